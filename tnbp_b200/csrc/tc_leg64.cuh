// Leg contraction on tcgen05 for bond dimensions above 32 (chi = 32 requests
// run BP at D = 64):  out[l, k, r] = sum_j in[l, j, r] * M[j, k],
// complex64 tensors, 32 < max(Din, Dout) <= 64.
//
// The product and the 3xTF32 split are those of k_leg_apply_tc
// (tc_leg.cuh): real GEMM [A_re | A_im] (128 x 2Dp) x [[M_re, M_im],
// [-M_im, M_re]] (2Dp x 2Dq).  With Dp, Dq up to 64 the operands no longer
// fit shared memory at once, so K (2Dp <= 128) is walked in chunks of 64:
// the message operand stays resident (N2 x K2, hi and lo: up to 128 KB), the
// tile operand is built one K chunk at a time (128 x 64, hi and lo: 64 KB),
// and the chunks' MMAs accumulate into one TMEM accumulator of N2 <= 128
// columns.  256 threads, two per tile row: half h loads and converts
// j in [32h, 32h + 32) and stores output columns [Dq h / 2, Dq (h+1) / 2);
// warps w and w + 4 read TMEM lane quadrant w & 3.  The next tile's loads
// are issued before the wait on the last chunk's MMAs.
//
// Every wait is bounded: on timeout the CTA records g_tc_error, waits once
// more (bounded) for its MMAs, frees its TMEM and returns.
#pragma once
#include <cstdint>

#include "tc_leg.cuh"

namespace tnbp {
namespace tc {

constexpr int kTcMaxD64 = 64;
constexpr int kChunkK = 64;  // real K per chunk

__host__ __device__ constexpr size_t leg64_smem_bytes() {
  // A chunk (hi, lo): 128 x 64 fp32 each; B (hi, lo): 128 x 128 fp32 each
  return 1024 + (size_t)2 * kTcRows * kChunkK * 4 + (size_t)2 * (2 * kTcMaxD64) * (2 * kTcMaxD64) * 4 + 64;
}
__host__ __device__ inline bool leg64_ok(int Din, int Dout) {
  return Din <= kTcMaxD64 && Dout <= kTcMaxD64 && (Din > kTcMaxD || Dout > kTcMaxD);
}

}  // namespace tc

template <typename MR>
__global__ void __launch_bounds__(256) k_leg_apply_tc64(const LegTask* __restrict__ tasks,
                                                        const long long* __restrict__ begins, int ntask,
                                                        long long total_tiles) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char t64_smem_raw[];
  unsigned char* smem = t64_smem_raw + ((1024 - (smem_u32(t64_smem_raw) & 1023)) & 1023);
  unsigned char* a_hi = smem;                                    // 128 x 64 fp32
  unsigned char* a_lo = a_hi + kTcRows * kChunkK * 4;
  unsigned char* b_hi = a_lo + kTcRows * kChunkK * 4;            // up to 128 x 128 fp32
  unsigned char* b_lo = b_hi + (2 * kTcMaxD64) * (2 * kTcMaxD64) * 4;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(b_lo + (2 * kTcMaxD64) * (2 * kTcMaxD64) * 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = tid & 127, half = tid >> 7;
  constexpr int kHalfD = kTcMaxD64 / 2;  // j per thread

  const long long per = (total_tiles + gridDim.x - 1) / gridDim.x;
  const long long t_begin = (long long)blockIdx.x * per;
  const long long t_end = min(total_tiles, t_begin + per);
  if (t_begin >= t_end) return;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  float2 nxt[kHalfD];
  // this thread's half of one tile row (j in [32 half, 32 half + 32)) into
  // registers; rows < 2^31, 32-bit row split
  auto load_row = [&](long long tile, int task_id) {
    const LegTask t = tasks[task_id];
    const unsigned q = (unsigned)((tile - t.block_begin) * kTcRows) + (unsigned)row;
    const unsigned rows = (unsigned)(t.L * t.R), L = (unsigned)t.L;
    const int j0 = kHalfD * half;
    if (q < rows && j0 < t.Din) {
      const unsigned l = q % L, r = q / L;
      const float2* __restrict__ p =
          static_cast<const float2*>(t.in) + (size_t)l + (size_t)L * ((size_t)t.Din * r + j0);
#pragma unroll
      for (int j = 0; j < kHalfD; ++j) nxt[j] = j0 + j < t.Din ? __ldg(p + (size_t)L * j) : make_float2(0.f, 0.f);
    } else {
#pragma unroll
      for (int j = 0; j < kHalfD; ++j) nxt[j] = make_float2(0.f, 0.f);
    }
  };

  int cur_task = -1;
  LegTask tk;
  int Din = 0, Dout = 0, Dp = 4, Dq = 8;
  int task_of_next = find_task(begins, ntask, t_begin);
  load_row(t_begin, task_of_next);
  uint32_t phase = 0;
  bool failed = false;
  for (long long tile = t_begin; tile < t_end && !failed; ++tile) {
    const int task_id = task_of_next;
    if (task_id != cur_task) {  // the previous tile's MMAs completed: B is free
      cur_task = task_id;
      tk = tasks[task_id];
      Din = tk.Din;
      Dout = tk.Dout;
      Dp = (Din + 3) & ~3;
      Dq = (Dout + 7) & ~7;
      const int K2 = 2 * Dp, N2 = 2 * Dq;
      const typename cvec<MR>::type* __restrict__ mat = static_cast<const typename cvec<MR>::type*>(tk.mat);
      // B_real[k2][n2] = [[M_re, M_im], [-M_im, M_re]], stored N2 x K2 K-major
      for (int n2 = warp; n2 < N2; n2 += 8) {
        const int nr = n2 < Dq ? n2 : n2 - Dq, pn = n2 < Dq ? 0 : 1;
        for (int k2 = lane; k2 < K2; k2 += 32) {
          const int kr = k2 < Dp ? k2 : k2 - Dp, pk = k2 < Dp ? 0 : 1;
          double v = 0.0;
          if (kr < Din && nr < Dout) {
            const double2 m = to_d2(mat[kr + (long long)Din * nr]);
            v = (pk == pn) ? m.x : (pk == 0 ? m.y : -m.y);
          }
          const float h = to_tf32((float)v), lo = to_tf32((float)(v - (double)h));
          *reinterpret_cast<float*>(b_hi + kmajor_off(n2, k2, N2)) = h;
          *reinterpret_cast<float*>(b_lo + kmajor_off(n2, k2, N2)) = lo;
        }
      }
    }
    const int K2 = 2 * Dp, N2 = 2 * Dq;
    const int nchunk = (K2 + kChunkK - 1) / kChunkK;
    const uint32_t row_off = (uint32_t)((row >> 3) * 128 + (row & 7) * 16);
    for (int ch = 0; ch < nchunk; ++ch) {
      const int kc0 = ch * kChunkK, kcn = min(kChunkK, K2 - kc0);
      // operand chunk: K2 index x = j (re) or Dp + j (im); groups of 4 j
#pragma unroll
      for (int g = 0; g < kHalfD / 4; ++g) {
        const int j = kHalfD * half + 4 * g;  // first j of the group
        if (j >= Dp) continue;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          const int x = part * Dp + j;  // K2 index of the group
          if (x < kc0 || x >= kc0 + kcn) continue;
          float4 v;
          float* pv = &v.x;
#pragma unroll
          for (int i = 0; i < 4; ++i) pv[i] = part == 0 ? nxt[4 * g + i].x : nxt[4 * g + i].y;
          const float4 h = make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
          const float4 lo = make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z),
                                        to_tf32(v.w - h.w));
          const uint32_t o = (uint32_t)((x - kc0) >> 2) * (kTcRows * 16) + row_off;
          *reinterpret_cast<float4*>(a_hi + o) = h;
          *reinterpret_cast<float4*>(a_lo + o) = lo;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
        const uint32_t idesc = idesc_tf32(kTcRows, N2);
        const uint32_t a_lbo = kTcRows * 16, b_lbo = N2 * 16;
        const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
        const uint32_t bh = smem_u32(b_hi) + (uint32_t)(kc0 >> 2) * b_lbo, bl = smem_u32(b_lo) + (uint32_t)(kc0 >> 2) * b_lbo;
        for (int s = 0; s < kcn / 8; ++s) {
          const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
          const uint32_t acc0 = (ch > 0 || s > 0) ? 1u : 0u;
          mma_tf32(tmem, smem_desc(ah + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, acc0);
          mma_tf32(tmem, smem_desc(ah + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
          mma_tf32(tmem, smem_desc(al + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(mbar))
                     : "memory");
      }
      if (ch + 1 == nchunk && tile + 1 < t_end) {  // next tile's loads during the last chunk's MMAs
        task_of_next = (tile + 1 >= tk.block_begin + ((tk.L * tk.R + kTcRows - 1) / kTcRows))
                           ? find_task(begins, ntask, tile + 1)
                           : task_id;
        load_row(tile + 1, task_of_next);
      }
      const bool ok = mbar_wait(smem_u32(mbar), phase);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicExch(&g_tc_error, 1);
        if (!ok) mbar_wait(smem_u32(mbar), phase);
        failed = true;
        break;
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (failed) break;
    // epilogue: row's output columns n in [Dq h / 2, Dq (h+1) / 2): re in
    // TMEM column n, im in column Dq + n
    const int nh = Dq / 2, n0 = nh * half;
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    float cre[32], cim[32];
    tmem_ld32(lane_addr + (uint32_t)n0, cre);
    tmem_ld32(lane_addr + (uint32_t)(Dq + n0), cim);
    const unsigned q = (unsigned)((tile - tk.block_begin) * kTcRows) + (unsigned)row;
    if (q < (unsigned)(tk.L * tk.R)) {
      const unsigned L = (unsigned)tk.L, l = q % L, r = q / L;
      float2* __restrict__ p = static_cast<float2*>(tk.out) + (size_t)l + (size_t)L * ((size_t)Dout * r + n0);
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (i < nh && n0 + i < Dout) p[(size_t)L * i] = make_float2(cre[i], cim[i]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
}

}  // namespace tnbp
