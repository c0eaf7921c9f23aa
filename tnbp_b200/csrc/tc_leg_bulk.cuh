// Leg contraction on tcgen05 with asynchronous bulk staging of the input:
//   out[l, k, r] = sum_j in[l, j, r] * M[j, k]   (in, out complex64)
//
// Same product and 3xTF32 split as k_leg_apply_tc (tc_leg.cuh); what
// changes is how a 128-row tile reaches shared memory.  One thread issues
// cp.async.bulk copies (global -> shared, completion counted in bytes on an
// mbarrier) of the raw complex64 tile into a ring of kStages buffers, up to
// kStages tiles ahead of the tile being computed.  The threads then turn the
// raw tile into the UMMA operand (TF32 hi/lo, canonical K-major core
// matrices) with shared-memory reads and 16-byte stores only, so no warp
// waits on a global load.  The accumulator is double-buffered in TMEM: the
// epilogue of tile i-1 (tcgen05.ld, global stores) runs while the MMAs of
// tile i execute.
//
// A tile is a contiguous byte range of the input for the layouts that occur
// with power-of-two bond dimensions, selected per task by bulk_mode():
//   mode 1  L % 32 == 0 and (L >= 128 ? L % 128 == 0 : 128 % L == 0):
//           L >= 128: one copy of 128 rows per j (Din copies of 1 KB);
//           L = 32, 64: one copy of 128 / L whole (l, j) blocks.
//           Operand K order: [re j = 0..Dp) | im j = 0..Dp)] (planar).
//   mode 2  L == 1: one copy of the tile's rows (row q = Din contiguous
//           complex numbers).  Operand K order (re j, im j) interleaved, so
//           every 16-byte chunk of a raw row is one 16-byte operand chunk.
// Tasks of any other shape use k_leg_apply_tc or the CUDA-core kernel.
// Copies start 16-byte aligned and move a multiple of 16 bytes (Din even,
// tensors 256-byte aligned); none uses cluster multicast.
//
// Every wait is bounded: on timeout the CTA records g_tc_error, waits
// (bounded) for its copies and MMAs in flight, frees its TMEM and returns.
#pragma once
#include <climits>
#include <cstdint>

#include "tc_leg.cuh"

namespace tnbp {
namespace tc {

constexpr int kStages = 3;
constexpr int kRawBytes = kTcRows * kTcMaxD * 8;  // one raw tile: 128 rows x 32 complex64

__host__ __device__ constexpr size_t bulk_smem_bytes() {
  return 1024 + (size_t)kStages * kRawBytes + (size_t)2 * kTcRows * (2 * kTcMaxD) * 4 +
         (size_t)2 * (2 * kTcMaxD) * (2 * kTcMaxD) * 4 + 128;
}

// 0: not eligible; 1: planar (L multiple of 32); 2: interleaved (L == 1).
__host__ __device__ inline int bulk_mode(long long L, int Din, int Dout) {
  if (Din > kTcMaxD || Dout > kTcMaxD || Din < 2 || (Din & 1)) return 0;
  if (L == 1) return 2;
  if (L % 32 == 0 && (L >= 128 ? L % 128 == 0 : 128 % L == 0)) return 1;
  return 0;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// global -> shared bulk copy (no multicast); completion in bytes on bar
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Half h of an output row: out[l + L k] = (c[k], c[DQ + k]) for
// k in [h DQ/2, (h+1) DQ/2), k < Dout.
template <int DQ>
__device__ __forceinline__ void store_row_half(float2* __restrict__ p, unsigned L, int Dout, const float* c, int h) {
  if (h == 0) {
#pragma unroll
    for (int k = 0; k < DQ / 2; ++k)
      if (k < Dout) p[(size_t)L * k] = make_float2(c[k], c[DQ + k]);
  } else {
#pragma unroll
    for (int k = DQ / 2; k < DQ; ++k)
      if (k < Dout) p[(size_t)L * k] = make_float2(c[k], c[DQ + k]);
  }
}

__device__ __forceinline__ float4 tf32_hi4(float4 v) {
  return make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
}
__device__ __forceinline__ float4 tf32_lo4(float4 v, float4 h) {
  return make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z), to_tf32(v.w - h.w));
}

}  // namespace tc

template <typename MR>
__global__ void __launch_bounds__(256) k_leg_apply_tc_bulk(const LegTask* __restrict__ tasks,
                                                           const long long* __restrict__ begins, int ntask,
                                                           long long total_tiles) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char tcb_smem_raw[];
  unsigned char* smem = tcb_smem_raw + ((1024 - (smem_u32(tcb_smem_raw) & 1023)) & 1023);
  unsigned char* raw = smem;                                  // kStages x 32 KB
  unsigned char* a_hi = raw + kStages * kRawBytes;            // 128 x 64 fp32
  unsigned char* a_lo = a_hi + kTcRows * 2 * kTcMaxD * 4;
  unsigned char* b_hi = a_lo + kTcRows * 2 * kTcMaxD * 4;     // up to 64 x 64 fp32
  unsigned char* b_lo = b_hi + (2 * kTcMaxD) * (2 * kTcMaxD) * 4;
  uint64_t* full = reinterpret_cast<uint64_t*>(b_lo + (2 * kTcMaxD) * (2 * kTcMaxD) * 4);
  uint64_t* mma_bar = full + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
  // 256 threads: tile row q = tid & 127 (TMEM lane), half = tid >> 7 splits
  // the operand conversion and the output columns of the epilogue; warps w
  // and w + 4 share TMEM lane quadrant w & 3
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = tid & 127, half = tid >> 7;

  const long long per = (total_tiles + gridDim.x - 1) / gridDim.x;
  const long long t_begin = (long long)blockIdx.x * per;
  const long long t_end = min(total_tiles, t_begin + per);
  if (t_begin >= t_end) return;
  const int n = (int)(t_end - t_begin);

  if (warp == 0) {  // two 64-column accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(smem_u32(&full[s]), 1);
    mbar_init(smem_u32(mma_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // producer (thread 0): raw copy of one tile into a stage
  int ptask = find_task(begins, ntask, t_begin);
  auto issue = [&](long long tile, int stage) {
    while (ptask + 1 < ntask && begins[ptask + 1] <= tile) ++ptask;
    const LegTask t = tasks[ptask];
    const long long q0 = (tile - t.block_begin) * kTcRows;
    const int nrows = (int)min((long long)kTcRows, t.L * t.R - q0);
    const uint32_t bar = smem_u32(&full[stage]);
    const uint32_t dst = smem_u32(raw + stage * kRawBytes);
    const float2* in = static_cast<const float2*>(t.in);
    mbar_expect_tx(bar, (uint32_t)nrows * t.Din * 8u);
    if (t.L >= kTcRows) {  // mode 1, one copy of 128 rows per j
      const long long l0 = q0 % t.L, r = q0 / t.L;
      const float2* src = in + l0 + t.L * (long long)t.Din * r;
      for (int j = 0; j < t.Din; ++j)
        bulk_g2s(dst + (uint32_t)j * kTcRows * 8u, src + t.L * j, (uint32_t)nrows * 8u, bar);
    } else {  // L divides 128: the tile is nrows / L whole (l, j) blocks
      bulk_g2s(dst, in + (long long)t.Din * q0, (uint32_t)nrows * t.Din * 8u, bar);
    }
  };
  if (tid == 0)
    for (int s = 0; s < kStages && s < n; ++s) issue(t_begin + s, s);

  int ctask = find_task(begins, ntask, t_begin);
  long long cnext = ctask + 1 < ntask ? begins[ctask + 1] : LLONG_MAX;  // first tile of the next task
  int cur_b = -1;  // task whose message is in b_hi / b_lo
  LegTask tk = tasks[ctask], prev_tk = tk;
  long long prev_q0 = 0;
  bool failed = false;
  int li = 0;
  for (; li < n; ++li) {
    const long long tile = t_begin + li;
    while (tile >= cnext) {
      ++ctask;
      cnext = ctask + 1 < ntask ? begins[ctask + 1] : LLONG_MAX;
    }
    if (ctask != cur_b) {  // MMAs of the previous tile completed: B is free
      tk = tasks[ctask];
      cur_b = ctask;
      const int Din = tk.Din, Dout = tk.Dout, Dp = (Din + 3) & ~3, Dq = (Dout + 7) & ~7;
      const int K2 = 2 * Dp, N2 = 2 * Dq;
      const bool inter = bulk_mode(tk.L, Din, Dout) == 2;
      const typename cvec<MR>::type* __restrict__ mat = static_cast<const typename cvec<MR>::type*>(tk.mat);
      // out_re[n] = sum_j a_re M_re - a_im M_im ; out_im[n] = sum_j a_re M_im + a_im M_re
      for (int n2 = warp; n2 < N2; n2 += 8) {
        const int nr = n2 < Dq ? n2 : n2 - Dq, pn = n2 < Dq ? 0 : 1;
        for (int k2 = lane; k2 < K2; k2 += 32) {
          int kr, pk;
          if (inter) { kr = k2 >> 1; pk = k2 & 1; }
          else { kr = k2 < Dp ? k2 : k2 - Dp; pk = k2 < Dp ? 0 : 1; }
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
    const int Din = tk.Din, Dp = (Din + 3) & ~3, Dq = (tk.Dout + 7) & ~7;
    const int K2 = 2 * Dp, N2 = 2 * Dq;
    const long long q0 = (tile - tk.block_begin) * kTcRows;
    const int nrows = (int)min((long long)kTcRows, tk.L * tk.R - q0);
    const int stage = li % kStages;
    // 1. raw tile landed
    const bool ok = mbar_wait(smem_u32(&full[stage]), (uint32_t)((li / kStages) & 1));
    if (__syncthreads_or(!ok)) { failed = true; break; }
    // 2. raw -> UMMA operand (rows >= nrows are zero)
    const unsigned char* rs = raw + stage * kRawBytes;
    if (bulk_mode(tk.L, Din, tk.Dout) == 1) {
      const int q = row;
      const unsigned Ls = (unsigned)min(tk.L, (long long)kTcRows);
      const float2* rp = reinterpret_cast<const float2*>(rs) + (q / Ls) * Ls * Din + q % Ls;
      const uint32_t row_off = (uint32_t)((q >> 3) * 128 + (q & 7) * 16);
      const uint32_t im_off = (uint32_t)(Dp >> 2) * (kTcRows * 16);
      for (int g4 = half; g4 < Dp / 4; g4 += 2) {
        float4 re, im;
        float* pr = &re.x;
        float* pi = &im.x;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = 4 * g4 + j;
          const float2 v = (k < Din && q < nrows) ? rp[k * Ls] : make_float2(0.f, 0.f);
          pr[j] = v.x;
          pi[j] = v.y;
        }
        const float4 rh = tf32_hi4(re), ih = tf32_hi4(im);
        const uint32_t o = (uint32_t)g4 * (kTcRows * 16) + row_off;
        *reinterpret_cast<float4*>(a_hi + o) = rh;
        *reinterpret_cast<float4*>(a_hi + o + im_off) = ih;
        *reinterpret_cast<float4*>(a_lo + o) = tf32_lo4(re, rh);
        *reinterpret_cast<float4*>(a_lo + o + im_off) = tf32_lo4(im, ih);
      }
    } else {
      // interleaved: chunk g of row q = floats [4g, 4g+4) of the raw row;
      // a warp instruction covers 8 rows x 4 chunks
      const int nchunk = Dp / 2, real_chunks = Din / 2, nb4 = (nchunk + 3) / 4;
      for (int blk = warp; blk < 16 * nb4; blk += 8) {
        const int q = (blk % 16) * 8 + (lane & 7);
        const int g = (blk / 16) * 4 + (lane >> 3);
        if (g < nchunk) {
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (g < real_chunks && q < nrows) v = *reinterpret_cast<const float4*>(rs + (size_t)q * Din * 8 + 16 * g);
          const float4 h = tf32_hi4(v);
          const uint32_t o = (uint32_t)g * (kTcRows * 16) + (uint32_t)((q >> 3) * 128 + (q & 7) * 16);
          *reinterpret_cast<float4*>(a_hi + o) = h;
          *reinterpret_cast<float4*>(a_lo + o) = tf32_lo4(v, h);
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // 3. refill this stage, then the MMAs of this tile into buffer li & 1
    if (tid == 0) {
      if (li + kStages < n) issue(tile + kStages, stage);
      const uint32_t d = tmem + (uint32_t)(li & 1) * 64u;
      const uint32_t idesc = idesc_tf32(kTcRows, N2);
      const uint32_t a_lbo = kTcRows * 16, b_lbo = N2 * 16;
      const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
      for (int s = 0; s < K2 / 8; ++s) {
        const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
        mma_tf32(d, smem_desc(ah + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, s > 0 ? 1u : 0u);
        mma_tf32(d, smem_desc(ah + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
        mma_tf32(d, smem_desc(al + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mma_bar))
                   : "memory");
    }
    // 4. epilogue of the previous tile while these MMAs run
    if (li > 0) {
      float c[64];
      const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((li - 1) & 1) * 64u;
      const int pDq = (prev_tk.Dout + 7) & ~7;
      tmem_ld32(lane_addr, c);
      if (2 * pDq > 32) tmem_ld32(lane_addr + 32, c + 32);
      const unsigned q = (unsigned)prev_q0 + (unsigned)row;
      if (q < (unsigned)(prev_tk.L * prev_tk.R)) {
        const unsigned L = (unsigned)prev_tk.L, l = q % L, r = q / L;
        float2* __restrict__ p = static_cast<float2*>(prev_tk.out) + (size_t)l + (size_t)L * (size_t)prev_tk.Dout * r;
        switch (pDq) {
          case 8: store_row_half<8>(p, L, prev_tk.Dout, c, half); break;
          case 16: store_row_half<16>(p, L, prev_tk.Dout, c, half); break;
          case 24: store_row_half<24>(p, L, prev_tk.Dout, c, half); break;
          default: store_row_half<32>(p, L, prev_tk.Dout, c, half); break;
        }
      }
    }
    // 5. this tile's MMAs done: A, B and its accumulator are settled
    const bool ok2 = mbar_wait(smem_u32(mma_bar), (uint32_t)(li & 1));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    if (__syncthreads_or(!ok2)) {
      failed = true;
      if (!ok2) mbar_wait(smem_u32(mma_bar), (uint32_t)(li & 1));
      ++li;  // this tile's copies were consumed
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    prev_tk = tk;
    prev_q0 = q0;
  }
  if (!failed) {
    // epilogue of the last tile
    float c[64];
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((n - 1) & 1) * 64u;
    const int pDq = (prev_tk.Dout + 7) & ~7;
    tmem_ld32(lane_addr, c);
    if (2 * pDq > 32) tmem_ld32(lane_addr + 32, c + 32);
    const unsigned q = (unsigned)prev_q0 + (unsigned)row;
    if (q < (unsigned)(prev_tk.L * prev_tk.R)) {
      const unsigned L = (unsigned)prev_tk.L, l = q % L, r = q / L;
      float2* __restrict__ p = static_cast<float2*>(prev_tk.out) + (size_t)l + (size_t)L * (size_t)prev_tk.Dout * r;
      switch (pDq) {
        case 8: store_row_half<8>(p, L, prev_tk.Dout, c, half); break;
        case 16: store_row_half<16>(p, L, prev_tk.Dout, c, half); break;
        case 24: store_row_half<24>(p, L, prev_tk.Dout, c, half); break;
        default: store_row_half<32>(p, L, prev_tk.Dout, c, half); break;
      }
    }
  } else {
    if (tid == 0) {
      atomicExch(&g_tc_error, 1);
      // copies issued for tiles li .. li + kStages - 1 may still be in flight
      for (int j = li; j < n && j < li + kStages; ++j) mbar_wait(smem_u32(&full[j % kStages]), (uint32_t)((j / kStages) & 1));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
}

}  // namespace tnbp
