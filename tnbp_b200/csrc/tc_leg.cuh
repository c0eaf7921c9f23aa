// Leg contraction on the 5th-generation tensor cores (tcgen05, sm_100a) for
// the complex64 and mixed paths:  out[l, k, r] = sum_j in[l, j, r] * M[j, k]
// (in, out complex64; M complex64 or complex128).
//
// A CTA (128 threads) works through 128-row tiles, rows q = l + L*r.  The complex
// product is one real GEMM
//     [A_re | A_im] (128 x 2Dp)  x  [[M_re, M_im], [-M_im, M_re]] (2Dp x 2Dq)
//   = [C_re | C_im] (128 x 2Dq)
// in TF32 with the 3xTF32 split x = hi + lo (hi = tf32(x), lo = tf32(x - hi)):
// C = A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated in FP32 in tensor
// memory (TMEM).  Operands are written by the threads into shared memory in
// the canonical K-major, no-swizzle UMMA layout (8-row x 16-byte core
// matrices), one thread issues tcgen05.mma, tcgen05.commit arrives on an
// mbarrier, and each warp reads its 32 accumulator lanes back with
// tcgen05.ld.  Dp = Din rounded up to 4, Dq = Dout rounded up to 8
// (zero padded); Din, Dout <= 32.
//
// Every wait is bounded: on timeout the CTA records an error in
// g_tc_error, waits once more (bounded) for MMAs in flight, skips its
// epilogue, frees its TMEM and returns.
#pragma once
#include <cstdint>

#include "kernels.cuh"

namespace tnbp {

__device__ int g_tc_error = 0;

namespace tc {

constexpr int kTcRows = 128;
constexpr int kTcMaxD = 32;
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor: start address, leading (K-direction core
// matrix) byte offset, stride (8-row group) byte offset, version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::tf32: D F32, A/B TF32, both K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Byte offset of element (row, k) in a canonical K-major operand of R rows.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int R) {
  return (uint32_t)((k >> 2) * (R * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase) {
  for (long long i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared memory bytes of one CTA (operands sized for dims up to 32).
__host__ __device__ constexpr size_t leg_smem_bytes() {
  return (size_t)2 * kTcRows * (2 * kTcMaxD) * 4 + (size_t)2 * (2 * kTcMaxD) * (2 * kTcMaxD) * 4 + 1024 + 64;
}

// One output row: out[l + L k] = (c[k], c[DQ + k]) for k < Dout.  With
// L == 1 and Dout even the row is contiguous and 16-byte aligned: two
// complex numbers per store.
template <int DQ>
__device__ __forceinline__ void store_row(float2* __restrict__ p, unsigned L, int Dout, const float* c) {
  if (L == 1 && (Dout & 1) == 0) {
    float4* __restrict__ p4 = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int k = 0; k < DQ; k += 2)
      if (k < Dout) p4[k >> 1] = make_float4(c[k], c[DQ + k], c[k + 1], c[DQ + k + 1]);
    return;
  }
#pragma unroll
  for (int k = 0; k < DQ; ++k)
    if (k < Dout) p[(size_t)L * k] = make_float2(c[k], c[DQ + k]);
}

}  // namespace tc

// Persistent over a contiguous range of 128-row tiles: TMEM is allocated
// once, the B operand is rebuilt only when the tile range crosses into a new
// task, and the global loads of the tile after next are issued before
// waiting for the current tile's MMAs so that loads, tensor-core work and
// the epilogue overlap.
template <typename MR>
__global__ void __launch_bounds__(128) k_leg_apply_tc(const LegTask* __restrict__ tasks,
                                                      const long long* __restrict__ begins, int ntask,
                                                      long long total_tiles) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* smem = tc_smem_raw + ((1024 - (smem_u32(tc_smem_raw) & 1023)) & 1023);
  unsigned char* a_hi = smem;                                // 128 x 64 fp32
  unsigned char* a_lo = a_hi + kTcRows * 2 * kTcMaxD * 4;
  unsigned char* b_hi = a_lo + kTcRows * 2 * kTcMaxD * 4;    // up to 64 x 64 fp32
  unsigned char* b_lo = b_hi + (2 * kTcMaxD) * (2 * kTcMaxD) * 4;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(b_lo + (2 * kTcMaxD) * (2 * kTcMaxD) * 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

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

  int cur_task = -1;
  LegTask tk;
  int Din = 0, Dout = 0, Dp = 4, Dq = 8;
  // Two register buffers: tile i+2 is loaded into the buffer tile i was
  // converted from, so a tile's loads have two tile periods to arrive.
  float2 bufA[kTcMaxD], bufB[kTcMaxD];
  // issue the global loads of one tile row (thread = row) into registers
  // Rows and row lengths of one task are < 2^31 (a site tensor has fewer
  // than 2^31 elements), so the row split uses 32-bit division.
  auto load_row = [&](long long tile, int task_id, float2 (&nxt)[kTcMaxD]) {
    const LegTask t = tasks[task_id];
    const unsigned q = (unsigned)((tile - t.block_begin) * kTcRows) + (unsigned)tid;
    const unsigned rows = (unsigned)(t.L * t.R), L = (unsigned)t.L;
    if (q < rows && L == 1 && (t.Din & 1) == 0) {
      // contiguous, 16-byte aligned row (tensors are 256-byte aligned)
      const float4* __restrict__ p4 = reinterpret_cast<const float4*>(static_cast<const float2*>(t.in) +
                                                                      (size_t)t.Din * q);
#pragma unroll
      for (int k = 0; k < kTcMaxD; k += 2) {
        const float4 v = k < t.Din ? __ldg(p4 + (k >> 1)) : make_float4(0.f, 0.f, 0.f, 0.f);
        nxt[k] = make_float2(v.x, v.y);
        nxt[k + 1] = make_float2(v.z, v.w);
      }
    } else if (q < rows) {
      const unsigned l = q % L, r = q / L;
      const float2* __restrict__ p =
          static_cast<const float2*>(t.in) + (size_t)l + (size_t)L * (size_t)t.Din * r;
#pragma unroll
      for (int k = 0; k < kTcMaxD; ++k) nxt[k] = k < t.Din ? __ldg(p + (size_t)L * k) : make_float2(0.f, 0.f);
    } else {
#pragma unroll
      for (int k = 0; k < kTcMaxD; ++k) nxt[k] = make_float2(0.f, 0.f);
    }
  };
  // Double-buffered accumulator: the MMAs of tile i write TMEM columns
  // [64 (i & 1), 64 (i & 1) + 64) while the threads drain tile i-1 from the
  // other half.  One mbarrier: the k-th commit completes phase k & 1.
  LegTask prev_tk{};
  long long prev_q0 = 0;
  int prev_Dq = 8;
  int issued = -1;  // local index of the newest tile whose MMAs were committed
  auto epilogue = [&](int li) {  // tile li's MMAs have completed
    float c[64];
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(li & 1) * 64u;
    tmem_ld32(lane_addr, c);
    if (2 * prev_Dq > 32) tmem_ld32(lane_addr + 32, c + 32);
    const unsigned q = (unsigned)prev_q0 + (unsigned)tid;
    if (q < (unsigned)(prev_tk.L * prev_tk.R)) {
      const unsigned L = (unsigned)prev_tk.L, l = q % L, r = q / L;
      const int pDout = prev_tk.Dout;
      float2* __restrict__ p = static_cast<float2*>(prev_tk.out) + (size_t)l + (size_t)L * (size_t)pDout * r;
      switch (prev_Dq) {  // imaginary parts start at column Dq
        case 8: store_row<8>(p, L, pDout, c); break;
        case 16: store_row<16>(p, L, pDout, c); break;
        case 24: store_row<24>(p, L, pDout, c); break;
        default: store_row<32>(p, L, pDout, c); break;
      }
    }
  };
  // one tile: its task in slot (replaced by the task of tile + 2), its rows
  // in nxt (replaced by the rows of tile + 2); false if a wait gave up
  auto step = [&](long long tile, int& slot, float2 (&nxt)[kTcMaxD]) -> bool {
    const int li = (int)(tile - t_begin);
    const int task_id = slot;
    // the MMAs of tile li - 1 read A and B: they must be done before both
    // are rewritten
    if (li > 0) {
      const bool okw = mbar_wait(smem_u32(mbar), (uint32_t)((li - 1) & 1));
      if (__syncthreads_or(!okw)) {
        if (tid == 0) atomicExch(&g_tc_error, 1);
        return false;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (task_id != cur_task) {
      cur_task = task_id;
      tk = tasks[task_id];
      Din = tk.Din;
      Dout = tk.Dout;
      Dp = (Din + 3) & ~3;
      Dq = (Dout + 7) & ~7;
      const int K2 = 2 * Dp, N2 = 2 * Dq;
      const typename cvec<MR>::type* __restrict__ mat = static_cast<const typename cvec<MR>::type*>(tk.mat);
      // B_real[k2][n2] = [[M_re, M_im], [-M_im, M_re]], stored N2 x K2 K-major
      for (int n2 = warp; n2 < N2; n2 += 4) {
        const int nr = n2 < Dq ? n2 : n2 - Dq, pn = n2 < Dq ? 0 : 1;
        for (int k2 = tid & 31; k2 < K2; k2 += 32) {
          const int kr = k2 < Dp ? k2 : k2 - Dp, pk = k2 < Dp ? 0 : 1;
          double v = 0.0;
          if (kr < Din && nr < Dout) {
            const double2 m = to_d2(mat[kr + (long long)Din * nr]);
            v = (pk == pn) ? m.x : (pk == 0 ? m.y : -m.y);
          }
          // hi = tf32(v); lo = tf32 of the remainder, taken in FP64 so that
          // complex128 messages keep their low bits
          const float h = to_tf32((float)v), lo = to_tf32((float)(v - (double)h));
          *reinterpret_cast<float*>(b_hi + kmajor_off(n2, k2, N2)) = h;
          *reinterpret_cast<float*>(b_lo + kmajor_off(n2, k2, N2)) = lo;
        }
      }
    }
    const int K2 = 2 * Dp, N2 = 2 * Dq;
    // A operand for this tile from the prefetched registers: per group of 4
    // k one 16-byte store each of re-hi, im-hi, re-lo, im-lo.  A thread's
    // row sits at a fixed offset inside every core matrix, and the imaginary
    // half starts Dp/4 core-matrix columns further (Dp is a multiple of 4);
    // a warp's 32 stores fill 512 contiguous bytes.
    {
      const uint32_t row_off = (uint32_t)((tid >> 3) * 128 + (tid & 7) * 16);
      const uint32_t im_off = (uint32_t)(Dp >> 2) * (kTcRows * 16);
#pragma unroll
      for (int g4 = 0; g4 < kTcMaxD / 4; ++g4) {
        if (4 * g4 < Dp) {
          float4 rh, ih, rl, il;
          float* prh = &rh.x; float* pih = &ih.x; float* prl = &rl.x; float* pil = &il.x;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float re = nxt[4 * g4 + j].x, im = nxt[4 * g4 + j].y;
            const float h1 = to_tf32(re), h2 = to_tf32(im);
            prh[j] = h1;
            pih[j] = h2;
            prl[j] = to_tf32(re - h1);
            pil[j] = to_tf32(im - h2);
          }
          const uint32_t o = (uint32_t)g4 * (kTcRows * 16) + row_off;
          *reinterpret_cast<float4*>(a_hi + o) = rh;
          *reinterpret_cast<float4*>(a_hi + o + im_off) = ih;
          *reinterpret_cast<float4*>(a_lo + o) = rl;
          *reinterpret_cast<float4*>(a_lo + o + im_off) = il;
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
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
                       smem_u32(mbar))
                   : "memory");
    }
    issued = li;
    // prefetch tile + 2 into the buffer just converted, while the tensor
    // cores work
    if (tile + 2 < t_end) {
      slot = (tile + 2 >= tk.block_begin + ((tk.L * tk.R + kTcRows - 1) / kTcRows))
                 ? find_task(begins, ntask, tile + 2)
                 : task_id;
      load_row(tile + 2, slot, nxt);
    }
    // epilogue of the previous tile from the other accumulator half
    if (li > 0) epilogue(li - 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    prev_tk = tk;
    prev_q0 = (tile - tk.block_begin) * kTcRows;
    prev_Dq = Dq;
    return true;
  };
  int slotA = find_task(begins, ntask, t_begin), slotB = 0;
  load_row(t_begin, slotA, bufA);
  if (t_begin + 1 < t_end) {
    slotB = find_task(begins, ntask, t_begin + 1);
    load_row(t_begin + 1, slotB, bufB);
  }
  bool ok_all = true;
  long long tile = t_begin;
  for (; tile < t_end; tile += 2) {
    if (!step(tile, slotA, bufA)) { ok_all = false; break; }
    if (tile + 1 < t_end && !step(tile + 1, slotB, bufB)) { ok_all = false; break; }
  }
  const int nt = (int)(t_end - t_begin);
  if (ok_all) {  // the last tile
    const bool okl = mbar_wait(smem_u32(mbar), (uint32_t)((nt - 1) & 1));
    if (__syncthreads_or(!okl)) {
      if (tid == 0) atomicExch(&g_tc_error, 1);
      if (!okl) mbar_wait(smem_u32(mbar), (uint32_t)((nt - 1) & 1));
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      epilogue(nt - 1);
    }
  } else {
    // a wait gave up: give the newest committed MMAs one more bounded wait
    // before TMEM is freed
    if (tid == 0 && issued >= 0) mbar_wait(smem_u32(mbar), (uint32_t)(issued & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
}

}  // namespace tnbp
