// Message Gram on tcgen05 for the complex64 sweeps:
//   N[c, c'] = sum_q A[q, c] * conj(B[q, c'])      (c, c' < C <= 32)
// with q = l + L*m over every leg but the target, A = the absorbed tensor T,
// B = the site tensor V (both complex64, element (l, c, m) at
// l + L*c + L*C*m), the same contraction as k_gram with P = 1 (bp.h:157-166).
//
// Real form: X = [A_re ; A_im] and Y = [B_re ; B_im] (2Cp rows each, Cp = C
// rounded up to 8, row index = c or Cp + c, column = q).  D = X Y^T gives
//   N_re = D[c, c'] + D[Cp+c, Cp+c'],   N_im = D[Cp+c, c'] - D[c, Cp+c'].
// 3xTF32 with two M = 128 MMAs per K step on one stacked A operand of 192
// rows  [X_lo (rows 0-63) ; X_hi (64-127) ; zeros (128-191)]:
//   MMA 1: rows   0-127 x Y_hi -> D[0:64] += X_lo Y_hi,  D[64:128] += X_hi Y_hi
//   MMA 2: rows  64-191 x Y_lo -> D[0:64] += X_hi Y_lo,  D[64:128] += 0
// so D[0:64] + D[64:128] = X_hi Y_hi + X_hi Y_lo + X_lo Y_hi.
//
// One CTA (256 threads) owns one split-K chunk of one task (the chunking of
// k_gram: chunk_rows, a multiple of 64 here) and walks it in 64-row tiles.
// Each tile accumulates afresh into one of two TMEM buffers (FP32 over 64
// rows); while the next tile's MMAs run, every thread adds its 32 columns of
// one TMEM lane to FP64 registers.  At the end of the chunk the two row
// halves are added through shared memory, N is formed in FP64 and written to
// the chunk's partial slot; k_msg_finalize reduces the chunks in a fixed
// order as before.  The next tile's global loads are issued before the wait
// on the current tile's MMAs.
//
// Every wait is bounded: on timeout the CTA records g_tc_error, waits once
// more (bounded) for its MMAs, frees its TMEM and returns.
#pragma once
#include <cstdint>

#include "tc_leg_bulk.cuh"

namespace tnbp {
namespace tc {

constexpr int kGramQ = 64;     // contraction rows per tile
constexpr int kGramArows = 192;
__host__ __device__ constexpr size_t gram_smem_bytes() {
  // A: 192 rows x 64 K fp32; B hi, lo: 64 rows x 64 K fp32 each
  return 1024 + (size_t)kGramArows * kGramQ * 4 + (size_t)2 * 64 * kGramQ * 4 + 64;
}
__host__ __device__ inline bool gram_tc_ok(int C, int P) { return P == 1 && C >= 1 && C <= kTcMaxD; }

}  // namespace tc

// grid: one CTA per chunk of every task; begins = exclusive prefix of nchunk
// Two CTAs per SM (at most 128 registers per thread): while one CTA waits on
// its loads or MMAs the other converts or drains.
__global__ void __launch_bounds__(256, 2) k_gram_tc(const GramTask* __restrict__ tasks,
                                                 const long long* __restrict__ begins, int ntask) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char tg_smem_raw[];
  unsigned char* smem = tg_smem_raw + ((1024 - (smem_u32(tg_smem_raw) & 1023)) & 1023);
  unsigned char* a_op = smem;                                  // 192 x 64 fp32
  unsigned char* y_hi = a_op + kGramArows * kGramQ * 4;        // 64 x 64 fp32
  unsigned char* y_lo = y_hi + 64 * kGramQ * 4;
  uint64_t* mma_bar = reinterpret_cast<uint64_t*>(y_lo + 64 * kGramQ * 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int ti = find_task(begins, ntask, blockIdx.x);
  const GramTask tk = tasks[ti];
  const int chunk = (int)(blockIdx.x - tk.block_begin);
  const long long qbeg = chunk * tk.chunk_rows;
  const long long qend = min(tk.Q, qbeg + tk.chunk_rows);
  const int ntile = (int)((qend - qbeg + kGramQ - 1) / kGramQ);
  const int C = tk.C, Cp = (C + 7) & ~7, N2 = 2 * Cp;
  const unsigned L = (unsigned)tk.L, LC = (unsigned)(tk.L * tk.C);
  const float2* __restrict__ A = static_cast<const float2*>(tk.A);
  const float2* __restrict__ B = static_cast<const float2*>(tk.B);

  if (warp == 0) {  // two 64-column accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mma_bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // rows 128-191 of A stay zero
  for (int i = tid; i < (kGramQ / 4) * 64; i += 256) {
    const int k4 = i / 64, r = 128 + i % 64;
    *reinterpret_cast<float4*>(a_op + (uint32_t)k4 * (kGramArows * 16) + (uint32_t)((r >> 3) * 128 + (r & 7) * 16)) =
        make_float4(0.f, 0.f, 0.f, 0.f);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // Work item of a thread in a tile: column c = item % 32, q4 = item / 32
  // (4 consecutive q of one column: one 16-byte operand chunk per re/im and
  // hi/lo).  Two items per operand per thread; lanes run over c so a warp's
  // chunk stores fill 512 contiguous bytes.
  float2 xa[2][4], yb[2][4];
  // q < Q < 2^31 (a site tensor has fewer than 2^31 elements): 32-bit split
  auto load_tile = [&](int t) {
    const unsigned q0 = (unsigned)(qbeg + (long long)t * kGramQ), qe = (unsigned)qend;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int item = tid + 256 * it;
      const int c = item & 31, q4 = item >> 5;
      unsigned q = q0 + 4u * q4, l = q % L, m = q / L;
      if ((L & 3) == 0 && q + 3 < qe) {
        // L % 4 == 0 and q multiple of 4: the four rows are 32 contiguous,
        // 32-byte aligned bytes of column c
        float4 a01 = make_float4(0.f, 0.f, 0.f, 0.f), a23 = a01, b01 = a01, b23 = a01;
        if (c < C) {
          const size_t off = (size_t)l + (size_t)L * c + (size_t)LC * m;
          const float4* pa = reinterpret_cast<const float4*>(A + off);
          const float4* pb = reinterpret_cast<const float4*>(B + off);
          a01 = __ldg(pa); a23 = __ldg(pa + 1);
          b01 = __ldg(pb); b23 = __ldg(pb + 1);
        }
        xa[it][0] = make_float2(a01.x, a01.y); xa[it][1] = make_float2(a01.z, a01.w);
        xa[it][2] = make_float2(a23.x, a23.y); xa[it][3] = make_float2(a23.z, a23.w);
        yb[it][0] = make_float2(b01.x, b01.y); yb[it][1] = make_float2(b01.z, b01.w);
        yb[it][2] = make_float2(b23.x, b23.y); yb[it][3] = make_float2(b23.z, b23.w);
        continue;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float2 va = make_float2(0.f, 0.f), vb = va;
        if (c < C && q < qe) {
          const size_t off = (size_t)l + (size_t)L * c + (size_t)LC * m;
          va = __ldg(A + off);
          vb = __ldg(B + off);
        }
        xa[it][j] = va;
        yb[it][j] = vb;
        ++q;
        if (++l == L) { l = 0; ++m; }
      }
    }
  };
  // FP64 accumulators: this thread's TMEM lane (row) and 32-column half
  const int trow = 32 * (warp & 3) + lane, chalf = warp >> 2;
  double acc[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) acc[i] = 0.0;
  auto drain = [&](int buf) {
    if (32 * chalf < N2) {
      const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)buf * 64u + (uint32_t)(32 * chalf);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float v[16];
        tmem_ld16(base + 16u * h, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[16 * h + i] += (double)v[i];
      }
    }
  };

  bool failed = false;
  load_tile(0);
  for (int t = 0; t < ntile; ++t) {
    // operands of tile t from registers
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int item = tid + 256 * it;
      const int c = item & 31, q4 = item >> 5;
      if (c < Cp) {
        float4 xr, xi, yr, yi;
        float* pxr = &xr.x; float* pxi = &xi.x; float* pyr = &yr.x; float* pyi = &yi.x;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          pxr[j] = xa[it][j].x; pxi[j] = xa[it][j].y;
          pyr[j] = yb[it][j].x; pyi[j] = yb[it][j].y;
        }
        const uint32_t kx = (uint32_t)q4 * (kGramArows * 16);
        const uint32_t ky = (uint32_t)q4 * (uint32_t)(N2 * 16);
        const int rr = c, ri = Cp + c;  // X / Y rows of the re and im parts
        const float4 hr = tf32_hi4(xr), hi = tf32_hi4(xi);
        auto arow = [](int r) { return (uint32_t)((r >> 3) * 128 + (r & 7) * 16); };
        *reinterpret_cast<float4*>(a_op + kx + arow(rr)) = tf32_lo4(xr, hr);
        *reinterpret_cast<float4*>(a_op + kx + arow(ri)) = tf32_lo4(xi, hi);
        *reinterpret_cast<float4*>(a_op + kx + arow(64 + rr)) = hr;
        *reinterpret_cast<float4*>(a_op + kx + arow(64 + ri)) = hi;
        const float4 gr = tf32_hi4(yr), gi = tf32_hi4(yi);
        *reinterpret_cast<float4*>(y_hi + ky + arow(rr)) = gr;
        *reinterpret_cast<float4*>(y_hi + ky + arow(ri)) = gi;
        *reinterpret_cast<float4*>(y_lo + ky + arow(rr)) = tf32_lo4(yr, gr);
        *reinterpret_cast<float4*>(y_lo + ky + arow(ri)) = tf32_lo4(yi, gi);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t d = tmem + (uint32_t)(t & 1) * 64u;
      const uint32_t idesc = idesc_tf32(128, N2);
      const uint32_t a_lbo = kGramArows * 16, b_lbo = (uint32_t)N2 * 16;
      const uint32_t a0 = smem_u32(a_op), a64 = a0 + 64 * 16, bh = smem_u32(y_hi), bl = smem_u32(y_lo);
      for (int s = 0; s < kGramQ / 8; ++s) {
        const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
        mma_tf32(d, smem_desc(a0 + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, s > 0 ? 1u : 0u);
        mma_tf32(d, smem_desc(a64 + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mma_bar))
                   : "memory");
    }
    if (t + 1 < ntile) load_tile(t + 1);
    if (t > 0) drain((t - 1) & 1);
    const bool ok = mbar_wait(smem_u32(mma_bar), (uint32_t)(t & 1));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    if (__syncthreads_or(!ok)) {
      failed = true;
      if (!ok) mbar_wait(smem_u32(mma_bar), (uint32_t)(t & 1));
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (failed) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
  } else {
    if (ntile > 0) drain((ntile - 1) & 1);
    // D = rows 0-63 + rows 64-127, through shared memory (the A operand is
    // free: every MMA has completed)
    double* dsum = reinterpret_cast<double*>(a_op);  // 64 x 64 FP64 = 32 KB
    if (trow >= 64 && 32 * chalf < N2) {
#pragma unroll
      for (int i = 0; i < 32; ++i) dsum[(trow - 64) * 64 + 32 * chalf + i] = acc[i];
    }
    __syncthreads();
    if (trow < 64 && 32 * chalf < N2) {
#pragma unroll
      for (int i = 0; i < 32; ++i) dsum[trow * 64 + 32 * chalf + i] += acc[i];
    }
    __syncthreads();
    double2* part = tk.partial + (long long)chunk * C * C;
    for (int o = tid; o < C * C; o += 256) {
      const int c = o % C, c2 = o / C;
      const double re = dsum[c * 64 + c2] + dsum[(Cp + c) * 64 + Cp + c2];
      const double im = dsum[(Cp + c) * 64 + c2] - dsum[c * 64 + Cp + c2];
      part[c + (long long)C * c2] = make_double2(re, im);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
}

}  // namespace tnbp

namespace tnbp {
namespace tc {
// Gram for 32 < C <= 64: X and Y have 2Cp <= 128 rows, so the stacked
// operand of k_gram_tc does not fit M = 128; three MMAs per K step instead
// (X_hi Y_hi, X_hi Y_lo, X_lo Y_hi), M = 128 (X rows), N = 2Cp.
__host__ __device__ constexpr size_t gram64_smem_bytes() {
  // X hi, lo and Y hi, lo: 128 rows x 64 K fp32 each (reused as the 128 x 128
  // FP64 sum at the end)
  return 1024 + (size_t)4 * 128 * kGramQ * 4 + 64;
}
__host__ __device__ inline bool gram64_ok(int C, int P) { return P == 1 && C > kTcMaxD && C <= 64; }
}  // namespace tc

// grid: one CTA per chunk of every task; begins = exclusive prefix of nchunk
__global__ void __launch_bounds__(256) k_gram_tc64(const GramTask* __restrict__ tasks,
                                                   const long long* __restrict__ begins, int ntask) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char g64_smem_raw[];
  unsigned char* smem = g64_smem_raw + ((1024 - (smem_u32(g64_smem_raw) & 1023)) & 1023);
  constexpr int kOp = 128 * kGramQ * 4;  // one 128 x 64 fp32 operand
  unsigned char* x_hi = smem;
  unsigned char* x_lo = x_hi + kOp;
  unsigned char* y_hi = x_lo + kOp;
  unsigned char* y_lo = y_hi + kOp;
  uint64_t* mma_bar = reinterpret_cast<uint64_t*>(y_lo + kOp);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int ti = find_task(begins, ntask, blockIdx.x);
  const GramTask tk = tasks[ti];
  const int chunk = (int)(blockIdx.x - tk.block_begin);
  const long long qbeg = chunk * tk.chunk_rows;
  const long long qend = min(tk.Q, qbeg + tk.chunk_rows);
  const int ntile = (int)((qend - qbeg + kGramQ - 1) / kGramQ);
  const int C = tk.C, Cp = (C + 7) & ~7, N2 = 2 * Cp;
  const unsigned L = (unsigned)tk.L, LC = (unsigned)(tk.L * tk.C);
  const float2* __restrict__ A = static_cast<const float2*>(tk.A);
  const float2* __restrict__ B = static_cast<const float2*>(tk.B);

  if (warp == 0) {  // one accumulator of up to 128 columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mma_bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // items (c, q4): c = item % 64, q4 = item / 64; four per thread per tile
  auto arow = [](int r) { return (uint32_t)((r >> 3) * 128 + (r & 7) * 16); };
  const int trow = 32 * (warp & 3) + lane, chalf = warp >> 2;  // TMEM lane, 64-column half
  double acc[64];
#pragma unroll
  for (int i = 0; i < 64; ++i) acc[i] = 0.0;
  bool failed = false;
  for (int t = 0; t < ntile; ++t) {
    const unsigned q0 = (unsigned)(qbeg + (long long)t * kGramQ), qe = (unsigned)qend;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int item = tid + 256 * it;
      const int c = item & 63, q4 = item >> 6;
      if (c >= Cp) continue;
      float2 xa[4], yb[4];
      unsigned q = q0 + 4u * q4, l = q % L, m = q / L;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float2 va = make_float2(0.f, 0.f), vb = va;
        if (c < C && q < qe) {
          const size_t off = (size_t)l + (size_t)L * c + (size_t)LC * m;
          va = __ldg(A + off);
          vb = __ldg(B + off);
        }
        xa[j] = va;
        yb[j] = vb;
        ++q;
        if (++l == L) { l = 0; ++m; }
      }
      const float4 xr = make_float4(xa[0].x, xa[1].x, xa[2].x, xa[3].x);
      const float4 xi = make_float4(xa[0].y, xa[1].y, xa[2].y, xa[3].y);
      const float4 yr = make_float4(yb[0].x, yb[1].x, yb[2].x, yb[3].x);
      const float4 yi = make_float4(yb[0].y, yb[1].y, yb[2].y, yb[3].y);
      const uint32_t kx = (uint32_t)q4 * (128 * 16), ky = (uint32_t)q4 * (uint32_t)(N2 * 16);
      const float4 hr = tf32_hi4(xr), hi = tf32_hi4(xi), gr = tf32_hi4(yr), gi = tf32_hi4(yi);
      *reinterpret_cast<float4*>(x_hi + kx + arow(c)) = hr;
      *reinterpret_cast<float4*>(x_hi + kx + arow(Cp + c)) = hi;
      *reinterpret_cast<float4*>(x_lo + kx + arow(c)) = tf32_lo4(xr, hr);
      *reinterpret_cast<float4*>(x_lo + kx + arow(Cp + c)) = tf32_lo4(xi, hi);
      *reinterpret_cast<float4*>(y_hi + ky + arow(c)) = gr;
      *reinterpret_cast<float4*>(y_hi + ky + arow(Cp + c)) = gi;
      *reinterpret_cast<float4*>(y_lo + ky + arow(c)) = tf32_lo4(yr, gr);
      *reinterpret_cast<float4*>(y_lo + ky + arow(Cp + c)) = tf32_lo4(yi, gi);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t idesc = idesc_tf32(128, N2);
      const uint32_t a_lbo = 128 * 16, b_lbo = (uint32_t)N2 * 16;
      const uint32_t ah = smem_u32(x_hi), al = smem_u32(x_lo), bh = smem_u32(y_hi), bl = smem_u32(y_lo);
      for (int s = 0; s < kGramQ / 8; ++s) {
        const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
        mma_tf32(tmem, smem_desc(ah + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, s > 0 ? 1u : 0u);
        mma_tf32(tmem, smem_desc(ah + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
        mma_tf32(tmem, smem_desc(al + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mma_bar))
                   : "memory");
    }
    const bool ok = mbar_wait(smem_u32(mma_bar), (uint32_t)(t & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      if (!ok) mbar_wait(smem_u32(mma_bar), (uint32_t)(t & 1));
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // this tile's FP32 sums (64 rows of K) into FP64: lane trow, columns
    // [64 chalf, 64 chalf + 64) of N2
    if (64 * chalf < N2) {
      const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(64 * chalf);
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        float v[16];
        tmem_ld16(base + 16u * h, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[16 * h + i] += (double)v[i];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (failed) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
  } else {
    // D (2Cp x 2Cp, FP64) through shared memory (every MMA has completed)
    double* dsum = reinterpret_cast<double*>(smem);  // 128 x 128 FP64 = 128 KB = the four operands
    if (64 * chalf < N2) {
#pragma unroll
      for (int i = 0; i < 64; ++i) dsum[trow * 128 + 64 * chalf + i] = acc[i];
    }
    __syncthreads();
    double2* part = tk.partial + (long long)chunk * C * C;
    for (int o = tid; o < C * C; o += 256) {
      const int c = o % C, c2 = o / C;
      const double re = dsum[c * 128 + c2] + dsum[(Cp + c) * 128 + Cp + c2];
      const double im = dsum[(Cp + c) * 128 + c2] - dsum[c * 128 + Cp + c2];
      part[c + (long long)C * c2] = make_double2(re, im);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
}

}  // namespace tnbp
