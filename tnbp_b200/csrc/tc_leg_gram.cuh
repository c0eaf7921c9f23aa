// Last leg absorption fused with the message Gram on tcgen05 (sm_100a), for
// the complex64 and mixed sweeps:
//
//   N_t[c, c'] = sum_{o, j'} ( sum_j X[c, j, o] E_w[j, j'] ) conj(V[c', j', o])
//
// X is the site tensor with every bond leg but t (the target) and w already
// absorbed, E_w the incoming message on leg w, V the site tensor, o every
// other index (the physical leg included).  This is the last absorption of
// bp.h:137-152 for target t followed by the Gram of bp.h:157-166, with the
// absorbed tensor T_t = X x_w E_w kept on chip: it goes from the first
// product's TMEM accumulator through registers straight into the second
// product's shared-memory operand and never reaches global memory.
//
// A tile is 4 outer indices o (all of legs t and w for each): 128 rows
// (o, c) of the first product, 4 Dwq contraction columns (o, j') of the
// second.  Per tile:
//   MMA1  P[(o,c), j'] = [X_re | X_im] [[E_re, E_im], [-E_im, E_re]]
//         M = 128, N = 2 Dwq, K = 2 Dwp; 3xTF32 (hi.hi + hi.lo + lo.hi)
//   MMA2  D = [P_hi ; P_lo] [V_hi ; V_lo]^T over K = (o, j') (the four
//         hi/lo products; rows 0-63 and 64-127 of D are added at the end)
//         M = 128, N = 2 Cp; real form of the complex Gram as in
//         k_gram_tc:  N_re = D[c, c'] + D[Cp+c, Cp+c'],
//                     N_im = D[Cp+c, c'] - D[c, Cp+c'].
// Each tile's FP32 Gram is added to FP64 registers (tile-sized FP32 sums,
// as k_gram_tc), and a CTA writes the FP64 Gram of its chunk of tiles to
// its partial slot; k_msg_finalize reduces the chunks in a fixed order.
//
// Dt, Dw <= 32; Cp = Dt rounded up to 8, Dwp = Dw rounded up to 4, Dwq = Dw
// rounded up to 8.  Thread-to-element order follows the unit-stride index
// (c, j or o) so that a warp's loads are coalesced.  Every wait is bounded:
// on timeout the CTA records g_tc_error, waits once more (bounded) for its
// MMAs, frees its TMEM and returns without writing its partial.
// LegGramTask is declared in kernels.cuh.
#pragma once
#include <cstdint>

#include "tc_gram.cuh"

namespace tnbp {

namespace tc {
constexpr int kLgOuter = 4;
constexpr uint32_t kLgA1 = 128 * 64 * 4;   // one 128-row x 64-K fp32 operand
constexpr uint32_t kLgB1 = 64 * 64 * 4;    // one 64-row x 64-K fp32 operand
constexpr uint32_t kLgA2 = 128 * 128 * 4;  // 128 rows x 128 K
constexpr uint32_t kLgY2 = 64 * 128 * 4;   // 64 rows x 128 K
__host__ __device__ constexpr size_t leg_gram_smem_bytes() {
  return 1024 + 2 * (size_t)kLgA1 + 2 * (size_t)kLgB1 + kLgA2 + 2 * (size_t)kLgY2 + 64;
}
__host__ __device__ inline bool leg_gram_ok(int Dt, int Dw) {
  return Dt >= 1 && Dt <= kTcMaxD && Dw >= 1 && Dw <= kTcMaxD;
}
}  // namespace tc

// grid: one CTA per chunk of every task; begins = exclusive prefix of nchunk.
// One 256-thread CTA per SM (about 226 KB of shared memory).
template <typename MR>
__global__ void __launch_bounds__(256, 1) k_leg_gram_tc(const LegGramTask* __restrict__ tasks,
                                                        const long long* __restrict__ begins, int ntask) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char lg_smem_raw[];
  unsigned char* smem = lg_smem_raw + ((1024 - (smem_u32(lg_smem_raw) & 1023)) & 1023);
  unsigned char* a1_hi = smem;
  unsigned char* a1_lo = a1_hi + kLgA1;
  unsigned char* b1_hi = a1_lo + kLgA1;
  unsigned char* b1_lo = b1_hi + kLgB1;
  unsigned char* a2 = b1_lo + kLgB1;
  unsigned char* y2_hi = a2 + kLgA2;
  unsigned char* y2_lo = y2_hi + kLgY2;
  uint64_t* bars = reinterpret_cast<uint64_t*>(y2_lo + kLgY2);  // [0] MMA1, [1] MMA2
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int ti = find_task(begins, ntask, blockIdx.x);
  const LegGramTask tk = tasks[ti];
  const int chunk = (int)(blockIdx.x - tk.block_begin);
  const long long ntile_all = (tk.n_outer + kLgOuter - 1) / kLgOuter;
  const long long tile0 = (long long)chunk * tk.chunk_tiles;
  const int ntile = (int)min((long long)tk.chunk_tiles, ntile_all - tile0);
  const int Dt = tk.Dt, Dw = tk.Dw;
  const int Cp = (Dt + 7) & ~7, Dwp = (Dw + 3) & ~3, Dwq = (Dw + 7) & ~7;
  const int K1 = 2 * Dwp, N1 = 2 * Dwq, K2 = kLgOuter * Dwq, N2 = 2 * Cp;
  const float2* __restrict__ X = static_cast<const float2*>(tk.X);
  const float2* __restrict__ V = static_cast<const float2*>(tk.V);

  if (warp == 0) {  // P: columns 0-63; Gram: columns 64-127
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bars[0])), "r"(1u));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bars[1])), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // A2 rows that no P row fills (2 Cp <= r < 64 in each half) stay zero
  for (uint32_t i = (uint32_t)tid * 16u; i < kLgA2; i += 256u * 16u)
    *reinterpret_cast<float4*>(a2 + i) = make_float4(0.f, 0.f, 0.f, 0.f);
  // B1 = [[E_re, E_im], [-E_im, E_re]] (K1 x N1), stored N1 rows x K1 K-major,
  // hi/lo split taken in FP64 so that complex128 messages keep their low bits
  {
    const typename cvec<MR>::type* __restrict__ E = static_cast<const typename cvec<MR>::type*>(tk.E);
    for (int n2 = warp; n2 < N1; n2 += 8) {
      const int nr = n2 < Dwq ? n2 : n2 - Dwq, pn = n2 < Dwq ? 0 : 1;
      for (int k2 = lane; k2 < K1; k2 += 32) {
        const int kr = k2 < Dwp ? k2 : k2 - Dwp, pk = k2 < Dwp ? 0 : 1;
        double v = 0.0;
        if (kr < Dw && nr < Dw) {
          const double2 m = to_d2(E[kr + (long long)Dw * nr]);
          v = (pk == pn) ? m.x : (pk == 0 ? m.y : -m.y);
        }
        const float h = to_tf32((float)v), lo = to_tf32((float)(v - (double)h));
        *reinterpret_cast<float*>(b1_hi + kmajor_off(n2, k2, N1)) = h;
        *reinterpret_cast<float*>(b1_lo + kmajor_off(n2, k2, N1)) = lo;
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // Work items of a tile: (o, c, j4) = four consecutive j of row (o, c);
  // four per thread, ordered so that lanes run along the unit-stride index.
  auto item_of = [&](int it, int& o, int& c, int& j4) {
    const int item = tid + 256 * it;
    if (tk.mode == 0) { c = item & 31; j4 = (item >> 5) & 7; o = item >> 8; }
    else if (tk.mode == 1) { j4 = item & 7; c = (item >> 3) & 31; o = item >> 8; }
    else { o = item & 3; c = (item >> 2) & 31; j4 = item >> 7; }
  };
  float2 xr[4][4], vr[4][4];
  auto load_tile = [&](long long tile) {
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      int o, c, j4;
      item_of(it, o, c, j4);
      // outer indices and their factors are < 2^31 (a site tensor has fewer
      // than 2^31 elements): 32-bit division, 64-bit offsets
      const long long og = tile * kLgOuter + o;
      const bool ok = og < tk.n_outer && c < Dt;
      long long base = 0;
      if (ok) {
        const unsigned ou = (unsigned)og, L1 = (unsigned)tk.L1, Mid = (unsigned)tk.Mid;
        const unsigned a = ou % L1, rest = ou / L1;
        base = (long long)a + tk.s_mid * (long long)(rest % Mid) + tk.s_r * (long long)(rest / Mid) + tk.st * c;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = 4 * j4 + q;
        float2 x = make_float2(0.f, 0.f), v = x;
        if (ok && j < Dw) {
          x = __ldg(X + base + tk.sw * j);
          v = __ldg(V + base + tk.sw * j);
        }
        xr[it][q] = x;
        vr[it][q] = v;
      }
    }
  };
  auto row16 = [](int r) { return (uint32_t)((r >> 3) * 128 + (r & 7) * 16); };

  const int trow = 32 * (warp & 3) + lane, half = warp >> 2;
  double acc[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) acc[i] = 0.0;
  auto drain = [&]() {
    if (32 * half < N2) {
      const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + 64u + (uint32_t)(32 * half);
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
  int issued1 = 0, issued2 = 0;  // MMA1 / MMA2 commits so far
  if (ntile > 0) load_tile(tile0);
  for (int t = 0; t < ntile && !failed; ++t) {
    // A1 <- X (MMA1 of the previous tile has completed: waited below)
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      int o, c, j4;
      item_of(it, o, c, j4);
      if (4 * j4 >= Dwp) continue;
      const float4 re = make_float4(xr[it][0].x, xr[it][1].x, xr[it][2].x, xr[it][3].x);
      const float4 im = make_float4(xr[it][0].y, xr[it][1].y, xr[it][2].y, xr[it][3].y);
      const float4 rh = tf32_hi4(re), ih = tf32_hi4(im);
      const uint32_t r = row16(32 * o + c);
      const uint32_t kre = (uint32_t)j4 * (128 * 16), kim = (uint32_t)((Dwp >> 2) + j4) * (128 * 16);
      *reinterpret_cast<float4*>(a1_hi + kre + r) = rh;
      *reinterpret_cast<float4*>(a1_hi + kim + r) = ih;
      *reinterpret_cast<float4*>(a1_lo + kre + r) = tf32_lo4(re, rh);
      *reinterpret_cast<float4*>(a1_lo + kim + r) = tf32_lo4(im, ih);
    }
    // the previous tile's MMA2 reads A2 and Y2: wait for it, then drain its Gram
    if (t > 0) {
      const bool ok = mbar_wait(smem_u32(&bars[1]), (uint32_t)((t - 1) & 1));
      if (__syncthreads_or(!ok)) { failed = true; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain();
    }
    // Y2 <- V: rows c (re) and Cp + c (im), K = o Dwq + j
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      int o, c, j4;
      item_of(it, o, c, j4);
      if (c >= Cp || 4 * j4 >= Dwq) continue;
      const float4 re = make_float4(vr[it][0].x, vr[it][1].x, vr[it][2].x, vr[it][3].x);
      const float4 im = make_float4(vr[it][0].y, vr[it][1].y, vr[it][2].y, vr[it][3].y);
      const float4 rh = tf32_hi4(re), ih = tf32_hi4(im);
      const uint32_t kc = (uint32_t)(o * (Dwq >> 2) + j4) * (uint32_t)(N2 * 16);
      *reinterpret_cast<float4*>(y2_hi + kc + row16(c)) = rh;
      *reinterpret_cast<float4*>(y2_hi + kc + row16(Cp + c)) = ih;
      *reinterpret_cast<float4*>(y2_lo + kc + row16(c)) = tf32_lo4(re, rh);
      *reinterpret_cast<float4*>(y2_lo + kc + row16(Cp + c)) = tf32_lo4(im, ih);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {  // MMA1 into TMEM columns 0 .. N1-1
      const uint32_t idesc = idesc_tf32(128, N1);
      const uint32_t a_lbo = 128 * 16, b_lbo = (uint32_t)N1 * 16;
      const uint32_t ah = smem_u32(a1_hi), al = smem_u32(a1_lo), bh = smem_u32(b1_hi), bl = smem_u32(b1_lo);
      for (int s = 0; s < K1 / 8; ++s) {
        const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
        mma_tf32(tmem, smem_desc(ah + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, s > 0 ? 1u : 0u);
        mma_tf32(tmem, smem_desc(ah + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
        mma_tf32(tmem, smem_desc(al + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bars[0]))
                   : "memory");
    }
    issued1 = t + 1;
    // the next tile's loads fly while the tensor cores work
    if (t + 1 < ntile) load_tile(tile0 + t + 1);
    {
      const bool ok = mbar_wait(smem_u32(&bars[0]), (uint32_t)(t & 1));
      if (__syncthreads_or(!ok)) { failed = true; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // A2 <- P: this thread's TMEM lane is row (o, c) = (warp & 3, lane);
    // warps 0-3 take j' in [0, Dwq/2), warps 4-7 [Dwq/2, Dwq)
    {
      const int o = warp & 3, c = lane;
      const int jh = Dwq >> 1, j0 = half * jh;
      float re[16], im[16];
      const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
      tmem_ld16(lane_base + (uint32_t)j0, re);
      tmem_ld16(lane_base + (uint32_t)(Dwq + j0), im);
      if (c < Cp) {
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          if (4 * g < jh) {
            const float4 r4 = make_float4(re[4 * g], re[4 * g + 1], re[4 * g + 2], re[4 * g + 3]);
            const float4 i4 = make_float4(im[4 * g], im[4 * g + 1], im[4 * g + 2], im[4 * g + 3]);
            const float4 rh = tf32_hi4(r4), ih = tf32_hi4(i4);
            const uint32_t kc = (uint32_t)((o * Dwq + j0) / 4 + g) * (128 * 16);
            *reinterpret_cast<float4*>(a2 + kc + row16(c)) = rh;
            *reinterpret_cast<float4*>(a2 + kc + row16(Cp + c)) = ih;
            *reinterpret_cast<float4*>(a2 + kc + row16(64 + c)) = tf32_lo4(r4, rh);
            *reinterpret_cast<float4*>(a2 + kc + row16(64 + Cp + c)) = tf32_lo4(i4, ih);
          }
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {  // MMA2 into TMEM columns 64 .. 64 + N2 - 1
      const uint32_t idesc = idesc_tf32(128, N2);
      const uint32_t a_lbo = 128 * 16, b_lbo = (uint32_t)N2 * 16;
      const uint32_t aa = smem_u32(a2), bh = smem_u32(y2_hi), bl = smem_u32(y2_lo);
      for (int s = 0; s < K2 / 8; ++s) {
        const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
        mma_tf32(tmem + 64u, smem_desc(aa + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc,
                 s > 0 ? 1u : 0u);
        mma_tf32(tmem + 64u, smem_desc(aa + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bars[1]))
                   : "memory");
    }
    issued2 = t + 1;
  }
  if (!failed && issued2 > 0) {
    const bool ok = mbar_wait(smem_u32(&bars[1]), (uint32_t)((issued2 - 1) & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain();
    }
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(&g_tc_error, 1);
      // one more bounded wait for the newest MMAs before TMEM is freed
      if (issued1 > 0) mbar_wait(smem_u32(&bars[0]), (uint32_t)((issued1 - 1) & 1));
      if (issued2 > 0) mbar_wait(smem_u32(&bars[1]), (uint32_t)((issued2 - 1) & 1));
    }
  } else {
    // D = rows 0-63 + rows 64-127 through shared memory (A1 is free)
    double* dsum = reinterpret_cast<double*>(a1_hi);  // 64 x 64 FP64 = 32 KB
    if (trow >= 64 && 32 * half < N2) {
#pragma unroll
      for (int i = 0; i < 32; ++i) dsum[(trow - 64) * 64 + 32 * half + i] = acc[i];
    }
    __syncthreads();
    if (trow < 64 && 32 * half < N2) {
#pragma unroll
      for (int i = 0; i < 32; ++i) dsum[trow * 64 + 32 * half + i] += acc[i];
    }
    __syncthreads();
    double2* part = tk.partial + (long long)chunk * Dt * Dt;
    for (int o = tid; o < Dt * Dt; o += 256) {
      const int c = o % Dt, c2 = o / Dt;
      const double re = dsum[c * 64 + c2] + dsum[(Cp + c) * 64 + Cp + c2];
      const double im = dsum[(Cp + c) * 64 + c2] - dsum[c * 64 + Cp + c2];
      part[c + (long long)Dt * c2] = make_double2(re, im);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
  }
}

}  // namespace tnbp
