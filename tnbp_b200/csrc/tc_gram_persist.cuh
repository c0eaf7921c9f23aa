// Persistent form of the tcgen05 message Gram (k_gram_tc) for the complex64
// sweeps:  N[c, c'] = sum_q A[q, c] * conj(B[q, c'])  (c, c' < C <= 32),
// the same contraction, operand layout, 3xTF32 split and accumulation order
// as k_gram_tc (see tc_gram.cuh): split-K chunks of chunk_rows rows each
// write their own FP64 partial, and inside a chunk every 64-row block is
// accumulated afresh in FP32 in tensor memory (TMEM) and added, block after
// block, to FP64 registers.  Results are bitwise those of k_gram_tc.
//
// What differs is the schedule.  k_gram_tc runs one CTA per chunk, two per
// SM, and each CTA converts a 64-row tile, waits for its MMAs, drains them
// and only then converts the next: its loads have one MMA period to arrive.
// Here one 256-thread CTA per SM walks the chunks blockIdx.x,
// blockIdx.x + gridDim.x, ... in tiles of 128 rows (two 64-row blocks, two
// TMEM accumulators per tile, two tiles' accumulators = 256 columns).  The
// global loads of tile i + 2 are issued into one of two register buffers
// right after the MMAs of tile i, so a tile's loads have two tile periods to
// arrive, and the FP64 drain of tile i - 1 runs while the MMAs of tile i do.
// TMEM is allocated once per CTA.
//
// Every wait is bounded: on timeout the CTA records g_tc_error, waits once
// more (bounded) for its MMAs, frees its TMEM and returns.
#pragma once
#include <cstdint>

#include "tc_gram.cuh"

namespace tnbp {
namespace tc {

constexpr int kGramTileQ = 2 * kGramQ;                // rows per pipeline tile
constexpr uint32_t kGramA = kGramArows * kGramQ * 4;  // 192 x 64 fp32
constexpr uint32_t kGramY = 64 * kGramQ * 4;          // 64 x 64 fp32
constexpr uint32_t kGramBlk = kGramA + 2 * kGramY;    // one block's A, Y_hi, Y_lo
__host__ __device__ constexpr size_t gram_persist_smem_bytes() {
  // two blocks' operands, the 64 x 64 FP64 chunk sum, barrier and TMEM slot
  return 1024 + 2 * (size_t)kGramBlk + 64 * 64 * 8 + 64;
}

// Position of a 128-row tile in a CTA's walk over its chunks.
struct GramPos {
  long long chunk;  // global chunk index (>= total: past the end)
  int task, tile, ntile;
};

}  // namespace tc

// grid: min(total chunks, SMs); begins = exclusive prefix of nchunk
__global__ void __launch_bounds__(256, 1) k_gram_tc_persist(const GramTask* __restrict__ tasks,
                                                         const long long* __restrict__ begins, int ntask,
                                                         long long nchunk_total) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char tp_smem_raw[];
  unsigned char* smem = tp_smem_raw + ((1024 - (smem_u32(tp_smem_raw) & 1023)) & 1023);
  double* dsum = reinterpret_cast<double*>(smem + 2 * kGramBlk);  // 64 x 64 FP64
  uint64_t* mma_bar = reinterpret_cast<uint64_t*>(dsum + 64 * 64);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if ((long long)blockIdx.x >= nchunk_total) return;

  if (warp == 0) {  // 2 tiles x 2 blocks x 64 columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mma_bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // rows 128-191 of both blocks' A operands stay zero
  for (int i = tid; i < 2 * (kGramQ / 4) * 64; i += 256) {
    const int b = i / ((kGramQ / 4) * 64), j = i % ((kGramQ / 4) * 64);
    const int k4 = j / 64, r = 128 + j % 64;
    *reinterpret_cast<float4*>(smem + (uint32_t)b * kGramBlk + (uint32_t)k4 * (kGramArows * 16) +
                               (uint32_t)((r >> 3) * 128 + (r & 7) * 16)) = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  auto at_chunk = [&](long long chunk) -> GramPos {
    GramPos p;
    p.chunk = chunk;
    p.tile = 0;
    p.task = 0;
    p.ntile = 0;
    if (chunk < nchunk_total) {
      p.task = find_task(begins, ntask, chunk);
      const GramTask& t = tasks[p.task];
      const long long cl = chunk - t.block_begin;
      const long long rows = min(t.Q, (cl + 1) * t.chunk_rows) - cl * t.chunk_rows;
      p.ntile = (int)((rows + kGramTileQ - 1) / kGramTileQ);
    }
    return p;
  };
  auto next_pos = [&](GramPos p) -> GramPos {
    if (p.tile + 1 < p.ntile) { ++p.tile; return p; }
    return at_chunk(p.chunk + gridDim.x);
  };

  // Work item of a thread in a tile: column c = item % 32, q4 = item / 32
  // (4 consecutive q of one column: one 16-byte operand chunk per re/im and
  // hi/lo; q4 < 16 is block 0, q4 >= 16 block 1).  Four items per operand per
  // thread; lanes run over c so a warp's chunk stores fill 512 contiguous
  // bytes.  q < Q < 2^31 (a site tensor has fewer than 2^31 elements): 32-bit
  // split.
  auto load_tile = [&](const GramPos& p, float2 (&xa)[4][4], float2 (&yb)[4][4]) {
    const GramTask& t = tasks[p.task];
    const long long cl = p.chunk - t.block_begin;
    const unsigned q0 = (unsigned)(cl * t.chunk_rows + (long long)p.tile * kGramTileQ);
    const unsigned qe = (unsigned)min(t.Q, (cl + 1) * t.chunk_rows);
    const unsigned L = (unsigned)t.L, LC = (unsigned)(t.L * t.C);
    const int C = t.C;
    const float2* __restrict__ A = static_cast<const float2*>(t.A);
    const float2* __restrict__ B = static_cast<const float2*>(t.B);
#pragma unroll
    for (int it = 0; it < 4; ++it) {
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
  // operands of one tile from registers into both blocks' shared memory
  auto convert = [&](int Cp, const float2 (&xa)[4][4], const float2 (&yb)[4][4]) {
    const int N2 = 2 * Cp;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int item = tid + 256 * it;
      const int c = item & 31, q4 = item >> 5;
      if (c < Cp) {
        unsigned char* a_op = smem + (uint32_t)(q4 >> 4) * kGramBlk;
        unsigned char* y_hi = a_op + kGramA;
        unsigned char* y_lo = y_hi + kGramY;
        float4 xr, xi, yr, yi;
        float* pxr = &xr.x; float* pxi = &xi.x; float* pyr = &yr.x; float* pyi = &yi.x;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          pxr[j] = xa[it][j].x; pxi[j] = xa[it][j].y;
          pyr[j] = yb[it][j].x; pyi[j] = yb[it][j].y;
        }
        const uint32_t kx = (uint32_t)(q4 & 15) * (kGramArows * 16);
        const uint32_t ky = (uint32_t)(q4 & 15) * (uint32_t)(N2 * 16);
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
  };

  // FP64 accumulators: this thread's TMEM lane (row) and 32-column half
  const int trow = 32 * (warp & 3) + lane, chalf = warp >> 2;
  double acc[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) acc[i] = 0.0;
  // add the two 64-row blocks of the tile in accumulator set `set`, block 0
  // first (the order of the 64-row blocks along q)
  auto drain = [&](int set, int N2, int nblk) {
    if (32 * chalf < N2) {
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (b >= nblk) break;
        const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(2 * set + b) * 64u +
                              (uint32_t)(32 * chalf);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float v[16];
          tmem_ld16(base + 16u * h, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[16 * h + i] += (double)v[i];
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };
  // the chunk of p is complete: D = rows 0-63 + rows 64-127 through shared
  // memory, N formed in FP64 into the chunk's partial slot
  auto finish_chunk = [&](const GramPos& p) {
    const GramTask& t = tasks[p.task];
    const int C = t.C, Cp = (C + 7) & ~7, N2 = 2 * Cp;
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
    double2* part = t.partial + (p.chunk - t.block_begin) * C * C;
    for (int o = tid; o < C * C; o += 256) {
      const int c = o % C, c2 = o / C;
      const double re = dsum[c * 64 + c2] + dsum[(Cp + c) * 64 + Cp + c2];
      const double im = dsum[(Cp + c) * 64 + c2] - dsum[c * 64 + Cp + c2];
      part[c + (long long)C * c2] = make_double2(re, im);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = 0.0;
  };

  float2 xa0[4][4], yb0[4][4], xa1[4][4], yb1[4][4];
  GramPos pos0 = at_chunk(blockIdx.x), pos1 = next_pos(pos0);
  load_tile(pos0, xa0, yb0);
  if (pos1.chunk < nchunk_total) load_tile(pos1, xa1, yb1);
  GramPos prev = pos0;
  int prevN2 = 0, prevNblk = 0;
  bool failed = false;
  int li = 0;  // local index of the tile being issued
  // One tile: `cur` is the tile held in (xa, yb), `other` the tile after it;
  // on return (xa, yb) hold the tile after `other` and cur its position.
  auto step = [&](GramPos& cur, const GramPos& other, float2 (&xa)[4][4], float2 (&yb)[4][4]) -> bool {
    const GramTask& t = tasks[cur.task];
    const int Cp = (t.C + 7) & ~7, N2 = 2 * Cp;
    // 64-row blocks of this tile inside its chunk (the last tile of a chunk
    // of an odd number of blocks has one)
    const long long cl = cur.chunk - t.block_begin;
    const long long left = min(t.Q, (cl + 1) * t.chunk_rows) - cl * t.chunk_rows - (long long)cur.tile * kGramTileQ;
    const int nblk = left > kGramQ ? 2 : 1;
    if (li > 0) {  // the MMAs of tile li - 1 read the shared operands
      const bool ok = mbar_wait(smem_u32(mma_bar), (uint32_t)((li - 1) & 1));
      if (__syncthreads_or(!ok)) return false;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    convert(Cp, xa, yb);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t idesc = idesc_tf32(128, N2);
      const uint32_t a_lbo = kGramArows * 16, b_lbo = (uint32_t)N2 * 16;
      for (int b = 0; b < nblk; ++b) {
        const uint32_t d = tmem + (uint32_t)(2 * (li & 1) + b) * 64u;
        const uint32_t a0 = smem_u32(smem + (uint32_t)b * kGramBlk), a64 = a0 + 64 * 16;
        const uint32_t bh = a0 + kGramA, bl = bh + kGramY;
        for (int s = 0; s < kGramQ / 8; ++s) {
          const uint32_t ao = (uint32_t)s * 2 * a_lbo, bo = (uint32_t)s * 2 * b_lbo;
          mma_tf32(d, smem_desc(a0 + ao, a_lbo, 128), smem_desc(bh + bo, b_lbo, 128), idesc, s > 0 ? 1u : 0u);
          mma_tf32(d, smem_desc(a64 + ao, a_lbo, 128), smem_desc(bl + bo, b_lbo, 128), idesc, 1u);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mma_bar))
                   : "memory");
    }
    const GramPos this_tile = cur;
    // prefetch the tile after `other` into the buffer just converted
    cur = next_pos(other);
    if (cur.chunk < nchunk_total) load_tile(cur, xa, yb);
    if (li > 0) {
      drain((li - 1) & 1, prevN2, prevNblk);
      if (prev.tile + 1 == prev.ntile) finish_chunk(prev);
    }
    prev = this_tile;
    prevN2 = N2;
    prevNblk = nblk;
    ++li;
    return true;
  };
  while (true) {
    if (pos0.chunk >= nchunk_total) break;
    if (!step(pos0, pos1, xa0, yb0)) { failed = true; break; }
    if (pos1.chunk >= nchunk_total) break;
    if (!step(pos1, pos0, xa1, yb1)) { failed = true; break; }
  }
  if (!failed && li > 0) {  // the last tile (the last of its chunk)
    const bool ok = mbar_wait(smem_u32(mma_bar), (uint32_t)((li - 1) & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain((li - 1) & 1, prevN2, prevNblk);
      finish_chunk(prev);
    }
  }
  if (failed && tid == 0) {
    atomicExch(&g_tc_error, 1);
    // one more bounded wait for the newest MMAs before TMEM is freed
    if (li > 0) mbar_wait(smem_u32(mma_bar), (uint32_t)((li - 1) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
  }
}

}  // namespace tnbp
