// Device kernels of the BP / truncation / measurement hot path.
//
// Every kernel takes a device array of task descriptors so that one launch
// covers all sites (or edges, or messages) of a stage, whatever their bond
// dimensions: uneven shapes share a launch.  Blocks find their task by a
// binary search over the tasks' exclusive prefix of block counts.
#pragma once
#include <cstdint>
#include "cplx.cuh"

namespace tnbp {

constexpr int kThreads = 256;
constexpr int kRowTile = 32;   // rows of a leg-apply / Gram tile
constexpr int kColTile = 32;   // output columns per inner chunk
constexpr int kMaxLegs = 8;    // maximum site degree supported
constexpr int kSvdMaxSweeps = 60;

// Division of unsigned values below 2^31 by an invariant divisor d >= 1
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): q = (mulhi(x, m) + x) >> s with
// s = ceil(log2 d) and m = floor(2^32 (2^s - d) / d) + 1, set up once on the
// host.  mulhi(x, m) < x, so the sum stays below 2^32 for x < 2^31.
struct FastDiv {
  uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t s = 0;
  while ((1ull << s) < d) ++s;
  const unsigned long long m = (((1ull << 32) * ((1ull << s) - d)) / d) + 1;
  return FastDiv{d, (uint32_t)m, s};
}
__host__ __device__ __forceinline__ uint32_t fast_div(uint32_t x, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(x, f.m) + x) >> f.s;
#else
  return (uint32_t)((((unsigned long long)x * f.m) >> 32) + x) >> f.s;
#endif
}

// ---------------------------------------------------------------------------
// Leg contraction  out[l, k, r] = sum_j in[l, j, r] * mat[j, k]
//   in : L x Din x R, out : L x Dout x R (column-major), mat : Din x Dout.
// Rows q = l + L*r are tiled by 32; a block owns one row tile and loops over
// the output columns in chunks of 32 with the input tile kept in shared
// memory.  This is the absorption of a message (bp.h:137-152) and of a
// truncation projector (truncation.h:175-185, 206-216).
// ---------------------------------------------------------------------------
struct LegTask {
  const void* in;
  void* out;
  const void* mat;
  long long L, R;         // L R < 2^31 (a site tensor has fewer than 2^31 elements)
  int Din, Dout;
  long long block_begin;  // exclusive prefix of row tiles over tasks
  FastDiv div_l;          // by L: the CUDA-core kernel's row split q = l + L r
  FastDiv div_din;        // by Din
};
inline void set_leg_divisors(LegTask& t) {
  t.div_l = make_fastdiv((uint32_t)t.L);
  t.div_din = make_fastdiv((uint32_t)t.Din);
}

__device__ __forceinline__ int find_task(const long long* begins, int n, long long b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (begins[mid] <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// R: arithmetic and tensor element type; MR: element type of mat (a message
// or projector), which may be wider than R (complex128 messages of the mixed
// path, rounded to R in shared memory).
template <typename R, typename MR = R>
__global__ void __launch_bounds__(kThreads) k_leg_apply(const LegTask* __restrict__ tasks,
                                                        const long long* __restrict__ begins,
                                                        int ntask, int max_din) {
  using C = typename cvec<R>::type;
  using CM = typename cvec<MR>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ti = find_task(begins, ntask, blockIdx.x);
  const LegTask tk = tasks[ti];
  const long long tile = blockIdx.x - tk.block_begin;
  const long long rows = tk.L * tk.R;
  const long long q0 = tile * kRowTile;
  const int Din = tk.Din, Dout = tk.Dout;
  const int ldA = Din + 1;
  C* As = reinterpret_cast<C*>(smem_raw);              // [32][Din+1]
  C* Ms = As + kRowTile * (max_din + 1);               // [Din][33]
  const C* in = static_cast<const C*>(tk.in);
  C* out = static_cast<C*>(tk.out);
  const CM* mat = static_cast<const CM*>(tk.mat);
  const long long L = tk.L;
  const bool qfast = L >= kRowTile;

  // input tile
  const int nA = kRowTile * Din;
  for (int idx = threadIdx.x; idx < nA; idx += kThreads) {
    int qq, j;
    if (qfast) { qq = idx % kRowTile; j = idx / kRowTile; }
    else { qq = (int)fast_div((uint32_t)idx, tk.div_din); j = idx - qq * Din; }
    const long long q = q0 + qq;
    C v = czero<C>();
    if (q < rows) {
      const uint32_t r = fast_div((uint32_t)q, tk.div_l);
      const long long l = (long long)((uint32_t)q - r * (uint32_t)L);
      v = in[l + L * j + L * Din * (long long)r];
    }
    As[qq * ldA + j] = v;
  }
  for (int k0 = 0; k0 < Dout; k0 += kColTile) {
    const int kc = min(kColTile, Dout - k0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < Din * kColTile; idx += kThreads) {
      const int kk = idx % kColTile, j = idx / kColTile;
      Ms[j * (kColTile + 1) + kk] = kk < kc ? from_d2<C>(to_d2(mat[j + (long long)Din * (k0 + kk)])) : czero<C>();
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < (kRowTile * kColTile) / kThreads; ++i) {
      const int o = threadIdx.x + i * kThreads;
      int qq, kk;
      if (qfast) { qq = o % kRowTile; kk = o / kRowTile; }
      else { kk = o % kColTile; qq = o / kColTile; }
      C acc = czero<C>();
      const C* a = As + qq * ldA;
      const C* m = Ms + kk;
      for (int j = 0; j < Din; ++j) cfma(acc, a[j], m[j * (kColTile + 1)]);
      const long long q = q0 + qq;
      if (q < rows && kk < kc) {
        const uint32_t r = fast_div((uint32_t)q, tk.div_l);
        const long long l = (long long)((uint32_t)q - r * (uint32_t)L);
        out[l + L * (k0 + kk) + L * (long long)Dout * (long long)r] = acc;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Gram with up to two kept legs:
//   N[c, c'] = sum_q A[q, c] * conj(B[q, c'])
// with q = l + L*m (l < L, m < M) and c = t + D*p (t < D, p < P) at address
// l + L*t + L*D*m + L*D*M*p.  P = 1 gives the message contraction of
// bp.h:157-166 (one kept leg); P = d gives the (d,d,D,D) environments of
// measure.h:194-205 (kept target leg and physical leg).
// Split-K: block = (row chunk, 32x32 tile of N); partial sums are written in
// FP64 and reduced in a fixed order by k_msg_finalize (no float atomics).
// ---------------------------------------------------------------------------
struct GramTask {
  const void* A;
  const void* B;
  long long L, M;
  int D, P, C, ctiles;
  long long Q, chunk_rows;
  int nchunk;
  double2* partial;       // [nchunk][C*C], N[c + C*c']
  long long block_begin;  // exclusive prefix of nchunk*ctiles*ctiles
};

template <typename R>
__global__ void __launch_bounds__(kThreads) k_gram(const GramTask* __restrict__ tasks,
                                                   const long long* __restrict__ begins, int ntask) {
  using C = typename cvec<R>::type;
  // rows padded to 34 elements: 16-byte aligned pairs for the 2x2 tiles
  __shared__ __align__(16) C As[kRowTile][kColTile + 2];
  __shared__ __align__(16) C Bs[kRowTile][kColTile + 2];
  const int ti = find_task(begins, ntask, blockIdx.x);
  const GramTask tk = tasks[ti];
  long long b = blockIdx.x - tk.block_begin;
  const int tiles2 = tk.ctiles * tk.ctiles;
  const int chunk = (int)(b / tiles2);
  const int tt = (int)(b % tiles2);
  const int ca0 = (tt % tk.ctiles) * kColTile;
  const int cb0 = (tt / tk.ctiles) * kColTile;
  const long long qbeg = chunk * tk.chunk_rows;
  const long long qend = min(tk.Q, qbeg + tk.chunk_rows);
  const C* A = static_cast<const C*>(tk.A);
  const C* B = static_cast<const C*>(tk.B);
  const long long L = tk.L, LD = tk.L * tk.D, LDM = tk.L * tk.D * tk.M;
  const bool qfast = L >= kRowTile;
  // complex64: each 32-row tile is summed in FP32 and added to an FP64
  // accumulator, so rounding does not grow with the chunk length (up to 4096
  // rows); complex128 accumulates directly.
  constexpr bool kPromote = sizeof(R) == 4;
  const int ga0 = 2 * (threadIdx.x % 16), gb0 = 2 * (threadIdx.x / 16);
  C acc[4];
  double2 accd[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) { acc[i] = czero<C>(); accd[i] = make_double2(0.0, 0.0); }
  for (long long q0 = qbeg; q0 < qend; q0 += kRowTile) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kRowTile * kColTile; idx += kThreads) {
      int qq, cc;
      if (qfast) { qq = idx % kRowTile; cc = idx / kRowTile; }
      else { cc = idx % kColTile; qq = idx / kColTile; }
      const long long q = q0 + qq;
      C va = czero<C>(), vb = czero<C>();
      if (q < qend) {
        const long long l = q % L, m = q / L;
        const long long base = l + LD * m;
        const int c1 = ca0 + cc, c2 = cb0 + cc;
        if (c1 < tk.C) va = A[base + L * (c1 % tk.D) + LDM * (c1 / tk.D)];
        if (c2 < tk.C) vb = B[base + L * (c2 % tk.D) + LDM * (c2 / tk.D)];
      }
      As[qq][cc] = va;
      Bs[qq][cc] = vb;
    }
    __syncthreads();
    // each thread owns the 2x2 block (a0..a0+1, b0..b0+1) of the 32x32 tile:
    // four smem reads per four complex FMAs
#pragma unroll 8
    for (int qq = 0; qq < kRowTile; ++qq) {
      const C x0 = As[qq][ga0], x1 = As[qq][ga0 + 1];
      const C y0 = Bs[qq][gb0], y1 = Bs[qq][gb0 + 1];
      cfma_conj(acc[0], x0, y0);
      cfma_conj(acc[1], x1, y0);
      cfma_conj(acc[2], x0, y1);
      cfma_conj(acc[3], x1, y1);
    }
    if (kPromote) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 t = to_d2(acc[i]);
        accd[i].x += t.x;
        accd[i].y += t.y;
        acc[i] = czero<C>();
      }
    }
  }
  double2* part = tk.partial + (long long)chunk * tk.C * tk.C;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int a = ca0 + ga0 + (i & 1), bb = cb0 + gb0 + (i >> 1);
    if (a < tk.C && bb < tk.C) part[a + (long long)tk.C * bb] = kPromote ? accd[i] : to_d2(acc[i]);
  }
}

// Fused last leg absorption + message Gram (tc_leg_gram.cuh):
//   N_t[c, c'] = sum_{o, j'} (sum_j X[c, j, o] E_w[j, j']) conj(V[c', j', o]).
struct LegGramTask {
  const void* X;         // complex64, same layout as V
  const void* V;         // complex64 site tensor
  const void* E;         // Dw x Dw message on leg w (element type MR)
  long long st, sw;      // element strides of legs t and w
  long long L1, Mid;     // outer index o = a + L1 (b + Mid c)
  long long s_mid, s_r;  // element offset of o = a + s_mid b + s_r c
  long long n_outer;     // number of outer indices
  int Dt, Dw;
  int mode;              // thread order: 0 c fastest, 1 j fastest, 2 o fastest
  int chunk_tiles;       // tiles of 4 outer indices per CTA
  int nchunk;
  double2* partial;      // [nchunk][Dt * Dt], N[c + Dt c']
  long long block_begin; // exclusive prefix of nchunk over tasks
};

// One small site's whole sweep (k_site_sweep, site_sweep.cuh).
struct SiteTask {
  const void* V;               // site tensor (R), column-major (D_0, ..., D_{g-1}, d)
  const void* E[kMaxLegs];     // incoming message of leg k (MR), D_k x D_k
  void* out[kMaxLegs];         // new outgoing message of leg k (MR)
  const void* old[kMaxLegs];   // stored outgoing message of leg k (MR)
  double* dist[kMaxLegs];      // || new/|new| - old/|old| ||_F of leg k
  int D[kMaxLegs];
  int g, d, n;                 // degree, physical dim, d prod D
};

// Shared memory of one site: V and two buffers of n complex FP64 values, the
// incoming messages, and max(256, C^2) partial sums of the Gram.
__host__ __device__ inline size_t site_sweep_smem_bytes(const int* D, int g, int d) {
  size_t n = (size_t)d, sd2 = 0, cmax2 = 0;
  for (int k = 0; k < g; ++k) {
    n *= (size_t)D[k];
    sd2 += (size_t)D[k] * D[k];
    cmax2 = cmax2 > (size_t)D[k] * D[k] ? cmax2 : (size_t)D[k] * D[k];
  }
  const size_t part = cmax2 > 256 ? cmax2 : 256;
  return 16 * (3 * n + sd2 + part);
}
// Sites up to 64 KB (1024 elements at degree 3 and 4: D <= 8 and D <= 4) are
// swept whole; larger ones (a degree-2 corner at D = 32 would take 147 KB and
// one CTA per SM) measured faster on the per-level tcgen05 path.
constexpr size_t kSiteSmemMax = 64 * 1024;

// ---------------------------------------------------------------------------
// Reduce Gram partials (fixed order), normalize by the Frobenius norm
// (bp.h:166), store the new message, and the distance to the normalized
// stored message (bp.h:341-350).  One block per message.
// ---------------------------------------------------------------------------
struct MsgTask {
  const double2* partial;
  int nchunk, C;
  void* out;        // new message (C x C), storage precision
  const void* old;  // stored message (same dim) or nullptr
  double* dist;     // || new/|new| - old/|old| ||_F
  double* norm_out; // |N| before normalization (may be nullptr)
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

// OR: element type of the stored messages (out and old).
template <typename R, typename OR = R>
__global__ void __launch_bounds__(kThreads) k_msg_finalize(const MsgTask* __restrict__ tasks) {
  using C = typename cvec<OR>::type;
  __shared__ double red[32];
  const MsgTask tk = tasks[blockIdx.x];
  const int n = tk.C * tk.C;
  const C* old = static_cast<const C*>(tk.old);
  double s_new = 0.0, s_old = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) {
    double2 v = make_double2(0.0, 0.0);
    for (int c = 0; c < tk.nchunk; ++c) v = v + tk.partial[(long long)c * n + i];
    s_new += abs2(v);
    if (old) s_old += abs2(to_d2(old[i]));
  }
  const double nn = sqrt(block_sum(s_new, red));
  const double no = old ? sqrt(block_sum(s_old, red)) : 0.0;
  const double inv_n = nn > 0.0 ? 1.0 / nn : 1.0;
  const double inv_o = no > 0.0 ? 1.0 / no : 1.0;
  double d2 = 0.0;
  C* out = static_cast<C*>(tk.out);
  for (int i = threadIdx.x; i < n; i += kThreads) {
    double2 v = make_double2(0.0, 0.0);
    for (int c = 0; c < tk.nchunk; ++c) v = v + tk.partial[(long long)c * n + i];
    v = inv_n * v;
    if (old) d2 += abs2(v - inv_o * to_d2(old[i]));
    out[i] = from_d2<C>(v);
  }
  d2 = block_sum(d2, red);
  if (threadIdx.x == 0) {
    if (tk.dist) *tk.dist = sqrt(d2);
    if (tk.norm_out) *tk.norm_out = nn;
  }
}

// complex128 -> complex64 copy (round to nearest): the sweep copy of the
// mixed path's site tensors.
static __global__ void k_narrow(const double2* __restrict__ in, float2* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    out[i] = make_float2((float)v.x, (float)v.y);
  }
}

// One block per job of a batch: out = scale * sum_i x[i] (fixed order).
struct SumTask {
  const double* x;
  int n;
  double scale;
  double* out;
};
static __global__ void k_segmented_sum(const SumTask* __restrict__ tasks) {
  __shared__ double red[32];
  const SumTask tk = tasks[blockIdx.x];
  double s = 0.0;
  for (int i = threadIdx.x; i < tk.n; i += blockDim.x) s += tk.x[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *tk.out = s * tk.scale;
}

// cond = scale * sum_i x[i], fixed-order tree (one block).
static __global__ void k_sum_scaled(const double* __restrict__ x, int n, double scale, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = s * scale;
}

// ---------------------------------------------------------------------------
// AbsorbTPO, site part (apply.h:43-66):
//   V'[(v_0,o_0),...,(v_{g-1},o_{g-1}), p'] = sum_p O[o..., p, p'] V[v..., p]
// merged bond index v + D*o (column-major reshape of (v, o)).
// ---------------------------------------------------------------------------
struct AbsorbTask {
  const void* V;
  void* out;
  const double2* O;  // op tensor (r_0..r_{g-1}, d, d'), complex128
  int g, d, dout;
  int Dv[kMaxLegs];
  int r[kMaxLegs];
  FastDiv div_m[kMaxLegs];  // by Dv[k] r[k] (the merged bond of leg k)
  FastDiv div_v[kMaxLegs];  // by Dv[k]
  long long n_out;          // < 2^31 (checked on the host)
  long long block_begin;
};

template <typename R>
__global__ void __launch_bounds__(kThreads) k_absorb_sites(const AbsorbTask* __restrict__ tasks,
                                                           const long long* __restrict__ begins,
                                                           int ntask) {
  using C = typename cvec<R>::type;
  const int ti = find_task(begins, ntask, blockIdx.x);
  const AbsorbTask& tk = tasks[ti];
  const long long i = (blockIdx.x - tk.block_begin) * kThreads + threadIdx.x;
  if (i >= tk.n_out) return;
  // the output index's digits: 32-bit, divisions by the legs' invariant
  // merged and bond dims
  uint32_t rem = (uint32_t)i;
  uint32_t voff = 0, vstride = 1, ooff = 0, ostride = 1;
  for (int k = 0; k < tk.g; ++k) {
    const uint32_t q = fast_div(rem, tk.div_m[k]);
    const uint32_t mk = rem - q * tk.div_m[k].d;
    rem = q;
    const uint32_t o = fast_div(mk, tk.div_v[k]);
    voff += (mk - o * tk.div_v[k].d) * vstride;
    ooff += o * ostride;
    vstride *= tk.div_v[k].d;
    ostride *= (uint32_t)tk.r[k];
  }
  const uint32_t pout = rem;  // < dout
  const C* V = static_cast<const C*>(tk.V);
  double2 acc = make_double2(0.0, 0.0);
  for (int p = 0; p < tk.d; ++p) {
    const double2 v = to_d2(V[voff + (size_t)vstride * p]);
    const double2 o = tk.O[ooff + (size_t)ostride * (p + (size_t)tk.d * pout)];
    acc = acc + v * o;
  }
  static_cast<C*>(tk.out)[i] = from_d2<C>(acc);
}

// AbsorbTPO, message part (apply.h:110-128): E'[(e,i),(e',i')] = E[e,e'] d_ii'.
struct MsgExpandTask {
  const void* E;
  void* out;
  int D, r;
  long long block_begin;
};

template <typename R>
__global__ void __launch_bounds__(kThreads) k_expand_msgs(const MsgExpandTask* __restrict__ tasks,
                                                          const long long* __restrict__ begins,
                                                          int ntask) {
  using C = typename cvec<R>::type;
  const int ti = find_task(begins, ntask, blockIdx.x);
  const MsgExpandTask& tk = tasks[ti];
  const long long N = (long long)tk.D * tk.r;
  const long long i = (blockIdx.x - tk.block_begin) * kThreads + threadIdx.x;
  if (i >= N * N) return;
  const long long row = i % N, col = i / N;
  const int e = (int)(row % tk.D), ii = (int)(row / tk.D);
  const int e2 = (int)(col % tk.D), i2 = (int)(col / tk.D);
  const C* E = static_cast<const C*>(tk.E);
  static_cast<C*>(tk.out)[i] = (ii == i2) ? E[e + (long long)tk.D * e2] : czero<C>();
}

// ---------------------------------------------------------------------------
// Sum of squares per range (site norms, tci::normalize on V), two passes:
// k_sumsq_partial writes one double per block; k_scale_ranges has every block
// re-add its range's partials in the same order and scale its elements.
// ---------------------------------------------------------------------------
struct RangeTask {
  void* data;
  long long n;
  long long block_begin;
  int nblocks;
  double* partial;  // nblocks entries
};

template <typename R>
__global__ void __launch_bounds__(kThreads) k_sumsq_partial(const RangeTask* __restrict__ tasks,
                                                            const long long* __restrict__ begins,
                                                            int ntask, int per_thread) {
  using C = typename cvec<R>::type;
  __shared__ double red[32];
  const int ti = find_task(begins, ntask, blockIdx.x);
  const RangeTask& tk = tasks[ti];
  const long long b = blockIdx.x - tk.block_begin;
  const long long beg = b * (long long)kThreads * per_thread;
  const long long end = min(tk.n, beg + (long long)kThreads * per_thread);
  const C* x = static_cast<const C*>(tk.data);
  double s = 0.0;
  for (long long i = beg + threadIdx.x; i < end; i += kThreads) s += abs2(to_d2(x[i]));
  s = block_sum(s, red);
  if (threadIdx.x == 0) tk.partial[b] = s;
}

template <typename R>
__global__ void __launch_bounds__(kThreads) k_scale_ranges(const RangeTask* __restrict__ tasks,
                                                           const long long* __restrict__ begins,
                                                           int ntask, int per_thread) {
  using C = typename cvec<R>::type;
  const int ti = find_task(begins, ntask, blockIdx.x);
  const RangeTask& tk = tasks[ti];
  double s = 0.0;
  for (int i = 0; i < tk.nblocks; ++i) s += tk.partial[i];
  const double nrm = sqrt(s);
  const R inv = nrm > 0.0 ? (R)(1.0 / nrm) : (R)1;
  const long long b = blockIdx.x - tk.block_begin;
  const long long beg = b * (long long)kThreads * per_thread;
  const long long end = min(tk.n, beg + (long long)kThreads * per_thread);
  C* x = static_cast<C*>(tk.data);
  for (long long i = beg + threadIdx.x; i < end; i += kThreads) x[i] = inv * x[i];
}

}  // namespace tnbp
