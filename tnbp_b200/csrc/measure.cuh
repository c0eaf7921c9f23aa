// Measurement: reduced density matrices from Gram partials, then the
// expectation-value ratios of measure.h and the FP64 sum over Pauli terms.
#pragma once
#include "kernels.cuh"

namespace tnbp {

// out[i] = sum over chunks of partial[c*n + i] (fixed order), FP64.
struct PartialSumTask {
  const double2* partial;
  int nchunk;
  int n;
  double2* out;
};
static __global__ void k_partial_sum(const PartialSumTask* __restrict__ tasks) {
  const PartialSumTask tk = tasks[blockIdx.x];
  for (int i = threadIdx.x; i < tk.n; i += blockDim.x) {
    double2 v = make_double2(0.0, 0.0);
    for (int c = 0; c < tk.nchunk; ++c) v = v + tk.partial[(long long)c * tk.n + i];
    tk.out[i] = v;
  }
}

// One-site term (measure.h:72-89): rho[p,p'] = sum_x W[x,p] conj(V[x,p']);
//   <O> = sum rho[p,p'] O[p,p'] / sum_p rho[p,p].
// Two-site term (measure.h:255-294): env[(t + D p), (t' + D p')] per side;
//   num = sum env_a[(t,p),(t',p')] O[p,c,p',c'] env_b[(t,c),(t',c')]
//   den = sum env_a[(t,p),(t',p)] env_b[(t,c),(t',c)].
struct TermTask {
  int kind;              // 1 or 2
  int d;                 // physical dim (2)
  int D;                 // target bond dim (kind 2)
  const double2* rho_a;  // kind 1: d x d; kind 2: (D d) x (D d)
  const double2* rho_b;  // kind 2 only
  double2 op[16];        // kind 1: O[p + d p']; kind 2: O[p + d c + d^2 p' + d^3 c']
  double2 coeff;
};

static __global__ void __launch_bounds__(kThreads) k_terms(const TermTask* __restrict__ tasks,
                                                    double2* __restrict__ values) {
  __shared__ double red[32];
  const TermTask& tk = tasks[blockIdx.x];
  const int d = tk.d;
  double nr = 0.0, ni = 0.0, dr = 0.0, di = 0.0;
  if (tk.kind == 1) {
    if (threadIdx.x == 0) {
      for (int p = 0; p < d; ++p)
        for (int q = 0; q < d; ++q) {
          const double2 v = tk.rho_a[p + d * q] * tk.op[p + d * q];
          nr += v.x; ni += v.y;
        }
      for (int p = 0; p < d; ++p) { dr += tk.rho_a[p + d * p].x; di += tk.rho_a[p + d * p].y; }
    }
  } else {
    const int D = tk.D, C = D * d;
    const long long tt = (long long)D * D;
    for (long long idx = threadIdx.x; idx < tt; idx += blockDim.x) {
      const int t = (int)(idx % D), t2 = (int)(idx / D);
      for (int p = 0; p < d; ++p)
        for (int p2 = 0; p2 < d; ++p2) {
          const double2 ea = tk.rho_a[(t + D * p) + (long long)C * (t2 + D * p2)];
          for (int c = 0; c < d; ++c)
            for (int c2 = 0; c2 < d; ++c2) {
              const double2 eb = tk.rho_b[(t + D * c) + (long long)C * (t2 + D * c2)];
              const double2 o = tk.op[p + d * c + d * d * p2 + d * d * d * c2];
              const double2 v = (ea * o) * eb;
              nr += v.x; ni += v.y;
              if (p == p2 && c == c2) { const double2 w = ea * eb; dr += w.x; di += w.y; }
            }
        }
    }
  }
  nr = block_sum(nr, red); ni = block_sum(ni, red);
  dr = block_sum(dr, red); di = block_sum(di, red);
  if (threadIdx.x == 0) {
    const double den = dr * dr + di * di;
    // complex division num / den_c
    values[blockIdx.x] = make_double2((nr * dr + ni * di) / den, (ni * dr - nr * di) / den);
  }
}

// Cluster measurement, one tree site: its Gram environment over (kept bond
// leg t, physical leg p) contracted with the site's one-site operator,
//   X[t + D t'] = sum_{p,p'} env[(t + D p) + C (t' + D p')] op[p + d p'],
// C = D d; written in FP64 and, for absorption at the parent site, in
// storage precision R.
struct EnvOpTask {
  const double2* env;
  int D, d;            // d <= 2
  double2 op[4];       // op[p + d p'] (reference layout)
  double2* out64;      // D x D
  void* out;           // D x D, storage precision (may be null)
};
template <typename R>
__global__ void __launch_bounds__(kThreads) k_env_op(const EnvOpTask* __restrict__ tasks) {
  using C = typename cvec<R>::type;
  const EnvOpTask& tk = tasks[blockIdx.x];
  const int D = tk.D, d = tk.d;
  const long long CC = (long long)D * d;
  for (long long idx = threadIdx.x; idx < (long long)D * D; idx += blockDim.x) {
    const int t = (int)(idx % D), t2 = (int)(idx / D);
    double2 acc = make_double2(0.0, 0.0);
    for (int p = 0; p < d; ++p)
      for (int p2 = 0; p2 < d; ++p2) acc = acc + tk.env[(t + D * p) + CC * (t2 + D * p2)] * tk.op[p + d * p2];
    tk.out64[idx] = acc;
    if (tk.out) static_cast<C*>(tk.out)[idx] = from_d2<C>(acc);
  }
}

// out = sum_i a[i] b[i] (FP64, fixed order), one block per task: the two
// halves of a tree cluster meeting on one bond, sum_{t,t'} X[t,t'] Y[t,t'].
struct PairTask {
  const double2* a;
  const double2* b;
  int n;
  double2* out;
};
static __global__ void __launch_bounds__(kThreads) k_pair_dot(const PairTask* __restrict__ tasks) {
  __shared__ double red[32];
  const PairTask& tk = tasks[blockIdx.x];
  double sr = 0.0, si = 0.0;
  for (int i = threadIdx.x; i < tk.n; i += blockDim.x) {
    const double2 v = tk.a[i] * tk.b[i];
    sr += v.x; si += v.y;
  }
  sr = block_sum(sr, red);
  si = block_sum(si, red);
  if (threadIdx.x == 0) *tk.out = make_double2(sr, si);
}

// sum_k c_k <P_k> (FP64, one block, fixed order)
static __global__ void k_weighted_sum(const TermTask* __restrict__ tasks, const double2* __restrict__ values,
                               int n, double2* out) {
  __shared__ double red[32];
  double sr = 0.0, si = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double2 v = tasks[i].coeff * values[i];
    sr += v.x; si += v.y;
  }
  sr = block_sum(sr, red);
  si = block_sum(si, red);
  if (threadIdx.x == 0) *out = make_double2(sr, si);
}

}  // namespace tnbp
