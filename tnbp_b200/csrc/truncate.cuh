// BP-gauge truncation of every edge, FP64 on the device, one block per edge.
//
// Follows truncation.h:57-219 and SquareRootAndInverse (root.h:66-148):
//   M_a = E[m] (computed at site a), M_b = E[m + ne]
//   M = U diag(s) Vh                        (SVD, descending s)
//   R = U diag(sqrt s  | s > sv_min) Vh
//   S = Vh^H diag(1/sqrt s | sqrt s > sqrt sv_min) U^H
//   T = R_a^T R_b / ||R_a^T R_b||_F
//   T = X diag(s) Y, keep s_i > sv_min, at most chi_max, at least one
//   P_a = S_a^T X diag(sqrt s)   (D x chi, applied to V_a's leg)
//   P_b = (diag(sqrt s) Y S_b)^T (D x chi, applied to V_b's leg)
//   E[m] = E[m + ne] = diag(s)
// The SVD is a one-sided (Hestenes) Jacobi SVD: column pairs are rotated in
// a round-robin order, one warp per pair, until no pair is rotated; the
// sweep count is bounded and a non-converged edge is reported, never spun on.
#pragma once
#include "kernels.cuh"

namespace tnbp {

struct TruncTask {
  const void* Ma;   // D x D, storage precision
  const void* Mb;
  int D;
  double2* work;    // 8 * D * D scratch
  double* sv;       // 3 * D: s of Ma, Mb, T (sorted)
  int* perm;        // 3 * D
  void* Pa;         // D x D capacity, storage precision (first keep columns valid)
  void* Pb;
  double* s_keep;   // D: kept singular values of T
  int* keep_out;
  double* err_out;
  int* status;      // 0 ok, 1 SVD sweep limit reached, 2 non-finite values
};

__device__ __forceinline__ double2 warp_sum2(double2 v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}
__device__ __forceinline__ double warp_sum1(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One-sided Jacobi on the n x n matrix A (column-major); V accumulates the
// rotations so that A_in = A_out * V^H.  Returns sweeps used, -1 if the
// sweep limit was reached.
__device__ int block_jacobi(double2* A, double2* V, int n, int* flag, double* red) {
  double fro = 0.0;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
    V[i] = (i % n == i / n) ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0);
    fro += abs2(A[i]);
  }
  fro = block_sum(fro, red);
  const int np = n + (n & 1);
  const int nwarps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Pairs count as orthogonal once |a_i^H a_j| <= n eps |a_i| |a_j|: the
  // rounding of the dot product itself is about sqrt(n) eps, so a tighter
  // threshold could keep rotating noise forever.  A column whose norm is at
  // the rounding level of the matrix (<= n eps ||A||_F) is numerically zero
  // and is not rotated (its singular value is noise, far below any cut).
  const double eps = 2.220446049250313e-16;
  const double tol = eps * (double)max(n, 8);
  const double zero2 = (tol * tol) * fro;
  for (int sweep = 0; sweep < kSvdMaxSweeps; ++sweep) {
    __syncthreads();
    if (threadIdx.x == 0) *flag = 0;
    __syncthreads();
    for (int round = 0; round < np - 1; ++round) {
      for (int pi = warp; pi < np / 2; pi += nwarps) {
        int a, b;
        if (pi == 0) { a = np - 1; b = round; }
        else { a = (round + pi) % (np - 1); b = (round - pi + np - 1) % (np - 1); }
        if (a >= n || b >= n) continue;
        const int i = min(a, b), j = max(a, b);
        double2* ai = A + (long long)n * i;
        double2* aj = A + (long long)n * j;
        double al = 0.0, be = 0.0;
        double2 ga = make_double2(0.0, 0.0);
        for (int r = lane; r < n; r += 32) {
          const double2 x = ai[r], y = aj[r];
          al += abs2(x);
          be += abs2(y);
          cfma(ga, conj(x), y);
        }
        al = warp_sum1(al);
        be = warp_sum1(be);
        ga = warp_sum2(ga);
        const double g = sqrt(abs2(ga));
        if (!(g > 0.0) || g <= tol * sqrt(al * be) || min(al, be) <= zero2) continue;
        const double2 ph = make_double2(ga.x / g, ga.y / g);
        const double zeta = (be - al) / (2.0 * g);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        if (fabs(t) < eps) continue;  // the rotation would not change a bit
        if (lane == 0) *flag = 1;
        const double c = 1.0 / sqrt(1.0 + t * t);
        const double s = c * t;
        const double2 sph = s * ph, sphc = s * conj(ph);
        for (int r = lane; r < n; r += 32) {
          const double2 x = ai[r], y = aj[r];
          ai[r] = c * x - sphc * y;
          aj[r] = sph * x + c * y;
        }
        double2* vi = V + (long long)n * i;
        double2* vj = V + (long long)n * j;
        for (int r = lane; r < n; r += 32) {
          const double2 x = vi[r], y = vj[r];
          vi[r] = c * x - sphc * y;
          vj[r] = sph * x + c * y;
        }
      }
      __syncthreads();
    }
    if (*flag == 0) return sweep + 1;
  }
  return -1;
}

// After block_jacobi: s[k] sorted descending, perm[k] = source column.
__device__ void block_sv_sort(const double2* A, int n, double* s_tmp, double* s, int* perm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = warp; c < n; c += nw) {
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) acc += abs2(A[(long long)n * c + r]);
    acc = warp_sum1(acc);
    if (lane == 0) s_tmp[c] = sqrt(acc);
  }
  __syncthreads();
  // Non-finite values (from non-finite messages) sort last as -1, so that
  // the ranks stay a permutation and every perm[] entry is a valid column;
  // the caller reports them.
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double si = s_tmp[i];
    const double ki = isfinite(si) ? si : -1.0;
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double kj = isfinite(s_tmp[j]) ? s_tmp[j] : -1.0;
      rank += (kj > ki) || (kj == ki && j < i);
    }
    s[rank] = si;
    perm[rank] = i;
  }
  __syncthreads();
}

// SquareRootAndInverse of the D x D message held in A (destroyed):
// R and S written (D x D).  U/V factors taken from the Jacobi result.
__device__ void block_sqrt_inv(double2* A, double2* V, int n, double sv_min, double* s_tmp,
                               double* s, int* perm, double2* Rout, double2* Sout, int* flag,
                               int* status, double* red) {
  if (block_jacobi(A, V, n, flag, red) < 0 && threadIdx.x == 0) *status = 1;
  block_sv_sort(A, n, s_tmp, s, perm);
  const double sq_min = sqrt(sv_min);
  // R[i,j] = sum_k U[i,k] sq_k conj(V[j,k]);  U[:,k] = A[:,perm k] / s_k
  // S[i,j] = sum_k V[i,k] isq_k conj(U[j,k])
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    double2 r = make_double2(0.0, 0.0), q = make_double2(0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      const double sk = s[k];
      if (!(sk > sv_min)) continue;  // sqrt(s) := 0 (root.h:316-318)
      const double sq = sqrt(sk);
      const int pk = perm[k];
      const double2 u_i = (1.0 / sk) * A[(long long)n * pk + i];
      const double2 u_j = (1.0 / sk) * A[(long long)n * pk + j];
      const double2 v_i = V[(long long)n * pk + i];
      const double2 v_j = V[(long long)n * pk + j];
      r = r + sq * (u_i * conj(v_j));
      if (sq > sq_min) q = q + (1.0 / sq) * (v_i * conj(u_j));  // root.h:324-326
    }
    Rout[idx] = r;
    Sout[idx] = q;
  }
  __syncthreads();
}

template <typename R>
__global__ void __launch_bounds__(kThreads) k_truncate_edges(const TruncTask* __restrict__ tasks,
                                                             int chi_max, double sv_min) {
  using C = typename cvec<R>::type;
  __shared__ double red[32];
  __shared__ int flag;
  const TruncTask tk = tasks[blockIdx.x];
  const int n = tk.D;
  const long long nn = (long long)n * n;
  double2* W0 = tk.work;
  double2* W1 = W0 + nn;
  double2* RA = W1 + nn;
  double2* SA = RA + nn;
  double2* RB = SA + nn;
  double2* SB = RB + nn;
  double* s_tmp = reinterpret_cast<double*>(SB + nn);  // uses part of the 7th slot
  if (threadIdx.x == 0) *tk.status = 0;
  const C* Ma = static_cast<const C*>(tk.Ma);
  const C* Mb = static_cast<const C*>(tk.Mb);
  for (long long i = threadIdx.x; i < nn; i += kThreads) W0[i] = to_d2(Ma[i]);
  block_sqrt_inv(W0, W1, n, sv_min, s_tmp, tk.sv, tk.perm, RA, SA, &flag, tk.status, red);
  for (long long i = threadIdx.x; i < nn; i += kThreads) W0[i] = to_d2(Mb[i]);
  __syncthreads();
  block_sqrt_inv(W0, W1, n, sv_min, s_tmp, tk.sv + n, tk.perm + n, RB, SB, &flag, tk.status, red);
  // T = RA^T RB, normalized (truncation.h:110-121)
  double ss = 0.0;
  for (long long idx = threadIdx.x; idx < nn; idx += kThreads) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < n; ++k) cfma(acc, RA[(long long)n * i + k], RB[(long long)n * j + k]);
    W0[idx] = acc;
    ss += abs2(acc);
  }
  const double tn = sqrt(block_sum(ss, red));
  const double inv_tn = tn > 0.0 ? 1.0 / tn : 1.0;
  for (long long idx = threadIdx.x; idx < nn; idx += kThreads) W0[idx] = inv_tn * W0[idx];
  __syncthreads();
  double* sT = tk.sv + 2 * n;
  int* pT = tk.perm + 2 * n;
  if (block_jacobi(W0, W1, n, &flag, red) < 0 && threadIdx.x == 0) *tk.status = 1;
  block_sv_sort(W0, n, s_tmp, sT, pT);
  for (int k = threadIdx.x; k < 3 * n; k += kThreads)
    if (!isfinite(tk.sv[k])) *tk.status = 2;  // non-finite message or T
  int keep = 0;
  while (keep < n && keep < chi_max && sT[keep] > sv_min) ++keep;
  if (keep == 0) keep = 1;
  double tot = 0.0, cut = 0.0;
  for (int k = 0; k < n; ++k) { tot += sT[k] * sT[k]; if (k >= keep) cut += sT[k] * sT[k]; }
  // P_a[i,c] = sum_k SA[k,i] X[k,c] sqrt(s_c);  X[:,c] = W0[:,pT c]/s_c
  // P_b[j,c] = sqrt(s_c) sum_k Y[c,k] SB[k,j];  Y[c,k] = conj(W1[k, pT c])
  C* Pa = static_cast<C*>(tk.Pa);
  C* Pb = static_cast<C*>(tk.Pb);
  for (long long idx = threadIdx.x; idx < (long long)n * keep; idx += kThreads) {
    const int i = (int)(idx % n), c = (int)(idx / n);
    const double sc = sT[c];
    const int pc = pT[c];
    const double xs = sc > 0.0 ? sqrt(sc) / sc : 0.0;
    double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      cfma(a, SA[(long long)n * i + k], W0[(long long)n * pc + k]);
      cfma(b, conj(W1[(long long)n * pc + k]), SB[(long long)n * i + k]);
    }
    Pa[idx] = from_d2<C>(xs * a);
    Pb[idx] = from_d2<C>(sqrt(sc) * b);
  }
  for (int c = threadIdx.x; c < keep; c += kThreads) tk.s_keep[c] = sT[c];
  if (threadIdx.x == 0) {
    *tk.keep_out = keep;
    *tk.err_out = tot > 0.0 ? cut / tot : 0.0;
  }
}

// Messages after truncation: E = diag(s) (truncation.h:137-149).
struct DiagTask {
  const double* s;
  void* out;
  int n;
};
template <typename R>
__global__ void k_write_diag(const DiagTask* __restrict__ tasks) {
  using C = typename cvec<R>::type;
  const DiagTask tk = tasks[blockIdx.x];
  C* out = static_cast<C*>(tk.out);
  for (int i = threadIdx.x; i < tk.n * tk.n; i += blockDim.x) {
    const int r = i % tk.n, c = i / tk.n;
    out[i] = r == c ? from_d2<C>(make_double2(tk.s[r], 0.0)) : czero<C>();
  }
}

}  // namespace tnbp
