// Every outgoing BP message of a small site in one CTA, in shared memory.
//
// For a site of degree g with bond dims D_k and physical dim d (n = d prod D
// elements), each target leg t gets
//   T_t = V x_{k != t} E_k                   (bp.h:137-152, legs in order)
//   N_t[c, c'] = sum_{q} T_t[.., c, ..] conj(V[.., c', ..])   (bp.h:157-166)
// normalized by its Frobenius norm, with the distance to the stored message
// (the condition's per-message term, bp.h:286-354), exactly as
// k_msg_finalize forms them.  The site tensor, two ping-pong buffers for the
// absorptions, the g incoming messages and the Gram's partial sums all stay
// in shared memory, in FP64 whatever the storage precision: nothing but V,
// the messages and the g results crosses HBM, and one launch covers every
// small site of a sweep (or of a server batch of many jobs), whatever their
// degrees and dims.  Sites too large for this (site_sweep_smem_bytes above
// kSiteSmemMax) take the per-level path of the sweep plan.
//
// The Gram's partial sums are formed by P = 256 / C^2 thread groups over
// strided rows and reduced in a fixed order, so results do not depend on
// anything but the site's own data.
#pragma once
#include <cstdint>

#include "kernels.cuh"

namespace tnbp {

// SiteTask and site_sweep_smem_bytes are declared in kernels.cuh.

template <typename R, typename MR>
__global__ void __launch_bounds__(kThreads) k_site_sweep(const SiteTask* __restrict__ tasks) {
  using CR = typename cvec<R>::type;
  using CM = typename cvec<MR>::type;
  extern __shared__ __align__(16) unsigned char site_smem[];
  __shared__ double red[32];
  __shared__ long long strides[kMaxLegs];
  __shared__ int eoff[kMaxLegs];
  const SiteTask* tk = tasks + blockIdx.x;
  const int g = tk->g, n = tk->n, tid = threadIdx.x;
  double2* Vs = reinterpret_cast<double2*>(site_smem);
  double2* buf[2] = {Vs + n, Vs + 2 * n};
  double2* Es = Vs + 3 * n;
  if (tid == 0) {
    long long s = 1;
    int o = 0;
    for (int k = 0; k < g; ++k) {
      strides[k] = s;
      s *= tk->D[k];
      eoff[k] = o;
      o += tk->D[k] * tk->D[k];
    }
  }
  __syncthreads();
  int sd2 = 0;
  for (int k = 0; k < g; ++k) sd2 += tk->D[k] * tk->D[k];
  double2* part = Es + sd2;
  {
    const CR* V = static_cast<const CR*>(tk->V);
    for (int i = tid; i < n; i += kThreads) Vs[i] = to_d2(V[i]);
    for (int k = 0; k < g; ++k) {
      const CM* E = static_cast<const CM*>(tk->E[k]);
      const int m = tk->D[k] * tk->D[k];
      for (int i = tid; i < m; i += kThreads) Es[eoff[k] + i] = to_d2(E[i]);
    }
  }
  __syncthreads();
  for (int t = 0; t < g; ++t) {
    // T_t: absorb the message of every other leg, in leg order
    const double2* src = Vs;
    int which = 0;
    for (int k = 0; k < g; ++k) {
      if (k == t) continue;
      double2* dst = buf[which];
      which ^= 1;
      const long long L = strides[k];
      const int Dk = tk->D[k];
      const double2* e = Es + eoff[k];
      for (int i = tid; i < n; i += kThreads) {
        const long long l = i % L, rest = i / L;
        const int kp = (int)(rest % Dk);
        const long long r = rest / Dk;
        const double2* a = src + l + L * Dk * r;
        const double2* ek = e + (long long)Dk * kp;
        double2 acc = make_double2(0.0, 0.0);
        for (int j = 0; j < Dk; ++j) cfma(acc, a[L * j], ek[j]);
        dst[i] = acc;
      }
      __syncthreads();
      src = dst;
    }
    // Gram over every index but leg t: C^2 outputs, P row groups each
    const int C = tk->D[t];
    const int C2 = C * C;
    const long long L = strides[t], LC = L * C, Q = n / C;
    const int P = C2 >= kThreads ? 1 : kThreads / C2;
    for (int w = tid; w < C2 * P; w += kThreads) {
      const int o = w % C2, p = w / C2;
      const int c = o % C, c2 = o / C;
      double2 acc = make_double2(0.0, 0.0);
      for (long long q = p; q < Q; q += P) {
        const long long l = q % L, m = q / L;
        cfma_conj(acc, src[l + L * c + LC * m], Vs[l + L * c2 + LC * m]);
      }
      part[w] = acc;
    }
    __syncthreads();
    // fixed-order reduction of the groups, in place into part[0 .. C^2)
    double s_new = 0.0, s_old = 0.0;
    const CM* old = static_cast<const CM*>(tk->old[t]);
    for (int o = tid; o < C2; o += kThreads) {
      double2 v = part[o];
      for (int p = 1; p < P; ++p) v = v + part[(long long)p * C2 + o];
      part[o] = v;
      s_new += abs2(v);
      if (old) s_old += abs2(to_d2(old[o]));
    }
    const double nn = sqrt(block_sum(s_new, red));
    const double no = old ? sqrt(block_sum(s_old, red)) : 0.0;
    const double inv_n = nn > 0.0 ? 1.0 / nn : 1.0;
    const double inv_o = no > 0.0 ? 1.0 / no : 1.0;
    double d2 = 0.0;
    CM* out = static_cast<CM*>(tk->out[t]);
    for (int o = tid; o < C2; o += kThreads) {
      const double2 v = inv_n * part[o];
      if (old) d2 += abs2(v - inv_o * to_d2(old[o]));
      out[o] = from_d2<CM>(v);
    }
    d2 = block_sum(d2, red);
    if (tid == 0 && tk->dist[t]) *tk->dist[t] = sqrt(d2);
    __syncthreads();
  }
}

}  // namespace tnbp
