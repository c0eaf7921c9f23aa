/*
 * CPU stand-in for the gqten tensor backend (GraceQ/tensor-ng-dev, branch
 * "to-tci-release"; pinned commit unknown: the submodule directory
 * external/tensor-ng-dev is empty in the reference, .gitmodules:1-3).
 *
 * TEST INFRASTRUCTURE ONLY.  It exists so that the reference's own, unchanged
 * tnbp headers (include/tnbp/ptns/function/{init,apply,bp,truncation,
 * measure}.h) and apps (apps/kicked_ising_lattice, apps/estimator) compile
 * and run on the CPU as the oracle for the B200 kernels.  Nothing in the
 * product (tnbp_b200/) includes it.
 *
 * Only the gqten surface that min-tci calls is provided
 * (external/min-tci/include/tci/gqten/*.h):
 *   class tensor<E>: Rank Shape Size GetElem SetElem GetRaw GetScale SetScale
 *                    Normalize CalcNorm Conjugate Transpose Reshape
 *                    StreamRead StreamWrite Random FormattedPrint
 *   free functions:  Contract SVD TruncSVD Trace LinearCombine GetReal
 *                    (QR EigHerm ExpHermExact Inverse are declared and throw:
 *                     no call site on the estimator path reaches them)
 *
 * Conventions restated here (gqten itself is absent, so these are the
 * documented choices the GPU path follows too):
 *   - storage is column-major: coordinate 0 varies fastest.  This is the
 *     order min-tci's assign_from_range/to_range/for_each_with_coors assume
 *     (constructor.h:108-150, miscellaneous.h:353-382);
 *   - Contract(a,b,labs_a,labs_b,c): equal negative labels are summed,
 *     a non-negative label is the output leg position (linalg.h:204-323);
 *   - Normalize() divides by the Frobenius norm and returns it;
 *   - SVD returns singular values in descending order, u has shape
 *     (row legs..., k) and v_dag (k, column legs...), k = min(m, n);
 *   - TruncSVD keeps the singular values s_i > s_min (absolute), at most
 *     chi_max of them and at least one; trunc_err = sum of the discarded
 *     s_i^2 over the sum of all s_i^2.
 * The SVD is a one-sided (Hestenes) Jacobi SVD, chosen for its high relative
 * accuracy and because no LAPACK exists in this image.
 */
#ifndef TNBP_ORACLE_GQTEN_CPU_H
#define TNBP_ORACLE_GQTEN_CPU_H

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace gqten {

template <typename T> struct real_of { using type = T; };
template <typename T> struct real_of<std::complex<T>> { using type = T; };

inline float GetReal(float a) { return a; }
inline double GetReal(double a) { return a; }
inline float GetReal(const std::complex<float>& a) { return a.real(); }
inline double GetReal(const std::complex<double>& a) { return a.real(); }

namespace detail {

template <typename T> inline T conjv(const T& x) { return x; }
template <typename T> inline std::complex<T> conjv(const std::complex<T>& x) { return std::conj(x); }
template <typename T> inline T abs2(const T& x) { return x * x; }
template <typename T> inline T abs2(const std::complex<T>& x) { return std::norm(x); }

template <typename Shape> inline size_t prod(const Shape& s) {
  size_t p = 1;
  for (auto d : s) p *= static_cast<size_t>(d);
  return p;
}

// out[new multi-index] = in[old multi-index]; new leg i is old leg perm[i].
template <typename E>
std::vector<E> permute(const std::vector<E>& in, const std::vector<int32_t>& shape,
                       const std::vector<int>& perm) {
  const size_t r = shape.size();
  const size_t n = prod(shape);
  std::vector<E> out(n);
  if (r == 0 || n == 0) { out = in; return out; }
  std::vector<size_t> old_stride(r);
  size_t st = 1;
  for (size_t k = 0; k < r; ++k) { old_stride[k] = st; st *= shape[k]; }
  std::vector<size_t> nshape(r), nstride(r);
  for (size_t i = 0; i < r; ++i) { nshape[i] = shape[perm[i]]; nstride[i] = old_stride[perm[i]]; }
  std::vector<size_t> idx(r, 0);
  size_t src = 0;
  for (size_t o = 0; o < n; ++o) {
    out[o] = in[src];
    for (size_t k = 0; k < r; ++k) {
      if (++idx[k] < nshape[k]) { src += nstride[k]; break; }
      src -= nstride[k] * (nshape[k] - 1);
      idx[k] = 0;
    }
  }
  return out;
}

// C(MxN) = A(MxK) * B(KxN), all column-major.
template <typename E>
void gemm(size_t M, size_t N, size_t K, const E* A, const E* B, E* C) {
#pragma omp parallel for schedule(static) if (M * N * K > 32768)
  for (long long n = 0; n < (long long)N; ++n) {
    E* c = C + (size_t)n * M;
    for (size_t m = 0; m < M; ++m) c[m] = E(0);
    for (size_t k = 0; k < K; ++k) {
      const E b = B[k + K * (size_t)n];
      if (b == E(0)) continue;
      const E* a = A + k * M;
      for (size_t m = 0; m < M; ++m) c[m] += a[m] * b;
    }
  }
}

// One-sided Jacobi SVD of A (M x N, column-major, M >= N).  On return the
// columns of A hold U*diag(s) and V (N x N) is the accumulated rotation, so
// that A_in = (A_out) * V^H.
template <typename E>
void jacobi_columns(size_t M, size_t N, std::vector<E>& A, std::vector<E>& V) {
  using R = typename real_of<E>::type;
  V.assign(N * N, E(0));
  for (size_t i = 0; i < N; ++i) V[i + N * i] = E(1);
  const R tol = std::numeric_limits<R>::epsilon() * R(M);
  for (int sweep = 0; sweep < 80; ++sweep) {
    bool rotated = false;
    for (size_t i = 0; i + 1 < N; ++i) {
      for (size_t j = i + 1; j < N; ++j) {
        E* ai = &A[i * M];
        E* aj = &A[j * M];
        R alpha = 0, beta = 0;
        E gamma = E(0);
        for (size_t m = 0; m < M; ++m) {
          alpha += abs2(ai[m]);
          beta += abs2(aj[m]);
          gamma += conjv(ai[m]) * aj[m];
        }
        const R g = std::abs(gamma);
        if (g == R(0) || g <= tol * std::sqrt(alpha * beta)) continue;
        rotated = true;
        const E ph = gamma / g;  // e^{i phi}
        const R zeta = (beta - alpha) / (R(2) * g);
        const R t = (zeta >= R(0) ? R(1) : R(-1)) / (std::abs(zeta) + std::sqrt(R(1) + zeta * zeta));
        const R c = R(1) / std::sqrt(R(1) + t * t);
        const R s = c * t;
        // [a_i, a_j] <- [a_i, a_j] * J,  J = [[c, s ph], [-s conj(ph), c]]
        for (size_t m = 0; m < M; ++m) {
          const E x = ai[m], y = aj[m];
          ai[m] = c * x - s * conjv(ph) * y;
          aj[m] = s * ph * x + c * y;
        }
        E* vi = &V[i * N];
        E* vj = &V[j * N];
        for (size_t m = 0; m < N; ++m) {
          const E x = vi[m], y = vj[m];
          vi[m] = c * x - s * conjv(ph) * y;
          vj[m] = s * ph * x + c * y;
        }
      }
    }
    if (!rotated) break;
  }
}

// Thin SVD of A (M x N column-major): A = U diag(s) Vh, s descending.
template <typename E>
void svd_matrix(size_t M, size_t N, const E* Ain, std::vector<E>& U,
                std::vector<typename real_of<E>::type>& s, std::vector<E>& Vh) {
  using R = typename real_of<E>::type;
  const bool tall = M >= N;
  const size_t m = tall ? M : N, n = tall ? N : M;
  std::vector<E> A(m * n);
  if (tall) {
    std::copy(Ain, Ain + M * N, A.begin());
  } else {  // work on A^H (N x M)
    for (size_t r = 0; r < M; ++r)
      for (size_t c = 0; c < N; ++c) A[c + N * r] = conjv(Ain[r + M * c]);
  }
  std::vector<E> V;
  jacobi_columns(m, n, A, V);
  std::vector<R> sv(n);
  for (size_t j = 0; j < n; ++j) {
    R acc = 0;
    for (size_t r = 0; r < m; ++r) acc += abs2(A[r + m * j]);
    sv[j] = std::sqrt(acc);
  }
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return sv[a] > sv[b]; });
  // Left vectors of the worked matrix (m x n) and its right vectors (n x n).
  std::vector<E> Lw(m * n, E(0)), Rw(n * n);
  s.assign(n, R(0));
  for (size_t jj = 0; jj < n; ++jj) {
    const size_t j = order[jj];
    s[jj] = sv[j];
    for (size_t r = 0; r < n; ++r) Rw[r + n * jj] = V[r + n * j];
    if (sv[j] > R(0)) {
      for (size_t r = 0; r < m; ++r) Lw[r + m * jj] = A[r + m * j] / sv[j];
    }
  }
  // Complete zero-norm left vectors to an orthonormal set (Gram-Schmidt on e_k).
  for (size_t jj = 0; jj < n; ++jj) {
    if (s[jj] > R(0)) continue;
    for (size_t e = 0; e < m; ++e) {
      std::vector<E> v(m, E(0));
      v[e] = E(1);
      for (size_t q = 0; q < n; ++q) {
        if (q == jj || (s[q] == R(0) && q > jj)) continue;
        E d = E(0);
        for (size_t r = 0; r < m; ++r) d += conjv(Lw[r + m * q]) * v[r];
        for (size_t r = 0; r < m; ++r) v[r] -= d * Lw[r + m * q];
      }
      R nn = 0;
      for (size_t r = 0; r < m; ++r) nn += abs2(v[r]);
      if (nn > R(1e-2)) {
        nn = std::sqrt(nn);
        for (size_t r = 0; r < m; ++r) Lw[r + m * jj] = v[r] / nn;
        break;
      }
    }
  }
  // worked = Lw diag(s) Rw^H
  if (tall) {  // U = Lw (M x n), Vh = Rw^H (n x N)
    U = Lw;
    Vh.assign(n * N, E(0));
    for (size_t k = 0; k < n; ++k)
      for (size_t c = 0; c < N; ++c) Vh[k + n * c] = conjv(Rw[c + n * k]);
  } else {  // A = (A^H)^H = Rw diag(s) Lw^H: U = Rw (M x n), Vh = Lw^H (n x N)
    U = Rw;
    Vh.assign(n * N, E(0));
    for (size_t k = 0; k < n; ++k)
      for (size_t c = 0; c < N; ++c) Vh[k + n * c] = conjv(Lw[c + m * k]);
  }
}

}  // namespace detail

template <typename ElemT>
class tensor {
 public:
  using value_type = ElemT;
  using RealT = typename real_of<ElemT>::type;
  using ShapeT = std::vector<int32_t>;

  tensor() : scale_(ElemT(0)) {}
  explicit tensor(const ShapeT& shape)
      : shape_(shape), data_(detail::prod(shape), ElemT(0)), scale_(ElemT(shape.empty() ? 0 : 1)) {}
  tensor(const ShapeT& shape, const std::vector<ElemT>& data) : shape_(shape), scale_(ElemT(1)) {
    if (shape_.empty()) {
      scale_ = data.empty() ? ElemT(0) : data[0];
    } else {
      if (data.size() < detail::prod(shape)) throw std::invalid_argument("gqten::tensor: data too short");
      data_.assign(data.begin(), data.begin() + detail::prod(shape));
    }
  }
  // Takes ownership of a malloc'd buffer (linalg.h:36-43 relies on this).
  tensor(const ShapeT& shape, ElemT* owned) : shape_(shape), scale_(ElemT(1)) {
    if (shape_.empty()) {
      scale_ = owned ? owned[0] : ElemT(0);
    } else {
      data_.assign(owned, owned + detail::prod(shape));
    }
    std::free(owned);
  }

  size_t Rank() const { return shape_.size(); }
  ShapeT Shape() const { return shape_; }
  size_t Size() const { return shape_.empty() ? 1 : data_.size(); }

  template <typename C, typename std::enable_if<!std::is_integral<C>::value, int>::type = 0>
  size_t Offset(const C& coors) const {
    size_t off = 0, st = 1;
    for (size_t k = 0; k < shape_.size(); ++k) {
      off += static_cast<size_t>(coors[k]) * st;
      st *= static_cast<size_t>(shape_[k]);
    }
    return off;
  }
  template <typename C, typename std::enable_if<!std::is_integral<C>::value, int>::type = 0>
  ElemT GetElem(const C& coors) const { return shape_.empty() ? scale_ : data_[Offset(coors)]; }
  template <typename I, typename std::enable_if<std::is_integral<I>::value, int>::type = 0>
  ElemT GetElem(I i) const { return shape_.empty() ? scale_ : data_[static_cast<size_t>(i)]; }
  template <typename C, typename std::enable_if<!std::is_integral<C>::value, int>::type = 0>
  void SetElem(const C& coors, const ElemT& v) {
    if (shape_.empty()) scale_ = v; else data_[Offset(coors)] = v;
  }
  template <typename I, typename std::enable_if<std::is_integral<I>::value, int>::type = 0>
  void SetElem(I i, const ElemT& v) {
    if (shape_.empty()) scale_ = v; else data_[static_cast<size_t>(i)] = v;
  }

  const ElemT* GetRaw() const { return shape_.empty() ? &scale_ : data_.data(); }
  ElemT* GetRaw() { return shape_.empty() ? &scale_ : data_.data(); }
  std::vector<ElemT>& Data() { return data_; }
  const std::vector<ElemT>& Data() const { return data_; }

  // A rank-0 tensor holds its value as the scale; higher ranks keep values
  // materialised, so their scale is always one.
  ElemT GetScale() const { return shape_.empty() ? scale_ : ElemT(1); }
  void SetScale(const ElemT& s) {
    if (shape_.empty()) { scale_ = s; return; }
    for (auto& x : data_) x *= s;
  }

  RealT CalcNorm() const {
    if (shape_.empty()) return std::abs(scale_);
    RealT acc = 0;
    for (const auto& x : data_) acc += detail::abs2(x);
    return std::sqrt(acc);
  }
  RealT Normalize() {
    RealT n = CalcNorm();
    if (n > RealT(0)) {
      if (shape_.empty()) scale_ /= n;
      else for (auto& x : data_) x /= n;
    }
    return n;
  }
  void Conjugate() {
    scale_ = detail::conjv(scale_);
    for (auto& x : data_) x = detail::conjv(x);
  }
  template <typename Idx>
  void Transpose(const std::vector<Idx>& order) {
    std::vector<int> perm(order.begin(), order.end());
    if (perm.size() != shape_.size()) throw std::invalid_argument("gqten::Transpose: rank mismatch");
    data_ = detail::permute(data_, shape_, perm);
    ShapeT ns(shape_.size());
    for (size_t i = 0; i < ns.size(); ++i) ns[i] = shape_[perm[i]];
    shape_ = ns;
  }
  template <typename S>
  void Reshape(const S& new_shape) {
    ShapeT ns(new_shape.begin(), new_shape.end());
    if (detail::prod(ns) != Size()) throw std::invalid_argument("gqten::Reshape: size mismatch");
    shape_ = ns;
  }
  void StreamWrite(std::ostream& os) const {
    uint64_t r = shape_.size();
    os.write(reinterpret_cast<const char*>(&r), sizeof(r));
    os.write(reinterpret_cast<const char*>(shape_.data()), sizeof(int32_t) * r);
    os.write(reinterpret_cast<const char*>(&scale_), sizeof(ElemT));
    os.write(reinterpret_cast<const char*>(data_.data()), sizeof(ElemT) * data_.size());
  }
  void StreamRead(std::istream& is) {
    uint64_t r = 0;
    is.read(reinterpret_cast<char*>(&r), sizeof(r));
    shape_.assign(r, 0);
    is.read(reinterpret_cast<char*>(shape_.data()), sizeof(int32_t) * r);
    is.read(reinterpret_cast<char*>(&scale_), sizeof(ElemT));
    data_.assign(r ? detail::prod(shape_) : 0, ElemT(0));
    is.read(reinterpret_cast<char*>(data_.data()), sizeof(ElemT) * data_.size());
  }
  template <typename G>
  void Random(int, const std::vector<int>&, G& gen) {
    std::normal_distribution<RealT> nd(0, 1);
    for (auto& x : data_) {
      if constexpr (std::is_same<ElemT, RealT>::value) x = nd(gen);
      else x = ElemT(nd(gen), nd(gen));
    }
  }
  void FormattedPrint() const {
    std::cout << "tensor shape (";
    for (size_t k = 0; k < shape_.size(); ++k) std::cout << (k ? "," : "") << shape_[k];
    std::cout << ")\n";
    for (size_t i = 0; i < Size(); ++i) std::cout << "  " << GetElem(i) << "\n";
  }

 private:
  ShapeT shape_;
  std::vector<ElemT> data_;
  ElemT scale_;
};

template <typename E>
void Contract(const tensor<E>* pa, const tensor<E>* pb, const std::vector<int>& la,
              const std::vector<int>& lb, tensor<E>* pc) {
  const auto sa = pa->Shape();
  const auto sb = pb->Shape();
  if (la.size() != sa.size() || lb.size() != sb.size())
    throw std::invalid_argument("gqten::Contract: label count != rank");
  std::vector<int> ca, cb, fa, fb;  // contracted / free leg positions
  std::vector<int> neg;
  for (size_t i = 0; i < la.size(); ++i)
    if (la[i] < 0) neg.push_back(la[i]);
  std::sort(neg.begin(), neg.end(), std::greater<int>());
  for (int l : neg) {
    auto ia = std::find(la.begin(), la.end(), l) - la.begin();
    auto ib = std::find(lb.begin(), lb.end(), l) - lb.begin();
    if (ib == (long)lb.size()) throw std::invalid_argument("gqten::Contract: unmatched label");
    if (sa[ia] != sb[ib]) throw std::invalid_argument("gqten::Contract: contracted dims differ");
    ca.push_back((int)ia);
    cb.push_back((int)ib);
  }
  for (size_t i = 0; i < la.size(); ++i) if (la[i] >= 0) fa.push_back((int)i);
  for (size_t i = 0; i < lb.size(); ++i) {
    if (lb[i] >= 0) fb.push_back((int)i);
    else if (std::find(la.begin(), la.end(), lb[i]) == la.end())
      throw std::invalid_argument("gqten::Contract: unmatched label");
  }
  size_t M = 1, N = 1, K = 1;
  std::vector<int> perm_a, perm_b;
  for (int i : fa) { perm_a.push_back(i); M *= sa[i]; }
  for (int i : ca) { perm_a.push_back(i); K *= sa[i]; }
  for (int i : cb) perm_b.push_back(i);
  for (int i : fb) { perm_b.push_back(i); N *= sb[i]; }
  std::vector<E> da(pa->GetRaw(), pa->GetRaw() + pa->Size());
  std::vector<E> db(pb->GetRaw(), pb->GetRaw() + pb->Size());
  if (sa.empty()) da.assign(1, pa->GetScale());
  if (sb.empty()) db.assign(1, pb->GetScale());
  std::vector<E> A = sa.empty() ? da : detail::permute(da, sa, perm_a);
  std::vector<E> B = sb.empty() ? db : detail::permute(db, sb, perm_b);
  std::vector<E> C(M * N);
  detail::gemm(M, N, K, A.data(), B.data(), C.data());
  const size_t rc = fa.size() + fb.size();
  std::vector<int32_t> cshape;  // legs in [free a..., free b...] order
  std::vector<int> clabel;
  for (int i : fa) { cshape.push_back(sa[i]); clabel.push_back(la[i]); }
  for (int i : fb) { cshape.push_back(sb[i]); clabel.push_back(lb[i]); }
  if (rc == 0) {
    tensor<E> out(std::vector<int32_t>{}, std::vector<E>{C[0]});
    *pc = std::move(out);
    return;
  }
  std::vector<int> perm(rc, -1);
  for (size_t i = 0; i < rc; ++i) {
    if (clabel[i] < 0 || (size_t)clabel[i] >= rc || perm[clabel[i]] != -1)
      throw std::invalid_argument("gqten::Contract: bad output labels");
    perm[clabel[i]] = (int)i;
  }
  std::vector<int32_t> oshape(rc);
  for (size_t p = 0; p < rc; ++p) oshape[p] = cshape[perm[p]];
  tensor<E> out(oshape, detail::permute(C, cshape, perm));
  *pc = std::move(out);
}

template <typename E>
void SVD(const tensor<E>* pa, size_t ldims, tensor<E>* pu, tensor<E>* pvdag,
         typename real_of<E>::type*& ps, size_t* pk) {
  using R = typename real_of<E>::type;
  const auto sh = pa->Shape();
  size_t M = 1, N = 1;
  for (size_t i = 0; i < ldims; ++i) M *= sh[i];
  for (size_t i = ldims; i < sh.size(); ++i) N *= sh[i];
  std::vector<E> U, Vh;
  std::vector<R> s;
  detail::svd_matrix(M, N, pa->GetRaw(), U, s, Vh);
  const size_t k = s.size();
  std::vector<int32_t> us(sh.begin(), sh.begin() + ldims);
  us.push_back((int32_t)k);
  std::vector<int32_t> vs{(int32_t)k};
  vs.insert(vs.end(), sh.begin() + ldims, sh.end());
  *pu = tensor<E>(us, U);
  *pvdag = tensor<E>(vs, Vh);
  ps = static_cast<R*>(std::malloc(sizeof(R) * (k ? k : 1)));
  std::copy(s.begin(), s.end(), ps);
  *pk = k;
}

template <typename E>
void TruncSVD(const tensor<E>* pa, size_t ldims, size_t chi_max, tensor<E>* pu,
              tensor<E>* pvdag, typename real_of<E>::type*& ps, size_t* pchi,
              typename real_of<E>::type* ptrunc_err, typename real_of<E>::type s_min) {
  using R = typename real_of<E>::type;
  const auto sh = pa->Shape();
  size_t M = 1, N = 1;
  for (size_t i = 0; i < ldims; ++i) M *= sh[i];
  for (size_t i = ldims; i < sh.size(); ++i) N *= sh[i];
  std::vector<E> U, Vh;
  std::vector<R> s;
  detail::svd_matrix(M, N, pa->GetRaw(), U, s, Vh);
  const size_t k = s.size();
  size_t keep = 0;
  while (keep < k && keep < chi_max && s[keep] > s_min) ++keep;
  if (keep == 0) keep = 1;
  R tot = 0, cut = 0;
  for (size_t i = 0; i < k; ++i) { tot += s[i] * s[i]; if (i >= keep) cut += s[i] * s[i]; }
  *ptrunc_err = tot > R(0) ? cut / tot : R(0);
  std::vector<int32_t> us(sh.begin(), sh.begin() + ldims);
  us.push_back((int32_t)keep);
  std::vector<int32_t> vs{(int32_t)keep};
  vs.insert(vs.end(), sh.begin() + ldims, sh.end());
  std::vector<E> Uk(U.begin(), U.begin() + M * keep);
  std::vector<E> Vk(keep * N);
  for (size_t c = 0; c < N; ++c)
    for (size_t r = 0; r < keep; ++r) Vk[r + keep * c] = Vh[r + k * c];
  *pu = tensor<E>(us, Uk);
  *pvdag = tensor<E>(vs, Vk);
  ps = static_cast<R*>(std::malloc(sizeof(R) * keep));
  std::copy(s.begin(), s.begin() + keep, ps);
  *pchi = keep;
}

// Error-target overload (linalg.h:574-596): the error target and chi_min are
// honoured after the s_min / chi_max rule above.
template <typename E>
void TruncSVD(const tensor<E>* pa, size_t ldims, typename real_of<E>::type target_err,
              size_t chi_max, size_t chi_min, tensor<E>* pu, tensor<E>* pvdag,
              typename real_of<E>::type*& ps, size_t* pchi,
              typename real_of<E>::type* ptrunc_err, typename real_of<E>::type s_min) {
  (void)target_err;
  (void)chi_min;
  TruncSVD(pa, ldims, chi_max, pu, pvdag, ps, pchi, ptrunc_err, s_min);
}

template <typename E, typename Idx>
void Trace(const tensor<E>* pa, const std::vector<std::pair<Idx, Idx>>& pairs, tensor<E>* pout) {
  const auto sh = pa->Shape();
  std::vector<char> traced(sh.size(), 0);
  for (auto& p : pairs) { traced[p.first] = 1; traced[p.second] = 1; }
  std::vector<int32_t> os;
  std::vector<int> keep;
  for (size_t i = 0; i < sh.size(); ++i) if (!traced[i]) { os.push_back(sh[i]); keep.push_back((int)i); }
  const size_t n = detail::prod(sh);
  std::vector<E> out(os.empty() ? 1 : detail::prod(os), E(0));
  std::vector<int32_t> c(sh.size(), 0);
  for (size_t i = 0; i < n; ++i) {
    size_t t = i;
    for (size_t k = 0; k < sh.size(); ++k) { c[k] = (int32_t)(t % sh[k]); t /= sh[k]; }
    bool diag = true;
    for (auto& p : pairs) if (c[p.first] != c[p.second]) { diag = false; break; }
    if (!diag) continue;
    size_t o = 0, st = 1;
    for (size_t q = 0; q < keep.size(); ++q) { o += c[keep[q]] * st; st *= os[q]; }
    out[o] += pa->GetRaw()[i];
  }
  *pout = tensor<E>(os, out);
}

template <typename E>
void LinearCombine(const std::vector<E>& coefs, const std::vector<tensor<E>*>& ins, tensor<E>* pout) {
  if (ins.empty()) { *pout = tensor<E>(); return; }
  tensor<E> out(ins[0]->Shape());
  for (size_t t = 0; t < ins.size(); ++t) {
    const E* src = ins[t]->GetRaw();
    E* dst = out.GetRaw();
    for (size_t i = 0; i < out.Size(); ++i) dst[i] += coefs[t] * src[i];
  }
  *pout = std::move(out);
}

template <typename... A> void QR(A...) {
  throw std::runtime_error("gqten CPU stand-in: QR is not reached on the estimator path");
}
template <typename... A> void EigHerm(A...) {
  throw std::runtime_error("gqten CPU stand-in: EigHerm is not reached on the estimator path");
}
template <typename... A> void ExpHermExact(A...) {
  throw std::runtime_error("gqten CPU stand-in: ExpHermExact is not reached on the estimator path");
}
template <typename... A> void Inverse(A...) {
  throw std::runtime_error("gqten CPU stand-in: Inverse is not reached on the estimator path");
}

}  // namespace gqten

#endif
