// gqten::tensor<E> for tnbp's apps running on tnbp_b200.
//
// tnbp's apps (apps/estimator, apps/kicked_ising_lattice) are written
// against the Tensor Computing Interface of min-tci, whose gqten backend
// includes "gqten/gqten.h" (external/min-tci/include/tci/gqten/inc_all.h).
// Putting this directory first on the include path makes those apps, their
// headers and min-tci compile unchanged on top of tnbp_b200:
//
//   * gqten::tensor<E> is a host tensor (column-major, coordinate 0 fastest,
//     the order min-tci's assign_from_range fills) with the member functions
//     min-tci calls, and Contract / SVD / TruncSVD / LinearCombine / Trace /
//     QR are host implementations.  They serve the parts of the apps that are
//     not the estimator's hot path: building the circuit's tensor-product
//     operators (QasmToTPO, CircuitTPO, OptTPObySVD), the product state and
//     the Pauli operators.
//   * The hot path -- AbsorbTPO, BeliefPropagation, BeliefPropagationCondition,
//     Truncation and both Measure overloads -- runs on the GPU: for the
//     apps' tensor type gqten::tensor<std::complex<double>> this header
//     declares non-template overloads of those tnbp functions (an exact
//     match, so overload resolution prefers them to tnbp's templates) whose
//     definitions (tnbp_b200/dropin/device_overloads.cpp) call the C ABI of
//     include/tnbp_b200.h on a device-resident copy of the caller's state.
//
// The apps' MPI calls go to the one-rank communicator of "mpi.h" beside this
// directory: tnbp_b200 runs one lattice per process on one GPU.
//
// Semantics restated here (gqten itself is not part of the reference tree):
// Normalize divides by the Frobenius norm and returns it; SVD returns the
// singular values in descending order; TruncSVD keeps the values above s_min
// (absolute), at most chi_max and at least one, with truncation error
// sum(cut s^2) / sum(s^2).  These are the rules the engine's truncation uses.
#ifndef TNBP_DROPIN_GQTEN_GQTEN_H
#define TNBP_DROPIN_GQTEN_GQTEN_H

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../mpi.h"

namespace gqten {

template <typename T> struct RealOf { using type = T; };
template <typename T> struct RealOf<std::complex<T>> { using type = T; };

inline float GetReal(float a) { return a; }
inline double GetReal(double a) { return a; }
inline float GetReal(const std::complex<float>& a) { return a.real(); }
inline double GetReal(const std::complex<double>& a) { return a.real(); }

namespace detail {

template <typename T> inline T cj(const T& x) { return x; }
template <typename T> inline std::complex<T> cj(const std::complex<T>& x) { return std::conj(x); }
template <typename T> inline T mag2(const T& x) { return x * x; }
template <typename T> inline T mag2(const std::complex<T>& x) { return std::norm(x); }

using Shape = std::vector<int32_t>;

inline size_t numel(const Shape& s) {
  size_t n = 1;
  for (int32_t d : s) {
    if (d < 0) throw std::invalid_argument("gqten::tensor: negative dimension");
    n *= static_cast<size_t>(d);
  }
  return n;
}

// out = in with its axes reordered: axis k of out is axis perm[k] of in.
template <typename E>
std::vector<E> reorder(const std::vector<E>& in, const Shape& shape, const std::vector<int>& perm) {
  const size_t r = shape.size(), n = in.size();
  bool identity = true;
  for (size_t k = 0; k < r; ++k) identity = identity && perm[k] == (int)k;
  if (identity || n <= 1) return in;
  std::vector<size_t> in_stride(r);
  size_t st = 1;
  for (size_t k = 0; k < r; ++k) { in_stride[k] = st; st *= (size_t)shape[k]; }
  std::vector<size_t> dim(r), step(r);
  for (size_t k = 0; k < r; ++k) { dim[k] = (size_t)shape[perm[k]]; step[k] = in_stride[perm[k]]; }
  std::vector<E> out(n);
  std::vector<size_t> ctr(r, 0);
  size_t src = 0;
  for (size_t o = 0; o < n; ++o) {
    out[o] = in[src];
    for (size_t k = 0; k < r; ++k) {  // odometer over out's coordinates
      src += step[k];
      if (++ctr[k] < dim[k]) break;
      src -= step[k] * dim[k];
      ctr[k] = 0;
    }
  }
  return out;
}

// C (m x n) = A (m x k) B (k x n), column-major.
template <typename E>
void matmul(size_t m, size_t n, size_t k, const E* A, const E* B, E* C) {
  std::fill(C, C + m * n, E(0));
  for (size_t j = 0; j < n; ++j)
    for (size_t l = 0; l < k; ++l) {
      const E b = B[l + k * j];
      if (b == E(0)) continue;
      const E* a = A + m * l;
      E* c = C + m * j;
      for (size_t i = 0; i < m; ++i) c[i] += a[i] * b;
    }
}

// One-sided (Hestenes) Jacobi on the columns of A (m x n, m >= n): on return
// the columns of A are mutually orthogonal and A_in = A_out W^H with W
// unitary (n x n).  A pair is treated as orthogonal when
// |a_p^H a_q| <= n eps |a_p| |a_q|.
template <typename E>
void orthogonalize_columns(size_t m, size_t n, std::vector<E>& A, std::vector<E>& W) {
  using R = typename RealOf<E>::type;
  W.assign(n * n, E(0));
  for (size_t i = 0; i < n; ++i) W[i + n * i] = E(1);
  const R eps = std::numeric_limits<R>::epsilon() * R(n > 1 ? n : 1);
  for (int sweep = 0; sweep < 100; ++sweep) {
    bool rotated = false;
    for (size_t p = 0; p + 1 < n; ++p)
      for (size_t q = p + 1; q < n; ++q) {
        E* ap = &A[m * p];
        E* aq = &A[m * q];
        R alpha = 0, beta = 0;
        E gamma(0);
        for (size_t i = 0; i < m; ++i) {
          alpha += mag2(ap[i]);
          beta += mag2(aq[i]);
          gamma += cj(ap[i]) * aq[i];
        }
        const R g = std::abs(gamma);
        if (g == R(0) || g <= eps * std::sqrt(alpha) * std::sqrt(beta)) continue;
        rotated = true;
        const E phase = gamma / g;  // a_q e^{-i phi} makes the pair's overlap real
        const R zeta = (beta - alpha) / (R(2) * g);
        const R t = (zeta >= R(0) ? R(1) : R(-1)) / (std::abs(zeta) + std::sqrt(R(1) + zeta * zeta));
        const R c = R(1) / std::sqrt(R(1) + t * t), s = c * t;
        for (size_t i = 0; i < m; ++i) {
          const E x = ap[i], y = aq[i] * cj(phase);
          ap[i] = c * x - s * y;
          aq[i] = s * x + c * y;
        }
        E* wp = &W[n * p];
        E* wq = &W[n * q];
        for (size_t i = 0; i < n; ++i) {
          const E x = wp[i], y = wq[i] * cj(phase);
          wp[i] = c * x - s * y;
          wq[i] = s * x + c * y;
        }
      }
    if (!rotated) return;
  }
}

// Thin SVD of the m x n column-major matrix M: U (m x r), s (r, descending),
// Vh (r x n), r = min(m, n).
template <typename E>
void thin_svd(size_t m, size_t n, const E* M, std::vector<E>& U, std::vector<typename RealOf<E>::type>& s,
              std::vector<E>& Vh) {
  using R = typename RealOf<E>::type;
  const bool wide = m < n;
  const size_t rows = wide ? n : m, cols = wide ? m : n;  // work on M or M^H, tall
  std::vector<E> A(rows * cols);
  for (size_t j = 0; j < cols; ++j)
    for (size_t i = 0; i < rows; ++i) A[i + rows * j] = wide ? cj(M[j + m * i]) : M[i + m * j];
  std::vector<E> W;
  orthogonalize_columns(rows, cols, A, W);
  std::vector<R> norm(cols);
  for (size_t j = 0; j < cols; ++j) {
    R acc = 0;
    for (size_t i = 0; i < rows; ++i) acc += mag2(A[i + rows * j]);
    norm[j] = std::sqrt(acc);
  }
  std::vector<size_t> order(cols);
  std::iota(order.begin(), order.end(), size_t(0));
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return norm[a] > norm[b]; });
  // tall factorization: A_in = Q diag(s) W^H, Q = normalized columns of A
  std::vector<E> Q(rows * cols, E(0)), Wk(cols * cols);
  s.assign(cols, R(0));
  for (size_t jj = 0; jj < cols; ++jj) {
    const size_t j = order[jj];
    s[jj] = norm[j];
    if (norm[j] > R(0))
      for (size_t i = 0; i < rows; ++i) Q[i + rows * jj] = A[i + rows * j] / norm[j];
    for (size_t i = 0; i < cols; ++i) Wk[i + cols * jj] = W[i + cols * j];
  }
  // columns of Q for zero singular values: complete to an orthonormal set
  for (size_t jj = 0; jj < cols; ++jj) {
    if (s[jj] > R(0)) continue;
    for (size_t e = 0; e < rows; ++e) {
      std::vector<E> v(rows, E(0));
      v[e] = E(1);
      for (size_t k = 0; k < cols; ++k) {
        if (k == jj || (s[k] == R(0) && k > jj)) continue;
        E d(0);
        for (size_t i = 0; i < rows; ++i) d += cj(Q[i + rows * k]) * v[i];
        for (size_t i = 0; i < rows; ++i) v[i] -= d * Q[i + rows * k];
      }
      R nv = 0;
      for (size_t i = 0; i < rows; ++i) nv += mag2(v[i]);
      nv = std::sqrt(nv);
      if (nv > R(0.5)) {
        for (size_t i = 0; i < rows; ++i) Q[i + rows * jj] = v[i] / nv;
        break;
      }
    }
  }
  if (!wide) {  // M = Q s W^H
    U = Q;
    Vh.assign(cols * n, E(0));
    for (size_t j = 0; j < n; ++j)
      for (size_t i = 0; i < cols; ++i) Vh[i + cols * j] = cj(Wk[j + cols * i]);
  } else {  // M^H = Q s W^H  =>  M = W s Q^H
    U = Wk;  // m x m
    Vh.assign(cols * n, E(0));
    for (size_t j = 0; j < n; ++j)
      for (size_t i = 0; i < cols; ++i) Vh[i + cols * j] = cj(Q[j + rows * i]);
  }
}

}  // namespace detail

template <typename ElemT>
class tensor {
 public:
  using value_type = ElemT;
  using RealT = typename RealOf<ElemT>::type;
  using ShapeT = std::vector<int32_t>;

  // rank 0: a scalar (0 until set)
  tensor() : data_(1, ElemT(0)) {}
  explicit tensor(const ShapeT& shape) : shape_(shape), data_(shape.empty() ? 1 : detail::numel(shape), ElemT(0)) {}
  tensor(const ShapeT& shape, const std::vector<ElemT>& data) : shape_(shape), data_(data) {
    if (data_.size() != (shape.empty() ? 1 : detail::numel(shape)))
      throw std::invalid_argument("gqten::tensor: data size does not match the shape");
  }
  // Takes ownership of a buffer from std::malloc / std::calloc holding
  // numel(shape) elements (released with std::free).
  tensor(const ShapeT& shape, ElemT* owned) : shape_(shape) {
    const size_t n = shape.empty() ? 1 : detail::numel(shape);
    data_.assign(owned, owned + n);
    std::free(owned);
  }

  size_t Rank() const { return shape_.size(); }
  ShapeT Shape() const { return shape_; }
  size_t Size() const { return data_.size(); }

  template <typename C>
  size_t Offset(const C& coors) const {
    size_t off = 0, st = 1;
    size_t k = 0;
    for (auto c : coors) {
      if (k >= shape_.size()) break;
      off += static_cast<size_t>(c) * st;
      st *= static_cast<size_t>(shape_[k++]);
    }
    return off;
  }
  template <typename C, typename std::enable_if<!std::is_integral<C>::value, int>::type = 0>
  ElemT GetElem(const C& coors) const { return data_.at(Offset(coors)); }
  template <typename I, typename std::enable_if<std::is_integral<I>::value, int>::type = 0>
  ElemT GetElem(I i) const { return data_.at(static_cast<size_t>(i)); }
  ElemT GetElem(std::initializer_list<int32_t> coors) const { return data_.at(Offset(coors)); }
  template <typename C, typename std::enable_if<!std::is_integral<C>::value, int>::type = 0>
  void SetElem(const C& coors, const ElemT& v) { data_.at(Offset(coors)) = v; }
  template <typename I, typename std::enable_if<std::is_integral<I>::value, int>::type = 0>
  void SetElem(I i, const ElemT& v) { data_.at(static_cast<size_t>(i)) = v; }
  void SetElem(std::initializer_list<int32_t> coors, const ElemT& v) { data_.at(Offset(coors)) = v; }

  const ElemT* GetRaw() const { return data_.data(); }
  ElemT* GetRaw() { return data_.data(); }
  const std::vector<ElemT>& Data() const { return data_; }
  std::vector<ElemT>& Data() { return data_; }

  // The value of a rank-0 tensor; 1 for a tensor of rank >= 1 (its elements
  // carry no separate factor).
  ElemT GetScale() const { return shape_.empty() ? data_[0] : ElemT(1); }
  void SetScale(const ElemT& s) {
    if (shape_.empty()) data_[0] = s;
    else for (auto& x : data_) x *= s;
  }

  RealT CalcNorm() const {
    RealT acc = 0;
    for (const auto& x : data_) acc += detail::mag2(x);
    return std::sqrt(acc);
  }
  RealT Normalize() {
    const RealT n = CalcNorm();
    if (n > RealT(0))
      for (auto& x : data_) x /= n;
    return n;
  }
  void Conjugate() {
    for (auto& x : data_) x = detail::cj(x);
  }
  // Axis k of the result is axis order[k] of this tensor.
  template <typename Idx>
  void Transpose(const std::vector<Idx>& order) {
    std::vector<int> perm(order.begin(), order.end());
    if (perm.size() != shape_.size()) throw std::invalid_argument("gqten::tensor::Transpose: wrong rank");
    data_ = detail::reorder(data_, shape_, perm);
    ShapeT ns(shape_.size());
    for (size_t k = 0; k < perm.size(); ++k) ns[k] = shape_[perm[k]];
    shape_ = ns;
  }
  template <typename S>
  void Reshape(const S& new_shape) {
    ShapeT ns(new_shape.begin(), new_shape.end());
    if ((ns.empty() ? 1 : detail::numel(ns)) != data_.size())
      throw std::invalid_argument("gqten::tensor::Reshape: element count changes");
    shape_ = ns;
  }

  // text form: rank, dims, then the elements in storage order
  void StreamWrite(std::ostream& os) const {
    os << shape_.size();
    for (auto d : shape_) os << ' ' << d;
    os << '\n' << std::setprecision(17);
    for (const auto& x : data_) os << x << '\n';
  }
  void StreamRead(std::istream& is) {
    size_t r = 0;
    is >> r;
    shape_.assign(r, 0);
    for (auto& d : shape_) is >> d;
    data_.assign(shape_.empty() ? 1 : detail::numel(shape_), ElemT(0));
    for (auto& x : data_) is >> x;
  }
  template <typename D, typename G>
  void Random(int, const std::vector<D>&, G& gen) {
    std::uniform_real_distribution<RealT> u(RealT(-1), RealT(1));
    for (auto& x : data_) x = random_value(u, gen);
  }
  void FormattedPrint() const {
    std::cout << "tensor of rank " << shape_.size() << ", shape (";
    for (size_t k = 0; k < shape_.size(); ++k) std::cout << (k ? "," : "") << shape_[k];
    std::cout << ")\n";
    for (size_t i = 0; i < data_.size(); ++i) std::cout << "  [" << i << "] " << data_[i] << '\n';
  }

 private:
  template <typename U, typename G>
  static ElemT random_value(U& u, G& gen) {
    if constexpr (std::is_same<ElemT, RealT>::value) return u(gen);
    else return ElemT(u(gen), u(gen));
  }
  ShapeT shape_;
  std::vector<ElemT> data_;
};

// C = A B contracted over the axes whose labels are negative (equal labels
// pair up); a non-negative label is the axis' position in C.
template <typename E>
void Contract(const tensor<E>* pa, const tensor<E>* pb, const std::vector<int>& la, const std::vector<int>& lb,
              tensor<E>* pc) {
  const auto sa = pa->Shape(), sb = pb->Shape();
  if (la.size() != sa.size() || lb.size() != sb.size()) throw std::invalid_argument("gqten::Contract: label count");
  std::vector<std::pair<int, int>> freeA, freeB;  // (output position, axis)
  std::vector<std::pair<int, int>> cntA, cntB;    // (label, axis)
  for (size_t k = 0; k < la.size(); ++k) (la[k] >= 0 ? freeA : cntA).push_back({la[k], (int)k});
  for (size_t k = 0; k < lb.size(); ++k) (lb[k] >= 0 ? freeB : cntB).push_back({lb[k], (int)k});
  std::sort(freeA.begin(), freeA.end());
  std::sort(freeB.begin(), freeB.end());
  std::sort(cntA.begin(), cntA.end(), [](auto x, auto y) { return x.first > y.first; });
  std::sort(cntB.begin(), cntB.end(), [](auto x, auto y) { return x.first > y.first; });
  if (cntA.size() != cntB.size()) throw std::invalid_argument("gqten::Contract: unpaired contracted label");
  size_t M = 1, N = 1, K = 1;
  std::vector<int> permA, permB;
  for (auto& f : freeA) { permA.push_back(f.second); M *= (size_t)sa[f.second]; }
  for (size_t i = 0; i < cntA.size(); ++i) {
    if (cntA[i].first != cntB[i].first || sa[cntA[i].second] != sb[cntB[i].second])
      throw std::invalid_argument("gqten::Contract: contracted axes do not match");
    permA.push_back(cntA[i].second);
    permB.push_back(cntB[i].second);
    K *= (size_t)sa[cntA[i].second];
  }
  for (auto& f : freeB) { permB.push_back(f.second); N *= (size_t)sb[f.second]; }
  const auto A = detail::reorder(pa->Data(), sa, permA);
  const auto B = detail::reorder(pb->Data(), sb, permB);
  std::vector<E> C(M * N);
  detail::matmul(M, N, K, A.data(), B.data(), C.data());
  // C's axes are (free A by position, free B by position); place them
  const size_t rc = freeA.size() + freeB.size();
  typename tensor<E>::ShapeT sc(rc), cur;
  std::vector<int> pos;
  for (auto& f : freeA) { cur.push_back(sa[f.second]); pos.push_back(f.first); }
  for (auto& f : freeB) { cur.push_back(sb[f.second]); pos.push_back(f.first); }
  std::vector<int> perm(rc, -1);
  for (size_t k = 0; k < rc; ++k) {
    if (pos[k] < 0 || (size_t)pos[k] >= rc || perm[pos[k]] != -1)
      throw std::invalid_argument("gqten::Contract: output positions must be 0 .. rank-1 once each");
    perm[pos[k]] = (int)k;
    sc[pos[k]] = cur[k];
  }
  *pc = tensor<E>(sc, rc == 0 ? C : detail::reorder(C, cur, perm));
}

// Thin SVD of A viewed as a matrix (first ldims axes as rows): U has A's row
// axes plus one, Vh one plus A's column axes; s (k values, descending) in a
// std::malloc'd buffer that the caller owns.
template <typename E>
void SVD(const tensor<E>* pa, size_t ldims, tensor<E>* pu, tensor<E>* pvh, typename RealOf<E>::type*& ps,
         size_t* pk) {
  using R = typename RealOf<E>::type;
  const auto sh = pa->Shape();
  size_t m = 1, n = 1;
  for (size_t i = 0; i < sh.size(); ++i) (i < ldims ? m : n) *= (size_t)sh[i];
  std::vector<E> U, Vh;
  std::vector<R> s;
  detail::thin_svd(m, n, pa->GetRaw(), U, s, Vh);
  const size_t k = s.size();
  typename tensor<E>::ShapeT su(sh.begin(), sh.begin() + ldims), sv{(int32_t)k};
  su.push_back((int32_t)k);
  sv.insert(sv.end(), sh.begin() + ldims, sh.end());
  *pu = tensor<E>(su, U);
  *pvh = tensor<E>(sv, Vh);
  ps = static_cast<R*>(std::malloc(sizeof(R) * (k ? k : 1)));
  std::copy(s.begin(), s.end(), ps);
  *pk = k;
}

namespace detail {
template <typename E>
void cut_svd(const tensor<E>* pa, size_t ldims, size_t keep_max, size_t keep_min,
             typename RealOf<E>::type target_err, tensor<E>* pu, tensor<E>* pvh, typename RealOf<E>::type*& ps,
             size_t* pchi, typename RealOf<E>::type* perr, typename RealOf<E>::type s_min) {
  using R = typename RealOf<E>::type;
  R* s_all = nullptr;
  size_t k = 0;
  tensor<E> U, Vh;
  SVD(pa, ldims, &U, &Vh, s_all, &k);
  R total = 0;
  for (size_t i = 0; i < k; ++i) total += s_all[i] * s_all[i];
  size_t keep = 0;
  while (keep < k && keep < keep_max && s_all[keep] > s_min) ++keep;
  // the smallest count (at least keep_min) whose discarded weight meets the target
  if (target_err > R(0)) {
    size_t need = std::max<size_t>(1, keep_min);
    R cut = 0;
    for (size_t i = need; i < keep; ++i) cut += s_all[i] * s_all[i];
    while (need < keep && total > R(0) && cut / total > target_err) {
      cut -= s_all[need] * s_all[need];
      ++need;
    }
    keep = std::min(keep, need);
  }
  keep = std::max<size_t>(keep, std::min<size_t>(1, k));
  R cut = 0;
  for (size_t i = keep; i < k; ++i) cut += s_all[i] * s_all[i];
  *perr = total > R(0) ? cut / total : R(0);
  const auto su = U.Shape(), sv = Vh.Shape();
  const size_t rows = U.Size() / (k ? k : 1), cols = Vh.Size() / (k ? k : 1);
  std::vector<E> Uk(U.Data().begin(), U.Data().begin() + rows * keep), Vk(keep * cols);
  for (size_t j = 0; j < cols; ++j)
    for (size_t i = 0; i < keep; ++i) Vk[i + keep * j] = Vh.Data()[i + k * j];
  auto su2 = su, sv2 = sv;
  su2.back() = (int32_t)keep;
  sv2.front() = (int32_t)keep;
  *pu = tensor<E>(su2, Uk);
  *pvh = tensor<E>(sv2, Vk);
  ps = static_cast<R*>(std::malloc(sizeof(R) * (keep ? keep : 1)));
  std::copy(s_all, s_all + keep, ps);
  std::free(s_all);
  *pchi = keep;
}
}  // namespace detail

template <typename E>
void TruncSVD(const tensor<E>* pa, size_t ldims, size_t chi_max, tensor<E>* pu, tensor<E>* pvh,
              typename RealOf<E>::type*& ps, size_t* pchi, typename RealOf<E>::type* perr,
              typename RealOf<E>::type s_min) {
  detail::cut_svd(pa, ldims, chi_max, 1, typename RealOf<E>::type(0), pu, pvh, ps, pchi, perr, s_min);
}
template <typename E>
void TruncSVD(const tensor<E>* pa, size_t ldims, typename RealOf<E>::type target_err, size_t chi_max,
              size_t chi_min, tensor<E>* pu, tensor<E>* pvh, typename RealOf<E>::type*& ps, size_t* pchi,
              typename RealOf<E>::type* perr, typename RealOf<E>::type s_min) {
  detail::cut_svd(pa, ldims, chi_max, chi_min, target_err, pu, pvh, ps, pchi, perr, s_min);
}

// out = sum_i coefs[i] * (*ins[i]) (all of one shape)
template <typename E, typename C>
void LinearCombine(const std::vector<C>& coefs, const std::vector<tensor<E>*>& ins, tensor<E>* pout) {
  if (ins.empty()) { *pout = tensor<E>(); return; }
  tensor<E> out(ins[0]->Shape());
  for (size_t i = 0; i < ins.size(); ++i) {
    if (ins[i]->Size() != out.Size()) throw std::invalid_argument("gqten::LinearCombine: shapes differ");
    const E c = static_cast<E>(coefs[i]);
    for (size_t k = 0; k < out.Size(); ++k) out.GetRaw()[k] += c * ins[i]->GetRaw()[k];
  }
  *pout = out;
}

// Trace over the axis pairs (a, b) of each entry of pairs (equal dims).
template <typename E, typename P>
void Trace(const tensor<E>* pin, const P& pairs, tensor<E>* pout) {
  const auto sh = pin->Shape();
  std::vector<int> traced(sh.size(), -1);  // partner axis
  for (const auto& pr : pairs) {
    const int a = (int)pr.first, b = (int)pr.second;
    if (sh[a] != sh[b]) throw std::invalid_argument("gqten::Trace: paired axes differ in size");
    traced[a] = b;
    traced[b] = a;
  }
  std::vector<int> keep;
  typename tensor<E>::ShapeT ks;
  for (size_t k = 0; k < sh.size(); ++k)
    if (traced[k] < 0) { keep.push_back((int)k); ks.push_back(sh[k]); }
  tensor<E> out(ks);
  std::vector<int32_t> c(sh.size(), 0);
  for (size_t i = 0; i < pin->Size(); ++i) {
    bool diag = true;
    for (size_t k = 0; k < sh.size() && diag; ++k) diag = traced[k] < 0 || c[k] == c[traced[k]];
    if (diag) {
      size_t o = 0, ost = 1;
      for (size_t j = 0; j < keep.size(); ++j) { o += (size_t)c[keep[j]] * ost; ost *= (size_t)ks[j]; }
      out.GetRaw()[o] += pin->GetRaw()[i];
    }
    for (size_t k = 0; k < sh.size(); ++k) {
      if (++c[k] < sh[k]) break;
      c[k] = 0;
    }
  }
  *pout = out;
}

// A = Q R with Q's columns orthonormal (modified Gram-Schmidt on A viewed as
// a matrix with the first ldims axes as rows).
template <typename E>
void QR(const tensor<E>* pa, size_t ldims, tensor<E>* pq, tensor<E>* pr) {
  using R = typename RealOf<E>::type;
  const auto sh = pa->Shape();
  size_t m = 1, n = 1;
  for (size_t i = 0; i < sh.size(); ++i) (i < ldims ? m : n) *= (size_t)sh[i];
  const size_t k = std::min(m, n);
  std::vector<E> Q(m * k, E(0)), Rm(k * n, E(0));
  std::vector<E> A(pa->Data());
  for (size_t j = 0; j < n; ++j) {
    E* a = &A[m * j];
    for (size_t i = 0; i < std::min(j, k); ++i) {
      E d(0);
      for (size_t r = 0; r < m; ++r) d += detail::cj(Q[r + m * i]) * a[r];
      Rm[i + k * j] = d;
      for (size_t r = 0; r < m; ++r) a[r] -= d * Q[r + m * i];
    }
    if (j < k) {
      R nv = 0;
      for (size_t r = 0; r < m; ++r) nv += detail::mag2(a[r]);
      nv = std::sqrt(nv);
      Rm[j + k * j] = E(nv);
      if (nv > R(0))
        for (size_t r = 0; r < m; ++r) Q[r + m * j] = a[r] / nv;
    }
  }
  typename tensor<E>::ShapeT sq(sh.begin(), sh.begin() + ldims), sr{(int32_t)k};
  sq.push_back((int32_t)k);
  sr.insert(sr.end(), sh.begin() + ldims, sh.end());
  *pq = tensor<E>(sq, Q);
  *pr = tensor<E>(sr, Rm);
}

// Named by min-tci's wrappers (eigh, exp_herm, inverse) but used by neither
// app: declared so that min-tci compiles; calling one throws.
template <typename E, typename W, typename V>
void EigHerm(const tensor<E>*, size_t, W*&, V*&, size_t*, char, char) {
  throw std::runtime_error("gqten::EigHerm is not provided by the tnbp_b200 drop-in");
}
template <typename E, typename O>
void ExpHermExact(const tensor<E>*, O, tensor<E>*) {
  throw std::runtime_error("gqten::ExpHermExact is not provided by the tnbp_b200 drop-in");
}
template <typename E, typename O>
void Inverse(const tensor<E>*, O, tensor<E>*) {
  throw std::runtime_error("gqten::Inverse is not provided by the tnbp_b200 drop-in");
}

}  // namespace gqten

// ------------------------------------------------------ GPU hot path
// Non-template overloads of tnbp's hot-path functions for the apps' tensor
// type; see tnbp_b200/dropin/device_overloads.cpp.  Parameter lists are
// those of the templates in include/tnbp/ptns/function/{apply,bp,truncation,
// measure}.h with TenT = gqten::tensor<std::complex<double>>.
namespace tci { struct gqten_handle; }
namespace tnbp {
using DropinTensor = gqten::tensor<std::complex<double>>;

void AbsorbTPO(tci::gqten_handle& ctx, const std::vector<DropinTensor>& O,
               const std::vector<std::pair<int, int>>& Edge, std::vector<DropinTensor>& V,
               const std::vector<int>& SiteIdx, const std::map<int, int>& Site_To_MpiRank,
               std::vector<DropinTensor>& E, const std::vector<int>& EdgeIdx, MPI_Comm comm);

void BeliefPropagation(tci::gqten_handle& ctx, const std::vector<std::pair<int, int>>& I,
                       const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                       const std::map<int, int>& Site_To_MpiRank, const std::vector<std::pair<int, int>>& J,
                       const std::vector<DropinTensor>& E, const std::vector<int>& EdgeIdx, MPI_Comm comm,
                       std::vector<DropinTensor>& F);

void BeliefPropagationCondition(tci::gqten_handle& ctx, const std::vector<std::pair<int, int>>& I,
                                const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                                const std::map<int, int>& Site_To_MpiRank, const std::vector<DropinTensor>& E,
                                const std::vector<int>& EdgeIdx, MPI_Comm comm, double& result);

void Truncation(tci::gqten_handle& ctx, const std::vector<std::pair<int, int>>& I, std::vector<DropinTensor>& V,
                const std::vector<int>& SiteIdx, const std::map<int, int>& Site_To_MpiRank,
                std::vector<DropinTensor>& E, const std::vector<int>& EdgeIdx, MPI_Comm comm, int32_t max_dim,
                double eps, double err, std::vector<int32_t>& res_bond_dim, std::vector<double>& res_trunc_err);

std::vector<std::complex<double>> Measure(tci::gqten_handle& ctx, const std::vector<std::pair<int, int>>& I,
                                          const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                                          const std::map<int, int>& Site_To_MpiRank,
                                          const std::vector<DropinTensor>& E, const std::vector<int> EdgeIdx,
                                          MPI_Comm comm, const std::vector<int>& Site,
                                          const std::vector<DropinTensor>& O);

std::vector<std::complex<double>> Measure(tci::gqten_handle& ctx, const std::vector<std::pair<int, int>>& I,
                                          const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                                          const std::map<int, int>& Site_To_MpiRank,
                                          const std::vector<DropinTensor>& E, const std::vector<int> EdgeIdx,
                                          MPI_Comm comm, const std::vector<std::pair<int, int>>& Edge,
                                          const std::vector<DropinTensor>& O);
}  // namespace tnbp

#endif
