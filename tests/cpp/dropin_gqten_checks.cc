// The drop-in tensor backend (include/tnbp_dropin/gqten/gqten.h) checked on
// the CPU: Contract against explicit loops, SVD / TruncSVD / QR by their
// defining identities (reconstruction, orthonormality, ordering, the
// truncation rule), Transpose and Reshape by element addresses, Trace and
// LinearCombine by hand.  Prints "ok <name>" per check; exits non-zero on the
// first failure.
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "gqten/gqten.h"

using cd = std::complex<double>;
using T = gqten::tensor<cd>;

static std::mt19937_64 rng(7);
static T random_tensor(const std::vector<int32_t>& sh) {
  std::normal_distribution<double> g;
  T t(sh);
  for (size_t i = 0; i < t.Size(); ++i) t.GetRaw()[i] = cd(g(rng), g(rng));
  return t;
}
static void expect(bool c, const char* what, double v = 0) {
  if (!c) {
    std::printf("FAIL %s (%g)\n", what, v);
    std::exit(1);
  }
  std::printf("ok %s\n", what);
}
static double err_identity(const std::vector<cd>& M, size_t n) {  // |M - I|max, n x n
  double e = 0;
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) e = std::max(e, std::abs(M[i + n * j] - (i == j ? 1.0 : 0.0)));
  return e;
}
// X^H X for an m x k column-major matrix
static std::vector<cd> gram(const cd* X, size_t m, size_t k) {
  std::vector<cd> G(k * k);
  for (size_t a = 0; a < k; ++a)
    for (size_t b = 0; b < k; ++b) {
      cd s = 0;
      for (size_t i = 0; i < m; ++i) s += std::conj(X[i + m * a]) * X[i + m * b];
      G[a + k * b] = s;
    }
  return G;
}

static void check_svd(size_t m, size_t n, bool deficient) {
  T A = random_tensor({(int32_t)m, (int32_t)n});
  if (deficient)  // rank 2
    for (size_t j = 2; j < n; ++j)
      for (size_t i = 0; i < m; ++i) A.GetRaw()[i + m * j] = A.GetRaw()[i] * cd(0.5, j) + A.GetRaw()[i + m] * 0.25;
  T U, Vh;
  double* s = nullptr;
  size_t k = 0;
  gqten::SVD(&A, 1, &U, &Vh, s, &k);
  expect(k == std::min(m, n), "svd rank count");
  for (size_t i = 1; i < k; ++i) expect(s[i] <= s[i - 1], "svd values descending");
  double rec = 0;
  for (size_t i = 0; i < m; ++i)
    for (size_t j = 0; j < n; ++j) {
      cd v = 0;
      for (size_t l = 0; l < k; ++l) v += U.GetRaw()[i + m * l] * s[l] * Vh.GetRaw()[l + k * j];
      rec = std::max(rec, std::abs(v - A.GetRaw()[i + m * j]));
    }
  expect(rec < 1e-12, "svd reconstructs A", rec);
  expect(err_identity(gram(U.GetRaw(), m, k), k) < 1e-12, "svd U orthonormal");
  std::vector<cd> V(n * k);  // Vh^H
  for (size_t l = 0; l < k; ++l)
    for (size_t j = 0; j < n; ++j) V[j + n * l] = std::conj(Vh.GetRaw()[l + k * j]);
  expect(err_identity(gram(V.data(), n, k), k) < 1e-12, "svd Vh rows orthonormal");
  std::free(s);
}

int main() {
  // Contract: C[i, j] = sum_{k, l} A[i, k, l] B[l, k, j]
  {
    T A = random_tensor({3, 4, 5}), B = random_tensor({5, 4, 2}), C;
    gqten::Contract(&A, &B, {0, -1, -2}, {-2, -1, 1}, &C);
    double e = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 2; ++j) {
        cd v = 0;
        for (int k = 0; k < 4; ++k)
          for (int l = 0; l < 5; ++l) v += A.GetElem({i, k, l}) * B.GetElem({l, k, j});
        e = std::max(e, std::abs(v - C.GetElem({i, j})));
      }
    expect(C.Shape() == std::vector<int32_t>({3, 2}) && e < 1e-12, "contract two labels", e);
    // output positions out of order: D[j, i] = sum_k A2[i, k] B2[k, j]
    T A2 = random_tensor({3, 4}), B2 = random_tensor({4, 5}), D;
    gqten::Contract(&A2, &B2, {1, -1}, {-1, 0}, &D);
    e = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 5; ++j) {
        cd v = 0;
        for (int k = 0; k < 4; ++k) v += A2.GetElem({i, k}) * B2.GetElem({k, j});
        e = std::max(e, std::abs(v - D.GetElem({j, i})));
      }
    expect(D.Shape() == std::vector<int32_t>({5, 3}) && e < 1e-12, "contract permuted output", e);
    // full contraction to a scalar, and an outer product
    T S;
    gqten::Contract(&A2, &A2, {-1, -2}, {-1, -2}, &S);
    cd ss = 0;
    for (size_t i = 0; i < A2.Size(); ++i) ss += A2.GetRaw()[i] * A2.GetRaw()[i];
    expect(S.Rank() == 0 && std::abs(S.GetScale() - ss) < 1e-12, "contract to scalar");
    T O;
    gqten::Contract(&A2, &B2, {2, 0}, {1, 3}, &O);
    expect(O.Shape() == std::vector<int32_t>({4, 4, 3, 5}) &&
               std::abs(O.GetElem({1, 2, 0, 4}) - A2.GetElem({0, 1}) * B2.GetElem({2, 4})) < 1e-14,
           "contract outer product");
  }
  // Transpose / Reshape
  {
    T A = random_tensor({2, 3, 4});
    T B = A;
    B.Transpose(std::vector<int>{2, 0, 1});
    bool same = B.Shape() == std::vector<int32_t>({4, 2, 3});
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 4; ++k) same = same && B.GetElem({k, i, j}) == A.GetElem({i, j, k});
    expect(same, "transpose moves axes");
    B.Reshape(std::vector<int32_t>{8, 3});
    expect(B.Shape() == std::vector<int32_t>({8, 3}) && B.GetElem({5, 2}) == B.GetRaw()[5 + 8 * 2],
           "reshape keeps storage order");
  }
  check_svd(7, 4, false);
  check_svd(4, 7, false);
  check_svd(6, 5, true);
  // TruncSVD: s_min (absolute) and chi_max, at least one value, error rule
  {
    T A = random_tensor({6, 6});
    T U, Vh;
    double* s_all = nullptr;
    size_t k = 0;
    gqten::SVD(&A, 1, &U, &Vh, s_all, &k);
    double tot = 0;
    for (size_t i = 0; i < k; ++i) tot += s_all[i] * s_all[i];
    const double smin = 0.5 * (s_all[2] + s_all[3]);  // keeps 3
    T Ut, Vt;
    double* s = nullptr;
    size_t chi = 0;
    double err = -1;
    gqten::TruncSVD(&A, 1, 5, &Ut, &Vt, s, &chi, &err, smin);
    double cut = 0;
    for (size_t i = 3; i < k; ++i) cut += s_all[i] * s_all[i];
    expect(chi == 3 && Ut.Shape()[1] == 3 && Vt.Shape()[0] == 3 && std::abs(err - cut / tot) < 1e-14,
           "truncsvd s_min cut", err);
    std::free(s);
    gqten::TruncSVD(&A, 1, 2, &Ut, &Vt, s, &chi, &err, 0.0);
    expect(chi == 2, "truncsvd chi_max cut");
    std::free(s);
    gqten::TruncSVD(&A, 1, 4, &Ut, &Vt, s, &chi, &err, 1e300);
    expect(chi == 1, "truncsvd keeps at least one");
    std::free(s);
    std::free(s_all);
  }
  // QR
  {
    T A = random_tensor({5, 3}), Q, R;
    gqten::QR(&A, 1, &Q, &R);
    T QR_;
    gqten::Contract(&Q, &R, {0, -1}, {-1, 1}, &QR_);
    double e = 0;
    for (size_t i = 0; i < A.Size(); ++i) e = std::max(e, std::abs(QR_.GetRaw()[i] - A.GetRaw()[i]));
    expect(e < 1e-12 && err_identity(gram(Q.GetRaw(), 5, 3), 3) < 1e-12, "qr", e);
  }
  // Trace and LinearCombine
  {
    T A = random_tensor({3, 2, 3}), t;
    gqten::Trace(&A, std::vector<std::pair<int, int>>{{0, 2}}, &t);
    cd v = A.GetElem({0, 1, 0}) + A.GetElem({1, 1, 1}) + A.GetElem({2, 1, 2});
    expect(t.Shape() == std::vector<int32_t>({2}) && std::abs(t.GetElem({1}) - v) < 1e-14, "trace");
    T B = random_tensor({3, 2, 3}), L;
    std::vector<T*> ins{&A, &B};
    gqten::LinearCombine(std::vector<cd>{cd(2, 0), cd(0, 1)}, ins, &L);
    expect(std::abs(L.GetRaw()[7] - (2.0 * A.GetRaw()[7] + cd(0, 1) * B.GetRaw()[7])) < 1e-14, "linear combine");
  }
  // Normalize / ownership constructor
  {
    T A = random_tensor({4, 4});
    const double n = A.Normalize();
    expect(n > 0 && std::abs(A.CalcNorm() - 1.0) < 1e-14, "normalize to unit Frobenius norm");
    cd* raw = static_cast<cd*>(std::malloc(2 * sizeof(cd)));
    raw[0] = 1.0;
    raw[1] = 2.0;
    T O({2}, raw);
    expect(O.GetElem({1}) == cd(2.0), "takes a malloc'd buffer");
  }
  return 0;
}
