// Host check of which sites the site-resident sweep kernel takes
// (site_sweep_smem_bytes against kSiteSmemMax in tnbp_b200/csrc/kernels.cuh):
// with physical dim 2, degree 4 up to D = 4, degree 3 up to D = 8, degree 2
// up to D = 21, degree 1 up to D = 43, and every shared-memory figure
// 16 (3n + sum D^2 + max(256, max D^2)) bytes.  Exits non-zero on a mismatch.
#include <cstdio>

#include "kernels.cuh"

int main() {
  int bad = 0;
  const int largest_ok[5] = {0, 43, 21, 8, 4};  // by degree
  for (int g = 1; g <= 4; ++g) {
    for (int D = 1; D <= 48; ++D) {
      int dims[tnbp::kMaxLegs];
      for (int k = 0; k < g; ++k) dims[k] = D;
      const size_t b = tnbp::site_sweep_smem_bytes(dims, g, 2);
      size_t n = 2, sd2 = 0;
      for (int k = 0; k < g; ++k) { n *= (size_t)D; sd2 += (size_t)D * D; }
      const size_t part = (size_t)D * D > 256 ? (size_t)D * D : 256;
      if (b != 16 * (3 * n + sd2 + part)) { std::printf("bytes g=%d D=%d: %zu\n", g, D, b); ++bad; }
      const bool ok = b <= tnbp::kSiteSmemMax;
      if (ok != (D <= largest_ok[g])) { std::printf("eligibility g=%d D=%d: %d\n", g, D, (int)ok); ++bad; }
    }
  }
  std::printf("mismatches %d\n", bad);
  return bad ? 1 : 0;
}
