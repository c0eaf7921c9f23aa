// Host check of the invariant-divisor arithmetic the index kernels use
// (FastDiv in tnbp_b200/csrc/kernels.cuh): for divisors 1..70000, powers of
// two and their neighbours, and dividends at the edges and spread over
// [0, 2^31), fast_div must equal exact division.  Prints the count of
// mismatches and of cases; exits non-zero on any mismatch.
#include <cstdint>
#include <cstdio>

#include "kernels.cuh"

int main() {
  unsigned long long cases = 0, bad = 0;
  uint64_t seed = 0x9E3779B97F4A7C15ull;
  auto next = [&]() {
    seed ^= seed << 13;
    seed ^= seed >> 7;
    seed ^= seed << 17;
    return seed;
  };
  auto check = [&](uint32_t d) {
    const tnbp::FastDiv f = tnbp::make_fastdiv(d);
    const uint32_t edge[] = {0u, 1u, d - 1u, d, d + 1u, 2u * d - 1u, 2u * d, 0x7FFFFFFFu, 0x7FFFFFFEu,
                             0x7FFFFFFFu / d * d, 0x7FFFFFFFu / d * d - 1u};
    for (uint32_t x : edge) {
      if (x > 0x7FFFFFFFu) continue;
      ++cases;
      if (tnbp::fast_div(x, f) != x / d) ++bad;
    }
    for (int i = 0; i < 64; ++i) {
      const uint32_t x = (uint32_t)(next() & 0x7FFFFFFFu);
      ++cases;
      if (tnbp::fast_div(x, f) != x / d) ++bad;
    }
  };
  for (uint32_t d = 1; d <= 70000; ++d) check(d);
  for (int k = 0; k < 31; ++k) {
    check(1u << k);
    if (k > 0) check((1u << k) - 1u);
    check((1u << k) + 1u);
  }
  for (int i = 0; i < 20000; ++i) check((uint32_t)(next() % 0x7FFFFFFFu) + 1u);
  std::printf("cases %llu mismatches %llu\n", cases, bad);
  return bad ? 1 : 0;
}
