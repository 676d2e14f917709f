// Host check that the 32-bit butterfly rotation (tx::B) is exact: every
// inverse transform that uses it (DCT of 4..64 points, ADST of 8 and 16) is
// driven with 16-bit inputs - every element at an extreme (-32768 / 32767,
// random signs), the full random range, and sparse rows - and each
// butterfly's two sums are formed again in 64 bits (MAV1_BUTTERFLY_CHECK).
// A sum outside 32 bits would make the 32-bit result differ from the
// specification's; the check fails if any sum reaches 2^31 and prints the
// largest magnitude seen. Built and run by tests/test_host.py.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>

static long long g_max = 0;
static long long g_over = 0;
static inline void check_sums(long long a, long long b, long long c, long long s) {
  long long x = a * c - b * s, y = a * s + b * c;
  for (long long v : {x, y}) {
    long long m = v < 0 ? -v : v;
    if (m > g_max) g_max = m;
    if (v > INT32_MAX || v < INT32_MIN) g_over++;
  }
}
#define MAV1_BUTTERFLY_CHECK(a, b, c, s) check_sums(a, b, c, s)

#include "tx.cuh"

template <int N>
static void run_dct(std::mt19937 &g, int trials) {
  constexpr int n = 1 << N;
  std::uniform_int_distribution<int> full(-32768, 32767), bit(0, 1), mode(0, 3);
  for (int t = 0; t < trials; t++) {
    int32_t v[n];
    int m = mode(g);
    for (int i = 0; i < n; i++)
      v[i] = m == 0 ? (bit(g) ? 32767 : -32768) : m == 1 ? full(g) : m == 2 ? (i < n / 2 && bit(g) ? full(g) : 0)
                                                                            : (bit(g) ? (bit(g) ? 32767 : -32768) : 0);
    tx::idct<N>(v, 16);
  }
}

template <int N>
static void run_adst(std::mt19937 &g, int trials) {
  constexpr int n = 1 << N;
  std::uniform_int_distribution<int> full(-32768, 32767), bit(0, 1), mode(0, 1);
  for (int t = 0; t < trials; t++) {
    int32_t v[n];
    int m = mode(g);
    for (int i = 0; i < n; i++) v[i] = m == 0 ? (bit(g) ? 32767 : -32768) : full(g);
    if (N == 3) tx::iadst8(v, 16);
    else tx::iadst16(v, 16);
  }
}

int main() {
  std::mt19937 g(20251203);
  run_dct<2>(g, 200000);
  run_dct<3>(g, 200000);
  run_dct<4>(g, 200000);
  run_dct<5>(g, 100000);
  run_dct<6>(g, 50000);
  run_adst<3>(g, 200000);
  run_adst<4>(g, 200000);
  printf("largest butterfly sum %lld (2^%.2f), sums outside 32 bits: %lld\n", g_max,
         g_max ? __builtin_log2((double)g_max) : 0.0, g_over);
  return g_over ? 1 : 0;
}
