// Host check of the split 32- and 64-point inverse DCT (tx::idct_odd and
// tx::idct_join_pair, run by two threads per row on the device): on seeded
// random inputs - full 16-bit range, small values, and sparse rows with the
// upper half zero as in 64-point rows - the even half (idct<N - 1> without
// its permutation), the odd half and the join give exactly idct<N>'s output.
// Built and run by tests/test_host.py.
#include <cstdio>
#include <random>

#include "tx.cuh"

template <int N>
static int mismatches(std::mt19937 &g, int trials) {
  constexpr int n0 = 1 << N, h = n0 / 2;
  std::uniform_int_distribution<int> full(-(1 << 15), (1 << 15) - 1), small(-300, 300), pick(0, 2);
  int bad = 0;
  for (int t = 0; t < trials; t++) {
    int32_t in[n0], ref[n0], a[h], b[h], out[n0];
    int mode = pick(g);
    for (int i = 0; i < n0; i++)
      in[i] = mode == 0 ? full(g) : mode == 1 ? small(g) : (i < h && (g() & 1) ? small(g) : 0);
    for (int i = 0; i < n0; i++) ref[i] = in[i];
    tx::idct<N>(ref, 16);
    for (int k = 0; k < h; k++) {
      a[k] = in[tx::brev(N, k)];
      b[k] = in[tx::brev(N, k + h)];
    }
    tx::idct<N - 1, false>(a, 16);
    tx::idct_odd<N>(b, 16);
    for (int k = 0; k < h; k++) {
      out[k] = a[k];
      out[k + h] = b[k];
    }
    for (int i = 0; i < h; i++) tx::idct_join_pair(&out[i], &out[n0 - 1 - i], 16);
    for (int i = 0; i < n0; i++)
      if (out[i] != ref[i]) {
        bad++;
        break;
      }
  }
  return bad;
}

int main() {
  std::mt19937 g(20261203);
  int b5 = mismatches<5>(g, 50000), b6 = mismatches<6>(g, 50000);
  printf("idct32 split mismatches %d, idct64 split mismatches %d\n", b5, b6);
  return b5 || b6;
}
