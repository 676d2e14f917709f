// Inverse transforms (AV1 specification section 7.13.2), the forward
// transform's quantiser and dequantiser.
//
// The inverse kernels follow the specification's butterfly lists step by
// step (the encoder must reproduce the decoder's reconstruction bit for bit,
// as the reference does in src/kernels/k_itx.h:11-296). Each length is a
// template so every index is a compile-time constant: the 64-entry working
// array stays in registers on the device, and the same code runs on the host
// where the forward matrices are derived from these kernels.
#pragma once

#include "common.cuh"

namespace tx {

HD constexpr int brev(int numBits, int x) {
  int t = 0;
  for (int i = 0; i < numBits; i++) t |= ((x >> i) & 1) << (numBits - 1 - i);
  return t;
}

HD int cos128(int angle) {
  int a = angle & 255;
  if (a <= 64) return T(Cos128_Lookup)[a];
  if (a <= 128) return -T(Cos128_Lookup)[128 - a];
  if (a <= 192) return -T(Cos128_Lookup)[a - 128];
  return T(Cos128_Lookup)[256 - a];
}
HD int sin128(int angle) { return cos128(angle - 64); }

// Butterfly rotation B( a, b, angle, flip ) (spec 7.13.2.1). T_ is an
// int32_t pointer or an Offset view. The products and their sums are formed
// in 32 bits: every input is a 16-bit value (a dequantised level or a row
// output, both clamped to 16 bits, or an H output clamped to r = 16 bits) or
// a butterfly output of such values, and the cosines have 12 bits, so the
// sums stay below 2^30 (tests/native/butterfly_range_check.cpp drives every
// transform with extreme inputs and checks each sum in 64 bits through
// MAV1_BUTTERFLY_CHECK).
template <class T_>
HD void B(T_ t, int a, int b, int angle, int flip) {
  int c = cos128(angle), s = sin128(angle);
  int ta = t[a], tb = t[b];
#ifdef MAV1_BUTTERFLY_CHECK
  MAV1_BUTTERFLY_CHECK(ta, tb, c, s);
#endif
  int x = ta * c - tb * s, y = ta * s + tb * c;
  int xa = (x + 2048) >> 12, yb = (y + 2048) >> 12;
  t[a] = flip ? yb : xa;
  t[b] = flip ? xa : yb;
}

// Hadamard rotation H( a, b, flip, r ) with the r-bit clamp (spec 7.13.2.1).
template <class T_>
HD void H(T_ t, int a, int b, int flip, int r) {
  int ia = flip ? b : a, ib = flip ? a : b;
  int32_t x = t[ia], y = t[ib];
  int lo = -(1 << (r - 1)), hi = (1 << (r - 1)) - 1;
  t[ia] = clip3(lo, hi, x + y);
  t[ib] = clip3(lo, hi, x - y);
}

// Elements O, O+1, ... of a length-2O vector held from p: t[i] is p[i - O].
template <int O>
struct Offset {
  int32_t *p;
  HDM int32_t &operator[](int i) const { return p[i - O]; }
};

// Inverse DCT of length 1 << N (spec 7.13.2.3).
template <int N, bool PERM = true>
HD void idct(int32_t *t, int r) {
  constexpr int n0 = 1 << N;
  if (PERM) {
    int32_t c[n0];
#pragma unroll
    for (int i = 0; i < n0; i++) c[i] = t[i];
#pragma unroll
    for (int i = 0; i < n0; i++) t[i] = c[brev(N, i)];
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 16; i++) B(t, 32 + i, 63 - i, 63 - 4 * brev(4, i), 0);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 8; i++) B(t, 16 + i, 31 - i, 6 + (brev(3, 7 - i) << 3), 0);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 16; i++) H(t, 32 + i * 2, 33 + i * 2, i & 1, r);
  }
  if (N >= 4) {
#pragma unroll
    for (int i = 0; i < 4; i++) B(t, 8 + i, 15 - i, 12 + (brev(2, 3 - i) << 4), 0);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 8; i++) H(t, 16 + 2 * i, 17 + 2 * i, i & 1, r);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) B(t, 62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * brev(2, i) + 64 * j, 1);
  }
  if (N >= 3) {
#pragma unroll
    for (int i = 0; i < 2; i++) B(t, 4 + i, 7 - i, 56 - 32 * i, 0);
  }
  if (N >= 4) {
#pragma unroll
    for (int i = 0; i < 4; i++) H(t, 8 + 2 * i, 9 + 2 * i, i & 1, r);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) B(t, 30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), 1);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) H(t, 32 + i * 4 + j, 35 + i * 4 - j, i & 1, r);
  }
#pragma unroll
  for (int i = 0; i < 2; i++) B(t, 2 * i, 2 * i + 1, 32 + 16 * i, 1 - i);
  if (N >= 3) {
#pragma unroll
    for (int i = 0; i < 2; i++) H(t, 4 + 2 * i, 5 + 2 * i, i, r);
  }
  if (N >= 4) {
#pragma unroll
    for (int i = 0; i < 2; i++) B(t, 14 - i, 9 + i, 48 + 64 * i, 1);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) H(t, 16 + 4 * i + j, 19 + 4 * i - j, i & 1, r);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) B(t, 61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, 1);
  }
#pragma unroll
  for (int i = 0; i < 2; i++) H(t, i, 3 - i, 0, r);
  if (N >= 3) B(t, 6, 5, 32, 1);
  if (N >= 4) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) H(t, 8 + 4 * i + j, 11 + 4 * i - j, i, r);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 4; i++) B(t, 29 - i, 18 + i, 48 + (i >> 1) * 64, 1);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) H(t, 32 + 8 * i + j, 39 + 8 * i - j, i & 1, r);
  }
  if (N >= 3) {
#pragma unroll
    for (int i = 0; i < 4; i++) H(t, i, 7 - i, 0, r);
  }
  if (N >= 4) {
#pragma unroll
    for (int i = 0; i < 2; i++) B(t, 13 - i, 10 + i, 32, 1);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) H(t, 16 + i * 8 + j, 23 + i * 8 - j, i, r);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 8; i++) B(t, 59 - i, 36 + i, i < 4 ? 48 : 112, 1);
  }
  if (N >= 4) {
#pragma unroll
    for (int i = 0; i < 8; i++) H(t, i, 15 - i, 0, r);
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 4; i++) B(t, 27 - i, 20 + i, 32, 1);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      H(t, 32 + i, 47 - i, 0, r);
      H(t, 48 + i, 63 - i, 1, r);
    }
  }
  if (N >= 5) {
#pragma unroll
    for (int i = 0; i < 16; i++) H(t, i, 31 - i, 0, r);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 8; i++) B(t, 55 - i, 40 + i, 32, 1);
  }
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 32; i++) H(t, i, 63 - i, 0, r);
  }
}

// ADST input / output permutations (spec 7.13.2.4, 7.13.2.5).
// The 2^N-point inverse DCT (N = 5, 6) as two halves and a join, for two
// threads. After the input permutation, the operations of idct<N> on
// elements 0 .. n0/2 - 1 are exactly idct<N - 1> without its permutation,
// and those on n0/2 .. n0 - 1 are the groups that only N adds (idct_odd,
// the same operations in the same order, on element indices n0/2 .. n0 - 1;
// `odd` holds those elements, odd[0] being element n0/2); the halves touch
// disjoint elements until the last stage, H(i, n0 - 1 - i) for i < n0/2
// (idct_join_pair). Running the halves concurrently and then the join gives
// idct<N>'s result exactly.
template <int N>
HD void idct_odd(int32_t *odd, int r) {
  Offset<(1 << N) / 2> t{odd};
  if (N == 6) {
#pragma unroll
    for (int i = 0; i < 16; i++) B(t, 32 + i, 63 - i, 63 - 4 * brev(4, i), 0);
#pragma unroll
    for (int i = 0; i < 16; i++) H(t, 32 + i * 2, 33 + i * 2, i & 1, r);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) B(t, 62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * brev(2, i) + 64 * j, 1);
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) H(t, 32 + i * 4 + j, 35 + i * 4 - j, i & 1, r);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) B(t, 61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, 1);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) H(t, 32 + 8 * i + j, 39 + 8 * i - j, i & 1, r);
#pragma unroll
    for (int i = 0; i < 8; i++) B(t, 59 - i, 36 + i, i < 4 ? 48 : 112, 1);
#pragma unroll
    for (int i = 0; i < 8; i++) {
      H(t, 32 + i, 47 - i, 0, r);
      H(t, 48 + i, 63 - i, 1, r);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) B(t, 55 - i, 40 + i, 32, 1);
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++) B(t, 16 + i, 31 - i, 6 + (brev(3, 7 - i) << 3), 0);
#pragma unroll
    for (int i = 0; i < 8; i++) H(t, 16 + 2 * i, 17 + 2 * i, i & 1, r);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) B(t, 30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), 1);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) H(t, 16 + 4 * i + j, 19 + 4 * i - j, i & 1, r);
#pragma unroll
    for (int i = 0; i < 4; i++) B(t, 29 - i, 18 + i, 48 + (i >> 1) * 64, 1);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) H(t, 16 + i * 8 + j, 23 + i * 8 - j, i, r);
#pragma unroll
    for (int i = 0; i < 4; i++) B(t, 27 - i, 20 + i, 32, 1);
  }
}

// One pair of the join stage: H(i, n0 - 1 - i) with the clamp to r bits.
HD void idct_join_pair(int32_t *a, int32_t *b, int r) {
  int32_t x = *a, y = *b;
  int lo = -(1 << (r - 1)), hi = (1 << (r - 1)) - 1;
  *a = clip3(lo, hi, x + y);
  *b = clip3(lo, hi, x - y);
}

template <int N>
HD void adst_in_perm(int32_t *t) {
  constexpr int n0 = 1 << N;
  int32_t c[n0];
#pragma unroll
  for (int i = 0; i < n0; i++) c[i] = t[i];
#pragma unroll
  for (int i = 0; i < n0; i++) t[i] = c[(i & 1) ? (i - 1) : (n0 - i - 1)];
}

template <int N>
HD void adst_out_perm(int32_t *t) {
  constexpr int n0 = 1 << N;
  int32_t c[n0];
#pragma unroll
  for (int i = 0; i < n0; i++) c[i] = t[i];
#pragma unroll
  for (int i = 0; i < n0; i++) {
    int a = (i >> 3) & 1, b = ((i >> 2) & 1) ^ ((i >> 3) & 1), cc = ((i >> 1) & 1) ^ ((i >> 2) & 1),
        d = (i & 1) ^ ((i >> 1) & 1);
    int idx = ((d << 3) | (cc << 2) | (b << 1) | a) >> (4 - N);
    t[i] = (i & 1) ? -c[idx] : c[idx];
  }
}

// Inverse ADST4 (spec 7.13.2.6), 64-bit intermediate products.
HD void iadst4(int32_t *t) {
  const int64_t S1 = 1321, S2 = 2482, S3 = 3344, S4 = 3803;
  int64_t s0 = S1 * t[0], s1 = S2 * t[0], s2 = S3 * t[1], s3 = S4 * t[2];
  int64_t s4 = S1 * t[2], s5 = S2 * t[3], s6 = S4 * t[3];
  int64_t a7 = (int64_t)t[0] - t[2];
  int64_t b7 = a7 + t[3];
  s0 = s0 + s3;
  s1 = s1 - s4;
  s3 = s2;
  s2 = S3 * b7;
  s0 = s0 + s5;
  s1 = s1 - s6;
  int64_t x0 = s0 + s3, x1 = s1 + s3, x2 = s2, x3 = s0 + s1;
  x3 = x3 - s3;
  t[0] = (int32_t)round2l(x0, 12);
  t[1] = (int32_t)round2l(x1, 12);
  t[2] = (int32_t)round2l(x2, 12);
  t[3] = (int32_t)round2l(x3, 12);
}

// Inverse ADST8 (spec 7.13.2.7).
HD void iadst8(int32_t *t, int r) {
  adst_in_perm<3>(t);
#pragma unroll
  for (int i = 0; i < 4; i++) B(t, 2 * i, 2 * i + 1, 60 - 16 * i, 1);
#pragma unroll
  for (int i = 0; i < 4; i++) H(t, i, 4 + i, 0, r);
#pragma unroll
  for (int i = 0; i < 2; i++) B(t, 4 + 3 * i, 5 + i, 48 - 32 * i, 1);
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) H(t, 4 * j + i, 2 + 4 * j + i, 0, r);
#pragma unroll
  for (int i = 0; i < 2; i++) B(t, 2 + 4 * i, 3 + 4 * i, 32, 1);
  adst_out_perm<3>(t);
}

// Inverse ADST16 (spec 7.13.2.8).
HD void iadst16(int32_t *t, int r) {
  adst_in_perm<4>(t);
#pragma unroll
  for (int i = 0; i < 8; i++) B(t, 2 * i, 2 * i + 1, 62 - 8 * i, 1);
#pragma unroll
  for (int i = 0; i < 8; i++) H(t, i, 8 + i, 0, r);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    B(t, 8 + 2 * i, 9 + 2 * i, 56 - 32 * i, 1);
    B(t, 13 + 2 * i, 12 + 2 * i, 8 + 32 * i, 1);
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) H(t, 8 * j + i, 4 + 8 * j + i, 0, r);
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) B(t, 4 + 8 * j + 3 * i, 5 + 8 * j + i, 48 - 32 * i, 1);
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) H(t, 4 * j + i, 2 + 4 * j + i, 0, r);
#pragma unroll
  for (int i = 0; i < 4; i++) B(t, 2 + 4 * i, 3 + 4 * i, 32, 1);
  adst_out_perm<4>(t);
}

// Inverse identity transform (spec 7.13.2.15).
template <int N>
HD void iidentity(int32_t *t) {
#pragma unroll
  for (int i = 0; i < (1 << N); i++) {
    if (N == 2) t[i] = (int32_t)round2l((int64_t)t[i] * 5793, 12);
    else if (N == 3) t[i] = t[i] * 2;
    else if (N == 4) t[i] = (int32_t)round2l((int64_t)t[i] * 11586, 12);
    else t[i] = t[i] * 4;
  }
}

// Inverse Walsh-Hadamard (spec 7.13.2.10) for lossless blocks.
HD void iwht(int32_t *t, int shift) {
  int32_t a = t[0] >> shift, c = t[1] >> shift, d = t[2] >> shift, b = t[3] >> shift;
  a += c;
  d -= b;
  int32_t e = (a - d) >> 1;
  b = e - b;
  c = e - c;
  a -= b;
  d += c;
  t[0] = a;
  t[1] = b;
  t[2] = c;
  t[3] = d;
}

// 1-D kernel classes of the 2-D transform.
enum { KIND_DCT = 0, KIND_ADST = 1, KIND_IDTX = 2 };

HD int row_kind(int txType) {
  if (txType == DCT_DCT || txType == ADST_DCT || txType == FLIPADST_DCT || txType == H_DCT) return KIND_DCT;
  if (txType == DCT_ADST || txType == ADST_ADST || txType == DCT_FLIPADST || txType == FLIPADST_FLIPADST ||
      txType == ADST_FLIPADST || txType == FLIPADST_ADST || txType == H_ADST || txType == H_FLIPADST)
    return KIND_ADST;
  return KIND_IDTX;
}
HD int col_kind(int txType) {
  if (txType == DCT_DCT || txType == DCT_ADST || txType == DCT_FLIPADST || txType == V_DCT) return KIND_DCT;
  if (txType == ADST_DCT || txType == ADST_ADST || txType == FLIPADST_DCT || txType == FLIPADST_FLIPADST ||
      txType == ADST_FLIPADST || txType == FLIPADST_ADST || txType == V_ADST || txType == V_FLIPADST)
    return KIND_ADST;
  return KIND_IDTX;
}
HD int flip_ud(int t) { return t == FLIPADST_DCT || t == FLIPADST_ADST || t == V_FLIPADST || t == FLIPADST_FLIPADST; }
HD int flip_lr(int t) { return t == DCT_FLIPADST || t == ADST_FLIPADST || t == H_FLIPADST || t == FLIPADST_FLIPADST; }

// One 1-D inverse transform of kind / length 1 << log2n on t[0 .. n-1].
// The same for a length fixed at compile time: every index of the working
// array is a constant, so it stays in registers.
template <int N>
HD void inverse_1d_n(int32_t *t, int kind, int r) {
  if (kind == KIND_DCT) {
    idct<N>(t, r);
  } else if (kind == KIND_ADST) {
    if constexpr (N == 2) iadst4(t);
    else if constexpr (N == 3) iadst8(t, r);
    else if constexpr (N == 4) iadst16(t, r);
  } else {
    if constexpr (N <= 5) iidentity<N>(t);
  }
}

HD void inverse_1d(int32_t *t, int kind, int log2n, int r) {
  if (kind == KIND_DCT) {
    switch (log2n) {
      case 2: idct<2>(t, r); break;
      case 3: idct<3>(t, r); break;
      case 4: idct<4>(t, r); break;
      case 5: idct<5>(t, r); break;
      default: idct<6>(t, r); break;
    }
  } else if (kind == KIND_ADST) {
    if (log2n == 2) iadst4(t);
    else if (log2n == 3) iadst8(t, r);
    else iadst16(t, r);
  } else {
    switch (log2n) {
      case 2: iidentity<2>(t); break;
      case 3: iidentity<3>(t); break;
      case 4: iidentity<4>(t); break;
      default: iidentity<5>(t); break;
    }
  }
}

// ---- quantisation ----------------------------------------------------------

// Dequantisation shift class of a transform size (spec 7.12.3 dqDenom).
HD int dq_denom(int txSz) {
  if (txSz == TX_32X32 || txSz == TX_16X32 || txSz == TX_32X16 || txSz == TX_16X64 || txSz == TX_64X16) return 2;
  if (txSz == TX_64X64 || txSz == TX_32X64 || txSz == TX_64X32) return 4;
  return 1;
}

// Dead-zone quantiser of one Q4 coefficient: level = (|v| * denom + q * rnd / 4)
// / 16 / q, capped at 0xFFFF, with the sign of v. The reference
// (src/kernels/k_fwd.h:66-90) divides by q through a 2^44 reciprocal that is
// exact for every quotient below 2^19 and falls back to a division above;
// both give the truncating quotient, which is what this computes.
HD int quant_level(int v, int q, int rnd, int denom, uint64_t inv) {
  int64_t a = (int64_t)iabs(v) * denom;
  int64_t t = (a + (((int64_t)q * rnd) >> 2)) >> 4;
  int level = t < ((int64_t)1 << 19) ? (int)(((uint64_t)t * inv) >> 44) : (int)(t / q);
  if (level > 0xFFFF) level = 0xFFFF;
  return v < 0 ? -level : level;
}
HD uint64_t quant_inv(int q) { return ((uint64_t)1 << 44) / (uint64_t)q + 1; }

// Dequantisation of one level (spec 7.12.3 step 1, no quantizer matrix).
HD int dequant_level(int level, int q, int denom) {
  int64_t d = (int64_t)level * q;
  int64_t ad = d < 0 ? -d : d;
  int64_t d2 = (ad & 0xFFFFFF) >> (denom >> 1);
  if (d < 0) d2 = -d2;
  return clip3(-(1 << 15), (1 << 15) - 1, (int)d2);
}

}  // namespace tx
