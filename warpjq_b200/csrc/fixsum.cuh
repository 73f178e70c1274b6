// Exact, order-independent sums of FP64 values.
//
// The reference sums fractional aggregate values in plain f64, in whatever
// order its CPU slices or GPU atomics happen to run
// (crates/warpjq-core/src/agg.rs:62-71, cuda/warpjq_kernels.cu:1564), so its
// last bits depend on the schedule.  Here every finite value is added exactly
// into a fixed-point accumulator, and only the final total is rounded (once,
// to nearest-even), so a sum does not depend on tiles, CTAs, batches or the
// order of atomics: the same input gives the same bits every run.
//
// Layout: kFixDigits signed 64-bit limbs; limb i holds a signed count of
// 2^(32 i - kFixLowBits).  A value's 53-bit significand spans at most three
// limbs, and each add puts less than 2^32 into a limb, so limbs never carry
// while summing (2^31 adds per limb before an overflow is possible) and can
// be added with independent atomics.  The window is [2^-128, 2^128):
//   - bits of a value below 2^-128 are rounded off (to nearest-even, per
//     value, so still deterministic);
//   - values of magnitude 2^128 or more (and infinities) are summed in a
//     separate FP64 total ("big"), which is order-dependent; JSON numbers
//     that large are not expected in logs.
#pragma once

#include <stdint.h>

namespace wjq {

constexpr int kFixDigits = 8;
constexpr int kFixLowBits = 128;  // limb 0 counts units of 2^-128

// One value's contribution: limbs d, d+1, d+2 receive part[0..2] (signed).
struct FixParts {
  int d;  // first limb; -1: nothing to add (zero); -2: too big for the limbs
  long long part[3];
};

__host__ __device__ inline FixParts fix_split(double v) {
  FixParts r;
  unsigned long long b;
  __builtin_memcpy(&b, &v, 8);
  const int ex = (int)((b >> 52) & 0x7FF);
  unsigned long long m = b & ((1ull << 52) - 1);
  if (ex == 0x7FF) {
    r.d = -2;
    return r;
  }
  int e;
  if (ex == 0) {
    if (!m) {
      r.d = -1;
      return r;
    }
    e = -1074;
  } else {
    m |= 1ull << 52;
    e = ex - 1075;
  }
  // value = m * 2^e; bit position of m's lowest bit in the accumulator
  int pos = e + kFixLowBits;
  if (pos + 52 >= 32 * kFixDigits) {
    r.d = -2;
    return r;
  }
  if (pos < 0) {  // round off the bits below 2^-128 (nearest, ties to even)
    const int s = -pos;
    if (s > 54) {
      m = 0;
    } else {
      const unsigned long long rem = m & ((1ull << s) - 1), half = 1ull << (s - 1);
      m >>= s;
      if (rem > half || (rem == half && (m & 1))) m++;
    }
    pos = 0;
    if (!m) {
      r.d = -1;
      return r;
    }
  }
  const int d = pos >> 5, sh = pos & 31;
  const unsigned long long lo = m << sh;                     // bits [0, 64) of m << sh
  const unsigned long long hi = sh ? (m >> (64 - sh)) : 0;  // bits [64, 85)
  long long p0 = (long long)(lo & 0xFFFFFFFFull), p1 = (long long)(lo >> 32), p2 = (long long)hi;
  if (b >> 63) {
    p0 = -p0;
    p1 = -p1;
    p2 = -p2;
  }
  r.d = d;
  r.part[0] = p0;
  r.part[1] = p1;
  r.part[2] = d + 2 < kFixDigits ? p2 : 0;  // hi is zero when d + 2 is past the window
  return r;
}

// The correctly rounded FP64 value of  sum_i limb[i] * 2^(32 i - 128)
// + isum (a 128-bit two's complement integer given as lo/hi words).
__host__ __device__ inline double fix_to_double(const long long *limb, unsigned long long isum_lo,
                                                unsigned long long isum_hi) {
  // Normalise into 12 32-bit digits of a two's complement integer (units of
  // 2^-128): the limbs, then the integer sum placed at 2^0 (digit 4).
  uint32_t dg[12];
  __int128 carry = 0;
  for (int i = 0; i < 12; i++) {
    const __int128 t = carry + (i < kFixDigits ? (__int128)limb[i] : (__int128)0);
    dg[i] = (uint32_t)(unsigned long long)t;
    carry = t >> 32;  // arithmetic shift: the signed rest
  }
  {
    const uint32_t is[4] = {(uint32_t)isum_lo, (uint32_t)(isum_lo >> 32), (uint32_t)isum_hi,
                            (uint32_t)(isum_hi >> 32)};
    const uint32_t ext = (isum_hi >> 63) ? 0xFFFFFFFFu : 0u;
    unsigned long long c = 0;
    for (int i = 4; i < 12; i++) {
      const uint32_t a = (i - 4) < 4 ? is[i - 4] : ext;
      const unsigned long long s = (unsigned long long)dg[i] + a + c;
      dg[i] = (uint32_t)s;
      c = s >> 32;
    }
  }
  const bool neg = (dg[11] >> 31) != 0;
  if (neg) {  // magnitude
    unsigned long long c = 1;
    for (int i = 0; i < 12; i++) {
      const unsigned long long s = (unsigned long long)(uint32_t)~dg[i] + c;
      dg[i] = (uint32_t)s;
      c = s >> 32;
    }
  }
  int top = -1;  // highest set bit of the magnitude
  for (int i = 11; i >= 0 && top < 0; i--)
    if (dg[i]) {
      int b = 31;
      while (!((dg[i] >> b) & 1u)) b--;
      top = 32 * i + b;
    }
  if (top < 0) return 0.0;
  auto bit = [&](int k) -> unsigned { return k < 0 ? 0u : (dg[k >> 5] >> (k & 31)) & 1u; };
  // 53 significant bits from `top` down, then round to nearest-even with the
  // rest as guard and sticky bits
  unsigned long long mant = 0;
  for (int k = top; k > top - 53; k--) mant = (mant << 1) | bit(k);
  const int g = top - 53;
  bool sticky = false;
  for (int k = g - 1; k >= 0 && !sticky; k--) sticky = bit(k) != 0;
  if (bit(g) && (sticky || (mant & 1))) mant++;
  int e2 = top - 52 - kFixLowBits;  // value = mant * 2^e2
  if (mant >> 53) {
    mant >>= 1;
    e2++;
  }
  // mant * 2^e2 as a double; every total here is in the normal range
  // (|total| < 2^260 and >= 2^-128), so the scaling is exact
  double x = (double)mant;
  while (e2 > 0) {
    const int s = e2 > 60 ? 60 : e2;
    x *= (double)(1ull << s);
    e2 -= s;
  }
  while (e2 < 0) {
    const int s = -e2 > 60 ? 60 : -e2;
    x /= (double)(1ull << s);
    e2 += s;
  }
  return neg ? -x : x;
}

}  // namespace wjq
