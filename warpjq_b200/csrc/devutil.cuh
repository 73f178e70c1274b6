// Device helpers for the scan kernels: byte classification, JSON string
// decoding, number parsing and the order-preserving float encoding.
#pragma once

#include <stdint.h>

#include "plan.h"

namespace wjq {

// ---------------------------------------------------------------------------
// Byte classes
// ---------------------------------------------------------------------------

// JSON insignificant whitespace inside a line (json.rs:123-128; '\n' never
// occurs inside a line).
__device__ __forceinline__ bool is_ws(uint32_t c) {
  return c == ' ' || c == '\t' || c == '\r' || c == '\n';
}

// Bytes that end an atom (number or literal): whitespace and the structural
// characters, plus the quote.
__device__ __forceinline__ bool ends_atom(uint32_t c) {
  return is_ws(c) || c == ',' || c == '}' || c == ']' || c == ':' || c == '"' || c == '{' ||
         c == '[';
}

__device__ __forceinline__ bool is_digit(uint32_t c) { return c - '0' < 10u; }

__device__ __forceinline__ int hex_val(uint32_t c) {
  if (c - '0' < 10u) return (int)(c - '0');
  uint32_t l = c | 0x20;
  if (l - 'a' < 6u) return (int)(l - 'a' + 10);
  return -1;
}

// SWAR: nonzero iff some byte of `x` is '"', '\\' or below 0x20.
// (x - 0x01..) & ~x & 0x80.. is the exact "has a zero byte" test.
__device__ __forceinline__ uint32_t swar_string_special(uint32_t x) {
  uint32_t q = x ^ 0x22222222u;
  uint32_t b = x ^ 0x5C5C5C5Cu;
  uint32_t zq = (q - 0x01010101u) & ~q;
  uint32_t zb = (b - 0x01010101u) & ~b;
  uint32_t lo = (x - 0x20202020u) & ~x;  // bytes < 0x20 (exact as a boolean)
  return (zq | zb | lo) & 0x80808080u;
}

// SWAR: nonzero iff some byte of `x` is '\n'.
__device__ __forceinline__ uint32_t swar_newline(uint32_t x) {
  uint32_t t = x ^ 0x0A0A0A0Au;
  return (t - 0x01010101u) & ~t & 0x80808080u;
}

// Exact per-byte newline flags: 0x80 in each byte lane holding '\n'.
__device__ __forceinline__ uint32_t swar_newline_exact(uint32_t x) {
  uint32_t t = x ^ 0x0A0A0A0Au;
  return ~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u;
}

// Gathers the four 0x80 flags of `m` into bits 0..3.
__device__ __forceinline__ uint32_t swar_movemask(uint32_t m) {
  return ((m >> 7) * 0x00204081u) >> 21 & 0xFu;
}

// ---------------------------------------------------------------------------
// Structural classification of 32-byte chunks (the scan's first stage)
// ---------------------------------------------------------------------------

// Exact per-byte flags (0x80 in each byte lane) of the bytes of x that are
// '"', '\\' or below 0x20.  Each test adds to the low seven bits, which never
// carries across a byte lane; bytes >= 0x80 are never flagged.
__host__ __device__ __forceinline__ uint32_t flags_special(uint32_t x) {
  const uint32_t t = x & 0x7F7F7F7Fu;
  const uint32_t sq = (t ^ 0x22222222u) + 0x7F7F7F7Fu;  // bit 7 clear iff '"'
  const uint32_t sb = (t ^ 0x5C5C5C5Cu) + 0x7F7F7F7Fu;  // bit 7 clear iff '\\'
  const uint32_t sc = t + 0x60606060u;                  // bit 7 clear iff < 0x20
  return ~((sq & sb & sc) | x) & 0x80808080u;
}

// Exact per-byte flags of the '\n' bytes of x.
__host__ __device__ __forceinline__ uint32_t flags_newline(uint32_t x) {
  const uint32_t sn = ((x ^ 0x0A0A0A0Au) & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
  return ~(sn | x) & 0x80808080u;
}

// Shifts the nibbles gathered so far up by four and moves the four flags of
// `f` (bit 7 of each byte) in below them, byte j's flag on bit j.  The
// multiply by 1 + 2^7 + 2^14 + 2^21 lands byte j's flag on bit 28 + j (no
// two partial products share a bit, so nothing carries); one funnel shift
// brings those four bits in.  Pushing a chunk's words from the last to the
// first leaves word k's flags on bits 4k..4k+3.
__host__ __device__ __forceinline__ uint32_t flags_push(uint32_t acc, uint32_t f) {
#ifdef __CUDA_ARCH__
  return __funnelshift_l(f * 0x00204081u, acc, 4);
#else
  return (acc << 4) | ((f * 0x00204081u) >> 28);
#endif
}

// Classifies one 32-byte chunk given as eight little-endian words: returns
// the newline mask (bit j: byte j is '\n') and stores the special mask (bit
// j: byte j is '"', '\\' or below 0x20) in *special.  The special mask is
// what string scanning needs: a string ends at its first unescaped '"', a
// '\\' starts an escape, and any byte below 0x20 (the line's own newline
// too) ends a malformed string.
__host__ __device__ __forceinline__ uint32_t classify_chunk(const uint32_t w[8], uint32_t *special) {
  uint32_t s = 0, nl = 0;
#pragma unroll
  for (int k = 7; k >= 0; k--) {
    s = flags_push(s, flags_special(w[k]));
    nl = flags_push(nl, flags_newline(w[k]));
  }
  *special = s;
  return nl;
}

// ---------------------------------------------------------------------------
// Order-preserving float encoding (agg.rs:205-212)
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long order_bits(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b ^ (1ull << 63));
}

__host__ __device__ inline double from_order_bits(unsigned long long o) {
  unsigned long long b = (o >> 63) ? (o ^ (1ull << 63)) : ~o;
  double d;
  __builtin_memcpy(&d, &b, 8);
  return d;
}

// The minimum / maximum recorded in order keys, or +inf / -inf when none
// was: the keys start at ~0 and 0, which no number encodes, and stay there
// when no value arrived or the aggregate does not track them (only min and
// max queries do).
__host__ __device__ inline double min_of_bits(unsigned long long o) {
  return o == ~0ull ? __builtin_huge_val() : from_order_bits(o);
}
__host__ __device__ inline double max_of_bits(unsigned long long o) {
  return o == 0ull ? -__builtin_huge_val() : from_order_bits(o);
}

// ---------------------------------------------------------------------------
// JSON string decoding (json.rs:594-654): yields the decoded bytes of a
// validated string body one at a time.  \u escapes become UTF-8; a lone
// surrogate becomes U+FFFD; a high+low pair becomes one code point.
// ---------------------------------------------------------------------------

struct StrDecoder {
  const uint8_t *p;
  uint32_t i, n;
  uint8_t pend[4];
  uint8_t npend, ipend;

  __device__ StrDecoder(const uint8_t *body, uint32_t len) : p(body), i(0), n(len), npend(0), ipend(0) {}

  __device__ uint32_t hex4(uint32_t at) const {
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) v = v * 16 + (uint32_t)hex_val(p[at + k]);
    return v;
  }

  // Returns the next decoded byte, or -1 at the end.
  __device__ int next() {
    if (ipend < npend) return pend[ipend++];
    if (i >= n) return -1;
    uint32_t c = p[i];
    if (c != '\\') {
      i++;
      return (int)c;
    }
    uint32_t e = p[i + 1];
    i += 2;
    switch (e) {
      case 'b': return 0x08;
      case 'f': return 0x0c;
      case 'n': return '\n';
      case 'r': return '\r';
      case 't': return '\t';
      case 'u': break;
      default: return (int)e;  // '"', '\\', '/'
    }
    uint32_t cp = hex4(i);
    i += 4;
    if (cp >= 0xD800 && cp < 0xDC00 && i + 6 <= n && p[i] == '\\' && p[i + 1] == 'u') {
      uint32_t lo = hex4(i + 2);
      if (lo >= 0xDC00 && lo < 0xE000) {
        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
        i += 6;
      }
    }
    if (cp >= 0xD800 && cp < 0xE000) cp = 0xFFFD;
    npend = 0;
    ipend = 1;
    if (cp < 0x80) return (int)cp;
    if (cp < 0x800) {
      pend[0] = (uint8_t)(0xC0 | (cp >> 6));
      pend[1] = (uint8_t)(0x80 | (cp & 0x3F));
      npend = 2;
    } else if (cp < 0x10000) {
      pend[0] = (uint8_t)(0xE0 | (cp >> 12));
      pend[1] = (uint8_t)(0x80 | ((cp >> 6) & 0x3F));
      pend[2] = (uint8_t)(0x80 | (cp & 0x3F));
      npend = 3;
    } else {
      pend[0] = (uint8_t)(0xF0 | (cp >> 18));
      pend[1] = (uint8_t)(0x80 | ((cp >> 12) & 0x3F));
      pend[2] = (uint8_t)(0x80 | ((cp >> 6) & 0x3F));
      pend[3] = (uint8_t)(0x80 | (cp & 0x3F));
      npend = 4;
    }
    return pend[0];
  }
};

// Lexicographic compare of a string body (possibly escaped) against literal
// bytes, by decoded value (json.rs:680-691).  Returns -1, 0, 1.
__device__ inline int cmp_str_body(const uint8_t *body, uint32_t n, bool has_escape,
                                   const uint8_t *lit, uint32_t lit_len) {
  if (!has_escape) {
    uint32_t m = n < lit_len ? n : lit_len;
    for (uint32_t k = 0; k < m; k++) {
      uint32_t a = body[k], b = lit[k];
      if (a != b) return a < b ? -1 : 1;
    }
    return n == lit_len ? 0 : (n < lit_len ? -1 : 1);
  }
  StrDecoder d(body, n);
  uint32_t k = 0;
  for (;;) {
    int a = d.next();
    if (a < 0) return k == lit_len ? 0 : -1;
    if (k == lit_len) return 1;
    uint32_t b = lit[k++];
    if ((uint32_t)a != b) return (uint32_t)a < b ? -1 : 1;
  }
}

// FNV-1a over the decoded bytes of a string body.
__device__ inline uint32_t hash_str_body(const uint8_t *body, uint32_t n, bool has_escape) {
  uint32_t h = 0x811c9dc5u;
  if (!has_escape) {
    for (uint32_t k = 0; k < n; k++) {
      h ^= body[k];
      h *= 0x01000193u;
    }
    return h;
  }
  StrDecoder d(body, n);
  for (int c; (c = d.next()) >= 0;) {
    h ^= (uint32_t)c;
    h *= 0x01000193u;
  }
  return h;
}

__device__ inline uint32_t hash_raw(const uint8_t *p, uint32_t n) {
  uint32_t h = 0x811c9dc5u;
  for (uint32_t k = 0; k < n; k++) {
    h ^= p[k];
    h *= 0x01000193u;
  }
  return h;
}

// ---------------------------------------------------------------------------
// Number parsing.
//
// A validated JSON number is converted to the correctly rounded double, as
// Rust's str::parse::<f64> does in the reference (json.rs:73-78).  Two
// published methods:
//   1. Clinger's fast path (W. D. Clinger, "How to Read Floating Point
//      Numbers Accurately", PLDI 1990): when the significand fits 53 bits and
//      |exp10| <= 22, one IEEE multiplication or division by an exact power of
//      ten is correctly rounded.
//   2. Otherwise the Simple Decimal Conversion algorithm (N. Tao, "The Simple
//      Decimal Conversion Algorithm", 2020): the decimal digits (up to 800,
//      with a sticky bit for the rest) are scaled by powers of two until the
//      binary exponent is known, then rounded half to even.
// ---------------------------------------------------------------------------

__device__ __forceinline__ double exact_pow10(int e) {
  // 10^0 .. 10^22 are exact doubles.
  double r = 1.0;
  double b = 10.0;
  while (e) {
    if (e & 1) r *= b;
    b *= b;
    e >>= 1;
  }
  return r;
}

struct BigDec {
  static constexpr int kCap = 800;
  uint8_t d[kCap + 24];  // digit values 0..9; headroom for left shifts
  int nd;                // digits in use
  int dp;                // decimal point position: value = 0.d[0..nd) * 10^dp
  bool trunc;            // nonzero digits were dropped past kCap

  __device__ void trim() {
    while (nd > 0 && d[nd - 1] == 0) nd--;
    if (nd == 0) dp = 0;
  }

  // Divides by 2^k, k <= 60.
  __device__ void right_shift(int k) {
    int r = 0, w = 0;
    unsigned long long n = 0;
    for (; (n >> k) == 0; r++) {
      if (r >= nd) {
        if (n == 0) {
          nd = 0;
          dp = 0;
          return;
        }
        while ((n >> k) == 0) {
          n *= 10;
          r++;
        }
        break;
      }
      n = n * 10 + d[r];
    }
    dp -= r - 1;
    unsigned long long mask = (1ull << k) - 1;
    for (; r < nd; r++) {
      unsigned long long c = d[r];
      d[w++] = (uint8_t)(n >> k);
      n = (n & mask) * 10 + c;
    }
    while (n > 0) {
      uint8_t dig = (uint8_t)(n >> k);
      n = (n & mask) * 10;
      if (w < kCap) d[w++] = dig;
      else if (dig > 0) trunc = true;
    }
    nd = w;
    trim();
  }

  // Multiplies by 2^k, k <= 60.  Works from the last digit, writing 20
  // places to the right, then slides the result back.
  __device__ void left_shift(int k) {
    int w = nd + 20;
    unsigned long long n = 0;
    for (int r = nd - 1; r >= 0; r--) {
      n += (unsigned long long)d[r] << k;
      unsigned long long q = n / 10;
      d[--w] = (uint8_t)(n - 10 * q);
      n = q;
    }
    while (n > 0) {
      unsigned long long q = n / 10;
      d[--w] = (uint8_t)(n - 10 * q);
      n = q;
    }
    int newnd = nd + 20 - w;
    dp += newnd - nd;
    for (int i = 0; i < newnd; i++) d[i] = d[w + i];
    if (newnd > kCap) {
      for (int i = kCap; i < newnd; i++)
        if (d[i]) trunc = true;
      newnd = kCap;
    }
    nd = newnd;
    trim();
  }

  __device__ void shift(int k) {
    const int kMax = 60;
    if (nd == 0) return;
    if (k > 0) {
      while (k > kMax) {
        left_shift(kMax);
        k -= kMax;
      }
      left_shift(k);
    } else if (k < 0) {
      while (k < -kMax) {
        right_shift(kMax);
        k += kMax;
      }
      right_shift(-k);
    }
  }

  __device__ bool should_round_up(int at) const {
    if (at < 0 || at >= nd) return false;
    if (d[at] == 5 && at + 1 == nd) {
      if (trunc) return true;
      return at > 0 && (d[at - 1] & 1);
    }
    return d[at] >= 5;
  }

  __device__ unsigned long long rounded_integer() const {
    if (dp > 20) return ~0ull;
    unsigned long long n = 0;
    int i = 0;
    for (; i < dp && i < nd; i++) n = n * 10 + d[i];
    for (; i < dp; i++) n *= 10;
    if (should_round_up(dp)) n++;
    return n;
  }
};

__device__ __noinline__ double slow_decimal_to_double(const uint8_t *p, uint32_t n) {
  BigDec a;
  a.nd = 0;
  a.dp = 0;
  a.trunc = false;
  bool neg = p[0] == '-';
  uint32_t i = neg ? 1 : 0;
  bool seen_dot = false;
  int dp = 0;
  for (; i < n; i++) {
    uint32_t c = p[i];
    if (c == '.') {
      seen_dot = true;
      continue;
    }
    if (!is_digit(c)) break;
    // value = 0.d[0..nd) * 10^dp: every integer digit moves the point right;
    // a zero before the first significant digit moves it back left.
    if (!seen_dot) dp++;
    if (c == '0' && a.nd == 0) {
      dp--;
      continue;
    }
    if (a.nd < BigDec::kCap) a.d[a.nd++] = (uint8_t)(c - '0');
    else if (c != '0') a.trunc = true;
  }
  long long e = 0;
  if (i < n && (p[i] == 'e' || p[i] == 'E')) {
    i++;
    bool eneg = false;
    if (p[i] == '+' || p[i] == '-') {
      eneg = p[i] == '-';
      i++;
    }
    for (; i < n && is_digit(p[i]); i++)
      if (e < 100000) e = e * 10 + (p[i] - '0');
    if (eneg) e = -e;
  }
  a.dp = dp + (int)e;
  a.trim();
  unsigned long long bits;
  const int kMantBits = 52, kBias = -1023;
  if (a.nd == 0) {
    bits = 0;
  } else if (a.dp > 310) {
    bits = 0x7FFull << 52;  // +inf
  } else if (a.dp < -330) {
    bits = 0;
  } else {
    static const int powtab[] = {1, 3, 6, 9, 13, 16, 19, 23, 26};
    int exp = 0;
    while (a.dp > 0) {
      int k = a.dp >= 9 ? 27 : powtab[a.dp];
      a.shift(-k);
      exp += k;
    }
    while (a.dp < 0 || (a.dp == 0 && a.d[0] < 5)) {
      int k = -a.dp >= 9 ? 27 : powtab[-a.dp];
      a.shift(k);
      exp -= k;
    }
    exp--;  // value in [1, 2) * 2^exp after this
    if (exp < kBias + 1) {
      int k = kBias + 1 - exp;
      a.shift(-k);
      exp += k;
    }
    if (exp - kBias >= 0x7FF) {
      bits = 0x7FFull << 52;
    } else {
      a.shift(1 + kMantBits);
      unsigned long long mant = a.rounded_integer();
      if (mant == (2ull << kMantBits)) {
        mant >>= 1;
        exp++;
      }
      if (exp - kBias >= 0x7FF) {
        bits = 0x7FFull << 52;
      } else {
        if ((mant & (1ull << kMantBits)) == 0) exp = kBias;  // subnormal
        bits = (mant & ((1ull << kMantBits) - 1)) | ((unsigned long long)((exp - kBias) & 0x7FF) << 52);
      }
    }
  }
  if (neg) bits |= 1ull << 63;
  return __longlong_as_double((long long)bits);
}

// Parses a validated JSON number.  `is_int` is set when the text is an
// integer literal (no fraction, no exponent) that fits in int64; `iv` then
// holds its exact value.
__device__ __forceinline__ double parse_number(const uint8_t *p, uint32_t n, bool &is_int,
                                               long long &iv) {
  if (n <= 9) {  // exact in 32 bits
    uint32_t v = 0;
    uint32_t k = 0;
    for (; k < n; k++) {
      uint32_t dgt = (uint32_t)p[k] - '0';
      if (dgt > 9) break;
      v = v * 10 + dgt;
    }
    if (k == n) {
      is_int = true;
      iv = (long long)v;
      return (double)v;
    }
  }
  bool neg = p[0] == '-';
  uint32_t i = neg ? 1 : 0;
  unsigned long long mant = 0;
  int nd = 0;              // significant digits held in mant
  int exp10 = 0;
  bool dropped = false;    // a digit did not fit in mant
  bool overflow = false;   // a nonzero digit did not fit in mant
  // integer part
  for (; i < n && is_digit(p[i]); i++) {
    uint32_t dgt = p[i] - '0';
    if (nd < 19) {
      mant = mant * 10 + dgt;
      if (mant) nd++;
    } else {
      dropped = true;
      if (dgt) overflow = true;
      exp10++;
    }
  }
  bool frac = false, has_exp = false;
  if (i < n && p[i] == '.') {
    frac = true;
    i++;
    for (; i < n && is_digit(p[i]); i++) {
      uint32_t dgt = p[i] - '0';
      if (nd < 19) {
        mant = mant * 10 + dgt;
        if (mant) nd++;
        exp10--;
      } else {
        dropped = true;
        if (dgt) overflow = true;
      }
    }
  }
  if (i < n && (p[i] == 'e' || p[i] == 'E')) {
    has_exp = true;
    i++;
    bool eneg = false;
    if (p[i] == '+' || p[i] == '-') {
      eneg = p[i] == '-';
      i++;
    }
    int e = 0;
    for (; i < n && is_digit(p[i]); i++)
      if (e < 100000) e = e * 10 + (int)(p[i] - '0');
    exp10 += eneg ? -e : e;
  }
  is_int = false;
  if (!frac && !has_exp && !dropped) {
    if (!neg && mant <= 0x7FFFFFFFFFFFFFFFull) {
      is_int = true;
      iv = (long long)mant;
    } else if (neg && mant <= 0x8000000000000000ull) {
      is_int = true;
      iv = (long long)(0ull - mant);
    }
  }
  if (mant == 0 && !overflow) return neg ? -0.0 : 0.0;
  if (!overflow && mant < (1ull << 53) && exp10 >= -22 && exp10 <= 22) {
    double d = (double)mant;
    d = exp10 >= 0 ? d * exact_pow10(exp10) : d / exact_pow10(-exp10);
    return neg ? -d : d;
  }
  return slow_decimal_to_double(p, n);
}

}  // namespace wjq
