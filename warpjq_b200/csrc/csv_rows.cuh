// CSV rows to NDJSON, one row per thread (device code of the CSV
// converter, warpjq_csv_convert): the field rules are those of csv.cu's
// header comment.  Plain bytes are found and moved four at a time (SWAR
// byte masks over aligned words); escapes, key texts and quotes are
// inserted around them.  Also the host-side header parsing.  Kept in a
// header so a host harness can compile the same code.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace wjq_csv {

typedef unsigned long long u64;

// Bit k (k < 4) set when byte k of `w` equals the byte repeated in `pat`.
__device__ __forceinline__ uint32_t eq4(uint32_t w, uint32_t pat) {
  const uint32_t x = w ^ pat;
  const uint32_t z = ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu);  // 0x80 at equal bytes
  return (((z >> 7) * 0x00204081u) >> 21) & 0xFu;  // gathers the four flags in byte order
}

// Input words: the aligned 4-byte word holding byte i, from a 16-byte
// aligned block kept in registers (a block that holds one byte of the input
// lies in the same page as that byte, so the loads stay in mapped memory).
struct WordIn {
  const uint8_t *d;
  uintptr_t blk;
  uint4 v;
  __device__ __forceinline__ explicit WordIn(const uint8_t *d_) : d(d_), blk(1) {}
  __device__ __forceinline__ uint32_t word(u64 i) {
    const uintptr_t p = (uintptr_t)(d + i), b = p & ~(uintptr_t)15;
    if (b != blk) {
      blk = b;
      v = __ldg(reinterpret_cast<const uint4 *>(b));
    }
    const uint32_t o = (uint32_t)(p >> 2) & 3;
    return o < 2 ? (o ? v.y : v.x) : (o == 2 ? v.z : v.w);
  }
  __device__ __forceinline__ uint32_t lane(u64 i) const { return (uint32_t)((uintptr_t)(d + i) & 3); }
  __device__ __forceinline__ uint8_t byte(u64 i) { return (uint8_t)(word(i) >> (8 * lane(i))); }
};

// Output from `p` on in aligned 4-byte stores; the first word of the line
// is written bytewise from p (the previous line's thread owns the bytes
// before it), and so is the last, partial word (flush).
struct WordOut {
  uint8_t *row0;
  uintptr_t w;  // aligned word being filled
  uint32_t off; // its bytes already filled (those before row0 count as filled)
  u64 acc;
  __device__ __forceinline__ explicit WordOut(uint8_t *p)
      : row0(p), w((uintptr_t)p & ~(uintptr_t)3), off((uint32_t)((uintptr_t)p & 3)), acc(0) {}
  // appends the k (1..4) low bytes of v
  __device__ __forceinline__ void put(uint32_t v, uint32_t k) {
    const uint32_t m = k >= 4 ? 0xFFFFFFFFu : (1u << (8 * k)) - 1;
    acc |= (u64)(v & m) << (8 * off);
    off += k;
    if (off >= 4) {
      store((uint32_t)acc);
      acc >>= 32;
      w += 4;
      off -= 4;
    }
  }
  __device__ __forceinline__ void store(uint32_t x) {
    if (w >= (uintptr_t)row0) {
      *reinterpret_cast<uint32_t *>(w) = x;
    } else {
      uint8_t *b = reinterpret_cast<uint8_t *>(w);
      for (uint32_t j = (uint32_t)((uintptr_t)row0 - w); j < 4; j++) b[j] = (uint8_t)(x >> (8 * j));
    }
  }
  __device__ __forceinline__ void flush() {
    uint8_t *b = reinterpret_cast<uint8_t *>(w);
    for (uint32_t j = w < (uintptr_t)row0 ? (uint32_t)((uintptr_t)row0 - w) : 0; j < off; j++)
      b[j] = (uint8_t)(acc >> (8 * j));
  }
};

// Bytes of `x` below 0x20, as a 4-bit mask.
__device__ __forceinline__ uint32_t ctl4(uint32_t x) { return eq4(x & 0xE0E0E0E0u, 0u); }

// JSON string bytes of a byte that needs an escape (0x22, 0x5C, below 0x20).
__device__ __forceinline__ uint32_t esc_len(uint8_t c) {
  return (c == '"' || c == '\\' || c == '\n' || c == '\r' || c == '\t' || c == 8 || c == 12) ? 2 : 6;
}

__device__ __forceinline__ void put_esc(WordOut &w, uint8_t c) {
  uint32_t two = 0;
  switch (c) {
    case '"': two = '"'; break;
    case '\\': two = '\\'; break;
    case '\n': two = 'n'; break;
    case '\r': two = 'r'; break;
    case '\t': two = 't'; break;
    case 8: two = 'b'; break;
    case 12: two = 'f'; break;
    default: break;
  }
  if (two) {
    w.put('\\' | two << 8, 2);
  } else {
    const uint32_t l = c & 15;
    w.put('\\' | 'u' << 8 | '0' << 16 | (uint32_t)'0' << 24, 4);
    w.put((uint32_t)('0' + (c >> 4)) | (uint32_t)(l < 10 ? '0' + l : 'a' + l - 10) << 8, 2);
  }
}

// Bytes [p, e) as JSON string content (escaped where needed).  With kQuoted
// a '"' stops the run (its position is returned); otherwise a '"' is
// escaped and the run ends at e.  Plain bytes move a word at a time.
template <bool kWrite, bool kQuoted>
__device__ __forceinline__ u64 esc_run(WordIn &in, u64 p, u64 e, WordOut &w, u64 &len) {
  while (p < e) {
    const uint32_t s0 = in.lane(p);
    const uint32_t x = in.word(p);
    const uint32_t t = e - p >= 4 - s0 ? 4 : s0 + (uint32_t)(e - p);
    const uint32_t range = ((1u << t) - 1) & ~((1u << s0) - 1);
    const uint32_t q = eq4(x, 0x22222222u) & range;
    const uint32_t special = (eq4(x, 0x5C5C5C5Cu) | ctl4(x) | (kQuoted ? 0u : q)) & range;
    const uint32_t any = special | (kQuoted ? q : 0u);
    if (!any) {
      len += t - s0;
      if (kWrite) w.put(x >> (8 * s0), t - s0);
      p += t - s0;
      continue;
    }
    const uint32_t f = __ffs(any) - 1;
    if (f > s0) {
      len += f - s0;
      if (kWrite) w.put(x >> (8 * s0), f - s0);
      p += f - s0;
    }
    if (kQuoted && ((q >> f) & 1)) return p;
    const uint8_t c = (uint8_t)(x >> (8 * f));
    len += esc_len(c);
    if (kWrite) put_esc(w, c);
    p++;
  }
  return p;
}

// First ',' in [p, e), or e.
__device__ __forceinline__ u64 find_comma(WordIn &in, u64 p, u64 e) {
  while (p < e) {
    const uint32_t s0 = in.lane(p);
    const uint32_t x = in.word(p);
    const uint32_t t = e - p >= 4 - s0 ? 4 : s0 + (uint32_t)(e - p);
    const uint32_t m = eq4(x, 0x2C2C2C2Cu) & ((1u << t) - 1) & ~((1u << s0) - 1);
    if (m) return p + (__ffs(m) - 1 - s0);
    p += t - s0;
  }
  return e;
}

// True when [a, b) is a JSON number: -?(0|[1-9][0-9]*)(.[0-9]+)?([eE][+-]?[0-9]+)?
__device__ bool is_number(WordIn &in, u64 a, u64 b) {
  u64 i = a;
  if (i < b && in.byte(i) == '-') i++;
  if (i >= b) return false;
  uint8_t c = in.byte(i);
  if (c < '0' || c > '9') return false;
  i++;
  if (c != '0')
    while (i < b && (c = in.byte(i)) >= '0' && c <= '9') i++;
  if (i < b && in.byte(i) == '.') {
    i++;
    if (i >= b || (c = in.byte(i)) < '0' || c > '9') return false;
    while (i < b && (c = in.byte(i)) >= '0' && c <= '9') i++;
  }
  if (i < b && ((c = in.byte(i)) == 'e' || c == 'E')) {
    i++;
    if (i < b && ((c = in.byte(i)) == '+' || c == '-')) i++;
    if (i >= b || (c = in.byte(i)) < '0' || c > '9') return false;
    while (i < b && (c = in.byte(i)) >= '0' && c <= '9') i++;
  }
  return i == b;
}

struct KeySet {
  const uint32_t *text;  // key k: `"name":` (a leading ',' for k > 0) from word meta[2k], meta[2k+1] bytes
  const uint32_t *meta;
  uint32_t n;
};

// One row [s, e) to NDJSON: its length, and with kWrite its bytes.
template <bool kWrite>
__device__ u64 row_json(WordIn &in, u64 s, u64 e, const KeySet &ks, WordOut &w) {
  if (e > s && in.byte(e - 1) == '\r') e--;
  if (e == s) {  // an empty row: an empty line
    if (kWrite) w.put('\n', 1);
    return 1;
  }
  u64 len = 3;  // "{" "}\n"
  if (kWrite) w.put('{', 1);
  u64 p = s;
  bool more = true;
  for (uint32_t k = 0; k < ks.n && more; k++) {
    const uint32_t kw = __ldg(ks.meta + 2 * k), kl = __ldg(ks.meta + 2 * k + 1);
    len += kl;
    if (kWrite)
      for (uint32_t j = 0; j < kl; j += 4) w.put(__ldg(ks.text + kw + (j >> 2)), kl - j < 4 ? kl - j : 4);
    if (p < e && in.byte(p) == '"') {  // quoted
      len += 2;
      if (kWrite) w.put('"', 1);
      p++;
      for (;;) {
        p = esc_run<kWrite, true>(in, p, e, w, len);
        if (p >= e) break;                          // no closing quote
        if (p + 1 < e && in.byte(p + 1) == '"') {  // a doubled quote
          len += 2;
          if (kWrite) w.put('\\' | '"' << 8, 2);
          p += 2;
          continue;
        }
        p++;  // the closing quote
        break;
      }
      if (p < e && in.byte(p) != ',') {  // bytes after the closing quote, kept
        const u64 q = find_comma(in, p, e);
        esc_run<kWrite, false>(in, p, q, w, len);
        p = q;
      }
      if (kWrite) w.put('"', 1);
    } else {
      const u64 q = find_comma(in, p, e);
      if (q == p) {
        len += 4;
        if (kWrite) w.put('n' | 'u' << 8 | 'l' << 16 | (uint32_t)'l' << 24, 4);
      } else if (is_number(in, p, q)) {
        esc_run<kWrite, false>(in, p, q, w, len);  // digits, signs, '.', 'e': copied as they are
      } else {
        len += 2;
        if (kWrite) w.put('"', 1);
        esc_run<kWrite, false>(in, p, q, w, len);
        if (kWrite) w.put('"', 1);
      }
      p = q;
    }
    more = p < e;  // a ',' follows
    p++;
  }
  if (kWrite) w.put('}' | '\n' << 8, 2);
  return len;
}

inline void escape_into(std::string &o, const uint8_t *s, size_t n) {
  static const char *hx = "0123456789abcdef";
  for (size_t i = 0; i < n; i++) {
    const uint8_t c = s[i];
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      case 8: o += "\\b"; break;
      case 12: o += "\\f"; break;
      default:
        if (c < 0x20) {
          o += "\\u00";
          o += hx[c >> 4];
          o += hx[c & 15];
        } else {
          o += (char)c;
        }
    }
  }
}

// Header names from the raw header row, by the field rules above, as the
// key texts `"name":` (with a leading ',' after the first).
inline void parse_header(const uint8_t *h, size_t n, std::string &text, std::vector<uint32_t> &offs) {
  text.clear();
  offs.assign(1, 0);
  if (n >= 3 && h[0] == 0xEF && h[1] == 0xBB && h[2] == 0xBF) {
    h += 3;
    n -= 3;
  }
  if (n && h[n - 1] == '\r') n--;
  if (!n) return;
  size_t p = 0;
  bool more = true;
  while (more) {
    std::string name;
    if (p < n && h[p] == '"') {
      p++;
      while (p < n) {
        if (h[p] == '"') {
          if (p + 1 < n && h[p + 1] == '"') {
            name += '"';
            p += 2;
            continue;
          }
          p++;
          break;
        }
        name += (char)h[p++];
      }
      while (p < n && h[p] != ',') name += (char)h[p++];
    } else {
      while (p < n && h[p] != ',') name += (char)h[p++];
    }
    more = p < n;
    p++;
    if (offs.size() > 1) text += ',';
    text += '"';
    escape_into(text, (const uint8_t *)name.data(), name.size());
    text += "\":";
    offs.push_back((uint32_t)text.size());
  }
}

// Key texts packed from word boundaries: meta = (first word, bytes) per key.
inline void pack_keys(const std::string &text, const std::vector<uint32_t> &offs, std::vector<uint32_t> &words,
                      std::vector<uint32_t> &meta) {
  words.clear();
  meta.clear();
  for (size_t k = 0; k + 1 < offs.size(); k++) {
    const uint32_t a = offs[k], b = offs[k + 1];
    meta.push_back((uint32_t)words.size());
    meta.push_back(b - a);
    for (uint32_t j = a; j < b; j += 4) {
      uint32_t wv = 0;
      for (uint32_t t = 0; t < 4 && j + t < b; t++) wv |= (uint32_t)(uint8_t)text[j + t] << (8 * t);
      words.push_back(wv);
    }
  }
}

}  // namespace wjq_csv
