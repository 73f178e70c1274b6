// Per-line walker: one thread validates one NDJSON line end to end and, in
// the same pass, records the value of every trie node of the query plan.
//
// Semantics restated from the reference CPU engine:
//   - strict RFC 8259 validation of exactly one value per line
//     (json.rs:198-421): strings reject raw bytes < 0x20 and bad escapes,
//     numbers follow the JSON grammar, literals must be exact, brackets must
//     match;
//   - blank lines are those made only of ASCII whitespace including form
//     feed (chunk.rs:436);
//   - path resolution follows json.rs:444-508: last duplicate key wins,
//     missing/null propagate as Missing, indexing a scalar is a type error,
//     and an invalid line beats a type error.
// The walk is iterative; container depth is tracked in a 64-bit register
// and, for the rare deeper line, in a caller-provided bit stack.
#pragma once

#include "devutil.cuh"
#include "plan.h"

namespace wjq {

enum LineStatus : int {
  LS_OK = 0,
  LS_INVALID = 1,
  LS_TYPE_ERROR = 2,
  LS_BLANK = 4,
  LS_DEEP = 5,       // deeper than the register stack; caller retries with a deep stack
  LS_DEEP_FULL = 6,  // deeper than the deep stack provided
  LS_FALLBACK = 7,   // not the fast path's shape; the general walker decides
};

// Values recorded per trie node for one line; offsets are relative to the
// line start.
struct NodeVals {
  uint8_t kind[kMaxNodes];
  uint8_t esc[kMaxNodes];
  uint32_t off[kMaxNodes];
  uint32_t len[kMaxNodes];
};

// A deep bit stack for levels >= 64 (bit = 1 for arrays), in global memory.
struct DeepStack {
  uint32_t *words;
  uint64_t cap_levels;
};

namespace detail {

enum Expect : int {
  EX_VALUE = 0,
  EX_KEY_OR_CLOSE = 1,
  EX_KEY = 2,
  EX_COLON = 3,
  EX_COMMA_OR_CLOSE = 4,
  EX_VALUE_OR_CLOSE = 5,
  EX_END = 6,
};

// Scans the string whose opening quote is at `s`.  Returns the index of the
// closing quote, or -1 when the string is malformed or unterminated.
__device__ __forceinline__ long long scan_string_bytes(const uint8_t *line, uint32_t n, uint32_t s,
                                                       bool &esc) {
  uint32_t j = s + 1;
  esc = false;
  for (;;) {
    // Aligned word steps over runs of ordinary bytes.
    while (((uintptr_t)(line + j) & 3u) == 0 && j + 4 <= n &&
           swar_string_special(*(const uint32_t *)(line + j)) == 0)
      j += 4;
    if (j >= n) return -1;
    uint32_t c = line[j];
    if (c == '"') return j;
    if (c == '\\') {
      if (j + 1 >= n) return -1;
      uint32_t e = line[j + 1];
      esc = true;
      if (e == '"' || e == '\\' || e == '/' || e == 'b' || e == 'f' || e == 'n' || e == 'r' ||
          e == 't') {
        j += 2;
      } else if (e == 'u') {
        if (j + 6 > n) return -1;
        if (hex_val(line[j + 2]) < 0 || hex_val(line[j + 3]) < 0 || hex_val(line[j + 4]) < 0 ||
            hex_val(line[j + 5]) < 0)
          return -1;
        j += 6;
      } else {
        return -1;
      }
      continue;
    }
    if (c < 0x20) return -1;
    j++;
  }
}

// Validates an atom (number or literal) occupying [s, e).
__device__ __forceinline__ bool valid_atom(const uint8_t *p, uint32_t n) {
  uint32_t c = p[0];
  if (c == 't') return n == 4 && p[1] == 'r' && p[2] == 'u' && p[3] == 'e';
  if (c == 'f') return n == 5 && p[1] == 'a' && p[2] == 'l' && p[3] == 's' && p[4] == 'e';
  if (c == 'n') return n == 4 && p[1] == 'u' && p[2] == 'l' && p[3] == 'l';
  // number: -?(0|[1-9][0-9]*)(\.[0-9]+)?([eE][+-]?[0-9]+)?   (json.rs:370-410)
  uint32_t i = 0;
  if (c == '-') i = 1;
  if (i >= n || !is_digit(p[i])) return false;
  if (p[i] == '0') {
    i++;
  } else {
    while (i < n && is_digit(p[i])) i++;
  }
  if (i < n && p[i] == '.') {
    i++;
    if (i >= n || !is_digit(p[i])) return false;
    while (i < n && is_digit(p[i])) i++;
  }
  if (i < n && (p[i] == 'e' || p[i] == 'E')) {
    i++;
    if (i < n && (p[i] == '+' || p[i] == '-')) i++;
    if (i >= n || !is_digit(p[i])) return false;
    while (i < n && is_digit(p[i])) i++;
  }
  return i == n;
}

__device__ __forceinline__ uint8_t kind_of(uint32_t c) {
  switch (c) {
    case '{': return JK_OBJ;
    case '[': return JK_ARR;
    case '"': return JK_STR;
    case 't': case 'f': return JK_BOOL;
    case 'n': return JK_NULL;
    default: return JK_NUM;
  }
}

// Key child of `node` whose decoded key equals the key body, or kNoNode.
__device__ __forceinline__ uint8_t match_key(const DevPlan &P, uint8_t node, const uint8_t *body,
                                             uint32_t len, bool esc) {
  for (uint8_t c = P.nodes[node].first_child; c != kNoNode; c = P.nodes[c].next_sibling) {
    const PlanNode &nd = P.nodes[c];
    if (nd.is_index) continue;
    if (!esc) {
      if (nd.key_len != len) continue;
      if (len && body[0] != nd.key_first) continue;
      const uint8_t *k = P.blob + nd.key_off;
      uint32_t t = 1;
      while (t < len && body[t] == k[t]) t++;
      if (t >= len) return c;
    } else if (cmp_str_body(body, len, true, P.blob + nd.key_off, nd.key_len) == 0) {
      return c;
    }
  }
  return kNoNode;
}

__device__ __forceinline__ uint8_t index_child(const DevPlan &P, uint8_t node, uint32_t idx) {
  if (node == kNoNode || !P.nodes[node].has_index_children) return kNoNode;
  for (uint8_t c = P.nodes[node].first_child; c != kNoNode; c = P.nodes[c].next_sibling) {
    const PlanNode &nd = P.nodes[c];
    if (nd.is_index && nd.index == idx) return c;
  }
  return kNoNode;
}

}  // namespace detail

// Walks `line[0, n)` (no newline; a trailing '\r' is JSON whitespace).
// `deep` may be null: a line nesting past 64 levels then returns LS_DEEP.
__device__ __noinline__ int walk_line(const DevPlan &P, const uint8_t *line, uint32_t n,
                                      NodeVals &v, const DeepStack *deep) {
  using namespace detail;
  const uint32_t n_nodes = P.n_nodes;
  for (uint32_t k = 0; k < n_nodes; k++) v.kind[k] = JK_MISSING;

  uint32_t i = 0;
  while (i < n && is_ws(line[i])) i++;
  if (i == n) return LS_BLANK;
  if (line[i] == 0x0C) {  // form feed counts toward a blank line, not toward JSON
    for (uint32_t j = i; j < n; j++) {
      uint32_t c = line[j];
      if (!(c == ' ' || c == '\t' || c == '\r' || c == 0x0C)) return LS_INVALID;
    }
    return LS_BLANK;
  }

  uint8_t node_at[kMaxDepthFast];  // trie node of the open container at each level
  uint32_t arr_idx[kMaxDepthFast];
  uint64_t stk = 0;                // bit d: container at level d is an array
  uint64_t depth = 0;
  uint8_t pending = n_nodes ? 0 : kNoNode;  // node the next value lands on
  int expect = EX_VALUE;

  for (;;) {
    while (i < n && is_ws(line[i])) i++;
    if (i >= n) break;
    uint32_t c = line[i];
    bool close = false;

    if (expect == EX_COLON) {
      if (c != ':') return LS_INVALID;
      i++;
      expect = EX_VALUE;
      continue;
    }
    if (expect == EX_KEY_OR_CLOSE || expect == EX_KEY) {
      if (c == '}' && expect == EX_KEY_OR_CLOSE) {
        close = true;
      } else {
        if (c != '"') return LS_INVALID;
        bool esc;
        long long e = scan_string_bytes(line, n, i, esc);
        if (e < 0) return LS_INVALID;
        uint8_t parent = depth <= kMaxDepthFast ? node_at[depth - 1] : kNoNode;
        pending = kNoNode;
        if (parent != kNoNode && P.nodes[parent].has_key_children)
          pending = match_key(P, parent, line + i + 1, (uint32_t)e - i - 1, esc);
        i = (uint32_t)e + 1;
        expect = EX_COLON;
        continue;
      }
    } else if (expect == EX_COMMA_OR_CLOSE) {
      uint32_t lvl = (uint32_t)depth - 1;
      bool arr;
      if (lvl < 64) {
        arr = (stk >> lvl) & 1;
      } else {
        uint64_t b = lvl - 64;
        arr = (deep->words[b >> 5] >> (b & 31)) & 1;
      }
      if (c == ',') {
        i++;
        if (arr) {
          pending = kNoNode;
          if (lvl < kMaxDepthFast) {
            uint32_t idx = ++arr_idx[lvl];
            pending = index_child(P, node_at[lvl], idx);
          }
          expect = EX_VALUE;
        } else {
          expect = EX_KEY;
        }
        continue;
      }
      if ((c == '}' && !arr) || (c == ']' && arr)) {
        close = true;
      } else {
        return LS_INVALID;
      }
    } else if (expect == EX_END) {
      return LS_INVALID;
    } else if (expect == EX_VALUE_OR_CLOSE && c == ']') {
      close = true;
    }

    if (close) {
      depth--;
      if (depth < kMaxDepthFast) {
        uint8_t cn = node_at[depth];
        if (cn != kNoNode) v.len[cn] = i + 1 - v.off[cn];
      }
      i++;
      expect = depth == 0 ? EX_END : EX_COMMA_OR_CLOSE;
      continue;
    }

    // A value starts at i (expect is EX_VALUE or EX_VALUE_OR_CLOSE).
    uint8_t vn = pending;
    if (vn != kNoNode) {
      for (uint32_t k = vn + 1u; k < P.nodes[vn].subtree_end; k++) v.kind[k] = JK_MISSING;
      v.kind[vn] = kind_of(c);
      v.off[vn] = i;
      v.esc[vn] = 0;
    }
    if (c == '{' || c == '[') {
      bool arr = c == '[';
      if (depth < 64) {
        if (arr) stk |= 1ull << depth;
        else stk &= ~(1ull << depth);
      } else {
        if (!deep) return LS_DEEP;
        uint64_t b = depth - 64;
        if (b >= deep->cap_levels) return LS_DEEP_FULL;
        uint32_t m = 1u << (b & 31);
        if (arr) deep->words[b >> 5] |= m;
        else deep->words[b >> 5] &= ~m;
      }
      if (depth < kMaxDepthFast) {
        node_at[depth] = vn;
        arr_idx[depth] = 0;
      }
      pending = arr ? index_child(P, vn, 0) : kNoNode;
      depth++;
      i++;
      expect = arr ? EX_VALUE_OR_CLOSE : EX_KEY_OR_CLOSE;
      continue;
    }
    uint32_t vend;
    if (c == '"') {
      bool esc;
      long long e = scan_string_bytes(line, n, i, esc);
      if (e < 0) return LS_INVALID;
      vend = (uint32_t)e + 1;
      if (vn != kNoNode) v.esc[vn] = esc;
    } else {
      uint32_t j = i + 1;
      while (j < n && !ends_atom(line[j])) j++;
      if (!valid_atom(line + i, j - i)) return LS_INVALID;
      vend = j;
    }
    if (vn != kNoNode) v.len[vn] = vend - i;
    i = vend;
    expect = depth == 0 ? EX_END : EX_COMMA_OR_CLOSE;
  }
  return expect == EX_END ? LS_OK : LS_INVALID;
}

// ---------------------------------------------------------------------------
// The window walker: the same semantics as walk_line for a line staged in a
// shared-memory window, where the line's own newline (or one stored after
// the data end) terminates every scan, so no step needs a bounds check.
// ---------------------------------------------------------------------------

namespace detail {

// JSON whitespace inside a line ('\n' ends the line).
__device__ __forceinline__ bool is_ws3(uint32_t c) { return c == ' ' || c == '\t' || c == '\r'; }

__device__ __forceinline__ uint32_t skip_ws3(const uint8_t *w, uint32_t i) {
  while (is_ws3(w[i])) i++;
  return i;
}

// Four bytes at any offset of a 4-byte-aligned window.
__device__ __forceinline__ uint32_t load4(const uint8_t *w, uint32_t i) {
  const uint32_t *p = (const uint32_t *)(w + (i & ~3u));
  return __funnelshift_r(p[0], p[1], (i & 3u) * 8u);
}

// Number of ASCII digits starting at w[j]; `term` receives the byte after
// them.
__device__ __forceinline__ uint32_t digit_run(const uint8_t *w, uint32_t j, uint32_t &term) {
  uint32_t n = 0;
  for (;;) {
    uint32_t x = load4(w, j + n);
    // a byte is a digit when its high nibble is 3 and its low nibble is <= 9
    uint32_t nd = ((x & 0xF0F0F0F0u) ^ 0x30303030u) | (((x & 0x0F0F0F0Fu) + 0x06060606u) & 0x10101010u);
    if (nd) {
      const uint32_t sh = ((uint32_t)__ffs(nd) - 1u) & ~7u;
      term = (x >> sh) & 0xFFu;
      return n + (sh >> 3);
    }
    n += 4;
  }
}

__device__ __forceinline__ bool simple_escape(uint32_t e) {
  return e == '"' || e == '\\' || e == '/' || e == 'b' || e == 'f' || e == 'n' || e == 'r' ||
         e == 't';
}

// Closing quote of the string opened at w[i], or 0 when the string is
// malformed (a bad escape, a raw control byte) or reaches the newline.
// `esc` reports whether the body holds a backslash.  `sm` has one bit per
// window byte that is '"', '\\' or below 0x20 (the stage-1 special mask), so
// the scan jumps from one such byte to the next: ordinary bytes are never
// looked at.  The line's own newline is such a byte, so no search passes
// it: every escape that moves past a byte has checked that byte first.
__device__ __forceinline__ uint32_t mask_string(const uint8_t *w, const uint32_t *sm, uint32_t i,
                                                bool &esc) {
  uint32_t p = i + 1;
  esc = false;
  for (;;) {
    uint32_t k = p >> 5;
    uint32_t m = sm[k] & (0xFFFFFFFFu << (p & 31u));
    while (!m) m = sm[++k];
    p = (k << 5) + (uint32_t)__ffs(m) - 1u;
    const uint32_t c = w[p];
    if (c == '"') return p;
    if (c != '\\') return 0;  // a byte below 0x20
    esc = true;
    const uint32_t e = w[p + 1];
    if (e == 'u') {
      if (hex_val(w[p + 2]) < 0 || hex_val(w[p + 3]) < 0 || hex_val(w[p + 4]) < 0 ||
          hex_val(w[p + 5]) < 0)
        return 0;
      p += 6;
    } else {
      if (!simple_escape(e)) return 0;
      p += 2;
    }
  }
}

// End (exclusive) of the number or literal starting at w[i] == c, or 0 when
// it is malformed.  The byte after it is checked by the caller.
__device__ __forceinline__ uint32_t win_atom(const uint8_t *w, uint32_t i, uint32_t c) {
  if (c == 't') return load4(w, i) == 0x65757274u ? i + 4 : 0;      // "true"
  if (c == 'n') return load4(w, i) == 0x6C6C756Eu ? i + 4 : 0;      // "null"
  if (c == 'f') return load4(w, i + 1) == 0x65736C61u ? i + 5 : 0;  // "alse"
  // -?(0|[1-9][0-9]*)(\.[0-9]+)?([eE][+-]?[0-9]+)?   (json.rs:370-410)
  uint32_t j = i;
  if (c == '-') c = w[++j];
  if (c - '0' >= 10u) return 0;
  uint32_t t;
  uint32_t d = digit_run(w, j, t);
  if (c == '0' && d > 1) return 0;
  j += d;
  if (t == '.') {
    d = digit_run(w, j + 1, t);
    if (!d) return 0;
    j += 1 + d;
  }
  if ((t | 0x20u) == 'e') {
    uint32_t sgn = w[++j];
    if (sgn == '+' || sgn == '-') j++;
    d = digit_run(w, j, t);
    if (!d) return 0;
    j += d;
  }
  return j;
}

// match_key for a key body at w[off, off + len) of a window: keys of up to
// 8 bytes compare as two words.
__device__ __forceinline__ uint8_t match_key_win(const DevPlan &P, uint8_t node, const uint8_t *w,
                                                 uint32_t off, uint32_t len, bool esc) {
  if (esc) return match_key(P, node, w + off, len, esc);
  const uint32_t w0 = load4(w, off), w1 = load4(w, off + 4);
  const uint32_t m0 = len >= 4 ? 0xFFFFFFFFu : (1u << (8 * len)) - 1u;
  const uint32_t m1 = len >= 8 ? 0xFFFFFFFFu : len > 4 ? (1u << (8 * (len - 4))) - 1u : 0u;
  for (uint8_t c = P.nodes[node].first_child; c != kNoNode; c = P.nodes[c].next_sibling) {
    const PlanNode &nd = P.nodes[c];
    if (nd.is_index || nd.key_len != len) continue;
    if ((w0 & m0) != nd.key_w[0] || (w1 & m1) != nd.key_w[1]) continue;
    if (len <= 8) return c;
    const uint8_t *k = P.blob + nd.key_off;
    uint32_t t = 8;
    while (t < len && w[off + t] == k[t]) t++;
    if (t >= len) return c;
  }
  return kNoNode;
}

}  // namespace detail

// Walks the line w[s, e) of a window.  w must be 4-byte aligned, w[e] must
// be '\n' and the 32 bytes after it readable; `sm` is the window's special
// mask (bit j of sm[j / 32]: byte j is '"', '\\' or below 0x20), complete at
// least up to e.  Offsets recorded in `v` are relative to s.  Lines nesting
// past 64 levels return LS_DEEP.
__device__ __noinline__ int walk_masked(const DevPlan &P, const uint8_t *w, const uint32_t *sm,
                                           uint32_t s, uint32_t e, NodeVals &v) {
  using namespace detail;
  const uint32_t n_nodes = P.n_nodes;
  for (uint32_t k = 0; k < n_nodes; k++) v.kind[k] = JK_MISSING;

  uint32_t i = s;
  uint32_t c = w[i];
  if (is_ws3(c)) {
    i = skip_ws3(w, i);
    c = w[i];
  }
  if (c == '\n') return LS_BLANK;
  if (c == 0x0C) {  // form feed counts toward a blank line, not toward JSON
    for (; i < e; i++) {
      c = w[i];
      if (!(is_ws3(c) || c == 0x0C)) return LS_INVALID;
    }
    return LS_BLANK;
  }

  uint64_t arrs = 0;  // bit d: the container open at depth d is an array
  uint32_t depth = 0;
  uint32_t cur = kNoNode, idx = 0;  // trie node and element index of the innermost container
  unsigned long long cur_lm = 0;    // key_len_mask of cur (0: no key is looked up)
  uint8_t stk_node[kMaxDepthFast];
  uint32_t stk_idx[kMaxDepthFast];
  uint32_t vn = n_nodes ? 0u : kNoNode;  // node the next value lands on
  bool want_key = false;

  for (;;) {
    if (want_key) {
      if (c != '"') return LS_INVALID;
      bool esc;
      const uint32_t q = mask_string(w, sm, i, esc);
      if (!q) return LS_INVALID;
      vn = kNoNode;
      if (cur_lm) {
        const uint32_t kl = q - i - 1;
        if (esc || ((cur_lm >> (kl < 63u ? kl : 63u)) & 1ull))
          vn = match_key_win(P, (uint8_t)cur, w, i + 1, kl, esc);
      }
      // ':' and the value's first byte, usually in one read
      const uint32_t la = load4(w, q + 1);
      if ((la & 0xFFu) == ':') {
        i = q + 2;
        c = (la >> 8) & 0xFFu;
      } else {
        i = skip_ws3(w, q + 1);
        if (w[i] != ':') return LS_INVALID;
        c = w[++i];
      }
      if (is_ws3(c)) {
        i = skip_ws3(w, i);
        c = w[i];
      }
    }
    // A value starts at w[i] == c.
    if (vn != kNoNode) {
      for (uint32_t k = vn + 1u; k < P.nodes[vn].subtree_end; k++) v.kind[k] = JK_MISSING;
      v.kind[vn] = kind_of(c);
      v.off[vn] = i - s;
      v.esc[vn] = 0;
    }
    if (c == '{' || c == '[') {
      if (depth >= kMaxDepthFast) return LS_DEEP;
      const bool arr = c == '[';
      if (arr) arrs |= 1ull << depth;
      else arrs &= ~(1ull << depth);
      stk_node[depth] = (uint8_t)cur;
      stk_idx[depth] = idx;
      depth++;
      cur = vn;
      idx = 0;
      cur_lm = (!arr && vn != kNoNode) ? P.nodes[vn].key_len_mask : 0ull;
      c = w[++i];
      if (is_ws3(c)) {
        i = skip_ws3(w, i);
        c = w[i];
      }
      if (c != (arr ? (uint32_t)']' : (uint32_t)'}')) {
        want_key = !arr;
        vn = arr ? index_child(P, (uint8_t)cur, 0) : kNoNode;
        continue;
      }
      // an empty container: its close is taken below
    } else {
      uint32_t j;
      if (c == '"') {
        bool esc;
        j = mask_string(w, sm, i, esc);
        if (!j) return LS_INVALID;
        j++;
        if (vn != kNoNode) v.esc[vn] = esc;
      } else {
        j = win_atom(w, i, c);
        if (!j) return LS_INVALID;
      }
      if (vn != kNoNode) v.len[vn] = j - i;
      i = j;
    }
    // After a value: commas and closing brackets, with the next bytes read
    // four at a time.
    uint32_t la = load4(w, i);
    for (;;) {
      c = la & 0xFFu;
      if (is_ws3(c)) {
        i = skip_ws3(w, i);
        la = load4(w, i);
        c = la & 0xFFu;
      }
      if (depth == 0) return c == '\n' ? LS_OK : LS_INVALID;
      const bool arr = (arrs >> (depth - 1)) & 1;
      if (c == ',') {
        i++;
        c = (la >> 8) & 0xFFu;
        if (is_ws3(c)) {
          i = skip_ws3(w, i);
          c = w[i];
        }
        if (arr) {
          idx++;
          vn = index_child(P, (uint8_t)cur, idx);
        }
        want_key = !arr;
        break;
      }
      if (c != (arr ? (uint32_t)']' : (uint32_t)'}')) return LS_INVALID;
      if (cur != kNoNode) v.len[cur] = i + 1 - s - v.off[cur];
      depth--;
      cur = stk_node[depth];
      idx = stk_idx[depth];
      const bool parent_obj = depth > 0 && !((arrs >> (depth - 1)) & 1);
      cur_lm = (parent_obj && cur != kNoNode) ? P.nodes[cur].key_len_mask : 0ull;
      i++;
      la = load4(w, i);
    }
  }
}

namespace detail {

// Four hex digits at w[i..i+3].
__device__ __forceinline__ bool hex4_at(const uint8_t *w, uint32_t i) {
  return hex_val(w[i]) >= 0 && hex_val(w[i + 1]) >= 0 && hex_val(w[i + 2]) >= 0 && hex_val(w[i + 3]) >= 0;
}

// Position of the next special byte (a set bit of the window's special mask)
// from the cursor (k, m), consuming it.  The line's newline is special, so
// a walk that reaches it stops there.
__device__ __forceinline__ uint32_t pop_special(const uint32_t *sm, uint32_t &k, uint32_t &m) {
  while (!m) m = sm[++k];
  const uint32_t b = (k << 5) + (uint32_t)__ffs(m) - 1u;
  m &= m - 1u;
  return b;
}

}  // namespace detail

// The fast path of the window walk, for the common shape of a log line: one
// object whose members are separated by single ',' and ':' with no
// whitespace, keys without escapes, and values that are scalars or objects
// of the same shape, at most 8 deep (no arrays).  It steps from special byte
// to special byte: a key is its two quotes, a string value its quotes and
// escapes, and only the bytes right after them are read ('"' ':' value, ','
// or '}').  Lines of that shape get exactly walk_masked's verdict and node
// values; a line it finds malformed where every check so far has passed (a
// raw control byte or the line's end inside a string, a value that is no
// number or literal) is LS_INVALID without the general walk; for any other
// line (whitespace, arrays, escaped keys, deeper nesting, anything else
// malformed) it returns LS_FALLBACK and records nothing that walk_masked
// does not overwrite.  Same window contract as walk_masked.
//
// Checks whose outcome does not steer the walk (that a key's quotes are
// quotes where they were expected, the ':' after it, an escape's letter)
// are folded into `bad` and decided once, when the line's object closes, so
// the shared-memory loads behind them do not stall each step.  Every pop is
// bounded by the line's newline (a special byte), so a walk over a line of
// another shape still ends at e.
__device__ __forceinline__ int walk_objects(const DevPlan &P, const uint8_t *w, const uint32_t *sm,
                                            uint32_t s, uint32_t e, NodeVals &v) {
  using namespace detail;
  if (w[s] != '{') return LS_FALLBACK;
  const uint32_t n_nodes = P.n_nodes;
  for (uint32_t k = 0; k < n_nodes; k++) v.kind[k] = JK_MISSING;
  uint32_t cur = n_nodes ? 0u : kNoNode;  // trie node of the innermost open object
  unsigned long long lm = 0;             // its key_len_mask (0: no key is looked up)
  if (cur != kNoNode) {
    v.kind[0] = JK_OBJ;
    v.off[0] = 0;
    v.esc[0] = 0;
    lm = P.nodes[0].key_len_mask;
  }
  unsigned long long stack = 0;  // trie nodes of the enclosing objects, 8 bits a level
  uint32_t depth = 1;
  uint32_t k = (s + 1) >> 5;
  uint32_t m = sm[k] & (0xFFFFFFFFu << ((s + 1) & 31u));
  uint32_t p = s + 1;  // where the next key's opening quote must be
  uint32_t bad = 0;    // deferred checks: nonzero when the line is not of this shape
  for (;;) {
    const uint32_t q0 = pop_special(sm, k, m);
    if (q0 >= e) return LS_FALLBACK;
    const uint32_t q1 = pop_special(sm, k, m);
    if (q1 >= e) return LS_FALLBACK;
    bad |= (q0 ^ p) | ((uint32_t)w[q0] ^ '"') | ((uint32_t)w[q1] ^ '"');
    uint32_t vn = kNoNode;
    const uint32_t kl = q1 - q0 - 1;
    if ((lm >> (kl < 63u ? kl : 63u)) & 1ull) vn = match_key_win(P, (uint8_t)cur, w, q0 + 1, kl, false);
    const uint32_t la = load4(w, q1 + 1);
    bad |= (la & 0xFFu) ^ ':';
    const uint32_t c = (la >> 8) & 0xFFu;
    const uint32_t vs = q1 + 2;
    if (vn != kNoNode) {
      for (uint32_t x = vn + 1u; x < P.nodes[vn].subtree_end; x++) v.kind[x] = JK_MISSING;
      v.kind[vn] = kind_of(c);
      v.off[vn] = vs - s;
      v.esc[vn] = 0;
    }
    if (c == '{') {
      if (depth >= 8) return LS_FALLBACK;
      stack = (stack << 8) | cur;
      depth++;
      cur = vn;
      lm = vn != kNoNode ? P.nodes[vn].key_len_mask : 0ull;
      p = vs + 1;
      continue;
    }
    uint32_t ve;
    if (c == '"') {
      const uint32_t r0 = pop_special(sm, k, m);  // the opening quote, at vs
      if (r0 >= e) return LS_FALLBACK;
      bad |= r0 ^ vs;
      bool esc = false;
      uint32_t r;
      for (;;) {
        r = pop_special(sm, k, m);
        const uint32_t b = w[r];
        if (b == '"') break;
        // a raw control byte or the newline inside a string: with every
        // earlier check passed, the line is malformed whatever its shape
        if (b != '\\') return bad ? LS_FALLBACK : LS_INVALID;
        esc = true;
        const uint32_t x = w[r + 1];
        if (x == '"' || x == '\\') {
          pop_special(sm, k, m);  // the escaped byte is special itself (r + 1 < e)
        } else if (x == 'u') {
          bad |= hex4_at(w, r + 2) ? 0u : 1u;
        } else {
          bad |= simple_escape(x) ? 0u : 1u;  // a special x stops the next pop
        }
      }
      ve = r + 1;
      if (vn != kNoNode) v.esc[vn] = esc;
    } else {
      if (c == '[') return LS_FALLBACK;
      ve = win_atom(w, vs, c);
      // no number or literal at the value's place (a bare word, a bad
      // number, a cut literal): malformed, unless an earlier check failed
      // or the value is only preceded by whitespace
      if (!ve) return (bad || c == ' ' || c == '\t' || c == '\r') ? LS_FALLBACK : LS_INVALID;
    }
    if (vn != kNoNode) v.len[vn] = ve - vs;
    // after a value: ',' and the next key, or '}' closing one or more objects
    uint32_t t = w[ve];
    while (t == '}') {
      if (cur != kNoNode) v.len[cur] = ve + 1 - s - v.off[cur];
      if (--depth == 0) return (ve + 1 == e && !bad) ? LS_OK : LS_FALLBACK;
      cur = (uint32_t)(stack & 0xFFu);
      stack >>= 8;
      lm = cur != kNoNode ? P.nodes[cur].key_len_mask : 0ull;
      t = w[++ve];
    }
    if (t != ',') return LS_FALLBACK;
    p = ve + 1;
  }
}

// ---------------------------------------------------------------------------
// Evaluation of a walked line.
// ---------------------------------------------------------------------------

enum SlotState : uint8_t { SS_FOUND = 0, SS_MISSING = 1, SS_TYPE_ERROR = 2 };

struct SlotVal {
  uint8_t state;  // SlotState
  uint8_t kind;   // JKind (JK_MISSING when not found)
  uint8_t esc;
  uint32_t off;
  uint32_t len;
};

// Resolves slot `s` from the node values (json.rs:461-507).  Walking up from
// the terminal node, the shallowest failing step decides Missing vs type
// error, exactly as the top-down lookup does.
__device__ __forceinline__ SlotVal resolve_slot(const DevPlan &P, const NodeVals &v, uint32_t s) {
  SlotVal r;
  uint8_t t = P.slot_node[s];
  uint8_t st = SS_FOUND;
  for (uint8_t c = t; c != 0;) {
    uint8_t p = P.nodes[c].parent;
    uint8_t kp = v.kind[p];
    if (kp == JK_MISSING || kp == JK_NULL) st = SS_MISSING;
    else if (!P.nodes[c].is_index && kp != JK_OBJ) st = SS_TYPE_ERROR;
    else if (P.nodes[c].is_index && kp != JK_ARR) st = SS_TYPE_ERROR;
    c = p;
  }
  r.state = st;
  if (st == SS_FOUND && v.kind[t] != JK_MISSING) {
    r.kind = v.kind[t];
    r.esc = v.esc[t];
    r.off = v.off[t];
    r.len = v.len[t];
  } else {
    if (st == SS_FOUND) r.state = SS_MISSING;
    r.kind = JK_MISSING;
    r.esc = 0;
    r.off = 0;
    r.len = 0;
  }
  return r;
}

__device__ __forceinline__ uint32_t slot_rank(const uint8_t *line, const SlotVal &s) {
  switch (s.kind) {
    case JK_MISSING: case JK_NULL: return 0;
    case JK_BOOL: return line[s.off] == 't' ? 2 : 1;
    case JK_NUM: return 3;
    case JK_STR: return 4;
    case JK_ARR: return 5;
    default: return 6;
  }
}

// Three-way compare of a slot with a literal (json.rs:662-693).
__device__ __forceinline__ int compare_slot(const DevPlan &P, const uint8_t *line, const SlotVal &s,
                                            const PlanCmp &c) {
  uint32_t sr = slot_rank(line, s);
  if (sr != c.lit_rank) return sr < c.lit_rank ? -1 : 1;
  if (c.lit_kind == 3 /* NUM */) {
    bool is_int;
    long long iv;
    double d = parse_number(line + s.off, s.len, is_int, iv);
    if (d < c.lit_num) return -1;
    if (d > c.lit_num) return 1;
    return 0;
  }
  if (c.lit_kind == 4 /* STR */)
    return cmp_str_body(line + s.off + 1, s.len - 2, s.esc, P.blob + c.lit_off, c.lit_len);
  return 0;
}

__device__ __forceinline__ bool op_accepts(uint32_t op, int o) {
  switch (op) {
    case 0: return o == 0;
    case 1: return o != 0;
    case 2: return o < 0;
    case 3: return o <= 0;
    case 4: return o > 0;
    default: return o >= 0;
  }
}

__device__ __forceinline__ bool truthy(const uint8_t *line, const SlotVal &s) {
  if (s.kind == JK_MISSING || s.kind == JK_NULL) return false;
  return !(s.kind == JK_BOOL && line[s.off] == 'f');
}

// Evaluates the RPN condition (exec/cpu.rs:443-453; And/Or short-circuit
// has no side effects here, so a strict evaluation gives the same verdict).
__device__ __forceinline__ bool eval_filter(const DevPlan &P, const uint8_t *line,
                                            const SlotVal *slots) {
  uint64_t st = 0;  // bit stack, top at bit 0
  for (uint32_t k = 0; k < P.n_cond; k++) {
    const PlanCond &o = P.cond[k];
    switch (o.op) {
      case 0: {
        const PlanCmp &c = P.cmps[o.arg];
        bool r = op_accepts(c.op, compare_slot(P, line, slots[c.slot], c));
        st = (st << 1) | (r ? 1u : 0u);
        break;
      }
      case 1:
        st = (st << 1) | (truthy(line, slots[o.arg]) ? 1u : 0u);
        break;
      case 2: {
        uint64_t b = st & 1, a = (st >> 1) & 1;
        st = (st >> 2 << 1) | (a & b);
        break;
      }
      case 3: {
        uint64_t b = st & 1, a = (st >> 1) & 1;
        st = (st >> 2 << 1) | (a | b);
        break;
      }
      default:
        st ^= 1;
    }
  }
  return st & 1;
}

}  // namespace wjq
