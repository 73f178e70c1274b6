// TEST INFRASTRUCTURE -- the oracle's JSON scanner.
// Restates crates/warpjq-core/src/json.rs of the reference project.
#include "oracle.h"

#include <cstdlib>
#include <cstring>
#include <clocale>

namespace oracle {

static inline bool json_ws(uint8_t c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

// json.rs:123-128
static inline size_t skip_ws(const uint8_t *b, size_t len, size_t i) {
  while (i < len && json_ws(b[i])) i++;
  return i;
}

static inline bool is_hex(uint8_t c) {
  return (c >= '0' && c <= '9') || (c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F');
}

static bool fail(JsonError &e, size_t at, const std::string &msg) {
  e.offset = at;
  e.detail = msg;
  return false;
}

// json.rs:325-334
static bool expect_lit(const uint8_t *b, size_t len, size_t i, const char *lit, size_t &end,
                       JsonError &e) {
  size_t n = std::strlen(lit);
  if (len >= i + n && std::memcmp(b + i, lit, n) == 0) {
    end = i + n;
    return true;
  }
  return fail(e, i, std::string("expected `") + lit + "`");
}

// json.rs:336-368
bool skip_string(const uint8_t *b, size_t len, size_t i, size_t &end, JsonError &e) {
  size_t j = i + 1;
  while (j < len) {
    uint8_t c = b[j];
    if (c == '"') {
      end = j + 1;
      return true;
    }
    if (c == '\\') {
      if (j + 1 >= len) return fail(e, j, "unterminated escape");
      uint8_t x = b[j + 1];
      switch (x) {
        case '"': case '\\': case '/': case 'b': case 'f': case 'n': case 'r': case 't':
          j += 2;
          break;
        case 'u':
          if (j + 6 > len || !is_hex(b[j + 2]) || !is_hex(b[j + 3]) || !is_hex(b[j + 4]) ||
              !is_hex(b[j + 5]))
            return fail(e, j, "malformed `\\u` escape");
          j += 6;
          break;
        default:
          return fail(e, j, std::string("invalid escape `\\") + (char)x + "`");
      }
      continue;
    }
    if (c < 0x20) return fail(e, j, "unescaped control character in string");
    j++;
  }
  return fail(e, i, "unterminated string");
}

// json.rs:370-410
static bool skip_number(const uint8_t *b, size_t len, size_t i, size_t &end, JsonError &e) {
  size_t j = i;
  if (b[j] == '-') j++;
  size_t int_start = j;
  while (j < len && b[j] >= '0' && b[j] <= '9') j++;
  if (j == int_start) return fail(e, i, "number with no digits");
  if (b[int_start] == '0' && j - int_start > 1) return fail(e, i, "number has a leading zero");
  if (j < len && b[j] == '.') {
    j++;
    size_t fs = j;
    while (j < len && b[j] >= '0' && b[j] <= '9') j++;
    if (j == fs) return fail(e, j, "number has no digits after `.`");
  }
  if (j < len && (b[j] == 'e' || b[j] == 'E')) {
    j++;
    if (j < len && (b[j] == '+' || b[j] == '-')) j++;
    size_t es = j;
    while (j < len && b[j] >= '0' && b[j] <= '9') j++;
    if (j == es) return fail(e, j, "number has no digits in its exponent");
  }
  end = j;
  return true;
}

// json.rs:198-323.  Iterative: nesting depth is bounded only by the line.
// The container stack is a bit vector (json.rs:135-189 keeps the first 64
// levels in a word and spills the rest; a vector<bool> does both jobs here).
bool skip_value(const uint8_t *b, size_t len, size_t start, size_t &end, JsonError &e) {
  enum { VALUE, KEY, AFTER } state = VALUE;
  std::vector<bool> stack;  // true = array
  size_t i = start;
  for (;;) {
    if (state == VALUE) {
      i = skip_ws(b, len, i);
      if (i >= len) return fail(e, i, "unexpected end of input");
      uint8_t c = b[i];
      if (c == '{') {
        i = skip_ws(b, len, i + 1);
        if (i < len && b[i] == '}') {
          i++;
          state = AFTER;
        } else {
          stack.push_back(false);
          state = KEY;
        }
      } else if (c == '[') {
        i = skip_ws(b, len, i + 1);
        if (i < len && b[i] == ']') {
          i++;
          state = AFTER;
        } else {
          stack.push_back(true);
          state = VALUE;
        }
      } else if (c == '"') {
        if (!skip_string(b, len, i, i, e)) return false;
        state = AFTER;
      } else if (c == 't') {
        if (!expect_lit(b, len, i, "true", i, e)) return false;
        state = AFTER;
      } else if (c == 'f') {
        if (!expect_lit(b, len, i, "false", i, e)) return false;
        state = AFTER;
      } else if (c == 'n') {
        if (!expect_lit(b, len, i, "null", i, e)) return false;
        state = AFTER;
      } else if (c == '-' || (c >= '0' && c <= '9')) {
        if (!skip_number(b, len, i, i, e)) return false;
        state = AFTER;
      } else {
        return fail(e, i, std::string("unexpected character `") + (char)c + "`");
      }
    } else if (state == KEY) {
      i = skip_ws(b, len, i);
      if (i >= len || b[i] != '"') return fail(e, i, "expected a string key");
      if (!skip_string(b, len, i, i, e)) return false;
      i = skip_ws(b, len, i);
      if (i >= len || b[i] != ':') return fail(e, i, "expected `:` after object key");
      i++;
      state = VALUE;
    } else {
      if (stack.empty()) {
        end = i;
        return true;
      }
      i = skip_ws(b, len, i);
      if (i >= len) return fail(e, i, "unexpected end of input");
      uint8_t c = b[i];
      bool arr = stack.back();
      if (c == ',') {
        i++;
        state = arr ? VALUE : KEY;
      } else if ((c == '}' && !arr) || (c == ']' && arr)) {
        i++;
        stack.pop_back();
      } else {
        return fail(e, i, arr ? "expected `,` or `]`" : "expected `,` or `}`");
      }
    }
  }
}

// json.rs:414-421
bool validate(const uint8_t *b, size_t len, JsonError &e) {
  size_t end = 0;
  if (!skip_value(b, len, 0, end, e)) return false;
  size_t rest = skip_ws(b, len, end);
  if (rest != len) return fail(e, rest, "trailing content after JSON value");
  return true;
}

// json.rs:423-432
static Kind kind_of(const uint8_t *b, size_t i) {
  switch (b[i]) {
    case '{': return Kind::Obj;
    case '[': return Kind::Arr;
    case '"': return Kind::Str;
    case 't': case 'f': return Kind::Bool;
    case 'n': return Kind::Null;
    default: return Kind::Num;
  }
}

// json.rs:510-519
static const char *type_name(Kind k) {
  switch (k) {
    case Kind::Missing: case Kind::Null: return "null";
    case Kind::Bool: return "boolean";
    case Kind::Num: return "number";
    case Kind::Str: return "string";
    case Kind::Arr: return "array";
    default: return "object";
  }
}

static const uint8_t kNullText[] = {'n', 'u', 'l', 'l'};

Slot missing_slot() {
  Slot s;
  s.kind = Kind::Missing;
  s.p = kNullText;
  s.n = 4;
  return s;
}

// json.rs:63-65
bool Slot::is_truthy() const {
  if (kind == Kind::Missing || kind == Kind::Null) return false;
  return !(n == 5 && std::memcmp(p, "false", 5) == 0);
}

// json.rs:73-78.  The reference parses with Rust's correctly rounded
// `str::parse::<f64>`; glibc's strtod is correctly rounded as well.
bool Slot::as_f64(double &v) const {
  if (kind != Kind::Num) return false;
  char buf[128];
  std::string big;
  const char *s;
  if (n < sizeof(buf)) {
    std::memcpy(buf, p, n);
    buf[n] = 0;
    s = buf;
  } else {
    big.assign((const char *)p, n);
    s = big.c_str();
  }
  v = std::strtod(s, nullptr);
  return true;
}

// json.rs:523-556.  Last duplicate key wins.
static bool object_get(const uint8_t *b, size_t len, size_t i, const std::string &key,
                       bool &found, size_t &vs, size_t &ve, JsonError &e) {
  found = false;
  size_t j = skip_ws(b, len, i + 1);
  if (j < len && b[j] == '}') return true;
  for (;;) {
    j = skip_ws(b, len, j);
    if (j >= len || b[j] != '"') return fail(e, j, "expected a string key");
    size_t key_start = j;
    if (!skip_string(b, len, j, j, e)) return false;
    const uint8_t *kraw = b + key_start + 1;
    size_t kn = j - 1 - (key_start + 1);
    j = skip_ws(b, len, j);
    if (j >= len || b[j] != ':') return fail(e, j, "expected `:` after object key");
    size_t val_start = skip_ws(b, len, j + 1);
    size_t val_end = 0;
    if (!skip_value(b, len, val_start, val_end, e)) return false;
    if (key_matches(kraw, kn, key)) {
      found = true;
      vs = val_start;
      ve = val_end;
    }
    j = skip_ws(b, len, val_end);
    if (j < len && b[j] == ',') {
      j++;
    } else if (j < len && b[j] == '}') {
      return true;
    } else {
      return fail(e, j, "expected `,` or `}`");
    }
  }
}

// json.rs:558-578
static bool array_get(const uint8_t *b, size_t len, size_t i, uint32_t idx, bool &found,
                      size_t &vs, size_t &ve, JsonError &e) {
  found = false;
  size_t j = skip_ws(b, len, i + 1);
  if (j < len && b[j] == ']') return true;
  uint32_t n = 0;
  for (;;) {
    size_t s = skip_ws(b, len, j);
    size_t en = 0;
    if (!skip_value(b, len, s, en, e)) return false;
    if (n == idx) {
      found = true;
      vs = s;
      ve = en;
      return true;
    }
    n++;
    j = skip_ws(b, len, en);
    if (j < len && b[j] == ',') {
      j++;
    } else if (j < len && b[j] == ']') {
      return true;
    } else {
      return fail(e, j, "expected `,` or `]`");
    }
  }
}

// json.rs:444-508
LookupRes lookup(const uint8_t *line, size_t len, const std::vector<Step> &steps, Slot &out,
                 std::string &msg) {
  size_t start = skip_ws(line, len, 0);
  JsonError e;
  if (start >= len) {
    msg = "empty value at byte 0";
    return LookupRes::Invalid;
  }
  Kind kind = kind_of(line, start);
  size_t end = len;
  if (steps.empty()) {
    if (!skip_value(line, len, start, end, e)) {
      msg = e.detail;
      return LookupRes::Invalid;
    }
  }
  for (const Step &st : steps) {
    if (kind == Kind::Missing || kind == Kind::Null) {
      out = missing_slot();
      return LookupRes::Found;
    }
    bool found = false;
    size_t s = 0, en = 0;
    if (!st.is_index) {
      if (kind != Kind::Obj) {
        msg = std::string("cannot index ") + type_name(kind) + " with \"" + st.key + "\"";
        return LookupRes::TypeError;
      }
      if (!object_get(line, len, start, st.key, found, s, en, e)) {
        msg = e.detail;
        return LookupRes::Invalid;
      }
    } else {
      if (kind != Kind::Arr) {
        msg = std::string("cannot index ") + type_name(kind) + " with number";
        return LookupRes::TypeError;
      }
      if (!array_get(line, len, start, st.index, found, s, en, e)) {
        msg = e.detail;
        return LookupRes::Invalid;
      }
    }
    if (!found) {
      out = missing_slot();
      return LookupRes::Found;
    }
    start = s;
    end = en;
    kind = kind_of(line, s);
  }
  out.kind = kind;
  out.p = line + start;
  out.n = end - start;
  return LookupRes::Found;
}

static void push_utf8(std::string &out, uint32_t cp) {
  if (cp < 0x80) {
    out.push_back((char)cp);
  } else if (cp < 0x800) {
    out.push_back((char)(0xC0 | (cp >> 6)));
    out.push_back((char)(0x80 | (cp & 0x3F)));
  } else if (cp < 0x10000) {
    out.push_back((char)(0xE0 | (cp >> 12)));
    out.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
    out.push_back((char)(0x80 | (cp & 0x3F)));
  } else {
    out.push_back((char)(0xF0 | (cp >> 18)));
    out.push_back((char)(0x80 | ((cp >> 12) & 0x3F)));
    out.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
    out.push_back((char)(0x80 | (cp & 0x3F)));
  }
}

// Rust's u32::from_str_radix(s, 16) on a 4-byte slice: an optional leading
// `+`, then hex digits only.
static bool hex4(const uint8_t *p, size_t avail, uint32_t &v) {
  if (avail < 4) return false;
  size_t k = 0;
  if (p[0] == '+') k = 1;
  if (k == 4) return false;
  v = 0;
  for (; k < 4; k++) {
    uint8_t c = p[k];
    uint32_t d;
    if (c >= '0' && c <= '9') d = c - '0';
    else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
    else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
    else return false;
    v = v * 16 + d;
  }
  return true;
}

// json.rs:594-654.  Invalid scalars (lone surrogates) decode to U+FFFD.
bool unescape_into(const uint8_t *raw, size_t n, std::string &out) {
  size_t i = 0;
  while (i < n) {
    if (raw[i] != '\\') {
      out.push_back((char)raw[i]);
      i++;
      continue;
    }
    if (i + 1 >= n) return false;
    uint8_t e = raw[i + 1];
    switch (e) {
      case '"': out.push_back('"'); break;
      case '\\': out.push_back('\\'); break;
      case '/': out.push_back('/'); break;
      case 'b': out.push_back('\x08'); break;
      case 'f': out.push_back('\x0c'); break;
      case 'n': out.push_back('\n'); break;
      case 'r': out.push_back('\r'); break;
      case 't': out.push_back('\t'); break;
      case 'u': {
        uint32_t cp = 0;
        if (i + 6 > n || !hex4(raw + i + 2, 4, cp)) return false;
        i += 6;
        if (cp >= 0xD800 && cp < 0xDC00 && i + 1 < n && raw[i] == '\\' && raw[i + 1] == 'u' &&
            i + 6 <= n) {
          uint32_t lo = 0;
          if (hex4(raw + i + 2, 4, lo) && lo >= 0xDC00 && lo < 0xE000) {
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
            i += 6;
          }
        }
        if (cp >= 0xD800 && cp < 0xE000) cp = 0xFFFD;  // char::from_u32 fails on surrogates
        push_utf8(out, cp);
        continue;
      }
      default:
        return false;
    }
    i += 2;
  }
  return true;
}

// json.rs:582-591
bool key_matches(const uint8_t *raw, size_t n, const std::string &decoded) {
  if (std::memchr(raw, '\\', n) == nullptr)
    return n == decoded.size() && std::memcmp(raw, decoded.data(), n) == 0;
  std::string buf;
  if (!unescape_into(raw, n, buf)) return false;
  return buf == decoded;
}

static int bytes_cmp(const uint8_t *a, size_t an, const uint8_t *b, size_t bn) {
  size_t m = an < bn ? an : bn;
  int c = m ? std::memcmp(a, b, m) : 0;
  if (c != 0) return c < 0 ? -1 : 1;
  if (an == bn) return 0;
  return an < bn ? -1 : 1;
}

static uint8_t slot_rank(const Slot &s) {  // json.rs:30-45
  switch (s.kind) {
    case Kind::Missing: case Kind::Null: return 0;
    case Kind::Bool: return (s.n == 4 && std::memcmp(s.p, "true", 4) == 0) ? 2 : 1;
    case Kind::Num: return 3;
    case Kind::Str: return 4;
    case Kind::Arr: return 5;
    default: return 6;
  }
}

uint8_t Literal::rank() const {
  switch (kind) {
    case LitKind::Null: return 0;
    case LitKind::False: return 1;
    case LitKind::True: return 2;
    case LitKind::Num: return 3;
    default: return 4;
  }
}

// json.rs:662-693.  Returns -1, 0, 1.
int compare(const Slot &s, const Literal &lit) {
  uint8_t lr = lit.rank(), sr = slot_rank(s);
  if (sr != lr) return sr < lr ? -1 : 1;
  switch (lit.kind) {
    case LitKind::Null: case LitKind::False: case LitKind::True: return 0;
    case LitKind::Num: {
      double v;
      if (!s.as_f64(v)) return 0;
      if (v < lit.num) return -1;
      if (v > lit.num) return 1;
      return 0;  // equal, or unordered (partial_cmp None => Equal)
    }
    default: {
      const uint8_t *inner = s.p + 1;
      size_t n = s.n - 2;
      const uint8_t *lp = (const uint8_t *)lit.str.data();
      if (std::memchr(inner, '\\', n) == nullptr) return bytes_cmp(inner, n, lp, lit.str.size());
      std::string buf;
      if (!unescape_into(inner, n, buf)) return 0;
      return bytes_cmp((const uint8_t *)buf.data(), buf.size(), lp, lit.str.size());
    }
  }
}

// ir.rs:66-76
bool cmp_accepts(CmpOp op, int o) {
  switch (op) {
    case CmpOp::Eq: return o == 0;
    case CmpOp::Ne: return o != 0;
    case CmpOp::Lt: return o < 0;
    case CmpOp::Le: return o <= 0;
    case CmpOp::Gt: return o > 0;
    default: return o >= 0;
  }
}

}  // namespace oracle
