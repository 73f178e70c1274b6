// TEST INFRASTRUCTURE -- the oracle's query front-end.
// Restates crates/warpjq-core/src/query/{lex.rs, parse.rs, ir.rs, mod.rs}
// and the QueryError rendering of error.rs.
#include "oracle.h"

#include <cerrno>
#include <cstdlib>
#include <cstring>

namespace oracle {

// ---------------------------------------------------------------------------
// IR helpers (ir.rs)
// ---------------------------------------------------------------------------

static bool is_bare_key(const std::string &k) {  // ir.rs:48-52
  if (k.empty() || (k[0] >= '0' && k[0] <= '9')) return false;
  for (unsigned char c : k)
    if (!(std::isalnum(c) || c == '_')) return false;
  return true;
}

// Rust's `{:?}` on a str: quoted, with \" \\ \n \r \t \0 and \u{..} for other
// control characters.
static std::string rust_debug_str(const std::string &s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      case 0: o += "\\0"; break;
      default:
        if (c < 0x20 || c == 0x7f) {
          char b[16];
          std::snprintf(b, sizeof b, "\\u{%x}", c);
          o += b;
        } else {
          o.push_back((char)c);
        }
    }
  }
  return o + "\"";
}

std::string Path::display() const {  // ir.rs:32-46
  if (steps.empty()) return ".";
  std::string o;
  for (const Step &s : steps) {
    if (s.is_index) {
      o += "[" + std::to_string(s.index) + "]";
    } else if (is_bare_key(s.key)) {
      o += "." + s.key;
    } else {
      o += "." + rust_debug_str(s.key);
    }
  }
  return o;
}

void Cond::visit_paths(std::vector<PathId> &out) const {  // ir.rs:128-137
  switch (tag) {
    case Cmp: case Truthy: out.push_back(path); break;
    case And: case Or: a->visit_paths(out); b->visit_paths(out); break;
    case Not: a->visit_paths(out); break;
  }
}

const char *agg_name(AggKind k) {
  switch (k) {
    case AggKind::Count: return "count";
    case AggKind::Sum: return "sum";
    case AggKind::Min: return "min";
    case AggKind::Max: return "max";
    default: return "avg";
  }
}

std::vector<PathId> Program::required_paths() const {  // ir.rs:206-234
  std::vector<PathId> ids, tmp;
  auto push = [&](PathId id) {
    for (PathId x : ids)
      if (x == id) return;
    ids.push_back(id);
  };
  if (filter) {
    filter->visit_paths(tmp);
    for (PathId p : tmp) push(p);
  }
  if (has_group) push(group_by);
  switch (output.tag) {
    case Output::Passthrough: break;
    case Output::PathOut: push(output.path); break;
    case Output::Project:
      for (auto &f : output.fields) push(f.second);
      break;
    case Output::Agg:
      if (output.has_arg) push(output.arg);
      break;
  }
  return ids;
}

bool Program::csv_headers(std::vector<std::string> &cols) const {  // ir.rs:237-251
  cols.clear();
  switch (output.tag) {
    case Output::Project:
      for (auto &f : output.fields) cols.push_back(f.first);
      return true;
    case Output::PathOut:
      cols.push_back(paths[output.path].display());
      return true;
    case Output::Agg:
      if (has_group) cols.push_back(paths[group_by].display());
      cols.push_back(agg_name(output.agg));
      return true;
    default:
      return false;
  }
}

// error.rs:36-49.  The caret column counts characters, not bytes.
std::string QueryError::render(const std::string &src) const {
  size_t col = 0;
  for (size_t i = 0; i < at && i < src.size(); i++)
    if (((unsigned char)src[i] & 0xC0) != 0x80) col++;
  std::string o = "invalid query: " + message + "\n  " + src + "\n  " + std::string(col, ' ') +
                  "^\n";
  if (!hint.empty()) o += "  help: " + hint;
  return o;
}

// ---------------------------------------------------------------------------
// Lexer (lex.rs)
// ---------------------------------------------------------------------------

namespace {

enum class T : uint8_t {
  Dot, Pipe, LParen, RParen, LBracket, RBracket, LBrace, RBrace, Colon, Comma, Op, Ident, Str,
  Num, Int, Eof
};

struct Tok {
  T t = T::Eof;
  CmpOp op = CmpOp::Eq;
  std::string s;
  double num = 0;
  int64_t i = 0;
  size_t at = 0;
};

// Rust's `{}` on an f64: shortest round-trip digits, never exponent form.
static std::string rust_display_f64(double v) {
  char buf[64];
  for (int prec = 1; prec <= 17; prec++) {
    std::snprintf(buf, sizeof buf, "%.*g", prec, v);
    if (std::strtod(buf, nullptr) == v) break;
  }
  // Expand any exponent form into positional notation.
  std::string s = buf;
  size_t e = s.find('e');
  if (e == std::string::npos) return s;
  char big[400];
  std::snprintf(big, sizeof big, "%.17f", v);
  std::string f = big;
  if (f.find('.') != std::string::npos) {
    while (!f.empty() && f.back() == '0') f.pop_back();
    if (!f.empty() && f.back() == '.') f.pop_back();
  }
  return f;
}

static std::string describe(const Tok &t) {  // lex.rs:27-46
  switch (t.t) {
    case T::Dot: return "`.`";
    case T::Pipe: return "`|`";
    case T::LParen: return "`(`";
    case T::RParen: return "`)`";
    case T::LBracket: return "`[`";
    case T::RBracket: return "`]`";
    case T::LBrace: return "`{`";
    case T::RBrace: return "`}`";
    case T::Colon: return "`:`";
    case T::Comma: return "`,`";
    case T::Op: {
      static const char *n[] = {"==", "!=", "<", "<=", ">", ">="};
      return std::string("`") + n[(int)t.op] + "`";
    }
    case T::Ident: return "`" + t.s + "`";
    case T::Str: return "string " + rust_debug_str(t.s);
    case T::Num: return "number `" + rust_display_f64(t.num) + "`";
    case T::Int: return "number `" + std::to_string(t.i) + "`";
    default: return "end of query";
  }
}

static bool ascii_ws(unsigned char c) {  // u8::is_ascii_whitespace
  return c == ' ' || c == '\t' || c == '\n' || c == '\x0c' || c == '\r';
}
static bool is_alpha(unsigned char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); }
static bool is_digit(unsigned char c) { return c >= '0' && c <= '9'; }
static bool is_alnum(unsigned char c) { return is_alpha(c) || is_digit(c); }

struct LexFail {
  size_t at;
  std::string msg;
};

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

// `&str::get(a..b)` is None when out of range or off a char boundary.
static bool str_get(const std::string &s, size_t a, size_t b) {
  if (b > s.size() || a > b) return false;
  auto boundary = [&](size_t k) {
    return k == s.size() || (((unsigned char)s[k]) & 0xC0) != 0x80;
  };
  return boundary(a) && boundary(b);
}

// u32::from_str_radix(text, 16): optional `+`, then at least one hex digit.
static bool from_hex(const std::string &s, size_t a, size_t b, uint32_t &v) {
  size_t k = a;
  if (k < b && s[k] == '+') k++;
  if (k == b) return false;
  uint64_t acc = 0;
  for (; k < b; k++) {
    unsigned char c = s[k];
    uint32_t d;
    if (is_digit(c)) d = c - '0';
    else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
    else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
    else return false;
    acc = acc * 16 + d;
  }
  v = (uint32_t)acc;
  return true;
}

// lex.rs:192-263
static bool lex_string(const std::string &src, size_t start, std::string &s, size_t &next,
                       LexFail &f) {
  size_t i = start + 1;
  while (i < src.size()) {
    unsigned char c = src[i];
    if (c == '"') {
      next = i + 1;
      return true;
    }
    if (c == '\\') {
      i++;
      if (i >= src.size()) {
        f = {start, "unterminated string"};
        return false;
      }
      unsigned char e = src[i];
      switch (e) {
        case '"': s.push_back('"'); break;
        case '\\': s.push_back('\\'); break;
        case '/': s.push_back('/'); break;
        case 'n': s.push_back('\n'); break;
        case 't': s.push_back('\t'); break;
        case 'r': s.push_back('\r'); break;
        case 'b': s.push_back('\x08'); break;
        case 'f': s.push_back('\x0c'); break;
        case 'u': {
          if (!str_get(src, i + 1, i + 5)) {
            f = {i, "truncated `\\u` escape"};
            return false;
          }
          uint32_t cp;
          if (!from_hex(src, i + 1, i + 5, cp)) {
            f = {i, "bad `\\u` escape"};
            return false;
          }
          i += 4;
          if (cp >= 0xD800 && cp < 0xDC00) {
            bool ok = i + 1 < src.size() && src[i + 1] == '\\' && i + 2 < src.size() &&
                      src[i + 2] == 'u';
            if (ok) {
              if (!str_get(src, i + 3, i + 7)) {
                f = {i, "truncated surrogate pair"};
                return false;
              }
              uint32_t lo;
              if (!from_hex(src, i + 3, i + 7, lo)) {
                f = {i, "bad surrogate pair"};
                return false;
              }
              if (lo >= 0xDC00 && lo < 0xE000) {
                i += 6;
                push_utf8(s, 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00));
              } else {
                push_utf8(s, 0xFFFD);
              }
            } else {
              push_utf8(s, 0xFFFD);
            }
          } else {
            if ((cp >= 0xD800 && cp < 0xE000) || cp > 0x10FFFF) cp = 0xFFFD;
            push_utf8(s, cp);
          }
          break;
        }
        default:
          f = {i, std::string("unknown escape `\\") + (char)e + "`"};
          return false;
      }
      i++;
      continue;
    }
    // Copy one whole UTF-8 sequence.
    size_t n = 1;
    if (c >= 0xF0) n = 4;
    else if (c >= 0xE0) n = 3;
    else if (c >= 0xC0) n = 2;
    s.append(src, i, n);
    i += n;
  }
  f = {start, "unterminated string"};
  return false;
}

// lex.rs:265-317
static bool lex_number(const std::string &src, size_t start, Tok &t, size_t &next, LexFail &f) {
  size_t i = start;
  if (src[i] == '-') i++;
  size_t int_start = i;
  while (i < src.size() && is_digit(src[i])) i++;
  if (i == int_start) {
    f = {start, "expected a number"};
    return false;
  }
  bool is_float = false;
  if (i < src.size() && src[i] == '.') {
    is_float = true;
    i++;
    while (i < src.size() && is_digit(src[i])) i++;
  }
  if (i < src.size() && (src[i] == 'e' || src[i] == 'E')) {
    is_float = true;
    i++;
    if (i < src.size() && (src[i] == '+' || src[i] == '-')) i++;
    size_t es = i;
    while (i < src.size() && is_digit(src[i])) i++;
    if (i == es) {
      f = {start, "number has no digits in its exponent"};
      return false;
    }
  }
  std::string text = src.substr(start, i - start);
  if (!is_float) {
    errno = 0;
    char *endp = nullptr;
    long long v = std::strtoll(text.c_str(), &endp, 10);
    if (errno == 0 && endp && *endp == 0) {
      t.t = T::Int;
      t.i = v;
      next = i;
      return true;
    }
  }
  t.t = T::Num;
  t.num = std::strtod(text.c_str(), nullptr);
  next = i;
  return true;
}

// lex.rs:56-188
static bool lex(const std::string &src, std::vector<Tok> &out, LexFail &f) {
  size_t i = 0;
  while (i < src.size()) {
    unsigned char c = src[i];
    if (ascii_ws(c)) {
      i++;
      continue;
    }
    if (c == '#') {
      while (i < src.size() && src[i] != '\n') i++;
      continue;
    }
    Tok t;
    t.at = i;
    switch (c) {
      case '.': t.t = T::Dot; i++; break;
      case '|': t.t = T::Pipe; i++; break;
      case '(': t.t = T::LParen; i++; break;
      case ')': t.t = T::RParen; i++; break;
      case '[': t.t = T::LBracket; i++; break;
      case ']': t.t = T::RBracket; i++; break;
      case '{': t.t = T::LBrace; i++; break;
      case '}': t.t = T::RBrace; i++; break;
      case ':': t.t = T::Colon; i++; break;
      case ',': t.t = T::Comma; i++; break;
      case '=':
        if (i + 1 < src.size() && src[i + 1] == '=') {
          t.t = T::Op; t.op = CmpOp::Eq; i += 2;
        } else {
          f = {i, "`=` is assignment in jq and is not supported; did you mean `==`?"};
          return false;
        }
        break;
      case '!':
        if (i + 1 < src.size() && src[i + 1] == '=') {
          t.t = T::Op; t.op = CmpOp::Ne; i += 2;
        } else {
          f = {i, "expected `!=`"};
          return false;
        }
        break;
      case '<':
        t.t = T::Op;
        if (i + 1 < src.size() && src[i + 1] == '=') { t.op = CmpOp::Le; i += 2; }
        else { t.op = CmpOp::Lt; i++; }
        break;
      case '>':
        t.t = T::Op;
        if (i + 1 < src.size() && src[i + 1] == '=') { t.op = CmpOp::Ge; i += 2; }
        else { t.op = CmpOp::Gt; i++; }
        break;
      case '"': {
        size_t next;
        t.t = T::Str;
        if (!lex_string(src, i, t.s, next, f)) return false;
        i = next;
        break;
      }
      default:
        if (c == '-' || is_digit(c)) {
          size_t next;
          if (!lex_number(src, i, t, next, f)) return false;
          i = next;
        } else if (is_alpha(c) || c == '_') {
          size_t st = i;
          while (i < src.size() && (is_alnum(src[i]) || src[i] == '_')) i++;
          t.t = T::Ident;
          t.s = src.substr(st, i - st);
        } else {
          // Rust prints `c as char`, i.e. the byte as a Latin-1 character.
          std::string ch;
          if (c < 0x80) ch.push_back((char)c);
          else push_utf8(ch, c);
          f = {i, "unexpected character `" + ch + "`"};
          return false;
        }
    }
    out.push_back(std::move(t));
  }
  Tok eof;
  eof.t = T::Eof;
  eof.at = src.size();
  out.push_back(eof);
  return true;
}

// ---------------------------------------------------------------------------
// Parser (parse.rs)
// ---------------------------------------------------------------------------

struct Unsupported { const char *name, *why; };
static const Unsupported KNOWN_UNSUPPORTED[] = {  // parse.rs:35-57
    {"reduce", "`reduce` is not in the v0.1 subset"},
    {"foreach", "`foreach` is not in the v0.1 subset"},
    {"def", "user-defined functions are not in the v0.1 subset"},
    {"if", "`if/then/else` is not in the v0.1 subset; use `select(...)`"},
    {"try", "`try/catch` is not in the v0.1 subset"},
    {"test", "regex (`test`) is on the roadmap, not in v0.1"},
    {"match", "regex (`match`) is on the roadmap, not in v0.1"},
    {"map", "`map` is not in the v0.1 subset"},
    {"keys", "`keys` is not in the v0.1 subset"},
    {"length", "`length` is not in the v0.1 subset; `count` counts lines"},
    {"tostring", "type coercions are not in the v0.1 subset"},
    {"tonumber", "type coercions are not in the v0.1 subset"},
    {"sort_by", "`sort_by` is not in the v0.1 subset"},
    {"unique", "`unique` is not in the v0.1 subset"},
    {"add", "`add` is not in the v0.1 subset; use `sum(.field)`"},
};
static const char *kLimitsHint = "see the Limitations section of the README for the full v0.1 subset";

static const char *find_unsupported(const std::string &w) {
  for (auto &u : KNOWN_UNSUPPORTED)
    if (w == u.name) return u.why;
  return nullptr;
}

// parse.rs:80-126
static bool unsupported_leading_keyword(const std::string &src, QueryError &err) {
  std::vector<std::pair<size_t, size_t>> stages;  // (start, end)
  size_t start = 0;
  int depth = 0;
  bool in_str = false;
  for (size_t i = 0; i < src.size(); i++) {
    char c = src[i];
    if (c == '\\' && in_str) {
      i++;
      continue;
    }
    if (c == '"') in_str = !in_str;
    else if (!in_str && (c == '(' || c == '[' || c == '{')) depth++;
    else if (!in_str && (c == ')' || c == ']' || c == '}')) depth--;
    else if (c == '|' && !in_str && depth == 0) {
      stages.push_back({start, i});
      start = i + 1;
    }
  }
  stages.push_back({start, src.size()});
  for (auto &st : stages) {
    size_t k = st.first;
    // str::trim_start trims Unicode whitespace; ASCII whitespace covers queries.
    while (k < st.second &&
           (ascii_ws((unsigned char)src[k]) || src[k] == '\x0b'))
      k++;
    size_t w = k;
    while (w < st.second && (is_alnum(src[w]) || src[w] == '_')) w++;
    if (w == k) continue;
    const char *why = find_unsupported(src.substr(k, w - k));
    if (why) {
      err.at = k;
      err.message = why;
      err.hint = kLimitsHint;
      return true;
    }
  }
  return false;
}

static const unsigned MAX_COND_DEPTH = 64;  // parse.rs:135

struct ParseFail {};

struct Parser {
  const std::string &src;
  std::vector<Tok> toks;
  size_t pos = 0;
  std::vector<Path> paths;
  unsigned depth = 0;
  QueryError err;

  explicit Parser(const std::string &s) : src(s) {}

  const Tok &peek() const { return toks[pos]; }
  const Tok &peek_at(size_t n) const {
    size_t k = pos + n;
    if (k > toks.size() - 1) k = toks.size() - 1;
    return toks[k];
  }
  size_t at() const { return toks[pos].at; }
  Tok bump() {
    Tok t = toks[pos];
    if (pos + 1 < toks.size()) pos++;
    return t;
  }
  bool eat(T t) {
    if (peek().t == t) {
      bump();
      return true;
    }
    return false;
  }
  [[noreturn]] void fail(size_t a, const std::string &m, const std::string &h = "") {
    err.at = a > src.size() ? src.size() : a;
    err.message = m;
    err.hint = h;
    throw ParseFail{};
  }
  void expect(T t, const std::string &ctx) {
    if (eat(t)) return;
    Tok want;
    want.t = t;
    fail(at(), "expected " + describe(want) + " " + ctx + ", found " + describe(peek()));
  }
  bool peek_keyword(const char *kw) const { return peek().t == T::Ident && peek().s == kw; }

  PathId intern(const Path &p) {  // parse.rs:198-204
    for (size_t i = 0; i < paths.size(); i++)
      if (paths[i] == p) return (PathId)i;
    paths.push_back(p);
    return (PathId)(paths.size() - 1);
  }

  enum StageKind { SFilter, SGroup, SOutput };

  static const char *describe_output(const Output &o) {  // parse.rs:639-646
    switch (o.tag) {
      case Output::Passthrough: return "`.`";
      case Output::PathOut: return "a field path";
      case Output::Project: return "an object projection";
      default: return "an aggregate";
    }
  }

  // parse.rs:208-289
  void program(Program &prog) {
    std::unique_ptr<Cond> filter;
    bool has_group = false;
    PathId group = 0;
    bool has_output = false;
    Output output;
    size_t output_at = 0;
    for (;;) {
      size_t stage_at = at();
      std::unique_ptr<Cond> c;
      PathId g = 0;
      Output o;
      StageKind k = stage(c, g, o);
      if (k == SFilter) {
        if (!filter) {
          filter = std::move(c);
        } else {
          auto n = std::make_unique<Cond>();
          n->tag = Cond::And;
          n->a = std::move(filter);
          n->b = std::move(c);
          filter = std::move(n);
        }
      } else if (k == SGroup) {
        if (has_group) fail(stage_at, "only one `group_by` per query is supported in v0.1");
        if (has_output)
          fail(stage_at, "`group_by` must come before the output stage",
               "write `group_by(.host) | count`, not `count | group_by(.host)`");
        has_group = true;
        group = g;
      } else {
        if (has_output)
          fail(stage_at, std::string("a second output stage follows ") + describe_output(output) +
                             "; v0.1 supports one output stage per query");
        output = std::move(o);
        has_output = true;
        output_at = stage_at;
      }
      if (!eat(T::Pipe)) break;
    }
    if (peek().t != T::Eof) fail(at(), "unexpected " + describe(peek()));
    if (!has_output) output.tag = Output::Passthrough;
    if (has_group && output.tag != Output::Agg)
      fail(output_at > 1 ? output_at : 1, "`group_by` must be followed by an aggregate",
           "try `group_by(.host) | count` or `group_by(.host) | sum(.bytes)`");
    prog.paths = std::move(paths);
    prog.filter = std::move(filter);
    prog.has_group = has_group;
    prog.group_by = group;
    prog.output = std::move(output);
    prog.source = src;
  }

  // parse.rs:291-384
  StageKind stage(std::unique_ptr<Cond> &c, PathId &g, Output &o) {
    size_t a = at();
    if (peek().t == T::Ident) {
      std::string name = peek().s;
      if (const char *why = find_unsupported(name)) fail(a, why, kLimitsHint);
      if (name == "select") {
        bump();
        expect(T::LParen, "after `select`");
        c = cond();
        expect(T::RParen, "to close `select(`");
        return SFilter;
      }
      if (name == "group_by") {
        bump();
        expect(T::LParen, "after `group_by`");
        Path p = path();
        if (p.steps.empty())
          fail(a, "`group_by(.)` would group by the whole line",
               "group by a field, e.g. `group_by(.status)`");
        g = intern(p);
        expect(T::RParen, "to close `group_by(`");
        return SGroup;
      }
      if (name == "count") {
        bump();
        if (peek().t == T::LParen)
          fail(at(), "`count` takes no argument",
               "write `count`, or `sum(.field)` to total a field");
        o.tag = Output::Agg;
        o.agg = AggKind::Count;
        o.has_arg = false;
        return SOutput;
      }
      if (name == "sum" || name == "min" || name == "max" || name == "avg") {
        bump();
        AggKind kind = name == "sum" ? AggKind::Sum
                       : name == "min" ? AggKind::Min
                       : name == "max" ? AggKind::Max
                                       : AggKind::Avg;
        expect(T::LParen, "after `" + name + "`");
        Path p = path();
        if (p.steps.empty())
          fail(a, "`" + name + "(.)` has no field to aggregate", "try `" + name + "(.bytes)`");
        PathId id = intern(p);
        expect(T::RParen, "to close `" + name + "(`");
        o.tag = Output::Agg;
        o.agg = kind;
        o.has_arg = true;
        o.arg = id;
        return SOutput;
      }
      fail(a, "unknown function `" + name + "`",
           "v0.1 supports: select, group_by, count, sum, min, max, avg");
    }
    if (peek().t == T::LBrace) {
      object(o);
      return SOutput;
    }
    Path p = path();
    if (p.steps.empty()) {
      o.tag = Output::Passthrough;
      return SOutput;
    }
    o.tag = Output::PathOut;
    o.path = intern(p);
    return SOutput;
  }

  // parse.rs:386-439
  void object(Output &o) {
    expect(T::LBrace, "to start an object");
    std::vector<std::pair<std::string, PathId>> fields;
    for (;;) {
      if (peek().t == T::RBrace) break;
      size_t key_at = at();
      Tok kt = bump();
      std::string key;
      if (kt.t == T::Ident || kt.t == T::Str) key = kt.s;
      else fail(key_at, "expected an object key, found " + describe(kt));
      PathId pid;
      if (eat(T::Colon)) {
        Path p = path();
        if (p.steps.empty())
          fail(key_at, "an object value of `.` would embed the whole line",
               "name a field, e.g. `{msg: .message}`");
        pid = intern(p);
      } else {
        Path p;
        Step s;
        s.key = key;
        p.steps.push_back(s);
        pid = intern(p);
      }
      for (auto &f : fields)
        if (f.first == key) fail(key_at, "duplicate key `" + key + "` in projection");
      fields.push_back({key, pid});
      if (!eat(T::Comma)) break;
    }
    expect(T::RBrace, "to close the object");
    if (fields.empty()) fail(at(), "empty projection `{}` produces no output");
    o.tag = Output::Project;
    o.fields = std::move(fields);
  }

  std::unique_ptr<Cond> cond() {  // parse.rs:443-451
    auto lhs = and_expr();
    while (peek_keyword("or")) {
      bump();
      auto rhs = and_expr();
      auto n = std::make_unique<Cond>();
      n->tag = Cond::Or;
      n->a = std::move(lhs);
      n->b = std::move(rhs);
      lhs = std::move(n);
    }
    return lhs;
  }

  std::unique_ptr<Cond> and_expr() {  // parse.rs:453-461
    auto lhs = term();
    while (peek_keyword("and")) {
      bump();
      auto rhs = term();
      auto n = std::make_unique<Cond>();
      n->tag = Cond::And;
      n->a = std::move(lhs);
      n->b = std::move(rhs);
      lhs = std::move(n);
    }
    return lhs;
  }

  std::unique_ptr<Cond> term() {  // parse.rs:463-520
    size_t a = at();
    std::unique_ptr<Cond> base;
    if (eat(T::LParen)) {
      depth++;
      if (depth > MAX_COND_DEPTH)
        fail(a, "conditions may not nest more than " + std::to_string(MAX_COND_DEPTH) + " deep");
      base = cond();
      expect(T::RParen, "to close the group");
      depth--;
    } else {
      if (peek().t == T::Ident) {
        std::string name = peek().s;
        fail(a, "expected a field path, found `" + name + "`", "did you mean `." + name + "`?");
      }
      Path p = path();
      if (p.steps.empty())
        fail(a, "`.` cannot be used as a condition in v0.1",
             "compare a field, e.g. `select(.status == 500)`");
      PathId id = intern(p);
      base = std::make_unique<Cond>();
      if (peek().t == T::Op) {
        CmpOp op = peek().op;
        bump();
        base->tag = Cond::Cmp;
        base->path = id;
        base->op = op;
        base->lit = literal();
      } else {
        base->tag = Cond::Truthy;
        base->path = id;
      }
    }
    while (peek().t == T::Pipe && peek_at(1).t == T::Ident && peek_at(1).s == "not") {
      bump();
      bump();
      auto n = std::make_unique<Cond>();
      n->tag = Cond::Not;
      n->a = std::move(base);
      base = std::move(n);
    }
    return base;
  }

  Literal literal() {  // parse.rs:522-561
    size_t a = at();
    Tok t = bump();
    Literal l;
    switch (t.t) {
      case T::Num: l.kind = LitKind::Num; l.num = t.num; return l;
      case T::Int: l.kind = LitKind::Num; l.num = (double)t.i; return l;
      case T::Str: l.kind = LitKind::Str; l.str = t.s; return l;
      case T::Ident:
        if (t.s == "true") { l.kind = LitKind::True; return l; }
        if (t.s == "false") { l.kind = LitKind::False; return l; }
        if (t.s == "null") { l.kind = LitKind::Null; return l; }
        fail(a, "expected a literal value, found `" + t.s + "`",
             "the right-hand side of a comparison must be a number, string, `true`, `false`, "
             "or `null`. Field-to-field comparison is not in v0.1");
      case T::Dot:
        fail(a, "field-to-field comparison is not supported in v0.1",
             "compare against a constant, e.g. `select(.status == 500)`");
      default:
        fail(a, "expected a literal value, found " + describe(t));
    }
  }

  Path path() {  // parse.rs:565-630
    size_t a = at();
    if (peek().t != T::Dot)
      fail(a, "expected a field path, found " + describe(peek()),
           "paths start with `.`, e.g. `.status` or `.req.path`");
    bump();
    Path p;
    for (;;) {
      const Tok &t = peek();
      if (t.t == T::Ident || t.t == T::Str) {
        Step s;
        s.key = t.s;
        bump();
        p.steps.push_back(s);
      } else if (t.t == T::LBracket) {
        bump();
        size_t idx_at = at();
        Tok it = bump();
        if (it.t == T::Int && it.i >= 0) {
          Step s;
          s.is_index = true;
          s.index = (uint32_t)it.i;  // `i as u32`
          p.steps.push_back(s);
        } else if (it.t == T::Int) {
          fail(idx_at, "negative array indices are not supported in v0.1");
        } else {
          fail(idx_at, "expected an array index, found " + describe(it),
               "slices (`.[1:3]`) and iteration (`.[]`) are not in v0.1");
        }
        expect(T::RBracket, "to close the index");
      } else {
        break;
      }
      if (peek().t == T::Dot) {
        T n = peek_at(1).t;
        if (n == T::Ident || n == T::Str || n == T::LBracket) bump();
        else break;
      } else if (peek().t != T::LBracket) {
        break;
      }
    }
    return p;
  }
};

}  // namespace

bool parse_query(const std::string &src, Program &out, QueryError &err) {
  if (unsupported_leading_keyword(src, err)) return false;
  Parser p(src);
  LexFail lf;
  if (!lex(src, p.toks, lf)) {
    err.at = lf.at > src.size() ? src.size() : lf.at;
    err.message = lf.msg;
    err.hint.clear();
    return false;
  }
  try {
    p.program(out);
  } catch (ParseFail &) {
    err = p.err;
    return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Flat tables (query/mod.rs:15-198)
// ---------------------------------------------------------------------------

uint32_t key_hash(const uint8_t *p, size_t n) {
  uint32_t h = 0x811c9dc5u;
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 0x01000193u;
  }
  return h;
}

static uint32_t push_blob(FlatProgram &f, const std::string &s, uint32_t &len) {
  uint32_t off = (uint32_t)f.blob.size();
  f.blob.insert(f.blob.end(), s.begin(), s.end());
  len = (uint32_t)s.size();
  return off;
}

static uint32_t flatten_cond(const Cond &c, FlatProgram &f) {  // query/mod.rs:141-198
  switch (c.tag) {
    case Cond::Cmp: {
      FlatCmp fc{};
      fc.path = c.path;
      fc.op = (uint32_t)c.op;
      switch (c.lit.kind) {
        case LitKind::Null: fc.lit_kind = 0; break;
        case LitKind::False: fc.lit_kind = 1; break;
        case LitKind::True: fc.lit_kind = 2; break;
        case LitKind::Num: fc.lit_kind = 3; fc.lit_num = c.lit.num; break;
        case LitKind::Str: fc.lit_kind = 4; fc.lit_off = push_blob(f, c.lit.str, fc.lit_len); break;
      }
      uint32_t idx = (uint32_t)f.cmps.size();
      f.cmps.push_back(fc);
      f.cond_rpn.push_back({0, idx});
      return 1;
    }
    case Cond::Truthy:
      f.cond_rpn.push_back({1, c.path});
      return 1;
    case Cond::Not: {
      uint32_t d = flatten_cond(*c.a, f);
      f.cond_rpn.push_back({4, 0});
      return d;
    }
    default: {
      uint32_t da = flatten_cond(*c.a, f);
      uint32_t db = flatten_cond(*c.b, f);
      f.cond_rpn.push_back({c.tag == Cond::And ? 2u : 3u, 0});
      return da > db + 1 ? da : db + 1;
    }
  }
}

FlatProgram flatten(const Program &p) {
  FlatProgram f;
  for (const Path &path : p.paths) {
    uint32_t off = (uint32_t)f.steps.size();
    for (const Step &s : path.steps) {
      FlatProgram::S gs{};
      if (s.is_index) {
        gs.kind = 1;
        gs.index = s.index;
      } else {
        gs.kind = 0;
        gs.key_off = push_blob(f, s.key, gs.key_len);
        gs.key_hash = key_hash((const uint8_t *)s.key.data(), s.key.size());
      }
      f.steps.push_back(gs);
    }
    f.paths.push_back({off, (uint32_t)path.steps.size()});
  }
  if (p.filter) f.cond_stack_depth = flatten_cond(*p.filter, f);
  return f;
}

}  // namespace oracle
