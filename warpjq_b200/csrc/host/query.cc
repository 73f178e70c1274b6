// jq-subset front-end for the GPU backend's host (see query.h).
#include "query.h"

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace wjqh {

namespace {

bool ascii_ws(unsigned char c) { return c == ' ' || c == '\t' || c == '\n' || c == 0x0C || c == '\r'; }
bool alpha(unsigned char c) { return (c | 0x20) >= 'a' && (c | 0x20) <= 'z'; }
bool digit(unsigned char c) { return c >= '0' && c <= '9'; }
bool alnum(unsigned char c) { return alpha(c) || digit(c); }

void utf8(std::string &o, uint32_t cp) {
  if (cp < 0x80) {
    o += (char)cp;
  } else if (cp < 0x800) {
    o += (char)(0xC0 | cp >> 6);
    o += (char)(0x80 | (cp & 0x3F));
  } else if (cp < 0x10000) {
    o += (char)(0xE0 | cp >> 12);
    o += (char)(0x80 | ((cp >> 6) & 0x3F));
    o += (char)(0x80 | (cp & 0x3F));
  } else {
    o += (char)(0xF0 | cp >> 18);
    o += (char)(0x80 | ((cp >> 12) & 0x3F));
    o += (char)(0x80 | ((cp >> 6) & 0x3F));
    o += (char)(0x80 | (cp & 0x3F));
  }
}

// Rust `{:?}` of a string, used in path display and token descriptions.
std::string debug_str(const std::string &s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    if (c == '"') o += "\\\"";
    else if (c == '\\') o += "\\\\";
    else if (c == '\n') o += "\\n";
    else if (c == '\r') o += "\\r";
    else if (c == '\t') o += "\\t";
    else if (c == 0) o += "\\0";
    else if (c < 0x20 || c == 0x7F) {
      char b[16];
      snprintf(b, sizeof b, "\\u{%x}", c);
      o += b;
    } else o += (char)c;
  }
  return o + "\"";
}

// ---- tokens (query/lex.rs) ------------------------------------------------

enum class TK : uint8_t { Dot, Pipe, LP, RP, LB, RB, LC, RC, Colon, Comma, Op, Ident, Str, Num, Int, Eof };

struct Token {
  TK k = TK::Eof;
  uint32_t op = 0;
  std::string s;
  double num = 0;
  long long iv = 0;
  size_t at = 0;
};

std::string f64_display(double v) {
  char b[64];
  for (int p = 1; p <= 17; p++) {
    snprintf(b, sizeof b, "%.*g", p, v);
    if (strtod(b, nullptr) == v) break;
  }
  if (!strchr(b, 'e')) return b;
  char big[400];
  snprintf(big, sizeof big, "%.17f", v);
  std::string f = big;
  while (!f.empty() && f.back() == '0') f.pop_back();
  if (!f.empty() && f.back() == '.') f.pop_back();
  return f;
}

std::string describe(const Token &t) {
  static const char *ops[] = {"==", "!=", "<", "<=", ">", ">="};
  switch (t.k) {
    case TK::Dot: return "`.`";
    case TK::Pipe: return "`|`";
    case TK::LP: return "`(`";
    case TK::RP: return "`)`";
    case TK::LB: return "`[`";
    case TK::RB: return "`]`";
    case TK::LC: return "`{`";
    case TK::RC: return "`}`";
    case TK::Colon: return "`:`";
    case TK::Comma: return "`,`";
    case TK::Op: return std::string("`") + ops[t.op] + "`";
    case TK::Ident: return "`" + t.s + "`";
    case TK::Str: return "string " + debug_str(t.s);
    case TK::Num: return "number `" + f64_display(t.num) + "`";
    case TK::Int: return "number `" + std::to_string(t.iv) + "`";
    default: return "end of query";
  }
}

struct Fail {
  size_t at;
  std::string msg, hint;
};

bool char_boundary(const std::string &s, size_t k) {
  return k == s.size() || (k < s.size() && ((unsigned char)s[k] & 0xC0) != 0x80);
}

// u32::from_str_radix(_, 16) over s[a, b): optional '+', then hex digits.
bool hexnum(const std::string &s, size_t a, size_t b, uint32_t &v) {
  if (b > s.size() || !char_boundary(s, a) || !char_boundary(s, b)) return false;
  if (a < b && s[a] == '+') a++;
  if (a >= b) return false;
  unsigned long long x = 0;
  for (size_t i = a; i < b; i++) {
    unsigned char c = s[i];
    int d = digit(c) ? c - '0' : (c | 0x20) >= 'a' && (c | 0x20) <= 'f' ? (c | 0x20) - 'a' + 10 : -1;
    if (d < 0) return false;
    x = x * 16 + d;
  }
  v = (uint32_t)x;
  return true;
}

void lex_string(const std::string &src, size_t start, Token &t, size_t &next) {
  size_t i = start + 1;
  std::string &s = t.s;
  while (i < src.size()) {
    unsigned char c = src[i];
    if (c == '"') {
      next = i + 1;
      return;
    }
    if (c == '\\') {
      if (++i >= src.size()) throw Fail{start, "unterminated string", ""};
      unsigned char e = src[i];
      if (e == 'u') {
        uint32_t cp;
        if (!(i + 5 <= src.size() && char_boundary(src, i + 1) && char_boundary(src, i + 5)))
          throw Fail{i, "truncated `\\u` escape", ""};
        if (!hexnum(src, i + 1, i + 5, cp)) throw Fail{i, "bad `\\u` escape", ""};
        i += 4;
        if (cp >= 0xD800 && cp < 0xDC00) {
          if (i + 2 < src.size() && src[i + 1] == '\\' && src[i + 2] == 'u') {
            if (!(i + 7 <= src.size() && char_boundary(src, i + 3) && char_boundary(src, i + 7)))
              throw Fail{i, "truncated surrogate pair", ""};
            uint32_t lo;
            if (!hexnum(src, i + 3, i + 7, lo)) throw Fail{i, "bad surrogate pair", ""};
            if (lo >= 0xDC00 && lo < 0xE000) {
              i += 6;
              utf8(s, 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00));
            } else {
              utf8(s, 0xFFFD);
            }
          } else {
            utf8(s, 0xFFFD);
          }
        } else {
          utf8(s, (cp >= 0xD800 && cp < 0xE000) ? 0xFFFD : cp);
        }
      } else {
        const char *from = "\"\\/ntrbf", *to = "\"\\/\n\t\r\b\f";
        const char *hit = strchr(from, e);
        if (!hit || !e) throw Fail{i, std::string("unknown escape `\\") + (char)e + "`", ""};
        s += to[hit - from];
      }
      i++;
      continue;
    }
    size_t n = c >= 0xF0 ? 4 : c >= 0xE0 ? 3 : c >= 0xC0 ? 2 : 1;
    s.append(src, i, n);
    i += n;
  }
  throw Fail{start, "unterminated string", ""};
}

void lex_number(const std::string &src, size_t start, Token &t, size_t &next) {
  size_t i = start;
  if (src[i] == '-') i++;
  size_t is = i;
  while (i < src.size() && digit(src[i])) i++;
  if (i == is) throw Fail{start, "expected a number", ""};
  bool flt = false;
  if (i < src.size() && src[i] == '.') {
    flt = true;
    i++;
    while (i < src.size() && digit(src[i])) i++;
  }
  if (i < src.size() && (src[i] | 0x20) == 'e') {
    flt = true;
    i++;
    if (i < src.size() && (src[i] == '+' || src[i] == '-')) i++;
    size_t es = i;
    while (i < src.size() && digit(src[i])) i++;
    if (i == es) throw Fail{start, "number has no digits in its exponent", ""};
  }
  std::string text = src.substr(start, i - start);
  next = i;
  if (!flt) {
    errno = 0;
    char *e = nullptr;
    long long v = strtoll(text.c_str(), &e, 10);
    if (!errno && e && !*e) {
      t.k = TK::Int;
      t.iv = v;
      return;
    }
  }
  t.k = TK::Num;
  t.num = strtod(text.c_str(), nullptr);
}

std::vector<Token> lex(const std::string &src) {
  std::vector<Token> out;
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
    Token t;
    t.at = i;
    static const char *punct = ".|()[]{}:,";
    const char *hit = c ? strchr(punct, c) : nullptr;
    if (hit) {
      t.k = (TK)(hit - punct);
      i++;
    } else if (c == '=' || c == '!' || c == '<' || c == '>') {
      bool eq = i + 1 < src.size() && src[i + 1] == '=';
      if (c == '=' && !eq) throw Fail{i, "`=` is assignment in jq and is not supported; did you mean `==`?", ""};
      if (c == '!' && !eq) throw Fail{i, "expected `!=`", ""};
      t.k = TK::Op;
      t.op = c == '=' ? WARPJQ_OP_EQ : c == '!' ? WARPJQ_OP_NE : c == '<' ? (eq ? WARPJQ_OP_LE : WARPJQ_OP_LT)
                                                                    : (eq ? WARPJQ_OP_GE : WARPJQ_OP_GT);
      i += eq ? 2 : 1;
    } else if (c == '"') {
      t.k = TK::Str;
      lex_string(src, i, t, i);
    } else if (c == '-' || digit(c)) {
      lex_number(src, i, t, i);
    } else if (alpha(c) || c == '_') {
      size_t s = i;
      while (i < src.size() && (alnum(src[i]) || src[i] == '_')) i++;
      t.k = TK::Ident;
      t.s = src.substr(s, i - s);
    } else {
      std::string ch;
      if (c < 0x80) ch += (char)c;
      else utf8(ch, c);
      throw Fail{i, "unexpected character `" + ch + "`", ""};
    }
    out.push_back(std::move(t));
  }
  Token eof;
  eof.at = src.size();
  out.push_back(eof);
  return out;
}

// ---- parser (query/parse.rs) ---------------------------------------------

const char *const kUnsupported[][2] = {
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
const char *kSubsetHint = "see the Limitations section of the README for the full v0.1 subset";

const char *unsupported(const std::string &w) {
  for (auto &u : kUnsupported)
    if (w == u[0]) return u[1];
  return nullptr;
}

// Names an unsupported construct at the start of any top-level pipeline
// stage before lexing can trip over its syntax (parse.rs:80-126).
void check_leading_keywords(const std::string &src) {
  size_t start = 0;
  int depth = 0;
  bool in_str = false;
  std::vector<std::pair<size_t, size_t>> stages;
  for (size_t i = 0; i < src.size(); i++) {
    char c = src[i];
    if (in_str && c == '\\') {
      i++;
      continue;
    }
    if (c == '"') in_str = !in_str;
    else if (!in_str && strchr("([{", c) && c) depth++;
    else if (!in_str && strchr(")]}", c) && c) depth--;
    else if (!in_str && c == '|' && depth == 0) {
      stages.push_back({start, i});
      start = i + 1;
    }
  }
  stages.push_back({start, src.size()});
  for (auto &st : stages) {
    size_t k = st.first;
    while (k < st.second && (ascii_ws(src[k]) || src[k] == 0x0B)) k++;
    size_t w = k;
    while (w < st.second && (alnum(src[w]) || src[w] == '_')) w++;
    if (w == k) continue;
    if (const char *why = unsupported(src.substr(k, w - k))) throw Fail{k, why, kSubsetHint};
  }
}

struct Parser {
  const std::string &src;
  std::vector<Token> tk;
  size_t pos = 0;
  std::vector<Path> paths;
  unsigned depth = 0;

  const Token &peek(size_t n = 0) const { return tk[std::min(pos + n, tk.size() - 1)]; }
  size_t at() const { return tk[pos].at; }
  Token bump() {
    Token t = tk[pos];
    if (pos + 1 < tk.size()) pos++;
    return t;
  }
  bool eat(TK k) {
    if (peek().k != k) return false;
    bump();
    return true;
  }
  void expect(TK k, const std::string &ctx) {
    if (eat(k)) return;
    Token w;
    w.k = k;
    throw Fail{at(), "expected " + describe(w) + " " + ctx + ", found " + describe(peek()), ""};
  }
  bool keyword(const char *kw) const { return peek().k == TK::Ident && peek().s == kw; }
  uint16_t intern(const Path &p) {
    for (size_t i = 0; i < paths.size(); i++)
      if (paths[i] == p) return (uint16_t)i;
    paths.push_back(p);
    return (uint16_t)(paths.size() - 1);
  }

  Path path() {
    size_t a = at();
    if (peek().k != TK::Dot)
      throw Fail{a, "expected a field path, found " + describe(peek()),
                 "paths start with `.`, e.g. `.status` or `.req.path`"};
    bump();
    Path p;
    for (;;) {
      const Token &t = peek();
      if (t.k == TK::Ident || t.k == TK::Str) {
        Step s;
        s.key = t.s;
        p.steps.push_back(s);
        bump();
      } else if (t.k == TK::LB) {
        bump();
        size_t ia = at();
        Token x = bump();
        if (x.k == TK::Int && x.iv >= 0) {
          Step s;
          s.is_index = true;
          s.index = (uint32_t)x.iv;
          p.steps.push_back(s);
        } else if (x.k == TK::Int) {
          throw Fail{ia, "negative array indices are not supported in v0.1", ""};
        } else {
          throw Fail{ia, "expected an array index, found " + describe(x),
                     "slices (`.[1:3]`) and iteration (`.[]`) are not in v0.1"};
        }
        expect(TK::RB, "to close the index");
      } else {
        break;
      }
      if (peek().k == TK::Dot) {
        TK n = peek(1).k;
        if (n == TK::Ident || n == TK::Str || n == TK::LB) bump();
        else break;
      } else if (peek().k != TK::LB) {
        break;
      }
    }
    return p;
  }

  std::unique_ptr<Cond> node(Cond::Tag t, std::unique_ptr<Cond> a, std::unique_ptr<Cond> b) {
    auto n = std::make_unique<Cond>();
    n->tag = t;
    n->a = std::move(a);
    n->b = std::move(b);
    return n;
  }

  std::unique_ptr<Cond> cond() {
    auto l = conj();
    while (keyword("or")) {
      bump();
      l = node(Cond::Or, std::move(l), conj());
    }
    return l;
  }
  std::unique_ptr<Cond> conj() {
    auto l = term();
    while (keyword("and")) {
      bump();
      l = node(Cond::And, std::move(l), term());
    }
    return l;
  }
  std::unique_ptr<Cond> term() {
    size_t a = at();
    std::unique_ptr<Cond> base;
    if (eat(TK::LP)) {
      if (++depth > 64) throw Fail{a, "conditions may not nest more than 64 deep", ""};
      base = cond();
      expect(TK::RP, "to close the group");
      depth--;
    } else {
      if (peek().k == TK::Ident)
        throw Fail{a, "expected a field path, found `" + peek().s + "`", "did you mean `." + peek().s + "`?"};
      Path p = path();
      if (p.steps.empty())
        throw Fail{a, "`.` cannot be used as a condition in v0.1", "compare a field, e.g. `select(.status == 500)`"};
      base = std::make_unique<Cond>();
      base->path = intern(p);
      if (peek().k == TK::Op) {
        base->tag = Cond::Cmp;
        base->op = bump().op;
        literal(*base);
      } else {
        base->tag = Cond::Truthy;
      }
    }
    while (peek().k == TK::Pipe && peek(1).k == TK::Ident && peek(1).s == "not") {
      bump();
      bump();
      base = node(Cond::Not, std::move(base), nullptr);
    }
    return base;
  }
  void literal(Cond &c) {
    size_t a = at();
    Token t = bump();
    switch (t.k) {
      case TK::Num: c.lit = LitKind::Num; c.num = t.num; return;
      case TK::Int: c.lit = LitKind::Num; c.num = (double)t.iv; return;
      case TK::Str: c.lit = LitKind::Str; c.str = t.s; return;
      case TK::Ident:
        if (t.s == "true") { c.lit = LitKind::True; return; }
        if (t.s == "false") { c.lit = LitKind::False; return; }
        if (t.s == "null") { c.lit = LitKind::Null; return; }
        throw Fail{a, "expected a literal value, found `" + t.s + "`",
                   "the right-hand side of a comparison must be a number, string, `true`, "
                   "`false`, or `null`. Field-to-field comparison is not in v0.1"};
      case TK::Dot:
        throw Fail{a, "field-to-field comparison is not supported in v0.1",
                   "compare against a constant, e.g. `select(.status == 500)`"};
      default:
        throw Fail{a, "expected a literal value, found " + describe(t), ""};
    }
  }

  void program(Program &P) {
    bool has_out = false;
    size_t out_at = 0;
    for (;;) {
      size_t sa = at();
      const Token &t = peek();
      if (t.k == TK::Ident) {
        std::string name = t.s;
        if (const char *why = unsupported(name)) throw Fail{sa, why, kSubsetHint};
        if (name == "select") {
          bump();
          expect(TK::LP, "after `select`");
          auto c = cond();
          expect(TK::RP, "to close `select(`");
          P.filter = P.filter ? node(Cond::And, std::move(P.filter), std::move(c)) : std::move(c);
        } else if (name == "group_by") {
          bump();
          expect(TK::LP, "after `group_by`");
          Path p = path();
          if (p.steps.empty())
            throw Fail{sa, "`group_by(.)` would group by the whole line", "group by a field, e.g. `group_by(.status)`"};
          uint16_t id = intern(p);
          expect(TK::RP, "to close `group_by(`");
          if (P.has_group) throw Fail{sa, "only one `group_by` per query is supported in v0.1", ""};
          if (has_out)
            throw Fail{sa, "`group_by` must come before the output stage",
                       "write `group_by(.host) | count`, not `count | group_by(.host)`"};
          P.has_group = true;
          P.group_by = id;
        } else if (name == "count" || name == "sum" || name == "min" || name == "max" || name == "avg") {
          bump();
          uint32_t kind = name == "count" ? WARPJQ_AGG_COUNT : name == "sum" ? WARPJQ_AGG_SUM
                          : name == "min" ? WARPJQ_AGG_MIN : name == "max" ? WARPJQ_AGG_MAX : WARPJQ_AGG_AVG;
          bool has_arg = kind != WARPJQ_AGG_COUNT;
          uint16_t arg = 0;
          if (!has_arg) {
            if (peek().k == TK::LP)
              throw Fail{at(), "`count` takes no argument", "write `count`, or `sum(.field)` to total a field"};
          } else {
            expect(TK::LP, "after `" + name + "`");
            Path p = path();
            if (p.steps.empty())
              throw Fail{sa, "`" + name + "(.)` has no field to aggregate", "try `" + name + "(.bytes)`"};
            arg = intern(p);
            expect(TK::RP, "to close `" + name + "(`");
          }
          set_output(P, has_out, out_at, sa);
          P.out = Out::Agg;
          P.agg = kind;
          P.has_arg = has_arg;
          P.arg = arg;
        } else {
          throw Fail{sa, "unknown function `" + name + "`",
                     "v0.1 supports: select, group_by, count, sum, min, max, avg"};
        }
      } else if (t.k == TK::LC) {
        std::vector<std::pair<std::string, uint16_t>> fields;
        object(fields);
        set_output(P, has_out, out_at, sa);
        P.out = Out::Project;
        P.fields = std::move(fields);
      } else {
        Path p = path();
        set_output(P, has_out, out_at, sa);
        if (p.steps.empty()) {
          P.out = Out::Passthrough;
        } else {
          P.out = Out::Path;
          P.out_path = intern(p);
        }
      }
      if (!eat(TK::Pipe)) break;
    }
    if (peek().k != TK::Eof) throw Fail{at(), "unexpected " + describe(peek()), ""};
    if (!has_out) P.out = Out::Passthrough;
    if (P.has_group && P.out != Out::Agg)
      throw Fail{out_at > 1 ? out_at : 1, "`group_by` must be followed by an aggregate",
                 "try `group_by(.host) | count` or `group_by(.host) | sum(.bytes)`"};
    P.paths = std::move(paths);
    P.source = src;
  }

  void set_output(Program &P, bool &has_out, size_t &out_at, size_t sa) {
    if (has_out) {
      const char *prev = P.out == Out::Passthrough ? "`.`" : P.out == Out::Path ? "a field path"
                         : P.out == Out::Project ? "an object projection" : "an aggregate";
      throw Fail{sa, std::string("a second output stage follows ") + prev +
                         "; v0.1 supports one output stage per query", ""};
    }
    has_out = true;
    out_at = sa;
  }

  void object(std::vector<std::pair<std::string, uint16_t>> &fields) {
    expect(TK::LC, "to start an object");
    while (peek().k != TK::RC) {
      size_t ka = at();
      Token k = bump();
      if (k.k != TK::Ident && k.k != TK::Str) throw Fail{ka, "expected an object key, found " + describe(k), ""};
      uint16_t id;
      if (eat(TK::Colon)) {
        Path p = path();
        if (p.steps.empty())
          throw Fail{ka, "an object value of `.` would embed the whole line", "name a field, e.g. `{msg: .message}`"};
        id = intern(p);
      } else {
        Path p;
        Step s;
        s.key = k.s;
        p.steps.push_back(s);
        id = intern(p);
      }
      for (auto &f : fields)
        if (f.first == k.s) throw Fail{ka, "duplicate key `" + k.s + "` in projection", ""};
      fields.push_back({k.s, id});
      if (!eat(TK::Comma)) break;
    }
    expect(TK::RC, "to close the object");
    if (fields.empty()) throw Fail{at(), "empty projection `{}` produces no output", ""};
  }
};

}  // namespace

std::string Path::display() const {
  if (steps.empty()) return ".";
  std::string o;
  for (auto &s : steps) {
    if (s.is_index) {
      o += "[" + std::to_string(s.index) + "]";
      continue;
    }
    bool bare = !s.key.empty() && !digit(s.key[0]);
    for (unsigned char c : s.key)
      if (!(alnum(c) || c == '_')) bare = false;
    o += "." + (bare ? s.key : debug_str(s.key));
  }
  return o;
}

const char *agg_name(uint32_t k) {
  static const char *n[] = {"count", "sum", "min", "max", "avg"};
  return k < 5 ? n[k] : "count";
}

std::vector<uint16_t> Program::required_paths() const {
  std::vector<uint16_t> ids;
  auto push = [&](uint16_t id) {
    for (auto x : ids)
      if (x == id) return;
    ids.push_back(id);
  };
  std::vector<const Cond *> st;
  std::vector<uint16_t> fp;
  if (filter) {
    // preorder, left before right (ir.rs:128-137)
    std::vector<const Cond *> stack{filter.get()};
    while (!stack.empty()) {
      const Cond *c = stack.back();
      stack.pop_back();
      if (c->tag == Cond::Cmp || c->tag == Cond::Truthy) push(c->path);
      else {
        if (c->b) stack.push_back(c->b.get());
        stack.push_back(c->a.get());
      }
    }
  }
  if (has_group) push(group_by);
  if (out == Out::Path) push(out_path);
  if (out == Out::Project)
    for (auto &f : fields) push(f.second);
  if (out == Out::Agg && has_arg) push(arg);
  return ids;
}

bool Program::csv_headers(std::vector<std::string> &cols) const {
  cols.clear();
  if (out == Out::Passthrough) return false;
  if (out == Out::Project)
    for (auto &f : fields) cols.push_back(f.first);
  if (out == Out::Path) cols.push_back(paths[out_path].display());
  if (out == Out::Agg) {
    if (has_group) cols.push_back(paths[group_by].display());
    cols.push_back(agg_name(agg));
  }
  return true;
}

std::string Program::group_key_name() const {
  if (!has_group || paths[group_by].steps.empty()) return "key";
  const Step &s = paths[group_by].steps.back();
  return s.is_index ? "[" + std::to_string(s.index) + "]" : s.key;
}

std::string QueryError::render(const std::string &src) const {
  size_t col = 0;
  for (size_t i = 0; i < at && i < src.size(); i++) col += ((unsigned char)src[i] & 0xC0) != 0x80;
  std::string o = "invalid query: " + message + "\n  " + src + "\n  " + std::string(col, ' ') + "^\n";
  if (!hint.empty()) o += "  help: " + hint;
  return o;
}

bool parse(const std::string &src, Program &out, QueryError &err) {
  try {
    check_leading_keywords(src);
    Parser p{src};
    p.tk = lex(src);
    p.program(out);
    return true;
  } catch (Fail &f) {
    err.at = f.at > src.size() ? src.size() : f.at;
    err.message = f.msg;
    err.hint = f.hint;
    return false;
  }
}

// ---- lowering (query/mod.rs:95-198, gpu/lower.rs:38-127) ------------------

namespace {

uint32_t fnv1a(const std::string &s) {
  uint32_t h = 0x811c9dc5u;
  for (unsigned char c : s) {
    h ^= c;
    h *= 0x01000193u;
  }
  return h;
}

uint32_t blob_push(std::vector<uint8_t> &b, const std::string &s) {
  uint32_t off = (uint32_t)b.size();
  b.insert(b.end(), s.begin(), s.end());
  return off;
}

void json_quote(std::string &o, const std::string &s) {
  o += '"';
  for (unsigned char c : s) {
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      case 0x08: o += "\\b"; break;
      case 0x0C: o += "\\f"; break;
      default:
        if (c < 0x20) {
          char b[8];
          snprintf(b, sizeof b, "\\u%04x", c);
          o += b;
        } else o += (char)c;
    }
  }
  o += '"';
}

void flatten(const Cond &c, Lowered &L) {
  switch (c.tag) {
    case Cond::Cmp: {
      warpjq_cmp m{};
      m.path = c.path;
      m.op = c.op;
      m.lit_kind = (uint32_t)c.lit;
      if (c.lit == LitKind::Num) m.lit_num = c.num;
      if (c.lit == LitKind::Str) {
        m.lit_off = blob_push(L.blob, c.str);
        m.lit_len = (uint32_t)c.str.size();
      }
      L.cond.push_back({WARPJQ_COND_CMP, (uint32_t)L.cmps.size()});
      L.cmps.push_back(m);
      return;
    }
    case Cond::Truthy: L.cond.push_back({WARPJQ_COND_TRUTHY, c.path}); return;
    case Cond::Not:
      flatten(*c.a, L);
      L.cond.push_back({WARPJQ_COND_NOT, 0});
      return;
    default:
      flatten(*c.a, L);
      flatten(*c.b, L);
      L.cond.push_back({c.tag == Cond::And ? (uint32_t)WARPJQ_COND_AND : (uint32_t)WARPJQ_COND_OR, 0});
  }
}

template <class T>
const T *ptr(const std::vector<T> &v) {
  static const T dummy{};
  return v.empty() ? &dummy : v.data();
}

}  // namespace

void Lowered::build(const Program &p, bool csv) {
  *this = Lowered();
  for (auto &path : p.paths) {
    warpjq_path wp{(uint32_t)steps.size(), (uint32_t)path.steps.size()};
    for (auto &s : path.steps) {
      warpjq_step ws{};
      if (s.is_index) {
        ws.kind = WARPJQ_STEP_INDEX;
        ws.index = s.index;
      } else {
        ws.kind = WARPJQ_STEP_KEY;
        ws.key_off = blob_push(blob, s.key);
        ws.key_len = (uint32_t)s.key.size();
        ws.key_hash = fnv1a(s.key);
      }
      steps.push_back(ws);
    }
    paths.push_back(wp);
  }
  if (p.filter) flatten(*p.filter, *this);
  slot_of_path.assign(p.paths.size(), 0xFFFFFFFFu);
  for (uint16_t id : p.required_paths()) {
    slot_of_path[id] = (uint32_t)needed.size();
    needed.push_back(id);
  }
  uint32_t suffix_off = 0, suffix_len = 0;
  uint32_t out_kind = WARPJQ_OUT_PASSTHROUGH;
  if (p.out == Out::Path) out_kind = WARPJQ_OUT_PATH;
  if (p.out == Out::Agg) out_kind = WARPJQ_OUT_AGG;
  if (p.out == Out::Project) {
    out_kind = WARPJQ_OUT_PROJECT;
    for (size_t i = 0; i < p.fields.size(); i++) {
      std::string pre;
      if (csv) {
        if (i) pre += ',';
      } else {
        pre += i ? ',' : '{';
        json_quote(pre, p.fields[i].first);
        pre += ':';
      }
      field_paths.push_back(p.fields[i].second);
      prefix_off.push_back(blob_push(blob, pre));
      prefix_len.push_back((uint32_t)pre.size());
    }
    if (!csv) {
      suffix_off = blob_push(blob, "}");
      suffix_len = 1;
    }
  }
  prog = warpjq_program{};
  prog.steps = ptr(steps);
  prog.n_steps = (uint32_t)steps.size();
  prog.paths = ptr(paths);
  prog.n_paths = (uint32_t)paths.size();
  prog.cmps = ptr(cmps);
  prog.n_cmps = (uint32_t)cmps.size();
  prog.cond_rpn = ptr(cond);
  prog.n_cond = (uint32_t)cond.size();
  prog.blob = ptr(blob);
  prog.n_blob = (uint32_t)blob.size();
  prog.needed_paths = ptr(needed);
  prog.n_needed = (uint32_t)needed.size();
  prog.slot_of_path = ptr(slot_of_path);
  prog.output_kind = out_kind;
  prog.output_path = p.out == Out::Path ? p.out_path : 0xFFFFFFFFu;
  prog.agg_kind = p.out == Out::Agg ? p.agg : WARPJQ_AGG_COUNT;
  prog.agg_path = (p.out == Out::Agg && p.has_arg) ? p.arg : 0xFFFFFFFFu;
  prog.group_path = p.has_group ? p.group_by : 0xFFFFFFFFu;
  prog.has_filter = p.filter ? 1 : 0;
  prog.n_fields = (uint32_t)field_paths.size();
  prog.field_paths = ptr(field_paths);
  prog.prefix_off = ptr(prefix_off);
  prog.prefix_len = ptr(prefix_len);
  prog.suffix_off = suffix_off;
  prog.suffix_len = suffix_len;
  prog.csv_mode = csv ? 1 : 0;
}

}  // namespace wjqh
