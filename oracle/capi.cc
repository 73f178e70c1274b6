// TEST INFRASTRUCTURE -- C entry points of the oracle, loaded by the tests
// and by bench.py's CPU-baseline leg through ctypes.  Not part of the product.
#include "oracle.h"

#include <cstdlib>
#include <cstring>
#include <functional>

using namespace oracle;

namespace {

void put_err(char *err, size_t n, const std::string &m) {
  if (!err || !n) return;
  size_t k = m.size() < n - 1 ? m.size() : n - 1;
  std::memcpy(err, m.data(), k);
  err[k] = 0;
}

std::string jstr(const std::string &s) {
  std::string o;
  write_json_string(o, (const uint8_t *)s.data(), s.size());
  return o;
}

std::string num_json(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

std::string cond_json(const Cond &c) {
  switch (c.tag) {
    case Cond::Cmp: {
      static const char *lk[] = {"null", "false", "true", "num", "str"};
      std::string lit = "{\"kind\":\"" + std::string(lk[(int)c.lit.kind]) + "\"";
      if (c.lit.kind == LitKind::Num) lit += ",\"num\":" + num_json(c.lit.num);
      if (c.lit.kind == LitKind::Str) lit += ",\"str\":" + jstr(c.lit.str);
      lit += "}";
      return "{\"cmp\":{\"path\":" + std::to_string(c.path) + ",\"op\":" +
             std::to_string((int)c.op) + ",\"lit\":" + lit + "}}";
    }
    case Cond::Truthy: return "{\"truthy\":" + std::to_string(c.path) + "}";
    case Cond::And: return "{\"and\":[" + cond_json(*c.a) + "," + cond_json(*c.b) + "]}";
    case Cond::Or: return "{\"or\":[" + cond_json(*c.a) + "," + cond_json(*c.b) + "]}";
    default: return "{\"not\":" + cond_json(*c.a) + "}";
  }
}

std::string program_json(const Program &p) {
  std::string o = "{\"paths\":[";
  for (size_t i = 0; i < p.paths.size(); i++) {
    if (i) o += ",";
    o += "[";
    for (size_t k = 0; k < p.paths[i].steps.size(); k++) {
      const Step &s = p.paths[i].steps[k];
      if (k) o += ",";
      o += s.is_index ? std::to_string(s.index) : jstr(s.key);
    }
    o += "]";
  }
  o += "],\"filter\":" + (p.filter ? cond_json(*p.filter) : std::string("null"));
  o += ",\"group_by\":" + (p.has_group ? std::to_string(p.group_by) : std::string("null"));
  o += ",\"output\":";
  switch (p.output.tag) {
    case Output::Passthrough: o += "\"passthrough\""; break;
    case Output::PathOut: o += "{\"path\":" + std::to_string(p.output.path) + "}"; break;
    case Output::Project: {
      o += "{\"project\":[";
      for (size_t i = 0; i < p.output.fields.size(); i++) {
        if (i) o += ",";
        o += "[" + jstr(p.output.fields[i].first) + "," +
             std::to_string(p.output.fields[i].second) + "]";
      }
      o += "]}";
      break;
    }
    default:
      o += "{\"agg\":\"" + std::string(agg_name(p.output.agg)) + "\",\"arg\":" +
           (p.output.has_arg ? std::to_string(p.output.arg) : std::string("null")) + "}";
  }
  std::vector<std::string> cols;
  if (p.csv_headers(cols)) {
    o += ",\"csv_headers\":[";
    for (size_t i = 0; i < cols.size(); i++) o += (i ? "," : "") + jstr(cols[i]);
    o += "]";
  } else {
    o += ",\"csv_headers\":null";
  }
  FlatProgram f = flatten(p);
  o += ",\"flat\":{\"steps\":[";
  for (size_t i = 0; i < f.steps.size(); i++) {
    auto &s = f.steps[i];
    o += (i ? "," : "") + std::string("[") + std::to_string(s.kind) + "," +
         std::to_string(s.index) + "," + std::to_string(s.key_off) + "," +
         std::to_string(s.key_len) + "," + std::to_string(s.key_hash) + "]";
  }
  o += "],\"paths\":[";
  for (size_t i = 0; i < f.paths.size(); i++)
    o += (i ? "," : "") + std::string("[") + std::to_string(f.paths[i].step_off) + "," +
         std::to_string(f.paths[i].step_count) + "]";
  o += "],\"cmps\":[";
  for (size_t i = 0; i < f.cmps.size(); i++) {
    auto &c = f.cmps[i];
    o += (i ? "," : "") + std::string("[") + std::to_string(c.path) + "," + std::to_string(c.op) +
         "," + std::to_string(c.lit_kind) + "," + std::to_string(c.lit_off) + "," +
         std::to_string(c.lit_len) + "," + num_json(c.lit_num) + "]";
  }
  o += "],\"cond_rpn\":[";
  for (size_t i = 0; i < f.cond_rpn.size(); i++)
    o += (i ? "," : "") + std::string("[") + std::to_string(f.cond_rpn[i].op) + "," +
         std::to_string(f.cond_rpn[i].arg) + "]";
  o += "],\"blob\":" + jstr(std::string(f.blob.begin(), f.blob.end()));
  o += ",\"cond_stack_depth\":" + std::to_string(f.cond_stack_depth) + "}}";
  return o;
}

char *dup_out(const std::string &s, size_t *n) {
  char *p = (char *)std::malloc(s.size() + 1);
  std::memcpy(p, s.data(), s.size());
  p[s.size()] = 0;
  if (n) *n = s.size();
  return p;
}

}  // namespace

extern "C" {

void oracle_free(char *p) { std::free(p); }

// 0 = ok, 1 = runtime error, 2 = query error.  `stats` receives
// bytes_in, lines_in, lines_out, malformed, type_errors.
int oracle_run(const char *query, const uint8_t *data, size_t len, int format, int on_invalid,
               size_t chunk_bytes, size_t threads, size_t max_line_bytes, char **out,
               size_t *out_len, uint64_t *stats, char *err, size_t err_len) {
  Program prog;
  QueryError qe;
  std::string q = query;
  if (!parse_query(q, prog, qe)) {
    put_err(err, err_len, qe.render(q));
    return 2;
  }
  Options opt;
  opt.format = (Format)format;
  opt.on_invalid = (OnInvalid)on_invalid;
  if (chunk_bytes) opt.chunk_bytes = chunk_bytes;
  if (max_line_bytes) opt.max_line_bytes = max_line_bytes;
  opt.threads = threads;
  std::string res, e;
  RunStats st;
  int rc = run_bytes(prog, data, len, opt, res, st, e);
  if (stats) {
    stats[0] = st.bytes_in;
    stats[1] = st.lines_in;
    stats[2] = st.lines_out;
    stats[3] = st.malformed;
    stats[4] = st.type_errors;
  }
  if (rc != 0) {
    put_err(err, err_len, e);
    *out = nullptr;
    if (out_len) *out_len = 0;
    return 1;
  }
  *out = dup_out(res, out_len);
  return 0;
}

// 1 when the line is one valid JSON value (json.rs:414); else 0 with the
// error offset and message.
int oracle_validate(const uint8_t *line, size_t len, size_t *offset, char *detail, size_t n) {
  JsonError e;
  if (validate(line, len, e)) return 1;
  if (offset) *offset = e.offset;
  put_err(detail, n, e.detail);
  return 0;
}

void oracle_format_number(double v, char *buf, size_t n) { put_err(buf, n, format_number(v)); }

// Parses a query; returns 0 and a JSON dump of the program (and its flat
// tables) on success, or 2 and the rendered QueryError.
int oracle_parse(const char *query, char **out, size_t *out_len) {
  Program prog;
  QueryError qe;
  std::string q = query;
  if (!parse_query(q, prog, qe)) {
    std::string m = "{\"error\":" + jstr(qe.message) + ",\"at\":" + std::to_string(qe.at) +
                    ",\"hint\":" + jstr(qe.hint) + ",\"rendered\":" + jstr(qe.render(q)) + "}";
    *out = dup_out(m, out_len);
    return 2;
  }
  *out = dup_out(program_json(prog), out_len);
  return 0;
}

// Resolves the single path of `path_query` (e.g. ".a.b[0]") against `line`
// (json.rs:444).  Returns 0 Found (kind, raw bytes), 1 TypeError, 2 Invalid,
// -1 if the path does not parse.
int oracle_lookup(const uint8_t *line, size_t len, const char *path_query, int *kind, char **raw,
                  size_t *raw_len) {
  Program prog;
  QueryError qe;
  if (!parse_query(path_query, prog, qe)) return -1;
  std::vector<Step> steps;
  if (prog.output.tag == Output::PathOut) steps = prog.paths[prog.output.path].steps;
  Slot s;
  std::string msg;
  LookupRes r = lookup(line, len, steps, s, msg);
  if (r == LookupRes::Found) {
    *kind = (int)s.kind;
    *raw = dup_out(std::string((const char *)s.p, s.n), raw_len);
    return 0;
  }
  *raw = dup_out(msg, raw_len);
  return r == LookupRes::TypeError ? 1 : 2;
}

// Three-way compare of the value at `path_query` in `line` with the literal
// of a `select(<path> <op> <literal>)` query (json.rs:662).  Returns the
// predicate's verdict (0/1), or -1 on a parse problem.
int oracle_eval_select(const uint8_t *line, size_t len, const char *select_query) {
  Program prog;
  QueryError qe;
  if (!parse_query(select_query, prog, qe) || !prog.filter) return -1;
  JsonError je;
  if (!validate(line, len, je)) return -1;
  std::vector<PathId> ids;
  prog.filter->visit_paths(ids);
  std::vector<Slot> slots(prog.paths.size(), missing_slot());
  for (PathId id : ids) {
    std::string msg;
    if (lookup(line, len, prog.paths[id].steps, slots[id], msg) != LookupRes::Found) return -1;
  }
  std::function<bool(const Cond &)> ev = [&](const Cond &c) -> bool {
    switch (c.tag) {
      case Cond::Cmp: return cmp_accepts(c.op, compare(slots[c.path], c.lit));
      case Cond::Truthy: return slots[c.path].is_truthy();
      case Cond::And: return ev(*c.a) && ev(*c.b);
      case Cond::Or: return ev(*c.a) || ev(*c.b);
      default: return !ev(*c.a);
    }
  };
  return ev(*prog.filter) ? 1 : 0;
}

// Correctly rounded decimal-to-double of a JSON number (json.rs:73-78).
double oracle_parse_f64(const uint8_t *p, size_t n) {
  Slot s;
  s.kind = Kind::Num;
  s.p = p;
  s.n = n;
  double v = 0;
  s.as_f64(v);
  return v;
}

}  // extern "C"

extern "C" {

// Per physical line, in the same shape as the walker test harness:
//   blank | invalid | type | filtered | selected<TAB>kind:raw[=hexfloat]...
// following exec/cpu.rs:299-371 with the chunk.rs line rules.
int oracle_eval_lines(const char *query, const uint8_t *data, size_t len, char **out,
                      size_t *out_len) {
  Program prog;
  QueryError qe;
  if (!parse_query(query, prog, qe)) return 2;
  std::vector<PathId> req = prog.required_paths(), fpaths;
  if (prog.filter) prog.filter->visit_paths(fpaths);
  std::string o;
  size_t pos = 0;
  std::vector<Slot> slots(prog.paths.size(), missing_slot());
  std::function<bool(const Cond &)> ev = [&](const Cond &c) -> bool {
    switch (c.tag) {
      case Cond::Cmp: return cmp_accepts(c.op, compare(slots[c.path], c.lit));
      case Cond::Truthy: return slots[c.path].is_truthy();
      case Cond::And: return ev(*c.a) && ev(*c.b);
      case Cond::Or: return ev(*c.a) || ev(*c.b);
      default: return !ev(*c.a);
    }
  };
  while (pos < len) {
    const uint8_t *nl = (const uint8_t *)std::memchr(data + pos, '\n', len - pos);
    size_t end = nl ? (size_t)(nl - data) : len;
    const uint8_t *line = data + pos;
    size_t n = end - pos;
    pos = end + 1;
    size_t e = n;
    if (e && line[e - 1] == '\r') e--;
    bool blank = true;
    for (size_t k = 0; k < e; k++) {
      uint8_t c = line[k];
      if (!(c == ' ' || c == '\t' || c == '\n' || c == 0x0C || c == '\r')) blank = false;
    }
    if (blank) {
      o += "blank\n";
      continue;
    }
    JsonError je;
    if (!validate(line, e, je)) {
      o += "invalid\n";
      continue;
    }
    for (auto &s : slots) s = missing_slot();
    bool type = false;
    for (PathId id : fpaths) {
      std::string msg;
      if (lookup(line, e, prog.paths[id].steps, slots[id], msg) != LookupRes::Found) type = true;
    }
    if (type) {
      o += "type\n";
      continue;
    }
    if (prog.filter && !ev(*prog.filter)) {
      o += "filtered\n";
      continue;
    }
    for (PathId id : req) {
      std::string msg;
      if (lookup(line, e, prog.paths[id].steps, slots[id], msg) != LookupRes::Found) type = true;
    }
    if (type) {
      o += "type\n";
      continue;
    }
    o += "selected";
    for (PathId id : req) {
      const Slot &s = slots[id];
      o += "\t" + std::to_string((int)s.kind) + ":";
      if (s.kind != Kind::Missing) o.append((const char *)s.p, s.n);
      if (s.kind == Kind::Num) {
        double d;
        s.as_f64(d);
        char b[64];
        std::snprintf(b, sizeof b, "=%a", d);
        o += b;
      }
    }
    o += "\n";
  }
  *out = dup_out(o, out_len);
  return 0;
}

}  // extern "C"
