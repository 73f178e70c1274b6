// TEST INFRASTRUCTURE -- the oracle's aggregation, output and CPU engine.
// Restates crates/warpjq-core/src/{agg.rs, output.rs, chunk.rs, exec/cpu.rs,
// exec/mod.rs} of the reference project.
#include "oracle.h"

#include <charconv>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <unordered_map>
#include <algorithm>

namespace oracle {

// ---------------------------------------------------------------------------
// agg.rs
// ---------------------------------------------------------------------------

void AggState::push_value(const Slot &s) {  // agg.rs:50-60
  count++;
  switch (s.kind) {
    case Kind::Missing: case Kind::Null: break;
    case Kind::Num: {
      double v;
      if (s.as_f64(v)) push_number(v);
      else saw_non_numeric = true;
      break;
    }
    default: saw_non_numeric = true;
  }
}

void AggState::push_number(double v) {  // agg.rs:62-71
  numeric++;
  sum += v;
  if (v < min) min = v;
  if (v > max) max = v;
}

void AggState::merge(const AggState &o) {  // agg.rs:73-84
  count += o.count;
  numeric += o.numeric;
  sum += o.sum;
  if (o.min < min) min = o.min;
  if (o.max > max) max = o.max;
  saw_non_numeric = saw_non_numeric || o.saw_non_numeric;
}

bool AggState::finish(AggKind k, double &v) const {  // agg.rs:88-97
  switch (k) {
    case AggKind::Count: v = (double)count; return true;
    case AggKind::Sum: v = sum; return true;
    case AggKind::Min: v = min; return numeric > 0;
    case AggKind::Max: v = max; return numeric > 0;
    default: v = sum / (double)numeric; return numeric > 0;
  }
}

uint64_t order_bits(double v) {  // agg.rs:205-212
  uint64_t b;
  std::memcpy(&b, &v, 8);
  return (b >> 63) ? ~b : (b ^ (1ull << 63));
}

GroupKey GroupKey::from_slot(const Slot &s) {  // agg.rs:121-144
  GroupKey k;
  switch (s.kind) {
    case Kind::Missing: case Kind::Null: k.rank = 0; break;
    case Kind::Bool: {
      bool t = s.n == 4 && std::memcmp(s.p, "true", 4) == 0;
      k.rank = t ? 2 : 1;
      break;
    }
    case Kind::Num: {
      double v;
      if (!s.as_f64(v)) v = std::nan("");
      k.rank = 3;
      k.bytes.assign((const char *)s.p, s.n);
      k.bits = order_bits(v);
      break;
    }
    case Kind::Str: {
      k.rank = 4;
      const uint8_t *inner = s.p + 1;
      size_t n = s.n - 2;
      if (std::memchr(inner, '\\', n)) {
        std::string buf;
        if (unescape_into(inner, n, buf)) {
          k.bytes = buf;
          break;
        }
      }
      k.bytes.assign((const char *)inner, n);
      break;
    }
    default:
      k.rank = 5;
      k.bytes.assign((const char *)s.p, s.n);
  }
  return k;
}

std::string GroupKey::to_json() const {  // agg.rs:158-171
  switch (rank) {
    case 0: return "null";
    case 1: return "false";
    case 2: return "true";
    case 4: {
      std::string o;
      write_json_string(o, (const uint8_t *)bytes.data(), bytes.size());
      return o;
    }
    default: return bytes;
  }
}

std::string GroupKey::to_plain() const { return rank == 4 ? bytes : to_json(); }

// agg.rs:182-195.  Numbers with equal values but different spellings ("1"
// and "1.0") are distinct groups that compare Equal there; the reference
// leaves their relative order to HashMap iteration.  Here ties break on the
// raw bytes so the oracle is deterministic.
bool GroupKey::operator<(const GroupKey &o) const {
  if (rank != o.rank) return rank < o.rank;
  if (rank == 3) {
    if (bits != o.bits) return bits < o.bits;
    return bytes < o.bytes;
  }
  return bytes < o.bytes;
}

size_t GroupKeyHash::operator()(const GroupKey &k) const {
  return std::hash<std::string>()(k.bytes) * 31 + k.rank;
}

// agg.rs:253-278.  Integral values below 2^53 print as integers; everything
// else prints the shortest round-trip digits placed the way the `ryu` crate's
// pretty printer places them, then `e` gets an explicit `+` for positive
// exponents.
std::string format_number(double v) {
  if (std::isnan(v)) return "null";
  if (std::isinf(v)) return v > 0 ? "1.7976931348623157e+308" : "-1.7976931348623157e+308";
  if (std::trunc(v) == v && std::fabs(v) < 9007199254740992.0) {
    return std::to_string((long long)v);
  }
  // Shortest digits and decimal exponent.
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string sci(buf, r.ptr);
  bool neg = false;
  size_t i = 0;
  if (sci[0] == '-') {
    neg = true;
    i = 1;
  }
  size_t epos = sci.find('e');
  std::string digits;
  for (size_t k = i; k < epos; k++)
    if (sci[k] != '.') digits.push_back(sci[k]);
  int e10 = std::atoi(sci.c_str() + epos + 1);  // value = d.ddd * 10^e10
  long length = (long)digits.size();
  long kk = e10 + 1;        // 10^(kk-1) <= v < 10^kk
  long k = kk - length;     // value = digits * 10^k
  std::string out = neg ? "-" : "";
  if (0 <= k && kk <= 16) {
    out += digits;
    out.append((size_t)(kk - length), '0');
    out += ".0";
  } else if (0 < kk && kk <= 16) {
    out += digits.substr(0, (size_t)kk);
    out += ".";
    out += digits.substr((size_t)kk);
  } else if (-5 < kk && kk <= 0) {
    out += "0.";
    out.append((size_t)(-kk), '0');
    out += digits;
  } else if (length == 1) {
    out += digits;
    out += "e" + std::to_string(kk - 1);
  } else {
    out += digits.substr(0, 1) + "." + digits.substr(1);
    out += "e" + std::to_string(kk - 1);
  }
  size_t e = out.find('e');
  if (e != std::string::npos && out[e + 1] != '-') out.insert(e + 1, "+");
  return out;
}

// ---------------------------------------------------------------------------
// output.rs
// ---------------------------------------------------------------------------

void write_json_string(std::string &out, const uint8_t *p, size_t n) {  // output.rs:24-42
  out.push_back('"');
  for (size_t i = 0; i < n; i++) {
    uint8_t c = p[i];
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\n': out += "\\n"; break;
      case '\r': out += "\\r"; break;
      case '\t': out += "\\t"; break;
      case 0x08: out += "\\b"; break;
      case 0x0c: out += "\\f"; break;
      default:
        if (c < 0x20) {
          char b[8];
          std::snprintf(b, sizeof b, "\\u%04x", c);
          out += b;
        } else {
          out.push_back((char)c);
        }
    }
  }
  out.push_back('"');
}

void write_csv_cell(std::string &out, const uint8_t *p, size_t n) {  // output.rs:45-61
  bool q = false;
  for (size_t i = 0; i < n; i++)
    if (p[i] == ',' || p[i] == '"' || p[i] == '\n' || p[i] == '\r') q = true;
  if (!q) {
    out.append((const char *)p, n);
    return;
  }
  out.push_back('"');
  for (size_t i = 0; i < n; i++) {
    if (p[i] == '"') out.push_back('"');
    out.push_back((char)p[i]);
  }
  out.push_back('"');
}

static void csv_value(std::string &out, const Slot &s) {  // output.rs:65-81
  switch (s.kind) {
    case Kind::Missing: case Kind::Null: return;
    case Kind::Str: {
      const uint8_t *inner = s.p + 1;
      size_t n = s.n - 2;
      if (std::memchr(inner, '\\', n)) {
        std::string buf;
        if (unescape_into(inner, n, buf)) {
          write_csv_cell(out, (const uint8_t *)buf.data(), buf.size());
          return;
        }
      }
      write_csv_cell(out, inner, n);
      return;
    }
    default: write_csv_cell(out, s.p, s.n);
  }
}

namespace {

// output.rs:87-334 (buffering omitted: everything lands in one string).
struct Writer {
  std::string buf;
  Format format;
  bool header_written = false;
  uint64_t rows = 0;
  explicit Writer(Format f) : format(f) {}

  void write_raw(const std::string &b, uint64_t r) {
    rows += r;
    if (format == Format::CountOnly) return;
    buf += b;
  }
  void write_header(const Program &p) {
    if (format != Format::Csv || header_written) return;
    header_written = true;
    std::vector<std::string> cols;
    if (p.csv_headers(cols)) {
      for (size_t i = 0; i < cols.size(); i++) {
        if (i) buf.push_back(',');
        write_csv_cell(buf, (const uint8_t *)cols[i].data(), cols[i].size());
      }
      buf.push_back('\n');
    }
  }
  void passthrough(const uint8_t *line, size_t n) {
    rows++;
    if (format == Format::CountOnly) return;
    if (format == Format::Csv) write_csv_cell(buf, line, n);
    else buf.append((const char *)line, n);
    buf.push_back('\n');
  }
  void value(const Slot &s) {
    rows++;
    if (format == Format::CountOnly) return;
    if (format == Format::Csv) csv_value(buf, s);
    else buf.append((const char *)s.p, s.n);
    buf.push_back('\n');
  }
  void projection(const std::vector<std::string> &keys, const std::vector<Slot> &slots) {
    rows++;
    if (format == Format::CountOnly) return;
    if (format == Format::Csv) {
      for (size_t i = 0; i < slots.size(); i++) {
        if (i) buf.push_back(',');
        csv_value(buf, slots[i]);
      }
    } else {
      buf.push_back('{');
      for (size_t i = 0; i < slots.size(); i++) {
        if (i) buf.push_back(',');
        write_json_string(buf, (const uint8_t *)keys[i].data(), keys[i].size());
        buf.push_back(':');
        buf.append((const char *)slots[i].p, slots[i].n);
      }
      buf.push_back('}');
    }
    buf.push_back('\n');
  }
  void aggregate(AggKind k, const AggState &st) {
    rows++;
    double v;
    std::string val = st.finish(k, v) ? format_number(v) : "null";
    if (format == Format::CountOnly) {
      rows = 0;
      buf.clear();
      buf += val;
      buf.push_back('\n');
      format = Format::Ndjson;
      return;
    }
    buf += val;
    buf.push_back('\n');
  }
  void groups(const std::string &key_name, AggKind k,
              const std::vector<std::pair<GroupKey, AggState>> &gs) {
    for (auto &g : gs) {
      rows++;
      double v;
      std::string val = g.second.finish(k, v) ? format_number(v) : "null";
      if (format == Format::Csv) {
        std::string plain = g.first.to_plain();
        write_csv_cell(buf, (const uint8_t *)plain.data(), plain.size());
        buf.push_back(',');
        buf += val;
      } else {
        buf.push_back('{');
        write_json_string(buf, (const uint8_t *)key_name.data(), key_name.size());
        buf.push_back(':');
        buf += g.first.to_json();
        buf.push_back(',');
        const char *an = agg_name(k);
        write_json_string(buf, (const uint8_t *)an, std::strlen(an));
        buf.push_back(':');
        buf += val;
        buf.push_back('}');
      }
      buf.push_back('\n');
    }
  }
  std::string finish() {
    if (format == Format::CountOnly) {
      buf.clear();
      buf += std::to_string(rows);
      buf.push_back('\n');
    }
    return buf;
  }
};

std::string group_key_name(const Program &p) {  // output.rs:338-347
  if (!p.has_group) return "key";
  const Path &path = p.paths[p.group_by];
  if (path.steps.empty()) return "key";
  const Step &s = path.steps.back();
  if (s.is_index) return "[" + std::to_string(s.index) + "]";
  return s.key;
}

// exec/mod.rs:113-138
struct Totals {
  enum { None, Scalar, Grouped } tag = None;
  AggState scalar;
  std::unordered_map<GroupKey, AggState, GroupKeyHash> groups;
  static Totals for_program(const Program &p) {
    Totals t;
    if (!p.is_aggregate()) t.tag = None;
    else if (p.has_group) t.tag = Grouped;
    else t.tag = Scalar;
    return t;
  }
  void merge(const Totals &o) {
    if (tag == Scalar && o.tag == Scalar) {
      scalar.merge(o.scalar);
    } else if (tag == Grouped && o.tag == Grouped) {
      for (auto &kv : o.groups) groups[kv.first].merge(kv.second);
    }
  }
};

// exec/cpu.rs:87-139
struct Plan {
  const Program *program;
  std::vector<PathId> filter_paths, post_paths;
  std::vector<std::string> proj_keys;
  std::vector<PathId> proj_paths;
  explicit Plan(const Program &p) : program(&p) {
    if (p.filter) {
      std::vector<PathId> tmp;
      p.filter->visit_paths(tmp);
      for (PathId id : tmp)
        if (std::find(filter_paths.begin(), filter_paths.end(), id) == filter_paths.end())
          filter_paths.push_back(id);
    }
    for (PathId id : p.required_paths())
      if (std::find(filter_paths.begin(), filter_paths.end(), id) == filter_paths.end())
        post_paths.push_back(id);
    if (p.output.tag == Output::Project)
      for (auto &f : p.output.fields) {
        proj_keys.push_back(f.first);
        proj_paths.push_back(f.second);
      }
  }
};

enum class Outcome { Emitted, NoRow, Malformed, TypeError };

bool eval_cond(const Cond &c, const std::vector<Slot> &slots) {  // exec/cpu.rs:443-453
  switch (c.tag) {
    case Cond::Cmp: return cmp_accepts(c.op, compare(slots[c.path], c.lit));
    case Cond::Truthy: return slots[c.path].is_truthy();
    case Cond::And: return eval_cond(*c.a, slots) && eval_cond(*c.b, slots);
    case Cond::Or: return eval_cond(*c.a, slots) || eval_cond(*c.b, slots);
    default: return !eval_cond(*c.a, slots);
  }
}

// exec/cpu.rs:299-371: the single source of truth for what a query means.
Outcome eval_line(const uint8_t *line, size_t n, const Plan &plan, std::vector<Slot> &slots,
                  Writer &out, Totals &totals, std::string &msg) {
  const Program &prog = *plan.program;
  JsonError je;
  if (!validate(line, n, je)) {
    msg = je.detail + " at byte " + std::to_string(je.offset);
    return Outcome::Malformed;
  }
  for (auto &s : slots) s = missing_slot();
  for (PathId id : plan.filter_paths) {
    switch (lookup(line, n, prog.paths[id].steps, slots[id], msg)) {
      case LookupRes::Found: break;
      case LookupRes::TypeError: return Outcome::TypeError;
      case LookupRes::Invalid: return Outcome::Malformed;
    }
  }
  if (prog.filter && !eval_cond(*prog.filter, slots)) return Outcome::NoRow;
  for (PathId id : plan.post_paths) {
    switch (lookup(line, n, prog.paths[id].steps, slots[id], msg)) {
      case LookupRes::Found: break;
      case LookupRes::TypeError: return Outcome::TypeError;
      case LookupRes::Invalid: return Outcome::Malformed;
    }
  }
  switch (prog.output.tag) {
    case Output::Passthrough: out.passthrough(line, n); return Outcome::Emitted;
    case Output::PathOut: out.value(slots[prog.output.path]); return Outcome::Emitted;
    case Output::Project: {
      std::vector<Slot> vals;
      for (PathId p : plan.proj_paths) vals.push_back(slots[p]);
      out.projection(plan.proj_keys, vals);
      return Outcome::Emitted;
    }
    default: {
      const Slot *value = prog.output.has_arg ? &slots[prog.output.arg] : nullptr;
      AggState *st = nullptr;
      if (totals.tag == Totals::Grouped && prog.has_group)
        st = &totals.groups[GroupKey::from_slot(slots[prog.group_by])];
      else if (totals.tag == Totals::Scalar)
        st = &totals.scalar;
      if (st) {
        if (value) st->push_value(*value);
        else st->push_count();
      }
      return Outcome::NoRow;
    }
  }
}

// chunk.rs:393-445: split on `\n`, trim one trailing `\r`, skip lines made only
// of u8::is_ascii_whitespace bytes (which includes form feed).
template <class F>
void for_each_line(const uint8_t *data, size_t len, uint64_t first, F f) {
  size_t pos = 0;
  uint64_t no = first;
  while (pos < len) {
    const uint8_t *nl = (const uint8_t *)std::memchr(data + pos, '\n', len - pos);
    size_t end = nl ? (size_t)(nl - data) : len;
    size_t s = pos;
    pos = end + 1;
    uint64_t number = no++;
    size_t e = end;
    if (e > s && data[e - 1] == '\r') e--;
    bool blank = true;
    for (size_t k = s; k < e; k++) {
      uint8_t c = data[k];
      if (!(c == ' ' || c == '\t' || c == '\n' || c == '\x0c' || c == '\r')) {
        blank = false;
        break;
      }
    }
    if (blank) continue;
    if (!f(data + s, e - s, number)) return;
  }
}

struct Partial {  // exec/cpu.rs:142-153
  std::string bytes;
  uint64_t rows = 0, physical_lines = 0, lines_in = 0;
  Totals totals;
  uint64_t malformed = 0, type_errors = 0;
  bool abort = false;
  uint64_t abort_line = 0;
  std::string abort_msg;
};

uint64_t count_physical_lines(const uint8_t *p, size_t n) {  // exec/cpu.rs:433-441
  uint64_t c = 0;
  for (size_t i = 0; i < n; i++) c += p[i] == '\n';
  if (n && p[n - 1] != '\n') c++;
  return c;
}

void process_slice(const uint8_t *p, size_t n, const Plan &plan, const Options &opt,
                   Partial &out) {  // exec/cpu.rs:373-424
  Writer w(opt.format);
  out.totals = Totals::for_program(*plan.program);
  std::vector<Slot> slots(plan.program->paths.size(), missing_slot());
  for_each_line(p, n, 0, [&](const uint8_t *line, size_t len, uint64_t number) {
    out.lines_in++;
    std::string msg;
    Outcome o = eval_line(line, len, plan, slots, w, out.totals, msg);
    if (o == Outcome::Malformed || o == Outcome::TypeError) {
      if (opt.on_invalid == OnInvalid::Abort) {
        out.abort = true;
        out.abort_line = number;
        out.abort_msg = msg;
        return false;
      }
      if (o == Outcome::Malformed) out.malformed++;
      else out.type_errors++;
    }
    return true;
  });
  out.physical_lines = count_physical_lines(p, n);
  out.bytes = std::move(w.buf);
  out.rows = w.rows;
}

// exec/cpu.rs:256-282
std::vector<std::pair<size_t, size_t>> split_chunk(const uint8_t *data, size_t len,
                                                   size_t threads) {
  const size_t MIN_SLICE = 64 << 10;
  size_t n = std::max<size_t>(threads, 1);
  n = std::min(n, std::max<size_t>(len / MIN_SLICE, 1));
  std::vector<std::pair<size_t, size_t>> out;
  if (n == 1) {
    out.push_back({0, len});
    return out;
  }
  std::vector<size_t> bounds{0};
  for (size_t i = 1; i < n; i++) {
    size_t want = (size_t)((unsigned __int128)len * i / n);
    size_t prev = bounds.back();
    const uint8_t *nl = (const uint8_t *)std::memchr(data + want, '\n', len - want);
    size_t cut = nl ? (size_t)(nl - data) + 1 : len;
    if (cut > prev && cut < len) bounds.push_back(cut);
  }
  bounds.push_back(len);
  bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
  for (size_t i = 0; i + 1 < bounds.size(); i++) out.push_back({bounds[i], bounds[i + 1]});
  return out;
}

}  // namespace

// exec/cpu.rs:160-239 driven by chunk.rs:292-387 (stream_chunks), which is
// what exec/cpu.rs:498 run_bytes uses for an in-memory buffer.
int run_bytes(const Program &program, const uint8_t *data, size_t len, const Options &opt,
              std::string &result, RunStats &stats, std::string &err) {
  if (opt.format == Format::Csv && program.output.tag == Output::Passthrough) {  // exec/mod.rs:256
    err = "--csv needs a query with named columns, but this one emits whole lines\n  help: "
          "project the fields you want, e.g. `{ts: .ts, status: .status}`, or use an aggregate";
    return 1;
  }
  Plan plan(program);
  Writer writer(opt.format);
  Totals totals = Totals::for_program(program);
  size_t threads = opt.threads ? opt.threads : std::max(1u, std::thread::hardware_concurrency());
  writer.write_header(program);
  stats = RunStats{};

  bool aborted = false;
  std::string abort_msg;
  const std::string file = "<memory>";

  auto on_chunk = [&](const uint8_t *c, size_t n, uint64_t first_line) -> uint64_t {
    if (aborted) return 0;
    stats.bytes_in += n;
    auto slices = split_chunk(c, n, threads);
    std::vector<Partial> parts(slices.size());
    if (slices.size() == 1) {
      process_slice(c + slices[0].first, slices[0].second - slices[0].first, plan, opt, parts[0]);
    } else {
      std::vector<std::thread> ws;
      for (size_t i = 0; i < slices.size(); i++)
        ws.emplace_back([&, i] {
          process_slice(c + slices[i].first, slices[i].second - slices[i].first, plan, opt,
                        parts[i]);
        });
      for (auto &t : ws) t.join();
    }
    uint64_t base = first_line, total = 0;
    for (auto &p : parts) {
      if (p.abort && !aborted) {
        aborted = true;
        abort_msg = "malformed JSON on line " + std::to_string(base + p.abort_line) + " of " +
                    file + ": " + p.abort_msg +
                    "\n  help: pass --skip-invalid to drop bad lines instead of stopping";
      }
      stats.lines_in += p.lines_in;
      stats.malformed += p.malformed;
      stats.type_errors += p.type_errors;
      writer.write_raw(p.bytes, p.rows);
      totals.merge(p.totals);
      base += p.physical_lines;
      total += p.physical_lines;
    }
    return total;
  };

  // chunk.rs:292-387
  {
    const size_t chunk_bytes = std::max<size_t>(opt.chunk_bytes, 1);
    std::vector<uint8_t> buf, carry;
    size_t rd = 0;  // read position in `data`
    uint64_t line_no = 1;
    bool first = true;
    for (;;) {
      buf.assign(carry.begin(), carry.end());
      carry.clear();
      size_t base = buf.size();
      size_t want = base >= chunk_bytes ? chunk_bytes : chunk_bytes - base;
      size_t got = std::min(want, len - rd);
      buf.insert(buf.end(), data + rd, data + rd + got);
      rd += got;
      size_t filled = base + got;
      if (first) {
        if (buf.size() >= 3 && buf[0] == 0xEF && buf[1] == 0xBB && buf[2] == 0xBF)
          buf.erase(buf.begin(), buf.begin() + 3);
        first = false;
      }
      if (buf.empty()) break;
      bool eof = filled < base + want;
      size_t end;
      if (eof) {
        end = buf.size();
      } else {
        size_t k = buf.size();
        while (k > 0 && buf[k - 1] != '\n') k--;
        if (k == 0) {
          if (buf.size() > opt.max_line_bytes) {
            err = "line " + std::to_string(line_no) + " exceeds the " +
                  std::to_string(opt.max_line_bytes) +
                  " byte limit (raise it with --max-line-bytes)";
            return 1;
          }
          carry.assign(buf.begin(), buf.end());
          continue;
        }
        end = k;
      }
      carry.assign(buf.begin() + end, buf.end());
      line_no += on_chunk(buf.data(), end, line_no);
      if (eof) break;
    }
  }

  if (aborted) {
    err = abort_msg;
    return 1;
  }
  // exec/mod.rs:321-339
  if (program.is_aggregate()) {
    if (totals.tag == Totals::Scalar) {
      writer.aggregate(program.output.agg, totals.scalar);
    } else if (totals.tag == Totals::Grouped) {
      std::vector<std::pair<GroupKey, AggState>> gs(totals.groups.begin(), totals.groups.end());
      std::sort(gs.begin(), gs.end(),
                [](const auto &a, const auto &b) { return a.first < b.first; });
      writer.groups(group_key_name(program), program.output.agg, gs);
    }
  }
  stats.lines_out = writer.rows;
  result = writer.finish();
  return 0;
}

}  // namespace oracle
