// Host driver of the GPU backend: the role the reference's Rust host plays
// around the device ABI (crates/warpjq-core/src/gpu/mod.rs:244-1259 and the
// formatting of agg.rs / output.rs / exec/mod.rs).
//
// It splits the input into newline-aligned chunks, keeps two device slots in
// flight (fill n+1 while n computes), merges every chunk's rows and
// aggregates in input order, and formats the output bytes.  There is no CPU
// evaluation of any line: every line of every chunk is decided on the device.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <cerrno>
#include <charconv>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../../include/warpjq_ext.h"
#include "../../../include/warpjq_host.h"

// The extension entry points are optional: with a backend that exports only
// the reference ABI (warpjq_kernels.h) the driver runs without them.
#pragma weak warpjq_autotile
#pragma weak warpjq_submit_host
#pragma weak warpjq_host_is_pinned
#pragma weak warpjq_slot_first_errors
#pragma weak warpjq_host_alloc_pinned
#pragma weak warpjq_host_free_pinned
#pragma weak warpjq_launch_device
#pragma weak warpjq_collect_device
#pragma weak warpjq_csv_create
#pragma weak warpjq_csv_destroy
#pragma weak warpjq_csv_reset
#pragma weak warpjq_csv_convert
#pragma weak warpjq_csv_gather
#pragma weak warpjq_csv_stage
#pragma weak warpjq_csv_stage_wait
#pragma weak warpjq_csv_carry
#pragma weak warpjq_device_read
#include "query.h"

namespace wjqh {

// ---------------------------------------------------------------------------
// Number formatting and value rendering (agg.rs:253-278, output.rs:24-81)
// ---------------------------------------------------------------------------

// Integral values below 2^53 print as integers; others print their shortest
// round-trip digits, placed as the `ryu` crate's pretty printer places them,
// with an explicit `+` on positive exponents.
std::string format_number(double v) {
  if (std::isnan(v)) return "null";
  if (std::isinf(v)) return v > 0 ? "1.7976931348623157e+308" : "-1.7976931348623157e+308";
  if (std::trunc(v) == v && std::fabs(v) < 9007199254740992.0) return std::to_string((long long)v);
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string s(buf, r.ptr), digits;
  bool neg = s[0] == '-';
  size_t e = s.find('e');
  for (size_t k = neg; k < e; k++)
    if (s[k] != '.') digits += s[k];
  long exp10 = std::strtol(s.c_str() + e + 1, nullptr, 10);
  long len = (long)digits.size(), kk = exp10 + 1, k = kk - len;
  std::string o = neg ? "-" : "";
  if (k >= 0 && kk <= 16) {
    o += digits + std::string((size_t)k, '0') + ".0";
  } else if (kk > 0 && kk <= 16) {
    o += digits.substr(0, (size_t)kk) + "." + digits.substr((size_t)kk);
  } else if (kk > -5 && kk <= 0) {
    o += "0." + std::string((size_t)-kk, '0') + digits;
  } else {
    o += digits.substr(0, 1);
    if (len > 1) o += "." + digits.substr(1);
    o += "e" + std::string(kk - 1 >= 0 ? "+" : "") + std::to_string(kk - 1);
  }
  return o;
}

void json_string(std::string &o, const uint8_t *p, size_t n) {
  o += '"';
  for (size_t i = 0; i < n; i++) {
    uint8_t c = p[i];
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

void csv_cell(std::string &o, const uint8_t *p, size_t n) {
  bool q = false;
  for (size_t i = 0; i < n && !q; i++) q = p[i] == ',' || p[i] == '"' || p[i] == '\n' || p[i] == '\r';
  if (!q) {
    o.append((const char *)p, n);
    return;
  }
  o += '"';
  for (size_t i = 0; i < n; i++) {
    if (p[i] == '"') o += '"';
    o += (char)p[i];
  }
  o += '"';
}

// Decodes a validated JSON string body (json.rs:594-654).
std::string unescape(const uint8_t *p, size_t n) {
  std::string o;
  auto hex4 = [&](size_t at) {
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) {
      uint8_t c = p[at + k];
      v = v * 16 + (c <= '9' ? c - '0' : (c | 0x20) - 'a' + 10);
    }
    return v;
  };
  for (size_t i = 0; i < n;) {
    if (p[i] != '\\') {
      o += (char)p[i++];
      continue;
    }
    uint8_t e = p[i + 1];
    i += 2;
    if (e != 'u') {
      const char *from = "\"\\/bfnrt", *to = "\"\\/\b\f\n\r\t";
      o += to[strchr(from, e) - from];
      continue;
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
    if (cp < 0x80) o += (char)cp;
    else if (cp < 0x800) {
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
  return o;
}

// ---------------------------------------------------------------------------
// Aggregation state and group keys (agg.rs:17-249)
// ---------------------------------------------------------------------------

struct Agg {
  uint64_t count = 0, numeric = 0;
  double sum = 0, min = INFINITY, max = -INFINITY;
  void merge(uint64_t c, uint64_t nu, double s, double mn, double mx) {
    count += c;
    numeric += nu;
    sum += s;
    if (mn < min) min = mn;
    if (mx > max) max = mx;
  }
  bool finish(uint32_t kind, double &v) const {
    switch (kind) {
      case WARPJQ_AGG_COUNT: v = (double)count; return true;
      case WARPJQ_AGG_SUM: v = sum; return true;
      case WARPJQ_AGG_MIN: v = min; return numeric > 0;
      case WARPJQ_AGG_MAX: v = max; return numeric > 0;
      default: v = sum / (double)numeric; return numeric > 0;
    }
  }
};

uint64_t order_bits(double v) {
  uint64_t b;
  memcpy(&b, &v, 8);
  return (b >> 63) ? ~b : (b ^ (1ull << 63));
}

// rank: 0 null, 1 false, 2 true, 3 number, 4 string, 5 array/object
struct GroupKey {
  uint8_t rank = 0;
  std::string bytes;
  uint64_t bits = 0;
  bool operator==(const GroupKey &o) const { return rank == o.rank && bytes == o.bytes; }
  // jq order; equal numbers with different spellings tie-break on the text.
  bool operator<(const GroupKey &o) const {
    if (rank != o.rank) return rank < o.rank;
    if (rank == 3 && bits != o.bits) return bits < o.bits;
    return bytes < o.bytes;
  }
  std::string json() const {
    if (rank == 0) return "null";
    if (rank == 1) return "false";
    if (rank == 2) return "true";
    if (rank == 4) {
      std::string o;
      json_string(o, (const uint8_t *)bytes.data(), bytes.size());
      return o;
    }
    return bytes;
  }
  std::string plain() const { return rank == 4 ? bytes : json(); }
};
struct KeyHash {
  size_t operator()(const GroupKey &k) const { return std::hash<std::string>()(k.bytes) ^ k.rank; }
};

// Rebuilds a key from a device group entry (gpu/mod.rs:1198-1221).
GroupKey device_key(const uint8_t *data, uint64_t off, uint32_t len, uint32_t kind) {
  GroupKey k;
  const uint8_t *raw = data + off;
  switch (kind) {
    case 0: case 1: k.rank = 0; break;
    case 2: k.rank = (len == 4 && memcmp(raw, "true", 4) == 0) ? 2 : 1; break;
    case 3: {
      k.rank = 3;
      k.bytes.assign((const char *)raw, len);
      k.bits = order_bits(strtod(k.bytes.c_str(), nullptr));
      break;
    }
    case 4:
      k.rank = 4;
      k.bytes = memchr(raw, '\\', len) ? unescape(raw, len) : std::string((const char *)raw, len);
      break;
    default:
      k.rank = 5;
      k.bytes.assign((const char *)raw, len);
  }
  return k;
}

// ---------------------------------------------------------------------------
// Output writer (output.rs:87-334)
// ---------------------------------------------------------------------------

// Growable malloc'd byte buffer for row output: realloc grows big blocks
// in place (remapped pages), and the finished buffer is handed to the
// caller without another copy.
struct Bytes {
  char *p = nullptr;
  size_t n = 0, cap = 0;
  ~Bytes() { free(p); }
  bool reserve(size_t want) {
    if (want <= cap) return true;
    char *q = (char *)realloc(p, want);
    if (!q) return false;
    p = q;
    cap = want;
    return true;
  }
  bool append(const void *src, size_t k) {
    if (n + k + 1 > cap && !reserve(std::max(n + k + 1, cap * 2))) return false;
    memcpy(p + n, src, k);
    n += k;
    return true;
  }
  char *release() {
    char *q = p;
    p = nullptr;
    n = cap = 0;
    return q;
  }
};

struct Writer {
  std::string buf;   // text output (header, aggregates, groups)
  Bytes bulk_rows;   // row output, after any header text
  bool oom = false;
  uint32_t fmt;  // WARPJQ_FMT_*
  uint64_t rows = 0;
  void header(const Program &p) {
    if (fmt != WARPJQ_FMT_CSV) return;
    std::vector<std::string> cols;
    if (!p.csv_headers(cols)) return;
    for (size_t i = 0; i < cols.size(); i++) {
      if (i) buf += ',';
      csv_cell(buf, (const uint8_t *)cols[i].data(), cols[i].size());
    }
    buf += '\n';
  }
  void bulk(const uint8_t *p, size_t n, uint64_t r) {
    rows += r;
    if (fmt == WARPJQ_FMT_COUNT) return;
    if (!bulk_rows.p && !buf.empty()) {
      oom |= !bulk_rows.append(buf.data(), buf.size());
      buf.clear();
    }
    oom |= !bulk_rows.append(p, n);
  }
  // Expected total row bytes, from the share of the input done so far.
  void reserve_rows(size_t total) {
    if (total > bulk_rows.cap) oom |= !bulk_rows.reserve(total + 1);
  }
  void aggregate(uint32_t kind, const Agg &a) {
    rows++;
    double v;
    std::string val = a.finish(kind, v) ? format_number(v) : "null";
    if (fmt == WARPJQ_FMT_COUNT) {
      rows = 0;
      buf = val + "\n";
      fmt = WARPJQ_FMT_NDJSON;
      return;
    }
    buf += val + "\n";
  }
  void groups(const std::string &name, uint32_t kind, const std::vector<std::pair<GroupKey, Agg>> &gs) {
    for (auto &g : gs) {
      rows++;
      double v;
      std::string val = g.second.finish(kind, v) ? format_number(v) : "null";
      if (fmt == WARPJQ_FMT_CSV) {
        std::string pl = g.first.plain();
        csv_cell(buf, (const uint8_t *)pl.data(), pl.size());
        buf += "," + val;
      } else {
        buf += '{';
        json_string(buf, (const uint8_t *)name.data(), name.size());
        buf += ':' + g.first.json() + ',';
        const char *an = agg_name(kind);
        json_string(buf, (const uint8_t *)an, strlen(an));
        buf += ':' + val + '}';
      }
      buf += '\n';
    }
  }
  // Hands the output to the caller as one malloc'd, NUL-terminated buffer.
  char *finish(size_t &len) {
    if (fmt == WARPJQ_FMT_COUNT) buf = std::to_string(rows) + "\n";
    if (bulk_rows.p) {
      if (!buf.empty()) oom |= !bulk_rows.append(buf.data(), buf.size());
      oom |= !bulk_rows.reserve(bulk_rows.n + 1);
      if (oom) return nullptr;
      bulk_rows.p[bulk_rows.n] = 0;
      len = bulk_rows.n;
      return bulk_rows.release();
    }
    char *o = (char *)malloc(buf.size() + 1);
    if (!o) return nullptr;
    memcpy(o, buf.data(), buf.size());
    o[buf.size()] = 0;
    len = buf.size();
    return o;
  }
};

}  // namespace wjqh

using namespace wjqh;

// A fixed set of threads for parallel reads: run(n, f) calls f(0..n-1) on
// the workers and returns when all have finished.
struct ReadPool {
  std::vector<std::thread> ws;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::function<void(unsigned)> job;
  unsigned n_jobs = 0, next_job = 0, done = 0;
  bool stop = false;
  explicit ReadPool(unsigned n) {
    for (unsigned t = 0; t < n; t++)
      ws.emplace_back([this] {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
          cv.wait(lk, [&] { return stop || next_job < n_jobs; });
          if (stop) return;
          const unsigned j = next_job++;
          lk.unlock();
          job(j);
          lk.lock();
          if (++done == n_jobs) done_cv.notify_all();
        }
      });
  }
  void run(unsigned n, std::function<void(unsigned)> f) {
    std::unique_lock<std::mutex> lk(mu);
    job = std::move(f);
    next_job = 0;
    done = 0;
    n_jobs = n;
    cv.notify_all();
    done_cv.wait(lk, [&] { return done == n_jobs; });
    n_jobs = 0;
  }
  ~ReadPool() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    for (auto &w : ws) w.join();
  }
};

struct warpjq_query {
  Program prog;
  Lowered low;
  uint32_t fmt = WARPJQ_FMT_NDJSON;
  warpjq_ctx *ctx = nullptr;
  uint64_t cap = 0;
  uint32_t n_slots = 2;
  bool tiled = false;  // device tiling chosen from the first bytes of a run
  // file input: read buffers (page-locked when `rpinned`) and read threads,
  // kept across runs
  std::vector<uint8_t *> rbufs;
  std::vector<uint64_t> rcaps;
  bool rpinned = false;
  std::unique_ptr<ReadPool> pool;
  // CSV input: the converter and, for input that is not page-locked, two
  // page-locked buffers its chunks are copied through
  warpjq_csv *csv = nullptr;
  uint8_t *csv_pin[2] = {nullptr, nullptr};
  uint64_t csv_pin_cap[2] = {0, 0};
  void free_read_bufs() {
    for (auto &b : rbufs) {
      if (!b) continue;
      if (rpinned) warpjq_host_free_pinned(b);
      else free(b);
    }
    rbufs.clear();
    rcaps.clear();
  }
  ~warpjq_query() {
    free_read_bufs();
    for (auto &b : csv_pin)
      if (b) warpjq_host_free_pinned(b);
    if (csv) warpjq_csv_destroy(csv);
  }
};

namespace {

void put_err(char *err, size_t n, const std::string &m) {
  if (!err || !n) return;
  size_t k = std::min(m.size(), n - 1);
  memcpy(err, m.data(), k);
  err[k] = 0;
}

// Copies into pinned memory with several threads (gpu/mod.rs:934-956).
void copy_to_pinned(uint8_t *dst, const uint8_t *src, size_t n) {
  const size_t kMin = 1 << 20;
  unsigned t = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 16);
  if (n < kMin || t == 1) {
    memcpy(dst, src, n);
    return;
  }
  size_t piece = (n + t - 1) / t;
  std::vector<std::thread> ws;
  for (unsigned i = 0; i < t; i++) {
    size_t a = i * piece, b = std::min(n, a + piece);
    if (a >= b) break;
    ws.emplace_back([=] { memcpy(dst + a, src + a, b - a); });
  }
  for (auto &w : ws) w.join();
}

struct Totals {
  Agg scalar;
  std::unordered_map<GroupKey, Agg, KeyHash> groups;
};

}  // namespace

extern "C" {

void warpjq_host_free(void *p) { free(p); }

// Parse and lowering, shared by both opens.
static int open_parsed(const char *query, uint32_t format, warpjq_query **out, char *err,
                       size_t err_len) {
  *out = nullptr;
  auto *q = new warpjq_query();
  QueryError qe;
  std::string src = query ? query : "";
  if (!parse(src, q->prog, qe)) {
    put_err(err, err_len, qe.render(src));
    delete q;
    return 2;
  }
  if (format == WARPJQ_FMT_CSV && q->prog.out == Out::Passthrough) {  // exec/mod.rs:256-266
    put_err(err, err_len,
            "--csv needs a query with named columns, but this one emits whole lines\n  help: project "
            "the fields you want, e.g. `{ts: .ts, status: .status}`, or use an aggregate");
    delete q;
    return 1;
  }
  q->fmt = format;
  q->low.build(q->prog, format == WARPJQ_FMT_CSV);
  *out = q;
  return 0;
}

int warpjq_query_open_host(const char *query, uint32_t format, warpjq_query **out, char *err,
                           size_t err_len) {
  return open_parsed(query, format, out, err, err_len);
}

int warpjq_query_is_grouped(const warpjq_query *q) { return q && q->prog.has_group; }

int warpjq_query_open(const char *query, uint32_t format, uint64_t chunk_bytes, warpjq_query **out,
                      char *err, size_t err_len) {
  *out = nullptr;
  warpjq_query *q = nullptr;
  int prc = open_parsed(query, format, &q, err, err_len);
  if (prc) return prc;
  // gpu/mod.rs:143-145: the GPU chunk is capped at 64 MiB.
  uint64_t cap = chunk_bytes ? chunk_bytes : (256ull << 20);
  cap = std::min<uint64_t>(cap, std::max<uint64_t>(64ull << 20, 1 << 20));
  q->cap = std::max<uint64_t>(cap, 1);
  char e[512] = {0};
  warpjq_status rc = warpjq_ctx_create(&q->low.prog, q->cap, q->n_slots, &q->ctx, e, sizeof e);
  if (rc != WARPJQ_OK) {
    put_err(err, err_len, std::string("CUDA error in creating the device context: ") + e);
    delete q;
    return 1;
  }
  *out = q;
  return 0;
}

void warpjq_query_close(warpjq_query *q) {
  if (!q) return;
  if (q->ctx) warpjq_ctx_destroy(q->ctx);
  delete q;
}

warpjq_ctx *warpjq_query_ctx(warpjq_query *q) { return q ? q->ctx : nullptr; }

int warpjq_query_is_aggregate(const warpjq_query *q) { return q && q->prog.is_aggregate(); }

// One newline-aligned chunk of input, at host address `data`; `pinned` when
// it is page-locked (copied to the device straight from there).
struct Chunk {
  const uint8_t *data = nullptr;
  uint64_t n = 0;
  bool pinned = false;
};

// The run loop shared by memory and file input: `next` yields chunks (false
// at the end; a nonempty error message stops the run), `total` is the input
// size (for sizing the output), `sample` the input's first bytes (for the
// tiling).  A chunk's bytes must stay valid until the chunk after the next
// one has been asked for.
static int run_chunks(warpjq_query *q, uint64_t total, const uint8_t *sample, size_t sample_len,
                      const std::function<bool(Chunk &, std::string &)> &next, const char *name,
                      uint32_t on_invalid, uint64_t max_line_bytes, char **out, size_t *out_len,
                      uint64_t *stats, char *err, size_t err_len) {
  *out = nullptr;
  if (out_len) *out_len = 0;
  if (!max_line_bytes) max_line_bytes = 64ull << 20;
  const Program &P = q->prog;
  Writer w;
  w.fmt = q->fmt;
  w.header(P);
  Totals tot;
  uint64_t st_lines = 0, st_malformed = 0, st_type = 0, lines_seen = 0, done_bytes = 0;
  char e[512] = {0};

  struct Flight {
    uint32_t slot;
    const uint8_t *data;
    uint64_t n;
  };
  std::vector<Flight> flight;
  uint32_t next_slot = 0;

  auto fail = [&](const std::string &m) {
    put_err(err, err_len, m);
    return 1;
  };

  bool reserved = false;
  auto drain = [&](const Flight &f) -> int {
    warpjq_chunk_result r;
    warpjq_status rc = warpjq_wait(q->ctx, f.slot, &r, e, sizeof e);
    if (rc != WARPJQ_OK) return fail(std::string("CUDA error in waiting for a chunk: ") + e);
    // A backend that leaves lines or groups to the host is not supported by
    // this driver (this project's backend never does).
    if (r.n_fallback || r.chunk_overflow || r.group_overflow)
      return fail("the device backend left work to the host (fallback lines or an overflow), "
                  "which this driver does not finish");
    uint64_t first_line = lines_seen + 1;
    lines_seen += r.n_lines;
    st_lines += r.n_lines - r.n_blank;
    st_malformed += r.n_invalid;
    st_type += r.n_type_error;
    done_bytes += f.n;
    if (on_invalid == WARPJQ_ON_INVALID_ABORT && (r.n_invalid || r.n_type_error)) {
      uint64_t fi = r.first_invalid == 0xFFFFFFFFu ? ~0ull : r.first_invalid;
      uint64_t ft = ~0ull, dummy = 0;
      if (warpjq_slot_first_errors) warpjq_slot_first_errors(q->ctx, f.slot, &dummy, &ft);
      uint64_t bad = std::min(fi, ft);
      return fail("malformed JSON on line " + std::to_string(first_line + (bad == ~0ull ? 0 : bad)) +
                  " of " + name + ": " +
                  (fi <= ft ? "line is not valid JSON" : "a path hit a value of the wrong type") +
                  "\n  help: pass --skip-invalid to drop bad lines instead of stopping");
    }
    if (P.is_aggregate()) {
      if (!P.has_group) {
        tot.scalar.merge(r.agg.count, r.agg.numeric, r.agg.sum, r.agg.min, r.agg.max);
      } else {
        for (uint32_t k = 0; k < r.n_groups; k++) {
          const warpjq_group &g = r.groups[k];
          GroupKey key = device_key(f.data, g.key_off, g.key_len, g.key_kind);
          tot.groups[key].merge(g.count, g.numeric, g.sum, g.min, g.max);
        }
      }
    } else if (r.n_selected) {
      w.bulk(r.out_bytes + r.out_row_off[0], (size_t)(r.out_row_off[r.n_selected] - r.out_row_off[0]),
             r.n_selected);
      // Size the output once from the first chunk's share of it.
      if (!reserved && done_bytes < total) {
        w.reserve_rows((size_t)((double)w.bulk_rows.n * (double)total / (double)done_bytes * 1.05));
        reserved = true;
      }
    }
    if (w.oom) return fail("out of host memory for the output");
    return 0;
  };

  // Tiles sized from the input's own line lengths (its first MiB).
  auto tile = [&]() -> bool {
    return !warpjq_autotile || !sample_len ||
           warpjq_autotile(q->ctx, sample, std::min<uint64_t>(sample_len, 1ull << 20), nullptr,
                           nullptr) == WARPJQ_OK;
  };
  if (!q->tiled) {
    if (!tile()) return fail("CUDA error in choosing the device tiling");
    q->tiled = true;
  }
  Chunk c;
  std::string why;
  while (next(c, why)) {
    const uint64_t n = c.n;
    // --max-line-bytes (chunk.rs:259-270): only a chunk without any newline
    // but its last byte can hold an over-long line.
    if (n > max_line_bytes) {
      const uint8_t *inner = (const uint8_t *)memchr(c.data, '\n', n - 1 > 0 ? n - 1 : 0);
      if (!inner)
        return fail("line " + std::to_string(lines_seen + 1) + " is at least " + std::to_string(n) +
                    " bytes, over the " + std::to_string(max_line_bytes) +
                    " byte limit (raise it with --max-line-bytes)");
    }
    if (n > q->cap) {  // one line longer than a slot: grow the slots to hold it
      for (auto &f : flight)
        if (drain(f)) return 1;
      flight.clear();
      warpjq_ctx_destroy(q->ctx);
      q->ctx = nullptr;
      q->cap = n;
      if (warpjq_ctx_create(&q->low.prog, q->cap, q->n_slots, &q->ctx, e, sizeof e) != WARPJQ_OK)
        return fail(std::string("CUDA error in creating the device context: ") + e);
      if (!tile()) return fail("CUDA error in choosing the device tiling");
      next_slot = 0;
    }
    uint32_t slot = next_slot;
    next_slot = (next_slot + 1) % q->n_slots;
    // The slot being refilled must have been drained (two slots: n and n-2).
    if (flight.size() >= q->n_slots) {
      if (drain(flight.front())) return 1;
      flight.erase(flight.begin());
    }
    warpjq_status sub;
    if (c.pinned && warpjq_submit_host) {
      sub = warpjq_submit_host(q->ctx, slot, c.data, n, e, sizeof e);
    } else {
      copy_to_pinned(warpjq_slot_buffer(q->ctx, slot), c.data, n);
      sub = warpjq_submit(q->ctx, slot, n, e, sizeof e);
    }
    if (sub != WARPJQ_OK) return fail(std::string("CUDA error in submitting a chunk: ") + e);
    flight.push_back({slot, c.data, n});
    if (flight.size() > 1) {
      if (drain(flight.front())) return 1;
      flight.erase(flight.begin());
    }
  }
  if (!why.empty()) return fail(why);
  for (auto &f : flight)
    if (drain(f)) return 1;

  // exec/mod.rs:321-339
  if (P.is_aggregate()) {
    if (!P.has_group) {
      w.aggregate(P.agg, tot.scalar);
    } else {
      std::vector<std::pair<GroupKey, Agg>> gs(tot.groups.begin(), tot.groups.end());
      std::sort(gs.begin(), gs.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
      w.groups(P.group_key_name(), P.agg, gs);
    }
  }
  uint64_t rows = w.rows;
  size_t res_len = 0;
  char *res = w.finish(res_len);
  if (!res) return fail("out of host memory for the output");
  if (stats) {
    stats[0] = total;
    stats[1] = st_lines;
    stats[2] = rows;
    stats[3] = st_malformed;
    stats[4] = st_type;
  }
  *out = res;
  if (out_len) *out_len = res_len;
  return 0;
}

int warpjq_query_run(warpjq_query *q, const uint8_t *data, size_t len, uint32_t on_invalid,
                     uint64_t max_line_bytes, char **out, size_t *out_len, uint64_t *stats,
                     char *err, size_t err_len) {
  // Strip a UTF-8 byte-order mark (chunk.rs:210-212).
  size_t pos = (len >= 3 && data[0] == 0xEF && data[1] == 0xBB && data[2] == 0xBF) ? 3 : 0;
  // Page-locked input is copied to the device straight from the caller's
  // memory; anything else is staged through the slots' pinned buffers.
  const bool pinned = len && warpjq_host_is_pinned && warpjq_submit_host &&
                      warpjq_host_is_pinned(data) && warpjq_host_is_pinned(data + len - 1);
  auto next = [&](Chunk &c, std::string &) -> bool {
    if (pos >= len) return false;
    // Next newline-aligned chunk of at most `cap` bytes (chunk.rs:234-278).
    uint64_t end = pos + std::min<uint64_t>(q->cap, len - pos);
    if (end < len) {
      const uint8_t *nl = nullptr;
      for (uint64_t k = end; k > pos; k--)
        if (data[k - 1] == '\n') {
          nl = data + k - 1;
          break;
        }
      if (nl) {
        end = (uint64_t)(nl - data) + 1;
      } else {  // one line longer than a slot
        const uint8_t *n2 = (const uint8_t *)memchr(data + end, '\n', len - end);
        end = n2 ? (uint64_t)(n2 - data) + 1 : len;
      }
    }
    c.data = data + pos;
    c.n = end - pos;
    c.pinned = pinned;
    pos = end;
    return true;
  };
  return run_chunks(q, len, data, len, next, "<memory>", on_invalid, max_line_bytes, out, out_len,
                    stats, err, err_len);
}

int warpjq_query_run_file(warpjq_query *q, const char *path, uint32_t on_invalid,
                          uint64_t max_line_bytes, char **out, size_t *out_len, uint64_t *stats,
                          char *err, size_t err_len) {
  *out = nullptr;
  const int fd = open(path, O_RDONLY);
  if (fd < 0) {
    put_err(err, err_len, std::string("cannot open ") + path + ": " + strerror(errno));
    return 1;
  }
  struct stat sb;
  if (fstat(fd, &sb) != 0) {
    put_err(err, err_len, std::string("cannot stat ") + path + ": " + strerror(errno));
    close(fd);
    return 1;
  }
  const uint64_t size = (uint64_t)sb.st_size;
  // Three buffers, kept with the query across runs: the chunk being read,
  // and the two the device may still be working on.  A chunk is filled up to
  // the context's slot size (a larger one would make the run loop grow the
  // context); only a longer line grows a buffer.  Page-locked when the
  // backend provides it (chunks then go to the device straight from them).
  const bool can_pin = warpjq_host_alloc_pinned && warpjq_host_free_pinned;
  auto host_alloc = [&](uint64_t n) -> uint8_t * {
    return can_pin ? (uint8_t *)warpjq_host_alloc_pinned(n) : (uint8_t *)malloc(n);
  };
  auto host_free = [&](uint8_t *b) {
    if (can_pin) warpjq_host_free_pinned(b);
    else free(b);
  };
  const uint64_t bufcap = std::max<uint64_t>(q->cap, 1 << 16);
  if (q->rbufs.size() != 3 || q->rpinned != can_pin) {
    q->free_read_bufs();
    q->rpinned = can_pin;
    q->rbufs.assign(3, nullptr);
    q->rcaps.assign(3, 0);
  }
  for (size_t i = 0; i < 3; i++) {
    if (q->rbufs[i] && q->rcaps[i] >= bufcap) continue;
    if (q->rbufs[i]) host_free(q->rbufs[i]);
    q->rbufs[i] = host_alloc(bufcap);
    q->rcaps[i] = bufcap;
    if (!q->rbufs[i]) {
      q->free_read_bufs();
      close(fd);
      put_err(err, err_len, "cannot allocate read buffers");
      return 1;
    }
  }
  std::vector<uint8_t *> &bufs = q->rbufs;
  std::vector<uint64_t> &caps = q->rcaps;
  const unsigned threads = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 16);
  uint64_t pos = 0;          // file offset of the next byte to read
  uint64_t carry_len = 0;    // bytes of a partial line waiting in `carry_from`
  const uint8_t *carry_from = nullptr;
  uint32_t k = 0;
  std::vector<uint8_t> sample;
  {  // the first MiB, for the tiling
    sample.resize(std::min<uint64_t>(size, 1 << 20));
    if (!sample.empty() && pread(fd, sample.data(), sample.size(), 0) != (ssize_t)sample.size())
      sample.clear();
  }
  if (!q->pool) q->pool.reset(new ReadPool(threads));
  // Reads [off, off + n) into dst with parallel preads.
  auto read_range = [&](uint8_t *dst, uint64_t off, uint64_t n) -> bool {
    if (n == 0) return true;
    const uint64_t piece = std::max<uint64_t>((n + threads - 1) / threads, 1 << 20);
    const unsigned parts = (unsigned)((n + piece - 1) / piece);
    std::atomic<bool> ok{true};
    q->pool->run(parts, [&](unsigned j) {
      const uint64_t a = (uint64_t)j * piece, b = std::min(n, a + piece);
      for (uint64_t at = a; at < b;) {
        const ssize_t got = pread(fd, dst + at, b - at, (off_t)(off + at));
        if (got <= 0) {
          ok = false;
          return;
        }
        at += (uint64_t)got;
      }
    });
    return ok;
  };
  auto grow = [&](uint32_t bi, uint64_t keep) -> bool {
    uint8_t *big = host_alloc(caps[bi] * 2);
    if (!big) return false;
    if (keep) memcpy(big, bufs[bi], keep);
    host_free(bufs[bi]);
    bufs[bi] = big;
    caps[bi] *= 2;
    return true;
  };
  auto next = [&](Chunk &c, std::string &why) -> bool {
    if (pos >= size && carry_len == 0) return false;
    const uint32_t bi = k % 3;
    // The partial line carried over first (from the buffer of the chunk
    // before, which the device does not read past that chunk's end).
    while (caps[bi] < carry_len + 1)
      if (!grow(bi, 0)) {
        why = "cannot allocate page-locked read buffers";
        return false;
      }
    if (carry_len) memmove(bufs[bi], carry_from, carry_len);
    uint64_t have = carry_len;
    // Fill up to the context's slot size (a larger chunk would make the run
    // loop grow the context); read on past it only for a longer line.
    uint64_t limit = std::max<uint64_t>(std::min<uint64_t>(caps[bi], std::max<uint64_t>(q->cap, 1 << 16)),
                                        have + 1);
    for (;;) {
      const bool at_start = pos == 0;
      const uint64_t want = std::min<uint64_t>(limit - have, size - pos);
      if (!read_range(bufs[bi] + have, pos, want)) {
        why = std::string("read error on ") + path;
        return false;
      }
      pos += want;
      have += want;
      uint8_t *buf = bufs[bi];
      if (at_start && have >= 3 && buf[0] == 0xEF && buf[1] == 0xBB && buf[2] == 0xBF) {
        memmove(buf, buf + 3, have - 3);  // a UTF-8 byte-order mark (chunk.rs:210-212)
        have -= 3;
      }
      if (pos >= size) {  // the rest of the file
        c.data = buf;
        c.n = have;
        c.pinned = can_pin;
        carry_len = 0;
        break;
      }
      uint64_t end = have;
      while (end > 0 && buf[end - 1] != '\n') end--;
      if (end > 0) {
        c.data = buf;
        c.n = end;
        c.pinned = can_pin;
        carry_from = buf + end;
        carry_len = have - end;
        break;
      }
      // No newline yet: a line longer than a chunk.  Read on, growing the
      // buffer when it is full (the bytes read so far move with it).
      if (have == caps[bi] && !grow(bi, have)) {
        why = "cannot allocate page-locked read buffers";
        return false;
      }
      limit = caps[bi];
    }
    k++;
    return c.n > 0;
  };
  int rc = run_chunks(q, size, sample.data(), sample.size(), next, path, on_invalid, max_line_bytes,
                      out, out_len, stats, err, err_len);
  close(fd);
  return rc;
}

// CSV input (warpjq_host.h): chunks of the input are converted to NDJSON on
// the device (warpjq_csv_convert) and scanned there (warpjq_launch_device),
// one chunk at a time; rows and aggregates merge in input order as for
// NDJSON, and group keys are gathered from the device copy.
int warpjq_query_run_csv(warpjq_query *q, const uint8_t *data, size_t len, uint32_t on_invalid,
                         char **out, size_t *out_len, uint64_t *stats, char *err, size_t err_len) {
  *out = nullptr;
  if (out_len) *out_len = 0;
  auto fail = [&](const std::string &m) {
    put_err(err, err_len, m);
    return 1;
  };
  if (!warpjq_csv_convert || !warpjq_csv_stage || !warpjq_csv_carry || !warpjq_launch_device ||
      !warpjq_collect_device || !warpjq_host_alloc_pinned)
    return fail("this device backend has no CSV input");
  if (!q->ctx) return fail("the query has no device context");
  if (!q->csv && warpjq_csv_create(&q->csv) != WARPJQ_OK) return fail("out of memory for the CSV converter");
  warpjq_csv_reset(q->csv);
  const Program &P = q->prog;
  Writer w;
  w.fmt = q->fmt;
  w.header(P);
  Totals tot;
  uint64_t st_lines = 0, st_malformed = 0, st_type = 0, records = 0;
  char e[512] = {0};
  const bool pinned = len && warpjq_host_is_pinned && warpjq_host_is_pinned(data) &&
                      warpjq_host_is_pinned(data + len - 1);
  uint64_t cap = std::max<uint64_t>(q->cap, 1 << 20);
  std::vector<uint64_t> k_off;
  std::vector<uint32_t> k_len;
  std::vector<uint8_t> k_bytes, rows;
  // Chunk k on the device: the row carried over from chunk k - 1 (`carry`
  // bytes just below offset `room` of its staging buffer), then its new
  // bytes from `room` on.  Chunk k + 1's new bytes are copied to the other
  // staging buffer while chunk k is converted and scanned.
  uint64_t room = 64 << 10;
  auto host_bytes = [&](uint32_t x, uint64_t hpos, uint64_t n, const uint8_t **src) -> bool {
    if (pinned || !n) {
      *src = data + hpos;
      return true;
    }
    if (q->csv_pin_cap[x] < n) {
      if (q->csv_pin[x]) warpjq_host_free_pinned(q->csv_pin[x]);
      const uint64_t want = std::max<uint64_t>(n, cap);
      q->csv_pin[x] = (uint8_t *)warpjq_host_alloc_pinned(want);
      q->csv_pin_cap[x] = q->csv_pin[x] ? want : 0;
      if (!q->csv_pin[x]) return false;
    }
    copy_to_pinned(q->csv_pin[x], data + hpos, n);
    *src = q->csv_pin[x];
    return true;
  };
  uint8_t *dbuf[2] = {nullptr, nullptr};
  auto stage = [&](uint32_t x, uint64_t at, uint64_t hpos, uint64_t n) -> int {
    const uint8_t *hs = nullptr;
    if (!host_bytes(x, hpos, n, &hs)) return fail("out of page-locked host memory for the CSV input");
    if (warpjq_csv_stage(q->csv, x, at, hs, n, &dbuf[x], e, sizeof e) != WARPJQ_OK)
      return fail(std::string("CUDA error in copying CSV to the device: ") + e);
    return 0;
  };
  uint64_t pos = 0, carry = 0, n_new = std::min<uint64_t>(cap, len);
  uint32_t b = 0;
  if (len && stage(0, room, 0, n_new)) return 1;
  while (len) {
    const uint64_t next = pos + n_new;
    const bool final_ = next == len;
    const uint64_t n_next = final_ ? 0 : std::min<uint64_t>(cap, len - next);
    if (!final_ && stage(b ^ 1, room, next, n_next)) return 1;
    const uint8_t *src = dbuf[b] + room - carry;
    const uint64_t n = carry + n_new;
    const uint8_t *d_nd = nullptr;
    uint64_t nd_len = 0, used = 0, recs = 0;
    if (warpjq_csv_convert(q->csv, src, n,
                           (final_ ? WARPJQ_CSV_FINAL : 0u) | (b ? WARPJQ_CSV_AFTER_STAGE1 : WARPJQ_CSV_AFTER_STAGE0),
                           nullptr, &d_nd, &nd_len, &used, &recs, e, sizeof e) != WARPJQ_OK)
      return fail(std::string("CUDA error in converting CSV: ") + e);
    if (nd_len && !q->tiled && warpjq_autotile) {  // tiles shaped by the converted lines
      std::vector<uint8_t> sample((size_t)std::min<uint64_t>(nd_len, 1 << 20));
      if (warpjq_device_read(sample.data(), d_nd, sample.size(), nullptr, e, sizeof e) != WARPJQ_OK ||
          warpjq_autotile(q->ctx, sample.data(), sample.size(), nullptr, nullptr) != WARPJQ_OK)
        return fail("CUDA error in choosing the device tiling");
      q->tiled = true;
    }
    if (nd_len) {
      warpjq_device_result r;
      if (warpjq_launch_device(q->ctx, d_nd, nd_len, nullptr, e, sizeof e) != WARPJQ_OK ||
          warpjq_collect_device(q->ctx, &r, e, sizeof e) != WARPJQ_OK)
        return fail(std::string("CUDA error in scanning converted CSV: ") + e);
      st_lines += r.n_lines - r.n_blank;
      st_malformed += r.n_invalid;
      st_type += r.n_type_error;
      if (on_invalid == WARPJQ_ON_INVALID_ABORT && (r.n_invalid || r.n_type_error)) {
        const uint64_t bad = std::min(r.first_invalid, r.first_type_error);
        return fail("bad value in CSV row " + std::to_string(records + bad + 1) + " (after the header): " +
                    (r.first_invalid <= r.first_type_error ? "row is not valid JSON once converted"
                                                           : "a path hit a value of the wrong type") +
                    "\n  help: pass --skip-invalid to drop bad rows instead of stopping");
      }
      if (P.is_aggregate()) {
        if (!P.has_group) {
          tot.scalar.merge(r.count, r.numeric, r.sum, r.min, r.max);
        } else if (r.n_groups) {
          k_off.resize(r.n_groups);
          k_len.resize(r.n_groups);
          uint64_t kb = 0;
          for (uint32_t k = 0; k < r.n_groups; k++) {
            k_off[k] = r.groups[k].key_off;
            k_len[k] = r.groups[k].key_len;
            kb += k_len[k];
          }
          k_bytes.resize(kb + 1);
          if (warpjq_csv_gather(q->csv, d_nd, k_off.data(), k_len.data(), r.n_groups, k_bytes.data(), nullptr, e,
                                sizeof e) != WARPJQ_OK)
            return fail(std::string("CUDA error in reading group keys: ") + e);
          uint64_t at = 0;
          for (uint32_t k = 0; k < r.n_groups; k++) {
            const warpjq_group_ext &g = r.groups[k];
            tot.groups[device_key(k_bytes.data(), at, g.key_len, g.key_kind)].merge(g.count, g.numeric, g.sum,
                                                                                     g.min, g.max);
            at += g.key_len;
          }
        }
      } else if (r.n_selected) {
        rows.resize(r.out_len + 1);
        if (warpjq_device_read(rows.data(), r.d_out_bytes, r.out_len, nullptr, e, sizeof e) != WARPJQ_OK)
          return fail(std::string("CUDA error in reading rows: ") + e);
        w.bulk(rows.data(), (size_t)r.out_len, r.n_selected);
        if (w.oom) return fail("out of host memory for the output");
      }
    }
    records += recs;
    if (final_) break;
    // the unconsumed end (a row that continues) goes in front of chunk k + 1
    const uint64_t tail = n - used;
    if (tail + 16 <= room) {
      if (warpjq_csv_carry(q->csv, src + used, tail, b ^ 1, room - tail, nullptr, e, sizeof e) != WARPJQ_OK)
        return fail(std::string("CUDA error in carrying a CSV row: ") + e);
    } else {  // longer than the room before a chunk: stage it again, from the host
      while (room < tail + 16) room *= 2;
      if (warpjq_csv_stage_wait && warpjq_csv_stage_wait(q->csv, b ^ 1, e, sizeof e) != WARPJQ_OK)
        return fail(std::string("CUDA error in copying CSV to the device: ") + e);
      if (stage(b ^ 1, room - tail, next - tail, tail + n_next)) return 1;
    }
    carry = tail;
    pos = next;
    n_new = n_next;
    b ^= 1;
  }
  if (P.is_aggregate()) {
    if (!P.has_group) {
      w.aggregate(P.agg, tot.scalar);
    } else {
      std::vector<std::pair<GroupKey, Agg>> gs(tot.groups.begin(), tot.groups.end());
      std::sort(gs.begin(), gs.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
      w.groups(P.group_key_name(), P.agg, gs);
    }
  }
  const uint64_t n_rows = w.rows;
  size_t res_len = 0;
  char *res = w.finish(res_len);
  if (!res) return fail("out of host memory for the output");
  if (stats) {
    stats[0] = len;
    stats[1] = st_lines;
    stats[2] = n_rows;
    stats[3] = st_malformed;
    stats[4] = st_type;
  }
  *out = res;
  if (out_len) *out_len = res_len;
  return 0;
}

int warpjq_run_bytes(const char *query, const uint8_t *data, size_t len, uint32_t format,
                     uint32_t on_invalid, uint64_t chunk_bytes, uint64_t max_line_bytes, char **out,
                     size_t *out_len, uint64_t *stats, char *err, size_t err_len) {
  warpjq_query *q = nullptr;
  *out = nullptr;
  int rc = warpjq_query_open(query, format, chunk_bytes, &q, err, err_len);
  if (rc) return rc;
  rc = warpjq_query_run(q, data, len, on_invalid, max_line_bytes, out, out_len, stats, err, err_len);
  warpjq_query_close(q);
  return rc;
}

// The head of one device-resident result (header, aggregate or groups)
// into a fresh writer: what warpjq_query_render_device prints.
static void render_head(const warpjq_query *q, Writer &w, uint64_t count, uint64_t numeric, double sum,
                        double mn, double mx, const warpjq_group_ext *groups, uint32_t n_groups,
                        uint64_t n_selected, const uint8_t *data) {
  const Program &P = q->prog;
  w.fmt = q->fmt;
  w.header(P);
  if (P.is_aggregate()) {
    if (!P.has_group) {
      Agg a;
      a.merge(count, numeric, sum, mn, mx);
      w.aggregate(P.agg, a);
    } else {
      std::vector<std::pair<GroupKey, Agg>> gs;
      gs.reserve(n_groups);
      for (uint32_t k = 0; k < n_groups; k++) {
        const warpjq_group_ext &g = groups[k];
        Agg a;
        a.merge(g.count, g.numeric, g.sum, g.min, g.max);
        gs.push_back({device_key(data, g.key_off, g.key_len, g.key_kind), a});
      }
      std::sort(gs.begin(), gs.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
      w.groups(P.group_key_name(), P.agg, gs);
    }
  } else {
    w.rows = n_selected;
  }
}

// Formats the result of a device-resident aggregate run (warpjq_ext.h) the
// way the CLI prints it.  `data` is a host copy of the input, needed to
// render group keys.
int warpjq_query_render_device(warpjq_query *q, const warpjq_device_result *r, const uint8_t *data,
                               char **out, size_t *out_len) {
  Writer w;
  render_head(q, w, r->count, r->numeric, r->sum, r->min, r->max, r->groups, r->n_groups, r->n_selected,
              data);
  size_t res_len = 0;
  char *res = w.finish(res_len);
  if (!res) return 1;
  *out = res;
  if (out_len) *out_len = res_len;
  return 0;
}

// Every input's output of a collected batch (warpjq_batch_collect), back to
// back in one malloc'd buffer: input i's bytes are out[offsets[i],
// offsets[i+1]).  `groups` is the batch's group array, `key_data` the host
// bytes its key_off values index; `rows` / `row_off` a host copy of the
// batch's rows and row offsets (may be null for aggregates).
int warpjq_query_render_batch(warpjq_query *q, const warpjq_batch_item *items, uint32_t n,
                              const warpjq_group_ext *groups, const uint8_t *key_data, const uint8_t *rows,
                              const uint64_t *row_off, char **out, size_t *out_len, uint64_t *offsets) {
  *out = nullptr;
  if (out_len) *out_len = 0;
  std::string all;
  offsets[0] = 0;
  for (uint32_t i = 0; i < n; i++) {
    const warpjq_batch_item &it = items[i];
    Writer w;
    render_head(q, w, it.count, it.numeric, it.sum, it.min, it.max, groups ? groups + it.group_begin : nullptr,
                it.n_groups, it.n_selected, key_data);
    size_t hl = 0;
    char *h = w.finish(hl);
    if (!h) return 1;
    all.append(h, hl);
    free(h);
    if (it.n_selected && rows && row_off) {
      const uint64_t a = row_off[it.row_begin], b = row_off[it.row_begin + it.n_selected];
      all.append((const char *)rows + a, b - a);
    }
    offsets[i + 1] = all.size();
  }
  char *res = (char *)malloc(all.size() + 1);
  if (!res) return 1;
  memcpy(res, all.data(), all.size());
  *out = res;
  if (out_len) *out_len = all.size();
  return 0;
}

}  // extern "C"
