// Seeded synthetic NDJSON (and a CSV rendering of the nginx schema) for
// benchmarks and tests.
//
// The nginx-style schema of the benchmark workload: keys in fixed order
//   ts          1700000000 + line index + uniform jitter 0..3
//   host        one of 8 names, uniform
//   method      GET 70%, POST 20%, PUT 5%, DELETE 5%
//   path        one of 32 fixed /api/v1/... paths, Zipf s = 1.1
//   status      200 80%, 304 5%, 404 9%, 500 5%, 503 1%
//   bytes       integer, log-uniform on [100, 10^7]
//   latency_ms  lognormal mu = 3, sigma = 1, three decimals
//   ua          40..120 printable ASCII characters (JSON-escaped)
// Lines are generated in independent blocks, each seeded from (seed, block),
// so any byte range can be produced in parallel and reproducibly.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Rng {  // splitmix64 seeding a xoshiro256** generator
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    for (auto &x : s) {
      seed += 0x9E3779B97F4A7C15ull;
      uint64_t z = seed;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      x = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  uint32_t below(uint32_t n) { return (uint32_t)((next() >> 32) * n >> 32); }
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

const char *kHosts[8] = {"api-01", "api-02", "api-03", "api-04", "web-01", "web-02", "web-03", "web-04"};
const char *kPaths[32] = {
    "/api/v1/users", "/api/v1/orders", "/api/v1/items", "/api/v1/cart", "/api/v1/login",
    "/api/v1/logout", "/api/v1/search", "/api/v1/health", "/api/v1/metrics", "/api/v1/config",
    "/api/v1/users/profile", "/api/v1/users/settings", "/api/v1/orders/history",
    "/api/v1/orders/status", "/api/v1/items/reviews", "/api/v1/items/stock", "/api/v1/payments",
    "/api/v1/payments/refund", "/api/v1/shipping", "/api/v1/shipping/track", "/api/v1/coupons",
    "/api/v1/notifications", "/api/v1/messages", "/api/v1/uploads", "/api/v1/downloads",
    "/api/v1/reports", "/api/v1/admin", "/api/v1/admin/users", "/api/v1/feedback",
    "/api/v1/sessions", "/api/v1/tokens", "/api/v1/webhooks"};

struct Tables {
  double path_cdf[32];
  Tables() {
    double z = 0;
    for (int k = 0; k < 32; k++) z += 1.0 / std::pow(k + 1, 1.1);
    double c = 0;
    for (int k = 0; k < 32; k++) {
      c += 1.0 / std::pow(k + 1, 1.1) / z;
      path_cdf[k] = c;
    }
    path_cdf[31] = 1.0;
  }
};
const Tables kT;

char *put(char *p, const char *s) {
  size_t n = strlen(s);
  memcpy(p, s, n);
  return p + n;
}

char *put_u64(char *p, uint64_t v) {
  char t[24];
  int n = 0;
  do {
    t[n++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (n) *p++ = t[--n];
  return p;
}

// Writes one line (with '\n') for line index `i`; returns the end.  With
// `csv` the same draws render as a CSV row of the columns in key order, ua
// always quoted (a '"' inside doubled).
char *nginx_line(char *p, Rng &r, uint64_t i, bool csv = false) {
  const char *sep_host = csv ? "," : ",\"host\":\"", *sep_method = csv ? "," : "\",\"method\":\"";
  const char *sep_path = csv ? "," : "\",\"path\":\"", *sep_status = csv ? "," : "\",\"status\":";
  if (!csv) p = put(p, "{\"ts\":");
  p = put_u64(p, 1700000000ull + i + r.below(4));
  p = put(p, sep_host);
  p = put(p, kHosts[r.below(8)]);
  p = put(p, sep_method);
  uint32_t m = r.below(100);
  p = put(p, m < 70 ? "GET" : m < 90 ? "POST" : m < 95 ? "PUT" : "DELETE");
  p = put(p, sep_path);
  double u = r.uniform();
  int k = 0;
  while (k < 31 && u > kT.path_cdf[k]) k++;
  p = put(p, kPaths[k]);
  p = put(p, sep_status);
  uint32_t s = r.below(100);
  p = put(p, s < 80 ? "200" : s < 85 ? "304" : s < 94 ? "404" : s < 99 ? "500" : "503");
  p = put(p, csv ? "," : ",\"bytes\":");
  p = put_u64(p, (uint64_t)std::floor(std::exp(std::log(100.0) + r.uniform() * (std::log(1e7) - std::log(100.0)))));
  p = put(p, csv ? "," : ",\"latency_ms\":");
  double lat = std::exp(3.0 + r.normal());
  uint64_t milli = (uint64_t)std::llround(lat * 1000.0);
  p = put_u64(p, milli / 1000);
  *p++ = '.';
  uint64_t f = milli % 1000;
  *p++ = (char)('0' + f / 100);
  *p++ = (char)('0' + f / 10 % 10);
  *p++ = (char)('0' + f % 10);
  p = put(p, csv ? ",\"" : ",\"ua\":\"");
  uint32_t n = 40 + r.below(81);
  for (uint32_t j = 0; j < n; j++) {
    char c = (char)(0x20 + r.below(95));
    if (csv ? c == '"' : (c == '"' || c == '\\')) *p++ = csv ? '"' : '\\';
    *p++ = c;
  }
  p = put(p, csv ? "\"\n" : "\"}\n");
  return p;
}

// ---------------------------------------------------------------------------
// Nested, dirty schema: objects 3-5 levels deep with shuffled key order,
// escaped strings, mixed number forms and a share of malformed lines.
//   ts     integer
//   req    {user: {id: "u<Zipf(0.9) over n_users>", tier, geo: {cc, lat, lon}}, method, path}
//   resp   {code, latency (decimal or exponent form of the same value), size}
//   meta   {trace: {span: {id, depth}}}
// About 10% of path strings carry a \uXXXX escape or an escaped quote; about
// 2% of lines are malformed: cut short, a bare NaN, or a leading zero.
// ---------------------------------------------------------------------------

const char *kTiers[4] = {"gold", "silver", "bronze", "free"};
const char *kCcs[6] = {"us", "de", "jp", "br", "in", "fr"};
const char *kMethods[4] = {"GET", "POST", "PUT", "DELETE"};

char *put_dec3(char *p, uint64_t milli) {  // milli/1000 with three decimals
  p = put_u64(p, milli / 1000);
  *p++ = '.';
  *p++ = (char)('0' + milli / 100 % 10);
  *p++ = (char)('0' + milli / 10 % 10);
  *p++ = (char)('0' + milli % 10);
  return p;
}

// The same value (milli / 1000) as a decimal, an exponent form, or a
// decimal exponent form.
char *put_mixed(char *p, Rng &r, uint64_t milli) {
  uint32_t form = r.below(3);
  if (form == 0) return put_dec3(p, milli);
  if (form == 1) {  // <milli>e-3
    p = put_u64(p, milli);
    return put(p, "e-3");
  }
  p = put_dec3(p, milli * 10);  // (milli*10/1000)E-1
  return put(p, "E-1");
}

uint64_t zipf(Rng &r, uint64_t n, double s) {
  // inverse of the continuous approximation of the Zipf CDF on [1, n]
  const double a = 1.0 - s;
  double k = std::pow(1.0 + r.uniform() * (std::pow((double)n, a) - 1.0), 1.0 / a);
  uint64_t v = (uint64_t)k;
  return v < 1 ? 1 : (v > n ? n : v);
}

char *nested_line(char *p, Rng &r, uint64_t i, uint64_t n_users) {
  char *start = p;
  const uint32_t bad = r.below(100) < 2 ? 1 + r.below(3) : 0;  // 1 cut, 2 NaN, 3 leading zero
  char buf[4][256];
  char *e[4];
  // req
  {
    char *q = buf[0];
    const char *parts[3];
    char user[160], *u = user;
    const char *uk[3];
    char idb[40], *ip = idb;
    ip = put(ip, "\"id\":\"u");
    ip = put_u64(ip, zipf(r, n_users, 0.9));
    ip = put(ip, "\"");
    *ip = 0;
    char tb[32], *tp = tb;
    tp = put(tp, "\"tier\":\"");
    tp = put(tp, kTiers[r.below(4)]);
    tp = put(tp, "\"");
    *tp = 0;
    char gb[96], *gp = gb;
    gp = put(gp, "\"geo\":{\"cc\":\"");
    gp = put(gp, kCcs[r.below(6)]);
    gp = put(gp, "\",\"lat\":");
    gp = put_dec3(gp, r.below(90000));
    gp = put(gp, ",\"lon\":-");
    gp = put_dec3(gp, r.below(180000));
    gp = put(gp, "}");
    *gp = 0;
    uk[0] = idb; uk[1] = tb; uk[2] = gb;
    for (int k = 2; k > 0; k--) { int j = r.below(k + 1); const char *t = uk[k]; uk[k] = uk[j]; uk[j] = t; }
    u = put(u, "\"user\":{");
    for (int k = 0; k < 3; k++) { if (k) *u++ = ','; u = put(u, uk[k]); }
    *u++ = '}';
    *u = 0;
    char mb[32], *mp = mb;
    mp = put(mp, "\"method\":\"");
    mp = put(mp, kMethods[r.below(4)]);
    mp = put(mp, "\"");
    *mp = 0;
    char pb[96], *pp = pb;
    pp = put(pp, "\"path\":\"/api/v2/");
    pp = put(pp, kTiers[r.below(4)]);
    const uint32_t esc = r.below(10);
    if (esc == 0) pp = put(pp, "/caf\\u00e9");
    else if (esc == 1) pp = put(pp, "/say \\\"hi\\\"");
    pp = put(pp, "\"");
    *pp = 0;
    parts[0] = user; parts[1] = mb; parts[2] = pb;
    for (int k = 2; k > 0; k--) { int j = r.below(k + 1); const char *t = parts[k]; parts[k] = parts[j]; parts[j] = t; }
    q = put(q, "\"req\":{");
    for (int k = 0; k < 3; k++) { if (k) *q++ = ','; q = put(q, parts[k]); }
    *q++ = '}';
    e[0] = q;
  }
  // resp
  {
    char *q = buf[1];
    const uint32_t c = r.below(100);
    const char *code = c < 75 ? "200" : c < 80 ? "201" : c < 84 ? "204" : c < 87 ? "301" : c < 92 ? "400"
                       : c < 96 ? "404" : c < 99 ? "500" : "503";
    char cb[32], *cp = cb;
    cp = put(cp, "\"code\":");
    if (bad == 3) *cp++ = '0';
    cp = put(cp, code);
    *cp = 0;
    char lb[48], *lp = lb;
    lp = put(lp, "\"latency\":");
    if (bad == 2) lp = put(lp, "NaN");
    else lp = put_mixed(lp, r, (uint64_t)std::llround(std::exp(3.0 + r.normal()) * 1000.0));
    *lp = 0;
    char sb[40], *sp = sb;
    sp = put(sp, "\"size\":");
    sp = put_u64(sp, r.below(1000000));
    *sp = 0;
    const char *f[3] = {cb, lb, sb};
    for (int k = 2; k > 0; k--) { int j = r.below(k + 1); const char *t = f[k]; f[k] = f[j]; f[j] = t; }
    q = put(q, "\"resp\":{");
    for (int k = 0; k < 3; k++) { if (k) *q++ = ','; q = put(q, f[k]); }
    *q++ = '}';
    e[1] = q;
  }
  // meta and ts
  {
    char *q = buf[2];
    q = put(q, "\"meta\":{\"trace\":{\"span\":{\"id\":\"");
    static const char hx[] = "0123456789abcdef";
    for (int k = 0; k < 16; k++) *q++ = hx[r.below(16)];
    q = put(q, "\",\"depth\":");
    q = put_u64(q, r.below(8));
    q = put(q, "}}}");
    e[2] = q;
    char *t = buf[3];
    t = put(t, "\"ts\":");
    t = put_u64(t, 1700000000ull + i);
    e[3] = t;
  }
  int order[4] = {0, 1, 2, 3};
  for (int k = 3; k > 0; k--) { int j = r.below(k + 1); int t = order[k]; order[k] = order[j]; order[j] = t; }
  *p++ = '{';
  for (int k = 0; k < 4; k++) {
    if (k) *p++ = ',';
    size_t n = (size_t)(e[order[k]] - buf[order[k]]);
    memcpy(p, buf[order[k]], n);
    p += n;
  }
  *p++ = '}';
  if (bad == 1) p = start + 1 + r.below((uint32_t)(p - start - 1));  // cut short
  *p++ = '\n';
  return p;
}

}  // namespace

extern "C" {

// The nested schema (above), like warpjq_gen_nginx_block; a line is at most
// 1 KiB.
uint64_t warpjq_gen_nested_block(uint64_t seed, uint64_t block, uint64_t first_line, uint64_t n_users,
                                 uint8_t *out, uint64_t cap, uint64_t *n_lines) {
  Rng r(seed * 0x100000001B3ull ^ (block * 0xD1B54A32D192ED03ull) ^ 0x5EED5EEDull);
  char *p = (char *)out, *end = (char *)out + cap;
  uint64_t i = first_line;
  while (end - p >= 1024) {
    p = nested_line(p, r, i, n_users ? n_users : 1);
    i++;
  }
  if (n_lines) *n_lines = i - first_line;
  return (uint64_t)(p - (char *)out);
}

// Fills `out[0, cap)` with whole nginx lines for the block `block` of `seed`,
// starting at line index `first_line`.  Returns bytes written and the number
// of lines in *n_lines.  A line is at most 512 bytes.
uint64_t warpjq_gen_nginx_block(uint64_t seed, uint64_t block, uint64_t first_line, uint8_t *out,
                                uint64_t cap, uint64_t *n_lines) {
  Rng r(seed * 0x100000001B3ull ^ (block * 0xD1B54A32D192ED03ull));
  char *p = (char *)out, *end = (char *)out + cap;
  uint64_t i = first_line;
  while (end - p >= 512) {
    p = nginx_line(p, r, i);
    i++;
  }
  if (n_lines) *n_lines = i - first_line;
  return (uint64_t)(p - (char *)out);
}

// The same records as CSV rows (no header), like warpjq_gen_nginx_block.
uint64_t warpjq_gen_nginx_csv_block(uint64_t seed, uint64_t block, uint64_t first_line, uint8_t *out,
                                    uint64_t cap, uint64_t *n_lines) {
  Rng r(seed * 0x100000001B3ull ^ (block * 0xD1B54A32D192ED03ull));
  char *p = (char *)out, *end = (char *)out + cap;
  uint64_t i = first_line;
  while (end - p >= 512) {
    p = nginx_line(p, r, i, true);
    i++;
  }
  if (n_lines) *n_lines = i - first_line;
  return (uint64_t)(p - (char *)out);
}

// Generates about `target` bytes of nginx NDJSON into `out` (capacity cap
// >= target), in parallel blocks of `block_bytes`.  Each block is padded
// with its lines only (no partial lines).  Returns the bytes written.
static uint64_t gen_parallel(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                             unsigned threads, uint64_t *total_lines, uint64_t n_users, int kind) {
  if (block_bytes < 4096) block_bytes = 4096;
  uint64_t nb = (target + block_bytes - 1) / block_bytes;
  std::vector<uint64_t> len(nb), lines(nb);
  std::vector<std::vector<uint8_t>> tmp(nb);
  if (!threads) threads = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> ws;
  for (unsigned t = 0; t < threads; t++) {
    ws.emplace_back([&, t] {
      for (uint64_t b = t; b < nb; b += threads) {
        // Blocks are generated in place at their nominal offset; lines of a
        // block never cross into the next block.
        uint64_t cap = std::min<uint64_t>(block_bytes, target - b * block_bytes);
        uint8_t *o = out + b * block_bytes;
        const uint64_t first = b * (block_bytes / 64);
        len[b] = kind == 1   ? warpjq_gen_nested_block(seed, b, first, n_users, o, cap, &lines[b])
                 : kind == 2 ? warpjq_gen_nginx_csv_block(seed, b, first, o, cap, &lines[b])
                             : warpjq_gen_nginx_block(seed, b, first, o, cap, &lines[b]);
      }
    });
  }
  for (auto &w : ws) w.join();
  // Compact the blocks (each ends a little short of its nominal size).
  uint64_t w = 0, total = 0;
  for (uint64_t b = 0; b < nb; b++) {
    if (w != b * block_bytes) memmove(out + w, out + b * block_bytes, len[b]);
    w += len[b];
    total += lines[b];
  }
  if (total_lines) *total_lines = total;
  return w;
}

uint64_t warpjq_gen_nginx(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                          unsigned threads, uint64_t *total_lines) {
  return gen_parallel(seed, out, target, block_bytes, threads, total_lines, 0, 0);
}

// Generates about `target` bytes of the nested schema with user ids drawn
// from [1, n_users].
uint64_t warpjq_gen_nested(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                           unsigned threads, uint64_t n_users, uint64_t *total_lines) {
  return gen_parallel(seed, out, target, block_bytes, threads, total_lines, n_users, 1);
}

// The NDJSON rendering of exactly the records warpjq_gen_nginx_csv(seed,
// .., target, block_bytes, ..) writes as CSV rows, in order (the expected
// input of a query over that CSV).  `out` must hold 2 * target bytes: a
// record's NDJSON line is under twice its CSV row.
uint64_t warpjq_gen_nginx_csv_as_ndjson(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                                        unsigned threads, uint64_t *total_lines) {
  static const uint64_t h = 47;  // the CSV header row's length
  if (target < h) {
    if (total_lines) *total_lines = 0;
    return 0;
  }
  target -= h;
  if (block_bytes < 4096) block_bytes = 4096;
  const uint64_t nb = (target + block_bytes - 1) / block_bytes;
  std::vector<uint64_t> len(nb), lines(nb);
  if (!threads) threads = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> ws;
  for (unsigned t = 0; t < threads; t++) {
    ws.emplace_back([&, t] {
      std::vector<uint8_t> tmp(block_bytes);
      for (uint64_t b = t; b < nb; b += threads) {
        const uint64_t cap = std::min<uint64_t>(block_bytes, target - b * block_bytes);
        const uint64_t first = b * (block_bytes / 64);
        uint64_t k = 0;
        warpjq_gen_nginx_csv_block(seed, b, first, tmp.data(), cap, &k);  // the block's row count
        // the same draws rendered as NDJSON
        Rng r(seed * 0x100000001B3ull ^ (b * 0xD1B54A32D192ED03ull));
        char *p = (char *)out + 2 * b * block_bytes;
        for (uint64_t i = 0; i < k; i++) p = nginx_line(p, r, first + i);
        len[b] = (uint64_t)(p - ((char *)out + 2 * b * block_bytes));
        lines[b] = k;
      }
    });
  }
  for (auto &w : ws) w.join();
  uint64_t w = 0, total = 0;
  for (uint64_t b = 0; b < nb; b++) {
    if (w != 2 * b * block_bytes) memmove(out + w, out + 2 * b * block_bytes, len[b]);
    w += len[b];
    total += lines[b];
  }
  if (total_lines) *total_lines = total;
  return w;
}

// About `target` bytes of the nginx records as CSV: a header row naming the
// columns (ts,host,method,path,status,bytes,latency_ms,ua), then the rows.
uint64_t warpjq_gen_nginx_csv(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                              unsigned threads, uint64_t *total_lines) {
  static const char kHead[] = "ts,host,method,path,status,bytes,latency_ms,ua\n";
  const uint64_t h = sizeof kHead - 1;
  if (target < h) {
    if (total_lines) *total_lines = 0;
    return 0;
  }
  memcpy(out, kHead, h);
  return h + gen_parallel(seed, out + h, target - h, block_bytes, threads, total_lines, 0, 2);
}

}  // extern "C"
