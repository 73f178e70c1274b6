// Seeded synthetic NDJSON for benchmarks and tests.
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

// Writes one line (with '\n') for line index `i`; returns the end.
char *nginx_line(char *p, Rng &r, uint64_t i) {
  p = put(p, "{\"ts\":");
  p = put_u64(p, 1700000000ull + i + r.below(4));
  p = put(p, ",\"host\":\"");
  p = put(p, kHosts[r.below(8)]);
  p = put(p, "\",\"method\":\"");
  uint32_t m = r.below(100);
  p = put(p, m < 70 ? "GET" : m < 90 ? "POST" : m < 95 ? "PUT" : "DELETE");
  p = put(p, "\",\"path\":\"");
  double u = r.uniform();
  int k = 0;
  while (k < 31 && u > kT.path_cdf[k]) k++;
  p = put(p, kPaths[k]);
  p = put(p, "\",\"status\":");
  uint32_t s = r.below(100);
  p = put(p, s < 80 ? "200" : s < 85 ? "304" : s < 94 ? "404" : s < 99 ? "500" : "503");
  p = put(p, ",\"bytes\":");
  p = put_u64(p, (uint64_t)std::floor(std::exp(std::log(100.0) + r.uniform() * (std::log(1e7) - std::log(100.0)))));
  p = put(p, ",\"latency_ms\":");
  double lat = std::exp(3.0 + r.normal());
  uint64_t milli = (uint64_t)std::llround(lat * 1000.0);
  p = put_u64(p, milli / 1000);
  *p++ = '.';
  uint64_t f = milli % 1000;
  *p++ = (char)('0' + f / 100);
  *p++ = (char)('0' + f / 10 % 10);
  *p++ = (char)('0' + f % 10);
  p = put(p, ",\"ua\":\"");
  uint32_t n = 40 + r.below(81);
  for (uint32_t j = 0; j < n; j++) {
    char c = (char)(0x20 + r.below(95));
    if (c == '"' || c == '\\') *p++ = '\\';
    *p++ = c;
  }
  p = put(p, "\"}\n");
  return p;
}

}  // namespace

extern "C" {

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

// Generates about `target` bytes of nginx NDJSON into `out` (capacity cap
// >= target), in parallel blocks of `block_bytes`.  Each block is padded
// with its lines only (no partial lines).  Returns the bytes written.
uint64_t warpjq_gen_nginx(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                          unsigned threads, uint64_t *total_lines) {
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
        len[b] = warpjq_gen_nginx_block(seed, b, b * (block_bytes / 64), out + b * block_bytes, cap,
                                        &lines[b]);
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

}  // extern "C"
