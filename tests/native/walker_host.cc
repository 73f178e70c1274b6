// TEST HARNESS (CPU): the device line walker and evaluator of
// warpjq_b200/csrc/walker.cuh compiled for the host, so their per-line
// semantics can be compared with the oracle without a GPU.  The product
// never runs this; it only exercises the same source on the CPU.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
static inline long long __double_as_longlong(double d) {
  long long x;
  std::memcpy(&x, &d, 8);
  return x;
}
static inline int __ffs(unsigned x) { return __builtin_ffs((int)x); }
static inline unsigned __funnelshift_r(unsigned lo, unsigned hi, unsigned sh) {
  sh &= 31u;
  return sh ? (lo >> sh) | (hi << (32u - sh)) : lo;
}
struct uint4 {
  unsigned x, y, z, w;
};
static inline double __longlong_as_double(long long x) {
  double d;
  std::memcpy(&d, &x, 8);
  return d;
}

#include "../../warpjq_b200/csrc/host/query.h"
#include "../../warpjq_b200/csrc/plan_build.h"
#include "../../warpjq_b200/csrc/walker.cuh"

using namespace wjq;

extern "C" {

// One output line per physical input line (mode 0: the bounded walker
// walk_line; mode 1: the window walker walk_masked, with the line copied at
// a varying offset into a window whose bytes past the newline are quotes,
// backslashes and digits, and the window's special mask made by the
// kernel's chunk classifier; mode 2: as mode 1, with the object fast path
// walk_objects tried first, as the scan kernel does):
//   blank | invalid | type | filtered | selected<TAB>kind:raw<TAB>...
// Returns 0, or 2 for a query error, 3 for a plan error.
int wh_eval(const char *query, const uint8_t *data, size_t len, int mode, char **out,
            size_t *out_len) {
  wjqh::Program prog;
  wjqh::QueryError qe;
  if (!wjqh::parse(query, prog, qe)) return 2;
  wjqh::Lowered low;
  low.build(prog, false);
  static DevPlan P;
  char err[256];
  if (build_plan(&low.prog, P, err, sizeof err) != WARPJQ_OK) return 3;
  std::vector<uint32_t> deep_words(1 << 16);
  DeepStack deep{deep_words.data(), (uint64_t)deep_words.size() * 32};
  static NodeVals nv;
  std::string o;
  std::vector<uint32_t> winbuf, smask;
  size_t pos = 0, line_no = 0;
  while (pos < len) {
    const uint8_t *nl = (const uint8_t *)std::memchr(data + pos, '\n', len - pos);
    size_t end = nl ? (size_t)(nl - data) : len;
    const uint8_t *line = data + pos;
    uint32_t n = (uint32_t)(end - pos);
    pos = end + 1;
    int st;
    if (mode == 1 || mode == 2) {
      // the line at a varying offset (across 32-byte chunk boundaries), its
      // newline, then quotes, backslashes and digits; the special mask of
      // the whole window is made by the kernel's own chunk classifier
      uint32_t s = (uint32_t)(line_no++ * 7 % 48);
      const uint32_t W = (s + n + 64 + 31) / 32 * 32;
      winbuf.assign(W / 4 + 8, 0);
      uint8_t *w = (uint8_t *)winbuf.data();
      std::memcpy(w + s, line, n);
      w[s + n] = '\n';
      for (uint32_t k = 1; k < 40; k++) w[s + n + k] = "\"\\9"[k % 3];
      smask.assign(W / 32 + 1, 0);
      for (uint32_t c = 0; c < W / 32; c++) classify_chunk(winbuf.data() + 8 * c, &smask[c]);
      line = w + s;
      st = mode == 2 ? walk_objects(P, w, smask.data(), s, s + n, nv) : LS_FALLBACK;
      if (st == LS_FALLBACK) st = walk_masked(P, w, smask.data(), s, s + n, nv);
    } else {
      st = walk_line(P, line, n, nv, nullptr);
    }
    if (st == LS_DEEP) st = walk_line(P, line, n, nv, &deep);
    if (st == LS_BLANK) {
      o += "blank\n";
      continue;
    }
    if (st != LS_OK) {
      o += "invalid\n";
      continue;
    }
    SlotVal slots[kMaxSlots];
    bool tf = false, tp = false;
    for (uint32_t s = 0; s < P.n_slots; s++) {
      slots[s] = resolve_slot(P, nv, s);
      if (slots[s].state == SS_TYPE_ERROR) ((P.filter_slot_mask >> s) & 1 ? tf : tp) = true;
    }
    if (tf) {
      o += "type\n";
    } else if (P.has_filter && !eval_filter(P, line, slots)) {
      o += "filtered\n";
    } else if (tp) {
      o += "type\n";
    } else {
      o += "selected";
      for (uint32_t s = 0; s < P.n_slots; s++) {
        o += "\t" + std::to_string(slots[s].kind) + ":";
        if (slots[s].kind != JK_MISSING) o.append((const char *)line + slots[s].off, slots[s].len);
        if (slots[s].kind == JK_NUM) {
          bool is_int;
          long long iv;
          double d = parse_number(line + slots[s].off, slots[s].len, is_int, iv);
          char b[64];
          std::snprintf(b, sizeof b, "=%a", d);
          o += b;
        }
      }
      o += "\n";
    }
  }
  *out = (char *)std::malloc(o.size() + 1);
  std::memcpy(*out, o.data(), o.size());
  *out_len = o.size();
  return 0;
}

void wh_free(char *p) { std::free(p); }

}  // extern "C"
