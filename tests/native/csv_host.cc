// TEST HARNESS (CPU): the CSV converter's per-row device code
// (warpjq_b200/csrc/csv_rows.cuh) compiled for the host.  Rows are split by
// the quote-parity rule, every row goes through the same row_json as on the
// device (length pass, then write pass at the prefix offset), so its bytes
// can be compared with the restated mapping without a GPU.  The product
// never runs this.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define __device__
#define __host__
#define __forceinline__ inline
struct uint4 {
  unsigned x, y, z, w;
};
static inline int __ffs(unsigned x) { return __builtin_ffs((int)x); }
template <typename T>
static inline T __ldg(const T *p) {
  return *p;
}

#include "../../warpjq_b200/csrc/csv_rows.cuh"

using namespace wjq_csv;

extern "C" {

// Converts `n` bytes of CSV placed at offset `shift` (0..15) of a 16-byte
// aligned buffer padded past its end (the device code reads whole aligned
// blocks).  Returns 0; 1 when a row's written bytes differ from its length.
int ch_convert(const uint8_t *src, size_t n, unsigned shift, char **out, size_t *out_len) {
  std::vector<uint4> store((n + shift) / 16 + 4);
  uint8_t *d = reinterpret_cast<uint8_t *>(store.data()) + shift;
  if (n) memcpy(d, src, n);
  std::vector<u64> row_end;
  bool inside = false;
  for (size_t i = 0; i < n; i++) {
    if (d[i] == '"') inside = !inside;
    else if (d[i] == '\n' && !inside) row_end.push_back(i);
  }
  if ((row_end.empty() ? 0 : row_end.back() + 1) < n) row_end.push_back(n);
  *out = nullptr;
  *out_len = 0;
  if (row_end.empty()) return 0;
  std::string text;
  std::vector<uint32_t> offs, words, meta;
  parse_header(d, row_end[0], text, offs);
  pack_keys(text, offs, words, meta);
  words.push_back(0);
  KeySet ks{words.data(), meta.data(), (uint32_t)(meta.size() / 2)};
  std::vector<u64> len(row_end.size(), 0);
  u64 total = 0;
  for (size_t r = 1; r < row_end.size(); r++) {
    WordIn in(d);
    WordOut w(nullptr);
    len[r] = row_json<false>(in, row_end[r - 1] + 1, row_end[r], ks, w);
    total += len[r];
  }
  std::vector<uint32_t> obuf(total / 4 + 4, 0xA5A5A5A5u);
  uint8_t *o = reinterpret_cast<uint8_t *>(obuf.data());
  u64 at = 0;
  int rc = 0;
  for (size_t r = 1; r < row_end.size(); r++) {
    WordIn in(d);
    WordOut w(o + at);
    row_json<true>(in, row_end[r - 1] + 1, row_end[r], ks, w);
    w.flush();
    const uint8_t *end = reinterpret_cast<const uint8_t *>(w.w) + w.off;
    if (end != o + at + len[r]) rc = 1;
    at += len[r];
  }
  *out = (char *)malloc(total ? total : 1);
  memcpy(*out, o, total);
  *out_len = total;
  return rc;
}

void ch_free(void *p) { free(p); }

}  // extern "C"
