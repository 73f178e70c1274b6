// CSV input: converts RFC 4180 CSV to NDJSON in device memory, so the scan
// kernels run on it unchanged.  The reference reads only NDJSON (its --csv
// flag is an output format, crates/warpjq-core/src/output.rs:45-85); this
// mapping is this library's own:
//
//   - a '\n' ends a row when the number of '"' bytes before it (from the
//     start of the input) is even; a '\r' just before it is dropped;
//   - the first row is the header; every later row becomes one NDJSON line,
//     an empty row an empty line (which the scan skips as blank);
//   - fields are separated by ','; a field that starts with '"' is quoted:
//     it runs to the next '"' not followed by another '"', a doubled '""'
//     inside stands for '"', and bytes after the closing quote up to the
//     next ',' are kept as they are; other fields run to the next ',';
//   - a row becomes an object with the header's names as keys, in order,
//     from its first min(fields, names) fields: missing trailing fields are
//     left out, extra fields are dropped;
//   - a value is the field's text as a JSON number when the field is not
//     quoted and its text is a JSON number; null when it is not quoted and
//     empty; else a JSON string ('"' and '\' escaped, control bytes as
//     \n \r \t \b \f or \u00XX, other bytes as they are).  Header names are
//     escaped the same way; a UTF-8 byte-order mark before the header is
//     dropped.
//
// Passes, none waiting on another CTA:
//   k_csv_stats     per 256-byte run: quote parity, newline count, newlines
//                   outside quotes if the run starts outside; per 64 KiB
//                   tile the same (16-byte loads, SWAR byte masks, a prefix
//                   XOR over the quote mask for the in-quote state)
//   k_csv_tiles     one block: each tile's start state and first row
//   k_csv_row_ends  each row's end offset
//   k_csv_close     the last row, the consumed length, the header's end
//   k_csv_json<0>   one thread per row: its NDJSON length
//   (exclusive scan of the lengths)
//   k_csv_json<1>   one thread per row: its NDJSON bytes
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/warpjq_ext.h"
#include "csv_rows.cuh"

using namespace wjq_csv;

namespace {

constexpr uint32_t kRun = 256;                     // bytes a thread owns in the row passes
constexpr int kCsvThreads = 256;                   // threads per tile
constexpr uint32_t kCsvTile = kRun * kCsvThreads;  // 64 KiB
constexpr int kScanBlock = 1024;                   // elements per block of the u64 scan
constexpr int kJsonThreads = 128;

void csv_err(char *err, size_t len, const char *fmt, ...) {
  if (!err || !len) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, len, fmt, ap);
  va_end(ap);
}

#define CSV_CK(call, what)                                                         \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      csv_err(err, err_len, "%s: %s", what, cudaGetErrorString(e_));                \
      return e_ == cudaErrorMemoryAllocation ? WARPJQ_ERR_OOM : WARPJQ_ERR_CUDA;    \
    }                                                                               \
  } while (0)

// Block-wide exclusive scan (+ or ^) of one u64 per thread; `total` gets
// the whole block's.  Every thread of the block must call it.
template <bool kXor>
__device__ u64 block_excl(u64 v, u64 &total) {
  __shared__ u64 s_w[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  u64 inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const u64 x = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc = kXor ? (inc ^ x) : (inc + x);
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  u64 before = 0, all = 0;
  for (int w = 0; w < nw; w++) {
    if (w < warp) before = kXor ? (before ^ s_w[w]) : (before + s_w[w]);
    all = kXor ? (all ^ s_w[w]) : (all + s_w[w]);
  }
  total = all;
  __syncthreads();
  return kXor ? (before ^ inc ^ v) : (before + inc - v);
}

// Quote and newline masks of the 16-byte aligned block at `blk`.
__device__ __forceinline__ void block_masks(const uint8_t *blk, uint32_t &q, uint32_t &nl) {
  const uint4 v = __ldg(reinterpret_cast<const uint4 *>(blk));
  q = eq4(v.x, 0x22222222u) | eq4(v.y, 0x22222222u) << 4 | eq4(v.z, 0x22222222u) << 8 |
      eq4(v.w, 0x22222222u) << 12;
  nl = eq4(v.x, 0x0A0A0A0Au) | eq4(v.y, 0x0A0A0A0Au) << 4 | eq4(v.z, 0x0A0A0A0Au) << 8 |
       eq4(v.w, 0x0A0A0A0Au) << 12;
}

// Inclusive prefix XOR of a 16-bit mask: bit j = parity of bits 0..j.
__device__ __forceinline__ uint32_t pxor16(uint32_t x) {
  x ^= x << 1;
  x ^= x << 2;
  x ^= x << 4;
  x ^= x << 8;
  return x & 0xFFFFu;
}

// Walks the bytes [a, b) of `d` in 16-byte aligned blocks (a block that
// holds one byte of the range lies in the same page as that byte, so the
// aligned loads stay in mapped memory).  For each block: f(block offset
// from d, quote mask, newline mask), both limited to the range.
template <typename F>
__device__ __forceinline__ void for_blocks(const uint8_t *d, u64 a, u64 b, F &&f) {
  if (a >= b) return;
  const uintptr_t pa = (uintptr_t)(d + a), pb = (uintptr_t)(d + b);
  for (uintptr_t blk = pa & ~(uintptr_t)15; blk < pb; blk += 16) {
    const uint32_t lo = blk < pa ? (uint32_t)(pa - blk) : 0;
    const uint32_t hi = pb - blk < 16 ? (uint32_t)(pb - blk) : 16;
    const uint32_t valid = ((1u << hi) - 1) & ~((1u << lo) - 1);
    uint32_t q, nl;
    block_masks(reinterpret_cast<const uint8_t *>(blk), q, nl);
    f((long long)(blk - (uintptr_t)d), q & valid, nl & valid);
  }
}

// Per run (u32): bit 0 quote parity, bits 1..11 newlines outside quotes
// when the run starts outside, bits 12..22 all newlines.  Per tile (u64):
// bit 0 parity, bits 1..31 the same outside count, bits 32..63 all newlines.
__global__ void __launch_bounds__(kCsvThreads) k_csv_stats(const uint8_t *d, u64 n, uint32_t *run_stat,
                                                           u64 *tile_stat) {
  const u64 a = (u64)blockIdx.x * kCsvTile + (u64)threadIdx.x * kRun;
  const u64 b = a + kRun < n ? a + kRun : n;
  uint32_t s = 0, c0 = 0, nlt = 0;
  for_blocks(d, a, b, [&](long long, uint32_t q, uint32_t nl) {
    const uint32_t inq = pxor16(q) ^ (s ? 0xFFFFu : 0u);
    c0 += __popc(nl & ~inq);
    nlt += __popc(nl);
    s ^= __popc(q) & 1;
  });
  run_stat[(u64)blockIdx.x * kCsvThreads + threadIdx.x] = s | c0 << 1 | nlt << 12;
  u64 ptot, ctot, ntot;
  const u64 sb = block_excl<true>(s, ptot);  // quote parity before this run, within the tile
  block_excl<false>(sb ? nlt - c0 : c0, ctot);
  block_excl<false>(nlt, ntot);
  if (threadIdx.x == 0) tile_stat[blockIdx.x] = (ptot & 1) | ctot << 1 | ntot << 32;
}

// One block: each tile's start state (inside quotes or not) and the rows
// ended before it; info[0] = rows ended by a newline.
__global__ void __launch_bounds__(1024) k_csv_tiles(const u64 *tile_stat, u64 n_tiles, uint32_t *tile_state,
                                                    u64 *tile_row, u64 *info) {
  const u64 per = (n_tiles + blockDim.x - 1) / blockDim.x;
  const u64 a = threadIdx.x * per < n_tiles ? threadIdx.x * per : n_tiles;
  const u64 b = a + per < n_tiles ? a + per : n_tiles;
  u64 p = 0;
  for (u64 t = a; t < b; t++) p ^= tile_stat[t] & 1;
  u64 ptot;
  const uint32_t s0 = (uint32_t)block_excl<true>(p, ptot);
  uint32_t s = s0;
  u64 rows = 0;
  for (u64 t = a; t < b; t++) {
    const u64 ts = tile_stat[t];
    const u64 c0 = (ts >> 1) & 0x7FFFFFFFull, nlt = ts >> 32;
    rows += s ? nlt - c0 : c0;
    s ^= (uint32_t)(ts & 1);
  }
  u64 rtot;
  u64 base = block_excl<false>(rows, rtot);
  s = s0;
  for (u64 t = a; t < b; t++) {
    const u64 ts = tile_stat[t];
    const u64 c0 = (ts >> 1) & 0x7FFFFFFFull, nlt = ts >> 32;
    tile_state[t] = s;
    tile_row[t] = base;
    base += s ? nlt - c0 : c0;
    s ^= (uint32_t)(ts & 1);
  }
  if (threadIdx.x == 0) info[0] = rtot;
}

// Writes the offset of every row-ending newline, in order.
__global__ void __launch_bounds__(kCsvThreads) k_csv_row_ends(const uint8_t *d, u64 n, const uint32_t *run_stat,
                                                              const uint32_t *tile_state, const u64 *tile_row,
                                                              u64 *row_end) {
  const u64 a = (u64)blockIdx.x * kCsvTile + (u64)threadIdx.x * kRun;
  const u64 b = a + kRun < n ? a + kRun : n;
  const uint32_t st = run_stat[(u64)blockIdx.x * kCsvThreads + threadIdx.x];
  const uint32_t p = st & 1, c0 = (st >> 1) & 0x7FF, nlt = (st >> 12) & 0x7FF;
  u64 tot;
  uint32_t s = (uint32_t)block_excl<true>(p, tot) ^ tile_state[blockIdx.x];
  u64 idx = block_excl<false>(s ? nlt - c0 : c0, tot) + tile_row[blockIdx.x];
  for_blocks(d, a, b, [&](long long off, uint32_t q, uint32_t nl) {
    const uint32_t inq = pxor16(q) ^ (s ? 0xFFFFu : 0u);
    uint32_t m = nl & ~inq;
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      row_end[idx++] = (u64)(off + j);
    }
    s ^= __popc(q) & 1;
  });
}

// info[0] (rows ended by a newline) -> rows; info[1] = bytes consumed (up
// to and with the last row's newline, or all when `final`); info[2] = the
// first row's end.  With `final`, a last row without a newline ends at n.
__global__ void k_csv_close(u64 *row_end, u64 n, int final_, u64 *info) {
  u64 r = info[0];
  const u64 start = r ? row_end[r - 1] + 1 : 0;
  if (final_ && start < n) row_end[r++] = n;
  info[0] = r;
  info[1] = final_ ? n : start;
  info[2] = r ? row_end[0] : 0;
}

// Rows [row0, rows) of the chunk, one thread each: pass 0 writes the NDJSON
// length of line r - row0 to len_off, pass 1 writes the line at out +
// len_off[r - row0] (len_off by then an exclusive prefix).
template <bool kWrite>
__global__ void __launch_bounds__(kJsonThreads) k_csv_json(const uint8_t *d, const u64 *row_end, u64 row0,
                                                           u64 rows, KeySet ks, u64 *len_off, uint8_t *out) {
  for (u64 r = row0 + blockIdx.x * (u64)blockDim.x + threadIdx.x; r < rows; r += (u64)gridDim.x * blockDim.x) {
    const u64 s = r ? __ldg(row_end + r - 1) + 1 : 0, e = __ldg(row_end + r);
    WordIn in(d);
    if (!kWrite) {
      WordOut w(nullptr);
      len_off[r - row0] = row_json<false>(in, s, e, ks, w);
    } else {
      WordOut w(out + len_off[r - row0]);
      row_json<true>(in, s, e, ks, w);
      w.flush();
    }
  }
}

// Exclusive prefix sum of v[0, m) in place, as block totals, one block over
// the totals, and a per-block add; the grand total goes to *total.
__global__ void __launch_bounds__(256) k_sum_blocks(u64 *v, u64 m, u64 *bt) {
  const u64 i0 = (u64)blockIdx.x * kScanBlock + threadIdx.x * (kScanBlock / 256);
  u64 loc[kScanBlock / 256];
  u64 s = 0;
#pragma unroll
  for (int k = 0; k < kScanBlock / 256; k++) {
    loc[k] = i0 + k < m ? v[i0 + k] : 0;
    s += loc[k];
  }
  u64 tot;
  u64 ex = block_excl<false>(s, tot);
#pragma unroll
  for (int k = 0; k < kScanBlock / 256; k++) {
    if (i0 + k < m) v[i0 + k] = ex;
    ex += loc[k];
  }
  if (threadIdx.x == 0) bt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_sum_totals(u64 *bt, u64 nb, u64 *total) {
  const u64 per = (nb + blockDim.x - 1) / blockDim.x;
  const u64 a = threadIdx.x * per < nb ? threadIdx.x * per : nb;
  const u64 b = a + per < nb ? a + per : nb;
  u64 s = 0;
  for (u64 i = a; i < b; i++) s += bt[i];
  u64 tot;
  u64 ex = block_excl<false>(s, tot);
  for (u64 i = a; i < b; i++) {
    const u64 x = bt[i];
    bt[i] = ex;
    ex += x;
  }
  if (threadIdx.x == 0) *total = tot;
}

__global__ void __launch_bounds__(256) k_sum_add(u64 *v, u64 m, const u64 *bt) {
  const u64 i0 = (u64)blockIdx.x * kScanBlock + threadIdx.x;
  const u64 base = bt[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanBlock; k += 256)
    if (i0 + k < m) v[i0 + k] += base;
}

// Copies slices src[off[i], off[i] + len[i]) to dst[dst_off[i], ...), a warp per slice.
__global__ void k_gather(const uint8_t *src, const u64 *off, const uint32_t *len, const u64 *dst_off, u64 n,
                         uint8_t *dst) {
  const u64 wid = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  for (u64 i = wid; i < n; i += ((u64)gridDim.x * blockDim.x) >> 5)
    for (uint32_t j = lane; j < len[i]; j += 32) dst[dst_off[i] + j] = src[off[i] + j];
}

template <typename T>
struct DBuf {  // device buffer that only grows
  T *p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t want) {  // grows by at least 1.5x (cudaFree synchronises the device)
    if (want <= n) return cudaSuccess;
    want = std::max(want + want / 8, n + n / 2);
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc((void **)&p, want * sizeof(T));
    if (e == cudaSuccess) n = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

}  // namespace

struct warpjq_csv {
  DBuf<uint8_t> in;  // device copy of host input
  DBuf<uint32_t> run_stat, tile_state, keys, key_off, g_len;  // keys: key texts by words; key_off: their meta
  DBuf<u64> tile_stat, tile_row, row_end, lens, bt, info, g_off, g_dst;
  DBuf<uint8_t> out, g_out;
  bool have_header = false;  // header names taken from an earlier chunk
  std::string key_text;
  std::vector<uint32_t> key_offs, key_words, key_meta;
  // chunks staged from host memory on a copy stream of their own
  DBuf<uint8_t> stage[2];
  cudaStream_t copy = nullptr;
  cudaEvent_t staged[2] = {nullptr, nullptr};
  ~warpjq_csv() {
    if (copy) cudaStreamSynchronize(copy);
    for (int b = 0; b < 2; b++) {
      stage[b].release();
      if (staged[b]) cudaEventDestroy(staged[b]);
    }
    if (copy) cudaStreamDestroy(copy);
    in.release();
    run_stat.release();
    tile_state.release();
    key_off.release();
    g_len.release();
    tile_stat.release();
    tile_row.release();
    row_end.release();
    lens.release();
    bt.release();
    info.release();
    g_off.release();
    g_dst.release();
    keys.release();
    out.release();
    g_out.release();
  }
};

extern "C" {

warpjq_status warpjq_csv_create(warpjq_csv **out) {
  if (!out) return WARPJQ_ERR_INVALID_ARG;
  *out = new (std::nothrow) warpjq_csv();
  return *out ? WARPJQ_OK : WARPJQ_ERR_OOM;
}

void warpjq_csv_destroy(warpjq_csv *c) { delete c; }

void warpjq_csv_reset(warpjq_csv *c) {
  if (!c) return;
  c->have_header = false;
  c->key_text.clear();
  c->key_offs.clear();
  c->key_words.clear();
  c->key_meta.clear();
}

warpjq_status warpjq_csv_convert(warpjq_csv *c, const uint8_t *src, uint64_t n, uint32_t flags, void *stream,
                                 const uint8_t **d_ndjson, uint64_t *ndjson_len, uint64_t *consumed,
                                 uint64_t *records, char *err, size_t err_len) {
  if (!c || (!src && n) || !d_ndjson || !ndjson_len || !consumed) {
    csv_err(err, err_len, "invalid argument");
    return WARPJQ_ERR_INVALID_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const bool final_ = (flags & WARPJQ_CSV_FINAL) != 0;
  *d_ndjson = nullptr;
  *ndjson_len = 0;
  *consumed = 0;
  if (records) *records = 0;
  if (n == 0) return WARPJQ_OK;
  const uint8_t *d = src;
  for (int b = 0; b < 2; b++)
    if ((flags & (WARPJQ_CSV_AFTER_STAGE0 << b)) && c->staged[b])
      CSV_CK(cudaStreamWaitEvent(st, c->staged[b], 0), "wait for a staged chunk");
  if (flags & WARPJQ_CSV_HOST_INPUT) {
    CSV_CK(c->in.ensure(n + 16), "device memory for the CSV input");
    CSV_CK(cudaMemcpyAsync(c->in.p, src, n, cudaMemcpyHostToDevice, st), "copy of the CSV input");
    d = c->in.p;
  }
  const u64 tiles = (n + kCsvTile - 1) / kCsvTile;
  CSV_CK(c->run_stat.ensure(tiles * kCsvThreads), "device memory for CSV rows");
  CSV_CK(c->tile_stat.ensure(tiles), "device memory for CSV rows");
  CSV_CK(c->tile_state.ensure(tiles), "device memory for CSV rows");
  CSV_CK(c->tile_row.ensure(tiles), "device memory for CSV rows");
  CSV_CK(c->info.ensure(4), "device memory for CSV rows");
  // rows ended by a newline outside quotes
  k_csv_stats<<<(unsigned)tiles, kCsvThreads, 0, st>>>(d, n, c->run_stat.p, c->tile_stat.p);
  k_csv_tiles<<<1, 1024, 0, st>>>(c->tile_stat.p, tiles, c->tile_state.p, c->tile_row.p, c->info.p);
  CSV_CK(cudaGetLastError(), "CSV row count");
  u64 nl_rows = 0;
  CSV_CK(cudaMemcpyAsync(&nl_rows, c->info.p, 8, cudaMemcpyDeviceToHost, st), "CSV row count");
  CSV_CK(cudaStreamSynchronize(st), "CSV row count");
  CSV_CK(c->row_end.ensure(nl_rows + 1), "device memory for CSV rows");
  k_csv_row_ends<<<(unsigned)tiles, kCsvThreads, 0, st>>>(d, n, c->run_stat.p, c->tile_state.p, c->tile_row.p,
                                                          c->row_end.p);
  k_csv_close<<<1, 1, 0, st>>>(c->row_end.p, n, final_ ? 1 : 0, c->info.p);
  CSV_CK(cudaGetLastError(), "CSV row ends");
  u64 info[3];
  CSV_CK(cudaMemcpyAsync(info, c->info.p, 24, cudaMemcpyDeviceToHost, st), "CSV row ends");
  CSV_CK(cudaStreamSynchronize(st), "CSV row ends");
  const u64 rows = info[0];
  u64 row0 = 0;
  if (!c->have_header) {
    if (rows == 0) return WARPJQ_OK;  // no whole row yet: the caller passes more bytes
    const u64 h_end = info[2];
    std::vector<uint8_t> head(h_end);
    if (h_end) {
      if (flags & WARPJQ_CSV_HOST_INPUT) memcpy(head.data(), src, h_end);
      else CSV_CK(cudaMemcpy(head.data(), d, h_end, cudaMemcpyDeviceToHost), "copy of the CSV header");
    }
    parse_header(head.data(), head.size(), c->key_text, c->key_offs);
    pack_keys(c->key_text, c->key_offs, c->key_words, c->key_meta);
    CSV_CK(c->keys.ensure(c->key_words.size() + 1), "device memory for CSV keys");
    CSV_CK(c->key_off.ensure(c->key_meta.size() + 1), "device memory for CSV keys");
    if (!c->key_words.empty())
      CSV_CK(cudaMemcpyAsync(c->keys.p, c->key_words.data(), c->key_words.size() * 4, cudaMemcpyHostToDevice, st),
             "copy of the CSV keys");
    if (!c->key_meta.empty())
      CSV_CK(cudaMemcpyAsync(c->key_off.p, c->key_meta.data(), c->key_meta.size() * 4, cudaMemcpyHostToDevice, st),
             "copy of the CSV keys");
    c->have_header = true;
    row0 = 1;
  }
  *consumed = info[1];
  const u64 m = rows - row0;
  if (records) *records = m;
  if (m == 0) return WARPJQ_OK;
  KeySet ks{c->keys.p, c->key_off.p, (uint32_t)(c->key_meta.size() / 2)};
  CSV_CK(c->lens.ensure(m + 1), "device memory for CSV lines");
  const unsigned grid = (unsigned)std::min<u64>((m + kJsonThreads - 1) / kJsonThreads, 148ull * 64);
  k_csv_json<false><<<grid, kJsonThreads, 0, st>>>(d, c->row_end.p, row0, rows, ks, c->lens.p, nullptr);
  const u64 nb = (m + kScanBlock - 1) / kScanBlock;
  CSV_CK(c->bt.ensure(nb), "device memory for CSV lines");
  k_sum_blocks<<<(unsigned)nb, 256, 0, st>>>(c->lens.p, m, c->bt.p);
  k_sum_totals<<<1, 1024, 0, st>>>(c->bt.p, nb, c->info.p + 3);
  k_sum_add<<<(unsigned)nb, 256, 0, st>>>(c->lens.p, m, c->bt.p);
  CSV_CK(cudaGetLastError(), "CSV line lengths");
  u64 total = 0;
  CSV_CK(cudaMemcpyAsync(&total, c->info.p + 3, 8, cudaMemcpyDeviceToHost, st), "CSV line lengths");
  CSV_CK(cudaStreamSynchronize(st), "CSV line lengths");
  CSV_CK(c->out.ensure(total + 16), "device memory for the NDJSON");
  k_csv_json<true><<<grid, kJsonThreads, 0, st>>>(d, c->row_end.p, row0, rows, ks, c->lens.p, c->out.p);
  CSV_CK(cudaGetLastError(), "CSV to NDJSON");
  *d_ndjson = c->out.p;
  *ndjson_len = total;
  return WARPJQ_OK;
}

warpjq_status warpjq_csv_stage(warpjq_csv *c, uint32_t buf, uint64_t at, const uint8_t *h_src, uint64_t n,
                               uint8_t **d_buf, char *err, size_t err_len) {
  if (!c || buf > 1 || (!h_src && n) || !d_buf) {
    csv_err(err, err_len, "invalid argument");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (!c->copy) {
    CSV_CK(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking), "copy stream");
    for (int b = 0; b < 2; b++) CSV_CK(cudaEventCreateWithFlags(&c->staged[b], cudaEventDisableTiming), "copy event");
  }
  if (c->stage[buf].n < at + n + 16) {  // the buffer's bytes do not survive growth
    CSV_CK(cudaStreamSynchronize(c->copy), "copy stream");
    CSV_CK(c->stage[buf].ensure(at + n + 16), "device memory for a staged chunk");
  }
  if (n) CSV_CK(cudaMemcpyAsync(c->stage[buf].p + at, h_src, n, cudaMemcpyHostToDevice, c->copy), "staging copy");
  CSV_CK(cudaEventRecord(c->staged[buf], c->copy), "staging copy");
  *d_buf = c->stage[buf].p;
  return WARPJQ_OK;
}

warpjq_status warpjq_csv_stage_wait(warpjq_csv *c, uint32_t buf, char *err, size_t err_len) {
  if (!c || buf > 1) return WARPJQ_ERR_INVALID_ARG;
  if (c->staged[buf]) CSV_CK(cudaEventSynchronize(c->staged[buf]), "staging copy");
  return WARPJQ_OK;
}

warpjq_status warpjq_csv_carry(warpjq_csv *c, const uint8_t *d_src, uint64_t n, uint32_t buf, uint64_t at,
                               void *stream, char *err, size_t err_len) {
  if (!c || buf > 1 || (!d_src && n) || at + n + 16 > c->stage[buf].n) {
    csv_err(err, err_len, "invalid argument");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (n)
    CSV_CK(cudaMemcpyAsync(c->stage[buf].p + at, d_src, n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream),
           "carried row copy");
  return WARPJQ_OK;
}

warpjq_status warpjq_csv_gather(warpjq_csv *c, const uint8_t *d_src, const uint64_t *offsets,
                                const uint32_t *lengths, uint64_t n, uint8_t *h_dst, void *stream, char *err,
                                size_t err_len) {
  if (!c || (n && (!offsets || !lengths || !h_dst))) {  // d_src null: offsets are addresses
    csv_err(err, err_len, "invalid argument");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (!n) return WARPJQ_OK;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<u64> dst(n);
  u64 total = 0;
  for (u64 i = 0; i < n; i++) {
    dst[i] = total;
    total += lengths[i];
  }
  CSV_CK(c->g_off.ensure(n), "device memory for a gather");
  CSV_CK(c->g_dst.ensure(n), "device memory for a gather");
  CSV_CK(c->g_len.ensure(n), "device memory for a gather");
  CSV_CK(c->g_out.ensure(total + 1), "device memory for a gather");
  CSV_CK(cudaMemcpyAsync(c->g_off.p, offsets, n * 8, cudaMemcpyHostToDevice, st), "gather offsets");
  CSV_CK(cudaMemcpyAsync(c->g_dst.p, dst.data(), n * 8, cudaMemcpyHostToDevice, st), "gather offsets");
  CSV_CK(cudaMemcpyAsync(c->g_len.p, lengths, n * 4, cudaMemcpyHostToDevice, st), "gather offsets");
  const unsigned grid = (unsigned)std::min<u64>((n + 7) / 8, 148ull * 16);
  k_gather<<<grid, 256, 0, st>>>(d_src, c->g_off.p, c->g_len.p, c->g_dst.p, n, c->g_out.p);
  CSV_CK(cudaGetLastError(), "gather");
  if (total) CSV_CK(cudaMemcpyAsync(h_dst, c->g_out.p, total, cudaMemcpyDeviceToHost, st), "gather copy");
  CSV_CK(cudaStreamSynchronize(st), "gather");
  return WARPJQ_OK;
}

warpjq_status warpjq_device_read(void *h_dst, const void *d_src, uint64_t n, void *stream, char *err,
                                 size_t err_len) {
  if (!n) return WARPJQ_OK;
  if (!h_dst || !d_src) return WARPJQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  CSV_CK(cudaMemcpyAsync(h_dst, d_src, n, cudaMemcpyDeviceToHost, st), "device to host copy");
  CSV_CK(cudaStreamSynchronize(st), "device to host copy");
  return WARPJQ_OK;
}

}  // extern "C"
