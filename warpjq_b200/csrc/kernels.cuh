// The sm_100a scan kernels.
//
// The hot path of the reference's k_nl_count / k_nl_write / k_build_lines /
// k_eval / DeviceSelect / k_row_len / k_emit chain (warpjq_kernels.cu:
// 1117-1849) as one scan pass plus, for row output, two small passes:
//
//   k_scan      One warp per CTA.  A warp takes the next tile from a work
//               ticket and stages tile + halo into shared memory with one
//               bulk (TMA) copy.  Stage 1 is lane-parallel over 32-byte
//               chunks: each chunk becomes two bit masks, its newlines and
//               its "special" bytes ('"', '\\', < 0x20).  The lines that
//               start in the tile are listed from the newline masks, and
//               stage 2 walks them one line per lane (walker.cuh), jumping
//               through strings by the special mask: validation, path
//               resolution, the filter, and either the aggregate or a
//               compact record per selected row (line offset, row length,
//               field spans).
//   k_rows_*    Rows only: block sums and an exclusive prefix over the
//               per-tile (rows, bytes, lines) totals, then the rows are
//               copied in line order from the input to the output.
//
// No host synchronisation happens inside a run and no kernel waits on
// another CTA.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/warpjq_kernels.h"
#include "devutil.cuh"
#include "fixsum.cuh"
#include "plan.h"
#include "walker.cuh"

namespace wjq {

constexpr int kThreads = 32;                 // one warp per CTA; each warp owns its tile
constexpr uint32_t kMaxLinesPerPass = 128;   // line-start list capacity per pass
constexpr int kReduceThreads = 128;          // block size of the per-tile reductions
// Register budgets of k_scan (warps per SM), measured per variant on the
// nginx workload: the ungrouped aggregate at 24 (80 registers; more warps
// hide more latency than its few spills cost), the row variant at 20 (96
// registers, which keep its record writing from spilling) and the group-by
// variants at 16 (128 registers).
constexpr int kScanBlocksPerSM = 24;
constexpr int kScanBlocksPerSMRows = 20;
constexpr int kScanBlocksPerSMGrouped = 16;

constexpr int kGroupCache = 16;  // per-CTA group accumulators kept in shared memory

// A CTA's line counts and ungrouped aggregate, in shared memory: each round
// of up to 32 lines is reduced in the warp (ballots, warp reductions) and
// lane 0 adds the round's totals here, so no lane keeps accumulators in
// registers through the walk.  Flushed to the run's counters at the end of
// the CTA (or of each tile, in a batch).
struct CtaAcc {
  unsigned long long lines, blank, invalid, type, sel;
  unsigned long long count, numeric, n_int;
  unsigned long long isum_lo, isum_hi;  // exact 128-bit sum of the integer values
  unsigned long long min_bits, max_bits;
  uint32_t saw;  // a selected line had a non-numeric, non-null value
  uint32_t pad;
  __device__ void clear() {
    lines = blank = invalid = type = sel = count = numeric = n_int = isum_lo = isum_hi = 0;
    min_bits = ~0ull;
    max_bits = 0;
    saw = 0;
  }
};

// Readable bytes kept past a window's data: the end sentinel, the walker's
// word reads after a line's newline, and the last chunk's 32-byte read.
constexpr uint32_t kWinSlack = 64;

// Shared-memory layout of k_scan for tile T and halo H: the window bytes,
// then the special and newline masks (one word per 32-byte chunk, the
// sentinel's chunk included), the CTA's exact FP sum, the mbarrier the
// tile copies complete on, the line-start list, and for grouped aggregates
// the group cache.  Nothing is static, so the dynamic size may be raised
// to the device's whole opt-in limit.
__host__ __device__ inline uint32_t scan_win_bytes(uint32_t T, uint32_t H) {
  return (T + H + kWinSlack + 15u) & ~15u;
}
__host__ __device__ inline uint32_t scan_chunk_words(uint32_t T, uint32_t H) {
  return ((T + H) / 32 + 2 + 3) & ~3u;
}
__host__ __device__ inline size_t scan_smem_base(uint32_t T, uint32_t H) {
  size_t s = scan_win_bytes(T, H);
  s += 2 * (size_t)scan_chunk_words(T, H) * sizeof(uint32_t);
  s += kFixDigits * sizeof(long long);
  s += sizeof(CtaAcc);
  s += sizeof(unsigned long long);  // the mbarrier of the tile copies
  s += (kMaxLinesPerPass + 2) * sizeof(uint16_t);
  return (s + 15) & ~(size_t)15;
}

// Record of one selected row, staged per CTA until the look-back resolves.
struct RowRec {
  unsigned long long line_start;  // absolute offset of the line
  uint32_t line_len;              // without '\n' and without a trailing '\r'
  uint32_t ordinal;               // line index within the tile
  uint32_t local_off;             // row offset within the tile's output
  uint32_t row_len;
  uint32_t pad[2];
  // followed by n_fields x {uint32 off (relative to line), uint32 len|kind<<28|esc<<27}
};
static_assert(sizeof(RowRec) == kRowRecBytes, "row record header size");

// One group key's accumulators, 128 bytes: the counts, the exact integer
// sum and min/max in the first 64, the exact sum of the non-integer values
// (fixsum.cuh) in the second.
struct GroupAcc {
  unsigned long long count, numeric, isum_lo, isum_hi, n_int, min_bits, max_bits;
  double fbig;                // non-integer values of magnitude >= 2^128
  long long fix[kFixDigits];  // the other non-integer values, exactly
};
static_assert(sizeof(GroupAcc) == 128, "group accumulator record");

__device__ __forceinline__ void group_acc_init(GroupAcc &a) {
  a.count = a.numeric = a.isum_lo = a.isum_hi = a.n_int = 0;
  a.min_bits = ~0ull;
  a.max_bits = 0;
  a.fbig = 0.0;
#pragma unroll
  for (int k = 0; k < kFixDigits; k++) a.fix[k] = 0;
}

// Adds a non-integer value to exact limbs (global or shared memory) with
// independent atomics; values too large for the limbs go to *big.
__device__ __forceinline__ void fix_atomic_add(long long *limbs, double *big, double v) {
  const FixParts pr = fix_split(v);
  if (pr.d == -2) {
    atomicAdd(big, v);
    return;
  }
  if (pr.d < 0) return;
#pragma unroll
  for (int k = 0; k < 3; k++)
    if (pr.part[k] && pr.d + k < kFixDigits)
      atomicAdd((unsigned long long *)&limbs[pr.d + k], (unsigned long long)pr.part[k]);
}

// Where a group key's bytes are (the first line that inserted it).
struct GroupKeyDesc {
  unsigned long long off;  // absolute input offset of the key bytes (string: body)
  uint32_t len;
  uint32_t input;           // batch input the key belongs to (0 for one input)
  uint8_t kind;
  uint8_t esc;
  uint8_t saw_non_numeric;  // a selected line had a non-numeric, non-null value
  uint8_t pad[5];
};
static_assert(sizeof(GroupKeyDesc) == 24, "group key descriptor");

// A CTA's private accumulators for up to kGroupCache keys (direct-mapped by
// key id), merged into the global records when the CTA finishes.  Hot keys
// then cost shared-memory atomics instead of contended global ones.
struct GroupCache {
  uint32_t tag[kGroupCache];  // key id held by the entry, or 0xFFFFFFFF
  GroupAcc acc[kGroupCache];
};

__host__ __device__ inline size_t scan_smem_bytes(uint32_t T, uint32_t H, bool groups) {
  return scan_smem_base(T, H) + (groups ? sizeof(GroupCache) : 0);
}

struct GroupTable {
  unsigned long long *slots;  // 0 = empty, else (hash << 32) | (key_id + 1)
  uint32_t cap_mask;
  uint32_t key_cap;
  GroupKeyDesc *keys;
  GroupAcc *acc;
};

// Per-tile totals of a rows run.
struct RowTile {
  unsigned long long rec_begin;  // the tile's first record in the record arena
  unsigned long long bytes;      // output bytes of the tile's rows
  uint32_t rows;
  uint32_t pad;
};

struct ScanParams {
  const uint8_t *data;
  unsigned long long n;
  uint32_t tile_bytes;
  uint32_t halo_bytes;
  unsigned long long n_tiles;
  RunCounters *ctr;
  TileDesc *tiles;
  // rows mode: per-tile totals and the record arena (rec_cap_per_cta
  // records per CTA, appended over all the CTA's tiles)
  RowTile *row_tiles;
  uint8_t *rec_scratch;
  unsigned long long rec_cap_per_cta;
  GroupTable g;
  // deep-nesting scratch, per CTA
  uint32_t *deep_words;
  unsigned long long deep_levels_per_cta;
  // Batched runs (tile_input null for one input): input i is
  // data[in_start[i], in_end[i]) and owns tiles [in_tile0[i], in_tile0[i+1]);
  // its counters and aggregate go to in_ctr[i].
  const uint32_t *tile_input;
  const unsigned long long *in_start;
  const unsigned long long *in_end;
  const unsigned long long *in_tile0;
  RunCounters *in_ctr;
  uint32_t any_rows;    // a mixed batch one of whose plans prints rows (its
                        // aggregate launches write empty row tiles)
  uint32_t rec_stride;  // bytes per row record (a mixed batch: the largest of its plans')
  // A mixed batch runs as one launch per distinct plan: this launch takes
  // its tiles from tile_list[0, n_list) (null: every tile) by tickets from
  // *ticket (null: ctr->next_tile), and a CTA's records follow those its
  // earlier launches of the batch appended (rec_cursor, one count per CTA,
  // read at the start and written back at the end; null: none).
  const uint32_t *tile_list;
  unsigned long long n_list;
  unsigned long long *ticket;
  unsigned long long *rec_cursor;
};

// Rows emission.
struct EmitParams {
  const uint8_t *data;
  const DevPlan *plan;
  // A mixed batch: tile t's rows are rendered by plans[in_plan[tile_input[t]]]
  // (null otherwise).
  const DevPlan *plans;
  const uint32_t *in_plan;
  const uint32_t *tile_input;
  uint32_t rec_stride;
  const RowTile *row_tiles;
  const TileDesc *tiles;
  unsigned long long n_tiles;
  const unsigned long long *block_prefix;  // 3 per block of tiles_per_block tiles
  uint32_t tiles_per_block;
  const uint8_t *recs;
  uint8_t *out;
  unsigned long long out_cap;
  unsigned long long *row_off;   // rows_cap + 1
  unsigned long long *line_idx;  // rows_cap
  unsigned long long rows_cap;
  RunCounters *ctr;
};

// ---------------------------------------------------------------------------
// Group table (open addressing; the key is published with one 64-bit CAS
// that carries its hash and a dense key id whose descriptor was written and
// fenced before the CAS).
// ---------------------------------------------------------------------------

struct KeyRef {
  const uint8_t *p;  // key bytes (string: body)
  uint32_t len;
  uint8_t kind;      // JK_NULL for missing/null keys
  uint8_t esc;
  uint32_t input;    // batch input of the line (keys of different inputs differ)
  unsigned long long abs_off;
};

__device__ __forceinline__ bool key_bytes_equal(const KeyRef &a, const uint8_t *bp, uint32_t blen,
                                                uint8_t besc) {
  if (!a.esc && !besc) {
    if (a.len != blen) return false;
    for (uint32_t k = 0; k < blen; k++)
      if (a.p[k] != bp[k]) return false;
    return true;
  }
  StrDecoder x(a.p, a.len), y(bp, blen);
  for (;;) {
    int u = x.next(), w = y.next();
    if (u != w) return false;
    if (u < 0) return true;
  }
}

// Returns the key id, or 0xFFFFFFFF when the table is full (the overflow flag
// is raised and the run is repeated with a bigger table).
__device__ uint32_t group_find_or_insert(const ScanParams &sp, const KeyRef &k, uint32_t h) {
  const GroupTable &g = sp.g;
  uint32_t pos = h & g.cap_mask;
  uint32_t mine = 0xFFFFFFFFu;
  for (uint32_t probe = 0; probe <= g.cap_mask; probe++) {
    unsigned long long w = *(volatile unsigned long long *)&g.slots[pos];
    if (w == 0) {
      if (mine == 0xFFFFFFFFu) {
        mine = atomicAdd(&sp.ctr->n_keys, 1u);
        if (mine >= g.key_cap) {
          atomicOr(&sp.ctr->overflow, 4u);
          return 0xFFFFFFFFu;
        }
        GroupKeyDesc d = {};
        d.off = k.abs_off;
        d.len = k.len;
        d.input = k.input;
        d.kind = k.kind;
        d.esc = k.esc;
        g.keys[mine] = d;
        __threadfence();
      }
      unsigned long long want = ((unsigned long long)h << 32) | (mine + 1ull);
      unsigned long long old = atomicCAS(&g.slots[pos], 0ull, want);
      if (old == 0) return mine;
      w = old;
    }
    if ((uint32_t)(w >> 32) == h) {
      uint32_t kid = (uint32_t)w - 1;
      __threadfence();
      const GroupKeyDesc d = g.keys[kid];
      if (d.kind == k.kind && d.input == k.input && key_bytes_equal(k, sp.data + d.off, d.len, d.esc))
        return kid;
    }
    pos = (pos + 1) & g.cap_mask;
  }
  atomicOr(&sp.ctr->overflow, 4u);
  return 0xFFFFFFFFu;
}

// ---------------------------------------------------------------------------
// Row rendering.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t csv_cell_len(const uint8_t *p, uint32_t n, bool decode) {
  // RFC 4180 quoting as output.rs:45-61 does it, over raw or decoded bytes.
  uint32_t len = 0, quotes = 0;
  bool need = false;
  if (!decode) {
    for (uint32_t k = 0; k < n; k++) {
      uint32_t c = p[k];
      if (c == '"') quotes++;
      if (c == ',' || c == '"' || c == '\n' || c == '\r') need = true;
    }
    len = n;
  } else {
    StrDecoder d(p, n);
    for (int c; (c = d.next()) >= 0;) {
      len++;
      if (c == '"') quotes++;
      if (c == ',' || c == '"' || c == '\n' || c == '\r') need = true;
    }
  }
  return need ? len + quotes + 2 : len;
}

__device__ __forceinline__ uint32_t csv_cell_write(uint8_t *dst, const uint8_t *p, uint32_t n,
                                                   bool decode, uint32_t expect_len) {
  // expect_len tells whether quoting applies (it differs from the bare length).
  uint32_t w = 0;
  uint32_t bare = 0;
  if (!decode) bare = n;
  else {
    StrDecoder d(p, n);
    while (d.next() >= 0) bare++;
  }
  bool quote = expect_len != bare;
  if (quote) dst[w++] = '"';
  if (!decode) {
    for (uint32_t k = 0; k < n; k++) {
      if (quote && p[k] == '"') dst[w++] = '"';
      dst[w++] = p[k];
    }
  } else {
    StrDecoder d(p, n);
    for (int c; (c = d.next()) >= 0;) {
      if (quote && c == '"') dst[w++] = '"';
      dst[w++] = (uint8_t)c;
    }
  }
  if (quote) dst[w++] = '"';
  return w;
}

// Length of a value cell in CSV mode (output.rs:65-81).
__device__ __forceinline__ uint32_t csv_value_len(const uint8_t *line, const SlotVal &s) {
  if (s.kind == JK_MISSING || s.kind == JK_NULL) return 0;
  if (s.kind == JK_STR) return csv_cell_len(line + s.off + 1, s.len - 2, s.esc);
  return csv_cell_len(line + s.off, s.len, false);
}

// Computes the row length of a selected line.
__device__ __forceinline__ uint32_t row_length(const DevPlan &P, const uint8_t *line,
                                               uint32_t line_len, const SlotVal *slots) {
  switch (P.output_kind) {
    case 0:  // passthrough (output.rs:204-217)
      return (P.csv_mode ? csv_cell_len(line, line_len, false) : line_len) + 1;
    case 1: {  // single value (output.rs:220-231)
      const SlotVal &s = slots[P.out_slot];
      if (P.csv_mode) return csv_value_len(line, s) + 1;
      return (s.kind == JK_MISSING ? 4 : s.len) + 1;
    }
    default: {  // projection (output.rs:234-264, prefixes rendered by lower.rs:63-87)
      uint32_t len = P.suffix_len + 1;
      for (uint32_t f = 0; f < P.n_fields; f++) {
        const SlotVal &s = slots[P.field_slot[f]];
        len += P.prefix_len[f];
        if (P.csv_mode) len += csv_value_len(line, s);
        else len += s.kind == JK_MISSING ? 4 : s.len;
      }
      return len;
    }
  }
}

// Warp-cooperative copy of n bytes: each lane loads four bytes 32 apart
// before storing them, so one step moves 128 bytes with the loads in flight
// together (lanes stride by 32: coalesced accesses).
__device__ __forceinline__ void warp_copy(uint8_t *dst, const uint8_t *src, uint32_t n, int lane) {
  for (uint32_t base = 0; base < n; base += 128) {
    const uint32_t k0 = base + lane;
    uint8_t b0 = 0, b1 = 0, b2 = 0, b3 = 0;
    if (k0 < n) b0 = src[k0];
    if (k0 + 32 < n) b1 = src[k0 + 32];
    if (k0 + 64 < n) b2 = src[k0 + 64];
    if (k0 + 96 < n) b3 = src[k0 + 96];
    if (k0 < n) dst[k0] = b0;
    if (k0 + 32 < n) dst[k0 + 32] = b1;
    if (k0 + 64 < n) dst[k0 + 64] = b2;
    if (k0 + 96 < n) dst[k0 + 96] = b3;
  }
}

// Segment s of a value or projection row (JSON output): the value of the
// single path, or prefix 0, value 0, prefix 1, value 1, ..., then the
// suffix; the last segment is the newline.
__device__ __forceinline__ const uint8_t *row_segment(const DevPlan &P, const uint8_t *line,
                                                      const uint32_t *fields, uint32_t nf,
                                                      uint32_t s, uint32_t &len) {
  const bool proj = P.output_kind == 2;
  const uint32_t n_before_suffix = proj ? 2 * nf : nf;
  if (s < n_before_suffix) {
    const uint32_t f = proj ? s >> 1 : s;
    if (proj && !(s & 1)) {
      len = P.prefix_len[f];
      return P.blob + P.prefix_off[f];
    }
    const uint32_t off = fields[2 * f], lk = fields[2 * f + 1];
    if ((lk >> 28) == JK_MISSING) {
      len = 4;
      return (const uint8_t *)"null";
    }
    len = lk & 0x07FFFFFFu;
    return line + off;
  }
  if (proj && s == n_before_suffix) {
    len = P.suffix_len;
    return P.blob + P.suffix_off;
  }
  len = 1;
  return (const uint8_t *)"\n";
}

// Writes one row.  All lanes of the warp call it together.
__device__ void emit_row(const DevPlan &P, const uint8_t *line, const RowRec &r,
                         const uint32_t *fields, uint8_t *dst, int lane) {
  if (P.output_kind == 0) {
    if (!P.csv_mode) {
      warp_copy(dst, line, r.line_len, lane);
      if (lane == 0) dst[r.line_len] = '\n';
    } else if (lane == 0) {
      uint32_t w = csv_cell_write(dst, line, r.line_len, false, r.row_len - 1);
      dst[w] = '\n';
    }
    return;
  }
  uint32_t nf = P.output_kind == 1 ? 1 : P.n_fields;
  if (P.csv_mode) {
    if (lane != 0) return;
    uint32_t w = 0;
    for (uint32_t f = 0; f < nf; f++) {
      if (P.output_kind == 2)
        for (uint32_t k = 0; k < P.prefix_len[f]; k++) dst[w++] = P.blob[P.prefix_off[f] + k];
      uint32_t off = fields[2 * f], lk = fields[2 * f + 1];
      uint32_t kind = lk >> 28, esc = (lk >> 27) & 1, len = lk & 0x07FFFFFFu;
      if (kind == JK_MISSING || kind == JK_NULL) continue;
      const uint8_t *vp = line + off;
      if (kind == JK_STR) {
        uint32_t L = csv_cell_len(vp + 1, len - 2, esc);
        w += csv_cell_write(dst + w, vp + 1, len - 2, esc, L);
      } else {
        uint32_t L = csv_cell_len(vp, len, false);
        w += csv_cell_write(dst + w, vp, len, false, L);
      }
    }
    dst[w] = '\n';
    return;
  }
  // The row as a list of segments (value, or prefix/value pairs then the
  // suffix, then the newline); lane l writes output bytes l, l+32, ...,
  // finding each byte's segment with a cursor that only moves forward, and
  // loads four bytes before storing them.
  const uint32_t L = r.row_len;
  uint32_t s = 0, soff = 0, slen;
  const uint8_t *sp = row_segment(P, line, fields, nf, 0, slen);
  for (uint32_t base = 0; base < L; base += 128) {
    uint8_t bb[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t b = base + lane + 32 * k;
      bb[k] = 0;
      if (b < L) {
        while (b >= soff + slen) {
          soff += slen;
          sp = row_segment(P, line, fields, nf, ++s, slen);
        }
        bb[k] = sp[b - soff];
      }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t b = base + lane + 32 * k;
      if (b < L) dst[b] = bb[k];
    }
  }
}

// ---------------------------------------------------------------------------
// The scan kernel.
// ---------------------------------------------------------------------------

// The 128-bit sum over the lanes of `grp` of their signed 64-bit values
// (0 where `on` is false): three parts of at most 22 bits, which cannot
// overflow 32 bits over 32 lanes, recombined with the negatives' borrow.
__device__ __forceinline__ void group_sum128(unsigned grp, bool on, long long v, unsigned long long &lo,
                                             unsigned long long &hi) {
  const unsigned long long u = on ? (unsigned long long)v : 0ull;
  const uint32_t p0 = __reduce_add_sync(grp, (uint32_t)(u & 0x1FFFFFu));
  const uint32_t p1 = __reduce_add_sync(grp, (uint32_t)((u >> 21) & 0x1FFFFFu));
  const uint32_t p2 = __reduce_add_sync(grp, (uint32_t)(u >> 42));
  const uint32_t nneg = __popc(__ballot_sync(0xffffffffu, on && v < 0) & grp);
  const unsigned __int128 t = (unsigned __int128)p0 + ((unsigned __int128)p1 << 21) +
                              ((unsigned __int128)p2 << 42) - ((unsigned __int128)nneg << 64);
  lo = (unsigned long long)t;
  hi = (unsigned long long)(t >> 64);
}

// The extreme (min or max) over the lanes of `grp` of 64-bit keys (lanes
// with `on` false hold none): the high words first, then the low words of
// the lanes holding the extreme high word.
__device__ __forceinline__ unsigned long long group_extreme(unsigned grp, bool on, unsigned long long ob,
                                                            bool mn) {
  const uint32_t none = mn ? 0xFFFFFFFFu : 0u;
  const uint32_t h = on ? (uint32_t)(ob >> 32) : none;
  const uint32_t eh = mn ? __reduce_min_sync(grp, h) : __reduce_max_sync(grp, h);
  const uint32_t l = (on && h == eh) ? (uint32_t)ob : none;
  const uint32_t el = mn ? __reduce_min_sync(grp, l) : __reduce_max_sync(grp, l);
  return ((unsigned long long)eh << 32) | el;
}

// One-CTA mbarrier (a tile's bulk copy completes on it) and the 1-D bulk
// (TMA) copy from this GPU's own global memory into shared memory.  The
// copy is single-CTA, with no cluster multicast.
constexpr uint32_t kWaitLimit = 1u << 22;  // try_wait rounds before a wait gives up

__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Issued by one lane: expects `bytes` (a multiple of 16, src and dst 16-byte
// aligned) on the barrier, then starts the copy.  The proxy fence orders the
// warp's earlier generic reads of `dst` before the copy's writes.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint32_t bar) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Hint: bring `bytes` (a multiple of 16, src 16-byte aligned) of this GPU's
// global memory into L2; nothing waits for it.
__device__ __forceinline__ void l2_prefetch(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}

// Waits (bounded) for the barrier's phase of parity `phase` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (uint32_t it = 0; it < kWaitLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16-byte global -> shared copy that does not go through registers; bytes
// past `src_bytes` (0..16) are zero-filled and not read.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes)
               : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(0xffffffffu, x, d);
  return x;
}

// Exclusive warp scan of (a, b) in lane order, with the warp totals.
__device__ __forceinline__ void warp_scan2(uint32_t a, unsigned long long b, uint32_t &ea,
                                           unsigned long long &eb, uint32_t &ta,
                                           unsigned long long &tb) {
  const int lane = threadIdx.x & 31;
  uint32_t ia = a;
  unsigned long long ib = b;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t xa = __shfl_up_sync(0xffffffffu, ia, d);
    unsigned long long xb = __shfl_up_sync(0xffffffffu, ib, d);
    if (lane >= d) {
      ia += xa;
      ib += xb;
    }
  }
  ea = ia - a;
  eb = ib - b;
  ta = __shfl_sync(0xffffffffu, ia, 31);
  tb = __shfl_sync(0xffffffffu, ib, 31);
}

// Adds the CTA's counts and (ungrouped) aggregate to `dst` and clears them;
// `also` (a batch's totals, may be null) receives the line counts too.  The
// non-integer values' exact sum, gathered in the CTA's shared limbs
// `cta_fix`, goes into dst's limbs (and the shared limbs are cleared).
__device__ __noinline__ void flush_counts(RunCounters *dst, RunCounters *also, const DevPlan &P, bool rows,
                                          int lane, CtaAcc *acc, long long *cta_fix) {
  __syncwarp();
  if (lane == 0) {
    for (RunCounters *c : {dst, also}) {
      if (!c) continue;
      if (acc->lines) atomicAdd(&c->n_lines, acc->lines);
      if (acc->blank) atomicAdd(&c->n_blank, acc->blank);
      if (acc->invalid) atomicAdd(&c->n_invalid, acc->invalid);
      if (acc->type) atomicAdd(&c->n_type_error, acc->type);
      if (acc->sel) atomicAdd(&c->n_selected, acc->sel);
    }
    if (!rows && P.group_slot < 0 && P.output_kind == 3) {
      if (acc->count) atomicAdd(&dst->agg_count, acc->count);
      if (acc->numeric) atomicAdd(&dst->agg_numeric, acc->numeric);
      if (acc->n_int) atomicAdd(&dst->agg_n_int, acc->n_int);
      const unsigned long long lo = acc->isum_lo, hi = acc->isum_hi;
      if (lo || hi) {
        const unsigned long long old = atomicAdd(&dst->agg_isum_lo, lo);
        const unsigned long long carry = (old + lo) < old;
        if (hi + carry) atomicAdd(&dst->agg_isum_hi, hi + carry);
      }
      if (acc->numeric) {
        atomicMin(&dst->agg_min_bits, acc->min_bits);
        atomicMax(&dst->agg_max_bits, acc->max_bits);
      }
    }
    if (!rows && acc->saw) atomicOr(&dst->agg_saw_non_numeric, 1u);
    acc->clear();
  }
  if (!rows && P.group_slot < 0 && P.output_kind == 3 && lane < kFixDigits) {
    const long long v = cta_fix[lane];
    cta_fix[lane] = 0;
    if (v) atomicAdd((unsigned long long *)&dst->fix[lane], (unsigned long long)v);
  }
  __syncwarp();
}

// The plan is a kernel parameter (constant bank): fields at fixed offsets
// are instruction operands, and no plan read goes through global memory.
// kGroups: the group-by path is compiled in (grouped aggregates); without
// it the kernel is lighter for every other query.
template <bool kRows, bool kGroups = false>
__global__ void __launch_bounds__(kThreads, kGroups ? kScanBlocksPerSMGrouped : (kRows ? kScanBlocksPerSMRows : kScanBlocksPerSM))
    k_scan(const __grid_constant__ ScanParams sp, const __grid_constant__ DevPlan plan) {
  extern __shared__ __align__(16) uint8_t smem[];
  const DevPlan &P = plan;
  const uint32_t T = sp.tile_bytes, H = sp.halo_bytes;
  const uint32_t nwords = scan_chunk_words(T, H);
  uint8_t *win = smem;                                              // window bytes (+ slack)
  uint32_t *smask = (uint32_t *)(smem + scan_win_bytes(T, H));      // special bytes per chunk
  uint32_t *nlmask = smask + nwords;                                // newlines per chunk
  long long *cta_fix = (long long *)(nlmask + nwords);              // the CTA's exact FP sum
  CtaAcc *acc = (CtaAcc *)(cta_fix + kFixDigits);                   // the CTA's counts and aggregate
  unsigned long long *s_bar = (unsigned long long *)(acc + 1);       // tile copies' mbarrier
  uint16_t *lstart = (uint16_t *)(s_bar + 1);                       // kMaxLinesPerPass + 2
  GroupCache *gcache = (GroupCache *)(smem + scan_smem_base(T, H));  // grouped aggregates only

  const int lane = threadIdx.x;
  const uint32_t rec_stride = sp.rec_stride;
  uint8_t *my_recs = sp.rec_scratch + (unsigned long long)blockIdx.x * sp.rec_cap_per_cta * rec_stride;
  DeepStack deep;
  deep.words = sp.deep_words + (unsigned long long)blockIdx.x * (sp.deep_levels_per_cta / 32);
  deep.cap_levels = sp.deep_levels_per_cta;

  // records this CTA has appended (rows mode)
  unsigned long long cta_recs = (kRows && sp.rec_cursor) ? sp.rec_cursor[blockIdx.x] : 0;
  NodeVals nv;
  SlotVal slots[kMaxSlots];

  if (lane < kFixDigits) cta_fix[lane] = 0;
  if (lane == 0) acc->clear();
  const bool grouped = kGroups && !kRows && P.group_slot >= 0;
  if (grouped) {
    for (int k = lane; k < kGroupCache; k += 32) {
      gcache->tag[k] = 0xFFFFFFFFu;
      group_acc_init(gcache->acc[k]);
    }
  }
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(s_bar);
  if (lane == 0) mbar_init(bar);
  __syncwarp();
  uint32_t phase = 0;  // parity of the barrier's current phase

  // Tickets are taken one tile ahead, so the atomic's latency overlaps a
  // tile's work.
  unsigned long long *const ticket_ctr = sp.ticket ? sp.ticket : &sp.ctr->next_tile;
  unsigned long long next_ticket = 0;
  if (lane == 0) next_ticket = atomicAdd(ticket_ctr, 1ull);
  const unsigned long long n_work = sp.tile_list ? sp.n_list : sp.n_tiles;
  for (;;) {
    const unsigned long long ticket = __shfl_sync(0xffffffffu, next_ticket, 0);
    if (ticket >= n_work) break;
    const unsigned long long tile = sp.tile_list ? sp.tile_list[ticket] : ticket;
    if (lane == 0) next_ticket = atomicAdd(ticket_ctr, 1ull);
    // The tile's input: the whole data, or one input of a batch (a window
    // never reaches past its input's end).
    uint32_t input = 0;
    unsigned long long data_start = 0, data_end = sp.n, ts = tile * T;
    RunCounters *ctr_in = sp.ctr;
    if (sp.tile_input) {
      input = sp.tile_input[tile];
      data_start = sp.in_start[input];
      data_end = sp.in_end[input];
      ts = data_start + (tile - sp.in_tile0[input]) * T;
      ctr_in = sp.in_ctr + input;
    }
    const uint32_t nf = P.output_kind == 2 ? P.n_fields : (P.output_kind == 1 ? 1u : 0u);
    const unsigned long long te = min(ts + T, data_end);
    const uint32_t tlen = (uint32_t)(te - ts);
    const uint32_t wlen = (uint32_t)min((unsigned long long)T + H, data_end - ts);
    const bool win_reaches_end = ts + wlen == data_end;

    // 1. Stage tile + halo: the window's 16-byte multiple by one bulk copy
    //    (inputs and tiles start 16-byte aligned), its last 0-15 bytes by
    //    plain loads, so nothing past the input is read.
    const uint32_t body = wlen & ~15u;
    __syncwarp();  // the previous tile's reads of the window are done
    if (lane == 0 && body) bulk_load(win, sp.data + ts, body, bar);
    if (lane < (wlen & 15u)) win[body + lane] = sp.data[ts + body + lane];
    const uint32_t prev_nl = (ts == data_start || sp.data[ts - 1] == '\n') ? 1u : 0u;
    if (body) {
      if (!mbar_wait(bar, phase)) {
        // the copy did not complete within the wait limit: report, give it
        // another bounded wait (it writes this CTA's shared memory), stop
        if (lane == 0) atomicOr(&sp.ctr->error, 2u);
        mbar_wait(bar, phase);
        return;
      }
      phase ^= 1u;
    }
    if (lane == 0 && win_reaches_end) win[wlen] = '\n';  // ends the last line for the walker
    __syncwarp();

    // 2. Stage 1, lane-parallel: every 32-byte chunk of the window (the end
    //    sentinel's too) becomes its special and newline masks; lane l owns
    //    chunks [l*K, l*K + K) and counts the line starts among them.
    const uint32_t limit = wlen + (win_reaches_end ? 1u : 0u);  // classified bytes
    const uint32_t nchunks = (limit + 31) >> 5;
    const uint32_t K = (nchunks + 31) >> 5;
    const uint32_t c0 = lane * K;
    const uint32_t nl_limit = tlen - 1;  // newlines below this start a line in the tile
    auto listed = [&](uint32_t c, uint32_t m) -> uint32_t {
      const uint32_t base = c * 32;
      if (base >= nl_limit) return 0u;
      if (nl_limit - base < 32) m &= (1u << (nl_limit - base)) - 1u;
      return m;
    };
    uint32_t my_nl = 0;
    unsigned long long nz = 0;  // bit k: chunk c0 + k lists a line start
    for (uint32_t k = 0; k < K; k++) {
      const uint32_t c = c0 + k;
      if (c >= nchunks) break;
      const uint4 u = ((const uint4 *)win)[2 * c];
      const uint4 v = ((const uint4 *)win)[2 * c + 1];
      const uint32_t w8[8] = {u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w};
      uint32_t sm_c;
      uint32_t nl_c = classify_chunk(w8, &sm_c);
      const uint32_t rem = limit - c * 32;
      if (rem < 32) {  // bytes past the window's data are stale
        sm_c &= (1u << rem) - 1u;
        nl_c &= (1u << rem) - 1u;
      }
      smask[c] = sm_c;
      nlmask[c] = nl_c;
      const uint32_t lm = listed(c, nl_c);
      if (lm) {
        my_nl += __popc(lm);
        nz |= 1ull << k;
      }
    }

    // The next tile's window is fetched into L2 now (its ticket has
    // arrived), so its bulk copy reads from L2 rather than waiting on HBM.
    if (lane == 0 && next_ticket < n_work) {
      const unsigned long long nt = sp.tile_list ? sp.tile_list[next_ticket] : next_ticket;
      {
        unsigned long long ns = nt * T, ne = sp.n;
        if (sp.tile_input) {
          const uint32_t ni = sp.tile_input[nt];
          ns = sp.in_start[ni] + (nt - sp.in_tile0[ni]) * T;
          ne = sp.in_end[ni];
        }
        const uint32_t nb = (uint32_t)min((unsigned long long)T + H, ne - ns) & ~15u;
        if (nb) l2_prefetch(sp.data + ns, nb);
      }
    }

    // 3. Lines starting in the tile: ts itself (after a newline) and q+1 for
    //    every newline q in [ts, te-1).
    uint32_t first_nl, tot_nl;
    unsigned long long dummy_e, dummy_t;
    warp_scan2(my_nl, 0ull, first_nl, dummy_e, tot_nl, dummy_t);
    const uint32_t lead = prev_nl;
    const uint32_t n_lines_tile = tot_nl + lead;

    // 4. Walk the lines, one per lane, in passes of the list's capacity.
    unsigned long long tile_rows = 0, tile_bytes = 0;
    const unsigned long long tile_rec0 = cta_recs;
    uint32_t tile_first_invalid = 0xFFFFFFFFu, tile_first_type = 0xFFFFFFFFu;
    for (uint32_t base = 0; base < n_lines_tile; base += kMaxLinesPerPass) {
      const uint32_t cnt = min(n_lines_tile - base, kMaxLinesPerPass);
      // list line starts [base, base + cnt] (one extra as the end marker)
      if (lead && lane == 0 && base == 0) lstart[0] = 0;
      {
        uint32_t idx = first_nl + lead;
        if (my_nl && idx <= base + cnt && idx + my_nl > base) {
          for (unsigned long long z = nz; z; z &= z - 1) {
            const uint32_t k = (uint32_t)__ffsll((long long)z) - 1u;
            uint32_t m = listed(c0 + k, nlmask[c0 + k]);
            while (m) {
              uint32_t b = (c0 + k) * 32 + (uint32_t)__ffs(m) - 1;
              m &= m - 1;
              if (idx >= base && idx <= base + cnt) lstart[idx - base] = (uint16_t)(b + 1);
              idx++;
            }
          }
        }
      }
      __syncwarp();
      for (uint32_t b0 = 0; b0 < cnt; b0 += 32) {
        const uint32_t li = b0 + lane;  // line index within the pass
        int status = -1;
        uint32_t has_row = 0, row_len = 0;
        unsigned long long line_abs = 0;
        uint32_t line_len = 0, ordinal = base + li;
        const uint8_t *lp = nullptr;
        bool has_group = false;
        KeyRef gk;
        uint32_t gh = 0;
        SlotVal aggv;
        aggv.kind = JK_MISSING;
        if (li < cnt) {
          uint32_t s = lstart[li];
          uint32_t e;  // window offset of the newline (or of the data end)
          bool found = true;
          if (base + li + 1 < n_lines_tile) {
            // the next line's start is listed (the list keeps one entry past
            // the pass for exactly this)
            e = (uint32_t)lstart[li + 1] - 1;
          } else {
            // last line of the tile: its newline is at or after te - 1 (the
            // sentinel's, when the window reaches the data's end)
            uint32_t q = tlen - 1;
            if (q < s) q = s;
            uint32_t c = q >> 5;
            uint32_t m = c < nchunks ? (nlmask[c] & (0xFFFFFFFFu << (q & 31))) : 0u;
            while (!m && ++c < nchunks) m = nlmask[c];
            if (m) e = c * 32 + (uint32_t)__ffs(m) - 1;
            else found = false;
          }
          line_abs = ts + s;
          if (found) {
            lp = win + s;
            line_len = e - s;
            status = walk_objects(P, win, smask, s, e, nv);
            if (status == LS_FALLBACK) status = walk_masked(P, win, smask, s, e, nv);
          } else {
            // longer than the window: walk it from global memory
            unsigned long long q = ts + wlen;
            while (q < data_end && sp.data[q] != '\n') q++;
            lp = sp.data + line_abs;
            line_len = (uint32_t)(q - line_abs);
            status = walk_line(P, lp, line_len, nv, nullptr);
          }
        }
        // Lines nesting past 64 levels share this CTA's deep stack, so they
        // are walked one at a time.
        if (__any_sync(0xffffffffu, status == LS_DEEP)) {
          for (int t = 0; t < 32; t++) {
            if (lane == t && status == LS_DEEP) {
              status = walk_line(P, lp, line_len, nv, &deep);
              if (status == LS_DEEP_FULL) {
                atomicOr(&sp.ctr->overflow, 8u);
                status = LS_INVALID;
              }
            }
            __syncwarp();
          }
        }
        // `line_len` for output excludes a trailing '\r' (chunk.rs:433-435).
        uint32_t out_len = line_len;
        if (status >= 0 && out_len && lp[out_len - 1] == '\r') out_len--;

        if (status == LS_OK) {
          uint32_t type_err_filter = 0, type_err_post = 0;
          for (uint32_t s = 0; s < P.n_slots; s++) {
            slots[s] = resolve_slot(P, nv, s);
            if (slots[s].state == SS_TYPE_ERROR) {
              if ((P.filter_slot_mask >> s) & 1) type_err_filter = 1;
              else type_err_post = 1;
            }
          }
          if (type_err_filter) {
            status = LS_TYPE_ERROR;
          } else if (P.has_filter && !eval_filter(P, lp, slots)) {
            status = 100;  // filtered out
          } else if (type_err_post) {
            status = LS_TYPE_ERROR;
          } else {
            status = 101;  // selected
          }
        }
        if (status == LS_INVALID) {
          tile_first_invalid = min(tile_first_invalid, ordinal);
        } else if (status == LS_TYPE_ERROR) {
          tile_first_type = min(tile_first_type, ordinal);
        } else if (status == 101) {
          if (kRows) {
            has_row = 1;
            row_len = row_length(P, lp, out_len, slots);
          } else {
            // aggregate (exec/cpu.rs:358-369, agg.rs:44-71)
            if (P.agg_slot >= 0) aggv = slots[P.agg_slot];
            if (kGroups && P.group_slot >= 0) {
              const SlotVal &g = slots[P.group_slot];
              has_group = true;
              gk.esc = 0;
              gk.input = input;
              if (g.kind == JK_MISSING || g.kind == JK_NULL) {
                gk.kind = JK_NULL;
                gk.p = lp;
                gk.len = 0;
                gk.abs_off = line_abs;
              } else if (g.kind == JK_STR) {
                gk.kind = JK_STR;
                gk.p = lp + g.off + 1;
                gk.len = g.len - 2;
                gk.esc = g.esc;
                gk.abs_off = line_abs + g.off + 1;
              } else {
                gk.kind = g.kind;
                gk.p = lp + g.off;
                gk.len = g.len;
                gk.abs_off = line_abs + g.off;
              }
              gh = (gk.kind == JK_STR ? hash_str_body(gk.p, gk.len, gk.esc) : hash_raw(gk.p, gk.len)) ^
                   (gk.kind * 0x9E3779B9u) ^ (input * 0x85EBCA6Bu);
              if (gh == 0) gh = 1;
            }
          }
        }

        // Aggregate contribution of this line.
        bool contrib = !kRows && status == 101;
        long long iv = 0;
        double fv = 0.0;
        bool is_int = false, is_num = false;
        bool saw = false;
        if (contrib && P.agg_slot >= 0) {
          if (aggv.kind == JK_NUM) {
            fv = parse_number(lp + aggv.off, aggv.len, is_int, iv);
            is_num = true;
          } else if (aggv.kind != JK_MISSING && aggv.kind != JK_NULL) {
            saw = true;
          }
        }
        // The round's counts and ungrouped aggregate, reduced in the warp
        // and added to the CTA's shared accumulator by lane 0.
        {
          const unsigned full = 0xffffffffu;
          const unsigned m_blank = __ballot_sync(full, status == LS_BLANK);
          const unsigned m_inv = __ballot_sync(full, status == LS_INVALID);
          const unsigned m_type = __ballot_sync(full, status == LS_TYPE_ERROR);
          const unsigned m_sel = __ballot_sync(full, status == 101);
          const unsigned m_saw = __ballot_sync(full, saw);
          const bool ung = contrib && !has_group;
          const unsigned m_cnt = __ballot_sync(full, ung);
          const unsigned m_num = __ballot_sync(full, ung && is_num);
          const unsigned m_int = __ballot_sync(full, ung && is_num && is_int);
          unsigned long long s_lo = 0, s_hi = 0, ext = 0;
          const uint32_t ak = P.agg_kind;
          if (m_int && (ak == WARPJQ_AGG_SUM || ak == WARPJQ_AGG_AVG))
            group_sum128(full, ung && is_num && is_int, iv, s_lo, s_hi);
          if (m_num && (ak == WARPJQ_AGG_MIN || ak == WARPJQ_AGG_MAX))
            ext = group_extreme(full, ung && is_num, order_bits(fv), ak == WARPJQ_AGG_MIN);
          if (ung && is_num && !is_int && (ak == WARPJQ_AGG_SUM || ak == WARPJQ_AGG_AVG))
            fix_atomic_add(cta_fix, &ctr_in->fbig, fv);  // exact, in the CTA's shared limbs
          if (lane == 0) {
            acc->blank += __popc(m_blank);
            acc->invalid += __popc(m_inv);
            acc->type += __popc(m_type);
            acc->sel += __popc(m_sel);
            if (m_saw) acc->saw = 1;
            if (m_cnt) {
              acc->count += __popc(m_cnt);
              acc->numeric += __popc(m_num);
              acc->n_int += __popc(m_int);
              if (s_lo || s_hi) {
                const unsigned long long o = acc->isum_lo;
                acc->isum_lo = o + s_lo;
                acc->isum_hi += s_hi + (acc->isum_lo < o ? 1ull : 0ull);
              }
              if (m_num && ak == WARPJQ_AGG_MIN) acc->min_bits = min(acc->min_bits, ext);
              if (m_num && ak == WARPJQ_AGG_MAX) acc->max_bits = max(acc->max_bits, ext);
            }
          }
        }
        if (kGroups && !kRows && P.group_slot >= 0) {
          // Lanes whose keys hash alike compare their key bytes with the
          // lowest such lane; only lanes that differ from it look up the
          // table themselves.
          const uint32_t hv = has_group ? gh : 0u;
          const unsigned peers = __match_any_sync(0xffffffffu, hv);
          const int leader = __ffs(peers) - 1;
          const unsigned long long lp = __shfl_sync(0xffffffffu, (unsigned long long)gk.p, leader);
          const uint32_t llen = __shfl_sync(0xffffffffu, gk.len, leader);
          const uint32_t lkind = __shfl_sync(0xffffffffu, (uint32_t)gk.kind, leader);
          const uint32_t lesc = __shfl_sync(0xffffffffu, (uint32_t)gk.esc, leader);
          const uint32_t linput = __shfl_sync(0xffffffffu, input, leader);
          const bool same = has_group && lane != leader && gk.kind == lkind && input == linput &&
                            key_bytes_equal(gk, (const uint8_t *)lp, llen, (uint8_t)lesc);
          uint32_t kid = 0xFFFFFFFFu;
          if (has_group && !same) kid = group_find_or_insert(sp, gk, gh);
          const uint32_t lkid = __shfl_sync(0xffffffffu, kid, leader);
          if (same) kid = lkid;
          // Lanes holding the same key add up their contributions in the
          // warp first; one lane per key then updates its accumulators
          // (counts, the exact integer sum, min or max).  Fractional values
          // go in per lane, exactly (fixsum.cuh).
          const unsigned grp = __match_any_sync(0xffffffffu, kid);
          const bool lead = kid != 0xFFFFFFFFu && lane == __ffs(grp) - 1;
          const bool num_int = is_num && is_int;
          const unsigned m_num = __ballot_sync(0xffffffffu, is_num) & grp;
          const unsigned m_int = __ballot_sync(0xffffffffu, num_int) & grp;
          const uint32_t ak = P.agg_kind;
          unsigned long long s_lo = 0, s_hi = 0, ext = 0;
          if ((ak == WARPJQ_AGG_SUM || ak == WARPJQ_AGG_AVG) && __any_sync(0xffffffffu, num_int))
            group_sum128(grp, num_int, iv, s_lo, s_hi);
          if ((ak == WARPJQ_AGG_MIN || ak == WARPJQ_AGG_MAX) && __any_sync(0xffffffffu, is_num))
            ext = group_extreme(grp, is_num, order_bits(fv), ak == WARPJQ_AGG_MIN);
          if (kid != 0xFFFFFFFFu && (lead || (is_num && !is_int))) {  // no key id: the table is full
            // This CTA's cached entry for the key if it has (or can claim)
            // one, else the global record.
            GroupAcc *ap = &sp.g.acc[kid];
            const uint32_t e = kid & (kGroupCache - 1);
            uint32_t t = *(volatile uint32_t *)&gcache->tag[e];
            if (t == 0xFFFFFFFFu) {
              const uint32_t prev = atomicCAS(&gcache->tag[e], 0xFFFFFFFFu, kid);
              t = prev == 0xFFFFFFFFu ? kid : prev;
            }
            if (t == kid) ap = &gcache->acc[e];
            GroupAcc &a = *ap;
            if (lead) {
              atomicAdd(&a.count, (unsigned long long)__popc(grp));
              if (m_num) atomicAdd(&a.numeric, (unsigned long long)__popc(m_num));
              if (m_int) {
                atomicAdd(&a.n_int, (unsigned long long)__popc(m_int));
                if (s_lo || s_hi) {
                  const unsigned long long old = atomicAdd(&a.isum_lo, s_lo);
                  const unsigned long long carry = (old + s_lo) < old ? 1ull : 0ull;
                  if (s_hi + carry) atomicAdd(&a.isum_hi, s_hi + carry);
                }
              }
              if (m_num && ak == WARPJQ_AGG_MIN) atomicMin(&a.min_bits, ext);
              if (m_num && ak == WARPJQ_AGG_MAX) atomicMax(&a.max_bits, ext);
            }
            if (is_num && !is_int && (ak == WARPJQ_AGG_SUM || ak == WARPJQ_AGG_AVG))
              fix_atomic_add(a.fix, &a.fbig, fv);
          }
          if (kid != 0xFFFFFFFFu && !is_num && aggv.kind != JK_MISSING && aggv.kind != JK_NULL &&
              P.agg_slot >= 0)
            sp.g.keys[kid].saw_non_numeric = 1;
        }

        if (kRows) {
          uint32_t er, tr;
          unsigned long long eb, tb;
          warp_scan2(has_row, (unsigned long long)row_len, er, eb, tr, tb);
          if (has_row) {
            unsigned long long ri = cta_recs + er;
            if (ri < sp.rec_cap_per_cta) {
              RowRec *r = (RowRec *)(my_recs + ri * rec_stride);
              r->line_start = line_abs;
              r->line_len = out_len;
              r->ordinal = ordinal;
              r->local_off = (uint32_t)(tile_bytes + eb);
              r->row_len = row_len;
              uint32_t *fl = (uint32_t *)(r + 1);
              for (uint32_t f = 0; f < nf; f++) {
                const SlotVal &s = slots[P.output_kind == 1 ? P.out_slot : P.field_slot[f]];
                fl[2 * f] = s.off;
                fl[2 * f + 1] = s.len | ((uint32_t)s.kind << 28) | ((uint32_t)s.esc << 27);
              }
            } else {
              atomicOr(&sp.ctr->overflow, 1u);
            }
          }
          tile_rows += tr;
          tile_bytes += tb;
          cta_recs += tr;
        }
      }
      __syncwarp();
    }
    if (lane == 0) acc->lines += n_lines_tile;

    // Per-tile bookkeeping.
    tile_first_invalid = __reduce_min_sync(0xffffffffu, tile_first_invalid);
    tile_first_type = __reduce_min_sync(0xffffffffu, tile_first_type);
    if (lane == 0) {
      sp.tiles[tile].n_lines = n_lines_tile;
      sp.tiles[tile].first_invalid = tile_first_invalid;
      sp.tiles[tile].first_type_error = tile_first_type;
      if (tile_first_invalid != 0xFFFFFFFFu) {
        atomicMin(&sp.ctr->first_invalid_tile, tile);
        if (sp.tile_input) atomicMin(&ctr_in->first_invalid_tile, tile);
      }
      if (tile_first_type != 0xFFFFFFFFu) {
        atomicMin(&sp.ctr->first_type_tile, tile);
        if (sp.tile_input) atomicMin(&ctr_in->first_type_tile, tile);
      }
    }
    if (kRows || sp.any_rows) {  // an aggregate tile of a batch with rows has none
      if (lane == 0) {
        RowTile rt;
        rt.rec_begin = (unsigned long long)blockIdx.x * sp.rec_cap_per_cta + tile_rec0;
        rt.bytes = tile_bytes;
        rt.rows = (uint32_t)tile_rows;
        rt.pad = 0;
        sp.row_tiles[tile] = rt;
      }
    }
    // A batch input's counts and aggregate go to its own record, tile by tile.
    if (sp.tile_input)
      flush_counts(ctr_in, sp.ctr, P, kRows, lane, acc, cta_fix);
  }

  // Merge this CTA's cached group accumulators into the global records.
  if (grouped) {
    __syncwarp();
    for (int k = lane; k < kGroupCache; k += 32) {
      const uint32_t kid = gcache->tag[k];
      if (kid == 0xFFFFFFFFu) continue;
      const GroupAcc c = gcache->acc[k];
      GroupAcc &a = sp.g.acc[kid];
      if (c.count) atomicAdd(&a.count, c.count);
      if (c.numeric) {
        atomicAdd(&a.numeric, c.numeric);
        atomicMin(&a.min_bits, c.min_bits);
        atomicMax(&a.max_bits, c.max_bits);
      }
      if (c.n_int) {
        const unsigned long long old = atomicAdd(&a.isum_lo, c.isum_lo);
        const unsigned long long carry = (old + c.isum_lo) < old ? 1ull : 0ull;
        if (c.isum_hi + carry) atomicAdd(&a.isum_hi, c.isum_hi + carry);
        atomicAdd(&a.n_int, c.n_int);
      }
      if (c.numeric > c.n_int) {
        for (int d = 0; d < kFixDigits; d++)
          if (c.fix[d]) atomicAdd((unsigned long long *)&a.fix[d], (unsigned long long)c.fix[d]);
        if (c.fbig != 0.0) atomicAdd(&a.fbig, c.fbig);
      }
    }
  }

  if (kRows && sp.rec_cursor && lane == 0) sp.rec_cursor[blockIdx.x] = cta_recs;
  // Flush this CTA's counters (a batch's were flushed per tile).
  flush_counts(sp.ctr, nullptr, P, kRows, lane, acc, cta_fix);
}

// The index of the first invalid / type-error line: lines of the tiles
// before the first tile holding one, summed in two passes (contiguous blocks
// of tiles, then one warp over the block sums).
__global__ void k_reduce_tiles(unsigned long long n_tiles, const TileDesc *tiles, RunCounters *ctr,
                               unsigned long long *block_lines) {
  __shared__ unsigned long long s_l[kReduceThreads], s_t[kReduceThreads];
  unsigned long long per = (n_tiles + gridDim.x - 1) / gridDim.x;
  unsigned long long b0 = blockIdx.x * per, b1 = min(b0 + per, n_tiles);
  unsigned long long cut = ctr->first_invalid_tile, cut_t = ctr->first_type_tile;
  unsigned long long lines = 0, lines_t = 0;
  unsigned long long chunk = (b1 > b0 ? b1 - b0 : 0);
  unsigned long long cper = (chunk + kReduceThreads - 1) / kReduceThreads;
  unsigned long long c0 = b0 + threadIdx.x * cper, c1 = min(c0 + cper, b1);
  for (unsigned long long t = c0; t < c1 && (t < cut || t < cut_t); t++) {
    if (t < cut) lines += tiles[t].n_lines;
    if (t < cut_t) lines_t += tiles[t].n_lines;
  }
  s_l[threadIdx.x] = lines;
  s_t[threadIdx.x] = lines_t;
  __syncthreads();
  for (int d = kReduceThreads / 2; d > 0; d >>= 1) {
    if (threadIdx.x < d) {
      s_l[threadIdx.x] += s_l[threadIdx.x + d];
      s_t[threadIdx.x] += s_t[threadIdx.x + d];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    block_lines[2 * blockIdx.x] = s_l[0];
    block_lines[2 * blockIdx.x + 1] = s_t[0];
  }
}

// The run's FP totals from its exact limbs (the integer sum joins them
// before the one rounding of sum_total).
__device__ __forceinline__ void finalize_sums(RunCounters &c) {
  c.fsum_total = fix_to_double(c.fix, 0, 0) + c.fbig;
  c.sum_total = fix_to_double(c.fix, c.agg_isum_lo, c.agg_isum_hi) + c.fbig;
}

// One warp: the block sums of k_reduce_tiles, then the first bad lines and
// the FP totals.
__global__ void k_finalize(const unsigned long long *block_lines, unsigned nblocks, const TileDesc *tiles,
                           RunCounters *ctr) {
  const int lane = threadIdx.x;
  unsigned long long lines = 0, lines_t = 0;
  for (unsigned b = lane; b < nblocks; b += 32) {
    lines += block_lines[2 * b];
    lines_t += block_lines[2 * b + 1];
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    lines += __shfl_down_sync(0xffffffffu, lines, d);
    lines_t += __shfl_down_sync(0xffffffffu, lines_t, d);
  }
  if (lane != 0) return;
  finalize_sums(*ctr);
  unsigned long long cut = ctr->first_invalid_tile, cut_t = ctr->first_type_tile;
  ctr->first_invalid = cut == ~0ull ? ~0ull : lines + tiles[cut].first_invalid;
  ctr->first_type_error = cut_t == ~0ull ? ~0ull : lines_t + tiles[cut_t].first_type_error;
}

// Batched runs: every input's record starts like a fresh run's.
__global__ void k_batch_reset(RunCounters *in_ctr, uint32_t n_inputs) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_inputs; i += gridDim.x * blockDim.x) {
    RunCounters z;
    memset(&z, 0, sizeof(z));
    z.first_invalid_tile = ~0ull;
    z.first_type_tile = ~0ull;
    z.agg_min_bits = ~0ull;
    z.first_invalid = ~0ull;
    z.first_type_error = ~0ull;
    in_ctr[i] = z;
  }
}

// The largest i in [0, n) with a[i] <= t (a[0] <= t, a ascending).
__device__ __forceinline__ uint32_t last_at_or_below(const unsigned long long *a, uint32_t n,
                                                     unsigned long long t) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (a[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// A batch's per-tile tables, built on the device from its per-input ones
// (host work stays proportional to the inputs, not the tiles): tile t
// belongs to the input i with in_tile0[i] <= t < in_tile0[i + 1] (an empty
// input owns none, so the last input starting at or below t is its owner).
// A mixed batch also lists, plan after plan, the tiles of each plan's
// inputs: position p of list_tiles is tile p - list_tile0[j] of input
// list_inputs[j] (list_tile0 running over the inputs in list order).
__global__ void k_batch_expand(unsigned long long n_tiles, uint32_t n_inputs, const unsigned long long *in_tile0,
                               uint32_t *tile_input, const uint32_t *list_inputs,
                               const unsigned long long *list_tile0, uint32_t *list_tiles) {
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_tiles;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    tile_input[t] = last_at_or_below(in_tile0, n_inputs, t);
    if (list_tiles) {
      const uint32_t j = last_at_or_below(list_tile0, n_inputs, t);
      const uint32_t i = list_inputs[j];
      list_tiles[t] = (uint32_t)(in_tile0[i] + (t - list_tile0[j]));
    }
  }
}

// Batched runs, one warp per input: the input's first invalid / type-error
// line (lane l sums a contiguous slice of the input's tiles' line counts)
// and its FP totals.
__global__ void k_batch_finalize(const TileDesc *tiles, const unsigned long long *in_tile0,
                                 RunCounters *in_ctr, uint32_t n_inputs) {
  const int lane = threadIdx.x & 31;
  const unsigned long long i = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n_inputs) return;  // uniform per warp
  const unsigned long long t0 = in_tile0[i], t1 = in_tile0[i + 1];
  RunCounters &c = in_ctr[i];
  const unsigned long long cut = c.first_invalid_tile, cut_t = c.first_type_tile;
  const unsigned long long per = (t1 - t0 + 31) / 32;
  const unsigned long long a = min(t0 + lane * per, t1), b = min(a + per, t1);
  unsigned long long lines = 0, lines_t = 0;
  for (unsigned long long t = a; t < b && (t < cut || t < cut_t); t++) {
    if (t < cut) lines += tiles[t].n_lines;
    if (t < cut_t) lines_t += tiles[t].n_lines;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    lines += __shfl_down_sync(0xffffffffu, lines, d);
    lines_t += __shfl_down_sync(0xffffffffu, lines_t, d);
  }
  if (lane != 0) return;
  finalize_sums(c);
  c.first_invalid = cut == ~0ull ? ~0ull : lines + tiles[cut].first_invalid;
  c.first_type_error = cut_t == ~0ull ? ~0ull : lines_t + tiles[cut_t].first_type_error;
}

// ---------------------------------------------------------------------------
// Rows: prefix over the per-tile totals, then emission in line order.
// ---------------------------------------------------------------------------

// Tiles per block of the rows passes (a multiple of 32, chosen per run by
// rows_tiles_per_block): small runs take 32 so their row copies still spread
// over hundreds of blocks, large ones 128 for fewer, fuller blocks.
constexpr int kEmitThreads = 128;
__host__ __device__ inline uint32_t rows_tiles_per_block(unsigned long long n_tiles) {
  return n_tiles < 148ull * 128 ? 32u : 128u;
}
constexpr int kPrefixThreads = 1024;  // the one block that scans the block sums

// Exclusive block scan of three u64 values in thread order, with totals.
template <int NT>
__device__ __forceinline__ void block_scan3(const unsigned long long v[3], unsigned long long ex[3],
                                            unsigned long long tot[3],
                                            unsigned long long (*s_w)[NT / 32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long inc[3] = {v[0], v[1], v[2]};
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      unsigned long long x = __shfl_up_sync(0xffffffffu, inc[k], d);
      if (lane >= d) inc[k] += x;
    }
  }
  if (lane == 31)
    for (int k = 0; k < 3; k++) s_w[k][warp] = inc[k];
  __syncthreads();
  for (int k = 0; k < 3; k++) {
    unsigned long long before = 0, all = 0;
    for (int w = 0; w < NT / 32; w++) {
      if (w < warp) before += s_w[k][w];
      all += s_w[k][w];
    }
    ex[k] = before + inc[k] - v[k];
    tot[k] = all;
  }
  __syncthreads();
}

// Pass 1: (rows, bytes, lines) summed per block of `tpb` tiles.
__global__ void __launch_bounds__(kEmitThreads)
    k_rows_block_sums(const RowTile *rt, const TileDesc *td, unsigned long long n_tiles,
                      uint32_t tpb, unsigned long long *bsum) {
  __shared__ unsigned long long s_w[3][kEmitThreads / 32];
  const unsigned long long t0 = (unsigned long long)blockIdx.x * tpb;
  unsigned long long v[3] = {0, 0, 0};
  for (uint32_t k = threadIdx.x; k < tpb; k += kEmitThreads) {
    unsigned long long t = t0 + k;
    if (t < n_tiles) {
      v[0] += rt[t].rows;
      v[1] += rt[t].bytes;
      v[2] += td[t].n_lines;
    }
  }
  unsigned long long ex[3], tot[3];
  block_scan3<kEmitThreads>(v, ex, tot, s_w);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) bsum[blockIdx.x * 3 + k] = tot[k];
}

// Pass 2 (one block): block sums -> exclusive block prefixes, in place; the
// totals give the output length and the closing row offset.  Output that
// does not fit raises the overflow flag (the run is repeated with room).
__global__ void __launch_bounds__(kPrefixThreads)
    k_rows_block_prefix(unsigned long long *bsum, unsigned nblocks, RunCounters *ctr,
                        unsigned long long *row_off, unsigned long long rows_cap,
                        unsigned long long out_cap) {
  __shared__ unsigned long long s_w[3][kPrefixThreads / 32];
  const unsigned per = (nblocks + kPrefixThreads - 1) / kPrefixThreads;
  const unsigned b0 = threadIdx.x * per, b1 = min(b0 + per, nblocks);
  unsigned long long v[3] = {0, 0, 0};
  for (unsigned b = b0; b < b1; b++)
    for (int k = 0; k < 3; k++) v[k] += bsum[b * 3 + k];
  unsigned long long ex[3], tot[3];
  block_scan3<kPrefixThreads>(v, ex, tot, s_w);
  for (unsigned b = b0; b < b1; b++)
    for (int k = 0; k < 3; k++) {
      unsigned long long x = bsum[b * 3 + k];
      bsum[b * 3 + k] = ex[k];
      ex[k] += x;
    }
  if (threadIdx.x == 0) {
    ctr->out_len = tot[1];
    if (tot[0] > rows_cap || tot[1] > out_cap) atomicOr(&ctr->overflow, 2u);
    else row_off[tot[0]] = tot[1];
  }
}

// Pass 3: each block takes its `tiles_per_block` tiles kEmitThreads at a time:
// per-tile prefixes by a block scan, then each warp copies whole tiles'
// rows, one row at a time, from the input to the output.
__global__ void __launch_bounds__(kEmitThreads) k_rows_emit(EmitParams ep) {
  __shared__ unsigned long long s_w[3][kEmitThreads / 32];
  __shared__ unsigned long long s_pre[3][kEmitThreads];
  __shared__ unsigned long long s_rec[kEmitThreads];
  __shared__ uint32_t s_rows[kEmitThreads];
  if (ep.ctr->overflow & 3u) return;  // the run is repeated with bigger buffers
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t rec_stride = ep.rec_stride;
  unsigned long long carry[3];
  for (int k = 0; k < 3; k++) carry[k] = ep.block_prefix[blockIdx.x * 3 + k];
  const uint32_t tpb = ep.tiles_per_block;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * tpb;
  for (uint32_t sub = 0; sub < tpb; sub += kEmitThreads) {
    if (t0 + sub >= ep.n_tiles) break;
    const unsigned long long t = t0 + sub + threadIdx.x;
    unsigned long long v[3] = {0, 0, 0};
    unsigned long long rec = 0;
    if (sub + threadIdx.x < tpb && t < ep.n_tiles) {
      const RowTile rt = ep.row_tiles[t];
      v[0] = rt.rows;
      v[1] = rt.bytes;
      v[2] = ep.tiles[t].n_lines;
      rec = rt.rec_begin;
    }
    unsigned long long ex[3], tot[3];
    block_scan3<kEmitThreads>(v, ex, tot, s_w);
    for (int k = 0; k < 3; k++) s_pre[k][threadIdx.x] = carry[k] + ex[k];
    s_rec[threadIdx.x] = rec;
    s_rows[threadIdx.x] = (uint32_t)v[0];
    __syncthreads();
    const int n_here = (int)min((uint32_t)kEmitThreads, tpb - sub);
    for (int i = warp; i < n_here; i += kEmitThreads / 32) {
      const uint32_t rows = s_rows[i];
      if (!rows) continue;
      const DevPlan &P = ep.plans ? ep.plans[ep.in_plan[ep.tile_input[t0 + sub + i]]] : *ep.plan;
      const unsigned long long row0 = s_pre[0][i], byte0 = s_pre[1][i], line0 = s_pre[2][i];
      for (uint32_t r = 0; r < rows; r++) {
        const RowRec *rr = (const RowRec *)(ep.recs + (s_rec[i] + r) * rec_stride);
        const uint32_t *fl = (const uint32_t *)(rr + 1);
        const unsigned long long dst_off = byte0 + rr->local_off;
        emit_row(P, ep.data + rr->line_start, *rr, fl, ep.out + dst_off, lane);
        if (lane == 0) {
          ep.row_off[row0 + r] = dst_off;
          ep.line_idx[row0 + r] = line0 + rr->ordinal;
        }
      }
    }
    for (int k = 0; k < 3; k++) carry[k] += tot[k];
    __syncthreads();
  }
}

}  // namespace wjq
