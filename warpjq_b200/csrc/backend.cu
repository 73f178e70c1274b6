// The warpjq device backend for sm_100a: the C ABI of warpjq_kernels.h
// (reference crates/warpjq-core/cuda/warpjq_kernels.h:238-274) and the
// device-resident extension of warpjq_ext.h.
//
// Per run the backend launches four kernels on one stream -- reset, scan,
// tile reduction, finalize -- with no host synchronisation in between.
// Device buffers that depend on the data (row records, output bytes, the
// group table, the deep-nesting stack) start at a size that fits ordinary
// input and are grown when the scan reports that one was too small; the run
// is then repeated on the device, so every line is always decided there.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/warpjq_ext.h"
#include "../../include/warpjq_kernels.h"
#include "kernels.cuh"
#include "plan.h"
#include "plan_build.h"

using namespace wjq;

namespace {


#define CK(call, what)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      set_err(err, err_len, "%s: %s", what, cudaGetErrorString(e_));                      \
      return e_ == cudaErrorMemoryAllocation ? WARPJQ_ERR_OOM : WARPJQ_ERR_CUDA;          \
    }                                                                                     \
  } while (0)

// ---------------------------------------------------------------------------
// Device buffers of one run, sized for an input length.
// ---------------------------------------------------------------------------

template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  // Grows to at least `want`; a buffer that grows again takes 1.5x its old
  // size, so inputs of varying size reallocate only a few times.  Growth is
  // stream-ordered on `st` (the launch stream, whose earlier runs on this
  // buffer have been collected): the old block returns to the device's
  // memory pool and the new one comes from it without synchronising the
  // device, so other streams' work runs on.  Never during a graph capture.
  cudaError_t ensure(size_t want, cudaStream_t st, bool capturing) {
    if (want <= n && p) return cudaSuccess;
    if (capturing) return cudaErrorStreamCaptureUnsupported;
    const size_t grown = n ? std::max(want, n + n / 2) : want;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMallocAsync((void **)&p, std::max<size_t>(grown, 1) * sizeof(T), st);
    if (e == cudaSuccess) n = grown;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct RunBufs {
  DevBuf<RunCounters> ctr;
  DevBuf<TileDesc> tiles;
  DevBuf<RowTile> row_tiles;
  DevBuf<unsigned long long> row_bsum;
  // batched runs: tile -> input table, inputs' extents and first tiles, and
  // one counter record per input
  DevBuf<uint32_t> b_tile_input;
  DevBuf<unsigned long long> b_in_start, b_in_end, b_in_tile0;
  DevBuf<RunCounters> b_in_ctr;
  // mixed batches: the inputs' distinct plans, each input's plan index, the
  // inputs in plan order with their running tile counts, the tiles of each
  // plan's inputs (one list after another, built on the device), each
  // plan's launch's ticket counter and the row launches' per-CTA record
  // counts
  DevBuf<DevPlan> b_plans;
  DevBuf<uint32_t> b_in_plan;
  DevBuf<uint32_t> b_list_inputs;
  DevBuf<unsigned long long> b_list_tile0;
  DevBuf<uint32_t> b_plan_tiles;
  DevBuf<unsigned long long> b_tickets, b_rec_cursor;
  DevBuf<uint8_t> recs;
  DevBuf<uint8_t> out;
  DevBuf<unsigned long long> row_off, line_idx;
  DevBuf<unsigned long long> block_lines;
  DevBuf<uint32_t> deep;
  // group table
  DevBuf<unsigned long long> g_slots;
  DevBuf<GroupKeyDesc> g_keys;
  DevBuf<GroupAcc> g_acc;

  // current capacities
  unsigned long long rec_cap_per_cta = 0;
  unsigned long long out_cap = 0;
  unsigned long long rows_cap = 0;
  uint32_t g_cap = 0;      // table slots (power of two)
  uint32_t g_key_cap = 0;
  unsigned long long deep_levels = 0;

  void release() {
    ctr.release(); tiles.release(); row_tiles.release(); row_bsum.release();
    b_tile_input.release(); b_in_start.release(); b_in_end.release(); b_in_tile0.release();
    b_in_ctr.release();
    b_plans.release();
    b_in_plan.release();
    b_list_inputs.release();
    b_list_tile0.release();
    b_plan_tiles.release();
    b_tickets.release();
    b_rec_cursor.release();
    recs.release(); out.release(); row_off.release(); line_idx.release();
    block_lines.release(); deep.release(); g_slots.release();
    g_keys.release(); g_acc.release();
  }
};

constexpr unsigned kReduceBlocks = 256;

__global__ void k_reset_run(RunCounters *ctr, GroupTable g, uint32_t g_cap, uint32_t key_cap) {
  unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  if (tid == 0) {
    RunCounters z;
    memset(&z, 0, sizeof(z));
    z.first_invalid_tile = ~0ull;
    z.first_type_tile = ~0ull;
    z.first_type_error = ~0ull;
    z.agg_min_bits = ~0ull;
    z.first_invalid = ~0ull;
    *ctr = z;
  }
  if (g.slots) {
    for (unsigned long long i = tid; i < g_cap; i += stride) g.slots[i] = 0;
    for (unsigned long long i = tid; i < key_cap; i += stride) group_acc_init(g.acc[i]);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Context.
// ---------------------------------------------------------------------------

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  uint8_t *h_chunk = nullptr;  // pinned staging
  uint8_t *d_chunk = nullptr;
  unsigned long long n_bytes = 0;
  RunBufs rb;
  RunCounters *h_ctr = nullptr;  // pinned mirror
  // pinned result mirrors
  std::vector<uint8_t> dummy;
  uint8_t *h_out = nullptr;
  size_t h_out_cap = 0;
  unsigned long long *h_row_off = nullptr;
  unsigned long long *h_line64 = nullptr;
  uint32_t *h_line32 = nullptr;
  size_t h_rows_cap = 0;
  warpjq_group *h_groups = nullptr;
  size_t h_groups_cap = 0;
  bool launched = false;
  uint32_t kernels = 0;
  // page-locked staging of a batch's tables (copied from here without a
  // host wait for the stream), and the event after its last copies
  uint8_t *h_btab = nullptr;
  size_t h_btab_cap = 0;
  cudaEvent_t btab_done = nullptr;
  cudaEvent_t scan_t0 = nullptr, scan_t1 = nullptr;  // around the scan kernel
  bool timed = false;  // the last run recorded scan_t0/scan_t1 (not a graph replay)
  unsigned long long last_first_invalid = ~0ull;
  unsigned long long last_first_type = ~0ull;
};

struct warpjq_ctx {
  int device = 0;
  int num_sms = 0;
  DevPlan plan;
  DevPlan *d_plan = nullptr;
  unsigned long long chunk_cap = 0;
  uint32_t tile_bytes = 6144;
  uint32_t halo_bytes = 2048;
  uint32_t group_keys0 = 1u << 16;  // distinct keys a fresh group table has room for
  unsigned grid = 0;        // CTAs per-CTA buffers are sized for (the largest variant's grid)
  unsigned grid_rows = 0, grid_agg = 0, grid_group = 0;  // persistent CTAs per variant
  size_t scan_smem = 0;
  std::vector<Slot> slots;
  // device-resident runs
  Slot dev;
  const uint8_t *dev_data = nullptr;
  unsigned long long dev_n = 0;
  cudaStream_t dev_stream = nullptr;
  std::vector<warpjq_group_ext> dev_groups;
  // batched runs (warpjq_batch_launch): host copies of the tables
  struct Batch {
    bool active = false;
    bool tables_on_device = false;  // enqueue without uploading the tables (graph capture)
    // a mixed batch: input i runs plans[in_plan[i]]; any_rows when one of
    // them prints rows (records then take the largest plan's stride)
    bool mixed = false, any_grouped = false, any_rows = false;
    uint32_t rec_stride = 0;
    std::vector<DevPlan> plans;
    std::vector<uint32_t> in_plan;
    // the inputs in plan order, their running tile counts (list_tile0, one
    // more entry than inputs), and plan k's share of those tiles
    // [plan_tile0[k], plan_tile0[k + 1])
    std::vector<uint32_t> list_inputs;
    std::vector<unsigned long long> list_tile0, plan_tile0;
    uint64_t epoch = 0;             // bumped whenever a plain batch replaces the device tables
    const uint8_t *d_data = nullptr;
    cudaStream_t stream = nullptr;
    unsigned long long n_tiles = 0, total = 0;
    std::vector<unsigned long long> start, end, tile0;
    std::vector<RunCounters> h_ctr;
    std::vector<warpjq_group_ext> groups;
    std::vector<uint32_t> group_input;
  } batch;
};

namespace {


warpjq_status configure_grid(warpjq_ctx *c, char *err, size_t err_len) {
  c->scan_smem = scan_smem_bytes(c->tile_bytes, c->halo_bytes,
                                 c->plan.output_kind == WARPJQ_OUT_AGG && c->plan.group_slot >= 0);
  int per_sm = 0;
  // The limit is a property of the kernel, shared by every context in the
  // process, so it is raised to the device maximum rather than to this
  // context's need (occupancy follows each launch's own request).
  int dev = 0, smem_max = 0;
  CK(cudaGetDevice(&dev), "device");
  CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "attribute");
  if (c->scan_smem > (size_t)smem_max) {
    set_err(err, err_len, "tiling needs %zu bytes of shared memory, over the %d available",
            c->scan_smem, smem_max);
    return WARPJQ_ERR_INVALID_ARG;
  }
  CK(cudaFuncSetAttribute(k_scan<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max),
     "cudaFuncSetAttribute(scan rows)");
  CK(cudaFuncSetAttribute(k_scan<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max),
     "cudaFuncSetAttribute(scan agg)");
  CK(cudaFuncSetAttribute(k_scan<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max),
     "cudaFuncSetAttribute(scan grouped)");
  // Each variant runs as many CTAs per SM as its own registers and shared
  // memory allow; buffers sized per CTA take the largest of them.
  int a = 0, b = 0, g = 0;
  const size_t grouped_smem = scan_smem_bytes(c->tile_bytes, c->halo_bytes, true);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_scan<true>, kThreads, c->scan_smem),
     "occupancy");
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_scan<false>, kThreads, c->scan_smem),
     "occupancy");
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g, k_scan<false, true>, kThreads, grouped_smem),
     "occupancy");
  c->grid_rows = (unsigned)(c->num_sms * std::max(1, a));
  c->grid_agg = (unsigned)(c->num_sms * std::max(1, b));
  c->grid_group = (unsigned)(c->num_sms * std::max(1, g));
  per_sm = std::max(std::max(a, b), g);
  c->grid = (unsigned)(c->num_sms * std::max(1, per_sm));
  return WARPJQ_OK;
}

// Sizes the buffers of `s` for an input of n bytes (first use, or growth).
warpjq_status ensure_bufs(warpjq_ctx *c, Slot &s, unsigned long long n,
                          unsigned long long n_tiles, cudaStream_t st, bool cap, char *err, size_t err_len,
                          bool grouped, bool rows, uint32_t rec_stride) {
  RunBufs &rb = s.rb;
  if (n_tiles == 0) n_tiles = 1;
  CK(rb.ctr.ensure(1, st, cap), "alloc counters");
  CK(rb.tiles.ensure(n_tiles, st, cap), "alloc tiles");
  CK(rb.block_lines.ensure(2 * kReduceBlocks, st, cap), "alloc reduce");
  if (!rb.deep_levels) rb.deep_levels = 1u << 16;
  CK(rb.deep.ensure((size_t)c->grid * (rb.deep_levels / 32), st, cap), "alloc deep stack");
  if (rows) {
    CK(rb.row_tiles.ensure(n_tiles, st, cap), "alloc row tiles");
    CK(rb.row_bsum.ensure(3 * ((n_tiles + 31) / 32), st, cap), "alloc row prefixes");
    // Records accumulate over all of a CTA's tiles: room for a row per KiB
    // of input, grown on overflow; output and row capacities follow the
    // input's size too (a larger input than the last does not overflow
    // for that reason alone).
    rb.rec_cap_per_cta = std::max(rb.rec_cap_per_cta, n / 1024 / std::max(1u, c->grid) + 1024);
    CK(rb.recs.ensure((size_t)c->grid * rb.rec_cap_per_cta * rec_stride, st, cap), "alloc records");
    rb.out_cap = std::max(rb.out_cap, n + n / 4 + (1u << 20));
    CK(rb.out.ensure(rb.out_cap, st, cap), "alloc output");
    rb.rows_cap = std::max(rb.rows_cap, n / 32 + 4096);
    CK(rb.row_off.ensure(rb.rows_cap + 1, st, cap), "alloc row offsets");
    CK(rb.line_idx.ensure(rb.rows_cap, st, cap), "alloc line index");
  }
  if (grouped) {
    if (!rb.g_cap) {
      rb.g_key_cap = c->group_keys0;
      rb.g_cap = 2 * c->group_keys0;
    }
    CK(rb.g_slots.ensure(rb.g_cap, st, cap), "alloc group table");
    CK(rb.g_keys.ensure(rb.g_key_cap, st, cap), "alloc group keys");
    CK(rb.g_acc.ensure(rb.g_key_cap, st, cap), "alloc group accumulators");
  }
  return WARPJQ_OK;
}

// Whether a run keeps a group table: the context's plan groups, or (a mixed
// batch) one of the inputs' plans does.
bool run_grouped(const warpjq_ctx *c, const warpjq_ctx::Batch *b) {
  if (b && b->mixed) return b->any_grouped;
  return c->plan.output_kind == WARPJQ_OUT_AGG && c->plan.group_slot >= 0;
}

// Whether a run prints rows (the context's plan does, or one of a mixed
// batch's plans does), and the bytes of its row records.
bool run_rows(const warpjq_ctx *c, const warpjq_ctx::Batch *b) {
  if (b && b->mixed) return b->any_rows;
  return c->plan.needs_rows != 0;
}
uint32_t run_rec_stride(const warpjq_ctx *c, const warpjq_ctx::Batch *b) {
  if (b && b->mixed) return b->rec_stride;
  return c->plan.rec_stride;
}

GroupTable group_view(RunBufs &rb, bool on) {
  GroupTable g{};
  if (!on) return g;
  g.slots = rb.g_slots.p;
  g.cap_mask = rb.g_cap - 1;
  g.key_cap = rb.g_key_cap;
  g.keys = rb.g_keys.p;
  g.acc = rb.g_acc.p;
  return g;
}

// Enqueues one run over n bytes at d_data on `st`.  No host synchronisation.
// With `b`, the run is a batch: n is the inputs' total size and the tiles
// come from the batch's tables.
warpjq_status enqueue_run(warpjq_ctx *c, Slot &s, const uint8_t *d_data, unsigned long long n,
                          cudaStream_t st, char *err, size_t err_len,
                          const warpjq_ctx::Batch *b = nullptr) {
  const unsigned long long n_tiles = b ? b->n_tiles : (n + c->tile_bytes - 1) / c->tile_bytes;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cap), "capture status");
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  const bool rows = run_rows(c, b);
  warpjq_status rc = ensure_bufs(c, s, n, n_tiles, st, capturing, err, err_len, run_grouped(c, b), rows,
                                 run_rec_stride(c, b));
  if (rc != WARPJQ_OK) return rc;
  RunBufs &rb = s.rb;
  const DevPlan &P = c->plan;
  const bool groups = run_grouped(c, b);
  const uint32_t n_inputs = b ? (uint32_t)b->start.size() : 0;
  if (b && !b->tables_on_device) {
    CK(rb.b_in_start.ensure(std::max<uint32_t>(n_inputs, 1), st, capturing), "alloc batch tables");
    CK(rb.b_in_end.ensure(std::max<uint32_t>(n_inputs, 1), st, capturing), "alloc batch tables");
    CK(rb.b_in_tile0.ensure(n_inputs + 1, st, capturing), "alloc batch tables");
    CK(rb.b_in_ctr.ensure(std::max<uint32_t>(n_inputs, 1), st, capturing), "alloc batch tables");
    CK(rb.b_tile_input.ensure(std::max<unsigned long long>(n_tiles, 1), st, capturing), "alloc batch tables");
    // The tables are packed into page-locked staging and copied from there:
    // a copy from pageable memory would make the host wait for the stream's
    // earlier work (the previous batches of a serving slot).
    // (Per-tile tables are built on the device from these, below.)
    const size_t n8 = n_inputs * 8ull, t8 = (n_inputs + 1) * 8ull, n4 = n_inputs * 4ull;
    const size_t p_pl = b->mixed ? b->plans.size() * sizeof(DevPlan) : 0, p_m4 = b->mixed ? n4 : 0,
                 p_m8 = b->mixed ? t8 : 0;
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t o_end = up16(n8), o_t0 = o_end + up16(n8), o_ip = o_t0 + up16(t8), o_pl = o_ip + up16(p_m4),
                 o_li = o_pl + up16(p_pl), o_lt = o_li + up16(p_m4), need = o_lt + p_m8;
    if (!s.btab_done) CK(cudaEventCreateWithFlags(&s.btab_done, cudaEventDisableTiming), "event");
    CK(cudaEventSynchronize(s.btab_done), "batch staging wait");  // the last batch's copies are done
    if (need > s.h_btab_cap) {
      if (s.h_btab) cudaFreeHost(s.h_btab);
      s.h_btab = nullptr;
      s.h_btab_cap = 0;
      const size_t cap = std::max<size_t>(need + need / 2, 1u << 16);
      CK(cudaMallocHost((void **)&s.h_btab, cap), "alloc batch staging");
      s.h_btab_cap = cap;
    }
    uint8_t *hb = s.h_btab;
    if (n8) {
      std::memcpy(hb, b->start.data(), n8);
      std::memcpy(hb + o_end, b->end.data(), n8);
    }
    std::memcpy(hb + o_t0, b->tile0.data(), t8);
    if (b->mixed) {
      CK(rb.b_plans.ensure(b->plans.size(), st, capturing), "alloc batch plans");
      CK(rb.b_in_plan.ensure(std::max<uint32_t>(n_inputs, 1), st, capturing), "alloc batch plans");
      CK(rb.b_list_inputs.ensure(std::max<uint32_t>(n_inputs, 1), st, capturing), "alloc batch plans");
      CK(rb.b_list_tile0.ensure(n_inputs + 1, st, capturing), "alloc batch plans");
      CK(rb.b_plan_tiles.ensure(std::max<unsigned long long>(n_tiles, 1), st, capturing), "alloc batch plans");
      std::memcpy(hb + o_pl, b->plans.data(), p_pl);
      if (n4) {
        std::memcpy(hb + o_ip, b->in_plan.data(), n4);
        std::memcpy(hb + o_li, b->list_inputs.data(), n4);
      }
      std::memcpy(hb + o_lt, b->list_tile0.data(), t8);
      CK(cudaMemcpyAsync(rb.b_plans.p, hb + o_pl, p_pl, cudaMemcpyHostToDevice, st), "H2D batch plans");
      if (n4) {
        CK(cudaMemcpyAsync(rb.b_in_plan.p, hb + o_ip, n4, cudaMemcpyHostToDevice, st), "H2D batch plans");
        CK(cudaMemcpyAsync(rb.b_list_inputs.p, hb + o_li, n4, cudaMemcpyHostToDevice, st), "H2D batch plans");
      }
      CK(cudaMemcpyAsync(rb.b_list_tile0.p, hb + o_lt, t8, cudaMemcpyHostToDevice, st), "H2D batch plans");
    }
    if (n8) {
      CK(cudaMemcpyAsync(rb.b_in_start.p, hb, n8, cudaMemcpyHostToDevice, st), "H2D batch tables");
      CK(cudaMemcpyAsync(rb.b_in_end.p, hb + o_end, n8, cudaMemcpyHostToDevice, st), "H2D batch tables");
    }
    CK(cudaMemcpyAsync(rb.b_in_tile0.p, hb + o_t0, t8, cudaMemcpyHostToDevice, st), "H2D batch tables");
    CK(cudaEventRecord(s.btab_done, st), "event record");
  }
  s.kernels = 0;
  if (b && n_inputs) {
    k_batch_reset<<<(n_inputs + 255) / 256, 256, 0, st>>>(rb.b_in_ctr.p, n_inputs);
    s.kernels++;
    if (n_tiles) {
      const unsigned nb = (unsigned)std::min<unsigned long long>((n_tiles + 255) / 256, 8ull * c->num_sms);
      k_batch_expand<<<nb, 256, 0, st>>>(n_tiles, n_inputs, rb.b_in_tile0.p, rb.b_tile_input.p,
                                         b->mixed ? rb.b_list_inputs.p : nullptr,
                                         b->mixed ? rb.b_list_tile0.p : nullptr,
                                         b->mixed ? rb.b_plan_tiles.p : nullptr);
      s.kernels++;
      CK(cudaGetLastError(), "launch batch tables");
    }
  }
  GroupTable g = group_view(rb, groups);
  k_reset_run<<<256, 256, 0, st>>>(rb.ctr.p, g, groups ? rb.g_cap : 0, groups ? rb.g_key_cap : 0);
  s.kernels++;
  CK(cudaGetLastError(), "launch reset");
  if (n > 0 && n_tiles > 0) {
    ScanParams sp{};
    sp.data = d_data;
    sp.n = n;
    sp.tile_bytes = c->tile_bytes;
    sp.halo_bytes = c->halo_bytes;
    sp.n_tiles = n_tiles;
    sp.ctr = rb.ctr.p;
    sp.tiles = rb.tiles.p;
    sp.row_tiles = rb.row_tiles.p;
    sp.rec_scratch = rb.recs.p;
    sp.rec_cap_per_cta = rb.rec_cap_per_cta;
    sp.g = g;
    sp.deep_words = rb.deep.p;
    sp.deep_levels_per_cta = rb.deep_levels;
    sp.rec_stride = run_rec_stride(c, b);
    if (b && b->mixed) {
      sp.any_rows = b->any_rows ? 1u : 0u;
      CK(rb.b_tickets.ensure(b->plans.size(), st, capturing), "alloc batch tickets");
      CK(rb.b_rec_cursor.ensure(c->grid, st, capturing), "alloc batch tickets");
      CK(cudaMemsetAsync(rb.b_tickets.p, 0, b->plans.size() * sizeof(unsigned long long), st), "reset tickets");
      if (b->any_rows)
        CK(cudaMemsetAsync(rb.b_rec_cursor.p, 0, c->grid * sizeof(unsigned long long), st), "reset tickets");
    }
    if (b) {
      sp.tile_input = rb.b_tile_input.p;
      sp.in_start = rb.b_in_start.p;
      sp.in_end = rb.b_in_end.p;
      sp.in_tile0 = rb.b_in_tile0.p;
      sp.in_ctr = rb.b_in_ctr.p;
    }
    if (!s.scan_t0 && !capturing) {
      CK(cudaEventCreate(&s.scan_t0), "event");
      CK(cudaEventCreate(&s.scan_t1), "event");
    }
    s.timed = !capturing;  // a captured sequence is not timed
    if (s.timed) CK(cudaEventRecord(s.scan_t0, st), "event record");
    if (b && b->mixed) {
      // One launch per distinct plan over its inputs' tiles, each the
      // variant specialised for that plan (the plan a kernel parameter, as
      // in a plain run).  The launches share the run's counters, per-tile
      // tables and group table; row launches append to the CTAs' record
      // arenas one after another.
      for (size_t k = 0; k < b->plans.size(); k++) {
        const unsigned long long n_k = b->plan_tile0[k + 1] - b->plan_tile0[k];
        if (!n_k) continue;
        const DevPlan &Pk = b->plans[k];
        const bool gk = Pk.output_kind == WARPJQ_OUT_AGG && Pk.group_slot >= 0;
        ScanParams spk = sp;
        spk.tile_list = rb.b_plan_tiles.p + b->plan_tile0[k];
        spk.n_list = n_k;
        spk.ticket = rb.b_tickets.p + k;
        spk.rec_cursor = Pk.needs_rows ? rb.b_rec_cursor.p : nullptr;
        const unsigned vg = Pk.needs_rows ? c->grid_rows : gk ? c->grid_group : c->grid_agg;
        const unsigned gr = (unsigned)std::min<unsigned long long>(vg, n_k);
        const size_t smem = scan_smem_bytes(c->tile_bytes, c->halo_bytes, gk);
        if (Pk.needs_rows)
          k_scan<true><<<gr, kThreads, smem, st>>>(spk, Pk);
        else if (gk)
          k_scan<false, true><<<gr, kThreads, smem, st>>>(spk, Pk);
        else
          k_scan<false><<<gr, kThreads, smem, st>>>(spk, Pk);
        s.kernels++;
        CK(cudaGetLastError(), "launch scan");
      }
    } else {
      const unsigned vgrid = P.needs_rows ? c->grid_rows : groups ? c->grid_group : c->grid_agg;
      const unsigned grid = (unsigned)std::min<unsigned long long>(vgrid, n_tiles);
      if (P.needs_rows)
        k_scan<true><<<grid, kThreads, c->scan_smem, st>>>(sp, c->plan);
      else if (groups)
        k_scan<false, true><<<grid, kThreads, c->scan_smem, st>>>(sp, c->plan);
      else
        k_scan<false><<<grid, kThreads, c->scan_smem, st>>>(sp, c->plan);
      s.kernels++;
      CK(cudaGetLastError(), "launch scan");
    }
    if (s.timed) CK(cudaEventRecord(s.scan_t1, st), "event record");
    if (rows) {
      const uint32_t tpb = rows_tiles_per_block(n_tiles);
      const unsigned nb = (unsigned)((n_tiles + tpb - 1) / tpb);
      k_rows_block_sums<<<nb, kEmitThreads, 0, st>>>(rb.row_tiles.p, rb.tiles.p, n_tiles, tpb,
                                                      rb.row_bsum.p);
      k_rows_block_prefix<<<1, kPrefixThreads, 0, st>>>(rb.row_bsum.p, nb, rb.ctr.p, rb.row_off.p,
                                                      rb.rows_cap, rb.out_cap);
      EmitParams ep{};
      ep.data = d_data;
      ep.plan = c->d_plan;
      ep.rec_stride = sp.rec_stride;
      if (b && b->mixed) {
        ep.plans = rb.b_plans.p;
        ep.in_plan = rb.b_in_plan.p;
        ep.tile_input = rb.b_tile_input.p;
      }
      ep.row_tiles = rb.row_tiles.p;
      ep.tiles = rb.tiles.p;
      ep.n_tiles = n_tiles;
      ep.block_prefix = rb.row_bsum.p;
      ep.tiles_per_block = tpb;
      ep.recs = rb.recs.p;
      ep.out = rb.out.p;
      ep.out_cap = rb.out_cap;
      ep.row_off = rb.row_off.p;
      ep.line_idx = rb.line_idx.p;
      ep.rows_cap = rb.rows_cap;
      ep.ctr = rb.ctr.p;
      k_rows_emit<<<nb, kEmitThreads, 0, st>>>(ep);
      s.kernels += 3;
      CK(cudaGetLastError(), "launch rows");
    }
    k_reduce_tiles<<<kReduceBlocks, kReduceThreads, 0, st>>>(n_tiles, rb.tiles.p, rb.ctr.p,
                                                             rb.block_lines.p);
    s.kernels++;
    CK(cudaGetLastError(), "launch reduce");
    k_finalize<<<1, 32, 0, st>>>(rb.block_lines.p, kReduceBlocks, rb.tiles.p, rb.ctr.p);
    s.kernels++;
    CK(cudaGetLastError(), "launch finalize");
    if (b && n_inputs) {
      k_batch_finalize<<<(n_inputs + 7) / 8, 256, 0, st>>>(rb.tiles.p, rb.b_in_tile0.p, rb.b_in_ctr.p,
                                                          n_inputs);
      s.kernels++;
      CK(cudaGetLastError(), "launch batch finalize");
    }
  }
  s.launched = true;
  return WARPJQ_OK;
}

// After a run finished: grows whatever overflowed.  Returns true if the run
// has to be repeated.
bool grow_after_overflow(warpjq_ctx *c, Slot &s, const RunCounters &h, unsigned long long n) {
  RunBufs &rb = s.rb;
  bool again = false;
  if (h.overflow & 1u) {  // records per CTA
    rb.rec_cap_per_cta *= 4;
    rb.recs.release();
    again = true;
  }
  if (h.overflow & 2u) {  // output bytes or row count; both totals are exact
    unsigned long long need_rows = h.n_selected + 1;
    if (need_rows > rb.rows_cap) {
      rb.rows_cap = need_rows + need_rows / 8;
      rb.row_off.release();
      rb.line_idx.release();
    }
    if (h.out_len > rb.out_cap) {
      rb.out_cap = h.out_len + h.out_len / 8 + 1;
      rb.out.release();
    }
    again = true;
  }
  if (h.overflow & 4u) {  // group table
    rb.g_key_cap = std::max<uint32_t>(rb.g_key_cap * 2, (uint32_t)std::min<unsigned long long>(h.n_keys * 2ull, 1u << 30));
    rb.g_cap = 1;
    while (rb.g_cap < rb.g_key_cap * 2u) rb.g_cap <<= 1;
    rb.g_key_cap = rb.g_cap / 2;
    rb.g_slots.release();
    rb.g_keys.release();
    rb.g_acc.release();
    again = true;
  }
  if (h.overflow & 8u) {  // deep nesting
    rb.deep_levels = std::min<unsigned long long>(rb.deep_levels * 16, ((n + 31) / 32) * 32 + 64);
    rb.deep.release();
    again = true;
  }
  return again;
}

// Runs synchronously until the result is complete; leaves counters in h.
warpjq_status run_to_completion(warpjq_ctx *c, Slot &s, const uint8_t *d_data,
                                unsigned long long n, cudaStream_t st, RunCounters &h,
                                bool already_enqueued, char *err, size_t err_len,
                                const warpjq_ctx::Batch *b = nullptr) {
  for (int attempt = 0; attempt < 16; attempt++) {
    if (!already_enqueued || attempt > 0) {
      warpjq_status rc = enqueue_run(c, s, d_data, n, st, err, err_len, b);
      if (rc != WARPJQ_OK) return rc;
    }
    CK(cudaMemcpyAsync(&h, s.rb.ctr.p, sizeof(RunCounters), cudaMemcpyDeviceToHost, st),
       "D2H counters");
    CK(cudaStreamSynchronize(st), "stream sync");
    if (h.error) {
      set_err(err, err_len, "the scan kernel raised its error flag");
      return WARPJQ_ERR_CUDA;
    }
    if (!h.overflow) return WARPJQ_OK;
    if (!grow_after_overflow(c, s, h, n)) return WARPJQ_OK;
  }
  set_err(err, err_len, "device buffers kept overflowing");
  return WARPJQ_ERR_OOM;
}

// Everything a captured batch bakes in from its context: buffer addresses
// and sizes, capacities, tiling and grid.  A graph replays only while this
// is unchanged (a grown or released buffer would leave it writing to freed
// memory).
uint64_t bufs_signature(const warpjq_ctx *c) {
  const RunBufs &rb = c->dev.rb;
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](uint64_t v) {
    h ^= v;
    h *= 0x100000001b3ull;
  };
  mix((uintptr_t)rb.ctr.p); mix(rb.ctr.n);
  mix((uintptr_t)rb.tiles.p); mix(rb.tiles.n);
  mix((uintptr_t)rb.row_tiles.p); mix(rb.row_tiles.n);
  mix((uintptr_t)rb.row_bsum.p); mix(rb.row_bsum.n);
  mix((uintptr_t)rb.b_tile_input.p); mix(rb.b_tile_input.n);
  mix((uintptr_t)rb.b_in_start.p); mix((uintptr_t)rb.b_in_end.p);
  mix((uintptr_t)rb.b_in_tile0.p); mix((uintptr_t)rb.b_in_ctr.p);
  mix((uintptr_t)rb.b_plans.p); mix((uintptr_t)rb.b_in_plan.p); mix((uintptr_t)rb.b_plan_tiles.p);
  mix((uintptr_t)rb.b_list_inputs.p); mix((uintptr_t)rb.b_list_tile0.p);
  mix(rb.b_plan_tiles.n); mix((uintptr_t)rb.b_tickets.p); mix(rb.b_tickets.n);
  mix((uintptr_t)rb.b_rec_cursor.p); mix(rb.b_rec_cursor.n);
  mix((uintptr_t)rb.recs.p); mix(rb.recs.n);
  mix((uintptr_t)rb.out.p); mix(rb.out.n);
  mix((uintptr_t)rb.row_off.p); mix((uintptr_t)rb.line_idx.p);
  mix((uintptr_t)rb.block_lines.p);
  mix((uintptr_t)rb.deep.p); mix(rb.deep.n);
  mix((uintptr_t)rb.g_slots.p); mix((uintptr_t)rb.g_keys.p); mix((uintptr_t)rb.g_acc.p);
  mix(rb.rec_cap_per_cta); mix(rb.out_cap); mix(rb.rows_cap); mix(rb.g_cap); mix(rb.g_key_cap);
  mix(rb.deep_levels); mix(c->tile_bytes); mix(c->halo_bytes); mix(c->grid); mix(c->scan_smem);
  return h;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

warpjq_status warpjq_probe(char *err, size_t err_len) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_err(err, err_len, "no CUDA device: %s", e == cudaSuccess ? "none found" : cudaGetErrorString(e));
    return WARPJQ_ERR_NO_DEVICE;
  }
  cudaDeviceProp p;
  e = cudaGetDeviceProperties(&p, 0);
  if (e != cudaSuccess) {
    set_err(err, err_len, "%s", cudaGetErrorString(e));
    return WARPJQ_ERR_NO_DEVICE;
  }
  if (p.major < 10) {
    set_err(err, err_len, "device 0 is sm_%d%d; this backend is built for sm_100a", p.major, p.minor);
    return WARPJQ_ERR_NO_DEVICE;
  }
  return WARPJQ_OK;
}

// Sizes of step, path, cmp, cond_op, agg_partial, group, in that order
// (reference warpjq_kernels.cu:2267-2277, gpu/ffi.rs:222-242).
warpjq_status warpjq_abi_check(const uint64_t *sizes, size_t n) {
  const uint64_t mine[6] = {sizeof(warpjq_step), sizeof(warpjq_path), sizeof(warpjq_cmp),
                            sizeof(warpjq_cond_op), sizeof(warpjq_agg_partial),
                            sizeof(warpjq_group)};
  if (!sizes || n != 6) return WARPJQ_ERR_ABI;
  for (int i = 0; i < 6; i++)
    if (sizes[i] != mine[i]) return WARPJQ_ERR_ABI;
  return WARPJQ_OK;
}

warpjq_status warpjq_device_name(char *buf, size_t len) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) return WARPJQ_ERR_NO_DEVICE;
  set_err(buf, len, "%s (sm_%d%d, %zu MiB)", p.name, p.major, p.minor,
          (size_t)(p.totalGlobalMem >> 20));
  return WARPJQ_OK;
}

warpjq_status warpjq_ctx_create(const warpjq_program *prog, uint64_t max_chunk_bytes,
                                uint32_t n_slots, warpjq_ctx **out, char *err, size_t err_len) {
  if (!out || n_slots == 0 || n_slots > 8 || max_chunk_bytes >= (1ull << 40)) {
    set_err(err, err_len, "invalid context arguments");
    return WARPJQ_ERR_INVALID_ARG;
  }
  *out = nullptr;
  warpjq_status rc = warpjq_probe(err, err_len);
  if (rc != WARPJQ_OK) return rc;
  std::unique_ptr<warpjq_ctx> c(new warpjq_ctx());
  rc = build_plan(prog, c->plan, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  CK(cudaGetDevice(&c->device), "cudaGetDevice");
  CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device), "attr");
  {
    // Run buffers grow from the device's default memory pool
    // (stream-ordered); keep up to 8 GiB of what they give back cached in
    // the pool instead of returning it to the driver at every
    // synchronisation.
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, c->device), "memory pool");
    uint64_t keep = 8ull << 30;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
  }
  CK(cudaMalloc((void **)&c->d_plan, sizeof(DevPlan)), "alloc plan");
  CK(cudaMemcpy(c->d_plan, &c->plan, sizeof(DevPlan), cudaMemcpyHostToDevice), "upload plan");
  rc = configure_grid(c.get(), err, err_len);
  if (rc != WARPJQ_OK) return rc;
  c->chunk_cap = max_chunk_bytes;
  c->slots.resize(n_slots);
  for (auto &s : c->slots) {
    CK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream");
    CK(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming), "event");
    CK(cudaHostAlloc((void **)&s.h_chunk, std::max<uint64_t>(max_chunk_bytes, 16), cudaHostAllocDefault),
       "pinned chunk");
    CK(cudaMalloc((void **)&s.d_chunk, max_chunk_bytes + 16), "device chunk");
    CK(cudaHostAlloc((void **)&s.h_ctr, sizeof(RunCounters), cudaHostAllocDefault), "pinned ctr");
    if (max_chunk_bytes) {
      rc = ensure_bufs(c.get(), s, max_chunk_bytes, (max_chunk_bytes + c->tile_bytes - 1) / c->tile_bytes,
                       s.stream, false, err, err_len, run_grouped(c.get(), nullptr), run_rows(c.get(), nullptr),
                       run_rec_stride(c.get(), nullptr));
      if (rc != WARPJQ_OK) return rc;
      CK(cudaStreamSynchronize(s.stream), "stream sync");
    }
  }
  CK(cudaHostAlloc((void **)&c->dev.h_ctr, sizeof(RunCounters), cudaHostAllocDefault), "pinned ctr");
  *out = c.release();
  return WARPJQ_OK;
}

static void free_slot(Slot &s) {
  s.rb.release();
  if (s.stream) cudaStreamDestroy(s.stream);
  if (s.done) cudaEventDestroy(s.done);
  if (s.h_chunk) cudaFreeHost(s.h_chunk);
  if (s.d_chunk) cudaFree(s.d_chunk);
  if (s.h_ctr) cudaFreeHost(s.h_ctr);
  if (s.h_out) cudaFreeHost(s.h_out);
  if (s.h_row_off) cudaFreeHost(s.h_row_off);
  if (s.h_line64) cudaFreeHost(s.h_line64);
  if (s.h_line32) cudaFreeHost(s.h_line32);
  if (s.h_groups) cudaFreeHost(s.h_groups);
  if (s.scan_t0) cudaEventDestroy(s.scan_t0);
  if (s.scan_t1) cudaEventDestroy(s.scan_t1);
  if (s.h_btab) cudaFreeHost(s.h_btab);
  if (s.btab_done) cudaEventDestroy(s.btab_done);
  s = Slot();
}

void warpjq_ctx_destroy(warpjq_ctx *ctx) {
  if (!ctx) return;
  cudaDeviceSynchronize();
  for (auto &s : ctx->slots) free_slot(s);
  free_slot(ctx->dev);
  if (ctx->d_plan) cudaFree(ctx->d_plan);
  delete ctx;
}

uint8_t *warpjq_slot_buffer(warpjq_ctx *ctx, uint32_t slot) {
  if (!ctx || slot >= ctx->slots.size()) return nullptr;
  return ctx->slots[slot].h_chunk;
}

uint64_t warpjq_slot_capacity(const warpjq_ctx *ctx) { return ctx ? ctx->chunk_cap : 0; }

// Every line of a chunk is decided on the device, however short, so the
// line budget is simply the byte capacity.
uint64_t warpjq_max_lines(const warpjq_ctx *ctx) { return ctx ? ctx->chunk_cap + 1 : 0; }

warpjq_status warpjq_submit(warpjq_ctx *ctx, uint32_t slot, uint64_t n_bytes, char *err,
                            size_t err_len) {
  if (!ctx || slot >= ctx->slots.size() || n_bytes > ctx->chunk_cap) {
    set_err(err, err_len, "submit: bad slot or %llu bytes over the slot capacity",
            (unsigned long long)n_bytes);
    return WARPJQ_ERR_INVALID_ARG;
  }
  Slot &s = ctx->slots[slot];
  s.n_bytes = n_bytes;
  if (n_bytes)
    CK(cudaMemcpyAsync(s.d_chunk, s.h_chunk, n_bytes, cudaMemcpyHostToDevice, s.stream), "H2D chunk");
  warpjq_status rc = enqueue_run(ctx, s, s.d_chunk, n_bytes, s.stream, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  CK(cudaEventRecord(s.done, s.stream), "event record");
  return WARPJQ_OK;
}

warpjq_status warpjq_submit_host(warpjq_ctx *ctx, uint32_t slot, const uint8_t *src,
                                 uint64_t n_bytes, char *err, size_t err_len) {
  if (!ctx || slot >= ctx->slots.size() || n_bytes > ctx->chunk_cap || (!src && n_bytes)) {
    set_err(err, err_len, "submit: bad slot or source, or %llu bytes over the slot capacity",
            (unsigned long long)n_bytes);
    return WARPJQ_ERR_INVALID_ARG;
  }
  Slot &s = ctx->slots[slot];
  s.n_bytes = n_bytes;
  if (n_bytes)
    CK(cudaMemcpyAsync(s.d_chunk, src, n_bytes, cudaMemcpyHostToDevice, s.stream), "H2D chunk");
  warpjq_status rc = enqueue_run(ctx, s, s.d_chunk, n_bytes, s.stream, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  CK(cudaEventRecord(s.done, s.stream), "event record");
  return WARPJQ_OK;
}

void *warpjq_host_alloc_pinned(uint64_t n_bytes) {
  void *p = nullptr;
  if (cudaHostAlloc(&p, n_bytes ? n_bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void warpjq_host_free_pinned(void *p) {
  if (p) cudaFreeHost(p);
}

int warpjq_host_is_pinned(const void *p) {
  if (!p) return 0;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the error state of the failed query
    return 0;
  }
  return a.type == cudaMemoryTypeHost ? 1 : 0;
}

static warpjq_status ensure_pinned(Slot &s, size_t out_bytes, size_t rows, size_t groups,
                                   char *err, size_t err_len) {
  if (out_bytes > s.h_out_cap || !s.h_out) {
    if (s.h_out) cudaFreeHost(s.h_out);
    s.h_out = nullptr;
    size_t cap = std::max<size_t>(out_bytes + out_bytes / 4, 1 << 16);
    CK(cudaHostAlloc((void **)&s.h_out, cap, cudaHostAllocDefault), "pinned rows");
    s.h_out_cap = cap;
  }
  if (rows + 1 > s.h_rows_cap || !s.h_row_off) {
    if (s.h_row_off) cudaFreeHost(s.h_row_off);
    if (s.h_line64) cudaFreeHost(s.h_line64);
    if (s.h_line32) cudaFreeHost(s.h_line32);
    size_t cap = std::max<size_t>(rows + rows / 4 + 1, 1024);
    CK(cudaHostAlloc((void **)&s.h_row_off, cap * 8, cudaHostAllocDefault), "pinned row offsets");
    CK(cudaHostAlloc((void **)&s.h_line64, cap * 8, cudaHostAllocDefault), "pinned line index");
    CK(cudaHostAlloc((void **)&s.h_line32, cap * 4, cudaHostAllocDefault), "pinned line index");
    s.h_rows_cap = cap;
  }
  if (groups > s.h_groups_cap || !s.h_groups) {
    if (s.h_groups) cudaFreeHost(s.h_groups);
    size_t cap = std::max<size_t>(groups + groups / 4, 256);
    CK(cudaHostAlloc((void **)&s.h_groups, cap * sizeof(warpjq_group), cudaHostAllocDefault),
       "pinned groups");
    s.h_groups_cap = cap;
  }
  return WARPJQ_OK;
}

// Copies the compacted group table of a finished run to the host.
static warpjq_status fetch_groups(warpjq_ctx *ctx, Slot &s, const RunCounters &h,
                                  std::vector<warpjq_group_ext> &out, char *err, size_t err_len,
                                  std::vector<uint32_t> *inputs = nullptr) {
  out.clear();
  if (inputs) inputs->clear();
  uint32_t nk = std::min<uint32_t>(h.n_keys, s.rb.g_key_cap);
  if (!nk) return WARPJQ_OK;
  std::vector<GroupKeyDesc> keys(nk);
  std::vector<GroupAcc> acc(nk);
  RunBufs &rb = s.rb;
  CK(cudaMemcpy(keys.data(), rb.g_keys.p, nk * sizeof(GroupKeyDesc), cudaMemcpyDeviceToHost),
     "D2H group keys");
  CK(cudaMemcpy(acc.data(), rb.g_acc.p, nk * sizeof(GroupAcc), cudaMemcpyDeviceToHost),
     "D2H group accumulators");
  for (uint32_t k = 0; k < nk; k++) {
    const GroupAcc &a = acc[k];
    if (a.count == 0) continue;  // an id allocated by a racing insert that lost
    warpjq_group_ext g{};
    g.key_off = keys[k].off;
    g.key_len = keys[k].len;
    g.key_kind = keys[k].kind;
    g.count = a.count;
    g.numeric = a.numeric;
    g.isum_lo = a.isum_lo;
    g.isum_hi = a.isum_hi;
    g.n_int = a.n_int;
    // exact sums, rounded once (fixsum.cuh)
    g.fsum = fix_to_double(a.fix, 0, 0) + a.fbig;
    g.min = a.numeric ? min_of_bits(a.min_bits) : __builtin_huge_val();
    g.max = a.numeric ? max_of_bits(a.max_bits) : -__builtin_huge_val();
    g.sum = fix_to_double(a.fix, a.isum_lo, a.isum_hi) + a.fbig;
    out.push_back(g);
    if (inputs) inputs->push_back(keys[k].input);
  }
  (void)ctx;
  return WARPJQ_OK;
}

warpjq_status warpjq_wait(warpjq_ctx *ctx, uint32_t slot, warpjq_chunk_result *out, char *err,
                          size_t err_len) {
  if (!ctx || slot >= ctx->slots.size() || !out) return WARPJQ_ERR_INVALID_ARG;
  Slot &s = ctx->slots[slot];
  std::memset(out, 0, sizeof(*out));
  out->first_invalid = 0xFFFFFFFFu;
  if (!s.launched) return WARPJQ_OK;
  RunCounters h;
  warpjq_status rc = run_to_completion(ctx, s, s.d_chunk, s.n_bytes, s.stream, h, true, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  const DevPlan &P = ctx->plan;
  out->n_lines = h.n_lines;
  out->n_blank = h.n_blank;
  out->n_invalid = h.n_invalid;
  out->n_type_error = h.n_type_error;
  out->n_selected = P.needs_rows ? h.n_selected : 0;
  out->first_invalid = h.first_invalid == ~0ull ? 0xFFFFFFFFu : (uint32_t)h.first_invalid;
  s.last_first_invalid = h.first_invalid;
  s.last_first_type = h.first_type_error;
  if (P.output_kind == WARPJQ_OUT_AGG) {
    out->n_selected = 0;
    if (P.group_slot < 0) {
      out->agg.count = h.agg_count;
      out->agg.numeric = h.agg_numeric;
      out->agg.sum = h.sum_total;
      out->agg.min = h.agg_numeric ? min_of_bits(h.agg_min_bits) : __builtin_huge_val();
      out->agg.max = h.agg_numeric ? max_of_bits(h.agg_max_bits) : -__builtin_huge_val();
      out->agg.saw_non_numeric = h.agg_saw_non_numeric;
    } else {
      std::vector<warpjq_group_ext> gs;
      rc = fetch_groups(ctx, s, h, gs, err, err_len);
      if (rc != WARPJQ_OK) return rc;
      rc = ensure_pinned(s, 0, 0, gs.size(), err, err_len);
      if (rc != WARPJQ_OK) return rc;
      for (size_t k = 0; k < gs.size(); k++) {
        warpjq_group &d = s.h_groups[k];
        d.key_off = (uint32_t)gs[k].key_off;
        d.key_len = gs[k].key_len;
        d.key_kind = gs[k].key_kind;
        d._pad = 0;
        d.count = gs[k].count;
        d.numeric = gs[k].numeric;
        d.sum = gs[k].sum;
        d.min = gs[k].min;
        d.max = gs[k].max;
      }
      out->groups = s.h_groups;
      out->n_groups = (uint32_t)gs.size();
    }
    return WARPJQ_OK;
  }
  size_t nsel = h.n_selected;
  rc = ensure_pinned(s, h.out_len, nsel, 0, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  if (nsel) {
    CK(cudaMemcpy(s.h_row_off, s.rb.row_off.p, (nsel + 1) * 8, cudaMemcpyDeviceToHost), "D2H row offsets");
    CK(cudaMemcpy(s.h_line64, s.rb.line_idx.p, nsel * 8, cudaMemcpyDeviceToHost), "D2H line index");
    if (h.out_len)
      CK(cudaMemcpy(s.h_out, s.rb.out.p, h.out_len, cudaMemcpyDeviceToHost), "D2H rows");
    for (size_t k = 0; k < nsel; k++) s.h_line32[k] = (uint32_t)s.h_line64[k];
  } else {
    s.h_row_off[0] = 0;
  }
  out->out_bytes = s.h_out;
  out->out_len = h.out_len;
  out->out_line_idx = s.h_line32;
  out->out_row_off = (const uint64_t *)s.h_row_off;
  return WARPJQ_OK;
}

// ---------------------------------------------------------------------------
// Device-resident extension
// ---------------------------------------------------------------------------

warpjq_status warpjq_slot_first_errors(warpjq_ctx *ctx, uint32_t slot, uint64_t *first_invalid,
                                       uint64_t *first_type_error) {
  if (!ctx || slot >= ctx->slots.size()) return WARPJQ_ERR_INVALID_ARG;
  if (first_invalid) *first_invalid = ctx->slots[slot].last_first_invalid;
  if (first_type_error) *first_type_error = ctx->slots[slot].last_first_type;
  return WARPJQ_OK;
}

warpjq_status warpjq_set_tiling(warpjq_ctx *ctx, uint32_t tile_bytes, uint32_t halo_bytes) {
  char *err = nullptr;
  size_t err_len = 0;
  if (!ctx) return WARPJQ_ERR_INVALID_ARG;
  uint32_t T = tile_bytes ? tile_bytes : ctx->tile_bytes;
  uint32_t H = halo_bytes ? halo_bytes : ctx->halo_bytes;
  if (T % 256 || T < 1024 || H % 256 || H < 512 || T + H > 65535 - 64) return WARPJQ_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize(), "sync");
  ctx->tile_bytes = T;
  ctx->halo_bytes = H;
  for (auto &s : ctx->slots) s.rb.release();
  ctx->dev.rb.release();
  return configure_grid(ctx, err, err_len);
}

warpjq_status warpjq_set_group_capacity(warpjq_ctx *ctx, uint32_t keys) {
  char *err = nullptr;
  size_t err_len = 0;
  if (!ctx || keys < 1024 || keys > (1u << 28) || (keys & (keys - 1))) return WARPJQ_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize(), "sync");
  ctx->group_keys0 = keys;
  auto drop = [](RunBufs &rb) {
    rb.g_slots.release();
    rb.g_keys.release();
    rb.g_acc.release();
    rb.g_cap = rb.g_key_cap = 0;
  };
  for (auto &s : ctx->slots) drop(s.rb);
  drop(ctx->dev.rb);
  return WARPJQ_OK;
}

warpjq_status warpjq_autotile(warpjq_ctx *ctx, const uint8_t *sample, uint64_t len,
                              uint32_t *tile_bytes, uint32_t *halo_bytes) {
  if (!ctx || (!sample && len)) return WARPJQ_ERR_INVALID_ARG;
  // Line-length statistics of the complete lines in the sample.
  uint64_t lines = 0, longest = 0;
  double sum = 0.0, sum2 = 0.0;
  const uint8_t *p = sample, *end = sample + len;
  const uint8_t *nl;
  while (p < end && (nl = (const uint8_t *)memchr(p, '\n', (size_t)(end - p))) != nullptr) {
    double l = (double)(nl - p) + 1.0;
    sum += l;
    sum2 += l * l;
    longest = std::max<uint64_t>(longest, (uint64_t)(nl - p) + 1);
    lines++;
    p = nl + 1;
  }
  uint32_t T = ctx->tile_bytes, H = ctx->halo_bytes;
  if (lines >= 16) {
    const double mean = sum / (double)lines;
    const double var = std::max(0.0, sum2 / (double)lines - mean * mean);
    const double cv = std::sqrt(var) / mean;
    // A tile's lines are walked in rounds of 32; each tile also costs about
    // as much as a few lines in staging and bookkeeping.  Score = lines per
    // walked lane slot, with the line count taken two deviations high.
    double best = -1.0;
    uint32_t best_T = T;
    for (uint32_t t = 1024; t <= 8192; t += 256) {
      double L = (double)t / mean;
      double hi = L + 2.0 * std::sqrt(L) * cv;
      double rounds = std::ceil(hi / 32.0);
      double score = L / (32.0 * rounds + 4.0);
      if (score >= best - 1e-9) {
        best = score;
        best_T = t;
      }
    }
    T = best_T;
    uint64_t h = (longest * 3 / 2 + 255) & ~255ull;
    H = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(h, 512), 16384);
    if (T + H > 65535 - 64) H = ((65535 - 64 - T) & ~255u);
  }
  if (tile_bytes) *tile_bytes = T;
  if (halo_bytes) *halo_bytes = H;
  if (T == ctx->tile_bytes && H == ctx->halo_bytes) return WARPJQ_OK;
  return warpjq_set_tiling(ctx, T, H);
}

warpjq_status warpjq_launch_device(warpjq_ctx *ctx, const uint8_t *d_data, uint64_t n_bytes,
                                   void *stream, char *err, size_t err_len) {
  if (!ctx || (!d_data && n_bytes)) return WARPJQ_ERR_INVALID_ARG;
  if (((uintptr_t)d_data & 15u) != 0) {
    set_err(err, err_len, "device input must be 16-byte aligned");
    return WARPJQ_ERR_INVALID_ARG;
  }
  ctx->dev_data = d_data;
  ctx->dev_n = n_bytes;
  ctx->dev_stream = (cudaStream_t)stream;
  return enqueue_run(ctx, ctx->dev, d_data, n_bytes, (cudaStream_t)stream, err, err_len);
}

warpjq_status warpjq_collect_device(warpjq_ctx *ctx, warpjq_device_result *out, char *err,
                                    size_t err_len) {
  if (!ctx || !out) return WARPJQ_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  Slot &s = ctx->dev;
  if (!s.launched) return WARPJQ_ERR_INVALID_ARG;
  RunCounters h;
  warpjq_status rc =
      run_to_completion(ctx, s, ctx->dev_data, ctx->dev_n, ctx->dev_stream, h, true, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  const DevPlan &P = ctx->plan;
  out->n_lines = h.n_lines;
  out->n_blank = h.n_blank;
  out->n_invalid = h.n_invalid;
  out->n_type_error = h.n_type_error;
  out->n_selected = h.n_selected;
  out->first_invalid = h.first_invalid;
  out->first_type_error = h.first_type_error;
  if (P.needs_rows) {
    out->d_out_bytes = s.rb.out.p;
    out->out_len = h.out_len;
    out->d_out_line_idx = (const uint64_t *)s.rb.line_idx.p;
    out->d_out_row_off = (const uint64_t *)s.rb.row_off.p;
  }
  out->count = h.agg_count;
  out->numeric = h.agg_numeric;
  out->isum_lo = h.agg_isum_lo;
  out->isum_hi = h.agg_isum_hi;
  out->n_int = h.agg_n_int;
  out->fsum = h.fsum_total;
  out->min = h.agg_numeric ? min_of_bits(h.agg_min_bits) : __builtin_huge_val();
  out->max = h.agg_numeric ? max_of_bits(h.agg_max_bits) : -__builtin_huge_val();
  out->sum = h.sum_total;
  out->saw_non_numeric = h.agg_saw_non_numeric;
  if (P.output_kind == WARPJQ_OUT_AGG && P.group_slot >= 0) {
    rc = fetch_groups(ctx, s, h, ctx->dev_groups, err, err_len);
    if (rc != WARPJQ_OK) return rc;
    out->groups = ctx->dev_groups.data();
    out->n_groups = (uint32_t)ctx->dev_groups.size();
  }
  out->kernels_launched = s.kernels;
  out->scan_ms = 0.0;
  if (s.scan_t0 && s.timed && ctx->dev_n) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s.scan_t0, s.scan_t1) == cudaSuccess) out->scan_ms = ms;
  }
  return WARPJQ_OK;
}

// The batch tables of warpjq_batch_launch(_mixed); the batch is left
// inactive until enqueued.
static warpjq_status batch_prepare(warpjq_ctx *ctx, const uint8_t *d_data, const uint64_t *offsets,
                                   const uint64_t *lengths, uint32_t n_inputs, void *stream, char *err,
                                   size_t err_len) {
  // d_data may be null: offsets are then device addresses, and the inputs
  // may lie in different allocations.
  if (!ctx || (n_inputs && (!offsets || !lengths))) return WARPJQ_ERR_INVALID_ARG;
  warpjq_ctx::Batch &b = ctx->batch;
  b.active = false;
  b.epoch++;
  b.d_data = d_data;
  b.stream = (cudaStream_t)stream;
  b.start.resize(n_inputs);
  b.end.resize(n_inputs);
  b.tile0.resize(n_inputs + 1);
  b.total = 0;
  const unsigned long long T = ctx->tile_bytes;
  unsigned long long tiles = 0;
  for (uint32_t i = 0; i < n_inputs; i++) {
    if (((uintptr_t)(d_data + offsets[i]) & 15u) != 0) {
      set_err(err, err_len, "batch input %u does not start on a 16-byte boundary", i);
      return WARPJQ_ERR_INVALID_ARG;
    }
    b.start[i] = offsets[i];
    b.end[i] = offsets[i] + lengths[i];
    b.tile0[i] = tiles;
    tiles += (lengths[i] + T - 1) / T;
    b.total += lengths[i];
  }
  b.tile0[n_inputs] = tiles;
  b.n_tiles = tiles;
  b.mixed = b.any_grouped = b.any_rows = false;
  b.rec_stride = 0;
  b.plans.clear();
  b.in_plan.clear();
  return WARPJQ_OK;
}

warpjq_status warpjq_batch_launch(warpjq_ctx *ctx, const uint8_t *d_data, const uint64_t *offsets,
                                  const uint64_t *lengths, uint32_t n_inputs, void *stream,
                                  char *err, size_t err_len) {
  warpjq_status rc = batch_prepare(ctx, d_data, offsets, lengths, n_inputs, stream, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  warpjq_ctx::Batch &b = ctx->batch;
  rc = enqueue_run(ctx, ctx->dev, d_data, b.total, b.stream, err, err_len, &b);
  if (rc == WARPJQ_OK) b.active = true;
  return rc;
}

warpjq_status warpjq_batch_launch_mixed(warpjq_ctx *ctx, warpjq_ctx *const *input_ctx, const uint8_t *d_data,
                                        const uint64_t *offsets, const uint64_t *lengths, uint32_t n_inputs,
                                        void *stream, char *err, size_t err_len) {
  if (!ctx || (n_inputs && !input_ctx)) return WARPJQ_ERR_INVALID_ARG;
  std::vector<const warpjq_ctx *> distinct;
  std::vector<uint32_t> in_plan(n_inputs);
  for (uint32_t i = 0; i < n_inputs; i++) {
    const warpjq_ctx *q = input_ctx[i];
    if (!q) {
      set_err(err, err_len, "input %u of a mixed batch has no query context", i);
      return WARPJQ_ERR_INVALID_ARG;
    }
    uint32_t k = 0;
    while (k < distinct.size() && distinct[k] != q) k++;
    if (k == distinct.size()) distinct.push_back(q);
    in_plan[i] = k;
  }
  warpjq_status rc = batch_prepare(ctx, d_data, offsets, lengths, n_inputs, stream, err, err_len);
  if (rc != WARPJQ_OK) return rc;
  warpjq_ctx::Batch &b = ctx->batch;
  b.mixed = true;
  b.rec_stride = kRowRecBytes;
  for (const warpjq_ctx *q : distinct) {
    b.plans.push_back(q->plan);
    b.any_grouped = b.any_grouped || (q->plan.output_kind == WARPJQ_OUT_AGG && q->plan.group_slot >= 0);
    b.any_rows = b.any_rows || q->plan.needs_rows;
    b.rec_stride = std::max(b.rec_stride, q->plan.rec_stride);
  }
  if (b.plans.empty()) b.plans.push_back(ctx->plan);
  b.in_plan = std::move(in_plan);
  // The inputs plan by plan (in input order within a plan) and their
  // running tile counts; the device lists each plan's tiles from these.
  const size_t n_plans = b.plans.size();
  std::vector<uint32_t> first(n_plans + 1, 0);
  for (uint32_t i = 0; i < n_inputs; i++) first[b.in_plan[i] + 1]++;
  for (size_t k = 0; k < n_plans; k++) first[k + 1] += first[k];
  b.list_inputs.resize(n_inputs);
  for (uint32_t i = 0; i < n_inputs; i++) b.list_inputs[first[b.in_plan[i]]++] = i;
  b.list_tile0.resize(n_inputs + 1);
  b.plan_tile0.assign(n_plans + 1, 0);
  unsigned long long run = 0;
  for (uint32_t j = 0; j < n_inputs; j++) {
    const uint32_t i = b.list_inputs[j];
    b.list_tile0[j] = run;
    run += b.tile0[i + 1] - b.tile0[i];
    b.plan_tile0[b.in_plan[i] + 1] = run;
  }
  b.list_tile0[n_inputs] = run;
  for (size_t k = 0; k < n_plans; k++) b.plan_tile0[k + 1] = std::max(b.plan_tile0[k + 1], b.plan_tile0[k]);
  rc = enqueue_run(ctx, ctx->dev, d_data, b.total, b.stream, err, err_len, &b);
  if (rc == WARPJQ_OK) b.active = true;
  return rc;
}

warpjq_status warpjq_batch_collect(warpjq_ctx *ctx, warpjq_batch_item *items,
                                   warpjq_device_result *all, char *err, size_t err_len) {
  if (!ctx || !ctx->batch.active) return WARPJQ_ERR_INVALID_ARG;
  warpjq_ctx::Batch &b = ctx->batch;
  Slot &s = ctx->dev;
  RunCounters h;
  warpjq_status rc =
      run_to_completion(ctx, s, b.d_data, b.total, b.stream, h, true, err, err_len, &b);
  if (rc != WARPJQ_OK) return rc;
  const uint32_t n = (uint32_t)b.start.size();
  b.h_ctr.resize(std::max<uint32_t>(n, 1));
  if (n)
    CK(cudaMemcpy(b.h_ctr.data(), s.rb.b_in_ctr.p, n * sizeof(RunCounters), cudaMemcpyDeviceToHost),
       "D2H batch counters");
  const DevPlan &P = ctx->plan;
  const bool grouped = run_grouped(ctx, &b);
  // Groups ordered by input (stable within an input).
  std::vector<uint32_t> first(n + 1, 0);
  if (grouped) {
    std::vector<warpjq_group_ext> gs;
    std::vector<uint32_t> gin;
    rc = fetch_groups(ctx, s, h, gs, err, err_len, &gin);
    if (rc != WARPJQ_OK) return rc;
    for (uint32_t in : gin) first[in + 1]++;
    for (uint32_t i = 0; i < n; i++) first[i + 1] += first[i];
    b.groups.assign(gs.size(), warpjq_group_ext{});
    std::vector<uint32_t> fill(first.begin(), first.end() - 1);
    for (size_t k = 0; k < gs.size(); k++) b.groups[fill[gin[k]]++] = gs[k];
  } else {
    b.groups.clear();
  }
  unsigned long long rows = 0, lines = 0;
  for (uint32_t i = 0; i < n && items; i++) {
    const RunCounters &c = b.h_ctr[i];
    warpjq_batch_item &it = items[i];
    std::memset(&it, 0, sizeof(it));
    it.n_lines = c.n_lines;
    it.n_blank = c.n_blank;
    it.n_invalid = c.n_invalid;
    it.n_type_error = c.n_type_error;
    const DevPlan &Pi = b.mixed ? b.plans[b.in_plan[i]] : P;
    it.n_selected = Pi.output_kind == WARPJQ_OUT_AGG ? 0 : c.n_selected;
    it.first_invalid = c.first_invalid;
    it.first_type_error = c.first_type_error;
    it.row_begin = rows;
    it.line_begin = lines;
    rows += it.n_selected;
    lines += c.n_lines;
    it.count = c.agg_count;
    it.numeric = c.agg_numeric;
    it.isum_lo = c.agg_isum_lo;
    it.isum_hi = c.agg_isum_hi;
    it.n_int = c.agg_n_int;
    it.fsum = c.fsum_total;
    it.min = c.agg_numeric ? min_of_bits(c.agg_min_bits) : __builtin_huge_val();
    it.max = c.agg_numeric ? max_of_bits(c.agg_max_bits) : -__builtin_huge_val();
    it.sum = c.sum_total;
    it.saw_non_numeric = c.agg_saw_non_numeric;
    it.group_begin = first[i];
    it.n_groups = first[i + 1] - first[i];
  }
  if (all) {
    std::memset(all, 0, sizeof(*all));
    all->n_lines = h.n_lines;
    all->n_blank = h.n_blank;
    all->n_invalid = h.n_invalid;
    all->n_type_error = h.n_type_error;
    // rows of the batch: every selected line, except a mixed batch's
    // aggregate inputs' (their selected lines print no row)
    unsigned long long n_rows = h.n_selected;
    if (b.mixed) {
      n_rows = 0;
      for (uint32_t i = 0; i < n; i++)
        if (b.plans[b.in_plan[i]].output_kind != WARPJQ_OUT_AGG) n_rows += b.h_ctr[i].n_selected;
    }
    all->n_selected = n_rows;
    all->first_invalid = ~0ull;
    all->first_type_error = ~0ull;
    if (run_rows(ctx, &b)) {
      all->d_out_bytes = s.rb.out.p;
      all->out_len = h.out_len;
      all->d_out_line_idx = (const uint64_t *)s.rb.line_idx.p;
      all->d_out_row_off = (const uint64_t *)s.rb.row_off.p;
    }
    all->groups = b.groups.data();
    all->n_groups = (uint32_t)b.groups.size();
    all->kernels_launched = s.kernels;
    if (s.scan_t0 && s.timed && b.total) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, s.scan_t0, s.scan_t1) == cudaSuccess) all->scan_ms = ms;
    }
  }
  return WARPJQ_OK;
}

struct warpjq_batch_graph {
  std::vector<warpjq_ctx *> ctxs;
  std::vector<uint64_t> epochs, sigs;
  std::vector<uint32_t> kernels;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

void warpjq_batch_graph_destroy(warpjq_batch_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

warpjq_status warpjq_batch_graph_create(warpjq_ctx *const *ctxs, uint32_t n_ctx, const uint8_t *const *d_data,
                                        const uint64_t *const *offsets, const uint64_t *const *lengths,
                                        const uint32_t *n_inputs, warpjq_batch_graph **out, char *err,
                                        size_t err_len) {
  if (!out || !ctxs || !n_ctx || !d_data || !offsets || !lengths || !n_inputs) return WARPJQ_ERR_INVALID_ARG;
  *out = nullptr;
  for (uint32_t i = 0; i < n_ctx; i++)
    for (uint32_t j = 0; j < i; j++)
      if (!ctxs[i] || ctxs[i] == ctxs[j]) {
        set_err(err, err_len, "each batch of a graph needs its own context");
        return WARPJQ_ERR_INVALID_ARG;
      }
  // 1. A plain run of every batch: sizes every buffer for this layout (and
  //    its contents) and leaves the batch tables on the device.
  for (uint32_t i = 0; i < n_ctx; i++) {
    warpjq_status rc = warpjq_batch_launch(ctxs[i], d_data[i], offsets[i], lengths[i], n_inputs[i], nullptr,
                                           err, err_len);
    if (rc != WARPJQ_OK) return rc;
    std::vector<warpjq_batch_item> items(std::max<uint32_t>(n_inputs[i], 1));
    rc = warpjq_batch_collect(ctxs[i], items.data(), nullptr, err, err_len);
    if (rc != WARPJQ_OK) return rc;
  }
  // 2. Capture every batch's launch sequence on its own stream, forked from
  //    and joined back to one capture stream.
  auto *g = new warpjq_batch_graph();
  cudaStream_t s0 = nullptr;
  std::vector<cudaStream_t> ss(n_ctx, nullptr);
  std::vector<cudaEvent_t> joins(n_ctx, nullptr);
  cudaEvent_t fork = nullptr;
  warpjq_status rc = WARPJQ_OK;
  auto fail = [&](cudaError_t e, const char *what) {
    set_err(err, err_len, "%s: %s", what, cudaGetErrorString(e));
    rc = WARPJQ_ERR_CUDA;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking);
  if (e != cudaSuccess) fail(e, "capture stream");
  if (rc == WARPJQ_OK && (e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming)) != cudaSuccess)
    fail(e, "capture event");
  for (uint32_t i = 0; rc == WARPJQ_OK && i < n_ctx; i++) {
    if ((e = cudaStreamCreateWithFlags(&ss[i], cudaStreamNonBlocking)) != cudaSuccess) fail(e, "capture stream");
    else if ((e = cudaEventCreateWithFlags(&joins[i], cudaEventDisableTiming)) != cudaSuccess) fail(e, "capture event");
  }
  bool began = false;
  if (rc == WARPJQ_OK) {
    if ((e = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) fail(e, "begin capture");
    else began = true;
  }
  if (rc == WARPJQ_OK && (e = cudaEventRecord(fork, s0)) != cudaSuccess) fail(e, "capture fork");
  for (uint32_t i = 0; rc == WARPJQ_OK && i < n_ctx; i++) {
    warpjq_ctx *c = ctxs[i];
    if ((e = cudaStreamWaitEvent(ss[i], fork, 0)) != cudaSuccess) {
      fail(e, "capture fork");
      break;
    }
    c->batch.tables_on_device = true;
    rc = enqueue_run(c, c->dev, c->batch.d_data, c->batch.total, ss[i], err, err_len, &c->batch);
    c->batch.tables_on_device = false;
    g->kernels.push_back(c->dev.kernels);
    if (rc != WARPJQ_OK) break;
    if ((e = cudaEventRecord(joins[i], ss[i])) != cudaSuccess) fail(e, "capture join");
    else if ((e = cudaStreamWaitEvent(s0, joins[i], 0)) != cudaSuccess) fail(e, "capture join");
  }
  if (began) {
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(s0, &graph);
    if (rc == WARPJQ_OK && e != cudaSuccess) fail(e, "end capture");
    if (rc == WARPJQ_OK) {
      g->graph = graph;
      if ((e = cudaGraphInstantiate(&g->exec, graph, 0)) != cudaSuccess) fail(e, "graph instantiate");
    } else if (graph) {
      cudaGraphDestroy(graph);
    }
  }
  for (uint32_t i = 0; i < n_ctx; i++) {
    if (ss[i]) cudaStreamDestroy(ss[i]);
    if (joins[i]) cudaEventDestroy(joins[i]);
  }
  if (fork) cudaEventDestroy(fork);
  if (s0) cudaStreamDestroy(s0);
  if (rc != WARPJQ_OK) {
    cudaGetLastError();
    warpjq_batch_graph_destroy(g);
    return rc;
  }
  for (uint32_t i = 0; i < n_ctx; i++) {
    g->ctxs.push_back(ctxs[i]);
    g->epochs.push_back(ctxs[i]->batch.epoch);
    g->sigs.push_back(bufs_signature(ctxs[i]));
  }
  *out = g;
  return WARPJQ_OK;
}

warpjq_status warpjq_batch_graph_launch(warpjq_batch_graph *g, void *stream, char *err, size_t err_len) {
  if (!g || !g->exec) return WARPJQ_ERR_INVALID_ARG;
  for (size_t i = 0; i < g->ctxs.size(); i++) {
    warpjq_ctx *c = g->ctxs[i];
    if (c->batch.epoch != g->epochs[i] || bufs_signature(c) != g->sigs[i]) {
      set_err(err, err_len,
              "batch %zu's context ran another batch or grew its buffers since the capture; create the graph again",
              i);
      return WARPJQ_ERR_INVALID_ARG;
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaGraphLaunch(g->exec, st), "graph launch");
  for (size_t i = 0; i < g->ctxs.size(); i++) {
    warpjq_ctx *c = g->ctxs[i];
    c->batch.active = true;
    c->batch.stream = st;
    c->dev.launched = true;
    c->dev.timed = false;
    c->dev.kernels = g->kernels[i];
  }
  return WARPJQ_OK;
}

}  // extern "C"
