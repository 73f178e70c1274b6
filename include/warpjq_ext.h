/* warpjq device backend -- extension entry points.
 *
 * These sit beside the drop-in ABI of warpjq_kernels.h and leave its structs
 * untouched.  They have no counterpart in the reference project: they serve
 * callers whose input is already resident in device memory (the
 * device-resident scan the benchmark measures), and they report aggregates
 * with exact 128-bit integer sums, which the reference's f64-only
 * warpjq_agg_partial cannot carry.
 *
 * Usage: warpjq_launch_device() enqueues the whole scan on a CUDA stream and
 * returns without synchronising; warpjq_collect_device() waits for it and
 * fills a warpjq_device_result.  Device buffers named in the result belong to
 * the context and stay valid until the next launch on it.
 */
#ifndef WARPJQ_EXT_H
#define WARPJQ_EXT_H

#include "warpjq_kernels.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One group of a device-resident run. */
typedef struct {
  uint64_t key_off;   /* byte offset of the key in the input (string: body) */
  uint32_t key_len;
  uint32_t key_kind;  /* JSON kind code 0..6 */
  uint64_t count;     /* lines that reached the aggregate */
  uint64_t numeric;   /* lines that contributed a number */
  uint64_t isum_lo;   /* exact sum of integer-literal values, two's complement */
  uint64_t isum_hi;
  uint64_t n_int;     /* how many values went into the exact sum */
  double fsum;        /* exact sum of the other numbers, rounded once to FP64 (independent of
                         tiling and of the order work runs in) */
  double min;
  double max;
  double sum;         /* isum + fsum rounded once to FP64 */
} warpjq_group_ext;

/* Aggregate and counters of a device-resident run. */
typedef struct {
  uint64_t n_lines;
  uint64_t n_blank;
  uint64_t n_invalid;
  uint64_t n_type_error;
  uint64_t n_selected;
  uint64_t first_invalid;    /* lowest invalid line index, or UINT64_MAX */
  uint64_t first_type_error; /* lowest line index with a type error, or UINT64_MAX */

  /* Rows (non-aggregate queries) stay in device memory. */
  const uint8_t *d_out_bytes;
  uint64_t out_len;
  const uint64_t *d_out_line_idx; /* n_selected entries */
  const uint64_t *d_out_row_off;  /* n_selected + 1 entries */

  /* Ungrouped aggregate. */
  uint64_t count;
  uint64_t numeric;
  uint64_t isum_lo;
  uint64_t isum_hi;
  uint64_t n_int;
  double fsum;
  double min;
  double max;
  double sum; /* isum + fsum rounded once */
  uint32_t saw_non_numeric;

  /* Grouped aggregate: host copy, valid until the next launch. */
  const warpjq_group_ext *groups;
  uint32_t n_groups;

  /* Device kernels launched by the last run (for launch accounting), and
   * the duration of its scan kernel, from CUDA events recorded around it on
   * the launch stream (the final attempt's, if the run was repeated). */
  uint32_t kernels_launched;
  double scan_ms;
} warpjq_device_result;

/* Enqueues the context's query over `n_bytes` of input at device address
 * `d_data` on `stream` (a cudaStream_t, or NULL for the default stream).
 * The input must stay unchanged until warpjq_collect_device returns.  Any
 * scratch that must grow is allocated here, synchronously, before enqueueing;
 * a later launch of the same or smaller size allocates nothing. */
warpjq_status warpjq_launch_device(warpjq_ctx *ctx, const uint8_t *d_data, uint64_t n_bytes,
                                   void *stream, char *err, size_t err_len);

/* Waits for the last launch and fills `out`.  If a device buffer proved too
 * small (an unusually selective projection, a very high group cardinality),
 * the buffers are grown and the run is repeated before returning, so the
 * result is always complete. */
warpjq_status warpjq_collect_device(warpjq_ctx *ctx, warpjq_device_result *out, char *err,
                                    size_t err_len);

/* Lowest line index (within the chunk last waited on) that was malformed,
 * and that hit a type error; UINT64_MAX for none.  warpjq_chunk_result
 * carries only the first; the second lets a host stop at the first bad
 * line of either kind, as --strict does on the CPU (exec/cpu.rs:394-407). */
warpjq_status warpjq_slot_first_errors(warpjq_ctx *ctx, uint32_t slot, uint64_t *first_invalid,
                                       uint64_t *first_type_error);

/* warpjq_submit with the chunk copied to the device straight from `src`
 * (n_bytes <= the slot capacity) instead of from the slot's pinned buffer.
 * For host memory that is already page-locked (cudaHostAlloc'd or
 * registered), this skips the staging copy; `src` must stay valid and
 * unmodified until warpjq_wait on this slot returns.  Errors as
 * warpjq_submit.  No reference counterpart. */
warpjq_status warpjq_submit_host(warpjq_ctx *ctx, uint32_t slot, const uint8_t *src,
                                 uint64_t n_bytes, char *err, size_t err_len);

/* 1 when `p` points into page-locked host memory the device can read by DMA,
 * else 0.  No reference counterpart. */
int warpjq_host_is_pinned(const void *p);

/* Page-locked host memory for input buffers (null on failure), and its
 * release (waits for the device).  No reference counterpart. */
void *warpjq_host_alloc_pinned(uint64_t n_bytes);
void warpjq_host_free_pinned(void *p);

/* One input's result within a batch (warpjq_batch_collect).  Line indexes
 * are relative to the input. */
typedef struct {
  uint64_t n_lines;
  uint64_t n_blank;
  uint64_t n_invalid;
  uint64_t n_type_error;
  uint64_t n_selected;
  uint64_t first_invalid;    /* lowest invalid line of the input, or UINT64_MAX */
  uint64_t first_type_error; /* lowest line with a type error, or UINT64_MAX */
  uint64_t row_begin;  /* the input's rows are rows [row_begin, row_begin + n_selected) of
                        * the batch's rows (see warpjq_batch_collect's `all`) */
  uint64_t line_begin; /* lines of the earlier inputs: subtract from the batch's line
                        * indexes to get the input's own */
  /* aggregate, as in warpjq_device_result */
  uint64_t count;
  uint64_t numeric;
  uint64_t isum_lo;
  uint64_t isum_hi;
  uint64_t n_int;
  double fsum;
  double min;
  double max;
  double sum;
  uint32_t saw_non_numeric;
  uint32_t group_begin; /* the input's groups: all->groups[group_begin, + n_groups) */
  uint32_t n_groups;
  uint32_t _pad;
} warpjq_batch_item;

/* Batched device-resident run: the context's query over n_inputs separate
 * inputs that are already in device memory, input i being
 * d_data[offsets[i], offsets[i] + lengths[i]) (each start 16-byte aligned;
 * with d_data NULL the offsets are device addresses, so the inputs may lie
 * in different allocations, and group key_off values are addresses too),
 * in one launch sequence on `stream` with no host synchronisation.  Every
 * input gets exactly the result a run over it alone would give; lines never
 * continue from one input into the next.  Use it when many small inputs
 * would each pay a run's fixed cost (launches, host round trip).  The
 * inputs must stay in place until warpjq_batch_collect returns.  No
 * reference counterpart. */
warpjq_status warpjq_batch_launch(warpjq_ctx *ctx, const uint8_t *d_data, const uint64_t *offsets,
                                  const uint64_t *lengths, uint32_t n_inputs, void *stream,
                                  char *err, size_t err_len);

/* A mixed batch: like warpjq_batch_launch, but input i runs the query of
 * input_ctx[i], so inputs with different queries share one launch sequence:
 * one launch of the persistent scan per distinct query, each over the tiles
 * of that query's inputs with its plan as a kernel parameter, then one set
 * of row, reduce and finalize passes.  Aggregate and row queries alike; each
 * input's rows are a contiguous range of the batch's output, in input
 * order.  `ctx` supplies the buffers, tiling and stream order, and is
 * collected with warpjq_batch_collect; each item is then rendered by its own
 * query (warpjq_query_render_batch).  The input contexts are only read
 * during this call.  No reference counterpart. */
warpjq_status warpjq_batch_launch_mixed(warpjq_ctx *ctx, warpjq_ctx *const *input_ctx,
                                        const uint8_t *d_data, const uint64_t *offsets,
                                        const uint64_t *lengths, uint32_t n_inputs, void *stream,
                                        char *err, size_t err_len);

/* Waits for the batch (repeating it once with larger buffers if one
 * overflowed) and fills items[0 .. n_inputs).  `all` (may be null) describes
 * the whole batch: its rows in input order in device memory (d_out_bytes,
 * d_out_row_off with n_selected + 1 entries, d_out_line_idx as batch line
 * numbers), and every input's groups, ordered by input (key_off is an offset
 * from d_data).  Pointers stay valid until the context's next device-resident
 * run or batch.  No reference counterpart. */
warpjq_status warpjq_batch_collect(warpjq_ctx *ctx, warpjq_batch_item *items,
                                   warpjq_device_result *all, char *err, size_t err_len);

/* A CUDA graph of batched runs: the launch sequences of one batch per
 * context (each context its own query, each batch its own inputs), captured
 * once on forked streams into one graph and replayed with one launch.  No
 * reference counterpart.
 *
 * warpjq_batch_graph_create first runs every batch once, plainly (this
 * sizes every device buffer for the layout and leaves the batch tables on
 * the device), then captures.  A replay re-reads the same device addresses:
 * change the inputs' bytes in place between replays, not their offsets or
 * lengths.  After warpjq_batch_graph_launch, collect each batch with
 * warpjq_batch_collect on its context, in any order.  A replay is refused
 * (WARPJQ_ERR_INVALID_ARG) once one of its contexts has run a plain batch
 * or grown a buffer (a collect that found an overflow reruns the batch
 * plainly with larger buffers, so its result stays complete): create the
 * graph again then.  The contexts must outlive the graph. */
typedef struct warpjq_batch_graph warpjq_batch_graph;

warpjq_status warpjq_batch_graph_create(warpjq_ctx *const *ctxs, uint32_t n_ctx,
                                        const uint8_t *const *d_data, const uint64_t *const *offsets,
                                        const uint64_t *const *lengths, const uint32_t *n_inputs,
                                        warpjq_batch_graph **out, char *err, size_t err_len);
warpjq_status warpjq_batch_graph_launch(warpjq_batch_graph *g, void *stream, char *err,
                                        size_t err_len);
void warpjq_batch_graph_destroy(warpjq_batch_graph *g);

/* Device-resident scan tunables: bytes per tile (one warp walks the lines
 * starting in a tile, one line per lane) and the halo staged after it (a line
 * that runs past tile + halo is walked from global memory, more slowly).
 * 0 keeps the current value.  Tile and halo must be multiples of 256 bytes,
 * the tile at least 1024 and the halo at least 512, with tile + halo below
 * 64 KiB.  Waits for the device and releases the context's buffers. */
warpjq_status warpjq_set_tiling(warpjq_ctx *ctx, uint32_t tile_bytes, uint32_t halo_bytes);

/* Room for `keys` distinct keys (a power of two, 1024 .. 2^28; the table
 * has twice as many slots) in a fresh group table of this context; it still
 * grows on overflow.  Default 65,536.  A table sized for the input's
 * cardinality avoids the rerun an overflow costs; a small one is cleared
 * faster.  Waits for the device and releases the context's group table.  No
 * reference counterpart (the reference's table is fixed at 65,536 slots,
 * warpjq_kernels.cu:1232-1345). */
warpjq_status warpjq_set_group_capacity(warpjq_ctx *ctx, uint32_t keys);

/* Chooses the tiling for input shaped like `sample` (host bytes, e.g. the
 * first megabyte of the input): tiles holding close to a whole number of
 * 32-line rounds, and a halo longer than the longest line seen.  With fewer
 * than 16 complete lines in the sample the tiling is left alone.  Applies it
 * with warpjq_set_tiling and reports it (either pointer may be null).  No
 * reference counterpart. */
warpjq_status warpjq_autotile(warpjq_ctx *ctx, const uint8_t *sample, uint64_t len,
                              uint32_t *tile_bytes, uint32_t *halo_bytes);

/* Result of warpjq_aggregate_noalloc, written to device memory the caller
 * owns. */
typedef struct {
  uint64_t n_lines;
  uint64_t n_blank;
  uint64_t n_invalid;
  uint64_t n_type_error;
  uint64_t n_selected;
  uint64_t first_invalid; /* lowest invalid line index, or UINT64_MAX */
  uint64_t count;
  uint64_t numeric;
  uint64_t isum_lo;       /* exact sum of integer-literal values, two's complement */
  uint64_t isum_hi;
  uint64_t n_int;
  double fsum;            /* exact sum of the other numbers, rounded once to FP64 */
  double min;
  double max;
  double sum;             /* isum + the other numbers, summed exactly and rounded once */
  uint32_t saw_non_numeric;
  uint32_t status;        /* 0 complete; 1 a fixed limit was hit, do not use the counts */
} warpjq_noalloc_result;

/* An ungrouped aggregate scan (count / sum / min / max / avg, with or without
 * select()) that allocates no device memory; it has no counterpart in the
 * reference.  It is for callers that cannot call cudaMalloc: an engine that
 * gives the whole device memory to its own pool allocator at start-up leaves
 * nothing for a library to allocate, and cudaMalloc may synchronise the
 * device, which a caller in the middle of a latency-critical stream schedule
 * cannot afford.
 *
 * The caller passes the program tables, its input in device memory (16-byte
 * aligned, at most 4 GiB, larger inputs are rejected with
 * WARPJQ_ERR_INVALID_ARG) and a warpjq_noalloc_result in device memory, which
 * is written when the work on `stream` completes.  All scratch lives in one
 * fixed array of about 10 MiB that every GPU loading this library holds
 * until exit; every call shares it and it keeps the last call's contents, so
 * calls that overlap on the GPU race -- order them on one stream.  The first
 * call on each device does a one-time set-up (it looks up the array's device
 * address); make that first call before any stream capture.  Lines nesting
 * deeper than 16,448 levels exceed the fixed nesting stack and set status 1. */
warpjq_status warpjq_aggregate_noalloc(const warpjq_program *prog, const uint8_t *d_data,
                                       uint64_t n_bytes, void *stream,
                                       warpjq_noalloc_result *d_result, char *err, size_t err_len);

/* CSV input.  The reference reads NDJSON only (its --csv flag formats
 * output, crates/warpjq-core/src/output.rs:45-85); these entry points have
 * no reference counterpart.  A converter turns RFC 4180 CSV into NDJSON in
 * device memory, which any query then scans like other input:
 *   - a '\n' ends a row when an even number of '"' bytes precede it; a
 *     '\r' before it is dropped;
 *   - the first row is the header (a UTF-8 byte-order mark before it is
 *     dropped); each later row becomes one line, an empty row an empty line;
 *   - fields are split at ','; a field starting with '"' is quoted up to the
 *     next '"' not doubled, "" inside it stands for '"', and bytes after the
 *     closing quote up to the next ',' are kept;
 *   - a row is an object of the header's names, in order, over its first
 *     min(fields, names) fields;
 *   - an unquoted field that is a JSON number stays a number, an unquoted
 *     empty field is null, anything else is a JSON string (escaped like
 *     the names).
 * Line i of the NDJSON is data row i (the scan's line numbers are row
 * numbers after the header). */
typedef struct warpjq_csv warpjq_csv;

#define WARPJQ_CSV_FINAL 1u      /* the input ends with this chunk */
#define WARPJQ_CSV_HOST_INPUT 2u /* `src` is host memory (copied to the device first) */
#define WARPJQ_CSV_AFTER_STAGE0 4u /* wait for staging buffer 0's last copy first */
#define WARPJQ_CSV_AFTER_STAGE1 8u /* wait for staging buffer 1's last copy first */

warpjq_status warpjq_csv_create(warpjq_csv **out);
void warpjq_csv_destroy(warpjq_csv *c);

/* The next chunk converted starts a new input (its first row is a header). */
void warpjq_csv_reset(warpjq_csv *c);

/* Converts the rows of one chunk, n bytes at `src` (device memory unless
 * WARPJQ_CSV_HOST_INPUT), enqueued on `stream` with a few host waits.  An
 * input can arrive in chunks: each chunk must start where the previous
 * one's *consumed bytes ended; without WARPJQ_CSV_FINAL, bytes after the last
 * row-ending newline are not consumed (pass them again at the start of the
 * next chunk), and a chunk with no whole row consumes nothing.  The header
 * row's names are kept for the later chunks until warpjq_csv_reset.
 * *d_ndjson (in the converter's memory, valid until its next call) holds
 * *ndjson_len bytes of NDJSON, one line per data row converted
 * (*records, may be null). */
warpjq_status warpjq_csv_convert(warpjq_csv *c, const uint8_t *src, uint64_t n, uint32_t flags,
                                 void *stream, const uint8_t **d_ndjson, uint64_t *ndjson_len,
                                 uint64_t *consumed, uint64_t *records, char *err, size_t err_len);

/* Staging for a pipelined host input: copies n bytes of host memory
 * (page-locked, for the copy to be asynchronous) to offset `at` of the
 * converter's device staging buffer `buf` (0 or 1) on the converter's own
 * copy stream, and returns the buffer's device address in *d_buf.  A
 * conversion passed WARPJQ_CSV_AFTER_STAGE0/1 waits on the device for that
 * buffer's last staging, so the next chunk can be copied while this one is
 * converted and scanned.  Growing a buffer drops its bytes.  The host bytes
 * must stay unchanged until warpjq_csv_stage_wait on the buffer returns or a
 * conversion that waited on it has returned. */
warpjq_status warpjq_csv_stage(warpjq_csv *c, uint32_t buf, uint64_t at, const uint8_t *h_src,
                               uint64_t n, uint8_t **d_buf, char *err, size_t err_len);
warpjq_status warpjq_csv_stage_wait(warpjq_csv *c, uint32_t buf, char *err, size_t err_len);

/* Copies n bytes of device memory (e.g. the unconsumed end of a chunk: a
 * row to be continued) to offset `at` of staging buffer `buf` on `stream`;
 * [at, at + n) must lie inside the buffer. */
warpjq_status warpjq_csv_carry(warpjq_csv *c, const uint8_t *d_src, uint64_t n, uint32_t buf,
                               uint64_t at, void *stream, char *err, size_t err_len);

/* Copies the device byte slices d_src[offsets[i], + lengths[i]), i < n, to
 * host memory h_dst back to back (d_src may be NULL: offsets are then
 * device addresses) (e.g. the group keys of a run over
 * converted CSV, whose NDJSON lives only on the device).  Synchronous. */
warpjq_status warpjq_csv_gather(warpjq_csv *c, const uint8_t *d_src, const uint64_t *offsets,
                                const uint32_t *lengths, uint64_t n, uint8_t *h_dst, void *stream,
                                char *err, size_t err_len);

/* Copies n bytes of device memory to host memory on `stream` and waits. */
warpjq_status warpjq_device_read(void *h_dst, const void *d_src, uint64_t n, void *stream,
                                 char *err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* WARPJQ_EXT_H */
