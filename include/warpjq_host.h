/* warpjq GPU backend -- host driver API.
 *
 * The reference runs its GPU backend from Rust (crates/warpjq-core/src/gpu/
 * mod.rs, exec/mod.rs); this C API is the same layer written in C++ so the
 * backend can be driven without a Rust toolchain: parse a jq-subset query,
 * lower it to the device tables of warpjq_kernels.h, stream a buffer through
 * warpjq_submit / warpjq_wait and format the output exactly as the reference
 * CPU engine does (exec/cpu.rs:498 run_bytes is the call it mirrors).
 *
 * Return codes: 0 success, 1 runtime error (message in err), 2 query error
 * (the rendered message in err), matching the CLI's exit codes for errors
 * (crates/warpjq-cli/src/main.rs:169-189).
 */
#ifndef WARPJQ_HOST_H
#define WARPJQ_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "warpjq_ext.h"
#include "warpjq_kernels.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Output formats (output.rs:14-21) and malformed-line policies
 * (exec/mod.rs:29-41). */
enum { WARPJQ_FMT_NDJSON = 0, WARPJQ_FMT_CSV = 1, WARPJQ_FMT_COUNT = 2 };
enum { WARPJQ_ON_INVALID_WARN = 0, WARPJQ_ON_INVALID_SKIP = 1, WARPJQ_ON_INVALID_ABORT = 2 };

typedef struct warpjq_query warpjq_query;

/* Parses and lowers `query`, and creates its device context with chunks of
 * at most min(chunk_bytes, 64 MiB) (gpu/mod.rs:143-145). */
int warpjq_query_open(const char *query, uint32_t format, uint64_t chunk_bytes,
                      warpjq_query **out, char *err, size_t err_len);
void warpjq_query_close(warpjq_query *q);

/* Parses and lowers `query` without a device context: enough to render
 * results (warpjq_query_render_device), e.g. on the rank that merges the
 * partial results of several GPUs; the query cannot run. */
int warpjq_query_open_host(const char *query, uint32_t format, warpjq_query **out, char *err,
                           size_t err_len);
int warpjq_query_is_grouped(const warpjq_query *q);

/* The device context, for device-resident runs through warpjq_ext.h. */
warpjq_ctx *warpjq_query_ctx(warpjq_query *q);
int warpjq_query_is_aggregate(const warpjq_query *q);

/* Runs the query over a host buffer.  On success *out is a malloc'd buffer
 * (free with warpjq_host_free) and stats receives bytes_in, lines_in,
 * lines_out, malformed, type_errors. */
int warpjq_query_run(warpjq_query *q, const uint8_t *data, size_t len, uint32_t on_invalid,
                     uint64_t max_line_bytes, char **out, size_t *out_len, uint64_t *stats,
                     char *err, size_t err_len);

/* Runs the query over a file: read with parallel preads into page-locked
 * buffers, in newline-aligned chunks, each chunk read while the device works
 * on the one before.  Output and stats as warpjq_query_run; error messages
 * name the file. */
int warpjq_query_run_file(warpjq_query *q, const char *path, uint32_t on_invalid,
                          uint64_t max_line_bytes, char **out, size_t *out_len, uint64_t *stats,
                          char *err, size_t err_len);

/* One-shot: open, run, close. */
int warpjq_run_bytes(const char *query, const uint8_t *data, size_t len, uint32_t format,
                     uint32_t on_invalid, uint64_t chunk_bytes, uint64_t max_line_bytes,
                     char **out, size_t *out_len, uint64_t *stats, char *err, size_t err_len);

/* Formats a device-resident aggregate result; `data` is a host copy of the
 * input (group keys are rendered from it). */
int warpjq_query_render_device(warpjq_query *q, const warpjq_device_result *r,
                               const uint8_t *data, char **out, size_t *out_len);

/* Every input's output of a collected batch (warpjq_batch_collect), back to
 * back in one buffer (free with warpjq_host_free): input i's bytes are
 * (*out)[offsets[i], offsets[i + 1]) -- what a run over it alone prints.
 * `groups` is the batch's group array (warpjq_device_result.groups) and
 * `key_data` the host bytes its key_off values index; `rows` and `row_off`
 * a host copy of the batch's rows and row offsets (null for aggregates).
 * offsets has n + 1 entries.  No reference counterpart. */
int warpjq_query_render_batch(warpjq_query *q, const warpjq_batch_item *items, uint32_t n,
                              const warpjq_group_ext *groups, const uint8_t *key_data, const uint8_t *rows,
                              const uint64_t *row_off, char **out, size_t *out_len, uint64_t *offsets);

void warpjq_host_free(void *p);

/* Runs the query over RFC 4180 CSV input in host memory: the header row
 * names the keys and each later row is one object, converted on the device
 * by the mapping warpjq_ext.h gives for warpjq_csv_convert, then scanned like
 * NDJSON.  Output, stats and return codes as warpjq_query_run (rows that a
 * query passes through print as the converted NDJSON; --strict errors name
 * the data row, counted after the header).  Chunks of the context's chunk
 * size are converted and scanned one after another.  The query must have a
 * device context (warpjq_query_open).  No reference counterpart: the
 * reference reads NDJSON only. */
int warpjq_query_run_csv(warpjq_query *q, const uint8_t *data, size_t len, uint32_t on_invalid,
                         char **out, size_t *out_len, uint64_t *stats, char *err, size_t err_len);

/* Seeded synthetic input in the benchmark's nginx-style schema (keys ts,
 * host, method, path, status, bytes, latency_ms, ua).  Writes whole lines,
 * about `target` bytes, into out (capacity >= target), generating blocks of
 * `block_bytes` on `threads` threads (0 = all cores).  Returns the bytes
 * written; *total_lines receives the line count. */
uint64_t warpjq_gen_nginx(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                          unsigned threads, uint64_t *total_lines);
uint64_t warpjq_gen_nginx_block(uint64_t seed, uint64_t block, uint64_t first_line, uint8_t *out,
                                uint64_t cap, uint64_t *n_lines);

/* The same records rendered as CSV: a header row naming the columns
 * (ts,host,method,path,status,bytes,latency_ms,ua), then one row per record
 * with ua always quoted ('"' doubled).  Returns the bytes written. */
uint64_t warpjq_gen_nginx_csv(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                              unsigned threads, uint64_t *total_lines);
uint64_t warpjq_gen_nginx_csv_block(uint64_t seed, uint64_t block, uint64_t first_line, uint8_t *out,
                                    uint64_t cap, uint64_t *n_lines);
/* The NDJSON lines of exactly the records warpjq_gen_nginx_csv writes with
 * the same seed, target and block size, in order; `out` holds 2 * target
 * bytes.  Returns the bytes written. */
uint64_t warpjq_gen_nginx_csv_as_ndjson(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                                        unsigned threads, uint64_t *total_lines);

/* The same for a nested, dirty schema: objects 3-5 levels deep with shuffled
 * key order (req.user.{id, tier, geo{cc, lat, lon}}, req.method, req.path,
 * resp.{code, latency, size}, meta.trace.span.{id, depth}, ts), about 10% of
 * strings with escapes, latencies in decimal and exponent forms, user ids
 * Zipf(0.9) over [1, n_users], and about 2% malformed lines (cut short, a
 * bare NaN, a leading zero). */
uint64_t warpjq_gen_nested(uint64_t seed, uint8_t *out, uint64_t target, uint64_t block_bytes,
                           unsigned threads, uint64_t n_users, uint64_t *total_lines);
uint64_t warpjq_gen_nested_block(uint64_t seed, uint64_t block, uint64_t first_line, uint64_t n_users,
                                 uint8_t *out, uint64_t cap, uint64_t *n_lines);

#ifdef __cplusplus
}
#endif

#endif /* WARPJQ_HOST_H */
