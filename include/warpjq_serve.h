/* warpjq GPU backend -- resident serving loop, C ABI.
 *
 * No reference counterpart: the reference runs one query per process
 * invocation (crates/warpjq-cli/src/run.rs:16-96), paying the device
 * context's set-up every time.  A server keeps, for a fixed list of
 * queries, every device context, compiled plan, stream, CSV converter and
 * staging buffer alive, and runs requests (one query over one input each)
 * with continuous batching (CSV requests first converted on the device by
 * a converter thread): a native loop thread admits waiting requests
 * into a free slot while earlier slots are still on the device, as long as
 * their device-memory footprints fit the budget beside what is in flight
 * (in arrival order, no overtaking), runs each slot's requests as one
 * batched scan per query (warpjq_batch_launch, or one mixed batch for many
 * requests, warpjq_batch_launch_mixed), and renders every
 * finished request's output on the host.  Each output is byte for byte what
 * a run over that input alone prints (warpjq_query_run).
 *
 * Return codes as warpjq_host.h: 0 success, 1 runtime error, 2 query error.
 */
#ifndef WARPJQ_SERVE_H
#define WARPJQ_SERVE_H

#include <stddef.h>
#include <stdint.h>

#include "warpjq_host.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct warpjq_server warpjq_server;

typedef struct {
  uint32_t n_slots;      /* batches in flight at once, each on its own stream (0: 3) */
  uint32_t max_batch;    /* requests one slot takes at most (0: no limit; 1 with one slot
                          * serves requests one at a time) */
  uint64_t budget_bytes; /* device memory admitted requests may hold at once (0: 120 GiB) */
  uint32_t format;       /* WARPJQ_FMT_* of every output */
  uint32_t mixed_min;    /* a slot's requests of two or more queries run as one mixed batch
                          * (one launch sequence, each input with its own plan) from this
                          * many on (0: never) */
  uint64_t chunk_bytes;  /* the contexts' chunk size (0: 1 MiB; only sizes host-run buffers) */
  uint64_t slot_bytes;   /* input bytes one slot takes at a time (0: 1 GiB; a larger request
                          * goes alone), so waiting work spreads over the slots */
} warpjq_serve_config;

/* Request flags. */
#define WARPJQ_SERVE_DEVICE 1u /* `data` is device memory (used in place when 16-byte aligned) */
#define WARPJQ_SERVE_CSV 2u    /* `data` is CSV (warpjq_ext.h warpjq_csv_convert's mapping) */

typedef struct {
  uint64_t id;         /* the id warpjq_serve_enqueue returned */
  uint32_t query;      /* index into the server's queries */
  int32_t rc;          /* 0, or 1 with `err` set (nothing else is valid then) */
  char *out;           /* the output (free with warpjq_host_free) */
  uint64_t out_len;
  uint64_t n_lines;    /* non-blank input lines */
  uint64_t n_invalid;  /* malformed lines (skipped, as --skip-invalid does) */
  double queue_ms;     /* arrival to admission */
  double latency_ms;   /* arrival to completion */
  char err[160];
} warpjq_serve_result;

/* Opens a server for `queries` (each parsed and compiled once per slot) on
 * the current device and starts its loop thread. */
int warpjq_serve_open(const char *const *queries, uint32_t n_queries, const warpjq_serve_config *cfg,
                      warpjq_server **out, char *err, size_t err_len);

/* Runs every slot's every query once over `reserve_bytes` of blank lines,
 * converts a CSV input of a quarter of that size and reserves each slot's
 * input arena and row buffers for inputs that large, so buffers reach their
 * working sizes and every kernel is loaded before requests arrive.  Call
 * before the first request. */
int warpjq_serve_warm(warpjq_server *s, uint64_t reserve_bytes, char *err, size_t err_len);

/* Queues one request: query `query` over `len` bytes at `data` (host memory
 * unless WARPJQ_SERVE_DEVICE).  The bytes must stay unchanged until the
 * request's result is returned by warpjq_serve_poll.  *id receives the
 * request's id.  A request whose footprint alone exceeds the budget is
 * completed at once with rc 1.  Thread-safe. */
int warpjq_serve_enqueue(warpjq_server *s, uint32_t query, const uint8_t *data, uint64_t len, uint32_t flags,
                         uint64_t *id, char *err, size_t err_len);

/* Moves up to `max_done` completed requests into `done` (in completion
 * order) and returns how many; waits up to `timeout_ms` for the first one
 * (0: no wait, negative: until one completes or nothing is pending).
 * Thread-safe. */
uint32_t warpjq_serve_poll(warpjq_server *s, warpjq_serve_result *done, uint32_t max_done, int timeout_ms);

/* Requests queued or on the device, not yet returned by a poll. */
uint64_t warpjq_serve_pending(warpjq_server *s);

/* Stops the loop after the requests in flight, drops the waiting ones and
 * frees everything (outputs not yet polled included). */
void warpjq_serve_close(warpjq_server *s);

#ifdef __cplusplus
}
#endif

#endif /* WARPJQ_SERVE_H */
