/* warpjq device backend -- the drop-in C ABI.
 *
 * This header declares exactly the entry points, enums and struct layouts of
 * the reference project's crates/warpjq-core/cuda/warpjq_kernels.h, so the
 * reference's Rust host (crates/warpjq-core/src/gpu/ffi.rs) links against this
 * backend unchanged.  The implementation behind it is new: sm_100a kernels
 * that decide every line on the device (no per-line or per-chunk CPU
 * fallback), so `n_fallback` is always 0 and the `fallback_*` arrays are
 * always empty, and `chunk_overflow` / `group_overflow` are never set.
 *
 * Conventions kept from the reference (warpjq_kernels.h:3-12):
 *   - plain C, fixed-width types, no ownership transfer; every pointer passed
 *     in is borrowed for the duration of the call;
 *   - errors are a warpjq_status plus a message in the caller's err[err_len];
 *   - results returned by warpjq_wait point into backend-owned pinned memory
 *     and stay valid until the next warpjq_submit on the same slot.
 */
#ifndef WARPJQ_KERNELS_H
#define WARPJQ_KERNELS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (reference warpjq_kernels.h:25-32). */
typedef enum {
  WARPJQ_OK = 0,
  WARPJQ_ERR_CUDA = 1,
  WARPJQ_ERR_NO_DEVICE = 2,
  WARPJQ_ERR_OOM = 3,
  WARPJQ_ERR_ABI = 4,
  WARPJQ_ERR_INVALID_ARG = 5
} warpjq_status;

/* Per-line outcome codes (reference warpjq_kernels.h:35-41). */
typedef enum {
  WARPJQ_LINE_OK = 0,
  WARPJQ_LINE_INVALID = 1,
  WARPJQ_LINE_TYPE_ERROR = 2,
  WARPJQ_LINE_FALLBACK = 3, /* never produced by this backend */
  WARPJQ_LINE_BLANK = 4
} warpjq_line_status;

/* Plan-table codes (reference warpjq_kernels.h:45-86; the values are part of
 * the ABI because the Rust side writes them into the tables). */
enum { WARPJQ_STEP_KEY = 0, WARPJQ_STEP_INDEX = 1 };
enum {
  WARPJQ_LIT_NULL = 0,
  WARPJQ_LIT_FALSE = 1,
  WARPJQ_LIT_TRUE = 2,
  WARPJQ_LIT_NUM = 3,
  WARPJQ_LIT_STR = 4
};
enum {
  WARPJQ_COND_CMP = 0,
  WARPJQ_COND_TRUTHY = 1,
  WARPJQ_COND_AND = 2,
  WARPJQ_COND_OR = 3,
  WARPJQ_COND_NOT = 4
};
enum {
  WARPJQ_OP_EQ = 0,
  WARPJQ_OP_NE = 1,
  WARPJQ_OP_LT = 2,
  WARPJQ_OP_LE = 3,
  WARPJQ_OP_GT = 4,
  WARPJQ_OP_GE = 5
};
enum {
  WARPJQ_OUT_PASSTHROUGH = 0,
  WARPJQ_OUT_PATH = 1,
  WARPJQ_OUT_PROJECT = 2,
  WARPJQ_OUT_AGG = 3
};
enum {
  WARPJQ_AGG_COUNT = 0,
  WARPJQ_AGG_SUM = 1,
  WARPJQ_AGG_MIN = 2,
  WARPJQ_AGG_MAX = 3,
  WARPJQ_AGG_AVG = 4
};

/* One path step: 20 bytes (reference warpjq_kernels.h:88-94). */
typedef struct {
  uint32_t kind;     /* WARPJQ_STEP_* */
  uint32_t index;    /* array index for WARPJQ_STEP_INDEX */
  uint32_t key_off;  /* decoded key bytes, offset into blob */
  uint32_t key_len;
  uint32_t key_hash; /* FNV-1a 32 of the decoded key (query/mod.rs:15-22) */
} warpjq_step;

/* A path is a run of steps: 8 bytes (reference warpjq_kernels.h:96-99). */
typedef struct {
  uint32_t step_off;
  uint32_t step_count;
} warpjq_path;

/* One comparison `path op literal`: 32 bytes (reference warpjq_kernels.h:101-109). */
typedef struct {
  uint32_t path;
  uint32_t op;       /* WARPJQ_OP_* */
  uint32_t lit_kind; /* WARPJQ_LIT_* */
  uint32_t lit_off;  /* string literal bytes in blob */
  uint32_t lit_len;
  uint32_t _pad;
  double lit_num;
} warpjq_cmp;

/* One reverse-Polish condition op: 8 bytes (reference warpjq_kernels.h:111-114). */
typedef struct {
  uint32_t op;  /* WARPJQ_COND_* */
  uint32_t arg; /* cmp index for CMP, path id for TRUTHY */
} warpjq_cond_op;

/* The compiled query as flat tables (reference warpjq_kernels.h:117-153).
 * warpjq_ctx_create copies everything it needs; nothing is retained. */
typedef struct {
  const warpjq_step *steps;
  uint32_t n_steps;
  const warpjq_path *paths;
  uint32_t n_paths;
  const warpjq_cmp *cmps;
  uint32_t n_cmps;
  const warpjq_cond_op *cond_rpn;
  uint32_t n_cond;
  const uint8_t *blob;
  uint32_t n_blob;

  /* Paths the backend must resolve; slot_of_path[path] is the slot index or
   * 0xFFFFFFFF. */
  const uint32_t *needed_paths;
  uint32_t n_needed;
  const uint32_t *slot_of_path;

  uint32_t output_kind; /* WARPJQ_OUT_* */
  uint32_t output_path; /* WARPJQ_OUT_PATH */
  uint32_t agg_kind;    /* WARPJQ_AGG_* */
  uint32_t agg_path;    /* 0xFFFFFFFF for count */
  uint32_t group_path;  /* 0xFFFFFFFF when ungrouped */
  uint32_t has_filter;

  /* Projection: value i is preceded by the literal bytes prefix[i] and the
   * row ends with the suffix; the host renders key names into these. */
  uint32_t n_fields;
  const uint32_t *field_paths;
  const uint32_t *prefix_off;
  const uint32_t *prefix_len;
  uint32_t suffix_off;
  uint32_t suffix_len;
  uint32_t csv_mode; /* 1: render values as CSV cells */
} warpjq_program;

/* Ungrouped aggregate of one chunk: 48 bytes (reference warpjq_kernels.h:159-167). */
typedef struct {
  uint64_t count;
  uint64_t numeric;
  double sum;
  double min;
  double max;
  uint32_t saw_non_numeric;
  uint32_t _pad;
} warpjq_agg_partial;

/* One group of one chunk: 56 bytes (reference warpjq_kernels.h:170-180).
 * key_off is an offset into the submitted chunk; for string keys it covers
 * the body between the quotes. */
typedef struct {
  uint32_t key_off;
  uint32_t key_len;
  uint32_t key_kind; /* JSON kind code 0..6: missing null bool num str arr obj */
  uint32_t _pad;
  uint64_t count;
  uint64_t numeric;
  double sum;
  double min;
  double max;
} warpjq_group;

/* What warpjq_wait reports for one chunk (reference warpjq_kernels.h:182-230). */
typedef struct {
  uint64_t n_lines;      /* physical lines, blank ones included */
  uint64_t n_blank;
  uint64_t n_invalid;
  uint64_t n_type_error;
  uint64_t n_fallback;   /* always 0 */
  uint64_t n_selected;

  const uint8_t *out_bytes;     /* assembled rows in input order */
  uint64_t out_len;
  const uint32_t *out_line_idx; /* chunk line index of each row, ascending */
  const uint64_t *out_row_off;  /* n_selected + 1 row offsets into out_bytes */

  const uint32_t *fallback_idx; /* always empty */
  const uint32_t *fallback_off;
  const uint32_t *fallback_len;
  uint32_t chunk_overflow;      /* always 0 */
  uint32_t first_invalid;       /* lowest invalid line index, or 0xFFFFFFFF */

  warpjq_agg_partial agg;

  const warpjq_group *groups;
  uint32_t n_groups;
  uint32_t group_overflow;      /* always 0 */
} warpjq_chunk_result;

typedef struct warpjq_ctx warpjq_ctx;

/* reference warpjq_kernels.h:238-274 */
warpjq_status warpjq_probe(char *err, size_t err_len);
warpjq_status warpjq_abi_check(const uint64_t *sizes, size_t n);
warpjq_status warpjq_ctx_create(const warpjq_program *prog, uint64_t max_chunk_bytes,
                                uint32_t n_slots, warpjq_ctx **out, char *err, size_t err_len);
void warpjq_ctx_destroy(warpjq_ctx *ctx);
uint8_t *warpjq_slot_buffer(warpjq_ctx *ctx, uint32_t slot);
uint64_t warpjq_slot_capacity(const warpjq_ctx *ctx);
uint64_t warpjq_max_lines(const warpjq_ctx *ctx);
warpjq_status warpjq_submit(warpjq_ctx *ctx, uint32_t slot, uint64_t n_bytes, char *err,
                            size_t err_len);
warpjq_status warpjq_wait(warpjq_ctx *ctx, uint32_t slot, warpjq_chunk_result *out, char *err,
                          size_t err_len);
warpjq_status warpjq_device_name(char *buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* WARPJQ_KERNELS_H */
