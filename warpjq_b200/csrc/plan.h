// Device plan: the compiled query in the form the sm_100a kernels read.
//
// warpjq_ctx_create turns the reference's flat warpjq_program tables
// (crates/warpjq-core/src/gpu/lower.rs:38-127) into this structure once per
// context.  The needed paths become a trie so one pass over a line resolves
// every path at once: each node is one path step, and a line's walker
// records, per node, the kind and byte span of the last value seen there
// (last duplicate key wins, json.rs:521-556).
#pragma once

#include <stdint.h>

namespace wjq {

constexpr int kMaxSlots = 16;   // needed paths per query (reference limit, cu:56)
constexpr int kMaxNodes = 64;   // trie nodes including the root
constexpr int kMaxCmps = 64;
constexpr int kMaxCond = 128;
constexpr int kMaxFields = 16;
constexpr int kMaxBlob = 4096;
constexpr int kMaxDepthFast = 64;  // container depth tracked in registers
constexpr uint8_t kNoNode = 0xFF;
constexpr uint32_t kRowRecBytes = 32;  // header of a staged row record (kernels.cuh RowRec)

// JSON kind codes shared with the ABI (warpjq_group.key_kind).
enum JKind : uint8_t {
  JK_MISSING = 0,
  JK_NULL = 1,
  JK_BOOL = 2,
  JK_NUM = 3,
  JK_STR = 4,
  JK_ARR = 5,
  JK_OBJ = 6
};

struct PlanNode {
  // Bit L set when a key child's key is L bytes long (bit 63: 63 or more);
  // a key of any other length cannot match and is skipped without compare.
  unsigned long long key_len_mask;
  uint32_t index;        // array index, for an index step
  uint16_t key_off;      // decoded key bytes in blob, for a key step
  uint16_t key_len;
  uint8_t parent;        // kNoNode for the root
  uint8_t is_index;      // step from the parent is an index step
  uint8_t first_child;   // kNoNode when a leaf
  uint8_t next_sibling;  // kNoNode at the end of the list
  uint8_t subtree_end;   // nodes are numbered in preorder: subtree = [id, subtree_end)
  uint8_t has_key_children;
  uint8_t has_index_children;
  uint8_t key_first;     // first key byte, a cheap reject before comparing
  uint32_t key_w[2];     // the key's first 8 bytes, little-endian, zero past its end
};

struct PlanCmp {
  double lit_num;
  uint16_t lit_off;  // string literal bytes in blob
  uint16_t lit_len;
  uint8_t slot;
  uint8_t op;        // WARPJQ_OP_*
  uint8_t lit_kind;  // WARPJQ_LIT_*
  uint8_t lit_rank;  // jq type rank of the literal (ir.rs:100-108)
};

struct PlanCond {
  uint8_t op;   // WARPJQ_COND_*
  uint8_t arg;  // cmp index, or slot for TRUTHY
};

struct DevPlan {
  uint32_t n_nodes;
  uint32_t n_slots;
  uint32_t n_cmps;
  uint32_t n_cond;
  uint32_t output_kind;  // WARPJQ_OUT_*
  uint32_t agg_kind;     // WARPJQ_AGG_*
  uint32_t csv_mode;
  uint32_t has_filter;
  int32_t out_slot;      // WARPJQ_OUT_PATH
  int32_t agg_slot;      // -1 for count
  int32_t group_slot;    // -1 when ungrouped
  uint32_t n_fields;
  uint32_t filter_slot_mask;  // slots the filter reads (type errors there always count)
  uint32_t rec_stride;        // bytes per selected-row record
  uint32_t needs_rows;        // passthrough / path / projection
  uint32_t suffix_off, suffix_len;
  int8_t field_slot[kMaxFields];
  uint16_t prefix_off[kMaxFields];
  uint16_t prefix_len[kMaxFields];
  uint8_t slot_node[kMaxSlots];
  PlanNode nodes[kMaxNodes];
  PlanCmp cmps[kMaxCmps];
  PlanCond cond[kMaxCond];
  uint8_t blob[kMaxBlob];
};

// Per-tile bookkeeping written by the scan kernel.
struct TileDesc {
  uint32_t n_lines;           // physical lines starting in the tile
  uint32_t first_invalid;     // tile-relative line ordinal, or 0xFFFFFFFF
  uint32_t first_type_error;  // tile-relative line ordinal, or 0xFFFFFFFF
  uint32_t pad;
};

// Everything the scan kernel accumulates for a run, in device memory.
struct RunCounters {
  unsigned long long next_tile;  // work ticket
  unsigned long long n_lines;
  unsigned long long n_blank;
  unsigned long long n_invalid;
  unsigned long long n_type_error;
  unsigned long long n_selected;
  unsigned long long out_len;
  unsigned long long first_invalid_tile;  // lowest tile holding an invalid line
  unsigned long long first_type_tile;     // lowest tile holding a type error
  // ungrouped aggregate
  unsigned long long agg_count;
  unsigned long long agg_numeric;
  unsigned long long agg_isum_lo;
  unsigned long long agg_isum_hi;
  unsigned long long agg_n_int;
  unsigned long long agg_min_bits;  // order-preserving encoding (agg.rs:205-212)
  unsigned long long agg_max_bits;
  unsigned int agg_saw_non_numeric;
  // group table
  unsigned int n_keys;
  unsigned int overflow;     // bit0 records, bit1 output, bit2 groups, bit3 deep stack
  unsigned int error;        // nonzero: a kernel found its own state inconsistent
  // exact sum of the non-integer aggregate values (fixsum.cuh): limb k
  // counts units of 2^(32 k - 128); values of magnitude >= 2^128 go to fbig
  long long fix[8];
  double fbig;
  double fsum_total;         // written by the finalize kernel: the rounded fix sum + fbig
  double sum_total;          // written by the finalize kernel: integer + fix sums rounded once, + fbig
  unsigned long long first_invalid;     // written by the finalize kernel
  unsigned long long first_type_error;  // written by the finalize kernel
};

}  // namespace wjq
