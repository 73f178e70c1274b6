// Host-side compilation of the flat warpjq_program tables into a DevPlan
// (see plan.h).  Header-only so the device backend and the host-compiled
// walker test share one implementation.
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/warpjq_kernels.h"
#include "plan.h"

namespace wjq {

inline void set_err(char *err, size_t n, const char *fmt, ...) {
  if (!err || !n) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, n, fmt, ap);
  va_end(ap);
}


struct TmpNode {
  bool is_index = false;
  uint32_t index = 0;
  uint32_t key_off = 0, key_len = 0;
  std::vector<int> kids;
  int parent = -1;
};

inline warpjq_status build_plan(const warpjq_program *p, DevPlan &P, char *err, size_t err_len) {
  std::memset(&P, 0, sizeof(P));
  if (!p) {
    set_err(err, err_len, "program is null");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (p->n_needed > (uint32_t)kMaxSlots) {
    set_err(err, err_len, "query needs %u field paths; this backend resolves at most %d",
            p->n_needed, kMaxSlots);
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (p->n_blob > (uint32_t)kMaxBlob || p->n_cmps > (uint32_t)kMaxCmps ||
      p->n_cond > (uint32_t)kMaxCond || p->n_fields > (uint32_t)kMaxFields) {
    set_err(err, err_len, "query is too large for the device plan");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (p->n_blob) std::memcpy(P.blob, p->blob, p->n_blob);
  auto slot_of = [&](uint32_t path) -> int {
    if (path >= p->n_paths) return -1;
    uint32_t s = p->slot_of_path[path];
    return s == 0xFFFFFFFFu ? -1 : (int)s;
  };

  // Trie over the needed paths.
  std::vector<TmpNode> tn(1);
  std::vector<int> slot_tmp(p->n_needed, 0);
  for (uint32_t s = 0; s < p->n_needed; s++) {
    uint32_t path = p->needed_paths[s];
    if (path >= p->n_paths) {
      set_err(err, err_len, "needed path %u out of range", path);
      return WARPJQ_ERR_INVALID_ARG;
    }
    const warpjq_path &wp = p->paths[path];
    if (wp.step_count == 0 || wp.step_count > (uint32_t)kMaxDepthFast - 2) {
      set_err(err, err_len, "path %u has %u steps; the device supports 1..%d", path, wp.step_count,
              kMaxDepthFast - 2);
      return WARPJQ_ERR_INVALID_ARG;
    }
    int cur = 0;
    for (uint32_t k = 0; k < wp.step_count; k++) {
      const warpjq_step &st = p->steps[wp.step_off + k];
      bool is_index = st.kind == WARPJQ_STEP_INDEX;
      if (!is_index && (st.key_off + st.key_len > p->n_blob)) {
        set_err(err, err_len, "step key out of the blob");
        return WARPJQ_ERR_INVALID_ARG;
      }
      int found = -1;
      for (int c : tn[cur].kids) {
        const TmpNode &x = tn[c];
        if (x.is_index != is_index) continue;
        if (is_index ? x.index == st.index
                     : (x.key_len == st.key_len &&
                        std::memcmp(p->blob + x.key_off, p->blob + st.key_off, st.key_len) == 0)) {
          found = c;
          break;
        }
      }
      if (found < 0) {
        TmpNode nn;
        nn.is_index = is_index;
        nn.index = st.index;
        nn.key_off = st.key_off;
        nn.key_len = st.key_len;
        nn.parent = cur;
        tn.push_back(nn);
        found = (int)tn.size() - 1;
        tn[cur].kids.push_back(found);
      }
      cur = found;
    }
    slot_tmp[s] = cur;
  }
  if (tn.size() > (size_t)kMaxNodes) {
    set_err(err, err_len, "query paths need %zu trie nodes; at most %d", tn.size(), kMaxNodes);
    return WARPJQ_ERR_INVALID_ARG;
  }
  // Preorder numbering.
  std::vector<int> order, newid(tn.size());
  std::vector<int> stack{0};
  while (!stack.empty()) {
    int x = stack.back();
    stack.pop_back();
    newid[x] = (int)order.size();
    order.push_back(x);
    for (auto it = tn[x].kids.rbegin(); it != tn[x].kids.rend(); ++it) stack.push_back(*it);
  }
  std::vector<int> subtree_end(tn.size());
  for (int i = (int)order.size() - 1; i >= 0; i--) {
    int x = order[i];
    int e = i + 1;
    for (int c : tn[x].kids) e = std::max(e, subtree_end[c]);
    subtree_end[x] = e;
  }
  P.n_nodes = p->n_needed ? (uint32_t)tn.size() : 0;
  for (size_t i = 0; i < order.size() && P.n_nodes; i++) {
    const TmpNode &x = tn[order[i]];
    PlanNode &d = P.nodes[i];
    d.index = x.index;
    d.key_off = (uint16_t)x.key_off;
    d.key_len = (uint16_t)x.key_len;
    d.parent = x.parent < 0 ? kNoNode : (uint8_t)newid[x.parent];
    d.is_index = x.is_index;
    d.first_child = x.kids.empty() ? kNoNode : (uint8_t)newid[x.kids[0]];
    d.next_sibling = kNoNode;
    d.subtree_end = (uint8_t)subtree_end[order[i]];
    d.key_first = (!x.is_index && x.key_len) ? p->blob[x.key_off] : 0;
    d.key_w[0] = d.key_w[1] = 0;
    for (uint32_t b = 0; !x.is_index && b < x.key_len && b < 8; b++)
      d.key_w[b >> 2] |= (uint32_t)p->blob[x.key_off + b] << (8 * (b & 3));
    d.key_len_mask = 0;
    for (size_t k = 0; k < x.kids.size(); k++) {
      const TmpNode &c = tn[x.kids[k]];
      if (c.is_index) {
        d.has_index_children = 1;
      } else {
        d.has_key_children = 1;
        d.key_len_mask |= 1ull << (c.key_len < 63 ? c.key_len : 63);
      }
    }
  }
  // Sibling links last: filling a node above resets its own link.
  for (size_t i = 0; i < order.size() && P.n_nodes; i++) {
    const TmpNode &x = tn[order[i]];
    for (size_t k = 0; k + 1 < x.kids.size(); k++)
      P.nodes[newid[x.kids[k]]].next_sibling = (uint8_t)newid[x.kids[k + 1]];
  }
  P.n_slots = p->n_needed;
  for (uint32_t s = 0; s < p->n_needed; s++) P.slot_node[s] = (uint8_t)newid[slot_tmp[s]];

  // Condition.
  P.n_cmps = p->n_cmps;
  for (uint32_t i = 0; i < p->n_cmps; i++) {
    const warpjq_cmp &c = p->cmps[i];
    int s = slot_of(c.path);
    if (s < 0 || c.op > 5 || c.lit_kind > 4 || c.lit_off + c.lit_len > p->n_blob) {
      set_err(err, err_len, "comparison %u is malformed", i);
      return WARPJQ_ERR_INVALID_ARG;
    }
    PlanCmp &d = P.cmps[i];
    d.lit_num = c.lit_num;
    d.lit_off = (uint16_t)c.lit_off;
    d.lit_len = (uint16_t)c.lit_len;
    d.slot = (uint8_t)s;
    d.op = (uint8_t)c.op;
    d.lit_kind = (uint8_t)c.lit_kind;
    d.lit_rank = (uint8_t)c.lit_kind;  // null 0, false 1, true 2, num 3, str 4 (ir.rs:100-108)
    P.filter_slot_mask |= 1u << s;
  }
  P.n_cond = p->n_cond;
  int depth = 0, max_depth = 0;
  for (uint32_t i = 0; i < p->n_cond; i++) {
    const warpjq_cond_op &o = p->cond_rpn[i];
    PlanCond &d = P.cond[i];
    d.op = (uint8_t)o.op;
    if (o.op == WARPJQ_COND_CMP) {
      if (o.arg >= p->n_cmps) {
        set_err(err, err_len, "condition references comparison %u", o.arg);
        return WARPJQ_ERR_INVALID_ARG;
      }
      d.arg = (uint8_t)o.arg;
      depth++;
    } else if (o.op == WARPJQ_COND_TRUTHY) {
      int s = slot_of(o.arg);
      if (s < 0) {
        set_err(err, err_len, "condition references an unresolved path");
        return WARPJQ_ERR_INVALID_ARG;
      }
      d.arg = (uint8_t)s;
      P.filter_slot_mask |= 1u << s;
      depth++;
    } else if (o.op == WARPJQ_COND_AND || o.op == WARPJQ_COND_OR) {
      depth--;
    } else if (o.op != WARPJQ_COND_NOT) {
      set_err(err, err_len, "unknown condition op %u", o.op);
      return WARPJQ_ERR_INVALID_ARG;
    }
    max_depth = std::max(max_depth, depth);
    if (depth < 1) {
      set_err(err, err_len, "condition stack underflows");
      return WARPJQ_ERR_INVALID_ARG;
    }
  }
  if (max_depth > 63) {
    set_err(err, err_len, "condition nests deeper than the device evaluator supports");
    return WARPJQ_ERR_INVALID_ARG;
  }
  P.has_filter = p->has_filter && p->n_cond > 0;

  // Output.
  P.output_kind = p->output_kind;
  P.agg_kind = p->agg_kind;
  P.csv_mode = p->csv_mode;
  P.out_slot = -1;
  P.agg_slot = -1;
  P.group_slot = -1;
  if (p->output_kind == WARPJQ_OUT_PATH) {
    P.out_slot = slot_of(p->output_path);
    if (P.out_slot < 0) {
      set_err(err, err_len, "output path has no slot");
      return WARPJQ_ERR_INVALID_ARG;
    }
  } else if (p->output_kind == WARPJQ_OUT_PROJECT) {
    P.n_fields = p->n_fields;
    for (uint32_t f = 0; f < p->n_fields; f++) {
      int s = slot_of(p->field_paths[f]);
      if (s < 0 || p->prefix_off[f] + p->prefix_len[f] > p->n_blob) {
        set_err(err, err_len, "projection field %u is malformed", f);
        return WARPJQ_ERR_INVALID_ARG;
      }
      P.field_slot[f] = (int8_t)s;
      P.prefix_off[f] = (uint16_t)p->prefix_off[f];
      P.prefix_len[f] = (uint16_t)p->prefix_len[f];
    }
    P.suffix_off = p->suffix_off;
    P.suffix_len = p->suffix_len;
  } else if (p->output_kind == WARPJQ_OUT_AGG) {
    if (p->agg_path != 0xFFFFFFFFu) P.agg_slot = slot_of(p->agg_path);
    if (p->group_path != 0xFFFFFFFFu) P.group_slot = slot_of(p->group_path);
    if ((p->agg_path != 0xFFFFFFFFu && P.agg_slot < 0) ||
        (p->group_path != 0xFFFFFFFFu && P.group_slot < 0)) {
      set_err(err, err_len, "aggregate path has no slot");
      return WARPJQ_ERR_INVALID_ARG;
    }
  } else if (p->output_kind != WARPJQ_OUT_PASSTHROUGH) {
    set_err(err, err_len, "unknown output kind %u", p->output_kind);
    return WARPJQ_ERR_INVALID_ARG;
  }
  P.needs_rows = p->output_kind != WARPJQ_OUT_AGG;
  uint32_t nf = p->output_kind == WARPJQ_OUT_PROJECT ? p->n_fields
                : p->output_kind == WARPJQ_OUT_PATH  ? 1
                                                     : 0;
  P.rec_stride = (uint32_t)kRowRecBytes + 8 * nf;
  return WARPJQ_OK;
}


}  // namespace wjq
