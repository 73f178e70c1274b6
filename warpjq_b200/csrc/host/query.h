// Host-side query front-end of the warpjq GPU backend: the jq-subset parser
// and the lowering to the flat warpjq_program tables.
//
// Restates the reference's crates/warpjq-core/src/query/{lex,parse,ir,mod}.rs
// and src/gpu/lower.rs, which the reference runs in Rust before calling the
// device ABI.  Query meaning must match the reference exactly, so the grammar,
// the error messages and the table layout follow those files; the code is
// this project's.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/warpjq_kernels.h"

namespace wjqh {

struct Step {
  bool is_index = false;
  std::string key;
  uint32_t index = 0;
  bool operator==(const Step &o) const {
    return is_index == o.is_index && key == o.key && index == o.index;
  }
};

struct Path {
  std::vector<Step> steps;
  bool operator==(const Path &o) const { return steps == o.steps; }
  std::string display() const;
};

enum class LitKind : uint8_t { Null = 0, False = 1, True = 2, Num = 3, Str = 4 };

struct Cond {
  enum Tag : uint8_t { Cmp, Truthy, And, Or, Not } tag = Cmp;
  uint16_t path = 0;
  uint32_t op = 0;
  LitKind lit = LitKind::Null;
  double num = 0;
  std::string str;
  std::unique_ptr<Cond> a, b;
};

enum class Out : uint8_t { Passthrough, Path, Project, Agg };

struct Program {
  std::vector<Path> paths;
  std::unique_ptr<Cond> filter;
  bool has_group = false;
  uint16_t group_by = 0;
  Out out = Out::Passthrough;
  uint16_t out_path = 0;
  std::vector<std::pair<std::string, uint16_t>> fields;
  uint32_t agg = WARPJQ_AGG_COUNT;
  bool has_arg = false;
  uint16_t arg = 0;
  std::string source;

  bool is_aggregate() const { return out == Out::Agg; }
  std::vector<uint16_t> required_paths() const;
  bool csv_headers(std::vector<std::string> &cols) const;
  std::string group_key_name() const;
};

struct QueryError {
  size_t at = 0;
  std::string message, hint;
  std::string render(const std::string &src) const;
};

bool parse(const std::string &src, Program &out, QueryError &err);

// Owns the flat tables a warpjq_program points into (gpu/lower.rs:17-35).
struct Lowered {
  std::vector<warpjq_step> steps;
  std::vector<warpjq_path> paths;
  std::vector<warpjq_cmp> cmps;
  std::vector<warpjq_cond_op> cond;
  std::vector<uint8_t> blob;
  std::vector<uint32_t> needed, slot_of_path, field_paths, prefix_off, prefix_len;
  warpjq_program prog{};
  void build(const Program &p, bool csv);
};

const char *agg_name(uint32_t k);

}  // namespace wjqh
