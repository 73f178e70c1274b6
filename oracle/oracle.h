// TEST INFRASTRUCTURE -- the oracle.
//
// A CPU restatement of warpjq's own CPU engine (the reference project's Rust
// crate `warpjq-core`), used only as the checker for the GPU backend: by the
// tests under tests/, by __graft_entry__.smoke(), and as the timed CPU
// baseline in bench.py.  Nothing in the product links or calls this code.
//
// Each function cites the reference file:line it restates.  Paths are relative
// to the reference project root (crates/warpjq-core/src/...).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>
#include <map>
#include <memory>

namespace oracle {

// ---------------------------------------------------------------------------
// Query IR  (query/ir.rs:10-252)
// ---------------------------------------------------------------------------

using PathId = uint16_t;

struct Step {
  bool is_index = false;   // Step::Index vs Step::Key
  std::string key;         // decoded key bytes
  uint32_t index = 0;
  bool operator==(const Step &o) const {
    return is_index == o.is_index && key == o.key && index == o.index;
  }
};

struct Path {
  std::vector<Step> steps;
  bool operator==(const Path &o) const { return steps == o.steps; }
  std::string display() const;  // ir.rs:32-46
};

enum class CmpOp : uint8_t { Eq = 0, Ne = 1, Lt = 2, Le = 3, Gt = 4, Ge = 5 };

enum class LitKind : uint8_t { Null, False, True, Num, Str };
struct Literal {
  LitKind kind = LitKind::Null;
  double num = 0.0;
  std::string str;
  uint8_t rank() const;  // ir.rs:100-108
};

struct Cond {
  enum Tag : uint8_t { Cmp, Truthy, And, Or, Not } tag = Cmp;
  PathId path = 0;
  CmpOp op = CmpOp::Eq;
  Literal lit;
  std::unique_ptr<Cond> a, b;
  void visit_paths(std::vector<PathId> &out) const;  // ir.rs:128-137, dedup by caller
};

enum class AggKind : uint8_t { Count = 0, Sum = 1, Min = 2, Max = 3, Avg = 4 };
const char *agg_name(AggKind k);  // ir.rs:150-158

struct Output {
  enum Tag : uint8_t { Passthrough, PathOut, Project, Agg } tag = Passthrough;
  PathId path = 0;                                         // PathOut
  std::vector<std::pair<std::string, PathId>> fields;      // Project
  AggKind agg = AggKind::Count;                            // Agg
  bool has_arg = false;
  PathId arg = 0;
};

struct Program {
  std::vector<Path> paths;
  std::unique_ptr<Cond> filter;
  bool has_group = false;
  PathId group_by = 0;
  Output output;
  std::string source;
  bool is_aggregate() const { return output.tag == Output::Agg; }
  std::vector<PathId> required_paths() const;              // ir.rs:206-234
  bool csv_headers(std::vector<std::string> &cols) const;  // ir.rs:237-251
};

struct QueryError {
  size_t at = 0;
  std::string message;
  std::string hint;
  std::string render(const std::string &src) const;  // error.rs:36-49
};

// query/parse.rs:59.  Returns false and fills `err` on a query error.
bool parse_query(const std::string &src, Program &out, QueryError &err);

// Flat tables (query/mod.rs:39-198); only what the tests inspect.
struct FlatCmp { uint32_t path, op, lit_kind, lit_off, lit_len; double lit_num; };
struct FlatProgram {
  struct S { uint32_t kind, index, key_off, key_len, key_hash; };
  struct P { uint32_t step_off, step_count; };
  struct C { uint32_t op, arg; };
  std::vector<S> steps;
  std::vector<P> paths;
  std::vector<FlatCmp> cmps;
  std::vector<C> cond_rpn;
  std::vector<uint8_t> blob;
  uint32_t cond_stack_depth = 0;
};
uint32_t key_hash(const uint8_t *p, size_t n);  // query/mod.rs:15-22
FlatProgram flatten(const Program &p);           // query/mod.rs:95-198

// ---------------------------------------------------------------------------
// JSON scanner  (json.rs)
// ---------------------------------------------------------------------------

enum class Kind : uint8_t { Missing = 0, Null = 1, Bool = 2, Num = 3, Str = 4, Arr = 5, Obj = 6 };

struct Slot {
  Kind kind = Kind::Missing;
  const uint8_t *p = nullptr;  // raw bytes; for Str includes the quotes
  size_t n = 0;
  bool is_truthy() const;       // json.rs:63-65
  bool as_f64(double &v) const; // json.rs:73-78
};
Slot missing_slot();            // json.rs:56-59 (raw "null")

struct JsonError { size_t offset = 0; std::string detail; };

bool skip_value(const uint8_t *b, size_t len, size_t start, size_t &end, JsonError &e);  // json.rs:213
bool skip_string(const uint8_t *b, size_t len, size_t i, size_t &end, JsonError &e);     // json.rs:336
bool validate(const uint8_t *b, size_t len, JsonError &e);                              // json.rs:414

enum class LookupRes { Found, TypeError, Invalid };
LookupRes lookup(const uint8_t *line, size_t len, const std::vector<Step> &steps, Slot &out,
                 std::string &msg);                                                     // json.rs:444
bool unescape_into(const uint8_t *raw, size_t n, std::string &out);                      // json.rs:594
bool key_matches(const uint8_t *raw, size_t n, const std::string &decoded);              // json.rs:582
int compare(const Slot &s, const Literal &lit);                                           // json.rs:662
bool cmp_accepts(CmpOp op, int ord);                                                      // ir.rs:66-76

// ---------------------------------------------------------------------------
// Aggregation  (agg.rs)
// ---------------------------------------------------------------------------

struct AggState {
  uint64_t count = 0;
  uint64_t numeric = 0;
  double sum = 0.0;
  double min = 1.0 / 0.0;
  double max = -1.0 / 0.0;
  bool saw_non_numeric = false;
  void push_count() { count++; }
  void push_value(const Slot &s);          // agg.rs:50-60
  void push_number(double v);              // agg.rs:62-71
  void merge(const AggState &o);           // agg.rs:73-84
  bool finish(AggKind k, double &v) const; // agg.rs:88-97 (false = None)
};

struct GroupKey {
  uint8_t rank = 0;        // agg.rs:146-155
  std::string bytes;       // Num raw / Str decoded / Composite raw
  uint64_t bits = 0;       // Num: order_bits
  static GroupKey from_slot(const Slot &s);  // agg.rs:121-144
  std::string to_json() const;               // agg.rs:158-171
  std::string to_plain() const;              // agg.rs:174-179
  bool operator==(const GroupKey &o) const { return rank == o.rank && bytes == o.bytes; }
  bool operator<(const GroupKey &o) const;   // agg.rs:182-195 (total order)
};
uint64_t order_bits(double v);               // agg.rs:205-212

struct GroupKeyHash { size_t operator()(const GroupKey &k) const; };

std::string format_number(double v);        // agg.rs:253-278

// ---------------------------------------------------------------------------
// Output  (output.rs)
// ---------------------------------------------------------------------------

enum class Format : uint8_t { Ndjson = 0, Csv = 1, CountOnly = 2 };

void write_json_string(std::string &out, const uint8_t *p, size_t n);  // output.rs:24-42
void write_csv_cell(std::string &out, const uint8_t *p, size_t n);     // output.rs:45-61

enum class OnInvalid : uint8_t { Warn = 0, Skip = 1, Abort = 2 };

struct Options {
  Format format = Format::Ndjson;
  size_t chunk_bytes = 256u << 20;    // chunk.rs:18
  size_t max_line_bytes = 64u << 20;  // chunk.rs:22
  OnInvalid on_invalid = OnInvalid::Warn;
  size_t threads = 0;                 // 0 = all cores
};

struct RunStats {
  uint64_t bytes_in = 0;
  uint64_t lines_in = 0;
  uint64_t lines_out = 0;
  uint64_t malformed = 0;
  uint64_t type_errors = 0;
};

// Runs `program` over an in-memory buffer the way exec/cpu.rs:498 does
// (streamed chunks, newline-aligned slices processed in parallel, merged in
// order).  Returns 0 on success, 1 on a runtime error (message in `err`).
int run_bytes(const Program &program, const uint8_t *data, size_t len, const Options &opt,
              std::string &out, RunStats &stats, std::string &err);

}  // namespace oracle
