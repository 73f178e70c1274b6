// An aggregate scan that allocates no device memory.
//
// Some callers cannot call cudaMalloc.  A database or stream engine that
// hands the whole device memory to its own pool allocator at start-up leaves
// nothing for a library to allocate behind its back, and cudaMalloc may
// synchronise the device, which a caller in the middle of a latency-critical
// stream schedule cannot afford.  For them, warpjq_aggregate_noalloc runs the
// ungrouped-aggregate variant of the scan (count / sum / min / max / avg,
// with or without a select()) using only:
//   - the input and the result struct, both in device memory the caller owns;
//   - a fixed scratch array in this file (g_noalloc_scratch, about 10 MiB),
//     which every GPU that loads the library holds until the process exits.
//
// Limits and caveats:
//   - input of at most kNoAllocMaxInput bytes (4 GiB); larger inputs are
//     rejected with WARPJQ_ERR_INVALID_ARG;
//   - lines nesting deeper than kNoAllocDeepLevels + 64 levels cannot be
//     decided in the fixed deep-nesting stack; the result then reports
//     status = 1 and its counts must not be used;
//   - every call shares the one scratch array, which keeps the previous
//     call's contents.  Calls whose work overlaps on the GPU (different
//     streams, or different host threads without ordering) race on it; order
//     them on one stream;
//   - the first call on each device performs set-up (it looks up the array's
//     device address and the kernel's occupancy); make that first call
//     before any stream capture.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/warpjq_ext.h"
#include "../../include/warpjq_kernels.h"

// The kernels are included with internal linkage so this file's
// instantiation of the scan kernel is its own.
namespace {
#include "kernels.cuh"
#include "plan_build.h"
}  // namespace

using namespace wjq;

namespace {

constexpr uint64_t kNoAllocMaxInput = 4ull << 30;
constexpr uint32_t kNoAllocTile = 16384;
constexpr uint32_t kNoAllocHalo = 2048;
constexpr uint64_t kNoAllocMaxTiles = kNoAllocMaxInput / kNoAllocTile;
constexpr uint32_t kNoAllocMaxGrid = 2048;
constexpr uint64_t kNoAllocDeepLevels = 1u << 14;  // per CTA, beyond the 64 in registers
constexpr unsigned kNoAllocReduceBlocks = 256;

constexpr uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }
constexpr uint64_t kOffCtr = 0;
constexpr uint64_t kOffTiles = align256(kOffCtr + sizeof(RunCounters));
constexpr uint64_t kOffBlockLines = align256(kOffTiles + kNoAllocMaxTiles * sizeof(TileDesc));
constexpr uint64_t kOffDeep =
    align256(kOffBlockLines + 2 * kNoAllocReduceBlocks * sizeof(unsigned long long));
constexpr uint64_t kScratchBytes =
    align256(kOffDeep + kNoAllocMaxGrid * (kNoAllocDeepLevels / 32) * sizeof(uint32_t));

}  // namespace

// The scratch.  In host code this name is only a stand-in for the symbol: its
// device address comes from cudaGetSymbolAddress in noalloc_setup().
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct DeviceSetup {
  bool done = false;
  unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
  unsigned grid = 0;
  size_t smem = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

// Once per device, with that device current.
warpjq_status noalloc_setup(int dev, DeviceSetup *&out, char *err, size_t err_len) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceSetup &s = g_setup[dev];
  if (!s.done) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_err(err, err_len, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
      return WARPJQ_ERR_CUDA;
    }
    size_t smem = scan_smem_bytes(kNoAllocTile, kNoAllocHalo, false);  // grouped queries are rejected
    e = cudaFuncSetAttribute(k_scan<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      set_err(err, err_len, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
      return WARPJQ_ERR_CUDA;
    }
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan<false>, kThreads, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
      set_err(err, err_len, "occupancy query: %s", cudaGetErrorString(e));
      return WARPJQ_ERR_CUDA;
    }
    unsigned grid = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
    s.grid = grid < kNoAllocMaxGrid ? grid : kNoAllocMaxGrid;
    s.scratch = (unsigned char *)ptr;
    s.smem = smem;
    s.done = true;
  }
  out = &s;
  return WARPJQ_OK;
}

__global__ void k_noalloc_reset(RunCounters *ctr) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    RunCounters z;
    memset(&z, 0, sizeof(z));
    z.first_invalid_tile = ~0ull;
    z.first_type_tile = ~0ull;
    z.agg_min_bits = ~0ull;
    z.first_invalid = ~0ull;
    z.first_type_error = ~0ull;
    *ctr = z;
  }
}

__global__ void k_noalloc_result(const RunCounters *ctr, warpjq_noalloc_result *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const RunCounters &c = *ctr;
  warpjq_noalloc_result r;
  memset(&r, 0, sizeof(r));
  r.n_lines = c.n_lines;
  r.n_blank = c.n_blank;
  r.n_invalid = c.n_invalid;
  r.n_type_error = c.n_type_error;
  r.n_selected = c.n_selected;
  r.first_invalid = c.first_invalid;
  r.count = c.agg_count;
  r.numeric = c.agg_numeric;
  r.isum_lo = c.agg_isum_lo;
  r.isum_hi = c.agg_isum_hi;
  r.n_int = c.agg_n_int;
  r.fsum = c.fsum_total;  // exact sums rounded once (fixsum.cuh)
  r.min = c.agg_numeric ? min_of_bits(c.agg_min_bits) : __builtin_huge_val();
  r.max = c.agg_numeric ? max_of_bits(c.agg_max_bits) : -__builtin_huge_val();
  r.sum = c.sum_total;
  r.saw_non_numeric = c.agg_saw_non_numeric;
  r.status = (c.overflow || c.error) ? 1u : 0u;
  *out = r;
}

}  // namespace

extern "C" warpjq_status warpjq_aggregate_noalloc(const warpjq_program *prog, const uint8_t *d_data,
                                                  uint64_t n_bytes, void *stream,
                                                  warpjq_noalloc_result *d_result, char *err,
                                                  size_t err_len) {
  if (!prog || !d_result || (!d_data && n_bytes)) {
    set_err(err, err_len, "null program, input or result");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (n_bytes > kNoAllocMaxInput) {
    set_err(err, err_len, "input of %llu bytes exceeds the %llu-byte limit of the no-allocation scan",
            (unsigned long long)n_bytes, (unsigned long long)kNoAllocMaxInput);
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (((uintptr_t)d_data & 15u) != 0) {
    set_err(err, err_len, "device input must be 16-byte aligned");
    return WARPJQ_ERR_INVALID_ARG;
  }
  if (prog->output_kind != WARPJQ_OUT_AGG || prog->group_path != 0xFFFFFFFFu) {
    set_err(err, err_len, "the no-allocation scan runs ungrouped aggregate queries only");
    return WARPJQ_ERR_INVALID_ARG;
  }
  DevPlan plan;
  warpjq_status rc = build_plan(prog, plan, err, err_len);
  if (rc != WARPJQ_OK) return rc;

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_err(err, err_len, "cudaGetDevice: %s", cudaGetErrorString(e));
    return WARPJQ_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_err(err, err_len, "device %d is beyond the %d devices the no-allocation scan sets up", dev,
            kMaxDevices);
    return WARPJQ_ERR_INVALID_ARG;
  }
  DeviceSetup *s = nullptr;
  rc = noalloc_setup(dev, s, err, err_len);
  if (rc != WARPJQ_OK) return rc;

  cudaStream_t st = (cudaStream_t)stream;
  unsigned char *base = s->scratch;
  RunCounters *ctr = (RunCounters *)(base + kOffCtr);
  TileDesc *tiles = (TileDesc *)(base + kOffTiles);
  unsigned long long *block_lines = (unsigned long long *)(base + kOffBlockLines);
  uint32_t *deep = (uint32_t *)(base + kOffDeep);

  // Each launch's own status is checked (cudaLaunchKernel returns it), so an
  // earlier, unrelated error of the caller is neither reported nor cleared.
  {
    void *args[] = {&ctr};
    e = cudaLaunchKernel((const void *)k_noalloc_reset, dim3(1), dim3(32), args, 0, st);
  }
  unsigned long long n_tiles = (n_bytes + kNoAllocTile - 1) / kNoAllocTile;
  if (n_bytes > 0) {
    ScanParams sp;
    memset(&sp, 0, sizeof(sp));
    sp.data = d_data;
    sp.n = n_bytes;
    sp.tile_bytes = kNoAllocTile;
    sp.halo_bytes = kNoAllocHalo;
    sp.n_tiles = n_tiles;
    sp.ctr = ctr;
    sp.tiles = tiles;
    sp.deep_words = deep;
    sp.deep_levels_per_cta = kNoAllocDeepLevels;
    unsigned grid = (unsigned)(n_tiles < s->grid ? n_tiles : s->grid);
    if (e == cudaSuccess) {
      void *args[] = {&sp, &plan};
      e = cudaLaunchKernel((const void *)k_scan<false>, dim3(grid), dim3(kThreads), args, s->smem, st);
    }
    if (e == cudaSuccess) {
      unsigned nb = kNoAllocReduceBlocks;
      void *args[] = {&n_tiles, &tiles, &ctr, &block_lines};
      e = cudaLaunchKernel((const void *)k_reduce_tiles, dim3(nb), dim3(kReduceThreads), args, 0, st);
    }
    if (e == cudaSuccess) {
      unsigned nb = kNoAllocReduceBlocks;
      void *args[] = {&block_lines, &nb, &tiles, &ctr};
      e = cudaLaunchKernel((const void *)k_finalize, dim3(1), dim3(32), args, 0, st);
    }
  }
  if (e == cudaSuccess) {
    void *args[] = {&ctr, &d_result};
    e = cudaLaunchKernel((const void *)k_noalloc_result, dim3(1), dim3(32), args, 0, st);
  }
  if (e != cudaSuccess) {
    set_err(err, err_len, "launch: %s", cudaGetErrorString(e));
    return WARPJQ_ERR_CUDA;
  }
  return WARPJQ_OK;
}
