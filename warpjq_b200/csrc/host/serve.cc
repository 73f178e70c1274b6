// The resident serving loop behind include/warpjq_serve.h.
//
// No reference counterpart: the reference CLI runs one query per process
// (crates/warpjq-cli/src/run.rs:16-96) and pays the device context's set-up
// each time.  Here a server owns, per slot, a CUDA stream, one query (and so
// one device context and compiled plan) per served query, a driver context
// for mixed batches, a device arena for inputs that are not usable in place,
// and page-locked buffers for row output; all of it lives as long as the
// server.  CSV requests are converted to NDJSON on the device by a converter
// thread (its own converter and stream) before they join the queue.  One
// loop thread runs the slots: it completes slots whose event has fired, then
// gives each free slot the longest prefix of the waiting requests that fits
// the memory budget beside what is in flight, so requests that arrive while
// others run are admitted as slots and memory free up and the slots' work
// overlaps on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/warpjq_serve.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

void put_err(char *err, size_t n, const std::string &s) {
  if (!err || !n) return;
  snprintf(err, n, "%s", s.c_str());
}

// Device bytes a request may hold while in flight: its NDJSON (CSV grows by
// at most 2x when converted), row output up to 1.25x, and a fixed part for
// tables.
uint64_t footprint(uint64_t n, uint32_t flags) {
  const uint64_t nd = (flags & WARPJQ_SERVE_CSV) ? 2 * n : n;
  return nd + nd + nd / 4 + (1ull << 20);
}

struct Req {
  uint64_t id = 0;
  uint32_t query = 0;
  const uint8_t *data = nullptr;
  uint64_t len = 0;
  uint32_t flags = 0;
  uint64_t fp = 0;
  Clock::time_point t_arrive, t_admit;
  uint64_t addr = 0;  // device address of the request's NDJSON in the slot
  uint64_t nd = 0;    // its length
  uint8_t *owned = nullptr;  // CSV converted ahead of admission: its NDJSON (freed at completion)
};

// A device buffer that grows stream-ordered (the slot's stream), keeping
// `keep` bytes of its contents.
struct DevBuf {
  uint8_t *p = nullptr;
  uint64_t cap = 0;
  bool reserve(uint64_t need, uint64_t keep, cudaStream_t st) {
    if (need <= cap) return true;
    const uint64_t ncap = std::max<uint64_t>(need + need / 2, 1ull << 20);
    uint8_t *np = nullptr;
    if (cudaMallocAsync((void **)&np, ncap, st) != cudaSuccess) return false;
    if (keep && p) cudaMemcpyAsync(np, p, keep, cudaMemcpyDeviceToDevice, st);
    if (p) cudaFreeAsync(p, st);
    p = np;
    cap = ncap;
    return true;
  }
  void release(cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
  }
};

// Page-locked host buffer that grows (its contents are not kept).
struct PinBuf {
  uint8_t *p = nullptr;
  uint64_t cap = 0;
  bool reserve(uint64_t need) {
    if (need <= cap) return true;
    if (p) cudaFreeHost(p);
    const uint64_t ncap = std::max<uint64_t>(need + need / 4, 1ull << 16);
    p = nullptr;
    cap = 0;
    if (cudaMallocHost((void **)&p, ncap) != cudaSuccess) return false;
    cap = ncap;
    return true;
  }
  ~PinBuf() {
    if (p) cudaFreeHost(p);
  }
};

struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<warpjq_query *> qs;  // one per served query
  warpjq_query *driver = nullptr;  // runs mixed batches
  warpjq_csv *conv = nullptr;
  DevBuf arena;
  PinBuf rows, row_off;
  std::vector<Req> reqs;
  std::vector<std::vector<size_t>> by_q;  // request indexes per query
  std::vector<size_t> mixed;              // request indexes of the mixed batch
  uint64_t fp = 0;
  bool busy = false;
};

}  // namespace

struct warpjq_server {
  std::vector<std::string> queries;
  warpjq_serve_config cfg{};
  int device = 0;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_loop, cv_done;
  std::deque<Req> waiting;
  std::deque<warpjq_serve_result> done;
  uint64_t in_flight_bytes = 0;  // footprints of admitted requests (loop thread only)
  uint64_t on_device = 0;        // admitted, not yet completed (guarded by mu)
  uint64_t next_id = 1;
  bool stop = false;
  std::thread loop;
  // CSV requests are converted by a thread of their own, on its own stream,
  // before they join the waiting queue, so the loop never waits on the
  // converter's host synchronisations
  std::deque<Req> to_convert;
  uint64_t converting = 0;  // taken by the converter, not yet queued
  std::condition_variable cv_conv;
  static constexpr int kConverters = 2;  // conversions overlap: each waits on its own kernels
  warpjq_csv *conv[kConverters] = {nullptr, nullptr};
  cudaStream_t conv_st[kConverters] = {nullptr, nullptr};
  std::thread converter[kConverters];
};

namespace {

warpjq_serve_result fail_result(const Req &r, const std::string &why) {
  warpjq_serve_result x;
  memset(&x, 0, sizeof x);
  x.id = r.id;
  x.query = r.query;
  x.rc = 1;
  put_err(x.err, sizeof x.err, why);
  x.latency_ms = ms_between(r.t_arrive, Clock::now());
  return x;
}

// Group keys of a collected batch, gathered from device memory into one
// host buffer; the groups' key_off values (device addresses) are rewritten
// to offsets into it.
bool gather_keys(Slot &s, const warpjq_device_result &all, std::vector<warpjq_group_ext> &groups,
                 std::vector<uint8_t> &keys, std::string &why) {
  groups.assign(all.groups, all.groups + all.n_groups);
  keys.assign(1, 0);
  if (groups.empty()) return true;
  std::vector<uint64_t> offs(groups.size());
  std::vector<uint32_t> lens(groups.size());
  uint64_t total = 0;
  for (size_t i = 0; i < groups.size(); i++) {
    offs[i] = groups[i].key_off;
    lens[i] = groups[i].key_len;
    groups[i].key_off = total;
    total += groups[i].key_len;
  }
  keys.assign(total + 1, 0);
  char e[256] = {0};
  if (warpjq_csv_gather(s.conv, nullptr, offs.data(), lens.data(), groups.size(), keys.data(), s.st, e,
                        sizeof e) != WARPJQ_OK) {
    why = std::string("gathering group keys: ") + e;
    return false;
  }
  return true;
}

// Renders every item of a collected batch with query q, appending one
// result per request (reqs[idx[i]] owns items[i]).
void render(warpjq_server *S, Slot &s, warpjq_query *q, const std::vector<warpjq_batch_item> &items,
            const std::vector<size_t> &idx, const warpjq_device_result &all,
            const std::vector<warpjq_group_ext> &groups, const std::vector<uint8_t> &keys,
            const uint8_t *rows, const uint64_t *row_off, std::vector<warpjq_serve_result> &out) {
  char *body = nullptr;
  size_t body_len = 0;
  std::vector<uint64_t> offs(items.size() + 1);
  const int rc = warpjq_query_render_batch(q, items.data(), (uint32_t)items.size(),
                                           groups.empty() ? nullptr : groups.data(), keys.data(), rows, row_off,
                                           &body, &body_len, offs.data());
  (void)all;
  const auto now = Clock::now();
  for (size_t i = 0; i < items.size(); i++) {
    const Req &r = s.reqs[idx[i]];
    if (rc) {
      out.push_back(fail_result(r, "rendering the output failed"));
      continue;
    }
    warpjq_serve_result x;
    memset(&x, 0, sizeof x);
    x.id = r.id;
    x.query = r.query;
    const uint64_t n = offs[i + 1] - offs[i];
    x.out = (char *)malloc(n + 1);
    if (!x.out) {
      out.push_back(fail_result(r, "out of host memory"));
      continue;
    }
    memcpy(x.out, body + offs[i], n);
    x.out_len = n;
    x.n_lines = items[i].n_lines - items[i].n_blank;
    x.n_invalid = items[i].n_invalid;
    x.queue_ms = ms_between(r.t_arrive, r.t_admit);
    x.latency_ms = ms_between(r.t_arrive, now);
    out.push_back(x);
  }
  free(body);
  (void)S;
}

// Collects one batch of context `ctx` (rendered by q, or per item by its own
// query for a mixed batch) and renders its requests' outputs.
void complete_batch(warpjq_server *S, Slot &s, warpjq_ctx *ctx, warpjq_query *q, const std::vector<size_t> &idx,
                    bool mixed, std::vector<warpjq_serve_result> &out) {
  std::vector<warpjq_batch_item> items(idx.size());
  warpjq_device_result all;
  memset(&all, 0, sizeof all);
  char e[512] = {0};
  std::string why;
  if (warpjq_batch_collect(ctx, items.data(), &all, e, sizeof e) != WARPJQ_OK) {
    why = std::string("CUDA error: ") + e;
  }
  std::vector<warpjq_group_ext> groups;
  std::vector<uint8_t> keys;
  const uint8_t *rows = nullptr;
  const uint64_t *row_off = nullptr;
  if (why.empty() && !gather_keys(s, all, groups, keys, why)) {
  }
  if (why.empty() && all.n_selected && all.d_out_bytes) {
    const uint64_t rb = std::max<uint64_t>(all.out_len, 1), ob = (all.n_selected + 1) * 8;
    if (!s.rows.reserve(rb) || !s.row_off.reserve(ob)) {
      why = "out of page-locked host memory for rows";
    } else {
      cudaMemcpyAsync(s.rows.p, all.d_out_bytes, all.out_len, cudaMemcpyDeviceToHost, s.st);
      cudaMemcpyAsync(s.row_off.p, all.d_out_row_off, ob, cudaMemcpyDeviceToHost, s.st);
      if (cudaStreamSynchronize(s.st) != cudaSuccess) why = "copying rows to the host failed";
      rows = s.rows.p;
      row_off = (const uint64_t *)s.row_off.p;
    }
  }
  if (!why.empty()) {
    for (size_t i : idx) out.push_back(fail_result(s.reqs[i], why));
    return;
  }
  if (!mixed) {
    render(S, s, q, items, idx, all, groups, keys, rows, row_off, out);
    return;
  }
  // a mixed batch: each request rendered by its own query, in groups of one
  // query (the items keep their group ranges into the batch's groups)
  std::vector<std::vector<size_t>> pos(S->queries.size());
  for (size_t i = 0; i < idx.size(); i++) pos[s.reqs[idx[i]].query].push_back(i);
  for (size_t qi = 0; qi < pos.size(); qi++) {
    if (pos[qi].empty()) continue;
    std::vector<warpjq_batch_item> sub;
    std::vector<size_t> sub_idx;
    for (size_t i : pos[qi]) {
      sub.push_back(items[i]);
      sub_idx.push_back(idx[i]);
    }
    render(S, s, s.qs[qi], sub, sub_idx, all, groups, keys, rows, row_off, out);
  }
}

void complete_slot(warpjq_server *S, Slot &s) {
  std::vector<warpjq_serve_result> out;
  // the requests this slot launched (those that failed at admission were
  // completed and counted off then, though they stay in s.reqs)
  size_t launched = s.mixed.size();
  for (auto &v : s.by_q) launched += v.size();
  if (!s.mixed.empty()) complete_batch(S, s, warpjq_query_ctx(s.driver), s.driver, s.mixed, true, out);
  for (size_t qi = 0; qi < s.by_q.size(); qi++)
    if (!s.by_q[qi].empty()) complete_batch(S, s, warpjq_query_ctx(s.qs[qi]), s.qs[qi], s.by_q[qi], false, out);
  S->in_flight_bytes -= s.fp;
  for (auto &r : s.reqs)
    if (r.owned) cudaFreeAsync(r.owned, s.st);  // after every use on this stream
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (auto &x : out) S->done.push_back(x);
    S->on_device -= launched;
  }
  S->cv_done.notify_all();
  s.reqs.clear();
  s.mixed.clear();
  for (auto &v : s.by_q) v.clear();
  s.fp = 0;
  s.busy = false;
}

// Places every request's NDJSON at a 16-byte aligned device address and
// launches the slot's batches.  Requests that fail here complete at once.
void admit(warpjq_server *S, Slot &s, std::vector<Req> take) {
  const auto now = Clock::now();
  const size_t n_take = take.size();  // counted on the device by the caller
  std::vector<warpjq_serve_result> failed;
  s.reqs.clear();
  // arena room for host inputs, unaligned device inputs and converted CSV
  uint64_t room = 16;
  for (auto &r : take) {
    r.t_admit = now;
    const bool dev = r.flags & WARPJQ_SERVE_DEVICE;
    if (!r.owned && (!dev || (uintptr_t)r.data % 16)) room += r.len + 16;
  }
  if (!s.arena.reserve(room, 0, s.st)) {
    for (auto &r : take) {
      failed.push_back(fail_result(r, "out of device memory for the request's input"));
      if (r.owned) cudaFreeAsync(r.owned, s.st);
    }
    take.clear();
  }
  uint64_t pos = 0;
  for (auto &r : take) {
    const bool dev = r.flags & WARPJQ_SERVE_DEVICE;
    std::string why;
    if (r.owned) {
      // CSV, converted by the converter thread: addr and nd are set
    } else if (dev && (uintptr_t)r.data % 16 == 0) {
      r.addr = (uint64_t)(uintptr_t)r.data;
      r.nd = r.len;
    } else {
      pos = (pos + 15) & ~15ull;
      if (r.len &&
          cudaMemcpyAsync(s.arena.p + pos, r.data, r.len, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                          s.st) != cudaSuccess)
        why = "copying the input to the device failed";
      r.addr = (uint64_t)(uintptr_t)(s.arena.p + pos);
      r.nd = r.len;
      pos += r.len;
    }
    if (!why.empty()) {
      failed.push_back(fail_result(r, why));
      if (r.owned) cudaFreeAsync(r.owned, s.st);
    } else {
      s.reqs.push_back(r);
    }
  }
  // batches: a slot's requests of several queries as one mixed batch (each
  // input with its own plan) from mixed_min requests on, else one batch per query
  s.by_q.assign(S->queries.size(), {});
  s.mixed.clear();
  for (size_t i = 0; i < s.reqs.size(); i++) s.by_q[s.reqs[i].query].push_back(i);
  if (S->cfg.mixed_min) {
    size_t n_q = 0;
    for (auto &v : s.by_q) n_q += !v.empty();
    if (n_q > 1 && s.reqs.size() >= S->cfg.mixed_min)
      for (auto &v : s.by_q) {
        s.mixed.insert(s.mixed.end(), v.begin(), v.end());
        v.clear();
      }
  }
  auto launch_failed = [&](const std::vector<size_t> &idx, const char *e) {
    for (size_t i : idx) failed.push_back(fail_result(s.reqs[i], std::string("CUDA error: ") + e));
  };
  std::vector<size_t> launched_none;
  if (!s.mixed.empty()) {
    std::vector<uint64_t> offs, lens;
    std::vector<warpjq_ctx *> ctxs;
    for (size_t i : s.mixed) {
      offs.push_back(s.reqs[i].addr);
      lens.push_back(s.reqs[i].nd);
      ctxs.push_back(warpjq_query_ctx(s.qs[s.reqs[i].query]));
    }
    char e[512] = {0};
    if (warpjq_batch_launch_mixed(warpjq_query_ctx(s.driver), ctxs.data(), nullptr, offs.data(), lens.data(),
                                  (uint32_t)offs.size(), s.st, e, sizeof e) != WARPJQ_OK) {
      launch_failed(s.mixed, e);
      s.mixed.clear();
    }
  }
  for (size_t qi = 0; qi < s.by_q.size(); qi++) {
    auto &idx = s.by_q[qi];
    if (idx.empty()) continue;
    std::vector<uint64_t> offs, lens;
    for (size_t i : idx) {
      offs.push_back(s.reqs[i].addr);
      lens.push_back(s.reqs[i].nd);
    }
    char e[512] = {0};
    if (warpjq_batch_launch(warpjq_query_ctx(s.qs[qi]), nullptr, offs.data(), lens.data(), (uint32_t)idx.size(),
                            s.st, e, sizeof e) != WARPJQ_OK) {
      launch_failed(idx, e);
      idx.clear();
    }
  }
  cudaEventRecord(s.ev, s.st);
  size_t launched = s.mixed.size();
  for (auto &v : s.by_q) launched += v.size();
  s.fp = 0;
  for (size_t i : s.mixed) s.fp += s.reqs[i].fp;
  for (auto &v : s.by_q)
    for (size_t i : v) s.fp += s.reqs[i].fp;
  S->in_flight_bytes += s.fp;
  s.busy = launched > 0;
  if (!s.busy)
    for (auto &r : s.reqs)
      if (r.owned) cudaFreeAsync(r.owned, s.st);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (auto &x : failed) S->done.push_back(x);
    S->on_device -= n_take - launched;
  }
  if (!failed.empty()) S->cv_done.notify_all();
}

// The converter thread: CSV requests in arrival order, each converted on the
// device into a buffer of its own and then queued for admission as NDJSON
// (a request that fails to convert completes with its error).
void converter_main(warpjq_server *S, int ci) {
  warpjq_csv *conv = S->conv[ci];
  cudaStream_t cst = S->conv_st[ci];
  cudaSetDevice(S->device);
  for (;;) {
    Req r;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_conv.wait(lk, [&] { return S->stop || !S->to_convert.empty(); });
      if (S->stop) break;
      r = S->to_convert.front();
      S->to_convert.pop_front();
      S->converting++;
    }
    std::string why;
    const uint8_t *d = nullptr;
    uint64_t nd = 0, consumed = 0, recs = 0;
    char e[512] = {0};
    warpjq_csv_reset(conv);
    const uint32_t fl = WARPJQ_CSV_FINAL | ((r.flags & WARPJQ_SERVE_DEVICE) ? 0u : WARPJQ_CSV_HOST_INPUT);
    if (warpjq_csv_convert(conv, r.data, r.len, fl, cst, &d, &nd, &consumed, &recs, e, sizeof e) !=
        WARPJQ_OK) {
      why = std::string("CSV conversion failed: ") + e;
    } else if (cudaMallocAsync((void **)&r.owned, nd + 16, cst) != cudaSuccess) {
      r.owned = nullptr;
      why = "out of device memory for the converted CSV";
    } else {
      if (nd) cudaMemcpyAsync(r.owned, d, nd, cudaMemcpyDeviceToDevice, cst);
      if (cudaStreamSynchronize(cst) != cudaSuccess) why = "CUDA error converting CSV";
      r.addr = (uint64_t)(uintptr_t)r.owned;
      r.nd = nd;
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->converting--;
      if (why.empty()) {
        S->waiting.push_back(r);
      } else {
        if (r.owned) cudaFreeAsync(r.owned, cst);
        S->done.push_back(fail_result(r, why));
      }
    }
    S->cv_loop.notify_one();
    S->cv_done.notify_all();
  }
}

void loop_main(warpjq_server *S) {
  cudaSetDevice(S->device);
  for (;;) {
    bool progress = false;
    for (auto &s : S->slots)
      if (s.busy && cudaEventQuery(s.ev) != cudaErrorNotReady) {
        complete_slot(S, s);
        progress = true;
      }
    for (auto &s : S->slots) {
      if (s.busy) continue;
      std::vector<Req> take;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        uint64_t total = 0;
        uint64_t bytes = 0;
        while (!S->waiting.empty()) {
          const Req &r = S->waiting.front();
          if (S->in_flight_bytes + total + r.fp > S->cfg.budget_bytes) break;
          if (S->cfg.max_batch && take.size() >= S->cfg.max_batch) break;
          if (!take.empty() && bytes + r.len > S->cfg.slot_bytes) break;
          bytes += r.len;
          total += r.fp;
          take.push_back(r);
          S->waiting.pop_front();
        }
        S->on_device += take.size();
      }
      if (!take.empty()) {
        admit(S, s, std::move(take));
        progress = true;
      }
    }
    bool any_busy = false;
    for (auto &s : S->slots) any_busy |= s.busy;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->stop && !any_busy) break;
    if (progress) continue;
    if (any_busy) {
      // a slot is on the device: look again shortly (new arrivals wake us)
      S->cv_loop.wait_for(lk, std::chrono::microseconds(50));
    } else {
      S->cv_loop.wait(lk, [&] { return S->stop || !S->waiting.empty(); });
      if (S->stop) break;
    }
  }
}

}  // namespace

extern "C" {

int warpjq_serve_open(const char *const *queries, uint32_t n_queries, const warpjq_serve_config *cfg,
                      warpjq_server **out, char *err, size_t err_len) {
  *out = nullptr;
  if (!n_queries) {
    put_err(err, err_len, "a server needs at least one query");
    return 1;
  }
  auto *S = new warpjq_server();
  if (cfg) S->cfg = *cfg;
  if (!S->cfg.n_slots) S->cfg.n_slots = 3;
  if (!S->cfg.budget_bytes) S->cfg.budget_bytes = 120ull << 30;
  if (!S->cfg.chunk_bytes) S->cfg.chunk_bytes = 1ull << 20;
  if (!S->cfg.slot_bytes) S->cfg.slot_bytes = 1ull << 30;
  cudaGetDevice(&S->device);
  for (uint32_t i = 0; i < n_queries; i++) S->queries.push_back(queries[i]);
  S->slots.resize(S->cfg.n_slots);
  auto fail = [&](int rc, const std::string &why) {
    put_err(err, err_len, why);
    warpjq_serve_close(S);
    return rc;
  };
  for (auto &s : S->slots) {
    if (cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming) != cudaSuccess)
      return fail(1, "CUDA error: creating a slot's stream");
    for (auto &q : S->queries) {
      warpjq_query *h = nullptr;
      char e[1024] = {0};
      const int rc = warpjq_query_open(q.c_str(), S->cfg.format, S->cfg.chunk_bytes, &h, e, sizeof e);
      if (rc) return fail(rc, e);
      s.qs.push_back(h);
    }
    char e[1024] = {0};
    if (warpjq_query_open("count", S->cfg.format, S->cfg.chunk_bytes, &s.driver, e, sizeof e))
      return fail(1, e);
    if (warpjq_csv_create(&s.conv) != WARPJQ_OK) return fail(1, "CUDA error: creating a CSV converter");
  }
  // the converter's stream at the highest priority: its kernels are short
  // and the converter thread waits on each of them, so they go ahead of the
  // slots' queued scans
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  for (int c = 0; c < warpjq_server::kConverters; c++)
    if (warpjq_csv_create(&S->conv[c]) != WARPJQ_OK ||
        cudaStreamCreateWithPriority(&S->conv_st[c], cudaStreamNonBlocking, prio_hi) != cudaSuccess)
      return fail(1, "CUDA error: creating a CSV converter");
  S->loop = std::thread(loop_main, S);
  for (int c = 0; c < warpjq_server::kConverters; c++) S->converter[c] = std::thread(converter_main, S, c);
  *out = S;
  return 0;
}

int warpjq_serve_warm(warpjq_server *S, uint64_t reserve_bytes, char *err, size_t err_len) {
  // blank lines (spaces, a newline every 4 KiB) and one line with every
  // kind of result, run by every slot's every query on the slot's stream
  if (reserve_bytes < 4096) reserve_bytes = 4096;
  std::vector<uint8_t> h(reserve_bytes, ' ');
  for (uint64_t i = 4095; i < reserve_bytes; i += 4096) h[i] = '\n';
  uint8_t *d = nullptr;
  if (cudaMalloc((void **)&d, reserve_bytes + 16) != cudaSuccess) {
    put_err(err, err_len, "CUDA error: out of device memory for warming");
    return 1;
  }
  cudaMemcpy(d, h.data(), reserve_bytes, cudaMemcpyHostToDevice);
  // CSV of about a quarter of the reserve: the converter's buffers grow to
  // what inputs that large need
  std::string rows = "a,b\n";
  const uint64_t csv_target = std::max<uint64_t>(reserve_bytes / 4, 1u << 16);
  rows.reserve(csv_target + 16);
  while (rows.size() < csv_target) rows += "\"x\",1\n";
  uint8_t *dc = nullptr;
  cudaMalloc((void **)&dc, rows.size() + 16);
  cudaMemcpy(dc, rows.data(), rows.size(), cudaMemcpyHostToDevice);
  int rc = 0;
  {
    // the loop thread must not touch the slots meanwhile: warm before the
    // first request only
    std::lock_guard<std::mutex> lk(S->mu);
    for (auto &s : S->slots) {
      for (auto *q : s.qs) {
        const uint64_t off = (uint64_t)(uintptr_t)d, len = reserve_bytes;
        char e[512] = {0};
        std::vector<warpjq_batch_item> it(1);
        warpjq_device_result all;
        if (warpjq_batch_launch(warpjq_query_ctx(q), nullptr, &off, &len, 1, s.st, e, sizeof e) != WARPJQ_OK ||
            warpjq_batch_collect(warpjq_query_ctx(q), it.data(), &all, e, sizeof e) != WARPJQ_OK) {
          put_err(err, err_len, std::string("CUDA error: ") + e);
          rc = 1;
        }
      }

      // room for host inputs and converted CSV of the reserve's size, and
      // page-locked room for a quarter of it in rows
      s.arena.reserve(reserve_bytes + reserve_bytes / 2, 0, s.st);
      s.rows.reserve(reserve_bytes / 4);
      s.row_off.reserve(reserve_bytes / 32);
      cudaStreamSynchronize(s.st);
    }
  }
  {
    // the converter thread's converter (idle: no request has arrived yet)
    const uint8_t *o = nullptr;
    uint64_t nd, consumed, recs;
    char e[512] = {0};
    for (int c = 0; c < warpjq_server::kConverters; c++) {
      warpjq_csv_reset(S->conv[c]);
      if (warpjq_csv_convert(S->conv[c], dc, rows.size(), WARPJQ_CSV_FINAL, S->conv_st[c], &o, &nd, &consumed,
                             &recs, e, sizeof e) != WARPJQ_OK) {
        put_err(err, err_len, std::string("CUDA error: ") + e);
        rc = 1;
      }
      cudaStreamSynchronize(S->conv_st[c]);
    }
  }
  cudaFree(d);
  cudaFree(dc);
  return rc;
}

int warpjq_serve_enqueue(warpjq_server *S, uint32_t query, const uint8_t *data, uint64_t len, uint32_t flags,
                         uint64_t *id, char *err, size_t err_len) {
  if (query >= S->queries.size()) {
    put_err(err, err_len, "no such query in this server");
    return 1;
  }
  if (len && !data) {
    put_err(err, err_len, "null input");
    return 1;
  }
  Req r;
  r.query = query;
  r.data = data;
  r.len = len;
  r.flags = flags;
  r.fp = footprint(len, flags);
  r.t_arrive = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    r.id = S->next_id++;
    if (id) *id = r.id;
    if (r.fp > S->cfg.budget_bytes) {
      S->done.push_back(fail_result(
          r, "request of " + std::to_string(len) + " bytes needs " + std::to_string(r.fp) +
                 " bytes of device memory, over the budget"));
      S->cv_done.notify_all();
      return 0;
    }
    if (flags & WARPJQ_SERVE_CSV) S->to_convert.push_back(r);
    else S->waiting.push_back(r);
  }
  if (flags & WARPJQ_SERVE_CSV) S->cv_conv.notify_one();
  else S->cv_loop.notify_one();
  return 0;
}

uint32_t warpjq_serve_poll(warpjq_server *S, warpjq_serve_result *done, uint32_t max_done, int timeout_ms) {
  std::unique_lock<std::mutex> lk(S->mu);
  auto ready = [&] {
    return !S->done.empty() ||
           (S->waiting.empty() && S->on_device == 0 && S->to_convert.empty() && S->converting == 0);
  };
  if (timeout_ms < 0) S->cv_done.wait(lk, ready);
  else if (timeout_ms > 0) S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
  uint32_t n = 0;
  while (n < max_done && !S->done.empty()) {
    done[n++] = S->done.front();
    S->done.pop_front();
  }
  return n;
}

uint64_t warpjq_serve_pending(warpjq_server *S) {
  std::lock_guard<std::mutex> lk(S->mu);
  return S->to_convert.size() + S->converting + S->waiting.size() + S->on_device + S->done.size();
}

void warpjq_serve_close(warpjq_server *S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    for (auto &r : S->waiting)
      if (r.owned) cudaFreeAsync(r.owned, S->conv_st[0]);
    S->waiting.clear();
    S->to_convert.clear();
  }
  S->cv_loop.notify_all();
  S->cv_conv.notify_all();
  if (S->loop.joinable()) S->loop.join();
  for (auto &t : S->converter)
    if (t.joinable()) t.join();
  // a conversion that finished while the threads stopped queued its request
  for (auto &r : S->waiting)
    if (r.owned) cudaFreeAsync(r.owned, S->conv_st[0]);
  S->waiting.clear();
  for (int c = 0; c < warpjq_server::kConverters; c++) {
    if (S->conv[c]) warpjq_csv_destroy(S->conv[c]);
    if (S->conv_st[c]) {
      cudaStreamSynchronize(S->conv_st[c]);
      cudaStreamDestroy(S->conv_st[c]);
    }
  }
  for (auto &x : S->done) free(x.out);
  for (auto &s : S->slots) {
    if (s.st) cudaStreamSynchronize(s.st);
    for (auto *q : s.qs) warpjq_query_close(q);
    if (s.driver) warpjq_query_close(s.driver);
    if (s.conv) warpjq_csv_destroy(s.conv);
    if (s.st) s.arena.release(s.st);
    if (s.st) cudaStreamSynchronize(s.st);
    if (s.ev) cudaEventDestroy(s.ev);
    if (s.st) cudaStreamDestroy(s.st);
  }
  delete S;
}

}  // extern "C"
