// The serving form: a request loop that takes solves of mixed sizes and
// precisions as they arrive and runs them with continuous batching.
//
// A scheduler thread owns the device work.  Requests are admitted against an
// HBM budget (one arena, allocated at creation, sub-allocated best-fit) and a
// cap on descriptor slots; an admitted request's field is copied into its
// arena buffer, and from then on every scheduling step carries it one pass
// further.  A step is, per precision, one persistent launch per pass kind
// present (the batch kernels of ff_batch_dev.cuh) over the tiles of every
// request at that pass, so requests that arrive while others run join the
// next step and their work shares the launches.  Axis tables (twiddles,
// digit reversals) stay resident per (length, precision); tile shapes are
// the tuned or default batch shapes, so a request's arithmetic is the same
// alone and in any mix.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "ff_batch.hpp"
#include "ff_status.hpp"

namespace ff {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Best-fit sub-allocator over one device region (offsets in 256-byte units
// of alignment).
struct Arena {
  size_t size = 0;
  std::map<size_t, size_t> free_;   // offset -> length
  size_t used = 0, peak = 0;

  void reset(size_t bytes) {
    size = bytes;
    free_.clear();
    free_[0] = bytes;
    used = peak = 0;
  }
  static size_t round(size_t b) { return (b + 255) & ~size_t(255); }
  bool alloc(size_t bytes, size_t *off) {
    bytes = round(bytes);
    auto best = free_.end();
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= bytes && (best == free_.end() || it->second < best->second)) best = it;
    if (best == free_.end()) return false;
    *off = best->first;
    const size_t rest = best->second - bytes;
    const size_t roff = best->first + bytes;
    free_.erase(best);
    if (rest) free_[roff] = rest;
    used += bytes;
    peak = std::max(peak, used);
    return true;
  }
  void release(size_t off, size_t bytes) {
    bytes = round(bytes);
    used -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

// kFetching: a finished request whose result ff_server_fetch is copying out;
// its buffers stay reserved until that copy has completed.
enum ReqState { kPending, kLoading, kRunning, kDone, kFetching };

struct Request {
  uint64_t id = 0;
  int n[3] = {0, 0, 0};
  int precision = FF_FP64;
  const void *f = nullptr;
  int f_on_host = 0;
  size_t bytes = 0;
  size_t off_d = 0, off_p = 0;
  int slot = -1;
  ReqState state = kPending;
  int next_pass = 0;         // passes already scheduled
  long finish_step = -1;     // step whose completion finishes the request
  bool desc_uploaded = false;
  cudaEvent_t src_ev = nullptr;   // the legacy default stream at submission (the input copy waits for it)
  cudaEvent_t in_ev = nullptr;
  Clock::time_point t_submit, t_admit, t_done;
  BatchGridHost g;
};

constexpr int kRing = 3;   // steps in flight per precision

// Per-precision launch state: descriptor table and the ring of step buffers.
struct Lane {
  int precision = FF_FP64;
  size_t dsz = 0;
  cudaStream_t stream = nullptr;
  // a step forks from `stream` into one stream per pass kind, so the kinds'
  // launches (independent requests) overlap, and joins back before its event
  cudaStream_t kstream[5] = {};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t kev[5] = {};
  void *desc = nullptr;                    // device descriptors [slots]
  unsigned char *desc_host = nullptr;      // pinned image
  CUtensorMap *maps = nullptr;             // device tensor maps [slots][2] (y, x boxes of the potential)
  CUtensorMap *maps_host = nullptr;        // pinned image
  std::vector<int> free_slots;
  // ring buffers: per step r and kind k: entries [slots] int2, starts [slots + 1] int, 5 tickets
  void *ring_dev = nullptr;
  unsigned char *ring_host = nullptr;
  size_t ring_bytes = 0;                   // one step's block
  cudaEvent_t ring_ev[kRing] = {};
  long ring_step[kRing] = {-1, -1, -1};    // step occupying each ring slot (-1: free)
  long next_step = 0;
  std::vector<uint64_t> step_members[kRing];
};

struct AxisEntry {
  void *mem = nullptr;
  AxisDev<double2> ad;
  AxisDev<float2> af;
};

}  // namespace
}  // namespace ff

using namespace ff;

struct ff_server {
  ff_server_config cfg{};
  int device = 0;
  int num_sms = 0;
  char *arena_base = nullptr;
  Arena arena;
  int *status = nullptr;
  cudaStream_t copy = nullptr, fetch = nullptr, setup = nullptr;
  Lane lane[2];
  std::map<std::tuple<int, int, int>, AxisEntry> axes;   // (n, precision, radix order)
  std::map<uint64_t, Request> reqs;
  std::deque<uint64_t> pending;
  std::vector<uint64_t> active;   // admitted, not yet done (loading or running)
  std::deque<uint64_t> finished;  // done, not yet claimed by ff_server_next
  bool admit_dirty = false;       // memory or slots freed, or requests arrived, since the last admission pass
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  int fatal = FF_OK;
  char fatal_msg[256] = {0};
  uint64_t next_id = 1;
  // statistics
  std::vector<double> lat_ms;
  uint64_t submitted = 0, completed = 0;
  double points_done = 0;
  Clock::time_point t_first, t_last;
  bool have_first = false;
  uint64_t steps = 0, launches = 0;
  int max_active_seen = 0;
};

namespace ff {
namespace {

size_t step_block_bytes(int slots) {
  auto r = [](size_t b) { return (b + 255) & ~size_t(255); };
  return 5 * (r(slots * sizeof(int2)) + r((slots + 1) * sizeof(int))) + r(5 * sizeof(int));
}

int lane_init(ff_server *s, Lane &L, int precision) {
  const int slots = s->cfg.max_active;
  L.precision = precision;
  L.dsz = precision == FF_FP64 ? batch_desc_size<double>() : batch_desc_size<float>();
  FF_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
  FF_CUDA(cudaEventCreateWithFlags(&L.fork_ev, cudaEventDisableTiming));
  for (int k = 0; k < 5; k++) {
    FF_CUDA(cudaStreamCreateWithFlags(&L.kstream[k], cudaStreamNonBlocking));
    FF_CUDA(cudaEventCreateWithFlags(&L.kev[k], cudaEventDisableTiming));
  }
  FF_CUDA(cudaMalloc(&L.desc, slots * L.dsz));
  FF_CUDA(cudaMallocHost((void **)&L.desc_host, slots * L.dsz));
  FF_CUDA(cudaMalloc((void **)&L.maps, (size_t)slots * 2 * sizeof(CUtensorMap)));
  FF_CUDA(cudaMallocHost((void **)&L.maps_host, (size_t)slots * 2 * sizeof(CUtensorMap)));
  L.ring_bytes = step_block_bytes(slots);
  FF_CUDA(cudaMalloc(&L.ring_dev, kRing * L.ring_bytes));
  FF_CUDA(cudaMallocHost((void **)&L.ring_host, kRing * L.ring_bytes));
  for (int r = 0; r < kRing; r++) FF_CUDA(cudaEventCreateWithFlags(&L.ring_ev[r], cudaEventDisableTiming));
  for (int q = slots - 1; q >= 0; q--) L.free_slots.push_back(q);
  for (int k = 0; k < 5; k++) {
    int per_sm = 0;
    int rc = precision == FF_FP64 ? batch_pass_prepare<double>(k, batch_budget(k), &per_sm)
                                  : batch_pass_prepare<float>(k, batch_budget(k), &per_sm);
    if (rc != FF_OK) return rc;
  }
  return FF_OK;
}

void lane_free(Lane &L) {
  for (int r = 0; r < kRing; r++)
    if (L.ring_ev[r]) cudaEventDestroy(L.ring_ev[r]);
  if (L.ring_host) cudaFreeHost(L.ring_host);
  if (L.ring_dev) cudaFree(L.ring_dev);
  if (L.desc_host) cudaFreeHost(L.desc_host);
  if (L.maps_host) cudaFreeHost(L.maps_host);
  if (L.maps) cudaFree(L.maps);
  if (L.desc) cudaFree(L.desc);
  for (int k = 0; k < 5; k++) {
    if (L.kev[k]) cudaEventDestroy(L.kev[k]);
    if (L.kstream[k]) cudaStreamDestroy(L.kstream[k]);
  }
  if (L.fork_ev) cudaEventDestroy(L.fork_ev);
  if (L.stream) cudaStreamDestroy(L.stream);
}

int axis_for(ff_server *s, int n, int precision, int order, AxisEntry **out) {
  auto key = std::make_tuple(n, precision, order);
  auto it = s->axes.find(key);
  if (it == s->axes.end()) {
    AxisEntry e;
    FF_CUDA(cudaMalloc(&e.mem, batch_axis_bytes(n, precision)));
    int rc = batch_axis_build(n, precision, order, e.mem, &e.ad, &e.af, s->setup);
    if (rc != FF_OK) {
      cudaFree(e.mem);
      return rc;
    }
    it = s->axes.emplace(key, e).first;
  }
  *out = &it->second;
  return FF_OK;
}

void fail(ff_server *s, int rc) {
  if (s->fatal == FF_OK) {
    s->fatal = rc;
    snprintf(s->fatal_msg, sizeof(s->fatal_msg), "%s", ff_last_error());
  }
}

// Admission of pending requests in arrival order; a request that does not
// fit now is passed over (later, smaller ones may fit) and retried when
// memory or slots are freed.  At most kAdmitWindow queued requests are
// examined per pass, so a long queue costs nothing while the budget is full.
constexpr int kAdmitWindow = 64;

int admit(ff_server *s) {
  int seen = 0;
  for (auto it = s->pending.begin(); it != s->pending.end() && seen < kAdmitWindow; seen++) {
    Request &q = s->reqs[*it];
    Lane &L = s->lane[q.precision == FF_FP64 ? 0 : 1];
    size_t od = 0, op = 0;
    if (L.free_slots.empty()) {
      ++it;
      continue;
    }
    if (!s->arena.alloc(q.bytes, &od)) {
      ++it;
      continue;
    }
    if (!s->arena.alloc(q.bytes, &op)) {
      s->arena.release(od, q.bytes);
      ++it;
      continue;
    }
    q.off_d = od;
    q.off_p = op;
    q.slot = L.free_slots.back();
    L.free_slots.pop_back();
    batch_grid_init(q.g, q.n, nullptr, nullptr, q.precision);
    for (int k = 0; k < 5; k++) q.g.shape[k] = batch_shape_for(q.precision, q.g, k);
    // axis d's tables in the radix order of the pass that owns it (z: 0, y: 1, x: 2)
    static const int owner[3] = {2, 1, 0};
    for (int d = 0; d < 3; d++) {
      AxisEntry *ax = nullptr;
      int rc = axis_for(s, q.n[d], q.precision, q.g.shape[owner[d]].order, &ax);
      if (rc != FF_OK) return rc;
      q.g.axd[d] = ax->ad;
      q.g.axf[d] = ax->af;
    }
    q.g.status = s->status;
    q.g.density = s->arena_base + q.off_d;
    q.g.potential = s->arena_base + q.off_p;
    const size_t esz = q.precision == FF_FP64 ? 8 : 4;
    const size_t fbytes = (size_t)q.n[0] * q.n[1] * q.n[2] * esz;
    // the copy stream does not synchronise with the legacy default stream:
    // the input copy waits explicitly for the work queued there before the
    // submission (a field produced by the caller on that stream)
    FF_CUDA(cudaStreamWaitEvent(s->copy, q.src_ev, 0));
    FF_CUDA(cudaMemcpyAsync(q.g.density, q.f, fbytes, q.f_on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            s->copy));
    if (!q.in_ev) FF_CUDA(cudaEventCreateWithFlags(&q.in_ev, cudaEventDisableTiming));
    FF_CUDA(cudaEventRecord(q.in_ev, s->copy));
    q.state = kLoading;
    q.t_admit = Clock::now();
    s->active.push_back(q.id);
    it = s->pending.erase(it);
  }
  return FF_OK;
}

// Builds and launches the next step of one precision lane; returns whether
// a step was issued.
int issue_step(ff_server *s, Lane &L, bool *issued) {
  *issued = false;
  int r = -1;
  for (int q = 0; q < kRing; q++)
    if (L.ring_step[q] < 0) {
      r = q;
      break;
    }
  if (r < 0) return FF_OK;
  std::vector<uint64_t> members;
  for (uint64_t id : s->active) {
    Request &q = s->reqs[id];
    if (q.state == kRunning && q.precision == L.precision && q.next_pass < 5) members.push_back(q.id);
  }
  if (members.empty()) return FF_OK;
  // compact layout of this step's work lists in ring block r: per kind the
  // entries (int2) and the prefix sums (int), then the five tickets
  int cnt[5] = {0, 0, 0, 0, 0};
  for (uint64_t id : members) cnt[s->reqs[id].next_pass]++;
  size_t e_off[5], s_off[5], off = 0;
  for (int k = 0; k < 5; k++) {
    e_off[k] = off;
    off += cnt[k] * sizeof(int2);
    s_off[k] = off;
    off += ((cnt[k] + 1) * sizeof(int) + 7) & ~size_t(7);
  }
  const size_t t_off = off;
  off += 5 * sizeof(int);
  unsigned char *hb = L.ring_host + (size_t)r * L.ring_bytes;
  char *db = static_cast<char *>(L.ring_dev) + (size_t)r * L.ring_bytes;
  int fill[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < 5; k++) reinterpret_cast<int *>(hb + s_off[k])[0] = 0;
  for (uint64_t id : members) {
    Request &q = s->reqs[id];
    if (!q.desc_uploaded) {
      unsigned char *img = L.desc_host + (size_t)q.slot * L.dsz;
      if (L.precision == FF_FP64) batch_desc_fill<double>(img, q.g);
      else batch_desc_fill<float>(img, q.g);
      FF_CUDA(cudaMemcpyAsync(static_cast<char *>(L.desc) + (size_t)q.slot * L.dsz, img, L.dsz,
                              cudaMemcpyHostToDevice, L.stream));
      CUtensorMap *mh = L.maps_host + 2 * (size_t)q.slot;
      const int rc = batch_grid_maps(q.g, q.precision, mh);
      if (rc != FF_OK) return rc;
      FF_CUDA(cudaMemcpyAsync(L.maps + 2 * (size_t)q.slot, mh, 2 * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                              L.stream));
      q.desc_uploaded = true;
    }
    const int k = q.next_pass;
    int *st = reinterpret_cast<int *>(hb + s_off[k]);
    reinterpret_cast<int2 *>(hb + e_off[k])[fill[k]] = make_int2(q.slot, k);
    st[fill[k] + 1] = st[fill[k]] + batch_tiles_of(q.g, k);
    fill[k]++;
    q.next_pass++;
    if (q.next_pass == 5) q.finish_step = L.next_step;
  }
  std::memset(hb + t_off, 0, 5 * sizeof(int));
  FF_CUDA(cudaMemcpyAsync(db, hb, off, cudaMemcpyHostToDevice, L.stream));
  FF_CUDA(cudaEventRecord(L.fork_ev, L.stream));
  for (int k = 0; k < 5; k++) {
    if (!cnt[k]) continue;
    const BatchWork wl{reinterpret_cast<const int2 *>(db + e_off[k]), reinterpret_cast<const int *>(db + s_off[k]),
                       cnt[k], reinterpret_cast<int *>(db + t_off) + k};
    const int tiles = reinterpret_cast<int *>(hb + s_off[k])[cnt[k]];
    const int blocks = std::max(1, std::min(tiles, batch_blocks_per_sm(k) * s->num_sms));
    cudaStream_t ks = L.kstream[k];
    FF_CUDA(cudaStreamWaitEvent(ks, L.fork_ev, 0));
    int rc = L.precision == FF_FP64 ? batch_pass_launch<double>(k, L.desc, L.maps, wl, blocks, batch_budget(k), ks)
                                    : batch_pass_launch<float>(k, L.desc, L.maps, wl, blocks, batch_budget(k), ks);
    if (rc != FF_OK) return rc;
    FF_CUDA(cudaEventRecord(L.kev[k], ks));
    FF_CUDA(cudaStreamWaitEvent(L.stream, L.kev[k], 0));
    s->launches++;
  }
  FF_CUDA(cudaEventRecord(L.ring_ev[r], L.stream));
  L.ring_step[r] = L.next_step++;
  L.step_members[r] = members;
  s->steps++;
  *issued = true;
  return FF_OK;
}

// Retires completed steps of a lane: members whose last pass ran in the step
// are done.
int retire_steps(ff_server *s, Lane &L, bool *progress) {
  for (;;) {
    int r = -1;
    long oldest = -1;
    for (int q = 0; q < kRing; q++)
      if (L.ring_step[q] >= 0 && (oldest < 0 || L.ring_step[q] < oldest)) {
        oldest = L.ring_step[q];
        r = q;
      }
    if (r < 0) return FF_OK;
    const cudaError_t e = cudaEventQuery(L.ring_ev[r]);
    if (e == cudaErrorNotReady) return FF_OK;
    if (e != cudaSuccess) FF_CUDA(e);
    const auto now = Clock::now();
    for (uint64_t id : L.step_members[r]) {
      auto it = s->reqs.find(id);
      if (it == s->reqs.end()) continue;
      Request &q = it->second;
      if (q.finish_step == oldest && q.state == kRunning) {
        s->active.erase(std::find(s->active.begin(), s->active.end(), id));
        q.state = kDone;
        q.t_done = now;
        s->finished.push_back(id);
        s->completed++;
        s->lat_ms.push_back(ms_between(q.t_submit, q.t_done));
        s->points_done += double(q.n[0]) * q.n[1] * q.n[2];
        s->t_last = now;
      }
    }
    L.step_members[r].clear();
    L.ring_step[r] = -1;
    *progress = true;
  }
}

void scheduler(ff_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    bool progress = false;
    int rc = FF_OK;
    for (int l = 0; l < 2 && rc == FF_OK; l++) rc = retire_steps(s, s->lane[l], &progress);
    if (progress) s->cv_done.notify_all();
    if (rc == FF_OK && !s->pending.empty() && s->admit_dirty) {
      s->admit_dirty = false;
      rc = admit(s);
    }
    if (rc == FF_OK) {
      for (uint64_t id : s->active) {
        Request &q = s->reqs[id];
        if (q.state != kLoading) continue;
        const cudaError_t e = cudaEventQuery(q.in_ev);
        if (e == cudaSuccess) {
          q.state = kRunning;
          progress = true;
        } else if (e != cudaErrorNotReady) {
          rc = set_error(FF_ERR_CUDA, "server input copy failed: %s", cudaGetErrorString(e));
          break;
        }
      }
    }
    for (int l = 0; l < 2 && rc == FF_OK; l++) {
      bool issued = false;
      rc = issue_step(s, s->lane[l], &issued);
      progress = progress || issued;
    }
    const bool busy = !s->active.empty();
    s->max_active_seen = std::max(s->max_active_seen, (int)s->active.size());
    if (rc != FF_OK) {
      fail(s, rc);
      s->cv_done.notify_all();
      break;
    }
    if (!progress) {
      // device work in flight: poll again shortly; idle: sleep until a submission
      if (busy) s->cv_work.wait_for(lk, std::chrono::microseconds(20));
      else s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
  }
}

}  // namespace
}  // namespace ff

// Frees a pending or finished request's buffers and slot and forgets it; the
// caller holds s->mu.
template <typename It> static void release_locked(ff_server *s, It it) {
  Request &q = it->second;
  if (q.state == kPending) {
    s->pending.erase(std::find(s->pending.begin(), s->pending.end(), q.id));
  } else {
    s->arena.release(q.off_d, q.bytes);
    s->arena.release(q.off_p, q.bytes);
    s->lane[q.precision == FF_FP64 ? 0 : 1].free_slots.push_back(q.slot);
    s->admit_dirty = true;
  }
  if (q.in_ev) cudaEventDestroy(q.in_ev);
  if (q.src_ev) cudaEventDestroy(q.src_ev);
  s->reqs.erase(it);
}

// Waits longer than this (about 31 years) are waits without limit; it keeps
// the deadline arithmetic in range for INFINITY and other huge values.
constexpr double kMaxTimeoutMs = 1e12;

extern "C" {

int ff_server_create(const ff_server_config *cfg, ff_server **out) {
  if (!cfg || !out) return set_error(FF_ERR_INVALID, "ff_server_create: null argument");
  *out = nullptr;
  if (cfg->hbm_budget < (1 << 20)) return set_error(FF_ERR_INVALID, "ff_server_create: budget below 1 MiB");
  if (cfg->max_active < 1 || cfg->max_active > (1 << 16))
    return set_error(FF_ERR_INVALID, "ff_server_create: max_active %d outside [1, 65536]", cfg->max_active);
  ff_server *s = new ff_server();
  s->cfg = *cfg;
  int rc = FF_OK;
  if (cudaGetDevice(&s->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess)
    rc = set_error(FF_ERR_CUDA, "ff_server_create: no current CUDA device");
  if (rc == FF_OK && cudaMalloc((void **)&s->arena_base, cfg->hbm_budget) != cudaSuccess) {
    cudaGetLastError();
    rc = set_error(FF_ERR_NOMEM, "ff_server_create: cannot reserve the HBM budget of %zu bytes", cfg->hbm_budget);
  }
  if (rc == FF_OK) {
    s->arena.reset(cfg->hbm_budget);
    if (cudaMalloc((void **)&s->status, sizeof(int)) != cudaSuccess || cudaMemset(s->status, 0, sizeof(int)) ||
        cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->fetch, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->setup, cudaStreamNonBlocking) != cudaSuccess)
      rc = set_error(FF_ERR_CUDA, "ff_server_create: streams");
  }
  if (rc == FF_OK) rc = lane_init(s, s->lane[0], FF_FP64);
  if (rc == FF_OK) rc = lane_init(s, s->lane[1], FF_FP32);
  if (rc != FF_OK) {
    ff_server_destroy(s);
    return rc;
  }
  s->worker = std::thread(scheduler, s);
  *out = s;
  return FF_OK;
}

int ff_server_submit(ff_server *s, const int n[3], int precision, const void *f, int f_on_host, uint64_t *id) {
  if (!s || !n || !f || !id) return set_error(FF_ERR_INVALID, "ff_server_submit: null argument");
  if (precision != FF_FP64 && precision != FF_FP32)
    return set_error(FF_ERR_INVALID, "ff_server_submit: precision %d", precision);
  int rc = batch_check_dims(n, nullptr, nullptr, "ff_server_submit", 0);
  if (rc != FF_OK) return rc;
  Request q;
  batch_grid_init(q.g, n, nullptr, nullptr, precision);
  q.bytes = batch_grid_bytes(q.g, precision);
  if (2 * Arena::round(q.bytes) > s->cfg.hbm_budget)
    return set_error(FF_ERR_NOMEM, "ff_server_submit: request needs %zu bytes, budget %zu", 2 * q.bytes,
                     s->cfg.hbm_budget);
  for (int d = 0; d < 3; d++) q.n[d] = n[d];
  q.precision = precision;
  q.f = f;
  q.f_on_host = f_on_host;
  // mark the legacy default stream of the server's device: the input copy is
  // ordered after the work the caller queued there before this call
  {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    cudaError_t e = cudaEventCreateWithFlags(&q.src_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(q.src_ev, 0);
    if (prev >= 0 && prev != s->device) cudaSetDevice(prev);
    if (e != cudaSuccess) {
      if (q.src_ev) cudaEventDestroy(q.src_ev);
      return set_error(FF_ERR_CUDA, "ff_server_submit: %s", cudaGetErrorString(e));
    }
  }
  q.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal != FF_OK) {
      cudaEventDestroy(q.src_ev);
      return set_error(s->fatal, "ff_server_submit: server stopped: %s", s->fatal_msg);
    }
    q.id = s->next_id++;
    *id = q.id;
    if (!s->have_first) {
      s->t_first = q.t_submit;
      s->have_first = true;
    }
    s->submitted++;
    s->reqs.emplace(q.id, q);
    s->pending.push_back(q.id);
    s->admit_dirty = true;
  }
  s->cv_work.notify_one();
  return FF_OK;
}

int ff_server_wait(ff_server *s, uint64_t id, double timeout_ms, ff_request_info *info) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_server_wait: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  const bool bounded = timeout_ms >= 0 && timeout_ms < kMaxTimeoutMs;
  const auto deadline = Clock::now() + std::chrono::microseconds(bounded ? (long long)(timeout_ms * 1000.0) : 0);
  for (;;) {
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(FF_ERR_INVALID, "ff_server_wait: unknown request %llu",
                                              (unsigned long long)id);
    const Request &q = it->second;
    if (q.state == kDone) {
      if (info) {
        info->latency_ms = ms_between(q.t_submit, q.t_done);
        info->queue_ms = ms_between(q.t_submit, q.t_admit);
        info->run_ms = ms_between(q.t_admit, q.t_done);
      }
      return FF_OK;
    }
    if (s->fatal != FF_OK) return set_error(s->fatal, "ff_server_wait: server stopped: %s", s->fatal_msg);
    if (bounded && Clock::now() >= deadline)
      return set_error(FF_ERR_TIMEOUT, "ff_server_wait: request %llu not done", (unsigned long long)id);
    if (bounded) s->cv_done.wait_until(lk, deadline);
    else s->cv_done.wait(lk);
  }
}

int ff_server_next(ff_server *s, double timeout_ms, uint64_t *id, ff_request_info *info) {
  if (!s || !id) return set_error(FF_ERR_INVALID, "ff_server_next: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  const bool bounded = timeout_ms >= 0 && timeout_ms < kMaxTimeoutMs;
  const auto deadline = Clock::now() + std::chrono::microseconds(bounded ? (long long)(timeout_ms * 1000.0) : 0);
  for (;;) {
    while (!s->finished.empty()) {
      const uint64_t q = s->finished.front();
      s->finished.pop_front();
      auto it = s->reqs.find(q);
      if (it == s->reqs.end()) continue;   // already released
      *id = q;
      if (info) {
        const Request &r = it->second;
        info->latency_ms = ms_between(r.t_submit, r.t_done);
        info->queue_ms = ms_between(r.t_submit, r.t_admit);
        info->run_ms = ms_between(r.t_admit, r.t_done);
      }
      return FF_OK;
    }
    if (s->fatal != FF_OK) return set_error(s->fatal, "ff_server_next: server stopped: %s", s->fatal_msg);
    if (bounded && Clock::now() >= deadline)
      return set_error(FF_ERR_TIMEOUT, "ff_server_next: no request finished");
    if (bounded) s->cv_done.wait_until(lk, deadline);
    else s->cv_done.wait(lk);
  }
}

int ff_server_fetch(ff_server *s, uint64_t id, void *phi, int phi_on_host) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_server_fetch: null server");
  void *src = nullptr;
  size_t bytes = 0;
  {
    // claim the request: a concurrent fetch or release of the same id is
    // refused until the copy below has finished, so its buffers cannot be
    // handed to another request while they are being read
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(FF_ERR_INVALID, "ff_server_fetch: unknown request");
    if (it->second.state == kFetching)
      return set_error(FF_ERR_INVALID, "ff_server_fetch: request %llu is being fetched by another call",
                       (unsigned long long)id);
    if (it->second.state != kDone) return set_error(FF_ERR_INVALID, "ff_server_fetch: request not done");
    Request &q = it->second;
    q.state = kFetching;
    src = q.g.potential;
    bytes = (size_t)q.n[0] * q.n[1] * q.n[2] * (q.precision == FF_FP64 ? 8 : 4);
  }
  cudaError_t e = cudaSuccess;
  if (phi) {
    e = cudaMemcpyAsync(phi, src, bytes, phi_on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s->fetch);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->fetch);
  }
  {
    // the claim ends: the request is released in the same critical section,
    // so no other call can see it between the copy and the release
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it != s->reqs.end()) release_locked(s, it);
  }
  s->cv_work.notify_one();
  if (e != cudaSuccess)
    return set_error(FF_ERR_CUDA, "ff_server_fetch: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e));
  return FF_OK;
}

int ff_server_release(ff_server *s, uint64_t id) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_server_release: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return set_error(FF_ERR_INVALID, "ff_server_release: unknown request");
  Request &q = it->second;
  if (q.state == kFetching)
    return set_error(FF_ERR_INVALID, "ff_server_release: request %llu is being fetched", (unsigned long long)id);
  if (q.state != kDone && q.state != kPending)
    return set_error(FF_ERR_INVALID, "ff_server_release: request %llu is on the device", (unsigned long long)id);
  release_locked(s, it);
  s->cv_work.notify_one();
  return FF_OK;
}

int ff_server_stats(ff_server *s, ff_server_report *st) {
  if (!s || !st) return set_error(FF_ERR_INVALID, "ff_server_stats: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof(*st));
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->steps = s->steps;
  st->launches = s->launches;
  st->peak_bytes = s->arena.peak;
  st->budget_bytes = s->cfg.hbm_budget;
  st->max_active = s->max_active_seen;
  if (!s->lat_ms.empty()) {
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = v.back();
    double sum = 0;
    for (double x : v) sum += x;
    st->mean_ms = sum / v.size();
    const double span = ms_between(s->t_first, s->t_last) * 1e-3;
    if (span > 0) {
      st->solves_per_s = s->completed / span;
      st->points_per_s = s->points_done / span;
    }
  }
  return FF_OK;
}

int ff_server_reset_stats(ff_server *s) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_server_reset_stats: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat_ms.clear();
  s->submitted = s->completed = 0;
  s->points_done = 0;
  s->have_first = false;
  s->steps = s->launches = 0;
  s->max_active_seen = 0;
  s->arena.peak = s->arena.used;
  return FF_OK;
}

int ff_server_check(ff_server *s) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_server_check: null server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal != FF_OK) return set_error(s->fatal, "server stopped: %s", s->fatal_msg);
  }
  int h = 0;
  FF_CUDA(cudaMemcpyAsync(&h, s->status, sizeof(int), cudaMemcpyDeviceToHost, s->fetch));
  FF_CUDA(cudaStreamSynchronize(s->fetch));
  if (h != kDevOk) {
    FF_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), s->fetch));
    FF_CUDA(cudaStreamSynchronize(s->fetch));
    return set_error(FF_ERR_TIMEOUT, "a served request's bulk copy did not complete within its wait limit");
  }
  return FF_OK;
}

int ff_server_destroy(ff_server *s) {
  if (!s) return FF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (int l = 0; l < 2; l++)
    if (s->lane[l].stream) cudaStreamSynchronize(s->lane[l].stream);
  if (s->copy) cudaStreamSynchronize(s->copy);
  for (auto &kv : s->reqs) {
    if (kv.second.in_ev) cudaEventDestroy(kv.second.in_ev);
    if (kv.second.src_ev) cudaEventDestroy(kv.second.src_ev);
  }
  for (auto &kv : s->axes) cudaFree(kv.second.mem);
  for (int l = 0; l < 2; l++) lane_free(s->lane[l]);
  if (s->copy) cudaStreamDestroy(s->copy);
  if (s->fetch) cudaStreamDestroy(s->fetch);
  if (s->setup) cudaStreamDestroy(s->setup);
  if (s->status) cudaFree(s->status);
  if (s->arena_base) cudaFree(s->arena_base);
  delete s;
  return FF_OK;
}

}  // extern "C"
