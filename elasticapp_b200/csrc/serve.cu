// Serving: continuous batching of rod-assembly simulations on one GPU.
//
// Requests (a set of straight rods, a time step, a horizon, gravity, clamp
// and damper options) arrive at any time.  The server owns a device pool of
// bins, each 520 slots (one CTA of the resident step kernels), sized from an
// HBM budget at creation.  A request is admitted when enough bins are free:
// its rods are packed into its own bins (next fit; a rod of 520 to 1039
// elements takes a pair of adjacent bins, run by a cluster of two CTAs),
// initialised on the host and copied in, and its initial energy is computed
// on the device.  Every tick is one launch of the resident kernel per
// precision (mixed, and FP64 for requests that fell back) over the bins of
// every active request: each CTA reads its bin, step count, time step and
// environment from a per-CTA table, so requests of different sizes, time
// steps and horizons share the launch.  The launch is always a cluster
// launch, pairs and single bins alike, so a request's arithmetic does not
// depend on whether long rods run beside it.  A request advances steps_per_launch steps per tick, counted from
// its own admission, so its result does not depend on what else is running.
//
// Retirement needs no host round trip: the host knows from the step counts
// which requests finish in a tick; right after that tick's launch it enqueues,
// on the same stream, their final energies and a copy of their state into a
// pinned host arena, records an event and returns their bins to the free list
// (stream order keeps the copy ahead of any later reuse).  eb_server_poll
// checks the events without blocking.  A mixed-precision result whose
// mechanical energy (kinetic, elastic and gravitational) grew by more than
// the tolerance, or is not finite, is run again in FP64 from its initial
// conditions.  At most two ticks are in flight.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <set>
#include <memory>
#include <string>
#include <vector>

#include "../../include/elastica_b200.h"
#include "eb_host.h"
#include "eb_internal.h"

namespace eb {
cudaError_t launch_rod_block_mixed_serve(const StepArgs& args, const ServeCta* serve, int n_ctas, int n_steps,
                                         bool damped, cudaStream_t stream);
cudaError_t launch_rod_block_fp64_serve(const StepArgs& args, const ServeCta* serve, int n_ctas, int n_steps,
                                        bool damped, cudaStream_t stream);
cudaError_t launch_rod_energy_list(int64_t n_rods, int64_t stride, const int64_t* start, const int32_t* n_el,
                                   const double* state, const double* params, const double gravity[3], double* out,
                                   cudaStream_t stream);
}  // namespace eb

namespace {

constexpr int64_t kBin = 520;                 // slots per bin (one CTA)
constexpr int64_t kPairSlots = 2 * kBin;      // a rod longer than a bin: two adjacent bins (a CTA pair)
// Packing fills a bin to at most 512 slots and a bin pair to 1024: the
// serving CTAs run 512 threads, and one slot more gives some threads a
// second round in every phase.  A single rod longer than that fills its unit
// alone.
constexpr int64_t kBinFill = 512;
constexpr int64_t kPairFill = 2 * kBinFill;
constexpr int64_t kRodsPerBin = kBin / 3;     // a rod takes at least 3 slots
constexpr size_t kArenaBytes = size_t(1) << 30;  // pinned result arena
constexpr size_t kUploadBytes = size_t(1) << 28;  // pinned staging of admitted requests' initial data
using Clock = std::chrono::steady_clock;

eb_status fail(eb_status st, const std::string& m) {
  eb::set_last_error(m);
  return st;
}

#define SV_CUDA(call)                                                                             \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(EB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// first-fit allocator of contiguous id ranges
struct RangeAlloc {
  std::map<int64_t, int64_t> free_;  // start -> length
  void init(int64_t cap) {
    free_.clear();
    if (cap > 0) free_[0] = cap;
  }
  int64_t alloc(int64_t n) {
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= n) {
        const int64_t s = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[s + n] = len - n;
        return s;
      }
    return -1;
  }
  void release(int64_t s, int64_t n) {
    auto it = free_.emplace(s, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && s + n == nx->first) {
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

// Bins and bin pairs: a pair is bins 2k and 2k + 1 (adjacent slot ranges).
// Free bins are kept as whole free pairs and as single bins whose buddy is in
// use; a single comes from the latter when there is one, else by splitting a
// pair, and a released bin rejoins its buddy when that is free.
struct BinPool {
  std::set<int64_t> pairs;   // even b with b and b + 1 free
  std::set<int64_t> halves;  // free b whose buddy is in use
  void init(int64_t n_bins) {
    pairs.clear();
    halves.clear();
    for (int64_t b = 0; b + 1 < n_bins; b += 2) pairs.insert(b);
  }
  int64_t free_bins() const { return static_cast<int64_t>(halves.size() + 2 * pairs.size()); }
  bool fits(int64_t n_pairs, int64_t n_singles) const {
    const int64_t p = static_cast<int64_t>(pairs.size());
    return n_pairs <= p && n_singles <= static_cast<int64_t>(halves.size()) + 2 * (p - n_pairs);
  }
  int64_t take_pair() {
    const int64_t b = *pairs.begin();
    pairs.erase(pairs.begin());
    return b;
  }
  int64_t take_single() {
    if (!halves.empty()) {
      const int64_t b = *halves.begin();
      halves.erase(halves.begin());
      return b;
    }
    const int64_t b = take_pair();
    halves.insert(b + 1);
    return b;
  }
  void give_pair(int64_t b) { pairs.insert(b); }
  void give_single(int64_t b) {
    auto it = halves.find(b ^ 1);
    if (it != halves.end()) {
      halves.erase(it);
      pairs.insert(b & ~int64_t(1));
    } else {
      halves.insert(b);
    }
  }
};

// FIFO ring of pinned host memory (allocations are freed in order)
struct Ring {
  unsigned char* base = nullptr;
  size_t cap = 0, head = 0, tail = 0, used = 0;
  std::deque<std::pair<size_t, size_t>> live;  // (offset, bytes incl. wrap padding)
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) / 256 * 256;
    if (bytes > cap) return false;
    size_t pad = 0;
    if (head + bytes > cap) pad = cap - head;  // wrap
    if (used + pad + bytes > cap) return false;
    if (pad) {
      head = 0;
      used += pad;
    }
    *off = head;
    live.emplace_back(head, bytes + pad);
    head = (head + bytes) % cap;
    used += bytes;
    return true;
  }
  void free_oldest() {
    if (live.empty()) return;
    used -= live.front().second;
    live.pop_front();
    if (live.empty()) head = tail = used = 0;
  }
};

enum ReqState { kQueued = 0, kActive = 1, kFinishing = 2, kDone = 3 };

struct Request {
  int64_t id = 0;
  std::vector<eb_straight_rod> rods;
  std::vector<double> velocities;  // concatenated per rod 3 x (n + 1), or empty
  double dt = 0.0;
  int64_t n_steps = 0;
  double gravity[3] = {0.0, 0.0, 0.0};
  uint32_t options = 0;
  double nu_t = 0.0, nu_r = 0.0;
  int precision = EB_PRECISION_MIXED;
  bool fell_back = false;
  bool damped = false;
  Clock::time_point t_submit;
  double latency_s = 0.0;
  double queued_s = -1.0;  // submission to first admission; < 0 until admitted
  ReqState state = kQueued;
  // placement: units of one bin, or of a bin pair holding one long rod
  std::vector<int64_t> bins;        // first bin of each unit
  std::vector<int32_t> bin_count;   // slots used in each unit
  std::vector<uint8_t> bin_pair;    // 1: the unit is a bin pair
  std::vector<int64_t> rod_bin, rod_off;  // bin and slot offset inside it, per rod
  int64_t rod0 = -1;
  int64_t elements = 0;
  int64_t steps_done = 0;
  // completion
  cudaEvent_t event = nullptr;
  size_t arena_off = 0;
  double e0 = 0.0, e1 = 0.0, escale = 0.0;
  std::vector<double> result;  // per rod, kStateFields rows of n + 1 slots
  std::vector<int64_t> result_off;
};

}  // namespace

struct eb_server {
  eb_server_config cfg{};
  cudaStream_t stream = nullptr;
  int64_t n_bins = 0, n_slots = 0, stride = 0, rod_cap = 0;
  double* state[2] = {nullptr, nullptr};
  double* par = nullptr;
  uint32_t* meta = nullptr;
  eb::RodInfo* rods = nullptr;
  int64_t* rod_start = nullptr;
  int32_t* rod_n = nullptr;
  double* e0 = nullptr;
  double* e1 = nullptr;
  uint32_t* status = nullptr;
  eb::ServeCta* d_cta[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [parity][precision]
  eb::ServeCta* h_cta[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  cudaEvent_t tick_event[2] = {nullptr, nullptr};
  bool tick_pending[2] = {false, false};
  // timing of each parity's step launches, summed when the tick is done
  cudaEvent_t launch_t0[2] = {nullptr, nullptr}, launch_t1[2] = {nullptr, nullptr};
  bool launch_timed[2] = {false, false};
  double kernel_seconds = 0.0;
  int cur = 0;
  int64_t ticks = 0;
  Ring arena;
  // pinned staging of initial data: copies from pageable memory would wait
  // for the stream (the running ticks) before each admission
  Ring upload;
  std::deque<cudaEvent_t> upload_events;  // one per live upload allocation, in order
  std::vector<cudaEvent_t> spare_events;
  BinPool bins;
  RangeAlloc rod_ids;
  int64_t next_id = 1;
  std::map<int64_t, std::unique_ptr<Request>> requests;
  std::deque<Request*> queue;
  std::vector<Request*> active;
  std::deque<Request*> finishing;
  std::deque<eb_completion> completed;
  int64_t n_completed = 0, n_fallbacks = 0;
  double element_steps = 0.0;
};

namespace {

void server_free(eb_server* s) {
  cudaSetDevice(s->cfg.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  void* dev[] = {s->state[0], s->state[1], s->par, s->meta, s->rods, s->rod_start, s->rod_n, s->e0, s->e1, s->status};
  for (void* p : dev)
    if (p) cudaFree(p);
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      if (s->d_cta[a][b]) cudaFree(s->d_cta[a][b]);
      if (s->h_cta[a][b]) cudaFreeHost(s->h_cta[a][b]);
    }
  for (auto& kv : s->requests)
    if (kv.second->event) cudaEventDestroy(kv.second->event);
  for (auto& e : s->tick_event)
    if (e) cudaEventDestroy(e);
  for (int p = 0; p < 2; ++p) {
    if (s->launch_t0[p]) cudaEventDestroy(s->launch_t0[p]);
    if (s->launch_t1[p]) cudaEventDestroy(s->launch_t1[p]);
  }
  if (s->arena.base) cudaFreeHost(s->arena.base);
  if (s->upload.base) cudaFreeHost(s->upload.base);
  for (cudaEvent_t e : s->upload_events) cudaEventDestroy(e);
  for (cudaEvent_t e : s->spare_events) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
}

// Placement units of the request, best fit decreasing: rods in order of
// decreasing length; a rod longer than a bin opens a bin pair (1040 slots,
// run by a CTA pair, which may split any rod of the unit); a shorter rod goes
// to the unit with the least room (below the fill limits above) that still
// holds it, else opens a single bin.
void pack(Request& r) {
  r.bins.clear();
  r.bin_count.clear();
  r.bin_pair.clear();
  r.rod_bin.assign(r.rods.size(), 0);
  r.rod_off.assign(r.rods.size(), 0);
  std::vector<size_t> order(r.rods.size());
  for (size_t k = 0; k < order.size(); ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return r.rods[a].n_elements > r.rods[b].n_elements; });
  std::multimap<int64_t, int64_t> room;  // free slots -> unit
  for (size_t k : order) {
    const int64_t w = r.rods[k].n_elements + 1;
    int64_t u = -1;
    if (w <= kBinFill) {
      auto it = room.lower_bound(w);
      if (it != room.end()) {
        u = it->second;
        room.erase(it);
      }
    }
    if (u < 0) {
      u = static_cast<int64_t>(r.bin_count.size());
      r.bin_count.push_back(0);
      r.bin_pair.push_back(w > kBin ? 1 : 0);
    }
    r.rod_bin[k] = u;
    r.rod_off[k] = r.bin_count[u];
    r.bin_count[u] += static_cast<int32_t>(w);
    const int64_t left = (r.bin_pair[u] ? kPairFill : kBinFill) - r.bin_count[u];
    if (left >= 3) room.emplace(left, u);  // a rod takes at least 3 slots
  }
}

void unit_counts(const Request& r, int64_t* n_pairs, int64_t* n_singles) {
  *n_pairs = 0;
  for (uint8_t p : r.bin_pair) *n_pairs += p;
  *n_singles = static_cast<int64_t>(r.bin_pair.size()) - *n_pairs;
}

uint32_t request_flags(const Request& r) {
  uint32_t f = 0;
  if (r.options & EB_REQUEST_GRAVITY) f |= eb::kSimGravity;
  if (r.options & EB_REQUEST_CLAMP) f |= eb::kSimClamp;
  if (r.options & EB_REQUEST_DAMPER) f |= eb::kSimDamper;
  return f;
}

// Space in the pinned staging ring: take back the staging of uploads that
// have landed, and wait for the oldest one while the ring is full.
eb_status upload_alloc(eb_server* s, size_t bytes, size_t* off) {
  auto take_oldest = [&]() {
    s->spare_events.push_back(s->upload_events.front());
    s->upload_events.pop_front();
    s->upload.free_oldest();
  };
  while (!s->upload_events.empty()) {
    const cudaError_t q = cudaEventQuery(s->upload_events.front());
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return fail(EB_ERR_CUDA, std::string("upload event: ") + cudaGetErrorString(q));
    take_oldest();
  }
  while (!s->upload.alloc(bytes, off)) {
    if (s->upload_events.empty())
      return fail(EB_ERR_OUT_OF_MEMORY, "request's initial data larger than the staging buffer");
    SV_CUDA(cudaEventSynchronize(s->upload_events.front()));
    take_oldest();
  }
  return EB_OK;
}

// Copy the request's initial rods into its bins (through pinned staging, so
// the copies queue behind the running ticks instead of waiting for them) and
// compute its initial energy.
eb_status place(eb_server* s, Request& r) {
  const int64_t S = s->stride;
  const size_t nu = r.bin_count.size(), nr = r.rods.size();
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  std::vector<size_t> ust(nu), upr(nu), umt(nu);
  size_t bytes = 0;
  for (size_t b = 0; b < nu; ++b) {
    const size_t c = static_cast<size_t>(r.bin_count[b]);
    ust[b] = bytes;
    bytes += up(c * eb::kStateFields * sizeof(double));
    upr[b] = bytes;
    bytes += up(c * eb::kParamFields * sizeof(double));
    umt[b] = bytes;
    bytes += up(c * sizeof(uint32_t));
  }
  const size_t uinfo = bytes;
  bytes += up(nr * sizeof(eb::RodInfo));
  const size_t ustart = bytes;
  bytes += up(nr * sizeof(int64_t));
  const size_t un = bytes;
  bytes += up(nr * sizeof(int32_t));
  size_t base_off = 0;
  if (eb_status st = upload_alloc(s, bytes, &base_off)) return st;
  unsigned char* base = s->upload.base + base_off;
  std::vector<double*> st(nu), pr(nu);
  std::vector<uint32_t*> mt(nu);
  for (size_t b = 0; b < nu; ++b) {
    st[b] = reinterpret_cast<double*>(base + ust[b]);
    pr[b] = reinterpret_cast<double*>(base + upr[b]);
    mt[b] = reinterpret_cast<uint32_t*>(base + umt[b]);
  }
  eb::RodInfo* info = reinterpret_cast<eb::RodInfo*>(base + uinfo);
  int64_t* rstart = reinterpret_cast<int64_t*>(base + ustart);
  int32_t* rn = reinterpret_cast<int32_t*>(base + un);
  // the staging space is reused once this event has passed (recorded on
  // every path, so the ring's allocations and the events stay paired)
  auto close_upload = [&]() -> eb_status {
    cudaEvent_t ev = nullptr;
    if (!s->spare_events.empty()) {
      ev = s->spare_events.back();
      s->spare_events.pop_back();
    } else {
      SV_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    s->upload_events.push_back(ev);
    SV_CUDA(cudaEventRecord(ev, s->stream));
    return EB_OK;
  };
  size_t voff = 0;
  for (size_t k = 0; k < r.rods.size(); ++k) {
    eb::HostRodData h;
    if (eb_status e = eb::host_straight_rod(r.rods[k], h)) {
      close_upload();
      return e;
    }
    const int64_t n = h.n, W = n + 1, b = r.rod_bin[k], o = r.rod_off[k], c = r.bin_count[b];
    if (!r.velocities.empty()) {
      for (int d = 0; d < 3; ++d)
        for (int64_t j = 0; j <= n; ++j) h.state[(eb::kStV + d) * W + j] = r.velocities[voff + d * W + j];
      voff += static_cast<size_t>(3 * W);
    }
    // (a unit's rods fill its slots [0, c) without gaps: every staged entry is written)
    for (int f = 0; f < eb::kStateFields; ++f)
      std::memcpy(&st[b][f * c + o], &h.state[f * W], W * sizeof(double));
    for (int f = 0; f < eb::kParamFields; ++f)
      std::memcpy(&pr[b][f * c + o], &h.param[f * W], W * sizeof(double));
    const int64_t rid = r.rod0 + static_cast<int64_t>(k);
    for (int64_t j = 0; j <= n; ++j) {
      uint32_t m = static_cast<uint32_t>(rid) << eb::kRodShift;
      if (j < n) m |= eb::kElem;
      if (j < n - 1) m |= eb::kVor;
      if (j == 0) m |= eb::kFirst;
      if (j == n) m |= eb::kLastNode;
      if (j == n - 1) m |= eb::kLastElem;
      mt[b][o + j] = m;
    }
    eb::RodInfo& ri = info[k];
    std::memset(&ri, 0, sizeof(ri));
    for (int d = 0; d < 3; ++d) ri.clamp_x[d] = h.state[(eb::kStX + d) * W];
    for (int q = 0; q < 9; ++q) ri.clamp_Q[q] = h.state[(eb::kStQ + q) * W];
    ri.damper_t = 1.0;
    ri.clamp_slot[1] = -1;
    ri.torque_slot = -1;
    ri.clamp_slot[0] = -1;
    if (r.options & EB_REQUEST_CLAMP) {
      ri.flags |= eb::kRodClamp;
      ri.clamp_slot[0] = r.bins[b] * kBin + o;  // node 0 / element 0 of the rod
    }
    if (r.options & EB_REQUEST_DAMPER) {
      ri.flags |= eb::kRodDamper;
      ri.damper_t = std::exp(-r.nu_t * r.dt);
      ri.damper_r = r.nu_r;
    }
    rstart[k] = r.bins[b] * kBin + o;
    rn[k] = static_cast<int32_t>(n);
    if (h.damped) r.damped = true;
  }
  for (size_t b = 0; b < r.bin_count.size(); ++b) {
    const int64_t c = r.bin_count[b], g0 = r.bins[b] * kBin;
    const size_t pitch = static_cast<size_t>(S) * sizeof(double), w = static_cast<size_t>(c) * sizeof(double);
    SV_CUDA(cudaMemcpy2DAsync(s->state[s->cur] + g0, pitch, st[b], w, w, eb::kStateFields,
                              cudaMemcpyHostToDevice, s->stream));
    SV_CUDA(cudaMemcpy2DAsync(s->par + g0, pitch, pr[b], w, w, eb::kParamFields, cudaMemcpyHostToDevice,
                              s->stream));
    SV_CUDA(cudaMemcpyAsync(s->meta + g0, mt[b], c * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  }
  SV_CUDA(cudaMemcpyAsync(s->rods + r.rod0, info, nr * sizeof(eb::RodInfo), cudaMemcpyHostToDevice, s->stream));
  SV_CUDA(cudaMemcpyAsync(s->rod_start + r.rod0, rstart, nr * sizeof(int64_t), cudaMemcpyHostToDevice, s->stream));
  SV_CUDA(cudaMemcpyAsync(s->rod_n + r.rod0, rn, nr * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
  if (eb_status st = close_upload()) return st;
  const double g[3] = {(r.options & EB_REQUEST_GRAVITY) ? r.gravity[0] : 0.0,
                       (r.options & EB_REQUEST_GRAVITY) ? r.gravity[1] : 0.0,
                       (r.options & EB_REQUEST_GRAVITY) ? r.gravity[2] : 0.0};
  SV_CUDA(eb::launch_rod_energy_list(static_cast<int64_t>(nr), S, s->rod_start + r.rod0, s->rod_n + r.rod0,
                                     s->state[s->cur], s->par, g, s->e0 + 5 * r.rod0, s->stream));
  return EB_OK;
}

eb_status admit(eb_server* s) {
  while (!s->queue.empty()) {
    Request& r = *s->queue.front();
    pack(r);
    int64_t n_pairs = 0, n_singles = 0;
    unit_counts(r, &n_pairs, &n_singles);
    if (!s->bins.fits(n_pairs, n_singles)) break;
    const int64_t rid = s->rod_ids.alloc(static_cast<int64_t>(r.rods.size()));
    if (rid < 0) break;
    r.rod0 = rid;
    r.bins.assign(r.bin_count.size(), -1);
    for (size_t b = 0; b < r.bin_count.size(); ++b)  // pairs first, so singles do not split them
      if (r.bin_pair[b]) r.bins[b] = s->bins.take_pair();
    for (size_t b = 0; b < r.bin_count.size(); ++b)
      if (!r.bin_pair[b]) r.bins[b] = s->bins.take_single();
    r.steps_done = 0;
    r.damped = false;
    if (eb_status e = place(s, r)) return e;
    if (r.queued_s < 0.0) r.queued_s = std::chrono::duration<double>(Clock::now() - r.t_submit).count();
    r.state = kActive;
    s->queue.pop_front();
    s->active.push_back(&r);
  }
  return EB_OK;
}

eb_status poll_events(eb_server* s, bool block_oldest);

// Enqueue the retirement of a request whose last step ran in this tick.
eb_status retire(eb_server* s, Request& r) {
  const int64_t S = s->stride, nr = static_cast<int64_t>(r.rods.size());
  const double g[3] = {(r.options & EB_REQUEST_GRAVITY) ? r.gravity[0] : 0.0,
                       (r.options & EB_REQUEST_GRAVITY) ? r.gravity[1] : 0.0,
                       (r.options & EB_REQUEST_GRAVITY) ? r.gravity[2] : 0.0};
  SV_CUDA(eb::launch_rod_energy_list(nr, S, s->rod_start + r.rod0, s->rod_n + r.rod0, s->state[s->cur], s->par, g,
                                     s->e1 + 5 * r.rod0, s->stream));
  size_t slots = 0;
  for (int32_t c : r.bin_count) slots += static_cast<size_t>(c);
  const size_t bytes = (slots * eb::kStateFields + 10 * static_cast<size_t>(nr)) * sizeof(double);
  size_t off = 0;
  while (!s->arena.alloc(bytes, &off)) {
    if (s->finishing.empty()) return fail(EB_ERR_OUT_OF_MEMORY, "request result larger than the host arena");
    // the arena is full: wait for the oldest retirement and take it out
    if (eb_status st = poll_events(s, true)) return st;
  }
  r.arena_off = off;
  double* dst = reinterpret_cast<double*>(s->arena.base + off);
  size_t pos = 0;
  for (size_t b = 0; b < r.bin_count.size(); ++b) {
    const int64_t c = r.bin_count[b], g0 = r.bins[b] * kBin;
    const size_t w = static_cast<size_t>(c) * sizeof(double);
    SV_CUDA(cudaMemcpy2DAsync(dst + pos, w, s->state[s->cur] + g0, static_cast<size_t>(S) * sizeof(double), w,
                              eb::kStateFields, cudaMemcpyDeviceToHost, s->stream));
    pos += static_cast<size_t>(c) * eb::kStateFields;
  }
  SV_CUDA(cudaMemcpyAsync(dst + pos, s->e0 + 5 * r.rod0, 5 * nr * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  SV_CUDA(cudaMemcpyAsync(dst + pos + 5 * nr, s->e1 + 5 * r.rod0, 5 * nr * sizeof(double), cudaMemcpyDeviceToHost,
                          s->stream));
  if (!r.event) SV_CUDA(cudaEventCreateWithFlags(&r.event, cudaEventDisableTiming));
  SV_CUDA(cudaEventRecord(r.event, s->stream));
  // bins and rod ids go back at once: the copies above run before any later
  // use of them on this stream
  for (size_t b = 0; b < r.bins.size(); ++b) {
    if (r.bin_pair[b])
      s->bins.give_pair(r.bins[b]);
    else
      s->bins.give_single(r.bins[b]);
  }
  s->rod_ids.release(r.rod0, nr);
  r.state = kFinishing;
  s->finishing.push_back(&r);
  return EB_OK;
}

// Take a landed retirement out of the arena: energies, drift check, result.
void land(eb_server* s, Request& r) {
  const int64_t nr = static_cast<int64_t>(r.rods.size());
  size_t slots = 0;
  for (int32_t c : r.bin_count) slots += static_cast<size_t>(c);
  const double* src = reinterpret_cast<const double*>(s->arena.base + r.arena_off);
  const double* e0 = src + slots * eb::kStateFields;
  const double* e1 = e0 + 5 * nr;
  double E0 = 0.0, E1 = 0.0, scale = 0.0;
  bool finite = true;
  for (int64_t k = 0; k < nr; ++k)
    for (int c = 0; c < 5; ++c) {
      E0 += e0[5 * k + c];
      E1 += e1[5 * k + c];
      scale += std::fabs(e0[5 * k + c]);
      finite = finite && std::isfinite(e1[5 * k + c]);
    }
  // plus the gravitational energy range of each rod over its own length, so a
  // rod that starts near the potential's zero is not held to a tighter check
  if (r.options & EB_REQUEST_GRAVITY) {
    const double g = std::sqrt(r.gravity[0] * r.gravity[0] + r.gravity[1] * r.gravity[1] +
                               r.gravity[2] * r.gravity[2]);
    for (const auto& p : r.rods)
      scale += p.density * (M_PI * p.radius * p.radius * p.length) * g * p.length;
  }
  r.e0 = E0;
  r.e1 = E1;
  r.escale = scale;
  // result per rod in the local slot layout
  r.result.clear();
  r.result_off.assign(r.rods.size(), 0);
  std::vector<size_t> bin_pos(r.bin_count.size(), 0);
  size_t pos = 0;
  for (size_t b = 0; b < r.bin_count.size(); ++b) {
    bin_pos[b] = pos;
    pos += static_cast<size_t>(r.bin_count[b]) * eb::kStateFields;
  }
  for (size_t k = 0; k < r.rods.size(); ++k) {
    const int64_t W = r.rods[k].n_elements + 1, b = r.rod_bin[k], o = r.rod_off[k], c = r.bin_count[b];
    r.result_off[k] = static_cast<int64_t>(r.result.size());
    for (int f = 0; f < eb::kStateFields; ++f) {
      const double* row = src + bin_pos[b] + static_cast<size_t>(f * c + o);
      r.result.insert(r.result.end(), row, row + W);
    }
  }
  s->arena.free_oldest();
  const bool drift_ok = finite && (E1 - E0) <= s->cfg.energy_tolerance * (scale > 0.0 ? scale : 1.0) &&
                       !(s->cfg.flags & EB_SERVER_FORCE_FALLBACK);
  if (!drift_ok && r.precision == EB_PRECISION_MIXED) {
    // rerun from the initial conditions in FP64
    r.precision = EB_PRECISION_FP64;
    r.fell_back = true;
    ++s->n_fallbacks;
    r.state = kQueued;
    r.result.clear();
    s->queue.push_front(&r);
    return;
  }
  r.latency_s = std::chrono::duration<double>(Clock::now() - r.t_submit).count();
  r.state = kDone;
  ++s->n_completed;
  eb_completion c{};
  c.request_id = r.id;
  c.precision = r.precision;
  c.fell_back = r.fell_back ? 1 : 0;
  c.latency_s = r.latency_s;
  c.queued_s = r.queued_s;
  c.energy_initial = E0;
  c.energy_final = E1;
  c.elements = r.elements;
  c.steps = r.n_steps;
  s->completed.push_back(c);
}

eb_status poll_events(eb_server* s, bool block_oldest) {
  while (!s->finishing.empty()) {
    Request* r = s->finishing.front();
    cudaError_t q = block_oldest ? cudaEventSynchronize(r->event) : cudaEventQuery(r->event);
    block_oldest = false;
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return fail(EB_ERR_CUDA, std::string("retirement event: ") + cudaGetErrorString(q));
    s->finishing.pop_front();
    land(s, *r);
  }
  return EB_OK;
}

}  // namespace

extern "C" {

EB_API eb_status eb_server_create(const eb_server_config* config, eb_server** out) {
  if (!out) return fail(EB_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = nullptr;
  eb_server_config cfg{};
  if (config) cfg = *config;
  if (cfg.precision != EB_PRECISION_MIXED && cfg.precision != EB_PRECISION_FP64)
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown precision");
  if (cfg.flags & ~static_cast<uint32_t>(EB_SERVER_FORCE_FALLBACK)) return fail(EB_ERR_INVALID_ARGUMENT, "unknown flag");
  if (cfg.steps_per_launch == 0) cfg.steps_per_launch = 128;
  if (cfg.steps_per_launch < 1 || cfg.steps_per_launch > 4096)
    return fail(EB_ERR_INVALID_ARGUMENT, "steps_per_launch must be in [1, 4096]");
  if (cfg.hbm_budget_bytes == 0.0) cfg.hbm_budget_bytes = 40e9;
  if (!(cfg.hbm_budget_bytes > 0.0)) return fail(EB_ERR_INVALID_ARGUMENT, "HBM budget must be positive");
  if (cfg.energy_tolerance == 0.0) cfg.energy_tolerance = 1e-3;
  if (!(cfg.energy_tolerance > 0.0)) return fail(EB_ERR_INVALID_ARGUMENT, "energy tolerance must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg.device < 0 || cfg.device >= ndev)
    return fail(EB_ERR_CUDA, "no such CUDA device");
  // bytes per bin: two state copies, parameters, metadata, rod table,
  // energies, rod lists, CTA tables
  const double per_bin = static_cast<double>(kBin) * (2 * eb::kStateFields + eb::kParamFields) * sizeof(double) +
                         kBin * sizeof(uint32_t) +
                         kRodsPerBin * (sizeof(eb::RodInfo) + 10 * sizeof(double) + sizeof(int64_t) + sizeof(int32_t)) +
                         4 * sizeof(eb::ServeCta);
  const int64_t n_bins = static_cast<int64_t>(cfg.hbm_budget_bytes / per_bin) / 2 * 2;  // whole bin pairs
  if (n_bins < 2) return fail(EB_ERR_INVALID_ARGUMENT, "HBM budget holds no bin pair");
  if (n_bins * kRodsPerBin >= (int64_t(1) << (32 - eb::kRodShift)))
    return fail(EB_ERR_UNSUPPORTED, "HBM budget too large for the rod id field");
  auto s = std::make_unique<eb_server>();
  s->cfg = cfg;
  s->n_bins = n_bins;
  s->n_slots = n_bins * kBin;
  s->stride = (s->n_slots + 31) / 32 * 32;
  s->rod_cap = n_bins * kRodsPerBin;
  cudaError_t e = cudaSetDevice(cfg.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  auto alloc = [&](auto** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s->stream);
  };
  const size_t S = static_cast<size_t>(s->stride);
  alloc(&s->state[0], S * eb::kStateFields * sizeof(double));
  alloc(&s->state[1], S * eb::kStateFields * sizeof(double));
  alloc(&s->par, S * eb::kParamFields * sizeof(double));
  alloc(&s->meta, S * sizeof(uint32_t));
  alloc(&s->rods, static_cast<size_t>(s->rod_cap) * sizeof(eb::RodInfo));
  alloc(&s->rod_start, static_cast<size_t>(s->rod_cap) * sizeof(int64_t));
  alloc(&s->rod_n, static_cast<size_t>(s->rod_cap) * sizeof(int32_t));
  alloc(&s->e0, static_cast<size_t>(s->rod_cap) * 5 * sizeof(double));
  alloc(&s->e1, static_cast<size_t>(s->rod_cap) * 5 * sizeof(double));
  alloc(&s->status, sizeof(uint32_t));
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      // one entry per bin, plus the padding entry of an odd count
      alloc(&s->d_cta[a][b], static_cast<size_t>(n_bins + 2) * sizeof(eb::ServeCta));
      if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void**>(&s->h_cta[a][b]),
                          static_cast<size_t>(n_bins + 2) * sizeof(eb::ServeCta), cudaHostAllocDefault);
    }
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&s->arena.base), kArenaBytes, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&s->upload.base), kUploadBytes, cudaHostAllocDefault);
  for (auto& ev : s->tick_event)
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  for (int p = 0; p < 2; ++p) {
    if (e == cudaSuccess) e = cudaEventCreate(&s->launch_t0[p]);
    if (e == cudaSuccess) e = cudaEventCreate(&s->launch_t1[p]);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    const std::string msg = std::string("server allocation: ") + cudaGetErrorString(e);
    server_free(s.get());
    return fail(e == cudaErrorMemoryAllocation ? EB_ERR_OUT_OF_MEMORY : EB_ERR_CUDA, msg);
  }
  s->arena.cap = kArenaBytes;
  s->upload.cap = kUploadBytes;
  s->bins.init(n_bins);
  s->rod_ids.init(s->rod_cap);
  *out = s.release();
  return EB_OK;
}

EB_API eb_status eb_server_destroy(eb_server* s) {
  if (!s) return EB_OK;
  server_free(s);
  delete s;
  return EB_OK;
}

EB_API eb_status eb_server_submit(eb_server* s, const eb_request* req, int64_t* request_id) {
  if (!s || !req || !request_id) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (req->n_rods < 1 || !req->rods) return fail(EB_ERR_INVALID_ARGUMENT, "a request needs at least one rod");
  if (!(req->dt > 0.0) || !std::isfinite(req->dt)) return fail(EB_ERR_INVALID_ARGUMENT, "dt must be positive");
  if (req->n_steps < 1) return fail(EB_ERR_INVALID_ARGUMENT, "a request needs at least one step");
  if (req->options & ~static_cast<uint32_t>(EB_REQUEST_CLAMP | EB_REQUEST_DAMPER | EB_REQUEST_GRAVITY))
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown request option");
  auto r = std::make_unique<Request>();
  r->rods.assign(req->rods, req->rods + req->n_rods);
  for (const auto& p : r->rods) {
    eb::HostRodData check;  // the reference initializer's argument checks
    if (p.n_elements >= 2 && p.n_elements + 1 <= kPairSlots)
      if (eb_status st = eb::host_straight_rod(p, check)) return st;
  }
  for (const auto& p : r->rods) {
    if (p.n_elements < 2) return fail(EB_ERR_INVALID_ARGUMENT, "a rod needs at least 2 elements");
    if (p.n_elements + 1 > kPairSlots)
      return fail(EB_ERR_UNSUPPORTED, "served rods hold at most " + std::to_string(kPairSlots - 1) + " elements");
    r->elements += p.n_elements;
  }
  pack(*r);
  int64_t n_pairs = 0, n_singles = 0;
  unit_counts(*r, &n_pairs, &n_singles);
  if (2 * n_pairs + n_singles > s->n_bins)
    return fail(EB_ERR_OUT_OF_MEMORY, "request larger than the server's HBM budget");
  if (req->velocities) {
    int64_t total = 0;
    for (const auto& p : r->rods) total += 3 * (p.n_elements + 1);
    r->velocities.assign(req->velocities, req->velocities + total);
  }
  r->dt = req->dt;
  r->n_steps = req->n_steps;
  for (int d = 0; d < 3; ++d) r->gravity[d] = req->gravity[d];
  r->options = req->options;
  r->nu_t = req->damper_translational;
  r->nu_r = req->damper_rotational;
  r->precision = s->cfg.precision;
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  Request* raw = r.get();
  s->requests[r->id] = std::move(r);
  s->queue.push_back(raw);
  *request_id = raw->id;
  return EB_OK;
}

EB_API eb_status eb_server_tick(eb_server* s, int64_t* in_flight) {
  if (!s) return fail(EB_ERR_INVALID_ARGUMENT, "null server");
  SV_CUDA(cudaSetDevice(s->cfg.device));
  const int parity = static_cast<int>(s->ticks & 1);
  // flow control: the tick that used this parity's tables must be done
  if (s->tick_pending[parity]) {
    SV_CUDA(cudaEventSynchronize(s->tick_event[parity]));
    s->tick_pending[parity] = false;
    if (s->launch_timed[parity]) {
      float ms = 0.0f;
      SV_CUDA(cudaEventElapsedTime(&ms, s->launch_t0[parity], s->launch_t1[parity]));
      s->kernel_seconds += 1e-3 * ms;
      s->launch_timed[parity] = false;
    }
  }
  if (eb_status st = poll_events(s, false)) return st;
  if (eb_status st = admit(s)) return st;
  const int K = s->cfg.steps_per_launch;
  int n_cta[2] = {0, 0};
  bool damped[2] = {false, false};
  // CTA tables: the two halves of each pair unit first (entries 2i, 2i + 1
  // form a cluster), then single bins, padded to an even count
  for (int pass = 0; pass < 2; ++pass)
    for (Request* r : s->active) {
      const int p = r->precision == EB_PRECISION_MIXED ? 0 : 1;
      const int32_t steps = static_cast<int32_t>(std::min<int64_t>(K, r->n_steps - r->steps_done));
      for (size_t b = 0; b < r->bins.size(); ++b) {
        if ((pass == 0) != (r->bin_pair[b] != 0)) continue;
        const int halves = r->bin_pair[b] ? 2 : 1;
        const int32_t W = r->bin_count[b], h = (W + 1) / 2;
        for (int k = 0; k < halves; ++k) {
          eb::ServeCta& c = s->h_cta[parity][p][n_cta[p]++];
          c.start = r->bins[b] * kBin + (k == 1 ? h : 0);
          c.count = halves == 1 ? W : (k == 0 ? h : W - h);
          c.steps = steps;
          c.dt = r->dt;
          c.half_dt = 0.5 * r->dt;
          for (int d = 0; d < 3; ++d) c.gravity[d] = r->gravity[d];
          c.flags = request_flags(*r);
          c.pair = halves == 2 ? 1u : 0u;
        }
      }
      damped[p] = damped[p] || r->damped;
    }
  for (int p = 0; p < 2; ++p)
    if (n_cta[p] % 2) {
      eb::ServeCta& c = s->h_cta[parity][p][n_cta[p]++];
      std::memset(&c, 0, sizeof(c));  // no slots, no steps: returns at once
    }
  if (n_cta[0] + n_cta[1] > 0) {
    eb::StepArgs a{};
    a.stride = s->stride;
    a.n_slots = s->n_slots;
    a.in = s->state[s->cur];
    a.out = s->state[s->cur ^ 1];
    a.par = s->par;
    a.meta = s->meta;
    a.rods = s->rods;
    a.status = s->status;
    for (int p = 0; p < 2; ++p) {
      if (!n_cta[p]) continue;
      SV_CUDA(cudaMemcpyAsync(s->d_cta[parity][p], s->h_cta[parity][p], n_cta[p] * sizeof(eb::ServeCta),
                              cudaMemcpyHostToDevice, s->stream));
      if (!s->launch_timed[parity]) {
        SV_CUDA(cudaEventRecord(s->launch_t0[parity], s->stream));
        s->launch_timed[parity] = true;
      }
      if (p == 0)
        SV_CUDA(eb::launch_rod_block_mixed_serve(a, s->d_cta[parity][p], n_cta[p], K, damped[p], s->stream));
      else
        SV_CUDA(eb::launch_rod_block_fp64_serve(a, s->d_cta[parity][p], n_cta[p], K, damped[p], s->stream));
    }
    if (s->launch_timed[parity]) SV_CUDA(cudaEventRecord(s->launch_t1[parity], s->stream));
    s->cur ^= 1;
    std::vector<Request*> still;
    for (Request* r : s->active) {
      const int64_t steps = std::min<int64_t>(K, r->n_steps - r->steps_done);
      r->steps_done += steps;
      s->element_steps += static_cast<double>(steps) * static_cast<double>(r->elements);
      if (r->steps_done >= r->n_steps) {
        if (eb_status st = retire(s, *r)) return st;
      } else {
        still.push_back(r);
      }
    }
    s->active.swap(still);
  }
  SV_CUDA(cudaEventRecord(s->tick_event[parity], s->stream));
  s->tick_pending[parity] = true;
  ++s->ticks;
  if (in_flight)
    *in_flight = static_cast<int64_t>(s->queue.size() + s->active.size() + s->finishing.size());
  return EB_OK;
}

EB_API eb_status eb_server_poll(eb_server* s, eb_completion* out, int32_t capacity, int32_t* count) {
  if (!s || !count || (capacity > 0 && !out)) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  SV_CUDA(cudaSetDevice(s->cfg.device));
  if (eb_status st = poll_events(s, false)) return st;
  int32_t n = 0;
  while (n < capacity && !s->completed.empty()) {
    out[n++] = s->completed.front();
    s->completed.pop_front();
  }
  *count = n;
  return EB_OK;
}

EB_API eb_status eb_server_result(eb_server* s, int64_t request_id, int64_t rod, int32_t field, double* values,
                                  int64_t count) {
  if (!s || !values) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  auto it = s->requests.find(request_id);
  if (it == s->requests.end()) return fail(EB_ERR_NOT_FOUND, "unknown request");
  const Request& r = *it->second;
  if (r.state != kDone) return fail(EB_ERR_INVALID_STATE, "request not completed");
  if (rod < 0 || rod >= static_cast<int64_t>(r.rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod");
  int row = 0, ncomp = 0;
  const int64_t n = r.rods[rod].n_elements, W = n + 1;
  int64_t per = 0;
  switch (field) {
    case EB_POSITION: row = eb::kStX; ncomp = 3; per = W; break;
    case EB_VELOCITY: row = eb::kStV; ncomp = 3; per = W; break;
    case EB_DIRECTOR: row = eb::kStQ; ncomp = 9; per = n; break;
    case EB_ANGULAR_VELOCITY: row = eb::kStW; ncomp = 3; per = n; break;
    default: return fail(EB_ERR_UNSUPPORTED, "served results hold the state fields only");
  }
  if (count != ncomp * per) return fail(EB_ERR_INVALID_ARGUMENT, "value count mismatch");
  const double* base = r.result.data() + r.result_off[rod];
  for (int c = 0; c < ncomp; ++c)
    std::memcpy(values + c * per, base + (row + c) * W, static_cast<size_t>(per) * sizeof(double));
  return EB_OK;
}

EB_API eb_status eb_server_release(eb_server* s, int64_t request_id) {
  if (!s) return fail(EB_ERR_INVALID_ARGUMENT, "null server");
  auto it = s->requests.find(request_id);
  if (it == s->requests.end()) return fail(EB_ERR_NOT_FOUND, "unknown request");
  if (it->second->state != kDone) return fail(EB_ERR_INVALID_STATE, "request not completed");
  if (it->second->event) cudaEventDestroy(it->second->event);
  s->requests.erase(it);
  return EB_OK;
}

EB_API eb_status eb_server_request_status(const eb_server* s, int64_t request_id, int32_t* state,
                                          double* age_s, double* queued_s) {
  if (!s || !state) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  auto it = s->requests.find(request_id);
  if (it == s->requests.end()) return fail(EB_ERR_NOT_FOUND, "unknown request");
  const Request& r = *it->second;
  const double age = std::chrono::duration<double>(Clock::now() - r.t_submit).count();
  *state = static_cast<int32_t>(r.state);
  if (age_s) *age_s = r.state == kDone ? r.latency_s : age;
  if (queued_s) *queued_s = r.queued_s >= 0.0 ? r.queued_s : age;
  return EB_OK;
}

EB_API eb_status eb_server_get_stats(const eb_server* s, eb_server_stats* out) {
  if (!s || !out) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  out->queued = static_cast<int64_t>(s->queue.size());
  out->active = static_cast<int64_t>(s->active.size());
  out->finishing = static_cast<int64_t>(s->finishing.size());
  out->completed = s->n_completed;
  out->fallbacks = s->n_fallbacks;
  out->bins_total = s->n_bins;
  out->bins_used = s->n_bins - s->bins.free_bins();
  out->ticks = s->ticks;
  out->element_steps = s->element_steps;
  out->kernel_seconds = s->kernel_seconds;
  return EB_OK;
}

}  // extern "C"
