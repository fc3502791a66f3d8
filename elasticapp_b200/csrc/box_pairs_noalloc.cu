// Candidate pairs of caller-provided boxes without any device allocation.
//
// This is the collision system's broad phase (a uniform grid hashed into a
// power-of-two table, a counting sort of the boxes by bucket, a search of the
// 27 neighbouring cells, closed-interval overlap tests) as a standalone entry
// point whose working memory is one fixed array in this file instead of
// buffers from cudaMalloc.  It exists for callers that cannot allocate device
// memory themselves: code embedded in a host framework that reserves the
// whole device memory pool up front and hands its operators their buffers
// (where a cudaMalloc of its own fails or is not allowed), and loops that
// cannot afford the device-wide synchronisation of cudaMalloc / cudaFree.
//
// Limits and sharing:
// * at most kMaxBoxes boxes per call (the scratch array is sized for that);
// * the scratch array is a file-scope device variable: every GPU that loads
//   this library holds it (16 MiB) until the process exits;
// * all calls on a device share it and it keeps the previous call's contents;
//   each call clears what it needs zeroed (bucket counts, largest extent,
//   status) before use.  Calls whose GPU work overlaps (two streams, two host
//   threads) race on it and give wrong results: serialise them;
// * the first call on a device looks up the array's device address (with that
//   device current) and caches it for later calls.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/elastica_b200.h"

namespace eb {
// records the message eb_last_error() returns on this thread (eb_capi.cu)
void set_last_error(const std::string& message);
}  // namespace eb

namespace {

constexpr int64_t kMaxBoxes = int64_t(1) << 17;  // 131,072 boxes per call
constexpr int64_t kTable = int64_t(1) << 18;     // hash table slots (>= 2 * kMaxBoxes)
constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr double kCellMargin = 1.0 + 1.0 / 1048576.0;
constexpr double kCellClamp = 1073741824.0;

// scratch layout, each part on a 256-byte boundary
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffExtent = 0;                                              // u64 largest extent bits
constexpr size_t kOffStatus = kOffExtent + 256;                               // u32 flags
constexpr size_t kOffCell = kOffStatus + 256;                                 // 3 x int32 per box
constexpr size_t kOffBucket = kOffCell + align256(3 * kMaxBoxes * 4);        // u32 per box
constexpr size_t kOffCount = kOffBucket + align256(kMaxBoxes * 4);           // int32 per table slot
constexpr size_t kOffStart = kOffCount + align256(kTable * 4);               // int32, table + 1
constexpr size_t kOffSortedId = kOffStart + align256((kTable + 1) * 4);      // int32 per box
constexpr size_t kOffSortedCell = kOffSortedId + align256(kMaxBoxes * 4);    // 3 x int32 per box
constexpr size_t kOffSortedBox = kOffSortedCell + align256(3 * kMaxBoxes * 4);  // 6 x double per box
constexpr size_t kOffPairCount = kOffSortedBox + align256(6 * kMaxBoxes * 8);   // int32 per box
constexpr size_t kOffPairOffset = kOffPairCount + align256(kMaxBoxes * 4);      // int64, boxes + 1
constexpr size_t kScratchBytes = kOffPairOffset + align256((kMaxBoxes + 1) * 8);
static_assert(kScratchBytes <= (size_t(16) << 20), "scratch layout exceeds 16 MiB");

static __device__ __align__(256) unsigned char g_box_pair_scratch[size_t(16) << 20];

enum NoAllocStatus : uint32_t { kBadBox = 1u };

struct Scratch {
  unsigned long long* extent;
  uint32_t* status;
  int32_t* cell;
  uint32_t* bucket;
  int32_t* count;
  int32_t* start;
  int32_t* sorted_id;
  int32_t* sorted_cell;
  double* sorted_box;
  int32_t* pair_count;
  int64_t* pair_offset;
};

Scratch carve(unsigned char* base) {
  Scratch s;
  s.extent = reinterpret_cast<unsigned long long*>(base + kOffExtent);
  s.status = reinterpret_cast<uint32_t*>(base + kOffStatus);
  s.cell = reinterpret_cast<int32_t*>(base + kOffCell);
  s.bucket = reinterpret_cast<uint32_t*>(base + kOffBucket);
  s.count = reinterpret_cast<int32_t*>(base + kOffCount);
  s.start = reinterpret_cast<int32_t*>(base + kOffStart);
  s.sorted_id = reinterpret_cast<int32_t*>(base + kOffSortedId);
  s.sorted_cell = reinterpret_cast<int32_t*>(base + kOffSortedCell);
  s.sorted_box = reinterpret_cast<double*>(base + kOffSortedBox);
  s.pair_count = reinterpret_cast<int32_t*>(base + kOffPairCount);
  s.pair_offset = reinterpret_cast<int64_t*>(base + kOffPairOffset);
  return s;
}

__device__ __forceinline__ uint32_t cell_hash(int32_t cx, int32_t cy, int32_t cz) {
  uint64_t h = static_cast<uint64_t>(static_cast<uint32_t>(cx)) * 0x9E3779B97F4A7C15ull ^
               static_cast<uint64_t>(static_cast<uint32_t>(cy)) * 0xC2B2AE3D27D4EB4Full ^
               static_cast<uint64_t>(static_cast<uint32_t>(cz)) * 0x165667B19E3779F9ull;
  h ^= h >> 29;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 32;
  return static_cast<uint32_t>(h);
}

__device__ __forceinline__ bool overlaps(const double* a, const double* b) {
  // closed intervals: a = (lo x, lo y, lo z, hi x, hi y, hi z)
  return !(b[0] > a[3] || b[1] > a[4] || b[2] > a[5] || b[3] < a[0] || b[4] < a[1] || b[5] < a[2]);
}

// largest box extent (block max, one atomic per CTA); non-finite or inverted
// boxes are flagged
__global__ void __launch_bounds__(kThreads) extent_kernel(const double* boxes, int64_t n, Scratch s) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  double ext = 0.0;
  if (i < n) {
    const double* b = boxes + 6 * i;
    for (int d = 0; d < 3; ++d) {
      const double x = b[3 + d] - b[d];
      if (!(x >= 0.0 && x < 1e300 && fabs(b[d]) < 1e300)) {
        atomicOr(s.status, kBadBox);
      } else {
        ext = fmax(ext, x);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
  __shared__ double wmax[kThreads / 32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = ext;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < kThreads / 32; ++k) m = fmax(m, wmax[k]);
    if (m > 0.0) atomicMax(s.extent, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

__global__ void __launch_bounds__(kThreads) cell_kernel(const double* boxes, int64_t n, Scratch s) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  double h = __longlong_as_double(static_cast<long long>(*s.extent)) * kCellMargin;
  if (!(h > 0.0)) h = 1.0;
  const double ih = 1.0 / h;
  int32_t c[3];
  for (int d = 0; d < 3; ++d) {
    double f = floor(boxes[6 * i + d] * ih);
    f = fmin(fmax(f, -kCellClamp), kCellClamp);
    c[d] = static_cast<int32_t>(f);
    s.cell[3 * i + d] = c[d];
  }
  const uint32_t b = cell_hash(c[0], c[1], c[2]) & static_cast<uint32_t>(kTable - 1);
  s.bucket[i] = b;
  atomicAdd(s.count + b, 1);
}

// single-CTA exclusive scan of n int32 counts; out[n] = total.  Optionally
// zeroes the input (the counts then serve as fill cursors).
template <typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_kernel(int32_t* in, Out* out, int64_t n, bool zero_in) {
  __shared__ Out warp_sums[kScanThreads / 32];
  const int64_t per = (n + kScanThreads - 1) / kScanThreads;
  const int64_t lo = static_cast<int64_t>(threadIdx.x) * per;
  const int64_t hi = lo + per < n ? lo + per : n;
  Out sum = 0;
  for (int64_t k = lo; k < hi; ++k) sum += static_cast<Out>(in[k]);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Out x = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const Out y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    Out ws = warp_sums[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const Out y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    warp_sums[lane] = ws;
  }
  __syncthreads();
  Out run = (wid > 0 ? warp_sums[wid - 1] : Out(0)) + x - sum;
  for (int64_t k = lo; k < hi; ++k) {
    const Out v = static_cast<Out>(in[k]);
    out[k] = run;
    run += v;
    if (zero_in) in[k] = 0;
  }
  if (threadIdx.x == kScanThreads - 1) out[n] = warp_sums[kScanThreads / 32 - 1];
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(const double* boxes, int64_t n, Scratch s) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  const uint32_t b = s.bucket[i];
  const int32_t pos = s.start[b] + atomicAdd(s.count + b, 1);
  if (pos < 0 || pos >= n) return;  // unreachable with consistent counts
  s.sorted_id[pos] = static_cast<int32_t>(i);
  for (int d = 0; d < 3; ++d) s.sorted_cell[3 * pos + d] = s.cell[3 * i + d];
  for (int d = 0; d < 6; ++d) s.sorted_box[6 * pos + d] = boxes[6 * i + d];
}

// Sort the partners (second entries) of one box's pair segment in place,
// ascending: heapsort, O(c log c) for c partners and no extra memory (the
// first entries are all the box's own index).
__device__ void sort_partners(int64_t* seg, int32_t c) {
  auto sift = [seg](int32_t root, int32_t end) {
    while (true) {
      int32_t child = 2 * root + 1;
      if (child >= end) return;
      if (child + 1 < end && seg[2 * child + 1] < seg[2 * child + 3]) ++child;
      if (seg[2 * root + 1] >= seg[2 * child + 1]) return;
      const int64_t t = seg[2 * root + 1];
      seg[2 * root + 1] = seg[2 * child + 1];
      seg[2 * child + 1] = t;
      root = child;
    }
  };
  for (int32_t k = c / 2 - 1; k >= 0; --k) sift(k, c);
  for (int32_t end = c - 1; end > 0; --end) {
    const int64_t t = seg[1];
    seg[1] = seg[2 * end + 1];
    seg[2 * end + 1] = t;
    sift(0, end);
  }
}

// every box counts (pass 1) or writes (pass 2) its partners with a larger
// index; the written segment of box i is sorted by partner.  The cell edge
// is the largest box extent, so one very large box puts many boxes in one
// cell: the search then costs up to O(n) per box (O(n^2) in all), which the
// box limit bounds.
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) pairs_kernel(int64_t n, Scratch s, int64_t* pairs, int64_t capacity) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (e >= n) return;
  const int32_t id = s.sorted_id[e];
  const int32_t cx = s.sorted_cell[3 * e], cy = s.sorted_cell[3 * e + 1], cz = s.sorted_cell[3 * e + 2];
  const double* me = s.sorted_box + 6 * e;
  int64_t* out = nullptr;
  if (kWrite) {
    if (s.pair_offset[n] > capacity) return;
    out = pairs + 2 * s.pair_offset[id];
  }
  int32_t cnt = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int32_t nx = cx + dx, ny = cy + dy, nz = cz + dz;
        const uint32_t b = cell_hash(nx, ny, nz) & static_cast<uint32_t>(kTable - 1);
        const int32_t k0 = max(s.start[b], 0);
        const int32_t k1 = min(s.start[b + 1], static_cast<int32_t>(n));
        for (int32_t k = k0; k < k1; ++k) {
          if (s.sorted_cell[3 * k] != nx || s.sorted_cell[3 * k + 1] != ny || s.sorted_cell[3 * k + 2] != nz)
            continue;
          const int32_t other = s.sorted_id[k];
          if (other <= id) continue;
          if (!overlaps(me, s.sorted_box + 6 * k)) continue;
          if (kWrite) {
            out[2 * cnt] = id;
            out[2 * cnt + 1] = other;
          }
          ++cnt;
        }
      }
  if constexpr (!kWrite) {
    s.pair_count[id] = cnt;
  } else {
    sort_partners(out, cnt);
  }
}

std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[64] = {nullptr};

}  // namespace

extern "C" EB_API eb_status eb_box_pairs_noalloc(const double* boxes, int64_t n_boxes, int64_t* pairs,
                                                 int64_t capacity, int64_t* count, void* stream) {
  auto fail = [](eb_status st, const std::string& m) {
    eb::set_last_error(m);
    return st;
  };
  if (!count) return fail(EB_ERR_INVALID_ARGUMENT, "null count pointer");
  *count = 0;
  if (n_boxes < 0) return fail(EB_ERR_INVALID_ARGUMENT, "negative box count");
  if (n_boxes > kMaxBoxes)
    return fail(EB_ERR_INVALID_ARGUMENT, "eb_box_pairs_noalloc takes at most " + std::to_string(kMaxBoxes) +
                                             " boxes per call (got " + std::to_string(n_boxes) + ")");
  if (capacity < 0 || (capacity > 0 && !pairs)) return fail(EB_ERR_INVALID_ARGUMENT, "bad pair buffer");
  if (n_boxes > 0 && !boxes) return fail(EB_ERR_INVALID_ARGUMENT, "null box array");
  if (n_boxes < 2) return EB_OK;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64)
    return fail(EB_ERR_CUDA, std::string("no usable current device: ") + cudaGetErrorString(e));
  unsigned char* base = nullptr;
  {
    // set-up, once per device, with that device current: the device address
    // of the scratch array (the array's name is only a host stand-in)
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_box_pair_scratch);
      if (e != cudaSuccess || !p)
        return fail(EB_ERR_CUDA, std::string("scratch address lookup: ") + cudaGetErrorString(e));
      g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    base = g_scratch_ptr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Scratch s = carve(base);
  const unsigned g = static_cast<unsigned>((n_boxes + kThreads - 1) / kThreads);
#define NA_CUDA(call)                                                                 \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return fail(EB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
  // what must start at zero: largest extent, status, bucket counts
  NA_CUDA(cudaMemsetAsync(s.extent, 0, sizeof(unsigned long long), st));
  NA_CUDA(cudaMemsetAsync(s.status, 0, sizeof(uint32_t), st));
  NA_CUDA(cudaMemsetAsync(s.count, 0, static_cast<size_t>(kTable) * sizeof(int32_t), st));
  extent_kernel<<<g, kThreads, 0, st>>>(boxes, n_boxes, s);
  cell_kernel<<<g, kThreads, 0, st>>>(boxes, n_boxes, s);
  scan_kernel<int32_t><<<1, kScanThreads, 0, st>>>(s.count, s.start, kTable, true);
  scatter_kernel<<<g, kThreads, 0, st>>>(boxes, n_boxes, s);
  pairs_kernel<false><<<g, kThreads, 0, st>>>(n_boxes, s, pairs, capacity);
  scan_kernel<int64_t><<<1, kScanThreads, 0, st>>>(s.pair_count, s.pair_offset, n_boxes, false);
  NA_CUDA(cudaGetLastError());
  int64_t total = 0;
  uint32_t flags = 0;
  NA_CUDA(cudaMemcpyAsync(&total, s.pair_offset + n_boxes, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(&flags, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  if (flags & kBadBox) return fail(EB_ERR_INVALID_ARGUMENT, "a box is not finite or has hi < lo");
  *count = total;
  if (total > capacity)
    return fail(EB_ERR_INVALID_ARGUMENT, "pair buffer too small: " + std::to_string(total) + " pairs, capacity " +
                                             std::to_string(capacity));
  if (total > 0) pairs_kernel<true><<<g, kThreads, 0, st>>>(n_boxes, s, pairs, capacity);
  NA_CUDA(cudaGetLastError());
  NA_CUDA(cudaStreamSynchronize(st));
#undef NA_CUDA
  return EB_OK;
}
