// k-way partition of rods by element count (largest differencing method of
// Karmarkar and Karp, the partitioner the reference ships for balancing
// blocks across threads, elastica/Utilities/KarmarkarKarpPartition.hpp:
// 332-422).  Every item starts as a partial partition with the item in one
// part and the other parts empty; the two partial partitions with the largest
// spread (largest minus smallest part) are merged by joining the largest part
// of one with the smallest of the other, the second largest with the second
// smallest, and so on, until one partition is left.  Ties are broken by
// creation order, so every rank computes the same partition.
#include <algorithm>
#include <cstdint>
#include <queue>
#include <string>
#include <vector>

#include "../../include/elastica_b200.h"
#include "eb_host.h"

namespace {

struct Partial {
  std::vector<int64_t> sum;                 // per part, descending
  std::vector<std::vector<int32_t>> items;  // per part
  int64_t order = 0;
  int64_t spread() const { return sum.front() - sum.back(); }
};

struct Wider {
  const std::vector<Partial>* pool;
  bool operator()(int32_t a, int32_t b) const {
    const Partial& x = (*pool)[a];
    const Partial& y = (*pool)[b];
    if (x.spread() != y.spread()) return x.spread() < y.spread();
    return x.order > y.order;  // earlier first among equal spreads
  }
};

}  // namespace

extern "C" EB_API eb_status eb_partition_rods(const int64_t* weights, int64_t n, int32_t n_parts, int32_t* part_of) {
  if (n < 0 || n_parts < 1 || (n > 0 && (!weights || !part_of))) {
    eb::set_last_error("bad partition arguments");
    return EB_ERR_INVALID_ARGUMENT;
  }
  if (n >= (int64_t(1) << 31)) {
    eb::set_last_error("too many items");
    return EB_ERR_UNSUPPORTED;
  }
  for (int64_t i = 0; i < n; ++i)
    if (weights[i] < 0) {
      eb::set_last_error("negative weight");
      return EB_ERR_INVALID_ARGUMENT;
    }
  if (n == 0) return EB_OK;
  const size_t k = static_cast<size_t>(n_parts);
  std::vector<Partial> pool(static_cast<size_t>(n));
  std::priority_queue<int32_t, std::vector<int32_t>, Wider> heap(Wider{&pool});
  int64_t order = 0;
  for (int64_t i = 0; i < n; ++i) {
    Partial& p = pool[static_cast<size_t>(i)];
    p.sum.assign(k, 0);
    p.items.assign(k, {});
    p.sum[0] = weights[i];
    p.items[0].push_back(static_cast<int32_t>(i));
    p.order = order++;
    heap.push(static_cast<int32_t>(i));
  }
  while (heap.size() > 1) {
    const int32_t a = heap.top();
    heap.pop();
    const int32_t b = heap.top();
    heap.pop();
    Partial& A = pool[static_cast<size_t>(a)];
    Partial& B = pool[static_cast<size_t>(b)];
    std::vector<std::pair<int64_t, std::vector<int32_t>>> parts(k);
    for (size_t j = 0; j < k; ++j) {
      parts[j].first = A.sum[j] + B.sum[k - 1 - j];
      parts[j].second = std::move(A.items[j]);
      auto& src = B.items[k - 1 - j];
      parts[j].second.insert(parts[j].second.end(), src.begin(), src.end());
    }
    std::stable_sort(parts.begin(), parts.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    for (size_t j = 0; j < k; ++j) {
      A.sum[j] = parts[j].first;
      A.items[j] = std::move(parts[j].second);
    }
    B.items.clear();
    B.sum.clear();
    A.order = order++;
    heap.push(a);
  }
  const Partial& last = pool[static_cast<size_t>(heap.top())];
  for (size_t j = 0; j < k; ++j)
    for (int32_t i : last.items[j]) part_of[i] = static_cast<int32_t>(j);
  return EB_OK;
}
