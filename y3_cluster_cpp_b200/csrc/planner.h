// planner.h -- scheduling policy of the request server (pure host C++, no CUDA).
//
// A request is a group of parameter points whose tables must sit in the
// device table pool while any of its points is being evaluated.  The planner
// decides three things:
//   * admission: requests enter the pool in arrival order, each taking one
//     contiguous run of slots (one table block per point, first fit).  The head
//     of the queue is never overtaken, so a large request cannot starve behind
//     a stream of small ones; it waits until enough finished requests have
//     released their slots;
//   * batching: every launch takes up to max_batch points from the admitted
//     requests, oldest first, splitting a request across launches when it does
//     not fit (continuous batching: requests admitted while a launch runs join
//     the next one);
//   * release: when every point of a request has come back, its run of slots
//     returns to the pool (neighbouring free runs are merged);
//   * cancellation: a cancelled request leaves the queue, or, once admitted,
//     gets no further points scheduled; its slots return when the points
//     already launched have come back.
#pragma once

#include <algorithm>
#include <deque>
#include <iterator>
#include <map>
#include <unordered_map>
#include <vector>

namespace y3b {

class SlotPool {
 public:
  explicit SlotPool(int cap) : cap_(cap)
  {
    if (cap > 0) free_[0] = cap;
  }
  // First run of n free slots, or -1.
  int alloc(int n)
  {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const int start = it->first, len = it->second;
      free_.erase(it);
      if (len > n) free_[start + n] = len - n;
      return start;
    }
    return -1;
  }
  void release(int start, int n)
  {
    auto it = free_.emplace(start, n).first;
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
  int free_slots() const
  {
    int t = 0;
    for (const auto& kv : free_) t += kv.second;
    return t;
  }
  int capacity() const { return cap_; }

 private:
  int cap_;
  std::map<int, int> free_;  // start -> length, disjoint and non-adjacent
};

struct PlanChunk {
  long long id;
  int first;  // index of the first point inside the request
  int count;
  int slot;   // pool slot of that first point
};

class Planner {
 public:
  Planner(int pool_slots, int max_batch) : pool_(pool_slots), max_batch_(max_batch) {}

  // 0 on success, 1 if the request can never fit (n > pool) or is malformed.
  int submit(long long id, int n)
  {
    if (n < 1 || n > pool_.capacity() || reqs_.count(id)) return 1;
    reqs_[id] = Req{n, -1, 0, 0, false};
    waiting_.push_back(id);
    return 0;
  }

  // Admit waiting requests in arrival order while the pool has room.
  void admit(std::vector<std::pair<long long, int>>* out)
  {
    while (!waiting_.empty()) {
      const long long id = waiting_.front();
      Req& r = reqs_[id];
      const int s = pool_.alloc(r.n);
      if (s < 0) break;
      r.slot0 = s;
      waiting_.pop_front();
      active_.push_back(id);
      out->emplace_back(id, s);
    }
  }

  // Chunks of the next launch (<= max_batch points, <= max_chunks chunks).
  int next_batch(std::vector<PlanChunk>* out, int max_chunks = 1 << 30)
  {
    int left = max_batch_, total = 0;
    for (auto it = active_.begin(); it != active_.end() && left > 0 &&
                                    (int)out->size() < max_chunks;) {
      Req& r = reqs_[*it];
      const int take = std::min(left, r.n - r.next);
      out->push_back(PlanChunk{*it, r.next, take, r.slot0 + r.next});
      r.next += take;
      left -= take;
      total += take;
      if (r.next == r.n)
        it = active_.erase(it);  // fully scheduled; waits for completion only
      else
        ++it;
    }
    return total;
  }

  // Marks `count` points of request `id` as returned.  Returns 1 when the
  // request is complete (its slots are released), 0 if points are still out,
  // -1 for an unknown request or a count beyond what was scheduled.
  int complete(long long id, int count)
  {
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -1;
    Req& r = it->second;
    if (r.slot0 < 0 || count < 0 || r.done + count > r.next) return -1;
    r.done += count;
    if (r.done < (r.cancelled ? r.next : r.n)) return 0;
    pool_.release(r.slot0, r.n);
    reqs_.erase(it);
    return 1;
  }

  // Stops scheduling request `id`.  Returns 1 when nothing of it is out any
  // more (it has left the planner and its slots are free), 0 when launched
  // points must still come back through complete(), -1 for an unknown id.
  int cancel(long long id)
  {
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -1;
    Req& r = it->second;
    if (r.slot0 < 0) {  // still waiting for admission
      waiting_.erase(std::find(waiting_.begin(), waiting_.end(), id));
      reqs_.erase(it);
      return 1;
    }
    auto a = std::find(active_.begin(), active_.end(), id);
    if (a != active_.end()) active_.erase(a);
    r.cancelled = true;
    if (r.done < r.next) return 0;
    pool_.release(r.slot0, r.n);
    reqs_.erase(it);
    return 1;
  }

  int free_slots() const { return pool_.free_slots(); }
  int capacity() const { return pool_.capacity(); }
  int waiting() const { return (int)waiting_.size(); }
  int unscheduled() const { return (int)active_.size(); }
  bool idle() const { return reqs_.empty(); }

 private:
  struct Req {
    int n, slot0, next, done;
    bool cancelled;
  };
  SlotPool pool_;
  int max_batch_;
  std::deque<long long> waiting_;  // not yet admitted, arrival order
  std::deque<long long> active_;   // admitted, points left to schedule
  std::unordered_map<long long, Req> reqs_;
};

}  // namespace y3b
