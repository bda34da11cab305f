// Admission policy of the serving scheduler: which probes of which requests start at each tick.
//
// Host-only and deterministic, so the policy is testable without a device (totem_plan_simulate).
// A tick advances every running probe group by one slice; a group of ``items`` probes of one
// request starts at some tick and finishes ``slices`` ticks later, holding ``items * item_bytes``
// of wave memory (the probes' waves and detector partial sums) meanwhile.
#pragma once
#include <algorithm>
#include <cstddef>
#include <numeric>
#include <vector>

namespace totem {

struct PlanRequest {
  unsigned long long id = 0;
  int n = 0;                 // window edge (groups of one edge share launches)
  long long items = 0;       // probes = w_num * depth
  int slices = 0;
  size_t item_bytes = 0;     // wave memory of one probe
  long long next = 0;        // first probe not yet started
};

struct PlanGroup {
  unsigned long long req = 0;
  long long item0 = 0;
  int items = 0;
  int start_tick = 0;
  int last_tick = 0;         // start_tick + slices - 1
  int n = 0;
  size_t bytes = 0;
  void* psi = nullptr;       // device buffers of the group (owned by the server)
  void* part = nullptr;
};

class Planner {
 public:
  static constexpr int kFifo = 0, kShortest = 1;
  static constexpr long long kMaxGroupItems = 1 << 20;

  Planner(size_t wave_bytes, size_t chunk_bytes, int policy, size_t max_groups)
      : wave_(wave_bytes), chunk_(std::max<size_t>(chunk_bytes, 1)), policy_(policy), max_groups_(max_groups) {}

  void add(const PlanRequest& r) { pending_.push_back(r); }
  bool idle() const { return active_.empty() && pending_.empty(); }
  size_t inflight() const { return inflight_; }
  const std::vector<PlanGroup>& active() const { return active_; }

  // Groups that start at ``tick``.  Requests are visited in arrival order, i.e. by ticket (FIFO;
  // with several preparation threads requests can become ready out of order, and a later one
  // that is ready does not wait for an earlier one still being prepared), or by least remaining
  // work, probes x slices (SHORTEST).  Each may start up to chunk_bytes of probes per
  // tick while the wave memory in flight stays within wave_bytes.  FIFO stops at the first
  // request that cannot start (no overtaking); SHORTEST lets smaller requests fill the gap.  A
  // single probe larger than wave_bytes starts alone when nothing else is in flight.
  std::vector<PlanGroup> start(int tick) {
    std::vector<PlanGroup> out;
    std::vector<size_t> order(pending_.size());
    std::iota(order.begin(), order.end(), 0);
    if (policy_ == kShortest)
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return work(pending_[a]) < work(pending_[b]);
      });
    else
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return pending_[a].id < pending_[b].id; });
    for (size_t idx : order) {
      if (active_.size() + out.size() >= max_groups_) break;
      PlanRequest& r = pending_[idx];
      const size_t free = wave_ > inflight_ ? wave_ - inflight_ : 0;
      long long cap = 0;
      if (free >= r.item_bytes) cap = (long long)std::max<size_t>(1, std::min(free, chunk_) / r.item_bytes);
      else if (inflight_ == 0 && r.item_bytes > wave_) cap = 1;
      const long long take = std::min({cap, r.items - r.next, kMaxGroupItems});
      if (take <= 0) {
        if (policy_ == kFifo) break;
        continue;
      }
      PlanGroup g;
      g.req = r.id;
      g.item0 = r.next;
      g.items = (int)take;
      g.start_tick = tick;
      g.last_tick = tick + r.slices - 1;
      g.n = r.n;
      g.bytes = (size_t)take * r.item_bytes;
      inflight_ += g.bytes;
      r.next += take;
      out.push_back(g);
    }
    pending_.erase(std::remove_if(pending_.begin(), pending_.end(),
                                  [](const PlanRequest& r) { return r.next >= r.items; }),
                   pending_.end());
    active_.insert(active_.end(), out.begin(), out.end());
    return out;
  }

  // Groups whose last slice runs at ``tick``; removed from the active set.
  std::vector<PlanGroup> finish(int tick) {
    std::vector<PlanGroup> done;
    std::vector<PlanGroup> keep;
    keep.reserve(active_.size());
    for (const PlanGroup& g : active_) {
      if (g.last_tick <= tick) {
        done.push_back(g);
        inflight_ -= g.bytes;
      } else {
        keep.push_back(g);
      }
    }
    active_.swap(keep);
    return done;
  }

  // Record device buffers on the active group that started as ``g``.
  void attach(const PlanGroup& g, void* psi, void* part) {
    for (PlanGroup& a : active_)
      if (a.req == g.req && a.item0 == g.item0) {
        a.psi = psi;
        a.part = part;
      }
  }

 private:
  static long long work(const PlanRequest& r) { return (r.items - r.next) * (long long)r.slices; }

  size_t wave_, chunk_;
  int policy_;
  size_t max_groups_;
  size_t inflight_ = 0;
  std::vector<PlanRequest> pending_;
  std::vector<PlanGroup> active_;
};

}  // namespace totem
