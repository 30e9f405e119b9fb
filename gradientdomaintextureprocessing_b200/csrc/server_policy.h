// HBM admission for the solve server (host only, no CUDA).
//
// Resident models (hierarchy + device systems) are charged their device bytes
// against a budget.  A model that must become resident is admitted when the
// budget has room after evicting idle models, least recently used first; busy
// models (a solve in flight) are never evicted.  The policy only decides; the
// server builds and frees the models.
#pragma once
#include <algorithm>
#include <cstdint>
#include <map>
#include <vector>

namespace gdtp {

class AdmissionPolicy {
 public:
  explicit AdmissionPolicy(int64_t budget) : budget_(budget) {}

  int64_t budget() const { return budget_; }
  int64_t used() const { return used_; }
  int64_t peak() const { return peak_; }
  int64_t evictions() const { return evictions_; }
  bool resident(int id) const { return models_.count(id) != 0; }
  bool busy(int id) const {
    auto it = models_.find(id);
    return it != models_.end() && it->second.busy;
  }

  // Idle models to evict, least recently used first, so that `bytes` more fit;
  // false (victims empty) when even evicting every idle model is not enough.
  bool plan(int64_t bytes, std::vector<int>& victims, int exclude = -1) const {
    victims.clear();
    if (bytes > budget_) return false;
    int64_t free = budget_ - used_;
    if (bytes <= free) return true;
    std::vector<std::pair<uint64_t, int>> idle;
    for (const auto& kv : models_)
      if (!kv.second.busy && kv.first != exclude) idle.push_back({kv.second.lastUse, kv.first});
    std::sort(idle.begin(), idle.end());
    for (const auto& v : idle) {
      victims.push_back(v.second);
      free += models_.at(v.second).bytes;
      if (bytes <= free) return true;
    }
    victims.clear();
    return false;
  }

  void add(int id, int64_t bytes, uint64_t tick) {
    Entry& e = models_[id];
    used_ += bytes - e.bytes;
    e.bytes = bytes;
    e.lastUse = tick;
    peak_ = std::max(peak_, used_);
  }
  void evict(int id) {
    auto it = models_.find(id);
    if (it == models_.end()) return;
    used_ -= it->second.bytes;
    models_.erase(it);
    evictions_++;
  }
  void set_busy(int id, bool b, uint64_t tick) {
    auto it = models_.find(id);
    if (it == models_.end()) return;
    it->second.busy = b;
    it->second.lastUse = tick;
  }

 private:
  struct Entry {
    int64_t bytes = 0;
    uint64_t lastUse = 0;
    bool busy = false;
  };
  int64_t budget_ = 0, used_ = 0, peak_ = 0, evictions_ = 0;
  std::map<int, Entry> models_;
};

}  // namespace gdtp
