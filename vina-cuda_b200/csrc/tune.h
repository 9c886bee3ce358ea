// Launch-shape autotuner.
//
// A kernel with several launch shapes (register budget per thread, tile
// size) whose results do not depend on the shape is tuned per workload key:
// the first calls with a new key each run one untried candidate, the cost
// of every run (kernel time per unit of work) is recorded, and once all
// candidates have run the cheapest one is used for that key from then on.
// Tuning therefore costs no extra kernel launches, only the slower
// candidates' share of the first few real calls.
#pragma once

#include <cstdint>
#include <map>
#include <vector>

namespace vd {

class Tuner {
  public:
    // Candidate to run for this key.
    int pick(uint64_t key, int n_cand) {
        Entry& e = table_[key];
        if (e.cost.empty()) e.cost.assign(n_cand, -1.0);
        if (e.best >= 0) return e.best;
        for (int i = 0; i < n_cand; ++i)
            if (e.cost[i] < 0) return i;
        return 0;
    }
    // Cost of one run of candidate `cand` (lower is better).
    void report(uint64_t key, int cand, double cost) {
        auto it = table_.find(key);
        if (it == table_.end() || cand < 0 || cand >= int(it->second.cost.size()) || !(cost >= 0)) return;
        Entry& e = it->second;
        if (e.cost[cand] < 0 || cost < e.cost[cand]) e.cost[cand] = cost;
        if (e.best >= 0) return;
        int best = -1;
        for (int i = 0; i < int(e.cost.size()); ++i) {
            if (e.cost[i] < 0) return;  // still exploring
            if (best < 0 || e.cost[i] < e.cost[best]) best = i;
        }
        e.best = best;
    }
    // Tuned candidate for a key, or -1 while it is still being explored.
    int best(uint64_t key) const {
        auto it = table_.find(key);
        return it == table_.end() ? -1 : it->second.best;
    }
    void clear() { table_.clear(); }

  private:
    struct Entry {
        int best = -1;
        std::vector<double> cost;  // -1 = not run yet
    };
    std::map<uint64_t, Entry> table_;
};

inline int ceil_log2(uint64_t v) {
    int k = 0;
    while ((uint64_t(1) << k) < v && k < 63) ++k;
    return k;
}

}  // namespace vd
