// Host check of the docking search's pair schedule (csrc/schedule.cpp):
// every pair scheduled exactly once with its type pair, 32-lane rounds with
// empty lanes {0, -1}, deterministic output, and a layout search that never
// raises a round's conflict cost.  Prints the mean per-ligand cost before
// and after the search and the build time.
#include <chrono>
#include <cstdio>
#include <map>
#include <random>
#include <utility>
#include <vector>

#include "schedule.h"

int main() {
    std::mt19937 rng(7);
    double before = 0, after = 0, ms = 0;
    const int kLigands = 200;
    for (int t = 0; t < kLigands; ++t) {
        const int na = 10 + int(rng() % 119);  // 10..128 heavy atoms
        std::vector<int2> pairs;
        std::map<std::pair<int, int>, int> want;
        const double keep = 0.2 + 0.6 * (rng() % 1000) / 1000.0;
        for (int a = 0; a < na && pairs.size() < 4096; ++a)
            for (int b = a + 1; b < na && pairs.size() < 4096; ++b)
                if ((rng() % 1000) < keep * 1000) {
                    const int tp = int(rng() % 153);
                    pairs.push_back(make_int2(a | (b << 16), tp));
                    want[{a, b}] = tp;
                }
        const auto t0 = std::chrono::steady_clock::now();
        const auto r1 = vd::schedule_pairs(pairs, na);
        ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        const auto r0 = vd::schedule_pairs(pairs, na, false);
        const auto r2 = vd::schedule_pairs(pairs, na);
        if (r0.size() != r1.size()) { std::printf("FAIL round count\n"); return 1; }
        std::map<std::pair<int, int>, int> seen;
        for (size_t k = 0; k < r1.size(); ++k) {
            if (r1[k].size() != 32) { std::printf("FAIL round size\n"); return 1; }
            const long c0 = vd::round_cost(r0[k]), c1 = vd::round_cost(r1[k]);
            if (c1 > c0) { std::printf("FAIL cost rose %ld -> %ld\n", c0, c1); return 1; }
            before += double(c0);
            after += double(c1);
            for (int l = 0; l < 32; ++l) {
                const int2 q = r1[k][l];
                if (q.x != r2[k][l].x || q.y != r2[k][l].y) { std::printf("FAIL not deterministic\n"); return 1; }
                if (q.y < 0) {
                    if (q.x != 0) { std::printf("FAIL empty lane\n"); return 1; }
                    continue;
                }
                int a = q.x & 0xffff, b = q.x >> 16;
                if (a > b) std::swap(a, b);
                if (a >= na || b >= na || seen.count({a, b})) { std::printf("FAIL pair %d %d\n", a, b); return 1; }
                seen[{a, b}] = q.y;
            }
        }
        if (seen != want) { std::printf("FAIL pairs differ\n"); return 1; }
    }
    std::printf("OK mean round cost per ligand %.1f -> %.1f, %.3f ms per ligand\n", before / kLigands,
                after / kLigands, ms / kLigands);
    return 0;
}
