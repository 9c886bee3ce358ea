// The docking search's intra-pair schedule: which pair each lane of the warp
// evaluates in each round of the pair phase, built on the host when a ligand
// is added.
//
// In one round the 32 lanes each load both atoms' coordinates (two 128-bit
// shared-memory loads) and add the pair force into both atoms' fixed-point
// accumulators (six 32-bit shared-memory atomics).  On B200 a 128-bit shared
// load is served in four phases of 8 lanes, each phase costing one wavefront
// per distinct atom in its most crowded bank group (atom mod 8: the
// coordinates are float4s); an atomic costs one wavefront per lane in its
// most crowded bank (atom mod 32), lanes on the same atom included.  The
// schedule is built in two steps: which pairs share a round (greedy, few
// lanes per atom), then where each pair sits in the round and which of its
// atoms comes first (a local search over the round's layout).
#include "schedule.h"

#include <algorithm>
#include <cstdint>
#include <cstring>

namespace vd {
namespace {

constexpr int kLanes = 32, kPhases = 4, kPhaseLanes = 8;
constexpr int kMaxAtoms = 128;
constexpr int kAtomicWeight = 3;  // three atomics (x, y, z) per atom per round

inline int first_atom(const int2& q) { return q.x & 0xffff; }
inline int second_atom(const int2& q) { return q.x >> 16; }
inline int2 flipped(const int2& q) { return make_int2(second_atom(q) | (first_atom(q) << 16), q.y); }

// Pairs that share a round: greedy over the remaining pairs, those whose
// atoms have the most pairs left first: take pairs whose first atom and
// second atom are each still unused in the round (either orientation: a
// pair's force is antisymmetric), then allow two lanes per atom, then three,
// and so on, until the round holds 32 pairs.  Within the round, lanes are
// then assigned so that each group of 8 lanes sees distinct atom residues
// mod 8 where possible (the starting point of the layout search).
std::vector<std::vector<int2>> greedy_rounds(const std::vector<int2>& pairs, int na) {
    std::vector<int> deg(na, 0);
    for (const int2& q : pairs) { ++deg[first_atom(q)]; ++deg[second_atom(q)]; }
    std::vector<int2> rem(pairs);
    std::vector<std::vector<int2>> rounds;
    std::vector<int> ca(na), cb(na);
    while (!rem.empty()) {
        std::stable_sort(rem.begin(), rem.end(), [&](const int2& x, const int2& y) {
            return deg[first_atom(x)] + deg[second_atom(x)] > deg[first_atom(y)] + deg[second_atom(y)];
        });
        std::fill(ca.begin(), ca.end(), 0);
        std::fill(cb.begin(), cb.end(), 0);
        std::vector<int2> take;
        for (int cap = 1; take.size() < size_t(kLanes) && !rem.empty(); ++cap) {
            std::vector<int2> keep;
            for (const int2& q : rem) {
                const int u = first_atom(q), v = second_atom(q);
                if (take.size() < size_t(kLanes) && ca[u] < cap && cb[v] < cap) {
                    take.push_back(q);
                    ++ca[u]; ++cb[v];
                } else if (take.size() < size_t(kLanes) && ca[v] < cap && cb[u] < cap) {
                    take.push_back(flipped(q));
                    ++ca[v]; ++cb[u];
                } else {
                    keep.push_back(q);
                }
            }
            rem.swap(keep);
        }
        for (const int2& q : take) { --deg[first_atom(q)]; --deg[second_atom(q)]; }
        // phases of 8 with distinct residues mod 8 of both atoms, then of one, then any
        std::vector<int2> left(take), order;
        while (!left.empty()) {
            std::vector<int2> phase;
            unsigned ga = 0, gb = 0;
            for (int strict = 2; strict >= 0; --strict) {
                std::vector<int2> keep;
                for (const int2& q : left) {
                    const unsigned ra = 1u << (first_atom(q) & 7), rb = 1u << (second_atom(q) & 7);
                    const bool oka = !(ga & ra), okb = !(gb & rb);
                    if (phase.size() < size_t(kPhaseLanes) &&
                        (strict == 0 || (strict == 1 && (oka || okb)) || (oka && okb))) {
                        phase.push_back(q);
                        ga |= ra; gb |= rb;
                    } else {
                        keep.push_back(q);
                    }
                }
                left.swap(keep);
            }
            order.insert(order.end(), phase.begin(), phase.end());
        }
        order.resize(kLanes, make_int2(0, -1));  // empty lanes
        rounds.push_back(order);
    }
    return rounds;
}

// Conflict counts of one round, updated lane by lane.  Side 0 is each
// pair's first atom, side 1 its second; an empty lane loads atom 0 on both
// sides (its schedule word names atoms 0 and 0) and adds no force.
struct Layout {
    int2 lane[kLanes];
    uint8_t occ[2][kPhases][kMaxAtoms];  // lanes of a phase loading an atom
    int grp[2][kPhases][8];              // distinct atoms of a phase per bank group
    int bank[2][32];                     // atomic lanes per bank
    long cost = 0;

    static bool empty(const int2& q) { return q.y < 0; }
    int atom(int i, int side) const {
        return empty(lane[i]) ? 0 : (side == 0 ? first_atom(lane[i]) : second_atom(lane[i]));
    }
    void load(int side, int p, int a, int d) {  // d = +1 add, -1 remove
        int& g = grp[side][p][a & 7];
        if (d > 0) {
            if (occ[side][p][a]++ == 0) { cost += 2 * g + 1; ++g; }
        } else {
            if (--occ[side][p][a] == 0) { --g; cost -= 2 * g + 1; }
        }
    }
    void atomic(int side, int a, int d) {
        int& b = bank[side][a & 31];
        if (d > 0) { cost += kAtomicWeight * (2 * b + 1); ++b; }
        else { --b; cost -= kAtomicWeight * (2 * b + 1); }
    }
    void place(int i, int d, bool atomics = true) {  // add (+1) or remove (-1) lane i's contributions
        for (int s = 0; s < 2; ++s) {
            load(s, i / kPhaseLanes, atom(i, s), d);
            if (atomics && !empty(lane[i])) atomic(s, atom(i, s), d);
        }
    }
    explicit Layout(const std::vector<int2>& r) {
        std::memset(occ, 0, sizeof(occ));
        std::memset(grp, 0, sizeof(grp));
        std::memset(bank, 0, sizeof(bank));
        for (int i = 0; i < kLanes; ++i) {
            lane[i] = r[i];
            place(i, +1);
        }
    }
    void swap_lanes(int i, int j) {  // the atomics do not depend on lane positions
        place(i, -1, false);
        place(j, -1, false);
        std::swap(lane[i], lane[j]);
        place(i, +1, false);
        place(j, +1, false);
    }
    void flip(int i) {
        place(i, -1);
        lane[i] = flipped(lane[i]);
        place(i, +1);
    }
};

// Local search over one round's layout: random lane swaps between phases
// and orientation flips, kept when the cost does not rise (the sum of
// squared occupancies, a smooth stand-in for the per-instruction maxima),
// until kStall moves in a row bring no strict improvement or kMoves moves
// have run.  A fixed-seed generator keeps schedules reproducible.
void refine_round(std::vector<int2>& r, uint64_t seed) {
    Layout L(r);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    auto next = [&x]() {
        x = x * 6364136223846793005ull + 1442695040888963407ull;
        return uint32_t(x >> 33);
    };
    // 1,500 moves: measured against 200-move stalls (lighter host work,
    // coordinate-load conflicts 7% higher) and 4,000 moves (3x the host work
    // for 1% fewer); ligand lists are packed on host threads (vd_add_ligands)
    constexpr int kMoves = 1500, kStall = 1500;
    long best = L.cost;
    for (int it = 0, stall = 0; it < kMoves && stall < kStall; ++it, ++stall) {
        if (L.cost < best) { best = L.cost; stall = 0; }
        const long before = L.cost;
        const uint32_t u = next();
        const int i = int(u % kLanes);
        if (u & (1u << 20)) {
            const int j = int((u >> 8) % kLanes);
            if (i / kPhaseLanes == j / kPhaseLanes) continue;  // same phase: no change
            L.swap_lanes(i, j);
            if (L.cost > before) L.swap_lanes(i, j);
        } else {
            if (Layout::empty(L.lane[i])) continue;
            L.flip(i);
            if (L.cost > before) L.flip(i);
        }
    }
    for (int i = 0; i < kLanes; ++i) r[i] = L.lane[i];
}

}  // namespace

long round_cost(const std::vector<int2>& round) { return Layout(round).cost; }

std::vector<std::vector<int2>> schedule_pairs(const std::vector<int2>& pairs, int na, bool refine) {
    std::vector<std::vector<int2>> rounds = greedy_rounds(pairs, na);
    if (refine)
        for (size_t k = 0; k < rounds.size(); ++k) refine_round(rounds[k], uint64_t(k) + 1);
    return rounds;
}

}  // namespace vd
