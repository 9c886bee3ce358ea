// The docking search's intra-pair schedule (host side, built once per ligand).
#pragma once

#include <vector>

#include <vector_functions.h>
#include <vector_types.h>

namespace vd {

// Splits a ligand's intra pairs {a | b << 16, type pair} (atoms < na) into
// rounds of 32 lanes, one pair per lane; an empty lane is {0, -1}.  Every
// pair appears once, as (a, b) or (b, a).  Deterministic.  refine = false
// skips the layout search (the greedy rounds only; for checks).
std::vector<std::vector<int2>> schedule_pairs(const std::vector<int2>& pairs, int na, bool refine = true);

// Smooth shared-memory conflict cost of one 32-lane round (lower is better):
// the sum, over both atoms of the pair, of the squared bank-group
// occupancies of the four 8-lane phases of the coordinate loads and three
// times the squared bank occupancies of the atomics.
long round_cost(const std::vector<int2>& round);

}  // namespace vd
