// Host check of the launch-shape autotuner (vina-cuda_b200/csrc/tune.h):
// every candidate is explored once per key on real calls, the cheapest is
// then kept, keys are independent, invalid reports are ignored.
#include <cstdio>

#include "tune.h"

#define CHECK(c)                                                  \
    do {                                                          \
        if (!(c)) {                                               \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            return 1;                                             \
        }                                                         \
    } while (0)

int main() {
    vd::Tuner t;
    const uint64_t k1 = 7, k2 = 9;
    // exploration: candidates in order, one per call, until each has a cost
    CHECK(t.best(k1) == -1);
    CHECK(t.pick(k1, 3) == 0);
    t.report(k1, 0, 5.0);
    CHECK(t.pick(k1, 3) == 1);
    t.report(k1, 1, 2.0);
    CHECK(t.best(k1) == -1);
    CHECK(t.pick(k1, 3) == 2);
    t.report(k1, 2, 3.0);
    CHECK(t.best(k1) == 1);           // cheapest
    for (int i = 0; i < 4; ++i) CHECK(t.pick(k1, 3) == 1);
    t.report(k1, 0, 1.0);             // later reports do not reopen a settled key
    CHECK(t.pick(k1, 3) == 1);
    // another key is independent
    CHECK(t.pick(k2, 2) == 0);
    t.report(k2, 0, -1.0);            // invalid cost: ignored
    t.report(k2, 5, 1.0);             // invalid candidate: ignored
    CHECK(t.pick(k2, 2) == 0);
    t.report(k2, 0, 4.0);
    CHECK(t.pick(k2, 2) == 1);
    t.report(k2, 1, 4.0);
    CHECK(t.best(k2) == 0);           // ties keep the first candidate
    // an unexplored key reported out of order settles once all have costs
    vd::Tuner u;
    u.pick(3, 2);
    u.report(3, 1, 1.0);
    CHECK(u.best(3) == -1 && u.pick(3, 2) == 0);
    u.report(3, 0, 0.5);
    CHECK(u.best(3) == 0);
    CHECK(vd::ceil_log2(1) == 0 && vd::ceil_log2(2) == 1 && vd::ceil_log2(6500) == 13 &&
          vd::ceil_log2(8192) == 13 && vd::ceil_log2(8193) == 14);
    std::printf("ok\n");
    return 0;
}
