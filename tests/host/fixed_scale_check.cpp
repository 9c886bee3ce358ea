// Host check of pair_force_scale (tables.cpp): for several weight sets the
// scale is a power of two, 128 x the largest pair force times the scale
// stays below 2^30, and the next power of two would not (unless the 2^24
// cap applies); the default weights give 2^19.  Prints "ok" on success.
#include <cmath>
#include <cstdio>
#include <vector>

#include "common.h"

int main() {
    using namespace vd;
    const double def[6] = {-0.035579, -0.005156, 0.840245, -0.035069, -0.587439, 1.923};
    const double mults[] = {1.0, 0.01, 0.5, 3.0, 40.0, 1000.0};
    for (double mult : mults) {
        double w[6];
        for (int i = 0; i < 5; ++i) w[i] = def[i] * mult;
        w[5] = def[5];
        std::vector<double> fast, se, sd;
        build_tables(w, fast, se, sd);
        const double scale = pair_force_scale(sd);
        int ex = 0;
        if (std::frexp(scale, &ex) != 0.5) { std::printf("scale %g is not a power of two\n", scale); return 1; }
        double bound = 0.0;
        for (int p = 0; p < kPairTypes; ++p)
            for (int i = 0; i + 1 < kBins; ++i) {
                const size_t b = size_t(p) * kN + i;
                bound = std::fmax(bound, std::fmax(std::fabs(sd[b]), std::fabs(sd[b + 1])) * std::sqrt((i + 1) / 32.0));
            }
        if (!(128.0 * bound * scale < 1073741824.0)) { std::printf("x%g: overflow margin\n", mult); return 1; }
        if (scale < 16777216.0 && !(128.0 * bound * 2.0 * scale >= 1073741824.0)) {
            std::printf("x%g: scale %g not the largest\n", mult, scale);
            return 1;
        }
        if (mult == 1.0 && scale != 524288.0) { std::printf("default scale %g\n", scale); return 1; }
    }
    std::printf("ok\n");
    return 0;
}
