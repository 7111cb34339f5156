// Pinning harness (test infrastructure).  Compiled by build_ref.sh against the
// reference's own src/MortonLUT.h, where it lies in the reference tree, into
// oracle/_ref/.  It prints the reference's Morton encode/decode results
// (its host LUT paths, src/MortonLUT.h:482-529) so tests/golden/make_golden.py
// can store them as fixtures.  The reference's __constant__ tables have no
// host copy; make_golden.py reads those from the source text instead.
#include <cstdio>
#include <cstdint>
#include <random>
#include "MortonLUT.h"

int main() {
    // per-axis encode, every coordinate below 4096 (exact below 1024,
    // truncated to 32 bits above)
    for (int axis = 0; axis < 3; ++axis)
        for (uint32_t v = 0; v < 4096; ++v) {
            uint16_t c[3] = {0, 0, 0};
            c[axis] = (uint16_t)v;
            printf("E %u %u %u %u\n", c[0], c[1], c[2], mortonEncode_LUT(c[0], c[1], c[2]));
        }
    std::mt19937 rng(12345);
    for (int i = 0; i < 4096; ++i) {
        uint16_t x = rng() & 1023, y = rng() & 1023, z = rng() & 1023;
        printf("E %u %u %u %u\n", x, y, z, mortonEncode_LUT(x, y, z));
    }
    for (int i = 0; i < 4096; ++i) {
        uint32_t m = rng() & 0x3FFFFFFFu;
        uint16_t x, y, z;
        morton3D_32_decode(m, x, y, z);
        printf("D %u %u %u %u\n", m, x, y, z);
    }
    return 0;
}
