// Test infrastructure: C entry points over the reference's own scalar helpers,
// compiled from the reference's source files where they lie (see the `ref`
// target of oracle/Makefile; output in oracle/_ref/, never committed).  They
// pin the oracle's restatements of the same functions (tests/test_oracle_ref_pin.py):
//   fraction_inside(l, r), fraction_inside(bl, br, tl, tr)  SIMD_UAAMG/levelset_util.cpp:4-100
//   volume_fraction(tet), volume_fraction(cube)              SIMD_UAAMG/volume_fractions.cpp:82-150
#include "levelset_util.h"
#include "volume_fractions.h"

extern "C" {
float ref_fraction_inside2(float l, float r) { return fraction_inside(l, r); }
float ref_fraction_inside4(float bl, float br, float tl, float tr) { return fraction_inside(bl, br, tl, tr); }
float ref_volume_fraction_tet(float p0, float p1, float p2, float p3) { return volume_fraction(p0, p1, p2, p3); }
float ref_volume_fraction_cube(float p000, float p100, float p010, float p110, float p001, float p101, float p011,
                               float p111) {
    return volume_fraction(p000, p100, p010, p110, p001, p101, p011, p111);
}
}
