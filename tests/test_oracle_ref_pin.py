"""Pins of the oracle against the reference's own code.

The reference's solvers need OpenVDB, TBB and Eigen, none of which is in this
image, but two of its source files are plain C++: SIMD_UAAMG/levelset_util.cpp
(fraction_inside, two- and four-corner forms, used by the pressure matrix and
the face weights) and SIMD_UAAMG/volume_fractions.cpp (volume_fraction of a
tetrahedron and of a cube, used by the viscosity construction).  oracle/Makefile
(`make -C oracle ref`, run by build() where the reference's sources are present)
compiles them where they lie, behind oracle/ref_shim.cpp, into oracle/_ref/:
once with the source's operation order (no contraction) and once as the
reference's CMake build would on an FMA host (-march, GCC's default contraction).

The oracle's restatements must equal the first bit for bit on seeded inputs
that cover both signs, zeros, ties and magnitudes from 1e-8 to 1e2; the CUDA
kernels are bit-exact against the oracle elsewhere, so the pin carries over.
The contracted build is allowed last-bit differences only.
"""
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.skipif(not os.path.exists(oracle.REF_LIB), reason="oracle/_ref not built")


def _samples(n, k, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, k))
    b = rng.standard_normal((n, k)) * 10.0 ** rng.integers(-8, 3, (n, k))
    c = rng.choice(np.array([0.0, -0.0, 1.0, -1.0, 0.5, -0.5, 1e-30, -1e-30]), (n, k))
    pick = rng.integers(0, 3, (n, 1))
    return np.where(pick == 0, a, np.where(pick == 1, b, c)).astype(np.float32)


def _same(x, y):
    x, y = np.float32(x), np.float32(y)
    return (np.isnan(x) and np.isnan(y)) or x.view(np.uint32) == y.view(np.uint32)


CASES = [
    ("orc_fraction_inside2", "ref_fraction_inside2", 2),
    ("orc_fraction_inside4", "ref_fraction_inside4", 4),
    ("orc_tet_fraction", "ref_volume_fraction_tet", 4),
    ("orc_cube_fraction", "ref_volume_fraction_cube", 8),
]


@pytest.mark.parametrize("orc,ref,k", CASES)
def test_oracle_equals_reference_build(orc, ref, k):
    O, R = oracle.lib(), oracle.ref_lib()
    of, rf = getattr(O, orc), getattr(R, ref)
    bad = []
    for i, row in enumerate(_samples(6000, k, seed=k)):
        args = [float(v) for v in row]
        o, r = of(*args), rf(*args)
        if not _same(o, r):
            bad.append((args, o, r))
    assert not bad, bad[:3]


@pytest.mark.parametrize("orc,ref,k", CASES)
def test_contracted_reference_build_differs_in_last_bits_only(orc, ref, k):
    R, RN = oracle.ref_lib(), oracle.ref_lib(native=True)
    if RN is None:
        pytest.skip("contracted build absent")
    rf, nf = getattr(R, ref), getattr(RN, ref)
    worst = 0.0
    for row in _samples(3000, k, seed=100 + k):
        args = [float(v) for v in row]
        r, n = np.float32(rf(*args)), np.float32(nf(*args))
        if _same(r, n) or not np.isfinite(r) or r == 0:
            continue
        worst = max(worst, abs(float(n) - float(r)) / abs(float(r)))
    assert worst <= 1e-6, worst
