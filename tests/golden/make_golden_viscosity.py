"""Regenerate the golden fixture of the viscosity oracle.

The reference cannot be built here (OpenVDB, TBB, Eigen absent) and ships no
golden vectors, so this fixture pins the CPU restatement itself: a change to
oracle/viscosity_oracle.c that alters any of these numbers fails
tests/test_oracle_viscosity.py::test_golden_fixture.  It also feeds the GPU
parity test of the same scene.

    python tests/golden/make_golden_viscosity.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import OracleViscosity  # noqa: E402
from uaamg_b200 import scenes  # noqa: E402

FILE = os.path.join(HERE, "viscosity_golden_24.npz")


def golden_scene():
    return scenes.viscosity_box_scene(24, 0.4, [((0.5, 0.7, 0.5), 0.15)], seed=7, mu=1e3,
                                      name="golden viscosity 24^3")


def warm_start(o, sc):
    """FLIP_vdb.cpp:3188-3198: the initial guess is the velocity at each DOF."""
    org, _ = o.topology(0)
    idx = o.dof_index(0)
    out = o.zeros(0)
    off = np.arange(512)
    xyz = np.stack([off >> 6, (off >> 3) & 7, off & 7], 1)
    for c, g in enumerate((sc.u, sc.v, sc.w)):
        lut = {tuple(x): i for i, x in enumerate(g.origins)}
        for li in range(org.shape[0]):
            j = lut.get(tuple(org[li]))
            if j is None:
                continue
            m = idx[c, li] >= 0
            out[c, li, m] = g.values[j].reshape(512)[m]
    return out


def make():
    sc = golden_scene()
    o = OracleViscosity(sc.liquid_phi, sc.solid_phi, sc.viscosity, sc.dt, sc.rho, sc.dx)
    out = {"levels": np.array(o.num_levels), "ndof": np.array([o.ndof(l) for l in range(o.num_levels)])}
    for l in range(o.num_levels):
        coef, trim = o.coefficients(l)
        org, masks = o.topology(l)
        out[f"l{l}_origins"] = org
        out[f"l{l}_dof"] = masks
        out[f"l{l}_coef"] = coef
        out[f"l{l}_trim"] = trim
    rhs = o.build_rhs(sc.u, sc.v, sc.w, sc.solid_velocity)
    out["rhs"] = rhs
    x0 = warm_start(o, sc)
    out["x0"] = x0
    x, st, it, nu = o.solve_pcg(x0, rhs, 1e-6, 100)
    out["pcg_x"] = x
    out["pcg_iters"] = np.array(it)
    out["pcg_status"] = np.array(st)
    np.savez_compressed(FILE, **out)


if __name__ == "__main__":
    make()
    print("wrote", FILE)
