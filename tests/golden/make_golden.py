"""Regenerate the golden fixtures of the Poisson oracle.

The reference cannot be built here (OpenVDB, TBB, Eigen absent) and ships no
golden vectors, so these fixtures pin the CPU restatement itself: a change to
oracle/poisson_oracle.c that alters any of these numbers fails
tests/test_oracle_poisson.py::test_golden_fixture.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import OraclePoisson  # noqa: E402
from uaamg_b200 import scenes  # noqa: E402


def golden_scene():
    return scenes.sdf_box_scene(40, 0.4, [((0.5, 0.7, 0.5), 0.15)], seed=3, dt=1.0, name="golden 40^3")


def make():
    sc = golden_scene()
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    out = {"levels": np.array(o.num_levels), "ndof": np.array([o.ndof(l) for l in range(o.num_levels)])}
    for l in range(o.num_levels):
        (d, cx, cy, cz), flags = o.coefficients(l)
        org, masks = o.topology(l)
        out[f"l{l}_origins"] = org
        out[f"l{l}_masks"] = masks
        out[f"l{l}_diag"] = d
        out[f"l{l}_cx"] = cx
        out[f"l{l}_cy"] = cy
        out[f"l{l}_cz"] = cz
        out[f"l{l}_flags"] = flags
    rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    out["rhs"] = rhs
    for sm in ("scheduled_jacobi", "weighted_jacobi", "rbgs", "spai0"):
        x, st, it, nu = o.solve_pcg(o.zeros(), rhs, smoother=sm)
        out[f"pcg_{sm}_x"] = x
        out[f"pcg_{sm}_iters"] = np.array(it)
        out[f"pcg_{sm}_status"] = np.array(st)
    np.savez_compressed(os.path.join(HERE, "poisson_golden_40.npz"), **out)


if __name__ == "__main__":
    make()
    print("wrote", os.path.join(HERE, "poisson_golden_40.npz"))
