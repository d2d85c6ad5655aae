"""Writes oracle_regression.npz: a small seeded channel release (64 x 64 DEM
at 5 m, ~400 particles) and the CPU oracle's state after 10 steps for a set
of options and precision modes.

The reference ships no tests or outputs and its Fortran is not compiled
here, so these vectors are the oracle's own, pinned by the known-answer
tests of test_oracle_kat.py: they lock the checker against unintended
change (test_oracle_golden.py replays the stored inputs and compares bit for
bit).  Rerun this script only after a deliberate change to the oracle.

    python tests/golden/make_oracle_regression.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "deslizamientos-y-flujos_b200"), os.path.join(ROOT, "oracle")]

import gfsph  # noqa: E402
import oracle  # noqa: E402
import workloads  # noqa: E402

NSTEPS = 10
PORE = {13: 0.02, 14: 1.0}
# name: (oracle mode, extra const(k), option overrides)
CASES = {
    "fp32": (0, {}, {}),
    "fp32_dacc": (1, {}, {}),
    "fp64": (2, {}, {}),
    "nor_density_cos_theta": (1, {16: 1.0}, {"nor_density": 1}),
    "gaussian_skf2": (1, {}, {"skf": 2}),
    "pore_pressure": (1, PORE, {"icpwp": 3, "pwp0rel": 0.8}),
}


def inputs():
    w = workloads.fractal_channel(n_target=400, dem_k=6, cell=5.0, semi_along=40.0, semi_across=25.0)
    return w


def case_run(w, mode, const_extra, over):
    const = {**w.const, **const_extra}
    opts = {**w.options, **over}
    p = gfsph.make_params(const, **opts)
    ny, nx = w.z.shape
    topol = oracle.initial_topol(w.z, w.dx, w.dy, const, deriv=p.dem_deriv, mode=mode)
    st = oracle.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    oracle.run(mode, p, nx, ny, w.dx, w.dy, st, NSTEPS)
    return st


def main():
    w = inputs()
    out = {"z": w.z, "x": w.x, "v": w.v, "rho": w.rho, "mass": w.mass, "hsml": w.hsml,
           "dxdy": np.array([w.dx, w.dy]),
           "meta": np.array(json.dumps({"const": {str(k): v for k, v in w.const.items()}, "options": w.options,
                                        "nsteps": NSTEPS,
                                        "cases": {k: [m, {str(a): b for a, b in c.items()}, o]
                                                  for k, (m, c, o) in CASES.items()}}))}
    for name, (mode, c, o) in CASES.items():
        st = case_run(w, mode, c, o)
        dtype = np.float64 if mode == 2 else np.float32  # modes 0 and 1 hold an FP32 state
        for key in ("x", "v", "rho", "mass", "hsml"):
            a = getattr(st, key)
            assert np.array_equal(a.astype(dtype).astype(np.float64), a)
            out[f"{name}.{key}"] = a.astype(dtype)
        out[f"{name}.flag"] = st.flag.astype(np.int8)
        out[f"{name}.t_dt"] = np.array([st.t, st.dt])
    np.savez_compressed(os.path.join(HERE, "oracle_regression.npz"), **out)
    print(f"{w.n} particles, {len(CASES)} cases, {NSTEPS} steps")


if __name__ == "__main__":
    main()
