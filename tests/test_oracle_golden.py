"""The oracle against its committed regression vectors (tests/golden/,
written by make_oracle_regression.py): the stored inputs replayed for 10
steps in every stored case must give the stored states bit for bit.  The
vectors are the oracle's own (the reference ships none); the known-answer
tests pin what they should be, this test that they stay."""
import json
import os

import numpy as np
import pytest

import gfsph
import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_regression.npz")
DATA = np.load(GOLDEN)
META = json.loads(str(DATA["meta"]))


@pytest.mark.parametrize("case", sorted(META["cases"]))
def test_oracle_reproduces_its_regression_vectors(case):
    mode, const_extra, over = META["cases"][case]
    const = {int(k): v for k, v in META["const"].items()}
    const.update({int(k): v for k, v in const_extra.items()})
    p = gfsph.make_params(const, **{**META["options"], **over})
    z = DATA["z"]
    dx, dy = (float(a) for a in DATA["dxdy"])
    ny, nx = z.shape
    topol = oracle.initial_topol(z, dx, dy, const, deriv=p.dem_deriv, mode=mode)
    st = oracle.State(DATA["x"], DATA["v"], DATA["rho"], DATA["mass"], DATA["hsml"], topol, dt=p.dt)
    oracle.run(mode, p, nx, ny, dx, dy, st, META["nsteps"])
    for key in ("x", "v", "rho", "mass", "hsml"):
        want = DATA[f"{case}.{key}"].astype(np.float64)
        assert np.array_equal(getattr(st, key), want), (case, key)
    assert np.array_equal(st.flag, DATA[f"{case}.flag"].astype(np.int32))
    assert (st.t, st.dt) == tuple(DATA[f"{case}.t_dt"])
