"""The largest configuration at full size: a 4096^2 DEM at 2 m with four
releases, ~4 million particles and the Bingham law.  One step is checked
against the serial oracle; over 12 steps, which the oracle would take minutes
for, the checks are the size-independent properties: volume conserved exactly
(no erosion), every state finite and inside the DEM box, smoothing lengths
updated, and a second handle on the same input giving bit-identical results."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu


def run(w, p, nsteps):
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(nsteps)
    out = sim.download(), sim.time(), sim.stats()
    sim.close()
    return out


def test_four_million_particles_bingham_multi_release(gfsph_lib):
    w = workloads.multi_release()
    assert 3_900_000 < w.n < 4_100_000
    p = workloads.make_params(w, gfsph)
    g, (t, dt), stats = run(w, p, 12)
    assert stats["active"] == w.n and stats["outside"] == 0
    assert np.array_equal(g["flag"], np.zeros(w.n, np.int32))
    for k in ("x", "v", "rho", "mass", "hsml"):
        assert np.all(np.isfinite(g[k])), k
    assert np.array_equal(g["mass"], w.mass)  # no erosion: every volume kept bit for bit
    assert not np.array_equal(g["hsml"], w.hsml)  # h_upgrade (sle 1) ran
    assert np.abs(g["v"]).max() > 0.0  # the releases started to move
    # adaptive dt grows by at most the single-precision factor 1.1 per step
    assert 0.0 < dt <= p.dt * 1.1 ** 12 * (1.0 + 1e-5) and t > 0.0
    g2, (t2, dt2), _ = run(w, p, 12)
    assert t2 == t and dt2 == dt
    for k in g:
        assert np.array_equal(g[k], g2[k]), k


def test_four_million_particles_one_step_matches_oracle(gfsph_lib, oracle_mod):
    """One step of the 4M-particle Bingham case against the serial oracle in
    the GPU's precision scheme (FP32 state, FP64 sums): every particle within
    1e-6 relative."""
    w = workloads.multi_release()
    p = workloads.make_params(w, gfsph)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(1)
    g = sim.download()
    t, dt = sim.time()
    sim.close()
    st = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    del topol
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, 1)
    assert np.array_equal(g["flag"], st.flag)
    for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
        ref = np.asarray(ref, np.float64)
        err = float(np.max(np.abs(g[key] - ref) / np.maximum(np.abs(ref), 1e-3)))
        assert err <= 1e-6, (key, err)
    assert abs(dt - st.dt) <= 1e-7 * st.dt
