"""The Monte-Carlo ensemble through the C ABI: every member advanced by
gfsph_ensemble_step is bit-identical to the same realization run alone with
gfsph_step, and the exceedance raster is the fraction of members whose
sampled maximum depth exceeds the threshold."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu


def realizations(w, nreal, seed=7):
    """Parameters and particle sets of nreal realizations: mu ~ U(0.08, 0.30),
    xi ~ LogNormal(ln 400, 0.3), release depth scaled by U(0.2, 2.0) — the
    volume scale changes the depth and mass of every particle."""
    rng = np.random.default_rng(seed)
    params, parts = [], []
    for _ in range(nreal):
        c = dict(w.const)
        c[9] = float(rng.uniform(0.08, 0.30))
        c[3] = float(np.exp(rng.normal(np.log(400.0), 0.3)))
        scale = float(rng.uniform(0.2, 2.0))
        wr = workloads.Workload(**{**w.__dict__, "const": c})
        params.append(workloads.make_params(wr, gfsph))
        rho = (w.rho * scale).astype(np.float32)
        mass = (w.mass * scale).astype(np.float32)
        parts.append((w.x, w.v, rho, mass, w.hsml))
    return params, parts


def test_members_match_standalone_runs(gfsph_lib):
    w = workloads.fractal_channel(n_target=5000, dem_k=8, cell=5.0)
    params, parts = realizations(w, 4)
    ens = gfsph.Ensemble(params, w.z, dx=w.dx, dy=w.dy)
    for m, pr in zip(ens.members, parts):
        m.upload(*pr)
    st, done = ens.step(15)
    assert st == 0 and done == 15
    for r, (p, pr) in enumerate(zip(params, parts)):
        sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        sim.upload(*pr)
        sim.step(15)
        a, b = ens.members[r].download(), sim.download()
        for k in a:
            assert np.array_equal(a[k], b[k]), (r, k)
        ta, tb = ens.members[r].time(), sim.time()
        assert ta == tb
        assert np.array_equal(ens.members[r].raster(gfsph.RASTER_Z), sim.raster(gfsph.RASTER_Z))
        sim.close()
    ens.close()


def test_exceedance_is_the_member_fraction(gfsph_lib):
    w = workloads.fractal_channel(n_target=4000, dem_k=8, cell=5.0)
    params, parts = realizations(w, 5, seed=11)
    ens = gfsph.Ensemble(params, w.z, dx=w.dx, dy=w.dy)
    for m, pr in zip(ens.members, parts):
        m.upload(*pr)
    for _ in range(3):
        ens.step(5)
        ens.sample()
    thr = 1.0
    prob = ens.exceedance(thr)
    maxd = np.stack([m.raster(gfsph.RASTER_MAX_DEPTH) for m in ens.members])
    ref = (maxd > thr).sum(axis=0).astype(np.float32) / np.float32(len(params))
    assert np.array_equal(prob, ref)
    assert 0.0 < prob.max() <= 1.0
    ens.close()


def test_t_end_stops_every_member(gfsph_lib):
    w = workloads.inclined_plane()
    params, parts = realizations(w, 3, seed=3)
    ens = gfsph.Ensemble(params, w.z, dx=w.dx, dy=w.dy)
    for m, pr in zip(ens.members, parts):
        m.upload(*pr)
    st, done = ens.step(100, t_end=0.0499)
    assert st == gfsph.T_END_REACHED and done == 5
    for m in ens.members:
        assert abs(m.time()[0] - 0.05) < 1e-6
    ens.close()


def test_rejects_mixed_dem_derivatives(gfsph_lib):
    w = workloads.inclined_plane()
    p0 = workloads.make_params(w, gfsph)
    p1 = workloads.make_params(w, gfsph)
    p1.dem_deriv = 1 - p0.dem_deriv
    with pytest.raises(gfsph.GfsphError) as e:
        gfsph.Ensemble([p0, p1], w.z, dx=w.dx, dy=w.dy)
    assert e.value.status == gfsph.ERR_ARG


def test_members_match_the_oracle(gfsph_lib, oracle_mod):
    """Two members of an ensemble (sharing the DEM rows of member 0) against
    the oracle in the GPU's precision scheme: the first member and the last."""
    w = workloads.fractal_channel(n_target=3000, dem_k=8, cell=5.0)
    params, parts = realizations(w, 6, seed=3)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=params[0].dem_deriv, mode=oracle_mod.MODE_FP32)
    ens = gfsph.Ensemble(params, w.z, dx=w.dx, dy=w.dy)
    for m, pr in zip(ens.members, parts):
        m.upload(*pr)
    ens.step(10)
    ny, nx = w.z.shape
    for r in (0, 5):
        x, v, rho, mass, hsml = parts[r]
        st = oracle_mod.State(x, v, rho, mass, hsml, topol, dt=params[r].dt)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, params[r], nx, ny, w.dx, w.dy, st, 10)
        g = ens.members[r].download()
        assert np.array_equal(g["flag"], st.flag)
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass)):
            ref = np.asarray(ref, np.float64)
            err = np.linalg.norm(g[key] - ref) / np.linalg.norm(ref)
            assert err <= 1e-5, (r, key, err)
    ens.close()
