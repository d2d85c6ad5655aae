"""Parity of the CUDA step (through the C ABI) with the CPU oracle.

Tolerances:
  - neighbour sets: bit-exact as sets, against the FP32 oracle;
  - one step, density, internal force: against the oracle in the GPU's own
    precision scheme (FP32 state and terms, FP64 sums; oracle mode 1), where
    the only freedom left is the order of the FP64 sums — relative error
    <= 1e-6 (in practice 0 or 1 ulp);
  - many steps: relative L2 of the depth field <= 1e-5 against oracle mode 1,
    and <= 2e-4 against the FP64 oracle (the reference's own FP32 build sits
    at ~2e-5..6e-5 from FP64 on these cases).
"""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def max_rel(a, b, floor=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def setup_pair(w, oracle_mod, **opts):
    """A GPU handle and an oracle state on identical inputs (same FP32 DEM rows)."""
    p = workloads.make_params(w, gfsph, **opts)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    st = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    return sim, st, p


def small_channel(n=6000, k=8):
    return workloads.fractal_channel(n_target=n, dem_k=k, cell=5.0)


@pytest.mark.parametrize("skf", [1, 2, 3])
def test_neighbour_sets_bit_exact(gfsph_lib, oracle_mod, skf):
    """The sets of grid_find against the oracle's literal restatement; with
    skf 2, 3 (support 3h) they include the drops of the reference's own grid.
    The first cloud has a few large smoothing lengths (coarse levels)."""
    rng = np.random.default_rng(11)
    clouds = []
    n = 4000
    x = rng.uniform(0, 60, size=(n, 2)).astype(np.float32) + np.float32(100.0)
    h = rng.uniform(0.5, 2.0, size=n).astype(np.float32)
    h[::400] *= np.float32(7.0)
    clouds.append((x, h))
    w = workloads.inclined_plane()
    clouds.append((w.x, w.hsml))
    wc = small_channel()
    clouds.append((wc.x, wc.hsml))
    for x, h in clouds:
        z = np.zeros((64, 64), np.float32)
        cell = float(np.ceil((x.max() + 10) / 63.0))
        p = gfsph.make_params({1: 9.8, 2: 2000, 3: 500, 5: 5, 9: 0.2, 10: 0.01, 15: 0.01}, skf=skf,
                              max_neighbours=256 if skf != 1 else 0)
        sim = gfsph.Sim(p, z, dx=cell, dy=cell)
        m = np.ones(x.shape[0], np.float32)
        sim.upload(x, np.zeros_like(x), m, m, h)
        rho = sim.density()
        off, idx = sim.neighbours()
        ref = oracle_mod.pairs(oracle_mod.MODE_FP32_DACC, p, x, h, mass=m, rho=m, want_rho=True)
        assert np.array_equal(off, ref["offsets"])
        assert np.array_equal(idx, ref["idx"])
        assert max_rel(rho, ref["rho"]) <= 1e-6
        sim.close()


def test_density_and_internal_force_match_oracle(gfsph_lib, oracle_mod):
    for w in (workloads.inclined_plane(), small_channel()):
        sim, st, p = setup_pair(w, oracle_mod)
        rho_g = sim.density()
        ref = oracle_mod.pairs(oracle_mod.MODE_FP32_DACC, p, w.x, w.hsml, mass=w.mass, rho=w.rho,
                               want_sets=False, want_rho=True, want_force=True)
        assert max_rel(rho_g, ref["rho"]) <= 1e-6
        sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
        f_g = sim.internal_forces()
        scale = np.abs(ref["force"]).max()
        assert np.abs(f_g - ref["force"]).max() <= 1e-6 * scale
        sim.close()


@pytest.mark.parametrize("case", ["plane", "channel_erosion"])
def test_one_step_matches_oracle(gfsph_lib, oracle_mod, case):
    w = workloads.inclined_plane() if case == "plane" else small_channel()
    sim, st, p = setup_pair(w, oracle_mod)
    sim.step(1)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, 1)
    assert np.array_equal(g["flag"], st.flag)
    for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
        err = max_rel(g[key], ref, floor=1e-3)
        assert err <= 1e-6, (key, err)
    t, dt = sim.time()
    assert abs(dt - st.dt) <= 1e-7 * st.dt
    sim.close()


def test_many_steps_inclined_plane(gfsph_lib, oracle_mod):
    w = workloads.inclined_plane()
    sim, st1, p = setup_pair(w, oracle_mod)
    st2 = st1.copy()
    nsteps = 200
    sim.step(nsteps)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st1, nsteps)
    oracle_mod.run(oracle_mod.MODE_FP64, p, nx, ny, w.dx, w.dy, st2, nsteps)
    assert rel_l2(g["rho"], st1.rho) <= 1e-5
    assert rel_l2(g["x"], st1.x) <= 1e-6
    assert rel_l2(g["rho"], st2.rho) <= 2e-4
    assert np.array_equal(g["mass"], w.mass)  # no erosion: volume exactly conserved
    sim.close()


def test_erosion_and_dem_rows_match_oracle(gfsph_lib, oracle_mod):
    w = small_channel()
    sim, st, p = setup_pair(w, oracle_mod)
    nsteps = 20
    sim.step(nsteps)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
    t = st.topol.reshape(ny, nx, 16)
    assert rel_l2(g["mass"], st.mass) <= 1e-6
    assert rel_l2(g["rho"], st.rho) <= 1e-5
    eroded = sim.raster(gfsph.RASTER_ERODED)
    assert eroded.max() > 0
    assert np.abs(eroded - t[..., 13]).max() <= 1e-6 + 1e-5 * t[..., 13].max()
    assert np.abs(sim.raster(gfsph.RASTER_Z) - t[..., 0]).max() <= 1e-3
    assert np.abs(sim.raster(gfsph.RASTER_AVAILABLE) - t[..., 14]).max() <= 1e-5
    sim.close()


EROSION_LAWS = {
    2: {17: 2650.0, 18: 1000.0, 21: 2, 22: 0.05, 23: 0.6},
    3: {17: 2650.0, 18: 1000.0, 21: 3, 22: 2e-3, 23: 500.0, 24: 0.1, 25: 0.5},
}


@pytest.mark.parametrize("law,rheo", [(2, "frictional_voellmy"), (2, "curvature"), (2, "mu_I_8"),
                                      (3, "frictional_voellmy"), (3, "hb_23_m1")])
def test_erosion_laws_2_and_3_match_oracle(gfsph_lib, oracle_mod, law, rheo):
    """Erosion law 2 (Get_Erosion_Rate_SW, SPH_SW_2019.f90:10332-10356): the
    rate C22 C23 |v| tan(theta - theta_e) from the bed angle along the flow
    and the equilibrium angle of the friction law's tanfi; law 3 (:10357-10376):
    C22 (Taub - Tauf) / dens_bar_eff from the basal shear of the friction
    after the reversal filter.  1 and 20 steps of the channel release against
    the oracle, mass and DEM rows included."""
    w = small_channel()
    w.const = {**w.const, **RHEOLOGIES[rheo], **EROSION_LAWS[law]}
    sim, st, p = setup_pair(w, oracle_mod)
    ny, nx = w.z.shape
    for nsteps in (1, 19):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps, rel_l2(g[key], ref))
    assert g["mass"].sum() > w.mass.sum() * 1.001
    t = st.topol.reshape(ny, nx, 16)
    eroded = sim.raster(gfsph.RASTER_ERODED)
    assert np.abs(eroded - t[..., 13]).max() <= 1e-6 + 1e-5 * t[..., 13].max()
    sim.close()


def test_rasters_match_oracle(gfsph_lib, oracle_mod):
    w = small_channel()
    sim, st, p = setup_pair(w, oracle_mod)
    ny, nx = w.z.shape
    sim.hazard_reset()
    haz = oracle_mod.Hazard(nx, ny, w.dx, w.dy)
    for _ in range(3):
        sim.step(5)
        g = sim.download()
        sim.hazard_sample()
        haz.sample(g["x"], g["v"], g["rho"], g["flag"])
    idw = sim.raster(gfsph.RASTER_DEPTH_IDW)
    ref = oracle_mod.raster_idw(nx, ny, w.dx, w.dy, g["x"], g["rho"], g["flag"])
    assert np.abs(idw - ref).max() <= 1e-5 * max(ref.max(), 1.0)
    cnt = sim.raster(gfsph.RASTER_COUNT).reshape(-1)
    assert np.array_equal(cnt.astype(np.int64), haz.cnt)
    assert np.array_equal(sim.raster(gfsph.RASTER_MAX_DEPTH).reshape(-1), haz.acc[:, 1].astype(np.float32))
    assert np.array_equal(sim.raster(gfsph.RASTER_MAX_VEL).reshape(-1), haz.acc[:, 3].astype(np.float32))
    sh = sim.raster(gfsph.RASTER_SUM_DEPTH).reshape(-1)
    assert np.abs(sh - haz.acc[:, 0]).max() <= 1e-5 * haz.acc[:, 0].max()
    sim.close()


def test_capacity_growth_gives_identical_results(gfsph_lib, oracle_mod):
    w = small_channel()
    sim_a, _, _ = setup_pair(w, oracle_mod)
    sim_b, _, _ = setup_pair(w, oracle_mod, max_neighbours=4)
    sim_a.step(6)
    sim_b.step(6)
    a, b = sim_a.download(), sim_b.download()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    sim_a.close()
    sim_b.close()


def test_runs_are_deterministic(gfsph_lib, oracle_mod):
    w = small_channel()
    outs = []
    for _ in range(2):
        sim, _, _ = setup_pair(w, oracle_mod)
        sim.step(12)
        outs.append(sim.download())
        sim.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_t_end_stops_the_loop(gfsph_lib, oracle_mod):
    w = workloads.inclined_plane()
    sim, _, _ = setup_pair(w, oracle_mod)
    st, t, done = sim.step(100, t_end=0.0499)
    assert st == gfsph.T_END_REACHED
    assert done == 5 and abs(t - 0.05) < 1e-6
    sim.close()


def test_particles_leaving_the_dem_are_frozen(gfsph_lib, oracle_mod):
    w = workloads.inclined_plane()
    x = w.x.copy()
    v = w.v.copy()
    x[0] = (0.2, 1000.0)        # next to the west edge, moving out
    v[0] = (-30.0, 0.0)
    sim, st, p = setup_pair(w, oracle_mod)
    sim.upload(x, v, w.rho, w.mass, w.hsml)
    sim.step(3)
    g = sim.download()
    assert g["flag"][0] == 1 and g["flag"][1:].sum() == 0
    frozen = g["x"][0].copy()
    sim.step(3)
    assert np.array_equal(sim.download()["x"][0], frozen)
    sim.close()


def test_full_size_channel_properties(gfsph_lib, oracle_mod):
    """The benchmark workload at full size (~200k particles, 1024^2 DEM)."""
    w = workloads.fractal_channel()
    sim, st, p = setup_pair(w, oracle_mod)
    sim.step(5)
    g = sim.download()
    assert all(np.all(np.isfinite(g[k])) for k in ("x", "v", "rho", "mass", "hsml"))
    assert g["mass"].sum() >= w.mass.sum()
    off, idx = sim.neighbours()
    counts = np.diff(off)
    assert counts.min() > 0
    # symmetry: j in N(i) <=> i in N(j)
    src = np.repeat(np.arange(w.n), counts)
    a = np.sort(src.astype(np.int64) * w.n + idx)
    b = np.sort(idx.astype(np.int64) * w.n + src)
    assert np.array_equal(a, b)
    # sets equal to the FP32 oracle's at this size (positions of the 5th step)
    sim2, _, _ = setup_pair(w, oracle_mod)
    sim2.upload(g["x"], g["v"], g["rho"], g["mass"], g["hsml"])
    sim2.density()
    off2, idx2 = sim2.neighbours()
    ref = oracle_mod.pairs(oracle_mod.MODE_FP32, p, g["x"], g["hsml"])
    assert np.array_equal(off2, ref["offsets"]) and np.array_equal(idx2, ref["idx"])
    sim.close()
    sim2.close()


def test_profile_counts_launches(gfsph_lib, oracle_mod):
    w = small_channel()
    sim, _, _ = setup_pair(w, oracle_mod)
    n0 = sim.launch_count()
    sim.step(16)
    per_step = (sim.launch_count() - n0) / 16
    assert per_step >= 14
    sim.profile(True)
    sim.step(4)
    prof = sim.profile_read()
    assert prof["k_force_rk"][1] == 4 and prof["k_density"][1] == 4
    assert all(ms >= 0 for ms, _ in prof.values())
    sim.close()


def test_release_outside_the_dem_box_is_flagged_at_the_first_step(gfsph_lib, oracle_mod):
    """Check_Out_Domain at the start of time_integration_sph: a release that
    overhangs the DEM box loses the overhanging particles before the search."""
    w = workloads.fractal_channel(n_target=4000, dem_k=7, cell=5.0)
    assert (w.x[:, 1] < 0).any()
    sim, st, p = setup_pair(w, oracle_mod)
    sim.step(2)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, 2)
    assert np.array_equal(g["flag"], st.flag)
    out = w.x[:, 1] < 0
    assert g["flag"][out].all()
    assert np.array_equal(g["x"][out], w.x[out])
    assert max_rel(g["x"], st.x, floor=1e-3) <= 1e-6
    sim.close()


def test_big_smoothing_lengths_sets_and_density(gfsph_lib, oracle_mod):
    """Particles whose hsml is far above the rest (the thin-front stragglers)
    are searched on a separate list; their sets and sums must not change."""
    rng = np.random.default_rng(5)
    n = 6000
    x = (rng.uniform(0, 80, size=(n, 2)) + 50.0).astype(np.float32)
    h = rng.uniform(0.8, 1.2, size=n).astype(np.float32)
    big = rng.choice(n, 40, replace=False)
    h[big] = rng.uniform(4.0, 40.0, size=40).astype(np.float32)
    m = rng.uniform(0.5, 1.5, size=n).astype(np.float32)
    p = gfsph.make_params({1: 9.8, 2: 2000, 3: 500, 5: 5, 9: 0.2, 10: 0.01, 15: 0.01})
    sim = gfsph.Sim(p, np.zeros((64, 64), np.float32), dx=4.0, dy=4.0)
    sim.upload(x, np.zeros_like(x), np.ones(n, np.float32), m, h)
    rho = sim.density()
    off, idx = sim.neighbours()
    ref = oracle_mod.pairs(oracle_mod.MODE_FP32, p, x, h)
    assert np.array_equal(off, ref["offsets"]) and np.array_equal(idx, ref["idx"])
    ref1 = oracle_mod.pairs(oracle_mod.MODE_FP32_DACC, p, x, h, mass=m, rho=np.ones(n), want_sets=False,
                            want_rho=True, want_force=True)
    assert max_rel(rho, ref1["rho"]) <= 1e-6
    sim.upload(x, np.zeros_like(x), np.ones(n, np.float32), m, h)
    f = sim.internal_forces()
    assert np.abs(f - ref1["force"]).max() <= 1e-6 * np.abs(ref1["force"]).max()
    sim.close()


def test_big_smoothing_lengths_one_step(gfsph_lib, oracle_mod):
    w = small_channel()
    rng = np.random.default_rng(9)
    big = rng.choice(w.n, 25, replace=False)
    w.hsml = w.hsml.copy()
    w.hsml[big] *= np.float32(6.0)
    sim, st, p = setup_pair(w, oracle_mod)
    sim.step(1)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, 1)
    assert np.array_equal(g["flag"], st.flag)
    for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
        assert max_rel(g[key], ref, floor=1e-3) <= 1e-6, key
    sim.close()


def test_long_run_with_growing_front(gfsph_lib, oracle_mod):
    """400 steps of a small channel release: the front spreads, some hsml grow
    far above the mean and move to the big list; the run stays on the oracle."""
    w = workloads.fractal_channel(n_target=3000, dem_k=8, cell=5.0)
    sim, st, p = setup_pair(w, oracle_mod)
    nsteps = 400
    sim.step(nsteps)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
    assert g["hsml"].max() > 2.5 * g["hsml"].mean()
    assert rel_l2(g["rho"], st.rho) <= 1e-4
    assert rel_l2(g["x"], st.x) <= 1e-5
    assert rel_l2(g["mass"], st.mass) <= 1e-5
    sim.close()


def test_far_apart_releases_on_a_large_dem(gfsph_lib, oracle_mod):
    """Two small releases 6 km apart on a 5 km x 5 km DEM with 0.5 m smoothing
    lengths: the bounding box holds ~2.6e8 cells of the finest level, but only
    the occupied 32 x 8-cell blocks get cells.  Sets stay exact and one step
    matches the oracle."""
    rng = np.random.default_rng(21)
    nc = 1500
    parts = []
    for cx, cy in ((300.0, 300.0), (4700.0, 4700.0)):
        parts.append(np.stack([rng.uniform(cx, cx + 20.0, nc), rng.uniform(cy, cy + 20.0, nc)], 1))
    x = np.concatenate(parts).astype(np.float32)
    n = x.shape[0]
    h = rng.uniform(0.4, 0.6, n).astype(np.float32)
    h[rng.choice(n, 6, replace=False)] = np.float32(3.0)  # a coarse level as well
    rho = rng.uniform(0.5, 1.5, n).astype(np.float32)
    mass = (rho * np.float32(0.25)).astype(np.float32)
    z = np.zeros((1024, 1024), np.float32)
    w = workloads.Workload(name="far_apart", const=workloads.voellmy_const(0.2, 500.0), options=dict(
        pa_sph=2, nnps=2, sle=1, skf=1, average_velocity=1, ic_adapt=0, h_inf=0.01, dt=0.01, dem_deriv=1),
        z=z, dx=5.0, dy=5.0, x=x, v=np.zeros_like(x), rho=rho, mass=mass, hsml=h)
    sim, st, p = setup_pair(w, oracle_mod)
    sim.density()
    off, idx = sim.neighbours()
    ref = oracle_mod.pairs(oracle_mod.MODE_FP32, p, x, h)
    assert np.array_equal(off, ref["offsets"]) and np.array_equal(idx, ref["idx"])
    s = sim.stats()
    assert s["levels"] >= 2 and s["cells"] < 2_000_000
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(1)
    g = sim.download()
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, 1024, 1024, w.dx, w.dy, st, 1)
    for key, r in (("x", st.x), ("v", st.v), ("rho", st.rho), ("hsml", st.hsml)):
        assert max_rel(g[key], r, floor=1e-3) <= 1e-6, key
    sim.close()


@pytest.mark.parametrize("icpwp,fct,staged", [(3, 0, ""), (3, 1, ""), (1, 0, ""), (1, 1, ""), (1, 0, "nor"),
                                              (1, 1, "cos")])
def test_pore_water_pressure_matches_oracle(gfsph_lib, oracle_mod, icpwp, fct, staged):
    """icpwp = 3 (Get_Pwp_SW with one point): Uaux starts at pwp0rel * h,
    lowers the basal friction by 1 - pwp/h, and relaxes towards the depth
    change of every step.  icpwp = 1: u starts the same way and the RK45
    integrates its dissipation stage by stage (ExtForces_SW :8648-8652).
    ic_fct_dens = 1 adds the buoyancy factor of tanfi and the negative pwp
    bounds.  With the staged RK45 (nor_density, ic_cosTheta = 1) u's bound
    in each stage is the depth the previous stage left."""
    w = small_channel()
    extra = {13: 0.02, 14: 1.0}
    if fct:
        extra.update({17: 2650.0, 18: 1000.0, 19: 0.5, 20: 1})
    if staged == "cos":
        extra[16] = 1.0
    w.const = {**w.const, **extra}
    kw = {"nor_density": 1} if staged == "nor" else {}
    sim, st, p = setup_pair(w, oracle_mod, icpwp=icpwp, pwp0rel=0.8, **kw)
    assert np.array_equal(sim.pwp(), (np.float32(0.8) * (w.rho * np.float32(1.0))).astype(np.float32))
    ny, nx = w.z.shape
    for nsteps in (1, 29):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps)
        assert rel_l2(sim.pwp(), st.pwp) <= tol
    # the friction really is lowered: without pore pressure the flow is slower
    sim0, st0, _ = setup_pair(w, oracle_mod, **kw)
    sim0.step(30)
    v0 = np.hypot(*sim0.download()["v"].T).mean()
    assert np.hypot(*g["v"].T).mean() > v0
    sim.close()
    sim0.close()


RHEOLOGIES = {
    "bingham": {5: 4, 6: 500.0, 7: 50.0, 3: 0.0, 9: 0.0},
    "frictional_voellmy": {5: 5},
    "coulomb_cf": {5: 6, 3: -200.0},
    "curvature": {5: 7},
    "mu_I_8": {5: 8, 3: 1.0, 6: 0.5, 7: 2.0, 9: 0.25},
    "mu_I_26": {5: 26, 3: 0.5, 6: 0.5, 7: 1.0, 9: 0.25},
    "mu_I_27": {5: 27, 3: 0.6, 6: 0.5, 7: 0.3, 9: 0.2},
    "manning_1": {5: 1, 3: 0.05},
    "laminar_2": {5: 2, 7: 5000.0},
    "bagnold_11": {5: 11, 3: 0.05},
    "hb_23_m1": {5: 23, 6: 3000.0, 7: 1000.0, 8: 1.0},
    "hb_23_m2": {5: 23, 6: 3000.0, 7: 1000.0, 8: 2.0},
    "hb_23_m05": {5: 23, 6: 3000.0, 7: 1000.0, 8: 0.5},
    "hb_23_m033": {5: 23, 6: 3000.0, 7: 1000.0, 8: 0.333333},
    "hb_24": {5: 24, 6: 3000.0, 7: 1000.0, 8: 0.5},
    "hb_25": {5: 25, 6: 3000.0, 7: 1000.0, 8: 0.5},
}


@pytest.mark.parametrize("rheo", sorted(RHEOLOGIES))
def test_rheologies_match_oracle(gfsph_lib, oracle_mod, rheo):
    """Every basal friction law on the path, 1 and 20 steps of the channel
    release against the oracle in the GPU's precision scheme."""
    w = small_channel()
    w.const = {**w.const, **RHEOLOGIES[rheo]}
    sim, st, p = setup_pair(w, oracle_mod)
    ny, nx = w.z.shape
    for nsteps in (1, 19):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps)
    sim.close()


def test_eroded_soil_bingham_matches_oracle(gfsph_lib, oracle_mod):
    """nfric 3 (SPH_SW_2019.f90:9443-9489) with Hungr erosion: the mass a
    particle gains by erosion, (m - m0)/m with m0 its mass at upload, turns
    on and scales its Bingham friction; 1 and 40 steps against the oracle,
    with the soil fraction past the 0.01 threshold for part of the flow.  A
    massless particle is refused at upload (the reference stops there)."""
    w = small_channel()
    w.const = {**w.const, 5: 3, 3: 2.0, 6: 3000.0, 7: 1000.0, 8: 0.05}
    sim, st, p = setup_pair(w, oracle_mod)
    m0 = st.mass.copy()
    ny, nx = w.z.shape
    for nsteps in (1, 39):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps, rel_l2(g[key], ref))
    soil = (g["mass"] - m0) / g["mass"]
    assert soil.max() > 0.05 and (soil > 0.01).mean() > 0.1, (soil.max(), (soil > 0.01).mean())
    mass = w.mass.copy()
    mass[7] = 0.0
    with pytest.raises(gfsph.GfsphError) as e:
        sim.upload(w.x, w.v, w.rho, mass, w.hsml)
    assert e.value.status == gfsph.ERR_ARG
    sim.close()


@pytest.mark.parametrize("rheo,staged", [("manning_1", "cos"), ("laminar_2", "nor"), ("bagnold_11", "cos"),
                                         ("hb_23_m2", "nor"), ("hb_25", "cos")])
def test_basal_laws_on_the_staged_path_match_oracle(gfsph_lib, oracle_mod, rheo, staged):
    """The same laws through the staged RK45 (ic_cosTheta = 1: g/sqrt(1 + |grad
    Z|^2) in the pressure and the friction; nor_density): 1 and 20 steps
    against the oracle."""
    w = small_channel()
    w.const = {**w.const, **RHEOLOGIES[rheo], **({16: 1.0} if staged == "cos" else {})}
    kw = {"nor_density": 1} if staged == "nor" else {}
    sim, st, p = setup_pair(w, oracle_mod, **kw)
    ny, nx = w.z.shape
    for nsteps in (1, 19):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps, rel_l2(g[key], ref))
    sim.close()


def test_basal_laws_outside_the_path_are_refused(gfsph_lib):
    """basal_friction_Ext_SW stops for nfric 23 with m other than 1, 2, 1/3,
    1/2 and for a yield stress below 1e-32 (SPH_SW_2019.f90:9547-9550,
    :9596-9598); nfric 24/25 with m <= 0 would divide by zero at rest; nfric
    9, 10, 22 and 201-203 are not on the path."""
    w = small_channel(n=500, k=6)
    cases = [({5: 23, 6: 3000.0, 7: 1000.0, 8: 0.7}, gfsph.ERR_UNSUPPORTED),
             ({5: 23, 6: 0.0, 7: 1000.0, 8: 1.0}, gfsph.ERR_ARG),
             ({5: 24, 6: 3000.0, 7: 1000.0, 8: 0.0}, gfsph.ERR_ARG),
             ({5: 25, 6: 3000.0, 7: 1000.0, 8: -1.0}, gfsph.ERR_ARG)]
    cases += [({5: nf}, gfsph.ERR_UNSUPPORTED) for nf in (9, 10, 22, 201)]
    # erosion law 2 needs a frictional law's tanfi, laws 2 and 3 the two densities; law 4 does not exist
    cases += [({5: 4, 6: 500.0, 7: 50.0, 17: 2650.0, 18: 1000.0, 21: 2, 22: 0.05}, gfsph.ERR_UNSUPPORTED),
              ({21: 2, 22: 0.05, 17: 0.0, 18: 1000.0}, gfsph.ERR_ARG), ({21: 3, 22: 0.05}, gfsph.ERR_ARG),
              ({21: 4, 22: 0.05}, gfsph.ERR_UNSUPPORTED)]
    # grain crushing const(36), the solid-end laws const(43) and the late
    # Voellmy xi const(41) (Input_SW :1312-1325, ExtForces_SW :8424-8434)
    cases += [({36: 1.0}, gfsph.ERR_UNSUPPORTED), ({43: 1.0}, gfsph.ERR_UNSUPPORTED),
              ({41: 300.0}, gfsph.ERR_UNSUPPORTED)]
    # icpwp 2 (a finite-difference column per particle) is not built
    for kw in ({"icpwp": 2}, {"icpwp": 4}):
        p = workloads.make_params(w, gfsph, pwp0rel=0.5, **kw)
        with pytest.raises(gfsph.GfsphError) as e:
            gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        assert e.value.status == gfsph.ERR_UNSUPPORTED, kw
    for const, status in cases:
        w.const = {**small_channel(n=500, k=6).const, **const}
        p = workloads.make_params(w, gfsph)
        with pytest.raises(gfsph.GfsphError) as e:
            gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        assert e.value.status == status, const


@pytest.mark.parametrize("skf", [2, 3])
def test_three_h_kernels_match_oracle(gfsph_lib, oracle_mod, skf):
    """skf 2 (Gaussian) and 3 (quintic), support 3h, on the channel release:
    one step and 20 steps against the oracle in the GPU's precision scheme
    (the pair sets follow the reference's own grid every step)."""
    w = small_channel()
    sim, st, p = setup_pair(w, oracle_mod, skf=skf, max_neighbours=256)
    ny, nx = w.z.shape
    for nsteps in (1, 19):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps, rel_l2(g[key], ref))
    sim.close()


STAGED = {
    "nor_density": ({}, {"nor_density": 1}),
    "cos_theta": ({16: 1.0}, {}),
    "both_pa1": ({16: 1.0}, {"nor_density": 1, "pa_sph": 1}),
}


@pytest.mark.parametrize("case", sorted(STAGED))
def test_staged_pressure_options_match_oracle(gfsph_lib, oracle_mod, case):
    """nor_density (sum_density_Tools :1841-1846) and ic_cosTheta = 1
    (IntForces_SW :6775-6783, Get_Grav_Ext_SW :9264-9270): the pressure then
    changes from stage to stage and the step runs stage by stage; 1 and 20
    steps of the channel release (with Hungr erosion and the curvature term)
    against the oracle in the GPU's precision scheme."""
    const, opts = STAGED[case]
    w = small_channel()
    w.const = {**w.const, **const, 5: 7}
    sim, st, p = setup_pair(w, oracle_mod, **opts)
    ny, nx = w.z.shape
    for nsteps in (1, 19):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        tol = 1e-6 if nsteps == 1 else 1e-5
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
            assert rel_l2(g[key], ref) <= tol, (key, nsteps, rel_l2(g[key], ref))
    t, dt = sim.time()
    assert abs(t - st.t) <= 1e-6 * st.t
    sim.close()


def test_staged_options_change_the_flow(gfsph_lib, oracle_mod):
    """The options are live: 20 steps with nor_density or ic_cosTheta = 1
    end elsewhere than the plain run."""
    out = {}
    for case, (const, opts) in [("plain", ({}, {})), *STAGED.items()]:
        wc = workloads.fractal_channel(n_target=6000, dem_k=8, cell=5.0)
        wc.const = {**wc.const, **const}
        sim, _, _ = setup_pair(wc, oracle_mod, **opts)
        sim.step(20)
        out[case] = sim.download()
        sim.close()
    for case in STAGED:
        assert rel_l2(out[case]["x"], out["plain"]["x"]) > 1e-6, case


def test_normalised_density_and_forces_match_oracle(gfsph_lib, oracle_mod):
    """One normalised sum_density_Tools call on the uploaded depths and the
    internal force that follows, against the oracle (mode 1)."""
    for w in (workloads.inclined_plane(), small_channel()):
        sim, st, p = setup_pair(w, oracle_mod, nor_density=1)
        rho_g = sim.density()
        ref = oracle_mod.pairs(oracle_mod.MODE_FP32_DACC, p, w.x, w.hsml, mass=w.mass, rho=w.rho,
                               want_sets=False, want_rho=True, want_force=True)
        assert max_rel(rho_g, ref["rho"]) <= 1e-6
        sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
        f_g = sim.internal_forces()
        scale = np.abs(ref["force"]).max()
        assert np.abs(f_g - ref["force"]).max() <= 1e-6 * scale
        sim.close()


def test_staged_profile_counts_launches(gfsph_lib, oracle_mod):
    w = small_channel()
    sim, _, _ = setup_pair(w, oracle_mod, nor_density=1)
    sim.profile(True)
    sim.step(3)
    prof = sim.profile_read()
    # per step: 5 normalised sums, k_stage_begin + 3 stages + the last, 4 internal forces
    assert prof["k_norm"][1] == 15 and prof["k_stage"][1] == 15 and prof["k_iforce"][1] == 12
    assert "k_force_rk" not in prof or prof["k_force_rk"][1] == 0
    sim.close()


@pytest.mark.parametrize("mode", [1, 2, 4, 10])
def test_adaptive_dt_modes_match_oracle(gfsph_lib, oracle_mod, mode):
    """Adaptive_dt_sph_SW modes 1, 2, 4 (DEM cell diagonal / |v|) and 10
    (the smaller of 1 and 4) over 30 steps of the channel release: the same
    dt sequence and state as the oracle in the GPU's precision scheme."""
    w = small_channel()
    sim, st, p = setup_pair(w, oracle_mod, ic_adapt=mode, dt=0.05)
    ny, nx = w.z.shape
    for nsteps in (1, 9, 20):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        t, dt = sim.time()
        assert abs(dt - st.dt) <= 1e-6 * st.dt, (nsteps, dt, st.dt)
        assert abs(t - st.t) <= 1e-6 * st.t, (nsteps, t, st.t)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho)):
            assert rel_l2(g[key], ref) <= 1e-5, (key, nsteps)
    sim.close()


@pytest.mark.parametrize("tune", [(2.5, 3.0), (3.0, 4.0), (2.0, 1.0), (1.0, 2.0)])
def test_search_tunables_keep_sets_and_results(gfsph_lib, oracle_mod, tune):
    """Other level bounds and cell sizes: the same neighbour sets, and one step
    still on the oracle."""
    w = small_channel()
    rng = np.random.default_rng(4)
    w.hsml = w.hsml.copy()
    w.hsml[rng.choice(w.n, 20, replace=False)] *= np.float32(5.0)
    sim, st, p = setup_pair(w, oracle_mod)
    sim.set_search(*tune)
    assert sim.get_search() == tune
    sim.density()
    off, idx = sim.neighbours()
    ref = oracle_mod.pairs(oracle_mod.MODE_FP32, p, w.x, w.hsml)
    assert np.array_equal(off, ref["offsets"]) and np.array_equal(idx, ref["idx"])
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(1)
    g = sim.download()
    ny, nx = w.z.shape
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, 1)
    for key, r in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
        assert max_rel(g[key], r, floor=1e-3) <= 1e-6, key
    sim.close()


def test_autotune_keeps_the_state(gfsph_lib, oracle_mod):
    w = small_channel()
    sim, _, _ = setup_pair(w, oracle_mod)
    sim.step(3)
    before = sim.download()
    t_before = sim.time()
    z_before = sim.raster(gfsph.RASTER_Z)
    lf, cd, ms = sim.autotune(steps=4)
    assert (lf, cd) == sim.get_search() and ms > 0
    after = sim.download()
    for k in before:
        assert np.array_equal(before[k], after[k]), k
    assert sim.time() == t_before
    assert np.array_equal(z_before, sim.raster(gfsph.RASTER_Z))
    sim.step(2)  # still steps
    sim.close()
