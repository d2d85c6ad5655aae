"""Parity pinned on the reference's own example and on the configurations at
their own sizes, through the C ABI against the oracle in the GPU's precision
scheme (FP32 state and terms, FP64 sums: oracle mode 1).

  - Picacho (the reference's shipped example, tests/golden/picacho): the
    inputs parsed by gfsph_run exactly as the Fortran driver would read them,
    100 steps (t = 17.9 s, adaptive dt, nnps 4, nfric 7 with v^2/R, basal
    pore pressure icpwp 3): every state array and the dt sequence identical
    bit for bit;
  - the 200k-particle fractal-channel workload: one step with every particle
    within 1e-6 (relative, the only freedom being the order of the FP64
    sums), then three steps within 1e-6 relative L2;
  - skf 4 (Wendland C2, kernel_TOOLS My_SPH_Tools_2019.f90:2157-2177):
    neighbour sets bit-exact, density, one step and 20 steps.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "deslizamientos-y-flujos_b200", "gfsph_run")
GOLDEN = os.path.join(ROOT, "tests", "golden", "picacho")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def max_rel(a, b, floor=1e-3):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def picacho(tmp_path):
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)
    import make_fixture
    make_fixture.extract(str(tmp_path))
    dump = os.path.join(str(tmp_path), "picacho.dump")
    out = subprocess.run([RUN, "Picacho", "--dir", str(tmp_path), "--dump", dump], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return workloads.from_driver_dump(dump, gfsph)


def test_picacho_example_matches_oracle_bit_for_bit(gfsph_lib, oracle_mod, tmp_path):
    w, p = picacho(tmp_path)
    assert w.n == 851 and w.z.shape == (291, 442)
    assert (p.nnps, p.icpwp, p.ic_adapt, int(p.cst[4] + 0.01)) == (4, 3, 1, 7)
    xmin, ymin = w.meta["xmin"], w.meta["ymin"]
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    sim = gfsph.Sim(p, w.z, xmin=xmin, ymin=ymin, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    st = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    ny, nx = w.z.shape
    for chunk in (1, 9, 40, 50):  # 1, 10, 50 and 100 steps
        sim.step(chunk)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, chunk, xmin=xmin, ymin=ymin)
        g = sim.download()
        t, dt = sim.time()
        assert np.float32(dt) == np.float32(st.dt), chunk
        assert abs(t - st.t) <= 1e-12 * st.t, chunk
        assert np.array_equal(g["flag"], st.flag), chunk
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
            assert np.array_equal(g[key], ref.astype(np.float32)), (key, chunk, max_rel(g[key], ref))
        assert np.array_equal(sim.pwp(), st.pwp.astype(np.float32)), chunk
    assert st.t > 17.8  # 100 steps of the adaptive dt
    sim.close()


def test_full_size_channel_state_matches_oracle(gfsph_lib, oracle_mod):
    """The benchmark workload itself: 200,011 particles on the 1024^2 DEM."""
    w = workloads.fractal_channel()
    assert 199_000 < w.n < 201_000
    p = workloads.make_params(w, gfsph)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    st = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    ny, nx = w.z.shape
    for nsteps, total in ((1, 1), (2, 3)):
        sim.step(nsteps)
        oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, nsteps)
        g = sim.download()
        assert np.array_equal(g["flag"], st.flag)
        for key, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("mass", st.mass), ("hsml", st.hsml)):
            if total == 1:
                assert max_rel(g[key], ref) <= 1e-6, (key, max_rel(g[key], ref))
            else:
                assert rel_l2(g[key], ref) <= 1e-6, (key, rel_l2(g[key], ref))
        t, dt = sim.time()
        assert abs(dt - st.dt) <= 1e-7 * st.dt
    # the eroded DEM rows: elevation and erodible depth
    for kind, row in ((gfsph.RASTER_Z, 0), (gfsph.RASTER_AVAILABLE, 14)):
        got = sim.raster(kind).reshape(-1)
        assert np.abs(got - st.topol[:, row]).max() <= 1e-5 * max(1.0, np.abs(st.topol[:, row]).max())
    sim.close()


def test_wendland_kernel_matches_oracle(gfsph_lib, oracle_mod):
    """skf 4 (Wendland C2, support 2h) on the channel release."""
    w = workloads.fractal_channel(n_target=6000, dem_k=8, cell=5.0)
    p = workloads.make_params(w, gfsph, skf=4)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    rho = sim.density()
    off, idx = sim.neighbours()
    ref = oracle_mod.pairs(oracle_mod.MODE_FP32_DACC, p, w.x, w.hsml, mass=w.mass, rho=w.rho, want_rho=True,
                           want_force=True)
    assert np.array_equal(off, ref["offsets"]) and np.array_equal(idx, ref["idx"])
    assert max_rel(rho, ref["rho"], floor=1e-6) <= 1e-6
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    f = sim.internal_forces()
    assert np.abs(f - ref["force"]).max() <= 1e-6 * np.abs(ref["force"]).max()
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    st = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
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
