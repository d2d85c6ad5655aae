"""The device adjoint of the step (gfsph_adjoint_*) against the oracle's FP64
forward-mode derivatives of the same run, along the rheology parameters,
the volumes, the initial positions and velocities, and random mixtures."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu

NSTEPS = 20


def case(oracle_mod, n=3000):
    w = workloads.fractal_channel(n_target=n, dem_k=8, cell=5.0, erosion=None)
    p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    return w, p, topol


def gpu_gradients(w, p, topol, gx, gv, gh, every=5):
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    adj = gfsph.Adjoint(sim, NSTEPS, every=every)
    final = sim.download()
    g = adj.backward(gx, gv, gh)
    after = sim.download()
    adj.close()
    sim.close()
    return g, final, after


def test_adjoint_matches_forward_mode_derivatives(gfsph_lib, oracle_mod):
    w, p, topol = case(oracle_mod)
    rng = np.random.default_rng(1)
    gx = rng.normal(size=(w.n, 2)).astype(np.float32)
    gv = rng.normal(size=(w.n, 2)).astype(np.float32)
    gh = rng.normal(size=w.n).astype(np.float32)
    g, final, after = gpu_gradients(w, p, topol, gx, gv, gh)
    for k in final:
        assert np.array_equal(final[k], after[k]), k  # the handle is left at the final state
    ny, nx = w.z.shape
    st0 = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)

    def directional(**seed):
        _, _, _, dx, dv, dh = oracle_mod.tangent(p, nx, ny, w.dx, w.dy, st0, NSTEPS, **seed)
        return float((gx * dx).sum() + (gv * dv).sum() + (gh * dh).sum())

    checks = {
        "tanfi": (directional(seed_mu=1.0), g["tanfi"]),
        "xi": (directional(seed_xi=1.0), g["xi"]),
    }
    dm = rng.normal(size=w.n) * w.mass
    checks["mass"] = (directional(seed_m=dm), float((g["mass"] * dm).sum()))
    dx0 = rng.normal(size=(w.n, 2))
    checks["x0"] = (directional(seed_x=dx0), float((g["x0"] * dx0).sum()))
    dv0 = rng.normal(size=(w.n, 2))
    checks["v0"] = (directional(seed_v=dv0), float((g["v0"] * dv0).sum()))
    for name, (ref, got) in checks.items():
        assert abs(got - ref) <= 2e-4 * abs(ref), (name, got, ref)


def test_checkpoint_interval_does_not_change_the_gradient(gfsph_lib, oracle_mod):
    w, p, topol = case(oracle_mod, n=1500)
    rng = np.random.default_rng(2)
    gx = rng.normal(size=(w.n, 2)).astype(np.float32)
    gv = rng.normal(size=(w.n, 2)).astype(np.float32)
    a, _, _ = gpu_gradients(w, p, topol, gx, gv, None, every=1)
    b, _, _ = gpu_gradients(w, p, topol, gx, gv, None, every=7)
    for k in ("x0", "v0", "mass"):
        assert np.allclose(a[k], b[k], rtol=1e-5, atol=1e-6 * np.abs(a[k]).max()), k
    assert abs(a["tanfi"] - b["tanfi"]) <= 1e-6 * abs(a["tanfi"])
    assert abs(a["xi"] - b["xi"]) <= 1e-6 * abs(a["xi"])


def test_adjoint_refuses_runs_outside_its_scope(gfsph_lib, oracle_mod):
    w = workloads.fractal_channel(n_target=1000, dem_k=8, cell=5.0)  # with erosion
    p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    with pytest.raises(gfsph.GfsphError) as e:
        gfsph.Adjoint(sim, 5)
    assert e.value.status == gfsph.ERR_UNSUPPORTED
    sim.close()
    # stage-dependent pressure (nor_density, ic_cosTheta = 1)
    w = workloads.fractal_channel(n_target=1000, dem_k=8, cell=5.0, erosion=None)
    for const, opts in (({}, {"nor_density": 1}), ({16: 1.0}, {})):
        w.const = {**w.const, **const}
        p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0, **opts)
        sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
        with pytest.raises(gfsph.GfsphError) as e:
            gfsph.Adjoint(sim, 5)
        assert e.value.status == gfsph.ERR_UNSUPPORTED
        sim.close()
    # a release that reaches past the DEM edge: particles leave the box
    w = workloads.fractal_channel(n_target=1000, dem_k=7, cell=5.0, erosion=None)
    p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    with pytest.raises(gfsph.GfsphError) as e:
        gfsph.Adjoint(sim, 5)
    assert e.value.status == gfsph.ERR_UNSUPPORTED
    sim.close()
