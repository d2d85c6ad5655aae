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
    """The device adjoint along the tangents of the rheology parameters, the
    volumes and the initial positions and velocities, against two exact
    forward-mode references: the derivative of the single-precision
    trajectory the device computes (the oracle's FP32 step carried on dual
    numbers, whose values equal the device state bit for bit), within 2e-5 of
    the sum of the direction's per-particle terms; and that of the FP64
    trajectory, within 2e-4."""
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

    def directional(single, **seed):
        _, _, _, dx, dv, dh = oracle_mod.tangent(p, nx, ny, w.dx, w.dy, st0, NSTEPS, single=single, **seed)
        return float((gx * dx).sum() + (gv * dv).sum() + (gh * dh).sum())

    dm = rng.normal(size=w.n) * w.mass
    dx0 = rng.normal(size=(w.n, 2))
    dv0 = rng.normal(size=(w.n, 2))
    checks = {  # name: (seed, the device's directional derivative, the scale of its terms)
        "tanfi": (dict(seed_mu=1.0), g["tanfi"], abs(g["tanfi"])),
        "xi": (dict(seed_xi=1.0), g["xi"], abs(g["xi"])),
        "mass": (dict(seed_m=dm), float((g["mass"] * dm).sum()), float(np.abs(g["mass"] * dm).sum())),
        "x0": (dict(seed_x=dx0), float((g["x0"] * dx0).sum()), float(np.abs(g["x0"] * dx0).sum())),
        "v0": (dict(seed_v=dv0), float((g["v0"] * dv0).sum()), float(np.abs(g["v0"] * dv0).sum())),
    }
    for name, (seed, got, scale) in checks.items():
        ref32 = directional(True, **seed)
        ref64 = directional(False, **seed)
        print(f"{name}: device {got:.9g} single-trajectory {ref32:.9g} FP64 {ref64:.9g} "
              f"|dev-32|/scale {abs(got - ref32) / scale:.2e} |dev-64|/|64| {abs(got - ref64) / abs(ref64):.2e}")
        assert abs(got - ref32) <= 2e-5 * scale, (name, got, ref32, scale)
        assert abs(got - ref64) <= 2e-4 * abs(ref64), (name, got, ref64)


@pytest.mark.parametrize("every", [1, 7])
def test_adjoint_with_the_smoothing_length_update(gfsph_lib, oracle_mod, every):
    """sle 1: every step ends with hsml' = 2 sqrt(m/h) (h_upgrade,
    SPH_MAIN_2019.f90:2925-2931), so the next step's kernel values depend on
    the depths and volumes of this one.  The device adjoint against the
    single-precision trajectory's exact derivative (within 2e-5 of the
    direction's scale) and the FP64 one (within 2e-4 of it), along tanfi, xi,
    the volumes and the initial positions and velocities; checkpoints every
    step or every 7 (the smoothing lengths are part of every stored state)."""
    w = workloads.fractal_channel(n_target=3000, dem_k=8, cell=5.0, erosion=None)
    p = workloads.make_params(w, gfsph, sle=1, ic_adapt=0)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    rng = np.random.default_rng(11)
    gx = rng.normal(size=(w.n, 2)).astype(np.float32)
    gv = rng.normal(size=(w.n, 2)).astype(np.float32)
    gh = rng.normal(size=w.n).astype(np.float32)
    g, final, _ = gpu_gradients(w, p, topol, gx, gv, gh, every=every)
    assert np.abs(final["hsml"] - w.hsml).max() > 1e-3  # the smoothing lengths did change
    ny, nx = w.z.shape
    st0 = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)

    def directional(single, **seed):
        _, _, _, dx, dv, dh = oracle_mod.tangent(p, nx, ny, w.dx, w.dy, st0, NSTEPS, single=single, **seed)
        return float((gx * dx).sum() + (gv * dv).sum() + (gh * dh).sum())

    dm = rng.normal(size=w.n) * w.mass
    dx0 = rng.normal(size=(w.n, 2))
    dv0 = rng.normal(size=(w.n, 2))
    for name, seed, got, scale in (
            ("tanfi", dict(seed_mu=1.0), g["tanfi"], abs(g["tanfi"])),
            ("xi", dict(seed_xi=1.0), g["xi"], abs(g["xi"])),
            ("mass", dict(seed_m=dm), float((g["mass"] * dm).sum()), float(np.abs(g["mass"] * dm).sum())),
            ("x0", dict(seed_x=dx0), float((g["x0"] * dx0).sum()), float(np.abs(g["x0"] * dx0).sum())),
            ("v0", dict(seed_v=dv0), float((g["v0"] * dv0).sum()), float(np.abs(g["v0"] * dv0).sum()))):
        ref32 = directional(True, **seed)
        ref64 = directional(False, **seed)
        print(f"sle 1, {name}: device {got:.9g} single-trajectory {ref32:.9g} FP64 {ref64:.9g} "
              f"|dev-32|/scale {abs(got - ref32) / scale:.2e}")
        assert abs(got - ref32) <= 2e-5 * scale, (name, got, ref32, scale)
        assert abs(got - ref64) <= 2e-4 * scale, (name, got, ref64, scale)


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


def test_twenty_directions_match_central_differences(gfsph_lib, oracle_mod):
    """20 seeded random directions in (tanfi, xi, the volumes) at once.  The
    device adjoint's directional derivative against (1) the exact derivative
    of the single-precision trajectory the device computes (the oracle's FP32
    step on dual numbers), within 1e-6 of the sum of the magnitudes of the
    direction's terms (the parameters' and every particle's), and (2) central
    differences of the FP64 oracle with relative steps of 1e-4, within 1e-4
    of that sum.  Relative to the directional derivative itself the FP64
    differences stay within 5e-4: the FP32 trajectory departs from the FP64
    one by ~1e-4 in the volume terms, and the terms of a random direction can
    cancel (e.g. -5.6 - 0.3 - 2.2 = -8.1 against a scale of 12).

    Directions in the initial positions and velocities are checked against
    the exact FP64 tangent instead (the test above): central differences are
    ill-posed there.  The release starts at rest, where the Coulomb friction's
    direction v/|v| is not differentiable (a step in v0 switches the reversal
    filter from its at-rest to its sliding branch once |v| > 1e-5), and the
    lattice puts pairs within ~1e-5 m of q = 1, where the reference's cubic
    spline jumps by 5e-8 W (its 2./3. is a single-precision literal in the
    FP64 build too, kernel_TOOLS My_SPH_Tools_2019.f90:2101), so steps of
    positions cross the jump."""
    w, p, topol = case(oracle_mod)
    rng = np.random.default_rng(20)
    gx = rng.normal(size=(w.n, 2)).astype(np.float32)
    gv = rng.normal(size=(w.n, 2)).astype(np.float32)
    gh = rng.normal(size=w.n).astype(np.float32)
    g, _, _ = gpu_gradients(w, p, topol, gx, gv, gh)
    ny, nx = w.z.shape
    eps = 1e-4
    m64 = w.mass.astype(np.float64)
    st0 = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)

    def loss(q, mass):
        st = oracle_mod.State(w.x, w.v, w.rho, mass, w.hsml, topol, dt=p.dt)
        oracle_mod.run(oracle_mod.MODE_FP64, q, nx, ny, w.dx, w.dy, st, NSTEPS)
        return float((gx * st.x).sum() + (gv * st.v).sum() + (gh * st.rho).sum())

    worst = worst_scaled = worst32 = 0.0
    for k in range(20):
        u = rng.normal(size=2)
        dm = rng.normal(size=w.n) * w.mass
        qp = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
        qm = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
        for idx, ui in ((8, u[0]), (2, u[1])):  # tanfi = const(9), xi = const(3)
            qp.cst[idx] = p.cst[idx] * (1 + eps * ui)
            qm.cst[idx] = p.cst[idx] * (1 - eps * ui)
        fd = (loss(qp, m64 + eps * dm) - loss(qm, m64 - eps * dm)) / (2 * eps)
        # the parameters travel as FP32: the steps actually taken
        dmu = (float(qp.cst[8]) - float(qm.cst[8])) / (2 * eps)
        dxi = (float(qp.cst[2]) - float(qm.cst[2])) / (2 * eps)
        _, _, _, tx, tv, th = oracle_mod.tangent(p, nx, ny, w.dx, w.dy, st0, NSTEPS, seed_mu=dmu, seed_xi=dxi,
                                                 seed_m=dm, single=True)
        t32 = float((gx * tx).sum() + (gv * tv).sum() + (gh * th).sum())
        terms = [g["tanfi"] * dmu, g["xi"] * dxi, float((g["mass"].astype(np.float64) * dm).sum())]
        got = sum(terms)
        scale = abs(terms[0]) + abs(terms[1]) + float(np.abs(g["mass"].astype(np.float64) * dm).sum())
        rel = abs(got - fd) / abs(fd)
        worst = max(worst, rel)
        worst_scaled = max(worst_scaled, abs(got - fd) / scale)
        worst32 = max(worst32, abs(got - t32) / scale)
        assert abs(got - t32) <= 1e-6 * scale, (k, got, t32, scale)
        assert abs(got - fd) <= 1e-4 * scale, (k, got, fd, scale)
        assert rel <= 5e-4, (k, got, fd, rel)
    print(f"over 20 directions: worst |dev-fd|/|fd| {worst:.2e}, |dev-fd|/sum|terms| {worst_scaled:.2e}, "
          f"|dev-single|/sum|terms| {worst32:.2e}")


def test_bingham_yield_stress_gradient(gfsph_lib, oracle_mod):
    """dL/d(yield stress const(6)) of the Bingham law (nfric 4) against the
    FP64 forward-mode oracle, with the positions and volumes."""
    w = workloads.fractal_channel(n_target=3000, dem_k=8, cell=5.0, erosion=None)
    w.const = {**w.const, 5: 4, 6: 1000.0, 7: 50.0, 3: 0.0, 9: 0.0}
    p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=oracle_mod.MODE_FP32)
    rng = np.random.default_rng(6)
    gx = rng.normal(size=(w.n, 2)).astype(np.float32)
    gv = rng.normal(size=(w.n, 2)).astype(np.float32)
    gh = rng.normal(size=w.n).astype(np.float32)
    g, final, _ = gpu_gradients(w, p, topol, gx, gv, gh)
    assert np.abs(final["v"]).max() > 0.1
    ny, nx = w.z.shape
    st0 = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)

    def directional(single=False, **seed):
        _, _, _, dx, dv, dh = oracle_mod.tangent(p, nx, ny, w.dx, w.dy, st0, NSTEPS, single=single, **seed)
        return float((gx * dx).sum() + (gv * dv).sum() + (gh * dh).sum())

    ref = directional(seed_ty=1.0)
    ref32 = directional(seed_ty=1.0, single=True)
    print(f"tauy: device {g['tauy']:.9g} single-trajectory {ref32:.9g} FP64 {ref:.9g}")
    assert ref != 0.0 and abs(g["tauy"] - ref) <= 2e-4 * abs(ref), (g["tauy"], ref)
    assert abs(g["tauy"] - ref32) <= 2e-5 * abs(ref32), (g["tauy"], ref32)
    dm = rng.normal(size=w.n) * w.mass
    dx0 = rng.normal(size=(w.n, 2))
    for name, seed, got, scale in (
            ("mass", dict(seed_m=dm), float((g["mass"] * dm).sum()), float(np.abs(g["mass"] * dm).sum())),
            ("x0", dict(seed_x=dx0), float((g["x0"] * dx0).sum()), float(np.abs(g["x0"] * dx0).sum()))):
        ref = directional(**seed)
        ref32 = directional(single=True, **seed)
        print(f"{name}: device {got:.9g} single-trajectory {ref32:.9g} FP64 {ref:.9g} scale {scale:.6g}")
        # Against the derivative of the trajectory the device computes, tight;
        # against FP64 within 2e-4 of the size of the terms: the regime of the
        # Bingham law is decided on single-precision values, so a particle near
        # a regime boundary can follow the other branch in FP64
        assert abs(got - ref32) <= 2e-5 * scale, (name, got, ref32, scale)
        assert abs(got - ref) <= 2e-4 * scale, (name, got, ref, scale)
    assert g["tanfi"] == 0.0  # no frictional term under the Bingham law


def idw_raster64(w, x, h):
    """The depth raster of SPH_SW_2019.f90:14310-14400 in FP64 (numpy): IDW of h
    over the 4x4 DEM nodes around each particle."""
    ny, nx = w.z.shape
    a1 = np.zeros(nx * ny)
    a5 = np.zeros(nx * ny)
    distg = np.hypot(w.dx, w.dy)
    ipx = ((x[:, 0] - 0.0) / w.dx + 1.0).astype(np.int64)
    ipy = ((x[:, 1] - 0.0) / w.dy + 1.0).astype(np.int64)
    for ox in range(-1, 3):
        for oy in range(-1, 3):
            ix, iy = ipx + ox, ipy + oy
            ok = (ix >= 1) & (ix <= nx) & (iy >= 1) & (iy <= ny)
            d = np.hypot(x[ok, 0] - (ix[ok] - 1) * w.dx, x[ok, 1] - (iy[ok] - 1) * w.dy)
            wgt = distg / np.maximum(d, 1e-6)
            ip = (iy[ok] - 1) * nx + (ix[ok] - 1)
            np.add.at(a1, ip, h[ok] * wgt)
            np.add.at(a5, ip, wgt)
    return np.where(a5.astype(np.float32) >= 1e-6, a1 / np.where(a5 > 0, a5, 1.0), a1)


def test_raster_misfit_and_its_gradient(gfsph_lib, oracle_mod):
    """gfsph_raster_misfit: L = sum (R - T)^2 of the IDW depth raster against a
    target, and dL/dx, dL/dh against central differences of an FP64 raster
    (steps of 1e-6 m and 1e-6 relative; particles on a DEM cell edge, where
    the raster is discontinuous, keep their positions)."""
    w = workloads.fractal_channel(n_target=3000, dem_k=8, cell=5.0, erosion=None)
    p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(10)
    st = sim.download()
    rng = np.random.default_rng(8)
    target = (sim.raster(gfsph.RASTER_DEPTH_IDW) * rng.uniform(0.5, 1.5, size=w.z.shape)).astype(np.float32)
    loss, gx, gh = sim.raster_misfit(target)
    sim.close()
    x64, h64 = st["x"].astype(np.float64), st["rho"].astype(np.float64)
    t64 = target.astype(np.float64).reshape(-1)
    L64 = float(((idw_raster64(w, x64, h64) - t64) ** 2).sum())
    assert abs(loss - L64) <= 1e-5 * L64
    # The raster jumps where a particle crosses a DEM cell edge (its 4x4 node
    # stencil moves): no step of a particle within 1e-4 m of an edge
    fx, fy = x64[:, 0] / w.dx, x64[:, 1] / w.dy
    edge = np.minimum(np.abs(fx - np.round(fx)) * w.dx, np.abs(fy - np.round(fy)) * w.dy)
    away = (edge > 1e-4)[:, None]
    for k in range(3):
        dx = rng.normal(size=x64.shape) * away
        dh = rng.normal(size=h64.shape) * h64
        e = 1e-6
        lp = float(((idw_raster64(w, x64 + e * dx, h64 + e * dh) - t64) ** 2).sum())
        lm = float(((idw_raster64(w, x64 - e * dx, h64 - e * dh) - t64) ** 2).sum())
        fd = (lp - lm) / (2 * e)
        got = float((gx.astype(np.float64) * dx).sum() + (gh.astype(np.float64) * dh).sum())
        assert abs(got - fd) <= 1e-4 * abs(fd), (k, got, fd)


def test_calibration_gradient_of_the_deposit_misfit(gfsph_lib, oracle_mod):
    """The deposit-raster calibration loss end to end: a target raster T from
    a run at mu = 0.18, xi = 350; L = sum (R - T)^2 after 100 steps at
    mu = 0.15, xi = 400; dL/dmu and dL/dxi from gfsph_raster_misfit followed
    by gfsph_adjoint_backward.  The reference is exact in FP64: the oracle's
    forward-mode tangents of the final positions and depths, composed with the
    gradient of the FP64 raster misfit (central differences of the raster
    along the tangent, steps of 1e-7 m that cross no DEM cell edge; central
    differences of the whole trajectory would be polluted by particles that
    cross one and jump the raster).  The misfit is ~1% of the raster after
    100 steps, so the FP32 trajectory's ~1e-5 drift from FP64 enters L and
    its gradient about 100-fold: the tolerance is 5e-3."""
    w, p, topol = case(oracle_mod)
    N = 100
    ny, nx = w.z.shape
    pt = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    pt.cst[8], pt.cst[2] = 0.18, 350.0
    st = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    oracle_mod.run(oracle_mod.MODE_FP64, pt, nx, ny, w.dx, w.dy, st, N)
    target = idw_raster64(w, st.x, st.rho).astype(np.float32).reshape(ny, nx)
    t64 = target.astype(np.float64).reshape(-1)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy, topol=topol.astype(np.float32))
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    adj = gfsph.Adjoint(sim, N, every=10)
    loss, gxr, ghr = sim.raster_misfit(target)
    g = adj.backward(gxr, np.zeros_like(gxr), ghr)
    adj.close()
    sim.close()
    s0 = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    oracle_mod.run(oracle_mod.MODE_FP64, p, nx, ny, w.dx, w.dy, s0, N)

    def L(x, h):
        return float(((idw_raster64(w, x, h) - t64) ** 2).sum())

    L64 = L(s0.x, s0.rho)
    assert abs(loss - L64) <= 5e-3 * L64, (loss, L64)
    st0 = oracle_mod.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    for key, seed in (("tanfi", "seed_mu"), ("xi", "seed_xi")):
        _, _, _, tx, _, th = oracle_mod.tangent(p, nx, ny, w.dx, w.dy, st0, N, **{seed: 1.0})
        tau = 1e-7 / np.abs(tx).max()
        ref = (L(s0.x + tau * tx, s0.rho + tau * th) - L(s0.x - tau * tx, s0.rho - tau * th)) / (2 * tau)
        rel = abs(g[key] - ref) / abs(ref)
        print(f"dL/d{key}: device {g[key]:.6e}, FP64 {ref:.6e}, relative difference {rel:.2e}")
        assert rel <= 5e-3, (key, g[key], ref)
