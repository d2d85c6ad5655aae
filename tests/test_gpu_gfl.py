"""The device GFL Taylor-Galerkin step (gfsph_gfl_*) against the
single-precision restatement (oracle/gfl_oracle.cpp): the set-up's
topography rows and the state after every friction law, both flow types,
one and three Gauss points, the WIR soil coupling and a 512 x 512 mesh, bit
for bit."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu

G = 9.8


def bed_and_state(nx, ny, d, seed, ntype, swl=0.0):
    intmat, coord = workloads.p1_mesh(nx, ny, d)
    rng = np.random.default_rng(seed)
    x, y = coord[:, 0], coord[:, 1]
    lx, ly = (nx - 1) * d, (ny - 1) * d
    z = 20.0 - 0.05 * x + 3.0 * np.sin(2 * np.pi * y / ly) * np.cos(np.pi * x / lx)
    z = z.astype(np.float32).astype(np.float64)
    u = np.zeros((coord.shape[0], 3))
    if ntype == 2:
        u[:, 0] = np.maximum(swl - z, 0.0)
        u[x < 0.3 * lx, 0] += 2.0
    else:
        u[:, 0] = np.where(x < 0.4 * lx, 3.0, 0.0) + rng.uniform(0.0, 0.2, size=x.size) * (x < 0.8 * lx)
    u[:, 1] = rng.normal(size=x.size) * 0.5 * u[:, 0]
    u[:, 2] = rng.normal(size=x.size) * 0.5 * u[:, 0]
    return intmat, coord, z, u.astype(np.float32)


def run_both(oracle_mod, intmat, coord, z, u, const, steps, dt, time=0.0, wir=None, **kw):
    g = gfsph.Gfl(coord, intmat, z, const, **kw)
    g.set_state(u, time)
    if wir is not None:
        g.set_wir(*wir)
    g.step(steps, dt)
    out, t = g.state()
    topol, topel = g.topol()
    launches = g.launch_count()
    g.close()
    ref, tref, rtopol, rtopel = oracle_mod.gfl_run(coord.astype(np.float32), intmat, z, const, u, steps, dt,
                                                   time=time, hs_w=None if wir is None else wir[0],
                                                   gradhs_w=None if wir is None else wir[1], **kw)
    return out, t, topol, topel, launches, ref, tref, rtopol, rtopel


LAWS = {
    0: {},
    1: {3: 0.04},
    2: {7: 5.0},
    3: {6: 200.0, 7: 20.0},
    4: {6: 500.0, 7: 30.0},
    5: {9: 0.2},
    6: {9: 0.25},
    7: {9: 0.2},
    8: {9: 0.2, 3: 0.02},
}


@pytest.mark.parametrize("nfric", sorted(LAWS))
@pytest.mark.parametrize("ntype", [2, 3])
def test_gfl_step_matches_oracle(gfsph_lib, oracle_mod, nfric, ntype):
    swl = 22.0
    intmat, coord, z, u = bed_and_state(41, 33, 5.0, 10 * nfric + ntype, ntype, swl)
    const = {1: G, 2: 1800.0, 4: 1e-4, 5: nfric, 10: 0.05, **LAWS[nfric]}
    if nfric == 5:
        const.update({12: 0.5, 13: 4.0})  # tanfi decays from 0.5 to 0.2 with Bfact 4 s
    out, t, topol, topel, launches, ref, tref, rtopol, rtopel = run_both(
        oracle_mod, intmat, coord, z, u, const, 30, 0.05, time=1.5, ntype=ntype, swl=swl, niter=3)
    assert np.array_equal(topol, rtopol.astype(np.float32)) and np.array_equal(topel, rtopel.astype(np.float32))
    assert np.isfinite(out).all() and np.abs(out - u).max() > 1e-3
    assert np.array_equal(out, ref.astype(np.float32)), np.abs(out - ref).max()
    assert t == tref
    assert launches == 30 * (3 + 2 + 1)


@pytest.mark.parametrize("ngaus,niter", [(1, 1), (1, 4), (3, 2)])
def test_gfl_quadrature_and_sweeps(gfsph_lib, oracle_mod, ngaus, niter):
    intmat, coord, z, u = bed_and_state(25, 40, 4.0, 7, 3)
    const = {1: G, 2: 2000.0, 3: 0.03, 5: 5, 9: 0.15, 10: 0.02}
    out, _, _, _, launches, ref, _, _, _ = run_both(oracle_mod, intmat, coord, z, u, const, 40, 0.04,
                                                    ngaus=ngaus, niter=niter)
    assert np.array_equal(out, ref.astype(np.float32)), np.abs(out - ref).max()
    assert launches == 40 * (3 + niter)


def test_gfl_with_the_soil_of_the_sph_flow(gfsph_lib, oracle_mod):
    """WIR: the soil depth hs_w under the water raises the bed in the still
    depth HH and its gradient adds to the slopes."""
    swl = 22.0
    intmat, coord, z, u = bed_and_state(41, 33, 5.0, 3, 2, swl)
    rng = np.random.default_rng(4)
    x, y = coord[:, 0], coord[:, 1]
    hs = np.maximum(0.0, 2.0 - ((x - 100.0) ** 2 + (y - 80.0) ** 2) / 800.0).astype(np.float32)
    grad = np.stack([-(x - 100.0) / 400.0, -(y - 80.0) / 400.0], 1) * (hs > 0)[:, None]
    grad = (grad + rng.normal(size=grad.shape) * 1e-3).astype(np.float32)
    const = {1: G, 2: 1000.0, 3: 0.03, 5: 0, 10: 0.05}
    out, _, _, _, _, ref, _, _, _ = run_both(oracle_mod, intmat, coord, z, u, const, 30, 0.05,
                                             wir=(hs, grad), ntype=2, swl=swl)
    assert np.array_equal(out, ref.astype(np.float32)), np.abs(out - ref).max()
    plain, *_ = run_both(oracle_mod, intmat, coord, z, u, const, 30, 0.05, ntype=2, swl=swl)
    assert np.abs(plain - out).max() > 1e-3  # the soil changes the flow


def test_gfl_large_mesh_matches_oracle(gfsph_lib, oracle_mod):
    """512 x 512 nodes (522,242 triangles), a dam break over the sloping bed,
    ten steps."""
    intmat, coord, z, u = bed_and_state(512, 512, 2.0, 11, 3)
    const = {1: G, 2: 2000.0, 3: 0.035, 5: 7, 9: 0.2, 10: 0.02}
    out, _, _, _, _, ref, _, _, _ = run_both(oracle_mod, intmat, coord, z, u, const, 10, 0.02)
    assert np.array_equal(out, ref.astype(np.float32)), np.abs(out - ref).max()


def test_gfl_refuses_what_it_does_not_build(gfsph_lib):
    intmat, coord, z, _ = bed_and_state(6, 5, 1.0, 0, 3)
    base = {1: G, 2: 1000.0, 10: 0.01}
    for const, kw, status in (({**base, 11: 1.0}, {}, gfsph.ERR_UNSUPPORTED),   # itens: viscous stresses
                              ({**base, 10: 0.0}, {}, gfsph.ERR_ARG),            # hfrict0 must exceed 1e-32
                              ({**base, 5: 2, 2: 0.0}, {}, gfsph.ERR_ARG),       # Julien friction without density
                              (base, {"ngaus": 2}, gfsph.ERR_UNSUPPORTED),
                              (base, {"ntype": 1}, gfsph.ERR_UNSUPPORTED)):
        with pytest.raises(gfsph.GfsphError) as e:
            gfsph.Gfl(coord, intmat, z, const, **kw)
        assert e.value.status == status
    with pytest.raises(gfsph.GfsphError) as e:  # clockwise triangles
        gfsph.Gfl(coord, intmat[:, ::-1], z, base)
    assert e.value.status == gfsph.ERR_ARG
