"""Soil and water particles (ic_ws_Interact = 1) on the device against the
oracle (FP32 state, FP64 sums): a Bingham soil cap on a gentle slope with a
water pond over its downslope edge, for both ic_SWalg forms, and the options
refused with them."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu

CONST = {1: 9.8, 2: 2000.0, 3: 0.03, 5: 4, 6: 1000.0, 7: 50.0, 10: 0.01, 15: 0.01, 18: 1000.0}


def soil_and_pond():
    w, a = workloads.soil_and_pond()
    return w, a["x"], a["v"], a["rho"], a["mass"], a["hsml"], a["itype"]


def run_pair(oracle_mod, sw_alg, steps):
    w, x, v, rho, mass, hsml, itype = soil_and_pond()
    p = gfsph.make_params(CONST, sle=1, ic_adapt=0, dt=0.01, ws_interact=1, sw_alg=sw_alg)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(x, v, rho, mass, hsml, itype=itype)
    sim.step(steps)
    got = sim.download()
    sim.close()
    ny, nx = w.z.shape
    topol = oracle_mod.initial_topol(w.z, w.dx, w.dy, CONST, deriv=p.dem_deriv)
    flag = np.where(itype == 2, 2, 0).astype(np.int32)
    st = oracle_mod.State(x, v, rho, mass, hsml, topol, flag=flag, dt=p.dt)
    oracle_mod.run(oracle_mod.MODE_FP32_DACC, p, nx, ny, w.dx, w.dy, st, steps)
    return got, st, itype


@pytest.mark.parametrize("sw_alg", [0, 1])
def test_soil_and_water_one_step_matches_oracle(gfsph_lib, oracle_mod, sw_alg):
    got, st, itype = run_pair(oracle_mod, sw_alg, 1)
    assert np.array_equal(got["flag"], st.flag & 1)
    for k, ref in (("x", st.x), ("v", st.v), ("rho", st.rho), ("hsml", st.hsml)):
        ref = ref.astype(np.float32)
        scale = np.abs(ref).max()
        assert np.abs(got[k] - ref).max() <= 1e-6 * max(scale, 1.0), (k, np.abs(got[k] - ref).max())
    assert np.abs(got["v"][itype == 2]).max() > 1e-3  # the water moves


@pytest.mark.parametrize("sw_alg", [0, 1])
def test_soil_and_water_thirty_steps_match_oracle(gfsph_lib, oracle_mod, sw_alg):
    """30 steps: relative L2 of positions 1e-6, of velocities and depths 1e-5
    (the soil surface is an FP64 atomic sum per DEM node, whose last bits can
    differ from the oracle's sequential sum)."""
    got, st, itype = run_pair(oracle_mod, sw_alg, 30)
    for k, ref, tol in (("x", st.x, 1e-6), ("v", st.v, 1e-5), ("rho", st.rho, 1e-5)):
        ref = ref.astype(np.float64)
        err = np.linalg.norm(got[k].astype(np.float64) - ref) / np.linalg.norm(ref)
        assert err <= tol, (k, err)


def test_water_changes_the_soil_flow(gfsph_lib):
    """The pond pushes the soil: the cap's velocities differ from the same cap
    run without the water."""
    w, x, v, rho, mass, hsml, itype = soil_and_pond()
    out = {}
    for with_water in (True, False):
        keep = slice(None) if with_water else slice(0, w.n)
        p = gfsph.make_params(CONST, sle=1, ic_adapt=0, dt=0.01, ws_interact=1, sw_alg=1)
        sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        sim.upload(x[keep], v[keep], rho[keep], mass[keep], hsml[keep], itype=itype[keep])
        sim.step(20)
        out[with_water] = sim.download()["v"][:w.n]
        sim.close()
    assert np.abs(out[True] - out[False]).max() > 1e-3


def test_soil_and_water_refusals(gfsph_lib):
    w, x, v, rho, mass, hsml, itype = soil_and_pond()
    # water particles without ic_ws_Interact = 1
    p = gfsph.make_params(CONST, sle=1, ic_adapt=0, dt=0.01)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    with pytest.raises(gfsph.GfsphError) as e:
        sim.upload(x, v, rho, mass, hsml, itype=itype)
    assert e.value.status == gfsph.ERR_UNSUPPORTED
    sim.close()
    # options outside the scope of the two materials
    # (interface erosion const(50) and friction const(55), Input_SW :1328-1345, too)
    for const, kw in (({21: 1, 22: 0.005}, {}), ({}, {"icpwp": 3}), ({}, {"nor_density": 1}), ({16: 1.0}, {}),
                      ({50: 1.0, 51: 0.001}, {}), ({55: 1.0, 56: 0.1}, {})):
        p = gfsph.make_params({**CONST, **const}, sle=1, ic_adapt=0, dt=0.01, ws_interact=1, **kw)
        with pytest.raises(gfsph.GfsphError) as e:
            gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        assert e.value.status == gfsph.ERR_UNSUPPORTED
    # the adjoint
    p = gfsph.make_params({**CONST, 5: 5, 9: 0.2}, sle=0, ic_adapt=0, dt=0.01, ws_interact=1)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(x, v, rho, mass, hsml, itype=itype)
    with pytest.raises(gfsph.GfsphError) as e:
        gfsph.Adjoint(sim, 5)
    assert e.value.status == gfsph.ERR_UNSUPPORTED
    sim.close()
