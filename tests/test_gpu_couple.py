"""The SPH -> FEM coupling pass (get_gradhs_w) through the C ABI against the
oracle's restatement, on a window of the DEM background triangulation."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def channel_after(nsteps):
    w = workloads.fractal_channel(n_target=6000, dem_k=8, cell=5.0)
    p = workloads.make_params(w, gfsph)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(nsteps)
    return w, sim, sim.download()


def test_gradhs_matches_oracle(gfsph_lib, oracle_mod):
    w, sim, g = channel_after(5)
    c = np.floor(g["x"][g["flag"] == 0].mean(axis=0) / w.dx).astype(int)
    ny, nx = w.z.shape
    nwx, nwy = 61, 81
    ix0 = int(np.clip(c[0] - 30, 0, nx - nwx))
    iy0 = int(np.clip(c[1] - 40, 0, ny - nwy))
    hs, grad = sim.gradhs(ix0, iy0, nwx, nwy, niter=5)
    hs_o, grad_o = oracle_mod.gradhs(oracle_mod.MODE_FP32_DACC, ix0, iy0, nwx, nwy, w.dx, w.dy, x=g["x"],
                                     rho=g["rho"], flag=g["flag"], niter=5)
    assert hs.max() > 1.0 and (hs > 0).sum() > 100
    assert np.abs(hs - hs_o).max() <= 1e-6 * hs_o.max()
    assert rel_l2(grad, grad_o) <= 1e-5
    # the reference's first sweep leaves the gradient at zero
    _, g1 = sim.gradhs(ix0, iy0, nwx, nwy, niter=1)
    assert np.all(g1 == 0)
    # niter = 0: the mass system solved by CG, against converged sweeps
    _, gcg = sim.gradhs(ix0, iy0, nwx, nwy, niter=0, tol=1e-14)
    _, gconv = oracle_mod.gradhs(oracle_mod.MODE_FP64, ix0, iy0, nwx, nwy, w.dx, w.dy, x=g["x"], rho=g["rho"],
                                 flag=g["flag"], niter=600)
    assert rel_l2(gcg, gconv) <= 1e-4
    sim.close()


def test_gradhs_rejects_windows_off_the_dem(gfsph_lib):
    w, sim, _ = channel_after(1)
    ny, nx = w.z.shape
    with pytest.raises(gfsph.GfsphError):
        sim.gradhs(nx - 10, 0, 20, 20)
    with pytest.raises(gfsph.GfsphError):
        sim.gradhs(0, 0, 1, 20)
    sim.close()
