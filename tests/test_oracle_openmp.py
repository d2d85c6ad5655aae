"""The OpenMP build of the oracle (the CPU baseline on all host cores) steps
the same physics as the serial checker: its pair sums are added in another
order, so the states agree to rounding, not bit for bit.  The grid search and
the erosion scatter keep the serial order, so volumes (erosion on) match to
rounding too."""
import numpy as np
import pytest

import gfsph
import oracle
import workloads


pytestmark = pytest.mark.skipif(not oracle.omp_available(), reason="no -fopenmp compiler here")


def run(mode, omp, nsteps=6, **opts):
    w = workloads.fractal_channel(n_target=6000, dem_k=8, cell=5.0)
    p = workloads.make_params(w, gfsph, **opts)
    ny, nx = w.z.shape
    topol = oracle.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv, mode=mode)
    st = oracle.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    r = oracle.Run(mode, p, nx, ny, w.dx, w.dy, st, omp=omp)
    assert r.advance(nsteps) == nsteps
    out = r.state()
    r.close()
    return out


@pytest.mark.parametrize("mode,rtol", [(oracle.MODE_FP64, 1e-12), (oracle.MODE_FP32_DACC, 1e-5)])
def test_openmp_build_matches_checker(mode, rtol):
    a = run(mode, omp=False)
    b = run(mode, omp=True)
    assert a.t == b.t and a.dt == b.dt
    assert np.array_equal(a.flag, b.flag)
    for k in ("x", "v", "rho", "mass", "hsml"):
        x, y = getattr(a, k), getattr(b, k)
        scale = np.abs(x).max()
        assert np.abs(x - y).max() <= rtol * scale, k


def test_thread_count_set_in_the_library():
    w = workloads.fractal_channel(n_target=6000, dem_k=8, cell=5.0)
    p = workloads.make_params(w, gfsph)
    ny, nx = w.z.shape
    topol = oracle.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv)
    st = oracle.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    r = oracle.Run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, st, omp=True)
    assert r.threads == oracle.omp_threads() >= 1
    r.close()
    assert oracle.Run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, st).threads == 1
