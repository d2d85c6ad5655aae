"""What a handle holds after a call fails.  A device allocation that fails
(here a neighbour table of 65536 slots for a million particles, ~262 GB)
leaves the handle without state: stepping or reading it returns
GFSPH_ERR_STATE, nothing runs on the freed buffers, and the next upload
starts afresh.  An adjoint record refuses a handle re-uploaded with another
particle count."""
import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu

ERR_CUDA, ERR_STATE = -2, -5


def small(**opts):
    w = workloads.fractal_channel(n_target=2000, dem_k=8, cell=5.0)
    return w, workloads.make_params(w, gfsph, **opts)


def million(w):
    rng = np.random.default_rng(5)
    ny, nx = w.z.shape
    n = 1_000_000
    x = np.stack([rng.uniform(0.1, 0.9, n) * nx * w.dx, rng.uniform(0.1, 0.9, n) * ny * w.dy], 1)
    return (x.astype(np.float32), np.zeros((n, 2), np.float32), np.ones(n, np.float32),
            np.ones(n, np.float32), np.full(n, 1.0, np.float32))


def status_of(fn, *a):
    with pytest.raises(gfsph.GfsphError) as e:
        fn(*a)
    return e.value.status


def test_failed_table_allocation_drops_the_state(gfsph_lib):
    w, p = small(max_neighbours=65536)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    assert status_of(sim.upload, *million(w)) == ERR_CUDA
    assert status_of(sim.step, 1) == ERR_STATE
    assert status_of(sim.download) == ERR_STATE
    sim.close()


def test_handle_recovers_after_a_failed_upload(gfsph_lib):
    w, p = small(max_neighbours=65536)  # 65536 slots x 2016 rows fit; a million rows do not
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(2)
    assert status_of(sim.upload, *million(w)) == ERR_CUDA
    assert status_of(sim.step, 1) == ERR_STATE  # the graphs and buffers of the old state are gone
    assert status_of(sim.download) == ERR_STATE
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(4)
    a = sim.download()
    sim.close()
    # the same calls without the failed upload (an upload keeps the time,
    # dt and the eroded DEM of the handle)
    ref = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    ref.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    ref.step(2)
    ref.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    ref.step(4)
    b = ref.download()
    ref.close()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_adjoint_refuses_a_resized_handle(gfsph_lib):
    w = workloads.fractal_channel(n_target=1500, dem_k=8, cell=5.0, erosion=None)
    p = workloads.make_params(w, gfsph, sle=0, ic_adapt=0)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    adj = gfsph.Adjoint(sim, 3, every=1)
    m = w.n - 7
    sim.upload(w.x[:m], w.v[:m], w.rho[:m], w.mass[:m], w.hsml[:m])
    g = np.zeros((w.n, 2), np.float32)
    assert status_of(adj.backward, g, g) == ERR_STATE
    adj.close()
    sim.close()


def test_every_particle_leaving_the_dem_ends_the_run(gfsph_lib, oracle_mod):
    """A patch launched across the +x edge of a flat, frictionless 95 m box:
    the first step that starts with no particle inside returns
    GFSPH_ERR_DOMAIN (-8), the time stops there, as the oracle's does (to
    one step: a particle's exit could flip by one step at the edge), and the
    state stays readable with every particle flagged."""
    nx = ny = 20
    d = 5.0
    g = np.arange(8) * 1.0 + 80.0
    X, Y = np.meshgrid(g, g - 40.0)  # x 80-87 m, y 40-47 m
    x = np.stack([X.ravel(), Y.ravel()], 1).astype(np.float32)
    n = x.shape[0]
    v = np.tile(np.float32([20.0, 0.0]), (n, 1))
    rho = np.full(n, 1.0, np.float32)
    mass = np.full(n, 1.0, np.float32)
    hsml = np.full(n, 1.3, np.float32)
    z = np.zeros((ny, nx), np.float32)
    p = gfsph.make_params({1: 9.8, 2: 2000.0, 3: 1e30, 5: 5, 9: 0.0, 10: 0.01, 15: 0.01},
                          sle=0, dt=0.01, ic_adapt=0, average_velocity=0)
    sim = gfsph.Sim(p, z, dx=d, dy=d)
    sim.upload(x, v, rho, mass, hsml)
    assert status_of(sim.step, 400) == -8
    t_gpu, _ = sim.time()
    out = sim.download()
    sim.close()
    assert np.all(out["flag"] == 1)
    topol = oracle_mod.initial_topol(z.astype(np.float64), d, d, {}, deriv=1, mode=oracle_mod.MODE_FP32_DACC)
    st = oracle_mod.State(x, v, rho, mass, hsml, topol, dt=0.01)
    run = oracle_mod.Run(oracle_mod.MODE_FP32_DACC, p, nx, ny, d, d, st)
    done = run.advance(400)
    t_ref = run.state().t
    run.close()
    assert 0 < done < 400
    assert abs(t_gpu - t_ref) <= 0.0101, (t_gpu, t_ref)

