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
