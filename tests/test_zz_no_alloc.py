"""The allocation-free depth raster, through the C ABI.

Callers that cannot allocate device memory mid-run (a host that reserves all
of it up front, or one embedded in a framework owning the allocator) use
gfsph_raster_idw_noalloc with their own device buffers; its accumulators are a
fixed device array inside the library.  This file is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import gfsph
import workloads

pytestmark = pytest.mark.gpu


def test_noalloc_raster_matches_the_handle_raster(gfsph_lib, oracle_mod):
    import torch

    w = workloads.fractal_channel(n_target=6000, dem_k=8, cell=5.0)
    p = workloads.make_params(w, gfsph)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(10)
    g = sim.download()
    ref = sim.raster(gfsph.RASTER_DEPTH_IDW)
    sim.close()
    ny, nx = w.z.shape
    dev = torch.device("cuda:0")
    x = torch.from_numpy(g["x"]).to(dev)
    rho = torch.from_numpy(g["rho"]).to(dev)
    flag = torch.from_numpy(g["flag"]).to(dev)
    out = torch.full((ny, nx), -1.0, dtype=torch.float32, device=dev)
    L = gfsph.lib()
    stream = torch.cuda.current_stream().cuda_stream
    tol = 1e-5 * max(float(ref.max()), 1.0)  # the tolerance of the handle raster against the oracle

    def call(depth, flags):
        st = L.gfsph_raster_idw_noalloc(w.n, C.c_void_p(x.data_ptr()), C.c_void_p(depth.data_ptr()),
                                        C.c_void_p(flags.data_ptr()), nx, ny, 0.0, 0.0, w.dx, w.dy,
                                        C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert st == 0, gfsph.strerror(st)
        torch.cuda.synchronize()
        return out.cpu().numpy()

    # Every call must start from cleared accumulators, and the calls differ in
    # their inputs so that sums left over from the call before would show: after
    # a call with every depth x7, a call with every particle flagged must give
    # zeros (not the x7 raster), and the real call must give the handle raster
    # (stale sums would give (7h + h)/2 = 4h at every node).
    got = call(rho * 7.0, flag)
    assert np.abs(got - 7.0 * ref).max() <= 7.0 * tol
    got = call(rho, torch.ones_like(flag))
    assert np.all(got == 0.0)
    for _ in range(2):  # then the real call twice in a row
        got = call(rho, flag)
        assert np.abs(got - ref).max() <= tol
        assert got.max() > 0
    # a misaligned position array is refused, not read
    xb = torch.zeros(2 * w.n + 1, dtype=torch.float32, device=dev)
    st = L.gfsph_raster_idw_noalloc(w.n, C.c_void_p(xb.data_ptr() + 4), C.c_void_p(rho.data_ptr()),
                                    C.c_void_p(flag.data_ptr()), nx, ny, 0.0, 0.0, w.dx, w.dy,
                                    C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert st == -1


def test_noalloc_raster_rejects_grids_above_its_fixed_size(gfsph_lib):
    L = gfsph.lib()
    big = 2048  # 2048 x 2048 nodes > 2^20
    st = L.gfsph_raster_idw_noalloc(0, None, None, None, big, big, 0.0, 0.0, 1.0, 1.0, C.c_void_p(256), None)
    assert st == -3
