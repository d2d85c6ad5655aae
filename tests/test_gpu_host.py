"""gfsph_run, the C++ host that reads the reference's input files, on the
GPU: it runs the step loop with the reference's plot cadence and writes
depth rasters."""
import json
import os
import subprocess

import numpy as np
import pytest

import workloads

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "deslizamientos-y-flujos_b200", "gfsph_run")


def read_asc(path):
    with open(path) as f:
        head = [next(f) for _ in range(6)]
        data = np.loadtxt(f)
    return head, data[::-1]


def test_gfsph_run_on_written_inputs(gfsph_lib, tmp_path):
    w = workloads.inclined_plane()
    d = str(tmp_path)
    workloads.write_reference_inputs(w, d, "plane")
    meta = json.loads(subprocess.run([RUN, "plane", "--dir", d, "--parse-only"], capture_output=True,
                                     text=True).stdout)
    out = subprocess.run([RUN, "plane", "--dir", d, "--out", d, "--max-steps", "300"], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    log = np.loadtxt(os.path.join(d, "plane.gfsph.log"))
    assert log.shape[0] == 3                         # plot every 100 steps (plot_step * dt)
    assert np.allclose(log[:, 3], meta["volume"], rtol=1e-6)   # no erosion: volume conserved
    assert log[-1, 2] == 300 and log[-1, 6] == meta["n"]
    head, depth = read_asc(os.path.join(d, "plane.depth_0002.asc"))
    assert depth.shape == (400, 200) and np.isfinite(depth).all() and depth.max() > 1.0
    _, hmax = read_asc(os.path.join(d, "plane.max_depth.asc"))
    assert hmax.max() >= log[:, 4].max() - 1e-4


def test_gfsph_run_with_basal_pore_pressure(gfsph_lib, tmp_path):
    """icpwp = 3 read from the .dat (with its pwp0rel line) reaches the step:
    a liquefied release (pwp0rel = 1, slow dissipation) runs out faster than
    the same release without pore pressure."""
    speeds = {}
    for icpwp in (0, 3):
        w = workloads.inclined_plane()
        w.const = {**w.const, 9: 0.55, 13: 0.001, 14: 1.0}
        w.options = {**w.options, "icpwp": icpwp, "pwp0rel": 1.0}
        d = os.path.join(str(tmp_path), "p%d" % icpwp)
        workloads.write_reference_inputs(w, d, "plane")
        meta = json.loads(subprocess.run([RUN, "plane", "--dir", d, "--parse-only"], capture_output=True,
                                         text=True).stdout)
        assert meta["icpwp"] == icpwp and (icpwp == 0 or meta["pwp0rel"] == 1.0)
        out = subprocess.run([RUN, "plane", "--dir", d, "--out", d, "--max-steps", "200"], capture_output=True,
                             text=True)
        assert out.returncode == 0, out.stderr
        speeds[icpwp] = np.loadtxt(os.path.join(d, "plane.gfsph.log"))[-1, 5]
    assert speeds[3] > 1.2 * speeds[0]


def test_kernels_report_sm100(gfsph_lib):
    """The runtime reports the loaded kernels as built for compute capability 10.0."""
    import ctypes as C
    v = C.c_int(0)
    assert gfsph_lib.lib().gfsph_binary_version(C.byref(v)) == 0
    assert v.value == 100
