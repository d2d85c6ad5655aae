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
    """icpwp = 1 and 3 read from the .dat (with their pwp0rel line) reach the
    step: a liquefied release (pwp0rel = 1, slow dissipation) runs out faster
    than the same release without pore pressure."""
    speeds = {}
    for icpwp in (0, 1, 3):
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
        # OutputRes_Classic writes the pore pressure at the nodes for icpwp 1 only
        res = open(os.path.join(d, "plane.post.res")).read()
        assert ('Result "Pwp"' in res) == (icpwp == 1)
    assert speeds[3] > 1.2 * speeds[0] and speeds[1] > 1.2 * speeds[0]


def test_kernels_report_sm100(gfsph_lib):
    """The runtime reports the loaded kernels as built for compute capability 10.0."""
    import ctypes as C
    v = C.c_int(0)
    assert gfsph_lib.lib().gfsph_binary_version(C.byref(v)) == 0
    assert v.value == 100


def parsed_count(d, name):
    """Particles the driver builds from the written .pts (Read_Source_plus_New
    fills the release on its own lattice, so the count is not the workload's)."""
    out = subprocess.run([RUN, name, "--dir", d, "--parse-only"], capture_output=True, text=True)
    return json.loads(out.stdout)["n"]


def run_driver(d, name, steps):
    out = subprocess.run([RUN, name, "--dir", d, "--out", d, "--max-steps", str(steps)], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stderr
    return out


@pytest.mark.parametrize("case", ["plane", "channel_erosion_pwp"])
def test_resume_from_restart_matches_the_uninterrupted_run(gfsph_lib, tmp_path, case):
    """OutputSave_SW's restart files (SPH_SW_2019.f90:12416-12485) written by
    gfsph_run after K steps, read back through icunk_s = 200 (and restart.top
    with erosion), and K more steps: the state equals that of 2K steps in one
    run, bit for bit (the files carry 9 significant digits, which read back
    into the same single-precision values).  Fixed dt: the reference starts a
    restarted run from the MASTER dt_sph, so adaptive dt would differ from
    the first step on."""
    if case == "plane":
        w = workloads.inclined_plane()
        name = "plane"
    else:
        w = workloads.fractal_channel(n_target=3000, dem_k=8, cell=5.0)
        w.const = {**w.const, 13: 0.001, 14: 1.0}
        w.options = {**w.options, "ic_adapt": 0, "icpwp": 3, "pwp0rel": 0.5}
        name = "chan"
    K = 30
    full, first, second = (os.path.join(str(tmp_path), k) for k in ("full", "first", "second"))
    for d in (full, first):
        workloads.write_reference_inputs(w, d, name, out_step=K)
    workloads.write_reference_inputs(w, second, name, out_step=K, restart=True)
    run_driver(full, name, 2 * K)
    run_driver(first, name, K)
    files = [".restart.dat"] + ([".restart.top"] if case != "plane" else [])
    for f in files:
        src = os.path.join(first, name + f)
        assert os.path.exists(src), f
        with open(src) as a, open(os.path.join(second, "restart" + f[len(".restart"):]), "w") as b:
            b.write(a.read())
    run_driver(second, name, K)
    with open(os.path.join(full, name + ".restart.dat")) as a, open(os.path.join(second, name + ".restart.dat")) as b:
        la, lb = a.read().splitlines(), b.read().splitlines()
    assert la[1:] == lb[1:]  # the state (and the time on its own line)
    if case != "plane":
        # Z and the eroded depth agree; the erodible depth does not, since
        # Input_SW sets it anew to const(48) after reading restart.top
        # (SPH_SW_2019.f90:1291-1301), and no node reached its limit here
        ta = np.loadtxt(os.path.join(full, name + ".restart.top"), skiprows=3)
        tb = np.loadtxt(os.path.join(second, name + ".restart.top"), skiprows=3)
        assert np.array_equal(ta[:, :3], tb[:, :3]) and ta[:, 2].max() > 0.0
    # the restart state moved away from the start
    st = np.loadtxt(os.path.join(full, name + ".restart.dat"), skiprows=3)
    assert st.shape[0] == parsed_count(full, name) and np.abs(st[:, 4:6]).max() > 0.1


def test_gid_results_agree_with_the_depth_raster(gfsph_lib, tmp_path):
    """The GiD files of OutputMesh_Classic / OutputRes_Classic: the mesh holds
    the DEM nodes, its quadrilaterals and the particles; at every plot time
    the nodal heights are the IDW depth raster written beside them."""
    w = workloads.inclined_plane()
    d = str(tmp_path)
    workloads.write_reference_inputs(w, d, "plane", out_step=50)
    run_driver(d, "plane", 150)
    ny, nx = w.z.shape
    msh = open(os.path.join(d, "plane.post.msh")).read().split("\n")
    i0 = next(k for k, l in enumerate(msh) if l.strip() == "coordinates")
    i1 = next(k for k, l in enumerate(msh) if l.strip() == "End coordinates")
    assert i1 - i0 - 1 == nx * ny + parsed_count(d, "plane")
    res = open(os.path.join(d, "plane.post.res")).read()
    assert res.startswith("GiD Post Results File 1.0")
    blocks = res.split(' Result "height"')[1:]
    assert len(blocks) == 3
    for k, blk in enumerate(blocks):
        vals = blk.split("Values")[1].split("End")[0].strip().split("\n")
        nodes = np.array([[float(t) for t in line.split()] for line in vals])
        _, depth = read_asc(os.path.join(d, "plane.depth_%04d.asc" % k))
        ip = nodes[:, 0].astype(int) - 1
        ref = depth.reshape(-1)[ip]
        assert np.allclose(nodes[:, 3], ref, rtol=2e-4, atol=1e-5)
        assert '"dis"' in blk and '"vel"' in blk


def test_driver_runs_soil_and_water(gfsph_lib, tmp_path):
    """gfsph_run on soil and water inputs (ic_soil = ic_water = 1, ic_SWAlg 1):
    the run steps both materials, and its restart file carries the water's
    itype 2 rows after the soil's, as OutputSave_SW writes them."""
    w, a = workloads.soil_and_pond()
    water = dict(x=a["x"][a["itype"] == 2], rho=a["rho"][a["itype"] == 2], lattice=1.5)
    d = str(tmp_path)
    workloads.write_reference_inputs(w, d, "pond", out_step=10, water=water)
    meta = json.loads(subprocess.run([RUN, "pond", "--dir", d, "--parse-only"], capture_output=True,
                                     text=True).stdout)
    run_driver(d, "pond", 20)
    st = np.loadtxt(os.path.join(d, "pond.restart.dat"), skiprows=3)
    assert st.shape[0] == meta["n"] and int((st[:, 1] == 2).sum()) == meta["n_water"] > 0
    assert (np.diff(st[:, 1]) >= 0).all()  # soil first, then water
    water_rows = st[:, 1] == 2
    assert np.abs(st[water_rows, 4:6]).max() > 1e-3  # the water moved
