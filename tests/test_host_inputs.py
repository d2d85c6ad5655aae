"""The C++ host driver's readers of the reference input files (no GPU):
MASTER.dat, the SW .dat, the .top DEM and the .pts source."""
import json
import os
import subprocess

import numpy as np
import pytest

import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "deslizamientos-y-flujos_b200", "gfsph_run")
GOLDEN = os.path.join(ROOT, "tests", "golden", "picacho")


def parse(name, directory):
    out = subprocess.run([RUN, name, "--dir", directory, "--parse-only"], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return json.loads(out.stdout)


def test_written_inputs_read_back(gfsph_lib, tmp_path):
    w = workloads.inclined_plane()
    workloads.write_reference_inputs(w, str(tmp_path), "plane")
    r = parse("plane", str(tmp_path))
    assert (r["nx"], r["ny"]) == (200, 400) and r["dx"] == 5.0 and r["fdiff"] == 1 and r["ictop"] == 0
    assert r["dt_sph"] == pytest.approx(0.01) and r["ic_adapt"] == 0
    assert (r["pa_sph"], r["nnps"], r["sle"], r["skf"], r["nfric"], r["icpwp"]) == (2, 2, 1, 1, 5, 0)
    assert r["const"][0] == pytest.approx(9.8) and r["const"][2] == 500 and r["const"][8] == pytest.approx(0.2)
    assert r["hsml"] == pytest.approx(4.0)
    # the lattice resample of Read_Source_plus_New reproduces the source nodes
    # and adds a halo of IDW-averaged nodes around them, at most 2 nodes deep
    assert r["n"] >= w.n and r["n"] < w.n * 1.5
    assert r["z_mean"] == pytest.approx(float(w.z.astype(np.float64).mean()), rel=1e-5)


def picacho_inputs(directory):
    """The reference's Picacho example inputs (tests/golden/picacho) in `directory`."""
    import sys
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)
    import make_fixture
    return make_fixture.extract(str(directory))


def test_picacho_example_reads(gfsph_lib, tmp_path):
    r = parse("Picacho", picacho_inputs(tmp_path))
    assert (r["nx"], r["ny"], r["dx"]) == (442, 291, 10.0)
    assert r["ictop"] == 10 and r["fdiff"] == 0
    assert (r["nnps"], r["skf"], r["nfric"], r["icpwp"]) == (4, 1, 7, 3)
    assert r["dt_sph"] == pytest.approx(0.1) and r["ic_adapt"] == 1 and r["plot_step"] == 50
    assert 800 < r["n"] < 900 and r["hsml"] == 20.0
    assert r["const"][2] == 300 and r["const"][8] == pytest.approx(0.6)


def test_reader_reports_unsupported_options(gfsph_lib, tmp_path):
    w = workloads.inclined_plane()
    workloads.write_reference_inputs(w, str(tmp_path), "bad")
    top = os.path.join(str(tmp_path), "bad.top")
    txt = open(top).read().replace("ictop\n100\n", "ictop\n3\n", 1)
    open(top, "w").write(txt)
    out = subprocess.run([RUN, "bad", "--dir", str(tmp_path), "--parse-only"], capture_output=True, text=True)
    assert out.returncode == 2 and "ictop 3" in out.stderr


@pytest.mark.parametrize("icpwp", [1, 3])
def test_written_inputs_with_pore_pressure_parse(gfsph_lib, tmp_path, icpwp):
    """icpwp 1 and 3 each read a pwp0rel line (Input_SW SPH_SW_2019.f90:1724-1729, 1829-1835)."""
    w = workloads.inclined_plane()
    w.options = {**w.options, "icpwp": icpwp, "pwp0rel": 0.75}
    workloads.write_reference_inputs(w, str(tmp_path), "pw")
    meta = parse("pw", str(tmp_path))
    assert meta["icpwp"] == icpwp and abs(meta["pwp0rel"] - 0.75) < 1e-7


def _damage(ext, how):
    def f(name, text):
        if not name.endswith(ext):
            return text
        if how == "missing":
            return None
        if how == "empty":
            return ""
        if how == "half":
            return text[: len(text) // 2]
        if how == "junk":
            return text.replace("0", "x")
        return how(text)
    return f


DAMAGE = [
    (ext, how) for ext in (".MASTER.dat", "plane.dat", ".top", ".pts") for how in ("missing", "empty", "half", "junk")
] + [
    (".top", lambda t: t.replace("200 400", "0 0", 1)),
    (".top", lambda t: t.replace("200 400", "-5 400", 1)),
    (".top", lambda t: t.replace("200 400", "2000000000 2000000000", 1)),
    ("plane.dat", lambda t: t.replace("ndimn\n  2", "ndimn\n  3", 1)),
    (".pts", lambda t: t.replace("1941 2 2 2 2", "1941 2 0 0 2", 1)),
]


@pytest.mark.parametrize("ext,how", DAMAGE)
def test_damaged_inputs_are_refused_with_a_message(gfsph_lib, tmp_path, ext, how):
    """A missing, empty, truncated or garbled input file, or a DEM grid, a
    dimension or a lattice outside what the step takes, ends the driver with
    status 2 and a message naming the file: never a crash or a silent run."""
    w = workloads.inclined_plane()
    src = tmp_path / "src"
    src.mkdir()
    workloads.write_reference_inputs(w, str(src), "plane")
    dst = tmp_path / "dst"
    dst.mkdir()
    mutate = _damage(ext, how)
    for name in os.listdir(src):
        text = mutate(name, (src / name).read_text())
        if text is not None:
            (dst / name).write_text(text)
    out = subprocess.run([RUN, "plane", "--dir", str(dst), "--parse-only"], capture_output=True, text=True)
    assert out.returncode == 2, (out.returncode, out.stderr)
    assert "plane" in out.stderr


def test_restart_input_reads_the_reference_layout(gfsph_lib, tmp_path):
    """icunk_s = 200: the particles come from restart.dat, written here in the
    layout of OutputSave_SW (SPH_SW_2019.f90:12416-12460: two header lines,
    npoin_s and the time, a column header, then i7, i5 and 8 values per line
    in g14.7); the driver reads them list-directed as Get_Restart_Info_SW
    does (:3270-3337) and hands them to the step unchanged."""
    import workloads
    w = workloads.inclined_plane()
    workloads.write_reference_inputs(w, str(tmp_path), "plane", restart=True)
    rng = np.random.default_rng(4)
    v = rng.normal(size=(w.n, 2)).astype(np.float32)
    pwp = np.zeros(w.n, np.float32)
    with open(tmp_path / "restart.dat", "w") as f:
        f.write(" ----- npoin_s      time at restart -----    12.50000    \n")
        f.write("        %d   12.50000    \n" % w.n)
        f.write(" ipoin...itype....x ............   y ..........   vx............. vy ..........   h........   "
                "mass..........   hsml ..........   pwp   \n")
        for i in range(w.n):
            vals = (w.x[i, 0], w.x[i, 1], v[i, 0], v[i, 1], w.rho[i], w.mass[i], w.hsml[i], pwp[i])
            f.write("%7d  %5d" % (i + 1, 1) + "".join("  %14.7E" % float(a) for a in vals) + "\n")
    r = parse("plane", str(tmp_path))
    assert r["n"] == w.n
    dump = str(tmp_path / "plane.dump")
    out = subprocess.run([RUN, "plane", "--dir", str(tmp_path), "--dump", dump], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    import gfsph
    got, _ = workloads.from_driver_dump(dump, gfsph)

    def g7(a):  # the value a g14.7 field carries, read back in single precision
        return np.array([np.float32(float("%14.7E" % float(b))) for b in np.ravel(a)], np.float32).reshape(np.shape(a))

    assert np.array_equal(got.x, g7(w.x)) and np.array_equal(got.v, g7(v))
    assert np.array_equal(got.rho, g7(w.rho)) and np.array_equal(got.mass, g7(w.mass))
    assert np.array_equal(got.hsml, g7(w.hsml))


def test_picacho_setup_matches_the_oracle_restatement(gfsph_lib, oracle_mod, tmp_path):
    """The C++ reader's DEM and particles for the reference's own example
    against the oracle's independent restatements of Get_DTM
    (SPH_FEM_topo_2019.f90:1155-1445, ictop 10: the scattered .top points to
    the grid by inverse-distance weights) and Read_Source_plus_New
    (SPH_SW_2019.f90:4999-5272: the .pts source resampled on its lattice),
    bit for bit; the driver leaves out the lattice nodes of zero volume."""
    import gfsph
    d = picacho_inputs(tmp_path)
    dump = os.path.join(str(tmp_path), "picacho.dump")
    out = subprocess.run([RUN, "Picacho", "--dir", d, "--dump", dump], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    w, p = workloads.from_driver_dump(dump, gfsph)
    dem = oracle_mod.get_dtm(os.path.join(d, "Picacho.top"))
    assert (dem["nx"], dem["ny"]) == (442, 291)
    assert np.float32(w.meta["xmin"]) == dem["xmin"] and np.float32(w.meta["ymin"]) == dem["ymin"]
    assert np.float32(w.dx) == dem["dx"] and np.float32(w.dy) == dem["dy"]
    assert np.array_equal(w.z, dem["z"])
    src = oracle_mod.read_source_plus_new(os.path.join(d, "Picacho.pts"), p.h_inf, dem["xshift"], dem["yshift"])
    keep = src["mass"] > 0
    assert keep.sum() == w.n
    for key, got in (("x", w.x), ("h", w.rho), ("mass", w.mass), ("hsml", w.hsml)):
        assert np.array_equal(got, src[key][keep]), key


def test_soil_and_water_inputs_parse(gfsph_lib, tmp_path):
    """ic_soil = ic_water = 1 with ic_SWAlg 1: the water points of
    Get_water_points (SPH_SW_2019.f90:2226-2273) through
    Read_Source_plus_New_WATER (icunk_w 7, a .pts named in the .dat) follow
    the soil's; the run takes ic_ws_Interact = 1.  Without water, ic_SWAlg 1
    is refused, and so is the debris-flow mixture (ic_SWAlg 3)."""
    w, a = workloads.soil_and_pond()
    w.meta["lattice"] = 1.5
    water = dict(x=a["x"][a["itype"] == 2], rho=a["rho"][a["itype"] == 2], lattice=1.5)
    d = str(tmp_path / "wir")
    workloads.write_reference_inputs(w, d, "pond", water=water)
    meta = parse("pond", d)
    assert meta["ws_interact"] == 1 and meta["sw_alg"] == 1
    soil_only = str(tmp_path / "soil")
    w.options = {**w.options, "sw_alg": 0}
    workloads.write_reference_inputs(w, soil_only, "pond")
    alone = parse("pond", soil_only)
    assert meta["n_water"] > 0 and meta["n"] == alone["n"] + meta["n_water"]
    assert abs(meta["n_water"] - len(water["rho"])) <= 0.1 * len(water["rho"])
    for sw, wat in ((1, False), (3, True)):
        dd = str(tmp_path / f"bad{sw}")
        w.options = {**w.options, "sw_alg": sw}
        workloads.write_reference_inputs(w, dd, "pond", water=water if wat else None)
        out = subprocess.run([RUN, "pond", "--dir", dd, "--parse-only"], capture_output=True, text=True)
        assert out.returncode != 0 and "ic_SWAlg" in out.stderr
