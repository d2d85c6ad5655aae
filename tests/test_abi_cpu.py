"""The C-ABI library without a GPU: it builds, loads, exports every symbol the
header declares, and its compute entry points refuse to run without a CUDA
device (no CPU fallback)."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gfsph.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gfsph_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_step_interface():
    syms = declared_symbols()
    for s in ("gfsph_create", "gfsph_upload", "gfsph_step", "gfsph_download", "gfsph_destroy",
              "gfsph_raster", "gfsph_neighbours", "gfsph_density"):
        assert s in syms


def test_library_exports_every_declared_symbol(gfsph_lib):
    L = gfsph_lib.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s
    assert set(declared_symbols()) <= set(gfsph_lib.SIGNATURES)


def test_library_is_built_for_sm100a(gfsph_lib):
    # the build compiles every CUDA source for sm_100a only; the GPU test
    # test_kernels_report_sm100 asks the runtime for the loaded kernels' version
    import build
    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "compute_90" not in flags and "sm_90" not in flags


def test_status_strings(gfsph_lib):
    assert gfsph_lib.strerror(0) == "ok"
    assert "CUDA device" in gfsph_lib.strerror(-6)
    assert gfsph_lib.strerror(-9) == "host memory allocation failed"
    assert gfsph_lib.lib().gfsph_version() >= 1


def test_rejects_unsupported_options_before_touching_the_device(gfsph_lib):
    z = np.zeros((8, 8), np.float32)
    base = {1: 9.8, 2: 2000, 3: 500, 5: 5, 9: 0.2, 10: 0.01, 15: 0.01}
    for const, bad in (({}, dict(skf=5)), ({}, dict(skf=2, nnps=4)), ({}, dict(nor_density=2)), ({}, dict(pa_sph=3)), ({16: 2.0}, {}),
                       ({}, dict(ic_adapt=3))):
        p = gfsph_lib.make_params({**base, **const}, **bad)
        with pytest.raises(gfsph_lib.GfsphError) as e:
            gfsph_lib.Sim(p, z, dx=1.0, dy=1.0)
        assert e.value.status == -4
    p = gfsph_lib.make_params({1: 9.8, 2: 2000, 3: 500, 5: 1, 9: 0.2, 10: 0.01, 15: 0.01})  # Manning
    with pytest.raises(gfsph_lib.GfsphError):
        gfsph_lib.Sim(p, z, dx=1.0, dy=1.0)
    for mn in (-1, 65537):  # initial neighbour-table capacity outside 0..65536
        p = gfsph_lib.make_params(base, max_neighbours=mn)
        with pytest.raises(gfsph_lib.GfsphError) as e:
            gfsph_lib.Sim(p, z, dx=1.0, dy=1.0)
        assert e.value.status == -1


def test_no_cpu_fallback_without_device(gfsph_lib):
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    p = gfsph_lib.make_params({1: 9.8, 2: 2000, 3: 500, 5: 5, 9: 0.2, 10: 0.01, 15: 0.01})
    with pytest.raises(gfsph_lib.GfsphError) as e:
        gfsph_lib.Sim(p, np.zeros((8, 8), np.float32), dx=1.0, dy=1.0)
    assert e.value.status == -6


def test_fortran_interface_names_every_symbol():
    src = open(os.path.join(ROOT, "deslizamientos-y-flujos_b200", "fortran", "gfsph_c.f90")).read().lower()
    for s in declared_symbols():
        assert f'bind(c, name="{s}")' in src, s


def test_fortran_module_names_every_status_code():
    """GFSPH_OK .. GFSPH_ERR_* of the header, each with the header's value."""
    hdr = open(os.path.join(ROOT, "include", "gfsph.h")).read()
    codes = {m.group(1): int(m.group(2)) for m in
             re.finditer(r"#define (GFSPH_(?:OK|T_END_REACHED|ERR_[A-Z_]+))\s+\(?(-?\d+)\)?", hdr)}
    assert len(codes) >= 11
    f90 = open(os.path.join(ROOT, "deslizamientos-y-flujos_b200", "fortran", "gfsph_c.f90")).read()
    for name, value in codes.items():
        m = re.search(rf"\b{name}\s*=\s*(-?\d+)", f90)
        assert m and int(m.group(1)) == value, name


def _c_declarations():
    """{name: argument count} of the functions include/gfsph.h declares."""
    src = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "gfsph.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(gfsph_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", src):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def _fortran_interfaces():
    """{C name: argument count} of the BIND(C) interfaces of the Fortran module."""
    path = os.path.join(os.path.dirname(os.path.dirname(__file__)), "deslizamientos-y-flujos_b200", "fortran",
                        "gfsph_c.f90")
    src = re.sub(r"&\s*\n\s*", " ", open(path).read())
    out = {}
    for m in re.finditer(r"function\s+\w+\s*\(([^)]*)\)\s*bind\(c,\s*name=\"(gfsph_[a-z0-9_]+)\"\)", src):
        args = m.group(1).strip()
        out[m.group(2)] = 0 if not args else args.count(",") + 1
    return out


def test_fortran_module_binds_every_entry_point():
    """The Fortran module (the reference's side of the boundary) declares every
    function of the C header, with the same number of arguments."""
    c, f = _c_declarations(), _fortran_interfaces()
    assert len(c) > 30
    assert sorted(set(c) - set(f)) == []
    for name, nargs in c.items():
        assert f[name] == nargs, (name, nargs, f[name])


def test_adjoint_record_refuses_a_closed_sim(gfsph_lib):
    """The record steps its handle: once the Sim is closed the binding refuses
    the backward pass (GFSPH_ERR_STATE) instead of passing a freed handle."""
    class ClosedSim:
        h = None
        n = 4
    adj = gfsph_lib.Adjoint.__new__(gfsph_lib.Adjoint)
    adj.sim, adj.h = ClosedSim(), None
    g = np.zeros((4, 2), np.float32)
    with pytest.raises(gfsph_lib.GfsphError) as e:
        adj.backward(g, g)
    assert e.value.status == -5
