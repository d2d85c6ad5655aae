"""Python binding of the gfsph C ABI (include/gfsph.h) over ctypes.

This is the host-side mirror of the reference's step interface for tests and
benchmarks: the Fortran host of the reference would bind the same symbols
through ISO_C_BINDING (fortran/gfsph_c.f90).  Arrays follow the Fortran
layout: particle vectors are (n, 2) float32 in C order, which is the (2, n)
column-major layout of the reference.

There is no CPU fallback: without libgfsph.so, or without a CUDA device, the
calls raise.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgfsph.so")

NCONST = 110
NTOPO = 16

OK = 0
T_END_REACHED = 1
ERR_ARG = -1
ERR_CUDA = -2
ERR_CAPACITY = -3
ERR_UNSUPPORTED = -4
ERR_STATE = -5
ERR_NO_DEVICE = -6

RASTER_DEPTH_IDW = 0
RASTER_MAX_DEPTH = 1
RASTER_MAX_VEL = 2
RASTER_SUM_DEPTH = 3
RASTER_SUM_VEL = 4
RASTER_COUNT = 5
RASTER_Z = 6
RASTER_ERODED = 7
RASTER_AVAILABLE = 8


class Params(C.Structure):
    _fields_ = [
        ("cst", C.c_float * NCONST),
        ("pa_sph", C.c_int), ("nnps", C.c_int), ("sle", C.c_int), ("skf", C.c_int),
        ("summation_density", C.c_int), ("average_velocity", C.c_int), ("nor_density", C.c_int),
        ("ic_adapt", C.c_int), ("h_inf", C.c_float), ("dt", C.c_float), ("dem_deriv", C.c_int),
        ("max_neighbours", C.c_int), ("icpwp", C.c_int), ("pwp0rel", C.c_float), ("ws_interact", C.c_int),
        ("sw_alg", C.c_int), ("reserved", C.c_int * 4),
    ]


class Dem(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("xmin", C.c_float), ("ymin", C.c_float),
        ("dx", C.c_float), ("dy", C.c_float), ("topol", C.POINTER(C.c_float)), ("ntopo", C.c_int),
        ("z", C.POINTER(C.c_float)),
    ]


_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_lib = None

# every symbol include/gfsph.h declares, with its ctypes signature
class GflParams(C.Structure):
    """gfsph_gfl_params: constF[k-1] = constF(k) of the GFL .dat, the flow
    type (2 under a still-water level, 3 over a dry bed), Gauss points per
    triangle, consistent-mass sweeps, still-water level, dry depth."""
    _fields_ = [("constF", C.c_float * 15), ("ntype", C.c_int), ("ngaus", C.c_int), ("niter", C.c_int),
                ("swl", C.c_float), ("comp", C.c_float)]


SIGNATURES = {
    "gfsph_create": (C.c_int, [C.POINTER(Params), C.POINTER(Dem), C.POINTER(C.c_void_p)]),
    "gfsph_destroy": (C.c_int, [C.c_void_p]),
    "gfsph_upload": (C.c_int, [C.c_void_p, C.c_int, _FP, _FP, _FP, _FP, _FP, _IP, _IP]),
    "gfsph_download": (C.c_int, [C.c_void_p, _FP, _FP, _FP, _FP, _FP, _IP]),
    "gfsph_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double), _IP]),
    "gfsph_get_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), _FP]),
    "gfsph_set_time": (C.c_int, [C.c_void_p, C.c_double, C.c_float]),
    "gfsph_density": (C.c_int, [C.c_void_p, _FP]),
    "gfsph_neighbours": (C.c_int, [C.c_void_p, C.c_int, _IP, _IP]),
    "gfsph_internal_forces": (C.c_int, [C.c_void_p, _FP]),
    "gfsph_raster": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "gfsph_hazard_sample": (C.c_int, [C.c_void_p]),
    "gfsph_raster_misfit": (C.c_int, [C.c_void_p, _FP, C.POINTER(C.c_double), _FP, _FP]),
    "gfsph_hazard_reset": (C.c_int, [C.c_void_p]),
    "gfsph_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gfsph_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "gfsph_profile_read": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "gfsph_num_kernels": (C.c_int, []),
    "gfsph_kernel_name": (C.c_char_p, [C.c_int]),
    "gfsph_launch_count": (C.c_longlong, [C.c_void_p]),
    "gfsph_stats": (C.c_int, [C.c_void_p, _IP, C.c_int]),
    "gfsph_dem_topol": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _FP]),
    "gfsph_raster_idw_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float,
                                           C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_void_p]),
    "gfsph_set_search": (C.c_int, [C.c_void_p, C.c_float, C.c_float]),
    "gfsph_get_search": (C.c_int, [C.c_void_p, _FP, _FP]),
    "gfsph_autotune": (C.c_int, [C.c_void_p, C.c_int, _FP, _FP, _FP]),
    "gfsph_adjoint_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "gfsph_adjoint_backward": (C.c_int, [C.c_void_p, _FP, _FP, _FP, _FP, _FP, _FP, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]),
    "gfsph_adjoint_param": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "gfsph_adjoint_destroy": (C.c_int, [C.c_void_p]),
    "gfsph_gradhs": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, _FP, _FP]),
    "gfsph_set_pwp": (C.c_int, [C.c_void_p, _FP]),
    "gfsph_get_pwp": (C.c_int, [C.c_void_p, _FP]),
    "gfsph_ensemble_create": (C.c_int, [C.POINTER(Params), C.POINTER(Dem), C.c_int, C.POINTER(C.c_void_p)]),
    "gfsph_ensemble_destroy": (C.c_int, [C.c_void_p]),
    "gfsph_ensemble_member": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "gfsph_ensemble_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _IP]),
    "gfsph_ensemble_sample": (C.c_int, [C.c_void_p]),
    "gfsph_ensemble_exceedance": (C.c_int, [C.c_void_p, C.c_float, _FP]),
    "gfsph_cg_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _IP, _FP, C.POINTER(C.c_void_p)]),
    "gfsph_cg_solve": (C.c_int, [C.c_void_p, _IP, _FP, _FP, _FP, C.c_float, _IP]),
    "gfsph_cg_destroy": (C.c_int, [C.c_void_p]),
    "gfsph_cg_launch_count": (C.c_longlong, [C.c_void_p]),
    "gfsph_cg_device_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "gfsph_solvegc2": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _IP, _IP, _FP, _FP, _FP, _FP, C.c_float, _IP]),
    "gfsph_gfl_create": (C.c_int, [C.POINTER(GflParams), C.c_int, C.c_int, _FP, _IP, _FP, C.POINTER(C.c_void_p)]),
    "gfsph_gfl_destroy": (C.c_int, [C.c_void_p]),
    "gfsph_gfl_set_state": (C.c_int, [C.c_void_p, _FP, C.c_double]),
    "gfsph_gfl_get_state": (C.c_int, [C.c_void_p, _FP, C.POINTER(C.c_double)]),
    "gfsph_gfl_set_wir": (C.c_int, [C.c_void_p, _FP, _FP]),
    "gfsph_gfl_step": (C.c_int, [C.c_void_p, C.c_int, C.c_float]),
    "gfsph_gfl_topol": (C.c_int, [C.c_void_p, _FP, _FP]),
    "gfsph_gfl_launch_count": (C.c_longlong, [C.c_void_p]),
    "gfsph_gfl_device_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "gfsph_strerror": (C.c_char_p, [C.c_int]),
    "gfsph_version": (C.c_int, []),
    "gfsph_binary_version": (C.c_int, [_IP]),
}


class GfsphError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {status} ({strerror(status)})")


def lib():
    """Loads libgfsph.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run build.py (the CUDA library is required)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def strerror(status):
    return lib().gfsph_strerror(status).decode()


def _check(st, what):
    if st < 0:
        raise GfsphError(st, what)
    return st


def _fp(a):
    return a.ctypes.data_as(_FP) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(_IP) if a is not None else None


def make_params(const=None, *, pa_sph=2, nnps=2, sle=1, skf=1, summation_density=1, average_velocity=1,
                nor_density=0, ic_adapt=0, h_inf=0.01, dt=0.01, dem_deriv=1, max_neighbours=0, icpwp=0, pwp0rel=0.0,
                ws_interact=0, sw_alg=0):
    """Params from a {k: value} map of the reference's const(k) (1-based)."""
    p = Params()
    for k, val in (const or {}).items():
        p.cst[k - 1] = float(val)
    p.pa_sph, p.nnps, p.sle, p.skf = pa_sph, nnps, sle, skf
    p.summation_density, p.average_velocity, p.nor_density = summation_density, average_velocity, nor_density
    p.ic_adapt, p.h_inf, p.dt, p.dem_deriv, p.max_neighbours = ic_adapt, h_inf, dt, dem_deriv, max_neighbours
    p.icpwp, p.pwp0rel = icpwp, pwp0rel
    p.ws_interact, p.sw_alg = ws_interact, sw_alg
    return p


def dem_topol(z, dx, dy, mode=1):
    """Slope/curvature rows topol(2..13) from Z with the library's host set-up."""
    ny, nx = z.shape
    t = np.zeros((ny * nx, NTOPO), dtype=np.float32)
    t[:, 0] = z.reshape(-1)
    _check(lib().gfsph_dem_topol(mode, nx, ny, dx, dy, _fp(t)), "gfsph_dem_topol")
    return t


class Sim:
    """One gfsph handle: a DEM, a particle set and the step state."""

    def __init__(self, params, z=None, *, xmin=0.0, ymin=0.0, dx=1.0, dy=1.0, topol=None):
        L = lib()
        if topol is not None:
            topol = np.ascontiguousarray(topol, dtype=np.float32)
            ny, nx = (z.shape if z is not None else (None, None))
            if nx is None:
                raise ValueError("pass z (for the grid shape) together with topol")
        else:
            z = np.ascontiguousarray(z, dtype=np.float32)
            ny, nx = z.shape
        self.nx, self.ny = nx, ny
        self.params = params
        self._z = np.ascontiguousarray(z, dtype=np.float32)
        self._topol = topol
        d = Dem()
        d.nx, d.ny, d.xmin, d.ymin, d.dx, d.dy = nx, ny, xmin, ymin, dx, dy
        d.topol = _fp(topol) if topol is not None else None
        d.ntopo = topol.shape[1] if topol is not None else 0
        d.z = _fp(self._z)
        self.dem = d
        h = C.c_void_p()
        _check(L.gfsph_create(C.byref(params), C.byref(d), C.byref(h)), "gfsph_create")
        self.h = h
        self.n = 0

    def close(self):
        if self.h:
            lib().gfsph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, x, v, rho, mass, hsml, flag=None, itype=None):
        """itype: the material of each particle (1 soil, 2 water; water only
        with ws_interact = 1); None is all soil."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        self._up = [x, np.ascontiguousarray(v, dtype=np.float32), np.ascontiguousarray(rho, dtype=np.float32),
                    np.ascontiguousarray(mass, dtype=np.float32), np.ascontiguousarray(hsml, dtype=np.float32),
                    None if flag is None else np.ascontiguousarray(flag, dtype=np.int32),
                    None if itype is None else np.ascontiguousarray(itype, dtype=np.int32)]
        a = self._up
        _check(lib().gfsph_upload(self.h, n, _fp(a[0]), _fp(a[1]), _fp(a[2]), _fp(a[3]), _fp(a[4]), _ip(a[6]),
                                  _ip(a[5])), "gfsph_upload")
        self.n = n

    def download(self, out=None):
        n = self.n
        if out is None:
            out = dict(x=np.empty((n, 2), np.float32), v=np.empty((n, 2), np.float32), rho=np.empty(n, np.float32),
                       mass=np.empty(n, np.float32), hsml=np.empty(n, np.float32), flag=np.empty(n, np.int32))
        _check(lib().gfsph_download(self.h, _fp(out["x"]), _fp(out["v"]), _fp(out["rho"]), _fp(out["mass"]),
                                    _fp(out["hsml"]), _ip(out["flag"])), "gfsph_download")
        return out

    def set_search(self, level_factor, cell_div):
        _check(lib().gfsph_set_search(self.h, level_factor, cell_div), "gfsph_set_search")

    def get_search(self):
        a, b = C.c_float(), C.c_float()
        _check(lib().gfsph_get_search(self.h, C.byref(a), C.byref(b)), "gfsph_get_search")
        return a.value, b.value

    def autotune(self, steps=8):
        """Picks the fastest search tunables on the current state: (level_factor, cell_div, ms/step)."""
        a, b, t = C.c_float(), C.c_float(), C.c_float()
        _check(lib().gfsph_autotune(self.h, steps, C.byref(a), C.byref(b), C.byref(t)), "gfsph_autotune")
        return a.value, b.value, t.value

    def gradhs(self, ix0, iy0, nwx, nwy, niter=5, tol=1e-10):
        """get_gradhs_w on a DEM node window: (hs_w (nwy, nwx), gradhs_w (nwy, nwx, 2))."""
        hs = np.empty((nwy, nwx), np.float32)
        g = np.empty((nwy, nwx, 2), np.float32)
        _check(lib().gfsph_gradhs(self.h, ix0, iy0, nwx, nwy, niter, tol, _fp(hs), _fp(g)), "gfsph_gradhs")
        return hs, g

    def pwp(self):
        """The basal pore-water pressure: u (icpwp = 1) or Uaux(1,:) (icpwp = 3)."""
        out = np.empty(self.n, np.float32)
        _check(lib().gfsph_get_pwp(self.h, _fp(out)), "gfsph_get_pwp")
        return out

    def set_pwp(self, pwp):
        a = np.ascontiguousarray(pwp, dtype=np.float32)
        _check(lib().gfsph_set_pwp(self.h, _fp(a)), "gfsph_set_pwp")

    def step(self, nsteps, t_end=1e300):
        t = C.c_double()
        done = C.c_int()
        st = _check(lib().gfsph_step(self.h, nsteps, t_end, C.byref(t), C.byref(done)), "gfsph_step")
        return st, t.value, done.value

    def time(self):
        t = C.c_double()
        dt = C.c_float()
        _check(lib().gfsph_get_time(self.h, C.byref(t), C.byref(dt)), "gfsph_get_time")
        return t.value, dt.value

    def set_time(self, t, dt):
        _check(lib().gfsph_set_time(self.h, t, dt), "gfsph_set_time")

    def density(self):
        rho = np.empty(self.n, np.float32)
        _check(lib().gfsph_density(self.h, _fp(rho)), "gfsph_density")
        return rho

    def internal_forces(self):
        a = np.empty((self.n, 2), np.float32)
        _check(lib().gfsph_internal_forces(self.h, _fp(a)), "gfsph_internal_forces")
        return a

    def neighbours(self):
        off = np.empty(self.n + 1, np.int32)
        st = lib().gfsph_neighbours(self.h, 0, _ip(off), None)
        if st < 0 and st != -3:
            _check(st, "gfsph_neighbours")
        cap = int(off[-1])
        idx = np.empty(max(cap, 1), np.int32)
        _check(lib().gfsph_neighbours(self.h, cap, _ip(off), _ip(idx)), "gfsph_neighbours")
        return off, idx[:cap]

    def raster(self, kind):
        out = np.empty((self.ny, self.nx), np.float32)
        _check(lib().gfsph_raster(self.h, kind, _fp(out)), "gfsph_raster")
        return out

    def raster_misfit(self, target):
        """L = sum (R - T)^2 of the depth raster R against `target` (ny, nx),
        with dL/dx (n, 2) and dL/dh (n,) of the current state."""
        t = np.ascontiguousarray(target, np.float32)
        loss = C.c_double()
        gx = np.empty((self.n, 2), np.float32)
        gh = np.empty(self.n, np.float32)
        _check(lib().gfsph_raster_misfit(self.h, _fp(t), C.byref(loss), _fp(gx), _fp(gh)), "gfsph_raster_misfit")
        return loss.value, gx, gh

    def hazard_sample(self):
        _check(lib().gfsph_hazard_sample(self.h), "gfsph_hazard_sample")

    def hazard_reset(self):
        _check(lib().gfsph_hazard_reset(self.h), "gfsph_hazard_reset")

    def set_stream(self, stream_ptr):
        _check(lib().gfsph_set_stream(self.h, C.c_void_p(stream_ptr)), "gfsph_set_stream")

    def profile(self, level):
        """0 off, 1 per-kernel events, 2 events around each step call."""
        _check(lib().gfsph_profile(self.h, int(level)), "gfsph_profile")

    def profile_read(self):
        L = lib()
        res = {}
        for k in range(L.gfsph_num_kernels()):
            ms = C.c_double()
            cnt = C.c_longlong()
            _check(L.gfsph_profile_read(self.h, k, C.byref(ms), C.byref(cnt)), "gfsph_profile_read")
            if cnt.value:
                res[L.gfsph_kernel_name(k).decode()] = (ms.value, cnt.value)
        return res

    def launch_count(self):
        return int(lib().gfsph_launch_count(self.h))

    def stats(self):
        v = np.zeros(8, np.int32)
        _check(lib().gfsph_stats(self.h, _ip(v), 8), "gfsph_stats")
        keys = ("active", "regular", "coarse", "levels", "cells", "table_capacity", "cell_capacity", "outside")
        return dict(zip(keys, (int(a) for a in v)))


class CG:
    """solvegc2 on the device for a fixed element system (gfsph_cg_*).

    intmat: (nelem, nnode) 1-based; gstif: (nelem, nevab, nevab) with
    [e, row, col]."""

    def __init__(self, intmat, gstif, ndofn=1):
        intmat = np.ascontiguousarray(intmat, np.int32)
        self.nelem, self.nnode = intmat.shape
        self.npoin = int(intmat.max())
        self.n = self.npoin * ndofn
        g = np.ascontiguousarray(np.transpose(gstif, (0, 2, 1)), np.float32)  # Fortran gstif(nevab, nevab, nelem)
        self._keep = (intmat, g)
        h = C.c_void_p()
        _check(lib().gfsph_cg_create(self.npoin, self.nelem, self.nnode, ndofn, _ip(intmat), _fp(g), C.byref(h)),
               "gfsph_cg_create")
        self.h = h

    def solve(self, rhs, iffix=None, fixed=None, tol=1e-10):
        n = self.n
        fix = np.zeros(n, np.int32) if iffix is None else np.ascontiguousarray(iffix, np.int32).copy()
        fx = np.zeros(n, np.float32) if fixed is None else np.ascontiguousarray(fixed, np.float32)
        r = np.ascontiguousarray(rhs, np.float32).copy()
        x = np.zeros(n, np.float32)
        it = C.c_int(0)
        _check(lib().gfsph_cg_solve(self.h, _ip(fix), _fp(fx), _fp(r), _fp(x), tol, C.byref(it)), "gfsph_cg_solve")
        return x, r, fix, it.value

    def launch_count(self):
        return int(lib().gfsph_cg_launch_count(self.h))

    def device_ms(self):
        """Device time of the last solve (its kernels, without the host copies)."""
        ms = C.c_double(0.0)
        _check(lib().gfsph_cg_device_ms(self.h, C.byref(ms)), "gfsph_cg_device_ms")
        return ms.value

    def close(self):
        if self.h:
            lib().gfsph_cg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Gfl:
    """The GFL Taylor-Galerkin shallow-water step on the device (gfsph_gfl_*).

    coord (npoin, 2), intmat (nelem, 3) 1-based counter-clockwise, z (npoin);
    const: {k: constF(k)}; the state unkno (npoin, 3) = h, hu, hv."""

    def __init__(self, coord, intmat, z, const, ntype=3, ngaus=3, niter=3, swl=0.0, comp=0.01):
        p = GflParams()
        for k, v in const.items():
            p.constF[k - 1] = v
        p.ntype, p.ngaus, p.niter, p.swl, p.comp = ntype, ngaus, niter, swl, comp
        c = np.ascontiguousarray(coord, np.float32)
        im = np.ascontiguousarray(intmat, np.int32)
        zz = np.ascontiguousarray(z, np.float32)
        self.npoin, self.nelem = c.shape[0], im.shape[0]
        h = C.c_void_p()
        _check(lib().gfsph_gfl_create(C.byref(p), self.npoin, self.nelem, _fp(c), _ip(im), _fp(zz), C.byref(h)),
               "gfsph_gfl_create")
        self.h = h

    def set_state(self, unkno, time=0.0):
        u = np.ascontiguousarray(unkno, np.float32)
        _check(lib().gfsph_gfl_set_state(self.h, _fp(u), time), "gfsph_gfl_set_state")

    def state(self):
        u = np.empty((self.npoin, 3), np.float32)
        t = C.c_double()
        _check(lib().gfsph_gfl_get_state(self.h, _fp(u), C.byref(t)), "gfsph_gfl_get_state")
        return u, t.value

    def set_wir(self, hs_w=None, gradhs_w=None):
        if hs_w is None:
            _check(lib().gfsph_gfl_set_wir(self.h, None, None), "gfsph_gfl_set_wir")
            return
        a = np.ascontiguousarray(hs_w, np.float32)
        b = np.ascontiguousarray(gradhs_w, np.float32)
        _check(lib().gfsph_gfl_set_wir(self.h, _fp(a), _fp(b)), "gfsph_gfl_set_wir")

    def step(self, nsteps, dt):
        _check(lib().gfsph_gfl_step(self.h, nsteps, dt), "gfsph_gfl_step")

    def topol(self):
        t = np.empty((self.npoin, 9), np.float32)
        e = np.empty((self.nelem, 9), np.float32)
        _check(lib().gfsph_gfl_topol(self.h, _fp(t), _fp(e)), "gfsph_gfl_topol")
        return t, e

    def launch_count(self):
        return int(lib().gfsph_gfl_launch_count(self.h))

    def device_ms(self):
        """Device time of the last step call (its kernels)."""
        ms = C.c_double(0.0)
        _check(lib().gfsph_gfl_device_ms(self.h, C.byref(ms)), "gfsph_gfl_device_ms")
        return ms.value

    def close(self):
        if self.h:
            lib().gfsph_gfl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Member(Sim):
    """A member handle of an ensemble (owned by the ensemble)."""

    def __init__(self, handle, nx, ny, params):
        self.h = handle
        self.nx, self.ny = nx, ny
        self.params = params
        self.n = 0

    def close(self):
        self.h = None


class Ensemble:
    """gfsph_ensemble: realizations with their own parameters on one DEM."""

    def __init__(self, params_list, z, *, xmin=0.0, ymin=0.0, dx=1.0, dy=1.0):
        L = lib()
        self._z = np.ascontiguousarray(z, dtype=np.float32)
        ny, nx = self._z.shape
        arr = (Params * len(params_list))(*params_list)
        self._params = arr
        d = Dem()
        d.nx, d.ny, d.xmin, d.ymin, d.dx, d.dy = nx, ny, xmin, ymin, dx, dy
        d.topol = None
        d.ntopo = 0
        d.z = _fp(self._z)
        self.dem = d
        h = C.c_void_p()
        _check(L.gfsph_ensemble_create(arr, C.byref(d), len(params_list), C.byref(h)), "gfsph_ensemble_create")
        self.h = h
        self.nx, self.ny = nx, ny
        self.members = []
        for r in range(len(params_list)):
            m = C.c_void_p()
            _check(L.gfsph_ensemble_member(h, r, C.byref(m)), "gfsph_ensemble_member")
            self.members.append(_Member(m, nx, ny, params_list[r]))

    def step(self, nsteps, t_end=1e300):
        done = C.c_int()
        st = _check(lib().gfsph_ensemble_step(self.h, nsteps, t_end, C.byref(done)), "gfsph_ensemble_step")
        return st, done.value

    def sample(self):
        _check(lib().gfsph_ensemble_sample(self.h), "gfsph_ensemble_sample")

    def exceedance(self, threshold):
        out = np.empty((self.ny, self.nx), np.float32)
        _check(lib().gfsph_ensemble_exceedance(self.h, threshold, _fp(out)), "gfsph_ensemble_exceedance")
        return out

    def close(self):
        if self.h:
            for m in self.members:
                m.close()
            lib().gfsph_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """gfsph_adjoint_*: records `nsteps` steps of `sim` (keeping the state
    every `every` steps) and returns gradients of a loss on the final state."""

    def __init__(self, sim, nsteps, every=1):
        self.sim = sim
        h = C.c_void_p()
        _check(lib().gfsph_adjoint_forward(sim.h, nsteps, every, C.byref(h)), "gfsph_adjoint_forward")
        self.h = h

    def backward(self, gx, gv, gh=None):
        """dL/dx, dL/dv (n, 2) and dL/dh (n,) of the final state -> dict of
        dL/dx0, dL/dv0, dL/dmass, dL/dtanfi (const(9)), dL/dxi (const(3)),
        dL/dtauy (const(6), the Bingham yield stress)."""
        if not self.h or not self.sim.h:  # the record steps its handle, which must still exist
            raise GfsphError(-5, "gfsph_adjoint_backward")
        n = self.sim.n
        gx = np.ascontiguousarray(gx, np.float32)
        gv = np.ascontiguousarray(gv, np.float32)
        ghh = None if gh is None else np.ascontiguousarray(gh, np.float32)
        out = dict(x0=np.empty((n, 2), np.float32), v0=np.empty((n, 2), np.float32), mass=np.empty(n, np.float32))
        mu, xi = C.c_double(), C.c_double()
        _check(lib().gfsph_adjoint_backward(self.h, _fp(gx), _fp(gv), _fp(ghh), _fp(out["x0"]), _fp(out["v0"]),
                                            _fp(out["mass"]), C.byref(mu), C.byref(xi)), "gfsph_adjoint_backward")
        out["tanfi"], out["xi"] = mu.value, xi.value
        ty = C.c_double()
        _check(lib().gfsph_adjoint_param(self.h, 2, C.byref(ty)), "gfsph_adjoint_param")
        out["tauy"] = ty.value  # dL/d(Bingham yield stress, const(6))
        return out

    def close(self):
        if self.h:
            lib().gfsph_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
