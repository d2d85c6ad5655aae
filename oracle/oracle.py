"""TEST INFRASTRUCTURE ONLY — Python binding of the CPU oracle (gfsph_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and
reference arm use this, as the checker or as the timed CPU baseline.
Parity status: unpinned (the reference ships no tests or golden outputs and
cannot be compiled here); see the header of gfsph_oracle.cpp.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libgfsph_oracle.so")
# the same source built with OpenMP: only for timing the CPU baseline on all
# host cores (its pair sums are added in another order than the checker's)
LIB_OMP = os.path.join(HERE, "_build", "libgfsph_oracle_omp.so")
NTOPO = 16

MODE_FP32 = 0        # reference FP32 build
MODE_FP32_DACC = 1   # FP32 state, FP64 sums (the GPU scheme)
MODE_FP64 = 2        # reference FP64 build
MODE_POS64 = 3       # precision experiment: mode 1 with the RK45 position updates in FP64 (Run only)

_libs = {}
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


def build():
    """Builds the checker library (and the OpenMP one where the compiler
    takes -fopenmp) when missing or older than the source."""
    def mtime(*names):
        return max(os.path.getmtime(os.path.join(HERE, f)) for f in names)

    hdr = os.path.join("..", "include", "gfsph.h")
    newest = mtime("gfsph_oracle.cpp", "gfl_oracle.cpp", hdr)
    newest_omp = mtime("gfsph_oracle.cpp", hdr)  # the OpenMP build holds the SPH step only
    if not (os.path.exists(LIB) and os.path.getmtime(LIB) >= newest
            and (not os.path.exists(LIB_OMP) or os.path.getmtime(LIB_OMP) >= newest_omp)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def omp_available():
    return os.path.exists(LIB_OMP)


def _cgroup_cpus():
    """CPUs the container's CPU quota allows (cgroup v2 or v1), else None."""
    try:
        with open("/sys/fs/cgroup/cpu.max") as f:
            q, per = f.read().split()[:2]
        if q != "max":
            return max(1, -(-int(q) // int(per)))
    except (OSError, ValueError):
        pass
    try:
        with open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us") as f:
            q = int(f.read())
        with open("/sys/fs/cgroup/cpu/cpu.cfs_period_us") as f:
            per = int(f.read())
        if q > 0 and per > 0:
            return max(1, -(-q // per))
    except (OSError, ValueError):
        pass
    return None


def omp_threads():
    """Threads the OpenMP library runs with: OMP_NUM_THREADS, else every
    host core this process may use, capped by the container's CPU quota."""
    env = os.environ.get("OMP_NUM_THREADS", "").split(",")[0].strip()
    if env.isdigit() and int(env) > 0:
        return int(env)
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    q = _cgroup_cpus()
    return min(n, q) if q else n


def lib(omp=False):
    path = LIB_OMP if omp else LIB
    if path not in _libs:
        if not os.path.exists(path):
            build()
        if not os.path.exists(path):
            raise RuntimeError("the OpenMP oracle library was not built (no compiler with -fopenmp)")
        L = C.CDLL(path)
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_double, _DP, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _DP, C.c_int, C.c_int,
                                 _DP, _DP, C.c_double, _IP]
        L.oracle_pairs.restype = C.c_int
        L.oracle_pairs.argtypes = [C.c_int, C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, _IP, C.c_int, _IP, _IP, _DP,
                                   _DP]
        L.oracle_kernel.restype = C.c_int
        L.oracle_kernel.argtypes = [C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP, _DP]
        L.oracle_dem_topol.restype = C.c_int
        L.oracle_dem_topol.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _DP]
        L.oracle_raster_idw.restype = C.c_int
        L.oracle_raster_idw.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                        _DP, _DP, _IP, _DP]
        L.oracle_hazard_sample.restype = C.c_int
        L.oracle_hazard_sample.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_int, _DP, _DP, _DP, _IP, _DP, _IP]
        L.oracle_new.restype = C.c_void_p
        L.oracle_new.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_double, _DP, C.c_int, _DP, _DP, _DP, _DP, _DP, _IP, _DP, C.c_double,
                                 C.c_double, _IP]
        L.oracle_advance.restype = C.c_int
        L.oracle_advance.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.oracle_get.restype = C.c_int
        L.oracle_get.argtypes = [C.c_void_p, _DP, _DP, _DP, _DP, _DP, _IP, _DP, _DP, _DP]
        L.oracle_gradhs.restype = C.c_int
        L.oracle_gradhs.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int, _DP, _DP, _IP, _DP, C.c_int, _DP, _DP]
        for fn in (L.oracle_tangent, L.oracle_tangent32):
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                           _DP, C.c_int, _DP, _DP, _DP, _DP, _DP, _IP, C.c_int, C.c_double, C.c_double,
                           C.c_double, C.c_double, C.c_double, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP]
        L.oracle_get_pwp.restype = C.c_int
        L.oracle_get_pwp.argtypes = [C.c_void_p, _DP]
        L.oracle_free.restype = None
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_set_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        if hasattr(L, "oracle_gfl_run"):
            L.oracle_gfl_run.restype = C.c_int
            L.oracle_gfl_run.argtypes = [C.c_int, C.c_int, _DP, _IP, _DP, _DP, C.c_int, C.c_int, C.c_int, C.c_double,
                                         C.c_double, _DP, _DP, _DP, C.c_int, C.c_double, _DP, _DP, _DP]
        L.oracle_solvegc2.restype = C.c_int
        L.oracle_solvegc2.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _IP, _IP, _DP, _DP, _DP, _DP,
                                      C.c_double, _IP]
        _libs[path] = L
    return _libs[path]


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dp(a):
    return a.ctypes.data_as(_DP) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(_IP) if a is not None else None


def dem_topol(z, dx, dy, deriv=1, mode=MODE_FP32):
    """topol (npoig, 16) with rows 2..13 derived from Z (Get_Topol / Fdiff_derivs)."""
    ny, nx = z.shape
    t = np.zeros((ny * nx, NTOPO), np.float64)
    t[:, 0] = z.reshape(-1)
    st = lib().oracle_dem_topol(mode, deriv, nx, ny, dx, dy, _dp(t))
    if st:
        raise RuntimeError(f"oracle_dem_topol: {st}")
    return t


def initial_topol(z, dx, dy, const, deriv=1, mode=MODE_FP32):
    """DEM rows as the reference has them before the time loop (slopes + erodible depth)."""
    t = dem_topol(z, dx, dy, deriv, mode)
    avail = 0.0
    if const.get(21, 0.0) > 1e-9:
        avail = const[48] if const.get(48, 0.0) > 1e-6 else 999.0
    t[:, 14] = np.float32(avail)
    return t


class State:
    """Particle state and DEM of an oracle run (float64 arrays)."""

    def __init__(self, x, v, rho, mass, hsml, topol, flag=None, dt=0.01, t=0.0, pwp=None, mass0=None):
        """pwp: u (icpwp = 1) or Uaux(1,:) (icpwp = 3); None starts it as Input_SW does.
        mass0: the masses at the start of the run (nfric 3); None takes mass."""
        self.x, self.v = _d(x).copy(), _d(v).copy()
        self.rho, self.mass, self.hsml = _d(rho).copy(), _d(mass).copy(), _d(hsml).copy()
        self.mass0 = self.mass.copy() if mass0 is None else _d(mass0).copy()
        n = self.x.shape[0]
        self.flag = np.zeros(n, np.int32) if flag is None else np.ascontiguousarray(flag, np.int32).copy()
        self.topol = _d(topol).copy()
        self.dt, self.t = float(dt), float(t)
        self.pwp = None if pwp is None else _d(pwp).copy()

    def copy(self):
        s = State(self.x, self.v, self.rho, self.mass, self.hsml, self.topol, self.flag, self.dt, self.t, self.pwp,
                  self.mass0)
        return s


def run(mode, params, nx, ny, dx, dy, state, nsteps, xmin=0.0, ymin=0.0, t_end=1e300):
    """Advances `state` in place by nsteps reference steps; returns steps done."""
    dt = C.c_double(state.dt)
    t = C.c_double(state.t)
    done = C.c_int(0)
    n = state.x.shape[0]
    init = 0
    if params.icpwp in (1, 3) and state.pwp is None:
        state.pwp, init = np.zeros(n), 1
    st = lib().oracle_run(mode, C.addressof(params), nx, ny, xmin, ymin, dx, dy, _dp(state.topol),
                          n, _dp(state.x), _dp(state.v), _dp(state.rho), _dp(state.mass), _dp(state.mass0),
                          _dp(state.hsml), _ip(state.flag), _dp(state.pwp), init,
                          nsteps, C.byref(dt), C.byref(t), t_end, C.byref(done))
    if st:
        raise RuntimeError(f"oracle_run: {st}")
    state.dt, state.t = dt.value, t.value
    return done.value


def pairs(mode, params, x, hsml, mass=None, rho=None, flag=None, want_sets=True, want_rho=False,
          want_force=False):
    """Neighbour sets (CSR), summation density, internal forces of one state."""
    x, hsml = _d(x), _d(hsml)
    n = x.shape[0]
    mass = _d(mass) if mass is not None else None
    rho = _d(rho) if rho is not None else None
    flag = np.zeros(n, np.int32) if flag is None else np.ascontiguousarray(flag, np.int32)
    L = lib()
    off = np.zeros(n + 1, np.int32) if want_sets else None
    rho_out = np.zeros(n) if want_rho or want_force else None
    force = np.zeros((n, 2)) if want_force else None
    idx = None
    if want_sets:
        st = L.oracle_pairs(mode, C.addressof(params), n, _dp(x), _dp(hsml), _dp(mass), _dp(rho), _ip(flag), 0,
                            _ip(off), None, None, None)
        cap = int(off[-1])
        idx = np.zeros(max(cap, 1), np.int32)
    else:
        cap = 0
    st = L.oracle_pairs(mode, C.addressof(params), n, _dp(x), _dp(hsml), _dp(mass), _dp(rho), _ip(flag), cap,
                        _ip(off), _ip(idx), _dp(rho_out), _dp(force))
    if st:
        raise RuntimeError(f"oracle_pairs: {st}")
    return dict(offsets=off, idx=None if idx is None else idx[:cap], rho=rho_out, force=force)


def kernel(skf, r, dx, dy, hs, mode=MODE_FP32):
    r, dx, dy, hs = (_d(np.atleast_1d(a)) for a in (r, dx, dy, hs))
    m = r.size
    w, d0, d1 = np.zeros(m), np.zeros(m), np.zeros(m)
    lib().oracle_kernel(mode, skf, m, _dp(r), _dp(dx), _dp(dy), _dp(hs), _dp(w), _dp(d0), _dp(d1))
    return w, d0, d1


def raster_idw(nx, ny, dx, dy, x, rho, flag, xmin=0.0, ymin=0.0):
    out = np.zeros(nx * ny)
    lib().oracle_raster_idw(nx, ny, xmin, ymin, dx, dy, x.shape[0], _dp(_d(x)), _dp(_d(rho)),
                            _ip(np.ascontiguousarray(flag, np.int32)), _dp(out))
    return out.reshape(ny, nx)


class Hazard:
    def __init__(self, nx, ny, dx, dy, xmin=0.0, ymin=0.0):
        self.geom = (nx, ny, xmin, ymin, dx, dy)
        self.acc = np.zeros((nx * ny, 4))
        self.cnt = np.zeros(nx * ny, np.int32)

    def sample(self, x, v, rho, flag):
        nx, ny, xmin, ymin, dx, dy = self.geom
        lib().oracle_hazard_sample(nx, ny, xmin, ymin, dx, dy, x.shape[0], _dp(_d(x)), _dp(_d(v)), _dp(_d(rho)),
                                   _ip(np.ascontiguousarray(flag, np.int32)), _dp(self.acc), _ip(self.cnt))


class Run:
    """A persistent oracle run: the state stays inside the oracle between
    advance() calls, so timing advance() measures only the steps."""

    def __init__(self, mode, params, nx, ny, dx, dy, state, xmin=0.0, ymin=0.0, omp=False):
        """omp=True runs the OpenMP library (timing only)."""
        self.params = params
        self.n = state.x.shape[0]
        self.topol_shape = state.topol.shape
        self.L = lib(omp)
        self.threads = self.L.oracle_set_threads(omp_threads() if omp else 0)
        stv = C.c_int(0)
        self.h = None
        self.h = self.L.oracle_new(mode, C.addressof(params), nx, ny, xmin, ymin, dx, dy, _dp(state.topol), self.n,
                                  _dp(state.x), _dp(state.v), _dp(state.rho), _dp(state.mass), _dp(state.hsml),
                                  _ip(state.flag), _dp(state.pwp), state.dt, state.t, C.byref(stv))
        if not self.h:
            raise RuntimeError(f"oracle_new: {stv.value}")

    def advance(self, nsteps, t_end=1e300):
        return self.L.oracle_advance(self.h, nsteps, t_end)

    def state(self, with_topol=False):
        n = self.n
        x, v = np.zeros((n, 2)), np.zeros((n, 2))
        rho, mass, hsml = np.zeros(n), np.zeros(n), np.zeros(n)
        flag = np.zeros(n, np.int32)
        dt, t = C.c_double(), C.c_double()
        topol = np.zeros(self.topol_shape) if with_topol else None
        self.L.oracle_get(self.h, _dp(x), _dp(v), _dp(rho), _dp(mass), _dp(hsml), _ip(flag), C.byref(dt), C.byref(t),
                         _dp(topol))
        pwp = None
        if self.params.icpwp in (1, 3):
            pwp = np.zeros(n)
            self.L.oracle_get_pwp(self.h, _dp(pwp))
        return State(x, v, rho, mass, hsml, topol if with_topol else np.zeros(1), flag, dt.value, t.value, pwp)

    def close(self):
        if self.h:
            self.L.oracle_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solvegc2(mode, intmat, gstif, rhs, iffix=None, fixed=None, tol=1e-10, ndofn=1):
    """solvegc2 on the element matrices gstif (nelem, nevab, nevab) with
    intmat (nelem, nnode) 1-based; returns (x, final residual, iffix, iters)."""
    intmat = np.ascontiguousarray(intmat, np.int32)
    nelem, nnode = intmat.shape
    npoin = int(intmat.max())
    n = npoin * ndofn
    g = np.ascontiguousarray(np.transpose(gstif, (0, 2, 1)), np.float64)  # element-major, column-major within
    fix = np.zeros(n, np.int32) if iffix is None else np.ascontiguousarray(iffix, np.int32).copy()
    fx = np.zeros(n) if fixed is None else _d(fixed).copy()
    r = _d(rhs).copy()
    x = np.zeros(n)
    it = C.c_int(0)
    st = lib().oracle_solvegc2(mode, npoin, nelem, nnode, ndofn, _ip(intmat), _ip(fix), _dp(fx), _dp(g), _dp(r),
                               _dp(x), tol, C.byref(it))
    if st:
        raise RuntimeError(f"oracle_solvegc2: {st}")
    return x, r, fix, it.value


def gradhs(mode, ix0, iy0, nwx, nwy, dx, dy, x=None, rho=None, flag=None, hs=None, niter=5, xmin=0.0, ymin=0.0):
    """get_gradhs_w on the node window [ix0, ix0+nwx) x [iy0, iy0+nwy) of the
    DEM background triangulation: (hs_w (nwy, nwx), gradhs_w (nwy, nwx, 2)).
    Either particles (x, rho, flag) or node depths hs (nwy, nwx)."""
    n = 0 if x is None else np.asarray(x).shape[0]
    xd = _d(x) if n else None
    rd = _d(rho) if n else None
    fl = np.ascontiguousarray(flag, np.int32) if (n and flag is not None) else None
    hin = _d(hs).reshape(-1) if hs is not None else None
    hs_out = np.zeros(nwx * nwy)
    g_out = np.zeros(2 * nwx * nwy)
    st = lib().oracle_gradhs(mode, ix0, iy0, nwx, nwy, xmin, ymin, dx, dy, n, _dp(xd), _dp(rd), _ip(fl), _dp(hin),
                             niter, _dp(hs_out), _dp(g_out))
    if st:
        raise RuntimeError(f"oracle_gradhs: {st}")
    return hs_out.reshape(nwy, nwx), g_out.reshape(nwy, nwx, 2)


def tangent(params, nx, ny, dx, dy, state, nsteps, seed_mu=0.0, seed_xi=0.0, seed_m=None, seed_x=None,
            seed_v=None, xmin=0.0, ymin=0.0, seed_ty=0.0, single=False):
    """Forward-mode derivative of nsteps steps from `state` along one
    direction (tangents of const(9), const(3), const(6), volumes, positions,
    velocities): returns (x, v, h, dx, dv, dh) at the end.  The FP64 step, or
    with single=True the single-precision step of MODE_FP32 (its values
    rounded as it rounds them, the derivatives in FP64): the exact
    derivative of the trajectory the device computes."""
    n = state.x.shape[0]
    out = [np.zeros((n, 2)), np.zeros((n, 2)), np.zeros(n), np.zeros((n, 2)), np.zeros((n, 2)), np.zeros(n)]
    sm = _d(seed_m) if seed_m is not None else None
    sx = _d(seed_x) if seed_x is not None else None
    sv = _d(seed_v) if seed_v is not None else None
    fn = lib().oracle_tangent32 if single else lib().oracle_tangent
    st = fn(C.addressof(params), nx, ny, xmin, ymin, dx, dy, _dp(state.topol), n, _dp(state.x),
                              _dp(state.v), _dp(state.rho), _dp(state.mass), _dp(state.hsml), _ip(state.flag),
                              nsteps, state.dt, state.t, seed_mu, seed_xi, seed_ty, _dp(sm), _dp(sx), _dp(sv),
                              *[_dp(a) for a in out])
    if st:
        raise RuntimeError(f"oracle_tangent: {st}")
    return tuple(out)


# ---------------------------------------------------------------- set-up
# Restatements of the reference's input set-up in single precision (irk =
# k_real), used to check the C++ host reader: every operation is an FP32
# numpy operation in the reference's order, and the inverse-distance sums
# are added with np.add.at in the reference's loop order (source point, then
# the node columns, then the node rows), so the sums round as the Fortran
# loops do.  Decimal input is converted straight to single precision
# (strtof), as a list-directed read of a default real does.

_strtof = None


def _f32(tokens):
    global _strtof
    if _strtof is None:
        libc = C.CDLL(None)
        _strtof = libc.strtof
        _strtof.restype = C.c_float
        _strtof.argtypes = [C.c_char_p, C.c_void_p]
    return np.array([_strtof(t.replace("d", "e").replace("D", "e").encode(), None) for t in tokens], np.float32)


def _lines(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f]


def _idw_block(px, py, x0, y0, dx, dy, nx, ny, lo, hi):
    """Node indices (row-major, 0-based) and validity of the block of nodes
    [ipx + lo, ipx + hi] x [ipy + lo', ...] around each point, flattened in
    the reference's loop order: point, node column, node row."""
    f1 = np.float32(1.0)
    ipx = ((px - x0) / dx + f1).astype(np.int64)  # Fortran real -> integer truncates
    ipy = ((py - y0) / dy + f1).astype(np.int64)
    return ipx, ipy


def get_dtm(top_path):
    """Get_DTM (SPH_FEM_topo_2019.f90:1155-1445) for ictop 10 and 11: the
    scattered (x, y, z) points of the .top file to the regular grid by
    inverse-distance weights over the 4x4 nodes around each point.  Returns
    dict(nx, ny, xmin, ymin, dx, dy, xshift, yshift, z (ny, nx) float32)."""
    L = _lines(top_path)
    ictop = int(L[1].split()[0])
    if ictop not in (10, 11):
        raise ValueError("get_dtm restates ictop 10 and 11")
    np_dtm, deltx = L[3].split()[:2]
    np_dtm = int(float(np_dtm))
    deltx = _f32([deltx])[0]
    tok = " ".join(L[5:5 + np_dtm]).split()
    pts = _f32(tok[:3 * np_dtm]).reshape(np_dtm, 3)
    xx, yy, zz = pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy()
    xming, xmaxg, yming, ymaxg = xx.min(), xx.max(), yy.min(), yy.max()
    zmaxg = zz.max()
    f1 = np.float32(1.0)
    npoigx = int((xmaxg - xming) / deltx + f1)
    npoigy = int((ymaxg - yming) / deltx + f1)
    deltxg = (xmaxg - xming) / np.float32(npoigx - 1)
    deltyg = (ymaxg - yming) / np.float32(npoigy - 1)
    xshift = yshift = np.float32(0.0)
    if ictop == 11:  # relative coordinates
        xshift, yshift = xming, yming
        xx = xx - xming
        yy = yy - yming
        xmaxg, ymaxg = xmaxg - xming, ymaxg - yming
        xming = yming = np.float32(0.0)
    cx = xming + np.arange(npoigx).astype(np.float32) * deltxg
    cy = yming + np.arange(npoigy).astype(np.float32) * deltyg
    distg = np.sqrt(deltxg * deltxg + deltyg * deltyg)
    inside = (xx >= xming) & (xx <= xmaxg) & (yy >= yming) & (yy <= ymaxg)
    ipx = ((xx - xming) / deltxg + f1).astype(np.int64)
    ipy = ((yy - yming) / deltyg + f1).astype(np.int64)
    a = np.arange(4)
    inx = (ipx[:, None, None] - 1 + a[None, :, None]) * np.ones((1, 1, 4), np.int64)   # columns ipx-1 .. ipx+2
    iny = (ipy[:, None, None] - 1 + a[None, None, :]) * np.ones((1, 4, 1), np.int64)   # rows ipy-1 .. ipy+2
    ok = inside[:, None, None] & (inx >= 1) & (inx <= npoigx) & (iny >= 1) & (iny <= npoigy)
    inx, iny, ok = inx.reshape(-1), iny.reshape(-1), ok.reshape(-1)
    src = np.repeat(np.arange(np_dtm), 16)[ok]
    inx, iny = inx[ok], iny[ok]
    dxs = xx[src] - cx[inx - 1]
    dys = yy[src] - cy[iny - 1]
    dist = np.maximum(np.float32(1.e-6), np.sqrt(dxs * dxs + dys * dys))
    dist = dist / distg
    node = (iny - 1) * npoigx + (inx - 1)
    a1 = np.zeros(npoigx * npoigy, np.float32)
    a2 = np.zeros(npoigx * npoigy, np.float32)
    np.add.at(a1, node, zz[src] / dist)
    np.add.at(a2, node, f1 / dist)
    z = np.where(a2 >= np.float32(1.e-6), a1 / np.where(a2 > 0, a2, f1), zmaxg).astype(np.float32)
    return dict(nx=npoigx, ny=npoigy, xmin=xming, ymin=yming, dx=deltxg, dy=deltyg, xshift=xshift, yshift=yshift,
                z=z.reshape(npoigy, npoigx))


def read_source_plus_new(pts_path, h_inf, xshift=0.0, yshift=0.0):
    """Read_Source_plus_New (SPH_SW_2019.f90:4999-5272): the source points of
    the .pts file resampled on a lattice by inverse-distance weights; every
    lattice node that received a weight becomes a particle with depth
    sum(h/d)/sum(1/d) (clamped to h_inf), volume dA * h * (number of its four
    lattice cells whose corners all received weights), dA = dx dy / 4, and
    smoothing length max(delt2Dx, delt2Dy) * facthsml as read.  Returns
    dict(x (n, 2), h, mass, hsml) in float32, lattice order."""
    L = _lines(pts_path)
    hdr = L[1].split()
    np_src = int(float(hdr[0]))
    dx_s, d2x, d2y, fact = _f32(hdr[1:5])
    delt2d = max(d2x, d2y)
    tok = " ".join(L[3:3 + np_src]).split()
    pts = _f32(tok[:3 * np_src]).reshape(np_src, 3)
    xs = pts[:, 0] - np.float32(xshift)
    ys = pts[:, 1] - np.float32(yshift)
    hs = pts[:, 2]
    f1 = np.float32(1.0)
    xmin, xmax, ymin, ymax = xs.min(), xs.max(), ys.min(), ys.max()
    npx = int((xmax - xmin) / d2x + f1)
    npy = int((ymax - ymin) / d2y + f1)
    d2x = (xmax - xmin) / np.float32(npx - 1)
    d2y = (ymax - ymin) / np.float32(npy - 1)
    gx = xmin + np.arange(npx).astype(np.float32) * d2x
    gy = ymin + np.arange(npy).astype(np.float32) * d2y
    dist2d = np.sqrt(d2x * d2x + d2y * d2y)
    ndx = int(max(np.float32(2.0), dx_s / d2x))
    ndy = int(max(np.float32(2.0), dx_s / d2y))
    ipx = ((xs - xmin) / d2x + f1).astype(np.int64)
    ipy = ((ys - ymin) / d2y + f1).astype(np.int64)
    ax = np.arange(-ndx + 1, ndx + 2)   # columns ipx - ndx + 1 .. ipx + ndx + 1
    ay = np.arange(-ndy, ndy + 1)       # rows ipy - ndy .. ipy + ndy
    inx = ipx[:, None, None] + ax[None, :, None] + 0 * ay[None, None, :]
    iny = ipy[:, None, None] + 0 * ax[None, :, None] + ay[None, None, :]
    ok = (inx >= 1) & (inx <= npx) & (iny >= 1) & (iny <= npy)
    inx, iny, ok = inx.reshape(-1), iny.reshape(-1), ok.reshape(-1)
    src = np.repeat(np.arange(np_src), ax.size * ay.size)[ok]
    inx, iny = inx[ok], iny[ok]
    dxs = xs[src] - gx[inx - 1]
    dys = ys[src] - gy[iny - 1]
    dist = np.maximum(np.float32(1.e-6), np.sqrt(dxs * dxs + dys * dys))
    dist = dist / dist2d
    node = (iny - 1) * npx + (inx - 1)
    a2 = np.zeros(npx * npy, np.float32)
    a3 = np.zeros(npx * npy, np.float32)
    np.add.at(a2, node, f1 / dist)
    np.add.at(a3, node, hs[src] / dist)
    w = (a2 >= np.float32(1.e-6)).reshape(npy, npx)
    full = w[:-1, :-1] & w[:-1, 1:] & w[1:, :-1] & w[1:, 1:]
    a4 = np.zeros((npy, npx), np.int64)
    a4[:-1, :-1] += full
    a4[:-1, 1:] += full
    a4[1:, :-1] += full
    a4[1:, 1:] += full
    keep = w.reshape(-1)
    h = (a3[keep] / a2[keep]).astype(np.float32)
    h = np.where(h < np.float32(h_inf), np.float32(h_inf), h).astype(np.float32)
    d_area = d2x * d2y / np.float32(4.0)
    mass = (d_area * h * a4.reshape(-1)[keep].astype(np.float32)).astype(np.float32)
    yy, xx = np.meshgrid(gy, gx, indexing="ij")
    x = np.stack([xx.reshape(-1)[keep], yy.reshape(-1)[keep]], 1).astype(np.float32)
    return dict(x=x, h=h, mass=mass, hsml=np.full(h.size, delt2d * fact, np.float32))


def gfl_run(coord, intmat, z, const, unkno, nsteps, dt, ntype=3, ngaus=3, niter=3, swl=0.0, comp=0.01, hs_w=None,
            gradhs_w=None, time=0.0):
    """The GFL Taylor-Galerkin step (gfl_oracle.cpp) nsteps times on the P1
    mesh coord (npoin, 2), intmat (nelem, 3) 1-based, nodal Z; const {k:
    constF(k)}; unkno (npoin, 3) of h, hu, hv.  Returns (unkno, time, topol
    (npoin, 9), topel (nelem, 9)) in float64 holding single-precision values."""
    coord = _d(coord)
    intmat = np.ascontiguousarray(intmat, np.int32)
    npoin, nelem = coord.shape[0], intmat.shape[0]
    c15 = np.zeros(15)
    for k, v in const.items():
        if 1 <= k <= 14:
            c15[k] = v
    u = _d(unkno).copy()
    t = C.c_double(time)
    topol = np.zeros((npoin, 9))
    topel = np.zeros((nelem, 9))
    hs = _d(hs_w) if hs_w is not None else None
    gh = _d(gradhs_w) if gradhs_w is not None else None
    st = lib().oracle_gfl_run(npoin, nelem, _dp(coord), _ip(intmat), _dp(_d(z)), _dp(c15), ntype, ngaus, niter, swl,
                              comp, _dp(hs), _dp(gh), _dp(u), nsteps, dt, C.byref(t), _dp(topol), _dp(topel))
    if st:
        raise RuntimeError(f"oracle_gfl_run: {st}")
    return u, t.value, topol, topel
