"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: every input (DEM, release area, depth field)
is generated here from a seed.  Particles are placed the way
Read_Source_plus_New does it (SPH_SW_2019.f90:4999-5272): one particle per
lattice node of spacing delt2D, volume mass = dA * h * fct_area with
dA = dx*dy/4 and fct_area the number of the node's four lattice cells whose
corners all carry material, smoothing length hsml = delt2D * facthsml, depth
clamped to h_inf.
"""
import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    const: dict                  # {k: const(k)} of the reference, 1-based
    options: dict                # pa_sph, nnps, sle, skf, ... for gfsph.make_params
    z: np.ndarray                # (ny, nx) float32 elevations
    dx: float
    dy: float
    x: np.ndarray                # (n, 2) float32
    v: np.ndarray                # (n, 2) float32
    rho: np.ndarray              # (n,) float32 depth
    mass: np.ndarray             # (n,) float32 volume
    hsml: np.ndarray             # (n,) float32
    steps: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.x.shape[0]


def lattice_particles(mask, depth, x0, y0, spacing, facthsml, h_inf):
    """Particles on the nodes of a lattice (mask True) as Read_Source_plus_New builds them."""
    ny, nx = mask.shape
    full = mask[:-1, :-1] & mask[1:, :-1] & mask[:-1, 1:] & mask[1:, 1:]
    fct = np.zeros(mask.shape, np.int32)
    fct[:-1, :-1] += full
    fct[1:, :-1] += full
    fct[:-1, 1:] += full
    fct[1:, 1:] += full
    keep = mask & (fct > 0)            # nodes with no complete cell would get zero volume
    iy, ix = np.nonzero(keep)
    xs = (np.float32(x0) + ix.astype(np.float32) * np.float32(spacing)).astype(np.float32)
    ys = (np.float32(y0) + iy.astype(np.float32) * np.float32(spacing)).astype(np.float32)
    h = depth[iy, ix].astype(np.float32)
    h = np.maximum(h, np.float32(h_inf)).astype(np.float32)
    d_area = np.float32(spacing) * np.float32(spacing) / np.float32(4.0)
    mass = (d_area * h * fct[iy, ix].astype(np.float32)).astype(np.float32)
    n = xs.size
    hsml = np.full(n, np.float32(spacing) * np.float32(facthsml), np.float32)
    x = np.stack([xs, ys], axis=1).astype(np.float32)
    return x, np.zeros((n, 2), np.float32), h, mass, hsml


def diamond_square(k, hurst, rng):
    """Fractional-Brownian surface on a (2^k+1)^2 grid by midpoint displacement."""
    n = 2 ** k + 1
    a = np.zeros((n, n), np.float64)
    a[0, 0], a[0, -1], a[-1, 0], a[-1, -1] = rng.standard_normal(4)
    step = n - 1
    scale = 1.0
    while step > 1:
        half = step // 2
        # diamond step: square centres
        c = (a[0:-1:step, 0:-1:step] + a[step::step, 0:-1:step] + a[0:-1:step, step::step] + a[step::step, step::step]) / 4.0
        a[half::step, half::step] = c + scale * rng.standard_normal(c.shape)
        # square step: edge midpoints, averaging the available neighbours
        p = np.pad(a, half, mode="constant", constant_values=np.nan)
        for (r0, c0) in ((0, half), (half, 0)):
            rows = np.arange(r0, n, step)
            cols = np.arange(c0, n, step)
            R, Cc = np.meshgrid(rows + half, cols + half, indexing="ij")
            nb = np.stack([p[R - half, Cc], p[R + half, Cc], p[R, Cc - half], p[R, Cc + half]])
            m = np.nanmean(nb, axis=0)
            a[np.ix_(rows, cols)] = m + scale * rng.standard_normal(m.shape)
        scale *= 2.0 ** (-hurst)
        step = half
    return a


def smooth_field(x, y, rng, nmodes=6, lmin=30.0, lmax=100.0):
    """Sum of seeded plane waves, normalised to zero mean and unit max."""
    f = np.zeros_like(x, dtype=np.float64)
    for _ in range(nmodes):
        lam = rng.uniform(lmin, lmax)
        th = rng.uniform(0, 2 * math.pi)
        ph = rng.uniform(0, 2 * math.pi)
        f += np.cos(2 * math.pi * (x * math.cos(th) + y * math.sin(th)) / lam + ph)
    f -= f.mean()
    m = np.abs(f).max()
    return f / m if m > 0 else f


def voellmy_const(mu, xi, dens=2000.0, g=9.8, erosion=None):
    """const(k) map of a frictional (nfric 5) + Voellmy run; erosion = (C22, C48) for Hungr."""
    c = {1: g, 2: dens, 3: xi, 5: 5, 9: mu, 10: 0.01, 15: 0.01}
    if erosion:
        c.update({21: 1, 22: erosion[0], 48: erosion[1]})
    return c


def inclined_plane(seed=1, spacing=2.0, facthsml=2.0, nx=200, ny=400, cell=5.0):
    """Granular collapse on an analytic DEM: 30 deg plane over the first 250
    rows then flat; paraboloid cap (10 m, radius 50 m) centred 200 m upslope
    of the toe on a 2 m lattice with seeded +-1% depth jitter; Voellmy
    mu = 0.2, xi = 500, density 2000, fixed dt = 0.01 s, 2000 steps."""
    rows = np.arange(ny, dtype=np.float64)[:, None] * np.ones((1, nx))
    z = np.where(rows < 250, (250 - rows) * cell * math.tan(math.radians(30.0)), 0.0).astype(np.float32)
    xc, yc, r0 = nx * cell / 2.0, 250 * cell - 200.0, 50.0
    m = int(math.ceil(r0 / spacing)) + 1
    gx0, gy0 = xc - m * spacing, yc - m * spacing
    ii = np.arange(2 * m + 1)
    X, Y = np.meshgrid(gx0 + ii * spacing, gy0 + ii * spacing)
    r2 = (X - xc) ** 2 + (Y - yc) ** 2
    mask = r2 < r0 * r0
    rng = np.random.default_rng(seed)
    depth = 10.0 * (1.0 - r2 / (r0 * r0)) * (1.0 + rng.uniform(-0.01, 0.01, size=X.shape))
    x, v, h, mass, hsml = lattice_particles(mask, depth, gx0, gy0, spacing, facthsml, 0.01)
    return Workload(
        name="inclined_plane_2k", const=voellmy_const(0.2, 500.0),
        options=dict(pa_sph=2, nnps=2, sle=1, skf=1, average_velocity=1, ic_adapt=0, h_inf=0.01, dt=0.01,
                     dem_deriv=1),
        z=z, dx=cell, dy=cell, x=x, v=v, rho=h, mass=mass, hsml=hsml, steps=2000,
        meta=dict(dem=f"{nx}x{ny} at {cell} m", lattice=spacing))


def fractal_channel(n_target=200_000, dem_k=10, cell=5.0, seed=2, facthsml=2.0, mean_depth=4.0,
                    semi_along=150.0, semi_across=80.0, erosion=(0.005, 2.0), mu=0.15, xi=400.0,
                    relief=800.0, z=None):
    """Seeded diamond-square fBm DEM (Hurst 0.8) of 2^dem_k nodes a side at
    `cell` m with a carved V-channel, relief `relief` m; an elliptical release
    (semi-axes 150 m along the channel, 80 m across) on the lattice spacing
    that gives ~n_target particles; smooth seeded depth field of mean 4 m;
    Voellmy mu = 0.15, xi = 400 with Hungr erosion 0.005 1/m over a 2 m
    erodible layer; adaptive dt (ic_adapt_dt_sph = 1).  `z` reuses a DEM
    made by an earlier call with the same dem_k, cell, seed and relief."""
    nx = ny = 2 ** dem_k
    L = nx * cell
    xc = L / 2.0
    if z is None:
        rng = np.random.default_rng(seed)
        f = diamond_square(dem_k, 0.8, rng)[: 2 ** dem_k, : 2 ** dem_k]
        f = (f - f.min()) / (f.max() - f.min())
        ys = np.arange(ny)[:, None] * cell
        xs = np.arange(nx)[None, :] * cell
        decay = 0.3125 * L
        base = (relief - 100.0) * np.exp(-ys / decay)
        rough = 100.0 * f * np.exp(-ys / (2 * decay))
        half_w = 0.04 * L
        carve = 40.0 * np.clip(1.0 - np.abs(xs - xc) / half_w, 0.0, None)
        z = (base + rough - carve).astype(np.float32)
    yc = 0.137 * L
    area = math.pi * semi_along * semi_across
    spacing = math.sqrt(area / n_target)
    mx = int(math.ceil(semi_across / spacing)) + 1
    my = int(math.ceil(semi_along / spacing)) + 1
    gx0, gy0 = xc - mx * spacing, yc - my * spacing
    X, Y = np.meshgrid(gx0 + np.arange(2 * mx + 1) * spacing, gy0 + np.arange(2 * my + 1) * spacing)
    mask = ((X - xc) / semi_across) ** 2 + ((Y - yc) / semi_along) ** 2 < 1.0
    fld = smooth_field(X, Y, np.random.default_rng(seed + 1000))
    depth = mean_depth * (1.0 + 0.25 * fld)
    depth *= mean_depth / depth[mask].mean()
    x, v, h, mass, hsml = lattice_particles(mask, depth, gx0, gy0, spacing, facthsml, 0.01)
    return Workload(
        name=f"fractal_channel_{x.shape[0] // 1000}k",
        const=voellmy_const(mu, xi, erosion=erosion),
        options=dict(pa_sph=2, nnps=2, sle=1, skf=1, average_velocity=1, ic_adapt=1, h_inf=0.01, dt=0.01,
                     dem_deriv=1),
        z=z, dx=cell, dy=cell, x=x, v=v, rho=h, mass=mass, hsml=hsml, steps=10_000,
        meta=dict(dem=f"{nx}x{ny} at {cell} m", lattice=spacing, relief=relief))


def multi_release(n_target=4_000_000, dem_k=12, cell=2.0, seed=3, nrel=4, facthsml=2.0, mean_depth=3.0,
                  tauy0=1000.0, constK=50.0, relief=1200.0):
    """Large-scale case: a seeded fBm DEM (Hurst 0.8) of 2^dem_k nodes a side
    at `cell` m (4096^2 at 2 m: 8.2 km) sloping down along y, with nrel
    elliptical releases (semi-axes 250 x 120 m) spread across the upper slope
    on the one lattice spacing that gives ~n_target particles in all;
    Bingham basal law (nfric 4, yield stress const(6) = tauy0, viscosity
    const(7) = constK), no erosion, adaptive dt."""
    nx = ny = 2 ** dem_k
    L = nx * cell
    rng = np.random.default_rng(seed)
    f = diamond_square(dem_k, 0.8, rng)[:ny, :nx]
    f = (f - f.min()) / (f.max() - f.min())
    ys = np.arange(ny)[:, None] * cell
    z = ((relief - 150.0) * (1.0 - ys / L) + 150.0 * f).astype(np.float32)
    sa, sc = 250.0, 120.0
    spacing = math.sqrt(nrel * math.pi * sa * sc / n_target)
    xs, ms, vs, hs, hl = [], [], [], [], []
    for r in range(nrel):
        xc, yc = L * (r + 0.5) / nrel, 0.2 * L
        mx = int(math.ceil(sc / spacing)) + 1
        my = int(math.ceil(sa / spacing)) + 1
        gx0, gy0 = xc - mx * spacing, yc - my * spacing
        X, Y = np.meshgrid(gx0 + np.arange(2 * mx + 1) * spacing, gy0 + np.arange(2 * my + 1) * spacing)
        mask = ((X - xc) / sc) ** 2 + ((Y - yc) / sa) ** 2 < 1.0
        fld = smooth_field(X, Y, np.random.default_rng(seed + 100 + r))
        depth = mean_depth * (1.0 + 0.25 * fld)
        x, v, h, mass, hsml = lattice_particles(mask, depth, gx0, gy0, spacing, facthsml, 0.01)
        xs.append(x); vs.append(v); hs.append(h); ms.append(mass); hl.append(hsml)
    c = {1: 9.8, 2: 2000.0, 3: 0.0, 5: 4, 6: tauy0, 7: constK, 9: 0.0, 10: 0.01, 15: 0.01}
    return Workload(
        name=f"multi_release_{sum(a.shape[0] for a in xs) // 1000}k", const=c,
        options=dict(pa_sph=2, nnps=2, sle=1, skf=1, average_velocity=1, ic_adapt=1, h_inf=0.01, dt=0.01,
                     dem_deriv=1),
        z=z, dx=cell, dy=cell, x=np.concatenate(xs), v=np.concatenate(vs), rho=np.concatenate(hs),
        mass=np.concatenate(ms), hsml=np.concatenate(hl), steps=2000,
        meta=dict(dem=f"{nx}x{ny} at {cell} m", lattice=spacing, releases=nrel))


def mc_ensemble(nreal, n_base=200_000, dem_k=10, cell=5.0, seed=2024, mu=(0.08, 0.30), xi=(400.0, 0.3),
                scale=(0.2, 2.0)):
    """Realizations of the Monte-Carlo hazard ensemble on the fractal channel
    DEM: mu ~ U(mu), xi ~ LogNormal(ln xi[0], xi[1]), release volume scaled by
    s ~ U(scale) — the release keeps its ellipse, its depth field is scaled by
    s and its lattice is refined so that the particle count is ~n_base * s
    (ragged counts).  Returns a list of Workloads sharing one DEM array."""
    rng = np.random.default_rng(seed)
    z = None
    out = []
    for _ in range(nreal):
        m = float(rng.uniform(*mu))
        x = float(np.exp(rng.normal(math.log(xi[0]), xi[1])))
        s = float(rng.uniform(*scale))
        w = fractal_channel(n_target=max(int(n_base * s), 100), dem_k=dem_k, cell=cell, mu=m, xi=x,
                            mean_depth=4.0 * s, z=z)
        z = w.z
        w.meta.update(mu=m, xi=x, volume_scale=s)
        out.append(w)
    return out


def soil_and_pond(spacing=1.5, scale=1.0):
    """Soil and water particles (ic_ws_Interact = 1): a gentle 2% slope
    (DEM at 2 m, Z = 0.02 (ymax - y)), a Bingham soil cap (radius 30 m, 6 m
    high) centred at (120, 80) m, and a 1.5 m-deep water pond over x 90..150,
    y 100..140 m, its first 10 m over the cap's edge; both on a lattice of
    `spacing`.  `scale` stretches the scene (and the DEM) in both directions.
    Returns the workload of the soil (its const and DEM) and the joint
    particle arrays with the material per particle (1 soil, 2 water)."""
    cell = 2.0
    n = int(round(120 * scale))
    yy = np.arange(n, dtype=np.float64)[:, None] * cell * np.ones((1, n))
    z = (0.02 * ((n - 1) * cell - yy)).astype(np.float32)
    g = np.arange(0.0, (n - 1) * cell, spacing)
    X, Y = np.meshgrid(g, g)
    cx, cy, r0 = 120.0 * scale, 80.0 * scale, 30.0 * scale
    r2 = (X - cx) ** 2 + (Y - cy) ** 2
    depth = 6.0 * (1.0 - r2 / r0 ** 2)
    xs, vs, hs_, ms, hsm = lattice_particles(r2 < r0 ** 2, depth, 0.0, 0.0, spacing, 2.0, 0.01)
    pond = (X >= 90.0 * scale) & (X <= 150.0 * scale) & (Y >= 100.0 * scale) & (Y <= 140.0 * scale)
    xw, vw, hw, mw, hsw = lattice_particles(pond, np.full(X.shape, 1.5), 0.0, 0.0, spacing, 2.0, 0.01)
    const = {1: 9.8, 2: 2000.0, 3: 0.03, 5: 4, 6: 1000.0, 7: 50.0, 10: 0.01, 15: 0.01, 18: 1000.0}
    w = Workload(name="soil_and_pond", const=const,
                 options=dict(pa_sph=2, nnps=2, sle=1, skf=1, average_velocity=1, ic_adapt=0, h_inf=0.01, dt=0.01,
                              dem_deriv=1, ws_interact=1, sw_alg=1),
                 z=z, dx=cell, dy=cell, x=xs, v=vs, rho=hs_, mass=ms, hsml=hsm, steps=1000,
                 meta=dict(dem=f"{n}x{n} at {cell} m", lattice=spacing))
    x = np.concatenate([xs, xw]).astype(np.float32)
    arrays = dict(x=x, v=np.zeros_like(x), rho=np.concatenate([hs_, hw]).astype(np.float32),
                  mass=np.concatenate([ms, mw]).astype(np.float32),
                  hsml=np.concatenate([hsm, hsw]).astype(np.float32),
                  itype=np.r_[np.ones(len(xs), np.int32), np.full(len(xw), 2, np.int32)])
    return w, arrays


def make_params(w, gfsph_module, **over):
    opts = dict(w.options)
    opts.update(over)
    return gfsph_module.make_params(w.const, **opts)


def p1_mesh(nx, ny, d):
    """The DEM background triangulation (SPH_FEM_topo_2019.f90:583-604): two
    triangles per grid cell, (n, n+1, n+1+nx) and (n, n+1+nx, n+nx), 1-based
    node numbers; returns intmat (nelem, 3), coords (npoin, 2)."""
    iy, ix = np.mgrid[0:ny - 1, 0:nx - 1]
    node = (iy * nx + ix).reshape(-1) + 1
    t1 = np.stack([node, node + 1, node + 1 + nx], 1)
    t2 = np.stack([node, node + 1 + nx, node + nx], 1)
    intmat = np.empty((2 * node.size, 3), np.int32)
    intmat[0::2] = t1
    intmat[1::2] = t2
    yy, xx = np.mgrid[0:ny, 0:nx]
    coords = np.stack([xx.reshape(-1) * d, yy.reshape(-1) * d], 1).astype(np.float64)
    return intmat, coords


def p1_mass_matrices(intmat, coords):
    """Consistent P1 mass matrices (2A/24)*[[2,1,1],[1,2,1],[1,1,2]] per
    triangle, the system of get_gradhs_w (SPH_GFL_SW_Interactions_2019.f90:483-540)."""
    p = coords[intmat - 1]
    a2 = np.abs((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    m = np.array([[2.0, 1.0, 1.0], [1.0, 2.0, 1.0], [1.0, 1.0, 2.0]])
    return (a2 / 24.0)[:, None, None] * m[None, :, :]


def write_reference_inputs(w, directory, name, out_step=100, restart=False, water=None):
    """Writes a workload in the reference's own input formats, so that the
    Fortran program (or gfsph_run) can read it: <name>.MASTER.dat,
    <name>.dat, <name>.top (ictop = 100: a grid file with finite-difference
    slopes) and <name>.pts (the particles as source points on their
    lattice).  w.options may carry icpwp (0, 1 or 3) and pwp0rel.  out_step is
    print_step = save_step = plot_step; restart=True writes icunk_s = 200,
    which reads the particles from restart.dat (Get_Restart_Info_SW).
    water: soil and water (ic_soil = ic_water = 1, ic_SWAlg = w.options'
    sw_alg): a dict with the water's x, rho and lattice, written as
    <name>_w.pts and read through Read_Source_plus_New_WATER (icunk_w 7)."""
    import os
    os.makedirs(directory, exist_ok=True)
    o = w.options
    c = [0.0] * 60
    for k, v in w.const.items():
        if k <= 60:
            c[k - 1] = float(v)
    blocks = 1
    if any(c[15:30]) or any(c[30:45]) or any(c[45:60]):
        c[10] = -1.0
        blocks = 2
    if any(c[30:45]) or any(c[45:60]):
        c[29] = -1.0
        blocks = 3
    if any(c[45:60]):
        c[44] = -1.0
        blocks = 4
    dt = float(o["dt"])
    with open(os.path.join(directory, name + ".MASTER.dat"), "w") as f:
        f.write("1\n" + name + " written by gfsph workloads\n")
        f.write("if_sph if_gfl ic_cases\n  1 0 0\n")
        f.write("SPH_problem_type SPH_t_integ_Alg\n  1 4\n")
        f.write("sph problem name\n" + name + "\n")
        f.write("dt time_end maxtimesteps\n  %g %g 1000000\n" % (dt, dt * w.steps))
        f.write("print_step save_step plot_step\n  %d %d %d\n" % (out_step, out_step, out_step))
        f.write("dt_sph ic_adapt\n  %g %d\n" % (dt, o["ic_adapt"]))
        f.write("Ntime curves max pts\n  0 6\nwin\n0\n")
    with open(os.path.join(directory, name + ".dat"), "w") as f:
        f.write("1\n " + name + "\n ic_SW_Alg\n  %d\nnhist\n  0\nndimn\n  2\n" % int(o.get("sw_alg", 0)))
        f.write("ic_soil ic_water ic_vps ic_abs\n  1 %d 0 0\n" % (1 if water is not None else 0))
        if restart:
            f.write("Soil unkno h_inf_SW\n  200 %g\n" % o["h_inf"])
            f.write("problem name (restart)\n  " + name + "\n")
        else:
            f.write("Soil unkno h_inf_SW\n  7 %g\n" % o["h_inf"])
            f.write("pts file name\n  " + name + "\n")
        if water is not None:
            f.write("Water unkno\n  7\n")
            f.write("water pts file name\n  " + name + "_w\n")
        f.write("pa_sph nnps sle skf\n  %d %d %d %d\n" % (o["pa_sph"], o["nnps"], o["sle"], o["skf"]))
        f.write("sum_den av_vel virt_part nor_dens\n  T %s F F\n" % ("T" if o["average_velocity"] else "F"))
        for b in range(blocks):
            f.write("constants %d-%d\n  " % (15 * b + 1, 15 * b + 15) + " ".join("%.9g" % v for v in c[15 * b:15 * b + 15]) + "\n")
        nfric = int(c[4] + 0.01)
        if 5 <= nfric <= 10 or nfric in (26, 27):  # if_frictional, SPH_SW_2019.f90:1252-1253, 1374
            f.write("K0 activated?\n  0\n")
        icpwp = int(o.get("icpwp", 0))
        f.write("icpwp\n  %d\n" % icpwp)
        if icpwp in (1, 3):
            f.write(" pwp0rel\n  %.9g\n" % float(o.get("pwp0rel", 0.0)))
        f.write("coarse mesh saving utility?\n  0\ncontrol points?\n  0\n")
        f.write("GID filter\n  1 1 1 1 0 1 0 0 0 1 0 0\nT_change_to_W\n  1.e+12\n")
    ny, nx = w.z.shape
    with open(os.path.join(directory, name + ".top"), "w") as f:
        f.write("ictop\n100\nnpoigx npoigy\n%d %d\nnode x y z\n" % (nx, ny))
        k = 1
        for iy in range(ny):
            for ix in range(nx):
                f.write("%d %.9g %.9g %.9g\n" % (k, float(np.float32(ix * w.dx)), float(np.float32(iy * w.dy)), float(w.z[iy, ix])))
                k += 1
    lattice = float(w.meta["lattice"])
    facthsml = float(w.hsml[0]) / lattice
    def write_pts(path, xs, hs, lat, fh):
        with open(path, "w") as f:
            f.write("npoin source  grid spacing  facthsml\n")
            f.write("%d %.9g %.9g %.9g %.9g\n" % (len(hs), lat, lat, lat, fh))
            f.write("X Y h\n")
            for (xx, yy), hh in zip(np.asarray(xs, np.float64), np.asarray(hs, np.float64)):
                f.write("%.9g %.9g %.9g\n" % (float(xx), float(yy), float(hh)))

    write_pts(os.path.join(directory, name + ".pts"), w.x, w.rho, lattice, facthsml)
    if water is not None:
        write_pts(os.path.join(directory, name + "_w.pts"), water["x"], water["rho"], float(water["lattice"]),
                  float(water.get("facthsml", facthsml)))


def from_driver_dump(path, gfsph_module):
    """A Workload and its params from `gfsph_run <problem> --dump FILE`: the
    run as the C++ driver parsed it from the reference's input files."""
    import ctypes as C
    with open(path, "rb") as f:
        b = f.read()
    if b[:8] != b"GFSPHDMP":
        raise ValueError(path + ": not a gfsph_run dump")
    ver, psz = np.frombuffer(b, np.int32, 2, 8)
    if ver not in (1, 2) or psz != C.sizeof(gfsph_module.Params):
        raise ValueError(path + ": dump version or params size mismatch")
    off = 16
    p = gfsph_module.Params.from_buffer_copy(b[off:off + psz])
    off += psz
    nx, ny = (int(v) for v in np.frombuffer(b, np.int32, 2, off))
    off += 8
    xmin, ymin, dx, dy = (float(v) for v in np.frombuffer(b, np.float32, 4, off))
    off += 16
    z = np.frombuffer(b, np.float32, nx * ny, off).reshape(ny, nx).copy()
    off += 4 * nx * ny
    n = int(np.frombuffer(b, np.int32, 1, off)[0])
    off += 4

    def take(count, shape):
        nonlocal off
        a = np.frombuffer(b, np.float32, count, off).reshape(shape).copy()
        off += 4 * count
        return a

    x = take(2 * n, (n, 2))
    v = take(2 * n, (n, 2))
    rho, mass, hsml = take(n, (n,)), take(n, (n,)), take(n, (n,))
    itype = np.frombuffer(b, np.int32, n, off).copy() if ver >= 2 else np.ones(n, np.int32)
    const = {k + 1: float(p.cst[k]) for k in range(len(p.cst)) if p.cst[k] != 0.0}
    w = Workload(name=os.path.basename(path), const=const, options={}, z=z, dx=dx, dy=dy, x=x, v=v, rho=rho,
                 mass=mass, hsml=hsml, meta=dict(xmin=xmin, ymin=ymin, itype=itype))
    return w, p
