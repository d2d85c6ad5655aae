"""Error of each output against FP64 at the configurations' full lengths.

Runs one case in one arm and saves its outputs, or compares saved outputs:

    python tests/golden/fp64_error_study.py oracle --case plane --mode 2 --out plane_fp64.npz
    python tests/golden/fp64_error_study.py oracle --case plane --mode 0 --out plane_fp32.npz
    python tests/golden/fp64_error_study.py gpu    --case plane --out plane_gpu.npz      (needs a GPU)
    python tests/golden/fp64_error_study.py report plane_fp64.npz plane_fp32.npz plane_gpu.npz

Cases (seeded synthetic inputs of the benchmark configurations):
  plane      the granular collapse on the 30-degree plane (~2k particles,
             200 x 400 DEM at 5 m, Voellmy mu 0.2 xi 500, fixed dt 0.01 s),
             2,000 steps, hazard samples every 50 steps;
  channel20k a 20k-particle release of the fractal-channel workload (1024^2
             DEM at 5 m, Voellmy mu 0.15 xi 400, Hungr erosion, adaptive dt),
             10,000 steps, hazard samples every 100 steps.
Arms: the serial oracle in the reference's FP32 scheme (mode 0, the shipped
build), in the GPU's scheme (mode 1: FP32 with FP64 sums), in FP64 (mode 2,
irk = k_double), or mode 1 with the RK45 position updates carried in FP64
(mode 3, a precision experiment), and the GPU through the C ABI.

Outputs, all evaluated in FP64 from each arm's particle states with the same
code (so only the states differ): the final IDW depth raster
(SPH_SW_2019.f90:14310-14400), the maximum-velocity raster over the hazard
samples (Get_MC_pixel_Vars_SW :20739-20812: each particle's |v| to the 4
nodes of its DEM cell), the runout (largest distance of a particle inside
the DEM from the release centroid) and the deposited volume (sum of the
volumes inside the DEM).  The report gives relative L2 errors of the rasters
and relative errors of the scalars against the FP64 arm.
"""
import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
for p in (os.path.join(ROOT, "deslizamientos-y-flujos_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import gfsph  # noqa: E402
import workloads  # noqa: E402

CASES = {
    "plane": dict(make=lambda: workloads.inclined_plane(), steps=2000, every=50),
    "channel20k": dict(make=lambda: workloads.fractal_channel(n_target=20_000), steps=10_000, every=100),
}


def idw_raster(w, x, h, flag):
    ny, nx = w.z.shape
    a1 = np.zeros(nx * ny)
    a5 = np.zeros(nx * ny)
    distg = np.hypot(w.dx, w.dy)
    keep = flag == 0
    x, h = x[keep], h[keep]
    ipx = (x[:, 0] / w.dx + 1.0).astype(np.int64)
    ipy = (x[:, 1] / w.dy + 1.0).astype(np.int64)
    for ox in range(-1, 3):
        for oy in range(-1, 3):
            ix, iy = ipx + ox, ipy + oy
            ok = (ix >= 1) & (ix <= nx) & (iy >= 1) & (iy <= ny)
            d = np.hypot(x[ok, 0] - (ix[ok] - 1) * w.dx, x[ok, 1] - (iy[ok] - 1) * w.dy)
            wgt = distg / np.maximum(d, 1e-6)
            ip = (iy[ok] - 1) * nx + (ix[ok] - 1)
            np.add.at(a1, ip, h[ok] * wgt)
            np.add.at(a5, ip, wgt)
    return np.where(a5 >= 1e-6, a1 / np.where(a5 > 0, a5, 1.0), a1)


def max_speed_sample(w, vmax, x, v, flag):
    ny, nx = w.z.shape
    keep = flag == 0
    x, v = x[keep], v[keep]
    ipx = np.clip((x[:, 0] / w.dx + 1.0).astype(np.int64), 1, nx - 1)
    ipy = np.clip((x[:, 1] / w.dy + 1.0).astype(np.int64), 1, ny - 1)
    ip = (ipy - 1) * nx + (ipx - 1)
    s = np.hypot(v[:, 0], v[:, 1])
    for node in (ip, ip + 1, ip + 1 + nx, ip + nx):
        np.maximum.at(vmax, node, s)


def outputs(w, x0, x, h, mass, flag, vmax):
    keep = flag == 0
    c = x0.astype(np.float64).mean(axis=0)
    return dict(depth=idw_raster(w, x, h, flag), vmax=vmax, runout=float(np.hypot(*(x[keep] - c).T).max()),
                volume=float(mass[keep].sum()), x=x, h=h, flag=flag)


def run_oracle(case, mode):
    import oracle
    cfg = CASES[case]
    w = cfg["make"]()
    p = workloads.make_params(w, gfsph)
    ny, nx = w.z.shape
    topol = oracle.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv,
                                 mode=oracle.MODE_FP64 if mode == 2 else oracle.MODE_FP32)
    st = oracle.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    run = oracle.Run(mode, p, nx, ny, w.dx, w.dy, st)
    vmax = np.zeros(nx * ny)
    done = 0
    while done < cfg["steps"]:
        k = min(cfg["every"], cfg["steps"] - done)
        run.advance(k)
        done += k
        s = run.state()
        max_speed_sample(w, vmax, s.x, s.v, s.flag)
    s = run.state()
    run.close()
    return dict(outputs(w, w.x, s.x, s.rho, s.mass, s.flag, vmax), time=s.t)


def run_gpu(case):
    cfg = CASES[case]
    w = cfg["make"]()
    p = workloads.make_params(w, gfsph)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    ny, nx = w.z.shape
    vmax = np.zeros(nx * ny)
    done = 0
    while done < cfg["steps"]:
        k = min(cfg["every"], cfg["steps"] - done)
        sim.step(k)
        done += k
        g = sim.download()
        max_speed_sample(w, vmax, g["x"].astype(np.float64), g["v"].astype(np.float64), g["flag"])
    g = sim.download()
    t, _ = sim.time()
    sim.close()
    return dict(outputs(w, w.x, g["x"].astype(np.float64), g["rho"].astype(np.float64),
                        g["mass"].astype(np.float64), g["flag"], vmax), time=t)


def report(ref_path, others):
    ref = np.load(ref_path)

    def rl2(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    print("arm | depth raster | max-velocity raster | runout | deposited volume | final time")
    for path in others:
        o = np.load(path)
        print("%s | %.3e | %.3e | %.3e | %.3e | %.6f" % (
            os.path.basename(path), rl2(o["depth"], ref["depth"]), rl2(o["vmax"], ref["vmax"]),
            abs(float(o["runout"]) - float(ref["runout"])) / float(ref["runout"]),
            abs(float(o["volume"]) - float(ref["volume"])) / float(ref["volume"]), float(o["time"])))
    print("FP64 final time %.6f" % float(ref["time"]))


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("oracle")
    a.add_argument("--case", choices=sorted(CASES), required=True)
    a.add_argument("--mode", type=int, choices=[0, 1, 2, 3], required=True)
    a.add_argument("--out", required=True)
    b = sub.add_parser("gpu")
    b.add_argument("--case", choices=sorted(CASES), required=True)
    b.add_argument("--out", required=True)
    c = sub.add_parser("report")
    c.add_argument("ref")
    c.add_argument("others", nargs="+")
    args = ap.parse_args()
    if args.cmd == "oracle":
        np.savez(args.out, **run_oracle(args.case, args.mode))
    elif args.cmd == "gpu":
        np.savez(args.out, **run_gpu(args.case))
    else:
        report(args.ref, args.others)


if __name__ == "__main__":
    main()
