"""Throughput benchmark of the SPH step: particle-steps/s on B200.

Workload: the fractal-channel configuration — seeded diamond-square DEM
1024 x 1024 at 5 m (Hurst 0.8, relief 800 m, carved V-channel), elliptical
release of ~200k particles (semi-axes 150 x 80 m, mean depth 4 m), Voellmy
mu = 0.15, xi = 400, Hungr erosion 0.005 1/m over a 2 m layer, adaptive dt.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gfsph|reference]

One JSON line on rank 0.  `value` is measured with the state resident in HBM:
every timed step is preceded by a 256 MiB write that flushes L2, and only the
device time of the step (CUDA events inside gfsph_step) is summed.  `e2e`
goes through the C ABI from pinned host buffers every step: upload of the
state, one step, download of the state.  With N > 1 every rank runs its own
replica (a different seed) on its own GPU: there is no exchange in the path.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "deslizamientos-y-flujos_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

METRIC = "SPH particle-steps/s"
UNIT = "particle-steps/s"
# Algorithmic bytes per particle and launch: the compulsory traffic of each
# pass, 168 B per particle-step in all (bin 28, density 24, force + RK4 +
# h-update 72, av_vel 44).  The force pass runs as two kernels: k_iforce reads
# x, y, hsml, m, h and the neighbour count (24 B); k_force_rk reads v and the
# flag (12 B) and writes x, y, v, hsml, flag and the step-start copies (36 B).
# The internal acceleration handed between them (8 B written, 8 B read) is an
# artefact of the split and is not counted.
B_ALG = {"k_density": 24, "k_iforce": 24, "k_force_rk": 48, "k_xsph": 44, "k_hist": 28}
# From ncu on this workload (200,011 particles), per particle: DRAM read +
# write bytes per launch and warp instructions per launch of k_density, the
# mean of its launches at steps 6, 16 and 25 (first, middle and last of the
# steps `bench.py --steps 20 --warmup 5` times; one launch each, cold caches).
# The issue-bound figure is printed only when the run times those same steps,
# since the neighbour work per step grows as the flow spreads.
NCU_STEPS = (6, 25)
NCU_PER_PARTICLE = {"k_density": {"warp_inst": 68.12e6 / 200011, "dram_bytes": 104.36e6 / 200011}}
NCU_SOURCE = "profiles/neighbour_kernels_fractal_channel_200k.md (ncu, cold caches, steps 6/16/25), scaled by active particles"
ISSUE_PEAK = 148 * 4 * 1.965e9  # warp instructions/s: SMs x schedulers x max SM clock


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def combine_ranks(ms_local, n_local, steps, dist=None, device="cpu"):
    """Whole-job throughput of N replicas: the slowest rank's device time
    (max over ranks) and the particle-steps of all ranks.  Returns
    (ms_max, total particles, particle-steps/s)."""
    import torch
    t = torch.tensor([float(ms_local), float(n_local)], dtype=torch.float64, device=device)
    if dist is not None:
        ms = t[:1].clone()
        nn = t[1:].clone()
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        dist.all_reduce(nn, op=dist.ReduceOp.SUM)
        t = torch.cat([ms, nn])
    ms_max, n_total = float(t[0].item()), float(t[1].item())
    return ms_max, n_total, n_total * steps / (ms_max / 1000.0)


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _oracle_case(n_target, seed=2):
    """The benchmark workload (the same release the GPU arm runs) as an
    oracle state."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gfsph
    import oracle
    import workloads
    w = workloads.fractal_channel(n_target=n_target, seed=seed)
    p = workloads.make_params(w, gfsph)
    topol = oracle.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv)
    ny, nx = w.z.shape
    st = oracle.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
    return oracle, w, p, nx, ny, st


def _warm_state(oracle, w, p, nx, ny, st, warm_steps):
    """The reference FP32 state after the GPU arm's warm-up steps (serial
    oracle, mode 0), so that the CPU legs time the same steps of the flow."""
    run = oracle.Run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, st)
    run.advance(warm_steps)
    snap = run.state(with_topol=True)
    run.close()
    return snap


def cpu_reference_rate(n_target, warm_steps, seconds_budget):
    """The reference path on the host (the FP32 oracle port) on the benchmark
    workload itself: the same ~200k-particle release, from the state after the
    GPU arm's warm-up steps, over as many of the following steps as fit the
    time budget.  One host thread (the reference is single-threaded), then the
    OpenMP build of the port over the same steps on every host core this
    process may use.  Returns the cpu_baseline object."""
    oracle, w, p, nx, ny, st = _oracle_case(n_target)
    snap = _warm_state(oracle, w, p, nx, ny, st, warm_steps)
    run = oracle.Run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, snap)
    t0 = time.perf_counter()
    run.advance(1)
    one = max(time.perf_counter() - t0, 1e-4)
    run.close()
    steps = max(1, min(400, int(seconds_budget / one)))

    def timed(omp):
        r = oracle.Run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, snap, omp=omp)
        t0 = time.perf_counter()
        r.advance(steps)
        el = time.perf_counter() - t0
        threads = r.threads
        r.close()
        return w.n * steps / el, threads

    where = (f"steps {warm_steps + 1}..{warm_steps + steps} of the benchmark workload itself ({w.n} particles, "
             f"the GPU arm's release), FP32 oracle port")
    rate, _ = timed(False)
    cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "sample": where + ", 1 host thread"}
    if oracle.omp_available():
        try:
            rate, threads = timed(True)
            cpu["openmp"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": where + f", OpenMP build, {threads} host threads"}
        except (OSError, RuntimeError) as e:
            cpu["openmp"] = {"unavailable": f"{type(e).__name__}: {e}"}
    else:
        cpu["openmp"] = {"unavailable": "the OpenMP build of the oracle was not made (no -fopenmp compiler)"}
    return cpu


def bench_config(n, w):
    """The `config` object both arms print: the same workload and steps."""
    return {"workload": "fractal_channel: 1024^2 DEM at 5 m, ~200k-particle elliptical release, "
                        "Voellmy + Hungr erosion, adaptive dt",
            "n_particles": n, "dem": w.meta["dem"], "lattice_m": round(w.meta["lattice"], 4),
            "timed_steps": "the K steps after the W warm-up steps of the flow, in both arms",
            "l2": "GPU arm: flushed before every timed step (256 MiB write)",
            "parallelism": "one GPU, or one host thread in the reference arm"}


def run_reference_arm(args, rank, world):
    """The reference's CPU path (the FP32 oracle port: the Fortran reference
    cannot be built here) on the GPU arm's workload: the same ~200k-particle
    release, W untimed warm-up steps, then K timed steps, one oracle step per
    bench step, on one host thread (the reference is single-threaded)."""
    if rank != 0:
        return 0
    oracle, w, p, nx, ny, st = _oracle_case(args.n)
    run = oracle.Run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, st)
    run.advance(args.warmup)
    el = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run.advance(1)
        el += time.perf_counter() - t0
    run.close()
    value = w.n * args.steps / el
    desc = (f"steps {args.warmup + 1}..{args.warmup + args.steps} of the benchmark workload itself ({w.n} "
            f"particles), FP32 oracle port (mode 0, the reference's FP32 scheme), 1 host thread")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * el / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(w.n, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def ensemble_bench(args, torch, gfsph, workloads):
    """Monte-Carlo ensemble: R realizations (mu ~ U(0.08, 0.30), xi ~
    LogN(ln 400, 0.3), release volume x U(0.2, 2.0): ragged particle counts,
    workloads.mc_ensemble) advanced S steps each, in waves of `wave` members
    that fit HBM (one gfsph_ensemble per wave: members on their own streams,
    one device copy of the DEM rows), against looping gfsph_step over the
    same members one at a time.  Both start from the same state after 3 warm
    steps (graph capture, capacity growth); times are host clocks around
    device-synchronised phases.  Realizations/s extrapolates realization-
    steps/s to the 5,000-step realization length.  Members are compared bit
    for bit between the two runs."""
    R, S, W = args.ensemble, args.ensemble_steps, max(1, args.ensemble_wave)
    t_batch = t_loop = 0.0
    npart = []
    identical = True
    err = 0.0
    for w0 in range(0, R, W):  # each wave drawn from its own seed
        ws = workloads.mc_ensemble(min(W, R - w0), n_base=args.n, seed=2024 + w0)
        params = [workloads.make_params(w, gfsph) for w in ws]
        npart += [w.n for w in ws]
        z = ws[0].z

        def fresh():
            e = gfsph.Ensemble(params, z, dx=ws[0].dx, dy=ws[0].dy)
            for m, w in zip(e.members, ws):
                m.upload(w.x, w.v, w.rho, w.mass, w.hsml)
            e.step(3)
            return e

        ens = fresh()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for m in ens.members:
            m.step(S)
        torch.cuda.synchronize()
        t_loop += time.perf_counter() - t0
        looped = [ens.members[k].download() for k in (0, len(ws) - 1)]
        ens.close()
        ens = fresh()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens.step(S)
        torch.cuda.synchronize()
        t_batch += time.perf_counter() - t0
        for a, k in zip(looped, (0, len(ws) - 1)):
            b = ens.members[k].download()
            identical &= all(np.array_equal(a[q], b[q]) for q in a)
            d = np.linalg.norm((b["rho"] - a["rho"]).astype(np.float64)) / max(np.linalg.norm(a["rho"]), 1e-30)
            err = max(err, float(d))
        ens.close()
    ps = sum(npart) * S
    return {
        "metric": "MC realizations/s", "realizations": R, "wave": W, "steps_per_realization_timed": S,
        "particles_min": min(npart), "particles_max": max(npart), "particles_total": sum(npart),
        "batched": {"realizations_per_s": R * S / t_batch / 5000.0, "seconds": t_batch,
                    "particle_steps_per_s": ps / t_batch},
        "looped": {"realizations_per_s": R * S / t_loop / 5000.0, "seconds": t_loop,
                   "particle_steps_per_s": ps / t_loop},
        "speedup_vs_looped": t_loop / t_batch,
        "max_rel_l2_depth_vs_looped": err, "bit_identical_to_looped": bool(identical),
        "note": "realizations/s = realization-steps/s / 5000 (extrapolated from the timed steps); "
                "device-synchronised host clock; the first and last member of every wave bit-compared with "
                "the looped run",
    }


def cg_bench(args, gfsph, workloads, peak):
    """The CG of the coupled large case: the P1 mass system of a 500 x 500-node
    window of the DEM background triangulation at 2 m (498,002 triangles,
    250,000 dofs), M x = b to r.r/r0.r0 <= 1e-10 (solvegc2's test), FP64 on the
    device.  Bytes per iteration: CSR values and column indices, row pointers
    and 6 FP64 vectors.  Host clock around each (synchronous) solve, which
    includes copying b in and x out (2 MB)."""
    nw = 500
    intmat, coords = workloads.p1_mesh(nw, nw, 2.0)
    g = workloads.p1_mass_matrices(intmat, coords)
    b = np.random.default_rng(3).normal(size=coords.shape[0]).astype(np.float32)
    cg = gfsph.CG(intmat, g)
    cg.solve(b, tol=1e-10)
    times, dev, its = [], [], 0
    for _ in range(5):
        t0 = time.perf_counter()
        _, _, _, its = cg.solve(b, tol=1e-10)
        times.append(time.perf_counter() - t0)
        dev.append(cg.device_ms())
    # the set-up and result kernels alone: a solve from a zero right-hand side
    # stops before the first iteration
    zero = np.zeros_like(b)
    cg.solve(zero, tol=1e-10)
    setup_ms = cg.device_ms()
    cg.close()
    n = coords.shape[0]
    nnz = 7 * n  # a structured P1 mesh: every node couples to itself and 6 neighbours (fewer on the edge)
    # per iteration: CSR values and columns, row pointers, the iffix gathers,
    # and the FP64 vectors read and written by the two phases
    # (A: s, p_old, fix read; p, ap written.  B: x, p, r, ap, q read; x, r1, s written)
    bytes_it = nnz * 12 + (n + 1) * 4 + n * 4 + 2 * 8 * n + 2 * 8 * n + 5 * 8 * n + 3 * 8 * n
    t = statistics.median(times)
    t_dev = statistics.median(dev) / 1e3
    per_it = max(t_dev - setup_ms / 1e3, 1e-9) / max(its, 1)
    out = {"system": f"P1 mass matrix, {intmat.shape[0]} triangles, {n} dofs", "tol": 1e-10,
           "iterations": its, "ms_per_solve": t * 1e3, "device_ms_per_solve": t_dev * 1e3,
           "device_setup_ms": setup_ms, "us_per_iteration": per_it * 1e6,
           "bytes_per_iteration": bytes_it, "achieved_gbs": bytes_it / per_it / 1e9,
           "frac_of_hbm": bytes_it / per_it / 1e9 / peak,
           "note": "device time (CUDA events around the solve's kernels) minus the set-up and result kernels, "
                   "per iteration; ms_per_solve is the host clock around the call, host copies included; the "
                   "working set (~50 MB) is L2-resident"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        gs = g.astype(np.float32).astype(np.float64)
        t0 = time.perf_counter()
        _, _, _, it_cpu = oracle.solvegc2(0, intmat, gs, b.astype(np.float64), tol=1e-10)
        out["cpu_port"] = {"ms_per_solve": (time.perf_counter() - t0) * 1e3, "iterations": it_cpu, "cores": 1,
                           "kind": "port", "sample": "the same solve, FP32 restatement of solvegc2"}
    return out


def plane_bench(args, gfsph, workloads, torch):
    """The granular collapse on the 30-degree plane (~2k particles, 200 x 400
    DEM at 5 m, Voellmy, fixed dt 0.01 s): all 2,000 steps on the device
    (CUDA events on the handle's stream), and on the CPU the FP32 oracle port
    over the same 2,000 steps, one thread."""
    w = workloads.inclined_plane()
    p = workloads.make_params(w, gfsph)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(w.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sim.close()
    out = {"workload": f"inclined plane: {w.n} particles, {w.meta['dem']}, Voellmy, {w.steps} steps",
           "device_s": ms / 1e3, "particle_steps_per_s": w.n * w.steps / (ms / 1e3),
           "note": "device time of the whole run (CUDA events); at 2k particles a step is launch-bound"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        topol = oracle.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv)
        st = oracle.State(w.x, w.v, w.rho, w.mass, w.hsml, topol, dt=p.dt)
        ny, nx = w.z.shape
        t0 = time.perf_counter()
        oracle.run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, st, w.steps)
        t_cpu = time.perf_counter() - t0
        out["cpu_port"] = {"s": t_cpu, "particle_steps_per_s": w.n * w.steps / t_cpu, "cores": 1, "kind": "port",
                           "sample": f"the same {w.steps} steps, FP32 oracle port"}
    return out


def wir_bench(args, gfsph, workloads, torch, nsteps=50):
    """Soil and water particles (ic_ws_Interact = 1, ic_SWalg = 1): the soil
    cap and water pond of workloads.soil_and_pond scaled to ~190k particles
    (0.33 m lattice, 240 x 240 DEM at 2 m).  The staged RK45 with the soil
    surface under the water rebuilt at every stage.  Device time from CUDA
    events on the handle's stream around `nsteps` steps after 10 warm-up
    steps; the oracle port times a bounded sample of the same state."""
    w, a = workloads.soil_and_pond(spacing=0.33, scale=2.0)
    n = a["x"].shape[0]
    p = workloads.make_params(w, gfsph)
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(a["x"], a["v"], a["rho"], a["mass"], a["hsml"], itype=a["itype"])
    sim.step(10)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nsteps
    st = sim.download()
    launches = sim.kernels_per_step() if hasattr(sim, "kernels_per_step") else None
    sim.close()
    out = {"workload": f"soil and water: {n} particles ({int((a['itype'] == 2).sum())} water), "
                       f"{w.meta['dem']}, Bingham soil, Manning water over the soil surface (ic_SWalg 1)",
           "steps": nsteps, "device_ms_per_step": ms, "particle_steps_per_s": n / (ms / 1e3),
           "finite": bool(np.isfinite(st["x"]).all()),
           "note": "device time (CUDA events on the handle's stream); per step 3 extra launches per RK stage "
                   "rebuild the soil surface"}
    if launches is not None:
        out["launches_per_step"] = launches
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        topol = oracle.initial_topol(w.z, w.dx, w.dy, w.const, deriv=p.dem_deriv)
        flag = np.where(a["itype"] == 2, 2, 0).astype(np.int32)
        so = oracle.State(st["x"], st["v"], st["rho"], st["mass"], st["hsml"], topol, flag=flag | st["flag"],
                          dt=p.dt)
        ny, nx = w.z.shape
        k = 2
        t0 = time.perf_counter()
        oracle.run(oracle.MODE_FP32, p, nx, ny, w.dx, w.dy, so, k)
        t_cpu = time.perf_counter() - t0
        out["cpu_port"] = {"particle_steps_per_s": n * k / t_cpu, "cores": 1, "kind": "port",
                           "sample": f"{k} steps of the same state after the GPU run, FP32 oracle port"}
    return out


def gfl_bench(args, gfsph, workloads, peak, nsteps=100):
    """The GFL Taylor-Galerkin step on the coupled case's mesh: the 500 x
    500-node window of the DEM background triangulation at 2 m (498,002
    triangles), a dam break over a sloping bed with Manning and Voellmy
    friction, 3 Gauss points, 3 consistent-mass sweeps.  Device time from CUDA
    events around `nsteps` steps (one call).  Algorithmic bytes per step: per
    node h, hu, hv read and written (24), Topol (36), the lumped mass (4) and
    its adjacency row pointer (4); per element the connectivity (12), the
    geometry (28), Topel (36) and its three adjacency entries (24); and per
    further sweep the adjacency, the element areas and three node vectors
    (rhs, the iterate in and out: 36 per node)."""
    nw = 500
    intmat, coord = workloads.p1_mesh(nw, nw, 2.0)
    x, y = coord[:, 0], coord[:, 1]
    z = (50.0 - 0.05 * x + 2.0 * np.sin(y / 40.0)).astype(np.float32)
    u = np.zeros((coord.shape[0], 3), np.float32)
    u[:, 0] = np.where(x < 300.0, 4.0, 0.0)
    const = {1: 9.8, 2: 2000.0, 3: 0.03, 5: 5, 9: 0.2, 10: 0.02}
    g = gfsph.Gfl(coord, intmat, z, const, ntype=3, ngaus=3, niter=3)
    g.set_state(u)
    dt = 0.02
    g.step(10, dt)
    t0 = time.perf_counter()
    g.step(nsteps, dt)
    host_s = time.perf_counter() - t0
    dev_ms = g.device_ms()
    launches = g.launch_count()
    out_state, _ = g.state()
    g.close()
    npoin, nelem = coord.shape[0], intmat.shape[0]
    niter = 3
    bytes_step = npoin * (24 + 36 + 4 + 4) + nelem * (12 + 28 + 36 + 24) + (niter - 1) * (nelem * 28 + npoin * 36)
    per_step = dev_ms / 1e3 / nsteps
    out = {"mesh": f"{npoin} nodes, {nelem} triangles (500 x 500 window at 2 m)", "steps": nsteps,
           "device_ms_per_step": per_step * 1e3, "host_ms_per_step": host_s * 1e3 / nsteps,
           "node_steps_per_s": npoin / per_step, "launches_per_step": launches / (nsteps + 10),
           "bytes_per_step": bytes_step, "achieved_gbs": bytes_step / per_step / 1e9,
           "frac_of_hbm": bytes_step / per_step / 1e9 / peak, "finite": bool(np.isfinite(out_state).all()),
           "note": "device time (CUDA events around the step call's kernels); the working set (~120 MB) is "
                   "about the size of L2"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        k = 4
        t0 = time.perf_counter()
        oracle.gfl_run(coord.astype(np.float32), intmat, z, const, u, 0, dt)
        t_setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        oracle.gfl_run(coord.astype(np.float32), intmat, z, const, u, k, dt)
        t_cpu = time.perf_counter() - t0 - t_setup
        out["cpu_port"] = {"ms_per_step": t_cpu * 1e3 / k, "setup_ms": t_setup * 1e3, "cores": 1, "kind": "port",
                           "sample": f"{k} steps of the same mesh (set-up timed apart), FP32 restatement"}
    return out


def adjoint_bench(gfsph, workloads, torch, nsteps=1000, every=100, sle=0):
    """The adjoint of the calibration case (config 5's shape): ~50k particles
    on a 512^2 DEM at 5 m (no erosion, fixed dt; fixed smoothing lengths, or
    with sle = 1 their update after every step), `nsteps` steps recorded with
    a checkpoint every `every` and swept back (the config runs 5,000 steps;
    the cost per step does not depend on how many).  Device time from CUDA
    events on the handle's stream around the plain forward run, the recording
    run and the backward sweep (which recomputes each step's forward pass from
    its segment's checkpoint)."""
    w = workloads.fractal_channel(n_target=50_000, dem_k=9, cell=5.0, erosion=None)
    p = workloads.make_params(w, gfsph, sle=sle, ic_adapt=0)
    stream = torch.cuda.Stream()
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.set_stream(stream.cuda_stream)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    sim.step(3)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / nsteps

    def restart():
        sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
        sim.set_time(0.0, p.dt)

    # one untimed run first: the buffers grow to the flow's extent once, so
    # the timed forward, recording and backward runs all start grown
    restart()
    sim.step(nsteps)
    restart()
    _, t_fwd = timed(lambda: sim.step(nsteps))
    restart()
    rng = np.random.default_rng(0)
    gx = rng.normal(size=(w.n, 2)).astype(np.float32)
    gv = rng.normal(size=(w.n, 2)).astype(np.float32)
    adj, t_rec = timed(lambda: gfsph.Adjoint(sim, nsteps, every=every))
    g, t_bwd = timed(lambda: adj.backward(gx, gv))
    adj.close()
    sim.close()
    hs = "hsml updated every step (sle 1)" if sle else "fixed hsml"
    return {"workload": f"{w.n} particles, {w.meta['dem']}, Voellmy, {hs}, fixed dt", "steps": nsteps,
            "checkpoint_every": every, "forward_ms_per_step": t_fwd, "recording_ms_per_step": t_rec,
            "backward_ms_per_step": t_bwd, "backward_over_forward": t_bwd / t_fwd, "dL_dtanfi": g["tanfi"],
            "dL_dxi": g["xi"],
            "note": "device time (CUDA events on the handle's stream); the backward step includes the forward "
                    "recomputation of its segment's states and of its own step from the kept checkpoints"}


def coupled_bench(gfsph, workloads, torch, nsteps=10):
    """Config 3 as one run: the 4M-particle Bingham case on the 4096^2 DEM at
    2 m with, every step, the SPH step and the coupling pass get_gradhs_w on
    a 500 x 500-node window of the DEM background triangulation (498,002
    triangles) around the first release, its projection solved by the device
    CG to 1e-10 (squared-norm ratio).  Device time from CUDA events around
    the steps, after 3 warm-up steps; the coupling pass copies its nodal
    outputs to the host each step, as a caller would read them."""
    w = workloads.multi_release()
    p = workloads.make_params(w, gfsph)
    stream = torch.cuda.Stream()
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.set_stream(stream.cuda_stream)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    ny, nx = w.z.shape
    nw = 500
    c = np.floor(w.x[: w.n // 8].mean(axis=0) / w.dx).astype(int)  # inside the first release
    ix0 = int(min(max(c[0] - nw // 2, 0), nx - nw))
    iy0 = int(min(max(c[1] - nw // 2, 0), ny - nw))

    def one():
        sim.step(1)
        sim.gradhs(ix0, iy0, nw, nw, niter=0, tol=1e-10)

    for _ in range(3):
        one()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(nsteps):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nsteps
    e0.record(stream)
    sim.step(nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / nsteps
    sim.close()
    return {"workload": f"{w.n} particles, {w.meta['dem']}, Bingham, coupling window {nw}x{nw} nodes "
                        f"({2 * (nw - 1) ** 2} triangles) with the CG projection every step",
            "steps": nsteps, "ms_per_coupled_step": ms, "ms_per_sph_step": ms_step,
            "particle_steps_per_s": w.n / (ms / 1e3), "sph_particle_steps_per_s": w.n / (ms_step / 1e3),
            "note": "device time (CUDA events), 3 warm-up steps; the config's 2,000 steps at this rate take "
                    f"{2000 * ms / 1e3:.1f} s"}


def couple_bench(sim, w, gfsph):
    """The coupling pass get_gradhs_w on the 500 x 500-node window of the DEM
    around the flow: node depths from the particles, element gradients,
    5 sweeps (the reference's) and, separately, the CG projection."""
    st = sim.download()
    act = st["flag"] == 0
    c = np.floor(st["x"][act].mean(axis=0) / w.dx).astype(int)
    ny, nx = w.z.shape
    nw = min(500, nx, ny)
    ix0 = int(min(max(c[0] - nw // 2, 0), nx - nw))
    iy0 = int(min(max(c[1] - nw // 2, 0), ny - nw))
    out = {"window": f"{nw}x{nw} nodes, {2 * (nw - 1) ** 2} triangles", "particles": int(act.sum())}
    for niter, key in ((5, "sweeps_5"), (0, "cg")):
        sim.gradhs(ix0, iy0, nw, nw, niter=niter)
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            sim.gradhs(ix0, iy0, nw, nw, niter=niter)
            ts.append(time.perf_counter() - t0)
        out[key + "_ms"] = statistics.median(ts) * 1e3
    out["note"] = "host clock, outputs copied to the host (3 MB)"
    return out


def run_leg(args):
    """One secondary leg alone (--leg), on one GPU: its JSON line."""
    import torch
    torch.cuda.set_device(0)
    import build as pkg_build
    pkg_build.build()
    import gfsph
    import workloads
    peak, _ = load_peaks()
    if args.leg == "gfl":
        out = gfl_bench(args, gfsph, workloads, peak)
    elif args.leg == "wir":
        out = wir_bench(args, gfsph, workloads, torch)
    elif args.leg == "plane":
        out = plane_bench(args, gfsph, workloads, torch)
    elif args.leg == "adjoint":  # --steps recorded steps, a checkpoint every --steps // 10
        out = adjoint_bench(gfsph, workloads, torch, nsteps=args.steps, every=max(1, args.steps // 10))
    else:
        out = cg_bench(args, gfsph, workloads, peak)
    print(json.dumps({"leg": args.leg, **out}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="gfsph", choices=["gfsph", "reference"])
    ap.add_argument("--n", type=int, default=200_000, help="particles per replica")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ensemble", type=int, default=512, help="realizations of the ensemble line (0: none)")
    ap.add_argument("--ensemble-steps", type=int, default=8)
    ap.add_argument("--ensemble-wave", type=int, default=64, help="members held on the device at once")
    ap.add_argument("--no-extras", action="store_true", help="only the step: no ensemble, CG, coupling, adjoint")
    ap.add_argument("--leg", choices=["gfl", "wir", "plane", "cg", "adjoint"],
                    help="run one secondary leg alone and print its line (for profiling it)")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    args.warmup = max(args.warmup, 3)
    if args.leg:
        return run_leg(args)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td

    import build as pkg_build
    pkg_build.build()
    import gfsph
    import workloads

    w = workloads.fractal_channel(n_target=args.n, seed=2 + rank)
    p = workloads.make_params(w, gfsph)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # the flush, the events and the library share one stream
    sim = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
    sim.set_stream(stream.cuda_stream)
    sim.upload(w.x, w.v, w.rho, w.mass, w.hsml)
    n = w.n
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # The clock sampler (200 ms period) runs from the warm-up through the
    # timed steps and their two replays below, so that the timed region,
    # a few ms long, is bracketed by samples taken under the same load.
    clk = ClockSampler(local).__enter__()
    # warm-up (graph capture, capacity growth)
    for _ in range(args.warmup):
        sim.step(1)

    # ---- timed: device-resident state, L2 flushed before every step
    sim.profile(2)
    l0 = sim.launch_count()
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        sim.step(1)
    barrier()
    launches = sim.launch_count() - l0
    ms_local, nsteps = sim.profile_read().get("step_batches", (0.0, 0))
    ms_total, n_job, value = combine_ranks(ms_local, n, args.steps, dist, "cuda")

    # The passes below replay the timed steps (warm-up + 1 .. warm-up + K) on a
    # fresh handle from the same release: the run is deterministic, and the
    # flow's cost per step changes as it spreads, so only the same steps
    # compare.
    def replay():
        s2 = gfsph.Sim(p, w.z, dx=w.dx, dy=w.dy)
        s2.set_stream(stream.cuda_stream)
        s2.upload(w.x, w.v, w.rho, w.mass, w.hsml)
        for _ in range(args.warmup):
            s2.step(1)
        return s2

    # ---- steady state: the K timed steps in one call, L2 not flushed
    s2 = replay()
    s2.profile(2)
    barrier()
    s2.step(args.steps)
    ms_steady = s2.profile_read().get("step_batches", (0.0, 0))[0]
    steady = n * args.steps / (ms_steady / 1000.0)
    s2.close()

    # ---- per-kernel device times (events around every launch) over the K
    # timed steps, L2 flushed before each
    s2 = replay()
    s2.profile(1)
    for _ in range(args.steps):
        flush.zero_()
        s2.step(1)
    kprof = s2.profile_read()
    s2.close()
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    clocks["window"] = "warm-up, timed steps and their two replays"
    tot = sum(ms for ms, _ in kprof.values())
    dom = max(kprof, key=lambda k: kprof[k][0])
    dom_ms = kprof[dom][0] / kprof[dom][1]
    peak, peak_kind = load_peaks()
    st_now = sim.download()
    search_stats = sim.stats()
    sim_search = sim.get_search()
    nact = int((st_now["flag"] == 0).sum())
    b_launch = B_ALG.get(dom, 0) * nact
    achieved = b_launch / (dom_ms / 1000.0) / 1e9
    shares = {k: round(ms / tot, 4) for k, (ms, _) in sorted(kprof.items(), key=lambda kv: -kv[1][0])}
    issue = None
    if dom in NCU_PER_PARTICLE and NCU_STEPS == (args.warmup + 1, args.warmup + args.steps):
        wi = NCU_PER_PARTICLE[dom]["warp_inst"] * nact
        issue = {"warp_inst_per_launch": wi, "achieved_warp_inst_per_s": wi / (dom_ms / 1000.0),
                 "peak_warp_inst_per_s": ISSUE_PEAK, "frac": wi / (dom_ms / 1000.0) / ISSUE_PEAK,
                 "ncu_steps": list(NCU_STEPS)}

    # ---- e2e through the C ABI with pinned host buffers
    pin = {k: torch.empty(a.shape, dtype=torch.float32 if a.dtype == np.float32 else torch.int32,
                          pin_memory=True).numpy() for k, a in st_now.items()}
    for k in pin:
        pin[k][...] = st_now[k]
    h2d = n * (8 + 8 + 4 + 4 + 4 + 4)
    d2h = n * (8 + 8 + 4 + 4 + 4 + 4)
    for _ in range(3):
        sim.upload(pin["x"], pin["v"], pin["rho"], pin["mass"], pin["hsml"], pin["flag"])
        sim.step(1)
        sim.download(pin)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = min(args.steps, 100)
    e0.record(stream)
    for _ in range(e2e_steps):
        sim.upload(pin["x"], pin["v"], pin["rho"], pin["mass"], pin["hsml"], pin["flag"])
        sim.step(1)
        sim.download(pin)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    _, _, e2e_value = combine_ranks(e2e_ms, n, e2e_steps, dist, "cuda")

    extras = world == 1 and not args.no_extras
    couple_line = couple_bench(sim, w, gfsph) if extras else None
    sim.close()
    cg_line = cg_bench(args, gfsph, workloads, peak) if extras else None
    gfl_line = gfl_bench(args, gfsph, workloads, peak) if extras else None
    wir_line = wir_bench(args, gfsph, workloads, torch) if extras else None
    plane_line = plane_bench(args, gfsph, workloads, torch) if extras else None
    adj_line = adjoint_bench(gfsph, workloads, torch) if extras else None
    adj1_line = None
    if extras:
        try:
            adj1_line = adjoint_bench(gfsph, workloads, torch, nsteps=200, every=20, sle=1)
        except gfsph.GfsphError as e:  # e.g. a coarse grid level appeared: outside the adjoint's scope
            adj1_line = {"unavailable": str(e)}
    big_line = coupled_bench(gfsph, workloads, torch) if extras else None
    ens_line = None
    if extras and args.ensemble > 0:
        ens_line = ensemble_bench(args, torch, gfsph, workloads)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(args.n, args.warmup, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**bench_config(n, w), **({"parallelism": "replicas, one per GPU"} if world > 1 else {})},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": (NCU_PER_PARTICLE[dom]["dram_bytes"] * nact) if dom in NCU_PER_PARTICLE else None,
                         "traffic_source": NCU_SOURCE,
                         "issue_bound": issue,
                         "alg_bytes_per_launch": b_launch, "avg_launch_ms": dom_ms,
                         "step_achieved_gbs": 168 * n * args.steps / (ms_total / 1000.0) / 1e9 / world},
            "kernel_shares": shares,
            "search": {**search_stats, "level_factor": sim_search[0], "cell_div": sim_search[1]},
            "steady_state": {"value": steady, "unit": UNIT, "note": "the same K steps in one call, L2 not flushed"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if cg_line:
            line["cg"] = cg_line
        if adj1_line:
            line["adjoint_sle1"] = adj1_line
        if gfl_line:
            line["gfl"] = gfl_line
        if wir_line:
            line["wir"] = wir_line
        if plane_line:
            line["plane"] = plane_line
        if adj_line:
            line["adjoint"] = adj_line
        if big_line:
            line["coupled_large_case"] = big_line
        if couple_line:
            line["couple"] = couple_line
        if ens_line:
            if cpu:
                mean_n = ens_line["particles_total"] / ens_line["realizations"]
                ens_line["cpu_sequential_realizations_per_s"] = cpu["value"] / mean_n / 5000.0
            line["ensemble"] = ens_line
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
