#!/usr/bin/env python
"""Benchmark of the B200 MHD stage engine (one JSON line on stdout, rank 0).

Workload (the metric's headline configuration): 3D Cartesian MHD blast on
256^3 zones over [-0.5,0.5]^3, periodic, gamma = 5/3, WENO-Z reconstruction,
HLLD flux, constrained transport, SSP-RK3, CFL 0.4.  A step is one full RK3
step (FINDDT + 3 stages) over all 256^3 zones; the workload is 200 steps.

  value   zone-updates/s, device-timed with CUDA events on the engine's stream,
          state resident in HBM (7 GB, far larger than the 126 MB L2);
  e2e     the same metric through the C-ABI with host buffers: pinned-host
          upload of the Fortran-layout state, INITIAL_UPDATE, the K steps and
          the download of the result, all inside the wall-clock window;
  roofline the dominant kernel (a flux sweep: reconstruction + Riemann)
          against the FP64 roofline: max(algorithmic bytes / measured copy
          bandwidth, exact FP64 operation count / measured DFMA peak) over
          its CUDA-event duration; the HBM side alongside;
  parity_sample  the engine and the CPU oracle on the same 256x256x64 slab
          of the blast for 2 steps, compared bit for bit;
  cpu_baseline  the CPU oracle (a restatement of the reference's Fortran,
          -march=native, OpenMP on all host cores) on that slab.

`--impl reference` times that CPU oracle alone (the reference itself is
Fortran and cannot be built on this image) on the same workload, each step a
256x256x64 slab of it.  For N > 1 (torchrun, or `--gpus N`, which launches
torchrun itself) the grid is cut into N z slabs, one per rank, with ghost
planes exchanged over NCCL (strong scaling); `--replicas` runs N independent
copies instead.  Time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic HBM bytes of the fused face-flux kernel per zone (per launch):
# read 5 primitives + 2 transverse cell fields + 1 face field, write 5 hydro
# fluxes + 2 face EMFs, all FP64
FLUX_BYTES_PER_ZONE = (8 + 7) * 8
# whole RK3 step: 8 FP64 state words read+written per stage, u_old re-read in
# stages 2 and 3: (64+64) + 3*64 + 3*64
STEP_BYTES_PER_ZONE = 512


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    """Rank, world and process group from the torchrun environment.  NCCL
    (one rank per GPU) unless --dry-run, which uses gloo on the CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if args.dry_run:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        else:
            # NCCL's init log (communicator, ranks, transports) on stderr
            os.environ.setdefault("NCCL_DEBUG", "INFO")
            os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                    device_id=torch.device("cuda", local))
    return world, rank, local, dist


def ranks_info(dist):
    """What the process group is: its backend, size and (NCCL) version."""
    if not dist:
        return {"world_size": 1, "backend": None}
    info = {"world_size": dist.get_world_size(), "backend": dist.get_backend()}
    if info["backend"] == "nccl":
        import torch
        v = torch.cuda.nccl.version()
        info["nccl_version"] = ".".join(str(x) for x in v) if isinstance(v, tuple) else v
    return info


def self_spawn(n):
    """`bench.py --gpus N` outside torchrun: launch N ranks through
    torch.distributed.run on this node and return its exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def oracle_recipe():
    """Switch the oracle to its -march=native build (compiled on this host)
    for timing; returns the recipe's description."""
    from oracle import oracle as O
    return O.use_native()


def cpu_baseline_of(build, steps, sample, keep=False):
    """The CPU oracle (a restatement of the reference's Fortran, OpenMP) on a
    bounded sample of a workload, on all host cores and on the reference's
    hard-coded 4 threads (solver/mhd/main.f90:31).  keep: also return the
    all-cores run's final state, time reached and fallback count (the
    parity sample's oracle side)."""
    from oracle import oracle as O
    recipe = oracle_recipe()
    out = {"unit": "zone-updates/s", "kind": "port", "sample": sample, "build": recipe}
    kept = None
    try:
        allc = len(os.sched_getaffinity(0))
        for threads, key in ((allc, "value"), (4, "value_4_threads")):
            O.set_num_threads(threads)
            spec, prim, eps = build()
            o = O.Oracle(spec)
            o.set_state(prim, eps)
            o.initial_update()
            t = 0.0
            t0 = time.perf_counter()
            for _ in range(steps):
                dt = o.finddt()
                o.rk3_step(dt)
                t += dt
            el = time.perf_counter() - t0
            out[key] = spec["nx"] * spec["ny"] * spec["nz"] * steps / el
            if key == "value":
                out["cores"] = O.num_threads()
                out["seconds"] = el
                if keep:
                    from cumc3d_b200 import capi
                    p, e = o.get_state()
                    kept = dict(prim=p, eps=e, bcell=o.get_array(capi.ARR_BCELL), cs=o.get_array(capi.ARR_CS),
                                t=t, fallback=o.fallback_count(), spec=spec, init=(prim, eps))
            o.close()
        O.set_num_threads(allc)
    except Exception as ex:  # the baseline must not hide the GPU number
        out.update({"value": None, "cores": None, "sample": "failed: %s" % ex})
    return (out, kept) if keep else out


def blast_slab(n, nz, recon, riemann):
    """The headline blast as an n x n x nz periodic z slab (same cross-section,
    same scheme and flags), the CPU-sized sample of the workload."""
    from cumc3d_b200 import models
    sp, pr, ep = models.blast_3d(n, nz=nz, recon=recon, riemann=riemann)
    sp["positivity_fallback"] = 1
    sp["fix_periodic_normal_faces"] = 1
    return sp, pr, ep


def blast_workload(n, recon, riemann):
    return "blast3d_%d^3_%s_%s_ct_rk3_cfl0.4" % (n, recon, riemann)


def reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    if args.workload == "batch1d":
        return reference_batch(args, world)
    recipe = oracle_recipe()
    # every host thread this process may use (torchrun sets OMP_NUM_THREADS=1)
    O.set_num_threads(len(os.sched_getaffinity(0)))
    # the sample shrinks with the step count so that the whole run stays
    # within a few minutes: a 64-plane slab up to 25 steps with warm-up, down
    # to 32 planes (the same cross-section and scheme; thinner slabs would
    # spend a larger share of the work on z ghosts) for the full 200
    n = args.n
    nz = int(max(32, min(64, 8 * round(64 * 25 / max(1, args.steps + args.warmup) / 8))))
    spec, prim, eps = blast_slab(n, nz, args.recon, args.riemann)
    o = O.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    for _ in range(args.warmup):
        o.rk3_step(o.finddt())
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.rk3_step(o.finddt())
    el = time.perf_counter() - t0
    zones = n * n * nz
    value = zones * args.steps / el
    sample = ("each step one RK3 step of a %dx%dx%d periodic z slab of the %d^3 blast (same cross-section, "
              "scheme and flags; %d of %d z planes), %d timed steps after %d warm-up; %s" % (
                  n, n, nz, n, nz, n, args.steps, args.warmup, recipe))
    line = {
        "impl": "reference", "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": blast_workload(n, args.recon, args.riemann), "grid": [n, n, n], "recon": args.recon,
                   "riemann": args.riemann, "precision": "fp64", "boundary": "periodic",
                   "positivity_fallback": 1, "fix_periodic_normal_faces": 1},
        "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def batch_specs(precision, t_end=0.1, count=512):
    """The batched workload: 512 seeded 1D Riemann problems, n log-uniform in
    [128, 4096] (seed 20261203), HLLD + PPM, CFL 0.8, t_end 0.1 (the first
    `count` of them for profiler runs)."""
    from cumc3d_b200 import models
    params = models.batch_problems(512)[:count]
    return params, [models.riemann_1d(p["n"], p["left"], p["right"], p["bx"], t_end=t_end, precision=precision)
                    for p in params]


def bench_batch(args, world, rank, local, dist):
    import numpy as np
    import torch

    from cumc3d_b200 import engine, shard
    params_all, probs_all = batch_specs(args.precision, count=args.batch_problems)
    # the problems are independent: each rank runs its share (cost ~ n^2:
    # the step count grows with n), no collective on the data path
    mine = shard.shard_problems([p["n"] ** 2 for p in params_all], rank, world)
    params = [params_all[i] for i in mine]
    probs = [probs_all[i] for i in mine]
    b = engine.BatchSolver([sp for sp, _, _ in probs], positivity_fallback=1)

    def upload():
        for i, (_, prim, eps) in enumerate(probs):
            b.set_state(i, prim, eps)

    for _ in range(args.warmup):
        upload()
        b.run()
    stream = torch.cuda.ExternalStream(b.stream())
    total_ms, zu = 0.0, 0
    clocks = ClockSampler(local)
    clocks.start()
    l0 = b.launch_count()
    for _ in range(args.steps):
        upload()  # untimed: the initial state of every problem
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, steps, status = b.run()
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        zu += int(sum(p["n"] * int(k) for p, k in zip(params, steps)))
    clk = clocks.stop()
    launches = b.launch_count() - l0
    ms = shard.max_over_ranks(total_ms, dist, "cuda")
    zu = shard.sum_over_ranks(zu, dist, "cuda")
    value = zu / (ms * 1e-3)
    # end to end through the C-ABI with host buffers: upload, run, download
    e2e = None
    if not args.no_e2e:
        rows = [(np.empty((p["n"] + 6, 8)), np.empty(p["n"] + 6)) for p in params]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        upload()
        _, steps, _ = b.run()
        for i, (pr, ep) in enumerate(rows):
            b.L.cumc_batch_get_state(b.h, i, pr.ctypes.data, ep.ctypes.data)
        el = shard.max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        zu1 = shard.sum_over_ranks(int(sum(p["n"] * int(k) for p, k in zip(params, steps))), dist, "cuda")
        h2d = shard.sum_over_ranks(sum(pr.nbytes + ep.nbytes for _, pr, ep in probs), dist, "cuda")
        d2h = shard.sum_over_ranks(sum(pr.nbytes + ep.nbytes for pr, ep in rows), dist, "cuda")
        e2e = {"value": zu1 / el, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "wall_s": el,
               "note": "a step is one whole batched run (all problems to t_end)"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        sample = [i for i in np.argsort([p["n"] for p in params])[::37]][:8]
        t0 = time.perf_counter()
        zc = 0
        for i in sample:
            sp, prim, eps = probs[i]
            o = O.Oracle(dict(sp, positivity_fallback=1))
            o.set_state(prim, eps)
            o.initial_update()
            _, k = o.evolve(sp["t_end"], 10 ** 7)
            zc += params[i]["n"] * k
            o.close()
        el = time.perf_counter() - t0
        cpu = {"value": zc / el, "unit": "zone-updates/s", "cores": O.num_threads(), "kind": "port",
               "sample": "CPU oracle, %d of the 512 problems run to t_end one after another (%.1f s)" % (
                   len(sample), el)}
    b.close()
    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
            "config": {"workload": "batch1d_512_riemann_ppm_hlld_cfl0.8_t0.1", "problems": len(params_all),
                       "n_range": [128, 4096], "seed": 20261203, "precision": args.precision,
                       "positivity_fallback": 1,
                       "step": "one whole batched run: INITIAL_UPDATE + every problem's time loop",
                       "l2": "per-problem rows are L2-resident by design; state re-uploaded between runs",
                       "parallelism": "problems sharded over %d ranks" % world if world > 1 else "single"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def reference_batch(args, world):
    """The CPU oracle on the batched workload: a sample of its problems, each
    run to t_end as the reference runs one problem per execution."""
    import numpy as np
    from oracle import oracle as O
    params, probs = batch_specs("fp64")
    sample = [i for i in np.argsort([p["n"] for p in params])[::37]][:6]

    def one_pass():
        zc = 0
        for i in sample:
            sp, prim, eps = probs[i]
            o = O.Oracle(dict(sp, positivity_fallback=1))
            o.set_state(prim, eps)
            o.initial_update()
            _, k = o.evolve(sp["t_end"], 10 ** 7)
            zc += params[i]["n"] * k
            o.close()
        return zc

    for _ in range(min(args.warmup, 1)):
        one_pass()
    t0 = time.perf_counter()
    zc = 0
    nsteps = max(1, min(args.steps, 3))
    for _ in range(nsteps):
        zc += one_pass()
    el = time.perf_counter() - t0
    value = zc / el
    sample_txt = "%d of the 512 problems (every 37th by size) run to t_end, %d passes" % (len(sample), nsteps)
    line = {
        "impl": "reference", "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
        "n_gpus": world, "steps": nsteps, "warmup": args.warmup, "ms_per_step": el / nsteps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batch1d_512_riemann_ppm_hlld_cfl0.8_t0.1 (reference arm: CPU oracle sample)"},
        "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample_txt},
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def bench_poisson(args, world, rank, local, dist):
    """Self-gravity of the collapsar model: the red-black SOR of the spherical
    Poisson equation (model/collapsar/src/custom.f90:511-620) on an
    nr x ntheta x nphi grid of the seeded star (models.star_sph).  A step =
    --sor-iters iterations continuing from the current potential (as the
    model re-solves every 10 hydro steps); metric = cell-updates/s (interior
    cells x iterations per second).  Also reported: a full solve from phi = 0
    to 1e-10, the initial model's solve."""
    import numpy as np
    import torch

    from cumc3d_b200 import engine, models, shard
    nr, nth, nph = (int(v) for v in args.sor_grid.split(","))
    spec, prim, eps = models.star_sph(nr, nth, nph)
    cells = nr * nth * nph
    ra = spec["rho_atm"]
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.poisson_setup(ra, 1.9)
    it_step = args.sor_iters
    for _ in range(args.warmup):
        s.poisson_solve(max_iter=it_step, tol=0.0)  # tol 0: exactly it_step iterations
    stream = torch.cuda.ExternalStream(s.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = s.launch_count()
    e0.record(stream)
    total = 0
    for _ in range(args.steps):
        it, _, _ = s.poisson_solve(max_iter=it_step, tol=0.0)
        total += it
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = s.launch_count() - l0
    ms = shard.max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    value = world * cells * total / (ms * 1e-3)
    t_iter = ms / total
    # one iteration moves 56 B per interior cell: the cell's own phi read and
    # written (16), its three coefficients (24), its source term (8), and its
    # phi once more as the other colour's neighbour (8)
    peak_gbs, peak_kind = load_peaks()
    achieved = 56.0 * cells / (t_iter * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_sor_sweep<0,2> + k_sor_sweep<1,2> + k_sor_ghosts (one iteration)",
                "achieved": achieved, "peak": peak_gbs,
                "unit": "GB/s", "frac": achieved / peak_gbs, "traffic": None, "bytes_per_cell_iteration": 56,
                "avg_iteration_ms": t_iter, "peak_source": "MEASURED_PEAKS.json hbm_gbs (%s)" % peak_kind}
    # the initial model's solve: phi = 0, to 1e-10
    full = None
    if args.sor_full:
        s.poisson_setup(ra, 1.9)
        torch.cuda.synchronize()
        e0.record(stream)
        it_full, err_full, conv_full = s.poisson_solve(max_iter=100000, tol=1e-10)
        e1.record(stream)
        s.sync()
        torch.cuda.synchronize()
        full = {"iterations": it_full, "converged": conv_full, "final_error": err_full,
                "ms": e0.elapsed_time(e1), "tol": 1e-10, "omega": 1.9}
    # end to end through the C-ABI with host buffers: density state and the
    # start potential up, one step of iterations, the potential back
    e2e = None
    if not args.no_e2e:
        phi0 = s.poisson_get()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_state(prim, eps)
        s.poisson_set(phi0)
        it_e, _, _ = s.poisson_solve(max_iter=it_step, tol=0.0)
        phi1 = s.poisson_get()
        el = time.perf_counter() - t0
        e2e = {"value": world * cells * it_e / el, "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(prim.nbytes + eps.nbytes + phi0.nbytes), "d2h_bytes_per_step": int(phi1.nbytes),
               "wall_s": el, "note": "set_state + poisson_set + one step of %d iterations + poisson_get" % it_step}
    s.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        sp2, pr2, _ = models.star_sph(128, 64, 64)
        n_it = 300
        t0 = time.perf_counter()
        O.poisson_solve(sp2, pr2[3:-3, 3:-3, 3:-3, 0], sp2["rho_atm"], omega=1.9, tol=0.0, max_iter=n_it)
        el = time.perf_counter() - t0
        cpu = {"value": 128 * 64 * 64 * n_it / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": "CPU oracle (the reference's loops in order, one thread), the star on a "
                         "128x64x64 grid, %d iterations (%.1f s; coefficient setup included)" % (n_it, el)}
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "collapsar_self_gravity_sor_%dx%dx%d_star" % (nr, nth, nph),
                       "iterations_per_step": it_step, "omega": 1.9,
                       "l2": "colour arrays %.1f GB, larger than L2" % (cells * 56 / 1e9),
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": roofline, "full_solve_from_zero": full, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def bench_collapsar(args, world, rank, local, dist):
    """The collapsar model from its shipped progenitor (156 x 44 x 128,
    spherical, PPM + HLLD, CFL 0.8; tests/golden/collapsar_profile.npz holds
    the files' values): INITIAL_UPDATE, the initial potential (red-black SOR
    from phi = 0 to 1e-10 at omega 1.9), then K host-driven steps (FINDDT,
    RUNGEKUTTA with the floors, the self-gravity + black hole source and the
    hole's growth) with the potential re-solved every n_pot = 10 steps from
    the last one, as main.f90 and CUSTOM_UPDATE do.  Metric: zone-updates/s
    of the run with its re-solves; device time (CUDA events on the engine
    stream) around the K steps."""
    import torch

    from cumc3d_b200 import engine, models
    spec, prim, eps = models.collapsar_model(os.path.join(ROOT, "tests", "golden", "collapsar_profile.npz"))
    zones = spec["nx"] * spec["ny"] * spec["nz"]
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    s.autotune()
    s.poisson_setup(spec["rho_atm"], 1.9)
    stream = torch.cuda.ExternalStream(s.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    it0, err0, conv0 = s.poisson_solve(100000, 1e-10)
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    initial = {"iterations": it0, "final_error": err0, "converged": conv0, "ms": e0.elapsed_time(e1)}
    phi0 = s.poisson_get()
    s.collapsar_set(spec["m_bh"], spec["c_code"])
    n_pot = spec["n_pot"]
    n_step = 0

    def step():
        nonlocal n_step
        s.rungekutta(s.finddt())
        resolves = 0
        if n_step % n_pot == 0:  # CUSTOM_UPDATE at p_in = 3
            s.poisson_solve(100000, 1e-10)
            resolves = 1
        n_step += 1
        return resolves
    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    clocks.start()
    l0 = s.launch_count()
    e0.record(stream)
    resolves = sum(step() for _ in range(args.steps))
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = s.launch_count() - l0
    ms = e0.elapsed_time(e1)
    m_bh, r_sh = s.collapsar_get()
    divb = s.find_divb()
    s.close()
    cpu = None
    if rank == 0 and not args.no_cpu:
        # the oracle on the same model from the same initial potential: 2 steps
        # (FINDDT + RUNGEKUTTA with the collapsar hooks), no re-solve
        from oracle import oracle as O
        o = O.Oracle(spec)
        o.set_state(prim, eps)
        o.initial_update()
        o.set_phi(phi0)
        o.collapsar_set(spec["m_bh"], spec["c_code"])
        t0 = time.perf_counter()
        for _ in range(2):
            o.rk3_step(o.finddt())
        el = time.perf_counter() - t0
        o.close()
        cpu = {"value": zones * 2 / el, "unit": "zone-updates/s", "cores": O.num_threads(), "kind": "port",
               "sample": "2 steps of the same model from the same initial potential, no potential re-solve"}
    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": zones * args.steps / (ms * 1e-3), "unit": "zone-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data":
                "the reference's shipped collapsar progenitor (model/collapsar/profile)",
            "config": {"workload": "collapsar_156x44x128_shipped_progenitor_ppm_hlld_ct_cfl0.8",
                       "n_pot": n_pot, "omega": 1.9, "tolerance": 1e-10,
                       "parallelism": "replicas" if world > 1 else "single"},
            "results": {"initial_potential_solve": initial, "potential_resolves_timed": resolves,
                        "m_bh": m_bh, "r_sh": r_sh, "max_divb": divb},
            "e2e": None, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line))
    return 0


def bench_snapshots(args, world, rank, local, dist):
    """Output without stalling: the 3D blast at --n^3 run for --steps steps,
    with a snapshot of the reference's output datasets every
    --snapshot-every steps (cumc_snapshot_start into page-locked buffers, the
    copy overlapping the next steps; wait before the next start), against the
    same run without output and with a blocking full-state download
    (cumc_get_state, what an UPDATE HOST + write would cost).  Metric =
    zone-updates/s of the run with snapshots; wall clock around each run."""
    import numpy as np
    import torch

    from cumc3d_b200 import engine, models, snapshot
    n, every = args.n, args.snapshot_every
    spec, prim, eps = models.blast_3d(n, recon=args.recon, riemann=args.riemann)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    zones = spec["nx"] * spec["ny"] * spec["nz"]
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    s.autotune()
    s.evolve(1e30, args.warmup)
    bufs = snapshot.buffers(spec, pinned=True)
    host_p = np.empty_like(prim)
    host_e = np.empty_like(eps)
    s.snapshot_start(*bufs)  # allocate the staging buffer before timing
    s.snapshot_wait()
    clocks = ClockSampler(local)
    clocks.start()

    def run(mode):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done = 0
        while done < args.steps:
            _, k = s.evolve(1e30, every)
            done += k
            if mode == "async":
                s.snapshot_start(*bufs)
            elif mode == "blocking":
                s.L.cumc_get_state(s.h, host_p.ctypes.data, host_e.ctypes.data)
        if mode == "async":
            s.snapshot_wait()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3, done
    ms_none, k_none = run("none")
    ms_async, k_async = run("async")
    ms_block, k_block = run("blocking")
    clk = clocks.stop()
    s.close()
    snap_bytes = sum(int(b.nbytes) for b in bufs)
    value = zones * k_async / (ms_async * 1e-3)
    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
            "steps": k_async, "warmup": args.warmup, "ms_per_step": ms_async / k_async, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "blast3d_%d^3_with_snapshots_every_%d_steps" % (n, every),
                       "snapshot_bytes": snap_bytes, "timing": "wall clock around each run (host-driven loop)"},
            "results": {"ms_per_step_no_output": ms_none / k_none,
                        "ms_per_step_async_snapshots": ms_async / k_async,
                        "ms_per_step_blocking_get_state": ms_block / k_block,
                        "snapshots": k_async // every},
            "e2e": None, "cpu_baseline": None, "clocks": clk,
        }
        print(json.dumps(line))
    return 0


def bench_slabs(args, world, rank, local, dist):
    """The 3D path cut along z into slabs (cumc_group_*, one process): the
    blast at --n^3 as --slabs slabs spread round-robin over the visible GPUs,
    against the undivided grid, both host-driven (FINDDT + RUNGEKUTTA per
    step).  Metric = zone-updates/s of the slab group (whole grid); with one
    GPU the slabs share it, which measures the exchange's cost.  Under
    torchrun (N > 1) one slab per rank instead (bench_slab_ranks)."""
    import torch

    from cumc3d_b200 import engine, models
    if world > 1:
        return bench_slab_ranks(args, world, rank, local, dist)
    n, ns = args.n, args.slabs
    spec, prim, eps = models.blast_3d(n, recon=args.recon, riemann=args.riemann)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    zones = spec["nx"] * spec["ny"] * spec["nz"]
    ndev = torch.cuda.device_count()
    sizes = [n // ns + (1 if i < n % ns else 0) for i in range(ns)]

    def run(obj, step, finddt):
        for _ in range(args.warmup):
            step(finddt())
        for d in range(ndev):
            torch.cuda.synchronize(d)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step(finddt())
        for d in range(ndev):
            torch.cuda.synchronize(d)
        return (time.perf_counter() - t0) * 1e3 / args.steps

    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    s.autotune()
    ms_single = run(s, s.rungekutta, s.finddt)
    s.close()
    g = engine.SlabGroup(spec, sizes, devices=[i % ndev for i in range(ns)])
    g.set_state(prim, eps)
    g.initial_update()
    for sl in g.slabs:
        sl.autotune()
    clocks = ClockSampler(local)
    clocks.start()
    ms_group = run(g, g.step, g.finddt)
    clk = clocks.stop()
    g.close()
    plane = (spec["nx"] + 6) * (spec["ny"] + 6) * 8
    cuts = ns  # a periodic ring
    xbytes = cuts * 2 * 3 * 3 * plane * (13 + 7)  # per step: sides x stages x planes x arrays
    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": zones / (ms_group * 1e-3), "unit": "zone-updates/s",
            "n_gpus": ndev, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_group,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "blast3d_%d^3_as_%d_z_slabs_on_%d_gpus" % (n, ns, ndev), "slabs": sizes,
                       "timing": "wall clock around host-driven steps, all devices synchronised"},
            "results": {"ms_per_step_undivided": ms_single, "ms_per_step_slabs": ms_group,
                        "ghost_bytes_per_step": xbytes},
            "e2e": None, "cpu_baseline": None, "clocks": clk,
        }
        print(json.dumps(line))
    return 0


def bench_slab_ranks(args, world, rank, local, dist):
    """One slab per rank (SlabRank): the blast at --n^3 cut into N z slabs,
    one per GPU, a periodic ring; ghost planes by NCCL send/recv into each
    receiver's memory, dt by an all-reduce (min), host-driven steps.  Strong
    scaling: the grid is fixed.  Time: CUDA events on each rank's engine
    stream around the K steps, the max over ranks.  e2e: each rank's slab
    uploaded from pinned host memory, INITIAL_UPDATE, the K steps and the
    slab's download, wall clock, max over ranks."""
    import torch

    from cumc3d_b200 import engine, models, shard
    n = args.n
    spec, prim, eps = models.blast_3d(n, recon=args.recon, riemann=args.riemann)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    zones = spec["nx"] * spec["ny"] * spec["nz"]
    sizes = [n // world + (1 if i < n % world else 0) for i in range(world)]
    r = engine.SlabRank(spec, sizes, rank)
    r.set_state(prim, eps)
    r.initial_update()
    tuning = r.solver.autotune()
    for _ in range(args.warmup):
        r.step(r.finddt())
    stream = torch.cuda.ExternalStream(r.solver.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = r.solver.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        r.step(r.finddt())
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = int(shard.sum_over_ranks(r.solver.launch_count() - l0, dist, "cuda"))
    ms = shard.max_over_ranks(e0.elapsed_time(e1), dist, "cuda") / args.steps
    xbytes = sum(r.send[k].numel() for k in r.send) * 3  # sent per step by this rank (3 stages)
    # this rank's flux sweeps against the FP64 roofline (its slab's zones)
    prof = r.solver.profile_step(args.profile_steps)
    try:
        fp64_peak = engine.fp64_peak_tflops()
    except Exception:
        fp64_peak = None
    roofline, _, _ = flux_roofline(args, prof, args.profile_steps, spec["nx"] * spec["ny"] * sizes[rank],
                                   tuning, fp64_peak)
    roofline["note"] = "rank 0's slab (%d z planes)" % sizes[0]
    r.close()
    # end to end: host slab in, K steps, slab out
    e2e = None
    if not args.no_e2e:
        o = sum(sizes[:rank])
        hp = torch.from_numpy(prim[o:o + sizes[rank] + 6].copy()).pin_memory()
        he = torch.from_numpy(eps[o:o + sizes[rank] + 6].copy()).pin_memory()
        r2 = engine.SlabRank(spec, sizes, rank)
        r2.set_state(prim, eps)  # untimed: the tuner needs a live state
        r2.initial_update()
        r2.solver.autotune()
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r2.solver.set_state_ptr(hp.data_ptr(), he.data_ptr())
        r2.initial_update()
        for _ in range(args.steps):
            r2.step(r2.finddt())
        out_p, out_e = r2.get_state()
        torch.cuda.synchronize()
        el = shard.max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        nbytes = shard.sum_over_ranks(int(hp.numel() * 8 + he.numel() * 8), dist, "cuda")
        r2.close()
        e2e = {"value": zones * args.steps / el, "unit": "zone-updates/s",
               "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": nbytes / args.steps,
               "wall_s": el, "steps": args.steps,
               "note": "each rank's slab uploaded and downloaded once per run of %d steps, amortised" % args.steps}
    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": zones / (ms * 1e-3), "unit": "zone-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": blast_workload(n, args.recon, args.riemann), "grid": [n, n, n],
                       "recon": args.recon, "riemann": args.riemann, "precision": "fp64", "boundary": "periodic",
                       "positivity_fallback": 1, "fix_periodic_normal_faces": 1, "slabs": sizes,
                       "parallelism": parallelism_of(args, world),
                       "l2": "state %.1f GB per rank, >> 126 MB L2 (no flush needed)" % (
                           7.0 * sizes[0] / n),
                       "timing": "CUDA events on each rank's engine stream, max over ranks", "autotuned": tuning},
            "roofline": roofline,
            "results": {"ghost_bytes_sent_per_step_rank0": xbytes},
            "e2e": e2e, "cpu_baseline": None, "gpu_launches": launches, "ranks": ranks_info(dist), "clocks": clk,
        }
        print(json.dumps(line))
    dist.barrier()
    dist.destroy_process_group()
    return 0


def _evolve_timed(engine, torch, spec, prim, eps, warmup, steps=None, t_end=None, tuning="auto", setup=None):
    """Run one handle: W warm-up steps, then time the rest (to t_end, or K
    more steps) with CUDA events on the engine stream.  Returns the handle
    (still open), timed steps and milliseconds."""
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    if setup is not None:
        setup(s)
    if tuning == "auto":
        s.autotune()
    te = t_end if t_end is not None else 1e30
    s.evolve(te, warmup)
    s.sync()
    stream = torch.cuda.ExternalStream(s.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    _, n = s.evolve(te, steps if steps is not None else 2 ** 31 - 1)
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    return s, n, e0.elapsed_time(e1)


def bench_config(args, world, rank, local, dist):
    """Other configurations of the path: Brio-Wu (1D, PPM + HLLD), the CP
    Alfven wave (256^3, one period, FP64 and FP32 with their relative L1), and
    the cylindrical torus (192 x 128 x 192, WENO + HLLD, 2000 steps)."""
    import numpy as np
    import torch

    from cumc3d_b200 import capi, engine, models
    extra = {}
    cpu = None
    clocks = ClockSampler(local)
    if args.workload == "briowu":
        spec, prim, eps = models.brio_wu(800, recon=args.recon_c or "ppm", riemann=args.riemann,
                                         precision=args.precision)
        zones = 800
        clocks.start()
        s, n, ms = _evolve_timed(engine, torch, spec, prim, eps, args.warmup, t_end=spec["t_end"])
        clk = clocks.stop()
        name = "briowu_800_%s_%s_cfl0.8_t0.1" % (spec["recon"], spec["riemann"])
        extra["time_reached"] = s.time
        s.close()
        # the same problem through the persistent 1D kernel (cumc_batch_*, one
        # problem; bit-identical to the 3D engine): one launch instead of ~60
        # graph nodes per step
        bs = engine.BatchSolver([spec])
        stb = torch.cuda.ExternalStream(bs.stream())
        pk = {}
        # one CTA (the batch default for problems of up to 1024 cells), and the
        # problem shared by an 8-CTA cluster (one cell per thread): a single
        # problem's time is its steps' latency, which more threads shorten
        for label, shape in (("one_cta", (8, 1024)), ("cluster_of_8", (8, 128))):
            bs.set_cluster(*shape)
            for _ in range(args.warmup):
                bs.set_state(0, prim, eps)
                bs.run()
            bs.set_state(0, prim, eps)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stb)
            _, bsteps, _ = bs.run()
            e1.record(stb)
            torch.cuda.synchronize()
            bms = e0.elapsed_time(e1)
            pk[label] = {"zone_updates_per_s": zones * int(bsteps[0]) / (bms * 1e-3), "steps": int(bsteps[0]),
                         "ms": bms}
        bs.close()
        extra["persistent_1d_kernel"] = dict(pk, note="cumc_batch_run with this one problem (INITIAL_UPDATE "
                                                      "included); results bit-identical for both shapes")
        if not args.no_cpu:
            cpu = cpu_baseline_of(lambda: models.brio_wu(800, recon=spec["recon"], riemann=spec["riemann"]), 100,
                                  "CPU oracle, Brio-Wu 800 zones, 100 RK3 steps")
    elif args.workload == "alfven3d":
        n3 = args.n
        recon = args.recon_c or "ppm"
        spec, prim, eps = models.alfven_3d(n3, recon=recon, riemann=args.riemann)
        zones = n3 ** 3
        out = {}
        forms = [("fp64", dict(spec, precision="fp64"), None), ("fp32", dict(spec, precision="fp32"), None)]
        lp = args.learned_params
        if recon == "weno" and lp and os.path.exists(lp):
            P = np.load(lp)

            def setup(s, P=P):
                s.learn_set(P, threshold=args.learn_threshold, audit_interval=args.audit_interval, audit_tol=1e-5,
                            flag_interval=args.flag_interval)
            forms.append(("fp32+learned", dict(spec, precision="fp32", learned=1), setup))
            forms.append(("fp64+learned", dict(spec, precision="fp64", learned=1), setup))
        clocks.start()
        for name_f, sp, setup in forms:
            s, k, t_ms = _evolve_timed(engine, torch, sp, prim, eps, args.warmup, t_end=spec["t_end"], setup=setup)
            out[name_f] = dict(cons=s.get_array(capi.ARR_CONS), divb=s.find_divb(), steps=k, ms=t_ms, t=s.time)
            if setup is not None:
                out[name_f]["stats"] = s.learn_stats()
            s.close()
        clk = clocks.stop()
        # the exact solution after one period is the initial state
        s0 = engine.Solver(spec)
        s0.set_state(prim, eps)
        s0.initial_update()
        c0 = s0.get_array(capi.ARR_CONS)
        s0.close()
        sl = (slice(3, n3 + 3),) * 3

        def rel_l1(a, b):
            a, b = a[sl].reshape(-1, 8), b[sl].reshape(-1, 8)
            den = np.abs(b).sum(axis=0)
            return (np.abs(a - b).sum(axis=0) / np.where(den == 0, 1, den)).tolist()
        l1_32 = rel_l1(out["fp32"]["cons"], out["fp64"]["cons"])
        extra.update({
            "l1_fp32_vs_fp64_per_var": l1_32, "l1_fp32_vs_fp64_max": max(l1_32),
            "l1_fp64_vs_exact_per_var": rel_l1(out["fp64"]["cons"], c0),
            "max_divb": {p: out[p]["divb"] for p in out},
            "fp32_zone_updates_per_s": zones * out["fp32"]["steps"] / (out["fp32"]["ms"] * 1e-3),
            "fp64_zone_updates_per_s": zones * out["fp64"]["steps"] / (out["fp64"]["ms"] * 1e-3),
            "period": spec["t_end"], "time_reached": {p: out[p]["t"] for p in out},
        })
        extra["fp32_over_fp64"] = extra["fp32_zone_updates_per_s"] / extra["fp64_zone_updates_per_s"]
        if not args.no_cpu:
            cpu = cpu_baseline_of(lambda: models.alfven_3d(128, recon=recon, riemann=args.riemann), 2,
                                  "CPU oracle, the same wave on a 128^3 grid, 2 RK3 steps")
        if "fp32+learned" in out:
            o = out["fp32+learned"]
            l1_l = rel_l1(o["cons"], out["fp64"]["cons"])
            st = o["stats"]
            extra.update({
                "l1_learned_vs_fp64_per_var": l1_l, "l1_learned_vs_fp64_max": max(l1_l),
                "l1_learned_vs_exact_per_var": rel_l1(o["cons"], c0),
                "learned_zone_updates_per_s": zones * o["steps"] / (o["ms"] * 1e-3),
                "learned_flagged_fraction_at_audits": st["flagged"] / max(1, st["audited"]),
                "learned_fallback_tiles": st["fallback_tiles"], "learned_audits": st["audits"],
                "learned_params": os.path.relpath(lp, ROOT),
                "learned_flag_interval": args.flag_interval, "learned_audit_interval": args.audit_interval,
                "learned_threshold": args.learn_threshold,
            })
            extra["learned_over_fp64"] = extra["learned_zone_updates_per_s"] / extra["fp64_zone_updates_per_s"]
            o64 = out["fp64+learned"]
            l1_64 = rel_l1(o64["cons"], out["fp64"]["cons"])
            extra.update({
                "fp64_learned_zone_updates_per_s": zones * o64["steps"] / (o64["ms"] * 1e-3),
                "l1_fp64_learned_vs_fp64_max": max(l1_64),
                "fp64_learned_flagged_fraction_at_audits": o64["stats"]["flagged"] / max(1, o64["stats"]["audited"]),
            })
            extra["fp64_learned_over_fp64"] = extra["fp64_learned_zone_updates_per_s"] / extra["fp64_zone_updates_per_s"]
        key = args.precision
        n, ms = out[key]["steps"], out[key]["ms"]
        name = "alfven3d_%d^3_%s_%s_cfl0.4_one_period" % (n3, recon, args.riemann)
    elif args.workload == "torus_sph":
        # the spherical torus on the refined grid its model reads (124 x 44 x
        # 128), PPM + HLLD at CFL 0.8 as the reference ships them, FP64 and FP32
        recon = args.recon_c or "ppm"
        spec, prim, eps = models.torus_sph(recon=recon, riemann=args.riemann)
        spec["positivity_fallback"] = 1 if recon == "weno" else 0
        # periodic phi: as for the cylindrical torus, the face-0 option keeps
        # the wound-up B_phi divergence-free at the seam
        spec["fix_periodic_normal_faces"] = 1
        zones = spec["nx"] * spec["ny"] * spec["nz"]
        out = {}
        clocks.start()
        for name_f, sp in (("fp64", dict(spec)), ("fp32", dict(spec, precision="fp32"))):
            s, k, t_ms = _evolve_timed(engine, torch, sp, prim, eps, args.warmup, steps=args.steps)
            out[name_f] = dict(cons=s.get_array(capi.ARR_CONS), divb=s.find_divb(), steps=k, ms=t_ms, t=s.time)
            s.close()
        clk = clocks.stop()
        sl = (slice(3, spec["nz"] + 3), slice(3, spec["ny"] + 3), slice(3, spec["nx"] + 3))
        a, b = out["fp32"]["cons"][sl].reshape(-1, 8), out["fp64"]["cons"][sl].reshape(-1, 8)
        den = np.abs(b).sum(axis=0)
        l1 = (np.abs(a - b).sum(axis=0) / np.where(den == 0, 1, den)).tolist()
        extra.update({"l1_fp32_vs_fp64_per_var": l1, "l1_fp32_vs_fp64_max": max(l1),
                      "max_divb": {f: out[f]["divb"] for f in out}, "time_reached": {f: out[f]["t"] for f in out},
                      "orbital_period": spec["t_orbit"]})
        for f in out:
            extra["%s_zone_updates_per_s" % f] = zones * out[f]["steps"] / (out[f]["ms"] * 1e-3)
        n, ms = out[args.precision]["steps"], out[args.precision]["ms"]
        name = "torus_sph_%dx%dx%d_%s_%s_ct_cfl0.8" % (spec["nx"], spec["ny"], spec["nz"], recon, args.riemann)
        if not args.no_cpu:
            cpu = cpu_baseline_of(lambda: models.torus_sph(recon=recon, riemann=args.riemann), 2,
                                  "CPU oracle, the same torus and grid, 2 RK3 steps")
    else:  # torus
        recon = args.recon_c or "weno"
        spec, prim, eps = models.torus_cyl(recon=recon, riemann=args.riemann, precision="fp64")
        spec["positivity_fallback"] = 1
        # phi is periodic: with the reference's frozen lower face the wound-up
        # B_phi of face n never reaches face 0, so div B is kept at roundoff
        # with the face-0 option (as for the blast)
        spec["fix_periodic_normal_faces"] = 1
        zones = spec["nx"] * spec["ny"] * spec["nz"]
        forms = [("fp64", dict(spec), None), ("fp32", dict(spec, precision="fp32"), None)]
        lp = args.learned_params
        if recon == "weno" and lp and os.path.exists(lp):
            P = np.load(lp)

            def setup(s, P=P):
                s.learn_set(P, threshold=args.learn_threshold, audit_interval=args.audit_interval, audit_tol=1e-5,
                            flag_interval=args.flag_interval)
            forms.append(("fp32+learned", dict(spec, precision="fp32", learned=1), setup))
        out = {}
        clocks.start()
        for name_f, sp, setup in forms:
            s, k, t_ms = _evolve_timed(engine, torch, sp, prim, eps, args.warmup, steps=args.steps, setup=setup)
            out[name_f] = dict(cons=s.get_array(capi.ARR_CONS), divb=s.find_divb(), steps=k, ms=t_ms, t=s.time,
                               stats=s.learn_stats() if setup is not None else None)
            s.close()
        clk = clocks.stop()
        sl = (slice(3, spec["nz"] + 3), slice(3, spec["ny"] + 3), slice(3, spec["nx"] + 3))

        def rel_l1(a, b):
            a, b = a[sl].reshape(-1, 8), b[sl].reshape(-1, 8)
            den = np.abs(b).sum(axis=0)
            return (np.abs(a - b).sum(axis=0) / np.where(den == 0, 1, den)).tolist()
        extra["max_divb"] = {f: out[f]["divb"] for f in out}
        extra["time_reached"] = {f: out[f]["t"] for f in out}
        for f in out:
            extra["%s_zone_updates_per_s" % f] = zones * out[f]["steps"] / (out[f]["ms"] * 1e-3)
            if f != "fp64":
                extra["l1_%s_vs_fp64_max" % f] = max(rel_l1(out[f]["cons"], out["fp64"]["cons"]))
        if "fp32+learned" in out:
            st = out["fp32+learned"]["stats"]
            extra["learned_flagged_fraction_at_audits"] = st["flagged"] / max(1, st["audited"])
            extra["learned_settings"] = {"flag_interval": args.flag_interval, "audit_interval": args.audit_interval,
                                         "threshold": args.learn_threshold, "audit_tol": 1e-5}
        key = args.precision if args.precision in out else "fp64"
        n, ms = out[key]["steps"], out[key]["ms"]
        name = "torus_cyl_192x128x192_%s_%s_ct_cfl0.4" % (recon, args.riemann)
        if not args.no_cpu:
            cpu = cpu_baseline_of(lambda: models.torus_cyl(nr=96, nphi=64, nz=96, recon=recon, riemann=args.riemann),
                                  2, "CPU oracle, the same torus on a 96x64x96 grid, 2 RK3 steps")
    value = zones * n / (ms * 1e-3)
    if rank == 0:
        line = {"metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
                "steps": n, "warmup": args.warmup, "ms_per_step": ms / max(n, 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
                "config": {"workload": name, "precision": args.precision}, "results": extra,
                "e2e": None, "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 200 RK3 steps of the blast; 5 whole runs of the batch)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="blast3d",
                    choices=["blast3d", "batch1d", "briowu", "alfven3d", "torus", "torus_sph", "poisson", "collapsar",
                             "snapshots",
                             "slabs"])
    ap.add_argument("--slabs", type=int, default=2, help="slabs: number of z slabs")
    ap.add_argument("--snapshot-every", type=int, default=10, help="snapshots: steps between two snapshots")
    ap.add_argument("--sor-grid", default="384,192,192", help="poisson: nr,ntheta,nphi of the star")
    ap.add_argument("--sor-iters", type=int, default=100, help="poisson: SOR iterations per step")
    ap.add_argument("--sor-full", type=int, default=1, help="poisson: also time the full solve from phi = 0 (0: skip)")
    ap.add_argument("--recon-c", default=None, help="reconstruction of the briowu/alfven3d/torus workloads")
    ap.add_argument("--batch-problems", type=int, default=512,
                    help="batch1d: run only the first N problems (profiler runs); the workload is 512")
    ap.add_argument("--learned-params", default=os.path.join(ROOT, "cumc3d_b200", "data", "flag_mlp.npy"),
                    help="trained flag network for the FP32+learned form of the alfven3d workload")
    ap.add_argument("--flag-interval", type=int, default=8,
                    help="learned forms: the flag network runs every this many steps")
    ap.add_argument("--audit-interval", type=int, default=24,
                    help="learned forms: full-WENO audit every this many steps (a multiple of --flag-interval)")
    ap.add_argument("--learn-threshold", type=float, default=-4.0,
                    help="learned forms: a cell is flagged smooth when the network's logit exceeds this; below 0 "
                         "also flags the borderline cells, whose scatter would otherwise keep whole warps on "
                         "WENO-Z (the audits bound the error)")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--recon", default="weno")
    ap.add_argument("--riemann", default="hlld")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--concurrent-sweeps", type=int, default=0,
                    help="1: each stage's three flux sweeps as concurrent graph branches (same bits)")
    ap.add_argument("--tuning", default="auto",
                    help="'auto' (the engine's autotuner) or split,tpb_recon,tpb_riemann,min_blocks[,recon_tile] "
                         "(pinned launch shape, e.g. for profiler runs where timing is distorted)")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: independent copies of the workload per rank instead of z slabs of one grid")
    ap.add_argument("--parity-sample", type=int, default=1,
                    help="1: check the engine bit for bit against the CPU oracle on the CPU baseline's slab")
    ap.add_argument("--precision-forms", type=int, default=1,
                    help="1: also time the FP64 / FP32 / FP32+learned forms on the 256^3 CP Alfven wave")
    ap.add_argument("--dry-run", action="store_true",
                    help="set up the ranks and the process group (gloo) and print the line's layout; no kernels")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"blast3d": 200, "batch1d": 5, "torus": 2000, "torus_sph": 1000, "poisson": 20, "snapshots": 60,
                      "slabs": 30, "collapsar": 200}.get(args.workload, 0)
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return self_spawn(args.gpus)
    if args.impl == "reference":
        return reference_arm(args)

    world, rank, local, dist = dist_setup(args)
    if args.dry_run:
        return dry_run(args, world, rank, dist)
    import torch

    from cumc3d_b200 import engine
    torch.cuda.set_device(local)
    engine.load_library()
    if args.workload == "batch1d":
        return bench_batch(args, world, rank, local, dist)
    if args.workload in ("briowu", "alfven3d", "torus", "torus_sph"):
        return bench_config(args, world, rank, local, dist)
    if args.workload == "poisson":
        return bench_poisson(args, world, rank, local, dist)
    if args.workload == "collapsar":
        return bench_collapsar(args, world, rank, local, dist)
    if args.workload == "snapshots":
        return bench_snapshots(args, world, rank, local, dist)
    if args.workload == "slabs":
        return bench_slabs(args, world, rank, local, dist)
    if world > 1 and not args.replicas:
        return bench_slab_ranks(args, world, rank, local, dist)
    return bench_blast(args, world, rank, local, dist)


def parallelism_of(args, world):
    if world == 1:
        return "single"
    if args.workload in ("blast3d", "slabs") and not args.replicas:
        return "z-slabs x %d (one per rank, NCCL send/recv of ghost planes, all-reduce min of dt)" % world
    if args.workload == "batch1d":
        return "problems sharded over %d ranks" % world
    return "replicas"


def dry_run(args, world, rank, dist):
    """The launch layout without a GPU: ranks, process group, parallelism."""
    info = ranks_info(dist)
    if dist:
        dist.barrier()
    if rank == 0:
        print(json.dumps({"metric": "zone-updates/s", "value": None, "unit": "zone-updates/s", "n_gpus": world,
                          "dry_run": True, "ranks": info,
                          "config": {"workload": blast_workload(args.n, args.recon, args.riemann),
                                     "parallelism": parallelism_of(args, world)},
                          "scaling": "strong" if world > 1 and not args.replicas else "weak"}))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def flux_roofline(args, prof, profile_steps, zones, tuning, fp64_peak):
    """Roofline of the dominant kernel class (a flux sweep on the FP64 path):
    bytes = 120 B/zone (the fused pass minimum), flops = the oracle's exact
    count per zone of a sweep; achieved = flops / launch time against the
    measured DFMA peak; frac = max(bytes / BW, flops / FP64 peak) / time, the
    FP64 roofline of the scope table; the HBM side and the measured traffic
    (ncu, profiles/traffic.json) alongside."""
    per_stage = {k: v for k, v in prof.items() if k != "dt"}
    dominant = max(per_stage, key=per_stage.get)
    avg_ms = prof[dominant] / (profile_steps * 3)
    peak_gbs, peak_kind = load_peaks()
    if dominant.startswith("flux"):
        bytes_launch = FLUX_BYTES_PER_ZONE * zones
        if tuning.get("split", True):
            kname = "%s + k_riemann, %s sweep (%s, %s)" % ("k_recon_tile" if tuning.get("recon_tile") else "k_recon",
                                                           dominant[-1], args.recon, args.riemann)
        else:
            kname = "k_flux<%s,%s,%s>" % (dominant[-1], args.recon, args.riemann)
    else:
        bytes_launch = None
        kname = dominant
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tdat = json.load(f)
        key = "%s/%s/%s/%s" % (dominant, args.recon, args.riemann, args.precision)
        if key in tdat:
            traffic = tdat[key]["bytes_per_zone"] * zones
    gbs = (bytes_launch / (avg_ms * 1e-3) / 1e9) if bytes_launch else None
    hbm = {"achieved": gbs, "peak": peak_gbs, "unit": "GB/s", "frac": (gbs / peak_gbs) if gbs else None,
           "bytes_per_launch": bytes_launch, "peak_source": "MEASURED_PEAKS.json hbm_gbs (%s)" % peak_kind,
           "traffic_over_algorithmic": (traffic / bytes_launch) if traffic and bytes_launch else None}
    ops = None
    okey = "blast3d_%s_%s" % (args.recon, args.riemann)
    opath = os.path.join(ROOT, "profiles", "op_counts.json")
    if args.precision == "fp64" and os.path.exists(opath):
        with open(opath) as f:
            ops = json.load(f).get(okey)
    roof = {"kernel": kname, "avg_launch_ms": avg_ms, "traffic": traffic, "hbm": hbm,
            "class_ms_per_step": {k: v / profile_steps for k, v in prof.items()}}
    if ops is not None and fp64_peak and dominant.startswith("flux"):
        fl = ops["flux_sweep_flops_per_zone"] * zones
        tf = fl / (avg_ms * 1e-3) / 1e12
        t_bound = max(bytes_launch / (peak_gbs * 1e9), fl / (fp64_peak * 1e12))
        roof.update({"bound": "fp64", "achieved": tf, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": t_bound / (avg_ms * 1e-3), "flops_per_launch": fl,
                     "peak_source": "cumc_fp64_peak (DFMA loop, measured in this run)",
                     "counts": "profiles/op_counts.json %s: flux_sweep_flops_per_zone (add, mul, div, sqrt one "
                               "flop each; a division or square root is several FP64 instructions)" % okey})
    else:
        roof.update({"bound": "hbm", "achieved": gbs, "peak": peak_gbs, "unit": "GB/s", "frac": hbm["frac"]})
    fpath = os.path.join(ROOT, "profiles", "fp64_pipe.json")
    if os.path.exists(fpath) and args.precision == "fp64":
        with open(fpath) as f:
            pipe = json.load(f).get("%s/%s/fp64" % (args.recon, args.riemann))
        if pipe is not None:
            roof["fp64_pipe_frac_ncu"] = pipe
    return roof, ops, peak_gbs


def parity_sample_check(args, kept, tuning):
    """The engine on the CPU baseline's slab, the same steps through the same
    captured step graph as the timed run, compared bit for bit with the
    oracle's state (prim incl. face B, epsilon, cell B, sound speed on the
    interior; the time reached)."""
    import numpy as np

    from cumc3d_b200 import capi, engine
    spec = kept["spec"]
    prim, eps = kept["init"]
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    # the launch shapes the timed run was tuned to
    s.set_tuning(tuning["split"], tuning["tpb_recon"], tuning["tpb_riemann"], tuning["riemann_min_blocks"],
                 tuning["recon_tile"])
    s.fallback_count(1)
    t, k = s.evolve(1e30, 2)
    p, e = s.get_state()
    got = dict(prim=p, eps=e, bcell=s.get_array(capi.ARR_BCELL), cs=s.get_array(capi.ARR_CS))
    fb = s.fallback_count()
    s.close()
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    sl = (slice(3, nz + 3), slice(3, ny + 3), slice(3, nx + 3))
    mism = {}
    for key in ("prim", "eps", "bcell", "cs"):
        a, b = got[key][sl], kept[key][sl]
        mism[key] = int(np.count_nonzero(~((a == b) | (np.isnan(a) & np.isnan(b)))))
    ok = all(v == 0 for v in mism.values()) and t == kept["t"] and fb == kept["fallback"]
    return {"bitwise": bool(ok), "cells": nx * ny * nz, "grid": [nx, ny, nz], "steps": k,
            "time_equal": t == kept["t"], "mismatched_values": mism,
            "fallback_cells_gpu": fb, "fallback_cells_oracle": kept["fallback"],
            "what": "prim (incl. face B), epsilon, cell B, c_s on the interior after 2 RK3 steps of the "
                    "captured step graph, the tuned launch shapes of the timed run"}


def precision_forms(args, learned_params):
    """The precision forms on the CP Alfven wave at 256^3 (WENO-Z + HLLD + CT,
    CFL 0.4): plain FP64, FP32 bulk, FP32 bulk + learned smooth-face flag
    (the bench's flag settings), each from the same initial state: 8 warm-up
    steps, then 24 timed steps (one audit cycle) with CUDA events on the
    engine stream; relative L1 per conserved variable of each form against
    the FP64 form after those 32 steps."""
    import numpy as np
    import torch

    from cumc3d_b200 import capi, engine, models
    from cumc3d_b200.accuracy import rel_l1
    n, warm, steps = 256, 8, 24
    spec, prim, eps = models.alfven_3d(n, recon="weno")
    forms = [("fp64", dict(spec, precision="fp64"), None), ("fp32", dict(spec, precision="fp32"), None)]
    if learned_params and os.path.exists(learned_params):
        P = np.load(learned_params)

        def setup(s, P=P):
            s.learn_set(P, threshold=args.learn_threshold, audit_interval=args.audit_interval, audit_tol=1e-5,
                        flag_interval=args.flag_interval)
        forms.append(("fp32+learned", dict(spec, precision="fp32", learned=1), setup))
    out, cons = {}, {}
    for name, sp, setup in forms:
        s = engine.Solver(sp)
        s.set_state(prim, eps)
        s.initial_update()
        if setup is not None:
            setup(s)
        s.autotune()
        s.evolve(1e30, warm)
        s.sync()
        stream = torch.cuda.ExternalStream(s.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        _, k = s.evolve(1e30, steps)
        e1.record(stream)
        s.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        cons[name] = s.get_array(capi.ARR_CONS)[3:n + 3, 3:n + 3, 3:n + 3]
        out[name] = {"zone_updates_per_s": n ** 3 / (ms * 1e-3), "ms_per_step": ms}
        if setup is not None:
            st = s.learn_stats()
            out[name]["flagged_fraction_at_audits"] = st["flagged"] / max(1, st["audited"])
        s.close()
    for name in out:
        if name != "fp64":
            l1 = rel_l1(cons[name], cons["fp64"])
            out[name]["l1_vs_fp64_max"] = float(l1.max())
            out[name]["l1_vs_fp64_per_var"] = l1.tolist()
            out[name]["speedup_vs_fp64"] = out[name]["zone_updates_per_s"] / out["fp64"]["zone_updates_per_s"]
    out["workload"] = "alfven3d_256^3_weno_hlld_ct_cfl0.4, %d warm-up + %d timed steps per form" % (warm, steps)
    return out


def bench_blast(args, world, rank, local, dist):
    """The headline workload on one GPU (or N replicas with --replicas)."""
    import numpy as np
    import torch

    from cumc3d_b200 import engine, models
    n = args.n
    spec, prim, eps = models.blast_3d(n, recon=args.recon, riemann=args.riemann, precision=args.precision)
    # the reference's WENO-Z + HLLD produces negative face pressure on this
    # blast within a few steps; both flags are mirrored by the CPU oracle
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    zones = spec["nx"] * spec["ny"] * spec["nz"]
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    if args.tuning == "auto":
        tuning = s.autotune()
    else:
        vals = [int(v) for v in args.tuning.split(",")] + [0]
        sp, tr, tm, mb, rt = vals[:5]
        s.set_tuning(bool(sp), tr, tm, mb, rt)
        tuning = dict(split=bool(sp), tpb_recon=tr, tpb_riemann=tm, riemann_min_blocks=mb, recon_tile=rt,
                      pinned=True)
    if args.concurrent_sweeps:
        s.set_concurrent_sweeps(True)
    tuning["concurrent_sweeps"] = bool(args.concurrent_sweeps)
    s.evolve(1e30, args.warmup)
    s.sync()
    stream = torch.cuda.ExternalStream(s.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = s.launch_count()
    e0.record(stream)
    _, nsteps = s.evolve(1e30, args.steps)
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = s.launch_count() - l0
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * zones * nsteps / (ms * 1e-3)

    # per-kernel-class timing (CUDA events on the engine stream, eager launches)
    prof = s.profile_step(args.profile_steps)
    try:
        fp64_peak = engine.fp64_peak_tflops()
    except Exception:
        fp64_peak = None
    roofline, ops, peak_gbs = flux_roofline(args, prof, args.profile_steps, zones, tuning, fp64_peak)
    step_gbs = STEP_BYTES_PER_ZONE * value / world / 1e9
    step_fp64 = None
    if ops is not None and fp64_peak:
        tf = ops["flops_per_zone_update"] * value / world / 1e12
        step_fp64 = {"flops_per_zone_update": ops["flops_per_zone_update"], "achieved_tflops": tf,
                     "frac": tf / fp64_peak}

    # end to end through the C-ABI with pinned host buffers; the same handle
    # counts the cells that took the positivity fallback
    e2e, fallback = None, None
    if not args.no_e2e:
        hp = torch.from_numpy(prim).pin_memory()
        he = torch.from_numpy(eps).pin_memory()
        out_p = torch.empty_like(hp).pin_memory()
        out_e = torch.empty_like(he).pin_memory()
        s2 = engine.Solver(spec)
        s2.set_state(prim, eps)  # untimed: the tuner needs a live state
        s2.initial_update()
        if args.tuning == "auto":
            s2.autotune()
        else:
            s2.set_tuning(tuning["split"], tuning["tpb_recon"], tuning["tpb_riemann"], tuning["riemann_min_blocks"],
                          tuning["recon_tile"])
        if args.concurrent_sweeps:
            s2.set_concurrent_sweeps(True)
        s2.fallback_count(1)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2.set_state_ptr(hp.data_ptr(), he.data_ptr())
        s2.initial_update()
        _, n2 = s2.evolve(1e30, args.steps)
        s2.get_state_ptr(out_p.data_ptr(), out_e.data_ptr())
        s2.sync()
        el = time.perf_counter() - t0
        if dist:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        fb = s2.fallback_count()
        s2.close()
        nbytes_in = hp.numel() * 8 + he.numel() * 8
        e2e = {"value": world * zones * n2 / el, "unit": "zone-updates/s",
               "h2d_bytes_per_step": nbytes_in / max(n2, 1), "d2h_bytes_per_step": nbytes_in / max(n2, 1),
               "wall_s": el, "steps": n2,
               "note": "state upload and result download once per run of %d steps, amortised per step" % n2}
        fallback = {"cells_per_step": fb / max(n2, 1), "steps": n2,
                    "fraction_of_reconstructions": fb / max(1, n2 * 9 * zones),
                    "what": "cells whose reconstruction took the first-order positivity fallback, per RK3 step "
                            "(3 stages x 3 sweeps reconstruct every zone 9 times a step), from t = 0"}

    forms = None
    if rank == 0 and world == 1 and args.precision_forms:
        forms = precision_forms(args, args.learned_params)

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        nz_slab = 64
        cpu, kept = cpu_baseline_of(lambda: blast_slab(n, nz_slab, args.recon, args.riemann), 2,
                                    "CPU oracle, %dx%dx%d periodic slab of the blast, 2 RK3 steps" % (n, n, nz_slab),
                                    keep=True)
        if kept is not None and args.parity_sample and args.precision == "fp64":
            parity = parity_sample_check(args, kept, tuning)

    s.close()
    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
            "steps": nsteps, "warmup": args.warmup, "ms_per_step": ms / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": blast_workload(n, args.recon, args.riemann),
                       "grid": [n, n, n], "recon": args.recon, "riemann": args.riemann,
                       "precision": args.precision, "boundary": "periodic", "steps_in_workload": 200,
                       "positivity_fallback": 1, "fix_periodic_normal_faces": 1,
                       "l2": "state 7 GB resident in HBM, >> 126 MB L2 (no flush needed)",
                       "parallelism": parallelism_of(args, world), "autotuned": tuning},
            "roofline": roofline,
            "step_hbm": {"bytes_per_zone_update": STEP_BYTES_PER_ZONE, "achieved_gbs": step_gbs,
                         "frac": step_gbs / peak_gbs},
            "step_fp64": step_fp64,
            "fp64_peak_tflops_measured": fp64_peak,
            "parity_sample": parity,
            "precision_forms": forms,
            "positivity_fallback": fallback,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "ranks": ranks_info(dist),
            "clocks": clk,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
