#!/usr/bin/env python
"""Throughput of the full PUFFY GR-RMHD + M1 RK2IMEX step (koral/sim.zig:1792
Sim.step) on the sm_100a engine, in zone-cycles/s (active cells x steps per
second, the reference's `znps`, koral/problems/puffy/main.zig:99).

Workload: the 3D wedge 192x180x64 MKS2 (periodic phi over +-pi/4, 3 ghost
zones, NV=13), the PUFFY torus from the engine's own init with seeded 1e-3
relative perturbations of u_int and rho, plain FP64. The state, metric cache
and stage buffers (several GB) are far larger than the 126 MB L2, so no flush
is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl koral|reference]

Under torchrun each rank runs an independent replica on its own GPU (the
path does not shard in this tier); `value` is the whole job's zone-cycles
over the slowest rank's device time. `--impl reference` times the CPU
restatement of the same step (the oracle; the reference's Zig toolchain is
not available) on all host cores, rank 0 only.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "zone-cycles/s (full GR-RMHD+M1 step)"
UNIT = "zone-cycles/s"
SAMPLE_NZ = 4  # phi cells of the CPU sample: same 192x180 meridional grid, 4 of the 64 phi cells

# Algorithmic HBM bytes per cell and launch of each step pass (FP64, SoA, the
# packed metric cache: center gcov10+gdet 11 f64, gcon16+gttpert 17 f64,
# Christoffels 40 f64, BL geometry 28 f64; face metric 11+17 f64 per face).
# Every cell's data counted once per launch; ghost/face overhangs ignored.
B = 8
PASS_BYTES_PER_CELL = {
    # p, u in; p, u out; center metric 28; radimp flag
    "implicit": (13 + 13 + 28 + 13 + 13) * B + 4,
    # per active dim: p in, face metric 28, wavespeeds 6, rijvisc 16; flb out 13
    "fluxes": None,  # dims-dependent, filled in by pass_bytes()
    # u, p in; center metric 28; p out (5 MHD + 4 rad + ENTR), 6 flags out
    "u2p": (13 + 13 + 28 + 13) * B + 6 * 4,
    # flb in (13 per face and dim), u in/out, metric 28, Christoffels 40
    "update": None,
    # p, center metric 28, BL geometry 28, wavespeeds 6 + cell dt 2 out
    "wavespeeds": (13 + 28 + 28 + 8) * B,
    # p in, rijvisc 16 out, metric 28, BL radius
    "radvisc": (13 + 28 + 16 + 1) * B,
}


def pass_bytes(name, ndim):
    if name == "fluxes":
        return ndim * (13 + 28 + 6 + 16 + 13) * B
    if name == "update":
        return (ndim * 13 + 13 + 13 + 28 + 40) * B
    return PASS_BYTES_PER_CELL.get(name)


def max_over_ranks(ms, dist, device):
    """The slowest rank's device time (every rank calls this, in the same order)."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(cells_per_rank, steps, world, ms_max):
    """Whole-job zone-cycles/s of `world` replicas: all ranks' cells x steps over
    the slowest rank's time."""
    return cells_per_rank * steps * world / (ms_max / 1e3)


def load_engine():
    spec = importlib.util.spec_from_file_location("koralcuda", os.path.join(ROOT, "koral-zig_b200", "koralcuda.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.lib()
    return mod


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0}, "fallback"


def profiled_figure(kernel, key):
    """A per-cell figure (`key`: dram_bytes_per_cell, fp64_flop_per_solve) of
    `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_traffic.txt")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def profiled_traffic(kernel):
    """dram bytes per cell of `kernel` from the committed ncu summary, or None."""
    return profiled_figure(kernel, "dram_bytes_per_cell")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while alive."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ident = vis.split(",")[device] if vis else str(device)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", ident, "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        for line in self.out.read().splitlines():
            cols = [c.strip() for c in line.split(",")]
            if len(cols) < 9:
                continue
            try:
                sm.append(float(cols[1]))
                smax.append(float(cols[2]))
            except ValueError:
                continue
            for name, v in zip(self.REASONS, cols[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.out.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def oracle_rate(nx, ny, nz, steps, warmup, threads, min_seconds=0.0):
    """zone-cycles/s of the CPU restatement (oracle/orc_sim.cpp) on a
    nx x ny x nz PUFFY wedge, after its own init and `warmup` steps."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    sys.path.insert(0, ROOT)
    from tests.orcsim import OracleSim, puffy_grid, puffy_options

    sim = OracleSim(puffy_grid(nx, ny, nz), puffy_options(), nthreads=threads)
    sim.init_puffy(1e-3, 1e-3, 1)
    sim.lib.orc_sim_init_timestep_guess(sim.h)
    for _ in range(warmup):
        sim.step()
    n, t = 0, 0.0
    while n < steps or t < min_seconds:
        t0 = time.perf_counter()
        sim.step()
        t += time.perf_counter() - t0
        n += 1
    sim.close()
    return nx * ny * nz * n / t, n, t


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    nz = SAMPLE_NZ
    rate, n, t = oracle_rate(args.nx, args.ny, nz, args.steps, args.warmup, threads)
    sample = (f"{args.nx}x{args.ny}x{nz} of the {args.nx}x{args.ny}x{args.nz} wedge (same meridional grid, "
              f"{nz} phi cells), {n} steps after {args.warmup} warm-up, oracle/orc_sim.cpp on {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (PUFFY torus init + seeded 1e-3 rho/u_int noise)",
        "config": {"workload": f"PUFFY 3D wedge {args.nx}x{args.ny}x{args.nz} MKS2, plain FP64, CPU sample"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


IMPLICIT_MODES = {"per-cell": 0, "compacting": 1, "split": 2, "sorted": 3, "rungs": 4, "iters": 5}


def batch_launches(opt, mode):
    """The engine's own kernel launches in one kc_implicit_batch call (the radix
    sort of the sorted forms runs CUB's kernels, not counted): the key kernel,
    the preparation and one launch per rung, or per rung and round of at most
    8 Newton iterations (the schedule of launch_iters in kc_abi_batch.inc)."""
    nrung = 6 * (opt.radimp_opdamp_maxlevels + 1)
    if mode in (0, 1):
        return 1
    if mode == 3:
        return 2
    if mode == 4:
        return 2 + nrung
    return 2 + nrung * (-(-(opt.radimp_maxiter + 1) // 8))
IMPL_METRIC = "implicit M1 solves/s (batched, independent cells)"
IMPL_UNIT = "solves/s"


def oracle_implicit_rate(geom, dt, pp, threads, min_seconds=10.0):
    """solves/s of the oracle's solveImplicitLab loop on host threads over the
    given cells, repeated until min_seconds of work (a bounded sample)."""
    import ctypes

    import numpy as np

    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.orc_implicit_batch_mt.argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
    n = len(dt)
    done, t = 0, 0.0
    while t < min_seconds:
        p = np.array(pp, copy=True)
        res = np.zeros((n, 3), dtype=np.int32)
        t0 = time.perf_counter()
        lib.orc_implicit_batch_mt(n, geom.ctypes.data, dt.ctypes.data, p.ctypes.data, res.ctypes.data, threads)
        t += time.perf_counter() - t0
        done += n
    return done / t, done, t


def implicit_battery(kc, opt, stream, rounds=30):
    """The reference's own implicit battery (koral tools/bench_implicit.zig:96-221):
    the 336 rad_implicit golden records (tests/golden, converted from the
    reference's rad_implicit.kgld), timed in ns/solve as that tool times them,
    on the GPU (the 336 cells per launch, and the battery replicated to 2^20
    cells so that it fills the device) and on the oracle port (one host thread,
    and all host threads with a dynamic ticket)."""
    import ctypes

    import numpy as np
    import torch

    z = np.load(os.path.join(ROOT, "tests", "golden", "rad__rad_implicit.npz"))
    d = np.ascontiguousarray(z["data"])
    geom, dt, pp = d[:, :23].copy(), d[:, 23].copy(), d[:, 24:37].copy()
    nrec = len(dt)
    out = {"records": nrec, "rounds": rounds}
    for label, reps in (("gpu_battery", 1), ("gpu_battery_x3121", 3121)):
        nround = rounds if reps == 1 else 3  # the replicated battery fills the device: 3 launches suffice
        g = torch.from_numpy(np.tile(geom, (reps, 1))).cuda()
        t = torch.from_numpy(np.tile(dt, reps)).cuda()
        p0 = torch.from_numpy(np.tile(pp, (reps, 1))).cuda()
        p = torch.empty_like(p0)
        r = torch.zeros((nrec * reps, 6), dtype=torch.int32, device="cuda")

        def go():
            p.copy_(p0)
            kc.implicit_batch_device(opt, nrec * reps, g.data_ptr(), t.data_ptr(), p.data_ptr(), r.data_ptr(),
                                     stream.cuda_stream, mode=0)

        go()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nround):
            go()
        e1.record(stream)
        torch.cuda.synchronize()
        out[label + "_ns_per_solve"] = e0.elapsed_time(e1) * 1e6 / (nround * nrec * reps)
        if reps == 1:
            out["converged"] = int((r[:, 0] == 1).sum().item())
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.orc_implicit_batch_mt.argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
    threads = os.cpu_count() or 1
    for label, th in (("oracle_1_thread", 1), (f"oracle_{threads}_threads", threads)):
        done, el = 0, 0.0
        while el < 2.0:
            q = pp.copy()
            res = np.zeros((nrec, 3), dtype=np.int32)
            t0 = time.perf_counter()
            lib.orc_implicit_batch_mt(nrec, geom.ctypes.data, dt.ctypes.data, q.ctypes.data, res.ctypes.data, th)
            el += time.perf_counter() - t0
            done += nrec
        out[label + "_ns_per_solve"] = el * 1e9 / done
    return out


def run_implicit(args, rank, world, local):
    """The batched implicit M1 solve over 2^22 independent seeded cells
    (kc_synth_implicit_cells), inputs resident in HBM, FP64."""
    import numpy as np

    kc = load_engine()
    opt = kc.puffy_options(device=local)
    n = args.cells
    geom, dt, pp = kc.synth_implicit_cells(opt, n, args.seed + rank)
    threads = os.cpu_count() or 1
    sample_n = min(n, 1 << 14)
    workload = f"{n} independent cells, seeded MKS2 states (kc_synth_implicit_cells), plain FP64"
    if args.impl == "reference":
        if rank != 0:
            return
        rate, done, t = oracle_implicit_rate(geom[:sample_n], dt[:sample_n], pp[:sample_n], threads)
        line = {"impl": "reference", "metric": IMPL_METRIC, "value": rate, "unit": IMPL_UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": {"workload": workload},
                "cpu_baseline": {"value": rate, "unit": IMPL_UNIT, "cores": threads, "kind": "port",
                                 "sample": f"first {sample_n} cells, {done} solves in {t:.1f} s"},
                "e2e": {"value": rate, "unit": IMPL_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch

    torch.cuda.set_device(local)
    dg = torch.from_numpy(geom).cuda()
    dd = torch.from_numpy(dt).cuda()
    dp0 = torch.from_numpy(pp).cuda()
    dp = torch.empty_like(dp0)
    dr = torch.zeros((n, 6), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def launch():
        dp.copy_(dp0)
        kc.implicit_batch_device(opt, n, dg.data_ptr(), dd.data_ptr(), dp.data_ptr(), dr.data_ptr(), stream.cuda_stream,
                                 mode=IMPLICIT_MODES[args.implicit_mode])

    for _ in range(args.warmup):
        launch()
    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    res = dr.cpu().numpy()
    ok = res[:, 0] == 1
    value = n * args.steps / (ms / 1e3)
    # end to end: host arrays through kc_implicit_batch (copies in and out inside)
    ke = max(1, min(3, args.steps))
    t0 = time.perf_counter()
    for _ in range(ke):
        kc.implicit_batch(opt, geom, dt, pp, mode=IMPLICIT_MODES[args.implicit_mode])
    te = time.perf_counter() - t0
    bpc = (23 + 1 + 13 + 13) * B + 6 * 4
    peaks, peak_kind = measured_peaks()
    achieved = bpc * n / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": IMPL_METRIC, "value": value, "unit": IMPL_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cells)",
        "config": {"workload": workload, "cells": n, "l2": "inputs larger than L2 (no flush)",
                   "implicit_mode": args.implicit_mode,
                   "converged": float(ok.mean()), "mean_iters": float(res[ok, 2].mean()),
                   "rungs": np.bincount(res[ok, 1], minlength=6).tolist()},
        "e2e": {"value": n * ke / te, "unit": IMPL_UNIT, "h2d_bytes_per_step": n * (23 + 1 + 13) * 8,
                "d2h_bytes_per_step": n * (13 * 8 + 24), "steps": ke, "timer": "host wall clock (synchronous API)"},
        "roofline": {"bound": "hbm", "kernel": "k_implicit_batch", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                     "algorithmic_bytes": bpc * n},
        "clocks": clk, "gpu_launches": args.steps * batch_launches(opt, IMPLICIT_MODES[args.implicit_mode]),
    }
    line["reference_battery"] = implicit_battery(kc, opt, stream)
    if rank == 0 and not args.no_cpu_baseline:
        rate, done, t = oracle_implicit_rate(geom[:sample_n], dt[:sample_n], pp[:sample_n], threads)
        line["cpu_baseline"] = {"value": rate, "unit": IMPL_UNIT, "cores": threads, "kind": "port",
                                "sample": f"first {sample_n} cells, {done} solves in {t:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)


PRIM_NAMES = ["rho", "uu", "vx", "vy", "vz", "entr", "b1", "b2", "b3", "ee", "fx", "fy", "fz"]
INTEGRATED = ("mass", "mdot", "radlum", "totallum", "scaleheight")


def measure_forms(kc, grid, local, steps, seed, graph):
    """The north-star forms on the benchmark's own wedge and init: plain FP64 and
    the mixed form (KC_MIXED), each from a fresh init, the mixed run forced to the
    plain run's dt sequence, timed with CUDA events on each engine's stream;
    returns ms per step of both, the mixed form's per-primitive field-scale error
    and the relative error of the integrated mass, accretion rate, luminosities
    and scale height (dump.scalarRow) after the steps."""
    import numpy as np
    import torch

    res, dts = {}, []
    # the learned guess of the combined form: pairs from one step of the same wedge
    src = kc.Sim(grid, kc.puffy_options(device=local))
    src.initPuffy(1e-3, 1e-3, seed)
    src.harvest_implicit(1000000)
    src.step()
    x, t = src.get_harvest(1000000)
    src.close()
    weights, _ = kc.mlp_train(x, t, steps=3000, batch=1024, lr=2e-3, seed=3)
    for form, mode, w in (("fp64", kc.KC_PLAIN_FP64, None), ("mixed", kc.KC_MIXED, None),
                          ("combined", kc.KC_MIXED, weights)):
        sim = kc.Sim(grid, kc.puffy_options(device=local, precision=mode))
        sim.initPuffy(1e-3, 1e-3, seed)
        if w is not None:
            sim.set_guess(w)
        sim.set_graph(graph)
        stream = torch.cuda.ExternalStream(sim.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(steps):
            if form == "fp64":
                dts.append(sim.step())
            else:
                sim.step(dts[k])
        e1.record(stream)
        torch.cuda.synchronize()
        res[form] = {"ms": e0.elapsed_time(e1) / steps, "p": sim.p, "scalars": sim.scalars(0.0, 5000.0, 15.0),
                     "t": sim.counters()["t"]}
        sim.close()
    b = res["fp64"]["p"]
    ok = np.all(np.isfinite(b), axis=1)
    out = {"steps": steps, "t": res["fp64"]["t"], "plain_fp64_ms_per_step": res["fp64"]["ms"]}
    for form in ("mixed", "combined"):
        a = res[form]["p"]
        dev = np.abs(a[ok] - b[ok]).max(axis=0) / np.maximum(np.abs(b[ok]).max(axis=0), 1e-300)
        out[form + "_ms_per_step"] = res[form]["ms"]
        out[form + "_speedup"] = res["fp64"]["ms"] / res[form]["ms"]
        out[form + "_field_scale_error"] = dict(zip(PRIM_NAMES, dev.tolist()))
        out[form + "_integrated_rel_error"] = {
            k: abs(res[form]["scalars"][k] / res["fp64"]["scalars"][k] - 1) for k in INTEGRATED}
    return {**out,
            "note": "mixed = FP32 LAXF dissipation and FP32 flux-CT corner averages, the rest FP64; "
                    "combined = mixed + the learned initial guess (network trained on the GPU on pairs "
                    "harvested from one step of the same wedge); same init and dt sequence as the plain run"}


def run_precision(args, rank, local):
    """Mixed forms (FP32 reconstruction, LAXF, flux-CT, or any set of those pieces
    and the rounded one-sided fluxes) against plain FP64 on the same wedge and
    init, each mixed run forced to the FP64 run's dt sequence:
    per-primitive field-scale error of the final state and the relative error of
    the integrated mass, accretion rate (horizon), luminosity and scale height."""
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    kc = load_engine()
    grid = kc.puffy_grid(args.nx, args.ny, args.nz)
    out = {}
    dts = []
    names = ["rho", "uu", "vx", "vy", "vz", "entr", "b1", "b2", "b3", "ee", "fx", "fy", "fz"]
    piece = {"all": kc.KC_MIXED, "ppm": kc.KC_FP32_PPM, "laxf": kc.KC_FP32_LAXF, "ct": kc.KC_FP32_CT,
             "flux": kc.KC_FP32_FLUX}
    variants = []
    for name in args.mixed_forms.split(","):
        mode = 0
        for part in name.split("+"):
            mode |= piece[part]
        variants.append(("mixed" if name == "all" else "mixed_" + name, mode))
    weights = None
    train = None
    if args.combined:
        # the learned guess of the combined form: pairs harvested from a separate
        # run of the same wedge and init, network trained on the GPU
        src = kc.Sim(grid, kc.puffy_options(device=local))
        src.initPuffy(1e-3, 1e-3, args.seed)
        src.harvest_implicit(args.pairs)
        hsteps = 0
        while True:
            src.step()
            hsteps += 1
            x, t = src.get_harvest(args.pairs)
            if x.shape[0] >= args.pairs or hsteps >= 20:
                break
        src.close()
        weights, loss = kc.mlp_train(x, t, steps=args.train_steps, batch=1024, lr=2e-3, seed=3)
        train = {"pairs": int(x.shape[0]), "harvest_steps": hsteps, "minibatches": args.train_steps,
                 "loss_first": float(loss[:10].mean()), "loss_last": float(loss[-100:].mean())}
        variants = variants + [("combined", kc.KC_MIXED, weights), ("fp64_guess", 0, weights),
                               ("fp64_nobisect", 0, None, {"radimp_start_with_bisect": 0})]
    variants = [tuple(v) + (None,) * (4 - len(v)) for v in variants]
    for form, mode, w, o in [("fp64", 0, None, None)] + variants + [("fp64_seeded", 0, None, None)]:
        sim = kc.Sim(grid, kc.puffy_options(device=local, precision=mode, **(o or {})))
        sim.initPuffy(1e-3, 1e-3, args.seed)
        if w is not None:
            sim.set_guess(w)
        if form == "fp64_seeded":
            # the FP64 run's own sensitivity: a 1e-15 relative seed on the conserved density
            u = sim.u
            u[:, 0] *= 1.0 + 1e-15 * np.random.default_rng(5).uniform(-1.0, 1.0, u.shape[0])
            sim.set_cons(u)
        stream = torch.cuda.ExternalStream(sim.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(args.steps):
            if form == "fp64":
                dts.append(sim.step())
            else:
                sim.step(dts[k])
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        c = sim.counters()
        out[form] = {"p": sim.p, "scalars": sim.scalars(0.0, 5000.0, 15.0), "ms_per_step": ms / args.steps,
                     "value": args.nx * args.ny * args.nz * args.steps / (ms / 1e3),
                     "newton_per_solve": c["n_radimp_iters"] / max(c["n_radimp_solves"], 1),
                     "implicit_failures": c["n_radimp_failures"]}
        sim.close()
    b = out["fp64"]["p"]
    ok = np.all(np.isfinite(b), axis=1)

    def dev_of(form):
        a = out[form]["p"]
        d = np.abs(a[ok] - b[ok]).max(axis=0) / np.maximum(np.abs(b[ok]).max(axis=0), 1e-300)
        r = {k: abs(out[form]["scalars"][k] / out["fp64"]["scalars"][k] - 1)
             for k in ("mass", "mdot", "radlum", "totallum", "scaleheight")}
        return d, r

    dev_s, rel_s = dev_of("fp64_seeded")
    line = {"metric": METRIC, "unit": UNIT, "workload": f"PUFFY 3D wedge {args.nx}x{args.ny}x{args.nz}, {args.steps} steps",
            "fp64": {"value": out["fp64"]["value"], "ms_per_step": out["fp64"]["ms_per_step"]},
            "fp64_seed_1e-15": {"field_scale": dict(zip(names, dev_s.tolist())), "integrated_rel": rel_s},
            "scalars_fp64": out["fp64"]["scalars"]}
    line["fp64"]["newton_per_solve"] = out["fp64"]["newton_per_solve"]
    if train is not None:
        line["guess_training"] = train
    for form, mode, w, _ in variants:
        dev, rel = dev_of(form)
        line[form] = {"precision_mode": mode, "learned_guess": w is not None, "value": out[form]["value"],
                      "ms_per_step": out[form]["ms_per_step"], "newton_per_solve": out[form]["newton_per_solve"],
                      "implicit_failures": out[form]["implicit_failures"],
                      "field_scale_error": dict(zip(names, dev.tolist())), "integrated_rel_error": rel,
                      "scalars": out[form]["scalars"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_guess(args, rank, local):
    """The learned initial guess: (pre-solve, converged) pairs harvested from the
    implicit passes of the 192x180x64 wedge, the network trained on the GPU,
    then the 256x256x128 wedge stepped with the reference's bisection warm
    start (plain), with the learned guess, and with the reference's own
    no-bisection start, on one dt sequence: zone-cycles/s, implicit-pass time,
    Newton iterations per solve, and the field-scale deviation of the final
    state from the plain run's."""
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    kc = load_engine()
    src = kc.Sim(kc.puffy_grid(192, 180, 64), kc.puffy_options(device=local))
    src.initPuffy(1e-3, 1e-3, args.seed)
    src.set_harvest_filter(1 if args.harvest == "hard" else 0)
    src.harvest_implicit(args.pairs)
    hsteps = 0
    while True:
        src.step()
        hsteps += 1
        x, t = src.get_harvest(args.pairs)
        if x.shape[0] >= args.pairs or hsteps >= 20:
            break
    src.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w, loss = kc.mlp_train(x, t, steps=args.train_steps, batch=1024, lr=2e-3, seed=3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0

    grid = kc.puffy_grid(args.nx, args.ny, args.nz)
    ncell = args.nx * args.ny * args.nz
    forms = (("plain", {}, False), ("learned", {}, True), ("no_bisect", {"radimp_start_with_bisect": 0}, False))
    out, dts, finals = {}, [], {}
    for name, o, learned in forms:
        sim = kc.Sim(grid, kc.puffy_options(device=local, **o))
        sim.initPuffy(1e-3, 1e-3, args.seed)
        if learned:
            sim.set_guess(w)
        k = 0
        for _ in range(args.warmup):
            if name == "plain":
                dts.append(sim.step())
            else:
                sim.step(dts[k])
            k += 1
        stream = torch.cuda.ExternalStream(sim.stream())
        c0 = sim.counters()
        sim.set_pass_timing(True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            if name == "plain":
                dts.append(sim.step())
            else:
                sim.step(dts[k])
            k += 1
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        c1 = sim.counters()
        solves = c1["n_radimp_solves"] - c0["n_radimp_solves"]
        out[name] = {"value": ncell * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "implicit_ms_per_step": sim.pass_times()["implicit"][0] / args.steps,
                     "newton_iters_per_solve": (c1["n_radimp_iters"] - c0["n_radimp_iters"]) / max(solves, 1),
                     "solve_failures": c1["n_radimp_failures"] - c0["n_radimp_failures"]}
        if learned:
            out[name]["fallbacks_to_plain"] = sim.guess_fallbacks()
        finals[name] = sim.p
        sim.close()
    b = finals["plain"]
    ok = np.all(np.isfinite(b), axis=1)
    names = ["rho", "uu", "vx", "vy", "vz", "entr", "b1", "b2", "b3", "ee", "fx", "fy", "fz"]
    for name in ("learned", "no_bisect"):
        d = np.abs(finals[name][ok] - b[ok]).max(axis=0) / np.maximum(np.abs(b[ok]).max(axis=0), 1e-300)
        out[name]["field_scale_dev_vs_plain"] = dict(zip(names, d.tolist()))
    line = {"metric": METRIC, "unit": UNIT, "workload": f"PUFFY 3D wedge {args.nx}x{args.ny}x{args.nz}, learned guess",
            "steps": args.steps, "warmup": args.warmup, "dtype": "f64 solve, bf16 network",
            "training": {"pairs": int(x.shape[0]), "harvest_steps": hsteps, "source": "PUFFY 3D wedge 192x180x64",
                         "harvest": args.harvest,
                         "train_steps": args.train_steps, "batch": 1024, "seconds": train_s,
                         "loss_first10": float(loss[:10].mean()), "loss_last100": float(loss[-100:].mean())},
            **out}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 20; 3 for --workload implicit)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="koral", choices=["koral", "reference"])
    ap.add_argument("--nx", type=int, default=192)
    ap.add_argument("--ny", type=int, default=180)
    ap.add_argument("--nz", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20250)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="step", choices=["step", "implicit", "precision", "guess"],
                    help="step: the RK2IMEX step on the wedge; implicit: the batched implicit-solve microbenchmark; "
                         "precision: mixed vs plain FP64 error study on the wedge; guess: the learned initial "
                         "guess against the plain one (use --nx 256 --ny 256 --nz 128)")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch the step's kernels eagerly instead of replaying a captured CUDA graph")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip the autotuner (implicit form and block sizes) before the timed steps")
    ap.add_argument("--no-forms", dest="forms", action="store_false",
                    help="skip the mixed-vs-plain comparison of the default workload")
    ap.add_argument("--combined", action="store_true",
                    help="precision workload: add the combined form (mixed + learned guess) and FP64 + learned guess")
    ap.add_argument("--mixed-forms", default="all",
                    help="precision workload: comma-separated FP32 piece sets (all, ppm, laxf, ct, flux, "
                         "or a+b combinations) run beside plain FP64")
    ap.add_argument("--pairs", type=int, default=1000000, help="training pairs of the guess workload")
    ap.add_argument("--harvest", default="all", choices=["hard", "all"],
                    help="guess workload: train on the solves whose pre-solve state must iterate (hard) or on all")
    ap.add_argument("--train-steps", type=int, default=3000, help="training minibatches of the guess workload")
    ap.add_argument("--cells", type=int, default=1 << 22, help="cells of the implicit microbenchmark")
    ap.add_argument("--face-tiles", type=int, default=None, choices=[0, 1, 2],
                    help="form of the y and z face sweeps (kc_set_face_tiles); default: the engine's")
    ap.add_argument("--implicit-mode", default=None, choices=["per-cell", "compacting", "split", "sorted", "rungs", "iters"],
                    help="implicit solve form: one thread per cell, the persistent lane-refilling state machine, the "
                         "split opening + compacted-ladder pair, or (batch workload only) the per-cell kernel over "
                         "key-sorted cells; default: sorted for --workload implicit, per-cell otherwise")
    args = ap.parse_args()
    if args.implicit_mode is None:  # iters is a batch form; the step's default form is per-cell
        args.implicit_mode = "iters" if args.workload == "implicit" else "per-cell"
    if args.steps is None:
        args.steps = 3 if args.workload == "implicit" else 20
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.workload == "implicit":
        return run_implicit(args, rank, world, local)
    if args.workload == "precision":
        return run_precision(args, rank, local)
    if args.workload == "guess":
        return run_guess(args, rank, local)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device (the engine has no CPU path)")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])

    kc = load_engine()
    grid = kc.puffy_grid(args.nx, args.ny, args.nz)
    opt = kc.puffy_options(device=local, implicit_mode=IMPLICIT_MODES[args.implicit_mode])
    t0 = time.perf_counter()
    sim = kc.Sim(grid, opt)
    create_s = time.perf_counter() - t0
    ncell = args.nx * args.ny * args.nz
    ndim = sum(1 for d in (args.nx, args.ny, args.nz) if d > 1)
    t0 = time.perf_counter()
    fac = sim.initPuffy(1e-3, 1e-3, args.seed)
    init_s = time.perf_counter() - t0
    if args.face_tiles is not None:
        sim.set_face_tiles(args.face_tiles)
    if args.graph:
        sim.set_graph(True)
    for _ in range(args.warmup):
        sim.step()
    tune = None
    if args.tune:
        # the autotuner times candidates from this state and restores it
        tune = sim.autotune(2)
        for _ in range(2):  # the chosen form's eager step and graph capture
            sim.step()
    stream = torch.cuda.ExternalStream(sim.stream())

    # ---- device-resident timing (value) ------------------------------------------
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    # pass timers record events on the stream; with the graph form they would run
    # the steps eagerly, so the graph run takes its pass table from a separate
    # eager window after the timed one
    sim.set_pass_timing(not args.graph)
    n0 = sim.launch_count()
    s0 = sim.counters()["n_radimp_solves"]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        sim.step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = sim.launch_count() - n0
    solves = sim.counters()["n_radimp_solves"] - s0
    pass_steps = args.steps
    if args.graph:
        pass_steps = min(args.steps, 5)
        sim.set_pass_timing(True)
        s0 = sim.counters()["n_radimp_solves"]
        for _ in range(pass_steps):
            sim.step()
        torch.cuda.synchronize()
        solves = sim.counters()["n_radimp_solves"] - s0
    passes = sim.pass_times()
    sim.set_pass_timing(False)
    ms_max = max_over_ranks(ms, dist, "cuda")
    value = job_rate(ncell, args.steps, world, ms_max)

    # ---- end to end through the C ABI with host buffers (e2e) ---------------------
    # Each step: pinned host p, u, flags -> device, Sim.step, device -> host; the
    # drop-in contract of a host-resident Sim whose step runs on the GPU.
    ke = args.e2e_steps if args.e2e_steps is not None else max(3, args.steps // 4)
    nc = sim.ncell
    hp = torch.empty((nc, kc.NV), dtype=torch.float64, pin_memory=True).numpy()
    hu = torch.empty((nc, kc.NV), dtype=torch.float64, pin_memory=True).numpy()
    hf = torch.empty((nc, kc.NFLAGS), dtype=torch.int32, pin_memory=True).numpy()
    lib, h = kc.lib(), sim._h
    for fn, buf in ((lib.kc_download_prims, hp), (lib.kc_download_cons, hu), (lib.kc_download_flags, hf)):
        sim._check(fn(h, buf.ctypes.data))
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        sim._check(lib.kc_upload_prims(h, hp.ctypes.data))
        sim._check(lib.kc_upload_cons(h, hu.ctypes.data))
        sim._check(lib.kc_upload_flags(h, hf.ctypes.data))
        sim.step()
        sim._check(lib.kc_download_prims(h, hp.ctypes.data))
        sim._check(lib.kc_download_cons(h, hu.ctypes.data))
        sim._check(lib.kc_download_flags(h, hf.ctypes.data))
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ems = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    e2e_bytes = hp.nbytes + hu.nbytes + hf.nbytes
    e2e = {"value": job_rate(ncell, ke, world, ems), "unit": UNIT, "h2d_bytes_per_step": e2e_bytes,
           "d2h_bytes_per_step": e2e_bytes, "steps": ke}

    # ---- the mixed form beside plain FP64 (the metric's "at stated error") ----------
    forms = None
    if world == 1 and args.forms:
        forms = measure_forms(kc, grid, local, args.steps, args.seed, args.graph)

    # ---- roofline of the dominant pass ---------------------------------------------
    peaks, peak_kind = measured_peaks()
    total = sum(v[0] for v in passes.values())
    table = {}
    for name, (pms, calls) in passes.items():
        if calls == 0:
            continue
        entry = {"ms_per_step": pms / pass_steps, "share": pms / total if total else 0.0,
                 "calls_per_step": calls / pass_steps}
        bpc = pass_bytes(name, ndim)
        if bpc is not None:
            entry["gbs"] = bpc * ncell / (pms / calls / 1e3) / 1e9
        table[name] = entry
    dom = max((n for n in table if n != "step"), key=lambda n: table[n]["ms_per_step"])
    dom_ms, dom_calls = passes[dom]
    bpc = pass_bytes(dom, ndim)
    kernel = {"implicit": "k_implicit", "fluxes": "k_face_flux", "u2p": "k_u2p", "update": "k_update",
              "wavespeeds": "k_wavespeeds", "radvisc": "k_rijvisc"}.get(dom, dom)
    achieved = bpc * ncell / (dom_ms / dom_calls / 1e3) / 1e9 if bpc else None
    tr = profiled_traffic(kernel)
    roofline = {
        "bound": "hbm", "kernel": kernel, "pass": dom, "achieved": achieved, "peak": peaks["hbm_gbs"],
        "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"] if achieved else None,
        "traffic": tr * ncell if tr else None, "algorithmic_bytes": bpc * ncell if bpc else None,
        "avg_launch_ms": dom_ms / dom_calls,
        "passes": table,
    }
    # the FP64 side of the implicit solve: ncu-counted FLOP per cell-solve (dadd +
    # dmul + 2 dfma) x this run's solves per launch over the live launch time,
    # against the DFMA peak measured now on this device
    fps = profiled_figure("k_implicit", "fp64_flop_per_solve")
    if dom == "implicit" and fps:
        solves_per_launch = solves / max(dom_calls, 1)
        peak64 = kc.fp64_peak()
        got = fps * solves_per_launch / (dom_ms / dom_calls / 1e3) / 1e12
        roofline["fp64"] = {"achieved": got, "peak": peak64, "unit": "TFLOP/s", "frac": got / peak64,
                            "flop_per_solve": fps, "solves_per_launch": solves_per_launch,
                            "peak_kind": "measured (kc_fp64_peak, DFMA chains)"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (PUFFY torus from the engine's init + seeded 1e-3 rho/u_int noise)",
        "config": {"workload": f"PUFFY 3D wedge {args.nx}x{args.ny}x{args.nz} MKS2 (periodic phi), plain FP64",
                   "cells": ncell, "ghosts": 3, "precision": "plain FP64", "l2": "inputs larger than L2 (no flush)",
                   "create_seconds": create_s, "init_seconds": init_s, "beta_norm_factor": fac, "parallelism": f"replicas x{world}",
                   "implicit_mode": args.implicit_mode if tune is None else
                   {0: "per-cell", 1: "compacting", 2: "split"}[tune["implicit_mode"]],
                   "cuda_graph": bool(args.graph), "autotune": tune,
                   "pass_table": "timed region" if not args.graph else f"{pass_steps} eager steps after it"},
        "e2e": e2e, "roofline": roofline, "clocks": clk, "gpu_launches": launches,
    }
    if forms is not None:
        line["forms"] = forms
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, t = oracle_rate(args.nx, args.ny, SAMPLE_NZ, 1, 1, threads, min_seconds=10.0)
        line["cpu_baseline"] = {
            "value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{args.nx}x{args.ny}x{SAMPLE_NZ} slice of the wedge, {n} steps ({t:.1f} s) after 1 warm-up, "
                      "oracle/orc_sim.cpp"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
