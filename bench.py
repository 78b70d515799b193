"""Benchmark of the SLIC/FORCE hot path on B200 (one JSON line on rank 0).

Workload (one "step" = one full split time step X(dt/2) Y(dt) X(dt/2) over the whole grid):
  2D Euler SLIC, 4096 x 4096 cells on [0,1]^2, gamma = 1.4, transmissive boundaries, four-quadrant
  Riemann initial data drawn from a seed (rho ~ U[0.1,2], u,v ~ U[-1,1], p ~ U[0.1,2]), superbee,
  CFL 0.8, dt computed on the device every step.  Inputs are larger than L2 (the FP64 state is 537 MB)
  so no L2 flush is needed between steps.

Arms:
  default              the CUDA path through the C ABI (libvanguard_slic.so); value = device-timed
                       cell-updates/s with the state resident in HBM; e2e = the same metric through
                       vg_solve() from pinned host buffers with H2D/D2H inside the timed region.
  --impl reference     the reference's own OpenMP C++ code (compiled unmodified into oracle/_ref) on
                       the host cores, on a bounded sample (a strip of the same grid) per step.

Multi-GPU (torchrun, N > 1): the path has no exchange step, so every rank runs an independent replica of
the workload; value = all ranks' cell-updates / the slowest rank's time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import threading
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s: mixed vs plain FP64 on GPU at ≤1e-6 L1 err; adjoint/fwd cost"
UNIT = "cell-updates/s"
NX = NY = 4096
CFL = 0.8
LIMITER = 0  # superbee
SEED = 2024
BYTES_PER_CELL_SWEEP = 2 * 4 * 8      # read + write of rho, rho u, rho v, E in FP64
BYTES_PER_CELL_UPDATE = 3 * BYTES_PER_CELL_SWEEP  # 192 B: three sweeps per step


def workload_config():
    return {
        "workload": "2D Euler SLIC 4096x4096, four-quadrant Riemann (seeded), gamma 1.4, superbee, CFL 0.8, transmissive",
        "nx": NX, "ny": NY, "limiter": "superbee", "cfl": CFL, "seed": SEED,
        "l2": "inputs larger than L2 (FP64 state 537 MB), no flush",
        "parallelism": "replicas",
    }


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons).  nvidia-smi needs longer to start
    than a short timed region lasts, so __enter__ returns only once the first sample has arrived (at most 5 s), a
    reader thread stamps every line on arrival, and only the lines that arrive between __enter__ and __exit__ count."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 25

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.stamped = []
        self.lines = []

    def _read(self):
        for line in self.proc.stdout:
            self.stamped.append((time.monotonic(), line))

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", str(self.PERIOD_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            t0 = time.monotonic()
            while not self.stamped and time.monotonic() - t0 < 5.0:
                time.sleep(0.005)
        except Exception:
            self.proc = None
        self.t_start = time.monotonic()
        return self

    def __exit__(self, *exc):
        t_end = time.monotonic()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.reader.join(timeout=5)
        late = 0.5 * self.PERIOD_MS / 1e3  # a sample taken inside the region may be read this much after it
        self.lines = [l for t, l in self.stamped if self.t_start <= t <= t_end + late and l.strip()]

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


class RankGroup:
    """One process per GPU (torchrun): the barrier and the max over ranks of the timing protocol.  NCCL on the
    GPUs; the same code runs with gloo on CPU tensors in the multi-process tests.  world == 1 needs no group."""

    def __init__(self, world, rank, backend, device):
        self.world, self.rank, self.device, self.dist = world, rank, device, None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        """The largest x over all ranks (every rank calls it, in the same order)."""
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def job_value(world, units_per_rank, slowest_seconds):
    """Whole-job throughput of `world` replicas that each processed units_per_rank, timed by the slowest rank."""
    return world * units_per_rank / slowest_seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ----------------------------------------------------------------------------------------- reference arm

def run_reference(args, world, rank):
    """The reference's own OpenMP C++ loop (compiled unmodified into oracle/_ref) on all host cores: the K timed
    steps run as ONE call of its per-step loop on a strip through the centre of the 4096^2 grid (ghost insertion,
    CFL time step, X(dt/2) Y(dt) X(dt/2) per step), after W warm-up steps in another call; the strip is sized from
    a probe so the timed call lasts about a minute."""
    if rank != 0:
        return 0
    import oracle as O
    from vanguard_b200 import workloads as wl
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvgref.so was not built"}))
        return 0
    cores = O.ref().vgref_set_threads(0)
    prm = wl.euler_params(1.4)
    full = wl.euler_quadrants_2d(NX, NY, seed=SEED)
    # per-step cost on a thin strip of the same grid, then size the sample so the timed call lasts ~60 s
    probe_rows = 16
    strip = np.ascontiguousarray(full[:, NY // 2 - probe_rows // 2: NY // 2 + probe_rows // 2, :])
    t0 = time.perf_counter()
    O.ref_run(O.EULER, strip.copy(), 1.0 / NX, CFL, steps=1, limiter=LIMITER, params=prm, threads=cores)
    per_cell = (time.perf_counter() - t0) / (NX * probe_rows)
    rows = int(max(16, min(NY, 60.0 / max(per_cell * NX * args.steps, 1e-12))))
    rows -= rows % 2
    sample = np.ascontiguousarray(full[:, NY // 2 - rows // 2: NY // 2 + rows // 2, :])
    O.ref_run(O.EULER, sample.copy(), 1.0 / NX, CFL, steps=args.warmup, limiter=LIMITER, params=prm, threads=cores)
    state = sample.copy()
    t0 = time.perf_counter()
    O.ref_run(O.EULER, state, 1.0 / NX, CFL, steps=args.steps, limiter=LIMITER, params=prm, threads=cores)
    total = time.perf_counter() - t0
    value = NX * rows * args.steps / total
    desc = (f"reference SecondOrderSolver per-step loop (oracle/_ref, OpenMP {cores} threads) on a {NX}x{rows} "
            f"strip through the centre of the 4096x4096 grid, {args.steps} steps in one call")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample():
    """The reference on the host cores for ~10-30 s on a strip of the workload (rank 0, N = 1)."""
    import oracle as O
    from vanguard_b200 import workloads as wl
    if not O.ref_available():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "oracle/_ref not built"}
    cores = O.ref().vgref_set_threads(0)
    prm = wl.euler_params(1.4)
    full = wl.euler_quadrants_2d(NX, NY, seed=SEED)
    probe_rows = 16
    strip = np.ascontiguousarray(full[:, NY // 2 - 8: NY // 2 + 8, :])
    t0 = time.perf_counter()
    O.ref_run(O.EULER, strip.copy(), 1.0 / NX, CFL, steps=1, limiter=LIMITER, params=prm, threads=cores)
    per_cell = (time.perf_counter() - t0) / (NX * probe_rows)
    steps = 2
    rows = int(max(16, min(NY, 15.0 / max(per_cell * NX * steps, 1e-12))))
    rows -= rows % 2
    sample = np.ascontiguousarray(full[:, NY // 2 - rows // 2: NY // 2 + rows // 2, :])
    t0 = time.perf_counter()
    O.ref_run(O.EULER, sample, 1.0 / NX, CFL, steps=steps, limiter=LIMITER, params=prm, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": NX * rows * steps / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{steps} steps of the reference per-step loop on a {NX}x{rows} strip of the workload "
                      f"({dt:.1f} s, OpenMP {cores} threads)"}


def hbm_roofline(rate, bytes_per_cell_update, basis):
    """HBM roofline of a whole leg: algorithmic bytes per cell-update (SURVEY's passes x 2 x components x 8 B) times
    the measured cell-update rate, against the measured copy bandwidth."""
    peak, kind = measured_peak()
    achieved = rate * bytes_per_cell_update / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "bytes_per_cell_update": bytes_per_cell_update, "basis": basis, "peak_source": kind}


def ref_cores():
    """Host threads for the reference's CPU baselines (0 when they are off or the reference was not built)."""
    import oracle as O
    if not CPU_LEGS or not O.ref_available():
        return 0
    return O.ref().vgref_set_threads(0)


# ---------------------------------------------------------------------------------------------- CUDA arm

def run_cuda(args, world, rank, local):
    import torch
    import vanguard_b200 as vg
    from vanguard_b200 import workloads as wl

    torch.cuda.set_device(local)
    group = RankGroup(world, rank, "nccl", f"cuda:{local}")
    barrier, max_over_ranks = group.barrier, group.max

    stream = torch.cuda.current_stream()
    sh = ctypes_stream(stream)
    legs = [x for x in args.legs.split(",") if x]
    global CPU_LEGS
    CPU_LEGS = world == 1 and rank == 0 and not args.no_cpu_baseline
    if "headline" not in legs:  # profiling / diagnostic runs of single legs (not a bench line)
        out = {}
        for leg in legs:
            out[leg] = LEGS[leg](local, stream, sh)
        if rank == 0:
            print(json.dumps({"legs": out}), flush=True)
        group.close()
        return 0

    prm = wl.euler_params(1.4)
    W0 = wl.euler_quadrants_2d(NX, NY, seed=SEED + rank)
    dx = 1.0 / NX

    results = {}
    wanted = args.forms.split(",")
    forms = [("fp64", vg.FP64)] if "fp64" in wanted else []
    if "mixed" in wanted and vg_mixed_available(vg):
        forms.append(("mixed", vg.MIXED))
    finals = {}
    for name, prec in forms:
        s = vg.Solver(vg.EULER, NX, NY, prm, precision=prec, device=local)
        s.upload(W0, stream=sh)
        # pick the sweep tile shapes on this grid (results do not depend on the choice)
        xt, yt = s.autotune(dx, CFL, limiter=LIMITER, stream=sh)
        tuned = s.launch_config()
        # warm-up (also captures the step graphs)
        s.run(dx, CFL, steps=max(args.warmup, 3), limiter=LIMITER, stream=sh)
        s.upload(W0, stream=sh)
        barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            start.record(stream)
            _, steps = s.run(dx, CFL, steps=args.steps, limiter=LIMITER, stream=sh, allow_nan=True)
            end.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = start.elapsed_time(end)
        ms = max_over_ranks(ms)
        launches = s.last_launch_count()
        finals[name] = s.download(stream=sh)

        # dominant kernel: an X half-sweep, timed alone (CUDA events on the launching stream)
        reps = max(5, min(args.steps, 20))
        s.sweep(0, dx, 1e-5, limiter=LIMITER, stream=sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            s.sweep(0, dx, 1e-5, limiter=LIMITER, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        xs_ms = e0.elapsed_time(e1) / reps
        e0.record(stream)
        for _ in range(reps):
            s.sweep(1, dx, 1e-5, limiter=LIMITER, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ys_ms = e0.elapsed_time(e1) / reps
        results[name] = {"ms": ms, "steps": steps, "launches": launches, "clocks": clk.summary(),
                         "x_sweep_ms": xs_ms, "y_sweep_ms": ys_ms,
                         "tuned": {"x": tuned[2], "y": tuned[3], "x_ms": xt, "y_ms": yt}}
        s.close()

    # The headline is the plain FP64 form: the reference's own arithmetic, bit-equal to it (the same grid and seed
    # are pinned against the oracle in tests/test_zs_config_shapes_gpu.py), so the comparison with the reference
    # arm is like for like.  The mixed form is reported beside it.
    head = "fp64" if "fp64" in results else "mixed"
    prec = vg.FP64 if head == "fp64" else vg.MIXED
    # end-to-end through the host-buffer API (vg_solve: upload + run + download inside the timed region)
    hin = torch.from_numpy(W0).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    s = vg.Solver(vg.EULER, NX, NY, prm, precision=prec, device=local)
    s.upload(W0, stream=sh)
    s.autotune(dx, CFL, limiter=LIMITER, measure=False, stream=sh)  # cached choice from the timed run
    s.solve(hin.numpy(), dx, CFL, steps=2, limiter=LIMITER, out=hout.numpy(), stream=sh)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.solve(hin.numpy(), dx, CFL, steps=args.steps, limiter=LIMITER, out=hout.numpy(), stream=sh)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    s.close()
    carried = 4  # rho, u, v, p cross the bus; w and lambda are validated on the host and not copied
    h2d = carried * NX * NY * 8
    d2h = carried * NX * NY * 8

    r = results[head]
    cells = NX * NY
    value = job_value(world, cells * args.steps, r["ms"] / 1000.0)
    peak, peak_kind = measured_peak()
    x_bytes = cells * BYTES_PER_CELL_SWEEP
    achieved = x_bytes / (r["x_sweep_ms"] / 1000.0) / 1e9
    traffic = load_traffic(head)

    if rank != 0:
        group.close()
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64", "data": "synthetic",
        "config": workload_config(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": ("sweep_x_kernel" if head == "fp64" else "sweep_x_pair_kernel") + " (X half-sweep, "
                               + r["tuned"]["x"] + ")",
                     "algorithmic_bytes_per_launch": x_bytes, "peak_source": peak_kind,
                     "note": ("the exact FP64 form is bound by the FP64 pipe (correctly rounded divisions and square "
                              "roots, no contraction), not by HBM: ncu shows the FP64 pipe 61 % busy and DRAM 10 % "
                              "(profiles/sweep_x_kernel_euler_fp64_2048.md); the mixed form's X sweep reaches 0.62 of "
                              "HBM (forms.mixed.x_sweep_hbm_frac)") if head == "fp64" else ""},
        "e2e": {"value": job_value(world, cells * args.steps, e2e_s), "unit": UNIT,
                "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "api": f"vg_solve ({head}; pinned host buffers; one upload + K steps + one download per call)"},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "form": head,
        "forms": {k: {"cell_updates_per_s": world * cells * args.steps / (v["ms"] / 1000.0),
                      "ms_per_step": v["ms"] / args.steps, "x_sweep_ms": v["x_sweep_ms"],
                      "y_sweep_ms": v["y_sweep_ms"], "autotune": v["tuned"],
                      "x_sweep_hbm_frac": x_bytes / (v["x_sweep_ms"] / 1000.0) / 1e9 / peak,
                      "y_sweep_hbm_frac": x_bytes / (v["y_sweep_ms"] / 1000.0) / 1e9 / peak,
                      "hbm_frac_of_step": world * cells * args.steps * BYTES_PER_CELL_UPDATE / (v["ms"] / 1000.0) / 1e9 / peak}
                  for k, v in results.items()},
    }
    if "mixed" in results and "fp64" in results:
        line["mixed_speedup"] = results["fp64"]["ms"] / results["mixed"]["ms"]
    if "mixed" in finals and "fp64" in finals:
        d = np.abs(finals["mixed"][0] - finals["fp64"][0])
        line["mixed_error_vs_fp64"] = {
            "rho_L1": float(d.mean()), "rho_Linf": float(d.max()), "steps": args.steps,
            "reference": "this run's FP64 form; tests/test_zs_config_shapes_gpu.py::test_euler_4096_five_steps checks "
                         "that form bit-equal to the oracle on this grid and seed, and the mixed form against the "
                         "oracle itself"}
    names = {"c5": "C5_ragged_batch_adjoint", "c4": "C4_hpr_1024", "c3": "C3_mhd_2048", "c1": "C1_sod_1000",
             "tm": "two_material_2048"}
    extra = {names[leg]: LEGS[leg](local, stream, sh) for leg in legs if leg in names}
    if extra:
        line["configs"] = extra
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    print(json.dumps(line), flush=True)
    group.close()
    return 0


C5_NINST, C5_STEPS, C5_CKPT = 4096, 500, 32


def ragged_adjoint_leg(local, stream, sh, reps=3):
    """C5: 4096 ragged 1D Euler Riemann problems (cells U{200..4000}), CFL 0.8, superbee, 500 steps per instance
    in one persistent launch per step (the whole loop one CUDA graph), then the discrete adjoint of
    L = sum (rho(T) - target)^2 with respect to the initial states and gamma.  Device-timed with CUDA events on the
    launching stream; the adjoint cost is reported against the forward for a binomial schedule with C5_CKPT state
    slots (recomputes forward segments) and with every state stored."""
    import torch
    import vanguard_b200 as vg
    from vanguard_b200 import workloads as wl

    ncell, dx, gamma, theta, W0 = wl.ragged_riemann_batch(ninst=C5_NINST, seed=SEED)
    total = int(W0.shape[1])
    target = np.random.default_rng(SEED + 1).uniform(0.1, 2.0, total)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"workload": f"{C5_NINST} ragged 1D Euler Riemann problems, cells U{{200..4000}} ({total} cells), "
                       f"gamma U[1.2,1.67], CFL 0.8, superbee, {C5_STEPS} steps, per-instance device dt",
           "cells": total}
    with vg.Batch(ncell, dx, gamma, device=local) as b:
        b.upload(W0, stream=sh)
        b.run(CFL, C5_STEPS, limiter=LIMITER, stream=sh)  # graph capture
        fwd = []
        for _ in range(reps):
            b.upload(W0, stream=sh)
            torch.cuda.synchronize()
            e0.record(stream)
            b.run(CFL, C5_STEPS, limiter=LIMITER, stream=sh)
            e1.record(stream)
            torch.cuda.synchronize()
            fwd.append(e0.elapsed_time(e1))
        fwd_ms = statistics.median(fwd)
        out["forward"] = {"ms": fwd_ms, "cell_updates_per_s": total * C5_STEPS / (fwd_ms / 1e3),
                          "launches": b.last_launch_count()}
        tgt = torch.from_numpy(target).to(f"cuda:{local}")
        g = torch.empty((6, total), dtype=torch.float64, device=f"cuda:{local}")
        gg = torch.empty((C5_NINST,), dtype=torch.float64, device=f"cuda:{local}")
        for name, ck in (("binomial", C5_CKPT), ("store_all", C5_STEPS)):
            b.upload(W0, stream=sh)
            b.gradient(tgt, CFL, C5_STEPS, limiter=LIMITER, checkpoints=ck, out=(g, gg), stream=sh)  # workspace
            torch.cuda.synchronize()
            e0.record(stream)
            L, _, _, fw, aw = b.gradient(tgt, CFL, C5_STEPS, limiter=LIMITER, checkpoints=ck, out=(g, gg), stream=sh)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            out[f"adjoint_{name}"] = {"checkpoints": ck, "ms": ms, "ratio_vs_forward": ms / fwd_ms,
                                      "forward_steps": fw, "reversed_steps": aw, "loss": L,
                                      "state_slot_bytes": (min(ck, C5_STEPS) + 1) * 3 * total * 8}
        # through the host-buffer API with pinned buffers, copies inside the timed region: the forward uploads the
        # initial planes and downloads the final ones; the gradient uploads the initial planes and the target and
        # downloads the gradient planes and the gamma gradient
        pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
        h_w0, h_out, h_tgt, h_g, h_gg = pin((6, total)), pin((6, total)), pin((total,)), pin((6, total)), pin((C5_NINST,))
        h_w0[:] = W0
        h_tgt[:] = target
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.upload(h_w0, stream=sh)
        b.run(CFL, C5_STEPS, limiter=LIMITER, stream=sh)
        b.download(out=h_out, stream=sh)
        fwd_host_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        b.upload(h_w0, stream=sh)
        b.gradient(h_tgt, CFL, C5_STEPS, limiter=LIMITER, checkpoints=C5_CKPT, out=(h_g, h_gg), stream=sh)
        grad_host_s = time.perf_counter() - t0
        out["forward"]["e2e_ms"] = fwd_host_s * 1e3
        out["adjoint_binomial"]["e2e_ms"] = grad_host_s * 1e3
        out["adjoint_binomial"]["e2e_ratio_vs_forward"] = grad_host_s / fwd_host_s
    out["forward"]["roofline"] = hbm_roofline(out["forward"]["cell_updates_per_s"], 48,
                                              "one pass per step x 2 x 3 components (rho, rho u, E) x 8 B")
    cores = ref_cores()
    if cores:
        # the reference's way: SecondOrderSolver::solve's loop once per problem, problems in parallel on the host
        # cores (one thread each); timed on every instance for a few steps
        import oracle as O
        probe = W0.copy()
        t0 = time.perf_counter()
        O.ref_batch_run(probe, ncell, dx, gamma, CFL, 1, limiter=LIMITER, threads=cores)
        one = time.perf_counter() - t0
        steps = int(max(1, min(C5_STEPS, 15.0 / max(one, 1e-9))))
        sample = W0.copy()
        t0 = time.perf_counter()
        O.ref_batch_run(sample, ncell, dx, gamma, CFL, steps, limiter=LIMITER, threads=cores)
        dt = time.perf_counter() - t0
        rate = total * steps / dt
        fwd_s = total * C5_STEPS / rate
        out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                               "sample": f"{steps} steps of all {C5_NINST} problems, each by the reference's 1D solve "
                                         f"loop, problems in parallel one thread each ({dt:.1f} s)"}
        out["forward"]["vs_cpu_reference"] = out["forward"]["cell_updates_per_s"] / rate
        # the reference has no derivatives: its gradient is central differences, 2 forward runs per parameter
        # (6 initial primitives + gamma per problem, all problems perturbed at once), estimated from the rate above
        out["cpu_fd_gradient_estimate_s"] = {"value": 14 * fwd_s, "forward_runs": 14, "forward_s": fwd_s,
                                             "basis": "14 full 500-step forward runs of the reference batch at the "
                                                      "measured sample rate"}
        out["adjoint_binomial"]["vs_cpu_fd_gradient"] = 14 * fwd_s / (out["adjoint_binomial"]["ms"] / 1e3)
    return out


C3_N, C3_STEPS = 2048, 500


def mhd_leg(local, stream, sh):
    """C3: 2D ideal MHD (GLM) 2048^2 periodic smooth vortex, superbee, CFL 0.8, 500 steps, FP64 and mixed."""
    import torch
    import vanguard_b200 as vg
    from vanguard_b200 import workloads as wl

    n, steps = C3_N, C3_STEPS
    W = wl.mhd_vortex_2d(n, seed=SEED)
    prm = wl.mhd_params()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res, finals = {}, {}
    for name, prec in (("fp64", vg.FP64), ("mixed", vg.MIXED)):
        with vg.Solver(vg.MHD, n, n, prm, precision=prec, boundary=vg.PERIODIC, device=local) as s:
            s.upload(W, stream=sh)
            s.autotune(1.0 / n, CFL, limiter=LIMITER, stream=sh)
            s.run(1.0 / n, CFL, steps=3, limiter=LIMITER, stream=sh)
            s.upload(W, stream=sh)
            torch.cuda.synchronize()
            e0.record(stream)
            s.run(1.0 / n, CFL, steps=steps, limiter=LIMITER, stream=sh)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            finals[name] = s.download(stream=sh)
            res[name] = {"ms": ms, "cell_updates_per_s": n * n * steps / (ms / 1e3)}
    d = np.abs(finals["mixed"][0] - finals["fp64"][0])
    res["mixed_error_vs_fp64"] = {"rho_L1": float(d.mean()), "rho_Linf": float(d.max())}
    res["mixed_speedup"] = res["fp64"]["ms"] / res["mixed"]["ms"]
    for form in ("fp64", "mixed"):
        res[form]["roofline"] = hbm_roofline(res[form]["cell_updates_per_s"], 336, "whole step: 3 sweeps x 2 x 7 "
                                             "components x 8 B (rho, rho u, rho v, E, Bx, By, psi)")
    res["workload"] = f"2D MHD {n}x{n} periodic vortex (seeded noise 1e-3), gamma 5/3, superbee, CFL 0.8, {steps} steps"
    cores = ref_cores()
    if cores:
        import oracle as O
        rows = 16
        strip = np.ascontiguousarray(W[:, n // 2 - rows // 2: n // 2 + rows // 2, :])
        t0 = time.perf_counter()
        O.ref_run(O.MHD, strip, 1.0 / n, CFL, steps=2, limiter=LIMITER, params=prm, bc=O.PERIODIC, threads=cores)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": n * rows * 2 / dt, "unit": UNIT, "cores": cores, "kind": "reference",
                               "sample": f"2 steps of the reference MHD per-step loop (c_h from the padded maximum "
                                         f"each step) on a {n}x{rows} periodic strip of the workload ({dt:.2f} s)"}
        res["fp64_vs_cpu_reference"] = res["fp64"]["cell_updates_per_s"] / res["cpu_baseline"]["value"]
    return res


C4_STEPS = 300


def hpr_leg(local, stream, sh):
    """C4: 2D HPR (GPR) 1024^2 smooth field (seeded), ideal gas via the stiffened-gas branch, thermal, tau1 and tau2
    log-uniform on [1e-6, 1e-2] from the seed, superbee, CFL 0.8, C4_STEPS steps, exact FP64.  The relaxation source
    runs as the reference runs it: the RK4 forcing solver with fractional-flux predictors, sub-cycled dt/(2 sub)
    before and after the sweeps, with sub chosen so each sub-step stays inside the explicit RK4 stability bound
    (0.5 dt / sub <= 2.5 min(tau1, tau2), dt estimated from the initial CFL speed with a 1.5x margin)."""
    import math
    import torch
    import vanguard_b200 as vg
    from vanguard_b200 import workloads as wl

    n = 1024
    tau1, tau2 = wl.hpr_relaxation_times(SEED)
    prm = wl.hpr_params(tau1=tau1, tau2=tau2)
    W = wl.hpr_smooth_2d(n, seed=SEED)
    res, finals, sub = {}, {}, 1
    for name, prec in (("fp64", vg.FP64), ("mixed", vg.MIXED)):
        with vg.Solver(vg.HPR, n, n, prm, precision=prec, device=local) as s:
            s.upload(W, stream=sh)
            if name == "fp64":
                S0 = s.max_wave_speed(stream=sh)
                dt_est = 1.5 * CFL * (1.0 / n) / S0
                sub = max(1, math.ceil(0.5 * dt_est / (2.5 * min(tau1, tau2))))
            s.autotune(1.0 / n, CFL, limiter=LIMITER, stream=sh)
            s.run(1.0 / n, CFL, steps=2, limiter=LIMITER, subcycles=sub, stream=sh)
            s.upload(W, stream=sh)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            t, it = s.run(1.0 / n, CFL, steps=C4_STEPS, limiter=LIMITER, subcycles=sub, stream=sh, allow_nan=True)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            finals[name] = s.download(stream=sh)
            res[name] = {"ms": ms, "steps": it, "t": t, "cell_updates_per_s": n * n * it / (ms / 1e3),
                         "launches": s.last_launch_count(), "finite": bool(np.isfinite(finals[name]).all())}
    # the stiff relaxation mode: one relaxation of dt/2 before and after the sweeps instead of the forcing, in the
    # FP64 form and in the configuration's chosen form (FP32 flux, FP64 source, pressure recovery, CFL and update)
    stiff = {}
    for name, prec in (("stiff_fp64", vg.FP64), ("stiff_mixed", vg.MIXED)):
        with vg.Solver(vg.HPR, n, n, prm, precision=prec, device=local) as s:
            s.upload(W, stream=sh)
            s.autotune(1.0 / n, CFL, limiter=LIMITER, stream=sh)
            s.run(1.0 / n, CFL, steps=2, limiter=LIMITER, stiff=True, stream=sh)
            s.upload(W, stream=sh)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            t, it = s.run(1.0 / n, CFL, steps=C4_STEPS, limiter=LIMITER, stiff=True, stream=sh, allow_nan=True)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            stiff[name] = s.download(stream=sh)
            res[name] = {"ms": ms, "steps": it, "t": t, "cell_updates_per_s": n * n * it / (ms / 1e3),
                         "launches": s.last_launch_count(), "speedup_vs_forcing_fp64": res["fp64"]["ms"] / ms,
                         "finite": bool(np.isfinite(stiff[name]).all())}

    def err(a, b):
        d = np.abs(a - b)
        return {"rho_L1": float(d[0].mean()), "rho_Linf": float(d[0].max()), "all_L1": float(d.mean())}

    res["stiff_fp64"]["difference_vs_forcing_fp64"] = err(stiff["stiff_fp64"], finals["fp64"])
    res["stiff_mixed"]["error_vs_stiff_fp64"] = err(stiff["stiff_mixed"], stiff["stiff_fp64"])
    res["stiff_mixed"]["difference_vs_forcing_fp64"] = err(stiff["stiff_mixed"], finals["fp64"])
    res["stiff_mixed"]["speedup_vs_stiff_fp64"] = res["stiff_fp64"]["ms"] / res["stiff_mixed"]["ms"]
    res["mixed_error_vs_fp64"] = err(finals["mixed"], finals["fp64"])
    res["mixed_speedup"] = res["fp64"]["ms"] / res["mixed"]["ms"]
    # algorithmic bytes: 3 sweeps + 2 source passes, each reading and writing the 11 non-trivial components
    for form in ("fp64", "mixed", "stiff_fp64", "stiff_mixed"):
        res[form]["roofline"] = hbm_roofline(res[form]["cell_updates_per_s"], 880, "whole step: (3 sweeps + 2 source "
                                             "passes) x 2 x 11 components x 8 B")
    res["source_adjoint"] = source_adjoint_cost(local, stream, sh, W, prm, tau1, tau2, S_dt=dt_sub_of(res, sub))
    res["chosen_form"] = ("stiff_mixed: the flux in FP32 (reconstruction, half-step evolution, FORCE) with the stiff "
                          "relaxation source, pressure recovery, CFL maximum and update in FP64")
    res["subcycles"] = sub
    res["workload"] = (f"2D HPR {n}x{n} smooth field (seeded), thermal ideal gas, tau1 {tau1:.3e}, tau2 {tau2:.3e}, "
                       f"superbee, CFL 0.8, {C4_STEPS} steps; fp64/mixed: the reference's RK4 forcing (FP64 in both "
                       f"forms) with {sub} sub-cycles per half step; stiff_*: the stiff relaxation source")
    cores = ref_cores()
    if cores:
        import oracle as O
        rows = 4
        strip = np.ascontiguousarray(W[:, n // 2 - rows // 2: n // 2 + rows // 2, :])
        t0 = time.perf_counter()
        O.ref_run(O.HPR, strip, 1.0 / n, CFL, steps=1, limiter=LIMITER, params=prm, subcycles=sub, threads=cores)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": n * rows / dt, "unit": UNIT, "cores": cores, "kind": "reference",
                               "sample": f"1 step of the reference HPR per-step loop with its RK4 forcing ({sub} "
                                         f"sub-cycles per half step) on a {n}x{rows} strip of the workload ({dt:.2f} s)"}
        res["fp64_vs_cpu_reference"] = res["fp64"]["cell_updates_per_s"] / res["cpu_baseline"]["value"]
    return res


def dt_sub_of(res, sub):
    """The RK4 forcing sub-step of the C4 run's last time step: 0.5 dt / sub (Solvers/hprsecondordersolver.cpp:516)."""
    t, it = res["fp64"]["t"], res["fp64"]["steps"]
    return 0.5 * (t / max(it, 1)) / sub


def source_adjoint_cost(local, stream, sh, W, prm, tau1, tau2, S_dt):
    """The HPR relaxation source's discrete adjoint at the C4 scale: every cell of the 1024^2 initial field as a
    homogeneous relaxation problem (vg_source_batch), one time step's worth of the forcing's sub-steps (2 sub of
    length S_dt), forward against the gradient of L = <lambda, W(T)> with binomial checkpointing and with every
    state stored; device-timed (CUDA events on the launching stream)."""
    import torch
    import vanguard_b200 as vg
    n = W.shape[1] * W.shape[2]
    W0 = np.ascontiguousarray(W.reshape(17, n))
    tau = np.stack([np.full(n, tau1), np.full(n, tau2)])
    steps = 26
    dev = f"cuda:{local}"
    lam = torch.from_numpy(np.random.default_rng(SEED + 7).standard_normal((17, n))).to(dev)
    g, gt = torch.empty((17, n), dtype=torch.float64, device=dev), torch.empty((2, n), dtype=torch.float64, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"workload": f"{n} homogeneous HPR cells (the C4 initial field), {steps} source steps of {S_dt:.3e}",
           "cells": n, "steps": steps}
    with vg.SourceBatch(n, prm, device=local) as b:
        b.upload(W0, tau, stream=sh)
        b.run(S_dt, steps, stream=sh)
        b.upload(W0, tau, stream=sh)
        torch.cuda.synchronize()
        e0.record(stream)
        b.run(S_dt, steps, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd = e0.elapsed_time(e1)
        out["forward_ms"] = fwd
        b.upload(W0, tau, stream=sh)
        for name, ck in (("binomial", 6), ("store_all", steps)):
            b.gradient(lam, S_dt, steps, checkpoints=ck, out=(g, gt), stream=sh)
            torch.cuda.synchronize()
            e0.record(stream)
            _, _, fw, aw = b.gradient(lam, S_dt, steps, checkpoints=ck, out=(g, gt), stream=sh)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            out[f"adjoint_{name}"] = {"checkpoints": ck, "ms": ms, "ratio_vs_forward": ms / fwd, "forward_steps": fw,
                                      "reversed_steps": aw}
    return out


def sod_leg(local, stream, sh):
    """C1: 1D Sod, 1000 cells, minbee, CFL 0.9, t_end 0.25 (time to solution, FP64), beside the reference's own
    SecondOrderSolver::solve called as-is on one thread and on all host cores."""
    import torch
    import vanguard_b200 as vg
    from vanguard_b200 import workloads as wl

    W = wl.sod_1d(1000)
    with vg.Solver(vg.EULER, 1000, 1, wl.euler_params(1.4), device=local) as s:
        s.upload(W, stream=sh)
        s.run(1e-3, 0.9, t_end=0.25, limiter=2, stream=sh)
        s.upload(W, stream=sh)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t, it = s.run(1e-3, 0.9, t_end=0.25, limiter=2, stream=sh)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        launches = s.last_launch_count()
    out = {"workload": "1D Sod 1000 cells, minbee, CFL 0.9, t_end 0.25", "steps": it, "t": t, "ms": sec * 1e3,
           "cell_updates_per_s": 1000 * it / sec, "launches": launches}
    out["roofline"] = hbm_roofline(out["cell_updates_per_s"], 48, "one pass per step x 2 x 3 components x 8 B; "
                                   "a 1000-cell grid is launch-latency bound (8 KB per plane), not HBM bound")
    cores = ref_cores()
    if cores:
        import oracle as O
        per = {}
        for thr in (1, cores):
            ref = W.copy()
            t0 = time.perf_counter()
            O.ref_run(O.EULER, ref, 1e-3, 0.9, t_end=0.25, limiter=2, params=wl.euler_params(1.4), threads=thr)
            per[thr] = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1000 * it / per[cores], "unit": UNIT, "cores": cores, "kind": "reference",
                               "sample": f"the reference's SecondOrderSolver::solve as-is, whole run ({per[cores]:.2f} "
                                         f"s on {cores} threads, {per[1]:.2f} s on 1)",
                               "one_thread_value": 1000 * it / per[1]}
        out["vs_cpu_reference"] = out["cell_updates_per_s"] / out["cpu_baseline"]["value"]
    return out


TM_N, TM_STEPS, TM_REINIT = 2048, 100, 10
CPU_LEGS = True  # run_cuda clears it unless this is rank 0 of a 1-GPU run with the CPU baseline on
TM_MODELS = None  # all of them; a comma list names a subset (profiling only)
TM_HPR_N, TM_HPR_STEPS = 1024, 20  # the HPR two-material models in 2D (19-20 planes, RK4 relaxation sub-cycle)
TM_1D_CELLS = 1 << 20  # the 1D-only multiphysics models (HPR multiphysics, MHD multiphysics)


def two_material_leg(local, stream, sh, n=TM_N, steps=TM_STEPS, models=None):
    """The two-material models on n^2 grids of the reference scenarios' 2D layouts (EulerReducedTests' bubble,
    MHDReducedTests' Dumbser disc; gamma 1.4 | 1.67), superbee, CFL 0.8, `steps` steps with the volume fraction
    reinitialised every TM_REINIT steps and one GLM damping sub-cycle for the MHD models: exact FP64 form (and the
    mixed form where the model has one), CUDA events on the launching stream; beside each, the compiled reference's
    per-step loop on a strip of the same grid on the host cores (its CPU baseline).  The HPR reduced and intermediate
    models run an elastic | plastic pair of ShockMieGruneisen solids in the layout of the reference's Zhang scenario
    (its deformation gradients and velocities) on TM_HPR_N^2 for TM_HPR_STEPS steps with one RK4 relaxation sub-cycle;
    the 1D-only multiphysics models run the same solids (HPR) and the Dumbser layout (MHD) on TM_1D_CELLS cells, the
    reference's sample being a TM_1D_CELLS / 64 cell segment about the interface."""
    import torch
    import oracle as O
    import vanguard_b200 as vg
    from vanguard_b200 import workloads as wl

    eu = wl.reduced_params(1.4, 0.0, 1.67, 0.0)
    mh = wl.mhd_reduced_params(1.4, 0.0, 1.67, 0.0)
    bubble, disc = wl.reduced_bubble_2d(n), wl.mhd_reduced_dumbser_2d(n)
    cases = [
        ("euler_reduced", vg.EULER_REDUCED, O.EULER_REDUCED, lambda: bubble, eu, 0, ("fp64", "mixed"), n, n, steps),
        ("euler_multiphysics", vg.EULER_MULTIPHYSICS, O.EULER_MULTIPHYSICS, lambda: wl.multiphysics_from_reduced(bubble),
         eu, 0, ("fp64",), n, n, steps),
        ("mhd_reduced", vg.MHD_REDUCED, O.MHD_REDUCED, lambda: disc, mh, 1, ("fp64",), n, n, steps),
        ("mhd_intermediate", vg.MHD_INTERMEDIATE, O.MHD_INTERMEDIATE, lambda: wl.mhd_intermediate_from_reduced(disc),
         mh, 1, ("fp64",), n, n, steps),
    ]
    hn, hs, m1d = TM_HPR_N, TM_HPR_STEPS, TM_1D_CELLS
    # two ShockMieGruneisen solids, elastic | plastic, in the layout of the reference's Zhang scenario of these models
    s1 = wl.hpr_shock_mg_params(tau1=0.05)
    s2 = wl.hpr_shock_mg_params(plastic=True, sigma0=1.0, n=1.0, tau1=1.0)
    hp = wl.hpr_two_params(s1, s2)
    zv = ((0.0, 0.2, 0.1), (0.0, -0.03, -0.01))
    cases += [
        ("hpr_reduced", vg.HPR_REDUCED, O.HPR_REDUCED,
         lambda: wl.hpr_two_solid_riemann(hn, s1, s2, *wl.ZHANG_F, *zv, ny=hn), hp, 1, ("fp64",), hn, hn, hs),
        ("hpr_intermediate", vg.HPR_INTERMEDIATE, O.HPR_INTERMEDIATE,
         lambda: wl.hpr_intermediate_from_reduced(wl.hpr_two_solid_riemann(hn, s1, s2, *wl.ZHANG_F, *zv, ny=hn)), hp,
         1, ("fp64",), hn, hn, hs),
        ("hpr_multiphysics", vg.HPR_MULTIPHYSICS, O.HPR_MULTIPHYSICS,
         lambda: wl.hpr_multiphysics_from_reduced(wl.hpr_two_solid_riemann(m1d, s1, s2, *wl.ZHANG_F, *zv)), hp, 0,
         ("fp64",), m1d, 1, steps),
        ("mhd_multiphysics", vg.MHD_MULTIPHYSICS, O.MHD_MULTIPHYSICS, lambda: wl.mhd_multiphysics_dumbser_1d(m1d),
         wl.mhd_multiphysics_params(1.4, 0.0, 1.67, 0.0), 0, ("fp64",), m1d, 1, steps),
    ]
    if models:  # profiling runs of a subset
        cases = [c for c in cases if c[0] in models]
    precisions = {"fp64": vg.FP64, "mixed": vg.MIXED}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cores = O.ref().vgref_set_threads(0) if (CPU_LEGS and O.ref_available()) else 0
    out = {"workload": f"2D {n}x{n}, gamma 1.4 | 1.67, superbee, CFL 0.8, {steps} steps, reinitialisation every "
                       f"{TM_REINIT} steps, MHD models with 1 GLM sub-cycle; HPR reduced and intermediate 2D {hn}x{hn} "
                       f"ShockMieGruneisen solids elastic | plastic, {hs} steps, 1 RK4 relaxation sub-cycle; HPR and "
                       f"MHD multiphysics 1D {m1d} cells, {steps} steps"}
    for name, model, omodel, make, prm, sub, forms, nx, ny, nsteps in cases:
        W = make()
        dx = 1.0 / nx
        res = {"grid": [nx, ny], "steps": nsteps}
        for form in forms:
            with vg.Solver(model, nx, ny, prm, precision=precisions[form], device=local) as s:
                s.upload(W, stream=sh)
                s.autotune(dx, CFL, limiter=LIMITER, stream=sh)
                s.run(dx, CFL, steps=3, limiter=LIMITER, subcycles=sub, reinit=TM_REINIT, stream=sh, allow_nan=True)
                s.upload(W, stream=sh)
                torch.cuda.synchronize()
                e0.record(stream)
                s.run(dx, CFL, steps=nsteps, limiter=LIMITER, subcycles=sub, reinit=TM_REINIT, stream=sh,
                      allow_nan=True)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                final = s.download(stream=sh)
            res[form] = {"ms": ms, "cell_updates_per_s": nx * ny * nsteps / (ms / 1e3),
                         "finite": bool(np.isfinite(final).all())}
        if cores:
            if ny > 1:
                rows = 4 if name.startswith("hpr") else 16  # the reference's HPR models run ~3e3 cell-updates/s
                strip = np.ascontiguousarray(W[:, ny // 2 - rows // 2: ny // 2 + rows // 2, :])
                what = f"a {nx}x{rows} strip"
            else:
                seg = nx // 64
                strip = np.ascontiguousarray(W[:, nx // 2 - seg // 2: nx // 2 + seg // 2])
                what = f"a {seg}-cell segment about the interface"
            t0 = time.perf_counter()
            O.run_two_material(omodel, strip, dx, CFL, steps=2, limiter=LIMITER, params=prm, reinit=TM_REINIT,
                               subcycles=sub, reference=True, threads=cores)
            dt = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": strip[0].size * 2 / dt, "unit": UNIT, "cores": cores, "kind": "reference",
                                   "sample": f"2 steps of the reference per-step loop on {what} ({dt:.2f} s)"}
            res["fp64_vs_cpu_reference"] = res["fp64"]["cell_updates_per_s"] / res["cpu_baseline"]["value"]
        out[name] = res
    return out


LEGS = {"c5": lambda l, st, sh: ragged_adjoint_leg(l, st, sh),
        "c4": lambda l, st, sh: hpr_leg(l, st, sh),
        "c3": lambda l, st, sh: mhd_leg(l, st, sh),
        "c1": lambda l, st, sh: sod_leg(l, st, sh),
        "tm": lambda l, st, sh: two_material_leg(l, st, sh, n=TM_N, steps=TM_STEPS, models=TM_MODELS)}


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def vg_mixed_available(vg):
    try:
        s = vg.Solver(vg.EULER, 8, 8, (1.4, 0.0), precision=vg.MIXED)
        s.close()
        return True
    except Exception:
        return False


def load_traffic(form):
    """DRAM bytes per X-sweep launch of `form` at the bench size, from the committed ncu summaries, if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(f"sweep_x_kernel_{form}_bytes_per_launch")
    except Exception:
        return None


def main():
    global NX, NY, C5_NINST, C5_STEPS, C4_STEPS, TM_N, TM_STEPS, TM_MODELS, C3_N, C3_STEPS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true", help="skip the C1/C3/C5 measurements")
    ap.add_argument("--legs", default="headline,c5,c4,c3,c1,tm",
                    help="comma list of headline (C2), c5, c4, c3, c1, tm (two-material models); without headline "
                         "only those legs run (profiling)")
    ap.add_argument("--forms", default="fp64,mixed", help="C2 forms to run (profiling)")
    ap.add_argument("--c5-ninst", type=int, default=4096, help="C5 instances (smaller is for profiling only)")
    ap.add_argument("--c5-steps", type=int, default=500, help="C5 steps (smaller is for profiling only)")
    ap.add_argument("--c4-steps", type=int, default=300, help="C4 steps (smaller is for profiling only)")
    ap.add_argument("--c3-steps", type=int, default=C3_STEPS, help="C3 steps (smaller is for profiling only)")
    ap.add_argument("--c3-n", type=int, default=C3_N, help="C3 grid size (smaller is for profiling only)")
    ap.add_argument("--tm-steps", type=int, default=TM_STEPS, help="two-material steps (smaller is for profiling only)")
    ap.add_argument("--tm-models", default="", help="two-material models to run, comma list (profiling only)")
    ap.add_argument("--tm-n", type=int, default=TM_N, help="two-material grid size (smaller is for profiling only)")
    ap.add_argument("--nx", type=int, default=4096, help="grid size (smaller grids are for profiling only)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    NX = NY = args.nx
    C5_NINST, C5_STEPS, C4_STEPS = args.c5_ninst, args.c5_steps, args.c4_steps
    C3_N, C3_STEPS = args.c3_n, args.c3_steps
    TM_N, TM_STEPS, TM_MODELS = args.tm_n, args.tm_steps, [m for m in args.tm_models.split(",") if m] or None
    if args.headline_only:
        args.legs = "headline"
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_cuda(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
