#!/usr/bin/env python
"""Benchmark of the tjsq hot path on B200: H*psi per second on a 4x24 t-J
cylinder superblock at m = 2000 multiplets (mid-chain, 12 holes, S = 0),
split-precision ("mixed": int8 slices on the tensor cores, FP64 elsewhere)
against the plain FP64 GPU path.

One "step" is one H*psi (hmerge'd model_wave) over the whole superblock with
operators and psi resident in HBM.  The superblock is synthetic (seeded):
sector tables, bases and operator blocks with the reference's quantum-number
structure at the sizes of that configuration (no DMRG run of the reference
can be reproduced here).  Its operators (about 0.2 GB), slice pools (about
0.5 GB) and phase-1 products (about 0.14 GB) exceed the 126 MB L2, so no
explicit L2 flush is done.

  python bench.py [--gpus N --steps K --warmup W --impl b200|reference
                   --precision mixed|fp64|ozaki --slices S]

mixed (default): the split-precision H*psi is the timed value; an FP64 leg
gives the speed-up, and Lanczos in both precisions from the same start
vector gives |dE|/site and ||psi - psi_FP64||.  The end-to-end leg is
tj_lanczos_memo_new through the C ABI with host buffers, followed by the
system-block truncation (one DMRG step of the hot path).

--impl reference times the oracle (the C restatement of the reference's
Fortran routines, FP64, OpenBLAS with every host thread) on the same
workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H·ψ/s & sweep time, 4×24 t-J m=2000: mixed vs FP64 GPU at ΔE/site≤1e-9"
UNIT = "H*psi/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="cyl4x24_m2000")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "ozaki"],
                    help="mixed: split-precision H*psi timed, FP64 leg for the speed-up and the accuracy check")
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end Lanczos leg (profiling runs)")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default tiling)")
    ap.add_argument("--no-microbench", action="store_true", help="skip the grouped block-GEMM microbenchmark")
    ap.add_argument("--sweep", default="cyl4x24_m2000", choices=["cyl4x24_m2000", "cyl4x24_m500", "ladder16_m256", "none"],
                    help="real DMRG run whose full sweep is timed (FP64 and split precision from the same state)")
    ap.add_argument("--sweep-prep", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the untimed warm-up and first half-sweeps before the timed sweeps")
    ap.add_argument("--config5", action="store_true",
                    help="also run configuration 5's four dopings as real DMRG runs on a 6-leg cylinder, with "
                         "their pair and density correlators and shared-launch H*psi")
    ap.add_argument("--config5-nx", type=int, default=12, help="columns of the 6-leg cylinder of --config5")
    ap.add_argument("--config5-m", type=int, default=500, help="kept multiplets of --config5")
    ap.add_argument("--config5-sweeps", type=int, default=2, help="full sweeps of each --config5 run")
    ap.add_argument("--instances", type=int, default=1,
                    help="K > 1: also time K independent superblocks (dopings 1/12, 1/10, 1/8, 1/6, ...) in shared "
                         "launches against the same K run one after another")
    return ap.parse_args()


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region can be shorter than nvidia-smi's start-up: wait
            # (up to 3 s) for its first sample, so that the region is covered
            t0 = time.time()
            while not self.rows and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, n in enumerate(names):
                    if r[4 + k].lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                pass
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return ws, rank, local, pg


def allmax(pg, x: float, impl: str) -> float:
    if pg is None:
        return x
    import torch
    dev = "cuda" if impl == "b200" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, impl):
    if pg is not None:
        if impl == "b200":
            import torch
            pg.barrier(device_ids=[torch.cuda.current_device()])
        else:
            pg.barrier()


def fp64_peak_tflops(device: int) -> float:
    """cuBLAS DGEMM throughput on this GPU (best of a few 8192^3 products)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda:%d" % device)
    b = torch.randn(n, n, dtype=torch.float64, device="cuda:%d" % device)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def cpu_reference(sb, steps: int, warmup: int, threads: int):
    """Times the oracle's model_wave (hmerge included) on the host."""
    from oracle import oracle
    oracle.lib(threads)
    oracle.set_threads(threads)
    for _ in range(warmup):
        oracle.model_wave(sb)
    t = time.perf_counter()
    for _ in range(steps):
        oracle.model_wave(sb)
    dt = time.perf_counter() - t
    return steps / dt, dt / steps


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def profile_traffic(workload: str, precision: str, launch: str):
    """DRAM bytes (read + write) of one launch from the committed ncu capture summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_inputs.json")) as f:
            d = json.load(f)
        return d.get(workload, {}).get(precision, {}).get(launch)
    except Exception:
        return None


def int8_peak_tops(device: int) -> float:
    """cuBLASLt int8 GEMM throughput on this GPU (torch._int_mm, best of a few 8192^3 products)."""
    import torch
    n = 8192
    a = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda:%d" % device)
    b = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda:%d" % device)
    torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def run_leg(ctx, sb, steps: int, warmup: int):
    """Device-timed H*psi on a resident superblock: (ms per H*psi, stats)."""
    ctx.model_wave_bench(sb, max(warmup, 3))
    ms, _ = ctx.model_wave_bench(sb, steps)
    return ms, ctx.stats()


def lanczos_leg(ctx, sb, lanzero: float, packed):
    """tj_lanczos_memo_new through the C ABI with host buffers: the timed call
    compiles the plan, uploads the operators from pinned host memory, runs the
    Lanczos iterations and downloads the Ritz vector into the caller's wave."""
    ctx.step_begin()
    w = sb.wave.copy()
    t0 = time.perf_counter()
    e0, iters, w = ctx.lanczos_memo_new(sb, lanzero, start=w, packed=packed, in_place=True)
    wall = time.perf_counter() - t0
    return e0, iters, w, wall, ctx.stats()


SWEEPS = {
    # nx, ny, electrons, kept_max: the 4x24 cylinder at 12 holes (delta = 1/8), the 2x16 ladder at 4 holes
    "cyl4x24_m2000": (24, 4, 84, 2000),
    "cyl4x24_m500": (24, 4, 84, 500),
    "ladder16_m256": (16, 2, 28, 256),
}


RESIDENCY_GB = 48.0   # blocks kept on the device during a sweep (tj_set_residency)


def sweep_leg(ctx64, ctxoz, name: str, prep: str, seed: int):
    """A real DMRG run of the reference's schedule (grand_sql_tj_b200.sweep,
    main.f90:96-187) through the C ABI on the device: warm-up and the first two
    half-sweeps untimed (at the reference's looser thresholds), then one full
    sweep (left to right and back, at lanzero = 2e-5) timed in FP64 and one in
    split precision, both from the same state (each after an untimed sweep
    of its own precision from it that fills the page-locked buffer pool).  Every DMRG step is Lanczos +
    truncation + operator renormalisation + wavefunction prediction, with
    host buffers in and out (the drop-in's calling pattern) and the blocks
    the library returns also kept on the device (tj_set_residency), so that
    the next steps read them without a host upload, and written into
    page-locked host buffers that are reused (HostPool)."""
    import numpy as np
    from grand_sql_tj_b200.lattice import Geometry
    from grand_sql_tj_b200.lib import DeviceBackend
    from grand_sql_tj_b200.sweep import Dmrg, DmrgParams
    nx, ny, ne, m = SWEEPS[name]
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=0.0, esite=0.0, up_bias=1)
    lanerr = float(np.float32(20.0e-6))
    p = DmrgParams(n_elec=ne, kept_min=3 * m // 4, kept_max=m, trun_err=1e-18, lanzero=lanerr,
                   lanzero_warm=lanerr * 1000, seed=seed)
    N = geo.num_site
    for c in (ctx64, ctxoz):
        if c is not None:
            c.set_residency(RESIDENCY_GB)
            c.use_host_pool(True)
    d = Dmrg(geo, DeviceBackend(ctxoz if (prep == "mixed" and ctxoz is not None) else ctx64), p)
    t0 = time.perf_counter()
    d.warm_up()
    d.left_to_right(N // 2 - 1, N - 2, restart=False, lanzero=lanerr * 30, trun_err=1e-18 * 15, phase="L->R0")
    d.right_to_left(N - 2, 1, restart=True, lanzero=lanerr * 30, trun_err=1e-18 * 15, phase="R->L0")
    prep_s = time.perf_counter() - t0
    snap = ({k: dict(getattr(d, k)) for k in ("sysblocks", "envblocks", "systruns", "envtruns", "sysbs", "envbs")},
            d.wave.copy(), d.rng.bit_generator.state)
    out = {"lattice": "%dx%d" % (ny, nx), "electrons": ne, "m": m, "prep_s": prep_s, "prep_precision": prep,
           "residency_gb": RESIDENCY_GB,
           "steps_per_sweep": 2 * (N - 3)}

    def one(ctx, tag):
        for k, v in snap[0].items():
            setattr(d, k, dict(v))
        d.wave = snap[1].copy()
        d.rng.bit_generator.state = snap[2]
        # both timed sweeps start with nothing kept on the device: the blocks
        # of the snapshot are uploaded once, then each new block stays resident
        for c in (ctx64, ctxoz):
            if c is not None:
                c.set_residency(0)
        ctx.set_residency(RESIDENCY_GB)
        trace = []
        d.be = DeviceBackend(ctx, trace)
        n0 = len(d.records)
        t = time.perf_counter()
        d.left_to_right(1, N - 2, restart=True, phase="L->R")
        d.right_to_left(N - 2, 1, restart=True, phase="R->L")
        wall = time.perf_counter() - t
        recs = d.records[n0:]
        agg = {k: sum(getattr(r, k) for r in recs) for k in ("t_lanczos", "t_trunc", "t_renorm", "t_pred")}
        out[tag] = {"sweep_s": wall, "steps": len(recs), "lanczos_vectors": sum(r.iters for r in recs),
                    "E_end": recs[-1].energy, "E_min": min(r.energy for r in recs),
                    "max_trunc_err": max(r.trunc_err for r in recs), "max_psi_dim": max(r.dim for r in recs),
                    "seconds": {k[2:]: v for k, v in agg.items()}}
        tr = [st for name, st, _, _ in trace if name == "truncation"]
        stages = ("rho", "tridiag", "eig", "select", "vec", "orth", "back", "total")
        out[tag]["truncation_ms"] = {k: sum(getattr(st, "trunc_ms_" + k) for st in tr) for k in stages}
        out[tag]["truncation_ms"]["max_sector"] = max(st.trunc_max_n for st in tr)
        out[tag]["truncation_ms"]["max_kept_block"] = max(st.trunc_max_kept for st in tr)
        rn = [st for name, st, _, _ in trace if name == "get_hamiltonian"]
        rh = [h for name, _, _, h in trace if name == "get_hamiltonian"]
        out[tag]["renorm_ms"] = {"plan": sum(st.renorm_plan_ms for st in rn), "gemm": sum(st.renorm_ms for st in rn),
                                 "call": sum(st.renorm_e2e_ms for st in rn),
                                 "tflops": sum(st.renorm_flops for st in rn) / max(sum(st.renorm_ms for st in rn), 1e-9) / 1e9,
                                 "wall": 1e3 * sum(w for name, _, w, _ in trace if name == "get_hamiltonian"),
                                 "host_pre": sum(st.renorm_pre_ms for st in rn),
                                 "host_post": sum(st.renorm_post_ms for st in rn)}
        for k in ("sizes", "alloc", "fill", "wrap"):
            out[tag]["renorm_ms"]["host_" + k] = 1e3 * sum(h.get(k, 0.0) for h in rh)
        lz = [st for name, st, _, _ in trace if name == "lanczos"]
        out[tag]["lanczos_ms"] = {"prepare": sum(st.prepare_ms for st in lz), "plan": sum(st.plan_ms for st in lz),
                                  "split_plan": sum(st.ozplan_ms for st in lz),
                                  "upload": sum(st.upload_ms for st in lz),
                                  "wall": 1e3 * sum(w for name, _, w, _ in trace if name == "lanczos"),
                                  "iterations": sum(st.lanczos_ms for st in lz)}
        # the prediction's library call; the rest of `pred` is the driver's
        # bases of the new superblock
        wt = [st for name, st, _, _ in trace if name == "wave_trans"]
        out[tag]["wave_trans_ms"] = {"wall": 1e3 * sum(w for name, _, w, _ in trace if name == "wave_trans"),
                                     "plan": sum(st.wt_plan_ms for st in wt), "device": sum(st.wt_ms for st in wt)}
        return recs

    # an untimed sweep from the same state before each timed one: a running
    # DMRG reuses the page-locked buffers of the blocks it replaces, and the
    # snapshot keeps the replaced blocks alive, so the pool is filled first
    # (with the sizes of that precision's run, which differ a little)
    one(ctx64, "untimed")
    r64 = one(ctx64, "fp64")
    if ctxoz is not None:
        one(ctxoz, "untimed")
        rmx = one(ctxoz, "mixed")
    del out["untimed"]
    if ctxoz is not None:
        out["speedup_vs_fp64"] = out["fp64"]["sweep_s"] / out["mixed"]["sweep_s"]
        out["dE_per_site_end"] = abs(out["fp64"]["E_end"] - out["mixed"]["E_end"]) / N
        out["dE_per_site_max_step"] = max(abs(a.energy - b.energy) for a, b in zip(r64, rmx)) / N
    return out


CONFIG5_DOPINGS = (1.0 / 12, 1.0 / 10, 1.0 / 8, 1.0 / 6)


def config5_leg(ctx, nx: int, m: int, sweeps: int, seed: int):
    """Configuration 5 at a size one run can take: the 6-leg cylinder of nx
    columns (y periodic, x open; t = 1, t' = -0.2, J = 1/3, S = 0) at the four
    dopings, holes rounded to even numbers.  Each is a DMRG run of the
    reference's schedule on the device (split-precision H*psi, FP64
    truncation, renormalisation and prediction; blocks kept resident),
    followed by the singlet pair (along y and x) and density correlators of
    Measurement (main.f90:191-332).  Then the H*psi of the four
    measurement-point superblocks in shared launches (tj_model_wave_multi)
    against the four one after another, with the two results compared."""
    import numpy as np
    from grand_sql_tj_b200.lattice import Geometry
    from grand_sql_tj_b200.lib import DeviceBackend
    from grand_sql_tj_b200.measure import measurement
    from grand_sql_tj_b200.sweep import Dmrg, DmrgParams
    n = 6 * nx
    out = {"lattice": "6x%d cylinder (y periodic, x open)" % nx, "t": 1.0, "t2": -0.2, "J": 1.0 / 3.0, "m": m,
           "sweeps": sweeps, "instances": []}
    ctx.set_residency(RESIDENCY_GB)
    ctx.use_host_pool(True)
    lasts = []
    for delta in CONFIG5_DOPINGS:
        holes = 2 * int(n * delta / 2.0 + 0.5)   # rounded half up to an even number
        geo = Geometry(nx, 6, t=1.0, J=1.0 / 3.0, t2=-0.2, esite=0.0, up_bias=1)
        d = Dmrg(geo, DeviceBackend(ctx), DmrgParams(n_elec=n - holes, kept_min=3 * m // 4, kept_max=m, seed=seed))
        t0 = time.perf_counter()
        d.ground_state(sweeps, final_half=True)
        run_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        cors = measurement(DeviceBackend(ctx), d)
        meas_s = time.perf_counter() - t0
        last_sweep = [r for r in d.records if r.phase == "R->L%d" % sweeps]
        lasts.append(d.last)
        out["instances"].append({
            "delta": delta, "holes": holes, "electrons": n - holes, "E_per_site": d.records[-1].energy / n,
            "max_trunc_err_last_sweep": max(r.trunc_err for r in last_sweep), "run_s": run_s, "steps": len(d.records),
            "measure_s": meas_s,
            "pair_y": [[*k, v] for k, v in sorted(cors["pair_y"].items())],
            "pair_x": [[*k, v] for k, v in sorted(cors["pair_x"].items())],
            "density": [[*k, v] for k, v in sorted(cors["density"].items())]})
    outs, ms_shared = ctx.model_wave_multi(lasts, reps=20)
    ms_seq, diff = 0.0, 0.0
    for sb, o in zip(lasts, outs):
        ms1, single = ctx.model_wave_bench(sb, 20)
        ms_seq += ms1
        a, b = o.data[:o.dim], single.data[:single.dim]
        diff = max(diff, float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)))
    out["shared_launch"] = {"psi_dims": [sb.wave.dim for sb in lasts], "shared_ms": ms_shared,
                            "sequential_ms": ms_seq, "speedup": ms_seq / ms_shared,
                            "max_rel_diff_shared_vs_single": diff}
    ctx.set_residency(0)
    return out


def main():
    args = parse()
    ws, rank, local, pg = dist_init(args)
    from grand_sql_tj_b200 import synth
    sb = synth.workload(args.workload, seed=args.seed + (rank if args.impl == "b200" else 0))
    cfg = {"workload": args.workload, "lattice": "4x24 cylinder (y periodic, x open)" if "4x24" in args.workload else args.workload,
           "m": 2000 if "m2000" in args.workload else None, "t": 1.0, "J": 1.0 / 3.0, "holes": 12,
           "sys_len": sb.sys.len, "env_len": sb.env.len, "psi_dim": sb.wave.dim,
           "sectors": len(sb.wave.sectors), "l2": "inputs larger than L2 (no flush)",
           "parallelism": "replicas" if ws > 1 else "single"}

    if args.impl == "reference":
        if rank != 0:
            barrier(pg, args.impl)
            return
        threads = os.cpu_count() or 1
        steps = max(1, min(args.steps, 8))
        warm = min(args.warmup, 1)
        rate, sec = cpu_reference(sb, steps, warm, threads)
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": ws,
                "steps": steps, "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": cfg,
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": "%d model_wave calls of the oracle (C restatement of get_sys.f90 "
                                           "model_wave + hmerge, OpenBLAS dgemm)" % steps},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        barrier(pg, args.impl)
        return

    from grand_sql_tj_b200 import build as B
    B.build()
    import numpy as np
    from grand_sql_tj_b200.lib import Context, TJ_PREC_OZAKI
    mixed = args.precision in ("mixed", "ozaki")
    ctx64 = Context(local)
    ctxoz = None
    if mixed:
        ctxoz = Context(local)
        ctxoz.set_precision(TJ_PREC_OZAKI, args.slices)
    head = ctxoz if mixed else ctx64
    # the autotuner's tiling for this superblock, in both precisions (untimed)
    tune = {}
    if not args.no_tune:
        if mixed:
            tune["mixed"] = ctxoz.autotune(sb).as_dict()
        if args.precision != "ozaki":
            tune["fp64"] = ctx64.autotune(sb).as_dict()
    # untimed legs first: the other precision (for the speed-up) and warm-up
    ms64 = st64 = None
    if args.precision == "mixed":
        ms64, st64 = run_leg(ctx64, sb, max(20, args.steps // 4), args.warmup)
    head.model_wave_bench(sb, max(args.warmup, 3))
    barrier(pg, args.impl)
    with Clocks(local) as clk:
        barrier(pg, args.impl)
        t0 = time.perf_counter()
        ms, _ = head.model_wave_bench(sb, args.steps)
        wall = time.perf_counter() - t0
        barrier(pg, args.impl)
    st = head.stats()
    ms_max = allmax(pg, ms, args.impl)
    value = ws * 1000.0 / ms_max

    e2e = accuracy = step = None
    if not args.no_e2e:
        # end to end through the reference-facing call (host buffers), at the
        # reference's sweep threshold lanzero = 2e-5
        lz = 20.0e-6
        from grand_sql_tj_b200.lib import PinnedHost, pack_superblock, packed_arrays
        packed = pack_superblock(sb)
        pinned = PinnedHost(packed_arrays(packed))
        # one untimed solve (first-use costs: graph instantiation, lazy module
        # loads), then the median of three timed solves
        lanczos_leg(head, sb, lz, packed)
        runs = sorted((lanczos_leg(head, sb, lz, packed) for _ in range(3)), key=lambda r: r[3])
        e0, iters, w, e2e_wall, st2 = runs[1]
        e2e_walls = [r[3] for r in runs]
        del runs
        nh = max(int(st2.lanczos_hpsi), 1)
        e2e_wall = allmax(pg, e2e_wall, args.impl)
        ops_bytes = 0
        for m in (sb.sys, sb.env):
            ops_bytes += sum(s.mat.size for s in m.ham.subs) * 8
            for bs in m.sub:
                for k in ("elec_up", "elec_down", "spin_sd", "num_sn"):
                    ops_bytes += sum(s.mat.size for s in getattr(bs, k).subs) * 8
        e2e = {"value": ws * nh / e2e_wall, "unit": UNIT, "via": "tj_lanczos_memo_new (plan + operator upload from "
               "pinned host memory + %d H*psi + Ritz vector download)" % nh,
               "h2d_bytes_per_step": int((ops_bytes + 8 * sb.wave.dim) / nh),
               "d2h_bytes_per_step": int(8 * sb.wave.dim / nh), "lanczos_iters": iters, "E0": e0,
               "timed_solves_s": e2e_walls, "statistic": "median of 3 solves after 1 untimed",
               "breakdown_ms": {"prepare": st2.prepare_ms, "plan_compile": st2.plan_ms,
                                "operator_upload": st2.upload_ms, "split_plan": st2.ozplan_ms,
                                "lanczos_iterations": st2.lanczos_ms}}
        # the same solve with the operators in ordinary (pageable) host memory,
        # as a Fortran driver that reads its blocks from disk each step holds them
        pinned.close()
        lanczos_leg(head, sb, lz, packed)
        runs = sorted((lanczos_leg(head, sb, lz, packed) for _ in range(3)), key=lambda r: r[3])
        st3 = runs[1][4]
        e2e["unpinned"] = {"value": ws * max(int(st3.lanczos_hpsi), 1) / allmax(pg, runs[1][3], args.impl),
                           "unit": UNIT, "timed_solves_s": [r[3] for r in runs],
                           "operator_upload_ms": st3.upload_ms, "prepare_ms": st3.prepare_ms}
        del runs
        # one DMRG step of the hot path: Lanczos + truncation of the system block
        # (a sweep calls it every step: one untimed call, then the median of three)
        t0 = time.perf_counter()
        kept = head.truncation(w, 0, 2000, 2000, 1e-12)
        trunc_first_s = time.perf_counter() - t0
        trunc_runs = []
        for _ in range(3):
            del kept
            t0 = time.perf_counter()
            kept = head.truncation(w, 0, 2000, 2000, 1e-12)
            trunc_runs.append(time.perf_counter() - t0)
        trunc_s = sorted(trunc_runs)[1]
        nsite = sb.geo.num_site
        step = {"lanczos_s": e2e_wall, "truncation_s": trunc_s, "truncation_first_call_s": trunc_first_s,
                "dmrg_step_s": e2e_wall + trunc_s,
                "note": "synthetic mid-chain superblock: Lanczos from its seeded start vector + truncation "
                        "(median of 3 calls after 1 untimed); the measured sweep is in `sweep`"}
        if mixed:
            # the split-precision result against FP64 on the same start vector and threshold
            e64, it64, w64, wall64, _ = lanczos_leg(ctx64, sb, lz, packed)
            ov = float(np.dot(w.data, w64.data))
            dpsi = float(np.linalg.norm(w.data - np.sign(ov) * w64.data))
            de = abs(e0 - e64) / nsite
            accuracy = {"E0_mixed": e0, "E0_fp64": e64, "dE_per_site": de, "psi_diff_norm": dpsi,
                        "iters_mixed": iters, "iters_fp64": it64, "ok": bool(de <= 1e-9),
                        "fp64_lanczos_s": wall64}
        del kept
        pinned.close()

    sweep = None
    if args.sweep != "none" and rank == 0 and not args.no_e2e:
        sweep = sweep_leg(ctx64, ctxoz, args.sweep, args.sweep_prep, args.seed)

    config5 = None
    if args.config5 and rank == 0:
        config5 = config5_leg(ctxoz if ctxoz is not None else ctx64, args.config5_nx, args.config5_m,
                              args.config5_sweeps, args.seed)

    shared = None
    if args.instances > 1:
        # independent instances of the same lattice at several dopings, one set of launches
        geo = {"cyl4x24_m2000": (24, 4, 47, 47, 2000, {}), "cyl4x24_m500": (24, 4, 47, 47, 500, {}),
               "cyl6x24_m6000": (24, 6, 71, 71, 6000, {"t2": -0.2})}[args.workload]
        nx, ny, ls, le, m, kw = geo
        dop = [1 / 12, 1 / 10, 1 / 8, 1 / 6, 1 / 14, 1 / 5, 1 / 16, 1 / 4][:args.instances]
        ns = nx * ny
        sbs = [synth.make_superblock(nx, ny, ls, le, m, ns - 2 * int(round(d * ns / 2)), args.seed + i, **kw)
               for i, d in enumerate(dop)]
        outs, ms_shared = head.model_wave_multi(sbs, reps=20)
        sep = [head.model_wave_bench(s_, 20)[0] for s_ in sbs]
        shared = {"instances": len(sbs), "dopings": dop, "holes": [ns - s_.tot_num_up if s_.tot_num_up else None
                                                                   for s_ in sbs],
                  "psi_dims": [s_.wave.dim for s_ in sbs], "shared_ms": ms_shared, "separate_ms": sep,
                  "separate_ms_sum": sum(sep), "shared_speedup": sum(sep) / ms_shared,
                  "hpsi_per_s_shared": len(sbs) * 1000.0 / ms_shared}
        del sbs, outs

    micro = None
    if rank == 0 and not args.no_microbench:
        # grouped block-GEMM microbenchmark: 400 sector pairs, dims log-uniform in
        # [8, 1024], 4..16 terms each; one persistent grouped launch (autotuned
        # tiling) against one launch per block GEMM
        from grand_sql_tj_b200 import gg
        gb = gg.make_batch(n_cells=400, seed=args.seed)
        g_ms, g_out, g_fl, g_tr = ctx64.grouped_gemm_bench(gb, 2, reps=3)
        p_ms, p_out, _, _ = ctx64.grouped_gemm_bench(gb, 1, reps=1)
        micro = {**gb.spec, "flops": g_fl, "grouped_ms": g_ms, "grouped_tflops": g_fl / (g_ms * 1e-3) / 1e12,
                 "per_block_ms": p_ms, "per_block_launches": gb.spec["terms"],
                 "per_block_tflops": g_fl / (p_ms * 1e-3) / 1e12, "grouped_speedup": p_ms / g_ms,
                 "max_diff_rel": float(np.max(np.abs(g_out - p_out)) / max(np.max(np.abs(p_out)), 1e-300)),
                 "tuned": g_tr.as_dict() if g_tr is not None else None, "dtype": "f64"}
        del gb, g_out, p_out

    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(local) if rank == 0 else None
    if mixed:
        i8 = int8_peak_tops(local) if rank == 0 else None
        t1, t2 = st.last_ms_phase1, st.last_ms_phase2
        dom = 1 if t1 >= t2 else 2
        tdom = max(t1, t2)
        s_ = args.slices
        alg = (st.flops_launch1 if dom == 1 else st.flops_launch2) * s_ * (s_ + 1) / 2
        issued = st.int8_ops_launch1 if dom == 1 else st.int8_ops_launch2
        achieved = alg / (tdom * 1e-3) / 1e12
        roof = {"bound": "tensor", "kernel": "oz_gemm_kernel (launch %d)" % dom, "achieved": achieved,
                "peak": i8, "unit": "TFLOP/s", "frac": (achieved / i8) if i8 else None,
                "traffic": profile_traffic(args.workload, "ozaki", "launch%d" % dom),
                "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                "peak_source": "measured cuBLASLt int8 GEMM 8192^3 (torch._int_mm) on this GPU; int8 ops",
                "work": "algorithmic int8 ops = FP64-equivalent flops of the launch x s(s+1)/2 slice products",
                "issued_int8_ops": issued, "launch_ms": tdom,
                "launch1_ms": t1, "launch2_ms": t2, "splits_ms": st.last_ms_split,
                "fp64_equiv_tflops": st.flops / (ms * 1e-3) / 1e12,
                "fp64_dgemm_peak_tflops": fp64}
    else:
        achieved = st.flops / (ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "kernel": "grouped_gemm_kernel (both phases)", "achieved": achieved,
                "peak": fp64, "unit": "TFLOP/s", "frac": (achieved / fp64) if fp64 else None,
                "traffic": profile_traffic(args.workload, "fp64", "per_hpsi"),
                "traffic_unit": "bytes per H*psi, both launches (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                "peak_source": "measured cuBLAS DGEMM 8192^3 on this GPU (FP64; not in MEASURED_PEAKS.json)",
                "phase1_ms": st.last_ms_phase1, "phase2_ms": st.last_ms_phase2}
    roof.update({"flops_per_hpsi": st.flops, "flops_ref_per_hpsi": st.flops_ref, "bytes_per_hpsi": st.bytes,
                 "hbm_frac": (st.bytes / (ms * 1e-3) / 1e9) / peaks.get("hbm_gbs", 6555.8)})
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, sec = cpu_reference(sb, 2, 0, threads)
        rate1, sec1 = cpu_reference(sb, 1, 0, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": "2 model_wave calls of the oracle on the same superblock",
               "single_thread": {"value": rate1, "unit": UNIT, "cores": 1,
                                 "sample": "1 model_wave call of the oracle, OPENBLAS 1 thread"}}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_max, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "int8 slices (s=%d) + f64" % args.slices if mixed else "f64",
                "data": "synthetic", "config": cfg,
                "precision": "mixed" if mixed else "fp64",
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
                "gpu_launches": int(st.kernels_per_hpsi) * args.steps, "wall_s_timed": wall}
        if ms64 is not None:
            line["fp64"] = {"value": ws * 1000.0 / ms64, "ms_per_step": ms64, "unit": UNIT,
                            "phase1_ms": st64.last_ms_phase1, "phase2_ms": st64.last_ms_phase2}
            line["speedup_vs_fp64"] = ms64 / ms
        if accuracy is not None:
            line["accuracy"] = accuracy
        if step is not None:
            line["dmrg_step"] = step
        if sweep is not None:
            line["sweep"] = sweep
        if config5 is not None:
            line["config5"] = config5
        if tune:
            line["autotune"] = tune
        if micro is not None:
            line["grouped_gemm_microbench"] = micro
        if shared is not None:
            line["shared_launch"] = shared
        print(json.dumps(line), flush=True)
    ctx64.close()
    if ctxoz is not None:
        ctxoz.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
