#!/usr/bin/env python
"""Benchmark: matrix-free H·v of the 2D extended Hubbard model on the 4x4 periodic square,
sector (N_up, N_dn) = (8, 8), dim C(16,8)^2 = 165,636,900, complex128 vectors,
t=1, t'=-0.25, U=8, V=1, phi_x=0.1, phi_y=0 (complex hoppings on the x-wrap bonds).

One step = one H·v (y = H x) through the C ABI (ftlm_gpu_apply).  Inputs (2.65 GB per vector)
are larger than L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: every rank applies H to its own vector (independent units, no collective on the data
path); value = all ranks' H·v / max-over-ranks device time ("scaling": "weak").
--impl reference times the reference's own CPU apply_extended_hubbard (oracle/_ref, built from the
reference sources) on bounded column samples of the same sector with all usable host threads.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LX, LY, NU, ND = 4, 4, 8, 8
PARAMS = dict(Lx=4, Ly=4, t=1.0, tp=-0.25, U=8.0, V=1.0, phi_x=0.1, phi_y=0.0)
METRIC = "4x4(8,8) complex128 H·v/s"
UNIT = "H·v/s"
WORKLOAD = "4x4 periodic, sector (8,8), dim 165636900, complex128 H·v, t=1 t'=-0.25 U=8 V=1 phi_x=0.1"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--sector", type=int, nargs=2, default=None, metavar=("NU", "ND"),
                    help="profile a smaller 4x4 sector instead (for ncu captures); not a bench line")
    ap.add_argument("--workload", default="hv", choices=["hv", "batched", "lanczos", "sweep-model", "orbit", "grad", "kresolved", "published", "sweep"],
                    help="hv: the H·v benchmark (the bench line).  Measurement aids (one JSON line each, not "
                         "bench lines): batched = 32-chain complex64 Lanczos steps on one sector; sweep-model = "
                         "per-sector step cost of the plain and batched paths over the full 4x4 sweep (R=32, "
                         "M=100) and the modelled sweep times; orbit = H_K·v of one momentum block; grad = "
                         "forward and backward of the differentiable 4x3 ln Z_GC (R=32, M=80); kresolved = k-resolved "
                         "sector ln Z (16 orbit blocks, R=24, M=100) against the unsymmetrised batched ln Z "
                         "(R=32, M=100) of the same sector; published = the reference's published n(mu) sweeps "
                         "(beta=20, R=12, M=72) timed on the GPU next to the published CPU times; sweep = the full 4x4 "
                         "grand-canonical sweep, batched complex64 and plain complex128 (same Philox starts), "
                         "R=32, M=100, T=0.1..2 x mu=-4..8 (tens of minutes)")
    ap.add_argument("--k", type=int, nargs=2, default=(1, 2), metavar=("KX", "KY"), help="orbit workload momentum")
    ap.add_argument("--hv-path", type=int, default=0, choices=[0, 1, 2, 3],
                    help="hv workload: pin the H·v kernel path (0 = the autotuner's choice)")
    ap.add_argument("--cols-variant", type=int, default=0, choices=[0, 1, 2, 3, 4, 5],
                    help="with --hv-path: column-slab width variant (0/1/2 = 256/128/512 columns; "
                         "3/4/5 = the same over the packed up list, path 3)")
    ap.add_argument("--bt-cols", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="batched workload: column-pass variant (-1 = the batched autotuner's choice)")
    ap.add_argument("--check", type=int, default=1,
                    help="sweep workload: chains per sector rerun in complex128 for the per-result error estimate")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def mem_available_bytes() -> int:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def usable_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- clocks during the timed region
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
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
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU baseline (oracle port)
def cpu_baseline_port(seconds: float):
    """The oracle restatement (row-gather, all host threads) on a bounded row sample of the sector."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import P, OracleSector  # noqa: E402  (CPU checker / baseline only)
    s = OracleSector(LX, LY, PARAMS["t"], PARAMS["tp"], PARAMS["U"], PARAMS["V"], PARAMS["phi_x"], PARAMS["phi_y"],
                     NU, ND)
    dim = s.dim
    rng = np.random.default_rng(7)
    x = np.empty(dim, np.complex128)
    step = 1 << 24
    for i in range(0, dim, step):
        k = min(step, dim - i)
        x[i:i + k] = rng.standard_normal(k) + 1j * rng.standard_normal(k)
    y = np.zeros(dim, np.complex128)
    th = usable_cores()
    r0 = dim // 3
    n = 200_000
    t0 = time.perf_counter()
    s.L.or_sector_apply_rows(s.h, P(x), P(y), r0, r0 + n, th)
    dt = time.perf_counter() - t0
    n2 = int(min(dim - r0, max(n, n * seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    s.L.or_sector_apply_rows(s.h, P(x), P(y), r0, r0 + n2, th)
    dt = time.perf_counter() - t0
    return {"value": (n2 / dt) / dim, "unit": UNIT, "cores": th, "kind": "port",
            "sample": f"rows [{r0},{r0 + n2}) of y = H x ({n2} of {dim} rows, {dt:.1f} s), oracle/ftlm_oracle.cpp "
                      f"row gather on {th} threads; H·v/s = rows/s / dim"}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C
    from oracle import reference  # noqa: E402  (the reference's own CPU code, timed as the baseline)
    L = reference()
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libftlm_ref.so not built and reference "
                                                               "sources absent"}))
        return 0
    dim = math.comb(16, 8) ** 2
    avail = mem_available_bytes()
    per_thread = 2 * dim * 16
    cores = usable_cores()
    threads = max(1, min(cores, 32, int((0.45 * avail - 12e9) // per_thread) if avail else 1))
    h = L.ref_sector_create(LX, LY, PARAMS["t"], PARAMS["tp"], PARAMS["U"], PARAMS["V"], PARAMS["phi_x"],
                            PARAMS["phi_y"], NU, ND)
    if not h:
        print(json.dumps({"impl": "reference", "unavailable": "reference FockBasis(16,8,8) construction failed"}))
        return 0
    ctx = L.ref_sample_create(h, threads)
    if not ctx:
        L.ref_sector_destroy(h)
        print(json.dumps({"impl": "reference", "unavailable": "host memory for the per-thread vectors"}))
        return 0
    done = C.c_longlong()
    # calibrate: per-call fixed cost (fill/scan) and per-column rate
    t_small = L.ref_sample_run(ctx, 0, 2000, C.byref(done))
    t_big = L.ref_sample_run(ctx, 0, 20000, C.byref(done))
    per_col = max((t_big - t_small) / 18000.0, 1e-7)
    budget = 120.0 / max(1, args.steps + args.warmup)
    ncols = int(max(5000, (budget - t_small) / per_col))
    col0 = 1234567
    for _ in range(args.warmup):
        L.ref_sample_run(ctx, col0, ncols, C.byref(done))
        col0 += threads * ncols
    tot_t, tot_c = 0.0, 0
    for _ in range(args.steps):
        tot_t += L.ref_sample_run(ctx, col0, ncols, C.byref(done))
        tot_c += done.value
        col0 += threads * ncols
    L.ref_sample_destroy(ctx)
    L.ref_sector_destroy(h)
    value = (tot_c / tot_t) / dim
    sample = (f"each step: {threads} threads x apply_extended_hubbard on x with {ncols} non-zero columns of {dim} "
              f"(reference skips zero columns; includes its O(dim) fill/scan per call); H·v/s = columns/s / dim")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1000.0 * tot_t / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": {"workload": WORKLOAD, "sample_columns_per_thread": ncols, "threads": threads,
                      "l2": "inputs larger than L2 (2.65 GB vectors)"},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------- our arm
def read_profile_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` at the benchmark size, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_4x4_6_6.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch_full_size:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def run_ours(args):
    import ctypes as C
    import numpy as np
    import torch
    import ftlm_extended_hubbard_b200 as F
    from ftlm_extended_hubbard_b200._lib import call

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    p = F.HubbardParams(**PARAMS)
    nu, nd = args.sector if args.sector else (NU, ND)
    sec = F.Sector(p, nu, nd)
    if args.hv_path:
        sec.set_apply_path(args.hv_path)
        call("ftlm_gpu_set_cols_variant", sec.handle, args.cols_variant)
        tuned_path, tuned_cols, chosen_by = args.hv_path, args.cols_variant, "command line"
    else:
        tuned_path, tuned_cols, _ = sec.autotune(3)  # project autotuner: H·v variant for this sector shape
        chosen_by = "autotuner"
    st = sec.stats()
    dim = sec.dim()
    g = torch.Generator(device="cuda")
    g.manual_seed(7 + rank)
    x = torch.randn(dim, dtype=torch.complex128, device="cuda", generator=g)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def apply():
        call("ftlm_gpu_apply", sec.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(sptr))

    for _ in range(max(3, args.warmup)):
        apply()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        apply()
    e1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    value = ws * args.steps / (ms_max / 1000.0)

    # per-pass device times (CUDA events on the launch stream between the two kernels)
    npass = C.c_int()
    buf = (C.c_float * 2)()
    rows_ms, cols_ms = [], []
    for _ in range(min(args.steps, 20)):
        call("ftlm_gpu_apply_profiled", sec.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
             C.c_void_p(sptr), buf, C.byref(npass))
        rows_ms.append(buf[0])
        cols_ms.append(buf[1])
    rows_avg, cols_avg = statistics.mean(rows_ms), statistics.mean(cols_ms)

    # end to end through the host-buffer C ABI call (pinned host memory, copies inside the timed region)
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    k_e2e = max(1, min(args.steps, 10))
    call("ftlm_gpu_apply_host", sec.handle, C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr()))
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        call("ftlm_gpu_apply_host", sec.handle, C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr()))
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if pg:
        pg.all_reduce(te, op=pg.ReduceOp.MAX)
    e2e_value = ws * k_e2e / float(te.item())

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    c = 16.0
    n_up = st["mean_up_sources"]
    # Algorithmic bytes per launch (row-gather model split over the two passes):
    #   hv_rows: read the own x row + write y            = 16 B x dim x 2
    #   hv_cols: read n_up distinct up-neighbour x rows + read and write y = 16 B x dim x (n_up + 2)
    alg = {"hv_rows": c * dim * 2.0, "hv_cols": c * dim * (n_up + 2.0)}
    avg_ms = {"hv_rows": rows_avg, "hv_cols": cols_avg}
    dom = max(avg_ms, key=avg_ms.get)
    achieved = alg[dom] / (avg_ms[dom] / 1000.0) / 1e9
    hv_bytes = c * dim * (2.0 + n_up)  # whole H·v, row-gather model (one read of own + neighbour rows, one write)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if not args.sector else f"4x4 sector {tuple(args.sector)} (profiling case)",
                   "vector": "torch.randn complex128, seed 7+rank",
                   "l2": "inputs larger than L2 (2.65 GB per vector); no flush",
                   "parallelism": f"independent H·v per rank x{ws}",
                   "hv_variant": {"path": tuned_path, "cols_slab": [256, 128, 512][tuned_cols % 3],
                                  "up_list": "packed" if tuned_cols >= 3 else "csr", "chosen_by": chosen_by}},
        "gpu_launches": 2 * args.steps,
        "kernels_ms": {"hv_rows": rows_avg, "hv_cols": cols_avg},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": read_profile_traffic(dom) if not args.sector else None,
                     "algorithmic_bytes_per_launch": alg[dom], "peak_source": peak_src,
                     "peak_note": ("hbm_gbs of MEASURED_PEAKS.json (burst copy)" if peaks else
                                   "fallback: MEASURED_PEAKS.json absent; 6650 GB/s, an earlier STREAM-style copy on B200"),
                     "hv_model_frac": hv_bytes / (ms_max / args.steps / 1000.0) / 1e9 / hbm,
                     "compulsory_frac": 2 * c * dim / (ms_max / args.steps / 1000.0) / 1e9 / hbm},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(dim * 16), "d2h_bytes_per_step": int(dim * 16),
                "steps": k_e2e, "call": "ftlm_gpu_apply_host (pinned host buffers)"},
        "clocks": clocks,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and not args.sector:
        del xh, yh
        try:
            out["cpu_baseline"] = cpu_baseline_port(args.cpu_seconds)
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(out))
    sec.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_batched(args):
    """32 complex64 chains of one 4x4 sector for `steps` Lanczos steps (one CUDA graph)."""
    import torch
    import ftlm_extended_hubbard_b200 as F
    nu, nd = args.sector if args.sector else (NU, ND)
    sec = F.Sector(F.HubbardParams(**PARAMS), nu, nd)
    if args.bt_cols >= 0:
        sec.batched_set_cols_variant(args.bt_cols)
        variant, tuned = args.bt_cols, None
    else:
        variant, tuned = sec.batched_autotune()
    sec.batched_lanczos(32, max(1, args.warmup), 7)  # allocation + warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sec.batched_lanczos(32, args.steps, 7)
    t = time.perf_counter() - t0
    print(json.dumps({"workload": f"batched Lanczos, 4x4 sector ({nu},{nd}), dim {sec.dim()}, 32 chains",
                      "cols_variant": variant, "autotune_ms": tuned,
                      "steps": args.steps, "seconds": t, "ms_per_chain_step": 1000.0 * t / (32 * args.steps)}))
    F.batched_release()
    return 0


def run_lanczos(args):
    """Plain complex128 Lanczos step on one 4x4 sector (the fused recurrence of ftlm_gpu_lanczos, Philox
    start, the autotuned H·v variant): wall time per step from a (warmup + steps)-step chain minus a
    warmup-step chain, so start-vector and set-up costs cancel."""
    import torch
    import ftlm_extended_hubbard_b200 as F
    nu, nd = args.sector if args.sector else (NU, ND)
    sec = F.Sector(F.HubbardParams(**PARAMS), nu, nd)
    path, cols, _ = sec.autotune(3)
    w = max(1, args.warmup)
    sec.lanczos(w, 7, start="philox")
    times = []
    for m in (w, w + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sec.lanczos(m, 7, start="philox")
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    print(json.dumps({"workload": f"plain complex128 Lanczos, 4x4 sector ({nu},{nd}), dim {sec.dim()}",
                      "hv_variant": {"path": path, "cols_variant": cols}, "steps": args.steps,
                      "ms_per_step": 1e3 * (times[1] - times[0]) / args.steps}))
    return 0


def run_sweep_model(args):
    """Per-sector Lanczos step cost of both paths on every 4x4 sector class (dims equal under
    N -> 16-N and spin exchange), combined into the time of a full R=32, M=100 sweep."""
    import torch
    import ftlm_extended_hubbard_b200 as F
    n, R, M, S = 16, 32, 100, max(1, args.steps)
    classes = {}
    for nu in range(n + 1):
        for nd in range(n + 1):
            a, b = min(nu, n - nu), min(nd, n - nd)
            classes.setdefault((min(a, b), max(a, b)), []).append((nu, nd))
    recs, t_plain, t_batched = [], 0.0, 0.0
    for (a, b), members in sorted(classes.items()):
        s = F.Sector(F.HubbardParams(**PARAMS), a, b)
        s.lanczos(1, 1, start="philox")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.lanczos(S, 5, start="philox")
        tp = (time.perf_counter() - t0) / S
        rec = {"nu": a, "nd": b, "dim": s.dim(), "sectors": len(members), "plain_chain_step_ms": 1e3 * tp}
        plain = R * M * tp
        bat = plain
        if s.dim() > 2 * M:
            s.batched_lanczos(32, 2, 1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.batched_lanczos(32, S, 1)
            tb = (time.perf_counter() - t0) / S
            rec["batched_block_step_ms"] = 1e3 * tb
            bat = M * tb * ((R + 31) // 32)
        t_plain += len(members) * plain
        t_batched += len(members) * bat
        recs.append(rec)
        s.close()
        F.batched_release()
    print(json.dumps({"workload": "4x4 sweep model, R=32, M=100, complex128 plain vs complex64 batched",
                      "plain_sweep_s": t_plain, "batched_sweep_s": t_batched, "ratio": t_plain / t_batched,
                      "steps_timed_per_sector": S, "sectors": recs}))
    return 0


def run_orbit(args):
    """H_K·v of one translation-orbit block (default 4x4 (8,8), K=(1,2), U=6, V=0.5, phi=0)."""
    import torch
    import ftlm_extended_hubbard_b200 as F
    nu, nd = args.sector if args.sector else (NU, ND)
    p = F.HubbardParams(4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0)
    s = F.Sector(p, nu, nd)
    t0 = time.perf_counter()
    o = s.orbit_block(*args.k)
    build = time.perf_counter() - t0
    x = torch.randn(o.dim, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    for _ in range(max(1, args.warmup)):
        o.apply(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        o.apply(x, y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"workload": f"orbit H_K v, 4x4 ({nu},{nd}) K={tuple(args.k)}", "block_dim": o.dim,
                      "ms_per_apply": ms, "reps_per_s": o.dim / ms * 1e3, "block_build_s": build}))
    o.close()
    return 0


def run_grad(args):
    """Forward + backward of ln Z_GC(U, V, t', mu, beta) on the 4x3 lattice (169 sectors, R=32, M=80,
    batched complex64 chains) at theta = (4, 1, -0.2, 2, 5)."""
    import numpy as np
    import torch
    from ftlm_extended_hubbard_b200 import autograd as AG
    theta = torch.tensor([4.0, 1.0, -0.2, 2.0, 5.0], dtype=torch.float64, requires_grad=True)
    t0 = time.perf_counter()
    lnz = AG.grand_canonical_logz(theta, AG.Lattice(4, 3), 32, 80, 7, method="batched")
    t1 = time.perf_counter()
    lnz.backward()
    t2 = time.perf_counter()
    print(json.dumps({"workload": "d lnZ_GC / d(U, V, t', mu, beta), 4x3, R=32, M=80", "lnZ": lnz.item(),
                      "grad": np.asarray(theta.grad).tolist(), "forward_s": t1 - t0, "backward_s": t2 - t1}))
    return 0


def run_kresolved(args):
    """One 4x4 sector (default (5,5); U=6, V=0.5, t'=-0.25, phi=0): ln Z from the 16 momentum blocks
    (R=24, M=100; batched complex64, and complex128 when dim <= 5e7) against the unsymmetrised
    batched ln Z (R=32, M=100) of the same sector, on T = 0.1..2.0.  --sector 8 8 is the k-block
    workload of the (8,8) sector (16 blocks of dim ~1.035e7)."""
    import numpy as np
    import torch
    import ftlm_extended_hubbard_b200 as F
    nu, nd = args.sector if args.sector else (5, 5)
    p = F.HubbardParams(4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0)
    s = F.Sector(p, nu, nd)
    T = np.round(np.arange(1, 21) * 0.1, 10)
    bts = 1.0 / T
    idx = nu * 17 + nd
    out = {"workload": f"k-resolved vs unsymmetrised ln Z, 4x4 ({nu},{nd}), dim {s.dim()}, R=24 (k) / 32, M=100",
           "T": T.tolist()}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lz_kb, _, dims = s.orbit_ftlm(bts, 24, 100, 7, sector_index=idx, method="batched")
    torch.cuda.synchronize()
    out["kresolved_batched_s"] = time.perf_counter() - t0
    out["block_dims"] = dims.ravel().tolist()
    out["lnz_k_batched"] = lz_kb.tolist()
    t0 = time.perf_counter()
    lz_b, _ = s.batched_ftlm(bts, 32, 100, 7)
    out["unsym_batched_s"] = time.perf_counter() - t0
    out["lnz_unsym"] = lz_b.tolist()
    out["max_abs_diff_lnz_k_vs_unsym"] = float(np.max(np.abs(lz_kb - lz_b)))
    out["abs_diff_lnz_k_vs_unsym_T1"] = float(abs(lz_kb[9] - lz_b[9]))
    F.batched_release()
    if s.dim() <= 50_000_000:
        t0 = time.perf_counter()
        lz_k, _, _ = s.orbit_ftlm(bts, 24, 100, 7, sector_index=idx, start="philox")
        out["kresolved_complex128_s"] = time.perf_counter() - t0
        out["max_rel_diff_batched_vs_complex128"] = float(np.max(np.abs(lz_kb - lz_k) / np.abs(lz_k)))
    print(json.dumps(out))
    return 0


def run_published(args):
    """The reference's published n(mu) workloads (benchmarks/data/n_vs_mu_*_beta20_*.tsv headers:
    t'=-0.35, U=5.75, V=0.9, beta=20, R=12, M=72, seed 7), same reference start vectors, timed end to end
    (sector plans, chains, quadrature, grid).  Published times are the reference's single-threaded
    CPU runs on the authors' macOS machine, as printed in those files."""
    import numpy as np
    import ftlm_extended_hubbard_b200 as F
    published_s = {"2x2": 0.4258, "3x2": 6.83, "4x2": 105.95, "3x3": 530.327, "2x5": 1877.38}
    rows = []
    for key, Lx, Ly in [("2x2", 2, 2), ("3x2", 3, 2), ("4x2", 4, 2), ("3x3", 3, 3), ("2x5", 2, 5)]:
        p = F.HubbardParams(Lx, Ly, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
        mus = np.linspace(-5.0, 20.0, 221)
        F.grand_canonical_sweep(F.HubbardParams(2, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0), 2, 4, 7, [0.05], mus[:2])
        ts = []
        for _ in range(3):  # median of three end-to-end runs
            t0 = time.perf_counter()
            F.grand_canonical_sweep(p, 12, 72, 7, [1.0 / 20.0], mus, start="reference")
            ts.append(time.perf_counter() - t0)
        t = sorted(ts)[1]
        rows.append({"lattice": key, "gpu_s": t, "published_cpu_s": published_s[key],
                     "speedup": published_s[key] / t})
    # the k-orbit solver run (3x2, momentum blocks; blocks of dim <= 64 exactly, larger by FTLM)
    p = F.HubbardParams(3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        for nu in range(7):
            for nd in range(7):
                s = F.Sector(p, nu, nd)
                s.orbit_ftlm([20.0], 12, 72, 7, sector_index=nu * 7 + nd, ed_cutoff=64)
                s.close()
        ts.append(time.perf_counter() - t0)
    t = sorted(ts)[1]
    rows.append({"lattice": "3x2 k-orbit (sector ln Z)", "gpu_s": t, "published_cpu_s": 9.05681,
                 "speedup": 9.05681 / t})
    print(json.dumps({"workload": "published n(mu) sweeps, beta=20, R=12, M=72 (plain complex128, reference "
                                  "start vectors)", "rows": rows}))
    return 0


def run_sweep(args):
    """The full 4x4 sweep (289 sectors, R=32, M=100) with both paths, end to end, and the batched
    path's errors against complex128 with the same Philox start vectors (both with the converged
    quadrature): measured against the plain sweep, and the batched path's own per-result estimate
    (chain 0 of every sector rerun in complex128, --check 1)."""
    import numpy as np
    import ftlm_extended_hubbard_b200 as F
    p = F.HubbardParams(**PARAMS)
    T = np.round(np.arange(1, 21) * 0.1, 10)
    mu = np.round(np.arange(49) * 0.25 - 4.0, 10)
    t0 = time.perf_counter()
    rb = F.grand_canonical_sweep(p, 32, 100, 7, T, mu, method="batched", check=args.check)
    tb = time.perf_counter() - t0
    F.batched_release()
    t0 = time.perf_counter()
    with F.quadrature("converged"):
        rp = F.grand_canonical_sweep(p, 32, 100, 7, T, mu, start="philox")
    tp = time.perf_counter() - t0
    ok = np.isfinite(rp.lnz_sector)
    rel_s = np.abs(rb.lnz_sector[ok] - rp.lnz_sector[ok]) / np.maximum(1.0, np.abs(rp.lnz_sector[ok]))
    rel_g = np.abs(rb.lnz_gc - rp.lnz_gc) / np.maximum(1.0, np.abs(rp.lnz_gc))
    out = {"workload": "full 4x4 grand-canonical sweep, 289 sectors, R=32, M=100, T 0.1..2 (20) x mu "
                       "-4..8 (49), t=1 t'=-0.25 U=8 V=1 phi_x=0.1",
           "batched_s": tb, "plain_s": tp, "ratio": tp / tb, "check_chains": args.check,
           "max_rel_err_sector_lnz": float(rel_s.max()), "max_rel_err_gc_lnz": float(rel_g.max()),
           "max_abs_err_n": float(np.abs(rb.n_avg - rp.n_avg).max())}
    if rb.lnz_gc_err is not None:
        out["estimated_max_rel_err_sector_lnz"] = float(
            (rb.lnz_sector_err[ok] / np.maximum(1.0, np.abs(rp.lnz_sector[ok]))).max())
        out["estimated_max_rel_err_gc_lnz"] = float((rb.lnz_gc_err / np.maximum(1.0, np.abs(rb.lnz_gc))).max())
        out["estimated_max_abs_err_n"] = float(rb.n_err.max())
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "lanczos":
        return run_lanczos(args)
    if args.workload == "sweep-model":
        return run_sweep_model(args)
    if args.workload == "orbit":
        return run_orbit(args)
    if args.workload == "grad":
        return run_grad(args)
    if args.workload == "kresolved":
        return run_kresolved(args)
    if args.workload == "published":
        return run_published(args)
    if args.workload == "sweep":
        return run_sweep(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
