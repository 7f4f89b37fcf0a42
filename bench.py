#!/usr/bin/env python
"""Benchmark of the no-pivot LU hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...   (the CPU restatement, host cores)

One step = one in-place factorization of a fresh, HBM-resident copy of the
workload matrix (each step factors its own copy, so no input reuse; a copy
is 1 GiB at n = 16384, far larger than the 126 MB L2).  For N > 1 (torchrun)
every rank factors its own matrices: replicas, no data-path collective;
time is the max over ranks.  Prints one JSON line on rank 0.

Fields beyond the value: `e2e` times the same factorization through the
public API from pinned host memory (H2D of A, factorization, D2H of the
factors), `roofline` reports the dominant kernel against the measured HBM
peak, `cpu_baseline` the CPU restatement of the reference algorithm on a
bounded sample of the same workload, `clocks` the SM clocks sampled during
the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # Mixed-precision reference path: fp32 storage, fp16 tensor-core Schur
    # update, fp32 accumulation, right-looking, nb = 256, n = 16384; matrix
    # A = R + D, R ~ N(0,1)/sqrt(n), row dominance 1.5.
    "lu_tc32_rl_n16384": dict(n=16384, nb=256, outer="TC32", kind=1, alpha=1.5,
                              kscale=0, oracle_fmt=1),
    # Plain FP32 right-looking, n = 4096, nb = 256, U[-1,1] + dominance 2.
    "lu_fp32_rl_n4096": dict(n=4096, nb=256, outer="FP32", kind=0, alpha=2.0,
                             kscale=0, oracle_fmt=0),
    # FP32 plain path at the mixed path's size (the comparison point of the
    # time-to-solution target).
    "lu_fp32_rl_n16384": dict(n=16384, nb=256, outer="FP32", kind=1, alpha=1.5,
                              kscale=0, oracle_fmt=0),
    "lu_bf16_rl_n16384": dict(n=16384, nb=256, outer="TC32_BF16", kind=1,
                              alpha=1.5, kscale=0, oracle_fmt=2),
    "lu_e4m3_rl_n16384": dict(n=16384, nb=256, outer="TC32_E4M3", kind=1,
                              alpha=1.5, kscale=0, oracle_fmt=3),
    "lu_split_rl_n16384": dict(n=16384, nb=256, outer="TC32_SPLIT", kind=1,
                               alpha=1.5, kscale=0, oracle_fmt=4),
}
# Workloads with their own step (see the run_* functions below).
SPECIAL = ("batch_10000_n16_512", "ll_f16_n16384", "precision_n32768", "adjoint_n8192",
           "c2_grid_n16384")
DEFAULT_WORKLOAD = "lu_tc32_rl_n16384"
NVML_REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x10: "sync_boost",
                0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
                0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting",
                0x100: "display_clock_setting"}


def lu_flops(n: int) -> float:
    return 2.0 * n ** 3 / 3.0


def max_over_ranks(x: float, dist, device) -> float:
    """The largest x over all ranks (every multi-GPU time is the slowest
    rank's); a collective, so every rank calls it at the same point."""
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, units_per_rank: float, ms: float) -> float:
    """Units per second over the whole job: each of `world` replicas
    processes units_per_rank in the slowest rank's time `ms`."""
    return world * units_per_rank / (ms / 1e3)


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def profiled_traffic(name: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/<name>.json), if present."""
    p = os.path.join(ROOT, "profiles", f"{name}.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


class ClockSampler:
    """Samples SM clocks and clock-event reasons through NVML every 20 ms."""

    def __init__(self, device_index: int):
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in NVML_REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self._nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t is not None:
            self._t.join()
        return False

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [],
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def cpu_baseline(wl: dict, budget_s: float = 12.0) -> dict:
    """The CPU restatement of the reference algorithm (oracle, all host
    threads) on a bounded sample of the same workload: the leading outer
    steps of the same n x n factorization, run until the time budget is
    spent.  TFLOP/s = (2n^3/3 - 2(n-k nb)^3/3) / time for k steps done."""
    import oracle as O
    n, nb = wl["n"], wl["nb"]
    a = O.gen_matrix(n, seed=1, kind=wl["kind"], alpha=wl["alpha"], kscale=wl["kscale"])
    t0 = time.perf_counter()
    k = 0
    nc = (n + nb - 1) // nb
    while k < nc and time.perf_counter() - t0 < budget_s:
        O.lu_rl_steps(a, nb, wl["oracle_fmt"], k, k + 1)
        k += 1
    dt = time.perf_counter() - t0
    rest = max(0, n - k * nb)
    flops = lu_flops(n) - lu_flops(rest)
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": O.num_threads(),
            "kind": "port",
            "sample": f"outer steps 0..{k - 1} of {nc} (nb={nb}) of the n={n} "
                      f"factorization, {dt:.1f} s, {flops / 1e12:.2f} TFLOP"}


def run_reference(args, wl) -> None:
    """--impl reference: the reference algorithm as its CPU restatement on
    the host cores (the reference itself has no CPU path), same workload,
    each step a bounded sample (the first outer step of a fresh copy)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    import oracle as O
    n, nb = wl["n"], wl["nb"]
    base = O.gen_matrix(n, seed=1, kind=wl["kind"], alpha=wl["alpha"], kscale=wl["kscale"])
    a = O.colmajor(n, n)
    steps_done = 0
    flops = lu_flops(n) - lu_flops(n - nb)
    times = []
    for i in range(args.warmup + args.steps):
        np.copyto(a, base)
        t0 = time.perf_counter()
        O.lu_rl_steps(a, nb, wl["oracle_fmt"], 0, 1)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            steps_done += 1
    total = sum(times)
    value = steps_done * flops / total / 1e12
    sample = (f"per step: outer step 0 (panel + trailing update, "
              f"{flops / 1e9:.1f} GFLOP) of the n={n} factorization on a fresh copy")
    line = {
        "metric": "LU TFLOP/s (2n^3/3)", "value": value, "unit": "TFLOP/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / max(1, steps_done),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if wl["oracle_fmt"] == 0 else "f32 storage, rounded-operand update",
        "data": "synthetic (seeded counter-based generator)",
        "config": config_of(args, wl),
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": O.num_threads(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_gpu(args, wl) -> None:
    """--impl reference --ref-device gpu: the reference's own GPU code
    (src/lu_nopiv.cu, gemm.cu, convert.cu, lu_nopiv.hxx compiled unmodified
    into oracle/_ref by oracle/Makefile; cuBLAS inside) on the same workload:
    remifa::lu_nopiv_rl<float, FP32, O, 8> with O = FP32 or TC32 (the fp16
    copy buffer it requires allocated beforehand), timed with CUDA events
    around each call.  The call allocates and frees its own workspace and
    synchronises, as the reference does.  Not part of any default line: it
    reproduces the reference-on-B200 figures next to this library's."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import ctypes
    import numpy as np
    import oracle as O
    import torch
    if wl["outer"] not in ("FP32", "TC32"):
        print(json.dumps({"impl": "reference", "workload": args.workload,
                          "unavailable": "the reference has no " + wl["outer"] +
                                         " trailing update"}))
        return
    so = os.path.join(ROOT, "oracle", "_ref", "libremifa_ref.so")
    if not os.path.exists(so):
        print(json.dumps({"impl": "reference", "workload": args.workload,
                          "unavailable": "oracle/_ref/libremifa_ref.so not built"}))
        return
    L = ctypes.CDLL(so)
    vp, i64, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    L.ref_lu_nopiv_rl_f32.argtypes = [vp, i64, i64, i64, vp, i64, vp, i, i, vp, i64]
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, nb = wl["n"], wl["nb"] if args.nb is None else args.nb
    tc = wl["outer"] == "TC32"
    a = O.gen_matrix(n, seed=1, kind=wl["kind"], alpha=wl["alpha"], kscale=wl["kscale"])
    base = torch.from_numpy(np.ascontiguousarray(a).T.copy()).cuda()  # column-major
    work = torch.empty_like(base)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    cpy = torch.empty((n, n), dtype=torch.float16, device="cuda") if tc else None
    st = torch.cuda.current_stream()
    times = []
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    try:
        for k in range(args.warmup + args.steps):
            work.copy_(base)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            sys.stdout.flush()
            os.dup2(devnull, 1)  # the reference prints a banner per call
            e0.record(st)
            rc = L.ref_lu_nopiv_rl_f32(ctypes.c_void_p(st.cuda_stream), n, n, nb,
                                       ctypes.c_void_p(work.data_ptr()), n,
                                       ctypes.c_void_p(info.data_ptr()), 0, int(tc),
                                       ctypes.c_void_p(cpy.data_ptr()) if tc else None,
                                       n if tc else 0)
            e1.record(st)
            torch.cuda.synchronize()
            os.dup2(saved, 1)
            if rc != 0:
                raise RuntimeError(f"reference call failed ({rc})")
            if k >= args.warmup:
                times.append(e0.elapsed_time(e1))
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)
    ms = statistics.median(times)
    value = lu_flops(n) / (ms * 1e-3) / 1e12
    line = {
        "metric": "LU TFLOP/s (2n^3/3)", "value": value, "unit": "TFLOP/s",
        "impl": "reference", "reference_device": "gpu", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "ms_all": times,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if not tc else "f32 storage, fp16 tensor-core update (cuBLAS)",
        "data": "synthetic (seeded generator of the tests, host)",
        "config": config_of(args, wl),
        "code": "the reference's src/lu_nopiv.cu, gemm.cu, convert.cu and lu_nopiv.hxx "
                "compiled unmodified for sm_100a (oracle/Makefile), cuBLAS 12.9 inside",
    }
    print(json.dumps(line), flush=True)


def time_to_solution(rb, torch, base, n, nb, outer, la, tol=1e-14, reps=2, solver="classic",
                     xt=None, b=None):
    """Time to an fp64-level solution of A x = b (b = A x_true, x_true ~
    N(0,1), fp64): copy A, factor with `outer`, refine in fp64 until the
    normwise backward error is <= tol -- classic refinement (`solver` =
    "classic", lu_refine_c) or GMRES-IR ("gmres", lu_gmres_ir_c).  Device
    time with CUDA events (the refinement reads its backward error back once
    per iteration)."""
    dev = base.device
    if xt is None:
        g = torch.Generator(device=dev)
        g.manual_seed(7)
        xt = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    if b is None:
        b = torch.zeros(n, dtype=torch.float64, device=dev)
        for j0 in range(0, n, 2048):  # b = A x_true in fp64, column blocks
            b += base[:, j0:j0 + 2048].double() @ xt[j0:j0 + 2048]
    lu = rb.colmajor_empty(n, n, n, torch.float32, dev)
    ws = torch.empty(rb.workspace_size(n, nb=nb, outer=outer), dtype=torch.uint8, device=dev)
    best = None
    for _ in range(reps):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        s0.record()
        lu.copy_(base)
        info = rb.lu_nopiv_rl(lu, nb=nb, outer=outer, workspace=ws, lookahead=la)
        if solver == "gmres":
            x, it, inner, be = rb.gmres_ir(base, lu, b, tol=tol, max_outer=20, restart=40)
        else:
            x, it, be = rb.refine(base, lu, b, tol=tol, max_iter=50)
            inner = None
        s1.record()
        torch.cuda.synchronize(dev)
        ms = s0.elapsed_time(s1)
        fe = float(((x - xt).abs().max() / xt.abs().max()).item())
        rec = {"ms": ms, "solver": solver, "iters": it, "berr": be, "fwd_err": fe,
               "info": int(info.item())}
        if inner is not None:
            rec["arnoldi_steps"] = inner
        if best is None or ms < best["ms"]:
            best = rec
    del lu, ws
    return best


def isolated_update_roofline(rb, torch, outer, n, nb, la, peaks, reps=3) -> dict:
    """The dominant kernel alone: the factorization's largest trailing-update
    launch shape -- under look-ahead with fp16 / bf16 updates the first bulk
    pass of six outer steps (M = N = n - 8 nb, K = 6 nb, the CTA-pair
    kernel), else the first step's bulk (M = N = n - 3 nb, K = nb) -- run
    through the library's update entry on one stream with nothing
    concurrent; the tensor-core launch is timed with CUDA events on its
    stream (the operand packing, a separate launch, is not counted).  At
    K = 6 nb = 1536 each C element's 8 bytes carry 2K = 3072 flops (AI 384
    flop/B, above the ridge of the measured peaks), so the bound reported
    is the tensor pipe; the HBM fraction is given beside it."""
    grouped = la and outer in (rb.TC32, rb.compute_type.TC32_BF16)
    q = 6 if grouped else 1
    m = n - (q + 2 if grouped else 3) * nb
    k = q * nb
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    a = rb.colmajor(torch.randn(m, k, device="cuda", generator=g))
    b = rb.colmajor(torch.randn(k, m, device="cuda", generator=g))
    c = rb.colmajor(torch.randn(m, m, device="cuda", generator=g))
    rb.gemmex(outer, -1.0, a, b, 1.0, c)  # warm-up
    torch.cuda.synchronize()
    with rb.profile() as pr:
        for _ in range(reps):
            rb.gemmex(outer, -1.0, a, b, 1.0, c)
        torch.cuda.synchronize()
    e = pr.entries["tc_update"]
    sec = e["total_ms"] / 1e3
    gbs = e["bytes"] / sec / 1e9
    tfs = e["flops"] / sec / 1e12
    alg = e["bytes"] / e["launches"]
    prof_name = "tc_update_pair_update_m8192_k1536" if grouped else "tc_update_update_m8192_k512"
    tr = profiled_traffic(prof_name)
    del a, b, c
    torch.cuda.empty_cache()
    out = {"kernel": ("tc_update_pair_kernel (CTA pairs, tcgen05 cta_group::2, 256 x 256 "
                      "tiles, TMA reduce-add)") if grouped else
                     "tc_update_kernel (persistent CTAs, C streamed by TMA, all SMs)",
           "shape": {"M": m, "N": m, "K": k},
           "algorithmic_bytes_per_launch": alg,
           "avg_launch_ms": e["total_ms"] / e["launches"], "launches": e["launches"],
           "traffic": tr["traffic_over_algorithmic"] * alg if tr else None,
           "traffic_source": (f"ncu dram bytes / algorithmic bytes of the same kernel at "
                              f"M = 8192 (profiles/{prof_name}.json), times this launch's "
                              "algorithmic bytes") if tr else None,
           "timing": "CUDA events on the launching stream, the launch alone, "
                     f"mean of {reps}"}
    if grouped:
        out.update({"bound": "tensor", "achieved": tfs, "peak": peaks["bf16_tflops"],
                    "unit": "TFLOP/s", "frac": tfs / peaks["bf16_tflops"],
                    "peak_source": peaks["source"] + " bf16_tflops (cuBLAS, burst)",
                    "frac_of_sustained": tfs / peaks["bf16_tflops_sustained"]
                    if peaks.get("bf16_tflops_sustained") else None,
                    "hbm_gbs": gbs, "hbm_frac": gbs / peaks["hbm_gbs"]})
    else:
        out.update({"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": gbs / peaks["hbm_gbs"],
                    "peak_source": peaks["source"] + " hbm_gbs (copy, burst)",
                    "tensor_tflops": tfs, "tensor_peak": peaks["bf16_tflops"],
                    "tensor_frac": tfs / peaks["bf16_tflops"]})
    return out


def config_of(args, wl) -> dict:
    return {"workload": args.workload, "n": wl["n"], "nb": getattr(args, "nb", None) or wl["nb"],
            "lookahead": not getattr(args, "no_lookahead", False),
            "diag_width": getattr(args, "diag_width", 0) or 128,
            "variant": "right-looking", "inner_update": "FP32",
            "outer_update": wl["outer"],
            "matrix": f"R + D, R ~ {'N(0,1)/sqrt(n)' if wl['kind'] else 'U[-1,1)'}, "
                      f"row dominance {wl['alpha']}",
            "l2": "inputs larger than L2: a distinct 4n^2-byte matrix per step",
            "parallelism": f"replicas x{args.gpus}"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + list(SPECIAL))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-device", default="cpu", choices=["cpu", "gpu"],
                    help="--impl reference: the CPU restatement on the host cores "
                         "(default) or the reference's own GPU code (oracle/_ref)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tts", action="store_true",
                    help="skip the time-to-solution measurements")
    ap.add_argument("--no-n32768", action="store_true",
                    help="skip the n = 32768 time-to-solution study of the default line")
    ap.add_argument("--no-isolated", action="store_true",
                    help="skip the dominant kernel's isolated timing (roofline): a launch "
                         "list of the factorization alone")
    ap.add_argument("--no-lookahead", action="store_true",
                    help="factor each outer block strictly after the previous update")
    ap.add_argument("--nb", type=int, default=None, help="override the outer block size")
    ap.add_argument("--diag-width", type=int, default=0,
                    help="override the diagonal-block width of the panel (0: library default)")
    ap.add_argument("--batch-count", type=int, default=10_000,
                    help="batched workload: the first N sizes of the seeded draw "
                         "(smaller cases for profiling)")
    args = ap.parse_args()
    if args.workload in SPECIAL:
        run_special(args)
        return
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        if args.ref_device == "gpu":
            run_reference_gpu(args, wl)
        else:
            run_reference(args, wl)
        return

    import torch
    import torch.distributed as dist
    import remifa_b200 as rb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    n, nb = wl["n"], (args.nb or wl["nb"])
    la = not args.no_lookahead
    outer = getattr(rb.compute_type, wl["outer"])
    nmat = args.warmup + args.steps
    base = rb.gen_matrix(n, seed=1 + rank, kind=wl["kind"], alpha=wl["alpha"],
                         kscale=wl["kscale"], device=dev)
    mats = []
    for _ in range(nmat):
        m = rb.colmajor_empty(n, n, n, torch.float32, dev)
        m.copy_(base)
        mats.append(m)
    ws = torch.empty(rb.workspace_size(n, nb=nb, outer=outer), dtype=torch.uint8, device=dev)
    infos = torch.zeros(nmat, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    for i in range(args.warmup):
        rb.lu_nopiv_rl(mats[i], nb=nb, outer=outer, info=infos[i:i + 1], workspace=ws,
                       lookahead=la, diag_width=args.diag_width)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()

    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    launches0 = rb.launch_count()
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for i in range(args.warmup, nmat):
            rb.lu_nopiv_rl(mats[i], nb=nb, outer=outer, info=infos[i:i + 1],
                           workspace=ws, lookahead=la, diag_width=args.diag_width)
        t_end.record(stream)
        torch.cuda.synchronize(dev)
    launches = rb.launch_count() - launches0
    ms = t_start.elapsed_time(t_end)
    # Per-kernel device times for the roofline: the same steps again on fresh
    # copies, every library launch bracketed by CUDA events on its own stream.
    # Those event records slow a step down, so `value` comes from the run
    # above, which has none.
    for i in range(args.warmup, nmat):
        mats[i].copy_(base)
    torch.cuda.synchronize(dev)
    p_start = torch.cuda.Event(enable_timing=True)
    p_end = torch.cuda.Event(enable_timing=True)
    with rb.profile() as prof:
        p_start.record(stream)
        for i in range(args.warmup, nmat):
            rb.lu_nopiv_rl(mats[i], nb=nb, outer=outer, info=infos[i:i + 1],
                           workspace=ws, lookahead=la, diag_width=args.diag_width)
        p_end.record(stream)
        torch.cuda.synchronize(dev)
    ms_prof = p_start.elapsed_time(p_end)
    if world > 1:
        ms = max_over_ranks(ms, dist, dev)
        dist.barrier()
    bad = int((infos != 0).sum().item())
    value = whole_job_rate(world, args.steps * lu_flops(n), ms) / 1e12

    # ---- end to end through lu_nopiv_rl_host_c: the pinned host matrix goes
    # in by column chunks while the device factors the chunks already in, and
    # each finished block column goes back while the factorization runs; the
    # host matrix is reset from a pinned source between steps (outside the
    # timed region)
    # (--e2e-steps 0 leaves it out: a profiling convenience, no e2e figure)
    e_ms = []
    if args.e2e_steps > 0:
        host_src = torch.empty((n, n), dtype=torch.float32, pin_memory=True).t()
        host_src.copy_(base)
        host_a = torch.empty((n, n), dtype=torch.float32, pin_memory=True).t()
        dA = mats[0]
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        host_a.copy_(host_src)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rb.lu_nopiv_rl_host(host_a, dA, nb=nb, outer=outer, info=infos[0:1], workspace=ws,
                            lookahead=la, diag_width=args.diag_width)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if i > 0:  # first iteration warms the pinned paths
            e_ms.append(e0.elapsed_time(e1))
    e2e_ms = sum(e_ms) / len(e_ms) if e_ms else None
    if world > 1 and e_ms:
        e2e_ms = max_over_ranks(e2e_ms, dist, dev)
    e2e_value = whole_job_rate(world, lu_flops(n), e2e_ms) / 1e12 if e_ms else None

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    peaks = measured_peaks()
    dom = "tc_update" if outer != rb.FP32 else "sgemm_update"
    ent = prof.entries.get(dom, {})
    roofline = None
    if ent.get("launches"):
        avg_ms = ent["total_ms"] / ent["launches"]
        if dom == "tc_update":
            roofline = ({} if args.no_isolated else
                        isolated_update_roofline(rb, torch, outer, n, nb, la, peaks))
            # inside the factorization (three concurrent streams, so per-launch
            # event times overlap): the update's algorithmic bytes per step
            # over the whole step's time -- a floor of its achieved rate
            per_step = ent["bytes"] / args.steps
            roofline["in_factorization"] = {
                "bytes_per_step": per_step, "flops_per_step": ent["flops"] / args.steps,
                "launches_per_step": ent["launches"] / args.steps,
                "rate_over_step_time_gbs": per_step / (ms / args.steps / 1e3) / 1e9,
                "frac_of_peak": per_step / (ms / args.steps / 1e3) / 1e9 / peaks["hbm_gbs"],
                "tensor_tflops_over_step_time":
                    ent["flops"] / args.steps / (ms / args.steps / 1e3) / 1e12,
                "avg_launch_event_ms": avg_ms,
                "event_time_over_wall": ent["total_ms"] / ms_prof,
                "note": "per-launch CUDA events from a second, profiled pass; launches on "
                        "the three streams overlap, so only the per-step ratio is a rate"}
        else:
            achieved = ent["flops"] / (ent["total_ms"] / 1e3) / 1e12
            roofline = {"kernel": dom, "bound": "fp32-simt", "achieved": achieved,
                        "peak": None, "unit": "TFLOP/s", "frac": None,
                        "note": "FP32 SIMT GEMM (no tensor cores on the FP32 plain path)",
                        "traffic": None, "avg_launch_ms": avg_ms,
                        "launches": ent["launches"],
                        "event_time_over_wall": ent["total_ms"] / ms_prof,
                        "timing": "per-launch CUDA events from a second, profiled pass "
                                  "of the same steps"}
    line = {
        "metric": "LU TFLOP/s (2n^3/3)",
        "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if outer == rb.FP32 else
                 f"f32 storage, {wl['outer']} update (fp32 accumulate)",
        "data": "synthetic (seeded counter-based generator on the device)",
        "config": config_of(args, wl),
        "e2e": {"value": e2e_value, "unit": "TFLOP/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": 4 * n * n, "d2h_bytes_per_step": 4 * n * n,
                "path": "lu_nopiv_rl_host_c via remifa_b200.lu_nopiv_rl_host: pinned host "
                        "matrix in by column chunks overlapping the factorization, finished "
                        "block columns streamed back"} if e_ms else None,
        "gpu_launches": launches,
        "roofline": roofline,
        "kernels": {k: {"launches": v["launches"], "ms": v["total_ms"]}
                    for k, v in prof.entries.items()},
        "clocks": clk.summary(),
        "bad_info_steps": bad,
    }
    if world == 1 and not args.no_tts:
        # time to an fp64-level solution: this workload's factorization vs
        # the plain FP32 path, both refined in fp64 to the same tolerance
        dA = None
        mats.clear()
        del ws
        torch.cuda.empty_cache()
        t_mixed = time_to_solution(rb, torch, base, n, nb, outer, la)
        t_fp32 = time_to_solution(rb, torch, base, n, nb, rb.FP32, la)
        line["time_to_solution"] = {
            "tol": 1e-14, "backward_error": "||b-Ax||inf/(||A||inf ||x||inf + ||b||inf)",
            wl["outer"]: t_mixed, "FP32": t_fp32,
            "speedup_vs_fp32_plain": t_fp32["ms"] / t_mixed["ms"]}
        if args.workload == DEFAULT_WORKLOAD and not args.no_n32768:
            # the time-to-solution target's own size: n = 32768, every
            # update precision against FP32 plain at kappa ~ 1e2 / 1e4 / 1e6
            del base
            torch.cuda.empty_cache()
            line["time_to_solution_n32768"] = precision_study(torch, rb, reps=1)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# special workloads: one JSON line each, same keys as the main line


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _base_line(args, metric, value, unit, ms, higher=True, dtype="f32", config=None):
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": higher, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype, "data": "synthetic (seeded counter-based generator on the device)",
            "config": config or {"workload": args.workload}}


def run_batch(args, torch, rb):
    """10,000 independent factorizations, n_i = floor(16 * 32**u_i) (seed
    11), A_i = R_i + D_i (R ~ U[-1,1), row dominance 1.5), fp32 storage,
    fp16 tensor-core outer updates, one persistent launch replayed as a CUDA
    graph; each step factors its own fresh copy of the batch (1.5 GB)."""
    from remifa_b200.batch import BatchPlan, MatrixBatch, batch_sizes
    import oracle as O
    sizes = batch_sizes(10_000, seed=11)[:args.batch_count]
    src = MatrixBatch(sizes, align=4).generate(seed=11)
    plan = BatchPlan(sizes, outer=rb.TC32)
    tuning = plan.autotune(reps=3)
    nrun = args.warmup + args.steps
    copies = [src.like(src.data.clone()) for _ in range(nrun)]
    info = torch.zeros(len(sizes), dtype=torch.int32, device=src.data.device)
    graphs = [plan.graph(m, info) for m in copies]
    stream = torch.cuda.current_stream()
    for i in range(args.warmup):
        graphs[i].launch(stream)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    with ClockSampler(torch.cuda.current_device()) as clk:
        with rb.profile() as prof:
            e0.record(stream)
            for i in range(args.warmup, nrun):
                graphs[i].launch(stream)
            e1.record(stream)
            torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    bad = int((info != 0).sum())
    flops = src.flops
    value = len(sizes) / (ms / 1e3)
    nbytes = float((sizes.astype("float64") * src.lda).sum() * 4)
    # end to end: pinned host batch -> device, factor, factors -> host
    host = torch.empty(src.data.numel(), dtype=torch.float32, pin_memory=True)
    host.copy_(src.data)
    back = torch.empty_like(host)
    dev = copies[0]
    e_ms = []
    for i in range(4):
        torch.cuda.synchronize()
        a0, a1 = _events(torch)
        a0.record(stream)
        dev.data.copy_(host, non_blocking=True)
        plan(dev, info)
        back.copy_(dev.data, non_blocking=True)
        a1.record(stream)
        torch.cuda.synchronize()
        if i:
            e_ms.append(a0.elapsed_time(a1))
    e2e_ms = sum(e_ms) / len(e_ms)
    peaks = measured_peaks()
    achieved = 2 * nbytes / (ms / 1e3) / 1e9
    line = _base_line(args, f"batched LU matrices/s ({len(sizes):,} sizes 16..511)", value,
                      "matrices/s", ms, dtype="f32 storage, fp16 tensor-core updates",
                      config={"workload": args.workload, "batch": len(sizes),
                              "sizes": "floor(16*32^u), u~U[0,1) seed 11",
                              "matrix": "R + D, R ~ U[-1,1), row dominance 1.5",
                              "tuning": tuning, "l2": "a distinct 1.5 GB copy per step",
                              "launch": "one persistent kernel per step, CUDA graph"})
    line.update({
        "tflops": flops / (ms / 1e3) / 1e12,
        "e2e": {"value": len(sizes) / (e2e_ms / 1e3), "unit": "matrices/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes,
                "path": "lu_batch_c via BatchPlan, pinned host buffers"},
        "gpu_launches": prof.launches,
        "roofline": {"kernel": "batch_lu_kernel", "bound": "hbm",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"],
                     "peak_source": peaks["source"] + " hbm_gbs",
                     "algorithmic_bytes_per_launch": 2 * nbytes, "traffic": None},
        "clocks": clk.summary(), "bad_info": bad,
    })
    # CPU baseline: the oracle's RL restatement per matrix on a sample
    import numpy as np
    idx = list(range(0, len(sizes), 50))
    t0 = time.perf_counter()
    fl = 0.0
    for i in idx:
        n = int(sizes[i])
        a = O.gen_matrix(n, seed=11 + i, kind=0, alpha=1.5)
        nb = tuning["nb"][rb.batch.bucket_of(n)]
        O.lu_rl(a, nb=nb, outer_fmt=1, threads=1)
        fl += lu_flops(n)
    dt = time.perf_counter() - t0
    line["cpu_baseline"] = {"value": len(idx) / dt, "unit": "matrices/s", "cores": 1,
                            "kind": "port",
                            "sample": f"{len(idx)} of the 10,000 matrices (every 50th), "
                                      f"{dt:.1f} s, {fl / dt / 1e9:.1f} GFLOP/s"}
    print(json.dumps(line), flush=True)


def run_ll16(args, torch, rb):
    """Left-looking factorization of an n = 16384 fp16 matrix (fp16
    storage, fp16 tensor-core updates, nb = 256 -- the reference's outer
    block for its fp16 wrappers -- or --nb), A = R + D with R ~
    N(0,1)/sqrt(n), row dominance 1.5."""
    n, nb = 16384, args.nb or 256
    base32 = rb.gen_matrix(n, seed=1, kind=1, alpha=1.5)
    base = rb.colmajor_empty(n, n, n, torch.float16)
    base.copy_(base32)
    del base32
    nrun = args.warmup + args.steps
    mats = [base.clone(memory_format=torch.preserve_format) for _ in range(nrun)]
    mats = [m if m.stride(0) == 1 else rb.colmajor(m) for m in mats]
    ws = torch.empty(rb.workspace_size(n, nb=nb, outer=rb.TC32, variant=1, dtype=torch.float16),
                     dtype=torch.uint8, device=base.device)
    infos = torch.zeros(nrun, dtype=torch.int32, device=base.device)
    stream = torch.cuda.current_stream()
    for i in range(args.warmup):
        rb.lu_nopiv_ll(mats[i], nb=nb, outer=rb.TC32, info=infos[i:i + 1], workspace=ws)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    launches0 = rb.launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for i in range(args.warmup, nrun):
            rb.lu_nopiv_ll(mats[i], nb=nb, outer=rb.TC32, info=infos[i:i + 1],
                           workspace=ws)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = rb.launch_count() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    # the per-kernel table from a separate, profiled factorization (CUDA
    # events around every launch would slow the timed steps)
    mats[0].copy_(base)
    with rb.profile() as prof:
        rb.lu_nopiv_ll(mats[0], nb=nb, outer=rb.TC32, info=infos[0:1], workspace=ws)
        torch.cuda.synchronize()
    host = torch.empty((n, n), dtype=torch.float16, pin_memory=True).t()
    host.copy_(base)
    back = torch.empty((n, n), dtype=torch.float16, pin_memory=True).t()
    e_ms = []
    for i in range(3):
        torch.cuda.synchronize()
        a0, a1 = _events(torch)
        a0.record(stream)
        mats[0].copy_(host, non_blocking=True)
        rb.lu_nopiv_ll(mats[0], nb=nb, outer=rb.TC32, info=infos[0:1], workspace=ws)
        back.copy_(mats[0], non_blocking=True)
        a1.record(stream)
        torch.cuda.synchronize()
        if i:
            e_ms.append(a0.elapsed_time(a1))
    e2e_ms = sum(e_ms) / len(e_ms)
    line = _base_line(args, "LU TFLOP/s (2n^3/3)", lu_flops(n) / (ms / 1e3) / 1e12,
                      "TFLOP/s", ms, dtype="f16 storage, fp16 tensor-core updates (fp32 accumulate)",
                      config={"workload": args.workload, "n": n, "nb": nb,
                              "variant": "left-looking", "storage": "fp16",
                              "matrix": "R + D, R ~ N(0,1)/sqrt(n), row dominance 1.5",
                              "l2": "a distinct 2n^2-byte matrix per step"})
    line.update({
        "e2e": {"value": lu_flops(n) / (e2e_ms / 1e3) / 1e12, "unit": "TFLOP/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": 2 * n * n,
                "d2h_bytes_per_step": 2 * n * n, "path": "lu_nopiv_ll_c, fp16 pinned host"},
        "gpu_launches": launches,
        "kernels": {k: {"launches": v["launches"], "ms": v["total_ms"]}
                    for k, v in prof.entries.items()},
        "kernels_note": "per-launch CUDA events of one separate factorization; "
                        "launches on several streams overlap",
        "clocks": clk.summary(), "bad_info_steps": int((infos != 0).sum())})
    print(json.dumps(line), flush=True)


def _condest(torch, rb, a, lu, n, iters=4):
    """Hager/Higham 1-norm estimate of ||A^-1||_1 with refined solves."""
    dev = a.device
    x = torch.full((n,), 1.0 / n, dtype=torch.float64, device=dev)
    est = 0.0
    from remifa_b200.autograd import refine_ex
    for _ in range(iters):
        y = torch.empty((n, 1), dtype=torch.float64, device=dev)
        refine_ex(a, lu, x.view(-1, 1).contiguous(), y, trans=False, tol=1e-12, max_iter=20)
        est = float(y.abs().sum())
        xi = torch.sign(y).view(-1, 1).contiguous()
        xi[xi == 0] = 1.0
        z = torch.empty((n, 1), dtype=torch.float64, device=dev)
        refine_ex(a, lu, xi, z, trans=True, tol=1e-12, max_iter=20)
        j = int(z.abs().argmax())
        if float(z.abs().max()) <= float((z.view(-1) * x).sum()):
            break
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        x[j] = 1.0
    return est


PRECISIONS = ["TC32_BF16", "TC32_E4M3", "TC32_SPLIT", "TC32", "FP32"]


def precision_study(torch, rb, n=32768, nb=256, reps=2, kappas=(1e2, 1e4, 1e6)):
    """Time to an fp64-level solution (backward error <= 1e-14) of A x = b,
    b = A x_true (x_true ~ N(0,1) seed 7, fp64), per Schur-update precision
    (bf16, e4m3 with per-tile 2^k scales, split fp16, fp16, fp32 plain) and
    per condition number.  A = alpha diag(|R| 1) - |R| with |R| ~ |N(0,1)|/sqrt(n)
    (generator kind 2): row dominance alpha = 1 + 1.06 / kappa sets
    kappa_2(A) ~ kappa.  Each precision is refined both ways (classic and
    GMRES-IR); its time to solution is the faster one that converged."""
    rows = []
    for target in kappas:
        alpha = 1.0 + 1.06 / target
        base = rb.gen_matrix(n, seed=1, kind=2, alpha=alpha)
        g = torch.Generator(device=base.device)
        g.manual_seed(7)
        xt = torch.randn(n, dtype=torch.float64, device=base.device, generator=g)
        b = torch.zeros(n, dtype=torch.float64, device=base.device)
        for j0 in range(0, n, 2048):
            b += base[:, j0:j0 + 2048].double() @ xt[j0:j0 + 2048]
        lu = rb.colmajor(base)
        rb.lu_nopiv_rl(lu, nb=nb, outer=rb.compute_type.TC32_SPLIT)
        kappa1 = float(base.abs().sum(dim=0).max()) * _condest(torch, rb, base, lu, n)
        del lu
        torch.cuda.empty_cache()
        row = {"kappa_target": target, "alpha": alpha, "kappa1_est": kappa1}
        for pr in PRECISIONS:
            outer = getattr(rb.compute_type, pr)
            c = time_to_solution(rb, torch, base, n, nb, outer, True, reps=reps,
                                 solver="classic", xt=xt, b=b)
            g2 = time_to_solution(rb, torch, base, n, nb, outer, True, reps=reps,
                                  solver="gmres", xt=xt, b=b)
            ok = [r for r in (c, g2) if r["berr"] <= 1e-14]
            row[pr] = {"classic": c, "gmres": g2,
                       "time_to_solution_ms": min(r["ms"] for r in ok) if ok else None}
            torch.cuda.empty_cache()
        fp32 = row["FP32"]["time_to_solution_ms"]
        mixed = [row[p]["time_to_solution_ms"] for p in PRECISIONS[:-1]
                 if row[p]["time_to_solution_ms"] is not None]
        row["speedup_best_mixed_vs_fp32"] = fp32 / min(mixed) if (fp32 and mixed) else None
        row["speedup_per_precision"] = {
            p: (fp32 / row[p]["time_to_solution_ms"]
                if fp32 and row[p]["time_to_solution_ms"] else None) for p in PRECISIONS[:-1]}
        rows.append(row)
        del base, b, xt
        torch.cuda.empty_cache()
    speed = [r["speedup_best_mixed_vs_fp32"] for r in rows]
    summary = {"n": n, "nb": nb, "reps": reps,
               "matrix": "alpha diag(|R| 1) - |R|, |R| ~ |N(0,1)|/sqrt(n) seed 1, "
                         "alpha = 1 + 1.06/kappa (kappa_2 ~ kappa)",
               "x_true": "N(0,1) seed 7, b = A x_true in fp64",
               "min_speedup_over_kappa": min(s for s in speed if s) if any(speed) else None,
               "results": rows}
    return summary


def run_precision(args, torch, rb):
    """n = 32768: precision_study at kappa ~ 1e2, 1e4, 1e6.  value = the
    smallest, over the three condition numbers, of (FP32-plain time to
    solution) / (best mixed-precision time to solution)."""
    st = precision_study(torch, rb, reps=max(1, min(args.steps, 2)))
    line = _base_line(args, "time-to-solution speedup vs FP32 plain (berr <= 1e-14), "
                      "smallest over kappa", st["min_speedup_over_kappa"], "x",
                      min(r[p]["time_to_solution_ms"] for r in st["results"]
                          for p in PRECISIONS[:-1] if r[p]["time_to_solution_ms"]),
                      dtype="f32 storage; bf16 / e4m3 / split-fp16 / fp16 updates; fp64 IR "
                            "(classic or GMRES)",
                      config={"workload": args.workload, "n": st["n"], "nb": st["nb"],
                              "matrix": st["matrix"], "x_true": st["x_true"]})
    line["results"] = st["results"]
    print(json.dumps(line), flush=True)


def run_adjoint(args, torch, rb):
    """Differentiable solve: n = 8192, 64 right-hand sides, fp16 tensor-core
    factors, dominance 2, loss sum(W * X), forward (factor + refined solves)
    and backward (refined transposed solves + outer product); plus the
    batched backward over 1,024 matrices of sizes U[64, 256]."""
    import numpy as np
    from remifa_b200.autograd import lu_solve_autograd
    from remifa_b200.batch import BatchPlan, MatrixBatch, RhsBatch, batched_lu_solve
    n, k = 8192, 64
    A0 = rb.gen_matrix(n, seed=2, kind=1, alpha=2.0)
    g = torch.Generator(device=A0.device)
    g.manual_seed(3)
    B = torch.randn(n, k, dtype=torch.float64, device=A0.device, generator=g)
    W = torch.randn(n, k, dtype=torch.float64, device=A0.device, generator=g)
    fw, bw = [], []
    for i in range(args.warmup + args.steps):
        A = A0.clone().requires_grad_(True)
        e0, e1 = _events(torch)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record()
        X = lu_solve_autograd(A, B, outer=rb.TC32, nb=256, refine=True)
        e1.record()
        (X * W).sum().backward()
        e2.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            fw.append(e0.elapsed_time(e1))
            bw.append(e1.elapsed_time(e2))
    rng = np.random.default_rng(12)
    sizes = rng.integers(64, 257, size=1024).astype(np.int32)
    layout = MatrixBatch(sizes, align=4).generate(seed=12, alpha=2.0)
    plan = BatchPlan(sizes, outer=rb.TC32)
    rhs = RhsBatch(sizes, 1)
    b = torch.randn(rhs.data.numel(), dtype=torch.float64, device=A0.device, generator=g)
    w = torch.randn(rhs.data.numel(), dtype=torch.float64, device=A0.device, generator=g)
    bfw, bbw = [], []
    for i in range(args.warmup + args.steps):
        a = layout.data.clone().requires_grad_(True)
        e0, e1 = _events(torch)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record()
        x = batched_lu_solve(a, b, layout, plan, refine_iters=4)
        e1.record()
        (x * w).sum().backward()
        e2.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            bfw.append(e0.elapsed_time(e1))
            bbw.append(e1.elapsed_time(e2))
    med = statistics.median
    line = _base_line(args, "differentiable solve forward+backward ms (n=8192, 64 rhs)",
                      med(fw) + med(bw), "ms", med(fw) + med(bw), higher=False,
                      dtype="f32 storage, fp16 tensor-core factors, fp64 refinement",
                      config={"workload": args.workload, "n": n, "nrhs": k,
                              "matrix": "R + D, R ~ N(0,1)/sqrt(n), row dominance 2",
                              "loss": "sum(W * X), W ~ N(0,1)"})
    line.update({"forward_ms": med(fw), "backward_ms": med(bw),
                 "batched": {"matrices": 1024, "sizes": "U[64,256] seed 12",
                             "forward_ms": med(bfw), "backward_ms": med(bbw),
                             "refine_iters": 4}})
    print(json.dumps(line), flush=True)


def run_c2_grid(args, torch, rb):
    """The n = 16384 mixed-precision workload over its matrix family: A = R +
    D (R ~ N(0,1)/sqrt(n)), row dominance alpha in {1.05, 1.5, 4}, entries
    scaled by 2^k, k in {0, 8} (seeds 1..6).  Per matrix: (i) right-looking,
    fp32 storage, fp16 tensor-core updates; (ii) left-looking with fp16
    storage (the matrix scaled by a power of two first if it exceeds the
    fp16 range, which rescales U exactly).  Reported per run: TFLOP/s, info,
    finite factors, the backward error of the unrefined solve and the FP64
    refinement steps to 1e-14.  value = the smallest right-looking TFLOP/s."""
    import math
    n = 16384
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    xt = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    runs = []

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = _events(torch)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sorted(ts)[len(ts) // 2]

    def solve_quality(a32, lu32):
        b = torch.zeros(n, dtype=torch.float64, device="cuda")
        for j0 in range(0, n, 2048):
            b += a32[:, j0:j0 + 2048].double() @ xt[j0:j0 + 2048]
        _, _, be0 = rb.refine(a32, lu32, b, tol=1e-14, max_iter=0)
        x, it, be = rb.refine(a32, lu32, b, tol=1e-14, max_iter=30)
        return be0, it, be

    seed = 1
    reps = max(args.steps, 1)
    with ClockSampler(torch.cuda.current_device()) as clk:
        for alpha in (1.05, 1.5, 4.0):
            for k in (0, 8):
                a = rb.gen_matrix(n, seed=seed, kind=1, alpha=alpha, kscale=k)
                amax = float(a.abs().max())
                lu = rb.colmajor_empty(n, n, n, torch.float32)
                info = torch.zeros(1, dtype=torch.int32, device="cuda")
                ms = timed(lambda: (lu.copy_(a), rb.lu_nopiv_rl(lu, nb=256, outer=rb.TC32,
                                                                 info=info)), reps)
                t_copy = timed(lambda: lu.copy_(a), reps)
                ms_f = max(ms - t_copy, 1e-6)
                lu.copy_(a)
                rb.lu_nopiv_rl(lu, nb=256, outer=rb.TC32, info=info)
                be0, it, be = solve_quality(a, lu)
                rl = {"tflops": lu_flops(n) / (ms_f / 1e3) / 1e12, "ms": ms_f,
                      "info": int(info.item()), "finite": bool(torch.isfinite(lu).all()),
                      "berr_unrefined": be0, "refine_iters": it, "berr": be}
                # (ii) fp16 storage, left-looking
                s_log2 = 0
                while amax * 2.0 ** (-s_log2) > 30000.0:
                    s_log2 += 1
                a16 = rb.colmajor_empty(n, n, n, torch.float16)
                a16.copy_(a * 2.0 ** (-s_log2))
                w16 = rb.colmajor_empty(n, n, n, torch.float16)
                ms16 = timed(lambda: (w16.copy_(a16), rb.lu_nopiv_ll(w16, nb=128, outer=rb.TC32,
                                                                      info=info)), reps)
                t16 = timed(lambda: w16.copy_(a16), reps)
                ms16_f = max(ms16 - t16, 1e-6)
                w16.copy_(a16)
                rb.lu_nopiv_ll(w16, nb=128, outer=rb.TC32, info=info)
                info16 = int(info.item())
                lu.copy_(w16)
                if s_log2:
                    lu.copy_(torch.tril(lu, -1) + torch.triu(lu) * 2.0 ** s_log2)
                be0h, ith, beh = solve_quality(a, lu)
                ll = {"tflops": lu_flops(n) / (ms16_f / 1e3) / 1e12, "ms": ms16_f,
                      "info": info16, "finite": bool(torch.isfinite(w16).all()),
                      "fp16_scale_log2": -s_log2, "berr_unrefined": be0h,
                      "refine_iters": ith, "berr": beh}
                runs.append({"alpha": alpha, "kscale": k, "seed": seed, "max_abs_a": amax,
                             "rl_tc32_f32": rl, "ll_f16": ll})
                del a, lu, a16, w16
                torch.cuda.empty_cache()
                seed += 1
    worst = min(r["rl_tc32_f32"]["tflops"] for r in runs)
    line = _base_line(args, "LU TFLOP/s (2n^3/3), smallest over the C2 matrix grid", worst,
                      "TFLOP/s", lu_flops(n) / worst / 1e9,
                      dtype="f32 storage + TC32 (RL); f16 storage + TC32 (LL)",
                      config={"workload": args.workload, "n": n, "nb_rl": 256, "nb_ll": 128,
                              "matrix": "2^k (R + D), R ~ N(0,1)/sqrt(n), dominance alpha",
                              "grid": "alpha in {1.05, 1.5, 4} x k in {0, 8}, seeds 1..6"})
    line["runs"] = runs
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def run_special(args) -> None:
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return  # under torchrun rank 0 alone reports
        print(json.dumps({"impl": "reference", "workload": args.workload,
                          "unavailable": "the reference has no batched, fp16-left-looking "
                                         "timing harness, refinement or adjoint for this "
                                         "workload; see the cpu_baseline field of our line"}))
        return
    import torch
    import remifa_b200 as rb
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    fn = {"batch_10000_n16_512": run_batch, "ll_f16_n16384": run_ll16,
          "precision_n32768": run_precision, "adjoint_n8192": run_adjoint,
          "c2_grid_n16384": run_c2_grid}[args.workload]
    fn(args, torch, rb)


if __name__ == "__main__":
    main()
