"""Benchmark of the KAMI block-GEMM hot path on B200.

Workload (default): FP16 block GEMM with FP32 accumulation, M = N = K = 128,
one problem per CTA, batch = 4 x SM count (592 on a 148-SM B200), the
reference's in-register repeat method with NUM_ITER = 1000 (every CTA
multiplies its resident A and B 1000 times; FLOPs = 2*M*N*K*batch*NUM_ITER,
block_gemm_1d_half_mma.cu:255-258).  Inputs: uniform[-1, 1] rounded to
FP16, seed 0, synthetic.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is device time of the GEMM launches only
(inputs resident in HBM; the 256 MiB L2 flush between steps is outside the
timed events); `e2e` is the same metric through the public C-ABI call on
host buffers (kami_gemm_batched_host: the inputs copied from pinned host
memory and C copied back inside the timed region; the batch in chunks whose
products start as their inputs land, so copies and products overlap).  With --gpus N > 1 every rank runs its own replica (weak scaling);
the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20


class L2Flush:
    """Between timed steps: write a buffer larger than the 126 MB L2, then read
    a second one, so the timed kernel finds neither its inputs in L2 nor
    dirty flush lines it would have to write back (both outside the events)."""

    def __init__(self, dev):
        import torch
        self.w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
        self.r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def zero_(self):
        self.w.zero_()
        self.r.sum()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--num-iter", type=int, default=1000)
    ap.add_argument("--variant", default="auto", choices=["auto", "mma_sync", "tcgen05", "tcgen05_ts"])
    ap.add_argument("--partition", default="auto", choices=["auto", "1d", "2d", "3d"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="bounded CPU-baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="block",
                    choices=["block", "block-sweep", "fp64", "split", "uneven", "spgemm", "spmm", "bmm",
                             "comparators", "ksplit", "case"],
                    help="block (default, the headline line) or one of the other configurations; "
                         "non-default workloads print one JSON line per measured case")
    ap.add_argument("--case", default="block128",
                    choices=["block128", "stream128", "fp64-64", "split-int8x7", "split-fp16x6", "spgemm-numeric",
                             "spgemm-symbolic",
                             "uneven-f16", "bmm-bf16"],
                    help="--workload case: run one benchmark case three times, untimed (for profiler captures)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("bf16_tflops"), d.get("hbm_gbs"), "measured"
    return 1590.0, 6650.0, "fallback"


def ncu_traffic(kernel_key: str):
    """DRAM bytes per launch from the committed ncu summary (profiles/*.md,
    a line `traffic_bytes_per_launch[<key>]: <int>`), else None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    tag = f"traffic_bytes_per_launch[{kernel_key}]:"
    for fn in sorted(os.listdir(d)):
        if fn.endswith((".md", ".txt")):
            for ln in open(os.path.join(d, fn)):
                if ln.strip().startswith(tag):
                    try:
                        return int(ln.split(":", 1)[1].strip())
                    except ValueError:
                        return None
    return None


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (restated reference check loop), bounded sample
# ---------------------------------------------------------------------------
def cpu_sample(M, N, K, seconds):
    import oracle
    rng = np.random.default_rng(0)
    A1 = rng.uniform(-1, 1, (1, M, K)).astype(np.float16)
    B1 = rng.uniform(-1, 1, (1, N, K)).astype(np.float16)
    t0 = time.perf_counter()
    oracle.gemm(A1, B1)
    t1 = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    n = int(max(1, min(4096, seconds / max(t1, 1e-6) * cores * 0.7)))
    A = rng.uniform(-1, 1, (n, M, K)).astype(np.float16)
    B = rng.uniform(-1, 1, (n, N, K)).astype(np.float16)
    t0 = time.perf_counter()
    oracle.gemm(A, B)
    dt = time.perf_counter() - t0
    flops = 2.0 * M * N * K * n
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": "port",
            "sample": f"{n} problems of {M}x{N}x{K} FP16 inputs, double accumulation (the reference's host "
                      f"check loop, OpenMP over problems), {dt:.2f} s"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (the oracle restatement of
    its host check GEMM) on the host cores, same metric and config."""
    if rank != 0:
        return
    M = N = K = args.size
    batch = 4 * 148
    for _ in range(args.warmup):
        cpu_sample(M, N, K, 1.0)
    vals = []
    t0 = time.perf_counter()
    last = None
    for _ in range(args.steps):
        last = cpu_sample(M, N, K, max(1.0, args.cpu_seconds / max(args.steps, 1)))
        vals.append(last["value"])
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    cfg = {"workload": f"fp16 block GEMM {M}x{N}x{K}, fp32 accumulate, batch {batch}", "M": M, "N": N, "K": K,
           "batch": batch, "num_iter": args.num_iter}
    out = {"impl": "reference", "metric": "block-GEMM TFLOPS", "value": v, "unit": "TFLOP/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16", "data": "synthetic",
           "config": cfg,
           "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": last["cores"], "kind": "port",
                            "sample": last["sample"]},
           "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def run_ours(args, rank, world):
    import torch
    from kami_b200 import api, replicas

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    M = N = K = args.size
    batch = 4 * sms
    num_iter = args.num_iter
    g = torch.Generator(device="cpu").manual_seed(0 + rank)
    A_h = (torch.rand((batch, M, K), generator=g) * 2 - 1).half()
    B_h = (torch.rand((batch, N, K), generator=g) * 2 - 1).half()
    A = A_h.to(dev)
    B = B_h.to(dev)
    C = torch.empty((batch, M, N), dtype=torch.float32, device=dev)
    flush = L2Flush(dev)
    stream = torch.cuda.current_stream(dev)
    plan = api.describe(M, N, K, batch, torch.float16, variant=args.variant, partition=args.partition)

    def step():
        api.gemm_batched(A, B, C, variant=args.variant, partition=args.partition, num_iter=num_iter)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # correctness spot check of one problem against a double reference on the host
    ref = (A_h[0].double() @ B_h[0].double().T) * num_iter
    got = C[0].double().cpu()
    rel = float((got - ref).norm() / ref.norm())

    replicas.barrier()
    sampler = ClockSampler(dev.index) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in times]
    replicas.barrier()
    # ---- end-to-end through the C ABI with host buffers ----
    A_pin = A_h.pin_memory()
    B_pin = B_h.pin_memory()
    C_pin = torch.empty((batch, M, N), dtype=torch.float32).pin_memory()
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # the public host-buffer call: copies in, products, copies out,
        # overlapped chunk by chunk
        api.gemm_batched_host(A_pin, B_pin, C_pin, variant=args.variant, partition=args.partition,
                              num_iter=num_iter, stream=stream)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    clocks = sampler.stop() if sampler else None
    # context only: this box's cuBLAS bf16 rate right now (8192^3), to tell a
    # slow box from a slow kernel; the roofline denominator stays the
    # driver-measured peak
    calib = None
    try:
        x = torch.randn(8192, 8192, device=dev, dtype=torch.bfloat16)
        y = torch.randn(8192, 8192, device=dev, dtype=torch.bfloat16)
        cm = _time_ms(lambda: torch.matmul(x, y), 3, 5)
        calib = {"cublas_bf16_8192_tflops": 2 * 8192 ** 3 / (min(cm) * 1e-3) / 1e12}
        del x, y
    except Exception as e:  # pragma: no cover
        calib = {"error": str(e)[:80]}

    step_ms = sum(ms) / len(ms)
    e2e_step = sum(e2e_ms) / len(e2e_ms)
    step_ms, e2e_step = replicas.max_over_ranks([step_ms, e2e_step], dev)
    flops_rank = 2.0 * M * N * K * batch * num_iter
    value = replicas.aggregate_rate(flops_rank, step_ms, world) / 1e12
    e2e_value = replicas.aggregate_rate(flops_rank, e2e_step, world) / 1e12
    if rank != 0:
        return
    peak_tf, peak_bw, src = measured_peaks()
    # the same statistic as `value`: mean device time of the timed launches
    achieved = flops_rank / (statistics.fmean(ms) * 1e-3) / 1e12
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": achieved / peak_tf, "peak_source": f"{src} bf16 dense (burst)",
            "traffic": ncu_traffic(f"gemm_{plan['variant']}_{M}"),
            "algorithmic_bytes_per_launch": batch * (M * K * 2 + N * K * 2 + M * N * 4)}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_sample(M, N, K, args.cpu_seconds)
    out = {"metric": "block-GEMM TFLOPS", "value": value, "unit": "TFLOP/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f16",
           "data": "synthetic (uniform[-1,1] rounded to fp16, seed 0)",
           "config": {"workload": f"fp16 block GEMM {M}x{N}x{K}, fp32 accumulate, batch {batch} "
                                  f"(4 x {sms} SMs), NUM_ITER {num_iter} in-register repeats",
                      "M": M, "N": N, "K": K, "batch": batch, "num_iter": num_iter,
                      "variant": plan["variant"], "partition": plan["partition"], "P": plan["P"],
                      "threads": plan["threads"], "l2": "256 MiB buffer written, then another 256 MiB read, between timed steps",
                      "parallelism": f"replicas x{world}"},
           "roofline": roof, "cpu_baseline": cpu,
           "e2e": {"value": e2e_value, "unit": "TFLOP/s",
                   "h2d_bytes_per_step": int(A_h.numel() * 2 + B_h.numel() * 2),
                   "d2h_bytes_per_step": int(C.numel() * 4)},
           "gpu_launches": args.steps, "clocks": clocks, "check_rel_err": rel, "box_calibration": calib}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# secondary workloads (one JSON line per case; the default run is `block`)
# ---------------------------------------------------------------------------
def _time_ms(fn, warmup, steps, flush=None):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        ts.append((e0, e1))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ts]


def _emit(d):
    print(json.dumps(d), flush=True)


def run_case(args):
    """One benchmark case, three times, untimed: the command the profiles under
    profiles/ were captured with (ncu -k <kernel> -s 2 -c 1 python bench.py
    --workload case --case <name>)."""
    import numpy as np
    import torch

    import oracle
    from kami_b200 import api
    from kami_b200.autograd import bmm

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    g = torch.Generator().manual_seed(0)
    c = args.case
    if c in ("block128", "stream128"):
        b = 4 * sms
        A = (torch.rand((b, 128, 128), generator=g) * 2 - 1).half().to(dev)
        B = (torch.rand((b, 128, 128), generator=g) * 2 - 1).half().to(dev)
        C = torch.empty((b, 128, 128), dtype=torch.float32, device=dev)
        it = args.num_iter if c == "block128" else 1
        fn = lambda: api.gemm_batched(A, B, C, variant=args.variant, partition=args.partition, num_iter=it)
    elif c == "fp64-64":
        A = (torch.rand((8192, 64, 64), generator=g, dtype=torch.float64) * 2 - 1).to(dev)
        B = (torch.rand((8192, 64, 64), generator=g, dtype=torch.float64) * 2 - 1).to(dev)
        C = torch.empty((8192, 64, 64), dtype=torch.float64, device=dev)
        fn = lambda: api.gemm_batched(A, B, C)
    elif c in ("split-int8x7", "split-fp16x6"):
        # the split-FP64 streamed workload: 8192 x 64^3, sign * 10^u, 7 int8 or 6 FP16 digits
        rng = np.random.default_rng(0)
        A = torch.tensor(rng.choice([-1.0, 1.0], (8192, 64, 64)) * 10.0 ** rng.uniform(-3, 3, (8192, 64, 64)),
                         device=dev)
        B = torch.tensor(rng.choice([-1.0, 1.0], (8192, 64, 64)) * 10.0 ** rng.uniform(-3, 3, (8192, 64, 64)),
                         device=dev)
        C = torch.empty((8192, 64, 64), dtype=torch.float64, device=dev)
        ns, sdt = (7, torch.int8) if c == "split-int8x7" else (6, torch.float16)
        fn = lambda: api.split_f64_gemm(A, B, C, nslices=ns, slice_dtype=sdt)
    elif c in ("spgemm-numeric", "spgemm-symbolic"):
        nb = 1024
        rpa, cia = oracle.bsr_pattern(nb, nb, 0.01, 1)
        rpb, cib = oracle.bsr_pattern(nb, nb, 0.01, 2)
        rng = np.random.default_rng(0)
        va = torch.tensor(rng.uniform(-1, 1, (len(cia), 16, 16)), dtype=torch.float16, device=dev)
        vb = torch.tensor(rng.uniform(-1, 1, (len(cib), 16, 16)), dtype=torch.float16, device=dev)
        Am = api.BSR(torch.tensor(rpa, device=dev), torch.tensor(cia, device=dev), va, nb)
        Bm = api.BSR(torch.tensor(rpb, device=dev), torch.tensor(cib, device=dev), vb, nb)
        rpc, nnzc = api.spgemm_symbolic(Am, Bm)
        cic = api.spgemm_fill_colidx(Am, Bm, rpc, nnzc)
        vc = torch.empty((nnzc, 16, 16), dtype=torch.float32, device=dev)
        cap = oracle.spgemm_nnzcub(cia, rpb)
        variant = args.variant if args.variant in ("mma_sync", "tcgen05") else "auto"
        fn = (lambda: api.spgemm_numeric(Am, Bm, rpc, cic, C_values=vc, variant=variant)) if c == "spgemm-numeric" \
            else (lambda: api.spgemm_symbolic_device(Am, Bm, cap))
    elif c == "uneven-f16":
        rng = np.random.default_rng(0)
        x = np.exp(rng.uniform(np.log(8), np.log(128), (20000, 3)))
        plan = api.GroupedPlan(np.clip(8 * np.round(x / 8), 8, 128).astype(np.int64), torch.float16)
        A = torch.rand(plan.sizes[0], device=dev).half()
        B = torch.rand(plan.sizes[1], device=dev).half()
        C = torch.empty(plan.sizes[2], dtype=torch.float32, device=dev)
        fn = lambda: plan.run(A, B, C)
    else:  # bmm-bf16: autograd forward + backward, 4096 x 64^3
        A = (torch.rand((4096, 64, 64), generator=g) * 2 - 1).bfloat16().to(dev).requires_grad_()
        B = (torch.rand((4096, 64, 64), generator=g) * 2 - 1).bfloat16().to(dev).requires_grad_()
        G = (torch.rand((4096, 64, 64), generator=g) * 2 - 1).bfloat16().to(dev)

        def fn():
            A.grad = B.grad = None
            bmm(A, B).backward(G)
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    print(json.dumps({"workload": "case", "case": c, "done": 3}), flush=True)


def run_secondary(args):
    import numpy as np
    import torch

    import oracle
    from kami_b200 import api
    from kami_b200.autograd import bmm

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    flush = L2Flush(dev)
    peak_tf, peak_bw, src = measured_peaks()
    W, K_ = max(args.warmup, 3), args.steps

    if args.workload == "block-sweep":
        cases = [(n, n, n) for n in (16, 32, 64, 128)] + [(128, 128, 8), (128, 128, 16), (128, 128, 32)]
        for (M, N, K) in cases:
            batch = 4 * sms
            g = torch.Generator().manual_seed(0)
            A = (torch.rand((batch, M, K), generator=g) * 2 - 1).half().to(dev)
            B = (torch.rand((batch, N, K), generator=g) * 2 - 1).half().to(dev)
            C = torch.empty((batch, M, N), dtype=torch.float32, device=dev)
            for variant in ("mma_sync", "tcgen05", "tcgen05_ts"):
                for part in ("1d", "2d", "3d"):
                    for it in (1000, 1):
                        try:
                            plan = api.describe(M, N, K, batch, variant=variant, partition=part)
                        except Exception as e:  # no kernel for this combination
                            _emit({"workload": "block-sweep", "M": M, "N": N, "K": K, "variant": variant,
                                   "partition": part, "unavailable": str(e)[:120]})
                            continue
                        ms = _time_ms(lambda: api.gemm_batched(A, B, C, variant=variant, partition=part,
                                                               num_iter=it), W, K_, flush)
                        t = min(ms)
                        fl = 2.0 * M * N * K * batch * it
                        by = batch * (M * K * 2 + N * K * 2 + M * N * 4)
                        _emit({"workload": "block-sweep", "M": M, "N": N, "K": K, "batch": batch, "num_iter": it,
                               "variant": plan["variant"], "partition": plan["partition"], "P": plan["P"],
                               "threads": plan["threads"], "ms": t, "tflops": fl / t / 1e9,
                               "frac_tensor_peak": fl / t / 1e9 / peak_tf,
                               "hbm_gbs": by / t / 1e6, "frac_hbm": by / t / 1e6 / peak_bw})
        return

    if args.workload == "fp64":
        # 1024 independent 32^3 FP64 problems, uniform[-1, 1], seed 0; streamed (NUM_ITER 1) and repeat
        rng = np.random.default_rng(0)
        for (n, batch) in [(32, 1024), (64, 8192), (32, 65536)]:
            A64 = rng.uniform(-1, 1, (batch, n, n))
            B64 = rng.uniform(-1, 1, (batch, n, n))
            A = torch.tensor(A64, device=dev)
            B = torch.tensor(B64, device=dev)
            C = torch.empty((batch, n, n), dtype=torch.float64, device=dev)
            ref = oracle.gemm(A64[:64], B64[:64])
            for part in ("1d", "2d", "3d"):
                for it in (1, 100):
                    try:
                        plan = api.describe(n, n, n, batch, torch.float64, partition=part)
                    except Exception as e:
                        _emit({"workload": "fp64", "n": n, "partition": part, "unavailable": str(e)[:100]})
                        continue
                    ms = _time_ms(lambda: api.gemm_batched(A, B, C, partition=part, num_iter=it), W, K_, flush)
                    err = float(np.max(np.abs(C[:64].cpu().numpy() / it - ref)))
                    t = min(ms)
                    fl = 2.0 * n ** 3 * batch * it
                    by = batch * 3 * n * n * 8
                    _emit({"workload": "fp64", "n": n, "batch": batch, "num_iter": it, "partition": part,
                           "P": plan["P"], "ms": t, "tflops": fl / t / 1e9, "hbm_gbs": by / t / 1e6,
                           "frac_hbm": by / t / 1e6 / peak_bw, "max_abs_err_vs_oracle": err})
        return

    if args.workload == "split":
        # batch 8192 of 64^3, entries sign * 10^u, u ~ U[-3, 3]
        rng = np.random.default_rng(0)
        batch, n = 8192, 64
        A64 = rng.choice([-1.0, 1.0], (batch, n, n)) * 10.0 ** rng.uniform(-3, 3, (batch, n, n))
        B64 = rng.choice([-1.0, 1.0], (batch, n, n)) * 10.0 ** rng.uniform(-3, 3, (batch, n, n))
        A = torch.tensor(A64, device=dev)
        B = torch.tensor(B64, device=dev)
        C = torch.empty((batch, n, n), dtype=torch.float64, device=dev)
        sub = 256
        hi, lo = oracle.gemm_dd(A64[:sub], B64[:sub])
        fl1 = 2.0 * n ** 3 * batch
        by = batch * 3 * n * n * 8
        for it in (1, 20):
            ms = _time_ms(lambda: api.gemm_batched(A, B, C, num_iter=it), W, K_, flush)
            e_nat = oracle.normwise_error_dd(C[:sub].cpu().numpy() / it, hi, lo)
            t = min(ms)
            _emit({"workload": "split", "kernel": "native-fp64 (DMMA mma.sync)", "num_iter": it, "ms": t,
                   "tflops_fp64_equiv": fl1 * it / t / 1e9, "hbm_gbs": by / t / 1e6, "normwise_err_dd": e_nat})
            for s_, sdt in [(3, torch.float16), (4, torch.float16), (5, torch.float16), (6, torch.float16),
                            (7, torch.float16), (8, torch.bfloat16), (6, torch.int8), (7, torch.int8),
                            (8, torch.int8)]:
                ms = _time_ms(lambda: api.split_f64_gemm(A, B, C, nslices=s_, slice_dtype=sdt, num_iter=it),
                              W, K_, flush)
                e = oracle.normwise_error_dd(C[:sub].cpu().numpy() / it, hi, lo) if it == 1 else None
                t = min(ms)
                sname = {torch.bfloat16: "bf16", torch.float16: "fp16", torch.int8: "int8"}[sdt]
                _emit({"workload": "split", "kernel": f"split {s_} x {sname}",
                       "num_iter": it, "ms": t, "tflops_fp64_equiv": fl1 * it / t / 1e9,
                       "hbm_gbs": by / t / 1e6, "normwise_err_dd": e})
        return

    if args.workload == "uneven":
        rng = np.random.default_rng(0)
        count = 20000
        x = np.exp(rng.uniform(np.log(8), np.log(128), (count, 3)))
        shapes = np.clip(8 * np.round(x / 8), 8, 128).astype(np.int64)
        for dt, tune, pack in ((torch.float16, False, False), (torch.float16, False, True),
                               (torch.float16, True, False), (torch.float64, False, False), (torch.float64, True, False)):
            if True:
                plan = api.GroupedPlan(shapes, dt, autotune=tune, pack=pack)
                info = plan.info()
                A = torch.rand(plan.sizes[0], device=dev).to(dt)
                B = torch.rand(plan.sizes[1], device=dev).to(dt)
                C = torch.empty(plan.sizes[2], dtype=plan.out_dtype, device=dev)
                plan.run(A, B, C)
                torch.cuda.synchronize()
                gph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(gph):
                    plan.run(A, B, C)
                ms = _time_ms(gph.replay, W, K_, flush)
                t = min(ms)
                _emit({"workload": "uneven", "dtype": str(dt).replace("torch.", ""), "autotune": tune,
                       "kernel": info["kernel"], "packed": pack and info["kernel"] == "tcgen05", "problems": count, "launches_per_step": 1, "cuda_graph": True, "ms": t,
                       "tflops": info["flops"] / t / 1e9, "hbm_gbs": info["bytes"] / t / 1e6,
                       "frac_hbm": info["bytes"] / t / 1e6 / peak_bw, "ctas": info["ctas"],
                       "partitions": info["partitions"], "flops": info["flops"], "bytes": info["bytes"]})
                del gph
        return

    if args.workload == "spgemm":
        # (a) the reference programs' method: one 128 x 128 BSR pair (8 x 8
        # tiles, the reference generator at sparsity 0.5, A = B as its
        # srand(0) reuse gives) per CTA, 16384 CTAs sharing it, NUM_ITER 1000,
        # FLOPs 2 * 16^3 * nnzCub * grid * NUM_ITER (spgemm/2d/...:763-768, 839-840)
        rp, ci, vals = oracle.bsr_generate(8, 8, 0.5)
        rpc_o, cic_o, vc_o = oracle.spgemm(8, 8, (rp, ci, vals), (rp, ci, vals), accum="double")
        nnzcub_b = oracle.spgemm_nnzcub(ci, rp)
        Ab = api.BSR(torch.tensor(rp, device=dev), torch.tensor(ci, device=dev), torch.tensor(vals, device=dev), 8)
        grid_b = 16384
        for part, P in [("1d", 4), ("1d", 8), ("2d", 2), ("3d", 2)]:
            for it in (1000,):
                Cb = api.BSR(torch.tensor(rpc_o, device=dev), torch.tensor(cic_o, device=dev),
                             torch.empty((grid_b, len(cic_o), 16, 16), dtype=torch.float32, device=dev), 8)
                ms = _time_ms(lambda: api.spgemm_block(Ab, Ab, Cb, partition=part, P=P, num_iter=it), W, K_, flush)
                t = statistics.fmean(ms)
                fl = 2.0 * 16 ** 3 * nnzcub_b * grid_b * it
                err = float(np.abs(Cb.values[grid_b - 1].double().cpu().numpy() / it - vc_o).max())
                _emit({"workload": "spgemm", "case": "reference block 128x128, 50 % tiles, 16384 CTAs",
                       "partition": part, "P": P, "nnzCub": nnzcub_b, "num_iter": it, "ms": t,
                       "tflops": fl / t / 1e9, "frac_tensor_peak": fl / t / 1e9 / peak_tf,
                       "max_abs_err_vs_oracle": err})
                del Cb
        nb = 1024  # n = 16384 with 16 x 16 blocks
        res = []
        for seed_a, seed_b in [(1, 2)]:
            rpa, cia = oracle.bsr_pattern(nb, nb, 0.01, seed_a)
            rpb, cib = oracle.bsr_pattern(nb, nb, 0.01, seed_b)
            rng = np.random.default_rng(0)
            va = torch.tensor(rng.uniform(-1, 1, (len(cia), 16, 16)), dtype=torch.float16, device=dev)
            vb = torch.tensor(rng.uniform(-1, 1, (len(cib), 16, 16)), dtype=torch.float16, device=dev)
            A = api.BSR(torch.tensor(rpa, device=dev), torch.tensor(cia, device=dev), va, nb)
            B = api.BSR(torch.tensor(rpb, device=dev), torch.tensor(cib, device=dev), vb, nb)
            nnzcub = oracle.spgemm_nnzcub(cia, rpb)
            rpc, nnzc = api.spgemm_symbolic(A, B)
            cic = api.spgemm_fill_colidx(A, B, rpc, nnzc)
            vc = torch.empty((nnzc, 16, 16), dtype=torch.float32, device=dev)

            def symbolic():
                r, _ = api.spgemm_symbolic(A, B)
                api.spgemm_fill_colidx(A, B, r, nnzc)

            ms_sym = _time_ms(symbolic, W, K_, flush)
            ms_var = {}
            for variant in ("mma_sync", "tcgen05"):
                ms_var[variant] = _time_ms(lambda: api.spgemm_numeric(A, B, rpc, cic, C_values=vc, variant=variant),
                                           W, K_, flush)
            ms_num = _time_ms(lambda: api.spgemm_numeric(A, B, rpc, cic, C_values=vc), W, K_, flush)
            # the same product with no host round trip: on-device symbolic pass
            # into a capacity of nnzCub (an upper bound of nnzC), then numeric
            cap = nnzcub
            vcap = torch.empty((cap, 16, 16), dtype=torch.float32, device=dev)
            ms_symd = _time_ms(lambda: api.spgemm_symbolic_device(A, B, cap), W, K_, flush)

            def device_pipeline():
                r, c_ = api.spgemm_symbolic_device(A, B, cap)
                api.spgemm_numeric_bound(A, B, r, c_, vcap)

            ms_dev = _time_ms(device_pipeline, W, K_, flush)
            fl = 2.0 * 16 ** 3 * nnzcub
            by = (len(cia) + len(cib)) * 512 + nnzc * 1024 + nnzc * 4 + (len(cia) + len(cib)) * 4
            t = min(ms_num)
            # check a sample of rows against the CPU oracle
            _emit({"workload": "spgemm", "n": nb * 16, "block": 16, "density": 0.01, "nnzA": len(cia),
                   "nnzB": len(cib), "nnzC": nnzc, "nnzCub": nnzcub, "numeric_ms": t,
                   "symbolic_ms": min(ms_sym), "tflops_numeric": fl / t / 1e9,
                   "hbm_gbs_numeric": by / t / 1e6, "frac_hbm": by / t / 1e6 / peak_bw,
                   "tflops_end_to_end": fl / (t + min(ms_sym)) / 1e9, "symbolic_device_ms": min(ms_symd),
                   "end_to_end_device_ms": min(ms_dev), "tflops_end_to_end_device": fl / min(ms_dev) / 1e9,
                   "numeric_ms_by_variant": {v: statistics.fmean(m) for v, m in ms_var.items()},
                   "frac_hbm_by_variant": {v: by / statistics.fmean(m) / 1e6 / peak_bw for v, m in ms_var.items()}})
        return

    if args.workload == "spmm":
        # (a) the reference programs' own shape and method: one 64 x 64 BSR block
        # (4 x 4 tiles, the reference generator at sparsity 0.5) times a dense
        # 64 x 64 B per CTA, 16384 CTAs sharing A and B, NUM_ITER 1000
        #  (spmm/1d/block_spmm_1d_half_mma.cu:229-285; FLOPs 2 * nnz * N).
        rp, ci, vals = oracle.bsr_generate(4, 4, 0.5, rule="spmm1d")
        rng = np.random.default_rng(0)
        Bh = torch.tensor(rng.integers(0, 3, (64, 64)), dtype=torch.float16, device=dev)
        d_rp, d_ci = torch.tensor(rp, device=dev), torch.tensor(ci, device=dev)
        d_v = torch.tensor(vals, device=dev)
        for batch, it in [(16384, 1000), (16384, 1)]:
            Cb = torch.empty((batch, 64, 64), dtype=torch.float32, device=dev)
            ms = _time_ms(lambda: api.spmm_batched(d_rp, d_ci, d_v, 4, Bh, Cb, b_layout="ref_nk", num_iter=it),
                          W, K_, flush)
            t = min(ms)
            fl = 2.0 * ci.size * 256 * 64 * batch * it
            ref = oracle.spmm(rp, ci, vals.astype(np.float64), 4, Bh.double().cpu().numpy(), "ref_nk")
            err = float(np.abs(Cb[batch - 1].double().cpu().numpy() / it - ref).max())
            _emit({"workload": "spmm", "case": "reference block 64x64x64, 50 % tiles, shared A/B",
                   "nnz_blocks": int(ci.size), "batch": batch, "num_iter": it, "ms": t, "tflops": fl / t / 1e9,
                   "frac_tensor_peak": fl / t / 1e9 / peak_tf, "max_abs_err_vs_oracle": err})
        # (b) a large SpMM, streamed: n = 16384 (1024 x 1024 tiles), 1 % tiles,
        # dense B 16384 x 256, FP16 in, FP32 out
        nb, Nd = 1024, 256
        rp, ci = oracle.bsr_pattern(nb, nb, 0.01, 1)
        va = torch.tensor(rng.uniform(-1, 1, (len(ci), 16, 16)), dtype=torch.float16, device=dev)
        A = api.BSR(torch.tensor(rp, device=dev), torch.tensor(ci, device=dev), va, nb)
        for lay in ("row_kn", "ref_nk"):
            Bd = torch.tensor(rng.uniform(-1, 1, (nb * 16, Nd) if lay == "row_kn" else (Nd, nb * 16)),
                              dtype=torch.float16, device=dev)
            C = torch.empty((nb * 16, Nd), dtype=torch.float32, device=dev)
            ms = _time_ms(lambda: api.spmm(A, Bd, C, b_layout=lay), W, K_, flush)
            t = min(ms)
            fl = 2.0 * len(ci) * 256 * Nd
            by = len(ci) * (512 + 4) + (nb + 1) * 4 + nb * 16 * Nd * 2 + nb * 16 * Nd * 4
            rows = slice(0, 64 * 16)
            ref = oracle.spmm(rp[:65], ci[: rp[64]], va[: rp[64]].double().cpu().numpy(), nb,
                              Bd.double().cpu().numpy(), lay)
            err = float(np.abs(C[rows].double().cpu().numpy() - ref).max())
            _emit({"workload": "spmm", "case": f"n=16384, 1 % tiles, dense {Nd} columns, B {lay}",
                   "nnz_blocks": int(len(ci)), "ms": t, "tflops": fl / t / 1e9, "hbm_gbs": by / t / 1e6,
                   "frac_hbm": by / t / 1e6 / peak_bw, "max_abs_err_first_64_block_rows": err})
        return

    if args.workload == "ksplit":
        # the register / shared-memory K split of the 1D mma.sync block GEMM at
        # 128^3 (the reference's reg_smem program: 1D FP16 128^3 with
        # REG_K_SPLIT_BLOCK of 8 k-steps in registers), in the reference's
        # repeat method, and the per-warp communication / computation cycles
        # of the traced instances (its usage_cycle programs)
        rng = np.random.default_rng(0)
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        b, n, it = 4 * sms, 128, 1000
        A = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).half()
        B = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).half()
        C = torch.empty((b, n, n), dtype=torch.float32, device=dev)
        fl = 2.0 * n ** 3 * b * it
        for P, rk in ((4, 0), (4, 2), (4, 4), (8, 0), (8, 4), (8, 8), (0, -1)):
            used = [None]

            def run():
                used[0] = api.gemm_batched_ksplit(A, B, C, P=P, reg_k_steps=rk, num_iter=it)[1]

            t = min(_time_ms(run, W, K_, flush))
            _emit({"workload": "ksplit", "tile": n, "P": P, "reg_k_steps": rk, "reg_k_used": used[0],
                   "num_iter": it, "ms": t, "tflops": fl / t / 1e9, "frac_tensor_peak": fl / t / 1e9 / peak_tf})
        for part, P, rk in (("1d", 8, -1), ("1d", 4, 4), ("1d", 4, 0), ("2d", 4, -1), ("3d", 2, -1)):
            _, cyc = api.gemm_trace(A[0], B[0], partition=part, P=P, reg_k_steps=rk, num_iter=10)
            _emit({"workload": "ksplit-trace", "tile": n, "partition": part, "P": P, "reg_k_steps": rk,
                   "num_iter": 10, "comm_cycles_per_iter": [int(x) // 10 for x in cyc[:, 0]],
                   "comp_cycles_per_iter": [int(x) // 10 for x in cyc[:, 1]]})
        return

    if args.workload == "comparators":
        # the vendor library (cuBLAS through torch) on the same workloads and
        # data as this library's kernels, side by side (context, not a target)
        rng = np.random.default_rng(0)

        def pair(name, ours, theirs, flops, by):
            for impl, fn in (("kami_b200", ours), ("cublas", theirs)):
                ms = _time_ms(fn, W, K_, flush)
                t = min(ms)
                _emit({"workload": "comparators", "case": name, "impl": impl, "ms": t, "ms_mean": statistics.fmean(ms),
                       "tflops": flops / t / 1e9, "hbm_gbs": by / t / 1e6 if by else None})

        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        # CUTLASS's own sm_100a batched GEMM (tcgen05 / TMA / TMEM collectives,
        # cluster 1 x 1 x 1) on the same buffers, reference B layout (N x K)
        import ctypes
        from kami_b200 import build as kbuild
        cmp_path = kbuild.build_comparators()
        if cmp_path:
            CL = ctypes.CDLL(cmp_path)
            CL.kami_cmp_cutlass_gemm_batched.argtypes = [ctypes.c_int] * 6 + [ctypes.c_int64] + \
                [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
            dtc = {torch.float16: 0, torch.bfloat16: 1, torch.float32: 3}
            for (b, n, idt, odt) in ((4 * sms, 128, torch.float16, torch.float32),
                                     (4 * sms, 128, torch.float16, torch.float16),
                                     (2048, 128, torch.bfloat16, torch.bfloat16),
                                     (4096, 64, torch.bfloat16, torch.bfloat16),
                                     (8192, 64, torch.float16, torch.float32)):
                A = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).to(idt)
                B = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).to(idt)
                C1 = torch.empty((b, n, n), dtype=odt, device=dev)
                C2 = torch.empty((b, n, n), dtype=odt, device=dev)
                need = ctypes.c_size_t(0)
                tile = 64 if n == 64 else 128
                args0 = (dtc[idt], dtc[odt], tile, n, n, n, b, A.data_ptr(), B.data_ptr(), C2.data_ptr())
                CL.kami_cmp_cutlass_gemm_batched(*args0, None, 0, ctypes.byref(need), None)
                ws = torch.empty(max(int(need.value), 16), dtype=torch.uint8, device=dev)
                strm = torch.cuda.current_stream(dev).cuda_stream

                def cutlass_run():
                    st = CL.kami_cmp_cutlass_gemm_batched(*args0, ws.data_ptr(), ws.numel(), None, strm)
                    if st != 0:
                        raise RuntimeError(f"CUTLASS comparator returned {st}")

                name = f"{str(idt).split('.')[-1]} {n}^3 x {b} streamed, {str(odt).split('.')[-1]} out, B as N x K"
                # cuBLAS (torch.bmm on B's transposed view) writes C in the input type
                C3 = torch.empty((b, n, n), dtype=idt, device=dev)
                Bt_ = B.transpose(1, 2)
                for impl, fn, cout in (("kami_b200", lambda: api.gemm_batched(A, B, C1), C1),
                                       ("cutlass_sm100", cutlass_run, C2),
                                       ("cublas", lambda: torch.bmm(A, Bt_, out=C3), C3)):
                    ms = _time_ms(fn, W, K_, flush)
                    t = min(ms)
                    by = b * n * n * (2 + 2 + cout.element_size())
                    _emit({"workload": "comparators", "case": name, "impl": impl, "ms": t,
                           "ms_mean": statistics.fmean(ms), "tflops": 2.0 * n ** 3 * b / t / 1e9,
                           "hbm_gbs": by / t / 1e6, "frac_hbm": by / t / 1e6 / peak_bw,
                           "c_dtype": str(cout.dtype).split('.')[-1]})
                diff = float((C1.float() - C2.float()).abs().max())
                _emit({"workload": "comparators", "case": name, "max_abs_diff_kami_vs_cutlass": diff})
        else:
            _emit({"workload": "comparators", "impl": "cutlass_sm100", "unavailable": "CUTLASS headers not found"})
        # FP16 128^3 x (4 x SMs), streamed (one product per problem)
        b, n = 4 * sms, 128
        A = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).half()
        B = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).half()
        Bt = B.transpose(1, 2)
        C = torch.empty((b, n, n), dtype=torch.float32, device=dev)
        C16 = torch.empty((b, n, n), dtype=torch.float16, device=dev)
        pair("fp16 128^3 x 592 streamed (ours FP32 out, cuBLAS FP16 out)",
             lambda: api.gemm_batched(A, B, C), lambda: torch.bmm(A, Bt, out=C16),
             2.0 * n ** 3 * b, b * n * n * (2 + 2 + 4))
        # FP64 64^3 x 8192 and 32^3 x 1024 streamed
        for b, n in ((8192, 64), (1024, 32)):
            A = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev)
            B = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev)
            Bt = B.transpose(1, 2)
            C = torch.empty((b, n, n), dtype=torch.float64, device=dev)
            pair(f"fp64 {n}^3 x {b} streamed", lambda: api.gemm_batched(A, B, C), lambda: torch.bmm(A, Bt, out=C),
                 2.0 * n ** 3 * b, b * n * n * 24)
        # BF16 bmm forward + backward, 4096 x 64^3
        b, n = 4096, 64
        A = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).bfloat16().requires_grad_()
        B = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).bfloat16().requires_grad_()
        G = torch.tensor(rng.uniform(-1, 1, (b, n, n)), device=dev).bfloat16()

        def fb(f):
            def step():
                A.grad = None
                B.grad = None
                f(A, B).backward(G)
            return step

        pair("bf16 bmm fwd+bwd 4096 x 64^3", fb(bmm), fb(torch.bmm), 6.0 * n ** 3 * b, b * n * n * 2 * 9)
        # uneven: 20000 problems in one graph launch vs one cuBLAS call per distinct shape (problems of equal
        # shape batched together)
        count = 20000
        x = np.exp(rng.uniform(np.log(8), np.log(128), (count, 3)))
        shapes = np.clip(8 * np.round(x / 8), 8, 128).astype(np.int64)
        plan = api.GroupedPlan(shapes, torch.float16)
        Ag = torch.rand(plan.sizes[0], device=dev).half()
        Bg = torch.rand(plan.sizes[1], device=dev).half()
        Cg = torch.empty(plan.sizes[2], dtype=plan.out_dtype, device=dev)
        groups = {}
        for (m_, n_, k_) in map(tuple, shapes):
            groups[(m_, n_, k_)] = groups.get((m_, n_, k_), 0) + 1
        tens = [(torch.rand((c_, m_, k_), device=dev).half(), torch.rand((c_, k_, n_), device=dev).half())
                for (m_, n_, k_), c_ in groups.items()]
        fl = float(sum(2 * m_ * n_ * k_ for m_, n_, k_ in map(tuple, shapes)))
        pair(f"fp16 uneven 20000 problems ({len(groups)} distinct shapes)", lambda: plan.run(Ag, Bg, Cg),
             lambda: [torch.bmm(a, b_) for a, b_ in tens], fl, None)
        return

    if args.workload == "bmm":
        batch, n = 4096, 64
        g = torch.Generator().manual_seed(0)
        A = (torch.rand((batch, n, n), generator=g) * 2 - 1).bfloat16().to(dev).requires_grad_()
        B = (torch.rand((batch, n, n), generator=g) * 2 - 1).bfloat16().to(dev).requires_grad_()
        G = (torch.rand((batch, n, n), generator=g) * 2 - 1).bfloat16().to(dev)

        def step():
            A.grad = None
            B.grad = None
            C = bmm(A, B)
            C.backward(G)

        ms = _time_ms(step, W, K_, flush)
        t = min(ms)
        fl = 3 * 2.0 * n ** 3 * batch
        # tensor passes of the step: forward reads A, B and writes C; the fused
        # backward reads A, B, dC and writes dA, dB
        by = batch * n * n * 2 * 8
        _emit({"workload": "bmm", "dtype": "bf16", "batch": batch, "M": n, "N": n, "K": n, "ms_fwd_bwd": t,
               "tflops": fl / t / 1e9, "hbm_gbs": by / t / 1e6, "frac_hbm": by / t / 1e6 / peak_bw})
        return


def main():
    args = parse()
    if args.workload == "case":
        run_case(args)
        return
    if args.workload != "block":
        run_secondary(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
