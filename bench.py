#!/usr/bin/env python
"""FRSZ2 compress/decompress throughput on B200.

Default workload: the 2 GiB fp64 array (2^28 values, random sign, magnitude
10^U(-30, 30), 1 % exact zeros, 0.1 % subnormals), exponent block 32, 21 bits
per value -- the single-array configuration with the 70 %-of-HBM target, at
its unaligned width.  One step = compress the whole array into its FRSZ2
buffer, then decompress it back.  The same line carries the other five cases
of that configuration (blocks of 32 and 64 at 16 / 21 / 32 bits), each timed
the same way on the same array, under "cases".

  value     whole-job GB/s of algorithmic bytes (compress: values read + exps
            and words written; decompress: the reverse; the 256 B pad is not
            counted), inputs resident in HBM, timed with CUDA events
  e2e       the same metric through the C ABI's host-buffer entry points
            (frsz2_compress_host / frsz2_decompress_host): pinned host buffers,
            H2D and D2H copies inside the timed region
  roofline  the dominant kernel's algorithmic GB/s over the measured HBM copy
            bandwidth
  cpu_baseline  the reference's own CPU codec (oracle/_ref, all host threads)
            on the same whole array
  extras    (default workload, one GPU) short runs of the batched (4,096
            arrays in one persistent launch per class vs per-array calls), fused
            basis dot / axpy and serving workloads, summarised

``--impl reference`` times that reference CPU codec alone on the same
workload (the whole array, the same values) and prints the reference-arm
line.  Under torchrun every rank compresses its own array (weak scaling, no
data-path collective), or with --shard one array split by block range (strong
scaling); the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FRSZ2 compress/decompress GB/s & % HBM peak; batched vs per-array; p50/p99 latency"

WORKLOADS = {
    # name: (kind, dtype, n, bits, E)
    "field512_f32_b16_e32": ("field", "float32", 512 ** 3, 16, 32),
    "loguniform_f64_2p28_b16_e32": ("loguniform", "float64", 1 << 28, 16, 32),
    "loguniform_f64_2p28_b21_e32": ("loguniform", "float64", 1 << 28, 21, 32),
    "loguniform_f64_2p28_b32_e32": ("loguniform", "float64", 1 << 28, 32, 32),
    "loguniform_f64_2p28_b16_e64": ("loguniform", "float64", 1 << 28, 16, 64),
    "loguniform_f64_2p28_b21_e64": ("loguniform", "float64", 1 << 28, 21, 64),
    "loguniform_f64_2p28_b32_e64": ("loguniform", "float64", 1 << 28, 32, 64),
    "normal_f64_2p20_b32_e32": ("normal", "float64", 1 << 20, 32, 32),
    # smaller cases (still larger than L2) for ncu captures
    "loguniform_f64_2p25_b21_e32": ("loguniform", "float64", 1 << 25, 21, 32),
    "loguniform_f64_2p25_b16_e64": ("loguniform", "float64", 1 << 25, 16, 64),
    # kernel families off the default path: blocks of fewer values than a lane,
    # padded blocks, fp64 below 8 bits, block sizes that are not powers of two
    "normal_f32_2p28_b16_e2": ("normal", "float32", 1 << 28, 16, 2),
    "normal_f64_2p27_b33_e32": ("normal", "float64", 1 << 27, 33, 32),
    "normal_f64_2p27_b5_e32": ("normal", "float64", 1 << 27, 5, 32),
    "normal_f32_2p28_b16_e5": ("normal", "float32", 1 << 28, 16, 5),
    "normal_f32_2p25_b16_e2": ("normal", "float32", 1 << 25, 16, 2),
    "normal_f64_2p24_b33_e32": ("normal", "float64", 1 << 24, 33, 32),
    "normal_f64_2p24_b5_e32": ("normal", "float64", 1 << 24, 5, 32),
    "normal_f32_2p25_b16_e5": ("normal", "float32", 1 << 25, 16, 5),
    "normal_f32_2p28_b16_e24": ("normal", "float32", 1 << 28, 16, 24),
    # values (and outputs) starting 1 element past a 32-byte boundary, as a
    # tensor view such as x[1:] does: (kind, dtype, n, bits, E, offset)
    "normal_f32_2p28_b16_e32_off1": ("normal", "float32", 1 << 28, 16, 32, 1),
    "normal_f64_2p27_b21_e32_off1": ("normal", "float64", 1 << 27, 21, 32, 1),
    "normal_f64_2p25_b21_e32_off1": ("normal", "float64", 1 << 25, 21, 32, 1),
}
DEFAULT_WORKLOAD = "loguniform_f64_2p28_b21_e32"


def workload_spec(name: str):
    """A named workload, or any `<normal|loguniform>_<f32|f64>_2p<K>_b<bits>_e<E>`
    (2^K values, `bits` per value, exponent block E), e.g. normal_f32_2p26_b28_e8."""
    import re

    if name in WORKLOADS:
        return WORKLOADS[name]
    m = re.fullmatch(r"(normal|loguniform)_f(32|64)_2p(\d+)_b(\d+)_e(\d+)", name)
    if not m:
        raise SystemExit(f"unknown workload {name}")
    kind, fb, k, bits, E = m.group(1), m.group(2), int(m.group(3)), int(m.group(4)), int(m.group(5))
    if not (10 <= k <= 30 and 4 <= bits <= int(fb) and 1 <= E <= 65536):
        raise SystemExit(f"workload {name} out of range")
    return (kind, "float32" if fb == "32" else "float64", 1 << k, bits, E)


# the six cases of the 2 GiB fp64 configuration: (bits, block size)
F64_2P28_CASES = ((16, 32), (21, 32), (32, 32), (16, 64), (21, 64), (32, 64))
BATCH_WORKLOADS = ("batched4096", "krylov100", "serving", "legacy_f32_2p28", "legacy_f64_2p27", "legacy_f32_2p25",
                   "plugin_grid")

# DRAM bytes (read + write) per launch from ncu captures, by (workload, kernel);
# profiles/ holds the captures' summaries and the commands that made them.
NCU_TRAFFIC = {
    ("loguniform_f64_2p28_b21_e32", "compress"): 2_862_649_600,
    ("loguniform_f64_2p28_b21_e32", "decompress"): 2_829_070_336,
    ("field512_f32_b16_e32", "compress"): 780_571_136,
    ("field512_f32_b16_e32", "decompress"): 755_632_128,
    ("loguniform_f64_2p25_b21_e32", "compress"): 338_155_520,
}


def algorithmic_bytes(dtype: str, n: int, bits: int, E: int) -> int:
    """Per-launch algorithmic bytes: n values + ceil(n/E) * (block bytes +
    exponent bytes); identical for compress and decompress."""
    es = 4 if dtype == "float32" else 8
    W = 8 if bits <= 8 else 16 if bits <= 16 else 32 if bits <= 32 else 64
    nb = -(-n // E)
    block_bytes = -(-E * bits // W) * (W // 8)
    return n * es + nb * (block_bytes + W // 8)


def load_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# ---------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile

            fd, self.path = tempfile.mkstemp(prefix="frsz2_clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "10"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- accuracy

def error_report(x, y, buf, bits: int, E: int) -> dict:
    """Max |x - x_hat|, max |x - x_hat| / |x| over nonzero x (both against the
    fp64 value of the input) and the number of values outside the per-block
    bound max(2^(e_b - bits + 2), 2^(e_b - 31)) that truncation guarantees."""
    import torch

    n = x.numel()
    w = 8 if bits <= 8 else 16 if bits <= 16 else 32 if bits <= 32 else 64
    nb = -(-n // E)
    exps = buf[: nb * (w // 8)].view({8: torch.int8, 16: torch.int16, 32: torch.int32, 64: torch.int64}[w])
    exps = exps.to(torch.float64)
    bound = torch.maximum(torch.exp2(exps - bits + 2), torch.exp2(exps - 31))
    max_abs, max_rel, bad = 0.0, 0.0, 0
    chunk = (1 << 24) // E * E
    for s0 in range(0, n, chunk):
        xe = x[s0:s0 + chunk].to(torch.float64)
        err = (xe - y[s0:s0 + chunk].to(torch.float64)).abs()
        b = bound[s0 // E:(s0 + xe.numel() + E - 1) // E].repeat_interleave(E)[: xe.numel()]
        bad += int((err > b).sum())
        max_abs = max(max_abs, float(err.max()))
        nz = xe != 0
        if bool(nz.any()):
            max_rel = max(max_rel, float((err[nz] / xe[nz].abs()).max()))
    out = {"max_abs": max_abs, "max_rel": max_rel, "bound_violations": bad, "against": "fp64 of the input"}
    if not math.isfinite(max_rel):
        # a value ~2^-1000 in a block whose maximum is ~2^+1000 decodes to the
        # block's zero level; the ratio overflows fp64 (strict JSON has no Inf)
        out["max_rel"] = None
        out["max_rel_note"] = "overflows fp64 (values far below their block maximum)"
    return out


# ---------------------------------------------------------------- inputs

def make_input_cuda(kind: str, dtype: str, n: int, seed: int):
    import torch

    from frsz_b200 import workloads

    tdt = torch.float32 if dtype == "float32" else torch.float64
    if kind == "field":
        side = round(n ** (1 / 3))
        return workloads.sinusoid_field_cuda(side, side, side, seed=seed, dtype=tdt)
    if kind == "loguniform":
        # generated on the host, as the reference arm does: both arms code the same values
        npdt = np.float32 if dtype == "float32" else np.float64
        return torch.from_numpy(workloads.loguniform_host(n, npdt, seed=seed)).to("cuda")
    return workloads.normal_cuda(n, tdt, seed=seed)


def make_input_host(kind: str, dtype: str, n: int, seed: int) -> np.ndarray:
    """The workload's values generated on the host (the same values as
    make_input_cuda for the log-uniform arrays; the field and the normal
    arrays come from the host generators of the same distributions)."""
    import torch

    from frsz_b200 import workloads

    npdt = np.float32 if dtype == "float32" else np.float64
    if kind == "field":
        side = round(n ** (1 / 3))
        f = workloads.sinusoid_field_cuda(side, side, side, seed=seed, dtype=torch.float32, device="cpu")
        return f.numpy().astype(npdt)
    if kind == "loguniform":
        return workloads.loguniform_host(n, npdt, seed=seed)
    return workloads.normal_np(n, npdt, seed=seed)


# ---------------------------------------------------------------- CPU reference codec

def cpu_reference_codec(x: np.ndarray, bits: int, E: int, threads: int, min_seconds: float):
    """Time the reference CPU codec (or, where it is not built, the oracle
    port) on `x`: compress + decompress per rep.  Returns (GB/s, kind, reps)."""
    import oracle

    kind = "reference" if oracle.ref_available() else "port"
    buf = np.zeros(oracle.compressed_bytes(bits, E, x.size), dtype=np.uint8)
    y = np.empty_like(x)

    def rep():
        if kind == "reference":
            oracle.ref_compress_into(x, buf, bits, E, threads)
            oracle.ref_decompress_into(buf, y, bits, E, threads)
        else:
            lib = oracle.oracle_lib()
            lib.frsz2o_compress_mt(int(x.dtype == np.float64), x.ctypes.data, x.size, bits, E, buf.ctypes.data,
                                   threads)
            lib.frsz2o_decompress_mt(int(x.dtype == np.float64), buf.ctypes.data, x.size, bits, E, y.ctypes.data,
                                     threads)

    rep()  # warm
    reps = 0
    t0 = time.perf_counter()
    while True:
        rep()
        reps += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    nbytes = 2 * algorithmic_bytes(str(x.dtype), x.size, bits, E)
    return nbytes * reps / dt / 1e9, kind, reps


# ---------------------------------------------------------------- reference arm

def run_reference_arm(args, rank: int, world: int) -> None:
    """The reference's own CPU codec (frsz2.hpp's compress_cpu_block /
    decompress_cpu_block over block ranges split across all host threads,
    built from the reference sources into oracle/_ref) on the whole workload:
    one step = compress + decompress of every value, as in our arm."""
    if rank != 0:
        return
    kind, dtype, n, bits, E = workload_spec(args.workload)[:5]
    threads = os.cpu_count() or 1
    x = make_input_host(kind, dtype, n, args.seed)
    import oracle

    impl_kind = "reference" if oracle.ref_available() else "port"
    buf = np.zeros(oracle.compressed_bytes(bits, E, x.size), dtype=np.uint8)
    y = np.empty_like(x)

    def step():
        if impl_kind == "reference":
            oracle.ref_compress_into(x, buf, bits, E, threads)
            oracle.ref_decompress_into(buf, y, bits, E, threads)
        else:
            lib = oracle.oracle_lib()
            lib.frsz2o_compress_mt(int(x.dtype == np.float64), x.ctypes.data, x.size, bits, E, buf.ctypes.data,
                                   threads)
            lib.frsz2o_decompress_mt(int(x.dtype == np.float64), buf.ctypes.data, x.size, bits, E, y.ctypes.data,
                                     threads)

    for _ in range(max(1, args.warmup)):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    nbytes = 2 * algorithmic_bytes(dtype, n, bits, E)
    value = nbytes * args.steps / dt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32" if dtype == "float32" else "u64", "data": "synthetic",
        "config": {"workload": args.workload, "dtype": dtype, "n": n, "bits": bits, "block_size": E},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": impl_kind,
                         "sample": f"all {n} values of the workload, compress+decompress per step"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm

def time_case(x, y, bits: int, E: int, warmup: int, K: int, stream):
    """Mean compress and decompress launch times (ms, CUDA events on the
    launching stream) of one (bits, E) case on the resident array x, and the
    number of values outside the per-block error bound."""
    import torch

    import frsz_b200

    n = x.numel()
    buf = torch.zeros(frsz_b200.compressed_size(x.dtype, bits, E, n), dtype=torch.uint8, device=x.device)
    for _ in range(warmup):
        frsz_b200.compress(x, bits, E, out=buf, stream=stream)
        frsz_b200.decompress(buf, n, x.dtype, bits, E, out=y, stream=stream)
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    for ev in evs:
        ev[0].record(stream)
        frsz_b200.compress(x, bits, E, out=buf, stream=stream)
        ev[1].record(stream)
        frsz_b200.decompress(buf, n, x.dtype, bits, E, out=y, stream=stream)
        ev[2].record(stream)
    torch.cuda.synchronize()
    c_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    d_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    viol = error_report(x, y, buf, bits, E)["bound_violations"]
    del buf
    return c_ms, d_ms, viol


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch

    import frsz_b200

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    kind, dtype, n, bits, E = workload_spec(args.workload)[:5]
    frsz_b200.lib()  # fail loudly if the library is missing
    x = make_input_cuda(kind, dtype, n, args.seed + rank)
    tdt = x.dtype
    size = frsz_b200.compressed_size(dtype, bits, E, n)
    buf = torch.zeros(size, dtype=torch.uint8, device="cuda")
    offset = workload_spec(args.workload)[5] if len(workload_spec(args.workload)) > 5 else 0
    if offset:
        xb = torch.empty(n + offset, dtype=tdt, device="cuda")
        xb[offset:] = x
        del x
        x = xb[offset:]
        y = torch.empty(n + offset, dtype=tdt, device="cuda")[offset:]
    else:
        y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    per_launch = algorithmic_bytes(dtype, n, bits, E)
    step_bytes = 2 * per_launch

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        frsz_b200.compress(x, bits, E, out=buf, stream=stream)
        if ev is not None:
            ev[1].record(stream)
        frsz_b200.decompress(buf, n, dtype, bits, E, out=y, stream=stream)
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    K = args.steps
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(K):
        step(evs[k])
    t_end.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop() if clocks else None

    elapsed_ms = t_start.elapsed_time(t_end)
    comp_ms = [e[0].elapsed_time(e[1]) for e in evs]
    decomp_ms = [e[1].elapsed_time(e[2]) for e in evs]
    if dist:
        t = torch.tensor([elapsed_ms, statistics.mean(comp_ms), statistics.mean(decomp_ms)], device="cuda",
                         dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms, comp_avg, decomp_avg = (float(v) for v in t)
    else:
        comp_avg, decomp_avg = statistics.mean(comp_ms), statistics.mean(decomp_ms)

    value = world * step_bytes * K / (elapsed_ms / 1e3) / 1e9
    errors = error_report(x, y, buf, bits, E)
    peaks = load_peaks()

    # ---- the other cases of the 2 GiB fp64 configuration, same array, same timing
    cases = None
    if args.workload.startswith("loguniform_f64_2p28_") and not args.no_cases:
        cases = {}
        for cb, cE in F64_2P28_CASES:
            key = f"b{cb}_e{cE}"
            if (cb, cE) == (bits, E):
                c_ms, d_ms, viol = comp_avg, decomp_avg, errors["bound_violations"]
            else:
                c_ms, d_ms, viol = time_case(x, y, cb, cE, args.warmup, K, stream)
            nb = algorithmic_bytes(dtype, n, cb, cE)
            cases[key] = {"compress_gbs": round(nb / c_ms / 1e6, 1), "decompress_gbs": round(nb / d_ms / 1e6, 1),
                          "compress_frac": round(nb / c_ms / 1e6 / peaks["hbm_gbs"], 4),
                          "decompress_frac": round(nb / d_ms / 1e6 / peaks["hbm_gbs"], 4),
                          "algorithmic_bytes": nb, "bound_violations": viol}

    # ---- end to end through the host-buffer C ABI
    e2e = None
    if not args.no_e2e:
        xh = x.cpu().pin_memory()
        ch = torch.zeros(size, dtype=torch.uint8).pin_memory()
        yh = torch.empty_like(xh).pin_memory()
        xn, cn, yn = xh.numpy(), ch.numpy(), yh.numpy()
        npdt = np.float32 if dtype == "float32" else np.float64

        def e2e_step():
            frsz_b200.compress_host(xn, bits, E, out=cn)
            frsz_b200.decompress_host(cn, n, npdt, bits, E, out=yn)

        e2e_step()
        K2 = max(3, min(K, args.e2e_steps))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K2):
            e2e_step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if dist:
            t = torch.tensor([dt], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t[0])
        comp_written = per_launch - n * (4 if dtype == "float32" else 8)
        e2e = {"value": round(world * step_bytes * K2 / dt / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": n * (4 if dtype == "float32" else 8) + comp_written,
               "d2h_bytes_per_step": comp_written + n * (4 if dtype == "float32" else 8), "steps": K2}
        if rank == 0:
            # the host path must agree with the device path
            assert torch.equal(torch.from_numpy(cn), buf.cpu()), "host-path bytes differ from the device path"
        del xh, ch, yh

    # ---- CPU baseline: reference codec on the host cores, rank 0 at N = 1
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        xs = x.cpu().numpy()
        threads = os.cpu_count() or 1
        gbs, ckind, reps = cpu_reference_codec(xs, bits, E, threads, args.cpu_seconds)
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": ckind,
               "sample": f"all {n} values of the workload, compress+decompress, {reps} reps"}
        del xs

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    # ---- the batched, fused-basis and serving measurements, summarised in the same line (N = 1,
    # default workload): batched, fused basis dot / axpy, serving
    extras = None
    if world == 1 and args.extras and args.workload == DEFAULT_WORKLOAD:
        del x, y, buf
        torch.cuda.empty_cache()
        extras = run_extras(args, local_rank)

    dom_ms = max(comp_avg, decomp_avg)
    dom = "compress" if comp_avg >= decomp_avg else "decompress"
    achieved = per_launch / (dom_ms / 1e3) / 1e9
    traffic = NCU_TRAFFIC.get((args.workload, dom))
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(elapsed_ms / K, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32" if dtype == "float32" else "u64",
        "data": "synthetic",
        "config": {"workload": args.workload, "dtype": dtype, "n": n, "bits": bits, "block_size": E,
                   "bytes_per_step": step_bytes, "l2": "inputs larger than L2, no flush",
                   "parallelism": f"replicas x{world}",
                   **({"values_offset_elems": offset} if offset else {})},
        "compress_gbs": round(per_launch / (comp_avg / 1e3) / 1e9, 2),
        "decompress_gbs": round(per_launch / (decomp_avg / 1e3) / 1e9, 2),
        "compress_ms": round(comp_avg, 5), "decompress_ms": round(decomp_avg, 5),
        "hbm_frac": {"compress": round(per_launch / (comp_avg / 1e3) / 1e9 / peaks["hbm_gbs"], 4),
                     "decompress": round(per_launch / (decomp_avg / 1e3) / 1e9 / peaks["hbm_gbs"], 4),
                     "of": peaks["source"]},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                     "algorithmic_bytes": per_launch, "peak_source": peaks["source"]},
        "errors": errors,
        **({"cases": {"of": f"measured HBM copy {peaks['hbm_gbs']} GB/s", "steps": K, **cases}} if cases else {}),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": 2 * K,
        "clocks": clk,
        **({"extras": extras} if extras else {}),
    }
    print(json.dumps(line), flush=True)


def run_extras(args, local_rank: int) -> dict:
    """Short runs of the batched (4,096 arrays), fused basis dot / axpy and
    serving workloads, summarised; each is the same code as its own
    --workload run (plan autotuning skipped, its default shape kept), and a
    failure is recorded instead of ending the benchmark."""
    import copy

    import torch

    out = {}
    for name, fn in (("batched4096", run_batched), ("krylov100", run_krylov), ("serving", run_serving)):
        a = copy.copy(args)
        a.batch_autotune = False
        t0 = time.perf_counter()
        try:
            line = fn(a, 0, 1, local_rank, emit=False)
        except Exception as e:  # recorded, the headline stands
            out[name] = {"error": repr(e)[:300]}
            continue
        finally:
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        if name == "batched4096":
            out[name] = {"gbs": line["value"], "hbm_frac": line["batched"]["hbm_frac"],
                         "compress_gbs": line["batched"]["compress_gbs"],
                         "decompress_gbs": line["batched"]["decompress_gbs"],
                         "per_array_plain_gbs": line["per_array_plain"]["gbs"],
                         "per_array_graph_gbs": line["per_array_graph"]["gbs"],
                         "speedup_vs_per_array_plain": line["speedup_vs_per_array_plain"],
                         "speedup_vs_per_array_graph": line["speedup_vs_per_array_graph"],
                         "bytes_per_step": line["config"]["bytes_per_step"], "steps": line["steps"]}
        elif name == "krylov100":
            out[name] = {"fused_dot": line["fused_dot"], "fused_axpy": line["fused_axpy"],
                         "uncompressed_torch_ms": line["uncompressed_torch"],
                         "compressed_basis_bytes": line["config"]["compressed_basis_bytes"]}
        else:
            out[name] = {"gbs": line["value"], "latency_us": line["latency_us"], "capacity": line["capacity"],
                         "requests": line["config"]["requests"], "load": line["config"]["load"]}
        out[name]["wall_s"] = round(time.perf_counter() - t0, 1)
    return out


# ---------------------------------------------------------------- one array over several GPUs

def run_shard(args, rank: int, world: int, local_rank: int) -> None:
    """One array split across the ranks by block range (strong scaling): rank
    r compresses and decompresses only its blocks, writing them into the
    whole array's layout (frsz2_compress_blocks / frsz2_decompress_blocks);
    there is no data-path collective.  value = the whole array's algorithmic
    bytes per step over the slowest rank's time."""
    import torch

    import frsz_b200
    from frsz_b200 import shard

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    kind, dtype, n, bits, E = workload_spec(args.workload)[:5]
    frsz_b200.lib()
    x_full = make_input_cuda(kind, dtype, n, args.seed)  # the same array on every rank
    b0, b1 = shard.shard_blocks(n, dtype, bits, E, world, rank)
    v0, v1 = b0 * E, min(n, b1 * E)
    xs = x_full[v0:v1].clone()
    ys = torch.empty_like(xs)
    buf = torch.zeros(frsz_b200.compressed_size(dtype, bits, E, n), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    mine = algorithmic_bytes(dtype, v1 - v0, bits, E) if v1 > v0 else 0

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        if v1 > v0:
            shard.compress_shard(xs, n, bits, E, b0, b1, buf, stream=stream)
        if ev is not None:
            ev[1].record(stream)
        if v1 > v0:
            shard.decompress_shard(buf, n, dtype, bits, E, b0, b1, ys, stream=stream)
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    K = args.steps
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(K):
        step(evs[k])
    t1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    elapsed_ms = t0.elapsed_time(t1)
    comp_avg = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    decomp_avg = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    # this rank's bytes equal a whole-array compress over its written ranges
    whole = frsz_b200.compress(x_full, bits, E)
    ok = all(torch.equal(buf[o:o + ln], whole[o:o + ln]) for o, ln in shard.written_ranges(n, bits, E, b0, b1))
    del whole
    if dist:
        t = torch.tensor([elapsed_ms, comp_avg, decomp_avg, 0.0 if ok else 1.0], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms, comp_avg, decomp_avg, bad = (float(v) for v in t)
        ok = bad == 0.0
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    assert ok, "a shard's bytes differ from the whole-array compress"
    peaks = load_peaks()
    per_launch = algorithmic_bytes(dtype, n, bits, E)
    dom_ms = max(comp_avg, decomp_avg)
    achieved = mine / (dom_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": round(2 * per_launch * K / (elapsed_ms / 1e3) / 1e9, 3), "unit": "GB/s",
        "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": round(elapsed_ms / K, 5),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32" if dtype == "float32" else "u64", "data": "synthetic",
        "config": {"workload": args.workload, "dtype": dtype, "n": n, "bits": bits, "block_size": E,
                   "bytes_per_step": 2 * per_launch, "l2": "inputs larger than L2, no flush",
                   "parallelism": f"block-range shards x{world}", "rank0_blocks": [b0, b1]},
        "roofline": {"bound": "hbm", "kernel": "compress" if comp_avg >= decomp_avg else "decompress",
                     "achieved": round(achieved, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                     "algorithmic_bytes": mine, "peak_source": peaks["source"], "of": "rank 0's shard"},
        "cpu_baseline": None, "e2e": None, "gpu_launches": 2 * K, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batched

def batched_specs(count: int = 4096, seed: int = 7):
    """The 4,096-array batch: byte sizes log-uniform in [1 KiB, 64 MiB], 50/50 fp32/fp64,
    bits uniform over {8, 12, 16, 24, 32}, block 32."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(count):
        nbytes = math.exp(rng.uniform(math.log(1024), math.log(64 << 20)))
        is64 = rng.random() < 0.5
        es = 8 if is64 else 4
        specs.append(("float64" if is64 else "float32", max(1, int(nbytes) // es), int(rng.choice([8, 12, 16, 24, 32])),
                      32))
    return specs


def run_batched(args, rank: int, world: int, local_rank: int, emit: bool = True):
    """One step = compress all arrays, then decompress all.  value = the
    batched plan (one graph launch per direction); the same arrays are also
    timed with one plain frsz2_compress / frsz2_decompress call per array
    (eager from the host, and recorded into a CUDA graph)."""
    import torch

    import frsz_b200

    torch.cuda.set_device(local_rank)
    specs = batched_specs(seed=args.seed + rank)
    align = 256
    off_v, off_c, items = 0, 0, []
    for dt, n, bits, E in specs:
        es = 4 if dt == "float32" else 8
        csize = frsz_b200.compressed_size(dt, bits, E, n)
        items.append((dt, n, bits, E, off_v, off_c, csize))
        off_v += -(-n * es // align) * align
        off_c += -(-csize // align) * align
    pool_in = torch.empty(off_v, dtype=torch.uint8, device="cuda")
    pool_out = torch.empty(off_v, dtype=torch.uint8, device="cuda")
    pool_c = torch.zeros(off_c, dtype=torch.uint8, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(args.seed + rank)
    arrays = []
    total_bytes = 0
    for dt, n, bits, E, ov, oc, csize in items:
        tdt = torch.float32 if dt == "float32" else torch.float64
        es = 4 if dt == "float32" else 8
        x = pool_in[ov:ov + n * es].view(tdt)
        x.normal_(generator=g)
        y = pool_out[ov:ov + n * es].view(tdt)
        c = pool_c[oc:oc + csize]
        arrays.append(frsz_b200.BatchArray(values=x, compressed=c, bits=bits, block_size=E, decompressed=y))
        total_bytes += algorithmic_bytes(dt, n, bits, E)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()  # graph capture needs a non-default stream
    torch.cuda.set_stream(stream)
    plan = frsz_b200.BatchPlan(arrays)
    tune_c = plan.autotune(compress=True, stream=stream) if args.batch_autotune else None
    tune_d = plan.autotune(compress=False, stream=stream) if args.batch_autotune else None

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    K = args.steps
    ms_c = timed(lambda: plan.compress(stream), K)
    ms_d = timed(lambda: plan.decompress(stream), K)
    # plain per-array calls
    lib = frsz_b200.lib()
    sp = stream.cuda_stream
    plain = [(frsz_b200.codec.dtype_code(a.values.dtype), a.bits, a.block_size, a.values.data_ptr(),
              a.values.numel(), a.compressed.data_ptr(), a.decompressed.data_ptr()) for a in arrays]

    def per_array_c():
        for code, bits, E, xp, n, cp, _ in plain:
            lib.frsz2_compress(code, bits, E, xp, n, cp, sp)

    def per_array_d():
        for code, bits, E, _, n, cp, yp in plain:
            lib.frsz2_decompress(code, bits, E, cp, n, yp, sp)

    K2 = max(1, min(K, 5))
    ms_pc = timed(per_array_c, K2)
    ms_pd = timed(per_array_d, K2)
    graphs = []
    for fn in (per_array_c, per_array_d):
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr, stream=stream):
            fn()
        graphs.append(gr)
    ms_gc = timed(graphs[0].replay, K2)
    ms_gd = timed(graphs[1].replay, K2)
    del graphs
    # parity spot check of a few arrays against the oracle
    import oracle
    rng = np.random.default_rng(1)
    for i in rng.choice(len(arrays), 6, replace=False):
        a = arrays[int(i)]
        if a.values.numel() > (1 << 22):
            continue
        xh = a.values.cpu().numpy()
        ref = oracle.compress(xh, a.bits, a.block_size, canary=0)
        got = a.compressed.cpu().numpy()
        w = frsz_b200.word_bits(a.bits) // 8
        nb = -(-xh.size // a.block_size)
        assert np.array_equal(got[:nb * w], ref[:nb * w]), "batched exponents differ from the oracle"
        eb = frsz_b200.exponent_size(xh.dtype, a.bits, a.block_size, xh.size)
        assert np.array_equal(got[eb:], ref[eb:]), "batched words differ from the oracle"
    info = plan.info()
    if rank != 0:
        return
    step_ms = ms_c + ms_d
    value = world * 2 * total_bytes / (step_ms / 1e3) / 1e9
    per_ms = ms_pc + ms_pd
    gper_ms = ms_gc + ms_gd
    peaks = load_peaks()
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32/u64", "data": "synthetic",
        "config": {"workload": "batched4096", "arrays": len(arrays), "bytes_per_step": 2 * total_bytes,
                   "sizes": "log-uniform 1 KiB-64 MiB", "dtypes": "50/50 fp32/fp64 N(0,1)",
                   "bits": [8, 12, 16, 24, 32], "block_size": 32, "l2": "inputs larger than L2, no flush"},
        "batched": {"compress_gbs": round(total_bytes / ms_c / 1e6, 1),
                    "decompress_gbs": round(total_bytes / ms_d / 1e6, 1),
                    "hbm_frac": round(2 * total_bytes / step_ms / 1e6 / peaks["hbm_gbs"], 4),
                    "autotune_ms": ({"compress": round(tune_c, 4), "decompress": round(tune_d, 4)}
                                    if args.batch_autotune else None),
                    "plan": info},
        "per_array_plain": {"gbs": round(2 * total_bytes / per_ms / 1e6, 1), "ms_per_step": round(per_ms, 3),
                            "launches_per_step": 2 * len(arrays), "host_loop": "python ctypes"},
        "per_array_graph": {"gbs": round(2 * total_bytes / gper_ms / 1e6, 1), "ms_per_step": round(gper_ms, 3)},
        "speedup_vs_per_array_plain": round(per_ms / step_ms, 2),
        "speedup_vs_per_array_graph": round(gper_ms / step_ms, 2),
        "gpu_launches": 2 * info["classes"] * K,
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


# ---------------------------------------------------------------- fused basis

def run_krylov(args, rank: int, world: int, local_rank: int, emit: bool = True):
    """The compressed basis: 100 fp64 vectors of 2^22 values, 32 bits (--krylov-bits
    for the other fused widths), block 32.  Times
    the fused h = V^T w and y += V c over the compressed basis, against
    decompress-then-torch and against torch on the uncompressed basis."""
    import torch

    import frsz_b200

    torch.cuda.set_device(local_rank)
    m, n, bits, E = args.krylov_vectors, 1 << 22, args.krylov_bits, 32
    g = torch.Generator(device="cuda").manual_seed(args.seed + rank)
    V = torch.randn(m, n, generator=g, device="cuda", dtype=torch.float64)
    basis = frsz_b200.CompressedBasis(m, n, bits=bits, block_size=E)
    for j in range(m):
        basis.append(V[j])
    Vd = torch.stack([basis.get(j) for j in range(m)])  # decompressed basis, for the checks and baselines
    w = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    c = torch.randn(m, generator=g, device="cuda", dtype=torch.float64)
    y = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    stream = torch.cuda.current_stream()
    tmp = torch.empty(n, dtype=torch.float64, device="cuda")
    h = torch.empty(m, dtype=torch.float64, device="cuda")

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    def unfused_dot():
        for j in range(m):
            frsz_b200.decompress(basis.buffers[j], n, torch.float64, bits, E, out=tmp)
            h[j] = torch.dot(tmp, w)

    K = args.steps
    ms_dot = timed(lambda: basis.dot(w, out=h), K)
    ms_axpy = timed(lambda: basis.axpy(c, y), K)
    ms_unfused = timed(unfused_dot, max(1, K // 10))
    ms_dense_dot = timed(lambda: torch.mv(V, w, out=h), K)
    ms_dense_axpy = timed(lambda: y.addmv_(V.t(), c), K)
    # accuracy of the fused results against torch on the decompressed basis
    hd = basis.dot(w)
    dot_err = float(((hd - Vd @ w).abs() / (Vd.abs() @ w.abs())).max())
    y0 = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    y1 = y0.clone()
    basis.axpy(c, y1)
    axpy_err = float(((y1 - (y0 + c @ Vd)).abs() / (y0.abs() + c.abs() @ Vd.abs())).max())
    comp_bytes = m * frsz_b200.compressed_size(np.float64, bits, E, n)
    dot_bytes = m * algorithmic_bytes("float64", n, bits, E) - m * n * 8 + n * 8
    axpy_bytes = dot_bytes + n * 8
    peaks = load_peaks()
    if rank != 0:
        return
    value = world * (dot_bytes + axpy_bytes) / ((ms_dot + ms_axpy) / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(ms_dot + ms_axpy, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": ("krylov100" if m == 100 else f"krylov{m}") + ("" if bits == 32 else f"_b{bits}"),
                   "vectors": m, "n": n, "bits": bits,
                   "block_size": E,
                   "compressed_basis_bytes": comp_bytes, "step": "fused dot h=V^T w, then fused axpy y+=V c"},
        "fused_dot": {"ms": round(ms_dot, 4), "gbs": round(dot_bytes / ms_dot / 1e6, 1),
                      "hbm_frac": round(dot_bytes / ms_dot / 1e6 / peaks["hbm_gbs"], 4), "max_rel_err": dot_err},
        "fused_axpy": {"ms": round(ms_axpy, 4), "gbs": round(axpy_bytes / ms_axpy / 1e6, 1),
                       "hbm_frac": round(axpy_bytes / ms_axpy / 1e6 / peaks["hbm_gbs"], 4),
                       "max_rel_err": axpy_err},
        "decompress_then_dot_ms": round(ms_unfused, 4),
        "uncompressed_torch": {"dot_ms": round(ms_dense_dot, 4), "axpy_ms": round(ms_dense_axpy, 4)},
        "speedup_fused_dot_vs_uncompressed": round(ms_dense_dot / ms_dot, 2),
        "speedup_fused_axpy_vs_uncompressed": round(ms_dense_axpy / ms_axpy, 2),
        "gpu_launches": 3 * K,  # dot: item kernel + final sum; axpy: one kernel
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


# ---------------------------------------------------------------- serving

def run_serving(args, rank: int, world: int, local_rank: int, emit: bool = True):
    """The request stream: Poisson arrivals, 60 % compress / 40 % decompress,
    input sizes log-normal (median 1 MB, sigma 1.5, capped at 256 MB), fp32 /
    fp64 50/50, bits from {12, 16, 32}, block 32, 32 GB admission budget.
    Offered load = 70 % of the capacity measured with the same requests all
    submitted at once.  Latency = completion - arrival, per request."""
    import torch

    import frsz_b200
    from frsz_b200 import serve

    torch.cuda.set_device(local_rank)
    rng = np.random.default_rng(args.seed + rank)
    pool = []
    for _ in range(512):  # distinct payloads; requests cycle through them
        nbytes = min(256 << 20, int(math.exp(rng.normal(math.log(1 << 20), 1.5))))
        is64 = bool(rng.random() < 0.5)
        es = 8 if is64 else 4
        n = max(1, nbytes // es)
        bits = int(rng.choice([12, 16, 32]))
        x = torch.randn(n, device="cuda", dtype=torch.float64 if is64 else torch.float32)
        pool.append(dict(is64=is64, n=n, bits=bits, x=x, comp=frsz_b200.compress(x, bits, 32)))
    torch.cuda.synchronize()
    R = args.requests
    picks = rng.integers(0, len(pool), R)
    ops = np.where(rng.random(R) < 0.6, serve.OP_COMPRESS, serve.OP_DECOMPRESS)

    def make(count, offsets):
        """Requests with arrival times relative to their submission."""
        reqs = (frsz_b200._lib.RequestC * count)()
        flags = serve.RELEASE_ON_COMPLETION | serve.ARRIVAL_RELATIVE
        for i in range(count):
            e = pool[picks[i]]
            inp = e["x"] if ops[i] == serve.OP_COMPRESS else e["comp"]
            r = reqs[i]
            r.op, r.dtype, r.bits, r.block_size, r.n = int(ops[i]), int(e["is64"]), e["bits"], 32, e["n"]
            r.input, r.output, r.arrival_ns, r.flags = inp.data_ptr(), None, int(offsets[i]), flags
        return reqs

    def drive(reqs, count):
        sv = serve.Server(memory_budget=32 << 30, max_batch=args.max_batch, streams=args.streams)
        sv.submit(reqs)
        got = []
        while len(got) < count:
            got += sv.poll(wait_ms=50)
        st = sv.stats()
        sv.close()
        assert all(c.status == 0 for c in got), "a serving request failed"
        return got, st

    # warm-up: loads every class kernel the stream uses (lazy module loading)
    drive(make(min(R, 2000), np.zeros(min(R, 2000))), min(R, 2000))
    # capacity: every request arrives at submission
    cap_n = min(R, args.capacity_requests)
    got, _ = drive(make(cap_n, np.zeros(cap_n)), cap_n)
    span = (max(c.done_ns for c in got) - min(c.arrival_ns for c in got)) / 1e9
    cap_bytes = sum(c.bytes for c in got) / span
    cap_rate = cap_n / span
    # Poisson stream at `load` of that capacity, starting 20 ms after submission
    lam = args.load * cap_rate
    offsets = 20_000_000 + np.cumsum(rng.exponential(1e9 / lam, R)).astype(np.int64)
    got, st = drive(make(R, offsets), R)
    lat = np.array([c.latency_ns for c in got], dtype=np.float64) / 1e3
    total = sum(c.bytes for c in got)
    span = (max(c.done_ns for c in got) - min(c.arrival_ns for c in got)) / 1e9
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(world * total / span / 1e9, 3), "unit": "GB/s", "n_gpus": world,
        "steps": R, "warmup": 0, "ms_per_step": round(span * 1e3 / R, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64", "data": "synthetic",
        "config": {"workload": "serving", "requests": R, "compress_fraction": 0.6,
                   "sizes": "log-normal median 1 MB sigma 1.5, cap 256 MB", "dtypes": "fp32/fp64 50/50",
                   "bits": [12, 16, 32], "block_size": 32, "budget_bytes": 32 << 30, "load": args.load,
                   "max_batch": args.max_batch, "streams": args.streams},
        "latency_us": {"p50": round(float(np.percentile(lat, 50)), 1), "p90": round(float(np.percentile(lat, 90)), 1),
                       "p99": round(float(np.percentile(lat, 99)), 1),
                       "p999": round(float(np.percentile(lat, 99.9)), 1), "max": round(float(lat.max()), 1)},
        "capacity": {"gbs": round(cap_bytes / 1e9, 1), "requests_per_s": round(cap_rate, 1),
                     "requests": cap_n},
        "offered_requests_per_s": round(lam, 1),
        "server": st,
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_plugin_grid(args, rank: int, world: int, local_rank: int) -> None:
    """Every (block size, bits) the frsz2 plugin offers (src/frsz2.cc:86-129:
    E = 2 .. 1024 in powers of two, bits 4..32 for fp32 and 4..64 for fp64) on
    one 1 GiB array of N(0,1) values per float type (2^28 fp32, 2^27 fp64):
    compress and decompress, each timed over `--steps` launches after
    `--warmup` untimed ones, as fractions of the measured HBM copy bandwidth.  Prints one summary line (per float type and
    block size: min / median of each direction and the widths below 0.85); with
    --grid-rows, every shape."""
    import torch

    import frsz_b200

    torch.cuda.set_device(local_rank)
    if rank != 0:
        return
    peak = load_peaks()["hbm_gbs"]
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    stream = torch.cuda.current_stream()
    K = max(1, args.steps)
    rows = []
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    t0 = time.perf_counter()
    for dt, tdt, maxb, n in (("float32", torch.float32, 32, 1 << 28), ("float64", torch.float64, 64, 1 << 27)):
        x = torch.randn(n, generator=g, device="cuda", dtype=tdt)
        y = torch.empty_like(x)
        for E in (2, 4, 8, 16, 32, 64, 128, 256, 512, 1024):
            for bits in range(4, maxb + 1):
                buf = frsz_b200.compress(x, bits, E)
                nb = algorithmic_bytes(dt, n, bits, E)
                frac = []
                for fn in (lambda: frsz_b200.compress(x, bits, E, out=buf),
                           lambda: frsz_b200.decompress(buf, n, tdt, bits, E, out=y)):
                    for _ in range(max(1, args.warmup)):
                        fn()
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    for _ in range(K):
                        fn()
                    b.record(stream)
                    torch.cuda.synchronize()
                    frac.append(round(nb / (a.elapsed_time(b) / K) / 1e6 / peak, 3))
                rows.append((dt, E, bits, frac[0], frac[1]))
                del buf
        del x, y
        torch.cuda.empty_cache()
    summary = {}
    for dt in ("float32", "float64"):
        for E in (2, 4, 8, 16, 32, 64, 128, 256, 512, 1024):
            rs = [r for r in rows if r[0] == dt and r[1] == E]
            c, d = sorted(r[3] for r in rs), sorted(r[4] for r in rs)
            summary[f"{dt}_e{E}"] = {"compress_min": c[0], "compress_median": c[len(c) // 2],
                                     "decompress_min": d[0], "decompress_median": d[len(d) // 2],
                                     "compress_below_0.85": [r[2] for r in rs if r[3] < 0.85],
                                     "decompress_below_0.85": [r[2] for r in rs if r[4] < 0.85]}
    allc, alld = sorted(r[3] for r in rows), sorted(r[4] for r in rows)
    line = {"metric": METRIC, "workload": "plugin_grid", "shapes": len(rows), "n": {"float32": 1 << 28, "float64": 1 << 27},
            "steps": K,
            "of": f"measured HBM copy {peak} GB/s", "data": "synthetic N(0,1)",
            "compress_median": allc[len(allc) // 2], "decompress_median": alld[len(alld) // 2],
            "compress_at_least_0.85": sum(v >= 0.85 for v in allc),
            "decompress_at_least_0.85": sum(v >= 0.85 for v in alld),
            "wall_s": round(time.perf_counter() - t0, 1), "clocks": clocks.stop(), "by_block_size": summary}
    if args.grid_rows:
        line["rows"] = [list(r) for r in rows]
    print(json.dumps(line), flush=True)


def run_legacy(args, rank: int, world: int, local_rank: int) -> None:
    """The legacy "frsz" codec (src/frsz.cc) on N(0,1) data, epsilon 1e-3:
    compress, then decompress as the reference does and with each block's
    own differences.  Bytes per launch: the values plus the int16 stream."""
    import torch

    from frsz_b200 import legacy

    torch.cuda.set_device(local_rank)
    dtype = torch.float32 if "_f32_" in args.workload else torch.float64
    n = 1 << int(args.workload.rsplit("2p", 1)[1])
    g = torch.Generator(device="cuda").manual_seed(args.seed + rank)
    x = torch.randn(n, generator=g, device="cuda", dtype=dtype)
    q = torch.empty(n, dtype=torch.int16, device="cuda")
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    ms_c = timed(lambda: legacy.compress(x, 1e-3, out=q))
    ms_d = timed(lambda: legacy.decompress(q, dtype, 1e-3, out=y))
    ms_o = timed(lambda: legacy.decompress(q, dtype, 1e-3, own_deltas=True, out=y))
    nbytes = n * (x.element_size() + 2)
    peak = load_peaks()["hbm_gbs"]
    gbs = [nbytes / ms / 1e6 for ms in (ms_c, ms_d, ms_o)]
    if rank == 0:
        print(json.dumps({"metric": "legacy frsz compress / decompress GB/s", "value": round(gbs[0], 1), "unit": "GB/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                          "dtype": str(dtype).replace("torch.", ""), "data": "synthetic N(0,1), epsilon 1e-3",
                          "config": {"workload": args.workload, "n": n},
                          "compress_gbs": round(gbs[0], 1), "decompress_reference_gbs": round(gbs[1], 1),
                          "decompress_own_deltas_gbs": round(gbs[2], 1),
                          "hbm_frac": [round(v / peak, 3) for v in gbs]}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    help="one of %s, %s, or <normal|loguniform>_<f32|f64>_2p<K>_b<bits>_e<E>"
                    % (", ".join(sorted(WORKLOADS)), ", ".join(BATCH_WORKLOADS)))
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=3.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="default workload: skip the batched / fused basis / serving summaries")
    ap.add_argument("--no-cases", action="store_true",
                    help="2 GiB fp64 workloads: skip timing the configuration's other five cases")
    ap.add_argument("--requests", type=int, default=100_000, help="serving: requests in the Poisson stream")
    ap.add_argument("--capacity-requests", type=int, default=20_000, help="serving: requests of the capacity probe")
    ap.add_argument("--load", type=float, default=0.7, help="serving: offered load as a fraction of capacity")
    ap.add_argument("--max-batch", type=int, default=256)
    ap.add_argument("--no-batch-autotune", dest="batch_autotune", action="store_false",
                    help="batched4096: keep the plan's default launch shape")
    ap.add_argument("--grid-rows", action="store_true", help="plugin_grid: print every shape too")
    ap.add_argument("--krylov-vectors", type=int, default=100, help="krylov100: basis size")
    ap.add_argument("--krylov-bits", type=int, default=32, choices=[16, 21, 24, 32, 48, 64],
                    help="krylov100: bits per value of the compressed basis")
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--shard", action="store_true",
                    help="split one array across the ranks by block range (strong scaling) instead of one "
                         "array per rank")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "batched4096":
        run_batched(args, rank, world, local_rank)
    elif args.workload == "krylov100":
        run_krylov(args, rank, world, local_rank)
    elif args.workload == "serving":
        run_serving(args, rank, world, local_rank)
    elif args.workload == "plugin_grid":
        run_plugin_grid(args, rank, world, local_rank)
    elif args.workload.startswith("legacy_"):
        run_legacy(args, rank, world, local_rank)
    elif args.impl == "reference":
        run_reference_arm(args, rank, world)
    elif args.shard:
        run_shard(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
