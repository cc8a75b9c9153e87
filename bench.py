#!/usr/bin/env python
"""Benchmark of the TBLIS-compatible contraction hot path on B200.

Headline workload (one "step" = one contraction through tblis_tensor_mult):
the ladder term C[abij] = A[abef] * B[efij] with o=48, v=160 (m=25600,
n=2304, k=25600; 3.02 TFLOP), FP64 inputs uniform(-1,1) * 2^k with k a
uniform integer in [-20, 20] per element, generated once on the host from
fixed seeds (the same bits in every arm), computed by the fastest method whose
normwise relative error is at most 1e-12.

Prints one JSON line (rank 0). Extra keys: the accuracy of the GPU results
against the reference's own FP64 output on the same inputs, the plain FP64
(DMMA) rate on the same workload, the roofline of the dominant kernel, the
CPU baseline (the TBLIS reference built from its own sources, timed on the
whole ladder on this host), the end-to-end rate through tblis_tensor_mult with
pinned host buffers, and the secondary workloads (DPD, batch, serving, ring,
transpose, dot/reduce), each with its own check against the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference's tblis_tensor_mult on the host cores on
the same inputs, one whole ladder contraction per step.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

O, V = 48, 160
FLOPS_LADDER = 2.0 * V * V * V * V * O * O
WORKLOAD = "ladder C[abij]=A[abef]*B[efij] o=48 v=160 fp64 exponent spread 2^[-20,20]"
METRIC = "contraction GFLOP/s at <=1e-12 normwise rel err"


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) leg")
    p.add_argument("--o", type=int, default=48, help="occupied extent (profiling runs use a smaller case)")
    p.add_argument("--v", type=int, default=160, help="virtual extent")
    p.add_argument("--case", default=None, choices=["ring", "transpose", "dot", "reduce", "dpd", "serve", "batch"],
                   help="run only one secondary kernel at extents --o/--v (profiling); prints its own line")
    p.add_argument("--batch-count", type=int, default=10000,
                   help="members of the --case batch workload (profiling runs use fewer)")
    a = p.parse_args(argv)
    global O, V, FLOPS_LADDER, WORKLOAD
    if (a.o, a.v) != (O, V):
        O, V = a.o, a.v
        FLOPS_LADDER = 2.0 * V * V * V * V * O * O
        WORKLOAD = "ladder C[abij]=A[abef]*B[efij] o=%d v=%d fp64 exponent spread 2^[-20,20]" % (O, V)
    return a


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ---------------------------------------------------------------------------------------
# Inputs: one host-side seeded recipe for every arm (GPU, end to end, CPU reference)
# ---------------------------------------------------------------------------------------

SEED_A, SEED_B = 1001, 1002
GEN_CHUNK = 1 << 24
INPUTS = ("host-generated FP64, numpy PCG64 stream per 16M-element chunk seeded (tensor seed, chunk) with "
          "A=1001, B=1002: uniform(-1,1) * 2^k, k uniform integer in [-20,20]; every arm uses the same bits")


def fill_spread(flat, seed):
    """Fills a flat float64 array (a tensor's storage in memory order) with
    uniform(-1,1) * 2^k, k a uniform integer in [-20, 20]; chunk c draws from
    numpy's PCG64 seeded with (seed, c), so the result does not depend on how
    many threads fill it."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor

    def one(c):
        s = c * GEN_CHUNK
        e = min(flat.size, s + GEN_CHUNK)
        rng = np.random.default_rng([seed, c])
        u = rng.uniform(-1.0, 1.0, e - s)
        k = rng.integers(-20, 21, e - s, dtype=np.int32)
        np.ldexp(u, k, out=flat[s:e])
    n = (flat.size + GEN_CHUNK - 1) // GEN_CHUNK
    with ThreadPoolExecutor(max_workers=max(1, min(16, len(os.sched_getaffinity(0))))) as ex:
        list(ex.map(one, range(n)))


def ladder_inputs(pinned=False):
    """A[abef] (V^4) and B[efij] (V^2 O^2), column-major in label order, as
    numpy arrays (backed by pinned torch host memory when `pinned`), plus a
    zeroed column-major C[abij]; the returned torch tensors keep the pinned
    storage alive."""
    import numpy as np
    keep = []

    def empty(shape):
        n = 1
        for x in shape:
            n *= x
        if pinned:
            import torch
            t = torch.empty(n, dtype=torch.float64).pin_memory()
            keep.append(t)
            flat = t.numpy()
        else:
            flat = np.empty(n, dtype=np.float64)
        return flat, flat.reshape(shape, order="F")
    fa, A = empty((V, V, V, V))
    fb, B = empty((V, V, O, O))
    fc, C = empty((V, V, O, O))
    fill_spread(fa, SEED_A)
    fill_spread(fb, SEED_B)
    fc[:] = 0.0
    return A, B, C, keep


def host_cpu():
    """(threads usable by this process, physical cores among them, CPU model)."""
    cpus = sorted(os.sched_getaffinity(0))
    model, phys, cur = None, set(), {}
    try:
        for line in open("/proc/cpuinfo"):
            if ":" not in line:
                if cur.get("processor") is not None and int(cur["processor"]) in cpus:
                    phys.add((cur.get("physical id"), cur.get("core id")))
                cur = {}
                continue
            k, v = [x.strip() for x in line.split(":", 1)]
            cur[k] = v
            if k == "model name" and model is None:
                model = v
        if cur.get("processor") is not None and int(cur["processor"]) in cpus:
            phys.add((cur.get("physical id"), cur.get("core id")))
    except OSError:
        pass
    return len(cpus), (len(phys) or len(cpus)), model


def normwise(got, want):
    """||got - want||_F / ||want||_F over numpy arrays."""
    import numpy as np
    return float(np.linalg.norm((got - want).ravel(order="K")) / np.linalg.norm(want.ravel(order="K")))


# ---------------------------------------------------------------------------------------
# CPU reference (oracle/_ref: the TBLIS reference compiled from its own sources)
# ---------------------------------------------------------------------------------------

def cpu_reference_ladder(A, B, reps=2):
    """Times the reference's tblis_tensor_mult on the whole ladder (the same
    inputs as the GPU arm), best of `reps`, with every usable host thread.
    Returns (GFLOP/s, threads, physical cores, model, sample text, C)."""
    import numpy as np
    import oracle
    if not oracle.have_ref():
        return None
    threads, phys, model = host_cpu()
    C = np.zeros((V, V, O, O), order="F")
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        oracle.ref_mult(1.0, A, "abef", B, "efij", 0.0, C, "abij", threads=threads)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    sample = ("the whole ladder (%.0f GFLOP, same inputs as the GPU arm), best of %d, tblis_tensor_mult of "
              "the reference built from its own sources, %d threads on %d physical cores (%s)"
              % (FLOPS_LADDER / 1e9, reps, threads, phys, model))
    return FLOPS_LADDER / best / 1e9, threads, phys, model, sample, C


def run_reference(args):
    """The reference arm: the reference's own tblis_tensor_mult on the host
    cores, one whole ladder contraction per step on the same seeded inputs
    as the GPU arm, exactly W warm-up and K timed steps (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference sources at build time)"}))
        return
    threads, phys, model = host_cpu()
    A, B, C, _ = ladder_inputs()

    def step():
        oracle.ref_mult(1.0, A, "abef", B, "efij", 0.0, C, "abij", threads=threads)
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    wall = sum(times)
    value = FLOPS_LADDER * len(times) / wall / 1e9
    sample = ("the whole ladder (%.0f GFLOP) per step, tblis_tensor_mult of the reference built from its own "
              "sources, %d threads on %d physical cores (%s)" % (FLOPS_LADDER / 1e9, threads, phys, model))
    print(json.dumps({
        "impl": "reference", "metric": METRIC,
        "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": 1e3 * wall / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(),
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": threads, "physical_cores": phys,
                         "cpu_model": model, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def headline_config():
    """The headline workload, identical in every arm."""
    return {"workload": WORKLOAD, "m": V * V, "n": O * O, "k": V * V, "inputs": INPUTS,
            "tolerance": "normwise relative error <= 1e-12 against the reference's FP64 result",
            "l2": "inputs larger than L2 (A is %.2f GB)" % (V ** 4 * 8 / 1e9),
            "parallelism": "replicas (one ladder contraction per GPU per step)"}


# ---------------------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_index):
        self.proc = None
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ids = [x.strip() for x in vis.split(",")] if vis else []
        self.gpu = ids[local_index] if local_index < len(ids) else str(local_index)
        # one file per rank: several ranks on one node must not share it
        name = "clocks_bench.csv" if local_index == 0 else "clocks_bench_rank%d.csv" % local_index
        # TBLIS_B200_CLOCKS_DIR names where the samples go (default: the
        # system's temporary directory)
        import tempfile
        self.path = os.path.join(os.environ.get("TBLIS_B200_CLOCKS_DIR") or tempfile.gettempdir(), name)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, window=None):
        """Median SM clock, max clock and throttle reasons of the samples
        taken inside `window` (host times (t0, t1) of the timed region), or of
        all samples when none fall inside it (then "window" says so)."""
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                t = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((t, float(parts[2]), float(parts[3]),
                             [nm for nm, v in zip(names, parts[6:10]) if v.lower().startswith("active")]))
            except ValueError:
                continue
        inside = [r for r in rows if window and window[0] <= r[0] <= window[1]]
        use = inside if inside else rows
        if not use:
            return None
        reasons = sorted({nm for r in use for nm in r[3]})
        return {"sm_mhz": statistics.median(r[1] for r in use), "sm_max_mhz": use[-1][2], "reasons": reasons,
                "samples": len(use), "window": "timed region" if inside else "warm-up and timed region"}


def time_steps(torch, fn, steps, stream):
    """Times `steps` calls of fn with CUDA events on `stream`; per-step event
    pairs give the kernel duration of the (single-launch) step."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(steps):
        starts[i].record(stream)
        fn()
        ends[i].record(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    return e0.elapsed_time(e1), per


def measure_fp64_peak(torch, dev):
    """cuBLAS DGEMM 8192^3 (best of 5): the FP64 tensor-core denominator."""
    n = 8192
    a = torch.rand((n, n), dtype=torch.float64, device=dev)
    b = torch.rand((n, n), dtype=torch.float64, device=dev)
    c = torch.empty((n, n), dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    best = None
    for _ in range(5):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b, out=c)
        e.record()
        torch.cuda.synchronize()
        t = s.elapsed_time(e)
        best = t if best is None else min(best, t)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measure_int8_peak(torch, dev):
    """cuBLAS int8 GEMM 8192^3 (torch._int_mm, best of 5): the dense INT8
    tensor-core denominator of the Ozaki kernel (TOP/s), or None."""
    try:
        n = 8192
        a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev)
        b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev).t().contiguous().t()
        for _ in range(2):
            torch._int_mm(a, b)
        best = None
        for _ in range(5):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            torch.cuda.synchronize()
            t = s.elapsed_time(e)
            best = t if best is None else min(best, t)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import tblis_b200 as tb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    stream = torch.cuda.current_stream()
    tb.set_stream(stream.cuda_stream)

    if args.case == "serve":
        print(json.dumps(serve_workloads(torch, tb, dev)))
        return
    if args.case == "batch":
        print(json.dumps(batch_workload(torch, tb, dev, stream, count=args.batch_count,
                                        serial_sample=min(500, args.batch_count),
                                        check_sample=min(400, args.batch_count))))
        return
    if args.case:
        print(json.dumps(single_case(torch, tb, dev, stream, args)))
        return

    # --- headline workload: ladder with exponent spread --------------------------------
    # the same host-generated bits on every rank and in every arm
    hA, hB, hC, keep = ladder_inputs(pinned=True)
    A = keep[0].to(dev).view(V, V, V, V).permute(3, 2, 1, 0)
    B = keep[1].to(dev).view(O, O, V, V).permute(3, 2, 1, 0)
    C = torch.zeros((O, O, V, V), dtype=torch.float64, device=dev).permute(3, 2, 1, 0)

    # method selection: Ozaki INT8 with the slice count the library picks for
    # 1e-12, kept when it meets 1e-12 against the FP64 path on this input, else
    # the plain FP64 DMMA path (its error is the FP64 rounding itself)
    method, method_name, cfg_name = 1, "fp64_dmma", "b200_fp64"
    used_method = 1
    Cfp = torch.zeros_like(C)
    tb.mult_ex(1.0, A, "abef", B, "efij", 0.0, Cfp, "abij", method=1)
    try:
        rep = tb.mult_ex(1.0, A, "abef", B, "efij", 0.0, C, "abij", method=2, tolerance=1e-12)
        torch.cuda.synchronize()
        err = (torch.linalg.vector_norm(C - Cfp) / torch.linalg.vector_norm(Cfp)).item()
        if err <= 1e-12:
            # the INT8 config picks slices (scheme I) or moduli (scheme II, reported as method 6)
            method, cfg_name = 2, "b200_ozaki_i8"
            method_name = ("ozaki_int8_%d_moduli" if rep["method"] == 6 else "ozaki_int8_%d_slices") % rep["slices"]
            used_method = rep["method"]
    except tb.TblisError:
        pass

    def step():
        tb.mult_ex(1.0, A, "abef", B, "efij", 0.0, C, "abij", method=method, tolerance=1e-12)

    def step_fp64():
        tb.mult_ex(1.0, A, "abef", B, "efij", 0.0, Cfp, "abij", method=1)

    # clocks sampled every 50 ms from before the warm-up on; the samples
    # inside the timed region are the ones reported
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    k0 = tb.kernel_count()
    tb.kernel_timer(True)
    t_timed0 = time.time()
    total_ms, per = time_steps(torch, step, args.steps, stream)
    t_timed1 = time.time()
    launches = tb.kernel_count() - k0
    kname = {1: "gemm_f64_kernel", 2: "ozaki_gemm_kernel", 6: "oz_crt_gemm"}[used_method]
    k_total_ms, k_launches = tb.kernel_time(kname)
    # device time per step of each stage of the contraction
    stages = {1: (kname,), 2: ("oz_stats", "oz_slice", kname), 6: ("oz_stats", "oz_slice", kname, "oz_crt_combine")}
    stage_ms = {n: tb.kernel_time(n)[0] / args.steps for n in stages[used_method]}
    tb.kernel_timer(False)
    clocks = sampler.stop((t_timed0, t_timed1))
    total_ms = max_over_ranks(dist, torch, total_ms, dev)
    ms_per_step = total_ms / args.steps
    value = job_value(world, args.steps, total_ms)

    # end to end through tblis_tensor_mult(NULL, tblis_get_config(cfg_name), ...)
    # with the pinned host buffers (copies inside the timed region), on every
    # rank, max over ranks
    e2e = None
    if not args.no_e2e:
        if dist:
            dist.barrier()
        e2e = e2e_ladder(torch, tb, cfg_name, max(2, min(args.steps, 3)), hA, hB, hC)
        e2e_ms = max_over_ranks(dist, torch, e2e["ms_per_step"], dev)
        e2e["ms_per_step"] = e2e_ms
        e2e["value"] = job_value(world, 1, e2e_ms)

    result = {
        "metric": METRIC,
        "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": headline_config(),
        "method": method_name,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if e2e:
        result["e2e"] = e2e

    if rank == 0:
        peaks = load_peaks()
        extra = {}
        # plain FP64 rate on the same workload and the roofline of its kernel
        fp64_peak = measure_fp64_peak(torch, dev)
        for _ in range(2):
            step_fp64()
        fp_ms, fp_per = time_steps(torch, step_fp64, max(3, args.steps // 2), stream)
        fp_kernel_ms = statistics.mean(fp_per)
        fp64_gflops = FLOPS_LADDER / (fp_kernel_ms * 1e-3) / 1e9
        extra["fp64_dmma_gflops"] = fp64_gflops
        extra["cublas_dgemm_8192_tflops"] = fp64_peak
        extra["fp64_path_frac_of_cublas_dgemm"] = fp64_gflops / 1e3 / fp64_peak
        extra["speedup_vs_fp64_path"] = value / world / fp64_gflops
        extra["stage_ms_per_step"] = stage_ms
        # the dominant kernel's own device time: CUDA events around each of its
        # launches on the launching stream, inside the timed steps
        launch_ms = k_total_ms / max(1, k_launches)
        units_per_launch = args.steps / max(1, k_launches)    # ladder contractions per launch
        if method == 1:
            achieved = FLOPS_LADDER * units_per_launch / (launch_ms * 1e-3) / 1e12
            result["roofline"] = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                                  "frac": achieved / fp64_peak, "traffic": None,
                                  "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor cores)",
                                  "kernel": "gemm_f64_kernel", "launch_ms": launch_ms,
                                  "share_of_step": k_total_ms / total_ms}
        else:
            # the dominant kernel is the INT8 GEMM: S(S+1)/2 GEMMs of m x n x k
            # for S slices (the fused slice-pair kernel), or one per modulus
            # (2 ops per MAC)
            S = int(method_name.split("_")[2])
            gemms = S if used_method == 6 else S * (S + 1) / 2
            int8_ops = gemms * FLOPS_LADDER * units_per_launch
            achieved = int8_ops / (launch_ms * 1e-3) / 1e12
            i8peak = measure_int8_peak(torch, dev)
            src = "cuBLAS int8 GEMM 8192^3 (torch._int_mm) measured in this run"
            if not i8peak:
                i8peak = 2.0 * peaks.get("bf16_tflops", 1590.0)
                src = "2 x measured bf16 dense GEMM (MEASURED_PEAKS.json)"
            # DRAM bytes (read + write) of one full-size oz_crt_gemm2 launch of this
            # workload with 13 moduli, from a one-pass ncu capture
            # (profiles/oz_crt_gemm_ladder.md): 15.79 GB read + 0.78 GB written
            traffic = None
            if used_method == 6 and gemms == 13 and (O, V) == (48, 160):
                traffic = 15.79e9 + 0.78e9
            m_, n_, k_ = V * V, O * O, V * V
            result["roofline"] = {"bound": "tensor", "achieved": achieved, "peak": i8peak, "unit": "TOP/s (int8)",
                                  "frac": achieved / i8peak, "traffic": traffic,
                                  "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                                    "full-size launch (profiles/oz_crt_gemm_ladder.md)"
                                                    if traffic else None,
                                  "algorithmic_bytes": gemms * (m_ * k_ + n_ * k_ + m_ * n_) if used_method == 6
                                                       else None,
                                  "peak_source": src,
                                  "kernel": kname, "launch_ms": launch_ms, "int8_gemms_per_launch": gemms,
                                  "share_of_step": k_total_ms / total_ms,
                                  "fp64_equivalent_tflops_kernel": FLOPS_LADDER * units_per_launch /
                                                                   (launch_ms * 1e-3) / 1e12}

        # accuracy: every GPU result against the reference's own FP64 output
        # on the same inputs (N=1: the CPU leg computes it); with several
        # ranks, against the library's FP64 path
        acc = {}
        Cref_dev = None
        if world == 1 and not args.no_cpu:
            cb = cpu_reference_ladder(hA, hB)
            if cb:
                v, threads, phys, model, sample, Cref = cb
                result["cpu_baseline"] = {"value": v, "unit": "GFLOP/s", "cores": threads, "physical_cores": phys,
                                          "cpu_model": model, "kind": "reference", "sample": sample}
                acc["against"] = "the reference's tblis_tensor_mult (FP64, CPU) on the same inputs"
                acc["normwise_rel_err_vs_reference"] = normwise(
                    C.permute(3, 2, 1, 0).cpu().numpy().transpose(3, 2, 1, 0), Cref)
                acc["fp64_path_normwise_rel_err_vs_reference"] = normwise(
                    Cfp.permute(3, 2, 1, 0).cpu().numpy().transpose(3, 2, 1, 0), Cref)
                if e2e:
                    e2e["normwise_rel_err_vs_reference"] = normwise(hC, Cref)
                Cref_dev = torch.from_numpy(Cref.transpose(3, 2, 1, 0).copy()).to(dev).permute(3, 2, 1, 0)
                del Cref
        if Cref_dev is None:
            acc["against"] = "the library's plain FP64 path on the same inputs"
            acc["normwise_rel_err_vs_fp64_path"] = (torch.linalg.vector_norm(C - Cfp) /
                                                    torch.linalg.vector_norm(Cfp)).item()
        err = acc.get("normwise_rel_err_vs_reference", acc.get("normwise_rel_err_vs_fp64_path"))
        acc["meets_1e-12"] = bool(err is not None and err <= 1e-12)
        result["accuracy"] = acc

        if not args.no_extra and world == 1:
            extra["precision_variants"] = precision_variants(torch, tb, A, B, C, stream,
                                                             Cref_dev if Cref_dev is not None else Cfp)
        del A, B, C, Cfp, Cref_dev
        torch.cuda.empty_cache()

        # the secondary workloads are single-GPU; with several ranks the others
        # would wait at the closing barrier for minutes
        if not args.no_extra and world == 1:
            extra.update(extra_workloads(torch, tb, dev, stream, peaks, check=not args.no_cpu))
        result["extra"] = extra
        print(json.dumps(result))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def precision_variants(torch, tb, A, B, C, stream, Cref):
    """The ladder under every arithmetic the library offers: plain FP64 DMMA,
    Ozaki INT8 slices (3..8), Ozaki INT8 moduli (8..16), Ozaki BF16 slices
    (3..8), one TF32 and one BF16 pass.
    Error = normwise relative difference to Cref (the reference's own FP64
    result on the same inputs at N=1); rate = FP64-equivalent GFLOP/s of the
    whole call (statistics, slicing and GEMM), mean of 2."""
    nref = torch.linalg.vector_norm(Cref).item()
    runs = [("fp64_dmma", 1, 0)]
    runs += [("ozaki_int8", 2, s) for s in range(3, 9)]
    runs += [("ozaki_int8_moduli", 6, n) for n in (8, 10, 11, 12, 13, 14, 16)]
    runs += [("ozaki_bf16", 3, s) for s in range(3, 9)]
    runs += [("tf32_single_pass", 4, 1), ("bf16_single_pass", 5, 1)]
    out = []
    for name, method, slices in runs:
        def call():
            tb.mult_ex(1.0, A, "abef", B, "efij", 0.0, C, "abij", method=method, slices=slices, tolerance=1e-12)
        call()
        torch.cuda.synchronize()
        err = (torch.linalg.vector_norm(C - Cref) / nref).item()
        total, _ = time_steps(torch, call, 2, stream)
        out.append({"variant": name, "slices": slices, "normwise_rel_err": err,
                    "gflops_fp64_equiv": FLOPS_LADDER * 2 / (total * 1e-3) / 1e9})
    return out


def max_over_ranks(dist, torch, value, dev):
    """The largest of one scalar over all ranks (the job's time is its
    slowest rank's); the value itself with one process."""
    if not dist:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return t.item()


def job_value(world, steps, total_ms):
    """Whole-job GFLOP/s: every rank contracts its own ladder per step."""
    return world * FLOPS_LADDER * steps / (total_ms * 1e-3) / 1e9


def e2e_ladder(torch, tb, cfg_name, steps, hA, hB, hC):
    """The same contraction through tblis_tensor_mult(NULL,
    tblis_get_config(cfg_name), ...) on pinned host buffers: the H2D copies of
    A and B and the D2H copy of C happen inside every call."""
    cfg = tb.get_config(cfg_name)
    h2d = (hA.size + hB.size) * 8
    d2h = hC.size * 8
    tb.mult(1.0, hA, "abef", hB, "efij", 0.0, hC, "abij", cfg=cfg)
    t0 = time.perf_counter()
    for _ in range(steps):
        tb.mult(1.0, hA, "abef", hB, "efij", 0.0, hC, "abij", cfg=cfg)
    dt = (time.perf_counter() - t0) / steps
    return {"value": FLOPS_LADDER / dt / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3,
            "call": "tblis_tensor_mult(NULL, tblis_get_config(\"%s\"), ...)" % cfg_name,
            "note": "host pinned buffers; H2D of A,B and D2H of C inside each call (the library copies A in "
                    "slabs of rows of C overlapped with the contraction of the slabs already copied, and each "
                    "slab of C back as soon as it is final)"}


OCC = [12, 4, 8, 6, 10, 3, 7, 5]
VIR = [60, 22, 40, 30, 52, 14, 36, 26]


def dpd_workload(torch, tb, dev, stream, check=True):
    """DPD ladder C[abij] = A[abef]*B[efij] under D2h (8 irreps, XOR, total
    irrep 0), occ [12,4,8,6,10,3,7,5], vir [60,22,40,30,52,14,36,26], default
    MArray layout; one grouped launch per call (graph-replayed). Returns the
    DPD rate and the dense-equivalent rate: dense FP64 GEMMs of the same
    per-irrep M x N x K on the same kernel; with `check`, the normwise error of
    C against the reference's own DPD contraction on the same inputs."""
    import numpy as np
    out = {}
    g = torch.Generator(device=dev)
    g.manual_seed(41)
    A = tb.DpdTensor(0, 8, [VIR, VIR, VIR, VIR])
    B = tb.DpdTensor(0, 8, [VIR, VIR, OCC, OCC])
    C = tb.DpdTensor(0, 8, [VIR, VIR, OCC, OCC])
    A.data = torch.empty(A.size(), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
    B.data = torch.empty(B.size(), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
    C.data = torch.zeros(C.size(), dtype=torch.float64, device=dev)
    rep = tb.dpd_mult(1.0, A, "abef", B, "efij", 0.0, C, "abij")      # plan, tuning, graph
    flops = rep["flops"]
    for _ in range(2):
        tb.dpd_mult(1.0, A, "abef", B, "efij", 0.0, C, "abij")
    ms, per = time_steps(torch, lambda: tb.dpd_mult(1.0, A, "abef", B, "efij", 0.0, C, "abij"), 5, stream)
    dpd_ms = statistics.median(per)
    out["dpd_gflop"] = flops / 1e9
    out["dpd_gflops"] = flops / (dpd_ms * 1e-3) / 1e9
    out["dpd_groups"] = rep["m"]
    out["dpd_tile_variant"] = rep["n"]
    # dense-equivalent: per irrep h, M_h = sum_g v_g v_{g^h}, N_h = sum_g o_g o_{g^h}, K_h = M_h
    tot_f, tot_ms = 0.0, 0.0
    for h in range(8):
        M = sum(VIR[x] * VIR[x ^ h] for x in range(8))
        N = sum(OCC[x] * OCC[x ^ h] for x in range(8))
        a = torch.empty((M, M), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
        b = torch.empty((M, N), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
        c = torch.zeros((M, N), dtype=torch.float64, device=dev)
        f = lambda: tb.mult(1.0, a, "ik", b, "kj", 0.0, c, "ij")
        f()
        _, p = time_steps(torch, f, 3, stream)
        tot_f += 2.0 * M * N * M
        tot_ms += statistics.median(p)
        del a, b, c
    out["dpd_dense_equiv_gflops"] = tot_f / (tot_ms * 1e-3) / 1e9
    out["dpd_frac_of_dense_equiv"] = out["dpd_gflops"] / out["dpd_dense_equiv_gflops"]
    if check:
        # the grouped launch's C against the reference's own DPD tblis::mult
        # (src/internal/3t/dpd/mult.cxx:1067-1267) on the host, same inputs
        import oracle
        if oracle.have_ref():
            threads, _, _ = host_cpu()
            oracle.ref().tblis_set_num_threads(threads)
            hA, hB = A.data.cpu().numpy(), B.data.cpu().numpy()
            want = np.zeros(C.size())
            t0 = time.perf_counter()
            oracle.ref_dpd_mult(8, 1.0, 0, [VIR] * 4, hA, "abef", 0, [VIR, VIR, OCC, OCC], hB, "efij",
                                0.0, 0, [VIR, VIR, OCC, OCC], want, "abij")
            out["dpd_reference_s"] = time.perf_counter() - t0
            out["dpd_normwise_rel_err_vs_reference"] = normwise(C.data.cpu().numpy(), want)
            del hA, hB, want
    del A, B, C
    torch.cuda.empty_cache()
    return out


def batch_workload(torch, tb, dev, stream, count=10000, serial_sample=500, check=True, check_sample=400):
    """A batch of `count` independent 4-index contractions (2 labels per group,
    extents uniform 4..32, random index order of every operand) in one grouped
    launch, against the same contractions issued one call at a time (timed on
    the first `serial_sample` and scaled); with `check`, a seeded sample of
    `check_sample` members against the reference on the host."""
    import random
    rnd = random.Random(0)
    g = torch.Generator(device=dev)
    g.manual_seed(43)
    items, flops = [], 0.0
    for _ in range(count):
        l = {c: rnd.randint(4, 32) for c in "abefij"}
        ia = "".join(rnd.sample("abef", 4))
        ib = "".join(rnd.sample("efij", 4))
        ic = "".join(rnd.sample("abij", 4))
        mk = lambda ix: torch.empty([l[c] for c in ix], dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
        items.append((1.0, mk(ia), ia, mk(ib), ib, 0.0, mk(ic), ic))
        flops += 2.0 * l["a"] * l["b"] * l["e"] * l["f"] * l["i"] * l["j"]
    prepared = tb.PreparedBatch(items)
    prepared.run()                          # plan + tuning + graph
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        prepared.run()
    torch.cuda.synchronize()
    batch_s = (time.perf_counter() - t0) / reps
    # device time of the grouped launch alone
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    prepared.run()
    e1.record()
    torch.cuda.synchronize()
    device_ms = e0.elapsed_time(e1)
    sample = items[:serial_sample]
    for it in sample[:20]:
        tb.mult(*it)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in sample:
        tb.mult(*it)
    torch.cuda.synchronize()
    serial_s = (time.perf_counter() - t0) * count / len(sample)
    out = {"batch_count": count, "batch_gflop": flops / 1e9, "batch_gflops": flops / batch_s / 1e9,
           "batch_wall_ms": batch_s * 1e3, "batch_event_ms": device_ms, "serial_gflops_est": flops / serial_s / 1e9,
           "batch_speedup_vs_serial": serial_s / batch_s}
    if check:
        # a seeded sample of members (their C holds the batch's last result:
        # beta is 0) against the reference's tblis_tensor_mult on the host
        import numpy as np
        import oracle
        if oracle.have_ref():
            errs = []
            for j in random.Random(1).sample(range(count), check_sample):
                al, a, ia, b, ib, be, c, ic = items[j]
                want = np.zeros(c.shape, order="F")
                oracle.ref_mult(al, a.cpu().numpy(), ia, b.cpu().numpy(), ib, 0.0, want, ic, threads=1)
                errs.append(normwise(c.cpu().numpy(), want))
            out["batch_checked_members"] = len(errs)
            out["batch_max_normwise_rel_err_vs_reference"] = max(errs)
    return out


SERVE_REQUESTS = 20000
SERVE_POOL_BYTES = 48 << 30
SERVE_RATES = (50, 200, 500, 1000, 2000)
SERVE_WINDOW_S = 4.0


def serve_pool(torch, dev, budget_bytes, seed=0):
    """Resident problems of the serving stream: 6 labels split 2/2/2 at random
    into contracted, A-only and B-only groups, every operand's index order
    permuted, extents log-uniform in 8..128, each operand at most 256 MB
    (resampled otherwise), FP64 uniform(-1,1); drawn until A, B and C of all
    problems fill budget_bytes of HBM (a solver's resident amplitudes)."""
    import math
    import random
    rnd = random.Random(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1)
    cap = (256 << 20) // 8
    pool, used = [], 0
    while True:
        labs = list("abcdef")
        rnd.shuffle(labs)
        AB, AC, BC = labs[0:2], labs[2:4], labs[4:6]
        l = {c: int(round(math.exp(rnd.uniform(math.log(8), math.log(128))))) for c in labs}
        ia, ib, ic = AB + AC, AB + BC, AC + BC
        sizes = [math.prod(l[c] for c in x) for x in (ia, ib, ic)]
        if max(sizes) > cap:
            continue
        if used + 8 * sum(sizes) > budget_bytes:
            break
        used += 8 * sum(sizes)
        rnd.shuffle(ia); rnd.shuffle(ib); rnd.shuffle(ic)
        ia, ib, ic = "".join(ia), "".join(ib), "".join(ic)
        mk = lambda ix: torch.empty([l[c] for c in ix], dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
        pool.append(dict(A=mk(ia), B=mk(ib), C=mk(ic), ia=ia, ib=ib, ic=ic, flops=2.0 * math.prod(l.values()),
                         c_bytes=8 * sizes[2]))
    return pool, used


def serve_stream(n, npool, rate, seed):
    """n requests: a uniformly drawn resident problem each, tolerance 1e-10 or
    1e-13 (50/50), Poisson gaps at `rate` per second."""
    import random
    rnd = random.Random(seed)
    picks = [rnd.randrange(npool) for _ in range(n)]
    tols = [1e-10 if rnd.random() < 0.5 else 1e-13 for _ in range(n)]
    gaps = [rnd.expovariate(rate) for _ in range(n)] if rate else [0.0] * n
    return picks, tols, gaps


def serve_run(torch, tb, pool, picks, tols, gaps, outs=None):
    """Submits the requests at their arrival times to a server with the
    150 GB admission budget and waits for all; returns (seconds from the
    first arrival to the last completion, arrival window, server stats)."""
    srv = tb.Server(hbm_budget_bytes=150 << 30, slots=4)
    ids = []
    t0 = time.perf_counter()
    due = t0
    for j, i in enumerate(picks):
        due += gaps[j]
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        p = pool[i]
        C = outs[j] if outs is not None else p["C"]
        ids.append(srv.submit(1.0, p["A"], p["ia"], p["B"], p["ib"], 0.0, C, p["ic"], tols[j]))
    for rid in ids:
        srv.wait(rid)
    served = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    return served, due - t0, st


def serial_run(torch, tb, pool, picks, gaps):
    """The same requests as plain tblis_tensor_mult calls (FP64 path), each
    waiting for its arrival and its predecessor; returns (seconds, latencies
    in ms, sorted)."""
    lat = []
    t0 = time.perf_counter()
    due = t0
    for j, i in enumerate(picks):
        due += gaps[j]
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        p = pool[i]
        tb.mult(1.0, p["A"], p["ia"], p["B"], p["ib"], 0.0, p["C"], p["ic"])
        if gaps[j]:
            torch.cuda.synchronize()
            lat.append((time.perf_counter() - due) * 1e3)
    torch.cuda.synchronize()
    return time.perf_counter() - t0, sorted(lat)


def serve_check(torch, tb, pool, picks, tols, chunk_bytes=8 << 30):
    """Every request of the stream again through the server (bursts of
    requests whose outputs fit chunk_bytes, each into its own output buffer),
    each result against the same problem computed alone on the plain FP64
    path; returns (requests checked, requests over their tolerance, largest
    error / tolerance)."""
    refs = {}
    for i in sorted(set(picks)):
        p = pool[i]
        r = torch.empty_like(p["C"])
        tb.mult(1.0, p["A"], p["ia"], p["B"], p["ib"], 0.0, r, p["ic"])
        refs[i] = (r, torch.linalg.vector_norm(r).item())
    checked, bad, worst = 0, 0, 0.0
    j = 0
    while j < len(picks):
        k, size = j, 0
        while k < len(picks) and (k == j or size + pool[picks[k]]["c_bytes"] <= chunk_bytes):
            size += pool[picks[k]]["c_bytes"]
            k += 1
        outs = [torch.empty_like(pool[picks[x]]["C"]) for x in range(j, k)]
        serve_run(torch, tb, pool, picks[j:k], tols[j:k], [0.0] * (k - j), outs)
        for x, o in zip(range(j, k), outs):
            r, nr = refs[picks[x]]
            err = torch.linalg.vector_norm(o - r).item() / (nr if nr else 1.0)
            worst = max(worst, err / tols[x])
            bad += err > tols[x]
            checked += 1
        del outs
        j = k
    del refs
    torch.cuda.empty_cache()
    return checked, bad, worst


def serve_workloads(torch, tb, dev):
    """Config 5: a stream of 20,000 pairwise 4-index contraction requests over
    a resident pool filling 48 GB of HBM, as a burst and under Poisson
    arrivals at 50-2,000 req/s (4 s of arrivals per rate), against serial
    plain calls under the same arrivals; every request of the burst checked
    against the same request run alone on the plain FP64 path."""
    out = {}
    pool, used = serve_pool(torch, dev, SERVE_POOL_BYTES)
    out["serve_pool"] = {"problems": len(pool), "operand_gb": used / 1e9}
    picks, tols, gaps = serve_stream(SERVE_REQUESTS, len(pool), 0, seed=3)
    flops = sum(pool[i]["flops"] for i in picks)
    # warm-up: the shapes' first plans
    serve_run(torch, tb, pool, picks[:64], tols[:64], [0.0] * 64)
    serial_s, _ = serial_run(torch, tb, pool, picks, gaps)
    served, _, st = serve_run(torch, tb, pool, picks, tols, gaps)
    out["serve_burst"] = {
        "requests": SERVE_REQUESTS, "tflop": flops / 1e12, "distinct_problems": len(set(picks)),
        "served_req_s": SERVE_REQUESTS / served, "served_gflops": flops / served / 1e9,
        "serial_req_s": SERVE_REQUESTS / serial_s, "serial_gflops": flops / serial_s / 1e9,
        "throughput_vs_serial": serial_s / served,
        "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
        "batches": st["batches"], "mean_batch": st["mean_batch"],
        "max_concurrent_batches": st["max_concurrent_batches"], "ozaki_requests": st["ozaki"],
        "shape_cache_hit_rate": st["shape_hits"] / max(1, st["shape_hits"] + st["shape_misses"])}
    checked, bad, worst = serve_check(torch, tb, pool, picks, tols)
    out["serve_burst"].update({"checked_requests": checked, "requests_over_tolerance": bad,
                               "max_err_over_tolerance": worst})
    for rate in SERVE_RATES:
        n = int(rate * SERVE_WINDOW_S)
        picks, tols, gaps = serve_stream(n, len(pool), rate, seed=rate)
        flops = sum(pool[i]["flops"] for i in picks)
        served, window, st = serve_run(torch, tb, pool, picks, tols, gaps)
        serial_s, lat = serial_run(torch, tb, pool, picks, gaps)
        out["serve_%d" % rate] = {
            "rate_req_s": rate, "requests": n, "arrival_window_s": window,
            "served_req_s": n / served, "served_gflops": flops / served / 1e9,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
            "batches": st["batches"], "mean_batch": st["mean_batch"],
            "shape_cache_hit_rate": st["shape_hits"] / max(1, st["shape_hits"] + st["shape_misses"]),
            "serial_same_arrivals": {"req_s": n / serial_s, "p50_ms": lat[len(lat) // 2],
                                     "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "throughput_vs_serial_same_arrivals": serial_s / served}
    del pool
    torch.cuda.empty_cache()
    return out


def single_case(torch, tb, dev, stream, args):
    """One secondary kernel alone at extents o, v (for profiling captures):
    ring C[aibj] += A[aeim]*B[mbej] (FP64 DMMA), transpose D[ijab] = C[abij],
    dot, NORM_2 reduce, or (dpd, fixed extents) the D2h DPD ladder of the
    secondary workloads in one grouped launch."""
    o, v = args.o, args.v
    g = torch.Generator(device=dev)
    g.manual_seed(7)

    def cm(shape):
        return torch.empty(list(reversed(shape)), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g) \
            .permute(*reversed(range(len(shape))))
    if args.case == "dpd":
        # per-irrep extents scaled by o/48 and v/160 (the defaults give the
        # secondary workload's D2h ladder itself)
        vir = [max(1, round(x * v / 160)) for x in VIR]
        occ = [max(1, round(x * o / 48)) for x in OCC]
        A = tb.DpdTensor(0, 8, [vir, vir, vir, vir])
        B = tb.DpdTensor(0, 8, [vir, vir, occ, occ])
        C = tb.DpdTensor(0, 8, [vir, vir, occ, occ])
        A.data = torch.empty(A.size(), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
        B.data = torch.empty(B.size(), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
        C.data = torch.zeros(C.size(), dtype=torch.float64, device=dev)

        def fn():
            return tb.dpd_mult(1.0, A, "abef", B, "efij", 0.0, C, "abij")
        work, unit = fn()["flops"] / 1e9, "GFLOP/s"
    elif args.case == "ring":
        A, B, C = cm([v, v, o, o]), cm([o, v, v, o]), cm([v, o, v, o])

        def fn():
            tb.mult_ex(1.0, A, "aeim", B, "mbej", 1.0, C, "aibj", method=1)
        work, unit = 2.0 * v ** 3 * o ** 3 / 1e9, "GFLOP/s"
    elif args.case == "transpose":
        C = cm([v, v, o, o])
        D = torch.zeros((v, v, o, o), dtype=torch.float64, device=dev).permute(3, 2, 1, 0)

        def fn():
            tb.add(1.0, C, "abij", 0.0, D, "ijab")
        work, unit = 2 * C.numel() * 8 / 1e9, "GB/s"
    elif args.case == "dot":
        C, E = cm([v, v, o, o]), cm([v, v, o, o])

        def fn():
            tb.dot(C, "abij", E, "abij")
        work, unit = 2 * C.numel() * 8 / 1e9, "GB/s"
    else:
        C = cm([v, v, o, o])

        def fn():
            tb.reduce(tb.REDUCE_NORM_2, C, "abij")
        work, unit = C.numel() * 8 / 1e9, "GB/s"
    for _ in range(args.warmup):
        fn()
    total, _ = time_steps(torch, fn, args.steps, stream)
    return {"case": args.case, "o": o, "v": v, "value": work * args.steps / (total * 1e-3), "unit": unit,
            "ms_per_step": total / args.steps}


def extra_workloads(torch, tb, dev, stream, peaks, check=True):
    out = {}
    try:
        out.update(serve_workloads(torch, tb, dev))
    except Exception as e:     # keep the headline line even if a secondary workload fails
        out["serve_error"] = str(e)[:200]
    try:
        out.update(dpd_workload(torch, tb, dev, stream, check))
    except Exception as e:     # keep the headline line even if a secondary workload fails
        out["dpd_error"] = str(e)[:200]
    try:
        out.update(batch_workload(torch, tb, dev, stream, check=check))
    except Exception as e:
        out["batch_error"] = str(e)[:200]
    torch.cuda.empty_cache()
    # ring: C[aibj] += A[aeim]*B[mbej], o=64, v=256 (8.8 TFLOP), FP64 DMMA
    o, v = 64, 256
    g = torch.Generator(device=dev)
    g.manual_seed(7)

    def cm(shape):
        return torch.empty(list(reversed(shape)), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g) \
            .permute(*reversed(range(len(shape))))
    A = cm([v, v, o, o])
    B = cm([o, v, v, o])
    C = cm([v, o, v, o])
    fl = 2.0 * v ** 3 * o ** 3

    def ring():
        tb.mult_ex(1.0, A, "aeim", B, "mbej", 1.0, C, "aibj", method=1)
    ring()
    ms, per = time_steps(torch, ring, 2, stream)
    out["ring_fp64_gflops"] = fl / (statistics.mean(per) * 1e-3) / 1e9
    del A, B
    # transpose D[ijab] = C[abij] at the same size (bytes = read + write)
    Cs = cm([v, v, o, o])
    D = torch.zeros((v, v, o, o), dtype=torch.float64, device=dev).permute(3, 2, 1, 0)

    def tr():
        tb.add(1.0, Cs, "abij", 0.0, D, "ijab")
    for _ in range(3):
        tr()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    pers = []
    for _ in range(5):
        flush.fill_(1)
        _, p = time_steps(torch, tr, 1, stream)
        pers.append(p[0])
    gbs = 2 * Cs.numel() * 8 / (statistics.median(pers) * 1e-3) / 1e9
    out["transpose_gbs"] = gbs
    if peaks.get("hbm_gbs"):
        out["transpose_frac_of_measured_hbm"] = gbs / peaks["hbm_gbs"]
    del D
    # dot of two 2.15 GB tensors (bytes = both reads) and a NORM_2 reduction
    # of one (its read), L2 flushed before each timed call
    E = cm([v, v, o, o])

    def bw(fn, nbytes):
        for _ in range(3):
            fn()
        pers = []
        for _ in range(5):
            flush.fill_(1)
            _, p = time_steps(torch, fn, 1, stream)
            pers.append(p[0])
        return nbytes / (statistics.median(pers) * 1e-3) / 1e9
    out["dot_gbs"] = bw(lambda: tb.dot(Cs, "abij", E, "abij"), 2 * Cs.numel() * 8)
    out["reduce_norm2_gbs"] = bw(lambda: tb.reduce(tb.REDUCE_NORM_2, Cs, "abij"), Cs.numel() * 8)
    if peaks.get("hbm_gbs"):
        out["dot_frac_of_measured_hbm"] = out["dot_gbs"] / peaks["hbm_gbs"]
        out["reduce_frac_of_measured_hbm"] = out["reduce_norm2_gbs"] / peaks["hbm_gbs"]
    del C, Cs, E, flush
    torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    main()
