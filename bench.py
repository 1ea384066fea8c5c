"""Benchmark: pi to 10^9 decimal digits on one B200 (Chudnovsky binary
splitting + Newton division / inverse square root on the GPU multiply engine),
digits identical to the reference's pi.txt.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--digits D]
                    [--impl ours|reference]

One step = one whole pi computation (the path's hot loop: every product,
carry and truncation of Pi(), PI.h:138-212).  `value` is device seconds per
computation measured with CUDA events on the library's stream, result left in
HBM; `e2e` is the same computation through the public C ABI call pic_pi_hex
writing the reference's text into pinned host memory (device->host copy inside
the timed region).  Multi-GPU runs are independent replicas (the path has no
exchange step); the reported time is the max over ranks.

--impl reference times the reference's own CPU program (oracle/_ref/picref_pi,
built from the reference sources) on this host's cores instead: each step is a
bounded pi run at --ref-sample digits, extrapolated to --digits with the
scaling exponent measured between two sample sizes in the same run.
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
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1e9-digit π wall time on 1 B200 vs plain GPU form & CPU; NTT HBM GB/s vs peak"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--digits", type=int, default=1_000_000_000)
    ap.add_argument("--form", choices=["chosen", "plain"], default="chosen")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--plain-digits", type=int, default=1_000_000,
                    help="size at which the plain per-product form is timed beside the chosen form")
    ap.add_argument("--ref-sample", type=int, default=10_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers ----
def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

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
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def run_reference_pi(digits: int, threads: int) -> float:
    from oracle.ffi import REF_PI
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([REF_PI, str(digits), str(threads)], cwd=d, capture_output=True, text=True,
                           check=True)
    return float(json.loads(r.stderr.strip().splitlines()[-1])["pi_s"])


def cpu_reference_estimate(target_digits: int, sample: int, threads: int):
    """Reference CPU time at `sample` digits and a scaled estimate for the
    target, exponent fitted between sample/10 and sample."""
    t_small = run_reference_pi(sample // 10, threads)
    t_big = run_reference_pi(sample, threads)
    expo = math.log10(max(t_big, 1e-6) / max(t_small, 1e-6))
    est = t_big * (target_digits / sample) ** expo
    return est, t_big, t_small, expo


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise max of per-rank timings (the slowest replica sets the
    job's time).  Identity when not distributed."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


# ---------------------------------------------------------- reference arm ----
def reference_arm(args):
    rank, _, world = rank_info()
    if rank != 0:
        return
    from oracle.ffi import REF_PI
    if not os.path.exists(REF_PI):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/picref_pi was not built (reference sources absent at build time)"}))
        return
    threads = os.cpu_count() or 1
    sample = args.ref_sample
    t_small = run_reference_pi(sample // 10, threads)  # calibration for the scaling exponent
    times = []
    for i in range(args.warmup + args.steps):
        t = run_reference_pi(sample, threads)
        if i >= args.warmup:
            times.append(t)
    t_big = statistics.mean(times)
    expo = math.log10(t_big / t_small)
    value = t_big * (args.digits / sample) ** expo
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_big * 1000.0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": f"pi_{args.digits:.0e}_digits", "digits": args.digits,
                                        "parallelism": "replicas"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                         "sample": f"reference Pi() at {sample} digits per step ({t_big:.2f} s mean), "
                                   f"scaled to {args.digits} digits with exponent {expo:.3f} fitted "
                                   f"against {sample // 10} digits ({t_small:.2f} s)"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def int_roof(P, torch, L, stream):
    """Row-pass butterflies per second on a 2^23-word three-prime product
    (3 row passes per product, each over 3 x 2^23 points and row_bits levels)
    against the register-only butterfly ceiling."""
    import ctypes as C

    k, n = 23, 1 << 23
    row_bits = P.get_ntt_geometry(k)[0]
    a = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda")
    b = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda")
    z = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    for _ in range(2):
        P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, "ntt3")
    torch.cuda.synchronize()
    P.check(L.pic_profile_begin())
    reps = 5
    for _ in range(reps):
        P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, "ntt3")
    stats = (P.KernelStat * 32)()
    cnt = C.c_int()
    P.check(L.pic_profile_end(stats, 32, C.byref(cnt)))
    rows = [s for s in stats[: cnt.value] if s.name.decode() == "ntt_rows"]
    if not rows or rows[0].seconds <= 0:
        return None
    bfly = rows[0].launches * 3 * (n // 2) * row_bits
    achieved = bfly / rows[0].seconds / 1e9
    ceiling = P.butterfly_rate()
    return {"kernel": "ntt_rows", "workload": "three-prime product of two 2^23-word operands",
            "row_bits": row_bits, "achieved": achieved, "ceiling": ceiling, "unit": "G butterflies/s",
            "frac": achieved / ceiling,
            "ceiling_basis": "lazy Shoup DIF butterflies with operands in registers, no memory traffic"}


def batched_products(P, torch, L, stream, count: int = 8192, top: int = 8192, seed: int = 7):
    """8192 independent products per call, operand sizes log-uniform in
    1..8192 limbs (splitmix64 seed 7), uniform random limbs: one pic_mul_batch
    call (persistent schoolbook + binned NTT, replayed from its CUDA graph)
    against one pic_mul launch sequence per product."""
    import numpy as np

    from oracle.ffi import splitmix64_np
    u = (splitmix64_np(seed, 2 * count) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    sizes = [max(1, min(top, int(math.exp(x * math.log(top))))) for x in u]
    na, nb = np.array(sizes[0::2]), np.array(sizes[1::2])
    rng = np.random.default_rng(seed)
    ta = torch.from_numpy(rng.integers(0, 2 ** 32, int(na.sum()), dtype=np.uint64).astype(np.uint32)
                          .view(np.int32)).cuda()
    tb = torch.from_numpy(rng.integers(0, 2 ** 32, int(nb.sum()), dtype=np.uint64).astype(np.uint32)
                          .view(np.int32)).cuda()
    tz = torch.zeros(int(na.sum() + nb.sum()), dtype=torch.int32, device="cuda")
    descs, oa, ob, oz = [], 0, 0, 0
    for x, y in zip(na.tolist(), nb.tolist()):
        descs.append((tz.data_ptr() + 4 * oz, ta.data_ptr() + 4 * oa, x, tb.data_ptr() + 4 * ob, y))
        oa += x
        ob += y
        oz += x + y
    torch.cuda.synchronize()

    def timed(fn, reps):
        fn()
        P.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    batched = timed(lambda: P.mul_batch_dev(descs, "auto"), 5)
    single = timed(lambda: [P.mul_dev(z, a, x, b, y, "auto") for (z, a, x, b, y) in descs], 1)
    return {"products": count, "sizes": "log-uniform 1..8192 limbs, splitmix64 seed 7",
            "batched_ms": batched, "one_launch_sequence_per_product_ms": single,
            "speedup": single / batched}


# ----------------------------------------------------------------- our arm ----
def ours(args):
    import ctypes as C

    import torch

    import piculator_b200 as P

    rank, local, world = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    P.init(local)
    L = P.lib()
    stream = torch.cuda.ExternalStream(L.pic_default_stream())
    form = P.PI_CHOSEN if args.form == "chosen" else P.PI_PLAIN
    hexd, pw, terms = P.pi_sizes(args.digits)

    def compute_step():
        h = C.c_void_p()
        st = P.PiStats()
        P.check(L.pic_pi_compute(args.digits, form, C.byref(h), C.byref(st)))
        L.pic_bf_free(h)
        return st

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        compute_step()
    barrier()
    # timed region: K whole computations, device time on the library's stream
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    phases = []
    for _ in range(args.steps):
        st = compute_step()
        launches += st.kernel_launches
        phases.append(st.as_dict())
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    dev_s = e0.elapsed_time(e1) / 1000.0 / args.steps
    barrier()

    # the same K computations again with every instrumented launch bracketed by
    # CUDA events on its own stream: per-kernel device time and algorithmic bytes
    P.check(L.pic_profile_begin())
    for _ in range(args.steps):
        compute_step()
    stats = (P.KernelStat * 32)()
    n = C.c_int()
    P.check(L.pic_profile_end(stats, 32, C.byref(n)))
    barrier()

    # e2e: the public call with the text delivered into pinned host memory
    cap = hexd + 64
    host = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
    outlen = C.c_size_t()
    st = P.PiStats()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        P.check(L.pic_pi_hex(args.digits, form, C.c_char_p(host.data_ptr()), cap, C.byref(outlen),
                             C.byref(st)))
    f1.record(stream)
    f1.synchronize()
    e2e_s = f0.elapsed_time(f1) / 1000.0 / args.steps
    text_head = bytes(host[:32].tolist()).decode(errors="replace")

    # max over ranks
    dev_s, e2e_s = max_over_ranks([dev_s, e2e_s], dist, device="cuda")

    kstats = [{"name": s.name.decode(), "launches": int(s.launches), "seconds": s.seconds,
               "bytes": s.bytes} for s in stats[: min(n.value, 32)]]
    for k in kstats:
        k["launches"] //= args.steps
        k["seconds"] /= args.steps
        k["bytes"] /= args.steps
    peak, peak_kind = measured_peaks()
    top = max(kstats, key=lambda k: k["seconds"])
    achieved = top["bytes"] / top["seconds"] / 1e9 if top["seconds"] > 0 else 0.0
    total_k = sum(k["seconds"] for k in kstats) or 1.0
    # DRAM bytes per algorithmic byte of the NTT passes, from one ncu capture of
    # the 2^23-word three-prime product (dram__bytes_read.sum +
    # dram__bytes_write.sum over 16 B per point): the row pass moves 14.9 B per
    # point, the column pass 30.8 B (data plus its twiddle table); both are per
    # point, so they scale to a launch of any size.
    dram_per_alg = {"ntt_rows": 14.9 / 16.0, "ntt_cols": 30.8 / 16.0}
    avg_bytes = top["bytes"] / max(top["launches"], 1)
    traffic = avg_bytes * dram_per_alg[top["name"]] if top["name"] in dram_per_alg else None
    roofline = {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_basis": "ncu DRAM bytes per point of the 2^23-word product, scaled "
                                                     "to the kernel's average launch",
                "launches": top["launches"],
                "avg_launch_ms": 1e3 * top["seconds"] / max(top["launches"], 1),
                "share_of_kernel_time": top["seconds"] / total_k,
                "measured": "CUDA events around every launch of the kernel, over K extra profiled steps"}

    # The integer roofline of the same passes: butterflies per second of the
    # row pass on the 2^23-word three-prime product against the register-only
    # butterfly rate of this GPU (pic_measure_butterfly_rate).
    int_roofline = None
    if rank == 0:
        int_roofline = int_roof(P, torch, L, stream)

    plain = None
    if not args.no_plain and rank == 0:
        def one(f):
            h = C.c_void_p()
            st2 = P.PiStats()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            P.check(L.pic_pi_compute(args.plain_digits, f, C.byref(h), C.byref(st2)))
            L.pic_bf_free(h)
            return time.perf_counter() - t0, st2.seconds_total, st2.kernel_launches
        one(P.PI_CHOSEN)
        c_wall, c_dev, c_l = one(P.PI_CHOSEN)
        p_wall, p_dev, p_l = one(P.PI_PLAIN)
        plain = {"digits": args.plain_digits, "chosen_s": c_wall, "plain_s": p_wall,
                 "speedup": p_wall / c_wall, "chosen_launches": c_l, "plain_launches": p_l}

    batch = None
    if not args.no_batch and rank == 0:
        batch = batched_products(P, torch, L, stream)

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        from oracle.ffi import REF_PI
        if os.path.exists(REF_PI):
            threads = os.cpu_count() or 1
            sample = min(args.ref_sample, args.digits)
            est, t_big, t_small, expo = cpu_reference_estimate(args.digits, sample, threads)
            cpu = {"value": est, "unit": "s", "cores": threads, "kind": "reference",
                   "sample": f"reference Pi() at {sample} digits ({t_big:.2f} s), scaled to {args.digits} "
                             f"digits with exponent {expo:.3f} fitted against {sample // 10} digits "
                             f"({t_small:.2f} s)"}

    if rank == 0:
        mean_phase = {k: statistics.mean(p[k] for p in phases)
                      for k in ("seconds_bsr", "seconds_div", "seconds_invsqrt", "seconds_final_mul")}
        mean_phase["step_seconds"] = [[round(p[k], 4) for k in ("seconds_total", "seconds_bsr", "seconds_div",
                                                                 "seconds_invsqrt", "seconds_final_mul")]
                                      for p in phases]
        line = {
            "metric": METRIC, "value": dev_s, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s * 1000.0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"pi_{args.digits:.0e}_digits", "digits": args.digits,
                       "hex_digits": hexd, "p_words": pw, "terms": terms, "form": args.form,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set larger than L2 (126 MB) in the dominant products"},
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(outlen.value), "text_head": text_head},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "int_roofline": int_roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
            "plain_vs_chosen": plain,
            "batched_products": batch,
            "phases": mean_phase,
            "kernels": kstats,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
