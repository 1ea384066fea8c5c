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
built from the reference sources) on this host's cores instead.  The first
warm-up step is a whole reference run at 10^8 digits, measured; every other
step is a bounded run at --ref-sample digits.  The 10^9 value is the measured
10^8 time on this host times the ratio of the reference's own 10^9 and 10^8
runs (both measured, same program and thread count, recorded in
tests/golden/reference_golden.json).  Power laws fitted between two smaller
sizes underestimate that ratio: the reference switches from its FFT to its
much slower NTT only near 10^8 digits (BigFloat.cpp:386).

--gpus N without a torchrun environment re-launches this script under
torch.distributed.run with N processes (one per GPU, independent replicas).
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
    ap.add_argument("--impl", choices=["ours", "reference", "replica-check"], default="ours",
                    help="replica-check: the launcher's self-test (no GPU, gloo ranks, no computation)")
    ap.add_argument("--plain-digits", type=int, default=1_000_000,
                    help="size at which the plain per-product form is timed beside the chosen form")
    ap.add_argument("--ref-sample", type=int, default=10_000_000)
    ap.add_argument("--ref-calibration", type=int, default=100_000_000,
                    help="size of the reference arm's measured calibration run")
    ap.add_argument("--no-isolated", action="store_true")
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


def run_reference_pi(digits: int, threads: int, with_tables: bool = False):
    """Seconds of one reference Pi() run (its own timer, table construction
    excluded); with_tables: (pi seconds, table seconds)."""
    from oracle.ffi import REF_PI
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([REF_PI, str(digits), str(threads)], cwd=d, capture_output=True, text=True,
                           check=True)
    rec = json.loads(r.stderr.strip().splitlines()[-1])
    return (float(rec["pi_s"]), float(rec["tables_s"])) if with_tables else float(rec["pi_s"])


def golden_pi():
    return json.load(open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")))["pi"]


def reference_ratio(hi: int, lo: int):
    """t(hi) / t(lo) of two whole reference runs at the same thread count,
    measured when the golden fixtures were generated (None if either is
    missing)."""
    g = golden_pi()
    a, b = g.get(str(hi)), g.get(str(lo))
    if not a or not b or "ref_seconds" not in a or "ref_seconds" not in b or a.get("threads") != b.get("threads"):
        return None
    return a["ref_seconds"] / b["ref_seconds"], a["threads"], a["ref_seconds"], b["ref_seconds"]


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
def reference_small_configs(threads: int) -> dict:
    """The reference program at its CPU-runnable configurations, on all host
    threads and on one: Pi() to 10^6 digits (its own timer, tables excluded;
    the table construction reported beside it) and isolated products BigFloat::mul(x, 0) of 2^12 / 2^16 / 2^20-word
    splitmix64 operands (seeds 42 and 43, the operands of the GPU arm's
    isolated products; best of three, one run at 2^20)."""
    from oracle.ffi import BF, REF_SO, Reference, random_words
    counts = sorted({1, threads})
    out = {"pi_1e6_s": {}, "pi_1e6_tables_s": {}}
    for th in counts:
        out["pi_1e6_s"][str(th)], out["pi_1e6_tables_s"][str(th)] = run_reference_pi(1_000_000, th, True)
    if os.path.exists(REF_SO):
        ref = Reference()
        prods = {}
        for lg in (12, 16, 20):
            a = BF(True, 0, random_words(42, 1 << lg))
            b = BF(True, 0, random_words(43, 1 << lg))
            row = {}
            for th in counts:
                best = float("inf")
                for _ in range(3 if lg < 20 else 1):
                    t0 = time.perf_counter()
                    ref.mul(a, b, 0, th)
                    best = min(best, time.perf_counter() - t0)
                row[str(th)] = best
            prods[str(lg)] = row
        out["isolated_products_s"] = prods
    out["unit"] = "s, keyed by host thread count"
    return out


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
    sample, calib = args.ref_sample, args.ref_calibration
    ratio = reference_ratio(args.digits, calib)
    times, t_calib = [], None
    for i in range(args.warmup + args.steps):
        if i == 0 and ratio is not None and calib != args.digits:
            t_calib = run_reference_pi(calib, threads)  # warm-up 0: the measured calibration run
            continue
        t = run_reference_pi(sample, threads)
        if i >= args.warmup:
            times.append(t)
    t_step = statistics.mean(times)
    if t_calib is not None:
        # value = t(calib) on this host x t_ref(digits) / t_ref(calib)
        value = t_calib * ratio[0]
        basis = (f"reference Pi() measured here at {calib} digits ({t_calib:.1f} s, {threads} threads) x "
                 f"{ratio[0]:.2f}, the ratio of the reference's own {args.digits}- and {calib}-digit runs "
                 f"({ratio[2]:.0f} s / {ratio[3]:.1f} s at {ratio[1]} threads, golden fixtures); timed steps "
                 f"are {sample}-digit runs ({t_step:.2f} s mean)")
    else:
        value = t_step * (args.digits / sample)
        basis = f"reference Pi() at {sample} digits per step, scaled linearly to {args.digits} digits"
    try:
        small = reference_small_configs(threads)
    except Exception as e:  # a reported baseline only: the line still prints
        small = {"error": f"{type(e).__name__}: {e}"}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1000.0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": f"pi_{args.digits:.0e}_digits", "digits": args.digits,
                                        "parallelism": "replicas"},
        "measured": {f"pi_{sample:.0e}_s": t_step, f"pi_{calib:.0e}_s": t_calib, "threads": threads},
        "cpu_runnable_configs": small,
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                         "sample": basis},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def replica_check(args):
    """The multi-process launcher's self-test: every rank joins a gloo group
    on 127.0.0.1, times a fixed amount of host work and rank 0 prints the
    bench line with n_gpus = the number of ranks and the max over ranks."""
    import datetime

    import torch.distributed as dist
    rank, _, world = rank_info()
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t0 = time.perf_counter()
    acc = 0
    for i in range(200_000 * (rank + 1)):
        acc += i * i
    dt = time.perf_counter() - t0
    (worst,) = max_over_ranks([dt], dist if world > 1 else None)
    if rank == 0:
        print(json.dumps({"impl": "replica-check", "metric": METRIC, "value": worst, "unit": "s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "per_rank_max_of": world}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def arith_roof(P, torch, L, stream):
    """Row-pass butterflies per second on a three-prime product of two
    0.8 * 2^23-word operands in the active form (a plain transform of length
    2^23 in both forms; 3 row passes per product, each over 3 x 2^23 points
    and row_bits levels) against the register-only butterfly ceiling of that
    form's arithmetic."""
    import ctypes as C

    form = P.get_tuning(P.TUNE_NTT_FORM)
    mode = "ntt3d" if form == P.FORM_DBL else "ntt3"
    k = 23
    n = int(0.8 * (1 << k))
    row_bits = P.get_ntt_geometry(k, form)[0]
    a = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda")
    b = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda")
    z = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    for _ in range(2):
        P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, mode)
    torch.cuda.synchronize()
    P.check(L.pic_profile_begin())
    reps = 5
    for _ in range(reps):
        P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, mode)
    stats = (P.KernelStat * 32)()
    cnt = C.c_int()
    P.check(L.pic_profile_end(stats, 32, C.byref(cnt)))
    rows = [s for s in stats[: cnt.value] if s.name.decode() == "ntt_rows"]
    if not rows or rows[0].seconds <= 0:
        return None
    bfly = rows[0].launches * 3 * (1 << (k - 1)) * row_bits
    achieved = bfly / rows[0].seconds / 1e9
    ceiling = P.butterfly_rate(form)
    basis = ("FP64 modular DIF butterflies (about nine FP64 instructions each)" if form == P.FORM_DBL
             else "lazy Shoup DIF butterflies") + " with operands in registers, no memory traffic"
    return {"kernel": "ntt_rows", "form": "fp64" if form == P.FORM_DBL else "integer",
            "workload": f"three-prime product of two {n}-word operands (transform length 2^{k})",
            "row_bits": row_bits, "achieved": achieved, "ceiling": ceiling, "unit": "G butterflies/s",
            "frac": achieved / ceiling, "ceiling_basis": basis}


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


def transform_bits(coefs: int, per_max: int) -> list:
    """Transform lengths (log2) of one three-prime product with `coefs`
    coefficients and operands of at most per_max pieces: one of 2^k, or the
    wrapped form's main 2^(k-1) and tail 2^kt (the rule of mul_ntt3 and
    mul_ntt3d with wrapped products on)."""
    k = max(1, (coefs - 1).bit_length())
    if k >= 4:
        nm = 1 << (k - 1)
        if per_max <= nm < coefs:
            kt = max(2, (2 * (coefs - nm) - 2).bit_length())
            if (1 << kt) <= nm // 2:
                return [k - 1, kt]
    return [k]


def isolated_products(P, torch, L, stream):
    """The isolated-multiply workload: two N-limb operands (splitmix64 seeds 42
    and 43), N = 2^12 ... 2^27, exact three-prime NTT product in both forms
    (integer and FP64) through pic_mul (inputs resident in HBM), its words
    checked against the reference's md5;
    where a proven FP64 piece width exists, the FFT product's time and its
    largest rounding distance.  B_mul = bytes of the transforms (two forward,
    one inverse; 16 B per point and pass, three primes) + 4 (na + nb + nz)."""
    import hashlib

    import numpy as np

    from oracle.ffi import random_words
    gold = {r["log2n"]: r for r in json.load(open(os.path.join(
        ROOT, "tests", "golden", "reference_golden.json")))["products"]["isolated"]}
    out = []
    for lg in (12, 16, 20, 24, 27):
        n = 1 << lg
        a = torch.from_numpy(random_words(42, n).view(np.int32)).cuda()
        b = torch.from_numpy(random_words(43, n).view(np.int32)).cuda()
        z = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        rec = {"log2n": lg}
        for mode in ("ntt3", "ntt3d", "fft"):
            if mode == "fft" and lg > 20:
                continue
            P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, mode)
            torch.cuda.synchronize()
            reps = 20 if lg <= 20 else 3
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, mode)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            w = z.cpu().numpy().view(np.uint32)
            L_ = w.size - (1 if w[-1] == 0 else 0)
            ok = hashlib.md5(w[:L_].tobytes()).hexdigest() == gold[lg]["md5"] if lg in gold else None
            rec[mode] = {"ms": ms, "matches_reference": ok}
            if mode in ("ntt3", "ntt3d"):
                # coefficients of the product: 64-bit pieces, or 56-bit in the FP64 form
                per = n // 2 if mode == "ntt3" else -(-32 * n // 56)
                form = P.FORM_DBL if mode == "ntt3d" else P.FORM_INT
                b_mul = 4.0 * 4 * n
                for k in transform_bits(2 * per - 1, per):
                    # passes of the tuned geometry: one up to 2^13 points, else
                    # ceil((k - row bits) / 11) column passes and the row pass
                    passes = 1 if k <= 13 else 1 + -(-(k - P.get_ntt_geometry(k, form)[0]) // 11)
                    b_mul += 3 * 3 * passes * 16.0 * (1 << k)
                rec[mode]["B_mul_GB"] = b_mul / 1e9
                rec[mode]["GBps"] = b_mul / (ms * 1e-3) / 1e9
            else:
                rec[mode]["max_err"] = L.pic_fft_last_max_err()
        out.append(rec)
        del a, b, z
    torch.cuda.empty_cache()
    return out


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
    # after the timed region: the text of the last step against the reference's pi.txt
    digits_check = None
    if rank == 0:
        import hashlib
        md5 = hashlib.md5(host[: outlen.value].numpy().tobytes()).hexdigest()
        g = golden_pi().get(str(args.digits))
        digits_check = {"md5": md5, "reference_md5": g["md5"] if g else None,
                        "matches_reference": (md5 == g["md5"]) if g else None}

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
    # DRAM bytes per algorithmic byte (16 B per point and pass) of the NTT
    # passes: dram__bytes_read.sum + dram__bytes_write.sum of every launch of
    # the kernel in one 1e9-digit computation (ncu, one pass per launch), over
    # the kernel's algorithmic bytes in the same computation.  FP64 form: rows
    # 1591.5 GB / 1739.5 GB, columns 1786.5 GB / 1763.6 GB (their per-point
    # twiddle tables mostly hit L2).  Integer form, from the 2^23-word product:
    # rows 14.9 B and columns 30.8 B per point.
    if P.get_tuning(P.TUNE_NTT_FORM) == P.FORM_DBL:
        dram_per_alg = {"ntt_rows": 1591.5 / 1739.5, "ntt_cols": 1786.5 / 1763.6}
        traffic_basis = ("ncu DRAM bytes of every launch of the kernel in one 1e9-digit computation over its "
                         "algorithmic bytes, times the kernel's average launch")
    else:
        dram_per_alg = {"ntt_rows": 14.9 / 16.0, "ntt_cols": 30.8 / 16.0}
        traffic_basis = "ncu DRAM bytes per point of the 2^23-word product, scaled to the kernel's average launch"
    avg_bytes = top["bytes"] / max(top["launches"], 1)
    traffic = avg_bytes * dram_per_alg[top["name"]] if top["name"] in dram_per_alg else None
    roofline = {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_basis": traffic_basis,
                "launches": top["launches"],
                "avg_launch_ms": 1e3 * top["seconds"] / max(top["launches"], 1),
                "share_of_kernel_time": top["seconds"] / total_k,
                "measured": "CUDA events around every launch of the kernel, over K extra profiled steps"}

    # The arithmetic roofline of the same passes: butterflies per second of
    # the row pass on a 2^23-point three-prime product in the active form
    # against the register-only butterfly rate of that arithmetic
    # (pic_measure_butterfly_rate_form).
    arith_roofline = None
    if rank == 0:
        arith_roofline = arith_roof(P, torch, L, stream)

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
                 "speedup": p_wall / c_wall, "chosen_launches": c_l, "plain_launches": p_l,
                 "plain_form": "the reference's recursion node by node, every product one three-prime NTT "
                               "launch sequence (pic_mul, NTT3), leaves by scalar multiplies"}

    batch = None
    if not args.no_batch and rank == 0:
        batch = batched_products(P, torch, L, stream)

    iso = None
    if not args.no_isolated and rank == 0:
        iso = isolated_products(P, torch, L, stream)

    # the two product forms of the same computation, cross-checked: NTT only,
    # and precision-selected (FP64 FFT for products up to 4 M words where its
    # proven piece width allows, NTT recompute past a rounding distance of 0.25)
    forms = None
    if rank == 0:
        import hashlib
        saved = P.get_tuning(P.TUNE_MUL_FFT_MAX)
        forms = {}
        try:
            for name, fmax in (("ntt_only", 0), ("precision_selected", 1 << 22)):
                P.set_tuning(P.TUNE_MUL_FFT_MAX, fmax)
                text, st2 = P.pi_hex(args.digits, form)
                forms[name] = {"md5": hashlib.md5(text).hexdigest(), "seconds": st2["seconds_total"],
                               "fft_max_err": st2["fft_max_err"], "fft_recomputes": st2["fft_recomputes"],
                               "products": st2["products"]}
                del text
        finally:
            P.set_tuning(P.TUNE_MUL_FFT_MAX, saved)
        forms["equal"] = forms["ntt_only"]["md5"] == forms["precision_selected"]["md5"]

    # the GPU's time at 10^8 digits, beside the reference arm's measured 10^8 run
    pi_1e8 = None
    if rank == 0 and args.digits > 100_000_000:
        h = C.c_void_p()
        st2 = P.PiStats()
        for _ in range(2):
            P.check(L.pic_pi_compute(100_000_000, P.PI_CHOSEN, C.byref(h), C.byref(st2)))
            L.pic_bf_free(h)
        pi_1e8 = st2.seconds_total

    cpu = None
    like = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        from oracle.ffi import REF_PI
        sample = min(args.ref_sample, args.digits)
        ratio = reference_ratio(args.digits, sample)
        if os.path.exists(REF_PI):
            threads = os.cpu_count() or 1
            # the GPU's own time on the same sample, for a measured ratio,
            # taken while the GPU is still busy from the runs above (after the
            # seconds of CPU-only work below its first runs were 2-7x slower)
            gpu_runs = []
            for _ in range(6):  # the first run at a new size builds its tables
                h = C.c_void_p()
                st2 = P.PiStats()
                P.check(L.pic_pi_compute(sample, P.PI_CHOSEN, C.byref(h), C.byref(st2)))
                L.pic_bf_free(h)
                gpu_runs.append(st2.seconds_total)
            gpu_s = min(gpu_runs[1:])
            t_ref = run_reference_pi(sample, threads)
            like = {"digits": sample, "reference_s": t_ref, "reference_threads": threads,
                    "gpu_s": gpu_s, "gpu_runs_s": gpu_runs, "ratio": t_ref / gpu_s}
            if ratio is not None:
                est = t_ref * ratio[0]
                basis = (f"reference Pi() measured here at {sample} digits ({t_ref:.2f} s) x {ratio[0]:.1f}, "
                         f"the ratio of the reference's own {args.digits}- and {sample}-digit runs "
                         f"({ratio[2]:.0f} s / {ratio[3]:.1f} s at {ratio[1]} threads, golden fixtures)")
            else:
                est = t_ref * args.digits / sample
                basis = f"reference Pi() measured here at {sample} digits, scaled linearly"
            cpu = {"value": est, "unit": "s", "cores": threads, "kind": "reference", "sample": basis}

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
            "digits_check": digits_check,
            "gpu_launches": int(launches),
            "roofline": roofline,
            "arith_roofline": arith_roofline,
            "cpu_baseline": cpu,
            "measured_vs_reference": like,
            "pi_1e8_s": pi_1e8,
            "clocks": clk,
            "plain_vs_chosen": plain,
            "batched_products": batch,
            "isolated_products": iso,
            "forms": forms,
            "phases": mean_phase,
            "kernels": kstats,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def relaunch(args) -> int:
    """--gpus N > 1 outside torchrun: N replicas under torch.distributed.run
    on 127.0.0.1, each rank on its own GPU; rank 0 prints the line."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args))
    _, _, world = rank_info()
    if args.gpus != world:
        raise SystemExit(f"--gpus {args.gpus} but {world} ranks were launched")
    if args.impl == "reference":
        reference_arm(args)
    elif args.impl == "replica-check":
        replica_check(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
