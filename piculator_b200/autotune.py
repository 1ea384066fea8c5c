"""Autotuner for the B200 engine: measures this GPU and writes tuning.json.

Size classes and what is chosen for each:
  * NTT transform length 2^k (k = 10..27): row-pass bits (11, 12, 13), radix
    of the register rounds (8 or 16) and column-tile width (automatic or
    4..32 columns), timed on three-prime products of that length; with
    --batched, the geometry of k = 14..27 is timed instead where the pi run
    uses it, on the batched merges of whole runs (one run per candidate,
    every merge level timed by stream-ordered events and attributed to its
    transform length);
  * single products by length: the form (schoolbook, three-prime NTT, FP64
    FFT, or the one-prime reference layout) -- i.e. the prime count and
    transform family -- as crossover thresholds;
  * binary splitting: the child length below which a level merges with the
    CTA schoolbook instead of batched NTTs, and the operand length from which
    that schoolbook takes a Karatsuba level, timed on whole 1e9-digit pi runs
    (--only-bsr reruns just this stage over an existing table).

    python -m piculator_b200.autotune [--quick] [--batched] [--out PATH]

`piculator_b200.init()` applies the file it finds next to this module.
Every candidate computes the same words (products are exact); only time
differs, measured with CUDA events on the library's stream.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import tempfile
import time

import numpy as np

import piculator_b200 as P

DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")


def _words(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)


class Timer:
    def __init__(self):
        import torch
        self.torch = torch
        self.stream = torch.cuda.ExternalStream(P.lib().pic_default_stream())

    def time(self, fn, reps: int = 3, warm: int = 1) -> float:
        for _ in range(warm):
            fn()
        e0 = self.torch.cuda.Event(enable_timing=True)
        e1 = self.torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(reps):
            fn()
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps


def tune_ntt(timer: Timer, ks, quick: bool) -> dict:
    torch = timer.torch
    out = {}
    for k in ks:
        n = 1 << k  # words per operand: the product fills 2^k three-prime points
        a = torch.from_numpy(_words(k, n).view(np.int32)).cuda()
        b = torch.from_numpy(_words(k + 100, n).view(np.int32)).cuda()
        z = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
        cands = []
        for rb in (3, 4):
            if k <= 13:
                # single-pass lengths keep the specialised radix-8 kernel: in
                # the binary-splitting merges it reads the child slots itself,
                # where the general kernels need a separate split first
                if rb == 3:
                    cands.append((12, 0, rb))
                continue
            for row in ((12,) if quick else (11, 12, 13)):
                for lw in ((0,) if quick else (0, 3, 5)):
                    cands.append((row, lw, rb))
        best = None
        for row, lw, rb in cands:
            P.set_ntt_geometry(k, row, lw, rb)
            try:
                ms = timer.time(lambda: P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, "ntt3"),
                                reps=2 if k >= 24 else 4)
            except P.PicError as e:  # a geometry this GPU cannot launch
                print(f"ntt k={k} {row}/{lw}/{rb}: skipped ({e})", flush=True)
                continue
            if best is None or ms < best[0]:
                best = (ms, row, lw, rb)
        P.set_ntt_geometry(k, best[1], best[2], best[3])
        out[str(k)] = {"row_bits": best[1], "col_width_log2": best[2], "radix_log2": best[3], "ms": best[0]}
        print(f"ntt k={k}: {out[str(k)]}", flush=True)
    return out


def _timeline_ms_by_k(stderr: str) -> dict:
    """Device ms per transform length from the last computation's timeline
    (the lines PIC_TIMELINE prints; the merges that end at a mark carry k)."""
    groups, cur = [], []
    for line in stderr.splitlines():
        line = line.strip()
        if not line.startswith("{"):
            continue
        d = json.loads(line)
        if "timeline" in d:
            cur.append(d)
        elif "timeline_alloc" in d:
            groups.append(cur)
            cur = []
    out: dict = {}
    for d in groups[-1] if groups else []:
        if "k" in d:
            out[d["k"]] = out.get(d["k"], 0.0) + d["ms"]
    return out


def tune_ntt_batched(digits: int, ks=range(14, 28), radices=(3, 4), form: int = P.FORM_INT,
                     rows=(11, 12, 13), pass_bits=(None,)) -> dict:
    """NTT geometry per length, timed on the batched merges of whole pi runs:
    each candidate is applied to every length at once, the second of two runs
    is timed, and each length takes the candidate whose merge levels of that
    length were fastest (a level's wrapped tail product, usually two lengths
    shorter, runs under the same candidate).  Radix 16 (radix_log2 4) applies
    to row passes of 2^11 .. 2^13 points and column passes of 2^8 .. 2^11
    rows; other passes stay radix 8.  With form FORM_DBL the runs use the
    FP64 product form and the geometry is that form's; pass_bits then lists
    the candidate FP64 pass-table limits (PIC_TUNE_DBL_PASS_TABLES), and the
    one with the fastest whole binary splitting is kept (returned under the
    key "dbl_pass_bits")."""
    import subprocess
    import sys
    import tempfile
    cands = [(row, lw, rb, pb) for row in rows for lw in (0, 3, 5) for rb in radices for pb in pass_bits]
    ms: dict = {}
    total: dict = {}
    env = dict(os.environ, PIC_TIMELINE="1")
    key = "ntt_fp64" if form == P.FORM_DBL else "ntt"
    for row, lw, rb, pb in cands:
        geo = {str(k): {"row_bits": row if k > 13 or form == P.FORM_INT else 12, "col_width_log2": lw,
                        "radix_log2": rb} for k in ks}
        tab = {key: geo}
        if form == P.FORM_DBL:
            tab["products"] = {"ntt_form": 1}
            if pb is not None:
                tab["products"]["dbl_pass_bits"] = pb
        with tempfile.NamedTemporaryFile("w", suffix=".json", delete=False) as f:
            json.dump(tab, f)
            path = f.name
        try:
            r = subprocess.run([sys.executable, "-m", "piculator_b200.cli", "pi", "--digits", str(digits),
                                "--repeat", "2", "--tuning", path], env=env, capture_output=True, text=True,
                               check=True)
        finally:
            os.unlink(path)
        by_k = _timeline_ms_by_k(r.stderr)
        for k, v in by_k.items():
            ms.setdefault(pb, {}).setdefault(k, {})[(row, lw, rb)] = v
        total.setdefault(pb, {})[(row, lw, rb)] = sum(by_k.values())
        print(f"ntt batched {key} {row}/{lw}/{rb}/{pb}: { {k: round(v, 2) for k, v in sorted(by_k.items())} }",
              flush=True)
    # the pass-table limit whose best per-length choices sum lowest
    def best_sum(pb):
        return sum(min(by.values()) for k, by in ms[pb].items() if k in ks)
    pb = min(ms, key=best_sum)
    out = {}
    for k, by in sorted(ms[pb].items()):
        if k not in ks:
            continue
        (row, lw, rb), best = min(by.items(), key=lambda kv: kv[1])
        out[str(k)] = {"row_bits": row, "col_width_log2": lw, "radix_log2": rb, "ms_batched": best}
        P.set_ntt_geometry(k, row, lw, rb, form)
    if form == P.FORM_DBL and pb is not None:
        out["dbl_pass_bits"] = pb
    return out


def tune_products(timer: Timer) -> dict:
    torch = timer.torch
    rows = []
    for lg in range(4, 21):
        n = 1 << (lg - 1)
        a = torch.from_numpy(_words(lg, n).view(np.int32)).cuda()
        b = torch.from_numpy(_words(lg + 50, n).view(np.int32)).cuda()
        z = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
        row = {"words": 2 * n}
        for mode in ("school", "ntt3", "fft", "ntt_ref"):
            if mode == "school" and 2 * n > 4096:
                continue
            row[mode] = timer.time(lambda: P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, mode))
        rows.append(row)
        print(f"product {2 * n} words: { {k: round(v, 4) for k, v in row.items()} }", flush=True)
    school_max = 0
    fft_max = 0
    for r in rows:
        if "school" in r and r["school"] <= r["ntt3"]:
            school_max = r["words"]
        if r["fft"] < r["ntt3"] and r["words"] > school_max:
            fft_max = r["words"]
    return {"school_max_words": school_max, "fft_max_words": fft_max, "table": rows}


def tune_bsr(quick: bool) -> dict:
    """Schoolbook threshold of the binary-splitting merges and the Karatsuba
    level of the CTA schoolbook kernel, timed on whole pi runs at the headline
    size (the best threshold moves with the size).  Every candidate computes
    the same words."""
    digits = 10_000_000 if quick else 1_000_000_000
    res = {}
    P.pi_hex(digits, P.PI_CHOSEN, want_text=False)
    cands = [(thr, kara) for thr in (300, 450, 600, 900, 1400) for kara in (0, 48, 96, 192)]
    for thr, kara in cands:
        P.set_tuning(P.TUNE_BSR_SCHOOL_MAX, thr)
        P.set_tuning(P.TUNE_BSR_KARATSUBA, kara)
        best = None
        for _ in range(2):
            _, st = P.pi_hex(digits, P.PI_CHOSEN, want_text=False)
            best = st["seconds_bsr"] if best is None else min(best, st["seconds_bsr"])
        res[f"{thr}/{kara}"] = best
        print(f"bsr school threshold {thr}, Karatsuba from {kara}: {best:.4f} s", flush=True)
    key = min(res, key=res.get)
    thr, kara = (int(x) for x in key.split("/"))
    P.set_tuning(P.TUNE_BSR_SCHOOL_MAX, thr)
    P.set_tuning(P.TUNE_BSR_KARATSUBA, kara)
    return {"bsr_school_max_words": thr, "bsr_karatsuba_min_words": kara, "digits": digits,
            "seconds": res}


def _read_table(path: str) -> dict:
    with open(path) as f:
        return json.load(f)


def _write_table(path: str, result: dict) -> None:
    """Write the table beside its destination and rename it over it, so an
    interrupted run never leaves a truncated file for init() to load."""
    d = os.path.dirname(os.path.abspath(path))
    with tempfile.NamedTemporaryFile("w", suffix=".json", dir=d, delete=False) as f:
        json.dump(result, f, indent=1)
        tmp = f.name
    try:
        os.replace(tmp, path)
    except BaseException:
        os.unlink(tmp)
        raise
    print("wrote", path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--batched", action="store_true",
                    help="time the geometry of k >= 14 on the merges of whole pi runs")
    ap.add_argument("--only-batched", action="store_true",
                    help="rerun only the batched geometry stage over the table in --out")
    ap.add_argument("--only-bsr", action="store_true",
                    help="rerun only the binary-splitting thresholds over the table in --out")
    ap.add_argument("--only-fp64", action="store_true",
                    help="rerun only the FP64 form's batched geometry and pass-table limit over the table in --out")
    args = ap.parse_args()
    if args.only_fp64:
        P.init(0, tuned=True)
        result = _read_table(args.out)
        got = tune_ntt_batched(1_000_000_000, ks=range(10, 28), form=P.FORM_DBL, rows=(11, 12),
                               pass_bits=(20, 24))
        result.setdefault("products", {})["dbl_pass_bits"] = got.pop("dbl_pass_bits", 20)
        result["ntt_fp64"] = got
        _write_table(args.out, result)
        return
    if args.only_bsr:
        P.init(0, tuned=True)
        result = _read_table(args.out)
        P.apply_tuning(args.out)
        result["bsr"] = tune_bsr(False)
        _write_table(args.out, result)
        return
    if args.only_batched:
        P.init(0, tuned=True)
        result = _read_table(args.out)
        result["ntt"].update(tune_ntt_batched(1_000_000_000))
        _write_table(args.out, result)
        return
    P.init(0, tuned=False)
    timer = Timer()
    result = {"gpu": None}
    try:
        import torch
        result["gpu"] = torch.cuda.get_device_name(0)
    except Exception:
        pass
    result["ntt"] = tune_ntt(timer, range(10, 28) if not args.quick else (14, 18, 22, 24, 26), args.quick)
    if args.batched:
        result["ntt"].update(tune_ntt_batched(10_000_000 if args.quick else 1_000_000_000))
    prod = tune_products(timer)
    result["products"] = prod
    P.set_tuning(P.TUNE_MUL_SCHOOL_MAX, prod["school_max_words"])
    P.set_tuning(P.TUNE_MUL_FFT_MAX, prod["fft_max_words"])
    result["bsr"] = tune_bsr(args.quick)
    _write_table(args.out, result)


if __name__ == "__main__":
    main()
