"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

Run in a checkout where oracle/_ref was built from the reference sources
(``make -C oracle ref``).  Every number below comes out of the reference's own
code: its Pi() driver (oracle/_ref/picref_pi, PI.h:138-212) for pi.txt, its
BigFloat methods (BigFloat.cpp) and NNT class (NTT.cpp) through
oracle/_ref/libpicref.so for the rest.  Inputs are seeded splitmix64 streams,
so the fixtures can be regenerated bit for bit:

    python tests/golden/make_golden.py [--big] [--odd]

--big adds the 10M- and 100M-digit pi runs (minutes of CPU); --huge also the
1e9-digit run (about two hours on 8 cores; its entry keeps the thread count
and time of the run that produced it); --odd the 3,141,593- and
27,182,818-digit runs.  Entries already in the file for sizes not generated
this time are kept.

    python tests/golden/make_golden.py --big-products

only adds the isolated products of 2^24 and 2^27 words (the reference's NTT
at k = 27 and k = 30; about 26 GB of host memory and several minutes for
2^27) to the existing file, leaving every other entry as it is;

    python tests/golden/make_golden.py --dec

only adds the decimal-output fixtures: BigFloat::to_string_dec
(BigFloat.cpp:83-94) of splitmix64 numbers and edge cases, and of Pi()'s
final number at 10^4 .. 10^6 digits (oracle/_ref/picref_dec).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.ffi import REF_PI, BF, Reference, random_words, splitmix64_np  # noqa: E402

REF_DEC = os.path.join(os.path.dirname(REF_PI), "picref_dec")


def md5(b: bytes) -> str:
    return hashlib.md5(b).hexdigest()


def words_md5(w: np.ndarray) -> str:
    return md5(np.ascontiguousarray(w, dtype="<u4").tobytes())


def run_pi(digits: int, threads: int) -> tuple[bytes, dict]:
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([REF_PI, str(digits), str(threads)], cwd=d, capture_output=True, text=True,
                           check=True)
        data = open(os.path.join(d, "pi.txt"), "rb").read()
        timing = json.loads(r.stderr.strip().splitlines()[-1])
    return data, timing


def gen_pi(big: bool, huge: bool = False, odd: bool = False) -> dict:
    out = {}
    sizes = [10_000, 100_000, 1_000_000] + ([10_000_000, 100_000_000] if big or huge else [])
    sizes += [1_000_000_000] if huge else []
    # sizes that are not powers of ten: other term counts, precisions and
    # top-level shapes of the binary splitting
    sizes += [3_141_593, 27_182_818] if odd else []
    for d in sizes:
        data, t = run_pi(d, os.cpu_count() or 1)
        out[str(d)] = {"md5": md5(data), "bytes": len(data), "head": data[:80].decode(),
                       "tail": data[-80:].decode(), "ref_seconds": t["pi_s"], "threads": t["threads"]}
        print(f"pi {d}: {out[str(d)]['md5']} ({t['pi_s']:.2f} s)", flush=True)
    return out


def gen_products(ref: Reference) -> dict:
    """Exact products through BigFloat::mul(x, 0) (BigFloat.cpp:326-444)."""
    cases = {}
    # small explicit cases: words stored in the fixture
    small = []
    seed = 1000
    for na, nb in [(1, 1), (1, 2), (2, 1), (3, 5), (7, 7), (16, 1), (1, 33), (31, 64), (100, 3),
                   (128, 128), (255, 257), (500, 700), (1024, 1024), (2048, 2047), (4095, 1)]:
        a = random_words(seed, na)
        b = random_words(seed + 1, nb)
        a[-1] |= 1
        b[-1] |= 1
        z = ref.mul(BF(True, 0, a), BF(True, 0, b))
        small.append({"seed_a": seed, "seed_b": seed + 1, "na": na, "nb": nb,
                      "z": z.words.tolist(), "L": z.L})
        seed += 2
    cases["small"] = small
    # all-ones / sparse / power-of-two edge operands
    edge = []
    for n in [1, 2, 3, 64, 1000, 4096]:
        ones = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
        z = ref.mul(BF(True, 0, ones), BF(True, 0, ones))
        edge.append({"kind": "ones", "n": n, "md5": words_md5(z.words), "L": z.L})
        sp = np.zeros(n, dtype=np.uint32)
        sp[-1] = 1
        sp[0] = 1
        z = ref.mul(BF(True, 0, sp), BF(True, 0, ones))
        edge.append({"kind": "sparse_x_ones", "n": n, "md5": words_md5(z.words), "L": z.L})
    cases["edge"] = edge
    # isolated-multiply workload (splitmix64 seed 42 / 43, N limbs each): hashes
    iso = []
    for lg in [12, 16, 20]:
        n = 1 << lg
        a = random_words(42, n)
        b = random_words(43, n)
        z = ref.mul(BF(True, 0, a), BF(True, 0, b), 0, threads=os.cpu_count() or 1)
        iso.append({"log2n": lg, "md5": words_md5(z.words), "L": z.L, "top": int(z.words[-1])})
        print(f"product 2^{lg}: {iso[-1]['md5']}", flush=True)
    cases["isolated"] = iso
    return cases


def gen_big_products(ref: Reference) -> list:
    """BigFloat::mul(x, 0) of 2^24- and 2^27-word splitmix64 operands (seeds
    42 / 43): the reference's NTT path (BigFloat.cpp:416-441) at k = 27 and
    k = 30.  Stored as md5 of the product words, length and top word."""
    out = []
    for lg in [24, 27]:
        n = 1 << lg
        a = random_words(42, n)
        b = random_words(43, n)
        t0 = time.time()
        z = ref.mul(BF(True, 0, a), BF(True, 0, b), 0, threads=os.cpu_count() or 1)
        out.append({"log2n": lg, "md5": words_md5(z.words), "L": z.L, "top": int(z.words[-1]),
                    "ref_seconds": round(time.time() - t0, 2), "threads": os.cpu_count() or 1})
        print(f"product 2^{lg}: {out[-1]['md5']} ({out[-1]['ref_seconds']} s)", flush=True)
        del z
    return out


def ref_dec_words(sign: bool, exp: int, words: np.ndarray, digits: int) -> bytes:
    """to_string_dec(digits) of a BigFloat, by the reference program."""
    with tempfile.NamedTemporaryFile(suffix=".bf", delete=False) as f:
        f.write(np.array([1 if sign else 0], dtype="<i4").tobytes())
        f.write(np.array([exp], dtype="<i8").tobytes())
        f.write(np.array([words.size], dtype="<u8").tobytes())
        f.write(np.ascontiguousarray(words, dtype="<u4").tobytes())
        path = f.name
    try:
        return _ref_dec_run(["words", path, str(digits)])
    finally:
        os.unlink(path)


def _ref_dec_run(args) -> bytes:
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "dec.txt")
        subprocess.run([REF_DEC, *args, out], capture_output=True, check=True)
        return open(out, "rb").read()


def gen_dec() -> dict:
    """BigFloat::to_string_dec (BigFloat.cpp:83-94): the text for seeded and
    edge-case numbers, and md5 / head / tail for Pi()'s number."""
    cases = []
    specs = [(5, 0), (5, 1), (5, 8), (5, 9), (5, 10), (5, 100), (1, 30), (2, 9), (3, 50), (40, 300),
             (200, 1900), (1000, 9000), (2500, 25000), (20000, 190000)]
    for i, (L, digits) in enumerate(specs):
        w = random_words(7000 + i, L)
        w[-1] = (w[-1] % 7) + 1 if i % 3 else w[-1]  # one-char and multi-char integer parts
        text = ref_dec_words(True, -L + 1, w, digits)
        rec = {"seed": 7000 + i, "L": L, "digits": digits, "top_mod7": bool(i % 3)}
        if len(text) <= 4000:
            rec["text"] = text.decode()
        rec["md5"] = md5(text)
        rec["len"] = len(text)
        cases.append(rec)
    edge = []
    for name, w in [("ones", np.full(300, 0xFFFFFFFF, dtype=np.uint32)),
                    ("zeros_below_top", np.array([0] * 299 + [3], dtype=np.uint32)),
                    ("single_low_bit", np.array([1] + [0] * 298 + [3], dtype=np.uint32))]:
        text = ref_dec_words(True, 0, w, 3000)
        edge.append({"kind": name, "digits": 3000, "md5": md5(text), "len": len(text), "tail": text[-60:].decode()})
    pi = {}
    for d in (10_000, 100_000, 1_000_000):
        t0 = time.time()
        text = _ref_dec_run(["pi", str(d), str(os.cpu_count() or 1)])
        pi[str(d)] = {"md5": md5(text), "len": len(text), "head": text[:80].decode(), "tail": text[-80:].decode(),
                      "ref_seconds": round(time.time() - t0, 2)}
        print(f"pi dec {d}: {pi[str(d)]['md5']} ({pi[str(d)]['ref_seconds']} s)", flush=True)
    return {"numbers": cases, "edge": edge, "pi": pi}


def gen_ntt(ref: Reference) -> dict:
    """NNT::NTT / iNTT (NTT.cpp:74-84) outputs at k = 11..16."""
    out = []
    for k in range(11, 17):
        n = 1 << k
        d, p, g, w = ref.ntt(k, splitmix64_np(7 + k, n) % np.uint64(9223372036854675457))
        x0 = splitmix64_np(7 + k, n) % np.uint64(p)
        f, p2, _, _ = ref.ntt(k, x0)
        inv, _, _, wi = ref.ntt(k, f, inverse=True)
        out.append({"k": k, "p": p, "g": g, "w": w, "w_inv": wi, "input_seed": 7 + k,
                    "fwd_md5": words_md5(f.view(np.uint32)), "fwd_head": [int(v) for v in f[:8]],
                    "roundtrip_ok": bool(np.array_equal(inv, x0))})
    return {"nnt": out}


def gen_bigfloat(ref: Reference) -> dict:
    """add/sub/mul/rcp/div/invsqrt with truncation (BigFloat.cpp:184-568)."""
    rng = np.random.default_rng(2024)
    cases = []
    for i in range(60):
        na, nb = (int(x) for x in rng.integers(1, 40, 2))
        a = random_words(5000 + 2 * i, na)
        b = random_words(5001 + 2 * i, nb)
        a[-1] |= 1
        b[-1] |= 1
        A = BF(bool(rng.integers(2)), int(rng.integers(-6, 6)), a)
        B = BF(bool(rng.integers(2)), int(rng.integers(-6, 6)), b)
        p = int(rng.integers(0, 30))
        rec = {"a": [A.sign, A.exp, A.words.tolist()], "b": [B.sign, B.exp, B.words.tolist()], "p": p}
        for name in ("add", "sub", "mul"):
            z = getattr(ref, name)(A, B, p)
            rec[name] = [z.sign, z.exp, z.words.tolist()]
        z = ref.rcp(A, p)
        rec["rcp"] = [z.sign, z.exp, z.words.tolist()]
        z = ref.div(A, B, p)
        rec["div"] = [z.sign, z.exp, z.words.tolist()]
        s = int(a[0])
        z = ref.mul_u32(A, s)
        rec["mul_u32"] = [s, z.sign, z.exp, z.words.tolist()]
        cases.append(rec)
    inv = []
    for x in (2, 3, 10005, 4294967295):
        for p in (0, 1, 2, 5, 40, 300):
            z = ref.invsqrt(x, p)
            inv.append({"x": x, "p": p, "z": [z.sign, z.exp, z.words.tolist()]})
    # the carry-loss case of uadd: low words below the window are dropped
    # before adding, so their carry is lost (BigFloat.cpp:222-224).
    A = BF(True, 0, np.array([0xFFFFFFFF, 0xFFFFFFFF, 5, 7], dtype=np.uint32))
    B = BF(True, 0, np.array([0x00000001, 0x00000001, 9], dtype=np.uint32))
    z = ref.add(A, B, 1)
    carry = {"a": [True, 0, A.words.tolist()], "b": [True, 0, B.words.tolist()], "p": 1,
             "add": [z.sign, z.exp, z.words.tolist()]}
    return {"ops": cases, "invsqrt": inv, "carry_loss": carry}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    ap.add_argument("--huge", action="store_true")
    ap.add_argument("--odd", action="store_true", help="also pi at 3,141,593 and 27,182,818 digits")
    ap.add_argument("--big-products", action="store_true",
                    help="only add the 2^24- and 2^27-word products to the existing file")
    ap.add_argument("--dec", action="store_true", help="only add the decimal-output fixtures")
    args = ap.parse_args()
    ref = Reference()
    path = os.path.join(HERE, "reference_golden.json")
    if args.dec:
        fixtures = json.load(open(path))
        fixtures["dec"] = gen_dec()
        json.dump(fixtures, open(path, "w"), indent=1, sort_keys=True)
        print("wrote", path)
        return
    if args.big_products:
        fixtures = json.load(open(path))
        big = gen_big_products(ref)
        iso = [e for e in fixtures["products"]["isolated"] if e["log2n"] not in (24, 27)]
        fixtures["products"]["isolated"] = sorted(iso + big, key=lambda e: e["log2n"])
        json.dump(fixtures, open(path, "w"), indent=1, sort_keys=True)
        print("wrote", path)
        return
    fixtures = {
        "pi": gen_pi(args.big, args.huge, args.odd),
        "products": gen_products(ref),
        "ntt": gen_ntt(ref),
        "bigfloat": gen_bigfloat(ref),
        "generator": "tests/golden/make_golden.py (reference compiled from its own sources)",
    }
    if os.path.exists(path):
        old = json.load(open(path))
        for d, v in old.get("pi", {}).items():
            fixtures["pi"].setdefault(d, v)
        fixtures["products"]["isolated"] += [e for e in old["products"]["isolated"]
                                             if e["log2n"] in (24, 27)]
        if "dec" in old:
            fixtures["dec"] = old["dec"]
    json.dump(fixtures, open(path, "w"), indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
