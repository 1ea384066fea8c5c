"""Command-line driver for the B200 engine.

    python -m piculator_b200.cli pi  --digits 1e9 [--repeat 2] [--form chosen|plain] [--out pi.txt]
                                     [--tuning FILE]
    python -m piculator_b200.cli mul --words 8388608 [--mode ntt3] [--repeat 3]
    torchrun --nproc-per-node N -m piculator_b200.cli pi --digits 1e9 --distributed

`pi --distributed` (under torchrun, one process per GPU, NCCL) splits the
binary splitting over the ranks (piculator_b200/shard.py); rank 0 prints the
line and writes the text.

`pi` runs the reference's Pi() (PI.h:138-212) on the GPU: it prints one JSON
line of phase times per run and, with --out, writes the same pi.txt text the
reference writes.  `mul` multiplies two splitmix64 operands of the given
length (the isolated-multiply workload) and prints the device time per
product.  Both are also the fixed commands the profiles in this repository
were captured with.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import time

import numpy as np

import piculator_b200 as P


def _splitmix_words(seed: int, n: int) -> np.ndarray:
    x = np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)
    z = x.copy()
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    z = z ^ (z >> np.uint64(31))
    return (z & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def cmd_pi(args) -> None:
    form = P.PI_CHOSEN if args.form == "chosen" else P.PI_PLAIN
    digits = int(float(args.digits))
    for r in range(args.repeat):
        t0 = time.perf_counter()
        text, st = P.pi_hex(digits, form, want_text=args.out is not None or args.md5)
        wall = time.perf_counter() - t0
        line = {"run": r, "digits": digits, "form": args.form, "wall_s": round(wall, 4),
                **{k: (round(v, 4) if isinstance(v, float) else v) for k, v in st.items()}}
        if args.md5 and text is not None:
            line["md5"] = hashlib.md5(text).hexdigest()
        print(json.dumps(line), flush=True)
    if args.out and text is not None:
        with open(args.out, "wb") as f:
            f.write(text)


def cmd_pi_distributed(args) -> None:
    import datetime
    import os

    import torch
    import torch.distributed as dist

    from piculator_b200.shard import DeviceBackend, pi_distributed
    digits = int(float(args.digits))
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        for r in range(args.repeat):
            dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            text = pi_distributed(DeviceBackend(), dist, digits, P.pi_sizes)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            dist.barrier()
            if dist.get_rank() == 0:
                line = {"run": r, "digits": digits, "ranks": dist.get_world_size(), "wall_s": round(wall, 4)}
                if args.md5:
                    line["md5"] = hashlib.md5(text).hexdigest()
                print(json.dumps(line), flush=True)
                if args.out:
                    with open(args.out, "wb") as f:
                        f.write(text)
    finally:
        dist.destroy_process_group()


def cmd_mul(args) -> None:
    import torch

    n = int(float(args.words))
    a = torch.from_numpy(_splitmix_words(42, n).view(np.int32)).cuda()
    b = torch.from_numpy(_splitmix_words(43, n).view(np.int32)).cuda()
    z = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.ExternalStream(P.lib().pic_default_stream())
    P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, args.mode)  # warm-up (tables)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.repeat):
        P.mul_dev(z.data_ptr(), a.data_ptr(), n, b.data_ptr(), n, args.mode)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.repeat
    print(json.dumps({"words": n, "mode": args.mode, "repeat": args.repeat, "ms_per_product": round(ms, 4),
                      "md5": hashlib.md5(z.cpu().numpy().tobytes()).hexdigest()}), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(prog="python -m piculator_b200.cli")
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("pi", help="compute pi in hex (the reference's Pi())")
    p.add_argument("--digits", default="1e6")
    p.add_argument("--repeat", type=int, default=1)
    p.add_argument("--form", choices=("chosen", "plain"), default="chosen")
    p.add_argument("--out", default=None, help="write the pi.txt text here")
    p.add_argument("--md5", action="store_true", help="print the md5 of the text")
    p.add_argument("--tuning", default=None, help="a tuning file applied over the default one")
    p.add_argument("--distributed", action="store_true",
                   help="split the binary splitting over the torchrun ranks (one GPU each)")
    m = sub.add_parser("mul", help="time an isolated product of two splitmix64 operands")
    m.add_argument("--words", default="8388608")
    m.add_argument("--mode", default="ntt3", choices=("auto", "school", "ntt3", "ntt3d", "fft", "ntt_ref"))
    m.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    import os
    local = int(os.environ.get("LOCAL_RANK", 0))
    if getattr(args, "distributed", False):
        import torch
        torch.cuda.set_device(local)
    P.init(local)
    if getattr(args, "tuning", None):
        P.apply_tuning(args.tuning)
    if args.cmd == "pi" and args.distributed:
        cmd_pi_distributed(args)
    elif args.cmd == "pi":
        cmd_pi(args)
    else:
        cmd_mul(args)


if __name__ == "__main__":
    main()
