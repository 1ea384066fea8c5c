"""Checkpoint files read on the host (no GPU): pic_checkpoint_inspect
accepts a well-formed file and rejects every damaged one with PIC_ERR_IO.
The files are written here byte for byte in the documented format
(piculator_b200/csrc/checkpoint.cu), so the format itself is pinned."""
from __future__ import annotations

import struct

import numpy as np
import pytest

import piculator_b200 as P

M64 = (1 << 64) - 1


def ckpt_hash(w: np.ndarray) -> int:
    h = 0x243F6A8885A308D3 ^ int(w.size)
    for x in w.tolist():
        h = ((h ^ x) * 0x9E3779B97F4A7C15) & M64
        h ^= h >> 29
    return h


def write_ckpt(path, digits=1000, p_words=93, terms=72, phase=1, numbers=None, magic=b"PICKPT01"):
    numbers = numbers if numbers is not None else [
        (True, -91, np.arange(1, 94, dtype=np.uint32)),
        (True, -90, np.arange(7, 99, dtype=np.uint32) * 3)]
    with open(path, "wb") as f:
        f.write(magic + struct.pack("<QQQII", digits, p_words, terms, phase, len(numbers)))
        for sign, exp, w in numbers:
            f.write(struct.pack("<iiqQQ", int(sign), 0, exp, w.size, ckpt_hash(w)))
        for _, _, w in numbers:
            f.write(w.astype("<u4").tobytes())


@pytest.fixture()
def ck(tmp_path):
    return str(tmp_path / "pi_1000.ckpt")


def test_inspect_valid(ck):
    write_ckpt(ck, phase=3)
    assert P.checkpoint_inspect(ck) == {"digits": 1000, "p_words": 93, "phase": 3}


def _expect_io(path, verify=True):
    with pytest.raises(P.PicError) as e:
        P.checkpoint_inspect(path, verify)
    assert e.value.status == P.ERR_IO
    return str(e.value)


def test_flipped_word_is_rejected(ck):
    write_ckpt(ck)
    raw = bytearray(open(ck, "rb").read())
    raw[-5] ^= 0x40
    open(ck, "wb").write(bytes(raw))
    assert "hash" in _expect_io(ck)
    # the header alone still reads without verification
    assert P.checkpoint_inspect(ck, verify=False)["phase"] == 1


@pytest.mark.parametrize("damage", ["magic", "truncated", "trailing", "phase", "count", "missing"])
def test_damaged_files_are_rejected(ck, damage):
    if damage == "magic":
        write_ckpt(ck, magic=b"PICKPT99")
    elif damage == "phase":
        write_ckpt(ck, phase=7)
    elif damage == "count":
        write_ckpt(ck, numbers=[])
    else:
        write_ckpt(ck)
        raw = open(ck, "rb").read()
        if damage == "truncated":
            open(ck, "wb").write(raw[:-9])
        elif damage == "trailing":
            open(ck, "wb").write(raw + b"\0")
        else:
            ck = ck + ".absent"
    _expect_io(ck)


def test_huge_length_field_is_rejected_before_any_allocation(ck):
    """A damaged length field (2^34 words, 64 GB) in a small file: the reader
    compares the lengths with the file's size first and never sizes a buffer
    from the field."""
    import struct as S
    w = np.arange(1, 94, dtype=np.uint32)
    with open(ck, "wb") as f:
        f.write(b"PICKPT01" + S.pack("<QQQII", 1000, 93, 72, 2, 1))
        f.write(S.pack("<iiqQQ", 1, 0, -91, 1 << 34, ckpt_hash(w)))
        f.write(w.astype("<u4").tobytes())
    assert "truncated" in _expect_io(ck)
