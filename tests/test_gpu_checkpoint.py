"""Checkpoint / resume of a pi computation: a run stopped right after the
checkpoint of phase 1 (binary splitting), 2 (division) or 3 (inverse square
root) -- as a crash there would stop it -- and resumed from the file gives the
reference's pi.txt byte for byte and skips the phases on disk.  A damaged
checkpoint is reported, never used.  The stop is a host-side hook; no GPU
fault is involved."""
from __future__ import annotations

import hashlib
import os

import pytest

pytestmark = pytest.mark.gpu

DIGITS = 1_000_000


@pytest.fixture()
def ckdir(pic, tmp_path):
    yield str(tmp_path)
    pic.lib().pic_debug_stop_after_phase(0)
    pic.set_checkpoint(None)


@pytest.mark.parametrize("phase", [1, 2, 3])
def test_stop_and_resume(pic, golden, ckdir, phase):
    pic.set_checkpoint(ckdir, pic.CKPT_WRITE)
    pic.lib().pic_debug_stop_after_phase(phase)
    with pytest.raises(pic.PicError) as e:
        pic.pi_hex(DIGITS, pic.PI_CHOSEN)
    assert e.value.status == pic.ERR_STOPPED
    path = os.path.join(ckdir, f"pi_{DIGITS}.ckpt")
    info = pic.checkpoint_inspect(path)
    assert info["phase"] == phase and info["digits"] == DIGITS
    pic.lib().pic_debug_stop_after_phase(0)
    pic.set_checkpoint(ckdir, pic.CKPT_RESUME)
    text, st = pic.pi_hex(DIGITS, pic.PI_CHOSEN)
    assert hashlib.md5(text).hexdigest() == golden["pi"][str(DIGITS)]["md5"]
    skipped = ["seconds_bsr", "seconds_div", "seconds_invsqrt"][:phase]
    for k in skipped:
        assert st[k] < 1e-3, (k, st[k])
    # every later phase ran
    assert st["seconds_final_mul"] > 0


def test_write_then_resume_every_phase_in_one_run(pic, golden, ckdir):
    pic.set_checkpoint(ckdir, pic.CKPT_WRITE | pic.CKPT_RESUME)
    text, _ = pic.pi_hex(DIGITS, pic.PI_CHOSEN)
    path = os.path.join(ckdir, f"pi_{DIGITS}.ckpt")
    assert pic.checkpoint_inspect(path)["phase"] == 3
    text2, st = pic.pi_hex(DIGITS, pic.PI_CHOSEN)  # resumes after phase 3
    assert text == text2
    assert hashlib.md5(text2).hexdigest() == golden["pi"][str(DIGITS)]["md5"]
    assert st["seconds_bsr"] < 1e-3


def test_damaged_checkpoint_is_rejected(pic, ckdir):
    pic.set_checkpoint(ckdir, pic.CKPT_WRITE)
    pic.lib().pic_debug_stop_after_phase(1)
    with pytest.raises(pic.PicError):
        pic.pi_hex(DIGITS, pic.PI_CHOSEN)
    pic.lib().pic_debug_stop_after_phase(0)
    path = os.path.join(ckdir, f"pi_{DIGITS}.ckpt")
    raw = bytearray(open(path, "rb").read())
    raw[len(raw) // 2] ^= 1
    open(path, "wb").write(bytes(raw))
    pic.set_checkpoint(ckdir, pic.CKPT_RESUME)
    with pytest.raises(pic.PicError) as e:
        pic.pi_hex(DIGITS, pic.PI_CHOSEN)
    assert e.value.status == pic.ERR_IO
