"""The C++ drop-in: the reference's own PI.h -- Pi() and Pi_BSR()
(PI.h:64-212), unmodified -- compiled against this library's pic::BigFloat
(oracle/Makefile target `dropin`, three stand-in headers in
oracle/dropin_shim/) writes the reference's pi.txt byte for byte.  Pi_BSR's
std::thread fork (PI.h:93-108) is active (threads > 1, more than 1000 terms),
so two host threads drive the library at the same time."""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import tempfile

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "picdropin_pi")


@pytest.mark.parametrize("digits,threads", [(10_000, 1), (100_000, 4), (1_000_000, 2)])
def test_reference_pi_h_on_pic_bigfloat(golden, digits, threads):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/picdropin_pi not built (the reference sources were absent at build time)")
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([DROPIN, str(digits), str(threads)], cwd=d, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        text = open(os.path.join(d, "pi.txt"), "rb").read()
    info = json.loads(r.stderr.strip().splitlines()[-1])
    assert info["threads"] == threads
    g = golden["pi"][str(digits)]
    assert len(text) == g["bytes"]
    assert hashlib.md5(text).hexdigest() == g["md5"]
