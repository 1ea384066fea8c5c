"""The C-ABI library: built, loadable, exports every symbol the header
declares, and reports errors as statuses (no GPU needed)."""
from __future__ import annotations

import ctypes
import os
import subprocess

import pytest

import piculator_b200 as P


def test_library_built_for_sm100a():
    assert os.path.exists(P.LIB_PATH), "run __graft_entry__.build()"
    out = subprocess.run(["cuobjdump", "--list-elf", P.LIB_PATH], capture_output=True, text=True)
    if out.returncode == 0:
        assert "sm_100a" in out.stdout


def test_every_declared_symbol_is_exported():
    names = P.declared_symbols()
    assert len(names) > 40
    L = ctypes.CDLL(P.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_primes(oracle):
    L = P.lib()
    assert L.pic_status_string(P.ERR_LENGTH) == b"FFT length is too small."
    assert L.pic_status_string(P.ERR_DIVIDE_BY_ZERO) == b"Divide by Zero"
    for k in range(11, 43):
        assert L.pic_ntt_prime(k) == oracle.prime(k)


def test_pi_sizes_host_only(oracle):
    for d in (1, 10, 10_000, 1_000_000, 1_000_000_000):
        assert P.pi_sizes(d) == oracle.pi_sizes(d)


def test_calls_before_init_fail_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = P.lib()
    assert L.pic_synchronize() == P.ERR_NOT_INITIALIZED
    assert L.pic_init(0) in (P.ERR_CUDA, P.ERR_INVALID)
    assert L.pic_last_error()


@pytest.mark.parametrize("lang", ["c99", "c++17"])
def test_header_is_plain_c_and_links(tmp_path, lang):
    """include/piculator_b200.h compiles warning-free as strict C99 and as
    C++17, and a C program links the library and calls a host-only entry
    point (the FFT piece width at 2^20 points) without a GPU."""
    import shutil
    cc = "gcc" if lang == "c99" else "g++"
    if shutil.which(cc) is None:
        pytest.skip(f"{cc} not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / ("main.c" if lang == "c99" else "main.cpp")
    src.write_text('#include "piculator_b200.h"\n'
                   "int main(void) { return pic_fft_piece_bits(20) == 11 ? 0 : 1; }\n")
    exe = tmp_path / "main"
    libdir = os.path.dirname(P.LIB_PATH)
    subprocess.run([cc, f"-std={lang}", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.join(root, "include"), str(src), "-L", libdir, "-lpiculator_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True)
    assert subprocess.run([str(exe)]).returncode == 0
