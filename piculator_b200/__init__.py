"""piculator_b200 -- B200-native engine for Piculator's big-integer multiply path.

The product is ``lib/libpiculator_b200.so`` (hand-written sm_100a CUDA behind
the C ABI in ``include/piculator_b200.h``).  This module is a thin ctypes
mirror of that ABI for Python callers, tests and the benchmark.  It never
computes anything itself: when the shared library is missing every entry point
raises ``LibraryMissing`` instead of falling back to another implementation.

Device buffers may be anything exposing a raw CUDA pointer (``int``); tests use
torch tensors for device memory and pass ``tensor.data_ptr()``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import NamedTuple, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PICULATOR_B200_LIB", os.path.join(HERE, "lib", "libpiculator_b200.so"))
HEADER = os.path.join(os.path.dirname(HERE), "include", "piculator_b200.h")

# pic_status (include/piculator_b200.h)
OK, ERR_INVALID, ERR_LENGTH, ERR_DIVIDE_BY_ZERO, ERR_LIMIT, ERR_CUDA, ERR_NO_MEMORY, \
    ERR_NOT_INITIALIZED, ERR_IO, ERR_TIMEOUT, ERR_STOPPED = range(11)
# checkpoint flags (pic_pi_set_checkpoint)
CKPT_WRITE, CKPT_RESUME = 1, 2
# product modes
MUL_AUTO, MUL_NTT_REF, MUL_NTT3, MUL_FFT, MUL_SCHOOL, MUL_NTT3D = range(6)
MUL_MODES = {"auto": MUL_AUTO, "ntt_ref": MUL_NTT_REF, "ntt3": MUL_NTT3, "fft": MUL_FFT,
             "school": MUL_SCHOOL, "ntt3d": MUL_NTT3D}
# three-prime product forms (PIC_TUNE_NTT_FORM; FORM_CHOSEN picks per product)
FORM_INT, FORM_DBL, FORM_CHOSEN = 0, 1, 2
# pi forms
PI_CHOSEN, PI_PLAIN = 0, 1


class LibraryMissing(RuntimeError):
    pass


class PicError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"pic status {status}: {message}")
        self.status = status


class PiStats(C.Structure):
    _fields_ = [("hex_digits", C.c_uint64), ("p_words", C.c_uint64), ("terms", C.c_uint64),
                ("seconds_bsr", C.c_double), ("seconds_div", C.c_double),
                ("seconds_invsqrt", C.c_double), ("seconds_final_mul", C.c_double),
                ("seconds_hex", C.c_double), ("seconds_total", C.c_double),
                ("kernel_launches", C.c_uint64), ("products", C.c_uint64),
                ("fft_max_err", C.c_double), ("fft_recomputes", C.c_uint64),
                ("transform_reuses", C.c_uint64)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("launches", C.c_uint64), ("seconds", C.c_double),
                ("bytes", C.c_double)]


class MulDesc(C.Structure):
    _fields_ = [("z", C.c_void_p), ("a", C.c_void_p), ("b", C.c_void_p),
                ("na", C.c_uint64), ("nb", C.c_uint64)]


_lib = None
_lock = threading.Lock()

_P, _U32P, _U64P, _DP = C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p
_SIGS = {
    "pic_init": ([C.c_int], C.c_int),
    "pic_shutdown": ([], C.c_int),
    "pic_last_error": ([], C.c_char_p),
    "pic_status_string": ([C.c_int], C.c_char_p),
    "pic_synchronize": ([], C.c_int),
    "pic_device_bytes_in_use": ([], C.c_uint64),
    "pic_debug_fail_allocations": ([C.c_int], None),
    "pic_debug_allocation_count": ([], C.c_uint64),
    "pic_pi_set_checkpoint": ([C.c_char_p, C.c_int], C.c_int),
    "pic_checkpoint_inspect": ([C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                C.POINTER(C.c_uint32), C.c_int], C.c_int),
    "pic_debug_stop_after_phase": ([C.c_int], None),
    "pic_default_stream": ([], C.c_void_p),
    "pic_profile_begin": ([], C.c_int),
    "pic_profile_end": ([C.POINTER(KernelStat), C.c_int, C.POINTER(C.c_int)], C.c_int),
    "pic_measure_butterfly_rate": ([C.POINTER(C.c_double)], C.c_int),
    "pic_measure_butterfly_rate_form": ([C.c_int, C.POINTER(C.c_double)], C.c_int),
    "pic_pi_compute": ([C.c_uint64, C.c_int, C.POINTER(C.c_void_p), C.POINTER(PiStats)], C.c_int),
    "pic_ntt_ensure_table": ([C.c_int], C.c_int),
    "pic_ntt_forward": ([_U64P, C.c_int, _P], C.c_int),
    "pic_ntt_inverse": ([_U64P, C.c_int, _P], C.c_int),
    "pic_ntt_pointwise": ([_U64P, _U64P, C.c_int, _P], C.c_int),
    "pic_int_to_ntt": ([_U64P, C.c_int, _U32P, C.c_size_t, _P], C.c_int),
    "pic_ntt_to_int": ([_U64P, C.c_int, _U32P, C.c_size_t, _P], C.c_int),
    "pic_ntt_prime": ([C.c_int], C.c_uint64),
    "pic_fft_ensure_table": ([C.c_int], C.c_int),
    "pic_fft_forward": ([_DP, C.c_int, _P], C.c_int),
    "pic_fft_inverse": ([_DP, C.c_int, _P], C.c_int),
    "pic_fft_pointwise": ([_DP, _DP, C.c_int, _P], C.c_int),
    "pic_int_to_fft": ([_DP, C.c_int, _U32P, C.c_size_t, _P], C.c_int),
    "pic_fft_to_int": ([_DP, C.c_int, _U32P, C.c_size_t, _P], C.c_int),
    "pic_fft_last_max_err": ([], C.c_double),
    "pic_fft_piece_bits": ([C.c_int], C.c_int),
    "pic_fft_error_bound": ([C.c_int, C.c_int], C.c_double),
    "pic_fft_recompute_count": ([], C.c_uint64),
    "pic_product_count": ([], C.c_uint64),
    "pic_mul": ([_U32P, _U32P, C.c_size_t, _U32P, C.c_size_t, C.c_int, _P], C.c_int),
    "pic_mul_batch": ([C.POINTER(MulDesc), C.c_size_t, C.c_int, _P], C.c_int),
    "pic_mul_noalloc": ([_U32P, _U32P, C.c_size_t, _U32P, C.c_size_t, _P], C.c_int),
    "pic_mul_host": ([_U32P, _U32P, C.c_size_t, _U32P, C.c_size_t, C.c_int], C.c_int),
    "pic_bf_from_words": ([C.POINTER(C.c_void_p), C.c_int, C.c_int64, _U32P, C.c_size_t], C.c_int),
    "pic_bf_from_u32": ([C.POINTER(C.c_void_p), C.c_uint32, C.c_int], C.c_int),
    "pic_bf_free": ([C.c_void_p], C.c_int),
    "pic_bf_info": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_size_t)],
                    C.c_int),
    "pic_bf_to_words": ([C.c_void_p, _U32P, C.c_size_t], C.c_int),
    "pic_bf_to_device": ([C.c_void_p, _U32P, C.c_size_t, _P], C.c_int),
    "pic_bf_from_device": ([C.POINTER(C.c_void_p), C.c_int, C.c_int64, _U32P, C.c_size_t, _P], C.c_int),
    "pic_bf_negate": ([C.c_void_p], C.c_int),
    "pic_bf_mul_u32": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_uint32], C.c_int),
    "pic_bf_add": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_size_t], C.c_int),
    "pic_bf_sub": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_size_t], C.c_int),
    "pic_bf_mul": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_size_t, C.c_int], C.c_int),
    "pic_bf_rcp": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_size_t, C.c_int], C.c_int),
    "pic_bf_div": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_size_t, C.c_int], C.c_int),
    "pic_bf_invsqrt": ([C.POINTER(C.c_void_p), C.c_uint32, C.c_size_t, C.c_int], C.c_int),
    "pic_bf_ucmp": ([C.c_void_p, C.c_void_p], C.c_int),
    "pic_bf_to_hex": ([C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t], C.c_int),
    "pic_bf_to_dec": ([C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t], C.c_int),
    "pic_transform_create": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_size_t, C.c_int], C.c_int),
    "pic_transform_mul": ([C.c_void_p, C.c_void_p], C.c_int),
    "pic_transform_to_bf": ([C.POINTER(C.c_void_p), C.c_void_p], C.c_int),
    "pic_transform_free": ([C.c_void_p], C.c_int),
    "pic_pi_hex": ([C.c_uint64, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t),
                    C.POINTER(PiStats)], C.c_int),
    "pic_bsr": ([C.c_uint32, C.c_uint32, C.c_size_t, C.c_int, C.POINTER(C.c_void_p),
                 C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)], C.c_int),
    "pic_set_tuning": ([C.c_int, C.c_int64], C.c_int),
    "pic_get_tuning": ([C.c_int], C.c_int64),
    "pic_set_ntt_geometry": ([C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
    "pic_get_ntt_geometry": ([C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "pic_set_ntt_geometry_form": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
    "pic_get_ntt_geometry_form": ([C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)], C.c_int),
    "pic_pi_sizes": ([C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                      C.POINTER(C.c_uint64)], C.c_int),
}


def declared_symbols(header: str = HEADER) -> list[str]:
    """Every function the C header declares (used by the ABI tests)."""
    import re
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pic_[a-z0-9_]+)\s*\(", src)))


def lib() -> C.CDLL:
    """Loads the shared library (raises LibraryMissing if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise LibraryMissing(f"{LIB_PATH} is not built; run __graft_entry__.build()")
            L = C.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = res
            _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        msg = lib().pic_last_error()
        raise PicError(status, msg.decode() if msg else "")


_initialised = False


TUNING_FILE = os.path.join(HERE, "tuning.json")


def apply_tuning(path: str = TUNING_FILE) -> bool:
    """Applies an autotuner result (piculator_b200/autotune.py) if present."""
    if not os.path.exists(path):
        return False
    import json
    with open(path) as f:
        t = json.load(f)
    L = lib()
    for k, g in t.get("ntt", {}).items():
        check(L.pic_set_ntt_geometry(int(k), g["row_bits"], g["col_width_log2"], g["radix_log2"]))
    for k, g in t.get("ntt_fp64", {}).items():
        check(L.pic_set_ntt_geometry_form(FORM_DBL, int(k), g["row_bits"], g["col_width_log2"], g["radix_log2"]))
    prod = t.get("products", {})
    if "school_max_words" in prod:
        check(L.pic_set_tuning(TUNE_MUL_SCHOOL_MAX, int(prod["school_max_words"])))
    if "fft_max_words" in prod:
        check(L.pic_set_tuning(TUNE_MUL_FFT_MAX, int(prod["fft_max_words"])))
    if "bsr_school_max_words" in t.get("bsr", {}):
        check(L.pic_set_tuning(TUNE_BSR_SCHOOL_MAX, int(t["bsr"]["bsr_school_max_words"])))
    if "bsr_karatsuba_min_words" in t.get("bsr", {}):
        check(L.pic_set_tuning(TUNE_BSR_KARATSUBA, int(t["bsr"]["bsr_karatsuba_min_words"])))
    if "ntt_form" in prod:
        check(L.pic_set_tuning(TUNE_NTT_FORM, int(prod["ntt_form"])))
    if "dbl_pass_bits" in prod:
        check(L.pic_set_tuning(TUNE_DBL_PASS_TABLES, int(prod["dbl_pass_bits"])))
    if "cols_bulk" in prod:
        check(L.pic_set_tuning(TUNE_COLS_BULK, int(prod["cols_bulk"])))
    return True


def init(device: int = 0, tuned: bool = True) -> None:
    """pic_init(device), then the autotuner's settings when tuned is set."""
    global _initialised
    check(lib().pic_init(device))
    _initialised = True
    if tuned:
        apply_tuning(TUNING_FILE)


def synchronize() -> None:
    check(lib().pic_synchronize())


def mode_id(mode) -> int:
    return MUL_MODES[mode] if isinstance(mode, str) else int(mode)


# ---- products ------------------------------------------------------------------
def mul_host(a: np.ndarray, b: np.ndarray, mode="auto") -> np.ndarray:
    """Exact product of two host word arrays through pic_mul_host."""
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    z = np.empty(a.size + b.size, dtype=np.uint32)
    check(lib().pic_mul_host(z.ctypes.data, a.ctypes.data, a.size, b.ctypes.data, b.size, mode_id(mode)))
    return z


def mul_dev(z_ptr: int, a_ptr: int, na: int, b_ptr: int, nb: int, mode="auto", stream: int = 0) -> None:
    check(lib().pic_mul(z_ptr, a_ptr, na, b_ptr, nb, mode_id(mode), stream or None))


def mul_batch_dev(descs: Sequence[tuple[int, int, int, int, int]], mode="auto", stream: int = 0) -> None:
    arr = (MulDesc * len(descs))(*[MulDesc(z, a, b, na, nb) for (z, a, na, b, nb) in descs])
    check(lib().pic_mul_batch(arr, len(descs), mode_id(mode), stream or None))


# ---- BigFloat handles ------------------------------------------------------------
class BF(NamedTuple):
    sign: bool
    exp: int
    words: np.ndarray


class DeviceBigFloat:
    """Owning wrapper around a pic_bf handle (BigFloat.h semantics)."""

    def __init__(self, handle: int):
        self.h = C.c_void_p(handle)

    @staticmethod
    def from_words(sign: bool, exp: int, words: np.ndarray) -> "DeviceBigFloat":
        w = np.ascontiguousarray(words, dtype=np.uint32)
        out = C.c_void_p()
        check(lib().pic_bf_from_words(C.byref(out), int(bool(sign)), int(exp),
                                      w.ctypes.data if w.size else None, w.size))
        return DeviceBigFloat(out.value)

    @staticmethod
    def from_bf(x) -> "DeviceBigFloat":
        return DeviceBigFloat.from_words(x.sign, x.exp, x.words)

    @staticmethod
    def from_u32(x: int, sign: bool = True) -> "DeviceBigFloat":
        out = C.c_void_p()
        check(lib().pic_bf_from_u32(C.byref(out), x, int(sign)))
        return DeviceBigFloat(out.value)

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value and _lib is not None:
            _lib.pic_bf_free(self.h)
            self.h = None

    def info(self):
        s, e, n = C.c_int(), C.c_int64(), C.c_size_t()
        check(lib().pic_bf_info(self.h, C.byref(s), C.byref(e), C.byref(n)))
        return bool(s.value), int(e.value), int(n.value)

    def to_bf(self) -> BF:
        s, e, n = self.info()
        w = np.zeros(max(n, 1), dtype=np.uint32)
        check(lib().pic_bf_to_words(self.h, w.ctypes.data, w.size))
        return BF(s, e, w[:n].copy())

    def _wrap(self, fn, *args) -> "DeviceBigFloat":
        out = C.c_void_p()
        check(fn(C.byref(out), *args))
        return DeviceBigFloat(out.value)

    def negate(self):
        check(lib().pic_bf_negate(self.h))

    def mul_u32(self, x: int):
        return self._wrap(lib().pic_bf_mul_u32, self.h, x)

    def add(self, other, p: int = 0):
        return self._wrap(lib().pic_bf_add, self.h, other.h, p)

    def sub(self, other, p: int = 0):
        return self._wrap(lib().pic_bf_sub, self.h, other.h, p)

    def mul(self, other, p: int = 0, mode="auto"):
        return self._wrap(lib().pic_bf_mul, self.h, other.h, p, mode_id(mode))

    def rcp(self, p: int, mode="auto"):
        return self._wrap(lib().pic_bf_rcp, self.h, p, mode_id(mode))

    def div(self, other, p: int, mode="auto"):
        return self._wrap(lib().pic_bf_div, self.h, other.h, p, mode_id(mode))

    @staticmethod
    def invsqrt(x: int, p: int, mode="auto"):
        out = C.c_void_p()
        check(lib().pic_bf_invsqrt(C.byref(out), x, p, mode_id(mode)))
        return DeviceBigFloat(out.value)

    def ucmp(self, other) -> int:
        r = lib().pic_bf_ucmp(self.h, other.h)
        if r == -2:
            check(ERR_INVALID)
        return r

    def to_hex(self, digits: int) -> bytes:
        buf = C.create_string_buffer(digits + 32)
        check(lib().pic_bf_to_hex(self.h, digits, buf, digits + 32))
        return buf.value

    def to_dec(self, digits: int) -> bytes:
        """to_string_dec (BigFloat.cpp:83-94)."""
        buf = C.create_string_buffer(digits + 32)
        check(lib().pic_bf_to_dec(self.h, digits, buf, digits + 32))
        return buf.value


class Transform:
    """Transform-domain operand (Transform.h)."""

    def __init__(self, x: DeviceBigFloat, p: int = 0, k: int = 0):
        out = C.c_void_p()
        check(lib().pic_transform_create(C.byref(out), x.h, p, k))
        self.h = out

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value and _lib is not None:
            _lib.pic_transform_free(self.h)
            self.h = None

    def mul(self, other: "Transform") -> None:
        check(lib().pic_transform_mul(self.h, other.h))

    def to_bigfloat(self) -> DeviceBigFloat:
        out = C.c_void_p()
        check(lib().pic_transform_to_bf(C.byref(out), self.h))
        return DeviceBigFloat(out.value)


(TUNE_BSR_SCHOOL_MAX, TUNE_MUL_SCHOOL_MAX, TUNE_MUL_FFT_MAX, TUNE_BATCH_GRAPHS, TUNE_BSR_WRAP,
 TUNE_BSR_SMALL_MERGE, TUNE_MUL_WRAP, TUNE_BSR_COMBINE, TUNE_FFT_ACCEPT_PPM, TUNE_BSR_KARATSUBA,
 TUNE_NTT_FORM, TUNE_DBL_PASS_TABLES, TUNE_COLS_BULK) = range(13)


def butterfly_rate(form: int = FORM_INT) -> float:
    """G butterflies per second with everything in registers (integer lazy
    Shoup, or the FP64 form's): the arithmetic ceiling of the NTT passes."""
    v = C.c_double(0.0)
    check(lib().pic_measure_butterfly_rate_form(form, C.byref(v)))
    return v.value


def set_tuning(knob: int, value: int) -> None:
    check(lib().pic_set_tuning(knob, value))


def get_tuning(knob: int) -> int:
    return int(lib().pic_get_tuning(knob))


def set_ntt_geometry(k: int, row_bits: int, col_width_log2: int, radix_log2: int, form: int = FORM_INT) -> None:
    check(lib().pic_set_ntt_geometry_form(form, k, row_bits, col_width_log2, radix_log2))


def get_ntt_geometry(k: int, form: int = FORM_INT) -> tuple[int, int, int]:
    r, c, x = C.c_int(), C.c_int(), C.c_int()
    check(lib().pic_get_ntt_geometry_form(form, k, C.byref(r), C.byref(c), C.byref(x)))
    return r.value, c.value, x.value


def bsr(a: int, b: int, p: int, form: int = 0):
    """Binary splitting over [a, b) at precision p: (P, Q, R) DeviceBigFloats."""
    hp, hq, hr = C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(lib().pic_bsr(a, b, p, form, C.byref(hp), C.byref(hq), C.byref(hr)))
    return DeviceBigFloat(hp.value), DeviceBigFloat(hq.value), DeviceBigFloat(hr.value)


# ---- pi ----------------------------------------------------------------------------
def pi_sizes(digits: int) -> tuple[int, int, int]:
    h, p, t = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(lib().pic_pi_sizes(digits, C.byref(h), C.byref(p), C.byref(t)))
    return int(h.value), int(p.value), int(t.value)


def pi_hex(digits: int, form: int = PI_CHOSEN, want_text: bool = True):
    """Runs Pi(digits) on the GPU.  Returns (text bytes or None, stats dict)."""
    hexd, _, _ = pi_sizes(digits)
    st = PiStats()
    n = C.c_size_t(0)
    if want_text:
        cap = hexd + 64
        buf = C.create_string_buffer(cap)
        check(lib().pic_pi_hex(digits, form, buf, cap, C.byref(n), C.byref(st)))
        return buf.raw[: n.value], st.as_dict()
    check(lib().pic_pi_hex(digits, form, None, 0, None, C.byref(st)))
    return None, st.as_dict()


def set_checkpoint(directory: str | None, flags: int = CKPT_WRITE | CKPT_RESUME) -> None:
    """pic_pi_set_checkpoint: write / resume pi computations in `directory`
    (None turns checkpoints off)."""
    check(lib().pic_pi_set_checkpoint(directory.encode() if directory else None, flags if directory else 0))


def checkpoint_inspect(path: str, verify: bool = True) -> dict:
    """Header of a checkpoint file (host only): digits, p_words, phase."""
    d, pw, ph = C.c_uint64(), C.c_uint64(), C.c_uint32()
    check(lib().pic_checkpoint_inspect(path.encode(), C.byref(d), C.byref(pw), C.byref(ph), int(verify)))
    return {"digits": d.value, "p_words": pw.value, "phase": ph.value}
