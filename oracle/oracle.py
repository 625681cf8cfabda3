"""ctypes wrapper of the C restatement in oracle/mcd_oracle.c.

TEST INFRASTRUCTURE ONLY: imported by tests/ (and by bench.py's CPU
baseline leg) as the checker; the product never imports it.  Determinants are
in the reference layout: interleaved spin-orbital bits in ``nw`` 64-bit words.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)


def build() -> str:
    """Compile liboracle.so (gcc) if it is missing or older than its sources."""
    src = [os.path.join(HERE, "mcd_oracle.c"), os.path.join(HERE, "mcd_oracle.h")]
    if not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in src):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        L.oracle_load.restype = ctypes.c_void_p
        L.oracle_load.argtypes = [ctypes.c_char_p, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_info.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p, _dp]
        L.oracle_integrals.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.oracle_hartree_fock.argtypes = [ctypes.c_void_p, _u64p]
        L.oracle_column.restype = ctypes.c_int64
        L.oracle_column.argtypes = [ctypes.c_void_p, _u64p, _u64p, _dp, ctypes.c_int64]
        L.oracle_diagonal.restype = ctypes.c_double
        L.oracle_diagonal.argtypes = [ctypes.c_void_p, _u64p]
        L.oracle_off_diagonal.restype = ctypes.c_double
        L.oracle_off_diagonal.argtypes = [ctypes.c_void_p, _u64p, _u64p]
        L.oracle_hsub.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_int32, _dp]
        _lib = L
    return _lib


def _u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(_u64p)


# ---------------------------------------------------------------------------
# Layout conversions between the reference's interleaved words and (alpha, beta).

def interleaved_to_ab(words, nw: int):
    """Reference words -> (alpha, beta) Python ints."""
    bits = 0
    for t in range(nw):
        bits |= int(words[t]) << (64 * t)
    a = b = 0
    p = 0
    while bits >> (2 * p):
        if (bits >> (2 * p)) & 1:
            a |= 1 << p
        if (bits >> (2 * p + 1)) & 1:
            b |= 1 << p
        p += 1
    return a, b


def ab_to_interleaved(a: int, b: int, nw: int):
    bits = 0
    p = 0
    while (a >> p) or (b >> p):
        if (a >> p) & 1:
            bits |= 1 << (2 * p)
        if (b >> p) & 1:
            bits |= 1 << (2 * p + 1)
        p += 1
    return [(bits >> (64 * t)) & 0xFFFFFFFFFFFFFFFF for t in range(nw)]


class Oracle:
    def __init__(self, path: str, threshold: float = 1e-13):
        L = lib()
        err = ctypes.create_string_buffer(512)
        self._h = L.oracle_load(path.encode(), float(threshold), err, 512)
        if not self._h:
            raise ValueError(err.value.decode())
        nso, ne, ms2, nw = (ctypes.c_int32() for _ in range(4))
        ec = ctypes.c_double()
        L.oracle_info(self._h, ctypes.byref(nso), ctypes.byref(ne), ctypes.byref(ms2), ctypes.byref(nw),
                      ctypes.byref(ec))
        self.nso, self.nelec, self.ms2, self.nw, self.ecore = nso.value, ne.value, ms2.value, nw.value, ec.value
        self.norb = self.nso // 2

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_free(self._h)
            self._h = None

    def integrals(self):
        n = self.nso
        h1 = np.zeros(n * n)
        g2 = np.zeros(n ** 4)
        lib().oracle_integrals(self._h, h1.ctypes.data_as(_dp), g2.ctypes.data_as(_dp))
        return h1.reshape(n, n), g2.reshape(n, n, n, n)

    def hartree_fock(self):
        d = np.zeros(self.nw, dtype=np.uint64)
        lib().oracle_hartree_fock(self._h, d.ctypes.data_as(_u64p))
        return [int(x) for x in d]

    def column(self, det_words):
        det, dp = _u64(det_words)
        cap = 1 << 16
        while True:
            out = np.zeros(cap * self.nw, dtype=np.uint64)
            vals = np.zeros(cap)
            n = lib().oracle_column(self._h, dp, out.ctypes.data_as(_u64p), vals.ctypes.data_as(_dp), cap)
            if n <= cap:
                return out[: n * self.nw].reshape(n, self.nw), vals[:n]
            cap = int(n)

    def diagonal(self, det_words) -> float:
        det, dp = _u64(det_words)
        return lib().oracle_diagonal(self._h, dp)

    def off_diagonal(self, d1, d2) -> float:
        a, ap = _u64(d1)
        b, bp = _u64(d2)
        return lib().oracle_off_diagonal(self._h, ap, bp)

    def hsub(self, dets):
        d, dp = _u64(np.asarray(dets, dtype=np.uint64).reshape(-1))
        k = len(dets)
        h = np.zeros(k * k)
        lib().oracle_hsub(self._h, dp, k, h.ctypes.data_as(_dp))
        return h.reshape(k, k)

    # alpha/beta helpers
    def column_ab(self, a: int, b: int):
        words, vals = self.column(ab_to_interleaved(a, b, self.nw))
        return [interleaved_to_ab(w, self.nw) for w in words], vals

    def column_ab_arrays(self, a: int, b: int):
        """get_column of (a, b) as numpy arrays (alpha, beta, value), for at
        most 64 spatial orbitals (two interleaved words)."""
        words, vals = self.column(ab_to_interleaved(a, b, self.nw))
        alpha = np.zeros(len(vals), dtype=np.uint64)
        beta = np.zeros(len(vals), dtype=np.uint64)
        for t in range(min(self.nw, 2)):
            w = words[:, t]
            alpha |= _compact_even(w) << np.uint64(32 * t)
            beta |= _compact_even(w >> np.uint64(1)) << np.uint64(32 * t)
        return alpha, beta, vals


def _compact_even(w):
    """Bits 0, 2, 4, ... of each uint64 packed into bits 0..31."""
    x = w & np.uint64(0x5555555555555555)
    for shift, mask in ((1, 0x3333333333333333), (2, 0x0F0F0F0F0F0F0F0F), (4, 0x00FF00FF00FF00FF),
                        (8, 0x0000FFFF0000FFFF), (16, 0x00000000FFFFFFFF)):
        x = (x | (x >> np.uint64(shift))) & np.uint64(mask)
    return x
