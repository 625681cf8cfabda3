"""mcdfci_b200: multi-coordinate-descent FCI (mCDFCI) on one B200.

Python binding of the C ABI in include/mcdfci.h (libmcdfci.so, built in-tree
by ``python -c "import __graft_entry__; __graft_entry__.build()"`` or
``make -C mcdfci_b200/csrc``).  The classes mirror the reference's interfaces
(ninotreve/mcdfci src/): ``Fcidump`` (input.h), ``Determinant``
(determinant.h), ``CDFCI`` (the Solver of solver.h, owning the Hamiltonian
tables and the hash WaveFunction on the GPU).

There is no CPU fallback: every compute call goes through libmcdfci.so and the
sm_100a kernels; importing the solver without the built library raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Callable, Iterable, List, Optional, Sequence, Tuple

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmcdfci.so")
CLI_PATH = os.path.join(_HERE, "mcdfci")

MCD_OK = 0
MCD_RESTART = -1
MCD_ERR_INVALID = 1
MCD_ERR_OVERFLOW = 2
MCD_ERR_EIG = 3
MCD_ERR_CUDA = 4
MCD_ERR_UNSUPPORTED = 5
MCD_ERR_NO_CANDIDATES = 6
MCD_STOPPED = 7
MCD_CB_RETIRE = 2  # batch report callback: stop advancing this instance only
MCD_PICK_GCD_GRAD = 0
MCD_UPDATE_EIG = 1
MCD_UPDATE_LS = 2

# Every symbol include/mcdfci.h declares.
EXPORTED_SYMBOLS = (
    "mcd_fcidump_read", "mcd_fcidump_problem", "mcd_fcidump_free", "mcd_options_default",
    "mcd_create", "mcd_create_from_fcidump", "mcd_destroy", "mcd_solve", "mcd_reset",
    "mcd_run_iterations", "mcd_run_iterations_timed", "mcd_get_report", "mcd_result", "mcd_stream", "mcd_scalars",
    "mcd_last_error", "mcd_run_json", "mcd_debug_column", "mcd_debug_hsub", "mcd_debug_eig",
    "mcd_debug_table_sums", "mcd_debug_picked", "mcd_debug_last_eig", "mcd_debug_launch_info", "mcd_debug_leader_sections",
    "mcd_debug_scatter_rate",
    "mcd_eig_update_static",
    "mcd_batch_create", "mcd_batch_destroy", "mcd_batch_size", "mcd_batch_solve", "mcd_batch_reset",
    "mcd_batch_run_iterations", "mcd_batch_run_iterations_timed", "mcd_batch_get_report", "mcd_batch_result",
    "mcd_rdm", "mcd_debug_wavefunction", "mcd_debug_compact", "mcd_checkpoint_save", "mcd_checkpoint_load",
    "mcd_debug_column_sections", "mcd_residual", "mcd_debug_slots", "mcd_debug_eig_shifted", "mcd_debug_eig_method",
    "mcd_debug_table_info", "mcd_debug_setup_times", "mcd_batch_residual", "mcd_debug_scatter_rate_mode",
    "mcd_debug_autotune_info", "mcd_batch_table_sums", "mcd_debug_grow",
)


class McdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class mcd_problem(ctypes.Structure):
    _fields_ = [
        ("norb", ctypes.c_int32), ("nelec", ctypes.c_int32), ("ms2", ctypes.c_int32), ("uhf", ctypes.c_int32),
        ("core_energy", ctypes.c_double),
        ("h1", ctypes.POINTER(ctypes.c_double)), ("g2", ctypes.POINTER(ctypes.c_double)),
        ("orbital_energy", ctypes.POINTER(ctypes.c_double)),
    ]


class mcd_options(ctypes.Structure):
    _fields_ = [
        ("num_iterations", ctypes.c_int64), ("report_interval", ctypes.c_int64),
        ("num_of_coordinate", ctypes.c_int32), ("estimate", ctypes.c_int32),
        ("z_threshold", ctypes.c_double), ("z_threshold_search", ctypes.c_int32),
        ("max_memory", ctypes.c_double), ("threshold", ctypes.c_double),
        ("ref_det_occ", ctypes.POINTER(ctypes.c_int32)), ("n_ref_det_occ", ctypes.c_int32),
        ("coordinate_pick", ctypes.c_int32), ("coordinate_update", ctypes.c_int32),
        ("groups", ctypes.c_int32), ("verbose", ctypes.c_int32),
        ("stream", ctypes.c_void_p), ("device", ctypes.c_int32), ("compaction", ctypes.c_int32),
        ("table_growth", ctypes.c_int32), ("eig_method", ctypes.c_int32), ("autotune", ctypes.c_int32),
    ]


class mcd_report(ctypes.Structure):
    _fields_ = [
        ("iteration", ctypes.c_int64), ("energy", ctypes.c_double), ("dx_max", ctypes.c_double),
        ("x_size", ctypes.c_uint64), ("z_size", ctypes.c_uint64), ("cols_size", ctypes.c_uint64),
        ("updates", ctypes.c_uint64), ("time_s", ctypes.c_double), ("scale", ctypes.c_double),
        ("max_residual", ctypes.c_double), ("z_threshold", ctypes.c_double),
        ("emitted_total", ctypes.c_uint64), ("updates_total", ctypes.c_uint64), ("occupied", ctypes.c_uint64),
        ("last_k", ctypes.c_int32), ("inv_steps_last", ctypes.c_int32), ("inv_updates", ctypes.c_uint64),
        ("inv_steps", ctypes.c_uint64), ("eig_fallbacks", ctypes.c_uint64), ("max_abs_evec", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


REPORT_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(mcd_report), ctypes.c_void_p)
BATCH_REPORT_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int32, ctypes.POINTER(mcd_report), ctypes.c_void_p)

_lib = None
_u64p = ctypes.POINTER(ctypes.c_uint64)
_dp = ctypes.POINTER(ctypes.c_double)


def library() -> ctypes.CDLL:
    """Load libmcdfci.so.  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {os.path.join(_HERE, 'csrc')}`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.mcd_fcidump_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
    L.mcd_fcidump_problem.argtypes = [vp, ctypes.POINTER(mcd_problem)]
    L.mcd_fcidump_free.argtypes = [vp]
    L.mcd_fcidump_free.restype = None
    L.mcd_options_default.argtypes = [ctypes.POINTER(mcd_options)]
    L.mcd_options_default.restype = None
    L.mcd_create.argtypes = [ctypes.POINTER(mcd_problem), ctypes.POINTER(mcd_options), ctypes.POINTER(vp)]
    L.mcd_create_from_fcidump.argtypes = [vp, ctypes.POINTER(mcd_options), ctypes.POINTER(vp)]
    L.mcd_destroy.argtypes = [vp]
    L.mcd_destroy.restype = None
    L.mcd_solve.argtypes = [vp, REPORT_CB, vp]
    L.mcd_reset.argtypes = [vp]
    L.mcd_run_iterations.argtypes = [vp, ctypes.c_int64]
    L.mcd_run_iterations_timed.argtypes = [vp, ctypes.c_int64, _dp, _dp, _dp]
    L.mcd_get_report.argtypes = [vp, ctypes.POINTER(mcd_report)]
    L.mcd_result.argtypes = [vp, _dp]
    L.mcd_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.mcd_scalars.argtypes = [vp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int64)]
    L.mcd_last_error.restype = ctypes.c_char_p
    L.mcd_last_error.argtypes = []
    L.mcd_run_json.argtypes = [ctypes.c_char_p]
    L.mcd_debug_column.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, _u64p, _u64p, _dp, ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_int64)]
    L.mcd_debug_hsub.argtypes = [vp, _u64p, _u64p, ctypes.c_int32, _dp]
    L.mcd_debug_eig.argtypes = [ctypes.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                ctypes.POINTER(ctypes.c_int32)]
    L.mcd_eig_update_static.argtypes = [ctypes.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                        ctypes.POINTER(ctypes.c_int32), vp]
    L.mcd_debug_eig_shifted.argtypes = [ctypes.c_int32, _dp, _dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp, _dp,
                                        ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.mcd_debug_eig_method.argtypes = [ctypes.c_int32, _dp, _dp, _dp, _dp, _dp, ctypes.c_int32, ctypes.c_double, _dp,
                                       _dp, _dp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.mcd_rdm.argtypes = [vp, _dp, _dp]
    L.mcd_debug_compact.argtypes = [vp, ctypes.c_double, _u64p]
    L.mcd_debug_grow.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
    L.mcd_debug_column_sections.argtypes = [vp, _u64p, ctypes.c_int32, ctypes.c_int32]
    L.mcd_checkpoint_save.argtypes = [vp, ctypes.c_char_p]
    L.mcd_checkpoint_load.argtypes = [vp, ctypes.c_char_p]
    L.mcd_debug_wavefunction.argtypes = [vp, _u64p, _u64p, _dp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    L.mcd_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ctypes.POINTER(mcd_options), ctypes.POINTER(vp)]
    L.mcd_batch_destroy.argtypes = [vp]
    L.mcd_batch_destroy.restype = None
    L.mcd_batch_size.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.mcd_batch_solve.argtypes = [vp, BATCH_REPORT_CB, vp]
    L.mcd_batch_reset.argtypes = [vp]
    L.mcd_batch_run_iterations.argtypes = [vp, ctypes.c_int64]
    L.mcd_batch_run_iterations_timed.argtypes = [vp, ctypes.c_int64, _dp, _dp, _dp]
    L.mcd_batch_get_report.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(mcd_report)]
    L.mcd_batch_result.argtypes = [vp, _dp]
    L.mcd_debug_table_sums.argtypes = [vp, _dp, _dp, _u64p]
    L.mcd_debug_picked.argtypes = [vp, _u64p, _u64p, _dp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    L.mcd_debug_last_eig.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    i32p = ctypes.POINTER(ctypes.c_int32)
    L.mcd_debug_launch_info.argtypes = [vp, i32p, i32p, i32p]
    L.mcd_debug_scatter_rate.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _dp]
    L.mcd_debug_leader_sections.argtypes = [vp, _u64p, ctypes.c_int32]
    L.mcd_residual.argtypes = [vp, _dp]
    L.mcd_debug_table_info.argtypes = [vp, _u64p, _u64p, ctypes.POINTER(ctypes.c_int32)]
    L.mcd_debug_setup_times.argtypes = [vp, _dp, ctypes.c_int32]
    L.mcd_batch_residual.argtypes = [vp, ctypes.c_int32, _dp]
    L.mcd_batch_table_sums.argtypes = [vp, ctypes.c_int32, _dp, _dp, _u64p]
    L.mcd_debug_autotune_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_int32), _dp, ctypes.c_int32,
                                          ctypes.POINTER(ctypes.c_int32)]
    L.mcd_debug_scatter_rate_mode.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_int32, _dp]
    L.mcd_debug_slots.argtypes = [vp, _u64p, _u64p, _dp, _dp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    _lib = L
    return L


def _check(rc: int) -> int:
    if rc != MCD_OK:
        raise McdError(rc, library().mcd_last_error().decode(errors="replace"))
    return rc


# ---------------------------------------------------------------------------

class Determinant:
    """A determinant as (alpha, beta) occupation strings (Determinant<N>,
    src/determinant.h:24-123, stores the same bits interleaved)."""

    __slots__ = ("alpha", "beta")

    def __init__(self, alpha: int, beta: int):
        self.alpha = int(alpha)
        self.beta = int(beta)

    @classmethod
    def from_spin_orbitals(cls, occ: Iterable[int]) -> "Determinant":
        a = b = 0
        for so in occ:
            if so & 1:
                b |= 1 << (so >> 1)
            else:
                a |= 1 << (so >> 1)
        return cls(a, b)

    def spin_orbitals(self) -> List[int]:
        out = []
        p = 0
        while (self.alpha >> p) or (self.beta >> p):
            if (self.alpha >> p) & 1:
                out.append(2 * p)
            if (self.beta >> p) & 1:
                out.append(2 * p + 1)
            p += 1
        return out

    def interleaved(self, nw: int) -> List[int]:
        """The reference's repr words."""
        bits = 0
        for so in self.spin_orbitals():
            bits |= 1 << so
        return [(bits >> (64 * t)) & 0xFFFFFFFFFFFFFFFF for t in range(nw)]

    @classmethod
    def from_interleaved(cls, words: Sequence[int]) -> "Determinant":
        bits = 0
        for t, w in enumerate(words):
            bits |= int(w) << (64 * t)
        occ = [i for i in range(bits.bit_length()) if (bits >> i) & 1]
        return cls.from_spin_orbitals(occ)

    def key(self) -> Tuple[int, int]:
        return (self.alpha, self.beta)

    def __eq__(self, other):
        return isinstance(other, Determinant) and self.key() == other.key()

    def __hash__(self):
        return hash(self.key())

    def __repr__(self):
        return f"Determinant(alpha={self.alpha:#x}, beta={self.beta:#x})"


class Fcidump:
    """A parsed FCIDUMP (Fcidump, src/input.h:57-338), host memory."""

    def __init__(self, path: str):
        L = library()
        h = ctypes.c_void_p()
        _check(L.mcd_fcidump_read(path.encode(), ctypes.byref(h)))
        self._h = h
        self.problem = mcd_problem()
        _check(L.mcd_fcidump_problem(self._h, ctypes.byref(self.problem)))
        self.path = path

    @property
    def norb(self) -> int:
        return self.problem.norb

    @property
    def nelec(self) -> int:
        return self.problem.nelec

    @property
    def ms2(self) -> int:
        return self.problem.ms2

    @property
    def core_energy(self) -> float:
        return self.problem.core_energy

    def arrays(self):
        """(h1[norb, norb], g2[norb]*4) as numpy views of the parsed data."""
        import numpy as np

        n = self.norb
        h1 = np.ctypeslib.as_array(self.problem.h1, shape=(n, n))
        g2 = np.ctypeslib.as_array(self.problem.g2, shape=(n, n, n, n))
        return h1, g2

    def __del__(self):
        if getattr(self, "_h", None):
            library().mcd_fcidump_free(self._h)
            self._h = None


def make_options(**kw) -> mcd_options:
    """mcd_options with the reference defaults, then keyword overrides
    (num_iterations, report_interval, num_of_coordinate, estimate, z_threshold,
    z_threshold_search, max_memory, threshold, ref_det_occ, coordinate_update
    ("eig"|"ls"), groups, verbose, stream, device, compaction, table_growth, eig_method)."""
    o = mcd_options()
    library().mcd_options_default(ctypes.byref(o))
    occ = kw.pop("ref_det_occ", None)
    upd = kw.pop("coordinate_update", None)
    if upd is not None:
        o.coordinate_update = {"eig": MCD_UPDATE_EIG, "ls": MCD_UPDATE_LS}[upd] if isinstance(upd, str) else int(upd)
    for k, v in kw.items():
        if k == "stream":
            o.stream = ctypes.c_void_p(int(v) if v else 0)
        elif k == "z_threshold_search":
            o.z_threshold_search = int(bool(v))
        elif k == "eig_method":
            o.eig_method = int(v)
        elif k in ("compaction", "table_growth", "autotune"):
            setattr(o, k, int(bool(v)))
        else:
            setattr(o, k, v)
    if occ:
        arr = (ctypes.c_int32 * len(occ))(*occ)
        o.ref_det_occ = ctypes.cast(arr, ctypes.POINTER(ctypes.c_int32))
        o.n_ref_det_occ = len(occ)
        o._occ_keepalive = arr  # type: ignore[attr-defined]
    return o


class CDFCI:
    """The mCDFCI solver on one GPU (CDFCI<N>, src/solver.h:621-920).

    ``CDFCI(Fcidump(path), num_of_coordinate=8, estimate=8, max_memory=0.005,
    num_iterations=20000, report_interval=1000)`` builds the Hamiltonian
    tables and the hash wavefunction on the GPU; ``solve()`` runs the
    reference's iteration and returns the energy.
    """

    def __init__(self, source, **options):
        L = library()
        self._opts = make_options(**options)
        h = ctypes.c_void_p()
        if isinstance(source, Fcidump):
            self._fcidump = source
            _check(L.mcd_create_from_fcidump(source._h, ctypes.byref(self._opts), ctypes.byref(h)))
        elif isinstance(source, mcd_problem):
            _check(L.mcd_create(ctypes.byref(source), ctypes.byref(self._opts), ctypes.byref(h)))
        else:
            self._fcidump = Fcidump(str(source))
            _check(L.mcd_create_from_fcidump(self._fcidump._h, ctypes.byref(self._opts), ctypes.byref(h)))
        self._h = h
        self.reports: List[dict] = []
        # spatial orbitals (the problem counts spin-orbitals)
        self.norb = (source.norb if isinstance(source, mcd_problem) else self._fcidump.norb) // 2

    def close(self):
        if getattr(self, "_h", None):
            library().mcd_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # -- solve ------------------------------------------------------------
    def solve(self, callback: Optional[Callable[[dict], bool]] = None) -> float:
        self.reports = []

        def cb(rep, _user):
            d = rep.contents.as_dict()
            self.reports.append(d)
            return 1 if (callback is not None and callback(d)) else 0

        c = REPORT_CB(cb)
        rc = library().mcd_solve(self._h, c, None)
        if rc not in (MCD_OK, MCD_STOPPED):
            _check(rc)
        return self.result_energy

    @property
    def result_energy(self) -> float:
        e = ctypes.c_double()
        _check(library().mcd_result(self._h, ctypes.byref(e)))
        return e.value

    # -- lower-level control ---------------------------------------------
    def reset(self):
        _check(library().mcd_reset(self._h))

    def run_iterations(self, n: int):
        _check(library().mcd_run_iterations(self._h, int(n)))

    def run_iterations_timed(self, n: int) -> dict:
        """n iterations with per-kernel CUDA events; device times in ms."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(library().mcd_run_iterations_timed(self._h, int(n), ctypes.byref(a), ctypes.byref(b),
                                                  ctypes.byref(c)))
        return {"leader_ms": a.value, "column_ms": b.value, "total_ms": c.value}

    def report(self) -> dict:
        r = mcd_report()
        _check(library().mcd_get_report(self._h, ctypes.byref(r)))
        return r.as_dict()

    def rdm(self):
        """Spin-summed spatial 1- and 2-RDM of the current wavefunction
        (mcd_rdm): arrays [n, n] and [n, n, n, n]."""
        import numpy as np

        n = self.norb
        g1 = np.zeros(n * n)
        g2 = np.zeros(n ** 4)
        _check(library().mcd_rdm(self._h, g1.ctypes.data_as(_dp), g2.ctypes.data_as(_dp)))
        return g1.reshape(n, n), g2.reshape(n, n, n, n)

    COLUMN_SECTIONS = ("decode", "probe", "update", "offer", "rounds", "prelude", "post", "merge", "ctas", "merges")

    def column_sections(self, enable: bool = True) -> dict:
        """Column-kernel phase cycles since the previous call; turns the
        timers on (or off) for later launches."""
        v = (ctypes.c_uint64 * len(self.COLUMN_SECTIONS))()
        _check(library().mcd_debug_column_sections(self._h, v, len(v), int(bool(enable))))
        return dict(zip(self.COLUMN_SECTIONS, list(v)))

    def save(self, path: str):
        """Checkpoint of the wavefunction and the iteration state."""
        _check(library().mcd_checkpoint_save(self._h, str(path).encode()))

    def load(self, path: str):
        """Continue from a checkpoint of the same problem, k and m."""
        _check(library().mcd_checkpoint_load(self._h, str(path).encode()))

    def compact(self, z_threshold: float) -> int:
        """One compaction with the given z_threshold; returns the occupied slots."""
        occ = ctypes.c_uint64()
        _check(library().mcd_debug_compact(self._h, float(z_threshold), ctypes.byref(occ)))
        return occ.value

    def wavefunction(self):
        """(alpha, beta, x) of the determinants with nonzero x."""
        import numpy as np

        cnt = ctypes.c_int64()
        _check(library().mcd_debug_wavefunction(self._h, None, None, None, 0, ctypes.byref(cnt)))
        n = cnt.value + 16
        a = np.zeros(n, dtype=np.uint64)
        b = np.zeros(n, dtype=np.uint64)
        x = np.zeros(n)
        _check(library().mcd_debug_wavefunction(self._h, a.ctypes.data_as(_u64p), b.ctypes.data_as(_u64p),
                                                x.ctypes.data_as(_dp), n, ctypes.byref(cnt)))
        k = min(cnt.value, n)
        return a[:k], b[:k], x[:k]

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(library().mcd_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def scalars(self) -> dict:
        xx, sc, xz = (ctypes.c_double * 2)(), (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
        it = ctypes.c_int64()
        _check(library().mcd_scalars(self._h, xx, sc, xz, ctypes.byref(it)))
        return {"xx": tuple(xx), "scale": tuple(sc), "xz": tuple(xz), "iteration": it.value}

    # -- parity / debug ---------------------------------------------------
    def column(self, det: Determinant):
        import numpy as np

        n = ctypes.c_int64()
        _check(library().mcd_debug_column(self._h, det.alpha, det.beta, None, None, None, 0, ctypes.byref(n)))
        cap = n.value
        a = np.zeros(cap, dtype=np.uint64)
        b = np.zeros(cap, dtype=np.uint64)
        v = np.zeros(cap)
        _check(library().mcd_debug_column(self._h, det.alpha, det.beta, a.ctypes.data_as(_u64p),
                                          b.ctypes.data_as(_u64p), v.ctypes.data_as(_dp), cap, ctypes.byref(n)))
        return a, b, v

    def hsub(self, dets: Sequence[Determinant]):
        import numpy as np

        k = len(dets)
        a = np.array([d.alpha for d in dets], dtype=np.uint64)
        b = np.array([d.beta for d in dets], dtype=np.uint64)
        h = np.zeros(k * k)
        _check(library().mcd_debug_hsub(self._h, a.ctypes.data_as(_u64p), b.ctypes.data_as(_u64p), k,
                                        h.ctypes.data_as(_dp)))
        return h.reshape(k, k)

    SETUP_STAGES = ("host_tables", "device_alloc", "upload", "table_fill", "graph_build", "growth", "reports",
                    "device_setup", "upload_copy", "upload_sync", "growth_alloc", "growth_rehash", "growth_free")

    def autotune_info(self) -> dict:
        rule, chosen, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        g = (ctypes.c_int32 * 16)()
        us = (ctypes.c_double * 16)()
        _check(library().mcd_debug_autotune_info(self._h, ctypes.byref(rule), ctypes.byref(chosen), g, us, 16,
                                                 ctypes.byref(n)))
        return {"rule": rule.value, "chosen": chosen.value,
                "trials": [{"groups": g[i], "column_us": us[i]} for i in range(min(n.value, 16))]}

    def grow(self, mode: int = 0) -> int:
        """One table growth now (mcd_debug_grow); returns the length of the
        old table's cluster through its last and first slots."""
        w = ctypes.c_int64()
        _check(library().mcd_debug_grow(self._h, int(mode), ctypes.byref(w)))
        return w.value

    def table_info(self) -> dict:
        c, mc, g = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int32()
        _check(library().mcd_debug_table_info(self._h, ctypes.byref(c), ctypes.byref(mc), ctypes.byref(g)))
        return {"capacity": c.value, "max_capacity": mc.value, "growths": g.value}

    def setup_times(self) -> dict:
        """Host wall time of the set-up stages (ms), summed since creation."""
        v = (ctypes.c_double * len(self.SETUP_STAGES))()
        _check(library().mcd_debug_setup_times(self._h, v, len(v)))
        return {k: float(x) for k, x in zip(self.SETUP_STAGES, v)}

    def residual(self) -> float:
        """||H c - E c|| / ||c|| of the current vector (mcd_residual)."""
        r = ctypes.c_double()
        _check(library().mcd_residual(self._h, ctypes.byref(r)))
        return r.value

    def slots(self):
        """(alpha, beta, x, z) of every occupied slot, in slot order."""
        import numpy as np

        cnt = ctypes.c_int64()
        _check(library().mcd_debug_slots(self._h, None, None, None, None, 0, ctypes.byref(cnt)))
        n = cnt.value
        a = np.zeros(max(n, 1), dtype=np.uint64)
        b = np.zeros(max(n, 1), dtype=np.uint64)
        x = np.zeros(max(n, 1))
        z = np.zeros(max(n, 1))
        _check(library().mcd_debug_slots(self._h, a.ctypes.data_as(_u64p), b.ctypes.data_as(_u64p),
                                         x.ctypes.data_as(_dp), z.ctypes.data_as(_dp), n, ctypes.byref(cnt)))
        k = min(cnt.value, n)
        return a[:k], b[:k], x[:k], z[:k]

    def table_sums(self) -> dict:
        xx, xz = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
        occ = ctypes.c_uint64()
        _check(library().mcd_debug_table_sums(self._h, xx, xz, ctypes.byref(occ)))
        return {"xx": tuple(xx), "xz": tuple(xz), "occupied": occ.value}

    LEADER_SECTIONS = ("state", "finish", "gather", "topk", "tie_sort", "picked", "hsub", "update_x",
                       "publish", "eig_setup", "tridiag", "multisection", "inv_iter", "backtransform",
                       "rayleigh", "eig_finish", "fast_solver", "fast_1", "fast_2", "fast_3", "fast_4",
                       "setup_fill", "setup_hx", "setup_sums", "rq_product")

    def leader_sections(self) -> dict:
        """SM cycles per leader-kernel phase since the previous call."""
        import numpy as np

        v = np.zeros(len(self.LEADER_SECTIONS), dtype=np.uint64)
        _check(library().mcd_debug_leader_sections(self._h, v.ctypes.data_as(_u64p), len(v)))
        return {name: int(c) for name, c in zip(self.LEADER_SECTIONS, v)}

    SCATTER_MODES = ("key_x_atomic", "key_x_loads", "atomic_only", "key_and_reduction")

    def scatter_rate(self, entries: int, reps: int = 20, ilp: int = 1, ctas_per_sm: int = 0, mode: int = 0) -> float:
        """Slots per second of the table's scattered-access probe (mode 0: a
        column entry's key read, x read and atomic z add, at pseudo-random
        slots; see SCATTER_MODES), with ctas_per_sm CTAs of 256 threads per
        SM (0: 8)."""
        r = ctypes.c_double()
        _check(library().mcd_debug_scatter_rate_mode(self._h, int(entries), int(reps), int(ilp), int(ctas_per_sm),
                                                     int(mode), ctypes.byref(r)))
        return r.value

    def launch_info(self) -> dict:
        c, mac, e = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _check(library().mcd_debug_launch_info(self._h, ctypes.byref(c), ctypes.byref(mac), ctypes.byref(e)))
        return {"groups": c.value, "list_size": mac.value, "entries_per_column": e.value}

    def picked(self):
        import numpy as np

        cap = 128
        a = np.zeros(cap, dtype=np.uint64)
        b = np.zeros(cap, dtype=np.uint64)
        dx = np.zeros(cap)
        k = ctypes.c_int32()
        _check(library().mcd_debug_picked(self._h, a.ctypes.data_as(_u64p), b.ctypes.data_as(_u64p),
                                          dx.ctypes.data_as(_dp), cap, ctypes.byref(k)))
        return a[: k.value], b[: k.value], dx[: k.value]

    def last_eig_inputs(self) -> dict:
        """The last iteration's subspace-eigenproblem inputs: H_sub, x, z,
        xx and xz (double-double pairs), as mcd_debug_eig takes them."""
        import numpy as np

        cap = 128
        h = np.zeros(cap * cap)
        x = np.zeros(cap)
        z = np.zeros(cap)
        xx = np.zeros(2)
        xz = np.zeros(2)
        k = ctypes.c_int32()
        _check(library().mcd_debug_last_eig(self._h, h.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                                            z.ctypes.data_as(_dp), xx.ctypes.data_as(_dp), xz.ctypes.data_as(_dp),
                                            cap, ctypes.byref(k)))
        n = k.value
        return {"k": n, "hsub": h[: n * n].reshape(n, n), "x": x[:n], "z": z[:n], "xx": xx, "xz": xz}


class CDFCIBatch:
    """Several mCDFCI instances on one GPU, advanced together (mcd_batch_*).

    ``CDFCIBatch([Fcidump(p) for p in paths], num_of_coordinate=16,
    estimate=16, max_memory=1.0, num_iterations=20000, report_interval=1000)``
    gives every FCIDUMP its own Hamiltonian tables and hash wavefunction;
    ``solve()`` runs all of them and returns their energies.  The reference
    has no equivalent: it solves a curve one point after another.
    """

    def __init__(self, sources, **options):
        L = library()
        self._fcidumps = [s if isinstance(s, Fcidump) else Fcidump(str(s)) for s in sources]
        self._opts = make_options(**options)
        arr = (ctypes.c_void_p * len(self._fcidumps))(*[f._h.value if isinstance(f._h, ctypes.c_void_p) else f._h
                                                          for f in self._fcidumps])
        h = ctypes.c_void_p()
        _check(L.mcd_batch_create(arr, len(self._fcidumps), ctypes.byref(self._opts), ctypes.byref(h)))
        self._h = h
        self.reports: List[List[dict]] = [[] for _ in self._fcidumps]

    def __len__(self) -> int:
        return len(self._fcidumps)

    def close(self):
        if getattr(self, "_h", None):
            library().mcd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def solve(self, callback: Optional[Callable[[int, dict], bool]] = None) -> List[float]:
        self.reports = [[] for _ in self._fcidumps]

        def cb(i, rep, _user):
            d = rep.contents.as_dict()
            self.reports[i].append(d)
            if callback is None:
                return 0
            v = callback(i, d)
            if v == "retire" or (not isinstance(v, bool) and v == MCD_CB_RETIRE):
                return MCD_CB_RETIRE
            return 1 if v else 0

        c = BATCH_REPORT_CB(cb)
        rc = library().mcd_batch_solve(self._h, c, None)
        if rc not in (MCD_OK, MCD_STOPPED):
            _check(rc)
        return self.result_energies

    @property
    def result_energies(self) -> List[float]:
        e = (ctypes.c_double * len(self))()
        _check(library().mcd_batch_result(self._h, e))
        return list(e)

    def reset(self):
        _check(library().mcd_batch_reset(self._h))

    def run_iterations(self, n: int):
        _check(library().mcd_batch_run_iterations(self._h, int(n)))

    def run_iterations_timed(self, n: int) -> dict:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(library().mcd_batch_run_iterations_timed(self._h, int(n), ctypes.byref(a), ctypes.byref(b),
                                                        ctypes.byref(c)))
        return {"leader_ms": a.value, "column_ms": b.value, "total_ms": c.value}

    def report(self, i: int) -> dict:
        r = mcd_report()
        _check(library().mcd_batch_get_report(self._h, int(i), ctypes.byref(r)))
        return r.as_dict()

    def table_sums(self, i: int) -> dict:
        xx, xz = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
        occ = ctypes.c_uint64()
        _check(library().mcd_batch_table_sums(self._h, int(i), xx, xz, ctypes.byref(occ)))
        return {"xx": tuple(xx), "xz": tuple(xz), "occupied": occ.value}

    def residual(self, i: int) -> float:
        """||H c - E c|| / ||c|| of instance i's current vector."""
        r = ctypes.c_double()
        _check(library().mcd_batch_residual(self._h, int(i), ctypes.byref(r)))
        return r.value


def _eig_inputs(hsub, x, z):
    """hsub as a contiguous k x k array and x, z of length k; ValueError
    otherwise (the C side copies k*k and k doubles from these buffers)."""
    import numpy as np

    hsub = np.ascontiguousarray(hsub, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    z = np.ascontiguousarray(z, dtype=np.float64).reshape(-1)
    if hsub.ndim != 2 or hsub.shape[0] != hsub.shape[1]:
        raise ValueError(f"hsub must be a square matrix, got shape {hsub.shape}")
    k = hsub.shape[0]
    if x.shape[0] != k or z.shape[0] != k:
        raise ValueError(f"x and z must have k = {k} elements, got {x.shape[0]} and {z.shape[0]}")
    return hsub, x, z, k


def debug_eig(hsub, x, z, xx, xz):
    """CoordinateUpdateEig on one subproblem (src/solver.h:333-609), on the GPU.
    xx, xz are (hi, lo) pairs.  Returns (dx, new_xx, new_scale, branch)."""
    import numpy as np

    hsub, x, z, k = _eig_inputs(hsub, x, z)
    dx = np.zeros(k)
    nxx, nsc = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
    br = ctypes.c_int32()
    xxa = (ctypes.c_double * 2)(*xx)
    xza = (ctypes.c_double * 2)(*xz)
    _check(library().mcd_debug_eig(k, hsub.ctypes.data_as(_dp), x.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                                   xxa, xza, dx.ctypes.data_as(_dp), nxx, nsc, ctypes.byref(br)))
    return dx, tuple(nxx), tuple(nsc), br.value


def debug_eig_shifted(hsub, x, z, xx, xz, drop):
    """debug_eig with the shifted solver first, as the leader runs it when
    the previous update's energy drop is known.  Returns (dx, new_xx,
    new_scale, branch, steps); steps = 0 when the full reduction ran."""
    import numpy as np

    hsub, x, z, k = _eig_inputs(hsub, x, z)
    dx = np.zeros(k)
    nxx, nsc = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
    br, st = ctypes.c_int32(), ctypes.c_int32()
    xxa = (ctypes.c_double * 2)(*xx)
    xza = (ctypes.c_double * 2)(*xz)
    _check(library().mcd_debug_eig_shifted(k, hsub.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                                           z.ctypes.data_as(_dp), xxa, xza, float(drop), dx.ctypes.data_as(_dp),
                                           nxx, nsc, ctypes.byref(br), ctypes.byref(st)))
    return dx, tuple(nxx), tuple(nsc), br.value, st.value


def debug_eig_method(hsub, x, z, xx, xz, method, drop=0.0):
    """debug_eig with a given method (mcd_options.eig_method): 0 the full
    reduction, 1 shifted inverse iteration first (drop > 0), 2 the bordered
    fixed point first.  Returns (dx, new_xx, new_scale, branch, steps); steps
    = 0 when the full reduction ran."""
    import numpy as np

    hsub, x, z, k = _eig_inputs(hsub, x, z)
    dx = np.zeros(k)
    nxx, nsc = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
    br, st = ctypes.c_int32(), ctypes.c_int32()
    xxa = (ctypes.c_double * 2)(*xx)
    xza = (ctypes.c_double * 2)(*xz)
    _check(library().mcd_debug_eig_method(k, hsub.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                                          z.ctypes.data_as(_dp), xxa, xza, int(method), float(drop),
                                          dx.ctypes.data_as(_dp), nxx, nsc, ctypes.byref(br), ctypes.byref(st)))
    return dx, tuple(nxx), tuple(nsc), br.value, st.value


def eig_update_static(hsub, x, z, xx, xz, stream=None):
    """debug_eig without allocation (mcd_eig_update_static): the device
    buffers are a static array in the library, k <= 128.  Same returns."""
    import numpy as np

    hsub, x, z, k = _eig_inputs(hsub, x, z)
    dx = np.zeros(max(k, 1))
    nxx, nsc = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
    br = ctypes.c_int32()
    xxa = (ctypes.c_double * 2)(*xx)
    xza = (ctypes.c_double * 2)(*xz)
    _check(library().mcd_eig_update_static(k, hsub.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                                           z.ctypes.data_as(_dp), xxa, xza, dx.ctypes.data_as(_dp), nxx, nsc,
                                           ctypes.byref(br), stream))
    return dx[:k], tuple(nxx), tuple(nsc), br.value


def run_json(path: str) -> int:
    """The cdfci_omp main on an input deck; returns 0 or 1."""
    return library().mcd_run_json(path.encode())
