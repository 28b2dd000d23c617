"""Test infrastructure only: ctypes binding of the CPU oracle (liboracle.so).

The oracle is a C++17 + OpenMP restatement of the reference's CPU path
(antequ/fastlinkingnumbers: src/compute_link.cpp, src/discretize.cpp,
src/potential_link_search.cpp, src/linking_number_certificate.cpp,
src/ModifiedKdBVH.h, src/curve.cpp, src/model.cpp). It is the checker for the
product and the timed CPU baseline; only tests/, __graft_entry__.smoke() and
the CPU legs of bench.py import this module. The product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_libs = {}
# The reference is built -O3 -march=native (its CMakeLists.txt:19). The timed
# CPU baseline uses the same flags (plus -ffp-contract=off, as every oracle
# build), compiled on the host that runs it into a folder keyed by that
# host's CPU, so a library built for one CPU is never loaded on another. The
# checker in the tests uses the portable x86-64-v3 build.
_NATIVE_FLAGS = "-O3 -march=native -ffp-contract=off -fopenmp -fPIC -std=c++17 -Wall -Wno-unknown-pragmas"

DIRECT_FAST, DIRECT_ONE_ARCTAN, BARNES_HUT = 0, 1, 2
SEG_BSPLINE, SEG_CATMULLROM, SEG_BEZIER, SEG_POLYLINE = 0, 1, 2, 3


def build(force: bool = False) -> str:
    """Compiles the oracle with its Makefile (g++ -O3 -fopenmp)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def native_key() -> str:
    """A short key of this host's CPU (model name and feature flags)."""
    import hashlib
    info = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.strip() == "":
                    break
    except OSError:
        import platform
        info = platform.processor()
    return hashlib.sha256(info.encode()).hexdigest()[:12]


def build_native() -> str:
    """Compiles the oracle with the reference's -O3 -march=native for this
    host's CPU (once per CPU model) and returns the library path."""
    out = os.path.join("_build", "native-" + native_key())
    path = os.path.join(_HERE, out, "liboracle.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", _HERE, f"OUT={out}", f"CXXFLAGS={_NATIVE_FLAGS}",
                        os.path.join(out, "liboracle.so")], check=True)
    return path


def lib(native: bool = False):
    path = build_native() if native else build()
    if path not in _libs:
        L = C.CDLL(path)
        vp, i32p, i64p, f64p, u64p = (C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_double), C.POINTER(C.c_uint64))
        L.orc_last_error.restype = C.c_char_p
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_load_bcc.argtypes = [vp, C.c_char_p]
        L.orc_set_curves.argtypes = [vp, C.c_int, C.c_int, i32p, f64p]
        L.orc_save_bcc.argtypes = [vp, C.c_char_p]
        L.orc_num_curves.argtypes = [vp]
        L.orc_prepare.argtypes = [vp, C.c_int]
        L.orc_rounds.argtypes = [vp]
        L.orc_num_pairs.argtypes = [vp]
        L.orc_num_pairs.restype = C.c_int64
        L.orc_get_pairs.argtypes = [vp, i32p]
        L.orc_poly_total.argtypes = [vp]
        L.orc_poly_total.restype = C.c_int64
        L.orc_get_poly.argtypes = [vp, i64p, f64p]
        L.orc_set_poly.argtypes = [vp, C.c_int, i64p, f64p]
        L.orc_eval_pairs.argtypes = [vp, C.c_int, i32p, i32p, C.c_int64, C.c_double, C.c_double,
                                     C.c_int, C.c_int, f64p, f64p, u64p, u64p]
        L.orc_eval_curve_bh.argtypes = [vp, i32p, i32p, C.c_int64, C.c_double, C.c_int, C.c_int,
                                         f64p, f64p, u64p, u64p]
        L.orc_eval_curve_bh2.argtypes = [vp, i32p, i32p, C.c_int64, C.c_double, C.c_double, C.c_int, C.c_int,
                                          f64p, f64p, u64p, u64p]
        L.orc_certificate.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, f64p, f64p]
        L.orc_certificate_text.argtypes = [vp, C.c_char_p]
        L.orc_certificate.restype = C.c_int64
        L.orc_max_threads.restype = C.c_int
        _libs[path] = L
    return _libs[path]


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleError(RuntimeError):
    pass


class Oracle:
    """One model in the oracle: load -> prepare (PLS, Discretize, PLS) -> evaluate."""

    def __init__(self, native: bool = False):
        self._L = lib(native)
        self._h = self._L.orc_create()

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    def _check(self, rc):
        if rc != 0:
            raise OracleError(self._L.orc_last_error().decode())

    def load_bcc(self, path: str):
        self._check(self._L.orc_load_bcc(self._h, os.fsencode(path)))
        return self

    def set_curves(self, seg_type: int, counts, xyz):
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._check(self._L.orc_set_curves(self._h, seg_type, len(counts), _p(counts, C.c_int32),
                                           _p(xyz, C.c_double)))
        return self

    def save_bcc(self, path: str):
        self._check(self._L.orc_save_bcc(self._h, os.fsencode(path)))

    def prepare(self, discretize: bool = True):
        self._check(self._L.orc_prepare(self._h, int(discretize)))
        return self

    def set_polylines(self, offsets, xyz):
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._check(self._L.orc_set_poly(self._h, len(offsets) - 1, _p(offsets, C.c_int64),
                                         _p(xyz, C.c_double)))
        return self

    @property
    def rounds(self) -> int:
        return self._L.orc_rounds(self._h)

    def pairs(self) -> np.ndarray:
        n = self._L.orc_num_pairs(self._h)
        out = np.zeros((n, 2), dtype=np.int32)
        if n:
            self._L.orc_get_pairs(self._h, _p(out, C.c_int32))
        return out

    def polylines(self):
        nc = self._L.orc_num_curves(self._h)
        tot = self._L.orc_poly_total(self._h)
        off = np.zeros(nc + 1, dtype=np.int64)
        xyz = np.zeros((max(tot, 1), 3), dtype=np.float64)
        self._L.orc_get_poly(self._h, _p(off, C.c_int64), _p(xyz, C.c_double))
        return off, xyz[:tot]

    def eval_pairs(self, method: int, pairs, beta0=2.0, betamax=10.0, bh_parallel=False,
                   nthreads=0):
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        pi = np.ascontiguousarray(pairs[:, 0])
        pj = np.ascontiguousarray(pairs[:, 1])
        n = len(pairs)
        lk = np.zeros(n)
        err = np.zeros(n)
        nfar = np.zeros(n, dtype=np.uint64)
        nleaf = np.zeros(n, dtype=np.uint64)
        if n:
            self._check(self._L.orc_eval_pairs(
                self._h, method, _p(pi, C.c_int32), _p(pj, C.c_int32), n, beta0, betamax,
                int(bh_parallel), nthreads, _p(lk, C.c_double), _p(err, C.c_double),
                _p(nfar, C.c_uint64), _p(nleaf, C.c_uint64)))
        return lk, err, nfar, nleaf

    def eval_curve_bh(self, pairs, beta=2.0, bucket=8, nthreads=0, continue_from=None):
        """One pass of the product's curve-order Barnes-Hut (FP64) per pair:
        (lk, err * 0.05, far node pairs, exact segment pairs). With
        continue_from = beta0 < beta, the pass at beta is continued from a
        pass at beta0 (its far node pairs, its exact terms reused)."""
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        pi = np.ascontiguousarray(pairs[:, 0])
        pj = np.ascontiguousarray(pairs[:, 1])
        n = len(pairs)
        lk = np.zeros(n)
        err = np.zeros(n)
        nfar = np.zeros(n, dtype=np.uint64)
        nex = np.zeros(n, dtype=np.uint64)
        if n:
            b0 = beta if continue_from is None else continue_from
            self._check(self._L.orc_eval_curve_bh2(
                self._h, _p(pi, C.c_int32), _p(pj, C.c_int32), n, b0, beta, int(bucket), nthreads,
                _p(lk, C.c_double), _p(err, C.c_double), _p(nfar, C.c_uint64), _p(nex, C.c_uint64)))
        return lk, err, nfar, nex

    def certificate(self, direct: bool, discretize=True, beta0=2.0, betamax=10.0):
        """Full reference pipeline; returns (text, mean_off, max_off)."""
        mean = C.c_double()
        mx = C.c_double()
        n = self._L.orc_certificate(self._h, int(direct), int(discretize), beta0, betamax,
                                    C.byref(mean), C.byref(mx))
        if n < 0:
            raise OracleError(self._L.orc_last_error().decode())
        buf = C.create_string_buffer(n + 1)
        self._L.orc_certificate_text(self._h, buf)
        return buf.value.decode(), mean.value, mx.value


def max_threads(native: bool = False) -> int:
    return lib(native).orc_max_threads()
