"""Host-side mirror of the reference's public interface for the linking-number
path, over the C ABI of libfln.so.

Names follow the reference (antequ/fastlinkingnumbers): ``Model``
(include/model.h:24-75), ``LinkingNumberCertificate``
(include/linking_number_certificate.h:25-131) and the per-pair functions of
src/compute_link.h:62-87. Errors raise ``FlnError`` (a RuntimeError) where the
reference throws std::runtime_error.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _native as N
from ._native import FlnError, default_params


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Engine:
    """One CUDA device and stream (fln_ctx). ``stream`` is an optional
    cudaStream_t handle (e.g. ``torch.cuda.current_stream().cuda_stream``)."""

    def __init__(self, device: int = 0, stream: int = 0):
        self._L = N.load()
        h = C.c_void_p()
        N.check(self._L.fln_ctx_create(int(device), C.c_void_p(stream or None), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.fln_ctx_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return self._h

    def stats(self) -> dict:
        s = N.Stats()
        N.check(self._L.fln_ctx_stats(self._h, C.byref(s)))
        return s.as_dict()

    def linking_numbers(self, xyz, loop_offsets, pairs, method: str = "barneshut",
                        params: Optional[N.Params] = None, **overrides):
        """Real-valued linking numbers of closed polylines for each (i, j) pair.

        xyz: (V, 3) float64 vertices; loop_offsets: (L + 1,) int64 CSR offsets;
        pairs: (P, 2) int32. Returns (lk, err, flags) numpy arrays."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        off = np.ascontiguousarray(loop_offsets, dtype=np.int64)
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        prm = params if params is not None else default_params(**overrides)
        n = len(pairs)
        lk = np.zeros(n)
        err = np.zeros(n)
        flags = np.zeros(n, dtype=np.int32)
        N.check(self._L.fln_linking_numbers(
            self._h, _ptr(xyz), _ptr(off), len(off) - 1, _ptr(pairs), n,
            N.METHOD_DIRECTSUM if method == "directsum" else _method(method), C.byref(prm),
            _ptr(lk), _ptr(err), _ptr(flags)))
        return lk, err, flags

    def linking_numbers_device(self, d_xyz: int, d_offsets: int, nloops: int, d_pairs: int,
                               npairs: int, d_lk: int, d_err: int = 0, d_flags: int = 0,
                               method: str = "barneshut", params: Optional[N.Params] = None,
                               **overrides):
        """Same as linking_numbers with every array already in device memory
        (raw device pointers, e.g. torch ``tensor.data_ptr()``)."""
        prm = params if params is not None else default_params(**overrides)
        N.check(self._L.fln_linking_numbers_device(
            self._h, C.c_void_p(d_xyz), C.c_void_p(d_offsets), int(nloops), C.c_void_p(d_pairs),
            int(npairs), _method(method), C.byref(prm), C.c_void_p(d_lk),
            C.c_void_p(d_err or None), C.c_void_p(d_flags or None)))

    def direct_pair(self, curve1, curve2, precision: int = N.PREC_FP64) -> float:
        a = np.ascontiguousarray(curve1, dtype=np.float64).reshape(-1, 3)
        b = np.ascontiguousarray(curve2, dtype=np.float64).reshape(-1, 3)
        out = C.c_double()
        N.check(self._L.fln_direct_pair(self._h, _ptr(a), len(a), _ptr(b), len(b), precision,
                                        C.byref(out)))
        return out.value

    def autotune(self, xyz, loop_offsets, pairs, tune_beta: bool = False, sample_pairs: int = 0,
                 params: Optional[N.Params] = None, tune_bucket: bool = False, **overrides):
        """Fastest Barnes-Hut settings on a seeded sample of the pairs:
        (tuned Params, result dict). The round budget always; beta only if
        tune_beta, the exact-bucket size only if tune_bucket."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        off = np.ascontiguousarray(loop_offsets, dtype=np.int64)
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        prm = params if params is not None else default_params(**overrides)
        out = N.Params()
        res = N.TuneResult()
        N.check(self._L.fln_autotune(self._h, _ptr(xyz), _ptr(off), len(off) - 1, _ptr(pairs), len(pairs),
                                     C.byref(prm), int(bool(tune_beta)) | (2 if tune_bucket else 0),
                                     int(sample_pairs), C.byref(out),
                                     C.byref(res)))
        return out, res.as_dict()

    def autotune_direct(self, xyz, loop_offsets, pairs, sample_pairs: int = 0,
                        params: Optional[N.Params] = None, **overrides):
        """Fastest direct-sum tile shape on a seeded sample of the pairs:
        (tuned Params, result dict)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        off = np.ascontiguousarray(loop_offsets, dtype=np.int64)
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        prm = params if params is not None else default_params(**overrides)
        out = N.Params()
        res = N.TuneResult()
        N.check(self._L.fln_autotune_direct(self._h, _ptr(xyz), _ptr(off), len(off) - 1, _ptr(pairs), len(pairs),
                                            C.byref(prm), int(sample_pairs), C.byref(out), C.byref(res)))
        return out, res.as_dict()

    # ---- learned opening criterion (no counterpart in the reference)
    def set_learned(self, model: Optional["LearnedCriterion"]):
        """Uses `model` for the Barnes–Hut opening decisions of this engine (None: off)."""
        N.check(self._L.fln_ctx_set_learned(self._h, model.handle if model is not None else None))

    def learned_collect(self, xyz, loop_offsets, pairs, cap: int, s_min: float = 1.0,
                        sample_keep: float = 0.05, max_terms: int = 1 << 16,
                        params: Optional[N.Params] = None, **overrides):
        """Training samples the way LearnedCriterion.train records them:
        (features (n, 8) float32, log10 true error (n,), separation (n,),
        log10 of the scaled Eq. 14 estimate (n,))."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        off = np.ascontiguousarray(loop_offsets, dtype=np.int64)
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        prm = params if params is not None else default_params(**overrides)
        X = np.zeros((max(cap, 1), 8), dtype=np.float32)
        T = np.zeros(max(cap, 1), dtype=np.float32)
        S = np.zeros(max(cap, 1), dtype=np.float32)
        E = np.zeros(max(cap, 1), dtype=np.float32)
        n = C.c_int64()
        N.check(self._L.fln_learned_collect(
            self._h, _ptr(xyz), _ptr(off), len(off) - 1, _ptr(pairs), len(pairs), C.byref(prm),
            float(s_min), float(sample_keep), int(cap), int(max_terms), _ptr(X), _ptr(T), _ptr(S),
            _ptr(E), C.byref(n)))
        k = n.value
        return X[:k].copy(), T[:k].copy(), S[:k].copy(), E[:k].copy()

    def mlp_predict(self, params, features, use_mma: bool = False) -> np.ndarray:
        """MLP outputs for rows of 8 features: FP32, or the traversal's BF16 warp-MMA path."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        X = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 8)
        if p.size != N.MLP_PARAMS:
            raise FlnError(1, f"expected {N.MLP_PARAMS} parameters")
        y = np.zeros(len(X), dtype=np.float32)
        N.check(self._L.fln_learned_predict(self._h, _ptr(p), _ptr(X), len(X), int(use_mma),
                                            _ptr(y)))
        return y

    def mlp_gradients(self, params, features, targets, quantile: float = 0.9):
        """(mean pinball loss, d loss / d params) from the training kernel."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        X = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 8)
        T = np.ascontiguousarray(targets, dtype=np.float32).reshape(-1)
        if p.size != N.MLP_PARAMS or len(T) != len(X):
            raise FlnError(1, "parameter or row count")
        g = np.zeros(N.MLP_PARAMS, dtype=np.float32)
        loss = C.c_double()
        N.check(self._L.fln_learned_gradients(self._h, _ptr(p), _ptr(X), _ptr(T), len(X),
                                              float(quantile), _ptr(g), C.byref(loss)))
        return loss.value, g


def learned_options(**overrides) -> N.LearnedOptions:
    o = N.LearnedOptions()
    N.load().fln_learned_default_options(C.byref(o))
    for k, v in overrides.items():
        if not hasattr(o, k):
            raise FlnError(1, f"unknown learned option {k}")
        setattr(o, k, v)
    return o


class LearnedCriterion:
    """The learned Barnes–Hut opening criterion (fln_learned)."""

    def __init__(self, handle):
        self._L = N.load()
        self._h = handle

    @classmethod
    def train(cls, engine: Engine, xyz, loop_offsets, pairs, params: Optional[N.Params] = None,
              options: Optional[N.LearnedOptions] = None, **option_overrides) -> "LearnedCriterion":
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        off = np.ascontiguousarray(loop_offsets, dtype=np.int64)
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        prm = params if params is not None else default_params()
        opt = options if options is not None else learned_options(**option_overrides)
        h = C.c_void_p()
        L = N.load()
        N.check(L.fln_learned_train(engine.handle, _ptr(xyz), _ptr(off), len(off) - 1, _ptr(pairs),
                                    len(pairs), C.byref(prm), C.byref(opt), C.byref(h)))
        return cls(h)

    @classmethod
    def from_params(cls, params, s_min: float, log10_tau: float,
                    min_candidates: int = 4) -> "LearnedCriterion":
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != N.MLP_PARAMS:
            raise FlnError(1, f"expected {N.MLP_PARAMS} parameters")
        h = C.c_void_p()
        L = N.load()
        N.check(L.fln_learned_create(_ptr(p), float(s_min), float(log10_tau), int(min_candidates),
                                     C.byref(h)))
        return cls(h)

    @property
    def handle(self):
        return self._h

    def params(self) -> np.ndarray:
        p = np.zeros(N.MLP_PARAMS, dtype=np.float32)
        N.check(self._L.fln_learned_get(self._h, _ptr(p), None))
        return p

    def configure(self, min_candidates: int = 4, min_node_segments: int = 0) -> "LearnedCriterion":
        """When the MLP runs in the traversal: warp steps with at least
        min_candidates candidates, candidates whose smaller node holds at
        least min_node_segments segments. Applies at the next set_learned."""
        N.check(self._L.fln_learned_configure(self._h, int(min_candidates), int(min_node_segments)))
        return self

    def info(self) -> dict:
        i = N.LearnedInfo()
        N.check(self._L.fln_learned_get(self._h, None, C.byref(i)))
        return i.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            self._L.fln_learned_destroy(self._h)
            self._h = None

    __del__ = close


def _method(m: str) -> int:
    if m == "directsum":
        return N.METHOD_DIRECTSUM
    if m == "barneshut":
        return N.METHOD_BARNESHUT
    raise FlnError(1, f"Invalid method: '{m}'.")


_default_engine: Optional[Engine] = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(0)
    return _default_engine


def ComputeLinkingNumberDirectFast(curve1, curve2, parallel: bool = False) -> float:
    """src/compute_link.h:86 — FP64 direct sum of two closed polylines ((n, 3) arrays)."""
    return default_engine().direct_pair(curve1, curve2, N.PREC_FP64)


def ComputeLinkingNumberDirectOneArctanPerPair(curve1, curve2, parallel: bool = False) -> float:
    """src/compute_link.h:62 — same integral; the GPU kernel serves both forms."""
    return default_engine().direct_pair(curve1, curve2, N.PREC_FP64)


class Model:
    """A collection of curves (include/model.h:24-75)."""

    def __init__(self):
        self._L = N.load()
        h = C.c_void_p()
        N.check(self._L.fln_model_create(C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.fln_model_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def ImportFromFile(self, filename: str):
        N.check(self._L.fln_model_load_bcc(self._h, os.fsencode(filename)))
        return self

    def ExportToFile(self, filename: str):
        N.check(self._L.fln_model_save_bcc(self._h, os.fsencode(filename)))

    def SetCurves(self, seg_type: int, counts, xyz):
        """counts[c] points per curve (negative = closed loop), xyz (P, 3)."""
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        N.check(self._L.fln_model_set_curves(self._h, int(seg_type), len(counts), _ptr(counts),
                                             _ptr(xyz)))
        return self

    def GetCurves(self):
        """Returns (seg_type, counts, xyz)."""
        nc = self._L.fln_model_num_curves(self._h)
        npnt = self._L.fln_model_num_points(self._h)
        t = C.c_int32()
        counts = np.zeros(nc, dtype=np.int32)
        xyz = np.zeros((max(npnt, 1), 3))
        N.check(self._L.fln_model_get_curves(self._h, C.byref(t), _ptr(counts), _ptr(xyz)))
        return t.value, counts, xyz[:npnt]

    def num_curves(self) -> int:
        return self._L.fln_model_num_curves(self._h)

    def Prepare(self, discretize: bool = True, engine: Optional["Engine"] = None):
        """PLS -> Discretize -> PLS. Returns (loop_offsets, xyz, pairs, rounds).
        With an engine the stages run on its GPU (same output bit for bit)."""
        r = C.c_int32()
        if engine is None:
            N.check(self._L.fln_model_prepare(self._h, int(discretize), C.byref(r)))
        else:
            N.check(self._L.fln_model_prepare_device(engine.handle, self._h, int(discretize), C.byref(r)))
        nv, npairs = C.c_int64(), C.c_int64()
        N.check(self._L.fln_model_prepared_sizes(self._h, C.byref(nv), C.byref(npairs)))
        off = np.empty(self.num_curves() + 1, dtype=np.int64)
        xyz = np.empty((max(nv.value, 1), 3))
        pairs = np.empty((max(npairs.value, 1), 2), dtype=np.int32)
        N.check(self._L.fln_model_get_prepared(self._h, _ptr(off), _ptr(xyz), _ptr(pairs)))
        return off, xyz[:nv.value], pairs[:npairs.value], r.value


class LinkingNumberCertificate:
    """include/linking_number_certificate.h:25-131."""

    def __init__(self, filename: Optional[str] = None):
        self._L = N.load()
        self._h = None
        if filename is not None:
            self.ImportFromFile(filename)

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.fln_certificate_destroy(self._h)
            self._h = None

    def _replace(self, h):
        if self._h:
            self._L.fln_certificate_destroy(self._h)
        self._h = h

    def ComputeFromModel(self, model: Model, force_direct_sum: bool = False,
                         discretize: bool = True, barnes_hut_init_beta: float = 2.0,
                         barnes_hut_beta_limit: float = 10.0, engine: Optional[Engine] = None,
                         **overrides):
        eng = engine or default_engine()
        prm = default_params(barnes_hut_init_beta=barnes_hut_init_beta,
                             barnes_hut_beta_limit=barnes_hut_beta_limit, **overrides)
        h = C.c_void_p()
        N.check(self._L.fln_certificate_compute(eng.handle, model.handle, int(force_direct_sum),
                                                int(discretize), C.byref(prm), C.byref(h)))
        self._replace(h)
        return self

    def ImportFromFile(self, filename: str):
        h = C.c_void_p()
        N.check(self._L.fln_certificate_load(os.fsencode(filename), C.byref(h)))
        self._replace(h)
        return self

    def ExportToFile(self, filename: str):
        N.check(self._L.fln_certificate_save(self._h, os.fsencode(filename)))

    def text(self) -> str:
        n = self._L.fln_certificate_text(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        self._L.fln_certificate_text(self._h, buf, n + 1)
        return buf.value.decode()

    def entries(self) -> np.ndarray:
        n = self._L.fln_certificate_num_entries(self._h)
        out = np.zeros((max(n, 1), 3), dtype=np.int32)
        N.check(self._L.fln_certificate_entries(self._h, _ptr(out)))
        return out[:n]

    def pairs(self):
        """Per evaluated pair: (pairs (P, 2), lk, err, flags)."""
        n = self._L.fln_certificate_num_pairs(self._h)
        pr = np.zeros((max(n, 1), 2), dtype=np.int32)
        lk, err = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        fl = np.zeros(max(n, 1), dtype=np.int32)
        N.check(self._L.fln_certificate_pairs(self._h, _ptr(pr), _ptr(lk), _ptr(err), _ptr(fl)))
        return pr[:n], lk[:n], err[:n], fl[:n]

    def ExportDiffsToFiles(self, out_diff_links_filename: str, out_diff_curves_filename: str,
                           other: "LinkingNumberCertificate"):
        N.check(self._L.fln_certificate_export_diffs(
            self._h, other._h, os.fsencode(out_diff_links_filename),
            os.fsencode(out_diff_curves_filename)))

    def Equals(self, other: "LinkingNumberCertificate") -> bool:
        return bool(self._L.fln_certificate_equals(self._h, other._h))

    def __eq__(self, other):
        return self.Equals(other)

    def __ne__(self, other):
        return not self.Equals(other)
