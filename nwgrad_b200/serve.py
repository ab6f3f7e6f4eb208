"""Serving: continuous batching of alignment requests on the GPU (nwg_server_* in the C ABI).

    srv = Server(params, grad_mode="soft", workers=3)
    t = srv.submit(seqs_a, seqs_b)            # returns at once; the request queues
    scores, grad, latency_ms = srv.wait(t)    # this request's results (AlignParams gradient)
    srv.stats()                               # {"p50_ms", "p99_ms", "gcups", "done", "batches"}

A request's scores and gradient are the same bits as ``SeqPairBatch(seqs_a, seqs_b, params,
...).score_and_grad(); compute_grad()`` on its pairs alone, whatever it was batched with.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import Job, check, ptr
from .batch import _GAP, _GRAD, _device_index, _encode_all, parse_mode
from .params import AlignParams


def _lib():
    L = _capi.lib()
    if not getattr(L, "_server_bound", False):
        L.nwg_server_create.argtypes = [C.c_int, C.POINTER(Job), C.c_int, _capi._dp, _capi._dp, C.c_int, C.c_int,
                                        C.c_int64, C.c_int64, C.POINTER(C.c_void_p)]
        L.nwg_server_set_params.argtypes = [C.c_void_p, _capi._dp, _capi._dp, C.c_int]
        L.nwg_server_submit.argtypes = [C.c_void_p, _capi._u8p, _capi._i64p, _capi._u8p, _capi._i64p, C.c_int64,
                                        C.POINTER(C.c_int64)]
        L.nwg_server_wait.argtypes = [C.c_void_p, C.c_int64, _capi._dp, _capi._dp, C.POINTER(C.c_double)]
        L.nwg_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.nwg_server_destroy.argtypes = [C.c_void_p]
        L.nwg_server_device_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                              C.POINTER(C.c_int64)]
        L.nwg_server_last_error.restype = C.c_char_p
        for f in ("nwg_server_create", "nwg_server_set_params", "nwg_server_submit", "nwg_server_wait",
                  "nwg_server_stats", "nwg_server_destroy", "nwg_server_device_stats"):
            getattr(L, f).restype = C.c_int
        L._server_bound = True
    return L


def _check(L, rc):
    if rc == 0:
        return
    msg = L.nwg_server_last_error().decode(errors="replace")
    if rc in (_capi.NWG_EINVAL, _capi.NWG_ERANGE):
        raise ValueError(msg)
    if rc == _capi.NWG_ENOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


class Server:
    """Continuous-batching alignment server on one GPU."""

    def __init__(self, params: AlignParams, *, gap_model="affine", mode="global", grad_mode="soft",
                 precision=32, temperature=1.0, workers=3, hbm_budget_gb=48.0, max_batch_pairs=65536,
                 device=None, free_ends=None):
        self._L = _lib()
        self._params = params.copy()
        self._alpha = params.alphabet_obj
        _, am, sg = parse_mode(mode, free_ends)
        self._job = Job(_GAP[gap_model], am, _GRAD[grad_mode], int(precision), -1, 0,
                        float(temperature), 0, 0, 0, 0, 0, sg)
        self._grad_mode = grad_mode
        m = np.ascontiguousarray(params._m, np.float64)
        g = np.ascontiguousarray(params._g, np.float64)
        h = C.c_void_p()
        _check(self._L, self._L.nwg_server_create(_device_index(device), C.byref(self._job), self._alpha.size,
                                                  ptr(m, _capi._dp), ptr(g, _capi._dp), params.num_sets,
                                                  int(workers), int(hbm_budget_gb * (1 << 30)),
                                                  int(max_batch_pairs), C.byref(h)))
        self._h = h

    def set_params(self, params: AlignParams):
        """Requests submitted from now on use a copy of params."""
        if params.alphabet_obj is not self._alpha:
            raise ValueError("nwgrad: params alphabet does not match the server's")
        m = np.ascontiguousarray(params._m, np.float64)
        g = np.ascontiguousarray(params._g, np.float64)
        _check(self._L, self._L.nwg_server_set_params(self._h, ptr(m, _capi._dp), ptr(g, _capi._dp),
                                                      params.num_sets))
        self._params = params.copy()

    def submit_codes(self, codes_a, off_a, codes_b, off_b) -> int:
        a = np.ascontiguousarray(codes_a, np.uint8) if len(codes_a) else np.zeros(1, np.uint8)
        b = np.ascontiguousarray(codes_b, np.uint8) if len(codes_b) else np.zeros(1, np.uint8)
        oa = np.ascontiguousarray(off_a, np.int64)
        ob = np.ascontiguousarray(off_b, np.int64)
        t = C.c_int64(0)
        _check(self._L, self._L.nwg_server_submit(self._h, ptr(a, _capi._u8p), ptr(oa, _capi._i64p),
                                                  ptr(b, _capi._u8p), ptr(ob, _capi._i64p), len(oa) - 1,
                                                  C.byref(t)))
        return int(t.value)

    def submit(self, seqs_a, seqs_b) -> int:
        if len(seqs_a) != len(seqs_b):
            raise ValueError("nwgrad: seqs_a and seqs_b need equal length")
        a, oa, _ = _encode_all(self._alpha, seqs_a, "A")
        b, ob, _ = _encode_all(self._alpha, seqs_b, "B")
        return self.submit_codes(a, oa, b, ob)

    def wait(self, ticket: int, n_pairs: int | None = None):
        """(scores, gradient AlignParams or None, latency ms) of a submitted request."""
        K, N = self._params.num_sets, self._alpha.size
        gs = K * N * N + 4 * K
        cap = n_pairs if n_pairs is not None else 1 << 16
        scores = np.zeros(max(cap, 1), np.float64)
        grad = np.zeros(gs, np.float64)
        lat = C.c_double(0)
        _check(self._L, self._L.nwg_server_wait(self._h, int(ticket), ptr(scores, _capi._dp),
                                                ptr(grad, _capi._dp), C.byref(lat)))
        g = None
        if self._grad_mode != "none":
            g = AlignParams._make(grad[:K * N * N].reshape(K, N, N).copy(), grad[K * N * N:].reshape(K, 4).copy(),
                                  self._alpha)
        return (scores[:n_pairs] if n_pairs is not None else scores), g, float(lat.value)

    def stats(self) -> dict:
        p50, p99, gc = C.c_double(), C.c_double(), C.c_double()
        done, batches = C.c_int64(), C.c_int64()
        _check(self._L, self._L.nwg_server_stats(self._h, C.byref(p50), C.byref(p99), C.byref(gc),
                                                 C.byref(done), C.byref(batches)))
        busy, total, nb = C.c_double(), C.c_double(), C.c_int64()
        _check(self._L, self._L.nwg_server_device_stats(self._h, C.byref(busy), C.byref(total), C.byref(nb)))
        return {"p50_ms": p50.value, "p99_ms": p99.value, "gcups": gc.value, "done": done.value,
                "batches": batches.value, "device_busy_ms": busy.value, "device_sum_ms": total.value,
                "device_overlap": (total.value / busy.value) if busy.value > 0 else None}

    def close(self):
        if getattr(self, "_h", None):
            self._L.nwg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:   # noqa: BLE001 - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
