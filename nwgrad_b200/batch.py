"""SeqPairBatch / SeqPairBatchDouble / SeqPair: the reference's batch API on the B200 path.

Mirrors michalsta/nwgrad's Python surface (py_exports.cpp:563-1262, docs/api.md) with the
same names, arguments, return types and exceptions.  The pairs are validated and encoded
once, uploaded to the GPU and kept there (the C ABI's store); every alignment runs on the
device through libnwgrad_b200.so.  CPU-only knobs of the reference (n_threads, kernel,
fill, schedule) are accepted and validated but have nothing to select here.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from . import _capi
from ._capi import Job, check, ptr
from .params import AlignParams, Alphabet

_GAP = {"linear": 0, "affine": 1}
_MODE = {"global": 0, "local": 1, "glocal": 2, "overlap": 2, "semiglobal": 2}
# semi-global free ends (the reference's kSgFree* bits, simd_levels.hpp:170-182)
_SG_NAMES = ("a_begin", "a_end", "b_begin", "b_end")
_SG_BITS = (1, 2, 4, 8)
SG_GLOCAL, SG_ALL = 12, 15
_CURRENT = object()   # a deferred soft guide due under the params current at its first use


def parse_mode(mode, free_ends=None):
    """(mode, free_ends) -> (mode name, align mode 0 global / 1 local / 2 semi-global, free-end
    bits), with the reference's rules and messages (py_exports.cpp:276-335): "semiglobal" takes
    free_ends -- four truth values (a_begin, a_end, b_begin, b_end) or the names of the free
    ones; "glocal" is (b_begin, b_end), "overlap" all four; other modes refuse free_ends."""
    if mode == "semiglobal":
        if free_ends is None:
            raise ValueError("nwgrad: mode \"semiglobal\" needs free_ends=(a_begin, a_end, b_begin, b_end)")
        return mode, 2, _parse_free_ends(free_ends)
    if free_ends is not None:
        raise ValueError(f"nwgrad: free_ends= goes with mode \"semiglobal\" (got mode \"{mode}\", "
                         f"whose ends are fixed)")
    if mode == "overlap":
        return mode, 2, SG_ALL
    if mode == "glocal":
        return mode, 2, SG_GLOCAL
    if mode in ("global", "local"):
        return mode, _MODE[mode], SG_GLOCAL
    raise ValueError(f"nwgrad: unknown mode \"{mode}\" (expected \"global\", \"local\", \"glocal\", "
                     f"\"overlap\" or \"semiglobal\")")


def _parse_free_ends(h):
    msg = ("nwgrad: free_ends must be four booleans (a_begin, a_end, b_begin, b_end) or the names of "
           "the free ends (\"a_begin\", \"a_end\", \"b_begin\", \"b_end\")")
    if isinstance(h, str):
        h = (h,)
    try:
        items = list(h)
    except TypeError:
        raise ValueError(msg) from None
    if not items:
        return 0
    if all(isinstance(x, str) for x in items):
        f = 0
        for nm in items:
            if nm not in _SG_NAMES:
                raise ValueError(f"nwgrad: unknown free end \"{nm}\" (expected \"a_begin\", \"a_end\", "
                                 f"\"b_begin\" or \"b_end\")")
            f |= _SG_BITS[_SG_NAMES.index(nm)]
        return f
    if len(items) != 4 or any(isinstance(x, str) for x in items):
        raise ValueError(msg)
    return sum(b for b, x in zip(_SG_BITS, items) if bool(x))
_GRAD = {"none": 0, "hard": 1, "soft": 2}
_TB = ("auto", "pointers", "scores", "hirschberg", "hirschberg_pmax", "grid")
_KERNELS = ("auto", "scalar_fallback", "sse2", "sse4", "avx2", "avx512", "neon")


def _device_index(device) -> int:
    if device is not None:
        return int(device)
    env = os.environ.get("NWGRAD_B200_DEVICE")
    if env:
        return int(env)
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.current_device()
    except Exception:   # noqa: BLE001 - torch is optional plumbing
        pass
    return 0


def _encode_all(alpha: Alphabet, seqs, which: str):
    """Concatenated codes and int64 offsets; a foreign character raises ValueError naming
    the pair and position (batch_engine.hpp:827-844)."""
    seqs = [s if isinstance(s, str) else str(s) for s in seqs]
    lens = np.fromiter((len(s) for s in seqs), dtype=np.int64, count=len(seqs))
    off = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    try:
        raw = np.frombuffer("".join(seqs).encode("latin-1"), dtype=np.uint8)
    except UnicodeEncodeError:
        raw = None
    if raw is None:
        for p, s in enumerate(seqs):
            for k, ch in enumerate(s):
                if ord(ch) > 255 or alpha.index_of(ch) < 0:
                    raise ValueError(f"nwgrad: pair {p}, sequence {which}: character '{ch}' at position {k} "
                                     f"is not in alphabet \"{alpha.symbols}\"")
    codes = alpha._lut[raw]
    bad = np.nonzero(codes == 255)[0]
    if bad.size:
        g = int(bad[0])
        p = int(np.searchsorted(off, g, side="right") - 1)
        k = g - int(off[p])
        raise ValueError(f"nwgrad: pair {p}, sequence {which}: character '{seqs[p][k]}' at position {k} "
                         f"is not in alphabet \"{alpha.symbols}\"")
    return np.ascontiguousarray(codes, dtype=np.uint8), off, seqs


def _flat_tracks(tracks, lens, name, per_pair_extra):
    """None, a flat 1-D integer array (sum of lens + extra entries), or one entry per pair
    (None entries: the default).  Returns (flat uint16 or None, mask of pairs given)."""
    if tracks is None:
        return None, None
    n = len(lens)
    need = lens + per_pair_extra
    if isinstance(tracks, np.ndarray) and tracks.ndim == 1 and tracks.dtype != object:
        t = np.asarray(tracks)
        if not np.issubdtype(t.dtype, np.integer):
            raise ValueError(f"nwgrad: {name} must be integers")
        if t.size != int(need.sum()):
            raise ValueError(f"nwgrad: {name} has {t.size} entries, the pairs need {int(need.sum())}")
        if t.size and (t.min() < 0 or t.max() > 65535):
            raise ValueError(f"nwgrad: {name} entries must be in [0, 65535]")
        return np.ascontiguousarray(t, dtype=np.uint16), np.ones(n, bool)
    tracks = list(tracks)
    if len(tracks) != n:
        raise ValueError(f"nwgrad: {name} needs one entry per pair ({len(tracks)} for {n} pairs)")
    out = []
    given = np.zeros(n, bool)
    for p, t in enumerate(tracks):
        if t is None:
            out.append(None)
            continue
        a = np.asarray(t, dtype=np.int64)
        if a.ndim != 1 or a.size != int(need[p]):
            if name == "gap_tracks":
                raise ValueError(f"nwgrad: gap_track has {a.size} entries, but sequence A of length "
                                 f"{int(lens[p])} needs {int(need[p])} (one per DP row 0..m)")
            raise ValueError(f"nwgrad: track has {a.size} entries, but sequence A has {int(lens[p])} "
                             f"residues (one set per residue)")
        if a.size and (a.min() < 0 or a.max() > 65535):
            raise ValueError(f"nwgrad: {name} entries must be in [0, 65535]")
        out.append(a.astype(np.uint16))
        given[p] = True
    return out, given


class _Store:
    """Owns one C-ABI store (device-resident pairs)."""

    def __init__(self, a, oa, b, ob, nalpha, tracks, gtracks, device):
        L = _capi.lib()
        self._L = L
        h = C.c_void_p()
        n = len(oa) - 1
        check(L.nwg_store_create(ptr(a, _capi._u8p), ptr(oa, _capi._i64p), ptr(b, _capi._u8p),
                                 ptr(ob, _capi._i64p), n, nalpha, ptr(tracks, _capi._u16p),
                                 ptr(gtracks, _capi._u16p), device, C.byref(h)))
        self.h = h
        self._fin = weakref.finalize(self, L.nwg_store_destroy, h)


class SeqPairBatch:
    """A batch of pairs (seqs_a[i], seqs_b[i]) of one problem type, aligned on the GPU.

    float32 DP (``SeqPairBatchDouble``: float64).  See the reference's docs/api.md
    "SeqPairBatch" for every argument and contract.
    """

    _precision = 32

    def __init__(self, seqs_a=None, seqs_b=None, params=None, *, n_threads=0, traceback="auto",
                 gap_model="affine", mode="global", grad_mode="hard", kernel="auto", tracks=None,
                 gap_tracks=None, free_ends=None, device=None):
        if isinstance(seqs_a, int) and seqs_b is None:   # SeqPairBatch(n_threads, traceback, ...)
            n_threads, seqs_a = seqs_a, None
        if int(n_threads) < 0:
            raise ValueError(f"nwgrad: n_threads must be >= 0 (0: the default thread count), got {n_threads}")
        if gap_model not in _GAP:
            raise ValueError(f"nwgrad: gap_model must be \"linear\" or \"affine\", got \"{gap_model}\"")
        mode, self._am, self._sg = parse_mode(mode, free_ends)
        if grad_mode not in _GRAD:
            raise ValueError(f"nwgrad: unknown grad_mode \"{grad_mode}\"")
        if traceback not in _TB:
            raise ValueError(f"nwgrad: unknown traceback \"{traceback}\"")
        if kernel not in _KERNELS:
            raise ValueError(f"nwgrad: unknown kernel \"{kernel}\"")
        self._n_threads = int(n_threads)
        self._traceback = traceback
        self._gap_model = gap_model
        self._mode = mode
        self._grad_mode = grad_mode
        self._kernel = kernel
        self._device = _device_index(device)
        self._hb_cutoff = 512
        self.soft_temperature = 1.0
        self.soft_impl = "scaled"
        self.soft_precision = "float32" if self._precision == 32 else "double"
        self._soft_guide = "eager"
        self.fill = "interpair"
        self.schedule = "dynamic"
        self.track_storage = "paths"
        self._tune = (0, 0)     # (lanes per pair, rows per lane): 0 = the planner's choice
        self._run_id = 0        # counts device runs (the autograd binding checks it)
        self._store = None
        self._n = 0
        self._params = None
        self._valid_scores = False
        self._valid_grads = False
        self._guides = None            # host copy, or None
        self._guides_pending = None    # params snapshot a deferred (soft) guide is due under
        self._have_guides = False
        self._paths = False
        if seqs_a is None:
            self._alpha = None
            return
        if params is None or not isinstance(params, AlignParams):
            raise TypeError("nwgrad: SeqPairBatch needs an AlignParams")
        if seqs_b is None or len(seqs_a) != len(seqs_b):
            raise ValueError("nwgrad: seqs_a and seqs_b need equal length")
        self._alpha = params.alphabet_obj
        self._params = params.copy()
        a, oa, sa = _encode_all(self._alpha, seqs_a, "A")
        b, ob, sb = _encode_all(self._alpha, seqs_b, "B")
        self._seqs_a, self._seqs_b = sa, sb
        self._n = len(sa)
        lens = np.diff(oa)
        K = self._params.num_sets
        tk, tgiven = _flat_tracks(tracks, lens, "tracks", 0)
        gk, ggiven = _flat_tracks(gap_tracks, lens, "gap_tracks", 1)
        self._tracked = tk is not None or gk is not None or K > 1
        flat_t = flat_g = None
        if tk is not None:
            if isinstance(tk, list):
                flat_t = np.zeros(int(lens.sum()), np.uint16)
                for p, t in enumerate(tk):
                    if t is not None:
                        flat_t[oa[p]:oa[p + 1]] = t
            else:
                flat_t = tk
        if gk is not None:
            flat_g = np.zeros(int(lens.sum()) + self._n, np.uint16)
            for p in range(self._n):
                lo = int(oa[p]) + p
                m = int(lens[p])
                if isinstance(gk, list) and gk[p] is not None:
                    flat_g[lo:lo + m + 1] = gk[p]
                elif not isinstance(gk, list):
                    flat_g[lo:lo + m + 1] = gk[lo:lo + m + 1]
                else:   # the default gap track of this pair, from its track
                    t = flat_t[oa[p]:oa[p + 1]] if flat_t is not None else np.zeros(m, np.uint16)
                    flat_g[lo] = t[0] if m else 0
                    flat_g[lo + 1:lo + m + 1] = t
        for name, arr in (("track", flat_t), ("gap_track", flat_g)):
            if arr is not None and arr.size and int(arr.max()) >= K:
                k = int(np.argmax(arr >= K))
                raise ValueError(f"nwgrad: {name}[{k}] = {int(arr[k])} is not a parameter set (params has {K})")
        self._oa, self._ob = oa, ob
        self._flat_t, self._flat_g = flat_t, flat_g
        self._store = _Store(a, oa, b, ob, self._alpha.size, flat_t, flat_g, self._device)
        self._push_params()

    @classmethod
    def from_codes(cls, codes_a, off_a, codes_b, off_b, params, **kw):
        """A batch from sequences already encoded in ``params``' alphabet: concatenated uint8
        codes with n_pairs + 1 int64 offsets per side (the store's own layout, uploaded as
        is).  Keywords as the constructor's; tracks / gap_tracks flat arrays only."""
        if not isinstance(params, AlignParams):
            raise TypeError("nwgrad: from_codes needs an AlignParams")
        self = cls.__new__(cls)
        rest = {k: v for k, v in kw.items() if k not in ("tracks", "gap_tracks")}
        cls.__init__(self, None, None, None, **rest)   # settings only; no pairs yet
        self._alpha = params.alphabet_obj
        self._params = params.copy()
        a = np.ascontiguousarray(codes_a, dtype=np.uint8)
        b = np.ascontiguousarray(codes_b, dtype=np.uint8)
        oa = np.ascontiguousarray(off_a, dtype=np.int64)
        ob = np.ascontiguousarray(off_b, dtype=np.int64)
        if oa.shape != ob.shape or oa.ndim != 1 or oa.size < 1:
            raise ValueError("nwgrad: off_a / off_b need n_pairs + 1 entries each")
        N = self._alpha.size   # codes >= N: the store refuses them (ValueError)
        tk = kw.get("tracks")
        gk = kw.get("gap_tracks")
        self._n = oa.size - 1
        self._oa, self._ob = oa - oa[0], ob - ob[0]
        self._seqs_a = self._seqs_b = None
        self._codes = (a, b)
        self._tracked = tk is not None or gk is not None or self._params.num_sets > 1
        tk = None if tk is None else np.ascontiguousarray(tk, dtype=np.uint16)
        gk = None if gk is None else np.ascontiguousarray(gk, dtype=np.uint16)
        self._flat_t, self._flat_g = tk, gk
        self._store = _Store(a if a.size else np.zeros(1, np.uint8), oa, b if b.size else np.zeros(1, np.uint8),
                             ob, N, tk, gk, self._device)
        self._push_params()
        return self

    # ── plumbing ──────────────────────────────────────────────────────────────
    def _push_params(self):
        p = self._params
        m = np.ascontiguousarray(p._m, dtype=np.float64)
        g = np.ascontiguousarray(p._g, dtype=np.float64)
        check(self._store._L.nwg_params_set(self._store.h, ptr(m, _capi._dp), ptr(g, _capi._dp),
                                            p.num_sets, p._alpha.size))

    def _job(self, grad_mode, band=-1, keep_paths=False):
        lanes, rows = self._tune
        soft_double = 1 if (self._precision == 64 or self.soft_precision == "double") else 0
        tb = {"hirschberg": 3, "hirschberg_pmax": 4, "grid": 5}.get(self._traceback, 0)
        if tb in (3, 4) and grad_mode != 2 and band < 0:
            self._check_hirschberg()
        if self._am == 2 and band >= 0 and self._sg != SG_GLOCAL:
            # aligner.hpp:2222-2231 (check_problem)
            raise ValueError("nwgrad: guide-banded alignment supports the semi-global ends of \"glocal\" "
                             "only; align these free ends with the full DP")
        return Job(_GAP[self._gap_model], self._am, grad_mode, self._precision, band,
                   int(bool(keep_paths)), float(self.soft_temperature), soft_double, lanes, rows,
                   tb, int(self._hb_cutoff), int(self._sg),
                   int(grad_mode == 2 and band < 0 and self._soft_guide == "posterior"))

    def _check_hirschberg(self):
        """Hirschberg splits pairs longer than hb_cutoff rows; this build implements the split
        for affine and linear gaps, Global, Local and glocal, tracked or not (the reference's
        viterbi_affine_hirschberg / _local / _glocal with hb_reverse_rows_ for tracks, and
        viterbi_linear_hirschberg) -- except linear glocal with tracks.  Other semi-global
        free-end sets run Pointers, as in the reference (aligner.hpp:2323-2330)."""
        if self._am != 2 or self._sg != SG_GLOCAL:
            return
        if self._tracked and self._gap_model == "linear" and self._n and \
                int(np.max(np.diff(self._oa))) > self._hb_cutoff:
            raise NotImplementedError(
                f"nwgrad_b200: traceback=\"{self._traceback}\" with mode \"{self._mode}\" splits tracked pairs "
                f"in this build only with affine gaps; use traceback=\"pointers\" or \"auto\"")

    @property
    def hb_cutoff(self) -> int:
        """Hirschberg base-case size in rows: pairs longer than this split."""
        return self._hb_cutoff

    @hb_cutoff.setter
    def hb_cutoff(self, v):
        v = int(v)
        if v < 1:
            raise ValueError("nwgrad: hb_cutoff must be >= 1")
        self._hb_cutoff = v

    def _run(self, grad_mode, band=-1, keep_paths=False, stream=None) -> float:
        if self._store is None:
            return 0.0
        job = self._job(grad_mode, band, keep_paths)
        self._run_id += 1
        self._path_cache = None
        tot = C.c_double(0.0)
        check(self._store._L.nwg_run(self._store.h, C.byref(job), stream, C.byref(tot)))
        return float(tot.value)

    def _gstride(self):
        K, N = self._params.num_sets, self._alpha.size
        return K * N * N + 4 * K

    def _vec_to_params(self, v) -> AlignParams:
        K, N = self._params.num_sets, self._alpha.size
        return AlignParams._make(v[:K * N * N].reshape(K, N, N).copy(), v[K * N * N:].reshape(K, 4).copy(),
                                 self._alpha)

    # ── batch operations ─────────────────────────────────────────────────────
    def __len__(self):
        return self._n

    def set_params(self, params: AlignParams):
        """Every pair gets a copy of params; clears scores, gradients and paths, keeps guides."""
        if not isinstance(params, AlignParams):
            raise TypeError("nwgrad: set_params needs an AlignParams")
        if self._alpha is not None and params.alphabet_obj is not self._alpha:
            raise ValueError(f"nwgrad: params alphabet \"{params.alphabet}\" does not match the batch's "
                             f"\"{self._alpha.symbols}\"")
        if self._params is not None and params.num_sets != self._params.num_sets:
            raise ValueError(f"nwgrad: set_params() cannot change the number of parameter sets "
                             f"({self._params.num_sets} -> {params.num_sets})")
        self._params = params.copy()
        if self._store is not None:
            self._push_params()
        self._valid_scores = self._valid_grads = False
        self._paths = False

    def score_and_grad(self, keep_paths: bool = False) -> float:
        """Full DP on every pair; returns the sum of scores in pair order."""
        gm = _GRAD[self._grad_mode]
        if gm == 2:
            tot = self._run(2)
            if self._soft_guide == "posterior":
                # the forward-backward left every pair's posterior guide
                self._guides_pending = None
                self._have_guides = True
            else:
                # the guide is deferred: computed on first use under the params scored now
                # ("eager") or under those current at that use ("lazy")
                self._guides_pending = self._params.copy() if self._soft_guide == "eager" else _CURRENT
                self._have_guides = False
            self._guides = None
            self._paths = False
        else:
            tot = self._run(gm, keep_paths=keep_paths)
            self._guides_pending = None
            self._have_guides = True
            self._guides = None
            self._paths = bool(keep_paths)
        self._valid_scores = True
        self._valid_grads = gm != 0
        return tot

    def banded_grad(self, bandwidth: int, keep_paths: bool = False) -> float:
        """Banded re-alignment + gradient around every pair's cached guide."""
        if int(bandwidth) <= 0:
            raise ValueError(f"nwgrad: banded_grad() needs bandwidth > 0 (got {bandwidth}); "
                             f"use score_and_grad() for full DP")
        self._resolve_guides()
        if not self._have_guides:
            raise RuntimeError("nwgrad: banded_grad() needs a guide; call score_and_grad() first")
        gm = _GRAD[self._grad_mode]
        tot = self._run(gm, band=int(bandwidth), keep_paths=keep_paths)
        self._valid_scores = True
        self._valid_grads = gm != 0
        self._paths = bool(keep_paths) and gm != 2
        self._guides = None
        return tot

    def _resolve_guides(self):
        """Compute deferred (soft) guides under the params snapshot they are due under; the
        batch's params and results are untouched (batch_soft_defer.inl)."""
        if self._guides_pending is None or self._store is None:
            return
        snap = self._params if self._guides_pending is _CURRENT else self._guides_pending
        m = np.ascontiguousarray(snap._m, dtype=np.float64)
        g = np.ascontiguousarray(snap._g, dtype=np.float64)
        job = self._job(0)
        check(self._store._L.nwg_resolve_guides(self._store.h, ptr(m, _capi._dp), ptr(g, _capi._dp),
                                                C.byref(job), None))
        self._guides_pending = None
        self._have_guides = True
        self._guides = None

    def _grads_raw(self) -> np.ndarray:
        out = np.zeros((self._n, self._gstride()), np.float64)
        if self._n:
            check(self._store._L.nwg_grads(self._store.h, ptr(out, _capi._dp)))
        return out

    def _check_grads(self):
        if self._grad_mode == "none":
            raise RuntimeError("nwgrad: grad_mode is None; construct with Hard or Soft to enable gradients")
        if not self._valid_grads:
            raise RuntimeError("nwgrad: gradient not computed; call score_and_grad() or banded_grad() first")

    def compute_grad(self) -> AlignParams:
        """The cached gradients summed over all pairs (fixed blocks of 4096, bit-reproducible)."""
        if self._n == 0:
            raise RuntimeError("nwgrad: empty batch")
        return self.weighted_grad(None)

    def weighted_grad(self, weights) -> AlignParams:
        """sum_i weights[i] * grad_i over the cached per-pair gradients."""
        if self._n == 0:
            raise RuntimeError("nwgrad: empty batch")
        self._check_grads()
        w = None
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.float64)
            if w.ndim != 1 or w.shape[0] != self._n:
                raise ValueError(f"nwgrad: weighted_grad needs one weight per pair ({self._n})")
        out = np.zeros(self._gstride(), np.float64)
        check(self._store._L.nwg_reduce(self._store.h, ptr(w, _capi._dp), ptr(out, _capi._dp)))
        return self._vec_to_params(out)

    def scores(self) -> np.ndarray:
        """The cached per-pair scores, in pair order."""
        if not self._valid_scores:
            raise RuntimeError("nwgrad: scores not computed; call score_and_grad() first")
        out = np.zeros(self._n, np.float64)
        if self._n:
            check(self._store._L.nwg_scores(self._store.h, ptr(out, _capi._dp)))
        return out

    def soft_status(self) -> np.ndarray:
        """Per pair, how the last soft pass computed it (low 8 bits): 0 in the batch's precision,
        1 refused by the float32 pass and computed in double -- the reference's kF32Refused flag
        (batch_engine.hpp:1285).  Bits 8 and up give the float32 pass's reasons: 1 a value out
        of range, 2 Z out of range, 4 a count's scale factor out of range, 8 a count out of
        range, 16 the lost-mass bound above 2^-24, 32 a weight out of range."""
        out = np.zeros(self._n, np.int32)
        if self._n:
            check(self._store._L.nwg_status(self._store.h, ptr(out, _capi._i32p)))
        return out

    def grads(self):
        """Per-pair gradients: (N, n, n) matrices and (N, 4) gaps; tracked: (N, K, n, n), (N, K, 4)."""
        if self._n == 0:
            raise RuntimeError("nwgrad: empty batch")
        self._check_grads()
        g = self._grads_raw()
        K, N = self._params.num_sets, self._alpha.size
        mats = g[:, :K * N * N].reshape(self._n, K, N, N)
        gaps = g[:, K * N * N:].reshape(self._n, K, 4)
        if not self._tracked:
            return mats[:, 0].copy(), gaps[:, 0].copy()
        return mats.copy(), gaps.copy()

    def guides(self) -> list:
        """Every pair's guide_j (m + 1 columns), resolving deferred guides first."""
        self._resolve_guides()
        if not self._have_guides:
            raise RuntimeError("nwgrad: no guide: run score_and_grad() first")
        if self._guides is None:
            g = np.zeros(int(self._oa[-1]) + self._n, np.int32)
            if g.size:
                check(self._store._L.nwg_guides(self._store.h, ptr(g, _capi._i32p)))
            self._guides = g
        return self._guides

    def align(self, seqs_a, seqs_b, params, band: int = 0, aligned_a=(), aligned_b=(), kernel="auto", *,
              tracks=None, gap_tracks=None) -> BatchResult:
        """Align (seqs_a[i], seqs_b[i]) under params WITHOUT adding them to this batch: the
        batch's problem type, grad mode and settings, one transient device store; returns the
        scores and the gradient summed over the pairs.  band > 0 bands every pair around the
        guide of aligned_a[i] / aligned_b[i] (the diagonal when none are given)."""
        if kernel not in _KERNELS:
            raise ValueError(f"nwgrad: unknown kernel \"{kernel}\"")
        if len(seqs_a) != len(seqs_b):
            raise ValueError("nwgrad: seqs_a and seqs_b need equal length")
        aligned_a, aligned_b = list(aligned_a), list(aligned_b)
        if (aligned_a or aligned_b) and (len(aligned_a) != len(seqs_a) or len(aligned_b) != len(seqs_a)):
            raise ValueError("nwgrad: aligned_a / aligned_b need one gapped string per pair")
        tmp = type(self)(seqs_a, seqs_b, params, gap_model=self._gap_model, mode=self._mode,
                         grad_mode=self._grad_mode, traceback=self._traceback, tracks=tracks,
                         gap_tracks=gap_tracks, device=self._device,
                         free_ends=self.free_ends if self._mode == "semiglobal" else None)
        tmp.soft_temperature = self.soft_temperature
        tmp.soft_precision = self.soft_precision
        tmp._hb_cutoff = self._hb_cutoff
        n = len(seqs_a)
        if n == 0:
            return BatchResult(np.zeros(0), AlignParams.zeros_like(params))
        if band and int(band) > 0:
            guides = []
            for i in range(n):
                m_i, n_i = len(seqs_a[i]), len(seqs_b[i])
                g = guide_j_from_aligned(aligned_a[i], aligned_b[i]) if aligned_a else _diagonal_guide(m_i, n_i)
                _validate_guide(g, m_i, n_i)
                guides.extend(g)
            gv = np.ascontiguousarray(guides, dtype=np.int32)
            check(tmp._store._L.nwg_set_guides(tmp._store.h, ptr(gv, _capi._i32p)))
            tmp._have_guides = True
            tmp._guides_pending = None
            gm = _GRAD[tmp._grad_mode]
            tmp._run(gm, band=int(band))
            tmp._valid_scores = True
            tmp._valid_grads = gm != 0
        else:
            tmp.score_and_grad()
        scores = tmp.scores()
        grad = tmp.compute_grad() if tmp._grad_mode != "none" else AlignParams.zeros_like(params)
        del tmp
        return BatchResult(scores, grad)

    def drop_paths(self):
        """Free the stored paths; scores, gradients and guides stay."""
        self._paths = False
        self._path_cache = None

    # ── stored paths (score_and_grad / banded_grad with keep_paths=True) ─────
    def _check_stored(self):
        if not self._valid_scores:
            raise RuntimeError("nwgrad: alignment not computed; call align() first")
        if not self._paths:
            raise RuntimeError("nwgrad: stored path unavailable; use align(keep_paths=True) or "
                               "banded_align(keep_paths=True)")

    def _stored(self):
        """(moves_off, moves in walk order, path_info [n_moves, start_i, start_j] per pair)."""
        self._check_stored()
        pc = getattr(self, "_path_cache", None)
        if pc is None:
            n = self._n
            mo = np.zeros(n + 1, np.int64)
            check(self._store._L.nwg_paths(self._store.h, ptr(mo, _capi._i64p), None, 0, None, None))
            mv = np.zeros(max(int(mo[-1]), 1), np.uint8)
            info = np.zeros(3 * max(n, 1), np.int32)
            check(self._store._L.nwg_paths(self._store.h, None, ptr(mv, _capi._u8p), int(mv.size),
                                           ptr(info, _capi._i32p), None))
            pc = (mo, mv, info.reshape(-1, 3))
            self._path_cache = pc
        return pc

    def _runs(self, i):
        """Pair i's path as (start_i, start_j, runs of (op, length)): op 0 aligned, 1 a residue
        of A against a gap, 2 a residue of B against a gap, start to end."""
        mo, mv, info = self._stored()
        k, si, sj = int(info[i, 0]), int(info[i, 1]), int(info[i, 2])
        ops = mv[mo[i]:mo[i] + k][::-1]
        runs = []
        for op in ops.tolist():
            if runs and runs[-1][0] == op:
                runs[-1][1] += 1
            else:
                runs.append([op, 1])
        return si, sj, runs

    def _codes_of(self, i):
        if getattr(self, "_codes", None) is not None:
            a, b = self._codes
            return a[self._oa[i]:self._oa[i + 1]], b[self._ob[i]:self._ob[i + 1]]
        return (self._alpha.encode(self._seqs_a[i]), self._alpha.encode(self._seqs_b[i]))

    def aligned(self, i: int):
        """Pair i's stored alignment as two gapped strings (batch_engine.hpp:515-535)."""
        si, sj, runs = self._runs(i)
        ca, cb = self._codes_of(i)
        sym = self._alpha.symbols
        a, b = [], []
        ia, jb = si, sj
        for op, ln in runs:
            a.append("".join(sym[x] for x in ca[ia:ia + ln]) if op != 2 else "-" * ln)
            b.append("".join(sym[x] for x in cb[jb:jb + ln]) if op != 1 else "-" * ln)
            if op != 2:
                ia += ln
            if op != 1:
                jb += ln
        return "".join(a), "".join(b)

    def coordinates(self, i: int) -> np.ndarray:
        """Biopython-style coordinates (2, k) of pair i's stored alignment (batch_engine.hpp:536-550)."""
        si, sj, runs = self._runs(i)
        x, y = si, sj
        ci, cj = [x], [y]
        for k, (op, ln) in enumerate(runs):
            if op != 2:
                x += ln
            if op != 1:
                y += ln
            if k + 1 < len(runs):
                ci.append(x); cj.append(y)
        ci.append(x); cj.append(y)
        return np.array([ci, cj], dtype=np.int64)

    def cigar(self, i: int, extended: bool = False, soft_clip: bool = False) -> str:
        """Pair i's stored alignment as a SAM CIGAR, seq_a the query (batch_engine.hpp:557-582)."""
        si, sj, runs = self._runs(i)
        ca, cb = self._codes_of(i)
        out = []
        state = {"op": None, "run": 0}

        def emit(op, n):
            if not n:
                return
            if op == state["op"]:
                state["run"] += n
                return
            if state["run"]:
                out.append(f"{state['run']}{state['op']}")
            state["op"], state["run"] = op, n

        if soft_clip:
            emit("S", si)
        ia, jb = si, sj
        for op, ln in runs:
            if op == 1:
                emit("I", ln); ia += ln
            elif op == 2:
                emit("D", ln); jb += ln
            elif not extended:
                emit("M", ln); ia += ln; jb += ln
            else:
                for _ in range(ln):
                    emit("=" if ca[ia] == cb[jb] else "X", 1)
                    ia += 1; jb += 1
        if soft_clip:
            emit("S", len(ca) - ia)
        if state["run"]:
            out.append(f"{state['run']}{state['op']}")
        return "".join(out)

    def cigars(self, extended: bool = False, soft_clip: bool = False) -> list:
        """Every pair's cigar(), in pair order."""
        return [self.cigar(i, extended, soft_clip) for i in range(self._n)]

    def __getitem__(self, i: int):
        n = self._n
        if i < 0:
            i += n
        if not 0 <= i < n:
            raise IndexError("SeqPairBatch index out of range")
        return SeqPair._view(self, i)

    # ── properties ───────────────────────────────────────────────────────────
    @property
    def n_threads(self):
        return self._n_threads

    @n_threads.setter
    def n_threads(self, v):
        if int(v) < 0:
            raise ValueError(f"nwgrad: n_threads must be >= 0 (0: the default thread count), got {v}")
        self._n_threads = int(v)

    @property
    def gap_model(self):
        return self._gap_model

    @property
    def mode(self):
        return self._mode

    @property
    def soft_guide(self):
        """When soft pairs compute their guide path (the Viterbi path banded_grad() bands
        around): "eager" (default) under the params score_and_grad() ran with, computed on
        first use from a snapshot of them; "lazy" under the params current at first use
        (after set_params() it follows the new params).  "posterior": the forward-backward's own
        guide -- per row the column of greatest exit mass, made non-decreasing -- left by
        score_and_grad() itself (full DP, untracked batches)."""
        return self._soft_guide

    @soft_guide.setter
    def soft_guide(self, v):
        if v not in ("eager", "lazy", "posterior"):
            raise ValueError(f"nwgrad: unknown soft_guide \"{v}\" (expected \"eager\", \"lazy\" or \"posterior\")")
        if v == "posterior" and self._tracked:
            raise NotImplementedError("nwgrad_b200: soft_guide=\"posterior\" is built for untracked batches; "
                                      "use \"eager\" or \"lazy\" with tracks")
        self._soft_guide = v

    @property
    def free_ends(self):
        """(a_begin, a_end, b_begin, b_end): which flanks are free; None for local."""
        if self._am == 1:
            return None
        sg = self._sg if self._am == 2 else 0
        return tuple(bool(sg & b) for b in _SG_BITS)

    @property
    def grad_mode(self):
        return self._grad_mode

    @property
    def traceback(self):
        return self._traceback

    @property
    def alphabet(self) -> str:
        if self._alpha is None or self._n == 0:
            raise RuntimeError("nwgrad: empty batch has no alphabet")
        return self._alpha.symbols

    @property
    def tracked(self) -> bool:
        return bool(getattr(self, "_tracked", False))

    @property
    def params(self) -> AlignParams:
        return self._params.copy()

    def autotune(self, sample_pairs: int = 65536, force: bool = False, verbose: bool = False) -> dict:
        """Pick the fastest kernel geometry per size class of this batch (measured on a sample of
        its own pairs, cached per device and problem type) and use it from now on.  Results do
        not change: every geometry computes the same cells.  Returns {size class: (lanes, rows)}."""
        from . import tune
        if self._store is None or self._n == 0:
            return {}
        table = tune.tune(self, sample_pairs=sample_pairs, force=force, verbose=verbose)
        tune.apply(self, table)
        return table

    def use_plain_fill(self) -> None:
        """Run every pair with one fixed geometry (32 lanes x 4 rows), bucketed by size only:
        the untuned baseline the autotuner is measured against."""
        from . import tune
        if self._store is not None:
            tune.plain(self)

    def set_memory(self, scratch_budget_bytes: int = -1, checkpoint_bytes: int = -1) -> None:
        """Device memory of soft runs: the forward-table budget of one call, and the per-pair
        table size above which only stripe boundaries are kept and each stripe is recomputed
        before its backward (bit-identical results).  -1 keeps the current value."""
        check(self._store._L.nwg_set_memory(self._store.h, int(scratch_budget_bytes), int(checkpoint_bytes)))

    def set_spin_limit(self, polls: int = 1 << 22) -> None:
        """Polls a wait between the warps of one long pair (soft gradient) makes before it gives
        up: the call then raises RuntimeError instead of hanging, and the batch stays usable."""
        check(self._store._L.nwg_set_spin_limit(self._store.h, int(polls)))

    def use_graphs(self, enable: bool = True) -> None:
        """Run each plan's per-bucket launches as one captured CUDA graph (the default): captured
        the second time the same launches run (a batch run once launches directly), replayed
        while they are unchanged (set_params steps keep them); False launches every bucket
        directly.  Results are the same either way."""
        check(self._store._L.nwg_set_graphs(self._store.h, 1 if enable else 0))

    def graph_stats(self):
        """(captures, replays) of bucket-sequence graphs since the batch was made."""
        cap = C.c_int64(0)
        rep = C.c_int64(0)
        check(self._store._L.nwg_graph_stats(self._store.h, C.byref(cap), C.byref(rep)))
        return int(cap.value), int(rep.value)

    def last_timing(self):
        """(device ms, kernel launches) of the last GPU call."""
        ms = C.c_double(0)
        n = C.c_int64(0)
        check(self._store._L.nwg_last_timing(self._store.h, C.byref(ms), C.byref(n)))
        return float(ms.value), int(n.value)


def guide_j_from_aligned(a_aligned: str, b_aligned: str) -> list:
    """The guide of a gapped alignment: guide[i] = the column of B reached after i residues of
    A (aligner.hpp:171-190)."""
    if len(a_aligned) != len(b_aligned):
        raise ValueError("aligned strings must have equal length")
    gj = [0]
    j = 0
    for x, y in zip(a_aligned, b_aligned):
        ag, bg = x == "-", y == "-"
        if ag and bg:
            raise ValueError("aligned strings have a column with two gaps")
        if not ag and not bg:
            j += 1
            gj.append(j)
        elif ag:
            j += 1
        else:
            gj.append(j)
    return gj


def _diagonal_guide(m: int, n: int) -> list:
    """round(i * n / m), halves away from zero (aligner.hpp:1781-1789)."""
    if m == 0:
        return [0]
    return [int(np.floor(i * n / m + 0.5)) for i in range(m + 1)]


def _validate_guide(g, m: int, n: int):
    """A guide must describe the pair: m + 1 columns of B, never moving left."""
    if len(g) != m + 1:
        raise ValueError(f"nwgrad: guide_j has {len(g)} entries, but sequence A of length {m} needs {m + 1}")
    for i, v in enumerate(g):
        if v < 0 or v > n:
            raise ValueError(f"nwgrad: guide_j[{i}] = {v} is outside [0, {n}] for sequence B of length {n}")
        if i > 0 and v < g[i - 1]:
            raise ValueError(f"nwgrad: guide_j decreases at row {i} ({g[i - 1]} -> {v})")


class BatchResult:
    """What a streaming align() returns: the pairs' scores and their summed gradient."""

    def __init__(self, scores: np.ndarray, grad: AlignParams):
        self._scores = scores
        self._grad = grad

    @property
    def scores(self) -> np.ndarray:
        """Alignment scores, shape (N,)."""
        return self._scores

    @property
    def grad(self) -> AlignParams:
        """Summed gradient over the batch as an AlignParams object."""
        return self._grad

    def __repr__(self):
        return f"BatchResult(n={len(self._scores)})"


class SeqPairBatchDouble(SeqPairBatch):
    """SeqPairBatch with the DP in float64."""
    _precision = 64


class SeqPair:
    """One pair: a view of pair i of a batch, or a standalone pair (a one-pair batch)."""

    def __init__(self, seq_a, seq_b, params, gap_model="affine", mode="global", grad_mode="hard",
                 kernel="auto", traceback="auto", *, track=None, gap_track=None, free_ends=None, device=None):
        cls = SeqPairBatchDouble if getattr(self, "_double", False) else SeqPairBatch
        self._batch = cls([seq_a], [seq_b], params, traceback=traceback, gap_model=gap_model, mode=mode,
                          grad_mode=grad_mode, kernel=kernel, free_ends=free_ends,
                          tracks=None if track is None else [track],
                          gap_tracks=None if gap_track is None else [gap_track], device=device)
        self._i = 0
        self._standalone = True

    @classmethod
    def _view(cls, batch, i):
        o = cls.__new__(cls)
        o._batch = batch
        o._i = i
        o._standalone = False
        return o

    def align(self, keep_paths=True) -> float:
        self._batch.score_and_grad(keep_paths=keep_paths)
        return self.score

    def score_and_grad(self, keep_paths=True):
        if self._batch.grad_mode == "none":
            raise RuntimeError("nwgrad: grad_mode is \"none\": use align()")
        self._batch.score_and_grad(keep_paths=keep_paths)
        return self.score, self.grad

    def banded_align(self, bandwidth, keep_paths=True) -> float:
        self._batch.banded_grad(bandwidth, keep_paths=keep_paths)
        return self.score

    def aligned(self):
        """The alignment as a pair of gapped strings (seq_a, seq_b)."""
        return self._batch.aligned(self._i)

    def coordinates(self) -> np.ndarray:
        """The alignment as Biopython-style coordinates, an int64 array of shape (2, k)."""
        return self._batch.coordinates(self._i)

    def cigar(self, *, extended: bool = False, soft_clip: bool = False) -> str:
        """The alignment as a SAM CIGAR string, seq_a the query and seq_b the reference."""
        return self._batch.cigar(self._i, extended, soft_clip)

    def formatted(self, width: int = 60) -> str:
        """Pretty-printed alignment block, wrapped at `width` columns (0 = no wrap)."""
        a, b = self.aligned()
        match = "".join(" " if (x == "-" or y == "-") else ("|" if x == y else ".") for x, y in zip(a, b))
        if width <= 0:
            width = len(a)
        blocks = []
        for off in range(0, len(a), max(width, 1)):
            blocks.append(a[off:off + width] + "\n" + match[off:off + width] + "\n" + b[off:off + width])
        return "\n\n".join(blocks)

    def drop_paths(self):
        self._batch.drop_paths()

    @property
    def stored_path_valid(self):
        b = self._batch
        return bool(b._valid_scores and b._paths)

    def set_params(self, params):
        if not self._standalone:
            raise RuntimeError("nwgrad: a batch view's params belong to the batch; set them on the batch")
        self._batch.set_params(params)

    @property
    def score(self):
        if not self._batch._valid_scores:
            return None
        return float(self._batch.scores()[self._i])

    @property
    def grad(self):
        b = self._batch
        if not b._valid_grads or b.grad_mode == "none":
            return None
        g = b._grads_raw()[self._i]
        return b._vec_to_params(g)

    @property
    def guide_j(self):
        b = self._batch
        try:
            g = b.guides()
        except RuntimeError:
            return None
        lo = int(b._oa[self._i]) + self._i
        m = int(b._oa[self._i + 1] - b._oa[self._i])
        return [int(x) for x in g[lo:lo + m + 1]]

    @property
    def seq_a(self):
        b = self._batch
        if b._seqs_a is None:
            a, _ = b._codes
            return b._alpha.decode(a[b._oa[self._i]:b._oa[self._i + 1]])
        return b._seqs_a[self._i]

    @property
    def seq_b(self):
        b = self._batch
        if b._seqs_b is None:
            _, bb = b._codes
            return b._alpha.decode(bb[b._ob[self._i]:b._ob[self._i + 1]])
        return b._seqs_b[self._i]

    @property
    def gap_model(self):
        return self._batch.gap_model

    @property
    def mode(self):
        return self._batch.mode

    @property
    def free_ends(self):
        return self._batch.free_ends

    @property
    def grad_mode(self):
        return self._batch.grad_mode

    @property
    def score_valid(self):
        return self._batch._valid_scores

    @property
    def grad_valid(self):
        return self._batch._valid_grads

    @property
    def path_valid(self):
        b = self._batch
        return b._have_guides or b._guides_pending is not None


class SeqPairDouble(SeqPair):
    _double = True
