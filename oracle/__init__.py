"""CPU oracle for the SeqPairBatch alignment path -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this
package, and only as the checker (or the timed CPU baseline); the product package
``nwgrad_b200`` never imports it.

Two back ends:

* ``liboracle.so`` -- the restatement of the reference's scalar algorithms in
  ``oracle/oracle.cpp`` (built by ``make -C oracle liboracle``), bit-exact for the hard path
  and a log-space double forward-backward for the soft path.
* ``_ref/libnwref*.so`` -- the reference's own C++ (michalsta/nwgrad, header-only core plus,
  for ``libnwref.so``, its SIMD level units) behind ``ref_driver.cpp``; built from the
  reference sources by ``make -C oracle ref`` / ``ref-simd`` where they are present.  Used to
  pin the restatement and as the CPU baseline.  Absent on a machine without the reference
  sources unless the built library travelled with the tree.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = {}

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_u16p = C.POINTER(C.c_uint16)


def build():
    """Compile liboracle.so (the restatement) in place."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(os.path.join(HERE, "oracle.cpp")):
            build()
        L = C.CDLL(path)
        L.orc_hard_batch.argtypes = [C.c_int] * 5 + [_dp, _dp, _u8p, _i64p, _u8p, _i64p, C.c_int64,
                                                      _u16p, _u16p, C.c_int, _i32p, C.c_int,
                                                      _dp, _dp, _i32p, _u8p, C.c_int64, _i64p, _i32p, C.c_int]
        L.orc_hard_batch.restype = C.c_int
        L.orc_soft_batch.argtypes = [C.c_int] * 4 + [_dp, _dp, _u8p, _i64p, _u8p, _i64p, C.c_int64,
                                                      _u16p, _u16p, C.c_double, _dp, _dp, _i32p, C.c_int, C.c_int,
                                                      _i32p]
        L.orc_soft_batch.restype = C.c_int
        L.orc_hb_batch.argtypes = [C.c_int] * 4 + [_dp, _dp, _u8p, _i64p, _u8p, _i64p, C.c_int64,
                                                    _dp, _dp, _i32p, _u8p, C.c_int64, _i64p, C.c_int, _i32p, C.c_int,
                                                    C.c_int, _u16p, _u16p]
        L.orc_hb_batch.restype = C.c_int
        L.orc_blocked_sum.argtypes = [_dp, C.c_int64, C.c_int64, _dp, _dp]
        L.orc_blocked_sum.restype = C.c_int
        _lib = L
    return _lib


def _p(x, t):
    return None if x is None else x.ctypes.data_as(t)


class Encoded:
    """A batch of pairs as the oracle reads it: concatenated u8 codes and int64 offsets."""

    def __init__(self, a_codes, b_codes, tracks=None, gap_tracks=None):
        self.la = np.array([len(x) for x in a_codes], dtype=np.int64)
        self.lb = np.array([len(x) for x in b_codes], dtype=np.int64)
        self.oa = np.zeros(len(a_codes) + 1, np.int64)
        self.ob = np.zeros(len(b_codes) + 1, np.int64)
        self.oa[1:] = np.cumsum(self.la)
        self.ob[1:] = np.cumsum(self.lb)
        self.a = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint8) for x in a_codes]) if len(a_codes) else np.zeros(0, np.uint8), dtype=np.uint8)
        self.b = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint8) for x in b_codes]) if len(b_codes) else np.zeros(0, np.uint8), dtype=np.uint8)
        if self.a.size == 0:
            self.a = np.zeros(1, np.uint8)
        if self.b.size == 0:
            self.b = np.zeros(1, np.uint8)
        self.n = len(a_codes)
        self.tracks = None if tracks is None else np.ascontiguousarray(tracks, dtype=np.uint16)
        self.gap_tracks = None if gap_tracks is None else np.ascontiguousarray(gap_tracks, dtype=np.uint16)


def hard(prec, gm, am, mat, gaps, enc: Encoded, tracked=False, guides_in=None, band=-1,
         moves_cap=0, free_ends=12):
    """Viterbi (Pointers semantics) + traceback + hard gradient for every pair.  am: 0 global,
    1 local, 2 semi-global with `free_ends` (1 a_begin, 2 a_end, 4 b_begin, 8 b_end; 12 glocal).

    Returns dict(scores (n,), grads (n, K*N*N + 4K), guides (sum(m+1),), ends (n, 4)
    [end_i, end_j, start_i, start_j], moves (n, moves_cap) walk order, nmoves (n,)).
    """
    L = lib()
    mat = np.ascontiguousarray(mat, np.float64)
    gaps = np.ascontiguousarray(gaps, np.float64)
    K, N = mat.shape[0], mat.shape[1]
    gs = K * N * N + 4 * K
    n = enc.n
    scores = np.zeros(n, np.float64)
    grads = np.zeros((n, gs), np.float64)
    guides = np.zeros(int(enc.oa[-1]) + n, np.int32)
    ends = np.zeros((n, 4), np.int32)
    nmoves = np.zeros(n, np.int64)
    moves = np.zeros((n, max(moves_cap, 1)), np.uint8) if moves_cap else None
    gi = None if guides_in is None else np.ascontiguousarray(guides_in, np.int32)
    rc = L.orc_hard_batch(prec, gm, am, N, K, _p(mat, _dp), _p(gaps, _dp), _p(enc.a, _u8p),
                          _p(enc.oa, _i64p), _p(enc.b, _u8p), _p(enc.ob, _i64p), n,
                          _p(enc.tracks, _u16p), _p(enc.gap_tracks, _u16p), int(bool(tracked)),
                          _p(gi, _i32p), int(band), _p(scores, _dp), _p(grads, _dp),
                          _p(guides, _i32p), _p(moves, _u8p), int(moves_cap), _p(nmoves, _i64p),
                          _p(ends, _i32p), int(free_ends))
    assert rc == 0
    return dict(scores=scores, grads=grads, guides=guides, ends=ends, moves=moves, nmoves=nmoves)


def hirschberg(prec, mat, gaps, enc: Encoded, cutoff=512, pmax=False, moves_cap=0, local=False, linear=False):
    """Hirschberg, affine (untracked, one parameter set) or linear (tracked or not: enc's tracks,
    K sets).  Pairs longer than `cutoff` rows split, shorter ones run the Pointers path; Local:
    the endpoint scans give the box that is solved as Global (pmax: the affine prefix-max
    carry; linear has one sweep).  Returns dict(scores, grads, guides, moves (n, moves_cap)
    path order start to end, nmoves, ends (n, 4): start i, start j, end i, end j)."""
    L = lib()
    N = np.shape(mat)[-1]
    mat = np.ascontiguousarray(mat, np.float64).reshape(-1, N, N)
    gaps = np.ascontiguousarray(gaps, np.float64).reshape(-1, 4)
    if not linear:
        mat, gaps = mat[:1], gaps[:1]
    K = mat.shape[0]
    n = enc.n
    scores = np.zeros(n, np.float64)
    grads = np.zeros((n, K * N * N + 4 * K), np.float64)
    guides = np.zeros(int(enc.oa[-1]) + n, np.int32)
    nmoves = np.zeros(n, np.int64)
    moves = np.zeros((n, max(moves_cap, 1)), np.uint8) if moves_cap else None
    ends = np.zeros((n, 4), np.int32)
    tk = enc.tracks if linear else None
    gk = enc.gap_tracks if linear else None
    rc = L.orc_hb_batch(prec, int(bool(pmax)), int(cutoff), N, _p(mat, _dp), _p(gaps, _dp), _p(enc.a, _u8p),
                        _p(enc.oa, _i64p), _p(enc.b, _u8p), _p(enc.ob, _i64p), n, _p(scores, _dp),
                        _p(grads, _dp), _p(guides, _i32p), _p(moves, _u8p), int(moves_cap), _p(nmoves, _i64p),
                        int(bool(local)), _p(ends, _i32p), int(bool(linear)), int(K), _p(tk, _u16p), _p(gk, _u16p))
    assert rc == 0
    return dict(scores=scores, grads=grads, guides=guides, moves=moves, nmoves=nmoves, ends=ends)


def soft(gm, am, mat, gaps, enc: Encoded, temperature=1.0, guides_in=None, band=-1, free_ends=12,
         posterior=False):
    """Log-space double forward-backward: (scores = T log Z, grads = expected counts); with
    guides_in and band >= 0 the guide-banded one; posterior=True adds the posterior guides
    (m + 1 columns per pair at off_a[p] + p, the reference's posterior_rows_log)."""
    L = lib()
    mat = np.ascontiguousarray(mat, np.float64)
    gaps = np.ascontiguousarray(gaps, np.float64)
    K, N = mat.shape[0], mat.shape[1]
    gs = K * N * N + 4 * K
    scores = np.zeros(enc.n, np.float64)
    grads = np.zeros((enc.n, gs), np.float64)
    post = np.zeros(int(enc.oa[-1]) + enc.n + 1, np.int32) if posterior else None
    rc = L.orc_soft_batch(gm, am, N, K, _p(mat, _dp), _p(gaps, _dp), _p(enc.a, _u8p),
                          _p(enc.oa, _i64p), _p(enc.b, _u8p), _p(enc.ob, _i64p), enc.n,
                          _p(enc.tracks, _u16p), _p(enc.gap_tracks, _u16p), float(temperature),
                          _p(scores, _dp), _p(grads, _dp),
                          _p(None if guides_in is None else np.ascontiguousarray(guides_in, np.int32), _i32p),
                          int(band), int(free_ends), _p(post, _i32p))
    assert rc == 0
    return (scores, grads, post) if posterior else (scores, grads)


def blocked_sum(grads, weights=None):
    """sum_p w[p] * grads[p], in the reference's fixed blocks of 4096 pairs."""
    L = lib()
    g = np.ascontiguousarray(grads, np.float64)
    out = np.zeros(g.shape[1], np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    L.orc_blocked_sum(_p(g, _dp), g.shape[0], g.shape[1], _p(w, _dp), _p(out, _dp))
    return out


# ── the reference itself (oracle/_ref) ───────────────────────────────────────

class _Problem(C.Structure):
    _fields_ = [("prec", C.c_int), ("gm", C.c_int), ("am", C.c_int), ("grad_mode", C.c_int),
                ("N", C.c_int), ("K", C.c_int), ("mat", _dp), ("gaps", _dp),
                ("alphabet", C.c_char_p), ("n_pairs", C.c_int64),
                ("a", C.c_char_p), ("oa", _i64p), ("b", C.c_char_p), ("ob", _i64p),
                ("tracks", _u16p), ("gtracks", _u16p), ("traceback", C.c_int), ("kernel", C.c_int),
                ("n_threads", C.c_int), ("temperature", C.c_double), ("soft_impl", C.c_int),
                ("soft_f32", C.c_int), ("hb_cutoff", C.c_int), ("inter_fill", C.c_int),
                ("free_ends", C.c_int), ("soft_guide", C.c_int)]


def ref_available(simd=False):
    name = "libnwref.so" if simd else "libnwref_scalar.so"
    return os.path.exists(os.path.join(HERE, "_ref", name))


def ref_lib(simd=False):
    name = "libnwref.so" if simd else "libnwref_scalar.so"
    if name not in _ref:
        L = C.CDLL(os.path.join(HERE, "_ref", name))
        L.ref_run.argtypes = [C.POINTER(_Problem), _dp, _dp, C.c_int, _dp, _dp, _i32p, _dp]
        L.ref_run.restype = C.c_int
        L.ref_time.argtypes = [C.POINTER(_Problem), C.c_int, C.c_int, _dp, _dp]
        L.ref_time.restype = C.c_int
        L.ref_info.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_char_p, C.c_int]
        L.ref_info.restype = C.c_int
        L.ref_last_error.restype = C.c_char_p
        _ref[name] = L
    return _ref[name]


_TB = {"auto": 0, "pointers": 1, "scores": 2, "hirschberg": 3, "hirschberg_pmax": 4, "grid": 5}


def _problem(prec, gm, am, grad_mode, alphabet, mat, gaps, seqs_a, seqs_b, tracks, gap_tracks,
             traceback, kernel, n_threads, temperature, soft_impl, soft_f32, hb_cutoff, inter_fill,
             free_ends=12, soft_guide=0):
    keep = []
    mat = np.ascontiguousarray(mat, np.float64)
    gaps = np.ascontiguousarray(gaps, np.float64)
    la = np.array([len(s) for s in seqs_a], np.int64)
    lb = np.array([len(s) for s in seqs_b], np.int64)
    oa = np.zeros(len(seqs_a) + 1, np.int64); oa[1:] = np.cumsum(la)
    ob = np.zeros(len(seqs_b) + 1, np.int64); ob[1:] = np.cumsum(lb)
    a = ("".join(seqs_a) + "\0").encode()
    b = ("".join(seqs_b) + "\0").encode()
    tk = None if tracks is None else np.ascontiguousarray(tracks, np.uint16)
    gk = None if gap_tracks is None else np.ascontiguousarray(gap_tracks, np.uint16)
    keep += [mat, gaps, oa, ob, a, b, tk, gk]
    alpha = alphabet.encode()
    keep.append(alpha)
    P = _Problem(prec, gm, am, grad_mode, mat.shape[1], mat.shape[0], _p(mat, _dp), _p(gaps, _dp),
                 alpha, len(seqs_a), a, _p(oa, _i64p), b, _p(ob, _i64p), _p(tk, _u16p),
                 _p(gk, _u16p), _TB[traceback], kernel, n_threads, float(temperature),
                 soft_impl, int(soft_f32), hb_cutoff, int(inter_fill), int(free_ends), int(soft_guide))
    return P, keep, oa


def ref_run(prec, gm, am, grad_mode, alphabet, mat, gaps, seqs_a, seqs_b, tracks=None,
            gap_tracks=None, traceback="pointers", kernel=-1, n_threads=1, temperature=1.0,
            soft_impl=0, soft_f32=True, hb_cutoff=0, inter_fill=True, band=-1, mat2=None,
            gaps2=None, simd=False, free_ends=12, soft_guide=0):
    """Run the reference batch once; returns dict(scores, grads, guides, total).  soft_guide: 0
    eager, 1 lazy, 2 posterior (the guides a soft run leaves)."""
    L = ref_lib(simd)
    if n_threads <= 0:
        n_threads = physical_cores()
    P, keep, oa = _problem(prec, gm, am, grad_mode, alphabet, mat, gaps, seqs_a, seqs_b, tracks,
                           gap_tracks, traceback, kernel, n_threads, temperature, soft_impl,
                           soft_f32, hb_cutoff, inter_fill, free_ends, soft_guide)
    K, N = np.asarray(mat).shape[0], np.asarray(mat).shape[1]
    n = len(seqs_a)
    scores = np.zeros(n, np.float64)
    grads = np.zeros((n, K * N * N + 4 * K), np.float64)
    guides = np.zeros(int(oa[-1]) + n, np.int32)
    total = np.zeros(1, np.float64)
    m2 = None if mat2 is None else np.ascontiguousarray(mat2, np.float64)
    g2 = None if gaps2 is None else np.ascontiguousarray(gaps2, np.float64)
    rc = L.ref_run(C.byref(P), _p(m2, _dp), _p(g2, _dp), int(band), _p(scores, _dp),
                   _p(grads, _dp) if grad_mode else None, _p(guides, _i32p), _p(total, _dp))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    return dict(scores=scores, grads=grads, guides=guides, total=float(total[0]))


def ref_time(prec, gm, am, grad_mode, alphabet, mat, gaps, seqs_a, seqs_b, tracks=None,
             gap_tracks=None, traceback="auto", kernel=-2, n_threads=0, temperature=1.0,
             warmup=1, reps=3, simd=True):
    """Time the reference's own batch path: per-pass seconds of score_and_grad()+compute_grad()."""
    L = ref_lib(simd)
    if n_threads <= 0:
        n_threads = physical_cores()
    P, keep, _ = _problem(prec, gm, am, grad_mode, alphabet, mat, gaps, seqs_a, seqs_b, tracks,
                          gap_tracks, traceback, kernel, n_threads, temperature, 0, True, 0, True)
    secs = np.zeros(reps, np.float64)
    total = np.zeros(1, np.float64)
    rc = L.ref_time(C.byref(P), warmup, reps, _p(secs, _dp), _p(total, _dp))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    return secs, float(total[0])


def physical_cores() -> int:
    """Physical cores among the CPUs this process may run on (the reference's default
    n_threads, parallel.hpp:165), counted here: the reference's own probe crashes when it
    runs inside a process that has numpy loaded."""
    cpus = sorted(os.sched_getaffinity(0))
    seen = set()
    for c in cpus:
        try:
            pkg = open(f"/sys/devices/system/cpu/cpu{c}/topology/physical_package_id").read().strip()
            core = open(f"/sys/devices/system/cpu/cpu{c}/topology/core_id").read().strip()
            seen.add((pkg, core))
        except OSError:
            seen.add(("?", str(c)))
    return max(1, len(seen))


def ref_bench_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "nwref_bench"))


def ref_time_codes(prec, gm, am, grad_mode, alphabet, mat, gaps, a, oa, b, ob, n_threads=0,
                   warmup=1, reps=3, kernel=-2, free_ends=12):
    """Time the reference's SIMD batch path (score_and_grad + compute_grad per pass) in its
    own process (_ref/nwref_bench) on pairs given as codes: returns (seconds per pass,
    total, threads, isa)."""
    import json
    import tempfile
    if n_threads <= 0:
        n_threads = physical_cores()
    mat = np.ascontiguousarray(mat, np.float64)
    gaps = np.ascontiguousarray(gaps, np.float64)
    K, N = mat.shape[0], mat.shape[1]
    sym = np.frombuffer(alphabet.encode(), dtype=np.uint8)
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        f.write(np.array([prec, gm, am, grad_mode, N, K, n_threads, warmup, reps, kernel, free_ends],
                         np.int32).tobytes())
        f.write(np.array([len(oa) - 1], np.int64).tobytes())
        f.write(np.array([len(alphabet)], np.int32).tobytes())
        f.write(alphabet.encode())
        f.write(mat.tobytes())
        f.write(gaps.tobytes())
        f.write(np.ascontiguousarray(oa - oa[0], np.int64).tobytes())
        f.write(sym[np.asarray(a[oa[0]:oa[-1]], np.int64)].tobytes())
        f.write(np.ascontiguousarray(ob - ob[0], np.int64).tobytes())
        f.write(sym[np.asarray(b[ob[0]:ob[-1]], np.int64)].tobytes())
        path = f.name
    try:
        r = subprocess.run([os.path.join(HERE, "_ref", "nwref_bench"), path], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nwref_bench failed: " + r.stderr.strip())
        out = json.loads(r.stdout.strip().splitlines()[-1])
    finally:
        os.unlink(path)
    return np.array(out["secs"]), out["total"], out["threads"], out["isa"]


def ref_info(n_threads=0, simd=True):
    if n_threads <= 0:
        n_threads = physical_cores()
    L = ref_lib(simd)
    r = C.c_int(0)
    buf = C.create_string_buffer(64)
    L.ref_info(n_threads, C.byref(r), buf, 64)
    return r.value, buf.value.decode()
