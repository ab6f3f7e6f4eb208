"""Semi-global ends on the GPU: mode "glocal" (A within B: row 0 a free start, row m's cells
ends), "overlap" (every flank free) and mode "semiglobal" with any free_ends set.

Hard results (scores, per-pair gradients, guides, stored paths) bit for bit the reference's
fixtures and the oracle's; soft within 1e-4 of the double log-space forward-backward.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402

SOFT_RTOL = 1e-4
SG_SETS = (12, 15, 9, 6, 3, 0)    # free_ends bits: 1 a_begin, 2 a_end, 4 b_begin, 8 b_end
NAMES = ("a_begin", "a_end", "b_begin", "b_end")


def _mode_kw(fe):
    """The API spelling of a free_ends bit set."""
    if fe == 12:
        return dict(mode="glocal")
    if fe == 15:
        return dict(mode="overlap")
    return dict(mode="semiglobal", free_ends=tuple(bool(fe & (1 << k)) for k in range(4)))


def _flat(b, n):
    gmat, ggap = b.grads()
    if gmat.ndim == 3:
        gmat, ggap = gmat[:, None], ggap[:, None]
    return np.concatenate([gmat.reshape(n, -1), ggap.reshape(n, -1)], axis=1)


def _soft_close(flat, ref):
    scale = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1.0)
    err = np.abs(flat - ref) / scale
    assert err.max() <= SOFT_RTOL, (err.max(), np.unravel_index(err.argmax(), err.shape))


@pytest.mark.parametrize("name", ["prot", "protf", "rna3"])
def test_semiglobal_reference_fixtures(name):
    """The GPU path against the reference engine's own semi-global outputs."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "semiglobal.npz"))
    pre = name + "_"
    alpha = str(z[pre + "alpha"])
    sa, sb = [str(s) for s in z[pre + "sa"]], [str(s) for s in z[pre + "sb"]]
    tr = z[pre + "tracks"] if pre + "tracks" in z.files else None
    gt = z[pre + "gap_tracks"] if pre + "gap_tracks" in z.files else None
    p = nw.AlignParams.from_arrays(z[pre + "mat"], z[pre + "gaps"], alphabet=alpha)
    for fe in SG_SETS:
        for gm in (0, 1):
            kw = dict(gap_model=("linear", "affine")[gm], tracks=tr, gap_tracks=gt, **_mode_kw(fe))
            for prec in (32, 64):
                cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
                b = cls(sa, sb, p, grad_mode="hard", **kw)
                b.score_and_grad()
                key = f"{pre}hard{prec}_g{gm}_e{fe}_"
                assert np.array_equal(b.scores(), z[key + "scores"]), key
                assert np.array_equal(_flat(b, len(sa)), z[key + "grads"]), key
                assert np.array_equal(b.guides(), z[key + "guides"]), key
            b = nw.SeqPairBatch(sa, sb, p, grad_mode="soft", **kw)
            b.score_and_grad()
            key = f"{pre}soft_g{gm}_e{fe}_"
            np.testing.assert_allclose(b.scores(), z[key + "scores"], rtol=SOFT_RTOL, atol=1e-5, err_msg=key)
            _soft_close(_flat(b, len(sa)), z[key + "grads"])
            if fe == 12 and tr is None:
                # banded re-alignment around the guides of the params scored, after a step
                p2 = nw.AlignParams.from_arrays(z[pre + "mat2"], z[pre + "gaps2"], alphabet=alpha)
                for prec in (32, 64):
                    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
                    hb = cls(sa, sb, p, grad_mode="hard", **kw)
                    hb.score_and_grad()
                    hb.set_params(p2)
                    hb.banded_grad(4)
                    key = f"{pre}band{prec}_g{gm}_e{fe}_"
                    assert np.array_equal(hb.scores(), z[key + "scores"]), key
                    assert np.array_equal(_flat(hb, len(sa)), z[key + "grads"]), key
                    assert np.array_equal(hb.guides(), z[key + "guides"]), key
                # the reference's soft fixtures ran in double: its guides are the float64 Viterbi's
                b = nw.SeqPairBatchDouble(sa, sb, p, grad_mode="soft", **kw)
                b.score_and_grad()
                b.set_params(p2)
                b.banded_grad(4)
                key = f"{pre}softband_g{gm}_e{fe}_"
                np.testing.assert_allclose(b.scores(), z[key + "scores"], rtol=SOFT_RTOL, atol=1e-5, err_msg=key)
                _soft_close(_flat(b, len(sa)), z[key + "grads"])


def _pairs(rng, long=False):
    """Empty and one-residue sides, miRNA-like short A in long B, homologs in several stripes,
    and (long) pairs of 1,600+ rows."""
    sa = rand_seqs(rng, 30, 1, 40, AA) + ["", "A", "", "ACDEF"] + rand_seqs(rng, 6, 18, 26, AA)
    sb = rand_seqs(rng, 30, 1, 40, AA) + ["KLM", "", "", "W"] + rand_seqs(rng, 6, 400, 1500, AA)
    homo = rand_seqs(rng, 6, 150, 330, AA)
    sa += homo
    sb += [mutate(rng, s, AA) for s in homo]
    if long:
        lng = rand_seqs(rng, 2, 1600, 2100, AA)
        sa += lng
        sb += ["".join(rng.choice(list(AA), size=200)) + mutate(rng, s, AA) for s in lng]
    return sa, sb


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("fe", [12, 15, 6, 9])
def test_semiglobal_hard_oracle(prec, gm, fe):
    rng = np.random.default_rng(3100 + prec + 7 * gm + fe)
    mat = rand_matrix(rng, 20, 1, True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if gm else np.array([[0.0, 3.0, 0.0, 2.0]])
    sa, sb = _pairs(rng, long=(prec == 32))
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), gap_model=("linear", "affine")[gm],
            grad_mode="hard", **_mode_kw(fe))
    tot = b.score_and_grad(keep_paths=True)
    cap = max(len(x) + len(y) for x, y in zip(sa, sb)) + 1
    o = oracle.hard(prec, gm, 2, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)), moves_cap=cap,
                    free_ends=fe)
    s = b.scores()
    assert np.array_equal(s, o["scores"]), np.nonzero(s != o["scores"])[0][:5]
    assert tot == float(np.cumsum(o["scores"])[-1])
    flat = _flat(b, len(sa))
    assert np.array_equal(flat, o["grads"]), np.nonzero((flat != o["grads"]).any(1))[0][:5]
    assert np.array_equal(b.guides(), o["guides"])
    mo, mv, info = b._stored()
    for i in range(len(sa)):
        k = int(info[i, 0])
        assert k == int(o["nmoves"][i])
        assert np.array_equal(mv[mo[i]:mo[i] + k], o["moves"][i, :k])
        assert (info[i, 1], info[i, 2]) == (o["ends"][i, 2], o["ends"][i, 3])
        a_al, b_al = b[i].aligned()
        si, sj, ei, ej = int(info[i, 1]), int(info[i, 2]), int(o["ends"][i, 0]), int(o["ends"][i, 1])
        assert a_al.replace("-", "") == sa[i][si:ei] and b_al.replace("-", "") == sb[i][sj:ej]


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("fe", [12, 15, 6, 9])
def test_semiglobal_soft_oracle(prec, gm, fe):
    rng = np.random.default_rng(3200 + prec + 7 * gm + fe)
    mat = rand_matrix(rng, 20, 1, True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if gm else np.array([[0.0, 3.0, 0.0, 2.0]])
    sa, sb = _pairs(rng, long=(prec == 32))
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), gap_model=("linear", "affine")[gm],
            grad_mode="soft", **_mode_kw(fe))
    b.score_and_grad()
    so, go = oracle.soft(gm, 2, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)), free_ends=fe)
    np.testing.assert_allclose(b.scores(), so, rtol=SOFT_RTOL, atol=1e-5)
    _soft_close(_flat(b, len(sa)), go)


@pytest.mark.parametrize("gm", [0, 1])
def test_semiglobal_soft_geometries_agree(gm):
    """Every soft geometry (a lane per pair, narrow and wide stripes, checkpointed) gives the
    glocal result within tolerance of the oracle."""
    rng = np.random.default_rng(3300 + gm)
    mat = rand_matrix(rng, 20, 1, True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa = rand_seqs(rng, 24, 5, 30, AA) + rand_seqs(rng, 8, 100, 260, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    so, go = oracle.soft(gm, 2, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)), free_ends=12)
    for geo in ((1, 16), (16, 4), (32, 2), (32, 8)):
        b = nw.SeqPairBatch(sa, sb, p, gap_model=("linear", "affine")[gm], mode="glocal", grad_mode="soft")
        b._tune = geo
        b.score_and_grad()
        np.testing.assert_allclose(b.scores(), so, rtol=SOFT_RTOL, atol=1e-5, err_msg=str(geo))
        _soft_close(_flat(b, len(sa)), go)


def test_semiglobal_refusals_and_api():
    rng = np.random.default_rng(3400)
    mat = rand_matrix(rng, 20, 1, True)
    p = nw.AlignParams.from_arrays(mat, [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    sa = rand_seqs(rng, 4, 600, 700, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    b = nw.SeqPairBatch(sa, sb, p, mode="glocal", grad_mode="hard")
    assert b.mode == "glocal" and b.free_ends == (False, False, True, True)
    b.score_and_grad()
    full = b.scores().copy()
    b.banded_grad(8)                          # glocal ends band (the reference's guide band)
    ov = nw.SeqPairBatch(sa, sb, p, mode="overlap", grad_mode="hard")
    ov.score_and_grad()
    with pytest.raises(ValueError, match="glocal"):
        ov.banded_grad(8)
    # glocal ends split pairs (the reference's glocal Hirschberg): the same optimal scores,
    # tracked affine too (tracked linear glocal splits are not built); other end sets run Pointers
    h = nw.SeqPairBatch(sa, sb, p, mode="glocal", grad_mode="hard", traceback="hirschberg")
    h.score_and_grad()
    assert np.array_equal(h.scores(), full)
    trk = np.zeros(sum(len(x) for x in sa), np.uint16)
    ht = nw.SeqPairBatch(sa, sb, p, mode="glocal", grad_mode="hard", traceback="hirschberg", tracks=trk)
    ht.score_and_grad()
    assert np.array_equal(ht.scores(), full)
    hov = nw.SeqPairBatch(sa, sb, p, mode="overlap", grad_mode="hard", traceback="hirschberg")
    hov.score_and_grad()
    assert np.array_equal(hov.scores(), ov.scores())
    # pairs within the Hirschberg cutoff run the Pointers path, as the reference's do
    short = nw.SeqPairBatch(sa[:2], sb[:2], p, mode="glocal", grad_mode="hard", traceback="hirschberg")
    short.hb_cutoff = 1000
    short.score_and_grad()
    assert np.array_equal(short.scores(), full[:2])
    o = nw.SeqPairBatch(sa, sb, p, mode="semiglobal", free_ends=("a_begin", "b_end"), grad_mode="soft")
    assert o.free_ends == (True, False, False, True)
    assert nw.SeqPairBatch(sa, sb, p, mode="overlap").free_ends == (True, True, True, True)
    assert nw.SeqPairBatch(sa, sb, p, mode="global").free_ends == (False, False, False, False)
    assert nw.SeqPairBatch(sa, sb, p, mode="local").free_ends is None
    # semiglobal with no free end is Global's DP
    g0 = nw.SeqPairBatch(sa, sb, p, mode="semiglobal", free_ends=(), grad_mode="hard")
    g1 = nw.SeqPairBatch(sa, sb, p, mode="global", grad_mode="hard")
    g0.score_and_grad()
    g1.score_and_grad()
    assert np.array_equal(g0.scores(), g1.scores())


@pytest.mark.parametrize("gm", [0, 1])
def test_glocal_banded_oracle(gm):
    """Banded re-alignment with glocal ends on multi-stripe pairs (miRNA-like A in long B and
    homologs): hard bit for bit, soft within tolerance of the oracle's banded forward-backward."""
    rng = np.random.default_rng(3500 + gm)
    mat = rand_matrix(rng, 20, 1, True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if gm else np.array([[0.0, 3.0, 0.0, 2.0]])
    sa = rand_seqs(rng, 8, 18, 26, AA) + rand_seqs(rng, 10, 60, 300, AA)
    sb = rand_seqs(rng, 8, 200, 600, AA) + [mutate(rng, s, AA) for s in sa[8:]]
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    q = nw.AlignParams.from_arrays(mat + 0.5, gaps + 0.25, alphabet=AA)
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    kw = dict(gap_model=("linear", "affine")[gm], mode="glocal")
    o = oracle.hard(32, gm, 2, mat, gaps, enc, free_ends=12)
    ob = oracle.hard(32, gm, 2, mat + 0.5, gaps + 0.25, enc, guides_in=o["guides"], band=6, free_ends=12)
    b = nw.SeqPairBatch(sa, sb, p, grad_mode="hard", **kw)
    b.score_and_grad()
    b.set_params(q)
    b.banded_grad(6)
    assert np.array_equal(b.scores(), ob["scores"])
    assert np.array_equal(_flat(b, len(sa)), ob["grads"])
    assert np.array_equal(b.guides(), ob["guides"])
    so, go = oracle.soft(gm, 2, mat + 0.5, gaps + 0.25, enc, 1.0, guides_in=o["guides"], band=6, free_ends=12)
    s = nw.SeqPairBatch(sa, sb, p, grad_mode="soft", **kw)
    s.score_and_grad()
    s.set_params(q)
    s.banded_grad(6)
    np.testing.assert_allclose(s.scores(), so, rtol=SOFT_RTOL, atol=1e-5)
    _soft_close(_flat(s, len(sa)), go)
