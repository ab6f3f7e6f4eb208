"""GPU soft path at the edges of float32's range, against the CPU oracle (double, log space).

The float32 pass either returns results within tolerance of the oracle or hands the pair to
double by itself (a value, Z or a count's scale factor out of range, or its lost-mass bound
above 2^-24), as the reference's run_fwdbwd does (aligner.hpp:6554-6626); a pair the double pass
refuses too is a ValueError.  Cases follow the reference's own tests:
test_soft_float32.py:145-158 (low temperatures, "a 31 x 4 Global pair once lost 20 % of a
count"), test_soft_denormal.py (long related protein pairs whose far cells go subnormal, low
temperature, banded), and a short A against a long B under global ends, whose long gap runs
once left a lane's exponent stale.
"""
import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402

SOFT_RTOL = 1e-4
MODES = [(gm, mode) for gm in ("linear", "affine") for mode in ("global", "local", "glocal")]
# every soft geometry the library compiles: (lanes per pair, rows per lane)
GEOS = [(1, 8), (1, 16), (1, 24), (1, 32), (8, 4), (16, 2), (16, 4), (16, 8), (32, 2), (32, 4), (32, 8)]


def _am(mode):
    return {"global": 0, "local": 1, "glocal": 2}[mode]


def _run(cls, alpha, mat, gaps, sa, sb, gm="affine", mode="global", T=1.0, geo=None, band=None):
    b = cls(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=alpha), gap_model=gm, mode=mode,
            grad_mode="soft")
    if geo is not None:
        b._tune = geo
    b.soft_temperature = T
    b.score_and_grad()
    if band is not None:
        b.set_params(nw.AlignParams.from_arrays(mat + 0.25, gaps + 0.1, alphabet=alpha))
        b.banded_grad(band)
    gmat, ggap = b.grads()
    flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
    return b.scores(), flat, b.soft_status() & 0xff


def _oracle(alpha, mat, gaps, sa, sb, gm="affine", mode="global", T=1.0):
    enc = oracle.Encoded(encode(alpha, sa), encode(alpha, sb))
    return oracle.soft(("linear", "affine").index(gm), _am(mode), mat, gaps, enc, T)


def _close(s, g, so, go, rtol=SOFT_RTOL, atol=1e-5):
    np.testing.assert_allclose(s, so, rtol=rtol, atol=atol)
    scale = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
    err = np.abs(g - go) / scale
    assert err.max() <= rtol, (err.max(), np.unravel_index(err.argmax(), err.shape))


def _mirna_case(rng, n=6):
    alpha = "ACGTU"
    mat = np.full((1, 5, 5), -4.0)
    for x, y in ((0, 3), (1, 2), (2, 1), (3, 0), (4, 0), (2, 4)):
        mat[0, x, y] = 5.0
    gaps = np.array([[5.0, 2.0, 5.0, 2.0]])
    sa = ["".join(rng.choice(list("ACGU"), size=22)) for _ in range(n)]
    sb = ["".join(rng.choice(list("ACGT"), size=int(rng.integers(500, 900)))) for _ in range(n)]
    return alpha, mat, gaps, sa, sb


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("geo", GEOS)
@pytest.mark.parametrize("T", [1.0, 2.0])
def test_short_a_long_b_global(prec, geo, T):
    """A 22-nt A against a 500-900-nt B under global ends: the long gap run at row m drives the
    exponent of row m's lane far down while the padding lanes below it hold zeros; every
    geometry computes the pair in its own precision (no rerun) and matches the oracle."""
    rng = np.random.default_rng(5100 + prec + geo[0] + geo[1] + int(T))
    alpha, mat, gaps, sa, sb = _mirna_case(rng)
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    s, g, st = _run(cls, alpha, mat, gaps, sa, sb, T=T, geo=geo)
    so, go = _oracle(alpha, mat, gaps, sa, sb, T=T)
    _close(s, g, so, go)
    if prec == 32 and geo[1] <= 4:
        # few rows per lane keep the lane's rows close in scale: the float32 pass accepts them
        assert not st.any(), st


@pytest.mark.parametrize("geo", GEOS)
def test_short_a_long_b_global_protein(geo):
    """The same shape over the 20-letter protein alphabet (whose per-lane histograms do not fit
    one lane per pair's shared memory), float32 at every geometry."""
    rng = np.random.default_rng(5200 + geo[0] + geo[1])
    mat = rng.integers(-4, 4, size=(1, 20, 20)).astype(np.float64)
    mat[0] = np.triu(mat[0]) + np.triu(mat[0], 1).T
    mat[0][np.diag_indices(20)] = rng.integers(4, 12, size=20)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa = ["".join(rng.choice(list(AA), size=22)) for _ in range(5)]
    sb = ["".join(rng.choice(list(AA), size=int(rng.integers(500, 900)))) for _ in range(5)]
    s, g, _ = _run(nw.SeqPairBatch, AA, mat, gaps, sa, sb, geo=geo)
    so, go = _oracle(AA, mat, gaps, sa, sb)
    _close(s, g, so, go)


def _pairs(rng, alpha, n):
    lens = [(1, 1), (1, 7), (7, 1), (22, 50), (50, 22), (33, 33), (31, 4)]
    lens += [(int(rng.integers(1, 60)), int(rng.integers(1, 60))) for _ in range(n)]
    return (["".join(rng.choice(list(alpha), a)) for a, _ in lens],
            ["".join(rng.choice(list(alpha), b)) for _, b in lens])


@pytest.mark.parametrize("gm,mode", MODES)
def test_low_temperature_in_range(gm, mode):
    """The reference's low-temperature grid (test_soft_float32.py:145-158): DNA matrices of
    scale 0.5, gaps (1.0, 0.5, 1.5, 0.3), T down to 0.04; float32 must be accurate or hand the
    pair to double."""
    for draw in range(4):
        rng = np.random.default_rng(6000 + 10 * draw + 3 * _am(mode) + ("linear", "affine").index(gm))
        mat = rng.normal(0.0, 0.5, (1, 4, 4))
        gaps = np.array([[1.0, 0.5, 1.5, 0.3]])
        sa, sb = _pairs(rng, "ACGT", 20)
        for T in (0.5, 0.2, 0.05, 0.04):
            so, go = _oracle("ACGT", mat, gaps, sa, sb, gm, mode, T)
            for cls in (nw.SeqPairBatch, nw.SeqPairBatchDouble):
                for geo in (None, (32, 4), (16, 2)):
                    s, g, _ = _run(cls, "ACGT", mat, gaps, sa, sb, gm, mode, T, geo=geo)
                    _close(s, g, so, go)


def _protein_case(rng, L, n):
    mat = rng.normal(-0.6, 0.6, (1, 20, 20)) + 2.0 * np.eye(20)
    gaps = np.array([[3.3, 0.3, 3.3, 0.3]])
    sa, sb = [], []
    for _ in range(n):
        a = rng.choice(list(AA), L)
        b = a.copy()
        mut = rng.random(L) < 0.2
        b[mut] = rng.choice(list(AA), int(mut.sum()))
        sa.append("".join(a))
        sb.append("".join(b[: L - int(rng.integers(0, 20))]))
    return mat, gaps, sa, sb


@pytest.mark.parametrize("gm,mode", MODES)
def test_denormal_long_pairs(gm, mode):
    """L ~250 related protein pairs (test_soft_denormal.py): cells far from the diagonal sit far
    below their lane's largest value.  Double within 1e-9 of the oracle, float32 within 1e-4."""
    rng = np.random.default_rng(7)
    mat, gaps, sa, sb = _protein_case(rng, 250, 3)
    so, go = _oracle(AA, mat, gaps, sa, sb, gm, mode)
    s, g, _ = _run(nw.SeqPairBatchDouble, AA, mat, gaps, sa, sb, gm, mode)
    _close(s, g, so, go, rtol=1e-9, atol=1e-9)
    s, g, _ = _run(nw.SeqPairBatch, AA, mat, gaps, sa, sb, gm, mode)
    _close(s, g, so, go)


@pytest.mark.parametrize("gm,mode", MODES)
@pytest.mark.parametrize("T", [0.3, 0.1])
def test_denormal_low_temperature(gm, mode, T):
    rng = np.random.default_rng(11)
    mat, gaps, sa, sb = _protein_case(rng, 60, 4)
    so, go = _oracle(AA, mat, gaps, sa, sb, gm, mode, T)
    s, g, _ = _run(nw.SeqPairBatchDouble, AA, mat, gaps, sa, sb, gm, mode, T)
    _close(s, g, so, go, rtol=1e-9, atol=1e-9)
    s, g, _ = _run(nw.SeqPairBatch, AA, mat, gaps, sa, sb, gm, mode, T)
    _close(s, g, so, go)


@pytest.mark.parametrize("gm", ["linear", "affine"])
@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("prec", [32, 64])
def test_banded_soft_both_precisions(gm, mode, prec):
    """Banded re-alignment (bandwidth 6) of L ~150 related protein pairs after a parameter
    step, in the batch's own precision (float32 banded runs in float32), against the oracle's
    banded pass around the same guides."""
    rng = np.random.default_rng(13)
    mat, gaps, sa, sb = _protein_case(rng, 150, 3)
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    s, g, st = _run(cls, AA, mat, gaps, sa, sb, gm, mode, band=6)
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    gi, ai = ("linear", "affine").index(gm), _am(mode)
    g0 = oracle.hard(prec, gi, ai, mat, gaps, enc)["guides"]
    so, go = oracle.soft(gi, ai, mat + 0.25, gaps + 0.1, enc, guides_in=g0, band=6)
    _close(s, g, so, go, rtol=SOFT_RTOL if prec == 32 else 1e-9, atol=1e-5 if prec == 32 else 1e-9)


def _long_homologs(rng, L, n):
    """Integer matrix with diagonal scores 4-11 (steps of up to e^11 per cell at T = 1); B is A
    with 20 % substitutions and single-residue insertions and deletions (2.5 % each)."""
    m = rng.integers(-4, 4, size=(20, 20)).astype(np.float64)
    m = np.triu(m) + np.triu(m, 1).T
    m[np.diag_indices(20)] = rng.integers(4, 12, size=20)
    sa, sb = [], []
    for _ in range(n):
        a = rng.integers(0, 20, L)
        b = a.copy()
        sub = rng.random(L) < 0.2
        b[sub] = rng.integers(0, 20, int(sub.sum()))
        out = []
        for x, u in zip(b, rng.random(L)):
            if u < 0.025:
                continue                                  # deletion
            out.append(x)
            if u > 0.975:
                out.append(int(rng.integers(0, 20)))      # insertion
        sa.append("".join(AA[i] for i in a))
        sb.append("".join(AA[i] for i in out))
    return m[None], sa, sb


@pytest.mark.parametrize("gm", ["linear", "affine"])
@pytest.mark.parametrize("mode", ["global", "local"])
def test_banded_soft_long_against_oracle(gm, mode):
    """Banded re-alignment (bandwidth 20) of 1,500-residue related pairs with insertions and
    deletions.  A stripe sweeps only the union of its rows' bands, so most stripes start far
    right of column 0 and read the stripe above (or below) outside its own columns as zero.
    Float32 and double against the oracle's banded pass around the same guides."""
    rng = np.random.default_rng(37)
    _, sa, sb = _long_homologs(rng, 1500, 3)
    mat = rng.normal(-0.6, 0.6, (1, 20, 20)) + 2.0 * np.eye(20)
    gaps = np.array([[3.3, 0.3, 3.3, 0.3]])
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    gi, ai = ("linear", "affine").index(gm), _am(mode)
    for prec, cls in ((32, nw.SeqPairBatch), (64, nw.SeqPairBatchDouble)):
        s, g, st = _run(cls, AA, mat, gaps, sa, sb, gm, mode, band=20)
        assert (st == 0).all(), st
        g0 = oracle.hard(prec, gi, ai, mat, gaps, enc)["guides"]
        so, go = oracle.soft(gi, ai, mat + 0.25, gaps + 0.1, enc, guides_in=g0, band=20)
        _close(s, g, so, go, rtol=SOFT_RTOL if prec == 32 else 1e-9, atol=1e-5 if prec == 32 else 1e-9)


@pytest.mark.parametrize("gm", ["linear", "affine"])
@pytest.mark.parametrize("mode", ["global", "local", "glocal"])
def test_banded_soft_late_starts_against_oracle(gm, mode):
    """B is a random prefix of 88-133 residues followed by a mutated copy of a 300-residue A,
    so the paths start far along row 0: Global through the origin and a long gap run on row 0,
    Local and glocal from row 0's start weights left of row 1's band.  Banded stripes below
    the first start right of column 0; the prefix lengths put band edges on multiples of 32.
    Float32 against the oracle's banded pass (bandwidth 6)."""
    rng = np.random.default_rng(41)
    mat = rng.normal(-0.6, 0.6, (1, 20, 20)) + 2.0 * np.eye(20)
    gaps = np.array([[3.3, 0.3, 3.3, 0.3]])
    sa, sb = [], []
    for P in range(88, 136, 3):
        a = rng.integers(0, 20, 300)
        b = a.copy()
        sub = rng.random(300) < 0.15
        b[sub] = rng.integers(0, 20, int(sub.sum()))
        sa.append("".join(AA[i] for i in a))
        sb.append("".join(AA[i] for i in np.concatenate([rng.integers(0, 20, P), b])))
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    gi, ai = ("linear", "affine").index(gm), _am(mode)
    fe = dict(free_ends=12) if mode == "glocal" else {}
    s, g, st = _run(nw.SeqPairBatch, AA, mat, gaps, sa, sb, gm, mode, band=6)
    assert (st == 0).all(), st
    g0 = oracle.hard(32, gi, ai, mat, gaps, enc, **fe)["guides"]
    so, go = oracle.soft(gi, ai, mat + 0.25, gaps + 0.1, enc, 1.0, guides_in=g0, band=6, **fe)
    _close(s, g, so, go)


@pytest.mark.parametrize("mode", ["global", "local"])
def test_banded_long_pairs_stay_float32(mode):
    """Banded re-alignment (bandwidth 64) of 3,000-residue related pairs after a parameter step.
    Between renormalisations both lanes hold values far above 1, so a count's scale
    2^(E_F + E_B - E_Z) falls below float32's normal range while F^ B^ nears 2^130; the step's
    F^ move into the scale, so float32 keeps every pair (no refusal to double) and matches the
    double batch."""
    rng = np.random.default_rng(31)
    mat, sa, sb = _long_homologs(rng, 3000, 3)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    s32, g32, st = _run(nw.SeqPairBatch, AA, mat, gaps, sa, sb, "affine", mode, band=64)
    s64, g64, _ = _run(nw.SeqPairBatchDouble, AA, mat, gaps, sa, sb, "affine", mode, band=64)
    assert (st == 0).all(), st
    _close(s32, g32, s64, g64)


def test_out_of_range_raises():
    """A step score of 800 nats overflows exp() in double too: ValueError naming the reason
    (test_soft_denormal.py: test_out_of_range_still_raises)."""
    mat = np.full((1, 20, 20), -1.0)
    np.fill_diagonal(mat[0], 800.0)
    gaps = np.array([[2.0, 0.5, 2.0, 0.5]])
    s = AA * 3
    for cls in (nw.SeqPairBatch, nw.SeqPairBatchDouble):
        b = cls([s], [s], nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="soft")
        with pytest.raises(ValueError, match="overflows"):
            b.score_and_grad()


def test_float32_out_of_range_reruns_in_double():
    """Step scores of ~100 nats overflow float32's exp but not double's: the float32 batch
    hands those pairs to double (soft_status 1) and matches the double batch
    (test_soft_float32.py: test_out_of_range_falls_back_to_double)."""
    rng = np.random.default_rng(21)
    mat = rng.normal(0.0, 1.0, (1, 4, 4)) + 100.0 * np.eye(4)
    gaps = np.array([[1.0, 0.5, 1.5, 0.3]])
    lens = [(int(rng.integers(1, 20)), int(rng.integers(1, 20))) for _ in range(12)]
    sa = ["".join(rng.choice(list("ACGT"), a)) for a, _ in lens]
    sb = ["".join(rng.choice(list("ACGT"), b)) for _, b in lens]
    s32, g32, st = _run(nw.SeqPairBatch, "ACGT", mat, gaps, sa, sb)
    s64, g64, _ = _run(nw.SeqPairBatchDouble, "ACGT", mat, gaps, sa, sb)
    assert (st == 1).all()
    np.testing.assert_allclose(s32, s64, rtol=1e-12)
    np.testing.assert_allclose(g32, g64, rtol=1e-12, atol=1e-12)


def test_wait_limit_fails_cleanly():
    """Soft long pairs with semi-global ends fill with several warps per pair that wait on one
    another with bounded polls.  With the limit at one poll the waits run out: the kernel
    marks the pair and returns, the call raises RuntimeError, and the same batch then runs to
    the oracle's result at the default limit.  (Other long pairs fill as tiles, a launch per
    anti-diagonal: no waits.)"""
    rng = np.random.default_rng(31)
    mat = rng.integers(-4, 4, size=(1, 20, 20)).astype(np.float64)
    mat[0] = np.triu(mat[0]) + np.triu(mat[0], 1).T
    mat[0][np.diag_indices(20)] = rng.integers(4, 12, size=20)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa = ["".join(rng.choice(list(AA), 2600)) for _ in range(2)]
    sb = ["".join(c if rng.random() > 0.2 else rng.choice(list(AA)) for c in a) for a in sa]
    b = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="soft",
                        mode="glocal")
    b.set_spin_limit(1)
    with pytest.raises(RuntimeError, match="ran out"):
        b.score_and_grad()
    b.set_spin_limit()
    b.score_and_grad()
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    so, go = oracle.soft(1, 2, mat, gaps, enc, free_ends=12)
    np.testing.assert_allclose(b.scores(), so, rtol=SOFT_RTOL)
