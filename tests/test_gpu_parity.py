"""GPU parity: the CUDA path through the C ABI against the CPU oracle on the same inputs.

Hard results (scores, per-pair gradient counts, guides) are compared bit for bit; soft
results within 1e-4 relative of the oracle's double log-space forward-backward (the
reference's float32-vs-double tolerance is 2e-4 / 1e-5 abs, test_soft_float32.py:26-29).
"""
import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402

SOFT_RTOL = 1e-4


def _problem(rng, alpha, n, lo, hi, K=1, integer=True, tracked=False, homolog=False, gap_tracks=False):
    N = len(alpha)
    mat = rand_matrix(rng, N, K, integer)
    if integer:
        gaps = np.tile([11.0, 1.0, 11.0, 1.0], (K, 1))
        if K > 1:
            gaps = gaps + rng.integers(0, 3, size=(K, 4))
    else:
        gaps = rng.uniform(0.3, 4.0, size=(K, 4))
    sa = rand_seqs(rng, n, lo, hi, alpha)
    sb = [mutate(rng, s, alpha) for s in sa] if homolog else rand_seqs(rng, n, lo, hi, alpha)
    tr = gt = None
    if tracked:
        tr = np.concatenate([rng.integers(0, K, size=len(s)) for s in sa] + [np.zeros(0, np.int64)]).astype(np.uint16)
        if gap_tracks:
            gt = np.concatenate([rng.integers(0, K, size=len(s) + 1) for s in sa]).astype(np.uint16)
    return mat, gaps, sa, sb, tr, gt


def _params(alpha, mat, gaps):
    return nw.AlignParams.from_arrays(mat, gaps, alphabet=alpha)


def _hard_check(prec, gm, am, alpha, mat, gaps, sa, sb, tr, gt, tracked):
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, _params(alpha, mat, gaps), gap_model=("linear", "affine")[gm],
            mode=("global", "local")[am], grad_mode="hard", tracks=tr, gap_tracks=gt)
    tot = b.score_and_grad()
    enc = oracle.Encoded(encode(alpha, sa), encode(alpha, sb), tr, gt)
    o = oracle.hard(prec, gm, am, mat, gaps, enc, tracked=tracked)
    s = b.scores()
    assert np.array_equal(s, o["scores"]), np.nonzero(s != o["scores"])[0][:5]
    # the reference sums in pair order (Python's sum() compensates: use a running sum)
    assert tot == (float(np.cumsum(o["scores"])[-1]) if len(sa) else 0.0)
    gmat, ggap = b.grads()
    K, N = mat.shape[0], mat.shape[1]
    if not tracked:
        gmat = gmat[:, None]
        ggap = ggap[:, None]
    flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
    assert np.array_equal(flat, o["grads"]), np.nonzero((flat != o["grads"]).any(1))[0][:5]
    gj = b.guides()
    assert np.array_equal(gj, o["guides"])
    cg = b.compute_grad()
    ref = oracle.blocked_sum(o["grads"])
    assert np.array_equal(np.concatenate([cg.matrices.ravel(), cg.gaps.ravel()]), ref)
    w = np.linspace(-1.0, 2.0, len(sa))
    wg = b.weighted_grad(w)
    ref = oracle.blocked_sum(o["grads"], w)
    assert np.array_equal(np.concatenate([wg.matrices.ravel(), wg.gaps.ravel()]), ref)


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
@pytest.mark.parametrize("integer", [True, False])
def test_hard_bit_exact(prec, gm, am, integer):
    rng = np.random.default_rng(100 + prec + 10 * gm + 20 * am + int(integer))
    # short (one lane per pair), medium and multi-stripe pairs, plus empty sequences
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 60, 0, 40, integer=integer)
    sa += ["", "ACD", "", "W" * 70] + rand_seqs(rng, 6, 200, 300, AA)
    sb += ["KLM", "", "", "W" * 3] + rand_seqs(rng, 6, 150, 320, AA)
    _hard_check(prec, gm, am, AA, mat, gaps, sa, sb, None, None, False)


@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
@pytest.mark.parametrize("gap_tracks", [False, True])
def test_hard_tracked_bit_exact(gm, am, gap_tracks):
    rng = np.random.default_rng(7 + gm + 2 * am + 4 * gap_tracks)
    alpha = "ACGTU"
    mat, gaps, sa, sb, tr, gt = _problem(rng, alpha, 50, 1, 45, K=3, tracked=True, gap_tracks=gap_tracks,
                                         integer=False)
    _hard_check(32, gm, am, alpha, mat, gaps, sa, sb, tr, gt, True)


def _soft_check(prec, gm, am, alpha, mat, gaps, sa, sb, tr, gt, T=1.0):
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, _params(alpha, mat, gaps), gap_model=("linear", "affine")[gm],
            mode=("global", "local")[am], grad_mode="soft", tracks=tr, gap_tracks=gt)
    b.soft_temperature = T
    b.score_and_grad()
    enc = oracle.Encoded(encode(alpha, sa), encode(alpha, sb), tr, gt)
    so, go = oracle.soft(gm, am, mat, gaps, enc, T)
    s = b.scores()
    np.testing.assert_allclose(s, so, rtol=SOFT_RTOL, atol=1e-5)
    K, N = mat.shape[0], mat.shape[1]
    gmat, ggap = b.grads()
    if gmat.ndim == 3:
        gmat = gmat[:, None]
        ggap = ggap[:, None]
    flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
    # relative to each pair's gradient scale (its largest entry), as the reference's tests do
    scale = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
    err = np.abs(flat - go) / scale
    assert err.max() <= SOFT_RTOL, (err.max(), np.unravel_index(err.argmax(), err.shape))


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_soft_within_tolerance(prec, gm, am):
    rng = np.random.default_rng(300 + prec + gm + 2 * am)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 40, 1, 40, homolog=True)
    sa += rand_seqs(rng, 4, 150, 260, AA) + ["", "A"]
    sb += [mutate(rng, s, AA) for s in sa[-6:-2]] + ["AC", ""]
    _soft_check(prec, gm, am, AA, mat, gaps, sa, sb, None, None)


@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_soft_tracked(gm, am):
    rng = np.random.default_rng(500 + gm + 2 * am)
    alpha = "ACGTU"
    mat, gaps, sa, sb, tr, gt = _problem(rng, alpha, 40, 1, 30, K=3, tracked=True, gap_tracks=True)
    _soft_check(32, gm, am, alpha, mat, gaps, sa, sb, tr, gt)


@pytest.mark.parametrize("T", [0.5, 2.0])
def test_soft_temperature(T):
    rng = np.random.default_rng(77)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 30, 5, 60, homolog=True)
    _soft_check(32, 1, 0, AA, mat, gaps, sa, sb, None, None, T=T)


@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
@pytest.mark.parametrize("bw", [1, 5, 64])
def test_banded_bit_exact(gm, am, bw):
    """set_params + banded_grad around the guides of a full pass (batch_engine.hpp:633-653)."""
    rng = np.random.default_rng(900 + gm + 2 * am + bw)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 40, 1, 60, integer=False, homolog=True)
    sa += rand_seqs(rng, 3, 150, 300, AA)
    sb += [mutate(rng, s, AA) for s in sa[-3:]]
    mat2 = mat + rng.normal(0, 0.3, size=mat.shape)
    gaps2 = gaps + rng.uniform(0, 0.2, size=gaps.shape)
    for prec in (32, 64):
        cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
        b = cls(sa, sb, _params(AA, mat, gaps), gap_model=("linear", "affine")[gm],
                mode=("global", "local")[am], grad_mode="hard")
        b.score_and_grad()
        b.set_params(_params(AA, mat2, gaps2))
        tot = b.banded_grad(bw)
        enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
        o0 = oracle.hard(prec, gm, am, mat, gaps, enc)
        o = oracle.hard(prec, gm, am, mat2, gaps2, enc, guides_in=o0["guides"], band=bw)
        assert np.array_equal(b.scores(), o["scores"]), np.nonzero(b.scores() != o["scores"])[0][:5]
        gmat, ggap = b.grads()
        flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
        assert np.array_equal(flat, o["grads"])
        assert np.array_equal(b.guides(), o["guides"])
        assert tot == float(np.cumsum(o["scores"])[-1])


@pytest.mark.parametrize("name", ["prot", "protf", "rna3"])
def test_golden_reference_batches(name):
    """The GPU path against the reference's own outputs (tests/golden/make_golden.py)."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_batches.npz"))
    pre = name + "_"
    alpha = str(z[pre + "alpha"])
    sa, sb = [str(s) for s in z[pre + "sa"]], [str(s) for s in z[pre + "sb"]]
    tr = z[pre + "tracks"] if pre + "tracks" in z.files else None
    gt = z[pre + "gap_tracks"] if pre + "gap_tracks" in z.files else None
    mat, gaps, mat2, gaps2 = z[pre + "mat"], z[pre + "gaps"], z[pre + "mat2"], z[pre + "gaps2"]
    for gm in (0, 1):
        for am in (0, 1):
            for prec in (32, 64):
                cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
                b = cls(sa, sb, _params(alpha, mat, gaps), gap_model=("linear", "affine")[gm],
                        mode=("global", "local")[am], grad_mode="hard", tracks=tr, gap_tracks=gt)
                b.score_and_grad()
                key = f"{pre}hard{prec}_g{gm}_m{am}_"
                assert np.array_equal(b.scores(), z[key + "scores"])
                gmat, ggap = b.grads()
                if gmat.ndim == 3:
                    gmat, ggap = gmat[:, None], ggap[:, None]
                flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
                assert np.array_equal(flat, z[key + "grads"])
                assert np.array_equal(b.guides(), z[key + "guides"])
                if tr is None:
                    b.set_params(_params(alpha, mat2, gaps2))
                    b.banded_grad(4)
                    key = f"{pre}band{prec}_g{gm}_m{am}_"
                    assert np.array_equal(b.scores(), z[key + "scores"])
                    gmat, ggap = b.grads()
                    flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
                    assert np.array_equal(flat, z[key + "grads"])
            for T in (1.0, 0.5):
                b = nw.SeqPairBatch(sa, sb, _params(alpha, mat, gaps), gap_model=("linear", "affine")[gm],
                                    mode=("global", "local")[am], grad_mode="soft", tracks=tr, gap_tracks=gt)
                b.soft_temperature = T
                b.score_and_grad()
                key = f"{pre}soft_T{T}_g{gm}_m{am}_"
                np.testing.assert_allclose(b.scores(), z[key + "scores"], rtol=SOFT_RTOL, atol=1e-5)
                gmat, ggap = b.grads()
                if gmat.ndim == 3:
                    gmat, ggap = gmat[:, None], ggap[:, None]
                flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
                ref = z[key + "grads"]
                scale = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1.0)
                assert (np.abs(flat - ref) / scale).max() <= SOFT_RTOL


@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
@pytest.mark.parametrize("geo", [(1, 8), (32, 2), (32, 4), (16, 4), (8, 4)])
def test_soft_checkpointed(gm, am, geo):
    """Stripe checkpoints (each stripe's forward recomputed before its backward) give the same
    bits as the whole-table pass, and both agree with the oracle."""
    rng = np.random.default_rng(1300 + gm + 2 * am + geo[1] + geo[0])
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 24, 1, 90, homolog=True)
    sa += rand_seqs(rng, 3, 200, 420, AA) + ["", "W"]
    sb += [mutate(rng, s, AA) for s in sa[-5:-2]] + ["MK", ""]
    alpha = AA
    if geo[0] == 1:   # one lane per pair keeps a per-lane histogram: a small alphabet
        alpha = "ACGT"
        mat, gaps, sa, sb, tr, gt = _problem(rng, alpha, 24, 1, 90, homolog=True)
        sa += rand_seqs(rng, 3, 200, 420, alpha)
        sb += [mutate(rng, s, alpha) for s in sa[-3:]]
    out = []
    for ckb in (-1, 0):
        b = nw.SeqPairBatch(sa, sb, _params(alpha, mat, gaps), gap_model=("linear", "affine")[gm],
                            mode=("global", "local")[am], grad_mode="soft")
        b._tune = geo
        b.set_memory(checkpoint_bytes=ckb)
        b.score_and_grad()
        gmat, ggap = b.grads()
        out.append((b.scores(), gmat.copy(), ggap.copy()))
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)
    enc = oracle.Encoded(encode(alpha, sa), encode(alpha, sb))
    so, go = oracle.soft(gm, am, mat, gaps, enc)
    np.testing.assert_allclose(out[1][0], so, rtol=SOFT_RTOL, atol=1e-5)
    flat = np.concatenate([out[1][1].reshape(len(sa), -1), out[1][2].reshape(len(sa), -1)], axis=1)
    scale = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(flat - go) / scale).max() <= SOFT_RTOL


def test_soft_small_scratch_budget():
    """A scratch budget of one table runs the pairs a few at a time, with the same bits."""
    rng = np.random.default_rng(1400)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 300, 10, 120, homolog=True)
    res = []
    for budget in (-1, 1):
        b = nw.SeqPairBatch(sa, sb, _params(AA, mat, gaps), grad_mode="soft")
        b.set_memory(scratch_budget_bytes=budget)
        b.score_and_grad()
        res.append((b.scores(), b.compute_grad()))
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1].matrices, res[1][1].matrices)
    assert np.array_equal(res[0][1].gaps, res[1][1].gaps)


@pytest.mark.parametrize("grad_mode", ["hard", "soft"])
def test_autotuned_and_plain_fill_same_results(grad_mode, tmp_path, monkeypatch):
    """The autotuned geometries and the plain fill compute the same results as the planner's."""
    monkeypatch.setenv("NWGRAD_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(1500)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 200, 5, 400, homolog=True)
    sa += rand_seqs(rng, 4, 1100, 1500, AA)
    sb += [mutate(rng, s, AA) for s in sa[-4:]]
    res = []
    from nwgrad_b200 import tune
    for how in ("planner", "tuned", "plain", "mixed"):
        b = nw.SeqPairBatch(sa, sb, _params(AA, mat, gaps), grad_mode=grad_mode)
        if how == "tuned":
            table = b.autotune(sample_pairs=64)
            assert table and all(isinstance(v, (tuple, dict)) for v in table.values())
        elif how == "plain":
            b.use_plain_fill()
        elif how == "mixed":
            # equal costs: every pair takes the geometry that pads it least (a mix of buckets)
            geos = tune.SOFT_GEOS if grad_mode == "soft" else tune.HARD_GEOS
            costs = [(g, r, 1.0) for g, r in geos if g > 1]
            tune.apply(b, {sc: {"costs": costs} for sc in tune._classes(b)})
        b.score_and_grad()
        gmat, ggap = b.grads()
        res.append((b.scores(), gmat.copy(), ggap.copy()))
    for other in res[1:]:
        if grad_mode == "hard":
            for x, y in zip(res[0], other):
                assert np.array_equal(x, y)
        else:
            np.testing.assert_allclose(other[0], res[0][0], rtol=1e-6, atol=1e-6)
            for x, y in zip(res[0][1:], other[1:]):
                scale = max(1.0, float(np.abs(x).max()))
                assert np.abs(x - y).max() <= 1e-5 * scale


@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_soft_long_pairs_tiles(gm, am):
    """Pairs of 1,600+ rows run as tiles (128 rows x 256 columns; forward and backward a launch
    per anti-diagonal): within tolerance of the oracle and of the one-warp kernel on the same
    pairs."""
    rng = np.random.default_rng(1600 + gm + 2 * am)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 6, 5, 200, homolog=True)
    sa += rand_seqs(rng, 3, 1600, 2400, AA)
    sb += [mutate(rng, s, AA) for s in sa[-3:]]
    kw = dict(gap_model=("linear", "affine")[gm], mode=("global", "local")[am], grad_mode="soft")
    b = nw.SeqPairBatch(sa, sb, _params(AA, mat, gaps), **kw)
    b.score_and_grad()
    one = nw.SeqPairBatch(sa, sb, _params(AA, mat, gaps), **kw)
    one._tune = (32, 4)                       # forced geometry: one warp per pair
    one.score_and_grad()
    np.testing.assert_allclose(b.scores(), one.scores(), rtol=1e-6, atol=1e-6)
    ga, gb = b.grads()
    oa_, ob_ = one.grads()
    scale = max(1.0, float(np.abs(oa_).max()))
    assert np.abs(ga - oa_).max() <= 1e-5 * scale and np.abs(gb - ob_).max() <= 1e-5 * max(1.0, float(np.abs(ob_).max()))
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    so, go = oracle.soft(gm, am, mat, gaps, enc)
    np.testing.assert_allclose(b.scores(), so, rtol=SOFT_RTOL, atol=1e-5)
    flat = np.concatenate([ga.reshape(len(sa), -1), gb.reshape(len(sa), -1)], axis=1)
    sc = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(flat - go) / sc).max() <= SOFT_RTOL


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_hard_long_pairs_tiles(prec, gm, am):
    """Untracked pairs of 1,536+ rows and 256+ columns fill as tiles (256 rows x 256 columns,
    a launch per anti-diagonal of tiles): bit for bit the oracle's (scores, per-pair
    gradients, guides), with short pairs in the same batch and ragged last tiles (B of 256,
    257, 511, 513 and 1,000+ residues; A of 1,536 rows exactly, one stripe of 256 rows more
    than a multiple, and longer)."""
    rng = np.random.default_rng(1700 + prec + gm + 2 * am)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 8, 1, 150, integer=(gm == 1), homolog=True)
    sa += rand_seqs(rng, 3, 1600, 2600, AA)
    sb += [mutate(rng, s, AA) for s in sa[-3:]]
    for la, lb in ((1536, 256), (1537, 257), (1800, 511), (2049, 513), (1600, 2900)):
        sa += rand_seqs(rng, 1, la, la, AA)
        sb += rand_seqs(rng, 1, lb, lb, AA)
    _hard_check(prec, gm, am, AA, mat, gaps, sa, sb, None, None, False)


@pytest.mark.parametrize("gm", [0, 1])
def test_hard_local_tiles_tied_best(gm):
    """Local, tiled: one segment twice in A (rows 100-199 and 1700-1799) and twice in B
    (columns 600-699 and 1000-1099) on backgrounds that score -5 against everything, so
    four end cells in different stripes and tiles tie for the best; the pair's end is the
    first in row-major order (200, 700), as the oracle's."""
    alpha = AA
    N = len(alpha)
    mat = np.full((1, N, N), -5.0)
    seg_letters = alpha[2:]
    for k in range(2, N):
        mat[0, k, k] = 5.0
    gaps = np.array([[11.0, 3.0, 11.0, 3.0]])
    rng = np.random.default_rng(1750 + gm)
    seg = "".join(rng.choice(list(seg_letters), 100))
    a = list(alpha[0] * 2000)
    b = list(alpha[1] * 1400)
    for o in (100, 1700):
        a[o:o + 100] = seg
    for o in (600, 1000):
        b[o:o + 100] = seg
    sa, sb = ["".join(a)], ["".join(b)]
    _hard_check(32, gm, 1, alpha, mat, gaps, sa, sb, None, None, False)
    bt = nw.SeqPairBatch(sa, sb, _params(alpha, mat, gaps), gap_model=("linear", "affine")[gm], mode="local",
                         grad_mode="hard")
    bt.score_and_grad()
    assert bt.scores()[0] == 500.0


def test_hard_long_tracked_tiles():
    """Tracked long pairs (three parameter sets, gap tracks) fill as tiles too: bit for bit."""
    rng = np.random.default_rng(1800)
    alpha = "ACGTU"
    mat, gaps, sa, sb, tr, gt = _problem(rng, alpha, 3, 1600, 2200, K=3, tracked=True, gap_tracks=True)
    _hard_check(32, 1, 0, alpha, mat, gaps, sa, sb, tr, gt, True)


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
@pytest.mark.parametrize("bw", [1, 5, 64])
def test_soft_banded(prec, gm, am, bw):
    """Soft banded re-alignment after set_params, around the Viterbi guides of the first
    parameters (the deferred soft guide), within tolerance of the oracle's banded pass."""
    rng = np.random.default_rng(1900 + prec + gm + 2 * am + bw)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 30, 1, 120, integer=False, homolog=True)
    sa += rand_seqs(rng, 2, 300, 500, AA) + ["", "C"]
    sb += [mutate(rng, s, AA) for s in sa[-4:-2]] + ["W", ""]
    mat2 = mat + rng.normal(0, 0.3, size=mat.shape)
    gaps2 = gaps + rng.uniform(0, 0.2, size=gaps.shape)
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, _params(AA, mat, gaps), gap_model=("linear", "affine")[gm], mode=("global", "local")[am],
            grad_mode="soft")
    b.score_and_grad()
    b.set_params(_params(AA, mat2, gaps2))
    b.banded_grad(bw)
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    g0 = oracle.hard(prec, gm, am, mat, gaps, enc)["guides"]
    so, go = oracle.soft(gm, am, mat2, gaps2, enc, guides_in=g0, band=bw)
    np.testing.assert_allclose(b.scores(), so, rtol=SOFT_RTOL, atol=1e-5)
    gmat, ggap = b.grads()
    flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
    scale = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(flat - go) / scale).max() <= SOFT_RTOL


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_score_only_bit_exact(prec, gm, am):
    """grad_mode="none" (the Viterbi fill and the walk for the guides, no gradient) against the
    oracle's Viterbi scores bit for bit: short pairs at a lane per pair, medium at a warp, and
    long pairs as tiles."""
    rng = np.random.default_rng(1300 + prec + 10 * gm + 20 * am)
    mat, gaps, sa, sb, tr, gt = _problem(rng, AA, 60, 0, 40, integer=False)
    sa += ["", "ACD", "W" * 70] + rand_seqs(rng, 6, 200, 400, AA) + rand_seqs(rng, 2, 1600, 2200, AA)
    sb += ["KLM", "", "W" * 3] + rand_seqs(rng, 6, 150, 420, AA) + rand_seqs(rng, 2, 1500, 2300, AA)
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, _params(AA, mat, gaps), gap_model=("linear", "affine")[gm],
            mode=("global", "local")[am], grad_mode="none")
    tot = b.score_and_grad()
    o = oracle.hard(prec, gm, am, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)))
    s = b.scores()
    assert np.array_equal(s, o["scores"]), np.nonzero(s != o["scores"])[0][:5]
    assert tot == float(np.cumsum(o["scores"])[-1])
