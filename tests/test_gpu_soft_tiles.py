"""Soft long pairs as tiles (soft_kernel<..., TL>): untracked pairs of 1,536+ DP rows and 256+
columns run the forward pass as a launch per anti-diagonal of tiles (128 rows x 256 columns),
then the backward pass a launch per anti-diagonal in reverse, each tile recomputing its forward
table from the saved rows and columns.  Scores and expected counts within the oracle's
tolerance (1e-4 relative, per pair scaled by its largest count), ragged last tiles included,
and the same bits on every run."""
import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402

SOFT_RTOL = 1e-4


def _pairs(rng):
    sa = rand_seqs(rng, 5, 5, 200, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    long_a = rand_seqs(rng, 2, 1600, 2600, AA)
    sa += long_a
    sb += [mutate(rng, s, AA) for s in long_a]
    for la, lb in ((1535, 256), (1536, 257), (2047, 511), (1600, 2900)):
        a = rand_seqs(rng, 1, la, la, AA)[0]
        sa.append(a)
        b = mutate(rng, a, AA)
        sb.append((b * (lb // max(len(b), 1) + 1))[:lb])
    return sa, sb


def _check(b, gm, am, mat, gaps, sa, sb, temperature=1.0):
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    so, go = oracle.soft(gm, am, mat, gaps, enc, temperature=temperature)
    np.testing.assert_allclose(b.scores(), so, rtol=SOFT_RTOL, atol=1e-5)
    ga, gb = b.grads()
    flat = np.concatenate([ga.reshape(len(sa), -1), gb.reshape(len(sa), -1)], axis=1)
    sc = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
    err = (np.abs(flat - go) / sc).max(axis=1)
    assert err.max() <= SOFT_RTOL, (np.argmax(err), err.max())


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_soft_tiles_match_oracle(prec, gm, am):
    rng = np.random.default_rng(3100 + prec + gm + 2 * am)
    mat = rand_matrix(rng, 20, 1, integer=False)
    gaps = np.array([[3.0, 1.0, 3.0, 1.0]]) if gm == 1 else np.array([[0.0, 1.5, 0.0, 1.5]])
    sa, sb = _pairs(rng)
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), gap_model=("linear", "affine")[gm],
            mode=("global", "local")[am], grad_mode="soft")
    b.score_and_grad()
    _check(b, gm, am, mat, gaps, sa, sb)
    # no pair refused everywhere; the narrow linear Global pairs (vertical gap runs far below
    # float32's range within one stripe) may be refused in float32 and rerun in double, as the
    # one-warp kernel refuses them too
    st = b.soft_status()
    assert ((st & 0xFF) <= 1).all()
    if gm == 1 or prec == 64:
        assert (st == 0).all()


@pytest.mark.parametrize("am", [0, 1])
def test_soft_tiles_deterministic_and_weighted(am):
    """Two runs and a parameter step: the same bits each time for the same parameters (every
    sum is in a fixed order), and compute_grad the pairs' blocked sum."""
    rng = np.random.default_rng(3150 + am)
    mat = rand_matrix(rng, 20, 1, integer=True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa, sb = _pairs(rng)
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    b = nw.SeqPairBatch(sa, sb, p, mode=("global", "local")[am], grad_mode="soft")
    b.score_and_grad()
    s1 = b.scores().copy()
    g1 = [x.copy() for x in b.grads()]
    b.score_and_grad()
    assert np.array_equal(s1, b.scores())
    for x, y in zip(g1, b.grads()):
        assert np.array_equal(x, y)
    cg = b.compute_grad()
    ga, gb = b.grads()
    flat = np.concatenate([ga.reshape(len(sa), -1), gb.reshape(len(sa), -1)], axis=1)
    ref = oracle.blocked_sum(flat)
    assert np.array_equal(np.concatenate([cg.matrices.ravel(), cg.gaps.ravel()]), ref)
    b.set_params(p + cg * 1e-3)
    b.score_and_grad()
    _check(b, 1, am, (p + cg * 1e-3).matrices, (p + cg * 1e-3).gaps, sa, sb)


def test_soft_tiles_temperature():
    """T = 0.5 and 2: the weights' range changes the renormalisation period; still within
    tolerance."""
    rng = np.random.default_rng(3170)
    mat = rand_matrix(rng, 20, 1, integer=True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa, sb = _pairs(rng)
    for T in (0.5, 2.0):
        b = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="soft")
        b.soft_temperature = T
        b.score_and_grad()
        _check(b, 1, 0, mat, gaps, sa, sb, temperature=T)
