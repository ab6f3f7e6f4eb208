"""Grid traceback (traceback="grid", aligner.hpp:89-100): pairs of 1,536+ rows and 256+ columns
fill score-only over tiles of 256 x 256 cells, keeping each stripe's bottom row and each tile's
last column, then walk back refilling only the tiles the path crosses.  The result is the
Pointers result bit for bit: scores, per-pair gradients, guides and every move of the stored
path, against the oracle."""
import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402


def _pairs(rng, homolog_long=True):
    sa = rand_seqs(rng, 6, 1, 150, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    long_a = rand_seqs(rng, 3, 1600, 2600, AA)
    sa += long_a
    sb += [mutate(rng, s, AA) for s in long_a] if homolog_long else rand_seqs(rng, 3, 1600, 2600, AA)
    for la, lb in ((1536, 256), (1537, 257), (2049, 513), (1600, 2900)):
        sa += rand_seqs(rng, 1, la, la, AA)
        sb += rand_seqs(rng, 1, lb, lb, AA)
    return sa, sb


def _check(prec, gm, am, mat, gaps, sa, sb, tracks=None, K=1):
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    kw = dict(gap_model=("linear", "affine")[gm], mode=("global", "local")[am], grad_mode="hard", tracks=tracks)
    g = cls(sa, sb, p, traceback="grid", **kw)
    tot = g.score_and_grad(keep_paths=True)
    cap = max(len(x) + len(y) for x, y in zip(sa, sb)) + 1
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb), tracks)
    o = oracle.hard(prec, gm, am, mat, gaps, enc, tracked=tracks is not None, moves_cap=cap)
    assert np.array_equal(g.scores(), o["scores"]), np.nonzero(g.scores() != o["scores"])[0][:5]
    assert tot == float(np.cumsum(o["scores"])[-1])
    gmat, ggap = g.grads()
    if tracks is None:
        gmat = gmat[:, None]
        ggap = ggap[:, None]
    flat = np.concatenate([gmat.reshape(len(sa), -1), ggap.reshape(len(sa), -1)], axis=1)
    assert np.array_equal(flat, o["grads"]), np.nonzero((flat != o["grads"]).any(1))[0][:5]
    assert np.array_equal(g.guides(), o["guides"])
    mo, mv, info = g._stored()
    for i in range(len(sa)):
        k = int(info[i, 0])
        assert k == int(o["nmoves"][i]), i
        assert np.array_equal(mv[mo[i]:mo[i] + k], o["moves"][i, :k]), i
        assert (info[i, 1], info[i, 2]) == (o["ends"][i, 2], o["ends"][i, 3]), i


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_grid_bit_exact(prec, gm, am):
    rng = np.random.default_rng(2700 + prec + gm + 2 * am)
    mat = rand_matrix(rng, 20, 1, integer=(gm == 1))
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if gm == 1 else np.array([[0.0, 2.5, 0.0, 2.5]])
    sa, sb = _pairs(rng)
    _check(prec, gm, am, mat, gaps, sa, sb)


@pytest.mark.parametrize("am", [0, 1])
def test_grid_unrelated_long_pairs(am):
    """Random (unrelated) long pairs: paths with long gap runs and, Local, short local
    alignments anywhere in the table."""
    rng = np.random.default_rng(2750 + am)
    mat = rand_matrix(rng, 20, 1, integer=True)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa, sb = _pairs(rng, homolog_long=False)
    _check(32, 1, am, mat, gaps, sa, sb)


def test_grid_tracked():
    """Tracked rows (three parameter sets): the tiles refill with each row's own set."""
    rng = np.random.default_rng(2780)
    mat = rand_matrix(rng, 20, 3, integer=True)
    gaps = np.tile([11.0, 1.0, 11.0, 1.0], (3, 1)) + rng.integers(0, 3, size=(3, 4))
    sa, sb = _pairs(rng)
    tr = np.concatenate([rng.integers(0, 3, size=len(s)) for s in sa]).astype(np.uint16)
    _check(32, 1, 0, mat, gaps, sa, sb, tracks=tr, K=3)


def test_grid_matches_pointers_after_set_params():
    """A parameter step: grid and Pointers batches agree on scores, gradients and guides."""
    rng = np.random.default_rng(2790)
    mat = rand_matrix(rng, 20, 1, integer=False)
    gaps = np.array([[10.0, 1.0, 10.0, 1.0]])
    sa, sb = _pairs(rng)
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    g = nw.SeqPairBatch(sa, sb, p, grad_mode="hard", traceback="grid")
    q = nw.SeqPairBatch(sa, sb, p, grad_mode="hard", traceback="pointers")
    for step in range(2):
        g.score_and_grad()
        q.score_and_grad()
        assert np.array_equal(g.scores(), q.scores())
        cg, cq = g.compute_grad(), q.compute_grad()
        assert np.array_equal(cg.matrices, cq.matrices) and np.array_equal(cg.gaps, cq.gaps)
        assert np.array_equal(g.guides(), q.guides())
        p2 = p + cg * 1e-3
        g.set_params(p2)
        q.set_params(p2)
