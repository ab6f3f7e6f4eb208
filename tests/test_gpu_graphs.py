"""Captured bucket sequences: a plan's per-bucket launches run as one CUDA graph, captured the
second time the same sequence runs (a batch run once launches directly) and replayed while the
launches are unchanged.  Results are bit-identical with graphs on and off; set_params steps
replay the captured graph (the weights live at a fixed address); a new batch or precision
captures again.
"""
import numpy as np
import pytest

from conftest import AA, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402


def _batch(rng, grad_mode, n=300, lo=20, hi=700, cls=None):
    mat = rand_matrix(rng, len(AA), 1, True)
    sa = rand_seqs(rng, n, lo, hi, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    p = nw.AlignParams.from_arrays(mat, [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    cls = cls or nw.SeqPairBatch
    return cls(sa, sb, p, grad_mode=grad_mode), p, mat


@pytest.mark.parametrize("grad_mode", ["soft", "hard"])
def test_graphs_same_results_and_replayed_across_set_params(grad_mode):
    rng = np.random.default_rng(41)
    b, p, mat = _batch(rng, grad_mode)
    ref, _, _ = _batch(np.random.default_rng(41), grad_mode)
    ref.use_graphs(False)
    for step in range(3):
        q = nw.AlignParams.from_arrays(mat + 0.25 * step, [[11.0 - step, 1.0, 11.0, 1.0 + 0.1 * step]], alphabet=AA)
        b.set_params(q)
        ref.set_params(q)
        t1 = b.score_and_grad()
        t0 = ref.score_and_grad()
        assert t1 == t0
        assert np.array_equal(b.scores(), ref.scores())
        g1, g0 = b.grads(), ref.grads()
        assert np.array_equal(g1[0], g0[0]) and np.array_equal(g1[1], g0[1])
    cap, rep = b.graph_stats()
    assert cap == 1 and rep == 1, (cap, rep)   # step 0 direct, step 1 captured, step 2 replayed
    assert ref.graph_stats() == (0, 0)


def test_graphs_banded_and_full_keep_their_own_capture():
    """Full and banded runs alternate without capturing again once the buffers they share have
    reached their sizes (a buffer that grows moves, which captures again)."""
    rng = np.random.default_rng(42)
    b, p, mat = _batch(rng, "hard", n=120, lo=50, hi=400)
    b.score_and_grad()
    b.banded_grad(16)
    b.score_and_grad()
    b.banded_grad(16)
    cap0, rep0 = b.graph_stats()
    for _ in range(2):
        b.score_and_grad()
        b.banded_grad(16)
    cap, rep = b.graph_stats()
    assert cap == cap0 and rep == rep0 + 4, (cap0, rep0, cap, rep)


def test_graphs_soft_refusal_rerun_unchanged():
    """A pair refused in float32 reruns in double outside the graph; the results match the
    graph-free run bit for bit."""
    rng = np.random.default_rng(43)
    mat = rand_matrix(rng, len(AA), 1, True)
    sa = rand_seqs(rng, 40, 50, 300, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    p = nw.AlignParams.from_arrays(mat, [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    out = []
    for graphs in (True, False):
        b = nw.SeqPairBatch(sa, sb, p, grad_mode="soft")
        b.soft_temperature = 0.05    # extreme weights: float32 refuses, double reruns
        b.use_graphs(graphs)
        try:
            tot = b.score_and_grad()
        except ValueError:
            tot = None
        out.append((tot, None if tot is None else b.scores().copy()))
    assert out[0][0] == out[1][0]
    if out[0][1] is not None:
        assert np.array_equal(out[0][1], out[1][1])
