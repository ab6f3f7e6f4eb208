"""Serving (continuous batching): every request's scores and gradient are the same bits as the
request aligned alone, whatever it was batched with; parameter updates apply to later requests."""
import numpy as np
import pytest

from conftest import AA, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402
from nwgrad_b200.serve import Server  # noqa: E402


def _requests(rng, k):
    out = []
    for _ in range(k):
        n = int(rng.integers(1, 40))
        sa = rand_seqs(rng, n, 5, 300, AA)
        sb = [mutate(rng, s, AA) for s in sa]
        out.append((sa, sb))
    return out


@pytest.mark.parametrize("grad_mode", ["hard", "soft"])
def test_request_results_alone_and_in_the_mix(grad_mode):
    rng = np.random.default_rng(5 if grad_mode == "hard" else 6)
    mat = rand_matrix(rng, 20)
    params = nw.AlignParams.from_arrays(mat, [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    reqs = _requests(rng, 24)
    with Server(params, grad_mode=grad_mode, workers=3, max_batch_pairs=200) as srv:
        tickets = [srv.submit(sa, sb) for sa, sb in reqs]          # submitted together: batched
        mixed = [srv.wait(t, len(r[0])) for t, r in zip(tickets, reqs)]
        alone = []
        for sa, sb in reqs:                                          # one at a time: alone
            alone.append(srv.wait(srv.submit(sa, sb), len(sa)))
        st = srv.stats()
    assert st["done"] == 2 * len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    assert st["batches"] < 2 * len(reqs)                             # some requests shared a batch
    for (sa, sb), (s1, g1, _), (s2, g2, _) in zip(reqs, mixed, alone):
        b = nw.SeqPairBatch(sa, sb, params, grad_mode=grad_mode)
        b.score_and_grad()
        g = b.compute_grad()
        assert np.array_equal(s1, s2) and np.array_equal(s1, b.scores())
        for x in (g1, g2):
            assert np.array_equal(x.matrices, g.matrices) and np.array_equal(x.gaps, g.gaps)


def test_set_params_applies_to_later_requests():
    rng = np.random.default_rng(8)
    p1 = nw.AlignParams.from_arrays(rand_matrix(rng, 20), [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    p2 = nw.AlignParams.from_arrays(rand_matrix(rng, 20), [[10.0, 2.0, 10.0, 2.0]], alphabet=AA)
    sa = rand_seqs(rng, 10, 20, 80, AA)
    sb = rand_seqs(rng, 10, 20, 80, AA)
    with Server(p1, grad_mode="hard", workers=2) as srv:
        t1 = srv.submit(sa, sb)
        srv.set_params(p2)
        t2 = srv.submit(sa, sb)
        s1, _, _ = srv.wait(t1, 10)
        s2, _, _ = srv.wait(t2, 10)
    for p, s in ((p1, s1), (p2, s2)):
        b = nw.SeqPairBatch(sa, sb, p)
        b.score_and_grad()
        assert np.array_equal(b.scores(), s)


def test_concurrent_batches_overlap_on_the_device():
    """A burst of requests larger than one worker's batch: the workers' batches are in flight
    on the device at the same time -- the sum of their device intervals (CUDA events around
    each batch's run) exceeds the time the device had any batch in flight."""
    rng = np.random.default_rng(9)
    mat = rand_matrix(rng, 20)
    params = nw.AlignParams.from_arrays(mat, [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    reqs = []
    for _ in range(12):
        sa = rand_seqs(rng, 150, 200, 400, AA)
        reqs.append((sa, [mutate(rng, s, AA) for s in sa]))
    with Server(params, grad_mode="soft", workers=3, max_batch_pairs=300) as srv:
        tickets = [srv.submit(sa, sb) for sa, sb in reqs]
        for t, (sa, _) in zip(tickets, reqs):
            srv.wait(t, len(sa))
        st = srv.stats()
    assert st["batches"] >= 6
    assert st["device_sum_ms"] > st["device_busy_ms"] > 0, st
