"""Several GPUs as replicas, host side on the CPU: two gloo ranks each take their contiguous,
cell-balanced pair range, compute their shard's summed gradient (the CPU oracle stands in
for the device here) and all-reduce it; the result is the whole batch's gradient."""
import os
import socket

import numpy as np
import pytest

from conftest import AA, ROOT, encode, mutate, rand_matrix, rand_seqs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    rng = np.random.default_rng(77)
    mat = rand_matrix(rng, 20)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa = rand_seqs(rng, 37, 1, 60, AA) + [""]
    sb = [mutate(rng, s, AA) for s in sa[:-1]] + ["ACD"]
    return mat, gaps, sa, sb


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from datetime import timedelta
    import oracle
    from nwgrad_b200.params import AlignParams
    from nwgrad_b200.replicas import allreduce_grad, shard_pairs
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mat, gaps, sa, sb = _problem()
        la = np.array([len(s) for s in sa]); lb = np.array([len(s) for s in sb])
        oa = np.concatenate([[0], np.cumsum(la)]); ob = np.concatenate([[0], np.cumsum(lb)])
        lo, hi = shard_pairs(oa, ob, world, rank)
        enc = oracle.Encoded(encode(AA, sa[lo:hi]), encode(AA, sb[lo:hi]))
        _, g = oracle.soft(1, 0, mat, gaps, enc)
        v = g.sum(axis=0) if hi > lo else np.zeros(20 * 20 + 4)
        part = AlignParams._make(v[:400].reshape(1, 20, 20), v[400:].reshape(1, 4), AlignParams.from_arrays(
            mat, gaps, alphabet=AA).alphabet_obj)
        tot = allreduce_grad(part)
        np.save(os.path.join(out, f"r{rank}.npy"), np.concatenate([tot.matrices.ravel(), tot.gaps.ravel(), [lo, hi]]))
    finally:
        dist.destroy_process_group()


def test_shard_pairs_covers_the_batch_in_order():
    from nwgrad_b200.replicas import shard_pairs
    rng = np.random.default_rng(3)
    la = rng.integers(0, 500, size=1001); lb = rng.integers(0, 500, size=1001)
    oa = np.concatenate([[0], np.cumsum(la)]); ob = np.concatenate([[0], np.cumsum(lb)])
    for world in (1, 2, 3, 8):
        cuts = [shard_pairs(oa, ob, world, r) for r in range(world)]
        assert cuts[0][0] == 0 and cuts[-1][1] == 1001
        assert all(cuts[r][1] == cuts[r + 1][0] for r in range(world - 1))
        cells = la.astype(float) * lb + 1
        share = [cells[lo:hi].sum() / cells.sum() for lo, hi in cuts]
        assert max(share) <= 1.0 / world + cells.max() / cells.sum() + 1e-12


def test_two_gloo_ranks_allreduce_the_shard_gradients(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"r{r}.npy") for r in range(2))
    assert r0[-2] == 0 and r0[-1] == r1[-2] and r1[-1] == 38      # the two ranges tile the batch
    mat, gaps, sa, sb = _problem()
    _, g = oracle.soft(1, 0, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)))
    full = g.sum(axis=0)
    for r in (r0, r1):
        np.testing.assert_allclose(r[:-2], full, rtol=1e-12, atol=1e-9)
