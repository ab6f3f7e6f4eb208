"""Stored paths (keep_paths=True): the moves bit for bit the oracle's, and their formats
(aligned strings, Biopython coordinates, SAM CIGAR, the formatted block) read off them."""
import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402


@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_moves_and_formats(gm, am):
    rng = np.random.default_rng(2300 + gm + 2 * am)
    mat = rand_matrix(rng, 20)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    sa = rand_seqs(rng, 20, 1, 150, AA) + ["", "ACD"]
    sb = [mutate(rng, s, AA) for s in sa[:-2]] + ["WW", ""]
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    b = nw.SeqPairBatch(sa, sb, p, gap_model=("linear", "affine")[gm], mode=("global", "local")[am], grad_mode="hard")
    b.score_and_grad(keep_paths=True)
    cap = max(len(x) + len(y) for x, y in zip(sa, sb)) + 1
    o = oracle.hard(32, gm, am, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)), moves_cap=cap)
    mo, mv, info = b._stored()
    for i in range(len(sa)):
        k = int(info[i, 0])
        assert k == int(o["nmoves"][i])
        assert np.array_equal(mv[mo[i]:mo[i] + k], o["moves"][i, :k])
        assert (info[i, 1], info[i, 2]) == (o["ends"][i, 2], o["ends"][i, 3])
        a_al, b_al = b[i].aligned()
        assert len(a_al) == len(b_al) == k
        si, sj = int(info[i, 1]), int(info[i, 2])
        ei, ej = int(o["ends"][i, 0]), int(o["ends"][i, 1])
        assert a_al.replace("-", "") == sa[i][si:ei] and b_al.replace("-", "") == sb[i][sj:ej]
        co = b[i].coordinates()
        assert co.shape[0] == 2 and (co[0, 0], co[1, 0]) == (si, sj) and (co[0, -1], co[1, -1]) == (ei, ej)
        cg = b[i].cigar()
        ops = [(int(n), t) for n, t in __import__("re").findall(r"(\d+)([MID])", cg)]
        assert sum(n for n, t in ops if t in "MI") == ei - si and sum(n for n, t in ops if t in "MD") == ej - sj
        ext = b[i].cigar(extended=True, soft_clip=True)
        lead = si if si else 0
        assert ext.startswith(f"{lead}S") or lead == 0
        fm = b[i].formatted(width=10)
        assert fm.replace("\n", "").count("|") == sum(1 for x, y in zip(a_al, b_al) if x == y and x != "-")
    assert b.cigars() == [b[i].cigar() for i in range(len(sa))]


def test_known_alignment_formats():
    """ACGT against AGT, +5 / -4, linear gap 3: one deletion of C."""
    mat = np.full((4, 4), -4.0)
    np.fill_diagonal(mat, 5.0)
    p = nw.AlignParams.from_arrays(mat, [[0.0, 3.0, 0.0, 3.0]], alphabet="ACGT")
    b = nw.SeqPairBatch(["ACGT"], ["AGT"], p, gap_model="linear", grad_mode="hard")
    b.score_and_grad(keep_paths=True)
    assert b[0].aligned() == ("ACGT", "A-GT")
    assert b[0].cigar() == "1M1I2M"
    assert b[0].cigar(extended=True) == "1=1I2="
    assert b[0].coordinates().tolist() == [[0, 1, 2, 4], [0, 1, 1, 3]]
    assert b[0].formatted() == "ACGT\n| ||\nA-GT"
    b.drop_paths()
    with pytest.raises(RuntimeError, match="stored path"):
        b[0].aligned()


@pytest.mark.parametrize("grad_mode", ["hard", "soft"])
def test_streaming_align(grad_mode):
    """align(): the batch's problem type on pairs it does not hold; full and banded."""
    rng = np.random.default_rng(2400)
    mat = rand_matrix(rng, 20, integer=False)
    gaps = np.array([[3.0, 0.5, 3.0, 0.5]])
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    host = nw.SeqPairBatch(["ACD"], ["ACE"], p, grad_mode=grad_mode)
    sa = rand_seqs(rng, 30, 5, 120, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    r = host.align(sa, sb, p)
    ref = nw.SeqPairBatch(sa, sb, p, grad_mode=grad_mode)
    ref.score_and_grad()
    assert np.array_equal(r.scores, ref.scores())
    g = ref.compute_grad()
    assert np.array_equal(r.grad.matrices, g.matrices) and np.array_equal(r.grad.gaps, g.gaps)
    # banded around the diagonal (no aligned strings) against the oracle's banded pass
    rb = host.align(sa, sb, p, band=6)
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    diag = np.concatenate([[int(np.floor(i * len(y) / len(x) + 0.5)) if len(x) else 0 for i in range(len(x) + 1)]
                           for x, y in zip(sa, sb)]).astype(np.int32)
    if grad_mode == "hard":
        o = oracle.hard(32, 1, 0, mat, gaps, enc, guides_in=diag, band=6)
        assert np.array_equal(rb.scores, o["scores"])
    else:
        so, _ = oracle.soft(1, 0, mat, gaps, enc, guides_in=diag, band=6)
        np.testing.assert_allclose(rb.scores, so, rtol=1e-4, atol=1e-5)
    # banded around given alignments
    aa = [x for x in sa]
    ab = [x for x in sa]      # the identity alignment of A with itself: guide i -> i
    with pytest.raises(ValueError):
        host.align(sa, sb, p, band=3, aligned_a=aa[:-1], aligned_b=ab[:-1])
    assert nw.guide_j_from_aligned("AC-GT", "A-TGT") == [0, 1, 1, 3, 4]
