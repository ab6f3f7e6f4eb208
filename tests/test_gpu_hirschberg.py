"""Hirschberg re-alignment on the GPU (traceback "hirschberg" / "hirschberg_pmax"; affine and
linear gaps, Global and Local, affine glocal ends): scores, gradients and guides bit for bit against the reference's own engine
(tests/golden/hirschberg.npz) and against the oracle's restatement on longer pairs."""
import os

import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _run(prec, tb, cut, mat, gaps, sa, sb, mode="global", gap_model="affine"):
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="hard", traceback=tb, mode=mode,
            gap_model=gap_model)
    b.hb_cutoff = cut
    tot = b.score_and_grad()
    gm, gg = b.grads()
    flat = np.concatenate([gm.reshape(len(sa), -1), gg.reshape(len(sa), -1)], axis=1)
    return b.scores(), flat, b.guides(), tot


@pytest.mark.parametrize("name", ["int", "flt"])
@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("tb", ["hirschberg", "hirschberg_pmax"])
@pytest.mark.parametrize("cut", [8, 64])
@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("gap_model", ["affine", "linear"])
def test_reference_fixtures(name, prec, tb, cut, mode, gap_model):
    z = np.load(os.path.join(GOLD, "hirschberg.npz"))
    sa, sb = [str(s) for s in z[f"{name}_sa"]], [str(s) for s in z[f"{name}_sb"]]
    s, g, gj, tot = _run(prec, tb, cut, z[f"{name}_mat"], z[f"{name}_gaps"], sa, sb, mode, gap_model)
    tag = ("lin" if gap_model == "linear" else "") + ("L" if mode == "local" else "")
    key = f"{name}_{tag + '_' if tag else ''}{tb}_{prec}_c{cut}_"
    assert np.array_equal(s, z[key + "scores"]), np.nonzero(s != z[key + "scores"])[0][:5]
    assert np.array_equal(g, z[key + "grads"])
    assert np.array_equal(gj, z[key + "guides"])
    assert tot == float(np.cumsum(z[key + "scores"])[-1])


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("tb", ["hirschberg", "hirschberg_pmax"])
@pytest.mark.parametrize("cut", [8, 64])
@pytest.mark.parametrize("mode", ["global", "local", "glocal"])
@pytest.mark.parametrize("use_gt", [False, True])
def test_tracked_affine_reference_fixtures(prec, tb, cut, mode, use_gt):
    """Tracked affine Hirschberg (three parameter sets per residue of A, gap sets per DP row
    or from the residues): every row's own substitution set and gap costs, the reverse sweep's
    rewritten vertical moves (hb_reverse_rows_, aligner.hpp:1848-1871), the open refunded at
    the cut from row p + 1 -- scores, gradients and guides bit for bit the reference engine's
    (tests/golden/hirschberg_tracked.npz)."""
    z = np.load(os.path.join(GOLD, "hirschberg_tracked.npz"))
    sa, sb = [str(s) for s in z["sa"]], [str(s) for s in z["sb"]]
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, nw.AlignParams.from_arrays(z["mat"], z["gaps"], alphabet=AA), grad_mode="hard", traceback=tb,
            mode=mode, tracks=z["tracks"], gap_tracks=z["gap_tracks"] if use_gt else None)
    b.hb_cutoff = cut
    b.score_and_grad()
    gm, gg = b.grads()
    flat = np.concatenate([gm.reshape(len(sa), -1), gg.reshape(len(sa), -1)], axis=1)
    key = f"{dict(global_='G_', local_='L_', glocal_='g_')[mode + '_']}{'gt_' if use_gt else ''}{tb}_{prec}_c{cut}_"
    assert np.array_equal(b.scores(), z[key + "scores"]), np.nonzero(b.scores() != z[key + "scores"])[0][:5]
    assert np.array_equal(flat, z[key + "grads"]), np.nonzero((flat != z[key + "grads"]).any(1))[0][:5]
    assert np.array_equal(b.guides(), z[key + "guides"])


@pytest.mark.parametrize("pmax", [False, True])
@pytest.mark.parametrize("mode", ["global", "local"])
def test_tiled_half_sweeps_against_the_oracle(pmax, mode):
    """Pairs of 7,000-9,000 residues: the half-sweeps of the top levels (8M cells and more) run
    as tiles over the whole device (hb_tile_kernel), the rest as one block each; scores,
    gradients and guides bit for bit the oracle's restatement of the reference's recursion."""
    rng = np.random.default_rng(2500 + pmax + 2 * (mode == "local"))
    mat = rand_matrix(rng, 20, integer=False)
    gaps = np.array([[3.1, 0.7, 2.9, 0.8]])
    sa = rand_seqs(rng, 3, 7000, 9000, AA) + rand_seqs(rng, 4, 600, 2000, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    tb = "hirschberg_pmax" if pmax else "hirschberg"
    s, g, gj, tot = _run(32, tb, 512, mat, gaps, sa, sb, mode)
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    o = oracle.hirschberg(32, mat, gaps, enc, cutoff=512, pmax=pmax, local=(mode == "local"))
    assert np.array_equal(s, o["scores"]), np.nonzero(s != o["scores"])[0][:5]
    assert np.array_equal(g, o["grads"])
    assert np.array_equal(gj, o["guides"])


@pytest.mark.parametrize("name", ["int", "flt"])
@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("tb", ["hirschberg", "hirschberg_pmax"])
@pytest.mark.parametrize("cut", [8, 64])
@pytest.mark.parametrize("gap_model", ["affine", "linear"])
def test_glocal_reference_fixtures(name, prec, tb, cut, gap_model):
    """Glocal ends (affine: viterbi_affine_hirschberg_glocal, aligner.hpp:4709; linear: the
    glocal branch of viterbi_linear_hirschberg, :5132): the end and start scans, the box's
    global solve with its free leading moves dropped -- scores, gradients and guides bit for
    bit the reference engine's (tests/golden/hirschberg_glocal.npz: A within a longer B,
    pairs without B)."""
    z = np.load(os.path.join(GOLD, "hirschberg_glocal.npz"))
    sa, sb = [str(s) for s in z[f"{name}_sa"]], [str(s) for s in z[f"{name}_sb"]]
    s, g, gj, tot = _run(prec, tb, cut, z[f"{name}_mat"], z[f"{name}_gaps"], sa, sb, "glocal", gap_model)
    key = f"{name}_{'lin_' if gap_model == 'linear' else ''}{tb}_{prec}_c{cut}_"
    assert np.array_equal(s, z[key + "scores"]), np.nonzero(s != z[key + "scores"])[0][:5]
    assert np.array_equal(g, z[key + "grads"]), np.nonzero((g != z[key + "grads"]).any(1))[0][:5]
    assert np.array_equal(gj, z[key + "guides"])


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("pmax", [False, True])
@pytest.mark.parametrize("gap_model", ["affine", "linear"])
def test_glocal_long_pairs_against_the_oracle(prec, pmax, gap_model):
    """Glocal pairs of 1,000-4,000 residues within longer B: the same score as the oracle's
    glocal Pointers (any optimal path), a path that scores it (the replayed gradient's
    substitution and gap counts give the score back), and keep_paths moves that start on
    row 0 and end on row m."""
    rng = np.random.default_rng(2600 + prec + pmax + 7 * (gap_model == "linear"))
    mat = rand_matrix(rng, 20, integer=True)
    gm = 1 if gap_model == "affine" else 0
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if gm else np.array([[0.0, 3.0, 0.0, 3.0]])
    sa = rand_seqs(rng, 5, 1000, 4000, AA) + rand_seqs(rng, 6, 1, 300, AA)
    sb = []
    for k, a in enumerate(sa):
        core = mutate(rng, a, AA) if k % 3 else rand_seqs(rng, 1, 200, 3000, AA)[0]
        sb.append(rand_seqs(rng, 1, 0, 500, AA)[0] + core + rand_seqs(rng, 1, 0, 500, AA)[0])
    tb = "hirschberg_pmax" if pmax else "hirschberg"
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    b = cls(sa, sb, p, grad_mode="hard", traceback=tb, mode="glocal", gap_model=gap_model)
    b.score_and_grad(keep_paths=True)
    o = oracle.hard(prec, gm, 2, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)), free_ends=12)
    np.testing.assert_array_equal(b.scores(), o["scores"])
    gm, gg = b.grads()
    flat = np.concatenate([gm.reshape(len(sa), -1), gg.reshape(len(sa), -1)], axis=1)
    w = np.concatenate([mat.reshape(-1), gaps.reshape(-1)])
    np.testing.assert_allclose(flat @ w, o["scores"], rtol=1e-6)
    for i in range(len(sa)):
        a_al, b_al = b[i].aligned()
        assert a_al.replace("-", "") == sa[i]


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("pmax", [False, True])
@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("gap_model", ["affine", "linear"])
def test_long_pairs_against_the_oracle(prec, pmax, mode, gap_model):
    """Pairs of 1,000-6,000 residues (several recursion levels, multi-round pipelines) mixed
    with short pairs that run the Pointers path; Local: homologous cores inside unrelated
    flanks (a box well inside the pair), and unrelated pairs."""
    rng = np.random.default_rng(2000 + prec + pmax + 10 * (mode == "local"))
    mat = rand_matrix(rng, 20, integer=False)
    gaps = np.array([[3.1, 0.7, 2.9, 0.8]])
    sa = rand_seqs(rng, 6, 1000, 6000, AA) + rand_seqs(rng, 10, 1, 300, AA)
    sb = [mutate(rng, s, AA) if k % 3 else rand_seqs(rng, 1, 500, 4000, AA)[0] for k, s in enumerate(sa)]
    if mode == "local":
        sb = [rand_seqs(rng, 1, 10, 400, AA)[0] + t + rand_seqs(rng, 1, 10, 400, AA)[0] if k % 3 else t
              for k, t in enumerate(sb)]
    cut = 256
    s, g, gj, _ = _run(prec, "hirschberg_pmax" if pmax else "hirschberg", cut, mat, gaps, sa, sb, mode, gap_model)
    o = oracle.hirschberg(prec, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb)), cutoff=cut, pmax=pmax,
                          local=mode == "local", linear=gap_model == "linear")
    assert np.array_equal(s, o["scores"]), np.nonzero(s != o["scores"])[0][:5]
    assert np.array_equal(g, o["grads"]), np.nonzero((g != o["grads"]).any(1))[0][:5]
    assert np.array_equal(gj, o["guides"])


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("cut", [8, 64])
@pytest.mark.parametrize("mode", ["global", "local"])
def test_tracked_linear_reference_fixtures(prec, cut, mode):
    """Linear Hirschberg with three parameter sets (per-residue tracks, per-row gap tracks)
    against the reference's own engine (tests/golden/hirschberg.npz, trk_*)."""
    z = np.load(os.path.join(GOLD, "hirschberg.npz"))
    sa, sb = [str(s) for s in z["trk_sa"]], [str(s) for s in z["trk_sb"]]
    cls = nw.SeqPairBatch if prec == 32 else nw.SeqPairBatchDouble
    b = cls(sa, sb, nw.AlignParams.from_arrays(z["trk_mat"], z["trk_gaps"], alphabet=AA), grad_mode="hard",
            traceback="hirschberg", mode=mode, gap_model="linear", tracks=z["trk_tracks"],
            gap_tracks=z["trk_gap_tracks"])
    b.hb_cutoff = cut
    b.score_and_grad()
    gm, gg = b.grads()
    flat = np.concatenate([gm.reshape(len(sa), -1), gg.reshape(len(sa), -1)], axis=1)
    key = f"trk_{'linLT_' if mode == 'local' else 'linT_'}hirschberg_{prec}_c{cut}_"
    assert np.array_equal(b.scores(), z[key + "scores"]), np.nonzero(b.scores() != z[key + "scores"])[0][:5]
    assert np.array_equal(flat, z[key + "grads"])
    assert np.array_equal(b.guides(), z[key + "guides"])


@pytest.mark.parametrize("mode", ["global", "local"])
def test_tracked_linear_long_pairs_against_the_oracle(mode):
    rng = np.random.default_rng(2300 + (mode == "local"))
    K = 3
    mat = rand_matrix(rng, 20, K, integer=False)
    gaps = rng.uniform(0.3, 3.0, size=(K, 4))
    sa = rand_seqs(rng, 5, 1000, 4000, AA) + rand_seqs(rng, 6, 1, 300, AA)
    sb = [mutate(rng, s, AA) if k % 3 else rand_seqs(rng, 1, 500, 3000, AA)[0] for k, s in enumerate(sa)]
    tr = np.concatenate([rng.integers(0, K, size=len(s)) for s in sa]).astype(np.uint16)
    gt = np.concatenate([rng.integers(0, K, size=len(s) + 1) for s in sa]).astype(np.uint16)
    b = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="hard",
                        traceback="hirschberg", mode=mode, gap_model="linear", tracks=tr, gap_tracks=gt)
    b.hb_cutoff = 200
    b.score_and_grad()
    gm, gg = b.grads()
    flat = np.concatenate([gm.reshape(len(sa), -1), gg.reshape(len(sa), -1)], axis=1)
    o = oracle.hirschberg(32, mat, gaps, oracle.Encoded(encode(AA, sa), encode(AA, sb), tr, gt), cutoff=200,
                          local=mode == "local", linear=True)
    assert np.array_equal(b.scores(), o["scores"]), np.nonzero(b.scores() != o["scores"])[0][:5]
    assert np.array_equal(flat, o["grads"]), np.nonzero((flat != o["grads"]).any(1))[0][:5]
    assert np.array_equal(b.guides(), o["guides"])


def test_score_matches_pointers_and_banded_follows():
    """Where the optimum is unique Hirschberg and Pointers agree; banded re-alignment then
    runs around the Hirschberg guide."""
    rng = np.random.default_rng(2100)
    mat = rand_matrix(rng, 20, integer=False)
    gaps = np.array([[3.0, 0.5, 3.0, 0.5]])
    sa = rand_seqs(rng, 4, 800, 1500, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    hb = nw.SeqPairBatch(sa, sb, p, grad_mode="hard", traceback="hirschberg")
    hb.hb_cutoff = 128
    hb.score_and_grad()
    pt = nw.SeqPairBatch(sa, sb, p, grad_mode="hard", traceback="pointers")
    pt.score_and_grad()
    np.testing.assert_allclose(hb.scores(), pt.scores(), rtol=1e-5)
    hb.set_params(nw.AlignParams.from_arrays(mat + 1e-3, gaps, alphabet=AA))
    hb.banded_grad(64)
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    o0 = oracle.hirschberg(32, mat, gaps, enc, cutoff=128)
    o = oracle.hard(32, 1, 0, mat + 1e-3, gaps, enc, guides_in=o0["guides"], band=64)
    assert np.array_equal(hb.scores(), o["scores"])


def test_errors():
    rng = np.random.default_rng(2200)
    mat = rand_matrix(rng, 20)
    sa = rand_seqs(rng, 2, 600, 700, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    neg = nw.AlignParams.from_arrays(mat, [[-1.0, 1.0, 11.0, 1.0]], alphabet=AA)
    b = nw.SeqPairBatch(sa, sb, neg, grad_mode="hard", traceback="hirschberg")
    with pytest.raises(ValueError, match="non-negative"):
        b.score_and_grad()
    # tracked linear glocal splits are not built (tracked affine ones are)
    tr = np.zeros(sum(len(s) for s in sa), np.uint16)
    trk = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, [[0.0, 1.0, 0.0, 1.0]], alphabet=AA),
                          grad_mode="hard", traceback="hirschberg", tracks=tr, mode="glocal", gap_model="linear")
    with pytest.raises(NotImplementedError):
        trk.score_and_grad()
    nlocal = nw.SeqPairBatch(sa, sb, neg, mode="local", grad_mode="hard", traceback="hirschberg_pmax")
    with pytest.raises(ValueError, match="non-negative"):
        nlocal.score_and_grad()
    with pytest.raises(ValueError):
        trk.hb_cutoff = 0
