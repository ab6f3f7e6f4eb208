"""The oracle pinned to the reference: its golden fixtures (the reference's brute-force
enumerator and its C++ batch engine, tests/golden/make_golden.py) and, where the reference
driver is built here, live random cases."""
import os

import numpy as np
import pytest

import oracle
from conftest import AA, encode, rand_matrix, rand_seqs

GOLD = os.path.join(os.path.dirname(__file__), "golden")
DNA = "ACGT"


def _enc1(alpha, a, b):
    return oracle.Encoded(encode(alpha, [a]), encode(alpha, [b]))


def test_bruteforce_fixtures():
    z = np.load(os.path.join(GOLD, "bruteforce.npz"))
    for k in range(len(z["a"])):
        a, b = str(z["a"][k]), str(z["b"][k])
        mat, gaps = z["mat"][k][None], z["gaps"][k][None]
        gm = 1 if bool(z["affine"][k]) else 0
        enc = _enc1(DNA, a, b)
        h = oracle.hard(64, gm, 0, mat, gaps, enc)
        assert h["scores"][0] == pytest.approx(z["global_score"][k], abs=1e-9)
        hl = oracle.hard(64, gm, 1, mat, gaps, enc)
        assert hl["scores"][0] == pytest.approx(z["local_score"][k], abs=1e-9)
        s, g = oracle.soft(gm, 0, mat, gaps, enc)
        assert s[0] == pytest.approx(z["log_z"][k], rel=1e-12, abs=1e-12)
        np.testing.assert_allclose(g[0], z["soft"][k], rtol=1e-9, atol=1e-12)
        if not np.isnan(z["hard"][k][0]):
            np.testing.assert_array_equal(h["grads"][0], z["hard"][k])


def _ref_cases():
    z = np.load(os.path.join(GOLD, "reference_batches.npz"))
    names = sorted({k.split("_")[0] for k in z.files})
    return z, names


@pytest.mark.parametrize("name", ["prot", "protf", "rna3"])
def test_reference_batch_fixtures(name):
    z, _ = _ref_cases()
    pre = name + "_"
    alpha = str(z[pre + "alpha"])
    sa, sb = [str(s) for s in z[pre + "sa"]], [str(s) for s in z[pre + "sb"]]
    tr = z[pre + "tracks"] if pre + "tracks" in z.files else None
    gt = z[pre + "gap_tracks"] if pre + "gap_tracks" in z.files else None
    enc = oracle.Encoded(encode(alpha, sa), encode(alpha, sb), tr, gt)
    tracked = tr is not None
    mat, gaps, mat2, gaps2 = z[pre + "mat"], z[pre + "gaps"], z[pre + "mat2"], z[pre + "gaps2"]
    for gm in (0, 1):
        for am in (0, 1):
            for prec in (32, 64):
                key = f"{pre}hard{prec}_g{gm}_m{am}_"
                o = oracle.hard(prec, gm, am, mat, gaps, enc, tracked=tracked)
                np.testing.assert_array_equal(o["scores"], z[key + "scores"])
                np.testing.assert_array_equal(o["grads"], z[key + "grads"])
                np.testing.assert_array_equal(o["guides"], z[key + "guides"])
                key = f"{pre}band{prec}_g{gm}_m{am}_"
                ob = oracle.hard(prec, gm, am, mat2, gaps2, enc, tracked=tracked, guides_in=o["guides"], band=4)
                np.testing.assert_array_equal(ob["scores"], z[key + "scores"])
                np.testing.assert_array_equal(ob["grads"], z[key + "grads"])
                np.testing.assert_array_equal(ob["guides"], z[key + "guides"])
            for T in (1.0, 0.5):
                key = f"{pre}soft_T{T}_g{gm}_m{am}_"
                s, g = oracle.soft(gm, am, mat, gaps, enc, T)
                np.testing.assert_allclose(s, z[key + "scores"], rtol=1e-11, atol=1e-11)
                np.testing.assert_allclose(g, z[key + "grads"], rtol=1e-9, atol=1e-10)


SG_SETS = (12, 15, 9, 6, 3, 0)   # free_ends bits: 1 a_begin, 2 a_end, 4 b_begin, 8 b_end


@pytest.mark.parametrize("name", ["prot", "protf", "rna3"])
def test_semiglobal_fixtures(name):
    """Semi-global ends (glocal, overlap, mixed free_ends) against the reference engine."""
    z = np.load(os.path.join(GOLD, "semiglobal.npz"))
    pre = name + "_"
    alpha = str(z[pre + "alpha"])
    sa, sb = [str(s) for s in z[pre + "sa"]], [str(s) for s in z[pre + "sb"]]
    tr = z[pre + "tracks"] if pre + "tracks" in z.files else None
    gt = z[pre + "gap_tracks"] if pre + "gap_tracks" in z.files else None
    enc = oracle.Encoded(encode(alpha, sa), encode(alpha, sb), tr, gt)
    mat, gaps = z[pre + "mat"], z[pre + "gaps"]
    for fe in SG_SETS:
        for gm in (0, 1):
            for prec in (32, 64):
                key = f"{pre}hard{prec}_g{gm}_e{fe}_"
                o = oracle.hard(prec, gm, 2, mat, gaps, enc, tracked=tr is not None, free_ends=fe)
                np.testing.assert_array_equal(o["scores"], z[key + "scores"], err_msg=key)
                np.testing.assert_array_equal(o["grads"], z[key + "grads"], err_msg=key)
                np.testing.assert_array_equal(o["guides"], z[key + "guides"], err_msg=key)
            key = f"{pre}soft_g{gm}_e{fe}_"
            s, g = oracle.soft(gm, 2, mat, gaps, enc, 1.0, free_ends=fe)
            np.testing.assert_allclose(s, z[key + "scores"], rtol=1e-11, atol=1e-11, err_msg=key)
            np.testing.assert_allclose(g, z[key + "grads"], rtol=1e-9, atol=1e-10, err_msg=key)
            if fe == 12 and tr is None:
                mat2, gaps2 = z[pre + "mat2"], z[pre + "gaps2"]
                for prec in (32, 64):
                    o = oracle.hard(prec, gm, 2, mat, gaps, enc, free_ends=fe)
                    key = f"{pre}band{prec}_g{gm}_e{fe}_"
                    ob = oracle.hard(prec, gm, 2, mat2, gaps2, enc, guides_in=o["guides"], band=4, free_ends=fe)
                    np.testing.assert_array_equal(ob["scores"], z[key + "scores"], err_msg=key)
                    np.testing.assert_array_equal(ob["grads"], z[key + "grads"], err_msg=key)
                    np.testing.assert_array_equal(ob["guides"], z[key + "guides"], err_msg=key)
                o = oracle.hard(64, gm, 2, mat, gaps, enc, free_ends=fe)
                key = f"{pre}softband_g{gm}_e{fe}_"
                s, g = oracle.soft(gm, 2, mat2, gaps2, enc, 1.0, guides_in=o["guides"], band=4, free_ends=fe)
                np.testing.assert_allclose(s, z[key + "scores"], rtol=1e-11, atol=1e-11, err_msg=key)
                np.testing.assert_allclose(g, z[key + "grads"], rtol=1e-9, atol=1e-10, err_msg=key)


def test_blocked_sum_order():
    """Blocks of 4096 in pair order, then the blocks in order (batch_engine.hpp:1788-1827)."""
    rng = np.random.default_rng(3)
    g = rng.normal(size=(9000, 7))
    w = rng.normal(size=9000)
    out = oracle.blocked_sum(g, w)
    ref = np.zeros(7)
    for b0 in range(0, 9000, 4096):
        acc = np.zeros(7)
        for p in range(b0, min(9000, b0 + 4096)):
            acc = acc + w[p] * g[p]
        ref = ref + acc
    np.testing.assert_array_equal(out, ref)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference driver not built here")
@pytest.mark.parametrize("gm", [0, 1])
@pytest.mark.parametrize("am", [0, 1])
def test_live_reference_random(gm, am):
    rng = np.random.default_rng(50 + gm + 2 * am)
    for prec in (32, 64):
        mat = rand_matrix(rng, 20, 1, integer=False)
        gaps = rng.uniform(0.2, 3.0, size=(1, 4))
        sa = rand_seqs(rng, 30, 0, 50, AA)
        sb = rand_seqs(rng, 30, 0, 50, AA)
        enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
        o = oracle.hard(prec, gm, am, mat, gaps, enc)
        r = oracle.ref_run(prec, gm, am, 1, AA, mat, gaps, sa, sb)
        np.testing.assert_array_equal(o["scores"], r["scores"])
        np.testing.assert_array_equal(o["grads"], r["grads"])
        np.testing.assert_array_equal(o["guides"], r["guides"])


def test_hirschberg_fixtures():
    """The Hirschberg restatement (affine exact and prefix-max carry, linear; Global and Local) against the
    reference's own engine with traceback hirschberg / hirschberg_pmax
    (tests/golden/hirschberg.npz)."""
    z = np.load(os.path.join(GOLD, "hirschberg.npz"))
    for name in ("int", "flt"):
        sa, sb = [str(s) for s in z[f"{name}_sa"]], [str(s) for s in z[f"{name}_sb"]]
        enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
        for prec in (32, 64):
            for tb in ("hirschberg", "hirschberg_pmax"):
                for cut in (8, 64):
                    for linear, local, tag in ((False, False, ""), (False, True, "L_"), (True, False, "lin_"),
                                               (True, True, "linL_")):
                        key = f"{name}_{tag}{tb}_{prec}_c{cut}_"
                        o = oracle.hirschberg(prec, z[f"{name}_mat"], z[f"{name}_gaps"], enc, cutoff=cut,
                                              pmax=tb.endswith("pmax"), local=local, linear=linear)
                        np.testing.assert_array_equal(o["scores"], z[key + "scores"])
                        np.testing.assert_array_equal(o["grads"], z[key + "grads"])
                        np.testing.assert_array_equal(o["guides"], z[key + "guides"])


def test_hirschberg_tracked_linear_fixtures():
    """Linear Hirschberg with three parameter sets (per-residue tracks, per-row gap tracks)
    against the reference's own engine (tests/golden/hirschberg.npz, trk_*)."""
    z = np.load(os.path.join(GOLD, "hirschberg.npz"))
    sa, sb = [str(s) for s in z["trk_sa"]], [str(s) for s in z["trk_sb"]]
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb), z["trk_tracks"], z["trk_gap_tracks"])
    for prec in (32, 64):
        for cut in (8, 64):
            for local, tag in ((False, "linT_"), (True, "linLT_")):
                key = f"trk_{tag}hirschberg_{prec}_c{cut}_"
                o = oracle.hirschberg(prec, z["trk_mat"], z["trk_gaps"], enc, cutoff=cut, local=local, linear=True)
                np.testing.assert_array_equal(o["scores"], z[key + "scores"])
                np.testing.assert_array_equal(o["grads"], z[key + "grads"])
                np.testing.assert_array_equal(o["guides"], z[key + "guides"])


def test_soft_banded_fixtures():
    """The guide-banded soft restatement against the reference's own engine
    (tests/golden/soft_banded.npz): guides from the Viterbi pass under the first parameters,
    the banded forward-backward under the second."""
    z = np.load(os.path.join(GOLD, "soft_banded.npz"))
    sa, sb = [str(s) for s in z["sa"]], [str(s) for s in z["sb"]]
    enc = oracle.Encoded(encode(AA, sa), encode(AA, sb))
    for gm in (0, 1):
        for am in (0, 1):
            g0 = oracle.hard(64, gm, am, z["mat"], z["gaps"], enc)["guides"]
            for bw in (1, 3, 8):
                s, g = oracle.soft(gm, am, z["mat2"], z["gaps2"], enc, guides_in=g0, band=bw)
                np.testing.assert_allclose(s, z[f"g{gm}_m{am}_b{bw}_scores"], rtol=1e-12, atol=1e-12)
                np.testing.assert_allclose(g, z[f"g{gm}_m{am}_b{bw}_grads"], rtol=1e-10, atol=1e-12)


def test_posterior_guides_pinned_to_the_reference():
    """The oracle's soft_guide="posterior" (per-row argmax of exit mass, made monotone) against
    the reference engine's guides (tests/golden/posterior.npz, make_golden.py post): every gap
    model and end mode, DNA and protein, T 1 and 0.5; the scores to 1e-9."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "posterior.npz"))
    for N in (4, 20):
        key = f"N{N}_"
        alpha = str(z[key + "alpha"])
        sa, sb = [str(s) for s in z[key + "sa"]], [str(s) for s in z[key + "sb"]]
        lut = {c: i for i, c in enumerate(alpha)}
        enc = oracle.Encoded([[lut[c] for c in s] for s in sa], [[lut[c] for c in s] for s in sb])
        n = sum(len(s) + 1 for s in sa)
        for gm in (0, 1):
            for am, fe in ((0, 12), (1, 12), (2, 12), (2, 15)):
                for T in (1.0, 0.5):
                    pre = f"{key}g{gm}_m{am}_e{fe}_T{T}_"
                    s, _, post = oracle.soft(gm, am, z[key + "mat"], z[key + "gaps"], enc, T, free_ends=fe,
                                             posterior=True)
                    np.testing.assert_allclose(s, z[pre + "scores"], rtol=1e-9, atol=1e-9)
                    assert np.array_equal(post[:n], z[pre + "guides"][:n]), pre
