"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Run in a checkout that has the reference sources (michalsta/nwgrad) at REF below and the
reference driver built (``make -C oracle ref``):

    python tests/golden/make_golden.py

Two sources, both the reference's own code run here:

* ``bruteforce.npz`` -- the reference test suite's exhaustive path enumerator
  (tests/Python/bruteforce.py, imported from the reference tree): global / local scores,
  global log Z and expected (soft) counts, and hard counts on unique optima, for tiny pairs.
* ``reference_batches.npz`` -- the reference's C++ batch engine (SeqPairBatchT, scalar
  backend, traceback "pointers"; soft: SeqPairBatchT<double>, log space) on seeded random
  batches: per-pair scores, gradients and guides, hard at float32 and float64, soft at
  T = 1 and 0.5, tracked with three parameter sets, and banded re-alignment after a step.
* ``hirschberg.npz`` -- the same engine with traceback "hirschberg" and "hirschberg_pmax"
  (affine Global, small hb_cutoff so pairs split several times), float32 and float64.
* ``soft_banded.npz`` -- SeqPairBatchT<double> soft (log space): score_and_grad, set_params,
  banded_grad(bw) around the Viterbi guides, every gap model and mode, bw 1, 3, 8.
* ``semiglobal.npz`` -- the batch engine with AlignMode::Glocal and free_ends sets (glocal,
  overlap, mixed): hard float32 / float64 with guides, soft log space at T = 1.
* ``hirschberg_tracked.npz`` -- tracked affine Hirschberg (three parameter sets, with and without
  gap tracks), Global, Local and glocal, both carries, float32 and float64.
* ``hirschberg_glocal.npz`` -- the batch engine with glocal ends and traceback "hirschberg" /
  "hirschberg_pmax" (affine and linear, small hb_cutoff): A within a longer B, float32 and
  float64.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("NWGRAD_REFERENCE", "/root/reference")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(REF, "tests", "Python"))

import oracle  # noqa: E402
from nwgrad_b200.params import AlignParams  # noqa: E402

DNA = "ACGT"


def brute_fixtures():
    import bruteforce as bf   # the reference's own enumerator
    rng = np.random.default_rng(2024)
    rows = []
    for case in range(40):
        la, lb = int(rng.integers(1, 6)), int(rng.integers(1, 6))
        a = "".join(rng.choice(list(DNA), size=la))
        b = "".join(rng.choice(list(DNA), size=lb))
        mat = rng.integers(-3, 6, size=(4, 4)).astype(np.float64)
        gaps = rng.uniform(0.5, 3.0, size=4).round(2)
        p = AlignParams(mat, *gaps, alphabet=DNA)
        for affine in (True, False):
            gs = bf.global_score(a, b, p, affine)
            ls = bf.local_score(a, b, p, affine)
            lz = bf.global_log_z(a, b, p, affine)
            pairs, oa, ea, ob, eb = bf.global_soft_counts(a, b, p, affine)
            soft = np.zeros(16 + 4)
            for (x, y), v in pairs.items():
                soft[DNA.index(x) * 4 + DNA.index(y)] += v
            soft[16:] = [-oa, -ea, -ob, -eb]   # counts -> gradient sign convention
            # hard counts only where the optimum is unique
            scored = list(bf._scored_paths(a, b, p, affine))
            best = max(s for _, s in scored)
            unique = sum(1 for _, s in scored if s == best) == 1
            hard = np.full(20, np.nan)
            if unique:
                hp, hoa, hea, hob, heb = bf.global_hard_counts(a, b, p, affine)
                hard[:] = 0
                for (x, y), v in hp.items():
                    hard[DNA.index(x) * 4 + DNA.index(y)] += v
                hard[16:] = [-hoa, -hea, -hob, -heb]
            rows.append(dict(a=a, b=b, mat=mat, gaps=gaps, affine=affine, global_score=gs, local_score=ls,
                             log_z=lz, soft=soft, hard=hard))
    np.savez_compressed(os.path.join(HERE, "bruteforce.npz"),
                        a=np.array([r["a"] for r in rows]), b=np.array([r["b"] for r in rows]),
                        mat=np.stack([r["mat"] for r in rows]), gaps=np.stack([r["gaps"] for r in rows]),
                        affine=np.array([r["affine"] for r in rows]),
                        global_score=np.array([r["global_score"] for r in rows]),
                        local_score=np.array([r["local_score"] for r in rows]),
                        log_z=np.array([r["log_z"] for r in rows]),
                        soft=np.stack([r["soft"] for r in rows]), hard=np.stack([r["hard"] for r in rows]))
    print("bruteforce.npz:", len(rows), "cases")


def ref_fixtures():
    rng = np.random.default_rng(99)
    AA = "ACDEFGHIKLMNPQRSTVWY"
    out = {}
    cases = []
    for name, alpha, K, n, lo, hi, integer in (("prot", AA, 1, 24, 0, 60, True),
                                                ("protf", AA, 1, 16, 1, 50, False),
                                                ("rna3", "ACGTU", 3, 24, 1, 40, False)):
        N = len(alpha)
        if integer:
            mat = rng.integers(-4, 4, size=(K, N, N)).astype(np.float64)
            for k in range(K):
                mat[k][np.diag_indices(N)] = rng.integers(4, 12, size=N)
            gaps = np.tile([11.0, 1.0, 11.0, 1.0], (K, 1))
        else:
            mat = rng.normal(0, 2, size=(K, N, N)).round(3)
            gaps = rng.uniform(0.3, 4.0, size=(K, 4)).round(3)
        sa = ["".join(rng.choice(list(alpha), size=int(rng.integers(lo, hi + 1)))) for _ in range(n)]
        sb = ["".join(rng.choice(list(alpha), size=int(rng.integers(lo, hi + 1)))) for _ in range(n)]
        tr = gt = None
        if K > 1:
            tr = np.concatenate([rng.integers(0, K, size=len(s)) for s in sa]).astype(np.uint16)
            gt = np.concatenate([rng.integers(0, K, size=len(s) + 1) for s in sa]).astype(np.uint16)
        mat2 = (mat + rng.normal(0, 0.3, size=mat.shape)).round(3)
        gaps2 = (gaps + rng.uniform(0, 0.2, size=gaps.shape)).round(3)
        cases.append((name, alpha, mat, gaps, sa, sb, tr, gt, mat2, gaps2))
    for name, alpha, mat, gaps, sa, sb, tr, gt, mat2, gaps2 in cases:
        pre = f"{name}_"
        out[pre + "alpha"] = np.array(alpha)
        out[pre + "mat"] = mat
        out[pre + "gaps"] = gaps
        out[pre + "mat2"] = mat2
        out[pre + "gaps2"] = gaps2
        out[pre + "sa"] = np.array(sa)
        out[pre + "sb"] = np.array(sb)
        if tr is not None:
            out[pre + "tracks"] = tr
            out[pre + "gap_tracks"] = gt
        for gm in (0, 1):
            for am in (0, 1):
                for prec in (32, 64):
                    r = oracle.ref_run(prec, gm, am, 1, alpha, mat, gaps, sa, sb, tracks=tr, gap_tracks=gt)
                    key = f"{pre}hard{prec}_g{gm}_m{am}_"
                    out[key + "scores"] = r["scores"]
                    out[key + "grads"] = r["grads"]
                    out[key + "guides"] = r["guides"]
                    rb = oracle.ref_run(prec, gm, am, 1, alpha, mat, gaps, sa, sb, tracks=tr, gap_tracks=gt,
                                        band=4, mat2=mat2, gaps2=gaps2)
                    key = f"{pre}band{prec}_g{gm}_m{am}_"
                    out[key + "scores"] = rb["scores"]
                    out[key + "grads"] = rb["grads"]
                    out[key + "guides"] = rb["guides"]
                for T in (1.0, 0.5):
                    r = oracle.ref_run(64, gm, am, 2, alpha, mat, gaps, sa, sb, tracks=tr, gap_tracks=gt,
                                       soft_impl=2, temperature=T)
                    key = f"{pre}soft_T{T}_g{gm}_m{am}_"
                    out[key + "scores"] = r["scores"]
                    out[key + "grads"] = r["grads"]
    np.savez_compressed(os.path.join(HERE, "reference_batches.npz"), **out)
    print("reference_batches.npz:", len(out), "arrays")


def sg_fixtures():
    """Semi-global ends (mode "glocal" = b_begin + b_end, "overlap" = all four, and other
    free_ends sets): hard at float32 / float64 with guides, soft (log space) at T = 1."""
    rng = np.random.default_rng(77)
    AA = "ACDEFGHIKLMNPQRSTVWY"
    out = {}
    cases = []
    for name, alpha, K, n, lo, hi, integer in (("prot", AA, 1, 24, 0, 60, True),
                                                ("protf", AA, 1, 16, 1, 50, False),
                                                ("rna3", "ACGTU", 3, 24, 1, 40, False)):
        N = len(alpha)
        if integer:
            mat = rng.integers(-4, 4, size=(K, N, N)).astype(np.float64)
            for k in range(K):
                mat[k][np.diag_indices(N)] = rng.integers(4, 12, size=N)
            gaps = np.tile([11.0, 1.0, 11.0, 1.0], (K, 1))
        else:
            mat = rng.normal(0, 2, size=(K, N, N)).round(3)
            gaps = rng.uniform(0.3, 4.0, size=(K, 4)).round(3)
        sa = ["".join(rng.choice(list(alpha), size=int(rng.integers(lo, hi + 1)))) for _ in range(n)]
        sb = ["".join(rng.choice(list(alpha), size=int(rng.integers(lo, hi + 1)))) for _ in range(n)]
        tr = gt = None
        if K > 1:
            tr = np.concatenate([rng.integers(0, K, size=len(s)) for s in sa]).astype(np.uint16)
            gt = np.concatenate([rng.integers(0, K, size=len(s) + 1) for s in sa]).astype(np.uint16)
        mat2 = (mat + rng.normal(0, 0.3, size=mat.shape)).round(3)
        gaps2 = (gaps + rng.uniform(0, 0.2, size=gaps.shape)).round(3)
        cases.append((name, alpha, mat, gaps, sa, sb, tr, gt, mat2, gaps2))
    for name, alpha, mat, gaps, sa, sb, tr, gt, mat2, gaps2 in cases:
        pre = f"{name}_"
        out[pre + "mat2"] = mat2
        out[pre + "gaps2"] = gaps2
        out[pre + "alpha"] = np.array(alpha)
        out[pre + "mat"] = mat
        out[pre + "gaps"] = gaps
        out[pre + "sa"] = np.array(sa)
        out[pre + "sb"] = np.array(sb)
        if tr is not None:
            out[pre + "tracks"] = tr
            out[pre + "gap_tracks"] = gt
        for fe in SG_SETS:
            for gm in (0, 1):
                for prec in (32, 64):
                    r = oracle.ref_run(prec, gm, 2, 1, alpha, mat, gaps, sa, sb, tracks=tr, gap_tracks=gt,
                                       free_ends=fe)
                    key = f"{pre}hard{prec}_g{gm}_e{fe}_"
                    out[key + "scores"] = r["scores"]
                    out[key + "grads"] = r["grads"]
                    out[key + "guides"] = r["guides"]
                r = oracle.ref_run(64, gm, 2, 2, alpha, mat, gaps, sa, sb, tracks=tr, gap_tracks=gt,
                                   soft_impl=2, temperature=1.0, free_ends=fe)
                key = f"{pre}soft_g{gm}_e{fe}_"
                out[key + "scores"] = r["scores"]
                out[key + "grads"] = r["grads"]
                if fe == 12 and tr is None:
                    # banded re-alignment (glocal only; the reference refuses other ends banded),
                    # around the guides of the params scored, after a parameter step
                    for prec in (32, 64):
                        rb = oracle.ref_run(prec, gm, 2, 1, alpha, mat, gaps, sa, sb, band=4, mat2=mat2,
                                            gaps2=gaps2, free_ends=fe)
                        key = f"{pre}band{prec}_g{gm}_e{fe}_"
                        out[key + "scores"] = rb["scores"]
                        out[key + "grads"] = rb["grads"]
                        out[key + "guides"] = rb["guides"]
                    rb = oracle.ref_run(64, gm, 2, 2, alpha, mat, gaps, sa, sb, soft_impl=2, temperature=1.0,
                                        band=4, mat2=mat2, gaps2=gaps2, free_ends=fe)
                    key = f"{pre}softband_g{gm}_e{fe}_"
                    out[key + "scores"] = rb["scores"]
                    out[key + "grads"] = rb["grads"]
    np.savez_compressed(os.path.join(HERE, "semiglobal.npz"), **out)
    print("semiglobal.npz:", len(out), "arrays")


# free_ends bit sets of the semi-global fixtures: glocal, overlap, and mixed ones
# (1 a_begin, 2 a_end, 4 b_begin, 8 b_end)
SG_SETS = (12, 15, 9, 6, 3, 0)


def hb_fixtures():
    rng = np.random.default_rng(123)
    AA = "ACDEFGHIKLMNPQRSTVWY"
    out = {}
    for name, integer in (("int", True), ("flt", False)):
        mat = rng.integers(-4, 4, size=(1, 20, 20)).astype(np.float64) if integer else \
            rng.normal(0, 2, size=(1, 20, 20)).round(3)
        if integer:
            mat[0][np.diag_indices(20)] = rng.integers(4, 12, size=20)
        gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if integer else rng.uniform(0.3, 4.0, size=(1, 4)).round(3)
        sa = ["".join(rng.choice(list(AA), size=int(rng.integers(1, 400)))) for _ in range(16)]
        sb = []
        for k, s in enumerate(sa):
            if k % 2:
                t = [c if rng.random() > 0.25 else str(rng.choice(list(AA))) for c in s]
                sb.append("".join(t))
            else:
                sb.append("".join(rng.choice(list(AA), size=int(rng.integers(1, 400)))))
        out[f"{name}_mat"], out[f"{name}_gaps"] = mat, gaps
        out[f"{name}_sa"], out[f"{name}_sb"] = np.array(sa), np.array(sb)
        for prec in (32, 64):
            for tb in ("hirschberg", "hirschberg_pmax"):
                for cut in (8, 64):
                    for gm, am, tag in ((1, 0, ""), (1, 1, "L_"), (0, 0, "lin_"), (0, 1, "linL_")):
                        r = oracle.ref_run(prec, gm, am, 1, AA, mat, gaps, sa, sb, traceback=tb, hb_cutoff=cut)
                        key = f"{name}_{tag}{tb}_{prec}_c{cut}_"
                        out[key + "scores"] = r["scores"]
                        out[key + "grads"] = r["grads"]
                        out[key + "guides"] = r["guides"]
    # tracked linear: three parameter sets picked per residue of A, gap sets per DP row
    K = 3
    mat = rng.integers(-4, 4, size=(K, 20, 20)).astype(np.float64)
    for k in range(K):
        mat[k][np.diag_indices(20)] = rng.integers(4, 12, size=20)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0], [9.0, 2.0, 10.0, 1.5], [12.0, 0.5, 8.0, 2.0]])
    sa = ["".join(rng.choice(list(AA), size=int(rng.integers(1, 400)))) for _ in range(16)]
    sb = ["".join(c if rng.random() > 0.25 else str(rng.choice(list(AA))) for c in s) if k % 2 else
          "".join(rng.choice(list(AA), size=int(rng.integers(1, 400)))) for k, s in enumerate(sa)]
    tr = np.concatenate([rng.integers(0, K, size=len(s)) for s in sa]).astype(np.uint16)
    gt = np.concatenate([rng.integers(0, K, size=len(s) + 1) for s in sa]).astype(np.uint16)
    out["trk_mat"], out["trk_gaps"], out["trk_sa"], out["trk_sb"] = mat, gaps, np.array(sa), np.array(sb)
    out["trk_tracks"], out["trk_gap_tracks"] = tr, gt
    for prec in (32, 64):
        for cut in (8, 64):
            for am, tag in ((0, "linT_"), (1, "linLT_")):
                r = oracle.ref_run(prec, 0, am, 1, AA, mat, gaps, sa, sb, tracks=tr, gap_tracks=gt,
                                   traceback="hirschberg", hb_cutoff=cut)
                key = f"trk_{tag}hirschberg_{prec}_c{cut}_"
                out[key + "scores"] = r["scores"]
                out[key + "grads"] = r["grads"]
                out[key + "guides"] = r["guides"]
    np.savez_compressed(os.path.join(HERE, "hirschberg.npz"), **out)
    print("hirschberg.npz:", len(out), "arrays")


def soft_banded_fixtures():
    rng = np.random.default_rng(321)
    AA = "ACDEFGHIKLMNPQRSTVWY"
    out = {}
    mat = rng.normal(0, 2, size=(1, 20, 20)).round(3)
    gaps = rng.uniform(0.3, 3.0, size=(1, 4)).round(3)
    mat2 = (mat + rng.normal(0, 0.3, size=mat.shape)).round(3)
    gaps2 = (gaps + rng.uniform(0, 0.2, size=gaps.shape)).round(3)
    sa = ["".join(rng.choice(list(AA), size=int(rng.integers(1, 90)))) for _ in range(14)]
    sb = []
    for s in sa:
        t = [c if rng.random() > 0.25 else str(rng.choice(list(AA))) for c in s]
        sb.append("".join(t) if rng.random() > 0.2 else "".join(rng.choice(list(AA), size=int(rng.integers(1, 90)))))
    out.update(mat=mat, gaps=gaps, mat2=mat2, gaps2=gaps2, sa=np.array(sa), sb=np.array(sb))
    for gm in (0, 1):
        for am in (0, 1):
            for bw in (1, 3, 8):
                r = oracle.ref_run(64, gm, am, 2, AA, mat, gaps, sa, sb, soft_impl=2, band=bw, mat2=mat2, gaps2=gaps2)
                out[f"g{gm}_m{am}_b{bw}_scores"] = r["scores"]
                out[f"g{gm}_m{am}_b{bw}_grads"] = r["grads"]
    np.savez_compressed(os.path.join(HERE, "soft_banded.npz"), **out)
    print("soft_banded.npz:", len(out), "arrays")


def posterior_fixtures():
    """soft_guide="posterior": the reference engine's guides after a double soft pass, every gap
    model and end mode (global, local, glocal, overlap), DNA and protein, T 1 and 0.5."""
    rng = np.random.default_rng(654)
    out = {}
    for alpha in ("ACGT", "ACDEFGHIKLMNPQRSTVWY"):
        N = len(alpha)
        mat = rng.normal(0, 1.5, size=(1, N, N)).round(3)
        gaps = rng.uniform(0.5, 3.0, size=(1, 4)).round(3)
        sa = ["".join(rng.choice(list(alpha), size=int(rng.integers(1, 110)))) for _ in range(24)]
        sb = []
        for s in sa:
            t = [c if rng.random() > 0.25 else str(rng.choice(list(alpha))) for c in s]
            sb.append("".join(t) if rng.random() > 0.2 else "".join(rng.choice(list(alpha), size=int(rng.integers(1, 110)))))
        key = f"N{N}_"
        out.update({key + "mat": mat, key + "gaps": gaps, key + "sa": np.array(sa), key + "sb": np.array(sb),
                    key + "alpha": np.array(alpha)})
        for gm in (0, 1):
            for am, fe in ((0, 12), (1, 12), (2, 12), (2, 15)):
                for T in (1.0, 0.5):
                    r = oracle.ref_run(64, gm, am, 2, alpha, mat, gaps, sa, sb, soft_guide=2, free_ends=fe,
                                       temperature=T)
                    out[f"{key}g{gm}_m{am}_e{fe}_T{T}_guides"] = r["guides"]
                    out[f"{key}g{gm}_m{am}_e{fe}_T{T}_scores"] = r["scores"]
    np.savez_compressed(os.path.join(HERE, "posterior.npz"), **out)
    print("posterior.npz:", len(out), "arrays")


def hb_tracked_fixtures():
    """Tracked affine Hirschberg (hb_reverse_rows_, aligner.hpp:1848-1871): three parameter
    sets picked per residue of A and gap sets per DP row, Global, Local and glocal, both carries."""
    rng = np.random.default_rng(456)
    AA = "ACDEFGHIKLMNPQRSTVWY"
    K = 3
    out = {}
    mat = rng.integers(-4, 4, size=(K, 20, 20)).astype(np.float64)
    for k in range(K):
        mat[k][np.diag_indices(20)] = rng.integers(4, 12, size=20)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0], [9.0, 2.0, 10.0, 1.5], [12.0, 0.5, 8.0, 2.0]])
    sa = ["".join(rng.choice(list(AA), size=int(rng.integers(1, 400)))) for _ in range(16)]
    sb = ["".join(c if rng.random() > 0.25 else str(rng.choice(list(AA))) for c in s) if k % 2 else
          "".join(rng.choice(list(AA), size=int(rng.integers(1, 400)))) for k, s in enumerate(sa)]
    tr = np.concatenate([rng.integers(0, K, size=len(s)) for s in sa]).astype(np.uint16)
    gt = np.concatenate([rng.integers(0, K, size=len(s) + 1) for s in sa]).astype(np.uint16)
    out["mat"], out["gaps"], out["sa"], out["sb"] = mat, gaps, np.array(sa), np.array(sb)
    out["tracks"], out["gap_tracks"] = tr, gt
    for prec in (32, 64):
        for tb in ("hirschberg", "hirschberg_pmax"):
            for cut in (8, 64):
                for am, tag in ((0, "G_"), (1, "L_"), (2, "g_")):
                    for use_gt in (False, True):
                        r = oracle.ref_run(prec, 1, am, 1, AA, mat, gaps, sa, sb, tracks=tr,
                                           gap_tracks=gt if use_gt else None, traceback=tb, hb_cutoff=cut,
                                           free_ends=12)
                        key = f"{tag}{'gt_' if use_gt else ''}{tb}_{prec}_c{cut}_"
                        out[key + "scores"] = r["scores"]
                        out[key + "grads"] = r["grads"]
                        out[key + "guides"] = r["guides"]
    np.savez_compressed(os.path.join(HERE, "hirschberg_tracked.npz"), **out)
    print("hirschberg_tracked.npz:", len(out), "arrays")


def hb_glocal_fixtures():
    """Glocal Hirschberg (viterbi_affine_hirschberg_glocal): A (a mutated stretch of B, or
    random) within B with random flanks, so the end and start scans pick columns inside B."""
    rng = np.random.default_rng(321)
    AA = "ACDEFGHIKLMNPQRSTVWY"
    out = {}
    for name, integer in (("int", True), ("flt", False)):
        mat = rng.integers(-4, 4, size=(1, 20, 20)).astype(np.float64) if integer else \
            rng.normal(0, 2, size=(1, 20, 20)).round(3)
        if integer:
            mat[0][np.diag_indices(20)] = rng.integers(4, 12, size=20)
        gaps = np.array([[11.0, 1.0, 11.0, 1.0]]) if integer else rng.uniform(0.3, 4.0, size=(1, 4)).round(3)
        sa, sb = [], []
        for k in range(16):
            core = "".join(rng.choice(list(AA), size=int(rng.integers(1, 300))))
            a = "".join(c if rng.random() > 0.25 else str(rng.choice(list(AA))) for c in core) if k % 3 else core
            if k % 4 == 0:
                a = "".join(rng.choice(list(AA), size=int(rng.integers(1, 300))))
            left = "".join(rng.choice(list(AA), size=int(rng.integers(0, 120))))
            right = "".join(rng.choice(list(AA), size=int(rng.integers(0, 120))))
            sa.append(a)
            sb.append(left + core + right if k % 5 else "")   # every fifth pair: no B
        out[f"{name}_mat"], out[f"{name}_gaps"] = mat, gaps
        out[f"{name}_sa"], out[f"{name}_sb"] = np.array(sa), np.array(sb)
        for prec in (32, 64):
            for tb in ("hirschberg", "hirschberg_pmax"):
                for cut in (8, 64):
                    for gm, tag in ((1, ""), (0, "lin_")):
                        r = oracle.ref_run(prec, gm, 2, 1, AA, mat, gaps, sa, sb, traceback=tb, hb_cutoff=cut,
                                           free_ends=12)
                        key = f"{name}_{tag}{tb}_{prec}_c{cut}_"
                        out[key + "scores"] = r["scores"]
                        out[key + "grads"] = r["grads"]
                        out[key + "guides"] = r["guides"]
    np.savez_compressed(os.path.join(HERE, "hirschberg_glocal.npz"), **out)
    print("hirschberg_glocal.npz:", len(out), "arrays")


if __name__ == "__main__":
    which = sys.argv[1:] or ["brute", "ref", "hb", "sb", "sg", "post", "hbg", "hbt"]
    if "hbg" in which:
        hb_glocal_fixtures()
    if "hbt" in which:
        hb_tracked_fixtures()
    if "post" in which:
        posterior_fixtures()
    if "brute" in which:
        brute_fixtures()
    if "ref" in which:
        ref_fixtures()
    if "hb" in which:
        hb_fixtures()
    if "sb" in which:
        soft_banded_fixtures()
    if "sg" in which:
        sg_fixtures()
