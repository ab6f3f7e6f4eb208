"""torch.autograd binding: the backward (the weighted FP64 reduction of the fused soft
forward-backward's per-pair gradients) against central finite differences of the scores,
and against compute_grad / weighted_grad."""
import numpy as np
import pytest

from conftest import AA, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import torch  # noqa: E402

import nwgrad_b200 as nw  # noqa: E402
from nwgrad_b200.autograd import align_scores  # noqa: E402


def _problem(seed, n=16, lo=5, hi=40):
    rng = np.random.default_rng(seed)
    mat = rand_matrix(rng, 20, integer=False)
    gaps = np.array([[3.0, 0.7, 2.5, 0.9]]) + rng.uniform(0, 0.3, size=(1, 4))
    sa = rand_seqs(rng, n, lo, hi, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    w = rng.normal(size=n)
    return rng, mat, gaps, sa, sb, w


def _loss(batch, mat, gaps, w):
    batch.set_params(nw.AlignParams.from_arrays(mat, gaps, alphabet=AA))
    batch.score_and_grad()
    return float(np.dot(w, batch.scores()))


@pytest.mark.parametrize("gm", ["affine", "linear"])
@pytest.mark.parametrize("am", ["global", "local"])
def test_backward_matches_finite_differences(gm, am):
    rng, mat, gaps, sa, sb, w = _problem(11 + (gm == "linear") + 2 * (am == "local"))
    b = nw.SeqPairBatchDouble(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA),
                              gap_model=gm, mode=am, grad_mode="soft")
    M = torch.tensor(mat, dtype=torch.float64, requires_grad=True)
    G = torch.tensor(gaps, dtype=torch.float64, requires_grad=True)
    loss = (align_scores(b, M, G) * torch.tensor(w)).sum()
    loss.backward()
    fd = nw.SeqPairBatchDouble(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA),
                               gap_model=gm, mode=am, grad_mode="soft")
    eps = 1e-5
    coords = [(0, int(i), int(j)) for i, j in rng.integers(0, 20, size=(12, 2))]
    for k, i, j in coords:
        mp, mm = mat.copy(), mat.copy()
        mp[k, i, j] += eps
        mm[k, i, j] -= eps
        num = (_loss(fd, mp, gaps, w) - _loss(fd, mm, gaps, w)) / (2 * eps)
        got = float(M.grad[k, i, j])
        assert abs(got - num) <= 1e-6 * max(1.0, abs(num)), ((k, i, j), got, num)
    for q in range(4):
        if gm == "linear" and q in (0, 2):
            continue                     # linear gaps read the extend costs only
        gp, gmn = gaps.copy(), gaps.copy()
        gp[0, q] += eps
        gmn[0, q] -= eps
        num = (_loss(fd, mat, gp, w) - _loss(fd, mat, gmn, w)) / (2 * eps)
        got = float(G.grad[0, q])
        assert abs(got - num) <= 1e-6 * max(1.0, abs(num)), (q, got, num)


def test_float32_backward_within_tolerance_of_double():
    rng, mat, gaps, sa, sb, w = _problem(21, n=40, lo=20, hi=120)
    grads = []
    for cls in (nw.SeqPairBatch, nw.SeqPairBatchDouble):
        b = cls(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="soft")
        M = torch.tensor(mat, dtype=torch.float64, requires_grad=True)
        G = torch.tensor(gaps, dtype=torch.float64, requires_grad=True)
        (align_scores(b, M, G) * torch.tensor(w)).sum().backward()
        grads.append(np.concatenate([M.grad.numpy().ravel(), G.grad.numpy().ravel()]))
    scale = max(1.0, np.abs(grads[1]).max())
    assert np.abs(grads[0] - grads[1]).max() <= 1e-4 * scale


@pytest.mark.parametrize("grad_mode", ["soft", "hard"])
def test_backward_is_the_weighted_gradient(grad_mode):
    rng, mat, gaps, sa, sb, w = _problem(31, n=50, lo=10, hi=200)
    b = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode=grad_mode)
    M = torch.tensor(mat[0], dtype=torch.float64, requires_grad=True)     # one set, 2-D
    G = torch.tensor(gaps[0], dtype=torch.float64, requires_grad=True)
    s = align_scores(b, M, G)
    assert s.shape == (len(sa),) and s.dtype == torch.float64
    s.sum().backward()
    ref = b.compute_grad()
    assert np.array_equal(M.grad.numpy(), ref.matrices[0]) and np.array_equal(G.grad.numpy(), ref.gaps[0])
    M.grad = None
    G.grad = None
    (align_scores(b, M, G) * torch.tensor(w)).sum().backward()
    ref = b.weighted_grad(w)
    assert np.array_equal(M.grad.numpy(), ref.matrices[0]) and np.array_equal(G.grad.numpy(), ref.gaps[0])


def test_backward_after_another_run_uses_its_own_parameters():
    rng, mat, gaps, sa, sb, w = _problem(41)
    b = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="soft")
    M1 = torch.tensor(mat, dtype=torch.float64, requires_grad=True)
    G1 = torch.tensor(gaps, dtype=torch.float64, requires_grad=True)
    s1 = align_scores(b, M1, G1)
    M2 = torch.tensor(mat + 0.5, dtype=torch.float64, requires_grad=True)
    G2 = torch.tensor(gaps, dtype=torch.float64, requires_grad=True)
    align_scores(b, M2, G2).sum().backward()
    s1.sum().backward()
    ref = nw.SeqPairBatch(sa, sb, nw.AlignParams.from_arrays(mat, gaps, alphabet=AA), grad_mode="soft")
    ref.score_and_grad()
    g = ref.compute_grad()
    assert np.array_equal(M1.grad.numpy(), g.matrices) and np.array_equal(G1.grad.numpy(), g.gaps)


def test_adam_steps_raise_the_margin():
    """A few Adam steps on the matrix and gap costs widen the homolog / decoy score margin."""
    rng = np.random.default_rng(51)
    mat = rand_matrix(rng, 20, integer=False)
    gaps = np.array([[3.0, 1.0, 3.0, 1.0]])
    sa = rand_seqs(rng, 64, 40, 120, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    decoy = ["".join(rng.permutation(list(s))) for s in sb]
    p0 = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    pos = nw.SeqPairBatch(sa, sb, p0, grad_mode="soft")
    neg = nw.SeqPairBatch(sa, decoy, p0, grad_mode="soft")
    M = torch.tensor(mat, dtype=torch.float64, requires_grad=True)
    G = torch.tensor(gaps, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([M, G], lr=1e-2)
    margins = []
    for _ in range(20):
        opt.zero_grad()
        margin = (align_scores(pos, M, G) - align_scores(neg, M, G)).mean()
        (-margin).backward()
        opt.step()
        margins.append(float(margin))
    assert margins[-1] > margins[0]
