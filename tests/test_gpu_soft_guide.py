"""soft_guide: when a soft batch computes the guide that banded_grad() bands around.
"eager" takes the params score_and_grad() ran with, "lazy" those current at first use."""
import numpy as np
import pytest

from conftest import AA, has_gpu, mutate, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

import nwgrad_b200 as nw  # noqa: E402


def _hard_guides(sa, sb, p):
    h = nw.SeqPairBatch(sa, sb, p, grad_mode="hard")
    h.score_and_grad()
    return h.guides()


def test_eager_and_lazy_guides():
    rng = np.random.default_rng(4100)
    mat = rand_matrix(rng, 20, 1, True)
    sa = rand_seqs(rng, 40, 20, 200, AA)
    sb = [mutate(rng, s, AA) for s in sa]
    p = nw.AlignParams.from_arrays(mat, [[11.0, 1.0, 11.0, 1.0]], alphabet=AA)
    q = nw.AlignParams.from_arrays(-mat * 0.5 + 2.0, [[3.0, 2.0, 4.0, 1.0]], alphabet=AA)
    gp, gq = _hard_guides(sa, sb, p), _hard_guides(sa, sb, q)
    assert not np.array_equal(gp, gq)
    out = {}
    for mode in ("eager", "lazy"):
        b = nw.SeqPairBatch(sa, sb, p, grad_mode="soft")
        b.soft_guide = mode
        assert b.soft_guide == mode
        b.score_and_grad()
        b.set_params(q)
        out[mode] = b.guides()
        b.banded_grad(8)                     # bands around that guide
    assert np.array_equal(out["eager"], gp)
    assert np.array_equal(out["lazy"], gq)
    b = nw.SeqPairBatch(sa, sb, p, grad_mode="soft")
    with pytest.raises(NotImplementedError):
        b.soft_guide = "posterior"
    with pytest.raises(ValueError, match="unknown soft_guide"):
        b.soft_guide = "viterbi"
    assert b.soft_guide == "eager"
