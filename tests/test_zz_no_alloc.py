"""nwg_scores_noalloc: the scores entry point that allocates no device memory, for callers
whose host framework owns every device allocation and forbids cudaMalloc.  Checked through
the C ABI against the store path's scores (nwg_run, score only) and the CPU oracle's Viterbi
scores, bit for bit as every hard result, on two calls in a row (the second reuses the
reserved scratch the first left dirty), and that the second call changes neither the device's
free memory nor torch's allocated bytes.  Collected last on purpose: it must also pass after
every other test in the same process."""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import AA, encode, has_gpu, rand_matrix, rand_seqs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]


def _encode(alpha, seqs):
    lut = {c: i for i, c in enumerate(alpha)}
    lens = np.array([len(s) for s in seqs], np.int64)
    off = np.zeros(len(seqs) + 1, np.int64)
    off[1:] = np.cumsum(lens)
    codes = np.array([lut[c] for s in seqs for c in s], np.uint8)
    return codes, off


def _lib():
    import nwgrad_b200 as nw
    L = nw.load_library()
    L.nwg_scores_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                     C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p]
    L.nwg_scores_noalloc.restype = C.c_int
    L.nwg_noalloc_last_error.restype = C.c_char_p
    return L


@pytest.mark.parametrize("gap_model", ["linear", "affine"])
@pytest.mark.parametrize("mode", ["global", "local"])
def test_noalloc_scores_match_store_path(gap_model, mode):
    import torch
    import nwgrad_b200 as nw
    L = _lib()
    rng = np.random.default_rng(11 if mode == "global" else 12)
    mat = rand_matrix(rng, 20, 1, integer=False)
    gaps = rng.uniform(0.3, 3.0, size=(1, 4))
    # short pairs, multi-stripe pairs (A longer than 128), empties, B up to 600
    sa = rand_seqs(rng, 200, 0, 60, AA) + rand_seqs(rng, 20, 150, 400, AA) + ["", "ACD"]
    sb = rand_seqs(rng, 200, 0, 60, AA) + rand_seqs(rng, 20, 100, 600, AA) + ["KL", ""]
    params = nw.AlignParams.from_arrays(mat, gaps, alphabet=AA)
    b = nw.SeqPairBatch(sa, sb, params, gap_model=gap_model, mode=mode, grad_mode="none")
    b.score_and_grad()
    ref = b.scores()
    o = oracle.hard(32, int(gap_model == "affine"), int(mode == "local"), mat, gaps,
                    oracle.Encoded(encode(AA, sa), encode(AA, sb)))
    assert np.array_equal(ref, o["scores"])
    ca, oa = _encode(AA, sa)
    cb, ob = _encode(AA, sb)
    dev = torch.device("cuda", torch.cuda.current_device())
    t_ca = torch.from_numpy(ca if ca.size else np.zeros(1, np.uint8)).to(dev)
    t_cb = torch.from_numpy(cb if cb.size else np.zeros(1, np.uint8)).to(dev)
    t_oa, t_ob = torch.from_numpy(oa).to(dev), torch.from_numpy(ob).to(dev)
    out = torch.full((len(sa),), -1.0, dtype=torch.float64, device=dev)
    m = np.ascontiguousarray(mat[0], np.float64)
    g = np.ascontiguousarray(gaps[0], np.float64)
    max_b = max(len(s) for s in sb)
    for call in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
        rc = L.nwg_scores_noalloc(t_ca.data_ptr(), t_oa.data_ptr(), t_cb.data_ptr(), t_ob.data_ptr(), len(sa),
                                  max_b, 20, m.ctypes.data_as(C.POINTER(C.c_double)),
                                  g.ctypes.data_as(C.POINTER(C.c_double)), int(gap_model == "affine"),
                                  int(mode == "local"), out.data_ptr(), None)
        assert rc == 0, L.nwg_noalloc_last_error()
        torch.cuda.synchronize()
        if call == 1:   # after the first call's one-time set-up, a call allocates nothing
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == alloc0
        got = out.cpu().numpy()
        assert np.array_equal(got, ref), (call, np.nonzero(got != ref)[0][:5])


def test_noalloc_rejects_b_over_the_limit():
    L = _lib()
    m = np.zeros(16)
    g = np.zeros(4)
    rc = L.nwg_scores_noalloc(None, None, None, None, 0, 5000, 4,
                              m.ctypes.data_as(C.POINTER(C.c_double)), g.ctypes.data_as(C.POINTER(C.c_double)),
                              1, 0, None, None)
    assert rc == 1 and b"2047" in L.nwg_noalloc_last_error()
