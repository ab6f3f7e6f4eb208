"""Shared fixtures: seeded problem generators and the gpu marker."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

AA = "ACDEFGHIKLMNPQRSTVWY"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def rand_matrix(rng, N, K=1, integer=True):
    """Symmetric-ish integer matrix in [-4, 11] with a positive diagonal, or Gaussian."""
    if integer:
        m = rng.integers(-4, 4, size=(K, N, N)).astype(np.float64)
        for k in range(K):
            m[k] = np.triu(m[k]) + np.triu(m[k], 1).T
            m[k][np.diag_indices(N)] = rng.integers(4, 12, size=N)
        return m
    return rng.normal(0.0, 2.0, size=(K, N, N))


def rand_seqs(rng, n, lo, hi, alpha):
    return ["".join(rng.choice(list(alpha), size=int(rng.integers(lo, hi + 1)))) for _ in range(n)]


def mutate(rng, s, alpha, sub=0.3, indel=0.05):
    out = []
    for c in s:
        r = rng.random()
        if r < indel / 2:
            continue
        if r < indel:
            out.append(c)
            out.extend(rng.choice(list(alpha), size=int(rng.geometric(1 / 3))))
            continue
        out.append(rng.choice(list(alpha)) if rng.random() < sub else c)
    return "".join(out)


def encode(alpha, seqs):
    lut = {c: i for i, c in enumerate(alpha)}
    return [[lut[c] for c in s] for s in seqs]


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
