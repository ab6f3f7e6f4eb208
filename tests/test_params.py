"""Host-side parameter types: the reference's AlignParams / SubstMatrix / Alphabet
semantics (align_params.hpp, subst_matrix.hpp, alphabet.hpp; docs/api.md)."""
import numpy as np
import pytest

import nwgrad_b200 as nw


def test_alphabet_interned_and_encode():
    assert nw.Alphabet.get("ACGT") is nw.DNA
    assert nw.DNA.index_of("G") == 2 and nw.DNA.index_of("N") == -1
    np.testing.assert_array_equal(nw.DNA.encode("GATTACA"), [2, 0, 3, 3, 0, 1, 0])
    assert nw.DNA.decode([2, 0]) == "GA"
    with pytest.raises(ValueError):
        nw.DNA.encode("ACGN")
    with pytest.raises(ValueError):
        nw.Alphabet.get("AAC")
    assert nw.PROTEIN.symbols == "ACDEFGHIKLMNPQRSTVWY"
    assert nw.PROTEIN_X.symbols[:20] == nw.PROTEIN.symbols


def test_params_arithmetic_and_sets():
    m = np.arange(16.0).reshape(4, 4)
    p = nw.AlignParams(nw.SubstMatrix(m, "ACGT"), 11, 1, 10, 2)
    q = p + 0.5 * p
    assert q.gap_open_a == 16.5 and q.gap_extend_b == 3.0
    np.testing.assert_array_equal(q.matrix.to_matrix(), 1.5 * m)
    r = p - p
    assert not np.any(r.matrices) and not np.any(r.gaps)
    with pytest.raises(ValueError):
        p + nw.AlignParams(np.zeros((20, 20)), 1, 1, 1, 1)
    s = nw.AlignParams.stack([p, q, r])
    assert s.num_sets == 3 and s[1].gap_open_a == 16.5
    with pytest.raises(ValueError):
        s + p                      # K differs
    s[2] = p
    assert s[2].gap_open_b == 10
    f = nw.AlignParams.from_arrays(np.ones((2, 4, 4)), [[1, 2, 3, 4], [5, 6, 7, 8]], alphabet="ACGT")
    assert f.num_sets == 2 and f.gaps[1, 3] == 8
    d = f.to_dict()
    assert d["num_sets"] == 2 and d["alphabet"] == "ACGT"


def test_params_copy_semantics():
    p = nw.AlignParams(np.eye(4), 1, 1, 1, 1, alphabet="ACGT")
    c = p.copy()
    p.gap_open_a = 7
    assert c.gap_open_a == 1
    p *= 2.0
    assert p.gap_open_a == 14 and c.gap_open_a == 1


def test_subst_matrix_score():
    sm = nw.SubstMatrix(np.arange(16.0).reshape(4, 4), "ACGT")
    assert sm.score("C", "G") == 6.0
    with pytest.raises(ValueError):
        sm.score("C", "N")


def test_mode_parsing():
    """Mode names and free_ends onto (align mode, free-end bits), with the reference's rules
    (py_exports.cpp:276-335)."""
    from nwgrad_b200.batch import parse_mode
    assert parse_mode("global") == ("global", 0, 12)
    assert parse_mode("local") == ("local", 1, 12)
    assert parse_mode("glocal") == ("glocal", 2, 12)
    assert parse_mode("overlap") == ("overlap", 2, 15)
    assert parse_mode("semiglobal", (True, False, False, True)) == ("semiglobal", 2, 9)
    assert parse_mode("semiglobal", ("a_end", "b_begin")) == ("semiglobal", 2, 6)
    assert parse_mode("semiglobal", "b_end") == ("semiglobal", 2, 8)
    assert parse_mode("semiglobal", ()) == ("semiglobal", 2, 0)
    with pytest.raises(ValueError, match="needs free_ends"):
        parse_mode("semiglobal")
    with pytest.raises(ValueError, match="goes with mode"):
        parse_mode("glocal", ("a_begin",))
    with pytest.raises(ValueError, match="unknown free end"):
        parse_mode("semiglobal", ("a_start",))
    with pytest.raises(ValueError, match="four booleans"):
        parse_mode("semiglobal", (True, False))
    with pytest.raises(ValueError, match="unknown mode"):
        parse_mode("fitting")


def test_tuner_size_classes():
    """The tuner's size classes: ceil(log2(rows x cols)) in integers (soft rows count row 0),
    the class set it keys the cache by equals the classes of the per-pair split, and every
    pair lands in exactly one class, in pair order."""
    from nwgrad_b200 import tune

    class FakeBatch:
        pass

    rng = np.random.default_rng(3)
    la = rng.integers(0, 700, 5000)
    lb = rng.integers(0, 700, 5000)
    for grad_mode in ("soft", "hard"):
        b = FakeBatch()
        b._oa = np.concatenate([[0], np.cumsum(la)]).astype(np.int64)
        b._ob = np.concatenate([[0], np.cumsum(lb)]).astype(np.int64)
        b._grad_mode = grad_mode
        sc = tune._class_of(b)
        rows = la + 1 if grad_mode == "soft" else la
        want = [tune.size_class(int(r), int(c)) for r, c in zip(rows, lb)]
        np.testing.assert_array_equal(sc, want)
        groups = tune._classes(b, sc)
        assert sorted(groups) == np.flatnonzero(np.bincount(sc)).tolist()
        idx = np.concatenate([groups[k] for k in sorted(groups)])
        assert np.array_equal(np.sort(idx), np.arange(la.size))
        for k, g in groups.items():
            assert np.all(sc[g] == k) and np.all(np.diff(g) > 0)
