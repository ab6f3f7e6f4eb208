"""Alphabet, SubstMatrix and AlignParams: the parameter types of the alignment path.

Host-side types with the reference's semantics (michalsta/nwgrad: alphabet.hpp,
subst_matrix.hpp, align_params.hpp; Python surface py_exports.cpp:1364-1537):

* alphabets are interned, so two matrices are compatible exactly when their alphabets are
  the same object;
* an AlignParams holds K >= 1 parameter sets (a stacked K x N x N matrix and K x 4 gap
  fields: open_a, extend_a, open_b, extend_b); set 0 is what the plain fields read;
* arithmetic (+, -, *) is element-wise over every field and needs the same alphabet and K;
  a gradient has the same type, so ``params + lr * grad`` is an update step.
"""
from __future__ import annotations

import threading

import numpy as np

AA20 = "ACDEFGHIKLMNPQRSTVWY"


class Alphabet:
    """Interned symbol <-> index map (alphabet.hpp)."""

    _interned: dict = {}
    _lock = threading.Lock()

    def __init__(self, symbols: str, _token=None):
        if _token is not Alphabet._lock:
            raise TypeError("use Alphabet.get(symbols)")
        self._symbols = symbols
        self._lut = np.full(256, 255, dtype=np.uint8)
        for i, c in enumerate(symbols.encode("latin-1")):
            self._lut[c] = i

    @staticmethod
    def get(symbols: str) -> "Alphabet":
        if not isinstance(symbols, str) or not symbols:
            raise ValueError("nwgrad: an alphabet needs at least one symbol")
        if len(set(symbols)) != len(symbols):
            raise ValueError(f"nwgrad: alphabet \"{symbols}\" has a repeated symbol")
        if len(symbols) > 255 or any(ord(c) > 255 for c in symbols):
            raise ValueError("nwgrad: alphabet symbols must be single-byte characters, at most 255")
        with Alphabet._lock:
            a = Alphabet._interned.get(symbols)
            if a is None:
                a = Alphabet(symbols, Alphabet._lock)
                Alphabet._interned[symbols] = a
            return a

    @property
    def symbols(self) -> str:
        return self._symbols

    @property
    def size(self) -> int:
        return len(self._symbols)

    def __len__(self):
        return len(self._symbols)

    def index_of(self, c: str) -> int:
        return self._symbols.find(c) if len(c) == 1 else -1

    def contains(self, c: str) -> bool:
        return self.index_of(c) >= 0

    def encode(self, s: str) -> np.ndarray:
        b = np.frombuffer(s.encode("latin-1"), dtype=np.uint8)
        codes = self._lut[b]
        bad = np.nonzero(codes == 255)[0]
        if bad.size:
            k = int(bad[0])
            raise ValueError(f"nwgrad: character '{s[k]}' is not in alphabet \"{self._symbols}\"")
        return codes

    def decode(self, indices) -> str:
        return "".join(self._symbols[int(i)] for i in indices)

    def __repr__(self):
        return f"Alphabet(\"{self._symbols}\")"


DNA = Alphabet.get("ACGT")
DNA_N = Alphabet.get("ACGTN")
RNA = Alphabet.get("ACGU")
RNA_N = Alphabet.get("ACGUN")
PROTEIN = Alphabet.get(AA20)
PROTEIN_X = Alphabet.get(AA20 + "X")
PROTEIN_UO = Alphabet.get(AA20 + "UO")
PROTEIN_UOX = Alphabet.get(AA20 + "UOX")
NCBI_PROTEIN = Alphabet.get("ARNDCQEGHILKMFPSTWYVBZX")
IUPAC_DNA = Alphabet.get("ATGCSWRYKMBVHDN")

K_MAX_SETS = 65536   # subst_matrix.hpp:177


def _alpha(a) -> Alphabet:
    if isinstance(a, Alphabet):
        return a
    return Alphabet.get(a)


class SubstMatrix:
    """A stack of K N x N substitution matrices over one alphabet (subst_matrix.hpp:35-183)."""

    def __init__(self, matrix, alphabet=AA20):
        self._alpha = _alpha(alphabet)
        m = np.array(matrix, dtype=np.float64)
        N = self._alpha.size
        if m.ndim == 2:
            m = m[None]
        if m.ndim != 3 or m.shape[1:] != (N, N):
            raise ValueError(f"nwgrad: matrix shape {np.shape(matrix)} does not match alphabet size {N}")
        if not 1 <= m.shape[0] <= K_MAX_SETS:
            raise ValueError("nwgrad: number of parameter sets out of range")
        self._m = np.ascontiguousarray(m)

    @classmethod
    def _wrap(cls, stack: np.ndarray, alpha: Alphabet) -> "SubstMatrix":
        o = cls.__new__(cls)
        o._alpha = alpha
        o._m = np.ascontiguousarray(stack, dtype=np.float64)
        return o

    @property
    def alphabet(self) -> str:
        return self._alpha.symbols

    @property
    def alphabet_obj(self) -> Alphabet:
        return self._alpha

    @property
    def size(self) -> int:
        return self._alpha.size

    @property
    def sets(self) -> int:
        return self._m.shape[0]

    def score(self, a: str, b: str) -> float:
        ia, ib = self._alpha.index_of(a), self._alpha.index_of(b)
        for c, i in ((a, ia), (b, ib)):
            if i < 0:
                raise ValueError(f"nwgrad: character '{c}' is not in alphabet \"{self.alphabet}\"")
        return float(self._m[0, ia, ib])

    def to_matrix(self) -> np.ndarray:
        return self._m[0].copy()

    def __repr__(self):
        return f"SubstMatrix(alphabet=\"{self.alphabet}\", sets={self.sets})"


class AlignParams:
    """K parameter sets: substitution matrices plus four gap costs each (align_params.hpp:45-203).

    ``AlignParams(matrix, gap_open_a=0, gap_extend_a=0, gap_open_b=0, gap_extend_b=0)`` with a
    SubstMatrix, or ``AlignParams(array, alphabet=..., ...)`` with a raw (N, N) array.
    """

    GAP_FIELDS = ("gap_open_a", "gap_extend_a", "gap_open_b", "gap_extend_b")

    def __init__(self, matrix, gap_open_a=0.0, gap_extend_a=0.0, gap_open_b=0.0, gap_extend_b=0.0,
                 *, alphabet=None):
        if isinstance(matrix, SubstMatrix):
            if alphabet is not None and _alpha(alphabet) is not matrix.alphabet_obj:
                raise ValueError("nwgrad: alphabet does not match the SubstMatrix's")
            sm = matrix
        else:
            sm = SubstMatrix(matrix, alphabet if alphabet is not None else AA20)
        self._alpha = sm.alphabet_obj
        self._m = sm._m.copy()
        K = self._m.shape[0]
        self._g = np.zeros((K, 4), dtype=np.float64)
        self._g[0] = [gap_open_a, gap_extend_a, gap_open_b, gap_extend_b]

    # ── constructors ──────────────────────────────────────────────────────────
    @classmethod
    def _make(cls, mats: np.ndarray, gaps: np.ndarray, alpha: Alphabet) -> "AlignParams":
        o = cls.__new__(cls)
        o._alpha = alpha
        o._m = np.ascontiguousarray(mats, dtype=np.float64)
        o._g = np.ascontiguousarray(gaps, dtype=np.float64).reshape(-1, 4)
        return o

    @classmethod
    def from_arrays(cls, matrices, gaps, alphabet=AA20) -> "AlignParams":
        al = _alpha(alphabet)
        m = np.array(matrices, dtype=np.float64)
        if m.ndim == 2:
            m = m[None]
        g = np.array(gaps, dtype=np.float64).reshape(-1, 4)
        N = al.size
        if m.ndim != 3 or m.shape[1:] != (N, N) or g.shape[0] != m.shape[0]:
            raise ValueError("nwgrad: from_arrays needs matrices (K, N, N) and gaps (K, 4) over the alphabet")
        if not 1 <= m.shape[0] <= K_MAX_SETS:
            raise ValueError("nwgrad: number of parameter sets out of range")
        return cls._make(m.copy(), g.copy(), al)

    @classmethod
    def stack(cls, parts) -> "AlignParams":
        parts = list(parts)
        if not parts:
            raise ValueError("nwgrad: AlignParams.stack() needs at least one set")
        al = parts[0]._alpha
        for p in parts[1:]:
            if p._alpha is not al:
                raise ValueError("nwgrad: AlignParams.stack() needs one alphabet")
        m = np.concatenate([p._m for p in parts])
        if m.shape[0] > K_MAX_SETS:
            raise ValueError("nwgrad: number of parameter sets out of range")
        return cls._make(m, np.concatenate([p._g for p in parts]), al)

    @classmethod
    def zeros_like(cls, p: "AlignParams") -> "AlignParams":
        return cls._make(np.zeros_like(p._m), np.zeros_like(p._g), p._alpha)

    # ── fields ────────────────────────────────────────────────────────────────
    @property
    def alphabet(self) -> str:
        return self._alpha.symbols

    @property
    def alphabet_obj(self) -> Alphabet:
        return self._alpha

    @property
    def num_sets(self) -> int:
        return self._m.shape[0]

    @property
    def matrix(self) -> SubstMatrix:
        return SubstMatrix._wrap(self._m[:1].copy(), self._alpha)

    @matrix.setter
    def matrix(self, sm: SubstMatrix):
        if sm.alphabet_obj is not self._alpha:
            raise ValueError("nwgrad: matrix alphabet does not match the params'")
        self._m[0] = sm._m[0]

    @property
    def matrices(self) -> np.ndarray:
        return self._m.copy()

    @matrices.setter
    def matrices(self, v):
        v = np.asarray(v, dtype=np.float64)
        if v.shape != self._m.shape:
            raise ValueError("nwgrad: matrices shape mismatch")
        self._m[...] = v

    @property
    def gaps(self) -> np.ndarray:
        return self._g.copy()

    @gaps.setter
    def gaps(self, v):
        v = np.asarray(v, dtype=np.float64).reshape(self._g.shape)
        self._g[...] = v

    def _gap_get(k):
        return property(lambda self: float(self._g[0, k]),
                        lambda self, v: self._g.__setitem__((0, k), float(v)))

    gap_open_a = _gap_get(0)
    gap_extend_a = _gap_get(1)
    gap_open_b = _gap_get(2)
    gap_extend_b = _gap_get(3)
    del _gap_get

    def __getitem__(self, k: int) -> "AlignParams":
        K = self.num_sets
        if k < 0:
            k += K
        if not 0 <= k < K:
            raise IndexError(f"nwgrad: parameter set {k} out of range (K = {K})")
        return AlignParams._make(self._m[k:k + 1].copy(), self._g[k:k + 1].copy(), self._alpha)

    def __setitem__(self, k: int, p: "AlignParams"):
        K = self.num_sets
        if k < 0:
            k += K
        if not 0 <= k < K:
            raise IndexError(f"nwgrad: parameter set {k} out of range (K = {K})")
        if p.num_sets != 1 or p._alpha is not self._alpha:
            raise ValueError("nwgrad: assign a one-set AlignParams over the same alphabet")
        self._m[k] = p._m[0]
        self._g[k] = p._g[0]

    def to_dict(self) -> dict:
        d = {"matrix": self._m[0].copy(), "alphabet": self.alphabet,
             "gap_open_a": float(self._g[0, 0]), "gap_extend_a": float(self._g[0, 1]),
             "gap_open_b": float(self._g[0, 2]), "gap_extend_b": float(self._g[0, 3])}
        if self.num_sets > 1:
            d.update(num_sets=self.num_sets, matrices=self._m.copy(), gaps=self._g.copy())
        return d

    def copy(self) -> "AlignParams":
        return AlignParams._make(self._m.copy(), self._g.copy(), self._alpha)

    # ── arithmetic ────────────────────────────────────────────────────────────
    def _check(self, o: "AlignParams"):
        if not isinstance(o, AlignParams):
            raise TypeError("nwgrad: AlignParams arithmetic needs another AlignParams")
        if o._alpha is not self._alpha:
            raise ValueError(f"nwgrad: alphabet mismatch (\"{self.alphabet}\" vs \"{o.alphabet}\")")
        if o.num_sets != self.num_sets:
            raise ValueError(f"nwgrad: parameter set count mismatch ({self.num_sets} vs {o.num_sets})")

    def __add__(self, o):
        self._check(o)
        return AlignParams._make(self._m + o._m, self._g + o._g, self._alpha)

    def __sub__(self, o):
        self._check(o)
        return AlignParams._make(self._m + (-1.0 * o._m), self._g + (-1.0 * o._g), self._alpha)

    def __mul__(self, s):
        s = float(s)
        return AlignParams._make(self._m * s, self._g * s, self._alpha)

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1.0

    def __iadd__(self, o):
        self._check(o)
        self._m += o._m
        self._g += o._g
        return self

    def __isub__(self, o):
        self._check(o)
        self._m += -1.0 * o._m
        self._g += -1.0 * o._g
        return self

    def __imul__(self, s):
        s = float(s)
        self._m *= s
        self._g *= s
        return self

    def __repr__(self):
        return (f"AlignParams(alphabet=\"{self.alphabet}\", sets={self.num_sets}, "
                f"gaps={self._g[0].tolist()})")
