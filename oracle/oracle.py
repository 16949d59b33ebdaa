"""ctypes bindings of the two CPU checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, never by the product.

* :class:`OracleCholesky` -- the project's C++ restatement (``oracle.cpp``).
* :class:`RefCholesky` -- the reference's own ``Sparse::CholeskyDecomposition``
  compiled from its headers (``ref_driver.cpp``, ``_ref/libtb_ref.so``).

Both expose the same small surface: symbolic arrays by name, numeric factor
arrays, solve, log-determinant.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtb_ref.so")

ARRAYS = {
    "perm": 0, "perm_inv": 1, "value_perm": 2, "SN_rp": 3, "SN_outer": 4, "SN_inner": 5,
    "row_to_SN": 6, "SN_tri_ptr": 7, "SN_rec_ptr": 8, "aTree_parents": 9, "eTree_parents": 10,
    "outer": 11, "inner": 12, "aTree_child_ptr": 13, "aTree_child_idx": 14,
}

STRATEGIES = {"maximal": 0, "fundamental": 1, "amalgamated": 2}

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_i64 = ctypes.c_int64


def build(with_reference: bool = True) -> None:
    """Compile the restatement (and the reference, when its checkout exists).

    The checkout's location is the Makefile's REFERENCE_DIR (override it in
    the environment); without a checkout the reference target is skipped."""
    targets = ["oracle"] + (["ref"] if with_reference else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _ptr(a):
    return a.ctypes.data if a is not None else None


def _load_oracle():
    if not os.path.exists(ORACLE_SO):
        build(with_reference=False)
    lib = ctypes.CDLL(ORACLE_SO)
    lib.tb_oracle_analyze.restype = _vp
    lib.tb_oracle_analyze.argtypes = [_i, _vp, _vp, _vp, _i, _i]
    lib.tb_oracle_destroy.argtypes = [_vp]
    lib.tb_oracle_sn_count.argtypes = [_vp]
    lib.tb_oracle_array_size.argtypes = [_vp, _i]
    lib.tb_oracle_array_size.restype = _i64
    lib.tb_oracle_array_copy.argtypes = [_vp, _i, _vp]
    lib.tb_oracle_factor.argtypes = [_vp, _vp, _d]
    for f in ("tb_oracle_tri_size", "tb_oracle_rec_size"):
        getattr(lib, f).argtypes = [_vp]
        getattr(lib, f).restype = _i64
    lib.tb_oracle_tri_copy.argtypes = [_vp, _vp]
    lib.tb_oracle_rec_copy.argtypes = [_vp, _vp]
    lib.tb_oracle_solve.argtypes = [_vp, _d, _vp, _i, _d, _vp, _i, _i]
    lib.tb_oracle_half_solve.argtypes = [_vp, _i, _d, _vp, _i, _d, _vp, _i, _i]
    lib.tb_oracle_log_det.argtypes = [_vp]
    lib.tb_oracle_log_det.restype = _d
    return lib


def _load_ref():
    if not os.path.exists(REF_SO):
        raise FileNotFoundError(f"{REF_SO} not built (needs the reference checkout; run make -C oracle ref)")
    lib = ctypes.CDLL(REF_SO)
    lib.tb_ref_create.restype = _vp
    lib.tb_ref_create.argtypes = [_i, _vp, _vp, _vp, _i]
    lib.tb_ref_destroy.argtypes = [_vp]
    lib.tb_ref_set_strategy.argtypes = [_vp, _i]
    lib.tb_ref_set_amalgamation_threshold.argtypes = [_vp, _i]
    lib.tb_ref_set_method.argtypes = [_vp, _i]
    lib.tb_ref_symbolic.argtypes = [_vp]
    lib.tb_ref_sn_count.argtypes = [_vp]
    lib.tb_ref_array_size.argtypes = [_vp, _i]
    lib.tb_ref_array_size.restype = _i64
    lib.tb_ref_array_copy.argtypes = [_vp, _i, _vp]
    lib.tb_ref_numeric.argtypes = [_vp, _vp, _d]
    lib.tb_ref_good.argtypes = [_vp]
    for f in ("tb_ref_tri_size", "tb_ref_rec_size"):
        getattr(lib, f).argtypes = [_vp]
        getattr(lib, f).restype = _i64
    lib.tb_ref_tri_copy.argtypes = [_vp, _vp]
    lib.tb_ref_rec_copy.argtypes = [_vp, _vp]
    lib.tb_ref_solve.argtypes = [_vp, _d, _vp, _i, _d, _vp, _i, _i, _i]
    lib.tb_ref_lower_solve.argtypes = [_vp, _d, _vp, _i, _d, _vp, _i, _i]
    lib.tb_ref_log_det.argtypes = [_vp]
    lib.tb_ref_log_det.restype = _d
    lib.tb_ref_set_quiet.argtypes = [_i]
    lib.tb_ref_set_blas_threads.argtypes = [_i]
    lib.tb_ref_mm_load.restype = _vp
    lib.tb_ref_mm_load.argtypes = [ctypes.c_char_p, _i]
    lib.tb_ref_mm_sizes.argtypes = [_vp, _vp, _vp, _vp]
    lib.tb_ref_mm_copy.argtypes = [_vp, _vp, _vp, _vp]
    lib.tb_ref_mm_free.argtypes = [_vp]
    lib.tb_ref_set_quiet(1)
    return lib


_ORACLE = None
_REF = None


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _load_oracle()
    return _ORACLE


def ref_lib():
    global _REF
    if _REF is None:
        _REF = _load_ref()
    return _REF


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _csr_args(outer, inner, perm):
    outer = np.ascontiguousarray(outer, dtype=np.int64)
    inner = np.ascontiguousarray(inner, dtype=np.int32)
    perm = None if perm is None else np.ascontiguousarray(perm, dtype=np.int32)
    return outer, inner, perm


class _Base:
    _prefix = ""

    def array(self, name: str) -> np.ndarray:
        w = ARRAYS[name]
        size = self._f("array_size")(self.h, w)
        out = np.zeros(size, dtype=np.int64)
        if size:
            self._f("array_copy")(self.h, w, out.ctypes.data)
        return out

    def sn_count(self) -> int:
        return int(self._f("sn_count")(self.h))

    def _f(self, name):
        return getattr(self.lib, self._prefix + name)

    def factor_values(self):
        tri = np.zeros(self._f("tri_size")(self.h))
        rec = np.zeros(self._f("rec_size")(self.h))
        if len(tri):
            self._f("tri_copy")(self.h, tri.ctypes.data)
        if len(rec):
            self._f("rec_copy")(self.h, rec.ctypes.data)
        return tri, rec

    def log_det(self) -> float:
        return float(self._f("log_det")(self.h))


class OracleCholesky(_Base):
    """The C++ restatement; symbolic analysis runs in the constructor."""

    _prefix = "tb_oracle_"

    def __init__(self, n, outer, inner, perm=None, strategy="maximal", amalgamation_threshold=4):
        self.lib = oracle_lib()
        self._keep = _csr_args(outer, inner, perm)
        o, i, p = self._keep
        self.n = int(n)
        self.h = self.lib.tb_oracle_analyze(self.n, _ptr(o), _ptr(i), _ptr(p),
                                            STRATEGIES[strategy], int(amalgamation_threshold))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.tb_oracle_destroy(self.h)
            self.h = None

    def factor(self, values, reg=0.0) -> int:
        v = np.ascontiguousarray(values, dtype=np.float64)
        return int(self.lib.tb_oracle_factor(self.h, v.ctypes.data, float(reg)))

    def solve(self, B, alpha=1.0, beta=0.0, X=None, which="full"):
        B = np.ascontiguousarray(B, dtype=np.float64)
        k = 1 if B.ndim == 1 else B.shape[1]
        X = np.zeros_like(B) if X is None else X
        if which == "full":
            self.lib.tb_oracle_solve(self.h, alpha, B.ctypes.data, k, beta, X.ctypes.data, k, k)
        else:
            self.lib.tb_oracle_half_solve(self.h, 0 if which == "lower" else 1, alpha,
                                          B.ctypes.data, k, beta, X.ctypes.data, k, k)
        return X


class RefCholesky(_Base):
    """The reference's own implementation (compiled headers)."""

    _prefix = "tb_ref_"

    def __init__(self, n, outer, inner, perm=None, strategy="maximal", threads=1,
                 amalgamation_threshold=4, method="multifrontal", blas_threads=1):
        self.lib = ref_lib()
        self.lib.tb_ref_set_blas_threads(int(blas_threads))
        self._keep = _csr_args(outer, inner, perm)
        o, i, p = self._keep
        self.n = int(n)
        self.h = self.lib.tb_ref_create(self.n, _ptr(o), _ptr(i), _ptr(p), int(threads))
        self.lib.tb_ref_set_strategy(self.h, STRATEGIES[strategy])
        self.lib.tb_ref_set_amalgamation_threshold(self.h, int(amalgamation_threshold))
        self.lib.tb_ref_set_method(self.h, 0 if method == "multifrontal" else 1)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.tb_ref_destroy(self.h)
            self.h = None

    def symbolic(self):
        self.lib.tb_ref_symbolic(self.h)

    def array(self, name):
        self.symbolic()
        return super().array(name)

    def sn_count(self):
        self.symbolic()
        return super().sn_count()

    def factor(self, values, reg=0.0) -> int:
        v = np.ascontiguousarray(values, dtype=np.float64)
        return int(self.lib.tb_ref_numeric(self.h, v.ctypes.data, float(reg)))

    def solve(self, B, alpha=1.0, beta=0.0, X=None, parallel=False):
        B = np.ascontiguousarray(B, dtype=np.float64)
        k = 1 if B.ndim == 1 else B.shape[1]
        X = np.zeros_like(B) if X is None else X
        self.lib.tb_ref_solve(self.h, alpha, B.ctypes.data, k, beta, X.ctypes.data, k, k, int(parallel))
        return X

    def lower_solve(self, B, alpha=1.0, beta=0.0, X=None):
        B = np.ascontiguousarray(B, dtype=np.float64)
        k = 1 if B.ndim == 1 else B.shape[1]
        X = np.zeros_like(B) if X is None else X
        self.lib.tb_ref_lower_solve(self.h, alpha, B.ctypes.data, k, beta, X.ctypes.data, k, k)
        return X


# ---------------------------------------------------------------- MatrixMarket

def ref_mm_read(path, threads: int = 1):
    """The reference's Sparse::MatrixCSR::LoadFromMatrixMarket (MatrixCSR/MatrixMarket.hpp:3-202):
    (rows, cols, outer, inner, values); a file it rejects gives a 0 x 0 matrix."""
    lib = ref_lib()
    h = lib.tb_ref_mm_load(os.fsencode(path), int(threads))
    try:
        rows, cols, nnz = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        lib.tb_ref_mm_sizes(h, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(nnz))
        m = max(rows.value, 0)
        outer = np.zeros(m + 1, dtype=np.int64)
        inner = np.zeros(max(nnz.value, 1), dtype=np.int32)
        values = np.zeros(max(nnz.value, 1), dtype=np.float64)
        lib.tb_ref_mm_copy(h, _ptr(outer), _ptr(inner), _ptr(values))
    finally:
        lib.tb_ref_mm_free(h)
    return rows.value, cols.value, outer, inner[:nnz.value], values[:nnz.value]


def mm_read_port(path):
    """Pure-Python restatement of the same reader for small files: banner and comment
    handling of MatrixMarket.hpp:19-138, triples of :146-174, and FromTriples
    (MatrixCSR/FromTriples.hpp:96-190): off-diagonal entries of a symmetric file
    mirrored, each row's entries in file order, stably sorted by column, repeated
    columns summed in that order.  Returns None for a file the reference rejects."""
    with open(path) as f:
        head = f.readline().split()
        words = [w.lower() for w in head]
        if len(words) < 5 or words[0] != "%%matrixmarket" or words[1] != "matrix" or words[2] != "coordinate":
            return None
        field, symmetry = words[3], words[4]
        if field == "complex" or symmetry not in ("general", "symmetric"):
            return None
        line = f.readline()
        while line and line.startswith("%"):
            line = f.readline()
        m, n, nnz = (int(t) for t in line.split()[:3])
        tokens = f.read().split()
    per = 2 if field == "pattern" else 3
    rows = [[] for _ in range(m)]
    for k in range(nnz):
        i = int(tokens[per * k]) - 1
        j = int(tokens[per * k + 1]) - 1
        a = 1.0 if per == 2 else float(tokens[per * k + 2])
        rows[i].append((j, a))
        if symmetry == "symmetric" and i != j:
            rows[j].append((i, a))
    outer, inner, values = [0], [], []
    for r in rows:
        r = sorted(r, key=lambda e: e[0])          # stable
        for j, a in r:
            if inner and len(inner) > outer[-1] and inner[-1] == j:
                values[-1] += a
            else:
                inner.append(j)
                values.append(a)
        outer.append(len(inner))
    return (m, n, np.asarray(outer, dtype=np.int64), np.asarray(inner, dtype=np.int32),
            np.asarray(values, dtype=np.float64))
