"""The header-only C++ mirror of the reference class compiles against the
C-ABI library and drives it like the reference's CholeskyDecomposition."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from tensors_b200 import _lib
from tensors_b200.cholesky import CholeskyDecomposition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def mirror_exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "mirror_check")
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "mirror_check.cpp"), "-o", out,
           "-L", libdir, "-ltensors_b200", f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def _grid_pattern(g):
    rows, cols = [], []
    for i in range(g):
        for j in range(g):
            r = i * g + j
            for (di, dj) in ((-1, 0), (0, -1), (0, 0), (0, 1), (1, 0)):
                if 0 <= i + di < g and 0 <= j + dj < g:
                    rows.append(r)
                    cols.append((i + di) * g + j + dj)
    outer = np.searchsorted(np.array(rows), np.arange(g * g + 1)).astype(np.int64)
    return outer, np.array(cols, dtype=np.int32)


def test_cpp_mirror_symbolic_matches_python_binding(mirror_exe):
    g = 17
    out = subprocess.run([mirror_exe, str(g)], check=True, capture_output=True, text=True).stdout
    sn = int(out.split()[1])
    outer, inner = _grid_pattern(g)
    perm = np.arange(g * g - 1, -1, -1, dtype=np.int32)
    c = CholeskyDecomposition(outer, inner, perm)
    c.SymbolicFactorization()
    assert sn == c.SN_Count()


@pytest.mark.gpu
def test_cpp_mirror_factor_and_solve(mirror_exe):
    run = subprocess.run([mirror_exe, "24", "numeric"], capture_output=True, text=True)
    assert run.returncode == 0, run.stdout + run.stderr
    out = run.stdout
    vals = dict(line.split() for line in out.strip().splitlines())
    assert int(vals["status"]) == 0
    assert float(vals["relres"]) < 1e-13
    assert int(vals["cg_ok"]) == 1 and 1 <= int(vals["cg_iter"]) <= 200
    assert int(vals["gmres_ok"]) == 1 and 1 <= int(vals["gmres_iter"]) <= 330
    assert float(vals["relres_f32_in"]) < 1e-13                        # float B, double X
    assert int(vals["status_f32"]) == 0
    assert float(vals["relres_f32_factor"]) <= 1e-12                   # Scal = float: refined to the default 1e-12
                                                                       # (for the float values it was given)
    assert int(vals["swap_moved"]) == 1
    assert float(vals["relres_swapped"]) < 1e-13


def test_cpp_mirror_matrix_market(mirror_exe, tmp_path):
    from tensors_b200 import matrices as M
    from tensors_b200.matrix_market import read_matrix_market, write_matrix_market

    A = M.grid_laplacian_2d(13, 0.5)
    src, dst = tmp_path / "a.mtx", tmp_path / "b.mtx"
    write_matrix_market(src, A)
    out = subprocess.run([mirror_exe, "mm", str(src), str(dst)], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[1]) == A.n and int(out[3]) == A.nnz
    c = CholeskyDecomposition(A.outer, A.inner)
    c.SymbolicFactorization()
    assert int(out[5]) == c.SN_Count()
    assert dst.read_text() == src.read_text()
    m, n, outer, inner, values = read_matrix_market(dst)
    assert np.array_equal(outer, A.outer) and np.array_equal(inner, A.inner) and np.array_equal(values, A.values)
