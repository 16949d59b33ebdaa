"""Python mirror of ``Sparse::CholeskyDecomposition`` over the C-ABI.

Method names, argument meanings and return conventions follow the reference
class (src/Sparse/CholeskyDecomposition.hpp and its CholeskyDecomposition/
subfiles); every call goes through ``include/tensors_b200.h`` into the CUDA
library.  Differences from the reference are deliberate and listed here:

* errors raise :class:`TBError` instead of printing and continuing (the
  reference ``eprint``s and returns, e.g. Solve.hpp:353-363);
* ``NumericFactorization`` returns 0 / 1 like the reference (Numeric.hpp:99)
  and additionally records the first failing supernode;
* ``LowerSolve`` solves with L = U^T as documented; the reference's public
  LowerSolve runs the upper solve (Solve.hpp:290-307).
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np

from ._lib import lib

__all__ = ["CholeskyDecomposition", "TBError", "SupernodeStrategy", "FactorizationMethod"]


class TBError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class SupernodeStrategy(enum.IntEnum):
    """CholeskyDecomposition.hpp:119-124."""

    Maximal = 0
    Fundamental = 1
    Amalgamated = 2


class FactorizationMethod(enum.IntEnum):
    """CholeskyDecomposition.hpp:126-130."""

    Multifrontal = 0
    LeftLooking = 1


_ARRAYS = {
    "perm": 0, "perm_inv": 1, "value_perm": 2, "SN_rp": 3, "SN_outer": 4, "SN_inner": 5,
    "row_to_SN": 6, "SN_tri_ptr": 7, "SN_rec_ptr": 8, "aTree_parents": 9, "eTree_parents": 10,
    "outer": 11, "inner": 12, "aTree_child_ptr": 13, "aTree_child_idx": 14,
}


def _check(status: int) -> int:
    if status < 0:
        raise TBError(status, lib().tb_last_error().decode("utf-8", errors="replace"))
    return status


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# scalar types at the boundary (tb_dtype)
TB_F64, TB_F32 = 0, 1


def _dtype_code(dt) -> int:
    return TB_F32 if np.dtype(dt) == np.float32 else TB_F64


class NumericalFactorization:
    """A numeric factor held apart from any decomposition (``NumericalFactorization_T``,
    CholeskyDecomposition.hpp:132-201): device storage exchanged with a decomposition's by
    ``CholeskyDecomposition.SwapNumericalFactorization``.  A new one is empty."""

    def __init__(self):
        h = ctypes.c_void_p()
        _check(lib().tb_factor_create(ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().tb_factor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _state(self):
        f, g, b, p = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int32()
        _check(lib().tb_factor_state(self._h, ctypes.byref(f), ctypes.byref(g), ctypes.byref(b), ctypes.byref(p)))
        return bool(f.value), bool(g.value), int(b.value), int(p.value)

    def NumericallyFactorizedQ(self) -> bool:
        return self._state()[0]

    def NumericallyGoodQ(self) -> bool:
        return self._state()[1]

    def AllocatedByteCount(self) -> int:
        return self._state()[2]

    def Precision(self):
        """'fp64' | 'mixed' of the stored factor, None when it never held one."""
        p = self._state()[3]
        return None if p < 0 else ("mixed" if p == 1 else "fp64")


class CholeskyDecomposition:
    """Supernodal Cholesky A = U^T U of a sparse SPD matrix on the GPU.

    ``CholeskyDecomposition(outer, inner, perm)`` mirrors the constructor with
    a fill-reducing permutation (CholeskyDecomposition.hpp:336: perm[i] is the
    original index placed at position i); ``perm=None`` means the matrix is
    already permuted (:350).  The pattern must be the full symmetric pattern
    with the diagonal present.
    """

    SupernodeStrategy_T = SupernodeStrategy
    FactorizationMethod_T = FactorizationMethod

    def __init__(self, outer, inner, perm=None, n: int | None = None, thread_count: int = 0):
        self._outer = np.ascontiguousarray(outer, dtype=np.int64)
        self._inner = np.ascontiguousarray(inner, dtype=np.int32)
        self._n = int(n) if n is not None else len(self._outer) - 1
        self._threads = int(thread_count)
        self._perm = None if perm is None else np.ascontiguousarray(perm, dtype=np.int32)
        if self._perm is not None and self._perm.shape != (self._n,):
            raise TBError(-1, "permutation has the wrong length")
        # the C-ABI reads outer[0..n] and inner[0..outer[n]): the arrays must hold that many
        if self._n < 0 or len(self._outer) < self._n + 1:
            raise TBError(-1, "row pointers shorter than n + 1")
        if self._n > 0 and not (0 <= int(self._outer[self._n]) <= len(self._inner)):
            raise TBError(-2, "row pointers run past the column indices")
        h = ctypes.c_void_p()
        _check(lib().tb_chol_create(ctypes.byref(h), self._n, self._outer.ctypes.data, self._inner.ctypes.data,
                                    None if self._perm is None else self._perm.ctypes.data, int(thread_count)))
        self._h = h
        self._owned = True

    @classmethod
    def _wrap(cls, h, n):
        """A view of a handle owned elsewhere (a batch's combined handle)."""
        obj = cls.__new__(cls)
        obj._h = h
        obj._n = int(n)
        obj._outer = obj._inner = obj._perm = None
        obj._owned = False
        return obj

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and getattr(self, "_owned", True):
            lib().tb_chol_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------------- setup
    def SetSupernodeStrategy(self, strategy) -> None:
        _check(lib().tb_chol_set_supernode_strategy(self._h, int(strategy)))
        self._strategy = SupernodeStrategy(int(strategy))

    def SetAmalgamationThreshold(self, threshold: int) -> None:
        _check(lib().tb_chol_set_amalgamation_threshold(self._h, int(threshold)))
        self._threshold = int(threshold)

    def SetFactorizationMethod(self, method) -> None:
        _check(lib().tb_chol_set_factorization_method(self._h, int(method)))
        self._method = FactorizationMethod(int(method))

    # the settings' getters (InputOutput.hpp), the reference's defaults until set
    def GetSupernodeStrategy(self) -> SupernodeStrategy:
        return getattr(self, "_strategy", SupernodeStrategy.Maximal)

    def AmalgamationThreshold(self) -> int:
        return getattr(self, "_threshold", 4)

    def GetFactorizationMethod(self) -> FactorizationMethod:
        return getattr(self, "_method", FactorizationMethod.Multifrontal)

    def ThreadCount(self) -> int:
        return self._threads

    def SetUseGraph(self, enabled: bool) -> None:
        _check(lib().tb_chol_set_graph(self._h, 1 if enabled else 0))

    def SetPrecision(self, precision) -> None:
        """'fp64' (default) or 'mixed' (FP32 factor with 3xTF32 updates, FP64 refinement in Solve)."""
        code = {"fp64": 0, "mixed": 1}[precision] if isinstance(precision, str) else int(precision)
        _check(lib().tb_chol_set_precision(self._h, code))

    def SetRefinement(self, tol: float = 1e-12, max_iterations: int = 30) -> None:
        _check(lib().tb_chol_set_refinement(self._h, float(tol), int(max_iterations)))

    def PrecisionInUse(self):
        """('fp64' | 'mixed', fell_back): the precision of the current factor; fell_back is True when a mixed
        solve's refinement broke down and the handle refactored in FP64."""
        p, f = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().tb_chol_precision_in_use(self._h, ctypes.byref(p), ctypes.byref(f)))
        return ("mixed" if p.value == 1 else "fp64"), bool(f.value)

    def RefinementInfo(self):
        """(iterations, relative residual) of the last mixed-precision solve."""
        it = ctypes.c_int32()
        rr = ctypes.c_double()
        _check(lib().tb_chol_refinement_info(self._h, ctypes.byref(it), ctypes.byref(rr)))
        return it.value, rr.value

    def PerturbedPivots(self) -> int:
        """Mixed precision: pivots raised to their floor in the last factorization."""
        v = ctypes.c_int32()
        _check(lib().tb_chol_perturbed_pivots(self._h, ctypes.byref(v)))
        return v.value

    def SetSchedule(self, schedule) -> None:
        """'levels' (default: one launch per kind, level and step), 'task_graph' (level launches, then one
        persistent launch for the levels with long panel chains) or 'task_graph_all' (every level in the
        persistent launch)."""
        code = {"levels": 0, "task_graph": 1, "task_graph_all": 2}[schedule] if isinstance(schedule, str) else int(schedule)
        _check(lib().tb_chol_set_schedule(self._h, code))

    def SetSolveSchedule(self, schedule) -> None:
        """Solve sweeps: 'levels' (default: one launch per level and step), 'task_graph' (level launches, then
        one persistent launch per sweep for the levels with 4 or more panel steps) or 'task_graph_all'."""
        code = {"levels": 0, "task_graph": 1, "task_graph_all": 2}[schedule] if isinstance(schedule, str) else int(schedule)
        _check(lib().tb_chol_set_solve_schedule(self._h, code))

    def SolveTrace(self) -> np.ndarray:
        """Trace of the persistent solve launches of the last solve: rows (sweep, task, taken_ns, ready_ns,
        done_ns, cta), forward sweep then back sweep."""
        cap = 12 * max(1, self.PlanStats().get("solve_graph_tasks", 0))
        out = np.zeros(cap, dtype=np.int64)
        m = _check(lib().tb_chol_solve_trace(self._h, out.ctypes.data, cap))
        return out[: 6 * m].reshape(m, 6)

    def Autotune(self, nrhs: int = 1) -> dict:
        """Time both factor schedules (on the last factorization's values) and both solve schedules (nrhs
        right-hand sides), keep the fastest of each; returns the choice and the times in ms."""
        choice = np.zeros(2, dtype=np.int32)
        times = np.zeros(4)
        _check(lib().tb_chol_autotune(self._h, int(nrhs), choice.ctypes.data, times.ctypes.data))
        names = {0: "levels", 1: "task_graph", 2: "task_graph_all"}
        return {"factor": names[int(choice[0])], "solve": names[int(choice[1])],
                "times_ms": {"factor_levels": times[0], "factor_task_graph": times[1],
                             "solve_levels": times[2], "solve_task_graph": times[3]}}

    def SetPlanOptions(self, defer_steps: int = 3, relax: int = 1, tc_width: int = 256) -> None:
        """Device-plan options: trailing-update deferral (1-4 panel steps), front relaxation (0 tight,
        1 default, 2 loose), widest tensor-core tile of the mixed path (128 / 256).  Leaves the object
        unfactorized."""
        _check(lib().tb_chol_set_plan_options(self._h, int(defer_steps), int(relax), int(tc_width)))

    def PlanOptions(self):
        d, r, w = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _check(lib().tb_chol_plan_options(self._h, ctypes.byref(d), ctypes.byref(r), ctypes.byref(w)))
        return d.value, r.value, w.value

    def AutotunePlan(self) -> dict:
        """After a factorization: factor the same values under every candidate plan-option set, keep the
        fastest (the object ends factored under it).  Returns {'choice': (defer, relax, width), 'times_ms': [...]}."""
        choice = (ctypes.c_int32 * 3)()
        times = np.full(64, np.inf)
        m = _check(lib().tb_chol_autotune_plan(self._h, choice, times.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 64))
        return {"choice": tuple(choice), "times_ms": times[:m].tolist()}

    def SetTrace(self, enabled: bool) -> None:
        _check(lib().tb_chol_set_trace(self._h, 1 if enabled else 0))

    def Trace(self) -> np.ndarray:
        """Trace of the last persistent factorization: rows (kind, index, taken_ns, ready_ns, done_ns, cta)."""
        cap = 6 * self.PlanStats()["graph_tasks"]
        out = np.zeros(cap, dtype=np.int64)
        m = _check(lib().tb_chol_trace(self._h, out.ctypes.data, cap))
        return out[: 6 * m].reshape(m, 6)

    def SetStream(self, stream) -> None:
        """Run on a torch.cuda.Stream (or raw handle); None = an owned stream."""
        ptr = None if stream is None else int(getattr(stream, "cuda_stream", stream))
        _check(lib().tb_chol_set_stream(self._h, ptr))

    # -------------------------------------------------------------- phases
    def SymbolicFactorization(self) -> None:
        _check(lib().tb_chol_symbolic(self._h))

    def NumericFactorization(self, values, reg: float = 0.0) -> int:
        """Values in the caller's CSR order (host array or CUDA torch tensor), float64 or float32
        (``NumericFactorization<ExtScal>``, Numeric.hpp:3-8: converted to FP64 on copy)."""
        if _is_cuda_tensor(values):
            import torch

            v = values.contiguous()
            if v.dtype == torch.float64:
                return _check(lib().tb_chol_numeric_device(self._h, v.data_ptr(), float(reg)))
            if v.dtype != torch.float32:
                raise TBError(-1, "NumericFactorization: values must be float64 or float32")
            return _check(lib().tb_chol_numeric_device_ex(self._h, v.data_ptr(), TB_F32, float(reg)))
        v = np.asarray(values)
        if v.dtype == np.float32:
            v = np.ascontiguousarray(v)
            code = TB_F32
        else:
            v = _f64(v)
            code = TB_F64
        if v.shape != (self.NonzeroCount(),):
            raise TBError(-1, "NumericFactorization: wrong number of values")
        return _check(lib().tb_chol_numeric_ex(self._h, v.ctypes.data, code, float(reg)))

    def _solve(self, which: str, B, X=None, alpha=1.0, beta=0.0):
        if _is_cuda_tensor(B):
            return self._solve_device(which, B, X, alpha, beta)
        B = np.asarray(B)
        B = np.ascontiguousarray(B) if B.dtype == np.float32 else _f64(B)
        one_d = B.ndim == 1
        k = 1 if one_d else B.shape[1]
        if B.shape[0] != self._n:
            raise TBError(-1, "Solve: B has the wrong number of rows")
        if X is None:
            X = np.zeros(B.shape, dtype=B.dtype)
            beta = 0.0
        elif not (X.flags.c_contiguous and X.dtype in (np.float64, np.float32) and X.shape == B.shape):
            raise TBError(-1, "Solve: X must be a C-contiguous float64 or float32 array shaped like B")
        if which == "full":
            # B and X may differ in type: each is cast on copy (Solve.hpp:20-27)
            _check(lib().tb_chol_solve_ex(self._h, float(alpha), B.ctypes.data, k, _dtype_code(B.dtype), float(beta),
                                          X.ctypes.data, k, _dtype_code(X.dtype), k))
            return X
        if B.dtype != np.float64 or X.dtype != np.float64:
            raise TBError(-1, "half solves take float64 arrays")
        fn = {"upper": lib().tb_chol_upper_solve, "lower": lib().tb_chol_lower_solve}[which]
        _check(fn(self._h, float(alpha), B.ctypes.data, k, float(beta), X.ctypes.data, k, k))
        return X

    def _solve_device(self, which, B, X, alpha, beta):
        import torch

        if which != "full":
            raise TBError(-1, "device half solves are not exposed")
        B = B.contiguous()
        k = 1 if B.dim() == 1 else B.shape[1]
        if X is None:
            X = torch.empty_like(B)
            beta = 0.0
        codes = {torch.float64: TB_F64, torch.float32: TB_F32}
        if B.dtype not in codes or X.dtype not in codes:
            raise TBError(-1, "Solve: B and X must be float64 or float32 tensors")
        if B.dtype == torch.float64 and X.dtype == torch.float64:
            _check(lib().tb_chol_solve_device(self._h, float(alpha), B.data_ptr(), k, float(beta), X.data_ptr(), k, k))
        else:
            _check(lib().tb_chol_solve_device_ex(self._h, float(alpha), B.data_ptr(), k, codes[B.dtype], float(beta),
                                                 X.data_ptr(), k, codes[X.dtype], k))
        return X

    def SwapNumericalFactorization(self, factor: "NumericalFactorization") -> None:
        """Exchanges this object's numeric factor with ``factor`` (Numeric.hpp:228-254).  A factor that
        says factorized but not good, or is too small for this symbolic analysis, is then treated as
        unfactorized; the object takes the incoming factor's precision."""
        _check(lib().tb_chol_swap_factor(self._h, factor._h))

    def Solve(self, B, X=None, alpha: float = 1.0, beta: float = 0.0):
        """X = alpha * A^{-1} B + beta * X  (Solve.hpp:22-80); B is n or n x nrhs."""
        return self._solve("full", B, X, alpha, beta)

    def UpperSolve(self, B, X=None, alpha: float = 1.0, beta: float = 0.0):
        """X = alpha * P^T U^{-1} P B + beta * X (Solve.hpp:182-243)."""
        return self._solve("upper", B, X, alpha, beta)

    def LowerSolve(self, B, X=None, alpha: float = 1.0, beta: float = 0.0):
        """X = alpha * P^T U^{-T} P B + beta * X (documented meaning of Solve.hpp:248)."""
        return self._solve("lower", B, X, alpha, beta)

    def Residual(self, B, X):
        """R = B - A X on CUDA tensors (row-major n x k), with the last factored values."""
        import torch

        k = 1 if B.dim() == 1 else B.shape[1]
        R = torch.empty_like(B)
        _check(lib().tb_chol_residual_device(self._h, B.data_ptr(), X.data_ptr(), R.data_ptr(), k))
        return R

    def ConjugateGradient(self, B, X=None, values=None, reg: float = 0.0, alpha: float = 1.0, beta: float = 0.0,
                          relative_tolerance: float = 1e-10, max_iter: int = 100, use_initial_guess: bool = False):
        """Conjugate gradients on (A' + reg I) X = B preconditioned by this factor, as the reference's
        ``ConjugateGradient::operator()`` (ConjugateGradient.hpp:109-356) with P = the factor's solve.

        ``values``: A' in the caller's CSR order (None: the values of the last factorization).
        X = alpha x + beta X; with ``use_initial_guess`` the iteration starts from X.  Returns
        ``(X, succeeded)``; ``IterationCount()`` and ``RelativeResiduals()`` report the end state
        (per column sqrt(|r.P r| / |b.P b|)).  Host arrays or CUDA tensors (all of one kind)."""
        cuda = _is_cuda_tensor(B)
        k = 1 if B.ndim == 1 else B.shape[1]
        rel = np.zeros(k, dtype=np.float64)
        iters = ctypes.c_int32()
        if cuda:
            import torch

            B = B.contiguous()
            if X is None:
                X = torch.zeros_like(B)           # the initial guess, if one is asked for: 0
                beta = 0.0
                torch.cuda.current_stream().synchronize()   # the handle's stream is not ordered after torch's
            v = 0 if values is None else values.contiguous().data_ptr()
            st = lib().tb_chol_cg_device(self._h, v, float(reg), float(alpha), B.data_ptr(), k, float(beta),
                                         X.data_ptr(), k, k, float(relative_tolerance), int(max_iter),
                                         int(bool(use_initial_guess)), ctypes.byref(iters), rel.ctypes.data)
        else:
            B = _f64(B)
            if X is None:
                X = np.zeros_like(B)
                beta = 0.0
            elif not (X.flags.c_contiguous and X.dtype == np.float64 and X.shape == B.shape):
                raise TBError(-1, "ConjugateGradient: X must be a C-contiguous float64 array shaped like B")
            v = None if values is None else _f64(values)
            if v is not None and v.shape != (self.NonzeroCount(),):
                raise TBError(-1, "ConjugateGradient: wrong number of values")
            st = lib().tb_chol_cg(self._h, None if v is None else v.ctypes.data, float(reg), float(alpha), B.ctypes.data,
                                  k, float(beta), X.ctypes.data, k, k, float(relative_tolerance), int(max_iter),
                                  int(bool(use_initial_guess)), ctypes.byref(iters), rel.ctypes.data)
        self._cg_iterations, self._cg_relres = iters.value, rel
        if st == -10:
            return X, False
        _check(st)
        return X, True

    def GMRES(self, B, X=None, values=None, reg: float = 0.0, alpha: float = 1.0, beta: float = 0.0,
              relative_tolerance: float = 1e-10, max_iter: int = 30, max_restarts: int = 10,
              use_initial_guess: bool = False):
        """Restarted GMRES on (A' + reg I) X = B, preconditioned from the left by this factor, as the
        reference's ``GMRES::operator()`` (GMRES.hpp:124-330): ``max_iter`` Arnoldi steps per restart.
        Returns ``(X, succeeded)``; ``IterationCount()``, ``GMRESRestarts()`` and ``RelativeResiduals()``
        (per column |P r| / |P b|) report the end state.  Host arrays or CUDA tensors."""
        cuda = _is_cuda_tensor(B)
        k = 1 if B.ndim == 1 else B.shape[1]
        rel = np.zeros(k, dtype=np.float64)
        iters, rests = ctypes.c_int32(), ctypes.c_int32()
        if cuda:
            import torch

            B = B.contiguous()
            if X is None:
                X = torch.zeros_like(B)
                beta = 0.0
                torch.cuda.current_stream().synchronize()
            v = 0 if values is None else values.contiguous().data_ptr()
            st = lib().tb_chol_gmres_device(self._h, v, float(reg), float(alpha), B.data_ptr(), k, float(beta),
                                            X.data_ptr(), k, k, float(relative_tolerance), int(max_iter),
                                            int(max_restarts), int(bool(use_initial_guess)), ctypes.byref(iters),
                                            ctypes.byref(rests), rel.ctypes.data)
        else:
            B = _f64(B)
            if X is None:
                X = np.zeros_like(B)
                beta = 0.0
            elif not (X.flags.c_contiguous and X.dtype == np.float64 and X.shape == B.shape):
                raise TBError(-1, "GMRES: X must be a C-contiguous float64 array shaped like B")
            v = None if values is None else _f64(values)
            st = lib().tb_chol_gmres(self._h, None if v is None else v.ctypes.data, float(reg), float(alpha),
                                     B.ctypes.data, k, float(beta), X.ctypes.data, k, k, float(relative_tolerance),
                                     int(max_iter), int(max_restarts), int(bool(use_initial_guess)),
                                     ctypes.byref(iters), ctypes.byref(rests), rel.ctypes.data)
        self._cg_iterations, self._cg_relres, self._gmres_restarts = iters.value, rel, rests.value
        if st == -10:
            return X, False
        _check(st)
        return X, True

    def GMRESRestarts(self) -> int:
        return getattr(self, "_gmres_restarts", 0)

    def GMRESIRIterations(self) -> int:
        """GMRES-IR steps of the last mixed-precision solve (-1: its CG refinement sufficed)."""
        v = ctypes.c_int32()
        _check(lib().tb_chol_gmres_ir_iterations(self._h, ctypes.byref(v)))
        return v.value

    def IterationCount(self) -> int:
        """Steps of the last ConjugateGradient call (ConjugateGradient.hpp:442)."""
        return getattr(self, "_cg_iterations", 0)

    def RelativeResiduals(self) -> np.ndarray:
        """Per column sqrt(|r.P r| / |b.P b|) after the last ConjugateGradient call (ConjugateGradient.hpp:459)."""
        return getattr(self, "_cg_relres", np.zeros(0))

    # ------------------------------------------------------------- getters
    def _array(self, name: str) -> np.ndarray:
        size = ctypes.c_int64()
        _check(lib().tb_chol_array_size(self._h, _ARRAYS[name], ctypes.byref(size)))
        out = np.zeros(size.value, dtype=np.int64)
        if size.value:
            _check(lib().tb_chol_array_copy(self._h, _ARRAYS[name], out.ctypes.data))
        return out

    def SymbolicArray(self, name: str) -> np.ndarray:
        return self._array(name)

    def RowCount(self) -> int:
        return self._n

    def ColCount(self) -> int:
        return self._n

    def NonzeroCount(self) -> int:
        v = ctypes.c_int64()
        _check(lib().tb_chol_nonzero_count(self._h, ctypes.byref(v)))
        return v.value

    def SN_Count(self) -> int:
        v = ctypes.c_int32()
        _check(lib().tb_chol_sn_count(self._h, ctypes.byref(v)))
        return v.value

    def SN_RowPointers(self):
        return self._array("SN_rp")

    def SN_Outer(self):
        return self._array("SN_outer")

    def SN_Inner(self):
        return self._array("SN_inner")

    def RowToSN(self):
        return self._array("row_to_SN")

    def SN_TrianglePointers(self):
        return self._array("SN_tri_ptr")

    def SN_RectanglePointers(self):
        return self._array("SN_rec_ptr")

    def GetPermutation(self):
        return self._array("perm")

    def GetInversePermutation(self):
        return self._array("perm_inv")

    def GetValuePermutation(self):
        return self._array("value_perm")

    def AssemblyTreeParents(self):
        return self._array("aTree_parents")

    def EliminationTreeParents(self):
        return self._array("eTree_parents")

    def RequiredTriangularSize(self) -> int:
        t, r = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().tb_chol_factor_sizes(self._h, ctypes.byref(t), ctypes.byref(r)))
        return t.value

    def RequiredRectangularSize(self) -> int:
        t, r = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().tb_chol_factor_sizes(self._h, ctypes.byref(t), ctypes.byref(r)))
        return r.value

    def FactorValues(self):
        """(SN_TriangleValues, SN_RectangleValues) in the reference layout."""
        tri = np.zeros(self.RequiredTriangularSize())
        rec = np.zeros(self.RequiredRectangularSize())
        _check(lib().tb_chol_factor_values(self._h, tri.ctypes.data, rec.ctypes.data))
        return tri, rec

    def SN_TriangleValues(self):
        return self.FactorValues()[0]

    def SN_RectangleValues(self):
        return self.FactorValues()[1]

    def NumericallyFactorizedQ(self) -> bool:
        f, g = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().tb_chol_factorized(self._h, ctypes.byref(f), ctypes.byref(g)))
        return bool(f.value)

    def NumericallyGoodQ(self) -> bool:
        f, g = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().tb_chol_factorized(self._h, ctypes.byref(f), ctypes.byref(g)))
        return bool(g.value)

    def FailedSupernode(self) -> int:
        v = ctypes.c_int32()
        _check(lib().tb_chol_failed_supernode(self._h, ctypes.byref(v)))
        return v.value

    def LogDeterminant(self) -> float:
        v = ctypes.c_double()
        _check(lib().tb_chol_log_det(self._h, ctypes.byref(v)))
        return v.value

    def FactorLogDeterminant(self) -> float:
        return 0.5 * self.LogDeterminant()

    def WriteFactorDiagonal(self):
        d = np.zeros(self._n)
        _check(lib().tb_chol_factor_diagonal(self._h, d.ctypes.data))
        return d

    def FlopCount(self):
        f, z = ctypes.c_double(), ctypes.c_double()
        _check(lib().tb_chol_flop_count(self._h, ctypes.byref(f), ctypes.byref(z)))
        return f.value, z.value

    def PlanStats(self) -> dict:
        out = np.zeros(32, dtype=np.int64)
        m = _check(lib().tb_chol_plan_stats(self._h, out.ctypes.data, 32))
        keys = ["arena_doubles", "update_doubles", "levels", "factor_launches", "gemm_tasks", "panel_tasks",
                "extend_tasks", "lower_launches", "upper_launches", "supernodes", "fronts", "front_flops", "graph_makespan_us", "graph_tasks",
                "solve_graph_tasks", "solve_split_level", "graph_ctas", "analyze_us", "plan_us", "tc_tiles",
                "image_blocks", "gemm_flops", "gemm_tile_flops", "super_panels", "lower_launches_super",
                "upper_launches_super"]
        return {k: int(out[i]) for i, k in enumerate(keys[:m])}

    def CheckPlan(self) -> None:
        """Host-side bounds check of every device task (raises TBError)."""
        _check(lib().tb_chol_check_plan(self._h))

    def DeviceBytes(self) -> int:
        v = ctypes.c_int64()
        _check(lib().tb_chol_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    def SetProfiling(self, enabled: bool) -> None:
        _check(lib().tb_chol_set_profiling(self._h, 1 if enabled else 0))

    def KernelProfile(self) -> dict:
        """Per launch kind of the last profiled factorization: ms, launches, flops."""
        ms = np.zeros(8)
        ln = np.zeros(8, dtype=np.int64)
        fl = np.zeros(8)
        _check(lib().tb_chol_kernel_profile(self._h, ms.ctypes.data, ln.ctypes.data, fl.ctypes.data))
        names = {0: "zero", 1: "extend", 2: "trsm", 3: "gemm", 4: "invert", 6: "potrf", 7: "assemble"}
        return {names[k]: {"ms": float(ms[k]), "launches": int(ln[k]), "flops": float(fl[k])} for k in names}

    def LaunchProfile(self):
        """Per launch of the last profiled factorization: (kind, level, step, tasks, ms)."""
        cap = 1 << 16
        info = np.zeros(4 * cap, dtype=np.int64)
        ms = np.zeros(cap)
        m = _check(lib().tb_chol_launch_profile(self._h, info.ctypes.data, ms.ctypes.data, cap))
        names = {0: "zero", 1: "extend", 2: "trsm", 3: "gemm", 4: "invert", 6: "potrf", 7: "assemble"}
        return [(names.get(int(info[4 * i]), "?"), int(info[4 * i + 1]), int(info[4 * i + 2]), int(info[4 * i + 3]),
                 float(ms[i])) for i in range(m)]

    def SolveProfile(self):
        """Per launch of the last profiled solve: (sweep, level, step, tasks, ms), sweep 0 forward / 1 back."""
        cap = 1 << 16
        info = np.zeros(4 * cap, dtype=np.int64)
        ms = np.zeros(cap)
        m = _check(lib().tb_chol_solve_profile(self._h, info.ctypes.data, ms.ctypes.data, cap))
        return [(int(info[4 * i]), int(info[4 * i + 1]), int(info[4 * i + 2]), int(info[4 * i + 3]), float(ms[i]))
                for i in range(m)]

    def LaunchCounts(self):
        a, b = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().tb_chol_launch_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def UNonzeroCount(self) -> int:
        v = ctypes.c_int64()
        _check(lib().tb_chol_u_nonzero_count(self._h, ctypes.byref(v)))
        return v.value

    def GetU(self):
        """U as a scipy CSR matrix in the permuted ordering (InputOutput.hpp:116-217)."""
        import scipy.sparse as sp

        rp = self.SN_RowPointers()
        so = self.SN_Outer()
        si = self.SN_Inner()
        tp = self.SN_TrianglePointers()
        rcp = self.SN_RectanglePointers()
        tri, rec = self.FactorValues()
        rows, cols, vals = [], [], []
        for s in range(len(rp) - 1):
            i0, i1 = rp[s], rp[s + 1]
            n0, n1 = i1 - i0, so[s + 1] - so[s]
            U0 = tri[tp[s]: tp[s] + n0 * n0].reshape(n0, n0)
            U1 = rec[rcp[s]: rcp[s] + n0 * n1].reshape(n0, n1)
            r, c = np.triu_indices(n0)
            rows.append(i0 + r); cols.append(i0 + c); vals.append(U0[r, c])
            if n1:
                rr = np.repeat(np.arange(n0), n1)
                rows.append(i0 + rr); cols.append(np.tile(si[so[s]: so[s + 1]], n0)); vals.append(U1.ravel())
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(self._n, self._n))

    def UNonzeroCount(self) -> int:
        """Nonzeros of U (tb_chol_u_nonzero_count; host-only after the symbolic phase)."""
        v = ctypes.c_int64()
        _check(lib().tb_chol_u_nonzero_count(self._h, ctypes.byref(v)))
        return v.value


def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


class BatchedCholesky:
    """Many independent SPD systems factored and solved together (tb_batch_*).

    ``systems`` is a list of ``(outer, inner, perm)`` (perm may be None).  The
    systems become the diagonal blocks of one matrix whose factorization runs
    as a single persistent launch; ``handle`` gives the underlying
    :class:`CholeskyDecomposition` for precision, refinement and statistics.
    """

    def __init__(self, systems, thread_count: int = 0):
        self._keep = []
        count = len(systems)
        n = np.zeros(count, dtype=np.int32)
        outer_p = (ctypes.c_void_p * count)()
        inner_p = (ctypes.c_void_p * count)()
        perm_p = (ctypes.c_void_p * count)()
        for s, (outer, inner, perm) in enumerate(systems):
            o = np.ascontiguousarray(outer, dtype=np.int64)
            i = np.ascontiguousarray(inner, dtype=np.int32)
            n[s] = len(o) - 1
            if n[s] > 0 and not (0 <= int(o[-1]) <= len(i)):
                raise TBError(-2, f"system {s}: row pointers run past the column indices")
            if perm is not None and len(perm) != n[s]:
                raise TBError(-1, f"system {s}: permutation has the wrong length")
            outer_p[s] = o.ctypes.data
            inner_p[s] = i.ctypes.data
            self._keep += [o, i]
            if perm is not None:
                p = np.ascontiguousarray(perm, dtype=np.int32)
                perm_p[s] = p.ctypes.data
                self._keep.append(p)
        self._b = ctypes.c_void_p()
        _check(lib().tb_batch_create(ctypes.byref(self._b), count, n.ctypes.data, ctypes.addressof(outer_p),
                                     ctypes.addressof(inner_p), ctypes.addressof(perm_p), int(thread_count)))
        self._keep.clear()
        self.count = count
        self.sizes = n.astype(np.int64)
        self.row_offsets = np.zeros(count + 1, dtype=np.int64)
        self.value_offsets = np.zeros(count + 1, dtype=np.int64)
        _check(lib().tb_batch_offsets(self._b, self.row_offsets.ctypes.data, self.value_offsets.ctypes.data))
        h = ctypes.c_void_p()
        _check(lib().tb_batch_handle(self._b, ctypes.byref(h)))
        self.handle = CholeskyDecomposition._wrap(h, self.row_offsets[-1])

    def close(self):
        if getattr(self, "_b", None):
            lib().tb_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def NumericFactorization(self, values, reg: float = 0.0) -> int:
        """values: list of per-system arrays, or one concatenated CUDA tensor / array."""
        if isinstance(values, (list, tuple)):
            vs = [np.ascontiguousarray(v, dtype=np.float64) for v in values]
            ptrs = (ctypes.c_void_p * self.count)(*[v.ctypes.data for v in vs])
            return _check(lib().tb_batch_numeric(self._b, ctypes.addressof(ptrs), float(reg)))
        if _is_cuda_tensor(values):
            return _check(lib().tb_batch_numeric_device(self._b, values.data_ptr(), float(reg)))
        return self.handle.NumericFactorization(np.ascontiguousarray(values, dtype=np.float64), reg)

    def FailedSystem(self) -> int:
        v = ctypes.c_int32()
        _check(lib().tb_batch_failed_system(self._b, ctypes.byref(v)))
        return v.value

    def Solve(self, B, X=None):
        """B: list of per-system (n_s,) or (n_s, k) arrays -> list of solutions; or a stacked CUDA tensor."""
        if _is_cuda_tensor(B):
            k = 1 if B.dim() == 1 else B.shape[1]
            if X is None:
                X = B.new_empty(B.shape)
            _check(lib().tb_batch_solve_device(self._b, B.data_ptr(), X.data_ptr(), int(k)))
            return X
        Bs = [np.ascontiguousarray(b, dtype=np.float64) for b in B]
        k = 1 if Bs[0].ndim == 1 else Bs[0].shape[1]
        Xs = [np.empty_like(b) for b in Bs]
        bp = (ctypes.c_void_p * self.count)(*[b.ctypes.data for b in Bs])
        xp = (ctypes.c_void_p * self.count)(*[x.ctypes.data for x in Xs])
        _check(lib().tb_batch_solve(self._b, ctypes.addressof(bp), ctypes.addressof(xp), int(k)))
        return Xs
