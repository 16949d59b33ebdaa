"""Python mirror of the request-serving runtime (tb_server_* in serve.cpp).

    srv = Server(hbm_cap_bytes=150 << 30, slots=4)
    mid = srv.add_matrix(outer, inner, perm)
    t = srv.submit(mid, values=vals, B=b)          # factor + solve
    t2 = srv.submit(mid, B=b2)                     # solve on the resident factor
    x, info = srv.wait(t)                          # info: status, latency_ms, run_ms, iterations, relres
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib
from .cholesky import CholeskyDecomposition, _check

PRECISIONS = {"fp64": 0, "mixed": 1}


def footprint_estimate(outer, inner, perm=None, precision: str = "mixed") -> int:
    """Device bytes of a handle for this pattern, from the host symbolic phase: the factor arena plus task
    tables, inverse diagonal blocks and work buffers (the server replaces it by the measured size)."""
    c = CholeskyDecomposition(outer, inner, perm)
    st = c.PlanStats()
    elem = 4 if precision == "mixed" else 8
    n = len(outer) - 1
    arena = st["arena_doubles"] * elem
    tasks = 64 * (st["gemm_tasks"] + st["panel_tasks"] + st["extend_tasks"]) + 48 * st.get("graph_tasks", 0)
    panels = 32768 * (st["panel_tasks"] // 2 + st["fronts"])
    return int(arena + tasks + panels + 64 * len(inner) + 256 * n + (32 << 20))


class Ticket:
    __slots__ = ("id", "B", "X", "k")

    def __init__(self, rid, B, X, k):
        self.id, self.B, self.X, self.k = rid, B, X, k


class Server:
    def __init__(self, hbm_cap_bytes: int, slots: int = 4, precision: str = "mixed", device: int = 0):
        self.precision = precision
        self._s = ctypes.c_void_p()
        _check(lib().tb_server_create(ctypes.byref(self._s), int(device), int(hbm_cap_bytes), int(slots),
                                      PRECISIONS[precision]))
        self._n = []

    def close(self):
        if getattr(self, "_s", None) is not None and self._s.value:
            lib().tb_server_destroy(self._s)
        self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_matrix(self, outer, inner, perm=None, footprint_bytes: int | None = None) -> int:
        o = np.ascontiguousarray(outer, dtype=np.int64)
        i = np.ascontiguousarray(inner, dtype=np.int32)
        p = None if perm is None else np.ascontiguousarray(perm, dtype=np.int32)
        fb = footprint_bytes or footprint_estimate(o, i, p, self.precision)
        mid = ctypes.c_int64()
        _check(lib().tb_server_add_matrix(self._s, len(o) - 1, o.ctypes.data, i.ctypes.data,
                                          None if p is None else p.ctypes.data, int(fb), ctypes.byref(mid)))
        self._n.append(len(o) - 1)
        return mid.value

    def submit(self, matrix_id: int, values=None, reg: float = 0.0, B=None, tol: float = 1e-10) -> Ticket:
        v = None if values is None else np.ascontiguousarray(values, dtype=np.float64)
        Bc = X = None
        k = 1
        if B is not None:
            Bc = np.ascontiguousarray(B, dtype=np.float64)
            k = 1 if Bc.ndim == 1 else Bc.shape[1]
            X = np.empty_like(Bc)
        rid = ctypes.c_int64()
        _check(lib().tb_server_submit(self._s, int(matrix_id), None if v is None else v.ctypes.data, float(reg),
                                      None if Bc is None else Bc.ctypes.data, None if X is None else X.ctypes.data,
                                      int(k), float(tol), ctypes.byref(rid)))
        return Ticket(rid.value, Bc, X, k)

    def wait(self, ticket: Ticket):
        st = ctypes.c_int32()
        lat, run, rr = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        it = ctypes.c_int32()
        _check(lib().tb_server_wait(self._s, ticket.id, ctypes.byref(st), ctypes.byref(lat), ctypes.byref(run),
                                    ctypes.byref(it), ctypes.byref(rr)))
        return ticket.X, {"status": st.value, "latency_ms": lat.value, "run_ms": run.value,
                          "iterations": it.value, "relres": rr.value}

    def stats(self) -> dict:
        r, p, e, f = (ctypes.c_int64() for _ in range(4))
        _check(lib().tb_server_stats(self._s, ctypes.byref(r), ctypes.byref(p), ctypes.byref(e), ctypes.byref(f)))
        return {"resident_bytes": r.value, "peak_resident_bytes": p.value, "evictions": e.value, "refactors": f.value}
