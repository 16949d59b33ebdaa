"""Serving runtime: continuous batching over resident factors under an HBM cap.

Each request's result in the mix must equal (within the refinement
tolerance) the result of the same request served alone."""
from __future__ import annotations

import numpy as np
import pytest

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import TBError
from tensors_b200.serving import Server, footprint_estimate


def _mats():
    out = []
    for A in (M.grid_laplacian_3d(14, 31, 1e-2), M.vector_laplacian_3d(6, 32, 1e-2), M.grid_laplacian_2d(60, 1e-2),
              M.grid_laplacian_3d(18, 33, 1e-2)):
        out.append((A, O.nested_dissection(A)))
    return out


MATS = _mats()


def test_server_validates_requests_without_running_them():
    A, p = MATS[2]
    srv = Server(hbm_cap_bytes=1 << 30, slots=2)
    mid = srv.add_matrix(A.outer, A.inner, p)
    with pytest.raises(TBError):
        srv.submit(mid + 5, values=A.values)                    # unknown matrix
    with pytest.raises(TBError):
        srv.submit(mid)                                          # neither a factorization nor a solve
    small = Server(hbm_cap_bytes=1024, slots=1)
    mid2 = small.add_matrix(A.outer, A.inner, p)
    with pytest.raises(TBError):
        small.submit(mid2, values=A.values)                      # footprint above the cap
    assert footprint_estimate(A.outer, A.inner, p) > 0
    srv.close()
    small.close()


@pytest.mark.gpu
def test_mixed_stream_matches_requests_served_alone():
    rng = np.random.default_rng(5)
    tol = 1e-10
    from tensors_b200.cholesky import CholeskyDecomposition

    foot = []
    for A, p in MATS:                                            # measured device bytes of a mixed factor
        c = CholeskyDecomposition(A.outer, A.inner, p)
        c.SetPrecision("mixed")
        assert c.NumericFactorization(A.values) == 0
        c.Solve(np.ones((A.n, 4)))
        foot.append(int(1.02 * c.DeviceBytes()))
        c.close()
    cap = max(foot) + sorted(foot)[-2]                           # two factors fit, four do not: evictions
    plan = []                                                    # (matrix, factor?, B)
    for j in range(40):
        m = int(rng.integers(0, len(MATS)))
        A = MATS[m][0]
        k = int(rng.integers(1, 5))
        plan.append((m, j < len(MATS) or rng.random() < 0.7, rng.standard_normal((A.n, k))))

    def serve(requests, slots):
        srv = Server(hbm_cap_bytes=cap, slots=slots)
        ids = [srv.add_matrix(A.outer, A.inner, p, footprint_bytes=f) for (A, p), f in zip(MATS, foot)]
        tickets, done = [], set()
        for m, fac, B in requests:
            if not fac and m not in done:
                fac = True                                       # the first request of a matrix factors it
            done.add(m)
            tickets.append(srv.submit(ids[m], values=MATS[m][0].values if fac else None, B=B, tol=tol))
        results = [srv.wait(t) for t in tickets]
        st = srv.stats()
        srv.close()
        return results, st

    mixed, st = serve(plan, slots=3)
    assert st["evictions"] > 0
    assert st["peak_resident_bytes"] <= cap
    for (m, fac, B), (X, info) in zip(plan, mixed):
        A = MATS[m][0]
        assert info["status"] == 0
        R = B - A.to_scipy() @ X
        assert np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)) <= 2 * tol
        alone, _ = serve([(m, True, B)], slots=1)
        Xa = alone[0][0]
        assert np.abs(X - Xa).max() <= 1e-7 * np.abs(Xa).max()
    lat = np.array([info["latency_ms"] for _, info in mixed])
    assert np.all(lat > 0)
