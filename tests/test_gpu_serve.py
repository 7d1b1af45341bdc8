"""Serving loop (pbg_server_*): sessions resident on the device, requests
batched continuously by a worker thread.

Checked: a request's result is bit-for-bit the same alone and in a mix of
concurrent requests on other sessions (other sizes, entering and leaving the
batch while it runs); host-submitted requests reach the FP64 true residual
1e-8 recomputed by the oracle, and warm starts from the session's previous
solution; admission refuses sessions beyond the HBM budget; many requests
from several threads all complete."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-8


def bubble_seq(n, k):
    """Request k of a rising-bubble sequence on an n^3 grid."""
    return dict(center=(n / 2, n / 2, n / 3 + 0.5 * k), radius=n / 5, ratio=1000.0, seed=1000 + k)


@pytest.mark.parametrize("precision", [0, 1])
def test_alone_equals_in_mix(engine, precision):
    n, steps = 28, 3
    h = 1.0 / n
    alone = []
    with engine.Server(precision=precision, slots=4) as S:
        sid = S.open_session((n, n, n), h)
        for k in range(steps):
            r, _ = S.wait(S.submit_bubble(sid, **bubble_seq(n, k)))
            assert r.converged
            alone.append((r.iterations, r.sweeps, S.get_x(sid)))
    mixed = []
    with engine.Server(precision=precision, slots=3) as S:
        others = [S.open_session((m, m, m), 1.0 / m) for m in (20, 33, 41, 24)]
        sid = S.open_session((n, n, n), h)
        pending = []
        for k in range(steps):
            # load the batch with other sessions' requests around each target request
            for j, o in enumerate(others):
                m = S.dims[o][0]
                pending.append(S.submit_bubble(o, **bubble_seq(m, 2 * k + j)))
            rid = S.submit_bubble(sid, **bubble_seq(n, k))
            for j, o in enumerate(others[:2]):
                m = S.dims[o][0]
                pending.append(S.submit_bubble(o, **bubble_seq(m, 2 * k + j + 1)))
            r, _ = S.wait(rid)
            assert r.converged
            mixed.append((r.iterations, r.sweeps, S.get_x(sid)))
        for p in pending:
            r, _ = S.wait(p)
            assert r.converged
    for (ia, sa, xa), (ib, sb, xb) in zip(alone, mixed):
        assert (ia, sa) == (ib, sb)
        assert np.array_equal(xa, xb)


def test_host_requests_reach_tolerance_with_warm_start(engine, oracle):
    P = oracle.Problem(oracle.KIND_CYL, 2, n=32, nb=4, rmin=2.0, rmax=5.0, rc=6.0)
    with engine.Server(precision=1, slots=2) as S:
        sid = S.open_session(P.dims, P.h)
        r1, lat1 = S.wait(S.submit(sid, P.b, rho=P.rho, solid=P.solid))
        x1 = S.get_x(sid)
        assert r1.converged and lat1 > 0
        assert np.linalg.norm(oracle.resid(P, x1, P.b)) / np.linalg.norm(P.b) <= TOL * 1.0001
        # same matrix, perturbed right-hand side: warm start from x1
        b2 = P.b * 1.001
        r2, _ = S.wait(S.submit(sid, b2))
        x2 = S.get_x(sid)
        assert r2.converged and r2.iterations < r1.iterations
        assert np.linalg.norm(oracle.resid(P, x2, b2)) / np.linalg.norm(b2) <= TOL * 1.0001


def test_admission_budget(engine):
    with engine.Server(precision=1, slots=2, hbm_budget=32 << 20) as S:
        a = S.open_session((40, 40, 40), 1 / 40)
        with pytest.raises(engine.PbgError) as e:
            S.open_session((64, 64, 64), 1 / 64)
        assert e.value.code == -6
        S.close_session(a)
        b = S.open_session((48, 48, 48), 1 / 48)
        assert S.stats()["sessions"] == 1 and b != a


def test_many_requests_from_threads(engine):
    with engine.Server(precision=1, slots=4) as S:
        sids = [S.open_session((m, m, m), 1.0 / m) for m in (16, 24, 30, 20, 36, 18)]
        rids, lock = [], threading.Lock()

        def client(t):
            for k in range(6):
                sid = sids[(t * 3 + k) % len(sids)]
                m = S.dims[sid][0]
                rid = S.submit_bubble(sid, **bubble_seq(m, k + 10 * t))
                with lock:
                    rids.append(rid)

        th = [threading.Thread(target=client, args=(t,)) for t in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        res = [S.wait(r, timeout=120.0) for r in rids]
        assert all(r.converged and r.relres <= TOL for r, _ in res)
        st = S.stats()
        assert st["submitted"] == st["completed"] == len(rids) and st["in_flight"] == 0
