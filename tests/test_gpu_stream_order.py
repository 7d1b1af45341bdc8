"""Device inputs that torch writes on its current stream are seen by the
session's calls, which run on the session's own non-blocking stream. The
tensor is filled behind ~25 ms of GPU spinning on torch's stream, so a call
that did not wait for torch's stream would read zeros.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _late_copy(torch, src):
    x = torch.zeros_like(src)
    torch.cuda._sleep(50_000_000)
    x.copy_(src)
    return x


def test_dot_waits_for_torch_stream(engine):
    import torch
    n = 32
    N = n ** 3
    src = (torch.arange(N, dtype=torch.float64, device="cuda") + 1.0) / N
    want = float(torch.dot(src, src))
    with engine.Session(n, n, n, 1.0 / n) as s:
        for _ in range(3):
            x = _late_copy(torch, src)
            got = s.dot(x, x)[0]
            assert abs(got - want) <= 1e-12 * want


def test_project_waits_for_torch_stream(engine, oracle):
    import torch
    import flow
    P = oracle.Problem(1, 5, n=32, nb=3, rmin=2.0, rmax=4.0, rc=5.0)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    p = np.random.default_rng(3).standard_normal(P.N)
    ru, rv, rw = flow.project(P.dims, P.h, 1e-3, p, col, ra, rb, u, v, w, solid=P.solid)
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        # every upload first (a pageable upload waits for the stream's earlier work)
        dev = [torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda() for a in (p, col, u, v, w)]
        sd = torch.from_numpy(P.solid).cuda()
        torch.cuda.synchronize()
        pd, cd, ud, vd, wd = (_late_copy(torch, t) for t in dev)
        s.project(pd, cd, ra, rb, 1e-3, ud, vd, wd, solid=sd)
        # torch work after the call sees its results
        for a, b in ((ud, ru), (vd, rv), (wd, rw)):
            assert np.array_equal(a.cpu().numpy(), b.reshape(-1))
