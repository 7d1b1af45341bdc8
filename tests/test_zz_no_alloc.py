"""pbg_dot_noalloc — the dot product for callers that cannot allocate.

Callers recording work into a CUDA graph (no cudaMalloc during stream
capture), or working in memory owned by another allocator, need a dot
product that allocates nothing. pbg_dot_noalloc keeps its scratch in a
fixed array inside the library; this test calls it through the C ABI on
device arrays, twice in a row (the second call reuses the array left by the
first), and checks both results against the session-based pbg_dot. The file
is collected last so that a failing run has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the sums are formed in the same order by both entry points; the tolerance
# is the one the dot-product tests use
RTOL = 1e-12


def test_dot_noalloc_matches_pbg_dot_twice():
    torch = pytest.importorskip("torch")
    import psiboil_b200 as pb
    assert pb.device_count() >= 1
    torch.cuda.set_device(0)
    rng = np.random.default_rng(11)
    nx, ny, nz, h = 40, 36, 44, 1.0 / 40
    n = nx * ny * nz
    dV = (h * h) * h
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pb.Session(nx, ny, nz, h) as s:
        for call in range(2):
            x = rng.standard_normal(n)
            y = rng.standard_normal(n)
            ref = s.dot(x, y)                      # session scratch
            xd = torch.from_numpy(x).cuda()
            yd = torch.from_numpy(y).cuda()
            pb.dot_noalloc(xd, yd, dV, out)        # fixed scratch, no allocation
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert got[0] == pytest.approx(ref[0], rel=RTOL, abs=1e-12 * np.abs(x * y).sum()), call
            assert got[1] == pytest.approx(ref[1], rel=RTOL), call


def test_dot_noalloc_rejects_bad_sizes():
    torch = pytest.importorskip("torch")
    import psiboil_b200 as pb
    L = pb.lib()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = L.pbg_dot_noalloc(x.data_ptr(), x.data_ptr(), (1 << 31), 1.0, out.data_ptr(), None)
    assert rc == -1 and b"2^31" in L.pbg_last_error()
    rc = L.pbg_dot_noalloc(x.data_ptr(), x.data_ptr(), 0, 1.0, out.data_ptr(), None)
    assert rc == -1
