"""pbg_dot_noalloc — the dot product for callers that cannot allocate.

Some callers cannot call cudaMalloc where they need a dot product: a host
code that hands all device memory to its own pool at start-up, or a
time-step loop that must not take an allocation's latency or failure path
in mid-step. pbg_dot_noalloc keeps its scratch in a fixed array inside the
library. This test calls it through the C ABI on device arrays, twice in a
row (the second call reuses the array the first one left), and checks both
results against the session-based pbg_dot. Both entry points launch the same
grid and add in the same order, so the results must be equal bit for bit.
One case is larger than the grid (more than 1,184 blocks of 256 elements),
so that the grid-stride loop and every partial-sum slot are used. The file
is collected last, so a run that stops at the first failure has already run
every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(40, 36, 44), (80, 72, 64)], ids=["small", "grid_stride"])
def test_dot_noalloc_matches_pbg_dot_twice(dims):
    torch = pytest.importorskip("torch")
    import psiboil_b200 as pb
    assert pb.device_count() >= 1
    torch.cuda.set_device(0)
    rng = np.random.default_rng(11)
    nx, ny, nz = dims
    h = 1.0 / nx
    n = nx * ny * nz
    if dims[0] == 80:
        assert n > 1184 * 256
    dV = (h * h) * h
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pb.Session(nx, ny, nz, h) as s:
        for call in range(2):
            x = rng.standard_normal(n)
            y = rng.standard_normal(n)
            ref = s.dot(x, y)                      # session scratch
            xd = torch.from_numpy(x).cuda()
            yd = torch.from_numpy(y).cuda()
            torch.cuda.synchronize()
            pb.dot_noalloc(xd, yd, dV, out)        # fixed scratch, no allocation
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert got[0] == ref[0], call
            assert got[1] == ref[1], call


def test_dot_noalloc_rejects_bad_arguments():
    torch = pytest.importorskip("torch")
    import psiboil_b200 as pb
    L = pb.lib()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = L.pbg_dot_noalloc(x.data_ptr(), x.data_ptr(), (1 << 31), 1.0, out.data_ptr(), None)
    assert rc == -1 and b"2^31" in L.pbg_last_error()
    rc = L.pbg_dot_noalloc(x.data_ptr(), x.data_ptr(), 0, 1.0, out.data_ptr(), None)
    assert rc == -1
    # the Python binding refuses what would reach the kernel as a bad pointer
    with pytest.raises(TypeError):
        pb.dot_noalloc(x.float(), x.float(), 1.0, out)
    with pytest.raises(TypeError):
        pb.dot_noalloc(x, x, 1.0, torch.zeros(2, dtype=torch.float64))
    with pytest.raises(ValueError):
        pb.dot_noalloc(torch.zeros(8, dtype=torch.float64, device="cuda")[::2], x, 1.0, out)
