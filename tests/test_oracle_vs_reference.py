"""Oracle vs the compiled reference run live (only where oracle/_ref was
built, i.e. where the reference sources exist)."""
import numpy as np
import pytest

import oracle_py


pytestmark = pytest.mark.skipif(not oracle_py.harness_available(),
                                reason="reference harness not built here")


@pytest.mark.parametrize("kind,kw", [(0, dict(n=20)), (1, dict(n=28, nb=4, rmin=2.0, rmax=5.0, rc=6.0)),
                                     (2, dict(index=5, n2d=8, s2=(30, 50)))])
def test_live_cg_and_ac(oracle, kind, kw):
    P = oracle.Problem(kind, 11, **kw)
    meta, arr = oracle.run_reference(P, "cg")
    x, st = oracle.cg(P)
    assert st["printed"] == int(meta["iterations"])
    assert np.array_equal(x, arr["x"])
    meta, arr = oracle.run_reference(P, "ac")
    x, st = oracle.AC(P).cycle()
    assert st["cycles"] == int(meta["cycles"])
    assert np.array_equal(x, arr["x"])
