"""The C-ABI library without a GPU: it loads, exports every declared symbol,
and its host-side generator matches the oracle's bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "psiboil_b200.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pbg_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import psiboil_b200 as pb
    L = ctypes.CDLL(pb.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    import psiboil_b200 as pb
    assert set(declared()) <= set(pb._SIGS)


def test_version_and_defaults():
    import psiboil_b200 as pb
    assert pb.lib().pbg_version() == 1
    p = pb.default_params(pb.SOLVER_CG)
    assert (p.min_iter, p.max_iter, p.res_rat, p.res_tol, p.stalecount) == (1, 20, 0.01, 1e-15, -1)
    a = pb.default_params(pb.SOLVER_AC)
    assert (a.max_cycles, a.min_cycles, a.stop_if_div, list(a.mv), list(a.ms)) == \
        (20, 0, 1, [20, 20, 20], [-1, -1, -1])


@pytest.mark.parametrize("kind,kw", [(0, dict(n=10)), (1, dict(n=20, nb=3, rmin=2.0, rmax=4.0, rc=4.0)),
                                     (2, dict(index=3, n2d=4, s2=(16, 30))),
                                     (2, dict(index=7, n2d=4, s3=(9, 13)))])
def test_generator_matches_oracle(oracle, kind, kw):
    import psiboil_b200 as pb
    dims, h, rho, solid, b = pb.generate(kind, 5, **kw)
    P = oracle.Problem(kind, 5, **kw)
    assert dims == P.dims and h == P.h
    assert np.array_equal(rho, P.rho) and np.array_equal(solid, P.solid) and np.array_equal(b, P.b)


def test_bad_arguments_fail_loudly():
    import psiboil_b200 as pb
    with pytest.raises(pb.PbgError):
        pb.Session(0, 4, 4, 0.25)
