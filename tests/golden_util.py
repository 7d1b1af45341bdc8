"""Loading of the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["single16", "single12", "cyl24", "odd15", "flat2d", "conv12", "per12", "per16"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def problem_of(g, oracle):
    kind = int(g["kind"])
    kw = {k[4:]: (tuple(v.tolist()) if v.ndim else v.item()) for k, v in g.items() if k.startswith("arg_")}
    return oracle.Problem(kind, int(g["seed"]), **kw)


def bc_of(P):
    """Session boundary types of a fixture problem: None (the default walls
    with a Dirichlet top) unless some axis is periodic."""
    per = getattr(P, "periodic", 0)
    if not per:
        return None
    bc = [0] * 6
    bc[5 if P.nz > 1 else 3] = 1
    for d in range(3):
        if (per >> d) & 1:
            bc[2 * d] = bc[2 * d + 1] = 2
    return bc
