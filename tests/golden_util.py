"""Loading of the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["single16", "single12", "cyl24", "odd15", "flat2d", "conv12"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def problem_of(g, oracle):
    kind = int(g["kind"])
    kw = {k[4:]: (tuple(v.tolist()) if v.ndim else v.item()) for k, v in g.items() if k.startswith("arg_")}
    return oracle.Problem(kind, int(g["seed"]), **kw)
