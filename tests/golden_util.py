"""Loading of the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["single16", "single12", "cyl24", "odd15", "flat2d", "conv12", "per12", "per16", "acx12"]

# AC runs beyond the default V/F/W loops (fixture acx12): the reference
# harness's arguments, the oracle AC's constructor arguments and the cycle's
# arguments (loop/init codes 1 V, 2 F, 4 W, 5 flex, -1 none = "just solve").
ACX_RUNS = {
    "acx_flex": (dict(cycle="flex", acresrat=0.1), dict(resrat=0.1), dict(loop=5)),
    "acx_solve": (dict(cycle="none"), {}, dict(loop=-1)),
    "acx_linf": (dict(cycle="V", linf=1), dict(use_linf=True), dict(loop=1)),
    "acx_linfw": (dict(cycle="W", linf=1), dict(use_linf=True), dict(loop=4)),
    "acx_fullv": (dict(cycle="V", init="V"), {}, dict(loop=1, init=1)),
    "acx_fullf": (dict(cycle="F", init="F"), {}, dict(loop=2, init=2)),
    "acx_fullflex": (dict(cycle="flex", init="V", acresrat=0.1), dict(resrat=0.1), dict(loop=5, init=1)),
    "acx_solgs": (dict(cycle="V", acsolver="gs"), dict(solver="gs"), dict(loop=1)),
    "acx_solbicgs": (dict(cycle="V", acsolver="bicgs"), dict(solver="bicgs"), dict(loop=1)),
    "acx_mincyc": (dict(cycle="V", mincyc=6), {}, dict(loop=1, min_cyc=6)),
}


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
