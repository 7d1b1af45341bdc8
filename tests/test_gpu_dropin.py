"""Drop-in through the reference's own Krylov virtual.

oracle/_ref/ref_harness_gpu is the reference harness built with
include/psiboil_b200_psiboil.hpp: `new pbg_psiboil::GpuCG(d, Prec::di())`
replaces `new CG(d, Prec::di())`, so the reference's Centered::solve and the
reference's own AC multigrid (its cycle logic, restriction, coarse
operators on the CPU) call the engine's GPU CG through Linear::solve. With
exact-order sums the results equal the reference's own, bit for bit.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from golden_util import load

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_harness_gpu")


def run(args):
    out = os.path.join(tempfile.mkdtemp(prefix="pbg_dropin_"), "r")
    subprocess.run([EXE] + args + ["--out", out], check=True, capture_output=True, timeout=600)
    x = np.fromfile(out + ".x", dtype=np.float64)
    meta = {}
    for line in open(out + ".txt"):
        p = line.split()
        if len(p) >= 2:
            meta[p[0]] = p[1:]
    return x, meta


@pytest.mark.skipif(not os.path.exists(EXE), reason="GPU-backed reference harness not built")
@pytest.mark.parametrize("solver,key", [("cg", "cg"), ("bicgs", "bicgs"), ("ac", "ac")])
def test_reference_with_gpu_krylov_is_bit_exact(solver, key):
    g = load("single16")
    x, meta = run(["--kind", "single", "--n", "16", "--seed", "7", "--solver", solver,
                   "--resrat", "1e-8", "--gpu", "1", "--exact", "1"])
    assert np.array_equal(x, g[key + "_x"])
    if solver == "ac":
        assert int(meta["cycles"][0]) == int(g["ac_cycles"])
    else:
        assert int(meta["iterations"][0]) == int(g[key + "_iterations"])


@pytest.mark.skipif(not os.path.exists(EXE), reason="GPU-backed reference harness not built")
def test_reference_ac_with_gpu_krylov_tree_sums():
    g = load("cyl24")
    x, meta = run(["--kind", "cyl", "--n", "24", "--nb", "3", "--rmin", "2.0", "--rmax", "4.0",
                   "--rc", "5.0", "--seed", "7", "--solver", "ac", "--resrat", "1e-8",
                   "--gpu", "1", "--exact", "0"])
    assert abs(int(meta["cycles"][0]) - int(g["ac_cycles"])) <= 2
    assert np.abs(x - g["ac_x"]).max() <= 1e-8 * np.abs(g["ac_x"]).max()


@pytest.mark.skipif(not os.path.exists(EXE), reason="GPU-backed reference harness not built")
@pytest.mark.parametrize("case,args,prec", [
    ("single16", ["--kind", "single", "--n", "16"], "ic0"),
    ("single16", ["--kind", "single", "--n", "16"], "ic2"),
    ("single16", ["--kind", "single", "--n", "16"], "ic3"),
    ("cyl24", ["--kind", "cyl", "--n", "24", "--nb", "3", "--rmin", "2.0", "--rmax", "4.0", "--rc", "5.0"], "ic2")])
def test_reference_with_gpu_ic_cg_is_bit_exact(case, args, prec):
    """`new GpuCG(d, Prec::ic2())` in place of `new CG(d, Prec::ic2())`: the
    reference's pressure solve gives the CPU reference's solution and
    iteration count bit for bit (golden fixtures from the CPU reference)."""
    g = load(case)
    x, meta = run(args + ["--seed", "7", "--solver", "cg", "--prec", prec, "--resrat", "1e-8",
                          "--gpu", "1", "--exact", "1"])
    assert np.array_equal(x, g["cg_" + prec + "_x"])
    assert int(meta["iterations"][0]) == int(g["cg_" + prec + "_iterations"])


@pytest.mark.skipif(not os.path.exists(EXE), reason="GPU-backed reference harness not built")
@pytest.mark.parametrize("case,args,key", [
    ("single16", ["--kind", "single", "--n", "16"], "cgs"),
    ("single16", ["--kind", "single", "--n", "16"], "bicgs_ic2"),
    ("single16", ["--kind", "single", "--n", "16"], "cgs_ic0"),
    ("conv12", ["--kind", "single", "--n", "12", "--convect", "2e-05"], "bicgs_ic0"),
    ("conv12", ["--kind", "single", "--n", "12", "--convect", "2e-05"], "cgs"),
    ("conv12", ["--kind", "single", "--n", "12", "--convect", "2e-05"], "cgs_ic3")])
def test_reference_with_gpu_bicgs_cgs_is_bit_exact(case, args, key):
    """`new GpuCGS(d, pc)` / `new GpuBiCGS(d, pc)` in place of the reference's
    CGS / BiCGS, on the pressure fixture and on its convected (non-symmetric)
    variant: the CPU reference's solution and iteration count bit for bit."""
    g = load(case)
    parts = key.split("_")
    prec = parts[1] if len(parts) > 1 else "di"
    x, meta = run(args + ["--seed", "7", "--solver", parts[0], "--prec", prec, "--resrat", "1e-8",
                          "--gpu", "1", "--exact", "1"])
    assert np.array_equal(x, g[key + "_x"])
    assert int(meta["iterations"][0]) == int(g[key + "_iterations"])


@pytest.mark.skipif(not os.path.exists(EXE), reason="GPU-backed reference harness not built")
@pytest.mark.parametrize("case,args", [
    ("cyl24", ["--kind", "cyl", "--n", "24", "--nb", "3", "--rmin", "2.0", "--rmax", "4.0", "--rc", "5.0"]),
    ("odd15", ["--kind", "batch", "--index", "40", "--n2d", "0", "--s3", "15", "16"])])
@pytest.mark.parametrize("solver", ["jacobi", "gs"])
def test_reference_with_gpu_stationary_is_bit_exact(case, args, solver):
    """`new GpuGaussSeidel(d)` / `new GpuJacobi(d)` in place of the reference's
    GaussSeidel / Jacobi behind Centered::solve; A.ci goes up with the matrix."""
    g = load(case)
    x, meta = run(args + ["--seed", "7", "--solver", solver, "--resrat", "0.01", "--maxit", "2000",
                          "--gpu", "1", "--exact", "1"])
    assert np.array_equal(x, g[solver + "_x"])
    assert int(meta["iterations"][0]) == int(g[solver + "_iterations"])


def _hist(meta):
    return np.array([float(meta["res0"][0])] + [float(v) for v in meta.get("cycle_res", [])])


GPUAC_CASES = [
    # golden fixture, harness problem args, harness AC args, golden run key
    ("single16", ["--kind", "single", "--n", "16"], [], "ac"),
    ("single12", ["--kind", "single", "--n", "12"], ["--cycle", "W"], "ac_w"),
    ("single12", ["--kind", "single", "--n", "12"], ["--guard", "0", "--maxcyc", "6"], "ac_noguard"),
    ("single12", ["--kind", "single", "--n", "12"], ["--acsm", "gs"], "acsm_gs"),
    ("cyl24", ["--kind", "cyl", "--n", "24", "--nb", "3", "--rmin", "2.0", "--rmax", "4.0", "--rc", "5.0"],
     [], "ac"),
    ("per12", ["--kind", "cyl", "--n", "12", "--nb", "2", "--rmin", "1.5", "--rmax", "2.5", "--rc", "3.0",
               "--periodic", "3"], [], "ac"),
    ("acx12", ["--kind", "single", "--n", "12"], ["--cycle", "flex", "--acresrat", "0.1"], "acx_flex"),
    ("acx12", ["--kind", "single", "--n", "12"], ["--cycle", "none"], "acx_solve"),
    ("acx12", ["--kind", "single", "--n", "12"], ["--linf", "1"], "acx_linf"),
    ("acx12", ["--kind", "single", "--n", "12"], ["--init", "V"], "acx_fullv"),
    ("acx12", ["--kind", "single", "--n", "12"], ["--acsolver", "bicgs"], "acx_solbicgs"),
]


@pytest.mark.skipif(not os.path.exists(EXE), reason="GPU-backed reference harness not built")
@pytest.mark.parametrize("case,args,acargs,key", GPUAC_CASES, ids=[c[0] + "-" + c[3] for c in GPUAC_CASES])
def test_reference_with_gpu_ac_is_bit_exact(case, args, acargs, key):
    """`pbg_psiboil::GpuAC multigrid(&pr)` in place of `AC multigrid(&pr)`
    (--gpu 2): the whole cycle on the GPU behind AC's own interface. With
    exact sums the cycle count, the residual history the harness parses from
    the log lines and the iterate are the CPU reference's, bit for bit."""
    g = load(case)
    x, meta = run(args + ["--seed", "7", "--solver", "ac", "--resrat", "1e-8", "--gpu", "2",
                          "--exact", "1"] + acargs)
    assert int(meta["cycles"][0]) == int(g[key + "_cycles"])
    assert int(meta["converged"][0]) == int(g[key + "_converged"])
    np.testing.assert_allclose(_hist(meta), g[key + "_hist"], rtol=1e-13)
    assert np.array_equal(x, g[key + "_x"])
