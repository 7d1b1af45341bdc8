"""Checkpoints in the reference's .bck format (pbg_bck_*), checked against
files written by the compiled reference itself (Centered::save on the
solved pressure of the fixture harness): the name follows name_file, the
interior of phi is bit for bit the reference's solution, and writing the
blocks back reproduces the reference's file byte for byte. Host code only:
no GPU needed."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

CASES = [(["--kind", "single", "--n", "8"], (8, 8, 8)),
         (["--kind", "batch", "--index", "1", "--n2d", "2", "--s2", "10", "14", "--s3", "6", "8"], (13, 13, 1)),
         (["--kind", "cyl", "--n", "12", "--nb", "2", "--rmin", "2", "--rmax", "3", "--rc", "3"], (12, 12, 12))]


def reference_checkpoint(tmp, args):
    out = os.path.join(tmp, "r")
    base = os.path.join(tmp, "pres")
    subprocess.run([HARNESS] + args + ["--seed", "3", "--solver", "cg", "--resrat", "1e-8", "--save", base,
                                       "--out", out], check=True, capture_output=True)
    x = np.fromfile(out + ".x")
    return base, x


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference harness not built")
@pytest.mark.parametrize("args,dims", CASES)
def test_reads_and_rewrites_reference_checkpoint(tmp_path, args, dims):
    import psiboil_b200 as pb
    base, x = reference_checkpoint(str(tmp_path), args)
    path = pb.bck_name(base, 0, 0)
    assert os.path.basename(path) == "pres_p000_000000.bck" and os.path.exists(path)
    phi, cold = pb.bck_read(path, 2, dims)
    assert np.array_equal(phi, x)
    blocks = tuple(d + 2 * pb.BW for d in dims)
    full = pb.bck_read(path, 2, blocks, compact=False)
    again = str(tmp_path / "again.bck")
    pb.bck_write(again, full, blocks, compact=False)
    assert open(again, "rb").read() == open(path, "rb").read()


def test_compact_round_trip_and_checks(tmp_path):
    import psiboil_b200 as pb
    dims = (5, 7, 3)
    rng = np.random.default_rng(1)
    phi, cold = rng.standard_normal(105), rng.standard_normal(105)
    path = str(tmp_path / "c.bck")
    pb.bck_write(path, [phi, cold], dims)
    a, b = pb.bck_read(path, 2, dims)
    assert np.array_equal(a, phi) and np.array_equal(b, cold)
    # halo written as zero, extents stored per field
    raw = np.fromfile(path, dtype=np.uint8)
    assert raw.size == 2 * (12 + 8 * 11 * 13 * 9)
    full = pb.bck_read(path, 2, (11, 13, 9), compact=False)
    assert full[0].reshape(11, 13, 9)[3:8, 3:10, 3:6].ravel().tolist() == phi.tolist()
    assert np.count_nonzero(full[0]) == np.count_nonzero(phi)
    with pytest.raises(pb.PbgError):
        pb.bck_read(path, 2, (5, 7, 4))       # other extents
    with pytest.raises(pb.PbgError):
        pb.bck_read(path, 3, dims)            # file ends early
    with pytest.raises(pb.PbgError):
        pb.bck_read(str(tmp_path / "none.bck"), 1, dims)
    assert pb.bck_name("p", -1, -1) == "p.bck" and pb.bck_name("p", 12, 3) == "p_p003_000012.bck"
