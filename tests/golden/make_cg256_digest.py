"""Digest of the compiled reference's CG solve of the 256^3 bubbles + cylinder
workload (32 bubbles of radius 4-16 cells, density ratio 1000, a solid
cylinder of radius 30 cells along z, seed 1).

Runs oracle/_ref/ref_harness (the unmodified reference library built from its
sources by oracle/build_ref.py): `CG(d, Prec::di())` through
`Centered::solve`, ResRat 1e-8, x0 = 0, one core. That takes about an hour.
The full solution (134 MB) is too large to commit, so this script stores a
digest of the run in tests/golden/cg256_digest.npz:

  * iterations, the final residual and ratio the reference logged, seconds;
  * sha256 of the matrix arrays c w e s n b t ci, of the right-hand side and
    of the solution (interior cells, float64 little-endian, k fastest: the
    engine's layout);
  * |x|_2, the means of x over the 4096 blocks of 16^3 cells, and 4096
    entries of x at seeded random cells (indices stored).

    python tests/golden/make_cg256_digest.py [--work DIR] [--n 256]

Test infrastructure only (the parity checker): tests/test_gpu_parity256.py
reads the digest.
"""
import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
WORKLOAD = dict(nb=32, rmin=4.0, rmax=16.0, rc=30.0, ratio=1000.0, seed=1)
SAMPLE_SEED = 20261203
NSAMPLE = 4096
BLOCK = 16


def digest_vector(x, n):
    """The digest fields of one solution vector (used by the tests too)."""
    x = np.ascontiguousarray(x, dtype="<f8")
    nb = n // BLOCK
    blocks = x.reshape(nb, BLOCK, nb, BLOCK, nb, BLOCK).mean(axis=(1, 3, 5)).ravel()
    idx = np.sort(np.random.default_rng(SAMPLE_SEED).choice(x.size, NSAMPLE, replace=False))
    return dict(sha_x=hashlib.sha256(x.tobytes()).hexdigest(), norm_x=float(np.linalg.norm(x)),
                block_means=blocks, sample_idx=idx.astype(np.int64), sample_x=x[idx].copy())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--work", default=None, help="directory for the harness's raw dumps")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--maxit", type=int, default=20000)
    a = ap.parse_args()
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(exe):
        raise SystemExit("build the reference harness first: python oracle/build_ref.py --ref <reference>")
    work = a.work or tempfile.mkdtemp(prefix="pbg_cg256_")
    os.makedirs(work, exist_ok=True)
    out = os.path.join(work, "cg%d" % a.n)
    w = WORKLOAD
    cmd = [exe, "--kind", "cyl", "--n", str(a.n), "--nb", str(w["nb"]), "--rmin", str(w["rmin"]),
           "--rmax", str(w["rmax"]), "--rc", str(w["rc"]), "--ratio", str(w["ratio"]),
           "--seed", str(w["seed"]), "--solver", "cg", "--resrat", "1e-8", "--maxit", str(a.maxit),
           "--out", out]
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise SystemExit("harness failed:\n" + r.stderr[-2000:])
    wall = time.time() - t0
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    run = json.loads(line)
    meta = {}
    for l in open(out + ".txt"):
        p = l.split()
        if len(p) >= 2:
            meta[p[0]] = p[1:]
    n = a.n
    N = n ** 3
    A = np.fromfile(out + ".A", dtype="<f8")
    assert A.size == 8 * N, A.size
    b = np.fromfile(out + ".b", dtype="<f8")
    x = np.fromfile(out + ".x", dtype="<f8")
    d = digest_vector(x, n)
    res = dict(n=np.array(n), iterations=np.array(int(meta["iterations"][0])),
               residual=np.array(float(meta["residual"][0])), ratio=np.array(float(meta["ratio"][0])),
               converged=np.array(int(meta["converged"][0])), seconds=np.array(float(run["seconds"])),
               wall=np.array(wall), sha_b=np.array(hashlib.sha256(b.tobytes()).hexdigest()),
               norm_b=np.array(float(np.linalg.norm(b))))
    for q, name in enumerate("c w e s n b t ci".split()):
        res["sha_A_" + name] = np.array(hashlib.sha256(A[q * N:(q + 1) * N].tobytes()).hexdigest())
    for k, v in w.items():
        res["arg_" + k] = np.array(v)
    for k, v in d.items():
        res[k] = np.array(v)
    path = os.path.join(HERE, "cg%d_digest.npz" % n)
    np.savez_compressed(path, **res)
    print(json.dumps({k: (v.item() if v.ndim == 0 else "array[%d]" % v.size) for k, v in res.items()}))
    print("wrote", path)


if __name__ == "__main__":
    sys.exit(main())
