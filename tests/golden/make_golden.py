"""Generate the golden fixtures from the compiled reference (PSI-BOIL).

Runs oracle/_ref/ref_harness (the unmodified reference library built from
its sources by oracle/build_ref.py, driven by the fixture harness) on small
seeded problems and stores its matrix, right-hand side, solutions,
iteration/cycle counts and residual histories under tests/golden/*.npz.
Only needed where the reference sources exist; the fixtures are committed.

    python tests/golden/make_golden.py            (everything)
    python tests/golden/make_golden.py --steps    (the step fixtures only)
    python tests/golden/make_golden.py NAME ...   (those solver fixtures only)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as O  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
from golden_util import ACX_RUNS  # noqa: E402

CASES = [
    # name, kind, problem kwargs, runs
    ("single16", O.KIND_SINGLE, dict(n=16), ["cg", "bicgs", "ac", "cg_ic0", "cg_ic2", "cg_ic3", "cgs",
                                             "bicgs_ic2", "cgs_ic0"]),
    ("single12", O.KIND_SINGLE, dict(n=12), ["cg", "ac_w", "ac_f", "ac_noguard", "jacobi", "gs",
                                             "acsm_gs", "acsm_bicgs", "acsm_cgs", "acsm_cg-ic0"]),
    ("cyl24", O.KIND_CYL, dict(n=24, nb=3, rmin=2.0, rmax=4.0, rc=5.0), ["cg", "ac", "cg_ic2", "jacobi",
                                                                          "gs", "acsm_gs", "acsm_jacobi"]),
    ("odd15", O.KIND_BATCH, dict(index=40, n2d=0, s3=(15, 16)), ["cg", "ac", "jacobi", "gs",
                                                                 "acsm_bicgs"]),
    ("flat2d", O.KIND_BATCH, dict(index=1, n2d=8, s2=(24, 40)), ["cg", "bicgs", "ac", "jacobi", "gs"]),
    # non-symmetric: upwind convection along +x added to the fixture
    ("conv12", O.KIND_SINGLE, dict(n=12, convect=2e-5), ["bicgs", "cgs", "bicgs_ic0", "bicgs_ic2",
                                                        "cgs_ic2", "cgs_ic3", "jacobi", "gs"]),
    # periodic boundaries (Periodic::yes grids, BndType::periodic): x and y
    # periodic around the cylinder case; x periodic on the single bubble
    ("per12", O.KIND_CYL, dict(n=12, nb=2, rmin=1.5, rmax=2.5, rc=3.0, periodic=3),
     ["cg", "bicgs", "ac", "jacobi", "gs", "cg_ic2", "acsm_gs", "ac_w"]),
    ("per16", O.KIND_SINGLE, dict(n=16, periodic=1), ["cg", "cgs", "ac", "gs", "acsm_jacobi"]),
    # the rest of AC's surface: flex cycle, "just solve", use_linf_error, a
    # full-cycle start, AC's own solver, min_cycles (golden_util.ACX_RUNS)
    ("acx12", O.KIND_SINGLE, dict(n=12), ["cg"] + sorted(ACX_RUNS)),
]

# Jacobi and Gauss-Seidel converge slowly on these density jumps: a looser
# ratio and an iteration cap (most runs stop at the cap, which pins the
# arithmetic of every sweep all the same)
STATIONARY = dict(resrat=1e-2, maxit=2000)


# pressure-correction steps (ref_harness --step 1): the reference's own
# Pressure::discretize of a two-phase Matter, update_rhs, CG and
# Momentum::project on the flow state of pbg_gen_flow
STEP_CASES = [
    # name, kind, problem kwargs, dt
    ("step8", O.KIND_SINGLE, dict(n=8), 0.003),
    ("step2d", O.KIND_BATCH, dict(index=0, n2d=1, s2=(32, 32)), 0.01),
    ("step12", O.KIND_SINGLE, dict(n=12), 1.0),
]
# the same with an immersed body: a sphere of 4.3 cells written as an STL
# and cut by the reference's own Body (fV, fS stored with the fixture)
BODY_STEP_CASES = [
    # name, kind, problem kwargs, dt, sphere radius in cells
    ("stepbody16", O.KIND_SINGLE, dict(n=16), 0.01, 4.3),
    ("stepbody32", O.KIND_SINGLE, dict(n=32), 0.003, 9.7),
]


def make_steps():
    import flow
    for name, kind, kw, dt in STEP_CASES:
        P = O.Problem(kind, 7, **kw)
        r = flow.run_reference_step(P, dt, res_rat=1e-10)
        out = dict(dims=np.array(P.dims), h=np.array(P.h), kind=np.array(kind), seed=np.array(7),
                   dt=np.array(dt), res_rat=np.array(1e-10),
                   iterations=np.array(r["meta"]["iterations"]))
        for k, v in kw.items():
            out["arg_" + k] = np.array(v)
        for k in "cwsb":
            out["A_" + k] = r["A"][k]
        out["rhs"] = r["b"]
        for k in "xuvw":
            out[k] = r[k]
        print(name, P.dims, dt, r["meta"]["iterations"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    for name, kind, kw, dt, radius in BODY_STEP_CASES:
        P = O.Problem(kind, 7, **kw)
        r = flow.run_reference_step(P, dt, res_rat=1e-10, body=radius)
        out = dict(dims=np.array(P.dims), h=np.array(P.h), kind=np.array(kind), seed=np.array(7),
                   dt=np.array(dt), res_rat=np.array(1e-10), body_radius=np.array(radius),
                   iterations=np.array(r["meta"]["iterations"]),
                   fV=r["body"]["fV"], fS=r["body"]["fS"])
        for k, v in kw.items():
            out["arg_" + k] = np.array(v)
        for k in "cwesnbt":
            out["A_" + k] = r["A"][k]
        out["ci"] = r["ci"]
        out["rhs"] = r["b"]
        for k in "xuvw":
            out[k] = r[k]
        print(name, P.dims, dt, radius, r["meta"]["iterations"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def main():
    O.build()
    if not O.harness_available():
        raise SystemExit("oracle/_ref/ref_harness missing: run python oracle/build_ref.py")
    only = [a for a in sys.argv[1:] if not a.startswith("--")]
    for name, kind, kw, runs in CASES:
        if only and name not in only:
            continue
        P = O.Problem(kind, 7, **kw)
        out = dict(dims=np.array(P.dims), h=np.array(P.h), kind=np.array(kind), seed=np.array(7))
        for k, v in kw.items():
            out["arg_" + k] = np.array(v)
        for run in runs:
            solver = "ac" if run.startswith("ac") else run.split("_")[0]
            extra = {}
            if run in ACX_RUNS:
                extra = dict(ACX_RUNS[run][0])
            if "_ic" in run:
                extra = dict(prec=run.split("_")[1])
            if run == "ac_w":
                extra = dict(cycle="W")
            elif run == "ac_f":
                extra = dict(cycle="F")
            elif run == "ac_noguard":
                extra = dict(guard=0, maxcyc=6)
            elif run.startswith("acsm_"):  # AC with the Pressure's solver of that kind
                # "acsm_<solver>" or "acsm_<solver>-<preconditioner>"
                sm, _, pr = run.split("_")[1].partition("-")
                extra = dict(acsm=sm)
                if pr:
                    extra["prec"] = pr
            kw_run = dict(resrat=1e-8)
            if solver in ("jacobi", "gs"):
                kw_run = dict(STATIONARY)
                out[run + "_resrat"] = np.array(kw_run["resrat"])
                out[run + "_maxit"] = np.array(kw_run["maxit"])
            meta, arr = O.run_reference(P, solver, **kw_run, **extra)
            if "A" not in out:
                for k in "cwesnbt":
                    out["A_" + k] = arr["A"][k]
                out["ci"] = arr["ci"]
                out["b"] = arr["b"]
            out[run + "_x"] = arr["x"]
            out[run + "_iterations"] = np.array(meta["iterations"])
            out[run + "_converged"] = np.array(meta["converged"])
            out[run + "_cycles"] = np.array(meta["cycles"])
            if solver == "ac":
                out[run + "_hist"] = np.array([meta["res0"]] + meta["cycle_res"])
            print(name, run, P.dims, {k: meta[k] for k in ("iterations", "cycles", "converged")})
            out["A"] = True
        del out["A"]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    if not only:
        make_steps()


if __name__ == "__main__":
    if sys.argv[1:] == ["--steps"]:
        O.build()
        make_steps()
    else:
        main()
