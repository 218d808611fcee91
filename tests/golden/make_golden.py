"""Generate the golden fixtures of tests/golden/ from the reference's own CUDA
build (oracle/_ref/ref_harness, built by `make -C oracle ref` from the
reference's unmodified headers; it needs a GPU).

    python tests/golden/make_golden.py --run            # on a GPU box: run the driver, then convert
    python tests/golden/make_golden.py --dumps DIR      # convert QAFDUMP1 files already in DIR
    python tests/golden/make_golden.py --run --only couple64   # one group only

Workloads (all FP64, the reference as shipped; parameters of the friction
solver with Re = 1, Er = 1, Rf = 0.1, lambda = 0.1, Ra = 1, L = 16 pi unless
noted; seeded random Q ~ U(-0.01, 0.01), w = 0, generator include/qaf_init.h):
  nl_rand32 / nl_rand64  one nonlinear evaluation (curr_func + wnonl_func +
                         r1nonl_func + r2nonl_func), seeds 4 / 3
  run32                  IF-RK4 dt = 1e-3, seed 5, states at steps 0 1 2 10 20
  run64                  IF-RK4 dt = 1e-3, seed 0, state at step 100
  run128                 IF-RK4 dt = 1e-3, seed 0, state at step 1000
  couple64               the coupled runs' step (no dealias, couple.cu:179-215)
                         and parameters (Re = Er = 0.1, Rf = 7.5e-5, lambda =
                         0.1, Ra = 0.2, dt = 1e-3) from their smooth initial
                         state (qaf_couple_init, seed 9) on 64^2, L = 8 pi
                         (their grid spacing), states at steps 0 1 10 1000
  dealiasw64             the same with the step of dealias/couple.cu:226-229
                         (wnew truncated, r1 and r2 not), seed 11, states at
                         steps 0 1 10 200
  grid3                  3 * 2^k grids (radix-3 transforms; the reference's
                         drivers run 768 = 512 * 3 / 2): one nonlinear
                         evaluation at 96^2 and 192^2 (seeds 12 / 13) and
                         IF-RK4 dt = 1e-3 at 96^2 and 192^2 (seeds 14 / 15),
                         states at steps 0 1 20
  rect                   grids with nx != ny (Mesh(Nx, Ny, Lx, Ly), Mesh.cuh:61-73):
                         one nonlinear evaluation at 96 x 64 (Lx = 16 pi,
                         Ly = 32 pi / 3, the same spacing; seed 16) and IF-RK4
                         dt = 1e-3 at 64 x 128 (Lx = 16 pi, Ly = 32 pi; seed 17),
                         states at steps 0 1 20
  kat summary            the reference's nonlinear terms for the analytic input
                         sets of UnitTest/Nonlinear/nlterms0-4 (N = 128, L = 2 pi,
                         Re = Er = 0.1, Ra = 0.2), reduced to their deviation from
                         the closed forms
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
TWO_PI = "6.283185307179586"
EIGHT_PI = "25.132741228718345"
GROUPS = ("nl", "run32", "run64", "run128", "kat", "couple64", "dealiasw64", "grid3", "rect")
SIXTEEN_PI = "50.26548245743669"
THIRTYTWO_PI = "100.53096491487338"
THIRTYTWO_PI_3 = "33.510321638291124"
GRID3_STEPS = (0, 1, 20)
COUPLE_STEPS = (0, 1, 10, 1000)
DEALIASW_STEPS = (0, 1, 10, 200)


def run_harness(out, only=GROUPS):
    H = HARNESS
    jobs = {
        "nl": [[H, "nonlinear", "--n", "32", "--init", "random", "--seed", "4", "--out", f"{out}/nl_rand32"],
               [H, "nonlinear", "--n", "64", "--init", "random", "--seed", "3", "--out", f"{out}/nl_rand64"]],
        "run32": [[H, "run", "--n", "32", "--steps", "20", "--seed", "5", "--dumps", "0,1,2,10,20",
                   "--out", f"{out}/run32"]],
        "run64": [[H, "run", "--n", "64", "--steps", "100", "--seed", "0", "--dumps", "0,100", "--out", f"{out}/run64"]],
        "run128": [[H, "run", "--n", "128", "--steps", "1000", "--seed", "0", "--dumps", "0,1000",
                    "--out", f"{out}/run128"]],
        "kat": [[H, "nonlinear", "--n", "128", "--L", TWO_PI, "--init", f"kat{k}", "--re", "0.1", "--er", "0.1",
                 "--alpha", "0.2", "--lambda", "0.1", "--rf", "0.000075", "--out", f"{out}/nl_kat{k}"]
                for k in range(5)],
        "couple64": [[H, "run", "--n", "64", "--L", EIGHT_PI, "--init", "couple", "--seed", "9", "--re", "0.1",
                      "--er", "0.1", "--rf", "0.000075", "--lambda", "0.1", "--alpha", "0.2", "--dt", "0.001",
                      "--dealias", "0", "--steps", str(COUPLE_STEPS[-1]),
                      "--dumps", ",".join(str(s) for s in COUPLE_STEPS), "--out", f"{out}/couple64"]],
        "dealiasw64": [[H, "run", "--n", "64", "--L", EIGHT_PI, "--init", "couple", "--seed", "11", "--re", "0.1",
                        "--er", "0.1", "--rf", "0.000075", "--lambda", "0.1", "--alpha", "0.2", "--dt", "0.001",
                        "--dealias", "2", "--steps", str(DEALIASW_STEPS[-1]),
                        "--dumps", ",".join(str(s) for s in DEALIASW_STEPS), "--out", f"{out}/dealiasw64"]],
        "grid3": [[H, "nonlinear", "--n", "96", "--init", "random", "--seed", "12", "--out", f"{out}/nl_rand96"],
                  [H, "nonlinear", "--n", "192", "--init", "random", "--seed", "13", "--out", f"{out}/nl_rand192"],
                  [H, "run", "--n", "96", "--steps", "20", "--seed", "14", "--dumps",
                   ",".join(str(s) for s in GRID3_STEPS), "--out", f"{out}/run96"],
                  [H, "run", "--n", "192", "--steps", "20", "--seed", "15", "--dumps",
                   ",".join(str(s) for s in GRID3_STEPS), "--out", f"{out}/run192"]],
        "rect": [[H, "nonlinear", "--n", "96", "--ny", "64", "--L", SIXTEEN_PI, "--Ly", THIRTYTWO_PI_3, "--init",
                  "random", "--seed", "16", "--out", f"{out}/nl_rect96x64"],
                 [H, "run", "--n", "64", "--ny", "128", "--L", SIXTEEN_PI, "--Ly", THIRTYTWO_PI, "--steps", "20",
                  "--seed", "17", "--dumps", ",".join(str(s) for s in GRID3_STEPS), "--out", f"{out}/run64x128"]],
    }
    for name in only:
        for c in jobs[name]:
            subprocess.run(c, check=True)


def kat_fields(k, n=128, L=2 * np.pi):
    """Closed-form inputs and nonlinear terms of UnitTest/Nonlinear/nlterms{k}.cu:46-94."""
    x = np.arange(n) * L / n
    X, Y = np.meshgrid(x, x)
    s, c = np.sin, np.cos
    if k == 0:
        return (-2 * s(X + Y), s(X), c(X), -60 * c(X),
                -4 * s(X) + 0.2 * s(X + Y) + c(X) * (c(X + Y) + 2 * s(X + Y)),
                -4 * c(X) - s(X) * (c(X + Y) + 2 * s(X + Y)))
    if k == 1:
        return (-2 * s(X + Y), c(X + Y), s(X + Y), 160 * c(X + Y),
                1 - 4 * c(X + Y) - c(2 * (X + Y)) + 0.2 * s(X + Y), s(X + Y) * (-4 - 2 * c(X + Y)))
    if k == 2:
        return (-5 * s(2 * X + Y), c(X + Y), s(X + Y), 160 * c(X + Y),
                -4 * c(X) * c(Y) + 4 * s(X) * s(Y) + c(2 * X + Y) * s(X + Y) + 0.4 * s(2 * X + Y)
                + 5 * s(X + Y) * s(2 * X + Y),
                -4 * c(Y) * s(X) - 4 * c(X) * s(Y) - 0.3 * s(2 * X + Y) - c(X + Y) * (c(2 * X + Y) + 5 * s(2 * X + Y)))
    if k == 3:
        return (-298 * s(17 * X + 3 * Y), c(5 * X + Y), s(5 * X + Y), 5600 * c(5 * X + Y) - 13440 * s(5 * X + Y),
                -4 * c(5 * X + Y) + 2 * c(17 * X + 3 * Y) * s(5 * X + Y) + 298 * (0.0342282 + s(5 * X + Y))
                * s(17 * X + 3 * Y),
                -4 * s(5 * X + Y) - 28 * s(17 * X + 3 * Y) - 2 * c(5 * X + Y) * (c(17 * X + 3 * Y) + 149 * s(17 * X + 3 * Y)))
    return (-13 * s(2 * X + 3 * Y), c(3 * X + 2 * Y), s(3 * X + 2 * Y), 3600 * c(3 * X + 2 * Y) - 1500 * s(3 * X + 2 * Y),
            6.5 * c(X - Y) - 6.5 * c(5 * (X + Y)) - 4.0 * c(3 * X + 2 * Y) - 2.5 * s(X - Y) - 2.5 * s(5 * (X + Y))
            + 1.2 * s(2 * X + 3 * Y),
            2.5 * c(X - Y) + 2.5 * c(5 * (X + Y)) + 6.5 * s(X - Y) - 6.5 * s(5 * (X + Y)) - 4.0 * s(3 * X + 2 * Y)
            + 0.5 * s(2 * X + 3 * Y))


def convert(d, only=GROUPS):
    def f(name):
        return O.read_dump(os.path.join(d, name))["fields"]

    def save(name, **arrs):
        np.savez_compressed(os.path.join(HERE, name), **arrs)

    def states(prefix, steps):
        arrs = {}
        for s in steps:
            st = f(f"{prefix}_s{s}.bin")
            arrs.update({f"w_{s}": st[0], f"r1_{s}": st[1], f"r2_{s}": st[2]})
        return arrs

    if "nl" in only:
        for n in (32, 64):
            i, nl = f(f"nl_rand{n}_in.bin"), f(f"nl_rand{n}_nl.bin")
            save(f"ref_nl_rand{n}.npz", w=i[0], r1=i[1], r2=i[2], wn=nl[0], r1n=nl[1], r2n=nl[2])
    if "run32" in only:
        save("ref_run32.npz", **states("run32", (0, 1, 2, 10, 20)))
    if "run64" in only:
        st = f("run64_s100.bin")
        save("ref_run64_s100.npz", w=st[0], r1=st[1], r2=st[2])
    if "run128" in only:
        st = f("run128_s1000.bin")
        save("ref_run128_s1000.npz", w=st[0], r1=st[1], r2=st[2])
    if "couple64" in only:
        save("ref_couple64.npz", **states("couple64", COUPLE_STEPS))
    if "dealiasw64" in only:
        save("ref_dealiasw64.npz", **states("dealiasw64", DEALIASW_STEPS))
    if "rect" in only:
        i, nl = f("nl_rect96x64_in.bin"), f("nl_rect96x64_nl.bin")
        save("ref_nl_rect96x64.npz", w=i[0], r1=i[1], r2=i[2], wn=nl[0], r1n=nl[1], r2n=nl[2])
        save("ref_run64x128.npz", **states("run64x128", GRID3_STEPS))
    if "grid3" in only:
        for n in (96, 192):
            i, nl = f(f"nl_rand{n}_in.bin"), f(f"nl_rand{n}_nl.bin")
            save(f"ref_nl_rand{n}.npz", w=i[0], r1=i[1], r2=i[2], wn=nl[0], r1n=nl[1], r2n=nl[2])
            save(f"ref_run{n}.npz", **states(f"run{n}", GRID3_STEPS))
    if "kat" not in only:
        return
    summary = {}
    for k in range(5):
        fields = kat_fields(k)
        nl = f(f"nl_kat{k}_nl.bin")
        dev = []
        for a, ex in zip(nl, fields[3:]):
            ph = O.bwd(a)
            dev.append(float(np.abs(ph - ex).max() / np.abs(ex).max()))
        summary[f"kat{k}"] = {"max_rel_dev_from_closed_form": dev}
    with open(os.path.join(HERE, "ref_kat_summary.json"), "w") as fh:
        json.dump(summary, fh, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--run", action="store_true")
    ap.add_argument("--dumps")
    ap.add_argument("--only", default=",".join(GROUPS), help="comma-separated groups of " + ", ".join(GROUPS))
    a = ap.parse_args()
    only = tuple(a.only.split(","))
    if any(g not in GROUPS for g in only):
        ap.error("unknown group in --only")
    if a.run:
        with tempfile.TemporaryDirectory() as d:
            run_harness(d, only)
            convert(d, only)
    elif a.dumps:
        convert(a.dumps, only)
    else:
        ap.error("give --run or --dumps DIR")


if __name__ == "__main__":
    main()
