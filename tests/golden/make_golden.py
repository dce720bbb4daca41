"""Generate the golden fixtures of the RD path from the reference itself.

Runs the reference's own operators (oracle/_ref/ref_harness_{f64,f32}, built
by ``make -C oracle ref`` from the reference sources) on seeded synthetic
inputs and stores, per case, the parameters, a SHA-256 of the exact inputs,
and the output: in full for small grids, else a SHA-256 of the exact output
bytes plus a strided subsample and summary statistics.

    python tests/golden/make_golden.py          # needs oracle/_ref
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gliomasolver_b200.anatomy import make_case  # noqa: E402
from gliomasolver_b200.schedule import make_schedule  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent

# name, n, seed, precision, Dw, rho, Tend, L, nsteps (None = the full schedule), mode
CASES = [
    ("rhs_n32_f64", 32, 1, "f64", 0.13, 0.025, 150.0, 25.6, 0, "rhs"),
    ("rhs_n32_f32", 32, 1, "f32", 0.13, 0.025, 150.0, 25.6, 0, "rhs"),
    ("steps_n32_f64", 32, 1, "f64", 0.13, 0.025, 150.0, 25.6, 50, "steps"),
    ("steps_n32_f32", 32, 1, "f32", 0.13, 0.025, 150.0, 25.6, 50, "steps"),
    ("steps_n16_f64_fast", 16, 3, "f64", 0.3, 0.2, 150.0, 25.6, 40, "steps"),
    # the parity configuration: 64^3 uniform, FP64, Dw=0.13, rho=0.025, T=150 d
    ("config1_n64_f64", 64, 0, "f64", 0.13, 0.025, 150.0, 25.6, None, "steps"),
]
FULL_OUTPUT_MAX_CELLS = 32 ** 3


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def make(case):
    name, n, seed, prec, Dw, rho, tend, L, nsteps, mode = case
    pw, pg, c0, x0 = make_case(n, seed)
    R = np.float64 if prec == "f64" else np.float32
    # the reference reads Real values: quantise the inputs first so the
    # fixture's inputs are exactly what both sides see
    pw, pg, c0 = (a.astype(R).astype(np.float64) for a in (pw, pg, c0))
    s = make_schedule(Dw, rho, tend, L, n // 8, prec)
    steps = s.nsteps if nsteps is None else nsteps
    if mode == "rhs":
        out = O.ref_rhs(pw, pg, c0, s.Dw, s.Dg, s.rho, prec)
    else:
        out = O.ref_uniform(pw, pg, c0, s.Dw, s.Dg, s.rho, s.dt, steps, prec)
    rec = dict(
        name=name, n=n, seed=seed, precision=prec, mode=mode, Dw_cm2_day=Dw, rho_day=rho, tend=tend, L=L,
        Dw=s.Dw, Dg=s.Dg, rho=s.rho, dt=s.dt, h=s.h, nsteps=steps, x0=x0,
        input_sha=sha(pw, pg, c0), output_sha=sha(out),
        out_sum=float(out.sum()), out_max=float(out.max()), out_l2=float(np.sqrt((out ** 2).sum())),
        out_sub=out[::4, ::4, ::4].copy(),
    )
    if out.size <= FULL_OUTPUT_MAX_CELLS:
        rec["out"] = out
    np.savez_compressed(OUT / f"{name}.npz", **rec)
    print(name, steps, rec["output_sha"][:16], rec["out_sum"])


if __name__ == "__main__":
    if not O.ref_available("f64") or not O.ref_available("f32"):
        sys.exit("oracle/_ref is not built: run `make -C oracle ref` where the reference sources are")
    only = set(sys.argv[1:])
    for c in CASES:
        if not only or c[0] in only:
            make(c)
