"""Pins the oracle build (oracle/_ref, the reference compiled from its sources with the project's FFT
substitute) against the reference's complete Fortran regression data, and records the result in
tests/golden/oracle_pin.json (committed).

For each golden case it runs the whole propagation (every analysis step of the input) with
`spo_ref_tool case <input> <out> --analysis-steps <all> --no-psi` and compares, as the reference's
gate 4 does (tests/regression_gate.hpp:19, tests/analysis_reference.hpp:556-580):
  - the BK coefficients of the kept analysis steps: max |C++ - Fortran| <= 1e-10 * scale;
  - the reaction probability per energy against the printed Fortran value (7 significant digits).
Takes minutes of CPU time; the tests check the committed record and re-run a short prefix.
"""

import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TOOL = os.path.join(ROOT, "oracle", "_ref", "spo_ref_tool")


def pin(case, work):
    d = os.path.join(HERE, case)
    cfg = json.load(open(os.path.join(d, "input.json")))
    n_analysis = int(round(cfg["nStep"] * cfg["dtStep"] / cfg["dtAna"]))
    out = os.path.join(work, case)
    t0 = time.time()
    subprocess.run([TOOL, "case", os.path.join(d, "input.json"), out, "--analysis-steps", str(n_analysis), "--no-psi"],
                   check=True, stdout=subprocess.DEVNULL)
    seconds = time.time() - t0
    ref = np.load(os.path.join(d, "bk_records.npy"))
    steps = np.load(os.path.join(d, "bk_steps.npy"))
    scale = float(np.load(os.path.join(d, "bk_scale.npy")))
    bk = np.fromfile(os.path.join(out, "bk_steps.c128"), dtype=np.complex128).reshape(n_analysis, -1)
    worst = float(np.max(np.abs(bk[steps] - ref)))
    p_ref = np.load(os.path.join(d, "p_reaction.npy"))
    p = np.fromfile(os.path.join(out, "p_reaction.f64"))
    p_dev = float(np.max(np.abs(p - p_ref)))
    return {"analysis_steps": n_analysis, "seconds": round(seconds, 1), "bk_worst_abs": worst, "bk_scale": scale,
            "bk_worst_over_scale": worst / scale, "bk_gate_1e-10": worst <= 1e-10 * scale,
            "p_reaction_max_abs_dev": p_dev, "p_reaction_within_print": p_dev <= 5e-7 * max(1.0, float(np.max(p_ref)))}


def main(work="/tmp/spo_pin"):
    os.makedirs(work, exist_ok=True)
    result = {}
    for case in ["hardwall_short", "cu111_dailight_short", "cu111_dailight_oblique"]:
        result[case] = pin(case, work)
        print(case, result[case], flush=True)
    result["threads"] = os.cpu_count()
    with open(os.path.join(HERE, "oracle_pin.json"), "w") as f:
        json.dump(result, f, indent=1)


if __name__ == "__main__":
    main(*sys.argv[1:])
