"""The precision form's error in the reaction and state-to-state probabilities: configuration 3 against 2.

Runs the configuration-2 input (tests/golden/inputs/config2_dz.json: Dai-Light PES, nZ 128, nR 48, nX = nY 16,
theta 16 x phi 32, nZSpecular 512, dt 2, 20000 steps = 40000 au, 81 analysis energies 0.2-1.0 eV) through the
reference program with the B200 backend (oracle/_ref/spodvr_b200), once in the FP64 form (configuration 2,
--device b200) and once in the mixed form (configuration 3, --device b200-mixed). The time loop, the BK
analysis at the analysis line and the S matrix are the reference's own (src/app/run.cpp,
src/analysis/s_matrix.cpp:118-176), so both runs differ only in the backend's arithmetic.

Writes tests/golden/precision_config3.json (or the path given as the first argument):
  p_reaction_fp64 / p_reaction_mixed   P_reaction per energy (scattering_summary.tsv)
  dp_reaction_max                      max over energies of |P_reaction(mixed) - P_reaction(FP64)|
  dp_state_max                         max over energies and open (v, j, mJ, n, m) channels of |P(mixed) - P(FP64)|
  p_state_max                          the largest state-to-state probability (for scale)
  seconds_fp64 / seconds_mixed         wall time of each program run (set-up on the host included)
bench.py copies dp_reaction_max and dp_state_max into its line.

  python tests/golden/precision_config3.py [OUT.json] [--steps N]
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROGRAM = os.path.join(ROOT, "oracle", "_ref", "spodvr_b200")
INPUT = os.path.join(HERE, "inputs", "config2_dz.json")


def read_tsv(path):
    rows = [ln.rstrip("\n").split("\t") for ln in open(path) if ln.strip() and not ln.startswith("#")]
    head = rows[0]
    return head, rows[1:]


def run(device, work, steps):
    cfg = json.load(open(INPUT))
    if steps:
        cfg.update({"nStep": steps, "tEnd": cfg["tStart"] + steps * cfg["dtStep"]})
    cfg.update({"writeSMatrix": True, "writeProbs": True})
    os.makedirs(work, exist_ok=True)
    path = os.path.join(work, "input.json")
    json.dump(cfg, open(path, "w"))
    out = os.path.join(work, "out")
    t0 = time.time()
    r = subprocess.run([PROGRAM, path, "--device", device, "--output-dir", out, "--no-color"], capture_output=True,
                       text=True)
    seconds = time.time() - t0
    if r.returncode != 0:
        sys.exit(f"{device}: exit {r.returncode}\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
    head, rows = read_tsv(os.path.join(out, "scattering_summary.tsv"))
    e = np.array([float(x[head.index("E_coll")]) for x in rows])
    p = np.array([float(x[head.index("P_reaction")]) for x in rows])
    shead, srows = read_tsv(os.path.join(out, "s_matrix.tsv"))
    keys = [tuple(x[shead.index(k)] for k in ("E_coll", "v", "j", "mJ", "n", "m")) for x in srows]
    ps = {k: float(x[shead.index("P")]) for k, x in zip(keys, srows)}
    return e, p, ps, seconds, cfg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out", nargs="?", default=os.path.join(HERE, "precision_config3.json"))
    ap.add_argument("--steps", type=int, default=0, help="time steps (default: the input's 20000)")
    ap.add_argument("--work", default=None)
    args = ap.parse_args()
    work = args.work or tempfile.mkdtemp(prefix="precision_config3_")
    e64, p64, s64, t64, cfg = run("b200", os.path.join(work, "fp64"), args.steps)
    e32, p32, s32, t32, _ = run("b200-mixed", os.path.join(work, "mixed"), args.steps)
    assert np.array_equal(e64, e32) and set(s64) == set(s32)
    dp = np.abs(p32 - p64)
    ds = {k: abs(s32[k] - s64[k]) for k in s64}
    worst = max(ds, key=ds.get)
    rec = {
        "input": "tests/golden/inputs/config2_dz.json",
        "time_steps": cfg["nStep"], "t_end_au": cfg["tEnd"], "energies": len(e64),
        "e_coll_ev": e64.tolist(),
        "p_reaction_fp64": p64.tolist(), "p_reaction_mixed": p32.tolist(),
        "dp_reaction_max": float(dp.max()), "dp_reaction_argmax_e_coll_ev": float(e64[int(dp.argmax())]),
        "p_scattered_range_fp64": [float((1 - p64).min()), float((1 - p64).max())],
        "open_channels": len(s64), "dp_state_max": float(ds[worst]),
        "dp_state_argmax": dict(zip(("E_coll", "v", "j", "mJ", "n", "m"), worst)),
        "p_state_max": float(max(s64.values())),
        "seconds_fp64": t64, "seconds_mixed": t32,
        "program": "oracle/_ref/spodvr_b200 (the reference's run_program with the B200 backend)",
    }
    with open(args.out, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps({k: v for k, v in rec.items() if not isinstance(v, list)}))


if __name__ == "__main__":
    main()
