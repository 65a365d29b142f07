"""A run that scatters, through the drop-in, against the Fortran reference data and the reference CPU backend
(needs a B200).

cu111_dailight_small is the reference's regression case whose packet reaches the analysis line and scatters
(Dai-Light H2/Cu(111), tEnd 14000 au = 7000 steps, 41 analysis energies 0.2-0.6 eV; P_reaction ~ 1e-2, most
of the packet is reflected). oracle/_ref/spodvr_b200 is the reference program (its run_program, time loop, BK
analysis and S matrix) with the B200 backend. The FP64 form is checked against
  - the Fortran data: averages to half a unit of their printed 8th digit, the BK coefficients of every 50th
    analysis step to 1e-10 of their scale (the reference's gate 4), P_reaction to its printed digits;
  - the reference CPU backend on the same input (tests/golden/cu111_dailight_small/cpu_backend.npz, made by
    tests/golden/make_cpu_golden.py): P_reaction to 1e-9 at every energy, and the final wave packet (fort.9)
    to 1e-10 relative L2, estimated on 16384 fixed random entries.
The mixed form is run on the same input and its reaction and state-to-state probabilities are compared with
the FP64 run's: max |dP_reaction| and max |dP(v, j, mJ, n, m)| are printed and bounded.
"""

import json
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

PROGRAM = os.path.join(ROOT, "oracle", "_ref", "spodvr_b200")
CASE = "cu111_dailight_small"


def run(tmp_path, device):
    cfg = json.load(open(os.path.join(GOLDEN, CASE, "input.json")))
    cfg.update({"CheckpointFormat": "both", "writeSMatrix": True})
    work = tmp_path / device
    work.mkdir()
    (work / "input.json").write_text(json.dumps(cfg))
    out = work / "out"
    r = subprocess.run([PROGRAM, str(work / "input.json"), "--device", device, "--output-dir", str(out), "--no-color"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return out


def fortran_records(path):
    raw = open(path, "rb").read()
    out, i = [], 0
    while i < len(raw):
        n = int.from_bytes(raw[i:i + 4], "little", signed=True)
        out.append(raw[i + 4:i + 4 + n])
        i += n + 8
    return out


def tsv(path):
    rows = [ln.rstrip("\n").split("\t") for ln in open(path) if ln.strip() and not ln.startswith("#")]
    return rows[0], rows[1:]


def p_reaction(out):
    head, rows = tsv(out / "scattering_summary.tsv")
    return np.array([float(r[head.index("P_reaction")]) for r in rows])


def state_probabilities(out):
    head, rows = tsv(out / "s_matrix.tsv")
    keys = [tuple(r[head.index(k)] for k in ("E_coll", "v", "j", "mJ", "n", "m")) for r in rows]
    return dict(zip(keys, (float(r[head.index("P")]) for r in rows)))


def half_unit(v):
    if v == 0:
        return 5e-9
    return 0.5 * 10.0 ** (math.floor(math.log10(abs(v))) + 1 - 8) * 1.0001


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    assert os.path.exists(PROGRAM), "build the drop-in: make -C oracle (needs the product library)"
    base = tmp_path_factory.mktemp("scattering")
    return {"b200": run(base, "b200"), "b200-mixed": run(base, "b200-mixed")}


def test_fp64_meets_the_fortran_gates(runs):
    out = runs["b200"]
    ref_avg = np.load(os.path.join(GOLDEN, CASE, "averages.npy"))
    avg = np.array([[float(x) for x in ln.split()] for ln in open(out / "averages.dat") if not ln.startswith("#")])
    assert avg.shape == ref_avg.shape
    for a, f in zip(avg.ravel(), ref_avg.ravel()):
        assert abs(a - f) <= half_unit(f), (a, f)
    bk = np.array([np.frombuffer(r, dtype=np.complex128) for r in fortran_records(out / "fort.21")[10:]])
    ref = np.load(os.path.join(GOLDEN, CASE, "bk_records.npy"))
    steps = np.load(os.path.join(GOLDEN, CASE, "bk_steps.npy"))
    scale = float(np.load(os.path.join(GOLDEN, CASE, "bk_scale.npy")))
    worst = float(np.max(np.abs(bk[steps] - ref)))
    print(f"{CASE} FP64: BK max |B200 - Fortran| = {worst:.2e} (gate {1e-10 * scale:.2e})")
    assert worst <= 1e-10 * scale
    p, p_ref = p_reaction(out), np.load(os.path.join(GOLDEN, CASE, "p_reaction.npy"))
    assert np.max(np.abs(p - p_ref)) <= 5e-7


def test_fp64_matches_the_reference_cpu_backend(runs):
    out = runs["b200"]
    cpu = np.load(os.path.join(GOLDEN, CASE, "cpu_backend.npz"))
    dp = float(np.max(np.abs(p_reaction(out) - cpu["p_reaction"])))
    recs = [r for r in fortran_records(out / "fort.9") if len(r) >= 1024 and len(r) % 16 == 0]
    psi = np.concatenate([np.frombuffer(r, dtype=np.complex128) for r in recs])
    norm2 = float(np.vdot(psi, psi).real)
    sample = psi[cpu["psi_index"]]
    e_psi = float(np.linalg.norm(sample - cpu["psi_values"]) / np.linalg.norm(cpu["psi_values"]))
    print(f"{CASE} FP64 vs the reference CPU backend: max |dP_reaction| {dp:.2e}, psi rel-L2 (sampled) {e_psi:.2e}, "
          f"norm^2 {norm2:.12f} vs {float(cpu['psi_norm2']):.12f}")
    assert dp <= 1e-9
    assert e_psi <= 1e-10
    assert abs(norm2 - float(cpu["psi_norm2"])) <= 1e-10 * float(cpu["psi_norm2"])


# The mixed form's bound on this case: its measured error is 2.3e-6 in P_reaction and 2.2e-6 in the
# state-to-state probabilities (FP32 storage and arithmetic of the wave packet; every constant factor exact to
# ~2^-48, the theta contractions of this grid summed in FP64).
MIXED_DP_BOUND = 5e-6


def test_mixed_form_reaction_and_state_probabilities(runs):
    p64, p32 = p_reaction(runs["b200"]), p_reaction(runs["b200-mixed"])
    s64, s32 = state_probabilities(runs["b200"]), state_probabilities(runs["b200-mixed"])
    assert set(s64) == set(s32)
    dp = float(np.max(np.abs(p32 - p64)))
    ds = max(abs(s32[k] - s64[k]) for k in s64)
    print(f"{CASE} mixed vs FP64: max |dP_reaction| {dp:.3e}, max |dP(v,j,mJ,n,m)| {ds:.3e} over {len(s64)} channels")
    assert dp <= MIXED_DP_BOUND and ds <= MIXED_DP_BOUND
