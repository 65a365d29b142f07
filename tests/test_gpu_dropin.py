"""The drop-in: the reference's own program (its run_program, time loop, BK analysis and S-matrix)
with the B200 backend in place of its CPU backend, on the reference's regression cases, against the
Fortran reference data (needs a B200).

oracle/_ref/spodvr_b200 is the reference program linked with the package's PropagationBackend
adapter (cpp-spo-dvr_b200/adapter/). For each case it runs the complete propagation and checks the
reference's gates 3 and 4 (tests/regression_gate.hpp of the reference):
  - averages (norm, <Z>, <r>, rest norm): to half a unit of the printed 8th digit;
  - BK coefficients of every kept analysis step: max |B200 - Fortran| <= 1e-10 * scale;
  - reaction probability per energy: to the 7 printed digits.
The mixed form (complex64 psi, FP32 FFTs) must keep |dP_reaction| <= 1e-6 against the FP64 form.
"""

import json
import math
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

PROGRAM = os.path.join(ROOT, "oracle", "_ref", "spodvr_b200")


def run_case(case, tmp_path, device="b200", extra=None):
    cfg = json.load(open(os.path.join(GOLDEN, case, "input.json")))
    cfg["CheckpointFormat"] = "both"  # also writes fort.21, the Fortran BK file
    if extra:
        cfg.update(extra)
    work = tmp_path / f"{case}_{device}"
    work.mkdir()
    path = work / "input.json"
    path.write_text(json.dumps(cfg))
    r = subprocess.run([PROGRAM, str(path), "--device", device, "--output-dir", str(work / "out"), "--no-color"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return work / "out"


def fortran_records(path):
    raw = open(path, "rb").read()
    out, i = [], 0
    while i < len(raw):
        n = struct.unpack("<i", raw[i:i + 4])[0]
        out.append(raw[i + 4:i + 4 + n])
        i += n + 8
    return out


def p_reaction(out):
    rows = [ln.split("\t") for ln in open(out / "scattering_summary.tsv") if ln.strip() and not ln.startswith("#")]
    head = rows[0]
    col = head.index("P_reaction")
    return np.array([float(r[col]) for r in rows[1:]])


def averages(out):
    return np.array([[float(x) for x in ln.split()] for ln in open(out / "averages.dat") if not ln.startswith("#")])


def half_unit(v):
    """Half a unit of the 8th significant digit of the Fortran E15.8 print of v."""
    if v == 0:
        return 5e-9
    e = math.floor(math.log10(abs(v))) + 1
    return 0.5 * 10.0 ** (e - 8) * 1.0001


@pytest.mark.parametrize("case", ["hardwall_short", "cu111_dailight_short", "cu111_dailight_oblique"])
def test_reference_program_with_b200_backend_meets_fortran_gates(case, tmp_path):
    assert os.path.exists(PROGRAM), "build the drop-in: make -C oracle (needs the product library)"
    out = run_case(case, tmp_path)
    ref_avg = np.load(os.path.join(GOLDEN, case, "averages.npy"))
    avg = averages(out)
    assert avg.shape == ref_avg.shape
    for a, f in zip(avg.ravel(), ref_avg.ravel()):
        assert abs(a - f) <= half_unit(f), (a, f)
    bk = np.array([np.frombuffer(r, dtype=np.complex128) for r in fortran_records(out / "fort.21")[10:]])
    ref = np.load(os.path.join(GOLDEN, case, "bk_records.npy"))
    steps = np.load(os.path.join(GOLDEN, case, "bk_steps.npy"))
    scale = float(np.load(os.path.join(GOLDEN, case, "bk_scale.npy")))
    assert bk.shape[1] == ref.shape[1]
    worst = float(np.max(np.abs(bk[steps] - ref)))
    assert worst <= 1e-10 * scale, (worst, scale)
    p = p_reaction(out)
    p_ref = np.load(os.path.join(GOLDEN, case, "p_reaction.npy"))
    assert np.max(np.abs(p - p_ref)) <= 5e-7 * max(1.0, float(np.max(p_ref)))


def test_mixed_form_reaction_probability_within_1e6(tmp_path):
    """The precision form's bar: |P_reaction(mixed) - P_reaction(FP64)| <= 1e-6 at every energy."""
    case = "cu111_dailight_short"
    p64 = p_reaction(run_case(case, tmp_path, "b200"))
    p32 = p_reaction(run_case(case, tmp_path, "b200-mixed"))
    dp = float(np.max(np.abs(p32 - p64)))
    print(f"max |dP_reaction| mixed vs FP64 = {dp:.3e}")
    assert dp <= 1e-6
