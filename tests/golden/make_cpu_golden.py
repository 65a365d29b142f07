"""Writes tests/golden/cu111_dailight_small/cpu_backend.npz: the reference CPU backend's own results on the
reference's cu111_dailight_small regression case (Dai-Light PES, tEnd 14000 au, a case whose packet scatters:
P_reaction ~ 6e-3), for the FP64 bars of tests/test_gpu_scattering.py.

The run is the reference's program (its run_program, time loop and analysis) with its CpuBackend, compiled from
the reference's sources (oracle/_ref/spodvr_b200 --device cpu), on the case's input with the Fortran and native
checkpoint files written (CheckpointFormat both) and the S matrix printed (writeSMatrix). It takes about an hour
on 8 threads, so its outputs are committed:
  p_reaction   P_reaction per analysis energy at full precision (scattering_summary.tsv)
  e_coll       the analysis energies (eV)
  psi_index    16384 indices into the final wave packet (the complex payload of fort.9, in file order),
               drawn without replacement by numpy's default_rng(2024), sorted
  psi_values   the wave packet at those indices (complex128)
  psi_norm2    the squared norm of the whole payload

  python tests/golden/make_cpu_golden.py [OUTDIR_OF_A_FINISHED_CPU_RUN]
Without an argument it runs the reference CPU backend in a temporary directory (SPODVR_REFERENCE not needed: the
case's input is tests/golden/cu111_dailight_small/input.json).
"""

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CASE = os.path.join(HERE, "cu111_dailight_small")
PROGRAM = os.path.join(ROOT, "oracle", "_ref", "spodvr_b200")


def fortran_records(path):
    raw = open(path, "rb").read()
    out, i = [], 0
    while i < len(raw):
        n = int.from_bytes(raw[i:i + 4], "little", signed=True)
        out.append(raw[i + 4:i + 4 + n])
        i += n + 8
    return out


def wave_packet(out):
    """The complex payload of fort.9 (the records that hold wave-function values), in file order."""
    recs = [r for r in fortran_records(os.path.join(out, "fort.9")) if len(r) >= 1024 and len(r) % 16 == 0]
    return np.concatenate([np.frombuffer(r, dtype=np.complex128) for r in recs])


def summary(out):
    rows = [ln.rstrip("\n").split("\t") for ln in open(os.path.join(out, "scattering_summary.tsv"))
            if ln.strip() and not ln.startswith("#")]
    head = rows[0]
    return (np.array([float(r[head.index("E_coll")]) for r in rows[1:]]),
            np.array([float(r[head.index("P_reaction")]) for r in rows[1:]]))


def run_cpu(work):
    cfg = json.load(open(os.path.join(CASE, "input.json")))
    cfg.update({"CheckpointFormat": "both", "writeSMatrix": True})
    path = os.path.join(work, "input.json")
    json.dump(cfg, open(path, "w"))
    out = os.path.join(work, "out")
    subprocess.run([PROGRAM, path, "--device", "cpu", "--output-dir", out, "--no-color"], check=True,
                   stdout=subprocess.DEVNULL)
    return out


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else run_cpu(tempfile.mkdtemp(prefix="small_cpu_"))
    e, p = summary(out)
    psi = wave_packet(out)
    idx = np.sort(np.random.default_rng(2024).choice(psi.size, 16384, replace=False))
    np.savez(os.path.join(CASE, "cpu_backend.npz"), e_coll=e, p_reaction=p, psi_index=idx, psi_values=psi[idx],
             psi_norm2=np.array(float(np.vdot(psi, psi).real)))
    print("P_reaction", p.min(), p.max(), "psi", psi.size, "norm2", float(np.vdot(psi, psi).real))


if __name__ == "__main__":
    main()
