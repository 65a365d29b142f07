"""Writes the committed golden fixtures of tests/golden/ from the reference's own regression data.

Run once in a checkout where the reference project is present (its path is the first argument, else
the SPODVR_REFERENCE environment variable); the outputs are committed, so the tests never read the
reference.

For each regression case of the reference (tests/reference/<case>/, Fortran outputs with their
input.json), it writes tests/golden/<case>/:
  input.json            the case's input, unchanged
  averages.npy          fortran_averages.out rows (time, norm, <Z>, <r>, rest norm) as printed (8 digits)
  bk_records.npy        every `stride`-th BK record of fortran_fort21.bin (complex128, the analysis
                        steps' (is, v) coefficients), with bk_steps.npy = their 0-based step indices
  bk_scale.npy          the gate-4 scale max(max |c| over all records, 1e-4)
                        (tests/analysis_reference.hpp:556-565 of the reference)
  p_reaction.npy        the reaction probability per analysis energy printed in fortran_stdout.txt
The gate-4 BK tolerance of the reference is 1e-10 of that scale (tests/regression_gate.hpp:19).
"""

import json
import os
import re
import shutil
import struct
import sys

import numpy as np

CASES = {"hardwall_short": 10, "cu111_dailight_short": 5, "cu111_dailight_oblique": 5, "cu111_dailight_small": 50}


def fortran_records(path):
    raw = open(path, "rb").read()
    out, i = [], 0
    while i < len(raw):
        n = struct.unpack("<i", raw[i:i + 4])[0]
        out.append(raw[i + 4:i + 4 + n])
        i += n + 8
    return out


def main(ref_root=None):
    ref_root = ref_root or os.environ.get("SPODVR_REFERENCE")
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "tests", "reference")):
        sys.exit("make_golden.py: give the reference checkout as the first argument or in SPODVR_REFERENCE")
    here = os.path.dirname(os.path.abspath(__file__))
    for case, stride in CASES.items():
        src = os.path.join(ref_root, "tests", "reference", case)
        dst = os.path.join(here, case)
        os.makedirs(dst, exist_ok=True)
        shutil.copy(os.path.join(src, "input.json"), os.path.join(dst, "input.json"))
        rows = []
        for line in open(os.path.join(src, "fortran_averages.out")):
            parts = line.split()
            if len(parts) == 5:
                try:
                    rows.append([float(x) for x in parts])
                except ValueError:
                    pass
        np.save(os.path.join(dst, "averages.npy"), np.array(rows))
        recs = fortran_records(os.path.join(src, "fortran_fort21.bin"))[10:]
        bk = np.array([np.frombuffer(r, dtype=np.complex128) for r in recs])
        scale = max(float(np.abs(bk).max()), 1e-4)
        steps = np.arange(0, bk.shape[0], stride)
        np.save(os.path.join(dst, "bk_records.npy"), bk[steps])
        np.save(os.path.join(dst, "bk_steps.npy"), steps)
        np.save(os.path.join(dst, "bk_scale.npy"), np.array(scale))
        p = [float(m.group(1).replace("D", "E")) for m in
             re.finditer(r"the reaction probability =\s*([-0-9.DE+]+)", open(os.path.join(src, "fortran_stdout.txt")).read())]
        np.save(os.path.join(dst, "p_reaction.npy"), np.array(p))
        print(case, "averages", len(rows), "bk", bk.shape, "kept", len(steps), "scale", scale, "P", len(p))


if __name__ == "__main__":
    main(*sys.argv[1:])
