"""Checkpoint and restart through the reference's own files (needs a B200).

oracle/_ref/spodvr_b200 is the reference program with the B200 backend in place of its CPU backend, so
its checkpoints are the reference's formats: checkpoint.bin and bk_coefficients.bin (io/checkpoint.hpp:
26-56), and the Fortran fort.9 / fort.21 (io/fortran_files.hpp:22-42), written from the wave packet
that the backend hands back on the host and read into it again on a restart (app/run.cpp:141-160).

As the reference's own restart test (tests/test_restart.cpp:241-255 and 475-480): a run split by a
restart (0 .. 60 and 60 .. 120 au) must write bitwise the same files as the unsplit run (0 .. 120 au),
restarted from the native files and from the Fortran ones, here on the B200 in both precision forms.
A restart on the B200 from the checkpoint of the reference's CPU backend continues that run: its wave
packet agrees with the unsplit B200 run to the FP64 bar (relative L2 1e-10).
"""

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

PROGRAM = os.path.join(ROOT, "oracle", "_ref", "spodvr_b200")

COMPARED = ["checkpoint.bin", "bk_coefficients.bin", "s_matrix.tsv", "scattering_summary.tsv", "fort.9", "fort.21"]


def base_input():
    cfg = json.load(open(os.path.join(GOLDEN, "hardwall_short", "input.json")))
    cfg["CheckpointFormat"] = "both"  # the native files and fort.9 / fort.21
    cfg["writeSMatrix"] = True
    return cfg


def with_times(cfg, t_start, t_end, n_steps):
    cfg = dict(cfg)
    cfg.update({"tStart": t_start, "tEnd": t_end, "nStep": n_steps})
    return cfg


def restart_from(cfg, directory, fmt="native"):
    cfg = dict(cfg)
    cfg.update({"NewCalc": False, "RestartDir": str(directory), "RestartFormat": fmt})
    return cfg


def run(cfg, work, device):
    work.mkdir(parents=True)
    path = work / "input.json"
    path.write_text(json.dumps(cfg))
    out = work / "out"
    r = subprocess.run([PROGRAM, str(path), "--device", device, "--output-dir", str(out), "--no-color"],
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


@pytest.mark.parametrize("device", ["b200", "b200-mixed"])
def test_split_run_is_bitwise_the_unsplit_run(device, tmp_path):
    assert os.path.exists(PROGRAM), "build the drop-in: make -C oracle (needs the product library)"
    cfg = base_input()
    full = run(with_times(cfg, 0.0, 120.0, 60), tmp_path / "full", device)
    first = run(with_times(cfg, 0.0, 60.0, 30), tmp_path / "first", device)
    second = run(restart_from(with_times(cfg, 60.0, 120.0, 30), first), tmp_path / "second", device)
    second_f = run(restart_from(with_times(cfg, 60.0, 120.0, 30), first, "fortran"), tmp_path / "second_f", device)
    for name in COMPARED:
        ref = (full / name).read_bytes()
        assert (second / name).read_bytes() == ref, name
        if name != "scattering_summary.tsv":
            assert (second_f / name).read_bytes() == ref, ("fortran restart", name)
    assert (second / "bk_coefficients.bin").stat().st_size > (first / "bk_coefficients.bin").stat().st_size


def wave_packet(out):
    """The complex payload of fort.9 (the records that hold wave-function values), in file order."""
    recs = [r for r in fortran_records(out / "fort.9") if len(r) >= 1024 and len(r) % 16 == 0]
    return np.concatenate([np.frombuffer(r, dtype=np.complex128) for r in recs])


def test_b200_continues_a_checkpoint_of_the_reference_cpu_backend(tmp_path):
    """The wave packet after the restart against the unsplit B200 run: relative L2 <= 1e-10 (the FP64 bar).
    At t = 120 au the packet has not reached the analysis line yet, so the BK coefficients are rounding
    noise (~1e-31) and are not compared here."""
    cfg = base_input()
    full = run(with_times(cfg, 0.0, 120.0, 60), tmp_path / "full", "b200")
    first_cpu = run(with_times(cfg, 0.0, 60.0, 30), tmp_path / "first_cpu", "cpu")
    second = run(restart_from(with_times(cfg, 60.0, 120.0, 30), first_cpu), tmp_path / "second", "b200")
    psi_full, psi = wave_packet(full), wave_packet(second)
    assert psi.shape == psi_full.shape and psi.size > 100000
    assert float(np.linalg.norm(psi - psi_full) / np.linalg.norm(psi_full)) <= 1e-10


FINE_ANALYSIS_FILES = ["fine_analysis/grid.json", "fine_analysis/scattering_summary.tsv", "fine_analysis/s_matrix.tsv",
                       "fine_analysis/probabilities_rovib.tsv", "fine_analysis/probabilities_diffraction.tsv",
                       "fine_analysis/spectrum/scattering_summary.tsv",
                       "fine_analysis/spectrum/probabilities_rovib.tsv",
                       "fine_analysis/spectrum/probabilities_diffraction.tsv"]


def fine_input(t_start, t_end):
    """The reference's fine-analysis runs (tests/test_restart.cpp:139-183): dtStep = dtAna = 10 au, 0 .. 600 au
    (60 BK records; the values are not physical, the runs are only compared with each other)."""
    cfg = base_input()
    cfg.update({"dtStep": 10.0, "dtAna": 10.0, "dtAve": 100.0, "alsoAnalysis": True})
    return with_times(cfg, t_start, t_end, int((t_end - t_start) / 10.0 + 0.5))


def test_fine_analysis_of_b200_bk_files_is_the_same_in_every_run_mode(tmp_path):
    """The fine analysis (§8(f)4: the reference's host post-processing of the BK file) of BK coefficients that
    the B200 computed: alsoAnalysis after the run, the same run split by a restart, and onlyAnalysis of the
    native and of the Fortran BK file give bitwise the same files (as tests/test_restart.cpp:204-219)."""
    full = run(fine_input(0.0, 600.0), tmp_path / "full", "b200")
    first = run(fine_input(0.0, 300.0), tmp_path / "first", "b200")
    second = run(restart_from(fine_input(300.0, 600.0), first), tmp_path / "second", "b200")
    outs = {"second": second}
    for fmt in ("native", "fortran"):
        cfg = fine_input(0.0, 600.0)
        cfg.update({"alsoAnalysis": False, "onlyAnalysis": True, "RestartDir": str(full), "RestartFormat": fmt})
        outs[fmt] = run(cfg, tmp_path / f"only_{fmt}", "b200")
    assert (full / "fine_analysis" / "s_matrix.tsv").exists()
    for name in FINE_ANALYSIS_FILES:
        ref = (full / name).read_bytes()
        assert ref, name
        for other, out in outs.items():
            assert (out / name).read_bytes() == ref, (other, name)
