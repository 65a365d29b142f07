"""The oracle is checked before it is trusted (CPU only).

1. The FFT substitute of the oracle build against a naive DFT, layout by layout (the reference's own
   FFT tests compare FFTW with a naive DFT the same way, tests/test_fft.cpp:118-240).
2. The reference build against the Fortran regression data: the committed record of the complete
   runs (tests/golden/oracle_pin.json, made by tests/golden/pin_oracle.py) and, re-run here, the first
   analysis steps of hardwall_short against fortran_fort21.bin.
3. The numpy restatement (oracle/spo_oracle.py) against the reference build, operator by operator
   and over two analysis steps, on five small cases (hard wall; Dai-Light corrugated PES; hetero-
   nuclear full theta grid; oblique incidence with the momentum shift; C6v surface symmetry).
"""

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REF_FFT_CHECK, REF_TOOL, TINY_CASES, _ensure_built, read_c128, rel_err

import spo_oracle as O


def test_fft_substitute_matches_naive_dft():
    _ensure_built()
    r = subprocess.run([REF_FFT_CHECK], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout


def test_reference_build_pinned_to_fortran_complete_runs():
    """The complete runs (every analysis step) met the reference's gate 4 for the BK coefficients."""
    pin = json.load(open(os.path.join(GOLDEN, "oracle_pin.json")))
    for case in ["hardwall_short", "cu111_dailight_short", "cu111_dailight_oblique"]:
        rec = pin[case]
        assert rec["bk_gate_1e-10"], (case, rec)
        assert rec["p_reaction_within_print"], (case, rec)


def test_reference_build_first_steps_match_fortran(tmp_path):
    _ensure_built()
    case = "hardwall_short"
    steps = 11
    out = str(tmp_path / case)
    subprocess.run([REF_TOOL, "case", os.path.join(GOLDEN, case, "input.json"), out, "--analysis-steps", str(steps),
                    "--no-psi"], check=True, stdout=subprocess.DEVNULL)
    bk = read_c128(os.path.join(out, "bk_steps.c128")).reshape(steps, -1)
    ref = np.load(os.path.join(GOLDEN, case, "bk_records.npy"))
    kept = np.load(os.path.join(GOLDEN, case, "bk_steps.npy"))
    scale = float(np.load(os.path.join(GOLDEN, case, "bk_scale.npy")))
    sel = kept[kept < steps]
    assert len(sel) >= 2
    worst = np.max(np.abs(bk[sel] - ref[: len(sel)]))
    assert worst <= 1e-10 * scale


def test_lcg_matches_reference(ref_case):
    d = ref_case("tiny_dailight")
    case = O.load_case(os.path.join(d, "case"))
    psi0 = read_c128(os.path.join(d, "psi_initial.c128"))
    chi0 = read_c128(os.path.join(d, "chi_start.c128"))
    assert np.array_equal(psi0, O.lcg_complex(psi0.size, 7))
    assert np.array_equal(chi0, O.lcg_complex(chi0.size, 8))
    assert psi0.size == case.nz * case.nr * case.nx * case.ny * case.n_rot


@pytest.mark.parametrize("name", TINY_CASES)
def test_restatement_matches_reference_build(ref_case, name):
    d = ref_case(name)
    case = O.load_case(os.path.join(d, "case"))
    shp = (case.nz, case.nr, case.nx, case.ny, case.n_rot)
    cshp = (case.nz_specular, case.nr)
    psi0 = read_c128(os.path.join(d, "psi_initial.c128"), shp)
    chi0 = read_c128(os.path.join(d, "chi_start.c128"), cshp)
    tol = 1e-13
    chi = O.specular_apply(chi0, case, O.FULL, False)
    assert rel_err(chi, read_c128(os.path.join(d, "stage_specular_chi.c128"), cshp)) < tol
    p = O.kinetic_zr(psi0, case, O.FULL)
    assert rel_err(p, read_c128(os.path.join(d, "stage_zr_psi.c128"), shp)) < tol
    p = O.kinetic_xy(p, case, O.FULL)
    assert rel_err(p, read_c128(os.path.join(d, "stage_xy_psi.c128"), shp)) < tol
    p, chi = O.potential_apply(p, chi, case)
    assert rel_err(p, read_c128(os.path.join(d, "stage_potential_psi.c128"), shp)) < tol
    assert rel_err(chi, read_c128(os.path.join(d, "stage_potential_chi.c128"), cshp)) < tol
    expia = O.exp_potential(case)
    p, chi = psi0, chi0
    for _ in range(2):
        p, chi = O.propagate_analysis_step(p, chi, case, expia)
    assert rel_err(p, read_c128(os.path.join(d, "psi_final.c128"), shp)) < tol
    chis = read_c128(os.path.join(d, "chi_steps.c128"), (2,) + cshp)
    assert rel_err(chi, chis[1]) < tol
    dens = np.fromfile(os.path.join(d, "block_densities.f64"))
    assert np.max(np.abs(O.block_densities(p) - dens)) <= 1e-13 * np.max(dens)


@pytest.mark.parametrize("name", ["tiny_dailight", "tiny_oblique"])
def test_averages_restatement_matches_reference_build(ref_case, name):
    """The oracle's averages against the reference's compute_averages (averages.cpp:37-80) on the final
    wave packet of two analysis steps, with the reference's own densities, grids and volume elements."""
    import json
    d = ref_case(name)
    case = O.load_case(os.path.join(d, "case"))
    g = json.load(open(os.path.join(d, "averages.json")))
    ref = np.fromfile(os.path.join(d, "averages.f64"))
    chis = read_c128(os.path.join(d, "chi_steps.c128"), (2, case.nz_specular, case.nr))
    got = O.averages(np.fromfile(os.path.join(d, "block_densities.f64")), chis[1],
                     np.fromfile(os.path.join(d, "grid_z.f64")), np.fromfile(os.path.join(d, "grid_z_specular.f64")),
                     np.fromfile(os.path.join(d, "grid_r.f64")), g["volume_scattering"], g["volume_specular"],
                     g["iz_analysis"], g["surface_index"])
    assert ref[3] > 0.0  # the rest-norm window is not empty
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-13
