"""The asymptotic analysis on the device (needs a B200): Balint-Kurti coefficients at the analysis line
and the on-the-fly S-matrix sums, in FP64, against the oracle.

The oracle's BK coefficients are those of the reference's BalintKurtiAnalyzer (balint_kurti.cpp:39-84)
after each analysis step of the LCG wave packet, with the reference's analysis surface (fixed or not,
recorded per step); the S sums restate SMatrixAccumulator::add (s_matrix.cpp:49-56) on them. The
tolerance is the BK gate of the reference, 1e-10 of the largest coefficient.
"""

import json
import os

import numpy as np
import pytest

from conftest import read_c128

import spo_oracle as O

pytestmark = pytest.mark.gpu


def analysis_of(d):
    a = json.load(open(os.path.join(d, "case", "analysis.json")))
    m = json.load(open(os.path.join(d, "case", "manifest.json")))
    n_dif = a["n_diffraction"]
    a["rotation_j"] = [a["state_j"][i * n_dif] for i in range(a["n_rotation"])]
    a["iz_analysis"] = m["iz_analysis"]
    a["dr"] = m["dr"]
    phi = np.fromfile(os.path.join(d, "case", "phi_vj.f64"))
    energies = np.fromfile(os.path.join(d, "case", "analysis_energies_hartree.f64"))
    return a, phi, energies


@pytest.mark.parametrize("name", ["tiny_dailight", "tiny_oblique", "tiny_dailight_sym"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bk_and_s_matrix_match_the_reference_analysis(ref_case, name, precision):
    from spo_b200 import B200Backend, CaseBundle
    d = ref_case(name)
    case = CaseBundle.load(os.path.join(d, "case"))
    a, phi, energies = analysis_of(d)
    be = B200Backend(case, precision=precision)
    be.read_wave_packet(read_c128(os.path.join(d, "psi_initial.c128")), read_c128(os.path.join(d, "chi_start.c128")))
    be.analysis_setup(a, phi, energies)
    ref_bk = read_c128(os.path.join(d, "bk_steps.c128")).reshape(2, -1)
    surface = np.fromfile(os.path.join(d, "surface_index.i32"), dtype=np.int32)
    times = np.fromfile(os.path.join(d, "analysis_times.f64"))
    got = []
    for step in range(2):
        be.propagate_analysis_step()
        fixed = surface[step] >= 0
        index = surface[step] if fixed else -1 - surface[step]
        got.append(be.bk_coefficients(times[step], fixed, index, accumulate=True))
    got = np.array(got)
    scale = np.max(np.abs(ref_bk))
    tol = 1e-10 if precision == "fp64" else 3e-5
    assert np.max(np.abs(got - ref_bk)) <= tol * scale
    sums = be.s_matrix_sums()
    ref_sums = O.s_matrix_sums(ref_bk, times, energies, a["analysis_time_step"])
    assert np.max(np.abs(sums - ref_sums)) <= tol * np.max(np.abs(ref_sums))
    be.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_averages_match_the_oracle(precision):
    """spo_averages (norm, <Z>, <r>, rest norm on the device) against compute_averages restated in the
    oracle (averages.cpp:37-80), on a random wave packet: FP64 sums in another order, so 1e-12; the
    mixed form holds the state in complex64, so its inputs differ by the rounding of psi (2e-6)."""
    from spo_b200 import B200Backend, workload
    case = workload.config_case({"nz": 48, "nr": 24, "nx": 4, "ny": 4, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 96, "nz_potential": 30})
    rng = np.random.default_rng(21)
    psi = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    z = 1.5 + 0.12 * np.arange(case.nz)
    zs = 1.5 + 0.12 * np.arange(case.nz_specular)
    r = 0.4 + 0.1 * np.arange(case.nr)
    vol_scat, vol_spec = 0.12 * 0.1 * 0.37, 0.12 * 0.1
    iz_analysis, surface = 30, 70
    with B200Backend(case, precision=precision) as be:
        be.read_wave_packet(psi, chi)
        got = be.averages(z, zs, r, vol_scat, vol_spec, iz_analysis, surface)
        dens = be.block_densities()
        psi_dev, chi_dev = be.wave_packet_on_host()
    ref = O.averages(dens, chi_dev, z, zs, r, vol_scat, vol_spec, iz_analysis, surface)
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-12
    exact = O.averages(O.block_densities(psi), chi, z, zs, r, vol_scat, vol_spec, iz_analysis, surface)
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert np.max(np.abs(got - exact) / np.abs(exact)) <= tol
