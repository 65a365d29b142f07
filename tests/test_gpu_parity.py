"""Parity of the sm_100a path with the oracle, through the C ABI (needs a B200).

The oracle is the reference's CPU path compiled from its own sources (oracle/_ref) on the same
inputs: the same case bundle (the reference's own set-up), the same LCG wave packet
(tests/cuda/cuda_test_setup.hpp:53-64 of the reference). As the reference's own GPU tests do
(tests/cuda/test_cuda_backend.cpp:86-106, :161-278), each operator is compared alone, then whole
analysis steps. Tolerances (FP64 form): 1e-12 relative per operator, 1e-10 relative L2 over analysis
steps (the FP64 bar); the mixed form (complex64 psi, FP32 FFTs): 3e-5 relative L2 over two steps.
"""

import os

import numpy as np
import pytest

from conftest import TINY_CASES, read_c128, rel_err, rel_l2

pytestmark = pytest.mark.gpu


def backend_for(d, precision="fp64"):
    from spo_b200 import B200Backend, CaseBundle
    case = CaseBundle.load(os.path.join(d, "case"))
    be = B200Backend(case, precision=precision)
    psi0 = read_c128(os.path.join(d, "psi_initial.c128"), case.psi_shape)
    chi0 = read_c128(os.path.join(d, "chi_start.c128"), case.chi_shape)
    be.read_wave_packet(psi0, chi0)
    return case, be, psi0, chi0


@pytest.mark.parametrize("name", TINY_CASES)
def test_each_operator_matches_oracle(ref_case, name):
    from spo_b200 import capi
    d = ref_case(name)
    case, be, _, _ = backend_for(d)
    shp, cshp = case.psi_shape, case.chi_shape
    be.apply_stage(capi.STAGE_SPECULAR)
    assert rel_err(be.specular(), read_c128(os.path.join(d, "stage_specular_chi.c128"), cshp)) < 1e-12
    be.apply_stage(capi.STAGE_ZR)
    psi, _ = be.wave_packet_on_host()
    assert rel_err(psi, read_c128(os.path.join(d, "stage_zr_psi.c128"), shp)) < 1e-12
    be.apply_stage(capi.STAGE_XY)
    psi, _ = be.wave_packet_on_host()
    assert rel_err(psi, read_c128(os.path.join(d, "stage_xy_psi.c128"), shp)) < 1e-12
    be.apply_stage(capi.STAGE_POTENTIAL)
    psi, chi = be.wave_packet_on_host()
    assert rel_err(psi, read_c128(os.path.join(d, "stage_potential_psi.c128"), shp)) < 1e-12
    assert rel_err(chi, read_c128(os.path.join(d, "stage_potential_chi.c128"), cshp)) < 1e-12
    be.close()


@pytest.mark.parametrize("name", TINY_CASES)
def test_analysis_steps_match_oracle(ref_case, name):
    d = ref_case(name)
    case, be, _, _ = backend_for(d)
    chis = read_c128(os.path.join(d, "chi_steps.c128"), (2,) + case.chi_shape)
    be.propagate_analysis_step()
    assert rel_l2(be.specular(), chis[0]) < 1e-10
    be.propagate_analysis_step()
    psi, chi = be.wave_packet_on_host()
    assert rel_l2(psi, read_c128(os.path.join(d, "psi_final.c128"), case.psi_shape)) < 1e-10
    assert rel_l2(chi, chis[1]) < 1e-10
    dens = np.fromfile(os.path.join(d, "block_densities.f64"))
    assert np.max(np.abs(be.block_densities() - dens)) <= 1e-10 * np.max(dens)
    assert be.last_launch_count() > 0
    be.close()


def test_readbacks_are_the_host_layout(ref_case):
    d = ref_case("tiny_dailight_sym")
    case, be, psi0, chi0 = backend_for(d)
    psi, chi = be.wave_packet_on_host()
    assert np.array_equal(psi, psi0) and np.array_equal(chi, chi0)
    for iz in (0, case.nz // 2, case.nz - 1):
        assert np.array_equal(be.z_plane(iz), psi0[iz])
    for ixy in (0, case.nx * case.ny - 1):
        col = be.site_column(ixy)  # (irot, izr) with izr fastest
        ix, iy = divmod(ixy, case.ny)
        expect = psi0[:, :, ix, iy, :].reshape(case.nz * case.nr, case.n_rot).T
        assert np.array_equal(col, expect)
    dens = be.block_densities()
    host = np.sum(np.abs(psi0.reshape(case.nz * case.nr, -1)) ** 2, axis=1)
    assert np.max(np.abs(dens - host)) <= 1e-13 * np.max(host)
    be.close()


def test_runs_are_bitwise_repeatable(ref_case):
    """Fixed launch shapes and fixed-order reductions, no atomics: two runs agree bitwise
    (the reference's GPU test of the same property: tests/cuda/test_cuda_backend.cpp:388)."""
    d = ref_case("tiny_oblique")
    out = []
    for _ in range(2):
        case, be, _, _ = backend_for(d)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("name", ["tiny_dailight", "tiny_oblique", "tiny_dailight_sym"])
def test_mixed_precision_form_stays_close(ref_case, name):
    d = ref_case(name)
    case, be, _, _ = backend_for(d, precision="mixed")
    for _ in range(2):
        be.propagate_analysis_step()
    psi, chi = be.wave_packet_on_host()
    chis = read_c128(os.path.join(d, "chi_steps.c128"), (2,) + case.chi_shape)
    assert rel_l2(psi, read_c128(os.path.join(d, "psi_final.c128"), case.psi_shape)) < 3e-5
    assert rel_l2(chi, chis[1]) < 3e-5
    be.close()


def test_errors_are_reported_not_thrown(ref_case):
    from spo_b200 import B200Error
    d = ref_case("tiny_hardwall")
    case, be, _, _ = backend_for(d)
    with pytest.raises(B200Error, match="iz out of range"):
        be.z_plane(case.nz)
    with pytest.raises(B200Error, match="ixy out of range"):
        be.site_column(-1)
    with pytest.raises(B200Error, match="unknown stage"):
        be.apply_stage(99)
    be.propagate_analysis_step()  # the handle stays usable after refused calls
    be.close()


@pytest.mark.parametrize("kernels", ["v3", "v4", "v5"])
@pytest.mark.parametrize("name", TINY_CASES)
def test_potential_kernels_match_oracle(ref_case, name, kernels, monkeypatch):
    """The potential step and two analysis steps with each chunked potential kernel forced (the default
    takes the first available of potential5, potential4, potential3, ...). Cases whose angular grid the
    kernel does not cover are skipped; potential5 exists in the mixed form only (3e-5 over two steps)."""
    monkeypatch.setenv("SPO_B200_KERNELS", kernels)
    from spo_b200 import capi
    d = ref_case(name)
    precision = "mixed" if kernels == "v5" else "fp64"
    case, be, psi0, chi0 = backend_for(d, precision=precision)
    if f"potential=potential{kernels[1]}" not in be.describe():
        be.close()
        pytest.skip(f"{kernels} does not cover ntheta {case.n_theta}, nphi {case.n_phi}")
    shp, cshp = case.psi_shape, case.chi_shape
    be.read_wave_packet(read_c128(os.path.join(d, "stage_xy_psi.c128"), shp),
                        read_c128(os.path.join(d, "stage_specular_chi.c128"), cshp))
    be.apply_stage(capi.STAGE_POTENTIAL)
    psi, chi = be.wave_packet_on_host()
    tol_stage, tol_steps = (1e-12, 1e-10) if precision == "fp64" else (3e-6, 3e-5)
    assert rel_err(psi, read_c128(os.path.join(d, "stage_potential_psi.c128"), shp)) < tol_stage
    assert rel_err(chi, read_c128(os.path.join(d, "stage_potential_chi.c128"), cshp)) < tol_stage
    be.read_wave_packet(psi0, chi0)
    be.propagate_analysis_step()
    be.propagate_analysis_step()
    psi, chi = be.wave_packet_on_host()
    chis = read_c128(os.path.join(d, "chi_steps.c128"), (2,) + cshp)
    assert rel_l2(psi, read_c128(os.path.join(d, "psi_final.c128"), shp)) < tol_steps
    assert rel_l2(chi, chis[1]) < tol_steps
    be.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_restart_is_bitwise(ref_case, precision):
    """Checkpoint/restart through the backend interface (wave_packet_on_host, then read_wave_packet into a
    fresh handle), as the reference's checkpoint files do (io/checkpoint.hpp; its restart test
    test_restart.cpp:241 wants split runs bitwise equal to straight ones): two analysis steps straight
    equal one step, a restart and one more step, bit for bit. The mixed form's complex64 state widens
    to complex128 on the host and narrows back exactly."""
    d = ref_case("tiny_oblique")
    case, be, _, _ = backend_for(d, precision=precision)
    be.propagate_analysis_step()
    be.propagate_analysis_step()
    straight = be.wave_packet_on_host()
    be.close()
    case, be, _, _ = backend_for(d, precision=precision)
    be.propagate_analysis_step()
    psi, chi = be.wave_packet_on_host()
    be.close()
    from spo_b200 import B200Backend
    with B200Backend(case, precision=precision) as again:
        again.read_wave_packet(psi, chi)
        again.propagate_analysis_step()
        split = again.wave_packet_on_host()
    assert np.array_equal(straight[0], split[0]) and np.array_equal(straight[1], split[1])
