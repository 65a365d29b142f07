"""The register-DFT kernels against the general kernels, on the shapes of the benchmark configuration
(needs a B200).

The tiny regression cases (test_gpu_parity.py) run the register-DFT kernels at their own sizes
against the oracle. The configuration-2 sizes (axis lengths 128 = 8 x 16 and 48 = 6 x 8, a 16 x 16
(x, y) grid, nphi 32 with ntheta 16) use other instantiations; here they are checked operator by
operator and over an analysis step against the general shared-memory Stockham kernels
(SPO_B200_KERNELS=v1), which the oracle checks on every case. All register potential kernels are
covered: v2 (potential2, one block per (Z, r) point looping over column chunks), v3 (potential3, one
block per point and chunk) and v4 (potential4, persistent blocks with register-tiled theta
contractions). v3 and v4 apply the same operations in the same order to every column and leave the
projection to a second kernel; they agree to rounding (not bitwise: the compiler may contract the
products of a complex multiply into FMAs differently in each kernel).

The tile widths of the register kernels (8, 16 or 32 batch lanes per block) compute every line with
the same operations in the same order, so they give bitwise equal wave packets; the autotuner's
choice between them can change the speed only.
"""

import os

import numpy as np
import pytest

from conftest import rel_err, rel_l2

pytestmark = pytest.mark.gpu

SHAPES = {
    # Z 128 = 16 x 8, r 48 = 8 x 6, (x, y) 4 x 4, theta 16 x phi 32 (8 columns per chunk)
    "axes_and_phi": {"nz": 128, "nr": 48, "nx": 4, "ny": 4, "j_max": 15, "mj_max": 15, "nz_specular": 256,
                     "nz_potential": 84},
    # (x, y) 16 x 16, Z 24 = 6 x 4, r 24, theta 4 x phi 8 (32 columns per chunk)
    "xy16": {"nz": 24, "nr": 24, "nx": 16, "ny": 16, "j_max": 3, "mj_max": 3, "nz_specular": 64, "nz_potential": 16},
}


def make(case, kernels, precision, tiles=None):
    from spo_b200 import B200Backend
    env = {"SPO_B200_KERNELS": kernels, "SPO_B200_TILES": tiles}
    old = {k: os.environ.get(k) for k in env}
    for k, v in env.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    try:
        return B200Backend(case, precision=precision)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("shape", list(SHAPES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kernels", ["v2", "v3", "v4", "v5", "v6"])
def test_register_kernels_match_general_kernels(shape, precision, kernels):
    from spo_b200 import capi, workload
    case = workload.config_case(SHAPES[shape])
    rng = np.random.default_rng(5)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    tol_stage, tol_step = (1e-12, 1e-11) if precision == "fp64" else (2e-6, 2e-5)
    ref = make(case, "v1", precision)
    new = make(case, kernels, precision)
    if kernels in ("v5", "v6") and precision == "fp64":  # potential5 and 6 are the mixed form's
        assert "potential=potential4" in new.describe(), new.describe()
    elif kernels == "v6" and shape == "xy16":  # potential6 needs theta 16 x phi 32: the best one below it
        assert "potential=potential5" in new.describe(), new.describe()
    else:
        assert f"potential=potential{kernels[1]}" in new.describe(), new.describe()
    for be in (ref, new):
        be.read_wave_packet(psi0, chi0)
    for stage in (capi.STAGE_ZR, capi.STAGE_XY, capi.STAGE_POTENTIAL):
        ref.apply_stage(stage)
        new.apply_stage(stage)
        p1, c1 = ref.wave_packet_on_host()
        p2, c2 = new.wave_packet_on_host()
        assert rel_err(p2, p1) < tol_stage, (shape, stage)
        assert rel_err(c2, c1) < tol_stage, (shape, stage)
    for be in (ref, new):
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
    p1, c1 = ref.wave_packet_on_host()
    p2, c2 = new.wave_packet_on_host()
    assert rel_l2(p2, p1) < tol_step and rel_l2(c2, c1) < tol_step
    ref.close()
    new.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tile_widths_are_bitwise_equal(precision):
    from spo_b200 import workload
    # Z 128 = 8 x 16 and (x, y) 16 x 16: the lengths whose kernels have 8, 16 and 32 lane tiles
    case = workload.config_case({"nz": 128, "nr": 24, "nx": 16, "ny": 16, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 256, "nz_potential": 40})
    rng = np.random.default_rng(9)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for tiles in ("8", "16", "32"):
        be = make(case, "v3", precision, tiles)
        assert f"z=axis2b<128,tb{tiles}>" in be.describe() and f"xy=xy2p<16,tb{tiles}>" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    for k in (1, 2):
        assert np.array_equal(out[0][0], out[k][0]) and np.array_equal(out[0][1], out[k][1]), k


@pytest.mark.parametrize("j_max", [15, 7, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_potential3_and_potential4_agree(j_max, precision):
    """ntheta 16 / nphi 32, ntheta 8 / nphi 16 and ntheta 4 / nphi 8: every instantiation family of
    potential4 against potential3 over an analysis step, to rounding (1e-13 FP64, 2e-6 mixed)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": 32, "nr": 24, "nx": 8, "ny": 8, "j_max": j_max, "mj_max": j_max,
                                 "nz_specular": 64, "nz_potential": 20})
    rng = np.random.default_rng(3)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for kernels in ("v3", "v4"):
        be = make(case, kernels, precision)
        assert f"potential=potential{kernels[1]}" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    tol = 1e-13 if precision == "fp64" else 2e-6
    assert rel_err(out[1][0], out[0][0]) < tol and rel_err(out[1][1], out[0][1]) < tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zr_windows_are_bitwise_equal(precision, monkeypatch):
    """T_Z and T_r run window by window over the (x, y, irot) lanes (Z then r per window, through L2):
    the same lines with the same operations as the two full passes, so bitwise the same wave packet;
    windows of 96 and 160 lanes (the last window of 160 is partial: 16 x 16 x 16 = 4096 lanes)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": 128, "nr": 24, "nx": 16, "ny": 16, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 256, "nz_potential": 40})
    rng = np.random.default_rng(13)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for window in ("0", "96", "160"):
        monkeypatch.setenv("SPO_B200_ZR_WINDOW", window)
        be = make(case, "v4", precision)
        assert f"zr_window={window}" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    for k in (1, 2):
        assert np.array_equal(out[0][0], out[k][0]) and np.array_equal(out[0][1], out[k][1]), k


@pytest.mark.parametrize("j_max", [15, 7, 3])
def test_potential5_agrees_with_potential4(j_max):
    """potential5 (bulk asynchronous copies, mixed form) against potential4 over an analysis step, on the
    three instantiation families: the same sums in the same order except the FMA contraction choices
    of each kernel, so they agree to FP32 rounding; then potential5 alone over four steps on a case
    whose x-y grid is not a multiple of the column chunk (n_xy 36, 8 or 16 columns per chunk)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": 32, "nr": 24, "nx": 8, "ny": 8, "j_max": j_max, "mj_max": j_max,
                                 "nz_specular": 64, "nz_potential": 20})
    rng = np.random.default_rng(5)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for kernels in ("v4", "v5"):
        be = make(case, kernels, "mixed")
        assert f"potential=potential{kernels[1]}" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    assert rel_err(out[1][0], out[0][0]) < 2e-6 and rel_err(out[1][1], out[0][1]) < 2e-6
    ragged = workload.config_case({"nz": 24, "nr": 24, "nx": 6, "ny": 6, "j_max": j_max, "mj_max": j_max,
                                   "nz_specular": 64, "nz_potential": 16})
    psi0 = rng.standard_normal(ragged.psi_shape) + 1j * rng.standard_normal(ragged.psi_shape)
    chi0 = rng.standard_normal(ragged.chi_shape) + 1j * rng.standard_normal(ragged.chi_shape)
    res = []
    for kernels in ("v1", "v5"):
        be = make(ragged, kernels, "mixed")
        be.read_wave_packet(psi0, chi0)
        for _ in range(4):
            be.propagate_analysis_step()
        res.append(be.wave_packet_on_host())
        be.close()
    assert rel_l2(res[1][0], res[0][0]) < 2e-5 and rel_l2(res[1][1], res[0][1]) < 2e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rxy_slabs_are_bitwise_equal(precision, monkeypatch):
    """T_r and T_xy slab by slab of Z planes (through L2), with the gas-phase step fused in the xy pass:
    the same lines with the same operations as the full passes, so bitwise the same wave packet; slabs
    of 1 and 3 planes (3 does not divide nz = 32: a partial last slab)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": 32, "nr": 24, "nx": 16, "ny": 16, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 64, "nz_potential": 20})
    rng = np.random.default_rng(17)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for planes in ("0", "1", "3"):
        monkeypatch.setenv("SPO_B200_RXY_PLANES", planes)
        be = make(case, "v4", precision)
        assert f"rxy_planes={planes}" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    for k in (1, 2):
        assert np.array_equal(out[0][0], out[k][0]) and np.array_equal(out[0][1], out[k][1]), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_kinetic_kernels_agree(precision, monkeypatch):
    """The persistent forms of the register kinetic kernels (next tile's loads in flight during the
    current tile) apply the same operations to every line, with the momentum shift of oblique incidence
    and the fused gas-phase step included: the same wave packet to rounding (1e-13 FP64, 2e-6 mixed; not
    bitwise, the compiler's FMA contractions may differ between the two kernels)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": 128, "nr": 24, "nx": 16, "ny": 16, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 256, "nz_potential": 40})
    rng = np.random.default_rng(23)
    n_xy = case.nx * case.ny
    phase = np.exp(1j * rng.uniform(0, 2 * np.pi, n_xy))
    case.a["shift_forward"] = phase
    case.a["shift_backward"] = np.conj(phase)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for persistent in ("0", "1"):
        monkeypatch.setenv("SPO_B200_PERSISTENT", persistent)
        be = make(case, "v4", precision)
        assert ("persistent=zrxy" in be.describe()) == (persistent == "1"), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    tol = 1e-13 if precision == "fp64" else 2e-6
    assert rel_err(out[1][0], out[0][0]) < tol and rel_err(out[1][1], out[0][1]) < tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nz,nr", [(128, 24), (48, 32)])
def test_balanced_axis_kernel_agrees(nz, nr, precision, monkeypatch):
    """The balanced axis kernel (lengths N1 x 2 N1: Z = 128 = 8 x 16, r = 32 = 4 x 8), in which every
    thread takes two first-level lines and one second-level line, against the plain one (N2 threads per
    lane, half of them idle in the second level): the same wave packet to rounding (1e-13 FP64, 2e-6
    mixed)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": nz, "nr": nr, "nx": 8, "ny": 8, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 2 * nz, "nz_potential": 40})
    rng = np.random.default_rng(31)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    n = nz if nz == 128 else nr
    axis = "z" if nz == 128 else "r"
    out = []
    for balanced in ("0", "1"):
        monkeypatch.setenv("SPO_B200_BALANCED", balanced)
        be = make(case, "v4", precision)
        form = "axis2b" if balanced == "1" else "axis2"
        assert f"{axis}={form}<{n}," in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    tol = 1e-13 if precision == "fp64" else 2e-6
    assert rel_err(out[1][0], out[0][0]) < tol and rel_err(out[1][1], out[0][1]) < tol


@pytest.mark.parametrize("nz,nr", [(48, 40), (56, 24), (80, 112)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_prime_factor_axis_kernel_agrees(nz, nr, precision, monkeypatch):
    """The prime-factor axis kernel (N = N1 N2 with N1, N2 coprime: 24 = 3 x 8, 40 = 5 x 8, 48 = 3 x 16,
    56 = 7 x 8, 80 = 5 x 16, 112 = 7 x 16; no twiddles, the factors in the permuted order) against the
    two-level kernel with twiddles (SPO_B200_PFA=0) over an analysis step: the same wave packet to rounding
    (1e-12 FP64, 1e-5 mixed)."""
    from spo_b200 import workload
    case = workload.config_case({"nz": nz, "nr": nr, "nx": 4, "ny": 4, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 2 * nz, "nz_potential": nz // 2})
    rng = np.random.default_rng(43)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    out = []
    for pfa in ("0", "1"):
        monkeypatch.setenv("SPO_B200_PFA", pfa)
        be = make(case, "v4", precision)
        desc = be.describe()
        if pfa == "1":
            assert f"z=axis2pfa<{nz}=" in desc and f"r=axis2pfa<{nr}=" in desc, desc
        else:
            assert "axis2pfa" not in desc, desc
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        out.append(be.wave_packet_on_host())
        be.close()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_l2(out[1][0], out[0][0]) < tol and rel_l2(out[1][1], out[0][1]) < tol


@pytest.mark.parametrize("j_max", [11, 13])
def test_potential5_pads_theta_12_and_14(j_max):
    """The angular grids of the ensemble workload, theta 12 x phi 24 (JMax 11) and theta 14 x phi 28
    (JMax 13), on potential5's 16-row tile (zero matrix rows for the missing theta, whose phi lines are
    skipped), and potential2/3 with phi 28, against the general kernels: the potential stage to 2e-6,
    an analysis step to 2e-5."""
    from spo_b200 import capi, workload
    case = workload.config_case({"nz": 32, "nr": 24, "nx": 4, "ny": 4, "j_max": j_max, "mj_max": j_max,
                                 "nz_specular": 64, "nz_potential": 20})
    assert case.m["n_theta"] == j_max + 1 and case.m["n_phi"] == 2 * j_max + 2
    rng = np.random.default_rng(17)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    ref = make(case, "v1", "mixed")
    ref.read_wave_packet(psi0, chi0)
    ref.apply_stage(capi.STAGE_POTENTIAL)
    p_stage, c_stage = ref.wave_packet_on_host()
    ref.read_wave_packet(psi0, chi0)
    ref.propagate_analysis_step()
    p_step, c_step = ref.wave_packet_on_host()
    ref.close()
    for kernels in ("v2", "v3", "v5"):
        be = make(case, kernels, "mixed")
        assert f"potential=potential{kernels[1]}" in be.describe(), be.describe()
        if kernels == "v5":
            assert f"(theta {j_max + 1} padded)" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.apply_stage(capi.STAGE_POTENTIAL)
        p, c = be.wave_packet_on_host()
        assert rel_err(p, p_stage) < 2e-6 and rel_err(c, c_stage) < 2e-6, kernels
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        p, c = be.wave_packet_on_host()
        assert rel_l2(p, p_step) < 2e-5 and rel_l2(c, c_step) < 2e-5, kernels
        be.close()


@pytest.mark.parametrize("nxy", [8, 16, 6])
def test_potential6_agrees_with_potential5_and_the_general_kernel(nxy):
    """potential6 (both theta contractions as split-precision TF32 tcgen05 GEMMs, 64-column tiles) on the
    configuration-2 angular grid (theta 16 x phi 32, JMax = MJMax = 15, n_rot 256): one tile (8 x 8), four
    tiles (16 x 16) and a partial tile (6 x 6: 36 columns). The potential stage alone against the general
    kernel and potential5 to FP32 rounding (2e-6 of the largest value), then two analysis steps to 2e-5
    relative L2."""
    from spo_b200 import capi, workload
    case = workload.config_case({"nz": 24, "nr": 16, "nx": nxy, "ny": nxy, "j_max": 15, "mj_max": 15,
                                 "nz_specular": 64, "nz_potential": 14})
    assert case.m["n_theta"] == 16 and case.m["n_phi"] == 32 and case.n_rot == 256
    rng = np.random.default_rng(23)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    stage, step = {}, {}
    for kernels in ("v1", "v5", "v6"):
        be = make(case, kernels, "mixed")
        if kernels != "v1":
            assert f"potential=potential{kernels[1]}" in be.describe(), be.describe()
        be.read_wave_packet(psi0, chi0)
        be.apply_stage(capi.STAGE_POTENTIAL)
        stage[kernels] = be.wave_packet_on_host()
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        be.propagate_analysis_step()
        step[kernels] = be.wave_packet_on_host()
        be.close()
    for ref in ("v1", "v5"):
        assert rel_err(stage["v6"][0], stage[ref][0]) < 2e-6, (ref, rel_err(stage["v6"][0], stage[ref][0]))
        assert rel_err(stage["v6"][1], stage[ref][1]) < 2e-6, ref
        assert rel_l2(step["v6"][0], step[ref][0]) < 2e-5 and rel_l2(step["v6"][1], step[ref][1]) < 2e-5, ref
