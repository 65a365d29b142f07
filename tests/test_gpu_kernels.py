"""The register-DFT kernels against the general kernels, on the shapes of the benchmark configuration
(needs a B200).

The tiny regression cases (test_gpu_parity.py) run the register-DFT kernels at their own sizes
against the oracle. The configuration-2 sizes (axis lengths 128 = 16 x 8 and 48 = 8 x 6, a 16 x 16
(x, y) grid, nphi 32 with ntheta 16) use other instantiations; here they are checked operator by
operator and over an analysis step against the general shared-memory Stockham kernels
(SPO_B200_KERNELS=v1), which the oracle checks on every case.
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


def make(case, kernels, precision):
    from spo_b200 import B200Backend
    old = os.environ.get("SPO_B200_KERNELS")
    os.environ["SPO_B200_KERNELS"] = kernels
    try:
        return B200Backend(case, precision=precision)
    finally:
        if old is None:
            del os.environ["SPO_B200_KERNELS"]
        else:
            os.environ["SPO_B200_KERNELS"] = old


@pytest.mark.parametrize("shape", list(SHAPES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_register_kernels_match_general_kernels(shape, precision):
    from spo_b200 import capi, workload
    case = workload.config_case(SHAPES[shape])
    rng = np.random.default_rng(5)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    tol_stage, tol_step = (1e-12, 1e-11) if precision == "fp64" else (2e-6, 2e-5)
    ref = make(case, "v1", precision)
    new = make(case, "v2", precision)
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
