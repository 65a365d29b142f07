"""The norm budget on the device (spo_norm_budget_*) against its numpy restatement (needs a B200).

NormBudget (src/analysis/norm_budget.cpp) is fed the cell probabilities after every analysis step; its windows
give the probability each absorber removed. The device computes the cells from the resident state and sums the
windows in FP64; oracle/norm_budget_oracle.py restates the reference's formulas on the same state read back
(block densities and the specular wave, both FP64). Bar: 1e-12 of the window's norm (sums in another order).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_norm_budget_matches_oracle(precision):
    import norm_budget_oracle

    from spo_b200 import B200Backend, workload
    case = workload.config_case({"nz": 48, "nr": 24, "nx": 4, "ny": 4, "j_max": 3, "mj_max": 3, "nz_specular": 96,
                                 "nz_potential": 30})
    vols = (0.12 * 0.16 * 0.3, 0.12 * 0.16)
    z_low, zs_low = (0, 3), (0, 2)
    a = case.a
    z_opt = a["z_optical"].copy()
    z_opt[:4] = np.exp(-0.01 * np.arange(4, 0, -1))  # a low-Z absorber over iz = 0..3
    zs_opt = a["z_specular_optical"].copy()
    zs_opt[:3] = np.exp(-0.02 * np.arange(3, 0, -1))
    a["z_optical"], a["z_specular_optical"] = z_opt, zs_opt
    ref = norm_budget_oracle.NormBudgetOracle(z_opt, a["r_optical"], zs_opt, case.steps_per_analysis, vols[0],
                                              vols[1], z_low, zs_low)
    rng = np.random.default_rng(4)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    with B200Backend(case, precision=precision) as be:
        assert be.norm_budget_setup(vols[0], vols[1], z_low, zs_low) == ref.n == 6
        be.read_wave_packet(psi0, chi0)
        windows = 0
        for step in range(4):
            got = be.norm_budget_add()
            want = ref.add(be.block_densities(), be.specular())
            assert (got is None) == (want is None)
            if got is not None:
                windows += 1
                scale = want[3]
                assert np.max(np.abs(got[0] - want[0])) <= 1e-12 * scale, (got[0], want[0])
                assert np.max(np.abs(got[1] - want[1])) <= 1e-12 * scale
                assert abs(got[2] - want[2]) <= 1e-12 * scale and abs(got[3] - want[3]) <= 1e-12 * scale
                assert np.all(want[0] >= -1e-12 * scale) and want[0].sum() > 0
            be.propagate_analysis_step()
        assert windows == 3
