"""The benchmarked kernels against the oracle on the benchmark's own input (needs a B200).

The configuration-2 input (tests/golden/inputs/config2_dz.json: Dai-Light PES, nZ 128, nR 48, theta 16 x phi
32, n_rot 256, nZSpecular 512) is set up by the reference itself (oracle/_ref/spo_ref_tool, the reference
compiled from its sources), with the reference GPU tests' LCG wave packet over the whole grid
(tests/cuda/cuda_test_setup.hpp:53-64 of the reference), and propagated by the reference's CpuBackend for one
analysis step (5 time steps). The same case bundle and packet then go through the C ABI:
  - nX = nY = 16 is the benchmark's grid itself: the FP64 form runs the kernels the FP64 line times
    (axis2b<128>, axis2pfa<48=3x16>, xy2p<16>, potential4<32,16>), the mixed form those of the headline
    (potential5<32,16> with exp(i A) rows through L2);
  - nX = nY = 4 runs the same Z, r and potential kernels on a smaller (x, y) grid.
Bars: the FP64 bar (relative L2 1e-10) and the mixed form's 3e-5, on psi and chi.
"""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, read_c128, rel_l2

pytestmark = pytest.mark.gpu


def config2_input(tmp_path, nx):
    cfg = json.load(open(os.path.join(GOLDEN, "inputs", "config2_dz.json")))
    cfg.update({"nX": nx, "nY": nx})
    path = tmp_path / f"config2_nx{nx}.json"
    path.write_text(json.dumps(cfg))
    return str(path)


@pytest.mark.parametrize("nx", [4, 16])
def test_config2_analysis_step_matches_oracle(ref_case, tmp_path, nx):
    from spo_b200 import B200Backend, CaseBundle

    d = ref_case(f"config2_nx{nx}", seed=7, analysis_steps=1, stages=False, input_path=config2_input(tmp_path, nx))
    case = CaseBundle.load(os.path.join(d, "case"))
    assert (case.nz, case.nr, case.nx, case.n_theta, case.n_phi, case.n_rot) == (128, 48, nx, 16, 32, 256)
    psi0 = read_c128(os.path.join(d, "psi_initial.c128"), case.psi_shape)
    chi0 = read_c128(os.path.join(d, "chi_start.c128"), case.chi_shape)
    ref_psi = read_c128(os.path.join(d, "psi_final.c128"), case.psi_shape)
    ref_chi = read_c128(os.path.join(d, "chi_steps.c128"), case.chi_shape)
    for precision, bar in (("fp64", 1e-10), ("mixed", 3e-5)):
        with B200Backend(case, precision=precision) as be:
            be.read_wave_packet(psi0, chi0)
            be.propagate_analysis_step()
            psi, chi = be.wave_packet_on_host()
            kernels = be.describe()
        e_psi, e_chi = rel_l2(psi, ref_psi), rel_l2(chi, ref_chi)
        print(f"config 2, nX = nY = {nx}, {precision}: rel-L2 psi {e_psi:.2e} chi {e_chi:.2e}; {kernels}")
        assert e_psi < bar and e_chi < bar, (precision, e_psi, e_chi)
        if nx == 16:
            if precision == "fp64":
                assert "potential4<nphi=32,nt=16" in kernels and "xy2p<16" in kernels, kernels
            else:
                assert "potential5<nphi=32,nt=16" in kernels, kernels
        del psi
