"""Ensembles of wave packets of uneven grid sizes, one CUDA graph launch per analysis step (needs a B200).

Each member keeps its own tables and state, so an ensemble step must give every member exactly the
wave packet that spo_propagate_analysis_step gives the same packet alone: bitwise, since the graph
replays the same kernels on the same data. The members below differ in every size (Z, r, x, y, the
angular basis, the specular grid) and in precision.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [
    ({"nz": 64, "nr": 24, "nx": 8, "ny": 8, "j_max": 5, "mj_max": 5, "nz_specular": 128, "nz_potential": 40}, "mixed"),
    ({"nz": 48, "nr": 32, "nx": 4, "ny": 4, "j_max": 7, "mj_max": 7, "nz_specular": 96, "nz_potential": 30}, "fp64"),
    ({"nz": 128, "nr": 24, "nx": 16, "ny": 16, "j_max": 3, "mj_max": 3, "nz_specular": 256, "nz_potential": 64},
     "mixed"),
]


def random_state(case, seed):
    rng = np.random.default_rng(seed)
    psi = (rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)) * 1e-2
    chi = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    return psi, chi


@pytest.mark.parametrize("chain", ["overlapped", "chained"])
def test_ensemble_steps_equal_each_member_alone(chain, monkeypatch):
    """Both graph shapes: members overlapped between the fork and the join (small members), and chained one
    after another (members that fill the GPU; forced here by a zero size threshold)."""
    from spo_b200 import B200Backend, Ensemble, workload

    if chain == "chained":
        monkeypatch.setenv("SPO_B200_ENSEMBLE_CHAIN_BYTES", "0")
    else:
        monkeypatch.delenv("SPO_B200_ENSEMBLE_CHAIN_BYTES", raising=False)

    cases = [workload.config_case(cfg) for cfg, _ in MEMBERS]
    states = [random_state(c, 100 + i) for i, c in enumerate(cases)]
    alone = []
    for (cfg, precision), case, (psi, chi) in zip(MEMBERS, cases, states):
        with B200Backend(case, precision=precision) as be:
            be.read_wave_packet(psi, chi)
            out = []
            for _ in range(2):
                be.propagate_analysis_step()
                out.append(be.wave_packet_on_host())
            alone.append((out, be.last_launch_count()))

    members = [B200Backend(case, precision=p) for (_, p), case in zip(MEMBERS, cases)]
    for be, (psi, chi) in zip(members, states):
        be.read_wave_packet(psi, chi)
    with Ensemble(members) as ens:
        assert ens.launch_count() == sum(n for _, n in alone)
        for step in range(2):
            ens.propagate_analysis_step()
            for k, be in enumerate(members):
                psi, chi = be.wave_packet_on_host()
                ref_psi, ref_chi = alone[k][0][step]
                assert np.array_equal(psi, ref_psi), (k, step)
                assert np.array_equal(chi, ref_chi), (k, step)
    for be in members:
        be.close()


def test_a_member_of_a_live_ensemble_cannot_be_destroyed():
    from spo_b200 import B200Backend, B200Error, Ensemble, workload

    cfg, precision = MEMBERS[1]
    be = B200Backend(workload.config_case(cfg), precision=precision)
    ens = Ensemble([be])
    with pytest.raises(B200Error, match="live ensemble"):
        be.close()
    ens.close()
    be.close()


def test_ensemble_refuses_a_member_twice():
    from spo_b200 import B200Backend, B200Error, Ensemble, workload

    cfg, precision = MEMBERS[1]
    with B200Backend(workload.config_case(cfg), precision=precision) as be:
        with pytest.raises(B200Error, match="appears twice"):
            Ensemble([be, be])
