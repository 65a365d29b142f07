"""Failure detection of the bounded device-side waits, without a GPU fault (needs a B200).

potential5 and potential6 move each item's data by bulk asynchronous copies whose completion is counted in
bytes on an mbarrier, and every wait on a barrier is bounded. spo_test_wait_timeout makes every item's
first barrier announce 16 bytes more than its copies deliver: every copy is valid and lands, but the
barrier's phase cannot complete. Each block's wait then gives up after a short poll limit, the block sets
the device error flag, waits (bounded) for its own work in flight, frees its tensor memory and leaves, and
the step returns SPO_ERR_TIMEOUT with the context intact. After the hook is cleared and the wave packet is
uploaded again, the next step is bitwise the step of a handle that never failed.
"""

import numpy as np
import pytest

from test_gpu_kernels import make

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernels", ["v5", "v6"])
def test_a_wait_that_gives_up_returns_timeout_and_the_handle_recovers(kernels):
    from spo_b200 import capi, workload
    case = workload.config_case({"nz": 24, "nr": 16, "nx": 8, "ny": 8, "j_max": 15, "mj_max": 15,
                                 "nz_specular": 64, "nz_potential": 14})
    rng = np.random.default_rng(31)
    psi0 = rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)
    chi0 = rng.standard_normal(case.chi_shape) + 1j * rng.standard_normal(case.chi_shape)
    with make(case, kernels, "mixed") as ref:
        assert f"potential=potential{kernels[1]}" in ref.describe(), ref.describe()
        ref.read_wave_packet(psi0, chi0)
        ref.propagate_analysis_step()
        expected = ref.wave_packet_on_host()
    with make(case, kernels, "mixed") as be:
        be.read_wave_packet(psi0, chi0)
        be.test_wait_timeout(1 << 16, 16)
        with pytest.raises(capi.B200Error) as err:
            be.propagate_analysis_step()
        assert err.value.status == capi.SPO_ERR_TIMEOUT, str(err.value)
        assert "gave up" in str(err.value)
        be.test_wait_timeout(0, 0)
        be.read_wave_packet(psi0, chi0)
        be.propagate_analysis_step()
        psi, chi = be.wave_packet_on_host()
    assert np.array_equal(psi, expected[0]) and np.array_equal(chi, expected[1])


def test_unmatched_bytes_must_be_a_multiple_of_16():
    from spo_b200 import capi, workload
    case = workload.config_case({"nz": 16, "nr": 16, "nx": 4, "ny": 4, "j_max": 3, "mj_max": 3,
                                 "nz_specular": 32, "nz_potential": 8})
    with make(case, "v5", "mixed") as be:
        with pytest.raises(capi.B200Error) as err:
            be.test_wait_timeout(100, 8)
        assert err.value.status == capi.SPO_ERR_INVALID
