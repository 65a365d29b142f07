"""spo_block_densities_noalloc against spo_block_densities (needs a B200).

The no-allocation entry point serves callers whose device memory belongs to their own pool allocator
and who therefore may not call cudaMalloc: they keep the wave packet in their own device buffers
(here a torch tensor, allocated by torch's caching allocator) and pass its address. Its per-block sums
go through the library's fixed device array, so two calls in a row must each give the densities of
their own input, equal to what a handle computes with its own scratch allocation.

This file is collected last, so that a run that stops at the first failure has run every other test.
It needs nothing from the other tests and runs alone in a fresh process.
"""

import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "cpp-spo-dvr_b200"))

pytestmark = pytest.mark.gpu


def small_case():
    from spo_b200 import workload
    return workload.config_case({"nz": 32, "nr": 24, "nx": 4, "ny": 4, "j_max": 5, "mj_max": 5, "nz_specular": 64,
                                 "nz_potential": 20})


def noalloc_densities(lib, tensor, precision, n_blocks, block_size, stream):
    from spo_b200 import capi
    out = np.empty(n_blocks, dtype=np.float64)
    st = lib.spo_block_densities_noalloc(ctypes.c_void_p(tensor.data_ptr()), precision, n_blocks, block_size,
                                         capi.dptr(out), ctypes.c_void_p(stream))
    assert st == capi.SPO_OK, lib.spo_last_error(None).decode()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_block_densities_match_the_handle_on_two_calls(precision):
    import torch

    from spo_b200 import B200Backend, capi

    lib = capi.lib()
    case = small_case()
    n_blocks = case.nz * case.nr
    block_size = case.nx * case.ny * case.n_rot
    rng = np.random.default_rng(11)
    dtype = torch.complex128 if precision == "fp64" else torch.complex64
    code = capi.PRECISION_FP64 if precision == "fp64" else capi.PRECISION_MIXED
    stream = torch.cuda.current_stream().cuda_stream
    with B200Backend(case, precision=precision) as be:
        for call in range(2):  # two calls in a row, different data: no state carried between them
            psi = (rng.standard_normal(case.psi_shape) + 1j * rng.standard_normal(case.psi_shape)) * (call + 1)
            chi = np.zeros(case.chi_shape, dtype=np.complex128)
            be.read_wave_packet(psi, chi)
            expected = be.block_densities()
            tensor = torch.from_numpy(np.ascontiguousarray(psi.reshape(-1))).to(dtype).cuda()
            torch.cuda.synchronize()
            got = noalloc_densities(lib, tensor, code, n_blocks, block_size, stream)
            assert np.max(np.abs(got - expected)) <= 1e-13 * np.max(expected), (call, precision)


def test_noalloc_refuses_sizes_beyond_its_limit():
    import torch

    from spo_b200 import capi

    lib = capi.lib()
    tensor = torch.zeros(16, dtype=torch.complex128, device="cuda")
    out = np.empty(1, dtype=np.float64)
    st = lib.spo_block_densities_noalloc(ctypes.c_void_p(tensor.data_ptr()), capi.PRECISION_FP64,
                                         capi.NOALLOC_MAX_BLOCKS + 1, 1, capi.dptr(out), None)
    assert st == capi.SPO_ERR_INVALID
    assert "exceeds SPO_NOALLOC_MAX_BLOCKS" in lib.spo_last_error(None).decode()


def test_noalloc_at_exactly_its_limit():
    """n_blocks = SPO_NOALLOC_MAX_BLOCKS: the last element of the shared array and the full grid are used."""
    import torch

    from spo_b200 import capi

    lib = capi.lib()
    n_blocks, block_size = capi.NOALLOC_MAX_BLOCKS, 4
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((n_blocks, block_size)) + 1j * rng.standard_normal((n_blocks, block_size))
    psi[-1] *= 3.0  # a distinct last block
    expected = np.sum(np.abs(psi) ** 2, axis=1)
    tensor = torch.from_numpy(psi.reshape(-1)).cuda()
    torch.cuda.synchronize()
    for _ in range(2):
        got = noalloc_densities(lib, tensor, capi.PRECISION_FP64, n_blocks, block_size,
                                torch.cuda.current_stream().cuda_stream)
        assert np.max(np.abs(got - expected)) <= 1e-13 * np.max(expected)
