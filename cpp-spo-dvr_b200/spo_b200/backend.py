"""B200Backend: the reference's PropagationBackend interface over the C ABI.

Mirrors spodvr::PropagationBackend (src/propagation/propagation_backend.hpp:34-59) member by
member, with the same layouts (src/propagation/wave_function.hpp) and the same meaning:

  read_wave_packet(psi, chi) ...... PropagationBackend::read_wave_packet (restart)
  wave_packet_on_host() ........... PropagationBackend::wave_packet_on_host (checkpoint, dump)
  propagate_analysis_step() ....... PropagationBackend::propagate_analysis_step
  specular() ...................... PropagationBackend::specular
  z_plane(iz) ..................... PropagationBackend::z_plane
  block_densities() ............... PropagationBackend::block_densities
  site_column(ixy) ................ PropagationBackend::site_column
  averages(...) ................... compute_averages (src/propagation/averages.cpp:37-80) on the device

Errors: the reference throws (InputError, CudaError); here a non-zero status raises B200Error
carrying the library's message. Construction takes a CaseBundle, the file form of BackendInput +
PotentialGrid + SpecularWave (propagation_backend.hpp:63-74).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import capi
from .case import CaseBundle


def _c(x):
    return np.ascontiguousarray(x, dtype=np.complex128)


def _f(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def _i(x):
    return np.ascontiguousarray(x, dtype=np.int32)


class B200Backend:
    """One wave packet resident on a B200, propagated by the sm_100a kernels of libspo_b200."""

    def __init__(self, case: CaseBundle, precision: str = "fp64", device: int = 0):
        self.case = case
        self._lib = capi.lib()
        m = case.m
        blocks = np.asarray(m["mj_blocks"], dtype=np.int32).reshape(-1, 3)
        keep = {
            "first": _i(blocks[:, 0]), "size": _i(blocks[:, 1]), "slot": _i(blocks[:, 2]),
        }
        for name in case.a:
            arr = case.a[name]
            keep[name] = _c(arr) if arr.dtype == np.complex128 else (_i(arr) if arr.dtype == np.int32 else _f(arr))
        self._keep = keep  # alive while the descriptor is read
        d = capi.SpoDesc()
        for key in ["n_rot", "nx", "ny", "nr", "nz", "nz_potential", "nz_specular", "n_theta", "n_phi",
                    "initial_channel", "r_absorber_first", "r_absorber_last", "steps_per_analysis", "n_rep",
                    "n_ops"]:
            setattr(d, key, int(m[key]))
        d.time_step = float(m["time_step"])
        for key in ["fft_scale_z", "fft_scale_r", "fft_scale_x", "fft_scale_y"]:
            setattr(d, key, float(m[key]))
        d.n_mj_blocks = int(blocks.shape[0])
        d.mj_fbr_first = capi.iptr(keep["first"])
        d.mj_fbr_size = capi.iptr(keep["size"])
        d.mj_phi_slot = capi.iptr(keep["slot"])
        for name in ["legendre", "z_kinetic_full", "z_kinetic_half", "r_kinetic_full", "r_kinetic_half",
                     "xy_kinetic_full", "xy_kinetic_half", "specular_kinetic_full", "specular_kinetic_half",
                     "rotation_half", "z_optical", "r_optical", "z_specular_optical", "gas_phase", "shift_forward",
                     "shift_backward", "specular_to_scattering", "scattering_to_specular", "potential",
                     "chi_initial"]:
            setattr(d, name, capi.dptr(keep[name]))
        for name in ["representative_of", "operation_of", "phi_index"]:
            setattr(d, name, capi.iptr(keep[name]))
        d.precision = capi.PRECISION_MIXED if precision == "mixed" else capi.PRECISION_FP64
        d.device = int(device)
        self.precision = precision
        h = ctypes.c_void_p()
        st = self._lib.spo_create(ctypes.byref(d), ctypes.byref(h))
        self._keep = None
        if st != capi.SPO_OK:
            raise capi.B200Error(st, self._lib.spo_last_error(None).decode())
        self._h = h

    # ------------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None):
            st = self._lib.spo_destroy(self._h)
            if st != capi.SPO_OK:  # a member of a live ensemble
                raise capi.B200Error(st, self._lib.spo_last_error(self._h).decode())
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int):
        if status != capi.SPO_OK:
            raise capi.B200Error(status, self._lib.spo_last_error(self._h).decode())

    # ------------------------------------------------------------------ PropagationBackend
    def read_wave_packet(self, psi: np.ndarray | None, chi: np.ndarray | None) -> None:
        p = None if psi is None else _c(psi).reshape(-1)
        c = None if chi is None else _c(chi).reshape(-1)
        if p is not None and p.size != int(np.prod(self.case.psi_shape)):
            raise ValueError("psi has the wrong size")
        if c is not None and c.size != int(np.prod(self.case.chi_shape)):
            raise ValueError("chi has the wrong size")
        self._check(self._lib.spo_upload_state(self._h, capi.dptr(p), capi.dptr(c)))

    def wave_packet_on_host(self):
        psi = np.empty(self.case.psi_shape, dtype=np.complex128)
        chi = np.empty(self.case.chi_shape, dtype=np.complex128)
        self._check(self._lib.spo_download_state(self._h, capi.dptr(psi), capi.dptr(chi)))
        return psi, chi

    def propagate_analysis_step(self) -> None:
        self._check(self._lib.spo_propagate_analysis_step(self._h))

    def specular(self, out: np.ndarray | None = None) -> np.ndarray:
        chi = np.empty(self.case.chi_shape, dtype=np.complex128) if out is None else out
        self._check(self._lib.spo_get_specular(self._h, capi.dptr(chi)))
        return chi

    def z_plane(self, iz: int, out: np.ndarray | None = None) -> np.ndarray:
        c = self.case
        plane = np.empty((c.nr, c.nx, c.ny, c.n_rot), dtype=np.complex128) if out is None else out
        self._check(self._lib.spo_get_z_plane(self._h, int(iz), capi.dptr(plane)))
        return plane

    def block_densities(self) -> np.ndarray:
        out = np.empty(self.case.nz * self.case.nr, dtype=np.float64)
        self._check(self._lib.spo_block_densities(self._h, capi.dptr(out)))
        return out

    def site_column(self, ixy: int) -> np.ndarray:
        c = self.case
        out = np.empty((c.n_rot, c.nz * c.nr), dtype=np.complex128)
        self._check(self._lib.spo_site_column(self._h, int(ixy), capi.dptr(out)))
        return out

    # ------------------------------------------------------------------ asymptotic analysis (FP64)
    def analysis_setup(self, analysis: dict, phi_vj: np.ndarray, energies_hartree: np.ndarray) -> None:
        """Balint-Kurti analysis data (AnalysisBasis, GasPhase, AnalysisEnergies of the reference):
        `analysis` holds n_v, n_rotation, n_diffraction, rotation_index, rotation_j, channel_ix,
        channel_iy, j_max_gas, initial_state, j_in, iz_analysis, dr, xy_scale, analysis_time_step."""
        a = analysis
        keep = {k: _i(a[k]) for k in ("rotation_index", "rotation_j", "channel_ix", "channel_iy")}
        keep["phi"] = _f(phi_vj)
        keep["e"] = _f(energies_hartree)
        d = capi.SpoAnalysisDesc()
        for k in ("n_v", "n_rotation", "n_diffraction", "j_max_gas", "initial_state", "j_in", "iz_analysis"):
            setattr(d, k, int(a[k]))
        for k in ("dr", "xy_scale", "analysis_time_step"):
            setattr(d, k, float(a[k]))
        for k in ("rotation_index", "rotation_j", "channel_ix", "channel_iy"):
            setattr(d, k, capi.iptr(keep[k]))
        d.phi_vj = capi.dptr(keep["phi"])
        d.n_energies = int(keep["e"].size)
        d.energies_hartree = capi.dptr(keep["e"])
        self._check(self._lib.spo_analysis_setup(self._h, ctypes.byref(d)))
        self._n_bk = int(a["n_v"]) * int(a["n_rotation"]) * int(a["n_diffraction"])
        self._n_e = int(keep["e"].size)

    def bk_coefficients(self, time: float = 0.0, surface_fixed: bool = False, surface_index: int = 0,
                        accumulate: bool = False) -> np.ndarray:
        """BK coefficients (n_v, n_states) of the current wave packet (BalintKurtiAnalyzer::coefficients)."""
        out = np.empty(self._n_bk, dtype=np.complex128)
        self._check(self._lib.spo_bk_coefficients(self._h, float(time), 1 if surface_fixed else 0,
                                                  int(surface_index), 1 if accumulate else 0, capi.dptr(out)))
        return out

    def s_matrix_sums(self) -> np.ndarray:
        """(n_energies, n_v * n_states): sum_t c(t) exp(i E t) dt_analysis (SMatrixAccumulator::add)."""
        out = np.empty(self._n_e * self._n_bk, dtype=np.complex128)
        self._check(self._lib.spo_s_matrix_sums(self._h, capi.dptr(out)))
        return out.reshape(self._n_e, self._n_bk)

    # ------------------------------------------------------------------ diagnostics
    def apply_stage(self, stage: int, half: bool = False) -> None:
        self._check(self._lib.spo_apply_stage(self._h, int(stage), 1 if half else 0))

    def set_stream(self, cuda_stream: int | None) -> None:
        """Run on the caller's cudaStream_t (an integer handle, e.g. torch.cuda.Stream().cuda_stream)."""
        self._check(self._lib.spo_set_stream(self._h, ctypes.c_void_p(cuda_stream or 0)))

    def norm_budget_setup(self, volume_scattering: float, volume_specular: float, z_low=None, zs_low=None) -> int:
        """The norm budget's tables on the device (NormBudget's constructor); returns the number of absorbers.
        z_low / zs_low: (first, last) of the low-Z absorber of each grid, or None."""
        d = capi.NormBudgetDesc(z_low[0] if z_low else -1, z_low[1] if z_low else -1,
                                zs_low[0] if zs_low else -1, zs_low[1] if zs_low else -1,
                                volume_scattering, volume_specular)
        n = ctypes.c_int(0)
        self._check(self._lib.spo_norm_budget_setup(self._h, ctypes.byref(d), ctypes.byref(n)))
        self._budget_absorbers = n.value
        return n.value

    def norm_budget_add(self):
        """NormBudget::add on the resident state: None at the first call, else (loss, loss_error, norm_start,
        norm_end) of the window since the previous call."""
        n = self._budget_absorbers
        loss, err, norms = np.zeros(n), np.zeros(n), np.zeros(2)
        has = ctypes.c_int(0)
        self._check(self._lib.spo_norm_budget_add(self._h, capi.dptr(loss), capi.dptr(err), capi.dptr(norms),
                                                  ctypes.byref(has)))
        return (loss, err, float(norms[0]), float(norms[1])) if has.value else None

    def test_wait_timeout(self, poll_limit: int, unmatched_bytes: int) -> None:
        """Failure-detection test of the bounded device waits (spo_test_wait_timeout): the potential kernel's
        barriers expect unmatched_bytes more than their copies deliver and give up after poll_limit polls;
        (0, 0) restores normal operation."""
        self._check(self._lib.spo_test_wait_timeout(self._h, poll_limit, unmatched_bytes))

    def profile(self, enable: bool) -> None:
        self._check(self._lib.spo_profile(self._h, 1 if enable else 0))

    def profile_records(self) -> list[dict]:
        n = ctypes.c_int()
        self._check(self._lib.spo_profile_count(self._h, ctypes.byref(n)))
        out = []
        for i in range(n.value):
            name = ctypes.create_string_buffer(64)
            ms, launches, nbytes = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
            self._check(self._lib.spo_profile_entry(self._h, i, name, 64, ctypes.byref(ms), ctypes.byref(launches),
                                                    ctypes.byref(nbytes)))
            out.append({"name": name.value.decode(), "ms": ms.value, "launches": launches.value,
                        "bytes_per_launch": nbytes.value})
        return out

    def device_bytes(self) -> int:
        v = ctypes.c_ulonglong()
        self._check(self._lib.spo_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    def last_launch_count(self) -> int:
        v = ctypes.c_int()
        self._check(self._lib.spo_last_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def describe(self) -> str:
        """The kernels and tile widths this handle uses, and whether the autotuner chose them."""
        buf = ctypes.create_string_buffer(512)
        self._check(self._lib.spo_describe(self._h, buf, 512))
        return buf.value.decode()

    def averages(self, z: np.ndarray, z_specular: np.ndarray, r: np.ndarray, volume_scattering: float,
                 volume_specular: float, iz_analysis: int, surface_index: int) -> np.ndarray:
        """[norm, <Z>, <r>, rest norm] of the resident wave packet, in FP64 on the device."""
        z, zs, r = _f(z), _f(z_specular), _f(r)
        if len(z) != self.case.nz or len(zs) != self.case.nz_specular or len(r) != self.case.nr:
            raise ValueError("averages: grid lengths must be nz, nz_specular and nr")
        out = np.empty(4)
        self._check(self._lib.spo_averages(self._h, capi.dptr(z), capi.dptr(zs), capi.dptr(r),
                                           float(volume_scattering), float(volume_specular), int(iz_analysis),
                                           int(surface_index), capi.dptr(out)))
        return out


class Ensemble:
    """Several B200Backend wave packets advanced together: one analysis step of every member is one
    CUDA graph launch (spo_ensemble_* of include/spo_b200.h). Members may differ in grid sizes and
    precision; each keeps its own state and stays usable on its own between ensemble steps."""

    def __init__(self, members: list[B200Backend]):
        if not members:
            raise ValueError("an ensemble needs at least one member")
        self._lib = capi.lib()
        self.members = list(members)  # the graph holds their device pointers: keep them alive
        arr = (ctypes.c_void_p * len(self.members))(*[m._h for m in self.members])
        e = ctypes.c_void_p()
        status = self._lib.spo_ensemble_create(arr, len(self.members), ctypes.byref(e))
        if status != 0:
            raise capi.B200Error(status, self._lib.spo_ensemble_last_error(None).decode())
        self._e = e

    def _check(self, status: int):
        if status != 0:
            raise capi.B200Error(status, self._lib.spo_ensemble_last_error(self._e).decode())

    def propagate_analysis_step(self) -> None:
        """One analysis step of every member (one graph launch); returns when all are done."""
        self._check(self._lib.spo_ensemble_step(self._e))

    def launch_count(self) -> int:
        v = ctypes.c_int()
        self._check(self._lib.spo_ensemble_launch_count(self._e, ctypes.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_e", None):
            self._lib.spo_ensemble_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
