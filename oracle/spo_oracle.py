"""CPU restatement of the split-operator propagation step of SPO-DVR, in numpy (FP64).

Test infrastructure: only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker. It is never called by the product path.

It restates, operator by operator, what the reference's CPU backend does in one analysis step
(file:line citations are into the reference project, SPO-DVR):

* ``analysis_step_schedule`` ....... src/propagation/split_operator_schedule.cpp:7-13
* ``propagate_analysis_step`` ...... src/propagation/split_operator.cpp:11-46
* ``specular_apply`` ............... src/propagation/specular_operator.cpp:40-71
* ``kinetic_zr`` ................... src/propagation/kinetic_operators.cpp:77-111
* ``kinetic_xy`` ................... src/propagation/kinetic_operators.cpp:134-172
* ``potential_apply`` .............. src/propagation/potential_operator.cpp:95-145, 158-201
* ``fbr_to_dvr`` / ``dvr_to_fbr`` .. src/propagation/angular_transform.cpp:54-114
* ``bk_coefficients`` .............. src/analysis/balint_kurti.cpp:39-84
* ``block_densities`` .............. src/propagation/averages.cpp:20-29
* ``averages`` ..................... src/propagation/averages.cpp:37-80

Its inputs are a *case bundle*: the data that cross the reference's PropagationBackend boundary
(src/propagation/propagation_backend.hpp:63-74: the tables, the angular transform matrices, the
symmetry maps, the potential grid and the initial specular wave), written by oracle/ref_tool.cpp.

Layouts (as the reference's host layout, src/propagation/wave_function.hpp:14-53):
  psi: numpy array (nz, nr, nx, ny, n_rot), i.e. flat index irot + n_rot*(iy + ny*(ix + nx*(ir + nr*iz)))
  chi: numpy array (nz_specular, nr), i.e. flat index ir + nr*iz

Parity: this restatement is pinned against the reference compiled from its own sources
(oracle/_ref, oracle/Makefile) on the same inputs, and that build against the reference's
Fortran regression fixtures (tests/golden).
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np


# --------------------------------------------------------------------------------------------
# Case bundle
# --------------------------------------------------------------------------------------------

@dataclass
class Case:
    """The boundary data of one run (what a PropagationBackend is built from)."""

    m: dict          # manifest: sizes and scalars
    t: dict          # arrays by name
    analysis: dict | None = None

    def __getattr__(self, name):
        m = self.__dict__.get("m")
        if m is not None and name in m:
            return m[name]
        raise AttributeError(name)

    @property
    def n_xy(self) -> int:
        return self.nx * self.ny


_ARRAYS_C128 = [
    "z_kinetic_full", "z_kinetic_half", "r_kinetic_full", "r_kinetic_half",
    "zr_kinetic_full", "zr_kinetic_half", "xy_kinetic_full", "xy_kinetic_half",
    "specular_kinetic_full", "specular_kinetic_half", "rotation_full", "rotation_half",
    "gas_phase", "shift_forward", "shift_backward", "specular_to_scattering",
    "scattering_to_specular", "chi_initial",
]
_ARRAYS_F64 = ["z_optical", "r_optical", "z_specular_optical", "xy_kinetic_energies",
               "rotational_energies", "legendre", "potential", "asymptotic"]
_ARRAYS_I32 = ["representative_of", "operation_of", "phi_index"]


def load_case(directory: str) -> Case:
    """Reads a bundle written by ``spo_ref_tool case`` (or by the synthetic workload builder)."""
    with open(os.path.join(directory, "manifest.json")) as f:
        m = json.load(f)
    t = {}
    for name in _ARRAYS_C128:
        t[name] = np.fromfile(os.path.join(directory, name + ".c128"), dtype=np.complex128)
    for name in _ARRAYS_F64:
        t[name] = np.fromfile(os.path.join(directory, name + ".f64"), dtype=np.float64)
    for name in _ARRAYS_I32:
        t[name] = np.fromfile(os.path.join(directory, name + ".i32"), dtype=np.int32)
    analysis = None
    apath = os.path.join(directory, "analysis.json")
    if os.path.exists(apath):
        with open(apath) as f:
            analysis = json.load(f)
        analysis["phi_vj"] = np.fromfile(os.path.join(directory, "phi_vj.f64"), dtype=np.float64)
    return Case(m=m, t=t, analysis=analysis)


def lcg_complex(n: int, seed: int) -> np.ndarray:
    """The reference GPU tests' 64-bit LCG (tests/cuda/cuda_test_setup.hpp:53-64): values in [-1, 1),
    real part then imaginary part per element. Vectorised by jumping ahead: x_(k+i) = A_i x_k + C_i."""
    mask = (1 << 64) - 1
    a, c = 6364136223846793005, 1442695040888963407
    block = 4096
    a_pow, c_pow = [], []
    ak, ck = 1, 0
    for _ in range(block):
        ak = (ak * a) & mask
        ck = (ck * a + c) & mask
        a_pow.append(ak)
        c_pow.append(ck)
    A = np.array(a_pow, dtype=np.uint64)
    C = np.array(c_pow, dtype=np.uint64)
    total = 2 * n
    out = np.empty(total, dtype=np.float64)
    x = np.uint64(seed & mask)
    done = 0
    with np.errstate(over="ignore"):
        while done < total:
            m = min(block, total - done)
            xs = A[:m] * x + C[:m]
            out[done:done + m] = (xs >> np.uint64(11)).astype(np.float64) / float(1 << 53) * 2.0 - 1.0
            x = xs[m - 1]
            done += m
    return out[0::2] + 1j * out[1::2]


# --------------------------------------------------------------------------------------------
# Operators
# --------------------------------------------------------------------------------------------

FULL, HALF = "full", "half"


def analysis_step_schedule(steps_per_analysis: int):
    """[(step, kinetic_only)]: T/2 V, (T V) n-1 times, T/2 (split_operator_schedule.cpp:7-13)."""
    s = [(HALF, False)]
    s += [(FULL, False)] * (steps_per_analysis - 1)
    s.append((HALF, True))
    return s


def _factors(case: Case, name: str, step: str) -> np.ndarray:
    return case.t[f"{name}_{step}"]


def specular_apply(chi: np.ndarray, case: Case, step: str, kinetic_only: bool) -> np.ndarray:
    """SpecularOperator::apply (specular_operator.cpp:40-71). chi: (nz_specular, nr)."""
    nzs, nr = chi.shape
    sz, sr = case.fft_scale_z, case.fft_scale_r
    f = _factors(case, "specular_kinetic", step).reshape(nzs, nr)
    x = np.fft.fft2(chi) * (sz * sr)                      # sign -1, then the forward scale
    x = f * x
    x = np.fft.ifft2(x) * (nzs * nr) * ((1.0 / (nzs * sz)) * (1.0 / (nr * sr)))  # sign +1, inverse scale
    if kinetic_only:
        return x
    i0 = case.initial_channel
    rot = case.t["rotation_half"].reshape(nr, case.n_rot)[:, i0]
    gas = rot * case.t["gas_phase"] * rot                  # specular_gas_phase_factors
    x[case.nz_potential:, :] = gas[None, :] * x[case.nz_potential:, :]
    x = case.t["z_specular_optical"][:, None] * x
    if nr != 1:
        a, b = case.r_absorber_first, case.r_absorber_last
        x[:, a:b + 1] = case.t["r_optical"][None, a:b + 1] * x[:, a:b + 1]
    return x


def kinetic_zr(psi: np.ndarray, case: Case, step: str) -> np.ndarray:
    """exp(-i (T_Z + T_r) dt) by a 2D (Z, r) FFT (kinetic_operators.cpp:77-111)."""
    nz, nr = psi.shape[0], psi.shape[1]
    sz, sr = case.fft_scale_z, case.fft_scale_r
    f = _factors(case, "zr_kinetic", step).reshape(nz, nr)
    x = np.fft.fftn(psi, axes=(0, 1)) * (sz * sr)
    x = f[:, :, None, None, None] * x
    return np.fft.ifftn(x, axes=(0, 1)) * (nz * nr) * ((1.0 / (nz * sz)) * (1.0 / (nr * sr)))


def kinetic_xy(psi: np.ndarray, case: Case, step: str) -> np.ndarray:
    """exp(-i T_xy dt) with the momentum shift (kinetic_operators.cpp:134-172)."""
    nx, ny = case.nx, case.ny
    sx = case.fft_scale_x if nx > 1 else 1.0
    sy = case.fft_scale_y if ny > 1 else 1.0
    f = _factors(case, "xy_kinetic", step).reshape(nx, ny)
    fwd = case.t["shift_forward"].reshape(nx, ny)
    shift = not np.all((fwd.real == 1.0) & (fwd.imag == 0.0))
    x = psi
    if shift:
        x = x * fwd[None, None, :, :, None]
    x = np.fft.fftn(x, axes=(2, 3)) * (sx * sy)
    x = f[None, None, :, :, None] * x
    x = np.fft.ifftn(x, axes=(2, 3)) * (nx * ny) * ((1.0 / (nx * sx)) * (1.0 / (ny * sy)))
    if shift:
        x = x * case.t["shift_backward"].reshape(nx, ny)[None, None, :, :, None]
    return x


def _mj_blocks(case: Case):
    """[(fbr_first, n_j, phi_slot, offset into legendre)] in mJ order (angular_transform.cpp:16-44)."""
    out = []
    off = 0
    for first, size, slot in case.mj_blocks:
        out.append((first, size, slot, off))
        off += case.n_theta * size
    return out


def fbr_to_dvr(c: np.ndarray, case: Case) -> np.ndarray:
    """FBR -> DVR (angular_transform.cpp:54-91). c: (..., n_rot) -> (..., n_theta, n_phi)."""
    nt, nphi = case.n_theta, case.n_phi
    dvr = np.zeros(c.shape[:-1] + (nt, nphi), dtype=np.complex128)
    M = case.t["legendre"]
    for first, nj, slot, off in _mj_blocks(case):
        mat = M[off:off + nt * nj].reshape(nt, nj)            # (theta, J)
        dvr[..., :, slot] = c[..., first:first + nj] @ mat.T
    return np.fft.ifft(dvr, axis=-1) * nphi                    # sign +1, scale 1


def dvr_to_fbr(dvr: np.ndarray, case: Case) -> np.ndarray:
    """DVR -> FBR (angular_transform.cpp:94-114): sign -1 phi FFT, then the transposed sums."""
    nt = case.n_theta
    x = np.fft.fft(dvr, axis=-1)
    c = np.zeros(dvr.shape[:-2] + (case.n_rot,), dtype=np.complex128)
    M = case.t["legendre"]
    for first, nj, slot, off in _mj_blocks(case):
        mat = M[off:off + nt * nj].reshape(nt, nj)
        c[..., first:first + nj] = x[..., :, slot] @ mat
    return c


def exp_potential(case: Case) -> np.ndarray:
    """exp(i A), A = -V dt, on the full (iz, ir, ixy, theta, phi) grid of the interaction region,
    through the symmetry maps (potential_operator.cpp:55-65, 187-195; potential_grid.hpp:28-36)."""
    nzp, nr, nt, nphi = case.nz_potential, case.nr, case.n_theta, case.n_phi
    n_rep = case.n_rep
    V = case.t["potential"].reshape(nzp, nr, n_rep, nt, nphi)   # (izr, irep, itp) reversed
    A = -V * case.time_step                                     # premultiply_with_time_step
    rep = case.t["representative_of"]
    op = case.t["operation_of"]
    phi_index = case.t["phi_index"].reshape(case.n_ops, nphi)
    idx_phi = phi_index[op]                                      # (n_xy, nphi)
    full = A[:, :, rep, :, :]                                    # (nzp, nr, n_xy, nt, nphi)
    full = np.take_along_axis(full, idx_phi[None, None, :, None, :].repeat(nt, axis=3), axis=4)
    return np.cos(full) + 1j * np.sin(full)


def potential_apply(psi: np.ndarray, chi: np.ndarray, case: Case, expia: np.ndarray | None = None):
    """PotentialOperator::apply_block for every (Z, r) point (potential_operator.cpp:95-136).
    Returns (psi, chi)."""
    nz, nr, nx, ny, n_rot = psi.shape
    nzp = case.nz_potential
    i0 = case.initial_channel
    rot_half = case.t["rotation_half"].reshape(nr, n_rot)
    opt_r = case.t["r_optical"] if nr != 1 else np.ones(nr)
    before = opt_r[:, None] * rot_half
    gas_step = opt_r[:, None] * rot_half * case.t["gas_phase"][:, None] * rot_half
    opt_z = case.t["z_optical"]
    sp2sc = case.t["specular_to_scattering"].reshape(nx, ny)
    sc2sp = case.t["scattering_to_specular"].reshape(nx, ny)
    psi = psi.copy()
    chi = chi.copy()
    # Gas-phase region.
    psi[nzp:] = opt_z[nzp:, None, None, None, None] * (gas_step[None, :, None, None, :] * psi[nzp:])
    # Interaction region.
    w = opt_z[:nzp, None, None, None, None] * (before[None, :, None, None, :] * psi[:nzp])
    incoming = chi[:nzp, :]                                      # (iz, ir)
    w[..., i0] = w[..., i0] + rot_half[None, :, None, None, i0] * (sp2sc[None, None] * incoming[:, :, None, None])
    if expia is None:
        expia = exp_potential(case)
    cols = w.reshape(nzp, nr, nx * ny, n_rot)
    dvr = fbr_to_dvr(cols, case)
    dvr = expia * dvr
    cols = dvr_to_fbr(dvr, case)
    cols = rot_half[None, :, None, :] * cols
    w = cols.reshape(nzp, nr, nx, ny, n_rot)
    proj = np.einsum("xy,zrxy->zr", sc2sp, w[..., i0])
    chi[:nzp, :] = proj
    w[..., i0] = w[..., i0] - sp2sc[None, None] * proj[:, :, None, None]
    psi[:nzp] = w
    return psi, chi


def propagate_analysis_step(psi, chi, case: Case, expia=None):
    """One analysis step (split_operator.cpp:11-46). Returns (psi, chi)."""
    if expia is None:
        expia = exp_potential(case)
    for step, kinetic_only in analysis_step_schedule(case.steps_per_analysis):
        chi = specular_apply(chi, case, step, kinetic_only)
        psi = kinetic_zr(psi, case, step)
        psi = kinetic_xy(psi, case, step)
        if not kinetic_only:
            psi, chi = potential_apply(psi, chi, case, expia)
    return psi, chi


def block_densities(psi: np.ndarray) -> np.ndarray:
    """sum |psi|^2 over (irot, ixy) per (Z, r) point (averages.cpp:20-29), izr = ir + nr*iz."""
    nz, nr = psi.shape[:2]
    return np.sum(np.abs(psi.reshape(nz * nr, -1)) ** 2, axis=1)


def averages(densities: np.ndarray, chi: np.ndarray, z: np.ndarray, z_specular: np.ndarray, r: np.ndarray,
             volume_scattering: float, volume_specular: float, iz_analysis: int, surface_index: int) -> np.ndarray:
    """Norm and position averages (averages.cpp:37-80): [norm, <Z>, <r>, rest norm].

    densities: block densities, izr = ir + nr*iz; chi: (nz_specular, nr). The norm is the scattering
    plus the specular norm, each times its volume element; <Z> and <r> divide the summed moments by
    it; the rest norm is the specular norm of iz_analysis < iz <= surface_index (times dZ dr).
    """
    nr = len(r)
    nz = len(densities) // nr
    d = np.asarray(densities, dtype=np.float64).reshape(nz, nr)
    c2 = np.abs(np.asarray(chi).reshape(len(z_specular), nr)) ** 2
    norm_scat = d.sum() * volume_scattering
    z_scat = (np.asarray(z)[:nz, None] * d).sum() * volume_scattering
    r_scat = (np.asarray(r)[None, :] * d).sum() * volume_scattering
    norm_spec = c2.sum() * volume_specular
    z_spec = (np.asarray(z_specular)[:, None] * c2).sum() * volume_specular
    r_spec = (np.asarray(r)[None, :] * c2).sum() * volume_specular
    rest = c2[iz_analysis + 1:surface_index + 1].sum() * volume_specular
    norm = norm_scat + norm_spec
    return np.array([norm, (z_scat + z_spec) / norm, (r_scat + r_spec) / norm, rest])


def bk_coefficients(z_plane: np.ndarray, chi: np.ndarray, case: Case, surface_fixed: bool,
                    surface_index: int) -> np.ndarray:
    """Balint-Kurti coefficients (balint_kurti.cpp:39-84). z_plane: (nr, nx, ny, n_rot) at Zana.
    Returns (n_v, n_states) complex."""
    a = case.analysis
    nx, ny, nr = case.nx, case.ny, case.nr
    n_v, n_rot_ana, n_dif = a["n_v"], a["n_rotation"], a["n_diffraction"]
    phi = a["phi_vj"].reshape(n_v, a["j_max_gas"] + 1, nr)
    shift = case.t["shift_forward"].reshape(nx, ny)
    bk = np.zeros((n_v, n_rot_ana * n_dif), dtype=np.complex128)
    ix = np.array(a["channel_ix"])
    iy = np.array(a["channel_iy"])
    for v in range(n_v):
        for irotana in range(n_rot_ana):
            irot = a["rotation_index"][irotana]
            j = a["state_j"][irotana * n_dif]
            rw = phi[v, j] * case.dr
            overlap = np.einsum("r,rxy->xy", rw, shift[None] * z_plane[:, :, :, irot])
            overlap = np.fft.fft2(overlap)
            bk[v, irotana * n_dif:(irotana + 1) * n_dif] = overlap[ix, iy] * a["xy_scale"]
    if surface_fixed:
        for v in range(n_v):
            bk[v, a["initial_state"]] = np.sum(chi[surface_index, :] * phi[v, a["j_in"]]) * case.dr
    return bk


def s_matrix_sums(bk_steps: np.ndarray, times: np.ndarray, energies_hartree: np.ndarray, dt_analysis: float):
    """SMatrixAccumulator::add over analysis steps (s_matrix.cpp:49-56): sums[ien, k] = sum_t bk_t[k]
    exp(i E_ien t) dt_analysis. bk_steps: (steps, n) with k = is + n_states v."""
    phase = np.exp(1j * np.outer(energies_hartree, times))          # (ien, t)
    return (phase @ bk_steps) * dt_analysis                          # (ien, k)
