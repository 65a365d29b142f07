"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference quotes its performance on runs of its own program, with no public data set. The
benchmark here runs the step on a case bundle built from the grid sizes of the configuration and
physically shaped tables: kinetic factors exp(-i E dt) from the momentum grids of H2 (M = 2 m_H,
mu = m_H / 2), quadratic absorbers exp(-V_opt dt) at the grid ends, the rotational energies
J(J+1) / (2 mu r^2), normalised associated Legendre functions on the Gauss-Legendre theta grid of a
homonuclear molecule (half grid, even J), a Morse gas-phase potential and a smooth corrugated
6D potential with the magnitudes of H2/Cu(111) (up to ~0.5 hartree). The throughput of the step does
not depend on the values; the physics tests use the reference's own set-up instead.

Config 2 (Dai-Light Cu(111) PES, FP64; config 3 = the same in the mixed form):
  nZ 128, nR 48, nX = nY 16 (hexagonal cell, 60 degree skew), JMax = MJMax = 15 on the full theta
  grid (HomoNuc false, which the reference accepts only for unequal masses: HD, m = 1.0078 + 2.0141)
  -> ntheta 16, nphi 32, n_rot 256; nZSpecular 512; dt 2; 5 time steps per analysis step; 84 of the
  128 Z points in the interaction region (switching to the gas phase ends at Z = 10 bohr);
  6D points nZ nR nX nY ntheta nphi = 8.05e8. No surface symmetry (every (x, y) point has its own
  exp(-iV dt) column: the largest table, the most bytes).
"""

from __future__ import annotations

import math

import numpy as np

from .case import CaseBundle

AMU = 1822.888486209  # electron masses per atomic mass unit
M_H = 1.0078 * AMU
EV = 1.0 / 27.211386245988

M_D = 2.0141 * AMU
CONFIG2 = dict(nz=128, nr=48, nx=16, ny=16, j_max=15, mj_max=15, homonuclear=False, nz_specular=512, dz=0.12,
               dr=0.16, z_start=0.0, r_start=0.5, cell=4.82, dt=2.0, steps_per_analysis=5, nz_potential=84)


def fft_momenta(n: int, d: float) -> np.ndarray:
    return 2.0 * math.pi * np.fft.fftfreq(n, d)


def step_factors(energy: np.ndarray, dt: float, half_by_sqrt: bool):
    full = np.exp(-1j * energy * dt)
    half = np.sqrt(full) if half_by_sqrt else np.exp(-1j * energy * dt / 2.0)
    return full, half


def absorber(q: np.ndarray, start: float, end: float, v0: float, dt: float) -> np.ndarray:
    x = np.clip((q - start) / (end - start), 0.0, None)
    v = np.where(q >= start, 1.5 * v0 * x * x, 0.0)
    return np.exp(-v * dt)


def normalized_legendre(l_max: int, m: int, x: np.ndarray) -> np.ndarray:
    """P_l^m(x) normalised to int_{-1}^{1} P^2 = 1, for l = |m| .. l_max: array (l_max - |m| + 1, len(x))."""
    m = abs(m)
    p_mm = np.ones_like(x) * math.sqrt(0.5)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    for k in range(1, m + 1):
        p_mm = -math.sqrt((2 * k + 1) / (2.0 * k)) * s * p_mm
    out = [p_mm]
    if l_max > m:
        p1 = math.sqrt(2 * m + 3) * x * p_mm
        out.append(p1)
        for l in range(m + 2, l_max + 1):
            a = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
            b = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
            out.append(a * (x * out[-1] - b * out[-2]))
    return np.array(out)


def angular_tables(j_max: int, mj_max: int, n_phi: int, homonuclear: bool):
    """Rotational basis (j_in = 0) and the FBR -> DVR matrices, in the reference's orders (mJ outer,
    J inner; matrix (block, theta, J)). Homonuclear: even J on the half theta grid with doubled
    weights; heteronuclear: every J on the full Gauss-Legendre grid."""
    roots, weights = np.polynomial.legendre.leggauss(j_max + 1)
    order = np.argsort(-roots)
    x, w = roots[order], weights[order]
    if homonuclear:
        keep = x >= -1e-15
        x, w = x[keep], 2.0 * w[keep]
        if j_max % 2 == 0:
            w[-1] *= 0.5  # theta = pi/2 is not doubled
    step = 2 if homonuclear else 1
    blocks, legendre, j_of = [], [], []
    first = 0
    for m in range(-mj_max, mj_max + 1):
        js = [j for j in range(0, j_max + 1, step) if j >= abs(m)]
        p = normalized_legendre(j_max, m, x)  # rows l = |m| ..
        rows = np.array([p[j - abs(m)] for j in js])  # (J, theta)
        mat = (rows * np.sqrt(w / n_phi)[None, :]).T  # (theta, J)
        legendre.append(mat.ravel())
        blocks.append([first, len(js), m if m >= 0 else n_phi + m])
        j_of += js
        first += len(js)
    return blocks, np.concatenate(legendre), np.array(j_of), x


def config_case(cfg: dict | None = None, seed: int = 2024) -> CaseBundle:
    """The case bundle of a configuration (default: config 2)."""
    c = dict(CONFIG2)
    if cfg:
        c.update(cfg)
    rng = np.random.default_rng(seed)
    nz, nr, nx, ny, nzs = c["nz"], c["nr"], c["nx"], c["ny"], c["nz_specular"]
    dt, dz, dr = c["dt"], c["dz"], c["dr"]
    m1, m2 = M_H, (M_H if c["homonuclear"] else M_D)
    mass = m1 + m2
    mu = m1 * m2 / mass
    n_phi = 2 * c["mj_max"] + 1
    while True:  # smallest 2^h 3^i 5 7 11 size >= 2 MjMax + 1
        m = n_phi
        for p in (2, 3, 5, 7, 11):
            while m % p == 0:
                m //= p
        if m == 1 and n_phi % 2 == 0:
            break
        n_phi += 1
    blocks, legendre, j_of, cos_theta = angular_tables(c["j_max"], c["mj_max"], n_phi, c["homonuclear"])
    n_rot = len(j_of)
    n_theta = len(cos_theta)
    nzp = min(int(c["nz_potential"]), nz)

    z = c["z_start"] + dz * np.arange(nz)
    zs = c["z_start"] + dz * np.arange(nzs)
    r = c["r_start"] + dr * np.arange(nr)
    ez = fft_momenta(nz, dz) ** 2 / (2 * mass)
    er = fft_momenta(nr, dr) ** 2 / (2 * mu)
    ezs = fft_momenta(nzs, dz) ** 2 / (2 * mass)
    a = c["cell"]
    dx, dy = a / nx, a / ny
    kx = fft_momenta(nx, dx)
    ky = fft_momenta(ny, dy)
    skew = math.pi / 3.0
    exy = (kx[:, None] ** 2 + ky[None, :] ** 2 - 2.0 * math.cos(skew) * kx[:, None] * ky[None, :]) / (
        2 * mass * math.sin(skew) ** 2)
    erot = (j_of * (j_of + 1))[None, :] / (2.0 * mu * r[:, None] ** 2)  # (ir, irot)

    t = {}
    t["z_kinetic_full"], t["z_kinetic_half"] = step_factors(ez, dt, True)
    t["r_kinetic_full"], t["r_kinetic_half"] = step_factors(er, dt, True)
    t["xy_kinetic_full"], t["xy_kinetic_half"] = step_factors(exy.ravel(), dt, False)
    espec = (ezs[:, None] + er[None, :]).ravel()  # (iz, ir) -> ir + nr*iz
    t["specular_kinetic_full"], t["specular_kinetic_half"] = step_factors(espec, dt, True)
    t["rotation_half"] = np.exp(-1j * erot.ravel() * dt / 2.0)  # irot + n_rot*ir
    t["z_optical"] = absorber(z, z[int(0.85 * nz)], z[-1], 0.2 * EV, dt)
    t["r_optical"] = absorber(r, r[int(0.75 * nr)], r[-1], 0.3 * EV, dt)
    t["z_specular_optical"] = absorber(zs, zs[int(0.85 * nzs)], zs[-1], 0.4 * EV, dt)
    de, alpha, re = 0.1745, 1.02, 1.40
    vasy = de * (1.0 - np.exp(-alpha * (r - re))) ** 2
    t["gas_phase"] = np.exp(-1j * vasy * dt)
    t["shift_forward"] = np.ones(nx * ny, dtype=np.complex128)
    t["shift_backward"] = np.ones(nx * ny, dtype=np.complex128)
    unit = 1.0 / math.sqrt(a * a * math.sin(skew))
    t["specular_to_scattering"] = np.full(nx * ny, unit, dtype=np.complex128)
    t["scattering_to_specular"] = np.full(nx * ny, unit * dx * dy * math.sin(skew), dtype=np.complex128)

    # V on (iz, ir, ixy, theta, phi): Morse in Z for the molecule at r with an r- and angle-dependent
    # corrugation, capped at 0.5 hartree; built as V = A(iz, ir) + B(iz, ir) * g(ixy, theta, phi).
    xg = (np.arange(nx) * dx)[:, None]
    yg = (np.arange(ny) * dy)[None, :]
    corr = (np.cos(2 * math.pi * xg / a) + np.cos(2 * math.pi * yg / a) + np.cos(2 * math.pi * (xg - yg) / a)).ravel()
    phi = 2 * math.pi * np.arange(n_phi) / n_phi
    sin2 = 1.0 - cos_theta ** 2
    g = (0.5 + 0.1 * corr[:, None, None]) * (1.0 + 0.3 * sin2[None, :, None] * np.cos(2 * phi)[None, None, :])
    g = g.reshape(nx * ny, n_theta * n_phi)
    zp = z[:nzp]
    morse = 0.07 * (np.exp(-2 * 1.1 * (zp - 2.5)) - 2 * np.exp(-1.1 * (zp - 2.5)))
    A = morse[:, None] + vasy[None, :]
    B = 0.05 * np.exp(-0.8 * (zp[:, None] - 1.5)).clip(max=10.0) * np.ones((1, nr))
    pot = np.empty((nzp, nr, nx * ny, n_theta * n_phi), dtype=np.float64)
    for iz in range(nzp):
        np.minimum(A[iz][:, None, None] + B[iz][:, None, None] * g[None], 0.5, out=pot[iz])
    t["potential"] = pot.reshape(-1)
    t["legendre"] = legendre
    t["representative_of"] = np.arange(nx * ny, dtype=np.int32)
    t["operation_of"] = np.zeros(nx * ny, dtype=np.int32)
    t["phi_index"] = np.arange(n_phi, dtype=np.int32)

    # Initial packet on the specular grid: Gaussian in Z moving to the surface times a Gaussian in r.
    z0 = zs[int(0.55 * nzs)]
    k0 = math.sqrt(2 * mass * 0.6 * EV)  # 0.6 eV collision energy
    alpha_z = 0.6
    chi_z = (2 * alpha_z / math.pi) ** 0.25 * np.exp(-alpha_z * (zs - z0) ** 2 - 1j * k0 * zs)
    chi_r = np.exp(-8.0 * (r - re) ** 2)
    chi_r /= math.sqrt(np.sum(chi_r ** 2) * dr)
    t["chi_initial"] = (chi_z[:, None] * chi_r[None, :]).ravel()
    _ = rng  # the tables are deterministic; the seed is kept for workloads with random states

    m = dict(n_rot=n_rot, nx=nx, ny=ny, nr=nr, nz=nz, nz_potential=nzp, nz_specular=nzs, n_theta=n_theta,
             n_phi=n_phi, mj_max=c["mj_max"], initial_channel=int(np.flatnonzero((j_of == 0))[0]),
             r_absorber_first=int(0.75 * nr), r_absorber_last=nr - 1,
             steps_per_analysis=c["steps_per_analysis"], time_step=dt, n_rep=nx * ny, n_ops=1,
             iz_analysis=int(0.7 * nz), dz=dz, dr=dr, fft_scale_z=dz / math.sqrt(2 * math.pi),
             fft_scale_r=dr / math.sqrt(2 * math.pi), fft_scale_x=math.sqrt(dx / nx), fft_scale_y=math.sqrt(dy / ny),
             mj_blocks=blocks, j=j_of.tolist(), system="synthetic H2/Cu(111)-shaped", workload="config2")
    return CaseBundle(m, t)
