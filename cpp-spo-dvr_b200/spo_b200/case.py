"""Case bundles: the data a propagation backend is built from, as files.

A bundle directory holds ``manifest.json`` (sizes and scalars) and one raw little-endian file per
array (``.c128`` complex128, ``.f64`` float64, ``.i32`` int32). It is the file form of what crosses
the reference's PropagationBackend boundary (BackendInput + PotentialGrid + SpecularWave,
src/propagation/propagation_backend.hpp:63-74). Bundles come from the reference's own set-up (a
maintainer's run of the reference with the recording factory) or from ``spo_b200.workload`` (the
seeded synthetic workloads of the benchmark).
"""

from __future__ import annotations

import json
import os

import numpy as np

C128 = ["z_kinetic_full", "z_kinetic_half", "r_kinetic_full", "r_kinetic_half", "xy_kinetic_full",
        "xy_kinetic_half", "specular_kinetic_full", "specular_kinetic_half", "rotation_half", "gas_phase",
        "shift_forward", "shift_backward", "specular_to_scattering", "scattering_to_specular", "chi_initial"]
F64 = ["z_optical", "r_optical", "z_specular_optical", "legendre", "potential"]
I32 = ["representative_of", "operation_of", "phi_index"]


class CaseBundle:
    """Sizes (``m``) and arrays (``a``) of one case."""

    def __init__(self, manifest: dict, arrays: dict):
        self.m = manifest
        self.a = arrays

    def __getattr__(self, name):
        m = self.__dict__.get("m")
        if m is not None and name in m:
            return m[name]
        raise AttributeError(name)

    @property
    def psi_shape(self):
        return (self.nz, self.nr, self.nx, self.ny, self.n_rot)

    @property
    def chi_shape(self):
        return (self.nz_specular, self.nr)

    @property
    def n_points(self) -> int:
        """Grid points of the 6D DVR grid, nZ nR nX nY ntheta nphi (the metric's unit)."""
        return self.nz * self.nr * self.nx * self.ny * self.n_theta * self.n_phi

    @staticmethod
    def load(directory: str) -> "CaseBundle":
        with open(os.path.join(directory, "manifest.json")) as f:
            m = json.load(f)
        a = {}
        for name in C128:
            a[name] = np.fromfile(os.path.join(directory, name + ".c128"), dtype=np.complex128)
        for name in F64:
            a[name] = np.fromfile(os.path.join(directory, name + ".f64"), dtype=np.float64)
        for name in I32:
            a[name] = np.fromfile(os.path.join(directory, name + ".i32"), dtype=np.int32)
        return CaseBundle(m, a)

    def save(self, directory: str) -> None:
        os.makedirs(directory, exist_ok=True)
        with open(os.path.join(directory, "manifest.json"), "w") as f:
            json.dump(self.m, f, indent=1)
        for name, ext, dt in [(n, ".c128", np.complex128) for n in C128] + [(n, ".f64", np.float64) for n in F64] + \
                [(n, ".i32", np.int32) for n in I32]:
            np.ascontiguousarray(self.a[name], dtype=dt).tofile(os.path.join(directory, name + ext))
