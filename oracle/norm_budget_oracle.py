"""The norm budget restated in numpy (test infrastructure: only the tests import it).

It follows the reference's NormBudget (src/analysis/norm_budget.cpp) and cell_probabilities
(src/propagation/averages.cpp:85-97):
  - absorbers, in order: ZOpt, [ZOptLow], ROpt (scattering grid), ZSpOpt, [ZSpOptLow], ROpt (specular grid)
    (norm_budget.cpp:39-50);
  - per cell (izr = ir + nr iz) of each grid: V_Z = -ln z_factor(iz), V_r = -ln r_factor(ir); cells with both zero
    do not absorb; window exponent 2 n (V_Z + V_r), the Z absorber (the low one inside its range) with share
    V_Z / (V_Z + V_r), the r absorber with the rest (norm_budget.cpp:52-71);
  - a window's loss per cell (norm_budget.cpp:24-35) and its shares summed per absorber, the norms at the window's
    start and end (norm_budget.cpp:75-112). Sums in the reference's cell order.
"""

import numpy as np


class NormBudgetOracle:
    def __init__(self, z_optical, r_optical, z_specular_optical, steps_per_window, volume_scattering,
                 volume_specular, z_low=None, zs_low=None):
        self.absorbers = ["ZOpt"] + (["ZOptLow"] if z_low else []) + ["ROpt"] + ["ZSpOpt"] + \
                         (["ZSpOptLow"] if zs_low else []) + ["ROpt"]
        n = 0
        z_opt, n = n, n + 1
        z_low_i, n = (n, n + 1) if z_low else (-1, n)
        r_opt, n = n, n + 1
        zsp_opt, n = n, n + 1
        zsp_low_i, n = (n, n + 1) if zs_low else (-1, n)
        r_spec, n = n, n + 1
        self.n = n
        self.vol = (volume_scattering, volume_specular)
        r = np.asarray(r_optical, dtype=np.float64)
        self.grids = [self._absorption(np.asarray(z_optical, np.float64), r, z_opt, z_low_i, z_low, r_opt,
                                       steps_per_window),
                      self._absorption(np.asarray(z_specular_optical, np.float64), r, zsp_opt, zsp_low_i, zs_low,
                                       r_spec, steps_per_window)]
        self.previous = None

    @staticmethod
    def _absorption(zf, rf, z_high, z_low, low_range, r_index, spw):
        nz, nr = zf.size, rf.size
        exponent = np.zeros(nz * nr)
        share = np.zeros(nz * nr)
        za = -np.ones(nz * nr, dtype=int)
        ra = -np.ones(nz * nr, dtype=int)
        for iz in range(nz):
            for ir in range(nr):
                v_z, v_r = -np.log(zf[iz]), -np.log(rf[ir])
                if v_z == 0.0 and v_r == 0.0:
                    continue
                k = ir + nr * iz
                exponent[k] = 2.0 * spw * (v_z + v_r)
                if v_z != 0.0:
                    za[k] = z_low if (low_range and low_range[0] <= iz <= low_range[1]) else z_high
                    share[k] = v_z / (v_z + v_r)
                if v_r != 0.0:
                    ra[k] = r_index
        return exponent, share, za, ra

    def add(self, block_densities, chi):
        """block_densities: (nz nr) sums of |psi|^2; chi: (nz_specular, nr) complex. None at the first call, else
        (loss, loss_error, norm_start, norm_end)."""
        cells = [np.asarray(block_densities, np.float64).ravel() * self.vol[0],
                 (np.abs(np.asarray(chi).ravel()) ** 2) * self.vol[1]]
        out = None
        if self.previous is not None:
            loss, err = np.zeros(self.n), np.zeros(self.n)
            for (exponent, share, za, ra), start, end in zip(self.grids, self.previous, cells):
                for k in np.flatnonzero((za >= 0) | (ra >= 0)):
                    g = exponent[k]
                    one_minus_f = -np.expm1(-g)
                    f = np.exp(-g)
                    c_loss = start[k] * one_minus_f + (end[k] - f * start[k]) * (g / one_minus_f - 1.0)
                    c_err = g * g / 6.0 * abs(end[k] - start[k] + c_loss)
                    if za[k] >= 0:
                        loss[za[k]] += share[k] * c_loss
                        err[za[k]] += share[k] * c_err
                    if ra[k] >= 0:
                        loss[ra[k]] += (1.0 - share[k]) * c_loss
                        err[ra[k]] += (1.0 - share[k]) * c_err
            out = (loss, err, float(sum(p.sum() for p in self.previous)), float(sum(c.sum() for c in cells)))
        self.previous = cells
        return out
