"""The CPU oracle of the learned potential's network (oracle/mlp_oracle.py): its gradients against
central finite differences in float64 (rounding off), and its BF16 rounding against known values."""

import numpy as np

import mlp_oracle as M


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -3.14159265, 65504.0], dtype=np.float64)
    got = M.bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0                      # exactly half an ulp (2^-7 at 1): tie -> even
    assert got[2] == 1.0 + 2 ** -7            # above half an ulp -> up
    assert got[3] == 1.0                      # below half an ulp -> down
    assert abs(got[4] - (-3.140625)) < 1e-12  # -3.14159 -> -3.140625
    assert got[5] == 65536.0                  # 65504 rounds up to 2^16 in BF16


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n_in, n_pad, width, depth = 3, 8, 8, 3
    n_par = n_pad * width + width + (depth - 1) * (width * width + width) + width + 1
    p = rng.standard_normal(n_par) * 0.5
    layers_first = p[:n_pad * width].reshape(width, n_pad)
    layers_first[:, n_in:] = 0.0                      # padded inputs carry no weight
    x = rng.standard_normal((16, n_in))
    y = rng.standard_normal(16)
    loss, g = M.gradients(p, x, y, n_pad, width, depth, rounding=False)
    h = 1e-6
    for k in rng.choice(n_par, 40, replace=False):
        if k < n_pad * width and (k % n_pad) >= n_in:
            continue
        q = p.copy()
        q[k] += h
        lp, _ = M.gradients(q, x, y, n_pad, width, depth, rounding=False)
        q[k] -= 2 * h
        lm, _ = M.gradients(q, x, y, n_pad, width, depth, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])
    assert loss > 0
