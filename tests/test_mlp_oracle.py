"""The network oracle (oracle/mlp_oracle.py) against finite differences of its
own loss, in FP64 (no BF16 rounding): pins the backward pass the GPU kernels
are checked against."""
import numpy as np

from oracle import mlp_oracle as mo


def random_params(rng):
    n = sum(o * i + o for o, i in zip(mo.DOUT, mo.DIN))
    p = np.empty(n)
    off = 0
    for l in range(6):
        k = mo.DOUT[l] * mo.DIN[l]
        bound = 1.0 / np.sqrt(mo.DIN[l])
        p[off:off + k + mo.DOUT[l]] = rng.uniform(-bound, bound, k + mo.DOUT[l])
        off += k + mo.DOUT[l]
    return p


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    p = random_params(rng)
    x = rng.uniform(-1, 1, (6, 4))
    t = rng.normal(0, 0.3, (6, 4))
    _, g, _ = mo.loss_and_grads(p, x, t, bf16_points=False)
    # a few entries of every layer's W and b
    offs, off = [], 0
    for l in range(6):
        k = mo.DOUT[l] * mo.DIN[l]
        offs += [off + int(rng.integers(k)), off + k + int(rng.integers(mo.DOUT[l]))]
        off += k + mo.DOUT[l]
    for i in offs:
        h = 1e-5 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_and_grads(pp, x, t, False)[0] - mo.loss_and_grads(pm, x, t, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-10, (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], dtype=np.float32)
    assert list(mo.bf16(x)) == [1.0, 1.0, 1.0 + 4 * 2 ** -8, 1.0, -2.5]
