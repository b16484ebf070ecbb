"""Test infrastructure only: a numpy restatement of the coordinate MLP of
supersonicflowsolver_b200/csrc/mlp.cu (forward, loss and backward), used to
check the GPU kernels' gradients. There is no reference counterpart (PSST has
no learned component), so this oracle is pinned only by finite differences of
its own loss (tests/test_mlp_oracle.py).

With bf16=True it rounds to BF16 at the points where the GPU path stores BF16
(features, hidden activations and pre-activations, the back-propagated
deltas, the tensor-core copies of W1..W5) and accumulates in FP64; with
bf16=False everything is FP64.
"""
import numpy as np

WIDTH, FEAT, FREQ, NIN, NOUT, HIDDEN = 256, 128, 15, 4, 4, 5
DIN = [FEAT, WIDTH, WIDTH, WIDTH, WIDTH, WIDTH]
DOUT = [WIDTH, WIDTH, WIDTH, WIDTH, WIDTH, NOUT]


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    """[(W, b)] per layer from the flat parameter array (W [out][in], then b)."""
    out, off = [], 0
    for l in range(6):
        n = DOUT[l] * DIN[l]
        W = np.asarray(p[off:off + n], dtype=np.float64).reshape(DOUT[l], DIN[l])
        off += n
        b = np.asarray(p[off:off + DOUT[l]], dtype=np.float64)
        off += DOUT[l]
        out.append((W, b))
    return out


def features(x):
    x = np.asarray(x, dtype=np.float64)
    cols = []
    for i in range(NIN):
        v = x[:, i]
        cols.append(v)
        w = np.pi
        for _ in range(FREQ):
            cols.append(np.sin(w * v))
            cols.append(np.cos(w * v))
            w *= 2.0
    f = np.stack(cols, axis=1)
    return np.concatenate([f, np.zeros((len(x), FEAT - f.shape[1]))], axis=1)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_and_grads(p, x, t, bf16_points=True):
    """Mean squared error over B x 4 and its gradient (flat, layout of p)."""
    r = bf16 if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(p)
    B = len(x)
    f = r(features(x))
    hs, zs = [f], []
    h = f
    for l in range(HIDDEN):
        W, b = layers[l]
        z = h @ r(W).T + b
        zs.append(r(z))
        h = r(silu(z))
        hs.append(h)
    W6, b6 = layers[5]
    y = h @ W6.T + b6
    d = y - np.asarray(t, dtype=np.float64)
    loss = float(np.mean(d * d))
    dy = 2.0 * d / (NOUT * B)
    grads = []
    grads.append((dy.T @ hs[HIDDEN], dy.sum(axis=0)))
    dz = r((dy @ W6) * dsilu(zs[HIDDEN - 1]))
    for l in range(HIDDEN - 1, -1, -1):
        W, _ = layers[l]
        grads.append((dz.T @ hs[l], dz.sum(axis=0)))
        if l > 0:
            dz = r((dz @ r(W)) * dsilu(zs[l - 1]))
    grads = grads[::-1]  # layer order 1..6
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat, y
