"""CPU oracle of the step scheduler's MLP (test infrastructure: only tests
import it, as the checker of the library's training kernels).

y = W2 relu(W1 x + b1) + b2, loss L = (1/n) sum_b sum_o (y_bo - t_bo)^2 / 2,
parameters flat as [W1 (32x20, row-major), b1 (32), W2 (5x32), b2 (5)].
Written in float64 so that the fp32 kernel's error can be stated against
it; the library MLP has no reference counterpart (the reference schedules
nothing)."""
import numpy as np

IN, HID, OUT = 20, 32, 5
NPARAM = HID * IN + HID + OUT * HID + OUT


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    w1 = p[o:o + HID * IN].reshape(HID, IN); o += HID * IN
    b1 = p[o:o + HID]; o += HID
    w2 = p[o:o + OUT * HID].reshape(OUT, HID); o += OUT * HID
    b2 = p[o:o + OUT]
    return w1, b1, w2, b2


def forward(p, x):
    w1, b1, w2, b2 = unpack(p)
    z = np.asarray(x, np.float64) @ w1.T + b1
    return z, np.maximum(z, 0.0) @ w2.T + b2


def loss_and_grad(p, x, t):
    """Loss and flat gradient, as the library's mgc_mlp_gradient defines them."""
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    n = x.shape[0]
    w1, b1, w2, b2 = unpack(p)
    z, y = forward(p, x)
    h = np.maximum(z, 0.0)
    d = (y - t) / n
    loss = 0.5 * np.sum((y - t) ** 2) / n
    gw2 = d.T @ h
    gb2 = d.sum(0)
    dz = (d @ w2) * (z > 0)
    gw1 = dz.T @ x
    gb1 = dz.sum(0)
    return loss, np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2])


def numeric_grad(p, x, t, eps=1e-6):
    """Central differences of loss_and_grad's loss (checks the oracle itself)."""
    p = np.asarray(p, np.float64).copy()
    g = np.zeros_like(p)
    for k in range(p.size):
        old = p[k]
        p[k] = old + eps
        lp = loss_and_grad(p, x, t)[0]
        p[k] = old - eps
        lm = loss_and_grad(p, x, t)[0]
        p[k] = old
        g[k] = (lp - lm) / (2 * eps)
    return g
