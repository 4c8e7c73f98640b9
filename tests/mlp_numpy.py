"""Float64 numpy restatement of the preconditioner MLP (8 -> 64 -> 64 -> 64 -> 1, tanh hidden
units, standardised inputs and labels) for checking the library's training kernels."""
import numpy as np

IN, HID = 8, 64
SIZES = [(HID, IN), (HID,), (HID, HID), (HID,), (HID, HID), (HID,), (1, HID), (1,)]


def unpack(p):
    out, off = [], 0
    for s in SIZES:
        c = int(np.prod(s))
        out.append(np.asarray(p[off:off + c], dtype=np.float64).reshape(s))
        off += c
    norm = np.asarray(p[off:off + 2 * IN + 2], dtype=np.float64)
    return out, norm


def loss_and_grad(p, X, y):
    (W1, b1, W2, b2, W3, b3, W4, b4), norm = unpack(p)
    x = (X - norm[:IN]) / norm[IN:2 * IN]
    t = (y - norm[2 * IN]) / norm[2 * IN + 1]
    a1 = np.tanh(x @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    a3 = np.tanh(a2 @ W3.T + b3)
    yh = (a3 @ W4.T)[:, 0] + b4[0]
    e = yh - t
    n = X.shape[0]
    loss = float(np.mean(e * e))
    d4 = 2 * e / n
    d3 = (d4[:, None] * W4) * (1 - a3 ** 2)
    d2 = (d3 @ W3) * (1 - a2 ** 2)
    d1 = (d2 @ W2) * (1 - a1 ** 2)
    g = [d1.T @ x, d1.sum(0), d2.T @ a1, d2.sum(0), d3.T @ a2, d3.sum(0), d4[None, :] @ a3, np.array([d4.sum()])]
    return loss, np.concatenate([gi.ravel() for gi in g])
