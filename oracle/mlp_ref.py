"""CPU reference of the preconditioner MLP (test infrastructure only).

Plain numpy FP64 forward and backward of 144 -> 256 -> 256 -> 225 with ReLU
and a mean-squared-error loss, on the packed weight layout of
rf_mlp_num_params (W1[256x144] b1 W2[256x256] b2 W3[225x256] b3, row-major
out x in).  The GPU trainer's gradients are checked against it.
"""
import numpy as np

IN, HID, OUT = 144, 256, 225


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    out = []
    for shape in [(HID, IN), (HID,), (HID, HID), (HID,), (OUT, HID), (OUT,)]:
        n = int(np.prod(shape))
        out.append(w[o:o + n].reshape(shape))
        o += n
    assert o == w.size
    return out


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.maximum(x @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h1, h2, h2 @ W3.T + b3


def loss_grad(w, x, y):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1, h2, o = forward(w, x)
    cnt = o.size
    loss = np.sum((o - y) ** 2) / cnt
    do = 2.0 * (o - y) / cnt
    gW3 = do.T @ h2
    gb3 = do.sum(0)
    dh2 = (do @ W3) * (h2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    gW1 = dh1.T @ x
    gb1 = dh1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g
