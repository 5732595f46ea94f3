"""CPU oracle of the lensing surrogate's network -- TEST INFRASTRUCTURE ONLY.

The reference renderer has no learned component, so this is not a
restatement of reference code: it restates, in float64 numpy, the network
that libbh.so implements (include/bh_surrogate_api.h): Fourier features, four
256-wide GELU layers, the 16-wide head, the training loss and its gradient.
BF16 rounding is applied at the same points as the CUDA path (weights,
features, activations, the loss gradient dY and the hidden gradients dZ fed
to the tensor-core GEMMs), so the comparison isolates the arithmetic of the
kernels.  Only the tests import this module.
"""
import numpy as np

N_IN, BANDS, WIDTH, HIDDEN, OUT, OUT_PAD = 7, 16, 256, 4, 16, 64
W_ESC, W_DISK_R, W_DISK_G, W_CONF, ESC_TOL = 100.0, 1.0, 1.0, 0.1, 1e-3
HID = WIDTH * WIDTH + WIDTH


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def layout(params):
    """Split the flat parameter vector into [(W_l, b_l)] for l = 0..4."""
    p = np.asarray(params, dtype=np.float64)
    out = []
    for l in range(HIDDEN):
        w = p[l * HID:l * HID + WIDTH * WIDTH].reshape(WIDTH, WIDTH)
        b = p[l * HID + WIDTH * WIDTH:(l + 1) * HID]
        out.append((w, b))
    base = HIDDEN * HID
    out.append((p[base:base + OUT * WIDTH].reshape(OUT, WIDTH), p[base + OUT * WIDTH:base + OUT * WIDTH + OUT]))
    return out


def band_w(b):
    return np.pi * 2.0 ** (0.5 * b)


def features(inp):
    """256 features per input row (float64 before BF16 rounding)."""
    x = np.asarray(inp, dtype=np.float64)[:, :N_IN]
    n = x.shape[0]
    f = np.zeros((n, WIDTH))
    for i in range(N_IN):
        for b in range(BANDS):
            t = band_w(b) * x[:, i]
            f[:, i * 32 + 2 * b] = np.sin(t)
            f[:, i * 32 + 2 * b + 1] = np.cos(t)
    f[:, 224:231] = x
    return f


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(0.7978845608 * (x + 0.044715 * x ** 3)))


def gelu_bf16(x):
    """The forward GELU of the CUDA path: BF16 operands and constants, BF16
    rounding after every operation (FMA rounded once); tanh exact then
    rounded (the device uses the hardware approximation)."""
    r = lambda v: bf16(v).astype(np.float64)
    x = r(x)
    c0, c1 = r(np.float32(0.7978845608)), r(np.float32(0.0356774081))
    u = r(r(x * x) * c1 + c0)
    v = r(x * u)
    t = r(np.tanh(v))
    h = r(x * 0.5)
    return r(h * t + h)


def gelu_grad(x):
    t = np.tanh(0.7978845608 * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * 0.7978845608 * (1 + 3 * 0.044715 * x * x)


def forward(X0, params):
    """Head outputs and the saved activations, from BF16 features X0 (n x 256)."""
    layers = layout(params)
    X = [np.asarray(X0, dtype=np.float64)]
    Z = []
    for l in range(HIDDEN):
        w, b = layers[l]
        z = X[-1] @ bf16(w).astype(np.float64).T + b
        Z.append(z)
        X.append(gelu_bf16(bf16(z).astype(np.float64)))
    wh, bh = layers[HIDDEN]
    Y = X[-1] @ bf16(wh).astype(np.float64).T + bh
    return Y, X, Z


def loss_grad(Y, inp, tgt):
    """Batch-mean loss terms (5) and dY (n x 16), as the loss kernel."""
    Y = np.asarray(Y, dtype=np.float64)
    n = Y.shape[0]
    cls = tgt[:, 0].astype(int)
    lg = Y[:, :3]
    m = lg.max(axis=1, keepdims=True)
    e = np.exp(lg - m)
    p = e / e.sum(axis=1, keepdims=True)
    g = np.zeros_like(Y)
    loss = np.zeros(5)
    loss[0] = -np.log(np.maximum(p[np.arange(n), cls], 1e-30)).sum()
    g[:, :3] = p
    g[np.arange(n), cls] -= 1.0
    esc = cls == 0
    r = inp[:, :3] + Y[:, 3:6] - tgt[:, 1:4]
    err = np.sqrt((r * r).sum(axis=1))
    loss[1] = (W_ESC * err[esc] ** 2).sum()
    g[esc, 3:6] = 2 * W_ESC * r[esc]
    hit = tgt[:, 6] > 0.5
    dr = Y[:, 6] - tgt[:, 4]
    dg = Y[:, 7] - tgt[:, 5]
    loss[2] = (W_DISK_R * dr[hit] ** 2).sum()
    loss[3] = (W_DISK_G * dg[hit] ** 2).sum()
    g[hit, 6] = 2 * W_DISK_R * dr[hit]
    g[hit, 7] = 2 * W_DISK_G * dg[hit]
    pred = np.argmax(p, axis=1)          # ties -> lowest index, as the kernel
    good = ((pred == cls) & (~esc | (err < ESC_TOL))).astype(np.float64)
    s = 1 / (1 + np.exp(-Y[:, 8]))
    loss[4] = (-W_CONF * (good * np.log(np.maximum(s, 1e-30)) + (1 - good) * np.log(np.maximum(1 - s, 1e-30)))).sum()
    g[:, 8] = W_CONF * (s - good)
    return loss / n, g / n


def gradients(X0, params, inp, tgt):
    """(flat gradient, loss terms) with the CUDA path's BF16 rounding points."""
    layers = layout(params)
    Y, X, Z = forward(X0, params)
    loss, dY = loss_grad(Y, inp, tgt)
    grads = np.zeros(len(params))
    base = HIDDEN * HID
    dYb = bf16(dY).astype(np.float64)
    grads[base:base + OUT * WIDTH] = (dYb.T @ X[HIDDEN]).ravel()
    grads[base + OUT * WIDTH:base + OUT * WIDTH + OUT] = dY.sum(axis=0)
    dX = dYb @ bf16(layers[HIDDEN][0]).astype(np.float64)
    for l in range(HIDDEN - 1, -1, -1):
        zb = bf16(Z[l]).astype(np.float64)
        dz = dX * gelu_grad(zb)
        dzb = bf16(dz).astype(np.float64)
        grads[l * HID:l * HID + WIDTH * WIDTH] = (dzb.T @ X[l]).ravel()
        grads[l * HID + WIDTH * WIDTH:(l + 1) * HID] = dz.sum(axis=0)
        if l > 0:
            dX = dzb @ bf16(layers[l][0]).astype(np.float64)
    return grads, loss
