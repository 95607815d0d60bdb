"""CPU oracle (numpy) for the ground-state CG preconditioners.

TEST INFRASTRUCTURE ONLY: the tests use it to check the CUDA kernels of
salmon_b200/csrc/k_fft.cu (TPA) and salmon_b200/csrc/k_net.cu (the learned
network); the library never calls it.

Neither preconditioner has a counterpart in the reference (SALMON's CG_ompk,
GS/CG.f90:34-139, is unpreconditioned).  The TPA factor follows Teter, Payne and
Allan, Phys. Rev. B 40, 12255 (1989); the network is the 3-layer linear 3D
convolution described in k_net.cu.
"""
from __future__ import annotations

import numpy as np

NTAP = 27
NET_C = 8
NW1, NW2, NW3 = NET_C * 1 * NTAP, NET_C * NET_C * NTAP, 1 * NET_C * NTAP
NET_NW = NW1 + NW2 + NW3
TAPS = [((t // 9) - 1, ((t // 3) % 3) - 1, (t % 3) - 1) for t in range(NTAP)]


# ------------------------------------------------------------------ TPA --
def fd_symbol(lap, nab, k, th):
    """-1/2 (lap0 + 2 sum lap_n cos(n th)) + 2 k sum nab_n sin(n th)."""
    t = lap[0] + sum(2.0 * lap[n] * np.cos(n * th) for n in range(1, 5))
    g = sum(nab[n] * np.sin(n * th) for n in range(1, 5))
    return -0.5 * t + 2.0 * k * g


def tpa_factor(x):
    p = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
    return p / (p + 16.0 * x ** 4)


def tpa_apply(g, shape, k, tband, lap3, nab3):
    """K g for one complex grid function g (NL,) at k-point k (3,), band kinetic
    energy tband; lap3/nab3: (3, 5) FD coefficients (already scaled by 1/H^2, 1/H)."""
    NLx, NLy, NLz = shape
    G = np.fft.fftn(g.reshape(shape))
    ms = [np.fft.fftfreq(n, 1.0 / n) for n in shape]  # 0, 1, ..., -1
    th = [2 * np.pi * m / n for m, n in zip(ms, shape)]
    T = 0.5 * float(np.dot(k, k)) + (fd_symbol(lap3[0], nab3[0], k[0], th[0])[:, None, None]
                                     + fd_symbol(lap3[1], nab3[1], k[1], th[1])[None, :, None]
                                     + fd_symbol(lap3[2], nab3[2], k[2], th[2])[None, None, :])
    x = np.maximum(T, 0.0) / max(tband, 1e-6)
    return np.fft.ifftn(G * tpa_factor(x)).ravel()


# -------------------------------------------------------------- network --
def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def split_weights(w):
    w = np.asarray(w)
    return (w[:NW1].reshape(NET_C, 1, NTAP), w[NW1:NW1 + NW2].reshape(NET_C, NET_C, NTAP),
            w[NW1 + NW2:].reshape(1, NET_C, NTAP))


def conv(x, W):
    """out[..., co] = sum_{tap, ci} W[co, ci, tap] x[i + d(tap), ci]; x: (NLx, NLy, NLz, CI)."""
    out = np.zeros(x.shape[:3] + (W.shape[0],))
    for t, (dx, dy, dz) in enumerate(TAPS):
        xs = np.roll(x, shift=(-dx, -dy, -dz), axis=(0, 1, 2))
        out += xs @ W[:, :, t].T
    return out


def conv_bwd_data(gout, W):
    gin = np.zeros(gout.shape[:3] + (W.shape[1],))
    for t, (dx, dy, dz) in enumerate(TAPS):
        gs = np.roll(gout, shift=(dx, dy, dz), axis=(0, 1, 2))
        gin += gs @ W[:, :, t]
    return gin


def conv_bwd_w(gout, x):
    dW = np.zeros((gout.shape[3], x.shape[3], NTAP))
    for t, (dx, dy, dz) in enumerate(TAPS):
        xs = np.roll(x, shift=(-dx, -dy, -dz), axis=(0, 1, 2))
        dW[:, :, t] = np.einsum("xyzo,xyzi->oi", gout, xs)
    return dW


def inv_rms(g):
    s = float(np.vdot(g, g).real)
    return np.sqrt(g.size / s) if s > 0 else 0.0


def _parts(g, shape, scale):
    """The two real one-channel samples (Re, Im) of a complex vector, scaled."""
    z = g.reshape(shape) * scale
    return [z.real[..., None], z.imag[..., None]]


def forward(g, shape, w, emulate_bf16=True):
    """The network on one complex vector g (NL,): f applied to Re and Im.
    Returns (output (NL,) complex, [(a0, a1, a2, y) per part], scale)."""
    rnd = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, W3 = (rnd(W) for W in split_weights(w))
    s = inv_rms(g)
    acts = []
    for x in _parts(g, shape, s):
        a0 = rnd(x)
        a1 = rnd(conv(a0, W1))
        a2 = rnd(conv(a1, W2))
        acts.append((a0, a1, a2, conv(a2, W3)))
    y = acts[0][3][..., 0] + 1j * acts[1][3][..., 0]
    out = y.ravel() / s if s > 0 else np.zeros_like(g)
    return out, acts, s


def loss_grad(gs, ts, shape, w, emulate_bf16=True):
    """Mean squared error over all samples, voxels and both parts of the
    network output against the targets (scaled like the inputs) and its
    gradient with respect to the flat weight vector."""
    rnd = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, W3 = (rnd(W) for W in split_weights(w))
    n = 2 * sum(g.size for g in gs)
    loss = 0.0
    d1, d2, d3 = np.zeros_like(W1), np.zeros_like(W2), np.zeros_like(W3)
    for g, t in zip(gs, ts):
        _, acts, s = forward(g, shape, w, emulate_bf16)
        for (a0, a1, a2, y), tt in zip(acts, _parts(t, shape, s)):
            if emulate_bf16:
                tt = tt.astype(np.float32).astype(np.float64)
            diff = y - tt
            loss += float((diff ** 2).sum())
            gy = 2.0 * diff / n
            d3 += conv_bwd_w(gy, a2)
            g2 = conv_bwd_data(gy, W3)
            d2 += conv_bwd_w(g2, a1)
            g1 = conv_bwd_data(g2, W2)
            d1 += conv_bwd_w(g1, a0)
    return loss / n, np.concatenate([d1.ravel(), d2.ravel(), d3.ravel()])


def identity_weights(noise=0.0, seed=0):
    """Weights for which the network is the identity (centre taps), plus noise."""
    rng = np.random.default_rng(seed)
    W1, W2, W3 = (np.zeros(x) for x in ((NET_C, 1, NTAP), (NET_C, NET_C, NTAP), (1, NET_C, NTAP)))
    W1[0, 0, 13] = 1.0
    W3[0, 0, 13] = 1.0
    for c in range(NET_C):
        W2[c, c, 13] = 1.0
    w = np.concatenate([W1.ravel(), W2.ravel(), W3.ravel()])
    if noise:
        w = w + noise * rng.standard_normal(w.size)
    return w.astype(np.float32)
