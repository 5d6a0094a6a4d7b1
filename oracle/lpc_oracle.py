"""CPU oracle of the learned preconditioner network (test infrastructure only).

A numpy restatement, in float64, of the network the library trains and applies: four 'same'
3x3x3 convolutions with channels 1-16-16-16-1, no biases, tanh after the first three, the
weights rounded to bfloat16 (round to nearest even) before use.  Layer l's weights are stored
[cout][cin][kz][ky][kx] and packed layer after layer (14688 values), as in the C ABI.

The loss is the mean squared error over the interior of zero-padded n^3 patches (``margin``
points in from every face), averaged over the patches, and :func:`loss_grad` returns its exact
gradient with respect to the (bfloat16-rounded) weights by reverse-mode differentiation.
:func:`fd_check` pins that gradient against central finite differences.

The network itself has no counterpart in the reference; it replaces the stencil-smoothing CG
preconditioner precond_hprsdft (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270).  The
training target, sigma (T + sigma)^-1 g with T the finite-difference kinetic operator, is
restated in :func:`screened_target` by FFT diagonalisation of the same operator.
"""
from __future__ import annotations

import numpy as np

CH = (1, 16, 16, 16, 1)
NW = sum(27 * CH[l] * CH[l + 1] for l in range(4))


def offsets():
    o = [0]
    for l in range(4):
        o.append(o[-1] + 27 * CH[l] * CH[l + 1])
    return o


def bf16_round(w: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 -> float32 with round-to-nearest-even (finite inputs)."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(w: np.ndarray, round_bf16: bool = True):
    w = np.asarray(w, np.float32)
    if round_bf16:
        w = bf16_round(w)
    o = offsets()
    return [w[o[l]:o[l + 1]].astype(np.float64).reshape(CH[l + 1], CH[l], 3, 3, 3) for l in range(4)]


def _shift(x: np.ndarray, dz: int, dy: int, dx: int, periodic: bool) -> np.ndarray:
    """s[..., z, y, x] = x[..., z+dz, y+dy, x+dx] (zero outside unless periodic)."""
    if periodic:
        return np.roll(x, (-dz, -dy, -dx), axis=(-3, -2, -1))
    out = np.zeros_like(x)
    n3, n2, n1 = x.shape[-3:]

    def rng(d, n):
        return (max(0, -d), min(n, n - d))

    (z0, z1), (y0, y1), (x0, x1) = rng(dz, n3), rng(dy, n2), rng(dx, n1)
    out[..., z0:z1, y0:y1, x0:x1] = x[..., z0 + dz:z1 + dz, y0 + dy:y1 + dy, x0 + dx:x1 + dx]
    return out


def conv(x: np.ndarray, w: np.ndarray, periodic: bool) -> np.ndarray:
    """'same' 3x3x3 convolution: out[b,co,p] = sum_{ci,tap} w[co,ci,tap] x[b,ci,p+tap-1]."""
    out = np.zeros((x.shape[0], w.shape[0]) + x.shape[2:])
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                xs = _shift(x, kz - 1, ky - 1, kx - 1, periodic)
                out += np.einsum("oi,bizyx->bozyx", w[:, :, kz, ky, kx], xs)
    return out


def conv_adjoint(d: np.ndarray, w: np.ndarray, periodic: bool) -> np.ndarray:
    """Adjoint of :func:`conv` in its input: din[b,ci,q] = sum w[co,ci,tap] d[b,co,q-tap+1]."""
    out = np.zeros((d.shape[0], w.shape[1]) + d.shape[2:])
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                ds = _shift(d, -(kz - 1), -(ky - 1), -(kx - 1), periodic)
                out += np.einsum("oi,bozyx->bizyx", w[:, :, kz, ky, kx], ds)
    return out


def conv_wgrad(x: np.ndarray, d: np.ndarray, periodic: bool) -> np.ndarray:
    """dW[co,ci,tap] = sum_{b,p} d[b,co,p] x[b,ci,p+tap-1]."""
    g = np.zeros((d.shape[1], x.shape[1], 3, 3, 3))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                xs = _shift(x, kz - 1, ky - 1, kx - 1, periodic)
                g[:, :, kz, ky, kx] = np.einsum("bozyx,bizyx->oi", d, xs)
    return g


def forward(w, x: np.ndarray, periodic: bool = False, keep: bool = False):
    """Network output for x of shape (nb, n3, n2, n1); keep=True also returns the activations."""
    ws = unpack(w) if not isinstance(w, list) else w
    a = [np.asarray(x, np.float64)[:, None]]
    for l in range(3):
        a.append(np.tanh(conv(a[-1], ws[l], periodic)))
    y = conv(a[-1], ws[3], periodic)[:, 0]
    return (y, a) if keep else y


def loss_grad(w, x: np.ndarray, t: np.ndarray, margin: int):
    """MSE over patch interiors and its gradient (packed like w) for zero-padded patches."""
    ws = unpack(w)
    y, a = forward(ws, x, False, keep=True)
    nb, n = x.shape[0], x.shape[1]
    mask = np.zeros(x.shape[1:])
    mask[margin:n - margin, margin:n - margin, margin:n - margin] = 1.0
    cnt = mask.sum() * nb
    diff = (y - t) * mask
    loss = float((diff ** 2).sum() / cnt)
    dy = (2.0 * diff / cnt)[:, None]
    grads = [None] * 4
    grads[3] = conv_wgrad(a[3], dy, False)
    dz = conv_adjoint(dy, ws[3], False) * (1.0 - a[3] ** 2)
    for l in (2, 1, 0):
        grads[l] = conv_wgrad(a[l], dz, False)
        if l > 0:
            dz = conv_adjoint(dz, ws[l], False) * (1.0 - a[l] ** 2)
    return loss, np.concatenate([g.ravel() for g in grads])


def fd_check(w, x, t, margin, idx, h=1e-3):
    """Central finite differences of the loss in the unrounded weights listed in idx.

    The network rounds weights to bfloat16, so the perturbation is applied to the float64
    weights that :func:`unpack` would produce (rounding switched off) and compared with the
    analytic gradient at those same weights."""
    ws0 = unpack(w)
    flat0 = np.concatenate([v.ravel() for v in ws0])
    o = offsets()

    def loss_at(flat):
        ws = [flat[o[l]:o[l + 1]].reshape(CH[l + 1], CH[l], 3, 3, 3) for l in range(4)]
        y = forward(ws, x, False)
        n = x.shape[1]
        m = np.zeros(x.shape[1:])
        m[margin:n - margin, margin:n - margin, margin:n - margin] = 1.0
        return float((((y - t) * m) ** 2).sum() / (m.sum() * x.shape[0]))

    out = []
    for i in idx:
        fp = flat0.copy()
        fm = flat0.copy()
        fp[i] += h
        fm[i] -= h
        out.append((loss_at(fp) - loss_at(fm)) / (2 * h))
    return np.array(out)


def init_weights(seed: int) -> np.ndarray:
    """Random weights with the same distribution as the library's initialiser (not its bits)."""
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.normal(0.0, 1.0 / np.sqrt(27.0 * CH[l]), 27 * CH[l] * CH[l + 1])
                           for l in range(4)]).astype(np.float32)


def kinetic_symbol(n, h, lap_coef, md):
    """Eigenvalues of the finite-difference -1/2 Laplacian on an n1 x n2 x n3 periodic grid,
    arranged (n3, n2, n1) (x fastest), for central weights lap_coef[md + m] (src/fd_module.f90:18-54)."""
    n1, n2, n3 = n

    def axis(nn):
        th = 2 * np.pi * np.fft.fftfreq(nn)
        return -0.5 * (lap_coef[md] + 2 * sum(lap_coef[md + m] * np.cos(m * th) for m in range(1, md + 1))) / h ** 2

    return axis(n3)[:, None, None] + axis(n2)[None, :, None] + axis(n1)[None, None, :]


def screened_target(g: np.ndarray, tsym: np.ndarray, sigma: float) -> np.ndarray:
    """sigma (T + sigma)^-1 g for fields g of shape (nb, n3, n2, n1), by FFT."""
    G = np.fft.fftn(g, axes=(1, 2, 3))
    return np.fft.ifftn(G * (sigma / (tsym + sigma)), axes=(1, 2, 3)).real
