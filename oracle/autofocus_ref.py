"""ORACLE (test infrastructure): FP64 reference of the image-entropy autofocus gradient.

The reference has no autofocus; this restates the objective the B200 engine differentiates, on top of
the reference's float PFA (src/form_image_pfa.py:165-246):

    x[i, k] = s[i, k] exp(-j theta_i)                      per-pulse phase correction
    z       = FFT2( W * R2( R1(x) ) )                      R1/R2: the two np.interp passes (or the float
                                                           32-tap sinc of oracle.float_pfa) as sparse
                                                           matrices, W: float64 Hamming product, pad
                                                           to pow2 (natural layout; |z| is invariant to
                                                           the reference's fftshift centring)
    I = |z|^2,  p = I / sum(I),  E = -sum p log p          image entropy (0 log 0 = 0)

``entropy_and_grad`` evaluates E and dE/dtheta with torch autograd in float64; ``fd_grad`` gives central
finite differences of the same float64 objective.
"""
from __future__ import annotations

import numpy as np

from . import float_pfa as fp


def _interp_matrix(x, xp):
    """Dense-free (rows, cols, vals) of the np.interp operator: out = M @ fp at queries x, zero outside."""
    n = xp.size
    k = np.searchsorted(xp, x, side="right") - 1
    live = (x >= xp[0]) & (x <= xp[-1])
    k = np.clip(k, 0, n - 2)
    f = (x - xp[k]) / (xp[k + 1] - xp[k])
    rows = np.nonzero(live)[0]
    kk, ff = k[live], f[live]
    return (np.concatenate([rows, rows]), np.concatenate([kk, kk + 1]), np.concatenate([1.0 - ff, ff]))


def _sinc_matrix(x, xp):
    """(rows, cols, vals) of the float 32-tap sinc resample of oracle.float_pfa._interp_sinc (ascending xp):
    interior brackets (15 <= k <= n-17) take tab[phase][t] / 32768 at k - 15 + t, the others the lerp."""
    from . import fixed_emulator as fe
    tab = fe._tab().astype(np.float64) / 32768.0
    n = xp.size
    k = np.searchsorted(xp, x, side="right") - 1
    live = (x >= xp[0]) & (x <= xp[-1])
    k = np.clip(k, 0, n - 2)
    f = (x - xp[k]) / (xp[k + 1] - xp[k])
    ph = np.clip(np.round(np.where(live, f, 0.0) * 32768.0), 0, 32767).astype(np.int64) >> 7
    interior = live & (k >= 15) & (k <= n - 17)
    edge = live & ~interior
    ri = np.nonzero(interior)[0]
    re_ = np.nonzero(edge)[0]
    rows = [np.repeat(ri, 32), re_, re_]
    cols = [(k[ri, None] - 15 + np.arange(32)[None, :]).ravel(), k[re_], k[re_] + 1]
    vals = [tab[ph[ri]].ravel(), 1.0 - f[re_], f[re_]]
    return np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)


def operators(tables, range_interp="lerp", az_interp="lerp"):
    """Per-pulse pass-1 operators and per-range-bin pass-2 operators of resample_kspace ("lerp": np.interp,
    "sinc": the float 32-tap sinc).  A descending source axis is resampled on its ascending view."""
    g = fp.geometry(tables["freq"], tables["ax"], tables["ay"])
    m, n = g["m"], g["n"]
    op1 = _sinc_matrix if range_interp == "sinc" else _interp_matrix
    op2 = _sinc_matrix if az_interp == "sinc" else _interp_matrix
    p1 = []
    for i in range(m):
        xp = g["kr"][i]
        rev = xp[0] > xp[-1]
        r, c, v = op1(g["KR"], xp[::-1] if rev else xp)
        if rev:
            c = n - 1 - c
        p1.append((r, c, v))
    tan_s = g["tan_phi"][g["order"]]
    p2 = []
    for j in range(n):
        src = g["KR"][j] * tan_s
        rev = src[0] > src[-1]
        r, c, v = op2(g["KC"], src[::-1] if rev else src)
        if rev:
            c = m - 1 - c
        p2.append((r, c, v))
    return g, p1, p2


def _forward_torch(sig, theta, g, p1, p2, torch):
    m, n = g["m"], g["n"]
    m2, n2 = fp.to_pow2(m), fp.to_pow2(n)
    s = torch.as_tensor(sig.astype(np.complex128))
    rot = torch.polar(torch.ones_like(theta), -theta)                 # exp(-j theta)
    x = s * rot[:, None]
    g1 = torch.zeros((m, n), dtype=torch.complex128)
    rows = []
    for i in range(m):
        r, c, v = p1[i]
        out = torch.zeros(n, dtype=torch.complex128)
        out = out.index_add(0, torch.as_tensor(r), x[i, torch.as_tensor(c)] * torch.as_tensor(v))
        rows.append(out)
    g1 = torch.stack(rows)                                            # (m, n) [pulse][range bin]
    g1s = g1[torch.as_tensor(g["order"])]
    cols = []
    for j in range(n):
        r, c, v = p2[j]
        out = torch.zeros(m, dtype=torch.complex128)
        out = out.index_add(0, torch.as_tensor(r), g1s[torch.as_tensor(c), j] * torch.as_tensor(v))
        cols.append(out)
    g2 = torch.stack(cols, 1)                                         # (m, n) [cross][range]
    w = torch.as_tensor(np.outer(np.hamming(m), np.hamming(n)))
    pad = torch.zeros((m2, n2), dtype=torch.complex128)
    pad[:m, :n] = g2 * w
    z = torch.fft.fft2(pad)
    inten = (z.real ** 2 + z.imag ** 2)
    p = inten / inten.sum()
    plogp = torch.where(p > 0, p * torch.log(torch.where(p > 0, p, torch.ones_like(p))), torch.zeros_like(p))
    return -plogp.sum()


def entropy_and_grad(sig, tables, theta, range_interp="lerp", az_interp="lerp"):
    import torch
    g, p1, p2 = operators(tables, range_interp, az_interp)
    th = torch.tensor(np.asarray(theta, np.float64), requires_grad=True)
    e = _forward_torch(sig, th, g, p1, p2, torch)
    e.backward()
    return float(e.item()), th.grad.numpy().copy()


def entropy(sig, tables, theta, ops=None):
    import torch
    g, p1, p2 = ops if ops is not None else operators(tables)
    with torch.no_grad():
        return float(_forward_torch(sig, torch.tensor(np.asarray(theta, np.float64)), g, p1, p2, torch).item())


def fd_grad(sig, tables, theta, idx, h=1e-4, range_interp="lerp", az_interp="lerp"):
    """Central differences of the float64 entropy w.r.t. theta[idx]."""
    ops = operators(tables, range_interp, az_interp)
    out = []
    for i in idx:
        tp = np.array(theta, np.float64)
        tm = tp.copy()
        tp[i] += h
        tm[i] -= h
        out.append((entropy(sig, tables, tp, ops) - entropy(sig, tables, tm, ops)) / (2 * h))
    return np.asarray(out)


def phase_error(m, seed=4, quad_edge=3.0, walk_std=0.05):
    """Injected per-pulse phase error: quadratic with `quad_edge` rad at the aperture edges plus a
    random walk of `walk_std` rad/pulse (seeded)."""
    rng = np.random.default_rng(seed)
    u = np.linspace(-1.0, 1.0, m)
    return quad_edge * u * u + np.cumsum(rng.normal(0.0, walk_std, m))
