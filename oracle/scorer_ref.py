"""CPU restatement of the learned-truncation scorer network (numpy, float32).

TEST INFRASTRUCTURE ONLY: tests compare the device scorer's scores and gradients against
this.  It computes the same network with the same rounding points as the device kernels
(BF16 weights; the first hidden activation, gelu'(z1) and dz2 rounded to BF16 where the
kernels store them; everything else float32), so the two agree to float32 summation-order
differences plus the tensor cores' accumulation order.

Network (parameters in the flat order of ``ps_scorer_get_params``):
    z1 = b1 + s0*weight*u[0] + s1*log|c|*u[1] + s2*remaining*u[2] + sum_q embed[q][p_q - 1]
    h1 = gelu(z1);  z2 = h1 @ w2;  y = b3 + sum_j gelu(z2_j + b2_j) * w3_j
with p_q = x_q | z_q << 1 over the term's non-identity qubits and gelu the tanh form.
Loss: mean over the batch of (y - target)^2.
"""

from __future__ import annotations

import numpy as np

H = 128
S = np.float32(0.7978845608028654)
A = np.float32(0.044715)

# EXACT = True computes in float64 with no rounding points (for finite-difference checks of
# the formulas themselves); the default mirrors the device's rounding.
EXACT = False


def f32(a):
    return np.asarray(a, np.float64) if EXACT else np.asarray(a).astype(np.float32)


def bf16(a):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    if EXACT:
        return np.asarray(a, np.float64)
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def gelu(x):
    t = np.tanh(S * (x + A * x * x * x))
    return np.float32(0.5) * x * (np.float32(1.0) + t)


def gelu_grad(x):
    x2 = x * x
    t = np.tanh(S * (x + A * x2 * x))
    return (np.float32(0.5) * (np.float32(1.0) + t)
            + np.float32(0.5) * x * (np.float32(1.0) - t * t) * S * (np.float32(1.0) + np.float32(3.0) * A * x2))


def unpack(params, nq):
    p = bf16(params)
    o = 0
    embed = p[o:o + nq * 3 * H].reshape(nq, 3, H); o += nq * 3 * H
    u = p[o:o + 3 * H].reshape(3, H); o += 3 * H
    b1 = p[o:o + H]; o += H
    w2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return embed, u, b1, w2, b2, w3, b3


def support(keys, nq, W):
    """(term, qubit, pauli index 0..2) triples of the non-identity qubits, ascending qubit."""
    keys = np.asarray(keys, np.uint64).reshape(-1, 2 * W)
    q = np.arange(nq)
    xb = ((keys[:, q // 64] >> (q % 64).astype(np.uint64)) & np.uint64(1)).astype(np.int64)
    zb = ((keys[:, W + q // 64] >> (q % 64).astype(np.uint64)) & np.uint64(1)).astype(np.int64)
    p = xb | (zb << 1)
    return p  # [n, nq], 0 = identity


def features(keys, logc, rem, nq, W, fscale, num_sites=None):
    p = support(keys, nq if num_sites is None else num_sites, W)
    weight = (p != 0).sum(axis=1).astype(np.float32)
    logc = np.maximum(np.asarray(logc, np.float32), np.float32(-200.0))
    f = np.stack([weight * np.float32(fscale[0]), logc * np.float32(fscale[1]),
                  np.asarray(rem, np.float32) * np.float32(fscale[2])], axis=1).astype(np.float32)
    return p, f


def f16(a):
    """Round float32 values to IEEE half (nearest even), returned as float32."""
    if EXACT:
        return np.asarray(a, np.float64)
    return np.asarray(a, np.float32).astype(np.float16).astype(np.float32)


def forward(params, keys, logc, rem, nq, W, fscale, site_row=None, tc=None):
    """``site_row``: embedding row of each qubit of the scored keys (-1: ignored), the inference
    site map; the keys then have len(site_row) qubits and W words per half.  ``tc``: the device's
    tensor-core inference path (scorers of at most 64 rows; the default decides by nq), whose
    first hidden activation is an f16 operand instead of bf16."""
    if tc is None:
        tc = nq <= 64 and not EXACT
    embed, u, b1, w2, b2, w3, b3 = unpack(params, nq)
    sites = nq if site_row is None else len(site_row)
    p, f = features(keys, logc, rem, nq, W, fscale, num_sites=sites)
    z1 = b1[None, :] + f[:, 0:1] * u[0][None, :] + f[:, 1:2] * u[1][None, :] + f[:, 2:3] * u[2][None, :]
    for q in range(sites):
        r = q if site_row is None else int(site_row[q])
        if r < 0:
            continue
        m = p[:, q] != 0
        if m.any():
            z1[m] += embed[r, p[m, q] - 1]
    h1 = f16(gelu(z1)) if tc else bf16(gelu(z1))
    z2 = f32(h1.astype(np.float64) @ w2.astype(np.float64)) + b2[None, :]
    h2 = gelu(z2)
    y = b3 + (h2 * w3[None, :]).sum(axis=1)
    return y, dict(p=p, f=f, z1=z1, h1=h1, z2=z2, h2=h2)


def gradients(params, keys, logc, rem, target, nq, W, fscale):
    embed, u, b1, w2, b2, w3, b3 = unpack(params, nq)
    y, c = forward(params, keys, logc, rem, nq, W, fscale, tc=False)  # training runs the bf16 kernels
    n = len(y)
    err = y - np.asarray(target, np.float32)
    dy = (2.0 / n) * err if EXACT else np.float32(2.0 / n) * err
    dz2 = dy[:, None] * w3[None, :] * gelu_grad(c["z2"])
    g = {}
    g["b3"] = np.array([dy.sum()])
    g["w3"] = (dy[:, None] * c["h2"]).sum(axis=0)
    g["b2"] = dz2.sum(axis=0)
    dz2b = bf16(dz2)
    g["w2"] = f32(c["h1"].T.astype(np.float64) @ dz2b.astype(np.float64))
    dh1 = f32(dz2b.astype(np.float64) @ w2.T.astype(np.float64))
    dz1 = dh1 * bf16(gelu_grad(c["z1"]))
    g["b1"] = dz1.sum(axis=0)
    g["u"] = np.stack([(dz1 * c["f"][:, k:k + 1]).sum(axis=0) for k in range(3)])
    ge = np.zeros((nq, 3, H), np.float64 if EXACT else np.float32)
    p = c["p"]
    for q in range(nq):
        for k in range(1, 4):
            m = p[:, q] == k
            if m.any():
                ge[q, k - 1] = dz1[m].sum(axis=0)
    g["embed"] = ge
    flat = f32(np.concatenate([g["embed"].reshape(-1), g["u"].reshape(-1), g["b1"], g["w2"].reshape(-1), g["b2"],
                               g["w3"], g["b3"]]))
    return flat, float((err * err).mean())
