"""Numpy restatement of the proposal model (test infrastructure, never the product).

The reference has no learned component; this is the specification the GPU kernels of
``akmc_b200/csrc/mlp.cu`` follow, restated independently:

* per-atom descriptors from the neighbours within ``RC`` (minimum image): 32 Gaussian radial
  functions G2_m = sum_j exp(-ETA_R (r_ij - mu_m)^2) fc(r_ij), mu_m evenly spaced on
  [0.5, 5.0] A; 32 angular functions (Behler's G4) G4 = 2^(1-zeta) sum_{j<k}
  (1 + lambda cos theta_ijk)^zeta exp(-eta (r_ij^2 + r_ik^2 + r_jk^2)) fc_ij fc_ik fc_jk for
  eta in ETA_A, zeta in ZETA, lambda in (+1, -1); fc(r) = (cos(pi r / RC) + 1) / 2;
* the MLP 64 -> 128 -> 128 -> 128 -> 3 with SiLU on the hidden layers: standardised
  inputs, inputs / weights / hidden activations rounded to BF16 (round to nearest even),
  FP32 accumulation;
* the equivariant readout: vectors B_m = sum_j phi_m(r_ij) (r_j - r_i) / r_ij with
  phi_m(r) = exp(-8 (r - nu_m)^2) fc(r), nu = NU; the displacement sum_m y_m B_m;
* its mean-squared-error gradient, in FP32.
"""
from __future__ import annotations

import numpy as np

RC = 5.0
N_RAD = 32
MU = 0.5 + np.arange(N_RAD) * (4.5 / (N_RAD - 1))
ETA_R = 1.0 / (2.0 * (4.5 / (N_RAD - 1)) ** 2)
ETA_A = (0.01, 0.03, 0.07, 0.15)
ZETA = (1, 2, 4, 8)
N_DESC = 64
SIZES = ((64, 128), (128, 128), (128, 128), (128, 3))
NU = (2.5, 3.6, 4.4)


def fc(r):
    return 0.5 * (np.cos(np.pi * r / RC) + 1.0)


def descriptors(pos, box):
    """(n, 64) float64 descriptors of every atom (brute-force minimum image)."""
    pos = np.asarray(pos, dtype=np.float64)
    box = np.asarray(box, dtype=np.float64)
    n = len(pos)
    out = np.zeros((n, N_DESC))
    for i in range(n):
        d = pos - pos[i]
        d -= box * np.rint(d / box)
        r2 = (d * d).sum(1)
        nb = np.where((r2 > 0) & (r2 < RC * RC))[0]
        v = d[nb]
        r = np.sqrt(r2[nb])
        f = fc(r)
        out[i, :N_RAD] = (np.exp(-ETA_R * (r[:, None] - MU[None, :]) ** 2) * f[:, None]).sum(0)
        m = len(nb)
        if m < 2:
            continue
        jj, kk = np.triu_indices(m, 1)
        cos = (v[jj] * v[kk]).sum(1) / (r[jj] * r[kk])
        djk = v[kk] - v[jj]
        djk -= box * np.rint(djk / box)
        rjk = np.sqrt((djk * djk).sum(1))
        fjk = np.where(rjk < RC, fc(rjk), 0.0)
        base = f[jj] * f[kk] * fjk
        rsum = r[jj] ** 2 + r[kk] ** 2 + rjk ** 2
        col = N_RAD
        for eta in ETA_A:
            g = base * np.exp(-eta * rsum)
            for z in ZETA:
                for lam in (1.0, -1.0):
                    out[i, col] = 2.0 ** (1 - z) * (g * (1.0 + lam * cos) ** z).sum()
                    col += 1
    return out


def basis(pos, box):
    """(n, 3, 3) float64 readout vectors (vector m, component c) of every atom."""
    pos = np.asarray(pos, dtype=np.float64)
    box = np.asarray(box, dtype=np.float64)
    out = np.zeros((len(pos), 3, 3))
    for i in range(len(pos)):
        d = pos - pos[i]
        d -= box * np.rint(d / box)
        r = np.sqrt((d * d).sum(1))
        nb = (r > 0) & (r < RC)
        u = d[nb] / r[nb, None]
        for m, nu in enumerate(NU):
            out[i, m] = ((np.exp(-8.0 * (r[nb] - nu) ** 2) * fc(r[nb]))[:, None] * u).sum(0)
    return out


def bf16(x):
    """Round float32 values to BF16 (nearest even), returned as float32."""
    a = np.asarray(x, dtype=np.float32).copy()
    u = a.view(np.uint32)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u + rounding) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def init_params(seed=0):
    """Flat FP32 parameter vector: W1 b1 W2 b2 W3 b3 W4 b4 (W stored [in][out])."""
    rng = np.random.default_rng(seed)
    parts = []
    for fi, fo in SIZES:
        parts.append(rng.normal(0.0, np.sqrt(1.0 / fi), (fi, fo)).astype(np.float32).ravel())
        parts.append(np.zeros(fo, np.float32))
    return np.concatenate(parts)


def unpack(p):
    out, o = [], 0
    for fi, fo in SIZES:
        W = p[o:o + fi * fo].reshape(fi, fo)
        o += fi * fo
        b = p[o:o + fo]
        o += fo
        out.append((W, b))
    return out


def readout(y, B):
    """The displacement sum_m y_m B_m of outputs y (n, 3) and vectors B (n, 3, 3)."""
    return np.einsum("nm,nmc->nc", y, B)


def forward(desc, norm, p, cache=False, rnd=bf16):
    """desc (n, 64); norm = (mean[64], inv_std[64]); p flat FP32 parameters.  rnd is the
    rounding of inputs, weights and hidden activations (BF16; identity for gradient
    checks).  Returns the three outputs y per row (``readout`` turns them into a
    displacement)."""
    x = rnd((np.asarray(desc, np.float32) - norm[0]) * norm[1])
    layers = unpack(p)
    acts, zs = [x], []
    h = x
    for li, (W, b) in enumerate(layers):
        z = h @ rnd(W) + b
        zs.append(z)
        if li < 3:
            h = rnd(silu(z))
            acts.append(h)
        else:
            h = z
    return (h, acts, zs) if cache else h


def loss_and_grad(desc, target, norm, p, rnd=bf16, B=None, rnd_grad=None):
    """Mean over rows of the squared error summed over the 3 components of the prediction
    (y, or readout(y, B) when B is given), and its gradient with respect to the FP32
    parameters (through the BF16-rounded weights as identity).  rnd_grad (e.g. bf16) rounds
    the hidden layers' errors dZ before they enter the products and the bias sums (the
    tensor-core training's operands)."""
    y, acts, zs = forward(desc, norm, p, cache=True, rnd=rnd)
    n = len(y)
    pred = y if B is None else readout(y, B)
    diff = pred - target
    loss = float((diff * diff).sum() / n)
    if B is not None:
        diff = np.einsum("nmc,nc->nm", B, diff)
    dz = (2.0 / n) * diff.astype(y.dtype)
    grads = []
    layers = unpack(p)
    for li in range(3, -1, -1):
        W, _ = layers[li]
        h = acts[li]
        if rnd_grad is not None and li < 3:
            dz = rnd_grad(dz)
        grads.append((h.T @ dz, dz.sum(0)))
        if li > 0:
            dh = dz @ rnd(W).T
            z = zs[li - 1]
            s = 1.0 / (1.0 + np.exp(-z))
            dz = dh * (s * (1.0 + z * (1.0 - s)))
    grads = grads[::-1]
    return loss, np.concatenate([np.concatenate([g[0].ravel(), g[1]]) for g in grads]).astype(np.float32)


def proposal_seeds(begin, pos, box, pred, score, threshold, min_score, scale, noise, radius,
                   seed, counter, score_stride=3, min_disp=0.0, center=None, region=0.0, group=0):
    """akmc_proposal_seeds restated: (disp, mode, chosen) of every walker.  Scores compare in
    float32 (the device's arithmetic); the uniforms are numpy.random.Philox(key=[seed, w],
    counter=[counter, 0, 0, 0]).random()."""
    begin = np.asarray(begin, dtype=np.int64)
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    box = np.asarray(box, dtype=np.float64).reshape(-1, 3)
    pred = np.asarray(pred, dtype=np.float32).reshape(-1, 3)
    score = np.asarray(score, dtype=np.float32).ravel()
    W = len(begin) - 1
    disp = np.zeros_like(pos)
    mode = np.zeros_like(pos)
    chosen = np.full(W, -1, dtype=np.int64)
    for w in range(W):
        a, b = int(begin[w]), int(begin[w + 1])
        n = b - a
        if n == 0:
            continue
        sc = score[(a + np.arange(n)) * score_stride]
        q = pred[a:b]
        elig = (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2]) >= np.float32(min_disp * min_disp)
        if center is not None and region > 0.0:
            dc = pos[a:b] - np.asarray(center, dtype=np.float64)[w]
            dc -= box[w] * np.rint(dc / box[w])
            elig &= (dc * dc).sum(1) < region * region
        if not elig.any():
            continue
        mx = sc[elig].max()
        if not mx >= np.float32(min_score):
            continue
        thr = np.float32(threshold) * mx
        cand = np.where(elig & (sc >= thr))[0]
        if len(cand) == 0:
            continue
        bg = np.random.Philox(key=np.array([seed, w], dtype=np.uint64),
                              counter=np.array([counter, 0, 0, 0], dtype=np.uint64))
        u = np.random.Generator(bg).random(1 + 6 * n)
        frac = ((w % group) + u[0]) / group if group > 1 else u[0]     # stratified over a group
        c = int(cand[min(int(frac * len(cand)), len(cand) - 1)])
        chosen[w] = c
        if noise > 0:
            d = pos[a:b] - pos[a + c]
            d -= box[w] * np.rint(d / box[w])
            near = np.where((d * d).sum(1) < radius * radius)[0]
            for j in near:
                for k in range(3):
                    ua, ub = u[1 + 6 * j + 2 * k], u[2 + 6 * j + 2 * k]
                    disp[a + j, k] = noise * (np.sqrt(-2.0 * np.log(1.0 - ua)) * np.cos(2.0 * np.pi * ub))
        mode[a + c] = pred[a + c].astype(np.float64)
        disp[a + c] += scale * mode[a + c]
    return disp, mode, chosen
