"""CPU oracle of the learned path guide (test infrastructure only).

The reference renderer has no learned guide, so nothing here restates reference code: it is
the specification the GPU kernels are checked against (guide.cuh, guide.cu):

* encode(): 144 inputs per shading point — 12 frequency bands 2^(k/2) per position axis, one-blob
  encodings of the outgoing direction's spherical angles (32 bins each), the shading normal.
* forward(): 144 -> 64 -> 64 -> 64 -> 64 -> 48 with ReLU; with fp16=True the weights, inputs
  and hidden activations are rounded to IEEE half where the GPU stores them, everything else
  is float64 (the GPU accumulates in float32, so results agree to accumulation order).
* decode() / mixture_pdf(): 8 von Mises-Fisher lobes plus the guide selection probability.
* loss_grad_out() / loss_and_grad(): the training loss mean(-wt log V + wt^2 qc / q) — the
  lobes' KL term and the estimator's second moment in alpha (q = alpha V + (1 - alpha)
  pdf_bsdf, V and qc held constant there) — and its analytic gradient, with the GPU's clamps
  and FP16 gradient storage (scale 8).
* adam(): beta1 0.9, beta2 0.99, eps 1e-8, bias-corrected.
* sample(): vMF mixture sampling by the inversion of Jakob (2012).

Parity status: there is no reference implementation to pin against. The analytic gradient is
pinned by central finite differences of the float64 loss (tests/test_guide_oracle.py).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT, N_LAYERS, N_LOBES = 144, 64, 48, 5, 8
ALPHA_MIN, ALPHA_SPAN = 0.05, 0.9
LOGK_MIN, LOGK_SPAN = -4.0, 12.0
WEIGHT_CLIP = 32.0
GRAD_CLAMP = 8192.0
GRAD_SCALE = 8.0


def layer_in(l):
    return N_IN if l == 0 else N_HID


def layer_out(l):
    return N_OUT if l == N_LAYERS - 1 else N_HID


def offsets():
    """(weight offset, bias offset) of each layer in the flat parameter vector."""
    off, res = 0, []
    for l in range(N_LAYERS):
        w = off
        b = w + layer_in(l) * layer_out(l)
        res.append((w, b))
        off = b + layer_out(l)
    return res, off


OFFSETS, N_PARAMS = offsets()


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    Ws, bs = [], []
    for l, (w, b) in enumerate(OFFSETS):
        Ws.append(p[w:b].reshape(layer_in(l), layer_out(l)))
        bs.append(p[b:b + layer_out(l)])
    return Ws, bs


def pack(Ws, bs):
    out = np.zeros(N_PARAMS, dtype=np.float64)
    for l, (w, b) in enumerate(OFFSETS):
        out[w:b] = np.asarray(Ws[l]).reshape(-1)
        out[b:b + layer_out(l)] = bs[l]
    return out


def h16(x):
    return np.asarray(x, dtype=np.float64).astype(np.float16).astype(np.float64)


def encode(q, bmin, bmax):
    """q: (B, 9) position, shading normal, outgoing direction -> (B, 144) float64."""
    q = np.asarray(q, dtype=np.float64)
    B = q.shape[0]
    e = np.zeros((B, N_IN))
    bmin = np.asarray(bmin, dtype=np.float32).astype(np.float64)
    inv = (1.0 / (np.asarray(bmax, dtype=np.float32) - np.asarray(bmin, dtype=np.float32))).astype(np.float32)
    u = np.clip(((q[:, :3].astype(np.float32) - bmin.astype(np.float32)) * inv).astype(np.float32), 0, 1)
    u = u.astype(np.float64)
    for a in range(3):
        for k in range(12):
            x = (u[:, a].astype(np.float32) * np.float32(2.0 ** (k / 2))).astype(np.float64)
            e[:, a * 24 + 2 * k] = np.sin(np.pi * x)
            e[:, a * 24 + 2 * k + 1] = np.cos(np.pi * x)
    th = np.arccos(np.clip(q[:, 8], -1, 1)) / np.pi
    ph = np.arctan2(q[:, 7], q[:, 6]) / (2 * np.pi) + 0.5
    i = np.arange(32)
    e[:, 72:104] = np.exp(-0.5 * (th[:, None] * 32 - (i + 0.5)) ** 2)
    e[:, 104:136] = np.exp(-0.5 * (ph[:, None] * 32 - (i + 0.5)) ** 2)
    e[:, 136:139] = q[:, 3:6]
    return e


def forward(params, X, fp16=True):
    """Returns (layer inputs [X0, H1..H4], raw outputs (B, 48))."""
    Ws, bs = unpack(params)
    r = h16 if fp16 else (lambda v: np.asarray(v, dtype=np.float64))
    acts = [r(X)]
    h = acts[0]
    for l in range(N_LAYERS - 1):
        h = r(np.maximum(h @ r(Ws[l]) + bs[l], 0.0))
        acts.append(h)
    out = h @ r(Ws[-1]) + bs[-1]
    return acts, out


def _sig(x):
    return 1.0 / (1.0 + np.exp(-x))


def decode(out):
    o = np.asarray(out, dtype=np.float64)
    L = o[:, :32].reshape(-1, N_LOBES, 4)
    th = np.pi * _sig(L[..., 0])
    ph = 2 * np.pi * _sig(L[..., 1])
    k = np.exp(LOGK_MIN + LOGK_SPAN * _sig(L[..., 2]))
    lg = L[..., 3] - L[..., 3].max(axis=1, keepdims=True)
    lam = np.exp(lg)
    lam /= lam.sum(axis=1, keepdims=True)
    mu = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=-1)
    alpha = ALPHA_MIN + ALPHA_SPAN * _sig(o[:, 32])
    return {"mu": mu, "kappa": k, "lam": lam, "alpha": alpha}


def vmf_norm(k):
    return k / (2 * np.pi * (-np.expm1(-2 * k)))


def guide_pdf(dec, w):
    c = (dec["mu"] * np.asarray(w, dtype=np.float64)[:, None, :]).sum(-1)
    return (dec["lam"] * vmf_norm(dec["kappa"]) * np.exp(dec["kappa"] * (c - 1))).sum(1)


def mixture_pdf(out, w, pdfb):
    d = decode(out)
    return d["alpha"] * guide_pdf(d, w) + (1 - d["alpha"]) * np.asarray(pdfb, dtype=np.float64)


def _lobe_terms(o, wi):
    B = o.shape[0]
    L = o[:, :32].reshape(B, N_LOBES, 4)
    sth, sph = _sig(L[..., 0]), _sig(L[..., 1])
    th, ph = np.pi * sth, 2 * np.pi * sph
    r = L[..., 2]
    lk = LOGK_MIN + LOGK_SPAN * _sig(r)
    k = np.exp(lk)
    lg = L[..., 3]
    lse_l = lg.max(1, keepdims=True) + np.log(np.exp(lg - lg.max(1, keepdims=True)).sum(1, keepdims=True))
    st, ct, sp, cp = np.sin(th), np.cos(th), np.sin(ph), np.cos(ph)
    c = st * cp * wi[:, 0:1] + st * sp * wi[:, 1:2] + ct * wi[:, 2:3]
    ls = (lg - lse_l) + lk - np.log(2 * np.pi) - np.log(-np.expm1(-2 * k)) + k * (c - 1)
    m = ls.max(1, keepdims=True)
    logV = (m + np.log(np.exp(ls - m).sum(1, keepdims=True)))[:, 0]
    return dict(sth=sth, sph=sph, st=st, ct=ct, sp=sp, cp=cp, r=r, k=k, c=c, ls=ls, logV=logV,
                lam=np.exp(lg - lse_l))


def loss_value(out, wi, pdfb, wt, V_fixed=None, q_fixed=None):
    """Per-row loss -wt log V + wt^2 qc / q, q = alpha Vc + (1 - alpha) pdf_bsdf, with Vc, qc
    the given constants (defaults: V and q at `out`); the second term trains alpha only."""
    o = np.asarray(out, dtype=np.float64)
    t = _lobe_terms(o, np.asarray(wi, dtype=np.float64))
    V = np.exp(t["logV"]) if V_fixed is None else V_fixed
    alpha = ALPHA_MIN + ALPHA_SPAN * _sig(o[:, 32])
    q = np.maximum(alpha * V + (1 - alpha) * pdfb, 1e-30)
    qc = q if q_fixed is None else q_fixed
    return -wt * t["logV"] + wt * wt * qc / q


def loss_grad_out(out, wi, pdfb, wt, clamp=True):
    """Per-row loss and d loss / d out (B, 48), V constant inside the alpha term."""
    o = np.asarray(out, dtype=np.float64)
    wi = np.asarray(wi, dtype=np.float64)
    B = o.shape[0]
    t = _lobe_terms(o, wi)
    V = np.exp(t["logV"])
    sa = _sig(o[:, 32])
    alpha = ALPHA_MIN + ALPHA_SPAN * sa
    q = np.maximum(alpha * V + (1 - alpha) * pdfb, 1e-30)
    loss = -wt * t["logV"] + wt * wt
    rr = np.exp(t["ls"] - t["logV"][:, None])
    k, c, st, ct, sp, cp = t["k"], t["c"], t["st"], t["ct"], t["sp"], t["cp"]
    dth = rr * k * (ct * cp * wi[:, 0:1] + ct * sp * wi[:, 1:2] - st * wi[:, 2:3]) * np.pi * t["sth"] * (1 - t["sth"])
    dph = rr * k * (-st * sp * wi[:, 0:1] + st * cp * wi[:, 1:2]) * 2 * np.pi * t["sph"] * (1 - t["sph"])
    with np.errstate(over="ignore", invalid="ignore"):
        frac = np.where(2 * k > 700, 0.0, 2 * k / np.expm1(np.minimum(2 * k, 700)))
    sk = _sig(t["r"])
    dk = rr * (1 - frac + k * (c - 1)) * LOGK_SPAN * sk * (1 - sk)
    dl = rr - t["lam"]
    g = np.zeros((B, N_OUT))
    g[:, 0:32:4] = -wt[:, None] * dth
    g[:, 1:32:4] = -wt[:, None] * dph
    g[:, 2:32:4] = -wt[:, None] * dk
    g[:, 3:32:4] = -wt[:, None] * dl
    g[:, 32] = -wt * wt * (V - pdfb) / q * ALPHA_SPAN * sa * (1 - sa)
    if clamp:
        g = np.clip(g, -GRAD_CLAMP, GRAD_CLAMP)
    return loss, g


def train_weights(w):
    w = np.asarray(w, dtype=np.float32)
    mean = np.float32(w.astype(np.float64).mean()) if w.size else np.float32(0)
    inv = np.float32(1.0) / mean if mean > 0 else np.float32(0)
    return np.minimum(w * inv, np.float32(WEIGHT_CLIP)).astype(np.float64)


def loss_fixed(params, q, dirs, pdfb, w, bmin, bmax, params_V):
    """float64 mean loss with the alpha term's V taken from `params_V` (finite-difference
    checks of loss_and_grad at params == params_V)."""
    X = encode(q, bmin, bmax)
    _, out = forward(params, X, fp16=False)
    _, outV = forward(params_V, X, fp16=False)
    V = np.exp(_lobe_terms(outV, np.asarray(dirs, dtype=np.float64))["logV"])
    pdfb = np.asarray(pdfb, dtype=np.float64)
    aV = ALPHA_MIN + ALPHA_SPAN * _sig(outV[:, 32])
    qc = np.maximum(aV * V + (1 - aV) * pdfb, 1e-30)
    wt = train_weights(w)
    return float(loss_value(out, dirs, pdfb, wt, V_fixed=V, q_fixed=qc).mean())


def loss_and_grad(params, q, dirs, pdfb, w, bmin, bmax, fp16=True):
    """Mean training loss and its gradient with respect to the flat parameters, following
    the GPU's rounding points when fp16 is True (float64 throughout otherwise)."""
    X = encode(q, bmin, bmax)
    acts, out = forward(params, X, fp16=fp16)
    wt = train_weights(w)
    pdfb = np.asarray(pdfb, dtype=np.float64)
    loss, g = loss_grad_out(out, dirs, pdfb, wt, clamp=fp16)
    B = X.shape[0]
    Ws, _ = unpack(params)
    r = h16 if fp16 else (lambda v: np.asarray(v, dtype=np.float64))
    scale = GRAD_SCALE if fp16 else 1.0
    G = r(g / scale)
    dWs, dbs = [None] * N_LAYERS, [None] * N_LAYERS
    for l in range(N_LAYERS - 1, -1, -1):
        dWs[l] = acts[l].T @ G * (scale / B)
        dbs[l] = G.sum(0) * (scale / B)
        if l > 0:
            G = r((G @ r(Ws[l]).T) * (acts[l] > 0))
    return float(loss.sum() / B), pack(dWs, dbs)


def adam(params, m, v, grad, step, lr, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step (float32, as on the GPU); returns (params, m, v)."""
    p = np.asarray(params, dtype=np.float32)
    g = np.asarray(grad, dtype=np.float32)
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    bc1 = np.float32(1 - b1 ** step)
    bc2 = np.float32(1 - b2 ** step)
    p = p - np.float32(lr) * (m / bc1) / (np.sqrt(v / bc2) + np.float32(eps))
    return p.astype(np.float32), m.astype(np.float32), v.astype(np.float32)


def _onb(n):
    sign = np.copysign(1.0, n[:, 2])
    a = -1.0 / (sign + n[:, 2])
    b = n[:, 0] * n[:, 1] * a
    t = np.stack([1.0 + sign * n[:, 0] ** 2 * a, sign * b, -sign * n[:, 0]], -1)
    bb = np.stack([b, sign + n[:, 1] ** 2 * a, -n[:, 1]], -1)
    return t, bb


def sample(out, u):
    """Direction samples of the vMF mixture from 3 uniforms per row."""
    d = decode(out)
    u = np.asarray(u, dtype=np.float64)
    B = u.shape[0]
    lam = d["lam"]
    j = np.zeros(B, dtype=np.int64)
    c = lam[:, 0].copy()
    for _ in range(N_LOBES - 1):
        adv = (j < N_LOBES - 1) & (u[:, 0] >= c)
        j = j + adv
        c = c + np.where(adv, lam[np.arange(B), np.minimum(j, N_LOBES - 1)], 0)
    k = d["kappa"][np.arange(B), j]
    mu = d["mu"][np.arange(B), j]
    xi = 1 - u[:, 1]
    w = np.clip(1 + np.log(xi + (1 - xi) * np.exp(-2 * k)) / k, -1, 1)
    s = np.sqrt(np.maximum(0, 1 - w * w))
    phi = 2 * np.pi * u[:, 2]
    t, b = _onb(mu)
    v = t * (s * np.cos(phi))[:, None] + b * (s * np.sin(phi))[:, None] + mu * w[:, None]
    return v / np.linalg.norm(v, axis=1, keepdims=True)
