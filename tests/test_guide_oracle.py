"""CPU checks of the path-guide oracle: the analytic loss gradient against central finite
differences (float64, no FP16 rounding), the encoding's layout and the mixture's
normalisation. These pin the oracle the GPU kernels are compared with."""
import numpy as np
import pytest

from oracle import guide_oracle as G

BMIN, BMAX = np.array([-2.0, 0.0, -2.0]), np.array([2.0, 2.5, 2.0])


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def random_batch(rng, B):
    p = rng.uniform(BMIN, BMAX, size=(B, 3))
    n = unit(rng.normal(size=(B, 3)))
    wo = unit(rng.normal(size=(B, 3)))
    q = np.concatenate([p, n, wo], 1)
    wi = unit(rng.normal(size=(B, 3)))
    pdfb = rng.uniform(0.05, 1.0, size=B)
    w = rng.lognormal(0.0, 1.0, size=B)
    return q, wi, pdfb, w


def init_params(rng, scale=1.0):
    Ws, bs = [], []
    for l in range(G.N_LAYERS):
        i, o = G.layer_in(l), G.layer_out(l)
        a = np.sqrt(6.0 / i) * scale
        Ws.append(rng.uniform(-a, a, size=(i, o)))
        bs.append(rng.uniform(-0.1, 0.1, size=o))
    return G.pack(Ws, bs)


def test_param_layout():
    assert G.N_PARAMS == 24880
    Ws, bs = G.unpack(np.arange(G.N_PARAMS, dtype=np.float64))
    assert Ws[0].shape == (144, 64) and Ws[4].shape == (64, 48) and bs[4].shape == (48,)
    assert np.array_equal(G.pack(Ws, bs), np.arange(G.N_PARAMS))


def test_encoding_layout():
    rng = np.random.default_rng(1)
    q, _, _, _ = random_batch(rng, 64)
    e = G.encode(q, BMIN, BMAX)
    assert e.shape == (64, 144)
    assert np.allclose(e[:, 139:], 0)
    assert np.allclose(e[:, 136:139], q[:, 3:6])
    s, c = e[:, 0:72:2], e[:, 1:72:2]
    assert np.allclose(s ** 2 + c ** 2, 1)
    # one-blob peaks at the bin of the angle
    th = np.arccos(q[:, 8]) / np.pi
    assert np.array_equal(np.argmax(e[:, 72:104], 1), np.minimum((th * 32).astype(int), 31))


def test_mixture_normalised():
    """The vMF mixture integrates to 1 over the sphere (Fibonacci-sphere quadrature)."""
    rng = np.random.default_rng(2)
    out = rng.normal(size=(4, 48))
    n = 200000
    i = np.arange(n) + 0.5
    z = 1 - 2 * i / n
    r = np.sqrt(1 - z * z)
    ph = np.pi * (1 + 5 ** 0.5) * i
    dirs = np.stack([r * np.cos(ph), r * np.sin(ph), z], 1)
    d = G.decode(out)
    for b in range(4):
        one = {k: v[b:b + 1].repeat(n, 0) for k, v in d.items()}
        integral = G.guide_pdf(one, dirs).mean() * 4 * np.pi
        assert abs(integral - 1) < 2e-3


def test_sampling_matches_density():
    """Histogram of oracle samples over 6 cube faces against the integrated density."""
    rng = np.random.default_rng(3)
    out = np.tile(rng.normal(size=(1, 48)), (400000, 1))
    dirs = G.sample(out, rng.uniform(size=(400000, 3)))
    assert np.allclose(np.linalg.norm(dirs, axis=1), 1, atol=1e-9)
    face = np.argmax(np.abs(dirs), 1) * 2 + (dirs[np.arange(len(dirs)), np.argmax(np.abs(dirs), 1)] > 0)
    hist = np.bincount(face, minlength=6) / len(dirs)
    m = 2000000  # Fibonacci-sphere quadrature of the density per face
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    rr = np.sqrt(1 - z * z)
    ph = np.pi * (1 + 5 ** 0.5) * i
    u = np.stack([rr * np.cos(ph), rr * np.sin(ph), z], 1)
    p = G.guide_pdf({k: v[:1].repeat(m, 0) for k, v in G.decode(out[:1]).items()}, u)
    fu = np.argmax(np.abs(u), 1) * 2 + (u[np.arange(m), np.argmax(np.abs(u), 1)] > 0)
    expect = np.array([(p * (fu == k)).mean() * 4 * np.pi for k in range(6)])
    assert np.allclose(hist, expect, atol=6e-3)


def test_output_gradient_finite_differences():
    rng = np.random.default_rng(4)
    B = 32
    out = rng.normal(size=(B, 48))
    out[:, 2:32:4] *= 2  # concentrations across most of (exp(-4), exp(8))
    _, wi, pdfb, w = random_batch(rng, B)
    wt = w / w.mean()
    _, g = G.loss_grad_out(out, wi, pdfb, wt, clamp=False)
    V0 = np.exp(G._lobe_terms(out, wi)["logV"])
    a0 = G.ALPHA_MIN + G.ALPHA_SPAN / (1 + np.exp(-out[:, 32]))
    q0 = a0 * V0 + (1 - a0) * pdfb
    h = 1e-6
    for j in list(range(33)):
        o1, o2 = out.copy(), out.copy()
        o1[:, j] += h
        o2[:, j] -= h
        fd = (G.loss_value(o1, wi, pdfb, wt, V_fixed=V0, q_fixed=q0) -
              G.loss_value(o2, wi, pdfb, wt, V_fixed=V0, q_fixed=q0)) / (2 * h)
        assert np.allclose(g[:, j], fd, rtol=1e-5, atol=1e-7), j
    assert np.all(g[:, 33:] == 0)


def test_lobe_loss_stable_far_from_every_lobe():
    """A sample opposite to sharp lobes keeps a finite, nonzero pull (log-sum-exp form)."""
    out = np.zeros((1, 48))
    out[0, 0:32:4] = -8.0  # theta ~ 0: all lobes at +z
    out[0, 2:32:4] = 3.0   # kappa ~ 1500
    loss, g = G.loss_grad_out(out, np.array([[0.0, 0.0, -1.0]]), np.array([0.3]), np.array([1.0]), clamp=False)
    assert np.all(np.isfinite(loss)) and np.all(np.isfinite(g))
    assert np.all(g[0, 2:32:4] > 0)  # every lobe is told to widen


def test_parameter_gradient_finite_differences():
    rng = np.random.default_rng(5)
    q, wi, pdfb, w = random_batch(rng, 64)
    p = init_params(rng)
    loss, g = G.loss_and_grad(p, q, wi, pdfb, w, BMIN, BMAX, fp16=False)
    assert np.isfinite(loss) and np.all(np.isfinite(g))
    assert abs(loss - G.loss_fixed(p, q, wi, pdfb, w, BMIN, BMAX, p)) < 1e-12 * max(1, abs(loss))
    idx = np.concatenate([rng.choice(G.N_PARAMS, 40, replace=False),
                          [G.OFFSETS[4][1] + 32, G.OFFSETS[0][1], G.OFFSETS[4][0] + 5]])
    h = 1e-5
    for i in idx:
        p1, p2 = p.copy(), p.copy()
        p1[i] += h
        p2[i] -= h
        l1 = G.loss_fixed(p1, q, wi, pdfb, w, BMIN, BMAX, p)
        l2 = G.loss_fixed(p2, q, wi, pdfb, w, BMIN, BMAX, p)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (i, fd, g[i])


def test_fp16_gradient_close_to_float64():
    """The FP16 rounding points change the gradient only slightly."""
    rng = np.random.default_rng(6)
    q, wi, pdfb, w = random_batch(rng, 512)
    p = init_params(rng)
    _, g64 = G.loss_and_grad(p, q, wi, pdfb, w, BMIN, BMAX, fp16=False)
    _, g16 = G.loss_and_grad(p, q, wi, pdfb, w, BMIN, BMAX, fp16=True)
    assert np.linalg.norm(g16 - g64) / np.linalg.norm(g64) < 2e-2


def test_adam_first_step_is_signed_lr():
    p = np.zeros(10, np.float32)
    g = np.linspace(-1, 1, 10).astype(np.float32)
    g[5] = 0
    p1, m, v = G.adam(p, np.zeros(10, np.float32), np.zeros(10, np.float32), g, 1, 1e-2)
    expect = -1e-2 * np.sign(g)
    assert np.allclose(p1, expect, atol=1e-6)


@pytest.mark.parametrize("seed", [0, 1])
def test_loss_decreases_under_gradient_descent(seed):
    """A few plain gradient steps on the float64 loss lower it (sanity of sign and scale)."""
    rng = np.random.default_rng(10 + seed)
    q, wi, pdfb, w = random_batch(rng, 256)
    p = init_params(rng, scale=0.5)
    l0, g = G.loss_and_grad(p, q, wi, pdfb, w, BMIN, BMAX, fp16=False)
    for _ in range(5):
        p = p - 0.05 * g
        l, g = G.loss_and_grad(p, q, wi, pdfb, w, BMIN, BMAX, fp16=False)
    assert l < l0
