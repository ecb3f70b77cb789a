"""The guiding network's CPU restatement: backpropagation against finite differences, and the
vMF-mixture sampler against its density (test infrastructure checks, no GPU)."""
import numpy as np

import oracle

LO, HI = np.array([-1, -1, -1], np.float32), np.array([2, 1, 3], np.float32)


def _params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(oracle.GUIDE_PARAMS, np.float32)
    offs = [0, 256 * 64] + [256 * 64 + k * 4096 for k in range(1, 5)] + [256 * 64 + 4 * 4096 + 64 * 48]
    shapes = [(256, 64), (64, 64), (64, 64), (64, 64), (64, 64), (64, 48)]
    for l, (k, n) in enumerate(shapes):
        w = rng.uniform(-1, 1, (k, n)) * np.sqrt(6.0 / (225 if l == 0 else 64)) * (0.3 if l == 5 else 1.0) * scale
        if l == 0:
            w[225:] = 0
        if l == 5:
            w[:, 40:] = 0
        p[offs[l]:offs[l + 1]] = w.astype(np.float32).ravel()
    return p, offs


def _records(n, seed=1):
    rng = np.random.default_rng(seed)
    pos = LO + rng.random((n, 3)) * (HI - LO)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.exponential(size=(n, 1))
    w[::5] = 0
    return np.concatenate([pos, nrm, wo, d, w], 1).astype(np.float32)


def test_backprop_matches_finite_differences():
    p, offs = _params()
    rec = _records(6)
    g, loss = oracle.guide_grad(p, rec, LO, HI, emulate=False)
    assert np.isfinite(loss) and np.abs(g).sum() > 0
    rng = np.random.default_rng(7)
    for l in range(6):
        v = np.zeros_like(p)
        seg = slice(offs[l], offs[l + 1])
        v[seg] = rng.normal(size=offs[l + 1] - offs[l]).astype(np.float32)
        if l == 0:
            v[seg].reshape(256, 64)[225:] = 0
        if l == 5:
            v[seg].reshape(64, 48)[:, 40:] = 0
        eps = 3e-6  # central differences converge as eps^2; small enough that no ReLU changes side
        pp, pm = (p + eps * v).astype(np.float32), (p - eps * v).astype(np.float32)
        _, lp = oracle.guide_grad(pp, rec, LO, HI, emulate=False)
        _, lm = oracle.guide_grad(pm, rec, LO, HI, emulate=False)
        fd = lp - lm
        an = float(g @ (pp.astype(np.float64) - pm.astype(np.float64)))
        assert abs(fd - an) <= 2e-5 * max(abs(an), 1e-9) + 1e-12, (l, fd, an)


def test_bf16_emulation_stays_close():
    p, _ = _params()
    x = _records(64)[:, :9]
    raw_e, mix_e = oracle.guide_forward(p, x, LO, HI, emulate=True)
    raw, mix = oracle.guide_forward(p, x, LO, HI, emulate=False)
    assert np.abs(raw_e - raw).max() < 0.05 * np.abs(raw).max()
    np.testing.assert_allclose(mix_e[:, 32:].sum(1), 1.0, rtol=1e-5)


def test_mixture_sampler_matches_its_density():
    rng = np.random.default_rng(3)
    mu = rng.normal(size=(8, 3))
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    kappa = np.array([0.01, 0.5, 2, 5, 20, 80, 300, 1000.0])
    w = rng.random(8) + 0.1
    w /= w.sum()
    mix = np.concatenate([np.concatenate([mu, kappa[:, None]], 1).ravel(), w]).astype(np.float32)
    n = 200_000
    u = rng.random((n, 3)).astype(np.float32)
    dirs, pdf = oracle.vmf_sample(np.tile(mix, (n, 1)), u)
    np.testing.assert_allclose(np.linalg.norm(dirs, axis=1), 1.0, atol=1e-5)
    # E[1/p] = area of the sphere; E[g] = integral of g p, by quadrature on a fine grid
    est = (1.0 / pdf.astype(np.float64))
    assert abs(est.mean() - 4 * np.pi) < 4 * est.std() / np.sqrt(n)
    th = (np.arange(1200) + 0.5) / 1200 * np.pi
    ph = (np.arange(2400) + 0.5) / 2400 * 2 * np.pi
    T, PH = np.meshgrid(th, ph, indexing="ij")
    grid = np.stack([np.sin(T) * np.cos(PH), np.sin(T) * np.sin(PH), np.cos(T)], -1).reshape(-1, 3)
    dA = (np.sin(T) * (np.pi / 1200) * (2 * np.pi / 2400)).ravel()
    pg = oracle.vmf_pdf(np.tile(mix, (grid.shape[0], 1)), grid.astype(np.float32)).astype(np.float64)
    assert abs((pg * dA).sum() - 1.0) < 2e-3
    for gfun in (lambda d: d[:, 0], lambda d: d[:, 2] ** 2, lambda d: (d @ mu[5] > 0.9).astype(float)):
        q = (gfun(grid) * pg * dA).sum()
        s = gfun(dirs.astype(np.float64))
        assert abs(s.mean() - q) < 4 * s.std() / np.sqrt(n) + 2e-3, (s.mean(), q)
