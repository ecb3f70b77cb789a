"""The guiding network on the GPU against its CPU restatement, and the guided renderer against the
plain one. Tolerances: the network runs bf16 weights/activations with f32 accumulation on the
tensor cores; the oracle emulates the same bf16 roundings in double precision, so outputs agree
to accumulation-order rounding (and the rare bf16 tie flip it causes)."""
import numpy as np
import pytest
import torch

import oracle
from liar_b200 import guiding as GD, render as R, scenes_guiding, scenes_render, tracers
from liar_b200._native import LiarGpuError
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu

LO, HI = np.array([-1, -1, -1], np.float32), np.array([2, 1, 3], np.float32)
OFFS = [0, 256 * 64] + [256 * 64 + k * 4096 for k in range(1, 5)] + [256 * 64 + 4 * 4096 + 64 * 48]


def _records(n, seed=1, zero_every=5):
    rng = np.random.default_rng(seed)
    pos = LO + rng.random((n, 3)) * (HI - LO)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.exponential(size=(n, 1))
    if zero_every:
        w[::zero_every] = 0
    return np.concatenate([pos, nrm, wo, d, w], 1).astype(np.float32)


def _guide(**kw):
    return GD.Guide(default_context(), (LO, HI), **kw)


def _cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_param_layout_and_initialisation():
    g = _guide(seed=3)
    p = g.params
    assert p.size == oracle.GUIDE_PARAMS == 35840
    assert np.all(p[:256 * 64].reshape(256, 64)[225:] == 0)
    assert np.all(p[OFFS[5]:].reshape(64, 48)[:, 40:] == 0)
    q = p.copy()
    q[100] = 0.5
    g.params = q
    np.testing.assert_array_equal(g.params, q)
    with pytest.raises(LiarGpuError):
        g.params = q[:-1]
    with pytest.raises(LiarGpuError):
        GD.Guide(default_context(), (HI, LO))


@pytest.mark.parametrize("n", [1, 31, 32, 1000, 4099])
def test_eval_matches_oracle(n):
    g = _guide(seed=5)
    x = _records(n, seed=n)[:, :9]
    mix = g.eval(_cuda(x)).cpu().numpy()
    _, ref = oracle.guide_forward(g.params, x, LO, HI, emulate=True)
    w, wr = mix[:, 32:], ref[:, 32:]
    np.testing.assert_allclose(w.sum(1), 1.0, rtol=1e-5)
    assert np.abs(w - wr).max() < 2e-3
    mu, mur = mix[:, :32].reshape(n, 8, 4), ref[:, :32].reshape(n, 8, 4)
    cos = (mu[..., :3] * mur[..., :3]).sum(-1)
    assert np.quantile(cos, 0.001) > 0.999
    np.testing.assert_allclose(mu[..., 3], mur[..., 3], rtol=2e-2)


@pytest.mark.parametrize("n", [1, 33, 5000, 40000])
def test_gradient_matches_oracle(n):
    """1 and 33 records: one CTA with a partial 32-record stage (the rows past the count read as
    zeros; the single record of n = 1 has weight zero, so its gradient is exactly zero); 5,000
    records: one or two stages per CTA of the weight-gradient kernel; 40,000: nine stages per CTA
    over its three stage buffers, accumulated in tensor memory."""
    g = _guide(seed=7)
    rec = _records(n, seed=2)
    loss, grad = g.train_step(_cuda(rec), apply=False, want_grad=True)
    ref, ref_loss = oracle.guide_grad(g.params, rec, LO, HI, emulate=True)
    assert abs(loss - ref_loss) < 1e-3 * abs(ref_loss) + 1e-6
    for l in range(6):
        a, b = grad[OFFS[l]:OFFS[l + 1]].astype(np.float64), ref[OFFS[l]:OFFS[l + 1]]
        if not np.any(b):
            assert not np.any(a), l
            continue
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert cos > 0.9995 and rel < 0.03, (l, cos, rel)
    # the gradient-only call leaves the weights alone; the padding rows and columns get none
    assert np.all(grad[:256 * 64].reshape(256, 64)[225:] == 0)
    assert np.all(grad[OFFS[5]:].reshape(64, 48)[:, 40:] == 0)


def test_adam_first_step():
    lr = 1e-3
    g = _guide(seed=9, learning_rate=lr)
    p0 = g.params
    rec = _cuda(_records(3000, seed=4))
    _, grad = g.train_step(rec, apply=False, want_grad=True)
    g.train_step(rec, apply=True)
    dp = g.params - p0
    big = np.abs(grad) > 1e-4
    # first Adam step: -lr * m_hat / (sqrt(v_hat) + eps) = -lr * sign(g) for |g| >> eps
    np.testing.assert_allclose(dp[big], -lr * np.sign(grad[big]), rtol=1e-3, atol=1e-7)
    assert np.all(dp[np.abs(grad) == 0] == 0)
    assert g.stats()["steps"] == 1


def test_sampler_matches_oracle():
    rng = np.random.default_rng(11)
    n = 20000
    mu = rng.normal(size=(n, 8, 3))
    mu /= np.linalg.norm(mu, axis=-1, keepdims=True)
    kappa = np.exp(rng.uniform(-6, 7, size=(n, 8, 1)))
    w = rng.random((n, 8)) + 0.01
    w /= w.sum(1, keepdims=True)
    mix = np.concatenate([np.concatenate([mu, kappa], -1).reshape(n, 32), w], 1).astype(np.float32)
    u = rng.random((n, 3)).astype(np.float32)
    d, p = _guide().sample(_cuda(mix), _cuda(u))
    d, p = d.cpu().numpy(), p.cpu().numpy()
    dr, pr = oracle.vmf_sample(mix, u)
    close = np.abs(d - dr).max(1) < 2e-3
    assert close.mean() > 0.999
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=2e-5)
    ok = close & (pr > 1e-3)
    np.testing.assert_allclose(p[ok], pr[ok], rtol=5e-3)


def test_training_learns_a_direction_field():
    """Records whose directions follow a position-dependent vMF: the loss falls and the guide's
    density at the true mean direction rises."""
    rng = np.random.default_rng(13)
    n = 1 << 16
    pos = LO + rng.random((n, 3)) * (HI - LO)
    ang = 2.0 * pos[:, 0]
    mean = np.stack([np.cos(ang), np.sin(ang), 0.3 * np.ones(n)], 1)
    mean /= np.linalg.norm(mean, axis=1, keepdims=True)
    mix = np.zeros((n, 40), np.float32)
    mix[:, 0:3] = mean
    mix[:, 3] = 30.0
    mix[:, 32] = 1.0
    d, _ = oracle.vmf_sample(mix, rng.random((n, 3)).astype(np.float32))
    nrm = np.tile([0, 0, 1.0], (n, 1))
    rec = np.concatenate([pos, nrm, nrm, d, np.ones((n, 1))], 1).astype(np.float32)
    g = _guide(seed=1, learning_rate=5e-3)
    rt = _cuda(rec)
    first, _ = g.train_step(rt)
    for _ in range(300):
        last, _ = g.train_step(rt)
    assert last < first - 1.0, (first, last)
    x = _cuda(rec[:4096, :9])
    m = g.eval(x)
    dens = np.array([oracle.vmf_pdf(m[i:i + 1].cpu().numpy(), mean[i:i + 1].astype(np.float32))[0] for i in range(0, 4096, 64)])
    assert np.median(dens) > 0.25 * 30 / (2 * np.pi)  # a fair share of the true peak density 30/2pi


def _tracer(max_gen=3, max_depth=8):
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = max_gen
    t.maxDepth = max_depth
    return t


def _film(desc):
    return torch.zeros((desc.height, desc.width, 8), dtype=torch.float32, device="cuda:0")


def test_guide_off_equals_plain_render():
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    desc = R.render_desc(cam, 48, 40, 6, _tracer(), seed=5)
    plain = _film(desc)
    gs.render_device(desc, plain.data_ptr())
    g = GD.Guide(default_context(), GD.scene_bounds(flat), guide_probability=0.0)
    guided = _film(desc)
    g.render(gs, desc, guided.data_ptr(), train=False)
    torch.cuda.synchronize()
    a, b = guided.cpu().numpy(), plain.cpu().numpy()
    np.testing.assert_allclose(a[..., :7], b[..., :7], rtol=2e-5, atol=2e-6 * np.abs(b[..., :7]).max())
    np.testing.assert_array_equal(a[..., 7], b[..., 7])
    st = GD.render_stats(default_context())
    assert st["paths"] == 48 * 40 * 6 and st["guided"] == 0


def _mean_within(a, b, min_fraction=0.99):
    ma, va = R.resolve(a)
    mb, vb = R.resolve(b)
    sig = np.sqrt(va + vb)
    ok = np.abs(ma[..., :3] - mb[..., :3]) <= 3 * sig + 1e-6 * np.maximum(np.abs(mb[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within 3 sigma"
    return ma, mb


def _image_mean_agrees(a, b, sigmas=4.0):
    """Image means of Y agree within `sigmas` standard errors (from the per-pixel variances)."""
    ma, va = R.resolve(a)
    mb, vb = R.resolve(b)
    n = ma[..., 1].size
    se = np.sqrt(va[..., 1].sum() + vb[..., 1].sum()) / n
    assert abs(ma[..., 1].mean() - mb[..., 1].mean()) < sigmas * se, (ma[..., 1].mean(), mb[..., 1].mean(), se)


def test_guided_white_furnace():
    """A random (untrained) guide sampled at 95% of the directional samples keeps Y = 1 on a
    Lambert(1) sphere under a unit sky: the mixture density matches what is sampled."""
    scene, cam = scenes_render.white_furnace()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    d = R.render_desc(cam, 32, 32, 256, _tracer(64, 64), seed=3)
    plain, guided = _film(d), _film(d)
    gs.render_device(d, plain.data_ptr())
    g = GD.Guide(default_context(), GD.scene_bounds(flat), guide_probability=0.95, seed=1)
    g.render(gs, d, guided.data_ptr(), train=False)
    torch.cuda.synchronize()
    assert GD.render_stats(default_context())["guided"] > 10000
    mp, _ = R.resolve(plain.cpu().numpy())
    mg, vg = R.resolve(guided.cpu().numpy())
    sphere = mp[..., 1] > 0.95  # pixels wholly on the sphere
    se = np.sqrt(vg[..., 1][sphere].sum()) / sphere.sum()
    assert abs(mg[..., 1][sphere].mean() - mp[..., 1][sphere].mean()) < 4 * se + 1e-3


def test_guided_render_is_unbiased():
    """Trained guide sampled at half the directional samples: same expectation as plain."""
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    g = GD.Guide(default_context(), GD.scene_bounds(flat), guide_probability=0.5, learning_rate=5e-3,
                 steps_per_pass=4, batch_records=32768, seed=1)
    warm = R.render_desc(cam, 64, 64, 8, _tracer(), seed=99, wave_paths=64 * 64)  # one pass per training round
    g.render(gs, warm, _film(warm).data_ptr(), train=True)
    st = g.stats()
    assert st["steps"] >= 8 * 4 - 4 and st["records"] > 0
    desc = R.render_desc(cam, 32, 32, 1024, _tracer(), seed=3)
    guided, plain = _film(desc), _film(desc)
    g.render(gs, desc, guided.data_ptr(), train=False)
    assert GD.render_stats(default_context())["guided"] > 0
    gs.render_device(desc, plain.data_ptr())
    torch.cuda.synchronize()
    a, b = guided.cpu().numpy(), plain.cpu().numpy()
    _mean_within(a, b)
    _image_mean_agrees(a, b)


def test_slit_room_guide_learns_the_slit():
    """After online training in the slit room, the guide at points of the wall facing the slit puts
    far more density toward the slit than a uniform hemisphere would: it has learned where the
    light comes from."""
    scene, cam = scenes_guiding.slit_room(n_triangles=20_000)
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    g = GD.Guide(default_context(), GD.scene_bounds(flat), guide_probability=0.3, learning_rate=5e-3,
                 steps_per_pass=8, batch_records=65536, seed=0)
    # online training from path records is noisy run to run (records arrive in atomic order, so
    # batches differ): the guide gets up to three rounds of 64 training passes to find the slit
    rng = np.random.default_rng(0)
    n = 256
    pts = np.stack([np.full(n, -4.99), rng.uniform(1.6, 2.4, n), rng.uniform(-0.8, 0.8, n)], 1)
    to_slit = np.array([5.0, 2.0, 0.0]) - pts
    to_slit /= np.linalg.norm(to_slit, axis=1, keepdims=True)
    x = np.concatenate([pts, np.tile([1.0, 0, 0], (n, 1)), np.tile([1.0, 0, 0], (n, 1))], 1).astype(np.float32)
    for round_ in range(3):
        train_d = R.render_desc(cam, 256, 256, 64, _tracer(), seed=7 + round_, wave_paths=256 * 256)
        g.render(gs, train_d, _film(train_d).data_ptr(), train=True)
        assert g.stats()["records"] > 20000
        mix = g.eval(torch.from_numpy(x).cuda()).cpu().numpy()
        q = oracle.vmf_pdf(mix, to_slit.astype(np.float32))
        ratio = np.median(q) * 2 * np.pi  # against a uniform density over the hemisphere
        print(f"slit room, round {round_ + 1}: guide density toward the slit / uniform hemisphere = {ratio:.1f}")
        if ratio > 5.0:
            break
    assert ratio > 5.0


def test_bounded_wait_times_out_and_the_context_stays_usable():
    """The tcgen05 inference kernel's mbarrier waits are bounded. Under the fault test mode no MMA
    is issued, so every wait runs out: the launch records a timeout, frees its tensor memory and
    returns; liar_gpu_synchronize reports LIAR_ERR_TIMEOUT, and afterwards the same guide on the
    same context evaluates normally."""
    import ctypes as C
    from liar_b200._native import LiarGpuError
    ctx = default_context()
    g = GD.Guide(ctx, (np.array([-1, -1, -1], np.float32), np.array([1, 1, 1], np.float32)), seed=3)
    x = torch.rand((3000, 9), device="cuda", generator=torch.Generator("cuda").manual_seed(1)) * 2 - 1
    ref = g.eval(x)
    ctx.synchronize()
    ref = ref.clone()
    ctx.check(ctx._lib.liar_gpu_set_fault_test(ctx.handle, C.c_int(1)))
    try:
        g.eval(x)
        with pytest.raises(LiarGpuError) as err:
            ctx.synchronize()
        assert err.value.code == -6  # LIAR_ERR_TIMEOUT
    finally:
        ctx.check(ctx._lib.liar_gpu_set_fault_test(ctx.handle, C.c_int(0)))
    again = g.eval(x)
    ctx.synchronize()
    torch.testing.assert_close(again, ref, rtol=0, atol=0)
    g.close()


def test_training_waits_time_out_and_training_recovers():
    """The training kernels' bounded waits (the forward and backward MMA chains, and the
    weight-gradient pipeline's TMA, encoder and commit barriers): under the fault test mode nothing
    is issued to the tensor core or the TMA unit, so the first wait of every kernel runs out; the
    step records a timeout, liar_gpu_synchronize reports LIAR_ERR_TIMEOUT, and afterwards the same
    guide computes the same gradient as before, bit for bit (the weight sum and the weight
    gradients' partial sums are added in fixed orders, so a step is reproducible)."""
    import ctypes as C
    from liar_b200._native import LiarGpuError
    ctx = default_context()
    g = _guide(seed=7)
    rec = _cuda(_records(5000, seed=2))
    _, ref = g.train_step(rec, apply=False, want_grad=True)
    ctx.check(ctx._lib.liar_gpu_set_fault_test(ctx.handle, C.c_int(1)))
    try:
        g.train_device(rec, apply=False)
        with pytest.raises(LiarGpuError) as err:
            ctx.synchronize()
        assert err.value.code == -6  # LIAR_ERR_TIMEOUT
    finally:
        ctx.check(ctx._lib.liar_gpu_set_fault_test(ctx.handle, C.c_int(0)))
    _, grad = g.train_step(rec, apply=False, want_grad=True)
    np.testing.assert_array_equal(grad, ref)
    g.close()
