"""The control-variate network's tensor-core kernels (tcgen05, BF16 inputs,
FP32 accumulation) against torch's FP32 products of the same BF16 values.
Tolerance: |D - D_ref| <= 1e-5 * sum_k |a_ik b_jk| (FP32 summation order)."""
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("m,n,k,batch", [(128, 128, 16, 1), (256, 128, 128, 2),
                                         (128, 16, 64, 3), (384, 128, 208, 1),
                                         (128, 16, 1024, 2)])
def test_gemm_bf16_matches_fp32_reference(cub, ctx, m, n, k, batch):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k + batch)
    a = torch.randn(batch, m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(batch, n, k, device="cuda", generator=g).to(torch.bfloat16)
    d = cub.mlp_gemm_bf16(a, b)
    ref = torch.bmm(a.float(), b.float().transpose(1, 2))
    scale = torch.bmm(a.float().abs(), b.float().abs().transpose(1, 2))
    err = (d - ref).abs()
    assert bool((err <= 1e-5 * scale + 1e-30).all()), float((err / scale).max())


def _peak_data(count, samples, seed):
    import numpy as np

    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (count, samples, 7))
    a = np.exp(rng.uniform(0, np.log(5), (count, 1, 7)))
    u = rng.uniform(0.2, 0.8, (count, 1, 7))
    y = np.prod(1.0 / (a ** -2 + (x - u) ** 2), axis=2)
    return x, y


def _blocks():
    import mlp_oracle as M

    return {"W0": (M.W0, M.B0), "b0": (M.B0, M.W1), "W1": (M.W1, M.B1), "b1": (M.B1, M.W2),
            "W2": (M.W2, M.B2), "b2": (M.B2, M.W3), "w3": (M.W3, M.B3), "b3": (M.B3, M.B3 + 1)}


def test_mlp_gradients_match_oracle(cub, ctx):
    """Tensor-core forward and backward of one minibatch against the CPU
    restatement with the same bf16 roundings: |dG| / |G| <= 1e-2 per
    parameter block, loss within 1e-3."""
    import numpy as np
    import mlp_oracle as M

    E, S = 3, 256
    x, y = _peak_data(E, S, 3)
    net = cub.Mlp(E, S, batch=256, seed=5)
    net.set_data(torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda"))
    loss, g = net.grad(0)
    p = net.params()
    for e in range(E):
        ys = y[e] / np.abs(y[e]).max()
        l_ref, g_ref = M.grad(p[e], x[e], ys)
        assert abs(loss[e] - l_ref) <= 1e-3 * l_ref
        for name, (a, b) in _blocks().items():
            ref = g_ref[a:b]
            d = np.linalg.norm(g[e, a:b] - ref) / max(np.linalg.norm(ref), 1e-30)
            assert d <= 1e-2, (e, name, d)


def test_mlp_training_and_inference(cub, ctx):
    """Adam on the tensor cores lowers the loss by a large factor, and
    inference at new points matches the restated forward pass."""
    import numpy as np
    import mlp_oracle as M

    E, S = 2, 4096
    x, y = _peak_data(E, S, 7)
    net = cub.Mlp(E, S, batch=1024, seed=9)
    net.set_data(torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda"))
    l0, _ = net.grad(0)
    l1 = net.train(30, 2e-3)
    assert (l1 < l0 / 3).all(), (l0, l1)
    rng = np.random.default_rng(11)
    xt = rng.uniform(0, 1, (E, 1000, 7))
    gt = net.eval(torch.tensor(xt, device="cuda")).cpu().numpy()
    p = net.params()
    for e in range(E):
        scale = np.abs(y[e]).max()
        ref, _ = M.forward(p[e], xt[e])
        assert np.abs(gt[e] - scale * ref).max() <= 1e-2 * scale


def _peak_params(cub, n, count, seed, amax):
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        a = np.exp(rng.uniform(0, np.log(amax), n))
        u = rng.uniform(0.1, 0.9, n)
        out.append((a, u))
    return out


def test_control_variate_is_correct_and_measured(cub, oracle, ctx):
    """The learned control variate (network trained on the tensor cores,
    integral of f - g plus integral of g) gives the analytic integral to the
    requested tolerance; its cost is measured against the plain method on
    the same integrands, and its gain in regions is asserted (in time it
    loses)."""
    import time

    n, eps, count = 7, 1e-4, 4
    cases = _peak_params(cub, n, count, 13, 8.0)
    params = [cub.make_params(n, list(a), list(u)) for a, u in cases]
    exact = [oracle.exact(oracle.make_integrand("product_peak", n, a, u)) for a, u in cases]
    t = time.perf_counter()
    res, st = ctx.cv_integrate_batch("product_peak", params, eps, 1e-14, epochs=30)
    t_cv = time.perf_counter() - t
    for r, ex in zip(res, exact):
        assert r.status == 0
        assert abs(r.integral - ex) <= 2 * eps * ex, (r.integral, ex)
    assert st["mean_residual_ratio"] < 1.0  # the network learned part of f
    t = time.perf_counter()
    plain = ctx.integrate_batch("product_peak", n, params, eps, 1e-14,
                                cub.options(policy=cub.POLICY_BREADTH))
    t_plain = time.perf_counter() - t
    for r, ex in zip(plain, exact):
        assert abs(r.integral - ex) <= 2 * eps * ex
    cv_regions = st["regions_residual"] + st["regions_network"]
    plain_regions = sum(r.nregions for r in plain)
    print(f"control variate: {st}; regions cv {cv_regions} plain {plain_regions}; "
          f"time cv {t_cv:.3f} s plain {t_plain:.3f} s")
    # What the trained network gains on these integrands: every integral
    # takes the control-variate route, and f - g plus g needs fewer regions
    # than f alone (measured 1.15x: 295 184 against 339 474).  In time it
    # loses by orders of magnitude: the network costs far more per rule
    # node than the integrand (1.32 s against 2.2 ms, measured); the time
    # ratio is printed above, not asserted.
    assert st["fallbacks"] == 0
    assert plain_regions / cv_regions >= 1.0, (plain_regions, cv_regions)
