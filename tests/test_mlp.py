"""The proposal network: the tensor-core GEMM against a float64 product of
the same bf16 operands, and the forward pass, gradients and Adam training of
the device network against the CPU oracle (oracle/mlp_oracle.py), which in
turn is checked against finite differences here on the CPU."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def batch(seed, rows, noise=0.0, task=0):
    """Inputs, targets of a fixed random linear task (`task` seeds it), mask."""
    proj = np.random.default_rng(1000 + task).standard_normal((MO.IN, MO.OUT))
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((rows, MO.IN)).astype(np.float32)
    t = (x @ proj + noise * rng.standard_normal((rows, MO.OUT)) > 0).astype(np.float32)
    mask = (rng.random((rows, MO.OUT)) > 0.1).astype(np.float32)
    return x, t, mask


# ---- CPU: the oracle itself ----------------------------------------------

def test_bf16_rounding_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3, 3.0e38], dtype=np.float32)
    r = MO.bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even mantissa
    assert r[2] == 1.0 + 2 ** -6            # tie -> even (rounds up)
    assert r[3] == -2.5
    assert abs(r[4] - 1e-3) / 1e-3 < 2 ** -8
    bits = MO.bf16_bits(np.array([1.0, -2.0], dtype=np.float32))
    assert list(bits) == [0x3F80, 0xC000]


def test_oracle_gradients_match_finite_differences():
    p = {k: v.astype(np.float64) for k, v in MO.init_params(3).items()}
    x, t, mask = batch(4, 12)
    _, g = MO.loss_and_grads(p, x, t, mask, exact=True)
    rng = np.random.default_rng(5)
    h = 1e-6
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        flat = p[name].reshape(-1)
        for idx in rng.choice(flat.size, size=6, replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _ = MO.loss_and_grads(p, x, t, mask, exact=True)
            flat[idx] = old - h
            lm, _ = MO.loss_and_grads(p, x, t, mask, exact=True)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 + 1e-4 * abs(fd), (name, idx, fd, an)


def test_rounded_oracle_stays_close_to_exact():
    p = MO.init_params(6)
    x, t, mask = batch(7, 256)
    l0, g0 = MO.loss_and_grads(p, x, t, mask, exact=True)
    l1, g1 = MO.loss_and_grads(p, x, t, mask, exact=False)
    assert abs(l0 - l1) < 1e-2 * abs(l0)
    for k in g0:
        assert rel(g1[k], g0[k]) < 5e-2, k


def test_param_layout(ld):
    assert ld.Mlp.param_count() == sum(int(np.prod(s)) for _, s in ld.MLP_SHAPES)
    p = MO.init_params(1)
    back = ld.unflatten_params(ld.flatten_params(p))
    for k in p:
        np.testing.assert_array_equal(back[k], p[k])


# ---- GPU -------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (128, 128, 128), (256, 256, 64), (384, 320, 192),
                                   (128, 64, 1024), (512, 192, 256)])
def test_tc_gemm_matches_float64(ld, M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    c = ld.tc_gemm(MO.bf16_bits(a), MO.bf16_bits(b))
    ref = MO.bf16(a) @ MO.bf16(b).T
    # fp32 accumulation of K products of bf16 values
    tol = 1e-6 * K * (np.abs(MO.bf16(a)) @ np.abs(MO.bf16(b)).T) + 1e-6
    assert np.all(np.abs(c - ref) <= tol)


@pytest.mark.gpu
def test_tc_gemm_exact_small_integers(ld):
    """Small integers are exact in bf16 and in fp32 accumulation: bit-exact."""
    rng = np.random.default_rng(11)
    a = rng.integers(-8, 9, size=(256, 128)).astype(np.float32)
    b = rng.integers(-8, 9, size=(128, 128)).astype(np.float32)
    c = ld.tc_gemm(MO.bf16_bits(a), MO.bf16_bits(b))
    np.testing.assert_array_equal(c, a @ b.T)


@pytest.mark.gpu
def test_tc_gemm_rejects_bad_shapes(ld):
    a = np.zeros((100, 64), dtype=np.uint16)
    b = np.zeros((64, 64), dtype=np.uint16)
    with pytest.raises(ld.LdError):
        ld.tc_gemm(a, b)


@pytest.mark.gpu
def test_params_roundtrip(ld):
    net = ld.Mlp(batch=128, seed=1)
    p = MO.init_params(2)
    net.set_params(p)
    back = net.get_params()
    for k in p:
        np.testing.assert_array_equal(back[k], p[k])
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("rows,skip", [(128, 0.0), (300, 0.0), (1024, 0.0), (300, 4.0)])
def test_forward_matches_oracle(ld, rows, skip):
    net = ld.Mlp(batch=256, seed=0, skip=skip)
    p = MO.init_params(8)
    net.set_params(p)
    x, _, _ = batch(9, rows)
    z = net.forward(x)
    zr, _ = MO.forward(p, x, skip=skip)
    assert z.shape == (rows, MO.OUT)
    assert rel(z, zr) < 1e-2
    assert np.mean(np.abs(z - zr) < 2e-2 * (np.abs(zr) + 1)) > 0.999
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("rows,skip", [(128, 0.0), (200, 0.0), (512, 0.0), (256, 1.5)])
def test_gradients_match_oracle(ld, rows, skip):
    net = ld.Mlp(batch=512, seed=0, skip=skip)
    p = MO.init_params(10)
    net.set_params(p)
    x, t, mask = batch(11, rows)
    g, loss = net.gradients(x, t, mask)
    lr, gr = MO.loss_and_grads(p, x, t, mask, skip=skip)
    assert abs(loss - lr) < 1e-3 * abs(lr) + 1e-5
    for k in gr:
        assert rel(g[k], gr[k]) < 2e-2, (k, rel(g[k], gr[k]))
    # and the bf16-free float64 gradient is still near
    _, ge = MO.loss_and_grads(p, x, t, mask, exact=True, skip=skip)
    for k in ge:
        assert rel(g[k], ge[k]) < 8e-2, k
    net.close()


@pytest.mark.gpu
def test_adam_step_matches_oracle(ld):
    net = ld.Mlp(batch=256, seed=0)
    p = MO.init_params(12)
    net.set_params(p)
    x, t, mask = batch(13, 256)
    lr = 1e-3
    g, _ = net.gradients(x, t, mask)
    net.train_step(x, t, mask, lr=lr)
    after = net.get_params()
    for k in p:
        # first Adam step: w - lr * g / (|g| + eps') with bias correction
        gi = g[k].astype(np.float64)
        step = lr * gi / (np.abs(gi) + 1e-8)
        np.testing.assert_allclose(after[k], p[k] - step, atol=2e-6, rtol=1e-5)
    net.close()


@pytest.mark.gpu
def test_training_reduces_loss(ld):
    net = ld.Mlp(batch=512, seed=3)
    x, t, mask = batch(14, 4096, noise=0.3)
    first = None
    for epoch in range(12):
        for i in range(0, 4096, 512):
            loss = net.train_step(x[i:i + 512], t[i:i + 512], mask[i:i + 512], lr=2e-3)
            first = loss if first is None else first
    xv, tv, mv = batch(15, 1024, noise=0.3)
    _, val = net.gradients(xv[:512], tv[:512], mv[:512])
    assert loss < 0.5 * first
    assert val < 0.6 * first
    z = net.forward(xv)
    acc = ((z > 0) == (tv > 0.5))[mv > 0].mean()
    assert acc > 0.85
    net.close()
