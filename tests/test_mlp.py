"""The cost model's network.  CPU: the float64 oracle's gradient against
central finite differences.  GPU: the CUDA kernels' forward pass and
gradient against the oracle, and training reducing the loss."""
import ctypes

import numpy as np
import pytest

from oracle import mlp as M
from tempi_b200 import _lib


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init(1) + rng.normal(0, 0.01, M.P)
    p[M.P - M.OUT:] = rng.normal(0, 0.1, M.OUT)  # non-zero output biases
    x = rng.uniform(0, 1, (16, M.IN))
    y = rng.normal(0, 1, (16, M.OUT))
    mask = (rng.uniform(size=(16, M.OUT)) < 0.7).astype(float)
    _, g = M.loss_and_grad(p, x, y, mask)
    idx = rng.choice(M.P, 200, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(M.P)
        e[i] = h
        num = (M.loss_and_grad(p + e, x, y, mask)[0] - M.loss_and_grad(p - e, x, y, mask)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), i


def test_parameter_count_matches_header():
    text = open(_lib.os.path.join(_lib.HERE, "..", "include", "tempi_b200.h")).read()
    assert f"#define TEMPI_MLP_PARAMS {M.P}" in text


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.gpu
def test_cuda_gradient_matches_oracle(cuda):
    """tempi_mlp_grad (float32 kernel) against the float64 oracle; tolerance
    1e-3 relative plus 1e-5 absolute per element."""
    import torch

    rng = np.random.default_rng(3)
    for n in (1, 17, 64):
        p = (M.init(n) + rng.normal(0, 0.02, M.P)).astype(np.float32)
        x = rng.uniform(0, 1, (n, M.IN)).astype(np.float32)
        y = rng.normal(0, 1, (n, M.OUT)).astype(np.float32)
        mask = (rng.uniform(size=(n, M.OUT)) < 0.8).astype(np.float32)
        mask[0, 0] = 1
        g = torch.zeros(M.P, dtype=torch.float32, device="cuda")
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        dp, dx, dy, dm = _dev(p), _dev(x), _dev(y), _dev(mask)
        _lib.check(_lib.tempi().tempi_mlp_grad(
            ctypes.c_void_p(dp.data_ptr()), ctypes.c_void_p(dx.data_ptr()),
            ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(dm.data_ptr()), n,
            ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(loss.data_ptr()), None))
        torch.cuda.synchronize()
        want_l, want_g = M.loss_and_grad(p.astype(np.float64), x, y, mask)
        got = g.cpu().numpy().astype(np.float64)
        assert abs(loss.item() - want_l) <= 1e-5 + 1e-4 * abs(want_l)
        np.testing.assert_allclose(got, want_g, rtol=1e-3, atol=1e-5)


@pytest.mark.gpu
def test_cuda_forward_matches_oracle(cuda):
    import torch

    rng = np.random.default_rng(4)
    members, n = 5, 300
    ps = np.stack([M.init(i) + rng.normal(0, 0.05, M.P) for i in range(members)]).astype(np.float32)
    x = rng.uniform(0, 1, (n, M.IN)).astype(np.float32)
    out = torch.zeros(members * n * M.OUT, dtype=torch.float32, device="cuda")
    dp, dx = _dev(ps), _dev(x)
    _lib.check(_lib.tempi().tempi_mlp_predict(ctypes.c_void_p(dp.data_ptr()), members,
                                               ctypes.c_void_p(dx.data_ptr()), n,
                                               ctypes.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(members, n, M.OUT)
    for m in range(members):
        want, _ = M.forward(ps[m].astype(np.float64), x)
        np.testing.assert_allclose(got[m], want, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_training_fits_a_smooth_target(cuda):
    """One launch trains all five members; the held-out error of a smooth
    synthetic target drops well below that of the untrained network."""
    import torch

    rng = np.random.default_rng(5)
    n = 4000
    x = rng.uniform(0, 1, (n, M.IN)).astype(np.float32)
    wtrue = rng.normal(0, 1, (M.IN, M.OUT))
    y = (np.sin(x @ wtrue) + 0.5 * x[:, :1]).astype(np.float32)
    mask = (rng.uniform(size=(n, M.OUT)) < 0.9).astype(np.float32)
    members = 5
    params = torch.zeros(members * M.P, dtype=torch.float32, device="cuda")
    _lib.check(_lib.tempi().tempi_mlp_init(ctypes.c_void_p(params.data_ptr()), members, 7))
    dx, dy, dm = _dev(x[:3000]), _dev(y[:3000]), _dev(mask[:3000])
    xt = _dev(x[3000:])

    def heldout_mse():
        out = torch.zeros(members * 1000 * M.OUT, dtype=torch.float32, device="cuda")
        _lib.check(_lib.tempi().tempi_mlp_predict(ctypes.c_void_p(params.data_ptr()), members,
                                                   ctypes.c_void_p(xt.data_ptr()), 1000,
                                                   ctypes.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        o = out.cpu().numpy().reshape(members, 1000, M.OUT).mean(0)
        return float(((o - y[3000:]) ** 2).mean())

    before = heldout_mse()
    losses = torch.zeros(members * 40, dtype=torch.float32, device="cuda")
    _lib.check(_lib.tempi().tempi_mlp_train(
        ctypes.c_void_p(params.data_ptr()), members, ctypes.c_void_p(dx.data_ptr()),
        ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(dm.data_ptr()), 3000, 40, 64,
        ctypes.c_float(3e-3), 11, ctypes.c_void_p(losses.data_ptr()), None))
    torch.cuda.synchronize()
    after = heldout_mse()
    l = losses.cpu().numpy().reshape(members, 40)
    assert (l[:, -1] < 0.5 * l[:, 0]).all()
    assert after < 0.25 * before, (before, after)
