"""The BF16 tensor-core MLP kernels against the CPU oracle (oracle/mlp.py).

GEMM: every epilogue against a float64 product of the same bf16 operands.
Training: loss and all weight and bias gradients of a small network against
the oracle's backward pass (which rounds to bf16 where the kernels store
bf16), and the oracle's gradient against central finite differences of its
own loss.  Adam: one step against the textbook update.
"""

import numpy as np
import pytest

from oracle import mlp as om

torch = pytest.importorskip("torch")


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    W = [rng.standard_normal((6, 5)).astype(np.float32) * 0.5, rng.standard_normal((3, 6)).astype(np.float32) * 0.5]
    b = [rng.standard_normal(6) * 0.1, rng.standard_normal(3) * 0.1]
    X = rng.standard_normal((7, 5)).astype(np.float32)
    T = rng.standard_normal((7, 3))

    # exact-arithmetic loss (no bf16 rounding) for the difference quotient
    def loss64(W0):
        a = X.astype(np.float64)
        z = a @ W0.T + b[0]
        y = om.gelu(z) @ W[1].astype(np.float64).T + b[1]
        return np.mean((y - T) ** 2)

    def grad64(W0):
        a = X.astype(np.float64)
        z = a @ W0.T + b[0]
        h = om.gelu(z)
        y = h @ W[1].astype(np.float64).T + b[1]
        d = 2.0 * (y - T) / y.size
        dz = (d @ W[1].astype(np.float64)) * om.gelu_grad(z)
        return dz.T @ a

    W0 = W[0].astype(np.float64)
    g = grad64(W0)
    eps = 1e-6
    for (i, j) in [(0, 0), (2, 3), (5, 4)]:
        Wp, Wm = W0.copy(), W0.copy()
        Wp[i, j] += eps
        Wm[i, j] -= eps
        fd = (loss64(Wp) - loss64(Wm)) / (2 * eps)
        assert abs(fd - g[i, j]) <= 1e-6 * max(1.0, abs(fd))


def _bf(x):
    return torch.from_numpy(om.bf16(np.asarray(x, dtype=np.float32))).to(torch.bfloat16).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("N,bn,kernel", [(384, 128, 0), (512, 256, 0), (384, 128, 1), (512, 256, 1)])
def test_gemm_epilogues_match_float64(N, bn, kernel):
    from hexdyn import mlp

    assert torch.cuda.is_available()
    rng = np.random.default_rng(N)
    M, K = 640, 192  # five row tiles: the persistent kernel loops over several tiles per CTA
    A = om.bf16(rng.standard_normal((M, K)).astype(np.float32))
    B = om.bf16(rng.standard_normal((N, K)).astype(np.float32) * 0.1)
    bias = rng.standard_normal(N).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    At, Bt = _bf(A), _bf(B)
    Cf = torch.empty(M, N, dtype=torch.float32, device="cuda")
    err = mlp.gemm(At, Bt, epilogue=mlp.EPI_F32, Cf=Cf, bn=bn, kernel=kernel)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    np.testing.assert_allclose(Cf.cpu().numpy(), ref, rtol=0, atol=1e-4 * np.abs(ref).max())
    # bias + GELU: Z, H and H^T
    H = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    Ht = torch.empty(N, M, dtype=torch.bfloat16, device="cuda")
    Z = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    mlp.gemm(At, Bt, epilogue=mlp.EPI_GELU, bias=torch.from_numpy(bias).cuda(), C_out=H, Ct=Ht, Z=Z, err=err, bn=bn, kernel=kernel)
    z = ref + bias
    np.testing.assert_allclose(Z.float().cpu().numpy(), z, rtol=1e-2, atol=1e-2)
    h = om.gelu(z)
    np.testing.assert_allclose(H.float().cpu().numpy(), h, rtol=1e-2, atol=1e-2)
    np.testing.assert_array_equal(Ht.float().cpu().numpy(), H.float().cpu().numpy().T)
    # GELU' epilogue on a given Z
    D = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    Dt = torch.empty(N, M, dtype=torch.bfloat16, device="cuda")
    mlp.gemm(At, Bt, epilogue=mlp.EPI_GELU_GRAD, C_out=D, Ct=Dt, Zin=Z, err=err, bn=bn, kernel=kernel)
    want = ref * om.gelu_grad(Z.float().cpu().numpy())
    np.testing.assert_allclose(D.float().cpu().numpy(), want, rtol=1e-2, atol=1e-2 * np.abs(want).max())
    np.testing.assert_array_equal(Dt.float().cpu().numpy(), D.float().cpu().numpy().T)
    torch.cuda.synchronize()
    assert int(err.item()) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("bn", [128, 256])
def test_gemm_gives_up_cleanly_when_its_wait_runs_out(bn):
    """The persistent GEMM's bounded waits: with the MMA issuer allowed no
    poll of its first loaded stage, every CTA gives up, reports through the
    error word and returns (its loads and MMAs drained, tensor memory freed);
    normal GEMMs right after it on every SM run and are correct."""
    import time

    from hexdyn import mlp

    assert torch.cuda.is_available()
    rng = np.random.default_rng(7)
    M, N, K = 128 * 160, 2 * bn, 256  # 320 tiles: every SM's CTA takes part
    A = om.bf16(rng.standard_normal((M, K)).astype(np.float32))
    B = om.bf16(rng.standard_normal((N, K)).astype(np.float32) * 0.1)
    At, Bt = _bf(A), _bf(B)
    Cf = torch.empty(M, N, dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    err = mlp.gemm(At, Bt, epilogue=mlp.EPI_F32, Cf=Cf, bn=bn, mma_wait_polls=0)
    torch.cuda.synchronize()
    assert int(err.item()) == 1
    assert time.perf_counter() - t0 < 30.0
    ref = A[:256].astype(np.float64) @ B.astype(np.float64).T
    for _ in range(2):
        err = mlp.gemm(At, Bt, epilogue=mlp.EPI_F32, Cf=Cf, bn=bn)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        np.testing.assert_allclose(Cf[:256].cpu().numpy(), ref, rtol=0, atol=1e-4 * np.abs(ref).max())


@pytest.mark.gpu
def test_training_gradients_match_oracle():
    from hexdyn import mlp

    rng = np.random.default_rng(1)
    net = mlp.TensorCoreMLP(50, 96, 2, 20, seed=3)
    M, m_valid = 256, 200
    X = np.zeros((M, net.p_in), dtype=np.float32)
    X[:m_valid, :50] = rng.standard_normal((m_valid, 50))
    T = np.zeros((M, net.p_out), dtype=np.float32)
    T[:m_valid, :20] = rng.standard_normal((m_valid, 20))
    # non-zero biases on the real units so that the bias path is exercised
    # (padded units keep a zero bias, hence zero activation)
    for i, lay in enumerate(net.layers):
        real = net.hidden if i < net.depth else net.n_out
        bias = np.zeros(lay.b.shape[0], dtype=np.float32)
        bias[:real] = rng.standard_normal(real) * 0.1
        lay.b.copy_(torch.from_numpy(bias))
    Xb = _bf(X)
    Xt = Xb.t().contiguous()
    loss = net.gradients(Xb, Xt, torch.from_numpy(T).cuda(), m_valid)
    torch.cuda.synchronize()
    net.check()
    W = [lay.w.cpu().numpy() for lay in net.layers]
    b = [lay.b.cpu().numpy().astype(np.float64) for lay in net.layers]
    ref_loss, gw, gb = om.gradients(W, b, X, T, m_valid, 20)
    assert abs(float(loss.item()) - ref_loss) <= 2e-3 * ref_loss
    for i, lay in enumerate(net.layers):
        g = lay.gw.cpu().numpy()
        rel = np.linalg.norm(g - gw[i]) / max(np.linalg.norm(gw[i]), 1e-30)
        assert rel < 2e-2, (i, rel)
        gbi = lay.gb.cpu().numpy()
        relb = np.linalg.norm(gbi - gb[i]) / max(np.linalg.norm(gb[i]), 1e-30)
        assert relb < 2e-2, (i, relb)
    # the padded rows and columns of every layer stay exactly zero
    for i, lay in enumerate(net.layers):
        g = lay.gw.cpu().numpy()
        rows = net.hidden if i < net.depth else net.n_out
        cols = net.n_in if i == 0 else net.hidden
        assert not np.any(g[rows:, :]) and not np.any(g[:, cols:])


@pytest.mark.gpu
def test_adam_step_matches_formula():
    from hexdyn import mlp

    net = mlp.TensorCoreMLP(16, 128, 1, 8, seed=0)
    lay = net.layers[0]
    rng = np.random.default_rng(2)
    g = rng.standard_normal(tuple(lay.gw.shape)).astype(np.float32)
    lay.gw.copy_(torch.from_numpy(g))
    w0 = lay.w.cpu().numpy().copy()
    net.adam(1e-3)
    torch.cuda.synchronize()
    m = 0.1 * g
    v = 0.001 * g * g
    want = w0 - 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    np.testing.assert_allclose(lay.w.cpu().numpy(), want, rtol=1e-5, atol=1e-7)
    np.testing.assert_array_equal(lay.wb.float().cpu().numpy(), om.bf16(lay.w.cpu().numpy()))
    np.testing.assert_array_equal(lay.wbt.float().cpu().numpy(), om.bf16(lay.w.cpu().numpy()).T)
