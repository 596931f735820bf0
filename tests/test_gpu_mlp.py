"""tcgen05 BF16 GEMM and the surrogate's training kernels: GEMM against a
float32 product of the same BF16 operands, gradients against the NumPy
oracle (oracle/mlp.py), and a short training run that must lower the loss."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import _lib, surrogate as sg  # noqa: E402
from oracle import mlp as omlp  # noqa: E402


def _toy_model(seed):
    prof = np.array([[0.0, 1.0], [1.0, 0.0]])
    return sg.FieldSurrogate(prof, np.ones(2), 1.0, np.ones(sg.N_SCALE_BINS), seed=seed)


def _mat(g, shape):
    return (torch.randn(shape, generator=g, device="cuda") * 0.5).to(torch.bfloat16)


@pytest.mark.parametrize("a_mn,b_mn", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_gemm_all_operand_layouts(a_mn, b_mn):
    g = torch.Generator(device="cuda").manual_seed(1)
    M, N, K = 256, 128, 192
    A = _mat(g, (M, K))
    B = _mat(g, (N, K))
    As = A.t().contiguous() if a_mn else A
    Bs = B.t().contiguous() if b_mn else B
    C = torch.full((M, N), float("nan"), device="cuda")
    sg._gemm(As, a_mn, M if a_mn else K, Bs, b_mn, N if b_mn else K, M, N, K, _lib.EPI_STORE, C=C, ldc=N,
             stream=sg._stream())
    ref = A.float() @ B.float().t()
    torch.cuda.synchronize()
    np.testing.assert_allclose(C.cpu().numpy(), ref.cpu().numpy(), rtol=1e-4, atol=1e-4)


def test_gemm_split_k_and_epilogues():
    g = torch.Generator(device="cuda").manual_seed(2)
    M, N, K = 128, 128, 512
    A, B = _mat(g, (M, K)), _mat(g, (N, K))
    part = torch.empty((4, M, N), device="cuda")
    sg._gemm(A, 0, K, B, 0, K, M, N, K, _lib.EPI_STORE, C=part, ldc=N, split=4, split_stride=M * N,
             stream=sg._stream())
    ref = A.float() @ B.float().t()
    torch.cuda.synchronize()
    np.testing.assert_allclose(part.sum(0).cpu().numpy(), ref.cpu().numpy(), rtol=1e-4, atol=1e-3)
    bias = torch.randn(N, generator=g, device="cuda")
    Z = torch.empty((M, N), device="cuda")
    H = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    sg._gemm(A[:, :128].contiguous(), 0, 128, B[:, :128].contiguous(), 0, 128, M, N, 128, _lib.EPI_BIAS_SILU, C=Z,
             bias=bias, H=H, stream=sg._stream())
    z_ref = A[:, :128].float() @ B[:, :128].float().t() + bias
    torch.cuda.synchronize()
    np.testing.assert_allclose(Z.cpu().numpy(), z_ref.cpu().numpy(), rtol=1e-4, atol=1e-4)
    h_ref = (z_ref * torch.sigmoid(z_ref)).to(torch.bfloat16).float()
    np.testing.assert_allclose(H.float().cpu().numpy(), h_ref.cpu().numpy(), rtol=1e-2, atol=1e-2)


def test_training_gradients_match_oracle():
    model = _toy_model(3)
    rng = np.random.default_rng(0)
    n = 256
    x = rng.uniform(-1, 1, (n, 2)).astype(np.float32)
    t = rng.normal(0, 1, (n, 2)).astype(np.float32)
    work = sg._Work(n, model.device, model.n_params)
    xb, tb = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    work.g.zero_()
    work.loss.zero_()
    sg.forward(model, xb, work, target=tb, inv_batch=1.0 / n)
    sg.backward(model, xb, work)
    torch.cuda.synchronize()
    loss, grads, y = omlp.forward_backward(model.params_dict(), x.astype(np.float64), t.astype(np.float64))
    assert abs(work.loss.item() - loss) <= 1e-4 * abs(loss)
    np.testing.assert_allclose(work.y.cpu().numpy(), y, rtol=2e-3, atol=2e-3)
    for name, _ in sg.PARAM_SHAPES:
        gg = model.view(work.g, name).cpu().numpy().astype(np.float64)
        ref = grads[name]
        rel = np.linalg.norm(gg - ref) / max(np.linalg.norm(ref), 1e-30)
        assert rel < 2e-2, (name, rel)


def test_short_training_lowers_loss():
    """Fit a smooth 2-D field for 300 steps: the loss must drop by 10x."""
    model = _toy_model(5)
    rng = np.random.default_rng(1)
    n = 1024
    x = rng.uniform(-1, 1, (n * 16, 2)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 1], np.cos(x[:, 0] + x[:, 1])], -1).astype(np.float32)
    X, T = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    work = sg._Work(n, model.device, model.n_params)
    m = torch.zeros(model.n_params, device="cuda")
    v = torch.zeros_like(m)
    losses = []
    for step in range(1, 301):
        sl = slice(((step - 1) % 16) * n, ((step - 1) % 16 + 1) * n)
        work.g.zero_()
        work.loss.zero_()
        sg.forward(model, X[sl], work, target=T[sl], inv_batch=1.0 / n)
        sg.backward(model, X[sl], work)
        sg.adam_step(model, work, m, v, 1e-3, step)
        losses.append(work.loss.item())
    assert np.mean(losses[-20:]) < 0.1 * np.mean(losses[:5]), (losses[:5], losses[-5:])
