"""Surrogate network kernels on the GPU: the tcgen05 BF16 GEMM against a
float32 product of the same bf16 operands, the network's gradients against
the float64 CPU oracle (oracle/mlp_oracle.py), and training reducing the
loss."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch.device("cuda:0")


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (256, 256, 128), (384, 64, 576),
                                   (1024, 512, 512), (128, 128, 8192)])
def test_gemm_bf16_matches_fp32_product(M, N, K):
    from openhurricane_b200.surrogate import gemm_bf16
    dev = _dev()
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(dev)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(dev)
    bias = torch.randn(N, generator=g).to(dev)
    ref = A.float() @ B.float().T + bias
    out = gemm_bf16(A, B, bias)
    torch.cuda.synchronize()
    err = (out - ref).abs().max().item() / ref.abs().max().item()
    # same bf16 operands, fp32 accumulation: only the summation order differs
    assert err < 1e-5 * max(1.0, (K / 512) ** 0.5), err
    ref_g = torch.nn.functional.gelu(ref)
    out_g = gemm_bf16(A, B, bias, act=1)
    assert (out_g - ref_g).abs().max().item() < 1e-4 * ref.abs().max().item() + 1e-5


def test_gemm_rejects_unpadded_shapes():
    from openhurricane_b200 import _capi
    from openhurricane_b200.surrogate import gemm_bf16
    dev = _dev()
    A = torch.zeros(100, 64, dtype=torch.bfloat16, device=dev)
    B = torch.zeros(32, 64, dtype=torch.bfloat16, device=dev)
    with pytest.raises(_capi.HcError):
        gemm_bf16(A, B)


@pytest.mark.parametrize("shape", [(12, 10, 3, 256), (56, 54, 2, 512)])
def test_mlp_gradients_match_cpu_oracle(shape):
    from oracle import mlp_oracle
    from openhurricane_b200.surrogate import MLP
    dev = _dev()
    n_in, n_out, nh, w = shape
    net = MLP(n_in, n_out, nh, w, max_batch=1024, seed=5)
    rng = np.random.default_rng(1)
    B = 1000
    X = rng.normal(size=(B, n_in)).astype(np.float32)
    Y = rng.normal(size=(B, n_out)).astype(np.float32)
    theta = net.get_params()
    loss, g = net.grad(torch.tensor(X, device=dev), torch.tensor(Y, device=dev))
    shp = net.shapes()
    # oracle on the bf16-rounded parameters and inputs the GPU multiplies
    bf = lambda a: torch.tensor(a).to(torch.bfloat16).float().numpy().astype(np.float64)
    th = theta.astype(np.float64).copy()
    off = 0
    for o, i in shp:
        th[off:off + o * i] = bf(theta[off:off + o * i])
        off += o * i + o
    ref_loss, ref_g = mlp_oracle.loss_and_grad(th, shp, bf(X), Y)
    assert abs(loss - ref_loss) / ref_loss < 2e-2
    off = 0
    for o, i in shp:
        for part in (o * i, o):
            a, r = g[off:off + part], ref_g[off:off + part]
            rel = np.linalg.norm(a - r) / np.linalg.norm(r)
            cos = float(a @ r / (np.linalg.norm(a) * np.linalg.norm(r)))
            assert rel < 5e-2 and cos > 0.998, (o, i, part, rel, cos)
            off += part


def test_mlp_training_reduces_loss():
    from openhurricane_b200.surrogate import MLP
    dev = _dev()
    net = MLP(12, 10, 3, 256, max_batch=8192, seed=3)
    gen = torch.Generator(device="cpu").manual_seed(0)
    X = torch.randn(8192, 12, generator=gen)
    Wt = torch.randn(12, 10, generator=gen) / 4
    Y = torch.tanh(X @ Wt) + 0.1 * torch.sin(3 * X[:, :10])
    X, Y = X.to(dev).contiguous(), Y.to(dev).contiguous()
    first = net.train_step(X, Y, 1e-3, want_loss=True, check=True)
    for _ in range(300):
        net.train_step(X, Y, 1e-3)
    last = net.train_step(X, Y, 1e-3, want_loss=True, check=True)
    assert last < 0.1 * first, (first, last)
    pred = net.forward(X)
    mse = ((pred - Y) ** 2).mean().item()
    assert abs(mse - last) / last < 0.2
