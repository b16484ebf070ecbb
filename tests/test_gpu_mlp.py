"""Tensor-core GEMM and coordinate-MLP kernels.

The GEMM (tcgen05, BF16 operands, FP32 accumulation) is compared with a plain
torch FP32 matmul of the same BF16-rounded operands; the network's gradients
with the CPU oracle (oracle/mlp_oracle.py, same BF16 rounding points, FP64
accumulation); and training must reduce the loss.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


# TMA-fed kernel: row strides that are multiples of 8 elements and split
# ranges of whole 64-wide chunks (ragged M, N, K edges arrive as zeros); the
# register-staged kernel: K = 100 or 300 (row strides of 200 / 600 bytes) and
# split ranges of 96.
@pytest.mark.parametrize("M,N,K,k_split", [(128, 256, 64, 64), (300, 256, 128, 128), (77, 128, 200, 200),
                                           (256, 256, 4096, 1024), (512, 128, 256, 256), (96, 200, 100, 100),
                                           (130, 256, 300, 96), (200, 72, 256, 256)])
def test_tc_gemm_matches_torch_fp32(M, N, K, k_split):
    from supersonicflowsolver_b200.mlp import tc_gemm

    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    D = tc_gemm(A, B, k_split=k_split).sum(dim=0)
    ref = A.float() @ B.float().T
    # FP32 accumulation in a different order: |error| <= K * 2^-23 * sum |a b|
    bound = (A.float().abs() @ B.float().abs().T) * (K * 2.0 ** -23) + 1e-6
    assert torch.all((D - ref).abs() <= bound), float(((D - ref).abs() / bound).max())


def test_tc_gemm_transposed_operands():
    """A and B given through strides (the weight-gradient form: A = X^T, B = Y^T)."""
    from supersonicflowsolver_b200.mlp import tc_gemm

    g = torch.Generator(device="cuda").manual_seed(3)
    X = torch.randn((1000, 256), generator=g, device="cuda").to(torch.bfloat16)  # [batch][256]
    Y = torch.randn((1000, 128), generator=g, device="cuda").to(torch.bfloat16)  # [batch][128]
    D = tc_gemm(X, Y, k_split=256, a_strides=(1, 256), b_strides=(1, 128), M=256, N=128, K=1000).sum(dim=0)
    ref = X.float().T @ Y.float()
    bound = (X.float().abs().T @ Y.float().abs()) * (1000 * 2.0 ** -23) + 1e-6
    assert torch.all((D - ref).abs() <= bound)


def batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 2]) * x[:, 0], x[:, 3] ** 2, 0.3 * x[:, 1] * x[:, 2], np.cos(x[:, 2] + x[:, 3])],
                 axis=1).astype(np.float32)
    return x, t


def test_mlp_gradients_match_cpu_oracle():
    from supersonicflowsolver_b200.mlp import MLP

    net = MLP(seed=11)
    x, t = batch(300, 1)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    g, loss = net.gradients(xd, td)
    p = net.params()
    oloss, og, oy = mo.loss_and_grads(p, x, t, bf16_points=True)
    y = net.forward(xd).cpu().numpy()
    assert rel_err(y, oy) < 2e-3
    assert abs(loss - oloss) <= 1e-3 * oloss
    off = 0
    for l in range(6):
        for n in (mo.DOUT[l] * mo.DIN[l], mo.DOUT[l]):
            a, b = g[off:off + n], og[off:off + n]
            # BF16 deltas agree up to one BF16 ulp flips; FP32 vs FP64 accumulation
            assert rel_err(a, b) < 2e-2, (l, n, rel_err(a, b))
            cos = float(np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos > 0.9999, (l, n, cos)
            off += n


def test_mlp_training_reduces_loss():
    from supersonicflowsolver_b200.mlp import MLP

    net = MLP(seed=5)
    x, t = batch(4096, 2)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = net.train_step(xd, td, 1e-3)
    for _ in range(300):
        last = net.train_step(xd, td, 1e-3)
    assert np.isfinite(last) and last < 0.1 * first, (first, last)
    # deterministic: same seed, same data, same steps -> same parameters
    net2 = MLP(seed=5)
    for _ in range(301):
        net2.train_step(xd, td, 1e-3)
    assert np.array_equal(net.params(), net2.params())


@pytest.mark.parametrize("M,N,K", [(200, 72, 1000), (256, 256, 4096), (40, 136, 64), (36, 100, 300), (44, 256, 520)])
def test_tc_gemm_transposed_ragged(M, N, K):
    """Operands contiguous along M and N (the weight-gradient form) with a
    ragged last K chunk: with 16-byte row strides (M, N multiples of 8) TMA
    loads them as they are and the MMA reads them MN-major; otherwise (36,
    100, 44) they are loaded as 16-byte vectors where aligned, element by
    element where not, and transposed in registers."""
    from supersonicflowsolver_b200.mlp import tc_gemm

    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    X = torch.randn((K, M), generator=g, device="cuda").to(torch.bfloat16)  # [batch][M]
    Y = torch.randn((K, N), generator=g, device="cuda").to(torch.bfloat16)  # [batch][N]
    D = tc_gemm(X, Y, k_split=512, a_strides=(1, M), b_strides=(1, N), M=M, N=N, K=K).sum(dim=0)
    ref = X.float().T @ Y.float()
    bound = (X.float().abs().T @ Y.float().abs()) * (K * 2.0 ** -23) + 1e-6
    assert torch.all((D - ref).abs() <= bound), float(((D - ref).abs() / bound).max())


def test_tc_gemm_wait_that_runs_out_is_reported():
    """A first mbarrier wait bounded at zero polls gives up at once: the call
    returns PSST_ERR_TIMEOUT (after draining the MMAs in flight), and the next
    call with the default bound computes the product."""
    from supersonicflowsolver_b200.mlp import tc_gemm
    from supersonicflowsolver_b200.psst import PsstError

    g = torch.Generator(device="cuda").manual_seed(11)
    A = torch.randn((256, 512), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((256, 512), generator=g, device="cuda").to(torch.bfloat16)
    for polls in (0, 0):
        with pytest.raises(PsstError) as e:
            tc_gemm(A, B, wait_polls=polls)
        assert e.value.status == 7
    D = tc_gemm(A, B, wait_polls=-1)[0]
    ref = A.float() @ B.float().T
    bound = (A.float().abs() @ B.float().abs().T) * (512 * 2.0 ** -23) + 1e-6
    assert torch.all((D - ref).abs() <= bound)


def test_network_runs_in_order_with_torch_default_stream():
    """With torch on its default stream (the legacy NULL stream, handle 0), the
    network's kernels are ordered after the kernels that made their input:
    an input copied in behind a 25 ms spin kernel is the one the forward pass
    reads."""
    from supersonicflowsolver_b200.mlp import MLP

    if not hasattr(torch.cuda, "_sleep"):
        pytest.skip("torch.cuda._sleep not available")
    assert torch.cuda.current_stream().cuda_stream == 0
    net = MLP(seed=1)
    x_real = torch.rand((1024, 4), device="cuda") * 2.0 - 1.0
    y_ref = net.forward(x_real).cpu()
    x = torch.zeros_like(x_real)
    torch.cuda.synchronize()
    torch.cuda._sleep(50_000_000)  # about 25 ms of clock cycles on torch's current stream
    x.copy_(x_real)
    y = net.forward(x).cpu()
    assert torch.equal(y, y_ref)
