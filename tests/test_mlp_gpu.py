"""The bracket-predictor network's tensor-core kernels against plain FP32 / FP64 arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 192), (512, 128, 1024), (128, 128, 2048),
                                   (2048, 128, 128)])
def test_gemm_bf16_tensor_cores(M, N, K):
    """C = A B^T on tcgen05 (BF16 operands, FP32 accumulation, two shared-memory stages; outputs of
    few tiles split over K across CTAs and summed in order: (512, 128, 1024) in 8 splits,
    (128, 128, 2048) -- the weight-gradient shape -- in 16) equals the FP32 product of the same BF16
    values to FP32 summation-order round-off; accumulate adds to C"""
    import torch
    from agama_b200 import _native
    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    C = torch.full((M, N), 7.0, dtype=torch.float32, device="cuda")
    ref = A.float() @ B.float().T
    L = _native.lib()
    _native.check(L.agama_gemmBf16Device(M, N, K, _native.VP(A.data_ptr()), _native.VP(B.data_ptr()),
                                         _native.VP(C.data_ptr()), N, 0, None))
    torch.cuda.synchronize()
    scale = np.sqrt(K)
    assert torch.max(torch.abs(C - ref)).item() <= 1e-5 * scale
    _native.check(L.agama_gemmBf16Device(M, N, K, _native.VP(A.data_ptr()), _native.VP(B.data_ptr()),
                                         _native.VP(C.data_ptr()), N, 1, None))
    torch.cuda.synchronize()
    assert torch.max(torch.abs(C - 2 * ref)).item() <= 2e-5 * scale


def _oracle():
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import mlp_ref
    return mlp_ref


def test_gradients_match_the_cpu_oracle():
    """the device loss and gradient (tcgen05 products in BF16, FP32 elsewhere) against the CPU FP64
    network: with the same BF16 rounding points to 1e-3 of the gradient norm per layer, and
    against pure FP64 to 3e-2"""
    import agama_b200
    R = _oracle()
    rng = np.random.default_rng(7)
    net = agama_b200.BracketNet(seed=3)
    p, _ = net.params()
    B = 256
    x = rng.normal(size=(B, 6)).astype(np.float32)
    t = rng.normal(size=(B, 3)).astype(np.float32)
    m = (rng.uniform(size=(B, 3)) > 0.25).astype(np.float32)
    loss, g = net.loss_grad(x, t, m)
    lb, gb = R.loss_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64), m.astype(np.float64), bf=True)
    l64, g64 = R.loss_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64), m.astype(np.float64))
    assert abs(loss - lb) <= 1e-4 * abs(lb)
    k = 0
    for o, i in R.SIZES:
        for sl in (slice(k, k + o * i), slice(k + o * i, k + o * i + o)):
            ref, ref64 = gb[sl], g64[sl]
            assert np.linalg.norm(g[sl] - ref) <= 1e-3 * np.linalg.norm(ref), (o, i, sl)
            assert np.linalg.norm(g[sl] - ref64) <= 3e-2 * np.linalg.norm(ref64), (o, i, sl)
        k += o * i + o


def test_fused_inference_matches_the_cpu_oracle():
    """the fused tcgen05 inference kernel against the CPU network with the same BF16 rounding
    points, including the input / output standardisation and a ragged last tile"""
    import agama_b200
    R = _oracle()
    rng = np.random.default_rng(11)
    net = agama_b200.BracketNet(seed=5)
    p, _ = net.params()
    scaling = np.concatenate([rng.normal(size=6), rng.uniform(0.5, 2, 6), rng.normal(size=3), rng.uniform(0.5, 2, 3)])
    net.set_params(scaling=scaling)
    n = 1000
    x = rng.normal(size=(n, 6)) * scaling[6:12] + scaling[:6]
    y = net.predict(x)
    xs = (x.astype(np.float32) - scaling[:6].astype(np.float32)) / scaling[6:12].astype(np.float32)
    yref = R.forward(p.astype(np.float64), xs.astype(np.float64), bf=True)[0] * scaling[15:18] + scaling[12:15]
    err = np.abs(y - yref) / scaling[15:18]
    assert np.max(err) <= 2e-3, np.max(err)


def test_training_learns_a_smooth_function():
    """Adam on the device: the loss of a smooth 6 -> 3 target falls by an order of magnitude and the
    trained network predicts held-out points"""
    import agama_b200
    rng = np.random.default_rng(1)
    n = 32768
    x = rng.normal(size=(n + 4096, 6))
    t = np.column_stack([np.sin(x[:, 0] + 0.5 * x[:, 1]), x[:, 2] * x[:, 3] * 0.5, np.tanh(x[:, 4] - x[:, 5])]) * 3 + 1
    m = np.ones_like(t)
    net = agama_b200.BracketNet(seed=2)
    hist = net.train(x[:n], t[:n], m[:n], epochs=8, batch=1024, lr=3e-3)
    assert hist[-1] < 0.1 * hist[0], hist
    y = net.predict(x[n:])
    resid = np.mean((y - t[n:]) ** 2, axis=0) / np.var(t[n:], axis=0)
    assert np.all(resid < 0.05), resid
