"""The warm start's network on the tensor cores (tcgen05, BF16 operands, FP32
accumulation), through the C-ABI.

* The GEMM alone against a torch FP32 product of the same BF16-rounded
  operands (relative error within FP32 accumulation: 1e-4 of the row scale).
* One forward + backward against the CPU oracle (oracle/mlp_oracle.py), which
  rounds to BF16 where the GPU path does and sums in FP64: every gradient
  tensor within 1e-2 of its largest entry, correlation above 0.9999.
* Training lowers the loss and the trained network's outputs match the
  oracle's forward pass of the same parameters.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(128, 128, 64), (256, 512, 64), (100, 70, 24), (512, 64, 256), (300, 200, 520),
          (8, 8, 8)]


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_matches_fp32_on_bf16_operands(pkg, m, n, k):
    import torch
    rng = np.random.default_rng(m * 1000 + n + k)
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((n, k)).astype(np.float32)
    bias = rng.standard_normal(n).astype(np.float32)
    ab = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64)
    bb = torch.from_numpy(b).to(torch.bfloat16).to(torch.float64)
    ref = (ab @ bb.T).numpy()
    scale = (ab.abs() @ bb.abs().T).numpy() + 1e-30
    c = pkg.mlp.gemm_bf16(a, b)
    assert np.all(np.abs(c - ref) <= 1e-4 * scale + 1e-6), np.max(np.abs(c - ref) / scale)
    c2 = pkg.mlp.gemm_bf16(a, b, bias=bias, relu=True)
    ref2 = np.maximum(ref + bias, 0.0)
    assert np.all(np.abs(c2 - ref2) <= 1e-4 * (scale + np.abs(bias)) + 1e-6)


DIMS = (64, 512, 512)


def _problem(n_in, n_out, rows, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((rows, n_in)).astype(np.float32)
    proj = rng.standard_normal((n_in, n_out)) / np.sqrt(n_in)
    t = np.tanh(x @ proj).astype(np.float32)
    return x, t


def test_gradients_match_the_cpu_oracle(pkg):
    import mlp_oracle as mo
    n_in, hidden, n_out = DIMS
    x, t = _problem(n_in, n_out, 256, 1)
    params = mo.init_params(n_in, hidden, n_out, seed=2)
    with pkg.mlp.Mlp(n_in, hidden, n_out, max_batch=256) as net:
        net.set_params(params)
        assert np.array_equal(net.get_params(), params)
        g, loss = net.gradients(x, t)
    g_ref, loss_ref = mo.gradients(params, x, t, n_in, hidden, n_out)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    sizes = [hidden * n_in, hidden, hidden * hidden, hidden, n_out * hidden, n_out]
    o = 0
    for i, s in enumerate(sizes):
        a, b = g[o:o + s].astype(np.float64), g_ref[o:o + s]
        o += s
        assert np.max(np.abs(a - b)) <= 1e-2 * np.max(np.abs(b)), (i, np.max(np.abs(a - b)))
        assert np.corrcoef(a, b)[0, 1] > 0.9999, i


def test_training_lowers_the_loss_and_forward_matches_the_oracle(pkg):
    import mlp_oracle as mo
    n_in, hidden, n_out = DIMS
    x, t = _problem(n_in, n_out, 2048, 3)
    with pkg.mlp.Mlp(n_in, hidden, n_out, max_batch=256) as net:
        net.set_params(mo.init_params(n_in, hidden, n_out, seed=4))
        losses = net.train(x, t, epochs=30, batch=256, lr=1e-3, seed=5)
        assert losses[-1] < 0.2 * losses[0], losses
        params = net.get_params()
        y = net.forward(x[:100])
    _, _, _, y_ref = mo.forward(params, x[:100], n_in, hidden, n_out)
    assert np.max(np.abs(y - y_ref)) <= 1e-2 * np.max(np.abs(y_ref)) + 1e-3
