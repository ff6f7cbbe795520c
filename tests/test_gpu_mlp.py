"""The warm-start MLP's tensor-core kernels (ofg_mlp_*: tcgen05.mma GEMMs)
against a plain FP32 restatement of the same network on the CPU: forward
within the BF16 rounding of weights and activations (tolerance 2e-2
relative), gradients to the same level, and Adam training that fits a smooth
field."""
import numpy as np
import pytest
import torch

from oneflow_b200.mlp import MLP

pytestmark = pytest.mark.gpu


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float32)


def torch_forward(net, flat, x, emulate_bf16=True):
    """FP32 reference; with emulate_bf16 the weights, inputs and hidden
    activations are rounded to BF16 where the kernels store them in BF16"""
    layers = net.unpack(flat)
    h = bf16(x) if emulate_bf16 else x
    for k, (W, b) in enumerate(layers):
        W = torch.tensor(W, device=x.device)
        b = torch.tensor(b, device=x.device)
        z = h @ (bf16(W) if emulate_bf16 else W) + b
        if k + 1 < len(layers):
            h = torch.nn.functional.gelu(z)
            h = bf16(h) if emulate_bf16 else h
        else:
            h = z
    return h


def data(n, n_in, n_out, seed=0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.rand((n, n_in), generator=g) * 2 - 1
    cols = [torch.sin(3 * x[:, 0]) * torch.cos(2 * x[:, 1 % n_in]), x[:, 0] * x[:, -1], torch.tanh(x.sum(1))]
    y = torch.stack([cols[k % 3] for k in range(n_out)], 1)
    return x.float().cuda().contiguous(), y.float().cuda().contiguous()


@pytest.mark.parametrize("shape", [(8, 64, 3, 4), (22, 256, 6, 5)])
def test_forward_matches_a_cpu_fp32_restatement(shape):
    net = MLP(*shape, seed=3)
    x, _ = data(1000, shape[0], shape[3])
    y = net.predict(x).cpu()
    ref = torch_forward(net, net.params(), x.cpu())
    err = (y - ref).abs().max().item() / ref.abs().max().item()
    assert err < 2e-2, err


@pytest.mark.parametrize("shape,rows", [((8, 64, 3, 4), 4096), ((22, 256, 6, 5), 4160)])
def test_gradient_matches_a_cpu_fp32_restatement(shape, rows):
    # rows 4,160 = 32.5 row tiles of 128: a partial tile; width 256 = two column tiles
    net = MLP(*shape, seed=5)
    x, y = data(rows, shape[0], shape[3], seed=1)
    loss, g = net.loss_grad(x, y)
    flat = torch.tensor(net.params(), device="cpu", requires_grad=True)
    x, y = x.cpu(), y.cpu()
    # the same network in FP32 on the CPU with torch's autograd, BF16 rounding
    # emulated in the forward (straight-through in the backward)
    layers, o = [], 0
    for fi, fo in net.layer_shapes():
        layers.append((flat[o:o + fi * fo].view(fi, fo), flat[o + fi * fo:o + fi * fo + fo]))
        o += fi * fo + fo
    h = bf16(x)
    for k, (W, b) in enumerate(layers):
        Wq = W + (bf16(W.detach()) - W.detach())
        z = h @ Wq + b
        if k + 1 < len(layers):
            a = torch.nn.functional.gelu(z)
            h = a + (bf16(a.detach()) - a.detach())
        else:
            h = z
    ref_loss = ((h - y) ** 2).mean()
    ref_loss.backward()
    gr = flat.grad.numpy()
    assert abs(loss - ref_loss.item()) <= 1e-2 * ref_loss.item()
    cos = float(np.dot(g, gr) / (np.linalg.norm(g) * np.linalg.norm(gr)))
    assert cos > 0.999, cos
    assert np.linalg.norm(g - gr) / np.linalg.norm(gr) < 3e-2


def test_training_fits_a_smooth_field():
    shape = (8, 64, 3, 4)
    net = MLP(*shape, seed=7)
    x, y = data(32768, shape[0], shape[3], seed=2)
    l0, _ = net.loss_grad(x[:8192], y[:8192])
    losses = net.train(x, y, steps=600, batch=4096, lr=2e-3, seed=11)
    l1, _ = net.loss_grad(x[:8192], y[:8192])
    assert np.all(np.isfinite(losses))
    assert l1 < 0.05 * l0, (l0, l1)
    # deterministic: the same seeds give the same weights
    net2 = MLP(*shape, seed=7)
    net2.train(x, y, steps=600, batch=4096, lr=2e-3, seed=11)
    assert np.array_equal(net.params(), net2.params())
