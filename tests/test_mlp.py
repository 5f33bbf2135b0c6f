"""The closure MLP: the CPU oracle's gradients against finite differences
(CPU), and the CUDA kernels (BF16 tensor cores, FP32 accumulate) against
the oracle (GPU).  Tolerances, normwise relative max|a-b|/max|b|:
  * oracle gradient vs central differences (FP64, no BF16): <= 1e-6;
  * kernel forward vs the BF16-emulating oracle: <= 2e-3;
  * kernel gradient vs the BF16-emulating oracle: <= 2e-2 (a BF16 rounding
    can fall the other way when the FP32 and FP64 sums differ);
  * Adam vs the oracle's Adam: <= 1e-5;
  * a 400-step training run cuts the loss of a smooth target 5-fold."""

import numpy as np
import pytest

from conftest import rel_err


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 48))
    x[:, :45] = rng.standard_normal((n, 45))
    t = np.stack([np.sin(x[:, 0] + 0.5 * x[:, 3]) * 0.7, np.tanh(x[:, 1] - x[:, 7] * x[:, 2] * 0.3)], 1)
    return x, t


def test_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle as mo
    x, t = _data(37, 1)
    p = mo.init_params(2).astype(np.float64)
    p[mo.OFF_B1:mo.OFF_W2] = 0.01 * np.arange(64)
    _, g = mo.loss_grad(p, x, t, emulate=False)
    rng = np.random.default_rng(3)
    idx = rng.choice(np.flatnonzero(g != 0), 60, replace=False)
    h = 1e-6
    fd = []
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd.append((mo.loss_grad(pp, x, t, False)[0] - mo.loss_grad(pm, x, t, False)[0]) / (2 * h))
    assert rel_err(g[idx], np.array(fd)) <= 1e-6


@pytest.mark.gpu
def test_kernels_match_oracle(gpu):
    import torch
    from oracle import mlp_oracle as mo
    from inmsom_elfs_b200.mlp import MLP
    x, t = _data(1024, 4)
    net = MLP(seed=5)
    p = net.host_params()
    xd = torch.from_numpy(x.astype(np.float32)).to("cuda").to(torch.bfloat16)
    td = torch.from_numpy(t.astype(np.float32)).to("cuda")
    y = net.forward(xd).cpu().numpy()
    yo, _ = mo.forward(p, x, emulate=True)
    assert rel_err(y, yo) <= 2e-3
    g = net.loss_grad(xd, td).cpu().numpy()
    lo, go = mo.loss_grad(p, x, t, emulate=True)
    assert abs(g[-1] - lo) <= 1e-3 * lo
    for a, b in ((mo.OFF_W1, mo.OFF_B1), (mo.OFF_B1, mo.OFF_W2), (mo.OFF_W2, mo.OFF_B2), (mo.OFF_B2, mo.OFF_W3),
                 (mo.OFF_W3, mo.OFF_B3), (mo.OFF_B3, mo.NPARAM)):
        assert rel_err(g[a:b], go[a:b]) <= 2e-2, (a, b, rel_err(g[a:b], go[a:b]))
    # gather through an index list: the same as the listed rows
    idx = torch.arange(1023, -1, -1, dtype=torch.int32, device="cuda")[:512]
    g2 = net.loss_grad(xd, td, idx, 512).cpu().numpy()
    _, go2 = mo.loss_grad(p, x[1023:511:-1], t[1023:511:-1], emulate=True)
    assert rel_err(g2[:-1], go2) <= 2e-2
    # Adam
    net.loss_grad(xd, td)
    gd = net.grad.cpu().numpy()[:-1].astype(np.float64)
    net.adam(lr=1e-3)
    pa, _, _ = mo.adam(p.astype(np.float64), np.zeros(mo.NPARAM), np.zeros(mo.NPARAM), gd, 1)
    assert rel_err(net.host_params(), pa) <= 1e-5


@pytest.mark.gpu
def test_training_reduces_loss(gpu):
    import torch
    from inmsom_elfs_b200.mlp import MLP
    x, t = _data(1 << 15, 6)
    xd = torch.from_numpy(x.astype(np.float32)).to("cuda").to(torch.bfloat16)
    td = torch.from_numpy(t.astype(np.float32)).to("cuda")
    net = MLP(seed=7)
    l0 = float(net.loss_grad(xd, td)[-1].item())
    net.train(xd, td, steps=400, batch=4096, lr=3e-3)
    l1 = float(net.loss_grad(xd, td)[-1].item())
    assert l1 < 0.2 * l0, (l0, l1)

