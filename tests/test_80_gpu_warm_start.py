"""The warm-start network (fg_ws_*): its tcgen05 forward convolutions, the
moment-matching statistics and every gradient against a plain PyTorch FP32
reference on the CPU (periodic conv3d by circular padding, autograd), with
the device's BF16 roundings of weights, activations and gradient operands
reproduced in the reference; and a short training that lowers the loss."""
import numpy as np
import pytest

from feram_b200 import warm_start as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
F = torch.nn.functional


class _RoundGrad(torch.autograd.Function):
    """Identity whose backward rounds the gradient to BF16 (the device feeds
    dL/dpre to the tensor cores as BF16)."""

    @staticmethod
    def forward(ctx, a):
        return a.clone()

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).to(torch.float32)


def _bf(a):
    return a.to(torch.bfloat16).to(torch.float32)


def _torch_stats(u, e):
    """site_stats of every sample; u (B, 3, Lz, Ly, Lx), e (B, 3)."""
    m = u.mean(dim=(2, 3, 4))
    axis = {0: 4, 1: 3, 2: 2}  # component -> tensor axis of its direction
    cl = sum((u[:, a] * torch.roll(u[:, a], -1, dims=axis[a] - 1)).mean(dim=(1, 2, 3)) for a in range(3))
    ct = sum((u[:, a] * torch.roll(u[:, a], -1, dims=axis[b] - 1)).mean(dim=(1, 2, 3))
             for a in range(3) for b in range(3) if b != a)
    return torch.stack([(m * e).sum(1), torch.sqrt((m * m).sum(1) + 1e-8), torch.sqrt(torch.sqrt((m ** 4).sum(1) + 1e-16)),
                        (u ** 2).sum(1).mean(dim=(1, 2, 3)),
                        (u ** 4).sum(1).mean(dim=(1, 2, 3)), cl, ct], dim=1)


def _reference(layers, B, L, x, cond, target, wts, extra=None):
    Lx, Ly, Lz = L
    h = torch.tensor(x).reshape(B, Lz, Ly, Lx, 16).permute(0, 4, 1, 2, 3).contiguous()
    params = []
    for l in range(4):
        w, b = layers[l]
        wt = torch.tensor(w).reshape(w.shape[0], 3, 3, 3, w.shape[2]).permute(0, 4, 1, 2, 3).contiguous()
        wt = _bf(wt).requires_grad_(True)
        bt = torch.tensor(b).requires_grad_(True)
        params.append((wt, bt))
    for l, (wt, bt) in enumerate(params):
        pre = F.conv3d(F.pad(h, (1, 1, 1, 1, 1, 1), mode="circular"), wt, bt)
        pre = _RoundGrad.apply(pre)
        h = _bf(F.silu(pre)) if l < 3 else pre
    u = 0.1 * h[:, :3]
    e = torch.tensor(np.asarray(cond)[:, 1:4] / 0.001, dtype=torch.float32)
    S = _torch_stats(u, e)
    loss = ((S - torch.tensor(target, dtype=torch.float32)) ** 2 * torch.tensor(wts, dtype=torch.float32)).sum(1).mean()
    total = loss
    if extra is not None:  # a loss term outside the statistics with dL/du = extra
        Lx, Ly, Lz = L
        ex = torch.tensor(extra, dtype=torch.float32).reshape(B, Lz, Ly, Lx, 3).permute(0, 4, 1, 2, 3)
        total = loss + (u * ex).sum()
    total.backward()
    return u, S, loss, params


@pytest.mark.parametrize("L,batch,extra", [((8, 8, 8), 2, False), ((12, 8, 4), 1, False), ((8, 8, 8), 2, True)])
def test_network_forward_and_gradients_match_torch(fg, L, batch, extra):
    """With extra: a further dL/du on the generated field (fg_ws_backward_du,
    the energy term's MD force in training)."""
    with W.WarmStartNet(L, batch=batch, seed=7) as net:
        rng = np.random.default_rng(3)
        for l in range(4):  # non-zero biases exercise the bias paths
            w, b, _, _ = net.layer(l)
            net.set_layer(l, w, rng.standard_normal(b.shape).astype(np.float32) * 0.1 * (b.shape[0] > 3))
        cond = np.array([[250.0 + 50 * i, 0.0, 0.0, 0.0005 * (i - 0.5), -5.0] for i in range(batch)])
        seeds = [11 + i for i in range(batch)]
        target = rng.standard_normal((batch, W.NSTAT)) * 0.01
        wts = np.abs(rng.standard_normal(W.NSTAT)) + 0.5
        nsite = L[0] * L[1] * L[2]
        dLdu = rng.standard_normal((batch, nsite, 3)).astype(np.float32) * 1e-3 if extra else None
        loss_dev = net.backward(cond, seeds, target, wts, dLdu)
        x, u_dev = net.io()
        S_dev = net.forward(cond, seeds)
        lay = [net.layer(l) for l in range(4)]
    grads = [(dw, db) for _, _, dw, db in lay]
    u_ref, S_ref, loss_ref, params = _reference([(w, b) for w, b, _, _ in lay], batch, L, x, cond, target, wts,
                                                dLdu)
    Lx, Ly, Lz = L
    u_ref = u_ref.detach().permute(0, 2, 3, 4, 1).reshape(-1, 3).numpy()
    assert np.abs(u_dev - u_ref).max() <= 1e-3 * np.abs(u_ref).max(), np.abs(u_dev - u_ref).max()
    assert np.allclose(S_dev, S_ref.detach().numpy(), rtol=2e-3, atol=1e-7), (S_dev, S_ref)
    assert abs(loss_dev - loss_ref.item()) <= 2e-3 * abs(loss_ref.item()), (loss_dev, loss_ref.item())
    for l, ((wt, bt), (dw, db)) in enumerate(zip(params, grads)):
        gw = wt.grad.permute(0, 2, 3, 4, 1).reshape(dw.shape).numpy()
        gb = bt.grad.numpy()
        ew = np.linalg.norm(dw - gw) / max(np.linalg.norm(gw), 1e-30)
        eb = np.linalg.norm(db - gb) / max(np.linalg.norm(gb), 1e-30)
        assert ew <= 2e-2 and eb <= 2e-2, (l, ew, eb)


def test_site_stats_match_device(fg):
    """The numpy statistics of the training targets are the device's."""
    with W.WarmStartNet((8, 8, 8), batch=1, seed=5) as net:
        cond = np.array([[300.0, 0.0, 0.0, 0.001, -5.0]])
        S = net.forward(cond, [9])
        _, u = net.io()
    ref = W.site_stats(u.reshape(8, 8, 8, 3), [0.0, 0.0, 0.001])
    assert np.allclose(S[0], ref, rtol=1e-4, atol=1e-9), (S[0], ref)


def test_training_lowers_the_loss(fg):
    """Adam on fixed targets: the loss falls by at least 10x in 300 steps."""
    rng = np.random.default_rng(1)
    cond = np.array([[150.0 + 25 * i, 0.0, 0.0, 0.0, -5.0] for i in range(4)])
    target = np.array([[0.0, 0.14 * (i < 2), 0.1 * (i < 2), 0.03, 0.0003, 0.02, 0.005] for i in range(4)])
    wts = 1.0 / np.maximum(target.var(axis=0), 1e-6)
    with W.WarmStartNet((8, 8, 8), batch=4, seed=2) as net:
        hist = []
        for it in range(300):
            hist.append(net.backward(cond, rng.integers(1, 2 ** 40, size=4), target, wts))
            net.adam(3e-3)
    ratio = np.mean(hist[-10:]) / np.mean(hist[:3])
    assert ratio < 0.1, (ratio, hist[:3], hist[-10:])


def test_training_is_reproducible_bit_for_bit(fg):
    """The weight gradient of several site splits (16^3 x 2 samples: 4
    splits of 2048 sites) is summed in a fixed order, so two trainings from
    the same seeds end with the same weights bit for bit."""
    rng = np.random.default_rng(4)
    cond = np.array([[200.0, 0.0, 0.0, 0.0, -5.0], [350.0, 0.0, 0.0, 0.0005, -5.0]])
    target = np.array([[0.0, 0.14, 0.1, 0.03, 0.0003, 0.02, 0.005], [0.0, 0.0, 0.0, 0.02, 0.0002, 0.0, 0.0]])
    wts = np.ones(W.NSTAT)
    seeds = [rng.integers(1, 2 ** 40, size=2) for _ in range(3)]
    out = []
    for _ in range(2):
        with W.WarmStartNet((16, 16, 16), batch=2, seed=9) as net:
            for sd in seeds:
                net.backward(cond, sd, target, wts)
                net.adam(1e-3)
            out.append([net.layer(l)[0] for l in range(4)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
