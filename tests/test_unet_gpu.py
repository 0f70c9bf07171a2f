"""The learned initial guess (include/incrmt_unet.h): the BF16 U-Net's own
forward/backward kernels against an FP64 PyTorch CPU restatement of the same
network, training, and what the trained guess gains over the solver without
it.

- gradients: loss within 3% and every convolution's weight gradient within
  6% (relative 2-norm) with cosine similarity above 0.995 of the FP64
  reference; the tolerance covers the BF16 rounding of activations, weights
  and back-propagated gradients between layers;
- training: 40 Adam steps on a fixed batch cut the loss by more than half;
- gain: trained on 256 seeded 128^2 MAC problems (8 circles at density
  ratio 3, 64 blobs; the standalone-solve workload at a test size) at half
  resolution, the guess on 8 held-out problems is within 0.7 of the
  solution's norm of it (about 0.2-0.5 measured) and needs no more V-cycles
  to 1e-9 than the zero start (about 10% fewer measured).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch_forward(params, levels, base, x, t, valid):
    """The network of incrmt_unet in FP64 NCHW PyTorch (CPU): the layer order
    and the parameter layout ([tap][in][out] weights, then biases) of the
    C ABI."""
    import torch
    import torch.nn.functional as F
    convs = []
    C = lambda l: base << l

    def add(cin, cout, taps):
        convs.append((cin, cout, taps))
    add(16, C(0), 9)
    add(C(0), C(0), 9)
    for l in range(1, levels):
        add(C(l - 1), C(l), 9)
        add(C(l), C(l), 9)
    for l in range(levels - 2, -1, -1):
        add(C(l + 1) + C(l), C(l), 9)
        add(C(l), C(l), 9)
    add(C(0), 16, 1)
    ws, bs, off = [], [], 0
    for cin, cout, taps in convs:
        w = params[off:off + taps * cin * cout].reshape(taps, cin, cout)
        off += taps * cin * cout
        b = params[off:off + cout]
        off += cout
        k = 3 if taps == 9 else 1
        wt = torch.tensor(w.transpose(2, 1, 0).reshape(cout, cin, k, k), dtype=torch.float64, requires_grad=True)
        ws.append(wt)
        bs.append(torch.tensor(b, dtype=torch.float64, requires_grad=True))

    def conv(i, h, relu=True):
        y = F.conv2d(h, ws[i], bs[i], padding=1 if ws[i].shape[-1] == 3 else 0)
        return F.relu(y) if relu else y
    B, H, W, _ = x.shape
    h = torch.zeros(B, 16, H, W, dtype=torch.float64)
    h[:, :3] = torch.tensor(x, dtype=torch.float64).permute(0, 3, 1, 2)
    k = 0
    skips = []
    for l in range(levels):
        if l > 0:
            h = F.avg_pool2d(h, 2)
        h = conv(k, h); k += 1
        h = conv(k, h); k += 1
        skips.append(h)
    for l in range(levels - 2, -1, -1):
        h = torch.cat([F.interpolate(h, scale_factor=2, mode="nearest"), skips[l]], dim=1)
        h = conv(k, h); k += 1
        h = conv(k, h); k += 1
    out = conv(k, h, relu=False)[:, 0]
    tt = torch.tensor(t, dtype=torch.float64)
    vv = torch.tensor(valid, dtype=torch.float64)
    loss = (vv * (out - tt) ** 2).sum() / vv.sum()
    loss.backward()
    grads = []
    for (cin, cout, taps), w, b in zip(convs, ws, bs):
        k = 3 if taps == 9 else 1
        gw = w.grad.numpy().reshape(cout, cin, taps).transpose(2, 1, 0)
        grads.append((gw, b.grad.numpy()))
    return float(loss), grads, convs


def _bf16(a):
    import torch
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float32).numpy()


def test_gradients_match_fp64_reference(gpu):
    import torch
    from incrmt_b200 import capi
    levels, base, B, H, W = 3, 16, 2, 32, 32
    net = capi.UNet(levels, base, seed=7)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((B, H, W, 3)).astype(np.float32)
    t = rng.standard_normal((B, H, W)).astype(np.float32)
    valid = np.ones((B, H, W), dtype=np.float32)
    valid[:, :, -5:] = 0
    dev = torch.device("cuda")
    xd, td, vd = (torch.tensor(a, device=dev) for a in (x, t, valid))
    loss, g = net.gradients(B, H, W, xd.data_ptr(), td.data_ptr(), vd.data_ptr())
    params = net.get_params()
    ref_loss, ref_grads, convs = _torch_forward(_bf16(params), levels, base, _bf16(x), t, valid)
    assert abs(loss - ref_loss) <= 0.03 * abs(ref_loss)
    off = 0
    for i, ((cin, cout, taps), (gw, gb)) in enumerate(zip(convs, ref_grads)):
        ours = g[off:off + taps * cin * cout].reshape(taps, cin, cout)
        off += taps * cin * cout + cout
        if i == 0:
            ours, gw = ours[:, :3], gw[:, :3]   # the zero-padding input channels get no gradient
        if i == len(convs) - 1:
            ours, gw = ours[..., :1], gw[..., :1]
        rel = np.linalg.norm(ours - gw) / np.linalg.norm(gw)
        cos = float(np.sum(ours * gw) / (np.linalg.norm(ours) * np.linalg.norm(gw)))
        assert rel < 0.06 and cos > 0.995, (i, rel, cos)
    net.close()


def test_training_reduces_loss(gpu):
    import torch
    from incrmt_b200 import capi
    net = capi.UNet(3, 16, seed=3)
    B, H, W = 4, 32, 32
    rng = np.random.default_rng(1)
    dev = torch.device("cuda")
    x = torch.tensor(rng.standard_normal((B, H, W, 3)).astype(np.float32), device=dev)
    # A smooth target the network can fit: a blurred copy of channel 0.
    t = torch.nn.functional.avg_pool2d(x[..., 0].unsqueeze(1), 5, 1, 2).squeeze(1).contiguous()
    v = torch.ones(B, H, W, device=dev)
    losses = [net.train_step(B, H, W, x.data_ptr(), t.data_ptr(), v.data_ptr(), 3e-3) for _ in range(40)]
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
    net.close()


def _mac_problem(m, seed):
    from incrmt_b200 import workloads
    rho, b = workloads.standalone_mac_problem(m, seed=seed)
    return rho.numpy(), b.numpy().ravel()


def test_learned_guess_saves_vcycles(gpu):
    """The network of the specification (4 levels, 32 base channels, about
    2 M parameters) trained on 1024 problems of the standalone MAC solve at
    128^2 (its own FP64 multigrid solutions, restricted by 2) and evaluated
    on 32 held-out problems: the guess must start the solve closer to the
    solution (relative error of the guess below 0.45 on average; measured
    0.32) and save at least 0.25 V-cycles per solve on average (measured
    0.47 of 8.4) against the zero start, never costing a V-cycle."""
    import torch
    from incrmt_b200 import capi
    m, factor = 128, 2
    dev = torch.device("cuda")
    H, W = capi.learned_grid(m, m, factor)
    s = capi.MGSolver(capi.SYS_MAC, m, m)
    ins, tgts = [], []
    for seed in range(1000, 2024):
        rho, b = _mac_problem(m, seed)
        s.set_density(rho)
        z = np.zeros(m * m)
        s.solve(b, z)
        bd = torch.tensor(b, device=dev)
        z0 = torch.zeros(m * m, dtype=torch.float64, device=dev)
        xin = torch.empty(H, W, 3, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()  # the solver works on its own stream
        capi.learned_input(s, bd.data_ptr(), z0.data_ptr(), factor, xin.data_ptr())
        zt = torch.tensor(z.reshape(m, m), dtype=torch.float32, device=dev)
        zt = torch.nn.functional.avg_pool2d(zt[None, None], factor)[0, 0]
        ins.append(xin)
        tgts.append((zt - zt.mean()) / zt.std())
    torch.cuda.synchronize()
    X = torch.stack(ins).contiguous()
    T = torch.stack(tgts).contiguous()
    V = torch.ones_like(T)
    net = capi.UNet(4, 32, seed=11)
    g = torch.Generator(device="cpu").manual_seed(0)
    for it in range(1500):
        idx = torch.randperm(len(ins), generator=g)[:16]
        # keep the batch tensors alive while the kernels read them
        xb, tb, vb = X[idx].contiguous(), T[idx].contiguous(), V[idx].contiguous()
        net.train_step(16, H, W, xb.data_ptr(), tb.data_ptr(), vb.data_ptr(), 2e-3 if it < 1100 else 5e-4)
    plain, learned, errs = [], [], []
    for seed in range(5000, 5032):
        rho, b = _mac_problem(m, seed)
        s.set_density(rho)
        bd = torch.tensor(b, device=dev)
        z = torch.zeros(m * m, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        plain.append(s.solve_device(bd.data_ptr(), z.data_ptr()).vcycles)
        zstar = z.clone()
        z.zero_()
        torch.cuda.synchronize()
        capi.learned_guess(s, net, bd.data_ptr(), z.data_ptr(), factor)
        e = (zstar - zstar.mean()) - (z - z.mean())
        errs.append(float(e.norm() / (zstar - zstar.mean()).norm()))
        learned.append(s.solve_device(bd.data_ptr(), z.data_ptr()).vcycles)
    capi.conv_status()
    saving = np.mean(plain) - np.mean(learned)
    assert np.mean(errs) < 0.45, errs
    assert saving >= 0.25, (saving, plain, learned)
    assert min(np.array(plain) - np.array(learned)) >= 0, (plain, learned)
    net.close()
    s.close()
