"""Training the learned warm start of the simulation's projections on the
method's own data (include/incrmt_unet.h).

A capture run records, for every MAC and FEM projection, the network input
of the warm start (the restricted residual of the previous step's pressure
and the restricted reciprocal density) and the target (the restricted
difference between the converged pressure and that warm start). The U-Net is
then trained on these samples by its own GPU kernels (forward, backward,
Adam). Torch tensors only hold the device buffers and pick the batches.
"""
import torch

from . import capi


def capture(sim, factor, steps, dt, device, systems=(capi.SYS_MAC, capi.SYS_FEM)):
    """Runs `steps` steps of `sim` capturing one sample per projection of
    each system. Returns {sys: (X, T)} with X (steps, H, W, 3) network inputs
    and T (steps, H, W) raw targets."""
    out = {}
    for sys in systems:
        H, W = sim.learned_grid(sys, factor)
        X = torch.zeros(steps, H, W, 3, dtype=torch.float32, device=device)
        T = torch.zeros(steps, H, W, dtype=torch.float32, device=device)
        out[sys] = (X, T)
    torch.cuda.synchronize(device)
    for sys, (X, T) in out.items():
        sim.learned_capture(sys, factor, X.data_ptr(), T.data_ptr(), steps)
    sim.step(dt, steps)
    for sys in out:
        assert sim.learned_stats(sys).captured == steps
        sim.learned_capture(sys, factor, 0, 0, 0)
    return out


def normalise(X, T):
    """Targets scaled to zero mean and unit variance over each sample's image
    (the pixels with a nonzero density feature; the step length along the
    network's output is chosen at solve time, so only the shape matters).
    Samples with a zero target are dropped. Returns X, T, valid masks."""
    V = (X[..., 1] != 0).float()
    n = V.sum((1, 2)).clamp(min=1)
    mean = (T * V).sum((1, 2)) / n
    var = (((T - mean[:, None, None]) * V) ** 2).sum((1, 2)) / n
    keep = var > 0
    X, T, V, mean, var = X[keep], T[keep], V[keep], mean[keep], var[keep]
    T = (T - mean[:, None, None]) / var.sqrt()[:, None, None] * V
    return X.contiguous(), T.contiguous(), V.contiguous()


def train(net, X, T, V, steps, batch=8, lr=2e-3, lr_late=5e-4, seed=0):
    """Adam steps of the network on random batches of the samples; returns
    the last batch loss."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    S, H, W = T.shape
    loss = None
    for it in range(steps):
        idx = torch.randint(0, S, (batch,), generator=g)
        # keep the batch tensors alive while the kernels read them
        xb, tb, vb = X[idx].contiguous(), T[idx].contiguous(), V[idx].contiguous()
        loss = net.train_step(batch, H, W, xb.data_ptr(), tb.data_ptr(), vb.data_ptr(),
                              lr if it < 0.75 * steps else lr_late)
    return loss
