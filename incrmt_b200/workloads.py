"""Seeded synthetic inputs for the benchmark configurations.

No public dataset is involved: each configuration is an IncRMT scenario or a
solver problem synthesised from a seed, identically for the GPU path and for
the CPU reference.

standalone_mac_problem: the standalone variable-density MAC pressure solve on
[-1,1]^2 with walls. The density comes from 8 seeded non-overlapping circles
(radius 0.02-0.1 of the domain length, rho_s=3, rho_f=1), blended by the
reference's smoothed Heaviside at eps=2.5*dx (obj_field.hh:102-112) and
combined as fluid_2d::set_rho does (fluid_2d.cc:1124-1137). The right-hand
side is the discrete MAC divergence (fluid_2d.cc:1179-1187) of an edge
velocity field built from 64 seeded Gaussian blobs (radius 0.02-0.1 of the
domain length, independent N(0,1) amplitudes on u and v), with zero normal
velocity on the walls, minus its mean.
"""
import math

import numpy as np
import torch


def _trans_func(phi, eps):
    """Smoothed Heaviside of obj_field::trans_func (obj_field.hh:102-112)."""
    t = 0.5 - phi * (0.5 / eps) - (0.5 / math.pi) * torch.sin((math.pi / eps) * phi)
    t = torch.where(phi < -eps, torch.ones_like(phi), t)
    return torch.where(phi > eps, torch.zeros_like(phi), t)


def circles(seed, count=8, rmin=0.04, rmax=0.2, box=(-1.0, 1.0, -1.0, 1.0), margin=0.05):
    """Rejection-sampled non-overlapping circles (cx, cy, r) inside the box."""
    rng = np.random.default_rng(seed)
    ax, bx, ay, by = box
    out = []
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place circles")
        r = rng.uniform(rmin, rmax)
        cx = rng.uniform(ax + r + margin, bx - r - margin)
        cy = rng.uniform(ay + r + margin, by - r - margin)
        if all((cx - x) ** 2 + (cy - y) ** 2 > (r + q + margin) ** 2 for x, y, q in out):
            out.append((cx, cy, r))
    return out


def circle_density(m, n, circ, rhos=3.0, rhof=1.0, tw=2.5, box=(-1.0, 1.0, -1.0, 1.0),
                   device="cpu"):
    """Ghosted (n+4, m+4) density of solid circles in fluid."""
    ax, bx, ay, by = box
    dx, dy = (bx - ax) / m, (by - ay) / n
    eps = tw * min(dx, dy)
    x = ax + dx * (torch.arange(-2, m + 2, device=device, dtype=torch.float64) + 0.5)
    y = ay + dy * (torch.arange(-2, n + 2, device=device, dtype=torch.float64) + 0.5)
    Y, X = torch.meshgrid(y, x, indexing="ij")
    rho = torch.zeros_like(X)
    sfrac = torch.zeros_like(X)
    for cx, cy, r in circ:
        phi = torch.sqrt((X - cx) ** 2 + (Y - cy) ** 2) - r
        tf = _trans_func(phi, eps)
        sfrac += tf
        rho += tf * rhos
    return torch.where(sfrac >= 1, rho / sfrac, (1 - sfrac) * rhof + rho)


def blob_divergence(m, n, seed, count=64, rmin=0.04, rmax=0.2, box=(-1.0, 1.0, -1.0, 1.0),
                    device="cpu"):
    """MAC divergence (n, m) of a sum of Gaussian velocity blobs, walls closed."""
    ax, bx, ay, by = box
    dx, dy = (bx - ax) / m, (by - ay) / n
    rng = np.random.default_rng(seed + 7919)
    ul = torch.zeros((n, m + 1), device=device, dtype=torch.float64)  # u on x-edges
    vd = torch.zeros((n + 1, m), device=device, dtype=torch.float64)  # v on y-edges
    xe = ax + dx * torch.arange(0, m + 1, device=device, dtype=torch.float64)
    yc = ay + dy * (torch.arange(0, n, device=device, dtype=torch.float64) + 0.5)
    xc = ax + dx * (torch.arange(0, m, device=device, dtype=torch.float64) + 0.5)
    ye = ay + dy * torch.arange(0, n + 1, device=device, dtype=torch.float64)
    for _ in range(count):
        cx, cy = rng.uniform(ax, bx), rng.uniform(ay, by)
        r = rng.uniform(rmin, rmax)
        au, av = rng.standard_normal(), rng.standard_normal()
        # Each blob is evaluated on its 4r bounding box only.
        def rng_idx(c0, lo, h, size):
            a = max(0, int(math.floor((c0 - 4 * r - lo) / h)))
            b = min(size, int(math.ceil((c0 + 4 * r - lo) / h)) + 1)
            return a, b
        i0, i1 = rng_idx(cx, ax, dx, m + 1)
        j0, j1 = rng_idx(cy, ay - 0.5 * dy, dy, n)
        if i1 > i0 and j1 > j0:
            gx = torch.exp(-((xe[i0:i1] - cx) / r) ** 2)
            gy = torch.exp(-((yc[j0:j1] - cy) / r) ** 2)
            ul[j0:j1, i0:i1] += au * gy[:, None] * gx[None, :]
        i0, i1 = rng_idx(cx, ax - 0.5 * dx, dx, m)
        j0, j1 = rng_idx(cy, ay, dy, n + 1)
        if i1 > i0 and j1 > j0:
            gx = torch.exp(-((xc[i0:i1] - cx) / r) ** 2)
            gy = torch.exp(-((ye[j0:j1] - cy) / r) ** 2)
            vd[j0:j1, i0:i1] += av * gy[:, None] * gx[None, :]
    ul[:, 0] = 0
    ul[:, m] = 0
    vd[0, :] = 0
    vd[n, :] = 0
    src = (1.0 / dx) * (ul[:, 1:] - ul[:, :-1]) + (1.0 / dy) * (vd[1:, :] - vd[:-1, :])
    return src - src.mean()


def standalone_mac_problem(m, n=None, seed=3, device="cpu"):
    """(rho (n+4,m+4), b (n,m)) for the standalone MAC solve, as float64 tensors."""
    n = m if n is None else n
    circ = circles(seed)
    rho = circle_density(m, n, circ, device=device)
    b = blob_divergence(m, n, seed, device=device)
    return rho, b


def standalone_fem_problem(m, n=None, seed=5, device="cpu"):
    """(rho (n+4,m+4), b (n+1,m+1)) for a standalone FEM solve: the same
    density model and a seeded smooth nodal right-hand side with zero mean."""
    n = m if n is None else n
    circ = circles(seed)
    rho = circle_density(m, n, circ, device=device)
    src = blob_divergence(m + 1, n + 1, seed, device=device)
    return rho, src


def sediment_bodies(seed=11, count=32, box=(-0.75, 0.75, -1.5, 1.5), rmin=0.03, rmax=0.06,
                    rho_min=1.5, rho_max=3.0, gap=0.02):
    """Seeded solids for the sediment configuration: `count` bodies in the
    walled box of the reference's sediment driver (sediment.cc:22,124),
    alternately circles and ellipses, sizes rmin-rmax, densities
    rho_min-rho_max, each falling with gravity (rho_s-1)/rho_s
    (sediment.cc:98). Placement is rejection-sampled so that bounding circles
    keep `gap` from each other and from the walls (as sediment.cc:91-121
    rejects overlaps). Returns a list of dicts: kind ('circle'|'ellipse'),
    cx, cy, r (circle radius / ellipse major semi-axis), b (minor semi-axis),
    theta, rhos, grav."""
    rng = np.random.default_rng(seed)
    ax, bx, ay, by = box
    out = []
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > 1000000:
            raise RuntimeError("could not place the bodies")
        r = rng.uniform(rmin, rmax)
        x = rng.uniform(ax + r + gap, bx - r - gap)
        y = rng.uniform(ay + r + gap, by - r - gap)
        if any(math.hypot(x - o["cx"], y - o["cy"]) <= r + o["r"] + gap for o in out):
            continue
        rhos = rng.uniform(rho_min, rho_max)
        kind = "circle" if len(out) % 2 == 0 else "ellipse"
        bsemi = r if kind == "circle" else r * rng.uniform(0.5, 0.8)
        theta = 0.0 if kind == "circle" else rng.uniform(0, math.pi)
        out.append(dict(kind=kind, cx=x, cy=y, r=r, b=bsemi, theta=theta, rhos=rhos,
                        grav=(rhos - 1) / rhos))
    return out
