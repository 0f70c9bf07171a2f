"""numpy restatement of IncRMT's two variable-density pressure operators.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). An independent way to
compute residuals b - A z of solutions produced on the GPU, restated from:
  - MAC: mgs_mac_varying_rho (mgs_mac.hh:64-102, mgs_mac.cc:49-54) with edge
    reciprocal densities from fluid_2d::set_edge_irho (fluid_2d.cc:1140-1160);
  - FEM: mgs_fem_varying_rho (mgs_fem.hh:86-136, mgs_fem.cc:12-21,126-162)
    with cell reciprocal densities from fluid_2d::set_corner_irho
    (fluid_2d.cc:1163-1170).
Only non-periodic grids are restated here (the configurations in use).
rho is the (n+4, m+4) ghosted cell-density array.
"""
import numpy as np


def mac_apply(rho, z, dx, dy, zpr=False):
    """A z for the MAC system; z is (n, m)."""
    n, m = z.shape
    ir = 1.0 / rho
    c = ir[2:n + 2, 2:m + 2]
    ex = 0.5 * ir[2:n + 2, 2:m + 3] + 0.5 * ir[2:n + 2, 1:m + 2]  # x-edges 0..m
    ey = 0.5 * ir[2:n + 3, 2:m + 2] + 0.5 * ir[1:n + 2, 2:m + 2]  # y-edges 0..n
    del c
    xx, yy = 1.0 / dx ** 2, 1.0 / dy ** 2
    el, er = ex[:, :m].copy(), ex[:, 1:].copy()
    ed, eu = ey[:n, :].copy(), ey[1:, :].copy()
    el[:, 0] = 0
    er_off = er.copy()
    er_off[:, m - 1] = 0
    ed[0, :] = 0
    eu[n - 1, :] = 0
    out = np.zeros_like(z)
    out[:, 1:] += xx * el[:, 1:] * z[:, :-1]
    out[:, :-1] += xx * er_off[:, :-1] * z[:, 1:]
    out[1:, :] += yy * ed[1:, :] * z[:-1, :]
    out[:-1, :] += yy * eu[:-1, :] * z[1:, :]
    er_diag = er_off.copy()
    if zpr:
        er_diag[:, m - 1] = 2 * er[:, m - 1]
    diag = -xx * (el + er_diag) - yy * (ed + eu)
    return out + diag * z


def fem_apply(rho, z, dx, dy, zpr=False):
    """A z for the FEM system; z is (n+1, m+1) corner nodes."""
    nf, mf = z.shape
    n, m = nf - 1, mf - 1
    cell = 1.0 / rho[1:n + 3, 1:m + 3]  # cell (i-1,j-1) for node (i,j), padded
    dydx, dxdy = dy / dx, dx / dy
    fm = 1.0 / 3.0 * (dxdy + dydx)
    hey = 0.5 * (1.0 / 3.0 * (-2 * dxdy + dydx))
    hex_ = 0.5 * (1.0 / 3.0 * (-2 * dydx + dxdy))
    fc = -1.0 / 6.0 * (dxdy + dydx)
    # Element (cell) contributions: each interior cell (ci,cj) couples its four
    # corner nodes with the bilinear-element stiffness scaled by 1/rho.
    cint = cell[1:n + 1, 1:m + 1]  # cells 0..n-1, 0..m-1 -> node (i,j) is its lower-left
    out = np.zeros_like(z)
    # local node order: 0=(i,j),1=(i+1,j),2=(i,j+1),3=(i+1,j+1).
    # Element matrix entries that reproduce the assembled stencil:
    # diagonal fm per element, edge neighbours hex (x) / hey (y), diagonal fc.
    zl = {0: z[:-1, :-1], 1: z[:-1, 1:], 2: z[1:, :-1], 3: z[1:, 1:]}
    E = {(0, 0): fm, (0, 1): hex_, (0, 2): hey, (0, 3): fc,
         (1, 1): fm, (1, 0): hex_, (1, 3): hey, (1, 2): fc,
         (2, 2): fm, (2, 3): hex_, (2, 0): hey, (2, 1): fc,
         (3, 3): fm, (3, 2): hex_, (3, 1): hey, (3, 0): fc}
    sl = {0: (slice(0, -1), slice(0, -1)), 1: (slice(0, -1), slice(1, None)),
          2: (slice(1, None), slice(0, -1)), 3: (slice(1, None), slice(1, None))}
    for (a, b), v in E.items():
        out[sl[a]] += cint * v * zl[b]
    if zpr:
        # Fixed right column: off-diagonal entries vanish (mgs_fem.hh:115-128).
        diag = np.zeros_like(z)
        for a in range(4):
            diag[sl[a]] += cint * fm
        out[:, m] = diag[:, m] * z[:, m]
    return out
