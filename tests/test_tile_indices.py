"""Index safety of the multigrid's shared-memory tile kernels, replayed on
the CPU (no GPU needed).

k_galerkin_tile and k_restrict_tile (incrmt_b200/csrc/mg.cu) stage a fixed
region of fine unknowns around each 32 x 8 tile of coarse unknowns, and wrap
a periodic index only once (wrap_idx). This test replays their staging
loops' index arithmetic, and the reads of their sums, over every level of
the hierarchies that build_hierarchy makes for the tested grids and the
benchmark's flag. On each level it checks that:
  - every staged point that is read from global memory lies inside the grid
    (a level smaller than the tile must not reach a second period);
  - every point the sums read was staged.
The replay mirrors the kernels' constants and formulas; it has to follow
any change to their staging.
"""
import pytest

CTW, CTH = 32, 8
K_SEMI_RATIO, K_COARSEST, K_MAX_LEVELS = 2.0, 16, 24


def wrap(i, m, p):
    """wrap_idx: one period at most."""
    if i < 0:
        return (i + m, True) if p else (i, False)
    if i >= m:
        return (i - m, True) if p else (i, False)
    return i, True


def can_coarsen(m, p):
    return (m % 2 == 0 and m // 2 >= 4) if p else m >= 5


def hierarchy(fm, fn, px, py, ratio):
    """The (fine m, fine n, coarse m, coarse n, kx, ky) steps of
    Multigrid::build_hierarchy."""
    out, mm, nn, r = [], fm, fn, ratio
    while len(out) + 1 < K_MAX_LEVELS and mm * nn > K_COARSEST:
        kx, ky = can_coarsen(mm, px), can_coarsen(nn, py)
        if kx and ky:
            if r > K_SEMI_RATIO:
                kx = False
            elif r < 1 / K_SEMI_RATIO:
                ky = False
        if not kx and not ky:
            break
        if kx and not ky:
            r *= 4
        elif ky and not kx:
            r /= 4
        mc = (mm // 2 if px else (mm + 1) // 2) if kx else mm
        nc = (nn // 2 if py else (nn + 1) // 2) if ky else nn
        out.append((mm, nn, mc, nc, kx, ky))
        mm, nn = mc, nc
    return out


def support(I, J, kx, ky):
    x0 = 2 * I - 1 if kx else I
    y0 = 2 * J - 1 if ky else J
    for v in range(3 if ky else 1):
        for u in range(3 if kx else 1):
            yield x0 + u, y0 + v


def replay_galerkin(fm, fn, cm, cn, kx, ky, px, py):
    sw = 2 * CTW + 1 if kx else CTW
    sh = 2 * CTH + 1 if ky else CTH
    nw, nh = sw + 2, sh + 2
    sxmax = 2 * cm - 1 if kx else cm - 1
    symax = 2 * cn - 1 if ky else cn - 1
    outside = missing = 0
    for bx in range((cm + CTW - 1) // CTW):
        for by in range((cn + CTH - 1) // CTH):
            x0, y0 = bx * CTW, by * CTH
            sx0 = 2 * x0 - 1 if kx else x0
            sy0 = 2 * y0 - 1 if ky else y0
            staged_p, staged_a = set(), set()
            for t in range(nw * nh):                       # weights: region grown by one
                xu, yu = sx0 - 1 + t % nw, sy0 - 1 + t // nw
                if xu > sxmax + 1 or yu > symax + 1:
                    continue
                (i, okx), (j, oky) = wrap(xu, fm, px), wrap(yu, fn, py)
                if okx and oky:
                    outside += not (0 <= i < fm and 0 <= j < fn)
                    staged_p.add((xu, yu))
            for t in range(sw * sh):                       # stencils of the supports
                xu, yu = sx0 + t % sw, sy0 + t // sw
                if xu > sxmax or yu > symax:
                    continue
                (i, okx), (j, oky) = wrap(xu, fm, px), wrap(yu, fn, py)
                if okx and oky:
                    outside += not (0 <= i < fm and 0 <= j < fn)
                    staged_a.add((xu, yu))
            for I in range(x0, min(x0 + CTW, cm)):
                for J in range(y0, min(y0 + CTH, cn)):
                    for fi, fj in support(I, J, kx, ky):
                        if not (wrap(fi, fm, px)[1] and wrap(fj, fn, py)[1]):
                            continue                       # weight zero outside the grid
                        missing += (fi, fj) not in staged_a
                        for dj in (-1, 0, 1):
                            for di in (-1, 0, 1):
                                g = (fi + di, fj + dj)
                                if wrap(g[0], fm, px)[1] and wrap(g[1], fn, py)[1]:
                                    missing += g not in staged_p
    return outside, missing


def replay_restrict(fm, fn, cm, cn, kx, ky, px, py):
    fw = 2 * CTW + 1 if kx else CTW
    fh = 2 * CTH + 1 if ky else CTH
    fxmax = 2 * cm - 1 if kx else cm - 1
    fymax = 2 * cn - 1 if ky else cn - 1
    outside = missing = 0
    for bx in range((cm + CTW - 1) // CTW):
        for by in range((cn + CTH - 1) // CTH):
            x0, y0 = bx * CTW, by * CTH
            fx0 = 2 * x0 - 1 if kx else x0
            fy0 = 2 * y0 - 1 if ky else y0
            staged = set()
            for t in range(fw * fh):
                xu, yu = fx0 + t % fw, fy0 + t // fw
                if xu > fxmax or yu > fymax:
                    continue
                (i, okx), (j, oky) = wrap(xu, fm, px), wrap(yu, fn, py)
                if okx and oky:
                    outside += not (0 <= i < fm and 0 <= j < fn)
                    staged.add((xu, yu))
            for I in range(x0, min(x0 + CTW, cm)):
                for J in range(y0, min(y0 + CTH, cn)):
                    for fi, fj in support(I, J, kx, ky):
                        if wrap(fi, fm, px)[1] and wrap(fj, fn, py)[1]:
                            missing += (fi, fj) not in staged
    return outside, missing


def _grids():
    # (name, system, cells m x n, x periodic, y periodic, domain width / height)
    cells = [("mac 1024 walls", 0, 1024, 1024, 0, 0, 1.0), ("fem 1024 walls", 1, 1024, 1024, 0, 0, 1.0),
             ("mac 768x512 y-prd", 0, 768, 512, 0, 1, 1.0), ("fem 768x512 y-prd", 1, 768, 512, 0, 1, 1.0),
             ("mac 512x384 prd", 0, 512, 384, 1, 1, 1.0), ("fem 1024x768 prd", 1, 1024, 768, 1, 1, 1.0),
             ("mac 1024x768 prd", 0, 1024, 768, 1, 1, 1.0), ("fem 64 prd", 1, 64, 64, 1, 1, 1.0),
             ("mac 128 prd", 0, 128, 128, 1, 1, 1.0), ("fem 256 walls", 1, 256, 256, 0, 0, 1.0),
             ("flag mac 2048", 0, 2048, 2048, 0, 1, 3.0), ("flag fem 2048", 1, 2048, 2048, 0, 1, 3.0),
             ("flag fem 384x128", 1, 384, 128, 0, 1, 1.0)]
    for name, sys_, m, n, px, py, aspect in cells:
        fm = m if (sys_ == 0 or px) else m + 1
        fn = n if (sys_ == 0 or py) else n + 1
        dx, dy = 2.0 * aspect / m, 2.0 / n
        yield pytest.param(fm, fn, px, py, (dx / dy) ** 2, id=name)


@pytest.mark.parametrize("fm,fn,px,py,ratio", list(_grids()))
def test_tile_staging_stays_in_grid(fm, fn, px, py, ratio):
    for (mm, nn, mc, nc, kx, ky) in hierarchy(fm, fn, px, py, ratio):
        if mm > 64 and nn > 16:
            # one period past the grid can only be reached from within 62
            # columns and 14 rows of it: such levels need no replay
            continue
        for replay in (replay_galerkin, replay_restrict):
            outside, missing = replay(mm, nn, mc, nc, kx, ky, px, py)
            assert outside == 0, (replay.__name__, mm, nn, mc, nc, kx, ky)
            assert missing == 0, (replay.__name__, mm, nn, mc, nc, kx, ky)


def test_replay_detects_unclipped_staging():
    """The replay finds the out-of-grid reads of the unclipped region on a
    small periodic level (the kernel before its region was clipped)."""
    fm, fn, cm, cn = 8, 6, 4, 6
    outside = 0
    for t in range((2 * CTW + 3) * (CTH + 2)):
        xu, yu = -2 + t % (2 * CTW + 3), -1 + t // (2 * CTW + 3)
        (i, okx), (j, oky) = wrap(xu, fm, 1), wrap(yu, fn, 1)
        if okx and oky:
            outside += not (0 <= i < fm and 0 <= j < fn)
    assert outside > 0
    assert replay_galerkin(fm, fn, cm, cn, True, False, 1, 1) == (0, 0)
