"""Seeded synthetic workloads of the benchmark (inputs only).

`perturbed_sphere` builds the precision-form geometry: a sphere of radius R
whose radius is modulated by real spherical harmonics of degree l <= lmax
with coefficients ~ N(0, rel_sigma * R) drawn from a fixed seed;
phi = (|x| - r(theta, varphi)) / gridDelta is kept where |phi| <= 1 (a
width-2 band) and the undefined runs take the sign of phi.  The field is
evaluated with torch on `device` (the GPU for the full-size case).
"""
import math

import numpy as np

from ._abi import BoundaryConditionEnum as BC
from .domain import Domain, Grid, lex_order, make_runs


def sh_coefficients(lmax, sigma, seed):
    rng = np.random.default_rng(seed)
    return [(l, m, float(rng.normal(0.0, sigma))) for l in range(lmax + 1)
            for m in range(-l, l + 1)]


def _radius_torch(torch, coeffs, ct, st, phi, radius):
    """r(theta, phi) = R + sum c_lm Y_lm (real, orthonormal)."""
    lmax = max(l for l, _, _ in coeffs)
    # associated Legendre P_l^m(cos t) without Condon-Shortley phase
    P = {}
    P[(0, 0)] = torch.ones_like(ct)
    for m in range(1, lmax + 1):
        P[(m, m)] = P[(m - 1, m - 1)] * (2 * m - 1) * st
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * ct * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * ct * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    r = torch.full_like(ct, radius)
    for l, m, c in coeffs:
        am = abs(m)
        norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
        if m == 0:
            y = norm * P[(l, 0)]
        elif m > 0:
            y = math.sqrt(2.0) * norm * P[(l, am)] * torch.cos(am * phi)
        else:
            y = math.sqrt(2.0) * norm * P[(l, am)] * torch.sin(am * phi)
        r = r + c * y
    return r


def perturbed_sphere(radius=40.0, grid_delta=0.05, lmax=8, rel_sigma=0.02, seed=1234,
                     device="cpu"):
    import torch

    grid = Grid(None, [BC.INFINITE_BOUNDARY] * 3, grid_delta)
    coeffs = sh_coefficients(lmax, rel_sigma * radius, seed)
    gd = grid_delta
    dev = torch.device(device)
    # range of r(theta, phi) from a fine angular sample
    th = torch.linspace(0, math.pi, 721, device=dev, dtype=torch.float64)
    pp = torch.linspace(-math.pi, math.pi, 1441, device=dev, dtype=torch.float64)
    T_, P_ = torch.meshgrid(th, pp, indexing="ij")
    rs_ = _radius_torch(torch, coeffs, torch.cos(T_).reshape(-1), torch.sin(T_).reshape(-1),
                        P_.reshape(-1), radius)
    span = float(rs_.max() - rs_.min())
    rmin = max(0.0, (float(rs_.min()) - 0.05 * span) / gd - 3.0)
    rmax = (float(rs_.max()) + 0.05 * span) / gd + 3.0
    n = int(math.ceil(rmax))

    def raw(x, y, z):
        """|x| - r(theta, phi) in physical units; x, y, z in index units."""
        rho = torch.sqrt(x * x + y * y + z * z)
        safe = torch.where(rho > 0, rho, torch.ones_like(rho))
        ct = z / safe
        st = torch.sqrt(torch.clamp(1 - ct * ct, min=0.0))
        ph = torch.atan2(y, x)
        return rho * gd - _radius_torch(torch, coeffs, ct, st, ph, radius)

    def phi_at(x, y, z):
        # first-order distance: (|x| - r) / |grad(|x| - r)|, in grid units
        f = raw(x, y, z)
        h = 1e-3
        g2 = torch.zeros_like(f)
        for d in range(3):
            o = [0.0, 0.0, 0.0]
            o[d] = h
            fp = raw(x + o[0], y + o[1], z + o[2])
            fm = raw(x - o[0], y - o[1], z - o[2])
            g2 = g2 + ((fp - fm) / (2 * h * gd)) ** 2
        return f / torch.sqrt(g2) / gd

    # 1. bricks of 8^3 cells whose centre lies near the surface
    B = 8
    nbk = (2 * n + 1) // B + 2
    base = -(nbk * B) // 2
    bax = torch.arange(nbk, device=dev, dtype=torch.float64)
    keep_b = []
    reach = 4.0 * math.sqrt(3.0) * 2.0 + 2.0  # half diagonal x Lipschitz bound + margin
    for bz in range(nbk):
        cz = base + bz * B + 3.5
        BY, BX = torch.meshgrid(bax, bax, indexing="ij")
        cx = base + BX.reshape(-1) * B + 3.5
        cy = base + BY.reshape(-1) * B + 3.5
        rr = torch.sqrt(cx * cx + cy * cy + cz * cz)
        near = (rr >= rmin - 8) & (rr <= rmax + 8)
        if not bool(near.any()):
            continue
        cx, cy = cx[near], cy[near]
        czt = torch.full_like(cx, cz)
        f = raw(cx, cy, czt) / gd
        sel = torch.abs(f) <= reach
        keep_b.append(torch.stack([cx[sel], cy[sel], czt[sel]], 1) - 3.5)
    bricks = torch.cat(keep_b)
    off = torch.arange(B, device=dev, dtype=torch.float64)
    OZ, OY, OX = torch.meshgrid(off, off, off, indexing="ij")
    offs = torch.stack([OX.reshape(-1), OY.reshape(-1), OZ.reshape(-1)], 1)
    # 2. cells of those bricks, evaluated in chunks
    idx_parts, val_parts = [], []
    per = max(1, (1 << 23) // (B ** 3))
    for s0 in range(0, len(bricks), per):
        cells = (bricks[s0:s0 + per, None, :] + offs[None, :, :]).reshape(-1, 3)
        v = phi_at(cells[:, 0], cells[:, 1], cells[:, 2])
        keep = torch.abs(v) <= 1.0
        idx_parts.append(cells[keep].to(torch.int32).cpu().numpy())
        val_parts.append(v[keep].cpu().numpy())
    idx = np.concatenate(idx_parts)
    vals = np.concatenate(val_parts)

    def sign_fn(x, y, z):
        out = np.empty(len(x), np.int64)
        step = 1 << 22
        for s in range(0, len(x), step):
            t = [torch.as_tensor(np.asarray(a[s:s + step], np.float64), device=dev) for a in (x, y, z)]
            out[s:s + step] = np.where(phi_at(*t).cpu().numpy() < 0, -1, 1)
        return out

    rs, sg = make_runs(idx, sign_fn, [-n - 1] * 3, [n + 1] * 3)
    return grid, Domain(grid, idx, vals, rs, sg, width=2)


def precision_velocity():
    """v = 1.0 + 0.3 n_z on the single material."""
    from .velocity import FunctorVelocity

    v = FunctorVelocity(1)
    v.set_rate(0, 1.0)
    v.set_linear(0, 2, 0.3)
    return v


def batch_domains(n=256, seed=7, points_range=(1e4, 2e6), device=None):
    """Inputs of the batching form: n independent planes, each with a random
    trench or cylindrical hole (width 0.5-4.0, depth 1-8), periodic in x/y,
    gridDelta 0.05-0.2 chosen so the band sizes spread log-uniformly over
    `points_range`, and a constant etch rate in [0.2, 1.5].  Returns a list
    of (grid, domain, velocity)."""
    import numpy as np

    from .geometry import sdf_box, sdf_levelset
    from .velocity import constant_scalar

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        hole = bool(rng.integers(2))
        width = float(rng.uniform(0.5, 4.0))
        depth = float(rng.uniform(1.0, 8.0))
        rate = float(rng.uniform(0.2, 1.5))
        target = float(np.exp(rng.uniform(np.log(points_range[0]), np.log(points_range[1]))))
        gd = float(np.exp(rng.uniform(np.log(0.05), np.log(0.2))))
        # a width-2 band holds ~2.5 points per cell of surface: the plane
        # (lateral^2) plus the walls (a trench's two walls along y, a hole's
        # cylinder); the lateral extent is chosen for the target band and kept
        # at least twice the feature (then gridDelta is made finer or coarser
        # within 0.05..0.2 to approach the target)
        area = target * gd * gd / 2.5
        if hole:
            lateral = math.sqrt(max(area - math.pi * width * depth, 0.0))
        else:
            lateral = -depth + math.sqrt(depth * depth + area)
        lmin = max(2.0 * width, width + 2.0)
        if lateral < lmin:
            lateral = lmin
            surf = lateral * lateral + (math.pi * width * depth if hole else 2.0 * lateral * depth)
            gd = float(np.clip(math.sqrt(2.5 * surf / target), 0.05, 0.2))
        # periodic extents in whole bricks (multiples of 8 points), which the
        # batching form's shared brick box needs
        cells = max(16, 8 * int(round(lateral / gd / 8.0)))
        c2 = cells // 2
        zlo, zhi = -depth - 1.5, 1.5
        grid = Grid(None, [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], gd,
                    index_min=[-c2, -c2, math.floor(zlo / gd)],
                    index_max=[c2, c2, math.ceil(zhi / gd)])
        r = width / 2.0
        lo = [grid.min[0], grid.min[1], grid.min[2]]
        hi = [grid.max[0] - 1, grid.max[1] - 1, grid.max[2]]
        if device is None:
            def sdf(x, y, z, hole=hole, r=r, depth=depth):
                if hole:
                    cut = np.maximum(np.sqrt(x * x + y * y) - r, -z - depth)
                else:
                    cut = sdf_box((x, y, z), (-r, -1e9, -depth), (r, 1e9, 1e9))
                return np.maximum(z, -cut)

            dom = sdf_levelset(grid, sdf, lo, hi)
        else:
            dom = _torch_domain(grid, _hole_or_trench_torch(hole, r, depth), lo, hi, device)
        out.append((grid, dom, constant_scalar(-rate)))
    return out


def _hole_or_trench_torch(hole, r, depth):
    """The batching form's plane with a cylindrical hole or a trench (along y)
    as a torch SDF."""
    import torch

    def sdf(x, y, z):
        if hole:
            cut = torch.maximum(torch.sqrt(x * x + y * y) - r, -z - depth)
        else:
            # box |x| <= r, z >= -depth (unbounded in y and upwards)
            qx = torch.abs(x) - r
            qz = -depth - z
            outside = torch.sqrt(torch.clamp(qx, min=0.0) ** 2 + torch.clamp(qz, min=0.0) ** 2)
            cut = outside + torch.clamp(torch.maximum(qx, qz), max=0.0)
        return torch.maximum(z, -cut)

    return sdf


def _torch_domain(grid, sdf, lo, hi, device):
    """Width-2 band and undefined runs of a torch SDF on `device`."""
    import torch

    idx, vals = _sdf_band_torch(grid, sdf, lo, hi, device)
    gd = grid.delta

    def sign_fn(x, y, z):
        out = np.empty(len(x), np.int64)
        step = 1 << 22
        for s in range(0, len(x), step):
            t = [torch.as_tensor(np.asarray(a[s:s + step], np.float64) * gd, device=device)
                 for a in (x, y, z)]
            out[s:s + step] = np.where(sdf(*t).cpu().numpy() < 0, -1, 1)
        return out

    rs, sg = make_runs(idx, sign_fn, [lo[0] - 1, lo[1] - 1, lo[2] - 1],
                       [hi[0] + 1, hi[1] + 1, hi[2] + 1])
    return Domain(grid, idx, vals, rs, sg, width=2)


def _sdf_band_torch(grid, sdf, lo, hi, device, chunk_cells=1 << 24):
    """Width-2 band (|sdf| <= gridDelta) of an SDF with Lipschitz constant 1
    over the index box [lo, hi], evaluated with torch on `device`: bricks of
    8^3 cells whose centre is further than half a diagonal plus 1.5 cells
    from the surface are skipped.  Returns (idx int32 (N,3), values)."""
    import torch

    gd = grid.delta
    dev = torch.device(device)
    B = 8
    nb = [(hi[d] - lo[d]) // B + 1 for d in range(3)]
    reach = (math.sqrt(3.0) * 4.0 + 1.5) * gd
    off = torch.arange(B, device=dev, dtype=torch.int64)
    OZ, OY, OX = torch.meshgrid(off, off, off, indexing="ij")
    offs = torch.stack([OX.reshape(-1), OY.reshape(-1), OZ.reshape(-1)], 1)
    by_, bx_ = torch.meshgrid(torch.arange(nb[1], device=dev), torch.arange(nb[0], device=dev),
                              indexing="ij")
    bx_, by_ = bx_.reshape(-1), by_.reshape(-1)
    idx_parts, val_parts = [], []
    for bz in range(nb[2]):
        cx = (lo[0] + bx_ * B + 3.5) * gd
        cy = (lo[1] + by_ * B + 3.5) * gd
        cz = torch.full_like(cx, (lo[2] + bz * B + 3.5) * gd, dtype=torch.float64)
        near = torch.abs(sdf(cx.double(), cy.double(), cz)) <= reach
        if not bool(near.any()):
            continue
        corner = torch.stack([lo[0] + bx_[near] * B, lo[1] + by_[near] * B,
                              torch.full_like(bx_[near], lo[2] + bz * B)], 1)
        per = max(1, chunk_cells // (B ** 3))
        for s in range(0, len(corner), per):
            cells = (corner[s:s + per, None, :] + offs[None, :, :]).reshape(-1, 3)
            inside = (cells[:, 0] <= hi[0]) & (cells[:, 1] <= hi[1]) & (cells[:, 2] <= hi[2])
            cells = cells[inside]
            v = sdf(cells[:, 0].double() * gd, cells[:, 1].double() * gd,
                    cells[:, 2].double() * gd) / gd
            keep = torch.abs(v) <= 1.0
            idx_parts.append(cells[keep].cpu().numpy())
            val_parts.append(v[keep].cpu().numpy())
    idx = np.concatenate(idx_parts) if idx_parts else np.zeros((0, 3), np.int64)
    vals = np.concatenate(val_parts) if val_parts else np.zeros(0)
    for d in range(3):
        if grid.is_periodic(d):
            idx[:, d] = grid.map_index(d, idx[:, d])
    return idx.astype(np.int32), vals


def hole_stack(lateral_cells=4096, grid_delta=0.02, pitch=1.28, radius=0.5, depth=2.0,
               layers=(0.1, 0.3), shift=(0.0, 0.0), device="cpu"):
    """The stacked-layer hole array: a substrate (material 0) with a square
    array of cylindrical holes (radius, depth, pitch; periodic in x/y) under
    two slabs on the flat top between the holes, of thickness layers[0]
    (material 1) and layers[1] (material 2, the top level set); every level
    set wraps the ones below.  Velocity per material 1.0 / 0.6 / 0.0 plus
    0.2 |n_z|.  The hole axes lie on grid points, `shift` cells away when
    given: cells at exactly the radius then carry values of order 1e-9, whose
    sign classes both precisions decide with the FP64 epsilon.
    Returns (grid, [three Domains], velocity)."""
    import torch

    from .velocity import FunctorVelocity

    half = lateral_cells * grid_delta / 2.0
    zlo, zhi = -depth - 0.5, layers[-1] + 0.5
    grid = Grid([-half, half, -half, half, zlo, zhi],
                [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], grid_delta)

    sx, sy = shift[0] * grid_delta, shift[1] * grid_delta

    def rho(x, y):
        px = torch.remainder(x + half - sx, pitch) - pitch / 2.0
        py = torch.remainder(y + half - sy, pitch) - pitch / 2.0
        return torch.sqrt(px * px + py * py)

    def substrate(x, y, z):
        return torch.maximum(z, -torch.maximum(rho(x, y) - radius, -z - depth))

    def stacked(h):
        def f(x, y, z):
            slab = torch.maximum(torch.maximum(z - h, -z), radius - rho(x, y))
            return torch.minimum(substrate(x, y, z), slab)
        return f

    lo = [grid.min[0], grid.min[1], grid.min[2]]
    hi = [grid.max[0] - 1, grid.max[1] - 1, grid.max[2]]
    doms = []
    for sdf in (substrate, stacked(layers[0]), stacked(layers[1])):
        idx, vals = _sdf_band_torch(grid, sdf, lo, hi, device)
        gd = grid.delta

        def sign_fn(x, y, z, sdf=sdf):
            out = np.empty(len(x), np.int64)
            step = 1 << 22
            for s in range(0, len(x), step):
                t = [torch.as_tensor(np.asarray(a[s:s + step], np.float64) * gd, device=device)
                     for a in (x, y, z)]
                out[s:s + step] = np.where(sdf(*t).cpu().numpy() < 0, -1, 1)
            return out

        rs, sg = make_runs(idx, sign_fn, [lo[0] - 1, lo[1] - 1, lo[2] - 1],
                           [hi[0] + 1, hi[1] + 1, hi[2] + 1])
        doms.append(Domain(grid, idx, vals, rs, sg, width=2))
    vel = FunctorVelocity(3)
    for m, rate in enumerate((1.0, 0.6, 0.0)):
        vel.set_rate(m, rate)
        vel.set_abs(m, 2, 0.2)
    return grid, doms, vel


def tiled_hole_stack(tiles, base_cells=1024, device="cuda", precision=1):
    """hole_stack at (tiles * base_cells)^2 lateral cells, built by tiling
    the base_cells^2 workload tiles x tiles times (the hole period divides
    base_cells): the points are shifted into every tile and the undefined
    runs rebuilt from the base level sets' signs (point queries on a context
    holding them).  Returns (grid, [three Domains], velocity, base grid,
    [three base Domains])."""
    from .advect import Context

    grid_s, doms_s, vel = hole_stack(lateral_cells=base_cells, device=device)
    n, half = base_cells, base_cells // 2
    big = tiles * n
    grid = Grid(None, grid_s.bc, grid_s.delta, index_min=[-big // 2, -big // 2, grid_s.min[2]],
                index_max=[big // 2, big // 2, grid_s.max[2]])
    q = Context(0, precision)
    q.set_grid(grid_s)
    q.set_level_set_count(len(doms_s))
    for i, d in enumerate(doms_s):
        q.upload(i, d)
    doms = []
    for i, d in enumerate(doms_s):
        parts = []
        for a in range(tiles):
            for b in range(tiles):
                t = d.idx.astype(np.int64)
                t = t + np.array([n * a - big // 2 + half, n * b - big // 2 + half, 0], np.int64)
                parts.append(t)
        idx = np.concatenate(parts)
        val = np.tile(d.values, tiles * tiles)
        o = lex_order(idx)
        idx, val = idx[o], val[o]
        del parts, o

        def sign_fn(x, y, z, i=i):
            out = np.empty(len(x), np.int64)
            step = 1 << 24
            for s0 in range(0, len(x), step):
                # big-grid x = -big/2 + n a + (x_base + half) in tile a
                w = np.stack([(np.asarray(x[s0:s0 + step]) + big // 2) % n - half,
                              (np.asarray(y[s0:s0 + step]) + big // 2) % n - half,
                              np.asarray(z[s0:s0 + step])], 1).astype(np.int32)
                out[s0:s0 + step] = np.where(q.values_at(i, w) < 0, -1, 1)
            return out

        rs, sg = make_runs(idx, sign_fn, idx.min(0) - 1, idx.max(0) + 1)
        doms.append(Domain(grid, idx.astype(np.int32), val, rs, sg, width=d.width))
    q.close()
    return grid, doms, vel, grid_s, doms_s
