"""Seeded synthetic initial conditions for the Euler workloads, evaluated at
the Gauss-Legendre nodes of every cell (what the reference's
adjustPointSolution does at t = 0, kernels/aderdg/generic/c/*/solutionAdjustment.cpph).

All workloads are analytic: no dataset is involved. Densities/pressures are
turned into conserved variables (rho, rho u, E) with gamma = 1.4.
"""
import functools
import os
import sys

import numpy as np

GAMMA = 1.4
_CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")


@functools.lru_cache(maxsize=None)
def _gl_nodes(order):
    sys.path.insert(0, _CSRC)
    try:
        import gen_tables
    finally:
        sys.path.pop(0)
    return tuple(gen_tables.build(order)["nodes"])


def gl_nodes(order):
    return np.array(_gl_nodes(order))


def node_coordinates(dim, order, cells, offset=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    """(ncells, b^dim, dim) coordinates of every node, cells in x-fastest order,
    nodes in (z, y, x) order with x fastest."""
    x = gl_nodes(order)
    b = order + 1
    dx = [size[d] / cells[d] for d in range(dim)]
    if dim == 2:
        j, i = np.meshgrid(np.arange(cells[1]), np.arange(cells[0]), indexing="ij")
        cy, cx = j.ravel(), i.ravel()
        ny, nx = np.meshgrid(x, x, indexing="ij")
        X = offset[0] + (cx[:, None] + nx.ravel()[None, :]) * dx[0]
        Y = offset[1] + (cy[:, None] + ny.ravel()[None, :]) * dx[1]
        return np.stack([X, Y], axis=-1)
    k, j, i = np.meshgrid(np.arange(cells[2]), np.arange(cells[1]), np.arange(cells[0]), indexing="ij")
    cz, cy, cx = k.ravel(), j.ravel(), i.ravel()
    nz, ny, nx = np.meshgrid(x, x, x, indexing="ij")
    X = offset[0] + (cx[:, None] + nx.ravel()[None, :]) * dx[0]
    Y = offset[1] + (cy[:, None] + ny.ravel()[None, :]) * dx[1]
    Z = offset[2] + (cz[:, None] + nz.ravel()[None, :]) * dx[2]
    assert X.shape[1] == b ** 3
    return np.stack([X, Y, Z], axis=-1)


def conserved(rho, vel, p):
    """rho: (...), vel: (..., 3), p: (...) -> Q (..., 5)"""
    Q = np.empty(rho.shape + (5,))
    Q[..., 0] = rho
    Q[..., 1:4] = rho[..., None] * vel
    Q[..., 4] = p / (GAMMA - 1) + 0.5 * rho * np.sum(vel * vel, axis=-1)
    return Q


def _periodic_d2(X, c):
    d = X - c
    d -= np.round(d)
    return np.sum(d * d, axis=-1)


def gaussian_pulse_2d(order, cells=(27, 27), seed=0, amplitude=0.5):
    """rho = 1 + a exp(-|x - x0|^2 / 0.01), x0 ~ U[0.3, 0.7]^2, u = (1, 1, 0),
    p = 1 on the periodic unit square (minimum-image distance); a = 0.5 unless
    given."""
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(0.3, 0.7, size=2)
    X = node_coordinates(2, order, cells)
    rho = 1.0 + amplitude * np.exp(-_periodic_d2(X, x0) / 0.01)
    vel = np.broadcast_to(np.array([1.0, 1.0, 0.0]), rho.shape + (3,))
    return conserved(rho, vel, np.ones_like(rho)), dict(x0=x0.tolist(), amplitude=amplitude)


def pulse_ensemble(n=256, seed=0, sides=(9, 27, 81), orders=(3, 5, 7)):
    """The ragged ensemble: n independent 2D periodic pulse problems, each with
    cells per side drawn from `sides`, order from `orders`, its own seeded
    centre and amplitude U[0.1, 0.5]. Returns a list of dicts (order, cells,
    seed, amplitude, luh)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        side = int(rng.choice(sides))
        order = int(rng.choice(orders))
        amp = float(rng.uniform(0.1, 0.5))
        iseed = int(rng.integers(0, 2 ** 31 - 1))
        luh, _ = gaussian_pulse_2d(order, (side, side), seed=iseed, amplitude=amp)
        out.append(dict(order=order, cells=(side, side), seed=iseed, amplitude=amp, luh=luh))
    return out


def gaussian_pulses_3d(order, cells=(27, 27, 27), seed=0, npulses=4):
    """rho = 1 + sum_k a_k exp(-|x - c_k|^2 / w_k^2), a_k ~ U[0.1, 0.5],
    w_k ~ U[0.05, 0.15], c_k ~ U[0, 1]^3; one velocity with components
    U[-0.5, 0.5]; p = 1; periodic unit cube."""
    rng = np.random.default_rng(seed)
    amps = rng.uniform(0.1, 0.5, size=npulses)
    widths = rng.uniform(0.05, 0.15, size=npulses)
    centres = rng.uniform(0.0, 1.0, size=(npulses, 3))
    vel0 = rng.uniform(-0.5, 0.5, size=3)
    # the Gaussian of the minimum-image distance factors by axis: per pulse
    # three 1-D factors over (cell, node) of each axis, one outer product
    x = gl_nodes(order)
    nx, ny, nz = cells
    rho = np.ones((nz, ny, nx) + (order + 1,) * 3)
    for a, w, c in zip(amps, widths, centres):
        f = []
        for d, n in enumerate((nx, ny, nz)):
            X = (np.arange(n)[:, None] + x[None, :]) * (1.0 / n)
            dd = X - c[d]
            dd -= np.round(dd)
            f.append(np.exp(-dd * dd / (w * w)))
        fx, fy, fz = f
        rho += a * (fz[:, None, None, :, None, None] * fy[None, :, None, None, :, None]) * \
            fx[None, None, :, None, None, :]
    rho = rho.reshape(nx * ny * nz, -1)
    vel = np.broadcast_to(vel0, rho.shape + (3,))
    return conserved(rho, vel, np.ones_like(rho)), dict(amps=amps.tolist(), widths=widths.tolist(),
                                                        centres=centres.tolist(), velocity=vel0.tolist())


def explosion_2d(order, cells=(81, 81), seed=0, radius=0.2):
    """Circular explosion: inside |x - c| < radius rho = 1, p = 1, outside
    rho = 0.125, p = 0.1, zero velocity; c ~ U[0.4, 0.6]^2."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.4, 0.6, size=2)
    X = node_coordinates(2, order, cells)
    r2 = np.sum((X - c) ** 2, axis=-1)
    inside = r2 < radius * radius
    rho = np.where(inside, 1.0, 0.125)
    p = np.where(inside, 1.0, 0.1)
    vel = np.zeros(rho.shape + (3,))
    return conserved(rho, vel, p), dict(centre=c.tolist())


def subcell_coordinates(dim, order, cells, offset=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    """(ncells, (2N+1)^dim, dim) centres of the FV subcells of every cell (the
    limiter's (2N+1)^d patch), subcells in (z, y, x) order with x fastest."""
    B = 2 * order + 1
    xs = (np.arange(B) + 0.5) / B
    dx = [size[d] / cells[d] for d in range(dim)]
    if dim == 2:
        j, i = np.meshgrid(np.arange(cells[1]), np.arange(cells[0]), indexing="ij")
        ny, nx = np.meshgrid(xs, xs, indexing="ij")
        X = offset[0] + (i.ravel()[:, None] + nx.ravel()[None, :]) * dx[0]
        Y = offset[1] + (j.ravel()[:, None] + ny.ravel()[None, :]) * dx[1]
        return np.stack([X, Y], axis=-1)
    k, j, i = np.meshgrid(np.arange(cells[2]), np.arange(cells[1]), np.arange(cells[0]), indexing="ij")
    nz, ny, nx = np.meshgrid(xs, xs, xs, indexing="ij")
    X = offset[0] + (i.ravel()[:, None] + nx.ravel()[None, :]) * dx[0]
    Y = offset[1] + (j.ravel()[:, None] + ny.ravel()[None, :]) * dx[1]
    Z = offset[2] + (k.ravel()[:, None] + nz.ravel()[None, :]) * dx[2]
    return np.stack([X, Y, Z], axis=-1)


def explosion(dim, order, cells, seed=0, radius=0.2):
    """Circular/spherical explosion at the GL nodes and at the FV subcell
    centres: inside |x - c| < radius rho = 1, p = 1, outside rho = 0.125,
    p = 0.1, zero velocity; c ~ U[0.4, 0.6]^dim. Returns (luh, fv, params)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.4, 0.6, size=dim)

    def state(pts):
        # |x - c|^2 summed over the axes in order, from per-axis squares over
        # (cell, point) of each axis (the coordinates are (cell + point) dx)
        sq = [((np.arange(cells[d])[:, None] + pts[None, :]) * (1.0 / cells[d]) - c[d]) ** 2 for d in range(dim)]
        if dim == 2:
            r2 = sq[0][None, :, None, :] + sq[1][:, None, :, None]  # (cy, cx, py, px)
        else:
            r2 = (sq[0][None, None, :, None, None, :] + sq[1][None, :, None, None, :, None]) + \
                sq[2][:, None, None, :, None, None]  # (cz, cy, cx, pz, py, px)
        inside = (r2 < radius * radius).reshape(int(np.prod(cells[:dim])), -1)
        Q = np.zeros(inside.shape + (5,))
        Q[..., 0] = np.where(inside, 1.0, 0.125)
        Q[..., 4] = np.where(inside, 1.0, 0.1) / (GAMMA - 1)
        return Q

    B = 2 * order + 1
    return state(gl_nodes(order)), state((np.arange(B) + 0.5) / B), dict(centre=c.tolist())


def elastic_pulse(dim, order, cells, seed=0):
    """Linear elastic waves on the periodic unit square/cube: a Gaussian
    velocity pulse (width 0.1, direction ~ U[-1, 1]^3, centre ~ U[0.3, 0.7]^d)
    with zero initial stress in a smoothly heterogeneous medium,
    rho = 1 + 0.3 s, lambda = 2 + 0.5 s, mu = 1 + 0.2 s with
    s = sin(2 pi (x + phase_x)) sin(2 pi (y + phase_y)), phases ~ U[0, 1].
    Returns luh (ncells, b^d, 12): sxx syy szz sxy syz sxz u v w lambda mu rho."""
    return _elastic_at(node_coordinates(dim, order, cells), dim, seed)


def _elastic_at(X, dim, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.3, 0.7, size=dim)
    direction = rng.uniform(-1.0, 1.0, size=3)
    phase = rng.uniform(0.0, 1.0, size=2)
    g = np.exp(-_periodic_d2(X, c) / 0.01)
    s = np.sin(2 * np.pi * (X[..., 0] + phase[0])) * np.sin(2 * np.pi * (X[..., 1] + phase[1]))
    Q = np.zeros(X.shape[:-1] + (12,))
    Q[..., 6:9] = g[..., None] * direction
    Q[..., 9] = 2.0 + 0.5 * s
    Q[..., 10] = 1.0 + 0.2 * s
    Q[..., 11] = 1.0 + 0.3 * s
    return Q, dict(centre=c.tolist(), direction=direction.tolist(), phase=phase.tolist())


def refined_node_coordinates(dim, order, cells, box_lo, box_hi, offset=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    """(ncells, b^dim, dim) node coordinates of a mesh made by
    exa_mesh_create_refined: the unrefined coarse cells (x fastest), then the
    fine cells of the refined box (x fastest)."""
    return nested_node_coordinates(dim, order, cells, [(box_lo, box_hi)], offset, size)


def nested_node_coordinates(dim, order, cells, boxes, offset=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    """(ncells, b^dim, dim) node coordinates of a mesh made by
    exa_mesh_create_nested: boxes[k] = (lo, hi) in level-k cell coordinates."""
    return boxes_node_coordinates(dim, order, cells, [(k, lo, hi) for k, (lo, hi) in enumerate(boxes)], offset, size)


def box_levels(dim, cells, boxes):
    """Per level: (r0, state) with r0 the bounding rectangle's lower corner
    and state an array over it (z, y, x order) holding 0 outside the level's
    region, 1 for a cell, 2 for a refined position; boxes = [(level, lo, hi)]."""
    L = max(b[0] for b in boxes) + 2
    out = []
    for lev in range(L):
        if lev == 0:
            r0, r1 = [0] * dim, list(cells[:dim])
        else:
            sub = [b for b in boxes if b[0] == lev - 1]
            r0 = [min(3 * b[1][d] for b in sub) for d in range(dim)]
            r1 = [max(3 * b[2][d] for b in sub) for d in range(dim)]
        shape = tuple(r1[d] - r0[d] for d in reversed(range(dim)))
        st = np.ones(shape, dtype=np.int8) if lev == 0 else np.zeros(shape, dtype=np.int8)
        if lev > 0:
            for b in boxes:
                if b[0] == lev - 1:
                    sl = tuple(slice(3 * b[1][d] - r0[d], 3 * b[2][d] - r0[d]) for d in reversed(range(dim)))
                    st[sl] = 1
        out.append([r0, st])
    for b in boxes:
        r0, st = out[b[0]]
        sl = tuple(slice(b[1][d] - r0[d], b[2][d] - r0[d]) for d in reversed(range(dim)))
        st[sl] = 2
    return out


def boxes_node_coordinates(dim, order, cells, boxes, offset=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    """(ncells, b^dim, dim) node coordinates of a mesh made by
    exa_mesh_create_boxes: level by level, the cells x fastest over the
    level's bounding rectangle. boxes = [(level, lo, hi)]."""
    out = []
    for lev, (r0, st) in enumerate(box_levels(dim, cells, boxes)):
        ext = list(reversed(st.shape))
        dx = [size[d] / (cells[d] * 3 ** lev) for d in range(dim)]
        off = [offset[d] + r0[d] * dx[d] for d in range(dim)] + [0.0] * (3 - dim)
        sz = [ext[d] * dx[d] for d in range(dim)] + [1.0] * (3 - dim)
        X = node_coordinates(dim, order, ext, off, sz)
        out.append(X[st.reshape(-1) == 1])
    return np.concatenate(out, axis=0)


def pulse_refined(dim, order, cells, box_lo, box_hi, seed=0):
    """Gaussian density pulse (amplitude 0.3, width 0.1) centred in the
    refined box plus a seeded offset U[-0.05, 0.05]^dim, carried by the
    velocity (1, 0.5, 0.25) through the box's faces; p = 1; periodic unit
    domain. Returns luh in the refined mesh's cell order."""
    return pulse_nested(dim, order, cells, [(box_lo, box_hi)], seed)


def pulse_nested(dim, order, cells, boxes, seed=0):
    """pulse_refined on a nested mesh (centre: the first box's centre plus a
    seeded offset U[-0.05, 0.05]^dim)."""
    return pulse_boxes(dim, order, cells, [(k, lo, hi) for k, (lo, hi) in enumerate(boxes)], seed)


def pulse_boxes(dim, order, cells, boxes, seed=0):
    """pulse_refined on a mesh refined by boxes = [(level, lo, hi)] (centre:
    the first box's centre plus a seeded offset U[-0.05, 0.05]^dim)."""
    rng = np.random.default_rng(seed)
    lev, box_lo, box_hi = boxes[0]
    c = np.array([(box_lo[d] + box_hi[d]) / (2.0 * cells[d] * 3 ** lev) for d in range(dim)])
    c = c + rng.uniform(-0.05, 0.05, size=dim)
    X = boxes_node_coordinates(dim, order, cells, boxes)
    rho = 1.0 + 0.3 * np.exp(-_periodic_d2(X, c) / 0.01)
    vel = np.zeros(rho.shape + (3,))
    vel[..., :dim] = np.array([1.0, 0.5, 0.25][:dim])
    return conserved(rho, vel, np.ones_like(rho))


def elastic_pulse_refined(dim, order, cells, box_lo, box_hi, seed=0):
    """elastic_pulse's fields at the nodes of a refined mesh (cell order of
    refined_node_coordinates). Returns luh (ncells, b^d, 12)."""
    return _elastic_at(refined_node_coordinates(dim, order, cells, box_lo, box_hi), dim, seed)[0]
