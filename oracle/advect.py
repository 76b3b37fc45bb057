"""Oracle (TEST INFRASTRUCTURE ONLY): FP64 numpy restatement of the
differentiable rollout -- semi-Lagrangian MAC self-advection, its adjoint, the
box loss, and advect->project rollouts with checkpointed reverse passes.

Used only by tests/ as the checker of xfluid_b200's CUDA kernels
(xfluid_b200/csrc/xfp_advect.cu) and rollout driver (xfluid_b200/rollout.py).
xFluid has no counterpart (it advects velocity with particles,
FluidSimulator.cpp:652-1085), so this oracle is pinned by FP64 central
differences instead of reference outputs (tests/test_rollout.py).

Definition (cell units, cell (i,j,k) centred at (i+.5, j+.5, k+.5)):
  u face (i,j,k) at (i, j+.5, k+.5); v at (i+.5, j, k+.5); w at (i+.5, j+.5, k)
  sample G(p): trilinear in G's node lattice, each lattice coordinate clamped
               to [0, n-1]; the derivative is 0 along a clamped coordinate
  advect:      out_G[f] = G(x_f - c * vel(x_f)), vel = (u, v, w) sampled at x_f
"""
from __future__ import annotations

import numpy as np

# lattice offsets per component (x, y, z)
_OFF = {0: (0.0, 0.5, 0.5), 1: (0.5, 0.0, 0.5), 2: (0.5, 0.5, 0.0)}


def _extents(comp, ni, nj, nk):
    return [(ni + 1, nj, nk), (ni, nj + 1, nk), (ni, nj, nk + 1)][comp]


def face_positions(comp, ni, nj, nk):
    na, nb, nc = _extents(comp, ni, nj, nk)
    ox, oy, oz = _OFF[comp]
    c, b, a = np.meshgrid(np.arange(nc), np.arange(nb), np.arange(na), indexing="ij")
    return a + ox, b + oy, c + oz


def _axis(x, o, n):
    f = x - o
    inside = (f > 0) & (f < n - 1)
    f = np.clip(f, 0, n - 1)
    a = np.clip(np.floor(f).astype(np.int64), 0, max(n - 2, 0))
    if n > 1:
        return a, a + 1, f - a, inside
    return a, a, np.zeros_like(f), inside


def stencil(comp, ni, nj, nk, x, y, z):
    """(flat indices[8], weights[8], d weights / d (x,y,z) [3][8])."""
    na, nb, nc = _extents(comp, ni, nj, nk)
    ox, oy, oz = _OFF[comp]
    a0, a1, ta, ia = _axis(x, ox, na)
    b0, b1, tb, ib = _axis(y, oy, nb)
    c0, c1, tc, ic = _axis(z, oz, nc)
    A, B, Cc = (a0, a1), (b0, b1), (c0, c1)
    wa, wb, wc = (1 - ta, ta), (1 - tb, tb), (1 - tc, tc)
    da = (-ia.astype(float), ia.astype(float))
    db = (-ib.astype(float), ib.astype(float))
    dc = (-ic.astype(float), ic.astype(float))
    idx, w, dw = [], [], [[], [], []]
    for q in range(8):
        qa, qb, qc = q & 1, (q >> 1) & 1, q >> 2
        idx.append((Cc[qc] * nb + B[qb]) * na + A[qa])
        w.append(wa[qa] * wb[qb] * wc[qc])
        dw[0].append(da[qa] * wb[qb] * wc[qc])
        dw[1].append(wa[qa] * db[qb] * wc[qc])
        dw[2].append(wa[qa] * wb[qb] * dc[qc])
    return idx, w, dw


def _gather(G, st):
    idx, w, _ = st
    flat = G.ravel()
    out = np.zeros(idx[0].shape)
    for q in range(8):
        out = out + w[q] * flat[idx[q]]
    return out


def advect(u, v, w, c):
    """Semi-Lagrangian self-advection (the definition in the module header)."""
    nk, nj, ni = u.shape[0], u.shape[1], u.shape[2] - 1
    G = (u, v, w)
    out = []
    for comp in range(3):
        x, y, z = face_positions(comp, ni, nj, nk)
        vel = [_gather(G[d], stencil(d, ni, nj, nk, x, y, z)) for d in range(3)]
        st = stencil(comp, ni, nj, nk, x - c * vel[0], y - c * vel[1], z - c * vel[2])
        out.append(_gather(G[comp], st).reshape(G[comp].shape))
    return tuple(out)


def advect_adjoint(u, v, w, gu, gv, gw, c):
    """J^T g of advect at state (u, v, w): weights at the departure point plus
    the departure point's dependence on vel(x_f)."""
    nk, nj, ni = u.shape[0], u.shape[1], u.shape[2] - 1
    G = (u, v, w)
    Gb = (gu, gv, gw)
    D = [np.zeros(a.size) for a in G]
    for comp in range(3):
        x, y, z = face_positions(comp, ni, nj, nk)
        g = Gb[comp].ravel()
        sv = [stencil(d, ni, nj, nk, x, y, z) for d in range(3)]
        vel = [_gather(G[d], sv[d]).ravel() for d in range(3)]
        x, y, z = x.ravel(), y.ravel(), z.ravel()
        idx, wt, dw = stencil(comp, ni, nj, nk, x - c * vel[0], y - c * vel[1], z - c * vel[2])
        flat = G[comp].ravel()
        grad = [np.zeros(g.shape) for _ in range(3)]
        for q in range(8):
            np.add.at(D[comp], idx[q], wt[q] * g)
            for d in range(3):
                grad[d] = grad[d] + dw[d][q] * flat[idx[q]]
        for d in range(3):
            pv = -c * grad[d] * g
            sidx, sw, _ = sv[d]
            for q in range(8):
                np.add.at(D[d], sidx[q].ravel(), sw[q].ravel() * pv)
    return tuple(Dd.reshape(a.shape) for Dd, a in zip(D, G))


def box_mask(comp, ni, nj, nk, box):
    x, y, z = face_positions(comp, ni, nj, nk)
    X, Y, Z = x / ni, y / nj, z / nk
    (x0, x1), (y0, y1), (z0, z1) = box
    return (X >= x0) & (X <= x1) & (Y >= y0) & (Y <= y1) & (Z >= z0) & (Z <= z1)


def box_loss(u, v, w, box):
    nk, nj, ni = u.shape[0], u.shape[1], u.shape[2] - 1
    loss, grads = 0.0, []
    for comp, a in enumerate((u, v, w)):
        m = box_mask(comp, ni, nj, nk, box)
        loss += float((a[m] ** 2).sum())
        grads.append(np.where(m, 2 * a, 0.0))
    return loss, tuple(grads)


# ---------------------------------------------------------------- rollouts
def _scene(mat, u, v, w):
    from xfluid_b200.scenes import Scene
    nk, nj, ni = mat.shape
    return Scene(ni, nj, nk, mat, u, v, w)


def project(O, mat, u, v, w, tol):
    out = O.project(_scene(mat, u, v, w), tol=tol, maxit=20000)
    return out["u"], out["v"], out["w"]


def project_adjoint(O, mat, gu, gv, gw, tol):
    """g - D^T A^{-1} G^T g with the oracle's assembly, PCG and transposes."""
    sc = _scene(mat, gu, gv, gw)
    A = O.assemble(sc)
    q = O.apply_T(sc, gu, gv, gw)
    lam = O.pcg(sc, dict(A, b=q), tol, 20000)["p"]
    du, dv, dw = O.rhs_T(sc, lam)
    return gu - du, gv - dv, gw - dw


def rollout_loss(O, mat, u, v, w, steps, c, box, tol):
    for _ in range(steps):
        u, v, w = project(O, mat, *advect(u, v, w, c), tol)
    return box_loss(u, v, w, box)[0]


def rollout_grad(O, mat, u0, v0, w0, steps, c, box, tol, checkpoint_every=4):
    """Loss and dL/d(u0,v0,w0): forward keeping a checkpoint every
    `checkpoint_every` steps, reverse pass recomputing each segment."""
    ck = {}
    u, v, w = u0, v0, w0
    for n in range(steps):
        if n % checkpoint_every == 0:
            ck[n] = (u, v, w)
        u, v, w = project(O, mat, *advect(u, v, w, c), tol)
    loss, g = box_loss(u, v, w, box)
    for s0 in sorted(ck, reverse=True):
        states = []
        u, v, w = ck[s0]
        for n in range(s0, min(s0 + checkpoint_every, steps)):
            states.append((u, v, w))
            u, v, w = project(O, mat, *advect(u, v, w, c), tol)
        for st in reversed(states):
            g = project_adjoint(O, mat, *g, tol)
            g = advect_adjoint(*st, *g, c)
    return loss, g
