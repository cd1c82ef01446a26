"""CPU restatement of the reference's multigrid building blocks (test
infrastructure only: the product never imports this module).

* ``coarse_nodes``   -- restrict_c (code/handwritten/grid/coordinates_extend.f90:336-356):
  every other node from the first physical one, then add_ghost_nodes
  (coordinates_extend.f90:529-538: ghost cells mirror the end cells).  The
  reference stops on an odd cell count; the library keeps the last fine
  cell as a coarse cell of its own, and on a periodic axis sizes a ghost cell
  like its periodic partner (the cell at the other end).  Both extensions
  are restated here as the library applies them.
* ``theta``          -- interpolation_stencil (grid/interpolation_stencils.f90:12-35):
  D(i) = (hn(i+1) - hc(i)) / (hc(i+1) - hc(i)), U = 1 - D.
* ``prolong_axis``   -- prolongate_C_GF (grid_field/GF_MG/GF_prolongate.f90:22-56)
  along one axis: for each coarse node i between cells i and i+1,
  node = u(i+1) D(i) + u(i) U(i) (coarse-grid theta), fine cell 2i-1 =
  (u(i) + node)/2 and fine cell 2i = (u(i+1) + node)/2; the coarse ghost
  cells hold the homogeneous BC images (apply_BCs_implicit: Dirichlet -u,
  Neumann u, periodic the far interior cell).  An unpaired last fine cell
  (odd count, library extension) takes its coarse cell's value.
* ``restrict``       -- the transpose of that prolongation (the library's
  restriction; the reference's restrict_C is a volume-weighted average).
* ``sor_pattern``    -- the point update of redBlack (solvers/SOR/SOR.f90:234-268)
  on the points of one parity pattern ``odd`` (every other point from
  2+odd along each axis): u = (1-w) u + w (sum_nb c_nb u_nb - f) / r with c
  the two-gradient Laplacian weights of the mesh's staggered stencils and r
  minus its diagonal (init_r_GF, SOR.f90:287-314).  The reference reads the
  ghost values stored before the sweep; ``ghost="implicit"`` instead moves
  the homogeneous ghost image of the point itself into r (the library's
  smoother), ``ghost="explicit"`` reads the images of the values before the
  sweep.  The library's red sweep is the patterns with an even index sum
  (000, 011, 101, 110), black the rest; points of one colour never
  neighbour each other, so the order of the patterns within a colour does
  not matter.
"""
from __future__ import annotations

import numpy as np

DIRICHLET, NEUMANN, PERIODIC = 1, 2, 3


def add_ghost_nodes(h):
    h = np.asarray(h, float)
    return np.concatenate([[h[0] - (h[1] - h[0])], h, [h[-1] + (h[-1] - h[-2])]])


def coarse_nodes(hn, periodic=False):
    """Node coordinates (with ghosts) of the coarsened axis."""
    hn = np.asarray(hn, float)
    sn = len(hn)
    phys = hn[1:sn - 1]
    c = list(phys[0::2])
    if (len(phys) - 1) % 2 == 1:  # odd cell count: keep the last node
        c.append(phys[-1])
    c = np.asarray(c)
    if not periodic:
        return add_ghost_nodes(c)
    h_first, h_last = c[1] - c[0], c[-1] - c[-2]
    return np.concatenate([[c[0] - h_last], c, [c[-1] + h_first]])


def theta(hn):
    """1-based arrays (index 0 unused) D, U of length sc."""
    hn = np.asarray(hn, float)
    hc = 0.5 * (hn[1:] + hn[:-1])
    sc = len(hc)
    D = np.zeros(sc)
    U = np.zeros(sc)
    for i in range(1, sc):  # 1-based i = 1..sc-1 -> 0-based hc[i-1], hn[i]
        D[i] = (hn[i] - hc[i - 1]) / (hc[i] - hc[i - 1])
        U[i] = 1.0 - D[i]
    return D, U


def fill_ghosts(u, axis, bc_lo, bc_hi):
    """Homogeneous (implicit) BC images on the two ghost planes of one axis."""
    u = np.moveaxis(u, axis, 0).copy()
    s = u.shape[0]
    if bc_lo == PERIODIC:
        u[0] = u[s - 2]
    else:
        u[0] = (-1.0 if bc_lo == DIRICHLET else 1.0) * u[1]
    if bc_hi == PERIODIC:
        u[s - 1] = u[1]
    else:
        u[s - 1] = (-1.0 if bc_hi == DIRICHLET else 1.0) * u[s - 2]
    return np.moveaxis(u, 0, axis)


def prolong_axis(u, hn_coarse, axis, nfine, bc_lo, bc_hi):
    """prolongate_C along ``axis``: u has coarse extent s along it (ghosts
    included); the result has the fine extent nfine + 2 (its ghost planes
    are left zero: extrap is not restated, only interior values are used)."""
    u = fill_ghosts(u, axis, bc_lo, bc_hi)
    u = np.moveaxis(u, axis, 0)
    s = u.shape[0]
    D, U = theta(hn_coarse)
    p = np.zeros((nfine + 2,) + u.shape[1:])
    odd = nfine % 2 == 1
    for i in range(1, s):  # 1-based coarse i = 1..s-1
        node = u[i] * D[i] + u[i - 1] * U[i]     # u(i+1)*D(i) + u(i)*U(i)
        iL, iR = 2 * i - 1, 2 * i                 # 1-based fine indices
        if 1 <= iL <= nfine + 2:
            p[iL - 1] = 0.5 * (u[i - 1] + node)
        if 1 <= iR <= nfine + 2:
            p[iR - 1] = 0.5 * (u[i] + node)
    if odd:  # unpaired last fine interior cell (library extension): injection
        p[nfine] = u[s - 2]
    return np.moveaxis(p, 0, axis)


def prolong(uc, coarse_hn, fine_shape, bcs):
    """3-D prolongation of a coarse correction (interior of the result is
    what matters): per axis, prolongate when the axis was coarsened."""
    v = np.asarray(uc, float)
    for d in range(3):
        nf = fine_shape[d] - 2
        if v.shape[d] - 2 == nf:
            continue
        v = prolong_axis(v, coarse_hn[d], d, nf, bcs[2 * d], bcs[2 * d + 1])
    return v


def _axis_matrix(coarse_hn, nc, nf, bc_lo, bc_hi):
    """1-D prolongation as a matrix (fine interior x coarse interior), the
    ghost images folded in."""
    P = np.zeros((nf, nc))
    for c in range(nc):
        e = np.zeros(nc + 2)
        e[c + 1] = 1.0
        P[:, c] = prolong_axis(e, coarse_hn, 0, nf, bc_lo, bc_hi)[1:-1]
    return P


def restrict(tf, coarse_hn, coarse_shape, bcs):
    """The transpose of ``prolong`` applied to a fine residual: result on the
    coarse level's interior (ghosts zero)."""
    t = np.asarray(tf, float)[1:-1, 1:-1, 1:-1]
    for d in range(3):
        nc, nf = coarse_shape[d] - 2, t.shape[d]
        if nc == nf:
            continue
        P = _axis_matrix(coarse_hn[d], nc, nf, bcs[2 * d], bcs[2 * d + 1])
        t = np.moveaxis(np.tensordot(P.T, np.moveaxis(t, d, 0), axes=(1, 0)), 0, d)
    out = np.zeros(coarse_shape)
    out[1:-1, 1:-1, 1:-1] = t
    return out


def _weights(hn):
    """Two-gradient Laplacian weights of one CC axis, 1-based t: wm(t), wp(t)
    for u(t-1), u(t+1) and the diagonal share w0(t) (stagCC2N then stagN2CC,
    derivative_stencils.f90)."""
    hn = np.asarray(hn, float)
    sn = len(hn)
    sc = sn - 1
    hc = 0.5 * (hn[1:] + hn[:-1])
    dhn = np.diff(hn)          # dhn[t-1] = hn(t+1) - hn(t), t = 1..sn-1
    dhc = np.diff(hc)          # dhc[t-1] = hc(t+1) - hc(t), t = 1..sc-1
    wm = np.zeros(sc + 1)
    wp = np.zeros(sc + 1)
    w0 = np.zeros(sc + 1)
    for t in range(2, sc):     # interior cells
        cD_lo, cU_lo = -1.0 / dhc[t - 2], 1.0 / dhc[t - 2]   # stagCC2N at t-1
        cD_hi, cU_hi = -1.0 / dhc[t - 1], 1.0 / dhc[t - 1]   # stagCC2N at t
        nD, nU = -1.0 / dhn[t - 1], 1.0 / dhn[t - 1]         # stagN2CC at t
        wm[t] = cD_lo * nD
        wp[t] = cU_hi * nU
        w0[t] = cU_lo * nD + cD_hi * nU
    return wm, wp, w0


def sor_pattern(u, f, hns, bcs, omega, odd, ghost="implicit"):
    """redBlack on pattern ``odd`` (3 ints 0/1), in place on u (CC, ghosts
    included); f is the unweighted right-hand side (the library's r / vol)."""
    W = [_weights(h) for h in hns]
    s = u.shape
    ref = u.copy() if ghost == "explicit" else None
    for k in range(2 + odd[2], s[2], 2):
        if k > s[2] - 1:
            break
        for j in range(2 + odd[1], s[1], 2):
            if j > s[1] - 1:
                break
            for i in range(2 + odd[0], s[0], 2):
                if i > s[0] - 1:
                    break
                I = (i, j, k)
                acc = 0.0
                r = 0.0
                for d in range(3):
                    wm, wp, w0 = W[d]
                    t = I[d]
                    r -= w0[t]
                    for side, w in ((-1, wm[t]), (1, wp[t])):
                        J = list(I)
                        J[d] = t + side
                        lo, hi = bcs[2 * d], bcs[2 * d + 1]
                        if J[d] == 1 or J[d] == s[d]:
                            b = lo if J[d] == 1 else hi
                            if b == PERIODIC:
                                J[d] = s[d] - 1 if J[d] == 1 else 2
                                acc += w * u[J[0] - 1, J[1] - 1, J[2] - 1]
                            else:
                                fac = -1.0 if b == DIRICHLET else 1.0
                                if ghost == "implicit":
                                    r -= w * fac
                                else:
                                    acc += w * fac * ref[i - 1, j - 1, k - 1]
                        else:
                            acc += w * u[J[0] - 1, J[1] - 1, J[2] - 1]
                u0 = u[i - 1, j - 1, k - 1]
                u[i - 1, j - 1, k - 1] = u0 * (1.0 - omega) + omega * (acc - f[i - 1, j - 1, k - 1]) / r
    return u


RED = ((0, 0, 0), (0, 1, 1), (1, 0, 1), (1, 1, 0))
BLACK = ((1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1))


def vol(hns):
    d = [np.diff(np.asarray(h, float)) for h in hns]
    return np.einsum("i,j,k->ijk", *d)


def red_black(e, r_vol, hns, bcs, omega, ghost="implicit"):
    """One red and one black sweep, the library's right-hand side r_vol =
    vol * f; returns the new e."""
    u = np.asarray(e, float).copy()
    V = vol(hns)
    f = np.zeros_like(u)
    f[1:-1, 1:-1, 1:-1] = r_vol[1:-1, 1:-1, 1:-1] / V[1:-1, 1:-1, 1:-1]
    for pats in (RED, BLACK):
        for odd in pats:
            sor_pattern(u, f, hns, bcs, omega, odd, ghost)
    return u


def residual(e, r_vol, hns, bcs):
    """r_vol - vol * L e at interior points (L the two-gradient Laplacian,
    ghost values the homogeneous BC images)."""
    u = np.asarray(e, float).copy()
    for d in range(3):
        u = fill_ghosts(u, d, bcs[2 * d], bcs[2 * d + 1])
    W = [_weights(h) for h in hns]
    s = u.shape
    Le = np.zeros(s)
    c = u[1:-1, 1:-1, 1:-1]
    acc = np.zeros_like(c)
    for d in range(3):
        wm, wp, w0 = W[d]
        sh = [1, 1, 1]
        sh[d] = s[d] - 2
        wm_, wp_, w0_ = (w[2:-1].reshape(sh) for w in (wm, wp, w0))
        lo = [slice(1, -1)] * 3
        hi = [slice(1, -1)] * 3
        lo[d] = slice(0, -2)
        hi[d] = slice(2, None)
        acc = acc + (wm_ * u[tuple(lo)] + w0_ * c + wp_ * u[tuple(hi)])
    Le[1:-1, 1:-1, 1:-1] = acc
    out = np.zeros(s)
    V = vol(hns)
    out[1:-1, 1:-1, 1:-1] = r_vol[1:-1, 1:-1, 1:-1] - V[1:-1, 1:-1, 1:-1] * Le[1:-1, 1:-1, 1:-1]
    return out
