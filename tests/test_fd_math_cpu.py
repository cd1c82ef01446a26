"""The algebra of the direct Poisson solve (MOONS_PREC_FD) against the oracle,
on the CPU: the reference's LAP_UNIFORM PCG operator on a CC field is
separable, A = V (Lx (+) Ly (+) Lz), so the fast-diagonalization formula
x = (Bx (x) By (x) Bz) diag(1/(lx+ly+lz)) (Fx (x) Fy (x) Fz) b -- restated
here in numpy with the same per-axis operator the CUDA build assembles --
must reproduce the oracle's converged Jacobi-PCG solution of A x = b."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200 import mesh_gen as mg

N, D, P = G.NEUMANN, G.DIRICHLET, G.PERIODIC


def axis_operator(hn, tlo, thi):
    """1-D two-gradient second difference over the interior cells of one CC
    axis (node coordinates with ghosts), homogeneous BCs folded in."""
    hn = np.asarray(hn, dtype=np.float64)
    hc = 0.5 * (hn[1:] + hn[:-1])
    dhn = np.diff(hn)   # cell widths, cells 0..sc-1 (0 and sc-1 are ghosts)
    dhc = np.diff(hc)   # centre distances between cells t and t+1
    sc = len(hc)
    n = sc - 2
    L = np.zeros((n, n))
    for t in range(1, sc - 1):        # interior cell t (0-based with ghosts)
        a = t - 1
        cm = (-1.0 / dhc[t - 1]) * (-1.0 / dhn[t])
        cp = (1.0 / dhc[t]) * (1.0 / dhn[t])
        c0 = (1.0 / dhc[t - 1]) * (-1.0 / dhn[t]) + (-1.0 / dhc[t]) * (1.0 / dhn[t])
        L[a, a] += c0
        for nb, w in ((t - 1, cm), (t + 1, cp)):
            if nb in (0, sc - 1):
                ty = tlo if nb == 0 else thi
                if ty == P:
                    nb = sc - 2 if nb == 0 else 1
                elif ty == N:
                    nb = t
                else:
                    nb, w = t, -w
            L[a, nb - 1] += w
    return L, dhn[1:-1]


def fd_solve(hs, bcs, b):
    fac = []
    for d in range(3):
        L, v = axis_operator(hs[d], bcs[2 * d], bcs[2 * d + 1])
        sv = np.sqrt(v)
        M = sv[:, None] * L / sv[None, :]
        assert np.abs(M - M.T).max() <= 1e-10 * np.abs(M).max()
        w, W = np.linalg.eigh(0.5 * (M + M.T))
        z = int(np.argmin(np.abs(w))) if D not in (bcs[2 * d], bcs[2 * d + 1]) else -1
        fac.append((w, W.T / sv[None, :], W / sv[:, None], z))
    T = b
    for d in range(3):
        T = np.moveaxis(np.tensordot(fac[d][1], np.moveaxis(T, d, 0), axes=1), 0, d)
    lam = fac[0][0][:, None, None] + fac[1][0][None, :, None] + fac[2][0][None, None, :]
    zero = all(f[3] >= 0 for f in fac)
    if zero:
        lam[fac[0][3], fac[1][3], fac[2][3]] = np.inf
    T = T / lam
    for d in range(3):
        T = np.moveaxis(np.tensordot(fac[d][2], np.moveaxis(T, d, 0), axes=1), 0, d)
    return T, zero


CASES = [
    ((9, 7, 11), [N, N, N, N, N, N]),
    ((8, 10, 12), [N, N, N, N, P, P]),
    ((10, 6, 9), [D, D, N, N, N, D]),
    ((12, 9, 8), [P, P, D, N, P, P]),
]


@pytest.mark.parametrize("n,bcs", CASES)
def test_fast_diagonalization_reproduces_the_oracle_solution(n, bcs):
    hs = [mg.add_ghost_nodes(mg.roberts_both(0.0, 1.0, n[0], 1.05)),
          mg.add_ghost_nodes(mg.roberts_both(0.0, 1.5, n[1], 1.2)),
          mg.add_ghost_nodes(mg.uniform(0.0, 2.0, n[2]))]
    m = O.Mesh(*hs)
    p = m.field(G.CC)
    alln = D not in bcs
    p.set_bcs(G.bc_spec(bcs, all_neumann=alln))
    rhs = m.field(G.CC)
    b = np.random.default_rng(1).standard_normal(rhs.shape)
    rhs.upload(b)
    s = O.PCG(m, G.OP_LAP_UNIFORM, G.PREC_LAP, [p], [p])
    info = s.solve([p], [rhs], G.isp(20000, 1e-13, 1e-300))
    assert info["exit_reason"] == 1
    x_or = p.download()[1:-1, 1:-1, 1:-1]
    # the PCG solves vol * L x = the RHS it was given, with the reference's
    # modify_RHS (homogeneous BCs: the RHS as uploaded, times the volumes) and,
    # when singular, the RHS mean removed; the residual the oracle reaches is
    # that of A x = b_int with A = V (Lx + Ly + Lz)
    b_int = b[1:-1, 1:-1, 1:-1]
    vol = [np.diff(h)[1:-1] for h in hs]
    V = vol[0][:, None, None] * vol[1][None, :, None] * vol[2][None, None, :]
    rhs_fd = V * b_int
    if alln:
        rhs_fd = rhs_fd - V * (rhs_fd.sum() / V.sum())
    x_fd, zero = fd_solve(hs, bcs, rhs_fd)
    assert zero == alln
    if alln:
        x_fd = x_fd - x_fd.mean()
        x_or = x_or - x_or.mean()
    err = np.abs(x_fd - x_or).max() / np.abs(x_or).max()
    assert err < 1e-8, err
