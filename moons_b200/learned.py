"""Training-loop shell of the learned preconditioner.

The network, its forward and backward passes and the Adam step run in the
library's CUDA kernels (``capi.UNet``); this module only drives them:

* ``ShellCase`` -- one draw of the sigma-shell Poisson case (sigma-weighted
  Laplacian, 10^U(-3,3) wall shell, RHS div(u x B), all-Neumann) on a shared
  mesh: coefficient fields, right-hand side, solvers;
* ``make_pairs`` -- (r, e) training pairs generated by the solver itself: the
  reference solution x* of each case (multigrid flexible CG to a tight
  tolerance) and iterates x_k of the reference's Jacobi-PCG; r is the
  solver's own residual at x_k (what a preconditioner is applied to) and
  e = x* - x_k (mean removed: the all-Neumann operator ignores constants);
  ``make_pairs_learned`` adds the iterates of the learned solve itself;
* ``train`` -- Adam epochs over the pairs, shuffled by PyTorch (the only
  PyTorch use: the data order), cosine learning-rate schedule; the default
  loss is the cosine in the energy norm of each case's own operator (the
  norm CG minimises), so the network is trained for what FCG needs;
* ``save`` / ``load`` -- the flat parameter array and the output scale.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from . import capi as G
from . import configs


def shell_mesh(n: int) -> G.Mesh:
    """The uniform unit-cube mesh of the sigma-shell case (n^3 cells)."""
    from . import mesh_gen as mg
    h = mg.add_ghost_nodes(mg.uniform(0.0, 1.0, n))
    return G.Mesh(h, h.copy(), h.copy())


@dataclass
class ShellCase:
    mesh: G.Mesh
    n: int
    shell: int
    seed: int
    k: List[G.Field] = field(default_factory=list)
    rhs: G.Field = None
    phi: G.Field = None
    op: G.PCG = None      # MG_MIXED solver: the reference solves and the loss's operator

    @classmethod
    def build(cls, mesh: G.Mesh, n: int, shell: int, seed: int) -> "ShellCase":
        _, sig, E = configs.sigma_shell(n, shell, seed)
        c = cls(mesh, n, shell, seed)
        es = []
        for d, dl in enumerate((G.FX, G.FY, G.FZ)):
            k = mesh.field(dl)
            k.upload(sig[d])
            c.k.append(k)
            e = mesh.field(dl)
            e.upload(E[d])
            es.append(e)
        c.rhs = mesh.field(G.CC)
        G.div(c.rhs, *es)
        c.phi = mesh.field(G.CC)
        c.phi.set_bcs(G.bc_spec([G.NEUMANN] * 6, all_neumann=True))
        c.op = c.solver(G.PREC_MG_MIXED)
        return c

    def solver(self, prec: int) -> G.PCG:
        return G.PCG(self.mesh, G.OP_LAP_PROPS, prec, [self.phi], [self.phi], self.k)


@dataclass
class Pair:
    r: G.Field
    e: G.Field
    case: int
    iterate: int


def _interior(a):
    return a[1:-1, 1:-1, 1:-1]


def make_pairs(cases: Sequence[ShellCase], iterates=(0, 2, 8, 32, 128), tol_ref: float = 1e-12) -> List[Pair]:
    """(r, e) pairs from the solver's own iterates (see the module text)."""
    pairs: List[Pair] = []
    for ci, c in enumerate(cases):
        ref = c.op
        c.phi.fill(0.0)
        ref.solve([c.phi], [c.rhs], G.isp(1000, tol_ref, 1e-300))
        xstar = c.phi.download()
        jac = c.solver(G.PREC_LAP)
        for k in iterates:
            c.phi.fill(0.0)
            if k > 0:
                jac.solve([c.phi], [c.rhs], G.isp(k, 1e-300, 1e-300))
            r = c.mesh.field(G.CC)
            ref.residual([c.phi], [c.rhs], [r])
            e = xstar - c.phi.download()
            e[1:-1, 1:-1, 1:-1] -= _interior(e).mean()
            e[0, :, :] = e[-1, :, :] = 0.0
            e[:, 0, :] = e[:, -1, :] = 0.0
            e[:, :, 0] = e[:, :, -1] = 0.0
            fe = c.mesh.field(G.CC)
            fe.upload(e)
            pairs.append(Pair(r, fe, ci, k))
        jac.close()
    return pairs


def make_pairs_learned(cases: Sequence[ShellCase], net: G.UNet, iterates=(1, 2, 4, 8, 16)) -> List[Pair]:
    """Pairs from the iterates of flexible CG with the current network
    (MOONS_PREC_UNET capped at k iterations): the residuals the learned solve
    itself meets, which the Jacobi iterates of make_pairs do not cover.  The
    reference solution of each case is recomputed with the multigrid solver."""
    pairs: List[Pair] = []
    for ci, c in enumerate(cases):
        c.phi.fill(0.0)
        c.op.solve([c.phi], [c.rhs], G.isp(1000, 1e-12, 1e-300))
        xstar = c.phi.download()
        fcg = c.solver(G.PREC_UNET)
        net.set_coeff(c.k)
        fcg.set_unet(net)
        for k in iterates:
            c.phi.fill(0.0)
            fcg.solve([c.phi], [c.rhs], G.isp(k, 1e-300, 1e-300))
            r = c.mesh.field(G.CC)
            c.op.residual([c.phi], [c.rhs], [r])
            e = xstar - c.phi.download()
            e[1:-1, 1:-1, 1:-1] -= _interior(e).mean()
            e[0, :, :] = e[-1, :, :] = 0.0
            e[:, 0, :] = e[:, -1, :] = 0.0
            e[:, :, 0] = e[:, :, -1] = 0.0
            fe = c.mesh.field(G.CC)
            fe.upload(e)
            pairs.append(Pair(r, fe, ci, 1000 + k))
        fcg.close()
    return pairs


def output_scale(pairs: Sequence[Pair]) -> float:
    """Median of rms(e) / rms(r) over the pairs: the network's output scale."""
    q = []
    for p in pairs:
        r = _interior(p.r.download())
        e = _interior(p.e.download())
        rr = math.sqrt(float((r * r).mean()))
        if rr > 0:
            q.append(math.sqrt(float((e * e).mean())) / rr)
    return float(np.median(q)) if q else 1.0


def train(net: G.UNet, cases: Sequence[ShellCase], pairs: Sequence[Pair], epochs: int = 4, lr: float = 1e-3,
          lr_min: float = 5e-5, seed: int = 0, loss: int = 2, log=None) -> List[float]:
    """Adam over the pairs for `epochs` passes; returns the mean loss of each
    epoch.  The data order is drawn by PyTorch (torch.randperm)."""
    import torch

    net.set_loss(loss)
    gen = torch.Generator().manual_seed(seed)
    steps = epochs * len(pairs)
    t = 0
    hist = []
    cur_case = -1
    for ep in range(epochs):
        order = torch.randperm(len(pairs), generator=gen).tolist()
        acc = 0.0
        for i in order:
            p = pairs[i]
            if p.case != cur_case:
                net.set_coeff(cases[p.case].k)
                if loss == 2:
                    net.set_operator(cases[p.case].op)
                cur_case = p.case
            a = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * t / max(1, steps)))
            acc += net.train_step(p.r, p.e, a)
            t += 1
        hist.append(acc / len(pairs))
        if log:
            log(f"epoch {ep}: mean loss {hist[-1]:.4f}")
    return hist


def save(net: G.UNet, path: str):
    np.savez_compressed(path, params=net.get_params(), out_scale=np.float64(net.out_scale))


def load(net: G.UNet, path: str):
    d = np.load(path)
    net.set_params(d["params"])
    net.out_scale = float(d["out_scale"])
