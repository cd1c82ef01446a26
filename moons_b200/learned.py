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
* ``make_pairs_two_stage`` -- pairs of the learned + mixed form
  (MOONS_PREC_UNET_MG, z = V(r) + N(r - A V(r))): at each iterate x_k the
  network's input is what one FP32 V-cycle leaves, t = r(x_k + V(r_k)), and
  its target the remaining error e = x* - x_k - V(r_k); the iterates come
  from the reference's Jacobi-PCG and from multigrid flexible CG (the
  residuals the two-stage solve itself meets);
* ``train`` -- Adam epochs over the pairs, shuffled by PyTorch (the only
  PyTorch use: the data order), cosine learning-rate schedule; the default
  loss is the cosine in the energy norm of each case's own operator (the
  norm CG minimises), so the network is trained for what FCG needs;
  ``blocked=True`` shuffles the draws and the pairs within each draw and
  builds a draw's operator only while its pairs run (for pair sets of
  hundreds of draws, whose operators would not all stay resident);
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

    def release(self, rhs: bool = True):
        """Free the operator's solver (rebuilt on demand by operator()) and,
        with `rhs`, the right-hand side, keeping what training reads (the
        coefficient fields and phi, whose BCs define the operator)."""
        if self.op is not None:
            self.op.close()
            self.op = None
        if rhs and self.rhs is not None:
            self.rhs.close()
            self.rhs = None

    def operator(self) -> G.PCG:
        if self.op is None:
            self.op = self.solver(G.PREC_MG_MIXED)
        return self.op


@dataclass
class UniformCase:
    """One draw of a constant-coefficient Poisson problem (the pressure or
    B-form cleaning-potential operator, LAP_UNIFORM) on a given mesh with
    given BCs: the right-hand side is the divergence of i.i.d. N(0,1) face
    values (seeded).  Same surface as ShellCase (k is empty: the network's
    coefficient feature stays 0, the value of a unit coefficient)."""
    mesh: G.Mesh
    bcs: object
    seed: int
    k: List[G.Field] = field(default_factory=list)
    rhs: G.Field = None
    phi: G.Field = None
    op: G.PCG = None

    @classmethod
    def build(cls, mesh: G.Mesh, bcs, seed: int) -> "UniformCase":
        rng = np.random.default_rng(seed)
        c = cls(mesh, bcs, seed)
        es = []
        for dl in (G.FX, G.FY, G.FZ):
            f = mesh.field(dl)
            f.upload(rng.standard_normal(f.shape))
            es.append(f)
        c.rhs = mesh.field(G.CC)
        G.div(c.rhs, *es)
        c.phi = mesh.field(G.CC)
        c.phi.set_bcs(bcs)
        c.op = c.solver(G.PREC_MG_MIXED)
        return c

    def solver(self, prec: int) -> G.PCG:
        return G.PCG(self.mesh, G.OP_LAP_UNIFORM, prec, [self.phi], [self.phi])

    release = ShellCase.release
    operator = ShellCase.operator


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


def _zero_ghosts(a):
    a[0, :, :] = a[-1, :, :] = 0.0
    a[:, 0, :] = a[:, -1, :] = 0.0
    a[:, :, 0] = a[:, :, -1] = 0.0
    return a


def make_pairs_two_stage(cases: Sequence[ShellCase], jacobi=(0, 8, 64), fcg=(1, 2, 3, 4, 5),
                         tol_ref: float = 1e-12, release: bool = False) -> List[Pair]:
    """(t, e) pairs of the learned + mixed form (see the module text): for
    each iterate x_k -- of the reference's Jacobi-PCG capped at k iterations
    (`jacobi`) and of multigrid flexible CG capped at k (`fcg`) -- the
    residual r_k, one FP32 V-cycle v = V(r_k) (moons_pcg_apply_prec), the
    network's input t = r(x_k + v) and its target e = x* - x_k - v (mean
    removed).  `release` frees each draw's solver and right-hand side once
    its pairs are made."""
    pairs: List[Pair] = []
    for ci, c in enumerate(cases):
        op = c.operator()
        c.phi.fill(0.0)
        op.solve([c.phi], [c.rhs], G.isp(1000, tol_ref, 1e-300))
        xstar = c.phi.download()
        iterates = []
        jac = c.solver(G.PREC_LAP)
        for k in jacobi:
            c.phi.fill(0.0)
            if k > 0:
                jac.solve([c.phi], [c.rhs], G.isp(k, 1e-300, 1e-300))
            iterates.append((k, c.phi.download()))
        jac.close()
        for k in fcg:
            c.phi.fill(0.0)
            op.solve([c.phi], [c.rhs], G.isp(k, 1e-300, 1e-300))
            iterates.append((1000 + k, c.phi.download()))
        r = c.mesh.field(G.CC)
        v = c.mesh.field(G.CC)
        for k, xk in iterates:
            c.phi.upload(xk)
            op.residual([c.phi], [c.rhs], [r])
            op.apply_prec([v], [r])
            x1 = xk + _zero_ghosts(v.download())
            c.phi.upload(x1)
            t = c.mesh.field(G.CC)
            op.residual([c.phi], [c.rhs], [t])
            e = xstar - x1
            e[1:-1, 1:-1, 1:-1] -= _interior(e).mean()
            fe = c.mesh.field(G.CC)
            fe.upload(_zero_ghosts(e))
            pairs.append(Pair(t, fe, ci, k))
        r.close()
        v.close()
        if release:
            c.release()
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


def _blocked_order(pairs: Sequence[Pair], gen) -> List[int]:
    import torch

    by_case = {}
    for i, p in enumerate(pairs):
        by_case.setdefault(p.case, []).append(i)
    keys = sorted(by_case)
    order = []
    for kc in torch.randperm(len(keys), generator=gen).tolist():
        idx = by_case[keys[kc]]
        order += [idx[j] for j in torch.randperm(len(idx), generator=gen).tolist()]
    return order


def train(net: G.UNet, cases: Sequence[ShellCase], pairs: Sequence[Pair], epochs: int = 4, lr: float = 1e-3,
          lr_min: float = 5e-5, seed: int = 0, loss: int = 2, log=None, blocked: bool = False) -> List[float]:
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
        order = _blocked_order(pairs, gen) if blocked else torch.randperm(len(pairs), generator=gen).tolist()
        acc = 0.0
        for i in order:
            p = pairs[i]
            if p.case != cur_case:
                if blocked and cur_case >= 0:
                    cases[cur_case].release(rhs=False)
                if cases[p.case].k:
                    net.set_coeff(cases[p.case].k)
                if loss == 2:
                    net.set_operator(cases[p.case].operator())
                cur_case = p.case
            a = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * t / max(1, steps)))
            acc += net.train_step(p.r, p.e, a)
            t += 1
        hist.append(acc / len(pairs))
        if blocked and cur_case >= 0:
            cases[cur_case].release(rhs=False)
            cur_case = -1
        if log:
            log(f"epoch {ep}: mean loss {hist[-1]:.4f}")
    return hist


def save(net: G.UNet, path: str, meta: dict | None = None):
    import json
    np.savez_compressed(path, params=net.get_params(), out_scale=np.float64(net.out_scale),
                        meta=np.array(json.dumps(meta or {})))


def load(net: G.UNet, path: str) -> dict:
    import json
    d = np.load(path)
    net.set_params(d["params"])
    net.out_scale = float(d["out_scale"])
    return json.loads(str(d["meta"])) if "meta" in d else {}


def train_two_stage(n: int = 128, shell: int = 4, draws: int = 250, epochs: int = 8, lr: float = 1e-3,
                    lr_min: float = 5e-5, seed: int = 0, log=None):
    """The learned + mixed network of the sigma-shell case: `draws` seeded
    draws (seeds 0 .. draws-1; held-out evaluation uses seeds from 1000), 8
    pairs each (Jacobi-PCG iterates 0, 8, 64 and multigrid-FCG iterates 1-5),
    Adam with the energy-norm cosine loss in blocked order.  Returns the
    network, its mesh and a summary."""
    import time
    mesh = shell_mesh(n)
    t0 = time.perf_counter()
    cases, pairs = [], []
    for s in range(draws):
        c = ShellCase.build(mesh, n, shell, s)
        ps = make_pairs_two_stage([c], release=True)   # keeps the coefficient fields and phi only
        for p in ps:
            p.case = s
        cases.append(c)
        pairs += ps
        if log and (s + 1) % 25 == 0:
            log(f"pairs: {s + 1} draws, {len(pairs)} pairs, {time.perf_counter() - t0:.0f} s")
    t1 = time.perf_counter()
    net = G.UNet(mesh, seed=seed)
    net.out_scale = output_scale(pairs)
    hist = train(net, cases, pairs, epochs=epochs, lr=lr, lr_min=lr_min, seed=seed, blocked=True, log=log)
    t2 = time.perf_counter()
    meta = {"n": n, "shell": shell, "draws": draws, "pairs": len(pairs), "epochs": epochs,
            "adam_steps": epochs * len(pairs), "loss": "energy-norm cosine (kind 2)",
            "loss_first_last": [hist[0], hist[-1]], "data_seconds": t1 - t0, "train_seconds": t2 - t1,
            "out_scale": net.out_scale}
    return net, mesh, meta


def train_two_stage_uniform(mesh: G.Mesh, bcs, draws: int = 25, epochs: int = 8, lr: float = 1e-3,
                            lr_min: float = 5e-5, seed: int = 0, seed0: int = 0, log=None):
    """The learned + mixed network of constant-coefficient solves (pressure
    and cleaning potential) on `mesh`: `draws` seeded right-hand sides (seeds
    seed0 ..), draw i with the BCs bcs[i % len(bcs)] (one BC set or a list),
    8 two-stage pairs each, Adam with the energy-norm cosine loss in blocked
    order.  Returns (net, summary)."""
    import time
    bl = list(bcs) if isinstance(bcs, (list, tuple)) else [bcs]
    t0 = time.perf_counter()
    cases, pairs = [], []
    for i in range(draws):
        c = UniformCase.build(mesh, bl[i % len(bl)], seed0 + i)
        ps = make_pairs_two_stage([c], release=True)
        for p in ps:
            p.case = i
        cases.append(c)
        pairs += ps
    t1 = time.perf_counter()
    net = G.UNet(mesh, seed=seed)
    net.out_scale = output_scale(pairs)
    hist = train(net, cases, pairs, epochs=epochs, lr=lr, lr_min=lr_min, seed=seed, blocked=True, log=log)
    t2 = time.perf_counter()
    meta = {"draws": draws, "pairs": len(pairs), "epochs": epochs, "adam_steps": epochs * len(pairs),
            "loss": "energy-norm cosine (kind 2)", "loss_first_last": [hist[0], hist[-1]],
            "data_seconds": t1 - t0, "train_seconds": t2 - t1, "out_scale": net.out_scale}
    return net, meta


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="train the learned + mixed (two-stage) network on the "
                                             "sigma-shell case and save its weights")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--shell", type=int, default=4)
    ap.add_argument("--draws", type=int, default=250)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--case", choices=["shell", "at_scale"], default="shell",
                    help="shell: the sigma-shell case (--n, --shell); at_scale: the pressure and cleaning-potential "
                         "solves of the 128 x 128 x 256 finite-Rem duct (its pressure and potential BCs alternate)")
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    log_ = lambda s: print(s, flush=True)
    if a.case == "shell":
        net_, _, meta_ = train_two_stage(a.n, a.shell, a.draws, a.epochs, log=log_)
    else:
        mom_, _, prm_, _ = configs.at_scale()
        mesh_ = G.Mesh(*mom_)
        net_, meta_ = train_two_stage_uniform(mesh_, [prm_.bc_p, prm_.bc_phi], draws=a.draws, epochs=a.epochs,
                                              log=log_)
        meta_["case"] = "at_scale 128x128x256, pressure and cleaning-potential BCs"
    save(net_, a.out, meta_)
    print(meta_, flush=True)
