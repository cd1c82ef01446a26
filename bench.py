#!/usr/bin/env python
"""Benchmark of the MOONS MHD time step on B200.

Workload (default): the fully developed MHD duct -- 64x64x256 fluid cells,
Roberts two-sided clustering (beta=1.05) across, periodic streamwise, mean
pressure gradient, Ha=100, Re=1000, B along y, a 4-cell conducting wall
layer (sigma=0.01) in the induction mesh, dt=5e-4, every PCG solve to a
relative residual of 1e-10.  A "step" is one full solve_MOONS step
(momentum + induction, four PCG solves).

Metric: steps/s (whole job; N GPUs run N independent replicas -- the path
does not shard) plus the pressure-Poisson time to 1e-10 on the same mesh.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl moons|reference]

The reference arm times the CPU restatement of the reference algorithm
(the oracle port) on the host, on a bounded sample scaled to the metric.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s & Poisson ms to 1e-10 residual: learned+mixed vs plain FP64 on one B200"
WORKLOAD = "MHD duct 64x64x256 fluid (+4-cell sigma=0.01 wall layer), Roberts beta=1.05, Ha=100, Re=1000, dt=5e-4"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="moons", choices=["moons", "reference"])
    ap.add_argument("--small", action="store_true", help="small mesh (debug only)")
    ap.add_argument("--profile", choices=["step", "jacobi", "mg", "mixed", "fd", "unet", "unet_train"], default=None,
                    help="profiling run for ncu launch lists: one duct step, one duct pressure solve with the "
                         "given preconditioner capped at --profile-iters iterations, or --profile-iters U-Net "
                         "forward applies / training steps on the 128^3 sigma-shell grid; prints what ran, no "
                         "bench line")
    ap.add_argument("--profile-iters", type=int, default=40)
    ap.add_argument("--leg", choices=["at_scale"], default=None,
                    help="run one leg alone and print its JSON (no bench line): at_scale = configuration 5 with "
                         "--leg-steps steps per variant")
    ap.add_argument("--leg-steps", type=int, default=200)
    ap.add_argument("--profile-mesh", choices=["duct", "at_scale", "shell"], default="duct",
                    help="mesh of the --profile Poisson solve: the duct fluid mesh (64x64x256), the "
                         "configuration-5 mesh (128x128x256, working set above the L2) or the 128^3 "
                         "sigma-shell case (sigma-weighted operator)")
    return ap.parse_args()


def run_profile(args):
    from moons_b200 import capi as G, configs
    kw = duct_kw(args.small)
    if args.profile == "step":
        sim = configs.make(G, configs.duct, seed=0, **kw)
        info = sim.step(1)
        print(json.dumps({"profile": "step", "workload": WORKLOAD, "info": info}), flush=True)
        return
    if args.profile in ("unet", "unet_train"):
        # U-Net forward applies (or training steps) on the sigma-shell grid
        from moons_b200 import learned as L
        n = 32 if args.small else 128
        mesh = L.shell_mesh(n)
        case = L.ShellCase.build(mesh, n, 2 if args.small else 4, 0)
        net = G.UNet(mesh, seed=0)
        net.set_coeff(case.k)
        r = mesh.field(G.CC)
        case.phi.fill(0.0)
        case.op.residual([case.phi], [case.rhs], [r])
        z = mesh.field(G.CC)
        if args.profile == "unet_train":
            net.set_operator(case.op)
            net.set_loss(2)
        for _ in range(args.profile_iters):
            if args.profile == "unet":
                net.apply(z, r)
            else:
                net.train_step(r, r, 1e-4)
        print(json.dumps({"profile": args.profile, "workload": f"U-Net {n}^3", "iters": args.profile_iters}),
              flush=True)
        return
    prec = {"jacobi": G.PREC_LAP, "mg": G.PREC_MG, "mixed": G.PREC_MG_MIXED, "fd": G.PREC_FD}[args.profile]
    if args.profile_mesh == "shell":
        # the sigma-weighted Poisson case (128^3, 4-cell shell, seed 0)
        from moons_b200 import learned as L
        n = 32 if args.small else 128
        case = L.ShellCase.build(L.shell_mesh(n), n, 2 if args.small else 4, 0)
        s = case.solver(prec)
        case.phi.fill(0.0)
        info = s.solve([case.phi], [case.rhs], G.isp(args.profile_iters, 1e-10, 1e-300))
        print(json.dumps({"profile": args.profile, "workload": f"sigma-shell Poisson {n}^3", "info": info}),
              flush=True)
        return
    mom, _, prm, _ = (configs.at_scale(**at_scale_kw(args.small)) if args.profile_mesh == "at_scale"
                      else configs.duct(**kw))
    m = G.Mesh(*mom)
    p = m.field(G.CC)
    p.set_bcs(prm.bc_p)
    b = m.field(G.CC)
    b.upload(np.random.default_rng(7).standard_normal(b.shape))
    s = G.PCG(m, G.OP_LAP_UNIFORM, prec, [p], [p])
    info = s.solve([p], [b], G.isp(args.profile_iters, 1e-10, 1e-300))
    print(json.dumps({"profile": args.profile, "workload": "duct pressure Poisson " + str(list(b.shape)),
                      "info": info}), flush=True)


def duct_kw(small):
    if small:
        return dict(nx=16, ny=16, nz=32)
    return dict(nx=64, ny=64, nz=256)


def at_scale_kw(small):
    """Configuration 5's mesh: 256 streamwise (z) x 128 x 128 cells."""
    return dict(nx=16, ny=16, nz=32) if small else {}


class Clocks:
    """Samples nvidia-smi during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.p = None
        self.out = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is None:
            return
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.out.append(parts)

    def summary(self):
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(p[1]) for p in self.out if p[1].replace(".", "").isdigit()]
        smax = [float(p[2]) for p in self.out if p[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for p in self.out for i in range(4) if p[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.out)}


def dist_setup(n, backend=None):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo for CPU tests.
    Ranks are independent replicas: the only collectives are the barrier and
    the max-over-ranks of the timings."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        return rank, world, local, dist
    return rank, world, local, None


def max_over_ranks(v, dist):
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, steps, ms_max):
    """Whole-job steps/s of `world` independent replicas (weak scaling)."""
    return world * steps / (ms_max / 1e3)


def poisson_ms(G, kw, prec=None, builder=None):
    """Pressure-Poisson time to 1e-10 on the duct fluid mesh, or the mesh of
    ``builder`` (random RHS), best of 3 solves from x = 0, with the given
    preconditioner (default the reference's Jacobi prec_Lap)."""
    from moons_b200 import configs
    mom, _, prm, _ = (builder or configs.duct)(**kw)
    m = G.Mesh(*mom)
    p = m.field(G.CC)
    p.set_bcs(prm.bc_p)
    b = m.field(G.CC)
    b.upload(np.random.default_rng(7).standard_normal(b.shape))
    s = G.PCG(m, G.OP_LAP_UNIFORM, G.PREC_LAP if prec is None else prec, [p], [p])
    best = None
    for _ in range(3):
        p.fill(0.0)
        info = s.solve([p], [b], G.isp(200000, 1e-10, 1e-300))
        if best is None or info["ms"] < best["ms"]:
            best = info
    s.close()
    return best, b.n


def vcycle_roofline(G, n=128, shell=4, reps=20, peak=None):
    """One V(2,2) cycle on the 128^3 sigma-shell case (seed 0), FP64 and
    FP32, applied through moons_pcg_apply_prec (separate launches, the call
    synchronises its stream): mean time over `reps` calls after 3 warm-up
    calls, and the algorithmic bytes of a V(nu1, nu2) cycle, (32 (nu1 + nu2)
    + 58) * 8/7 B per finest cell in FP64 and half that in FP32, over it."""
    from moons_b200 import learned as L
    mesh = L.shell_mesh(n)
    case = L.ShellCase.build(mesh, n, shell, 0)
    cells = n ** 3
    out = {}
    for name, prec, bpc in (("fp64", G.PREC_MG, (32 * 4 + 58) * 8.0 / 7.0),
                            ("fp32", G.PREC_MG_MIXED, (32 * 4 + 58) * 4.0 / 7.0)):
        s = case.solver(prec)
        r, z = mesh.field(G.CC), mesh.field(G.CC)
        case.phi.fill(0.0)
        s.residual([case.phi], [case.rhs], [r])
        for _ in range(3):
            s.apply_prec([z], [r])
        t0 = time.perf_counter()
        for _ in range(reps):
            s.apply_prec([z], [r])
        sec = (time.perf_counter() - t0) / reps
        gbs = bpc * cells / sec / 1e9
        out[name] = {"us_per_vcycle": sec * 1e6, "alg_bytes_per_cell": bpc, "achieved_gbs": gbs,
                     "frac": gbs / peak if peak else None}
        s.close()
    out["note"] = ("host-timed single V-cycles (launch latency included; inside the CUDA-graph solve the same "
                   "kernels run under dependent launch); the coarse levels are latency-bound in both precisions")
    return out


def sigma_shell_poisson(G, n=128, shell=4, seeds_plain=4, seeds_mg=64):
    """Mixed-precision Poisson case: div(sigma grad phi) = div(u x B) on a
    128^3 grid with a 10^U(-3,3) wall shell, to 1e-10 relative residual.
    Mean solve time of the reference's Jacobi-PCG (FP64) over `seeds_plain`
    seeds, and of multigrid-CG (FP64 V-cycle) and flexible CG with an FP32
    V-cycle over `seeds_mg` seeds; error of the mixed solution against the
    FP64 multigrid one (constant removed, all-Neumann)."""
    from moons_b200 import configs
    out = {}
    err = None
    for name, prec, ns in (("plain_fp64_jacobi", G.PREC_LAP, seeds_plain), ("mg_fp64", G.PREC_MG, seeds_mg),
                           ("mixed_fp32_vcycle", G.PREC_MG_MIXED, seeds_mg)):
        ms, its, rel = [], [], []
        for seed in range(ns):
            coords, sig, E = configs.sigma_shell(n, shell, seed)
            m = G.Mesh(*coords)
            phi = m.field(G.CC)
            phi.set_bcs(G.bc_spec([G.NEUMANN] * 6, all_neumann=True))
            ks, es = [], []
            for d, dl in enumerate((G.FX, G.FY, G.FZ)):
                k = m.field(dl)
                k.upload(sig[d])
                ks.append(k)
                e = m.field(dl)
                e.upload(E[d])
                es.append(e)
            rhs = m.field(G.CC)
            G.div(rhs, *es)
            s = G.PCG(m, G.OP_LAP_PROPS, prec, [phi], [phi], ks)
            par = G.isp(400000, 1e-10, 1e-300)
            phi.fill(0.0)
            s.solve([phi], [rhs], par)  # warm-up (graph build)
            phi.fill(0.0)
            info = s.solve([phi], [rhs], par)
            ms.append(info["ms"])
            its.append(info["iterations"])
            rel.append(info["rel"])
            if seed == 0 and name != "plain_fp64_jacobi":
                x = phi.download()[1:-1, 1:-1, 1:-1]
                x = x - x.mean()
                if name == "mg_fp64":
                    ref0 = x
                else:
                    err = float(np.abs(x - ref0).max() / np.abs(ref0).max())
            s.close()
        out[name] = {"ms_mean": float(np.mean(ms)), "iterations_mean": float(np.mean(its)),
                     "rel_max": float(np.max(rel)), "seeds": ns}
    out["speedup_mixed_vs_plain"] = out["plain_fp64_jacobi"]["ms_mean"] / out["mixed_fp32_vcycle"]["ms_mean"]
    out["speedup_mixed_vs_mg_fp64"] = out["mg_fp64"]["ms_mean"] / out["mixed_fp32_vcycle"]["ms_mean"]
    out["mixed_vs_fp64_solution_max_rel_err_seed0"] = err
    out["workload"] = f"sigma-weighted Poisson {n}^3 cells, 4-cell wall shell sigma=10^U(-3,3), RHS div(u x B)"
    return out


def unet_flops(n):
    """Algorithmic FLOPs of one U-Net forward on an n^3 grid: 2 * 27 * Cin *
    Cout per voxel and 3x3x3 convolution (real input channels; the head and
    the pooling are negligible)."""
    layers = [(2, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 128, 3),
              (128, 128, 3), (192, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]
    return sum(2 * 27 * ci * co * (n >> lv) ** 3 for ci, co, lv in layers)


def bf16_peak() -> float:
    """Dense bf16 TFLOP/s measured on this pool (burst), else the fallback."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
    except Exception:
        return 1590.0


WEIGHTS_TWO_STAGE = os.path.join(ROOT, "moons_b200", "weights", "unet_two_stage_shell128.npz")


def learned_mixed_poisson(G, n=128, shell=4, held=tuple(range(1000, 1064)), train_draws=8, epochs=8,
                          weights=WEIGHTS_TWO_STAGE):
    """Configuration 4, the learned + mixed form: flexible CG with the
    two-stage preconditioner z = V(r) + gamma N(r - A V(r)) (V the FP32
    V-cycle, N the U-Net, gamma its energy-optimal multiple), against
    flexible CG with V alone and CG with the FP64 V-cycle, to 1e-10 on
    held-out seeds.  The network is the committed one trained at the case's
    scale (moons_b200/learned.py, 250 draws / 2000 pairs) when its weights
    file is present; otherwise it is trained here on `train_draws` draws.
    A short training run is always timed (Adam steps on the GPU) so that
    the training cost is on record."""
    from moons_b200 import learned as L
    import torch
    mesh = L.shell_mesh(n)
    # training: a short run here (its cost), the full-scale weights if committed
    t0 = time.perf_counter()
    cases = []
    pairs = []
    for s in range(train_draws):
        c = L.ShellCase.build(mesh, n, shell, s)
        ps = L.make_pairs_two_stage([c], release=True)
        for q in ps:
            q.case = s
        cases.append(c)
        pairs += ps
    net = G.UNet(mesh, seed=0)
    net.out_scale = L.output_scale(pairs)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    hist = L.train(net, cases, pairs, epochs=epochs, lr=1e-3, lr_min=5e-5, blocked=True)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    short = {"draws": train_draws, "pairs": len(pairs), "adam_steps": epochs * len(pairs), "seconds": t_train,
             "ms_per_step": t_train / max(epochs * len(pairs), 1) * 1e3, "data_seconds": t1 - t0,
             "loss_first_last": [hist[0], hist[-1]], "loss": "energy-norm cosine (kind 2)"}
    # U-Net forward rate (host-synchronised applies on one input)
    z = mesh.field(G.CC)
    net.set_coeff(cases[0].k)
    for _ in range(3):
        net.apply(z, pairs[0].r)
    t2 = time.perf_counter()
    for _ in range(10):
        net.apply(z, pairs[0].r)
    fwd_ms = (time.perf_counter() - t2) / 10 * 1e3
    fl = unet_flops(n)
    del pairs, cases, z
    source = "trained here (short run)"
    meta = short
    if weights and os.path.exists(weights):
        meta = L.load(net, weights)
        source = "committed weights " + os.path.relpath(weights, ROOT)

    def solve(case, prec):
        s = case.solver(prec)
        if prec == G.PREC_UNET_MG:
            net.set_coeff(case.k)
            s.set_unet(net)
        par = G.isp(20000, 1e-10, 1e-300)
        case.phi.fill(0.0)
        s.solve([case.phi], [case.rhs], par)  # warm-up (graph build)
        case.phi.fill(0.0)
        info = s.solve([case.phi], [case.rhs], par)
        x = case.phi.download()[1:-1, 1:-1, 1:-1]
        s.close()
        return info, x - x.mean()

    names = (("cg_fp64_mg", G.PREC_MG), ("fcg_v", G.PREC_MG_MIXED), ("fcg_v_plus_n", G.PREC_UNET_MG))
    rows = []
    for sd in held:
        c = L.ShellCase.build(mesh, n, shell, sd)
        c.release(rhs=False)
        row = {"seed": sd}
        ref = None
        for name, prec in names:
            info, x = solve(c, prec)
            if ref is None:
                ref = x
            row[name] = {"ms": info["ms"], "iterations": info["iterations"], "exit_reason": info["exit_reason"],
                         "rel": info["rel"], "err_vs_fp64_mg": float(np.abs(x - ref).max() / np.abs(ref).max())}
        rows.append(row)
        del c
    summ = {}
    for name, _ in names:
        ms = [r[name]["ms"] for r in rows]
        it = [r[name]["iterations"] for r in rows]
        summ[name] = {"ms_mean": float(np.mean(ms)), "ms_min": float(np.min(ms)), "ms_max": float(np.max(ms)),
                      "iterations_mean": float(np.mean(it)), "iterations_max": int(np.max(it)),
                      "converged": sum(1 for r in rows if r[name]["exit_reason"] == 1),
                      "err_vs_fp64_mg_max": float(np.max([r[name]["err_vs_fp64_mg"] for r in rows]))}
    base = summ["cg_fp64_mg"]["ms_mean"]
    return {
        "workload": f"sigma-weighted Poisson {n}^3, {shell}-cell wall shell sigma=10^U(-3,3), RHS div(u x B), "
                    f"to 1e-10 relative residual; {len(held)} held-out seeds {held[0]}..{held[-1]}",
        "network": {"source": source, "training": meta, "short_training_run": short},
        "ablation": summ,
        "speedup_vs_cg_fp64_mg": {k: base / v["ms_mean"] for k, v in summ.items()},
        "gate_3x_vs_fp64_mg": {"met": base / summ["fcg_v_plus_n"]["ms_mean"] >= 3.0,
                               "measured": base / summ["fcg_v_plus_n"]["ms_mean"]},
        "per_seed": rows[:4],
        "unet_forward": {"ms_host_synced": fwd_ms, "gflop": fl / 1e9, "tflops": fl / (fwd_ms / 1e3) / 1e12,
                         "frac_of_measured_bf16": fl / (fwd_ms / 1e3) / 1e12 / bf16_peak()},
        "note": "fcg_v_plus_n: z = V(r) + gamma N(r - A V(r)) in FP64 flexible CG; exit_reason 11 means the "
                "learned phase stagnated and the FP32 V-cycle finished the solve (ms include both phases)",
    }


WEIGHTS_AT_SCALE = os.path.join(ROOT, "moons_b200", "weights", "unet_two_stage_at_scale.npz")


def at_scale_steps(G, small=False, steps=3, weights=WEIGHTS_AT_SCALE):
    """Configuration 5: the finite-Rem (constrained transport) MHD step on
    256 x 128 x 128 cells, plain FP64 Jacobi-PCG Poisson solves vs FP32
    V-cycle flexible CG vs the direct fast-diagonalization solve in CG vs the
    learned + mixed two-stage preconditioner in flexible CG;
    div(B) after every step, and the runs' fields against the plain one's
    after the last step (same seed, same tolerances)."""
    from moons_b200 import configs
    from moons_b200 import learned as L
    kw = dict(nx=16, ny=16, nz=32) if small else {}
    out, fields = {}, {}
    for name, prec in (("plain_fp64", 0), ("mixed_fp32_vcycle", G.PREC_MG_MIXED), ("fd_direct", G.PREC_FD),
                       ("learned_mixed", G.PREC_UNET_MG)):
        extra = {}
        if prec == G.PREC_UNET_MG:
            # one network for the pressure and the cleaning potential (same mesh):
            # the committed one when present, else trained here on seeded draws
            mom, _, prm, _ = configs.at_scale(**kw)
            mm = G.Mesh(*mom)
            if weights and os.path.exists(weights) and not small:
                net = G.UNet(mm, seed=0)
                meta = L.load(net, weights)
                meta["source"] = "committed weights " + os.path.relpath(weights, ROOT)
            else:
                net, meta = L.train_two_stage_uniform(mm, [prm.bc_p, prm.bc_phi], draws=4 if small else 16,
                                                      epochs=2 if small else 6)
                meta["source"] = "trained here"
            out["learned_mixed_network"] = meta
            extra = dict(meshes=(mm, mm), unets=(net, net))
        sim = configs.make(G, configs.at_scale, seed=0, prec_poisson=prec, **kw, **extra)
        sim.step(1)  # warm-up (graphs)
        divb, ms, its = [], 0.0, {}
        for _ in range(steps):
            info = sim.step(1)
            ms += info["ms"]
            for k in ("iters_U", "iters_p", "iters_B", "iters_phi"):
                its[k] = its.get(k, 0) + info[k] / steps
            divb.append(sim.divergence()[1])
        fields[name] = [sim.download(G.MHD_U, c) for c in range(3)] + [sim.download(G.MHD_B, c) for c in range(3)]
        out[name] = {"steps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps, "iters_per_step": its,
                     "div_B_l2sq_max": max(divb)}
        del sim
    rel = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
              for a, b in zip(fields["mixed_fp32_vcycle"], fields["plain_fp64"]))
    out["mixed_vs_plain_fields_max_rel_l2"] = rel
    out["speedup_mixed_vs_plain"] = out["plain_fp64"]["ms_per_step"] / out["mixed_fp32_vcycle"]["ms_per_step"]
    out["speedup_fd_vs_plain"] = out["plain_fp64"]["ms_per_step"] / out["fd_direct"]["ms_per_step"]
    out["fd_vs_plain_fields_max_rel_l2"] = max(
        float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)) for a, b in zip(fields["fd_direct"], fields["plain_fp64"]))
    out["learned_mixed_vs_plain_fields_max_rel_l2"] = max(
        float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        for a, b in zip(fields["learned_mixed"], fields["plain_fp64"]))
    out["speedup_learned_mixed_vs_plain"] = out["plain_fp64"]["ms_per_step"] / out["learned_mixed"]["ms_per_step"]
    n = kw.get("nx", 128), kw.get("ny", 128), kw.get("nz", 256)
    out["workload"] = (f"finite-Rem MHD with constrained transport, {n[0]}x{n[1]}x{n[2]} cells as (x, y, z): x and y "
                       f"the Roberts-stretched cross-section, z the uniform streamwise axis (the case's 256 x 128 x 128 "
                       f"lists the streamwise axis first), Re=1000, Ha=500, Rem=10, dt=2e-4; {steps} steps after 1 "
                       f"warm-up step" + ("" if steps >= 200 else " (the case's 200 steps shortened to keep the bench "
                                                                  "within minutes; bench.py --leg at_scale runs 200)"))
    return out


def full_bc_steps(G, small=False, steps=5, steps_tol=2):
    """The reference's full_BC case: lid-driven MHD cavity on the mesh bank's
    full_BC_w_vacuum_3D meshes (fluid 80 x 85 x 80, induction mesh with
    walls and vacuum 140 x 127 x 140), Re = 2000, Ha = 100, Rem = 2000,
    dt = 2.5e-3.  Two settings: the case's own PCG limits (U 5, p 20, B 20,
    phi 20 iterations at tol_rel 1e-6), and the same tolerance without the
    iteration caps; each with plain FP64 Jacobi-PCG, with FP32 V-cycle and
    with direct fast-diagonalization Poisson solves."""
    from moons_b200 import configs
    kw = dict(N=12, N_w=3) if small else {}
    out = {}
    for setting, extra, nst in (("case_caps", {}, steps), ("to_tol_1e-6", dict(iter_max=(20000,) * 4), steps_tol)):
        res = {}
        for name, prec in (("plain_fp64", 0), ("mixed_fp32_vcycle", G.PREC_MG_MIXED), ("fd_direct", G.PREC_FD)):
            sim = configs.make(G, configs.full_bc, seed=0, prec_poisson=prec, **kw, **extra)
            sim.step(1)  # warm-up (graphs)
            ms, its, divb = 0.0, {}, []
            for _ in range(nst):
                info = sim.step(1)
                ms += info["ms"]
                for k in ("iters_U", "iters_p", "iters_B", "iters_phi"):
                    its[k] = its.get(k, 0) + info[k] / nst
                divb.append(sim.divergence()[1])
            res[name] = {"steps_per_s": nst / (ms / 1e3), "ms_per_step": ms / nst, "iters_per_step": its,
                         "res_p_last": info["res_p"], "res_phi_last": info["res_phi"], "div_B_l2sq_max": max(divb)}
            sm, si = sim.shape(G.MHD_U, 0), sim.shape(G.MHD_B, 0)
            del sim
        res["speedup_mixed_vs_plain"] = res["plain_fp64"]["ms_per_step"] / res["mixed_fp32_vcycle"]["ms_per_step"]
        res["speedup_fd_vs_plain"] = res["plain_fp64"]["ms_per_step"] / res["fd_direct"]["ms_per_step"]
        res["steps"] = nst
        out[setting] = res
    out["workload"] = (f"full_BC case (mesh bank full_BC_w_vacuum_3D): fluid {sm[0] - 3}x{sm[1] - 2}x{sm[2] - 2} "
                       f"cells in an induction mesh of {si[0] - 3}x{si[1] - 2}x{si[2] - 2} (walls sigma=1, vacuum "
                       f"sigma=1e-3), Re=2000, Ha=100, Rem=2000, dt=2.5e-3; case_caps: the case's PCG limits "
                       f"U5/p20/B20/phi20 at tol 1e-6; to_tol_1e-6: the same tolerance without caps; timed steps "
                       f"after 1 warm-up step")
    return out


def cpu_sample(kw, steps=1, warmup=0):
    """The oracle (the C++ restatement of the reference's algorithm, on all
    host threads) stepping the full-size duct: `warmup` untimed steps, then
    `steps` full time steps timed one by one, every PCG solved to the case's
    1e-10 exactly as on the GPU path (no caps, no extrapolation).  Returns
    (steps_per_s, description, per-step iteration counts)."""
    import oracle.oracle as O
    from moons_b200 import configs
    sim = configs.make(O, configs.duct, seed=0, **kw)
    if warmup:
        sim.step(warmup)
    secs, its = [], {}
    for _ in range(steps):
        t0 = time.perf_counter()
        info = sim.step(1)
        secs.append(time.perf_counter() - t0)
        for k in ("iters_U", "iters_p", "iters_B", "iters_phi"):
            its[k] = its.get(k, 0) + info[k] / steps
    t = float(np.sum(secs))
    desc = (f"oracle (C++ restatement of the reference algorithm, {O.threads()} host threads), full-size duct, "
            f"seed 0: {steps} full time step(s) after {warmup} untimed step(s), every PCG to 1e-10 "
            f"({t:.1f} s; per step {[round(x, 2) for x in secs]} s)")
    return steps / t, desc, its


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    kw = duct_kw(args.small)
    import oracle.oracle as O
    cores = O.threads()
    # full, uncapped oracle steps (about 15 s each on the host cores): the
    # warm-up is one untimed step and at most 10 of the K steps are timed, so
    # that the arm ends within a few minutes; the rate is over the timed steps
    k_timed = max(1, min(args.steps, 10))
    value, desc, its = cpu_sample(kw, steps=k_timed, warmup=min(args.warmup, 1))
    desc += f"; {k_timed} of the requested {args.steps} steps timed, {min(args.warmup, 1)} of {args.warmup} warm-up"
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1e-4) velocity)",
        "config": {"workload": WORKLOAD, "mesh_fluid": [kw["nx"], kw["ny"], kw["nz"]], "pcg_tol_rel": 1e-10},
        "impl": "reference", "per_step": its,
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ldc32_config1(G, steps=1000):
    """Configuration 1 at its stated size: the MHD lid-driven cavity, uniform
    32^3, Re = 400, Ha = 10, potential form, dt = 1e-3, PCG to 1e-10, 1000
    steps from the seeded state; steps/s and the fields' relative L2 against
    the oracle's 1000-step fixture."""
    fx = os.path.join(ROOT, "tests", "golden", "ldc32_step1000.npz")
    from tests.golden import make_ldc32 as mk
    sim = mk.build_case(G)
    ms, tot = 0.0, {"iters_U": 0, "iters_p": 0, "iters_phi": 0}
    for _ in range(steps // 100):
        info = sim.step(100)
        ms += info["ms"]
        for k in tot:
            tot[k] += info[k]
    out = {"workload": "MHD lid-driven cavity 32^3 uniform, Re=400, Ha=10, low-Rem potential form, dt=1e-3, "
                       "PCG to 1e-10, 1000 steps from U0 = N(0,1e-6)",
           "steps": steps, "steps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps,
           "iters_per_step": {k: v / steps for k, v in tot.items()}}
    if os.path.exists(fx) and steps == 1000:
        z = np.load(fx)
        errs = {}
        for name, which, c in mk.FIELDS_LONG:
            a, b = sim.download(which, c), z[name]
            errs[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        out["rel_l2_vs_oracle_fixture"] = errs
        out["rel_l2_max"] = max(errs.values())
    return out


def main():
    args = parse()
    if args.profile:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    if args.leg == "at_scale":
        from moons_b200 import capi as G
        print(json.dumps({"leg": "at_scale", "result": at_scale_steps(G, small=args.small, steps=args.leg_steps)}),
              flush=True)
        return
    rank, world, local, dist = dist_setup(args.gpus)
    import torch
    from moons_b200 import capi as G, configs
    torch.cuda.set_device(local)
    kw = duct_kw(args.small)
    sim = configs.make(G, configs.duct, seed=rank, **kw)
    # warm-up (also builds the solver graphs)
    winfo = sim.step(args.warmup)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = G.kernel_launches()
    with Clocks(local) as clk:
        info = sim.step(args.steps)
    torch.cuda.synchronize()
    launches = G.kernel_launches() - launches0
    if dist is not None:
        dist.barrier()
    ms = max_over_ranks(info["ms"], dist)
    value = replica_rate(world, args.steps, ms)
    du, db = sim.divergence()
    its_v = {k: info[k] / max(args.steps, 1) for k in ("iters_U", "iters_p", "iters_B", "iters_phi")}

    # ---- end to end through the C-ABI with pinned host buffers, as a host
    # code driving the time loop: a second simulation from the same seed
    # takes the same warm-up steps on the device, then each of the same K
    # steps uploads the state (U, B) from the host, advances it, and
    # downloads it back into the same host buffers -- the same trajectory
    # and solver work as `value`, plus the copies.
    del sim
    sim_e = configs.make(G, configs.duct, seed=rank, **kw)
    sim_e.step(args.warmup)
    state = [sim_e.field(G.MHD_U, c) for c in range(3)] + [sim_e.field(G.MHD_B, c) for c in range(3)]
    host = [torch.from_numpy(f.download().ravel(order="F").copy()).pin_memory() for f in state]
    h2d = sum(f.n * 8 for f in state)
    d2h = h2d
    its_e = {}
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for f, h in zip(state, host):
            f.upload_ptr(h.data_ptr())
        ie = sim_e.step(1)
        for f, h in zip(state, host):
            f.download_ptr(h.data_ptr())
        for k in ("iters_U", "iters_p", "iters_B", "iters_phi"):
            its_e[k] = its_e.get(k, 0) + ie[k] / args.steps
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(t_e2e, dist)
    e2e = world * args.steps / t_e2e
    del sim_e

    # ---- the same step with multigrid (FP32 V-cycle) pressure / potential
    # solves: same systems and exit tests, far fewer iterations
    simx = configs.make(G, configs.duct, seed=rank, prec_poisson=G.PREC_MG_MIXED, **kw)
    simx.step(args.warmup)
    infox = simx.step(args.steps)
    msx = max_over_ranks(infox["ms"], dist)
    value_mixed = replica_rate(world, args.steps, msx)
    del simx
    # ... and with the direct (fast-diagonalization) pressure / potential solves
    simf = configs.make(G, configs.duct, seed=rank, prec_poisson=G.PREC_FD, **kw)
    simf.step(args.warmup)
    infof = simf.step(args.steps)
    msf = max_over_ranks(infof["ms"], dist)
    value_fd = replica_rate(world, args.steps, msf)
    del simf

    # ---- Poisson ms to 1e-10 + roofline of the pressure PCG iteration
    pinfo, ncc = poisson_ms(G, kw)
    mginfo, _ = poisson_ms(G, kw, G.PREC_MG)
    shell = sigma_shell_poisson(G, n=32 if args.small else 128, seeds_plain=1 if args.small else 4,
                                seeds_mg=2 if args.small else 16)
    mxinfo, _ = poisson_ms(G, kw, G.PREC_MG_MIXED)
    try:
        peak_v = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        peak_v = 6650.0
    vcyc = vcycle_roofline(G, n=32 if args.small else 128, shell=2 if args.small else 4, peak=peak_v)
    fdinfo, _ = poisson_ms(G, kw, G.PREC_FD)
    scale5 = at_scale_steps(G, small=args.small)
    fullbc = full_bc_steps(G, small=args.small)
    learned = learned_mixed_poisson(G, n=32 if args.small else 128, shell=2 if args.small else 4,
                                    held=(1000, 1001) if args.small else tuple(range(1000, 1064)),
                                    train_draws=2 if args.small else 8, epochs=2 if args.small else 8,
                                    weights=None if args.small else WEIGHTS_TWO_STAGE)
    # roofline: the pressure Jacobi-PCG on configuration 5's mesh (4.36 M
    # cells, 35 MB per array: the iteration's working set is above the L2)
    rinfo, ncc_r = poisson_ms(G, at_scale_kw(args.small), builder=configs.at_scale)
    alg_bytes = 88.0 * ncc_r * rinfo["iterations"]  # 88 B per cell per FP64 PCG iteration (algorithmic)
    achieved = alg_bytes / (rinfo["ms"] / 1e3) / 1e9
    ldc = ldc32_config1(G, steps=100 if args.small else 1000)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak = float(peaks["hbm_gbs"])
        peak_src = "measured"
    except Exception:
        peak = 6650.0
        peak_src = "fallback"
    traffic, traffic_src = None, None
    tf = os.path.join(ROOT, "profiles", "pcg_traffic_at_scale.json")
    if os.path.exists(tf):
        try:
            tj = json.load(open(tf))
            traffic = tj["bytes_per_cell_iter"] * ncc_r  # per PCG iteration, like alg_bytes_per_launch
            traffic_src = tj.get("source")
        except Exception:
            traffic = None

    if rank == 0:
        import oracle.oracle as O
        cpu_cores = O.threads()
        cpu_v, cpu_desc, cpu_its = cpu_sample(kw, steps=1, warmup=0)
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1e-4) velocity, uniform B0)",
            "config": {"workload": WORKLOAD, "mesh_fluid": [kw["nx"], kw["ny"], kw["nz"]],
                       "pcg_tol_rel": 1e-10, "parallelism": f"replicas x{world}",
                       "l2": "working set (~60 FP64 arrays x 10.7 MB) exceeds the 126 MB L2; no flush; the "
                             "roofline solve's iteration working set (5 arrays x 35 MB) exceeds it too"},
            "per_step": its_v,
            "div_U_l2sq": du, "div_B_l2sq": db,
            "steps_per_s_mixed_poisson": {"value": value_mixed, "per_step": {k: infox[k] / max(args.steps, 1) for k in (
                "iters_U", "iters_p", "iters_B", "iters_phi")}, "note": "pressure and potential solves by FP64 "
                "flexible CG + FP32 multigrid (MOONS_PREC_MG_MIXED); everything else as in value"},
            "steps_per_s_fd_poisson": {"value": value_fd, "per_step": {k: infof[k] / max(args.steps, 1) for k in (
                "iters_U", "iters_p", "iters_B", "iters_phi")}, "note": "pressure and cleaning-potential solves "
                "by CG with the direct fast-diagonalization solve of the separable operator (MOONS_PREC_FD); "
                "everything else as in value"},
            "poisson": {"ms_to_1e-10": pinfo["ms"], "iterations": pinfo["iterations"], "rel": pinfo["rel"],
                        "cells": ncc, "solver": "FP64 Jacobi-PCG (reference algorithm)",
                        "mg_fp64": {"ms_to_1e-10": mginfo["ms"], "iterations": mginfo["iterations"],
                                    "rel": mginfo["rel"], "solver": "CG + FP64 multigrid V(2,2), red-black SOR 1.15"},
                        "mixed": {"ms_to_1e-10": mxinfo["ms"], "iterations": mxinfo["iterations"],
                                  "rel": mxinfo["rel"], "solver": "FP64 flexible CG + FP32 multigrid V(2,2), red-black SOR 1.15"},
                        "fd": {"ms_to_1e-10": fdinfo["ms"], "iterations": fdinfo["iterations"],
                               "rel": fdinfo["rel"], "solver": "FP64 CG + direct fast-diagonalization solve"},
                        "speedup_mixed_vs_plain": pinfo["ms"] / mxinfo["ms"],
                        "speedup_fd_vs_plain": pinfo["ms"] / fdinfo["ms"]},
            "poisson_sigma_shell": shell,
            "vcycle_roofline_sigma_shell": vcyc,
            "poisson_learned_mixed": learned,
            "at_scale": scale5,
            "full_bc_vacuum": fullbc,
            "config1_ldc32": ldc,
            "roofline": {"bound": "hbm", "kernel": "pressure Jacobi-PCG iteration (the fused cell-centred pair "
                                                  "k_cc_lap + k_l_update) on configuration 5's mesh, 128x128x256 "
                                                  "cells",
                         "achieved": achieved, "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                         "alg_bytes_per_launch": 88.0 * ncc_r, "cells": ncc_r,
                         "iterations": rinfo["iterations"], "ms_to_1e-10": rinfo["ms"],
                         "us_per_iteration": rinfo["ms"] * 1e3 / max(rinfo["iterations"], 1)},
            "cpu_baseline": {"value": cpu_v, "unit": "steps/s", "cores": cpu_cores, "kind": "port",
                             "sample": cpu_desc, "per_step": cpu_its},
            "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "per_step": its_e, "note": "the same K steps as value (after the same warm-up), driven from "
                                              "the host with U and B copied up and down each step"},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
