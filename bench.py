"""Benchmark: simulated days per wall-clock hour of the adaptive ocean time step.

Workload (N=1, the default): the adaptive run J5..J9 (2,621,442 cells at J9),
32 Boussinesq layers, flat 4000 m bottom with a seeded Gaussian seamount
(2000 m, 50 km), zonal jet + 8 seeded Gaussian bumps (300 km, 0.05 m) in the
layer thicknesses, wavelet threshold tolerance 5e-3, explicit RK4 with
dt = 37.5 s (150 s at J7 scaled with the finest grid spacing, the reference's
CFL rule dt = cfl dx_min / c).  The initial grid is refined level by level as
the reference's initialize does (a partially refined patch tree, 4 x 4 node
patches).  One step is the reference's time_step (src/main.f90:405-444): RK4
of the hierarchy with WT_after_step per stage, adapt's mask sequence with
refine() of the patch tree and compression, and the inverse transform,
replayed as one captured CUDA graph.  With --gpus N>1
every rank advances its own ensemble member (independent seeds, no
collective): weak scaling, value = member-days per hour summed over ranks.

--impl reference times the CPU restatement of the reference's path (the
reference is Fortran; no Fortran compiler exists on the build or GPU hosts)
on the host cores, on bounded samples of the same workload (the whole step
on every level with a subset of the layers, extrapolated to 32 layers).

--mode uniform times the single-level TRiSK RK4 stepper (uniform J7 x 16
by default).  --kernels-only times that stepper alone on --level/--nz (the
small case kernel profiles are captured on); --wavelets-only does the same
for the wavelet transforms on the hierarchy --level-2 .. --level;
--elliptic-only runs the free-surface solve comparison on J5..--level.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 300.0      # uniform stepper (explicit RK4, J5 config)
TOL_AD = 5e-3   # wavelet threshold tolerance of the adaptive run
DAY = 86400.0


def dt_adaptive(lmax):
    """Explicit RK4 step of the adaptive run: 150 s at J7, scaled with the
    finest grid spacing (dt = cfl dx_min / c with the same cfl at every
    max_level, initialize_dt_viscosity_case in test/seamount/test_case_module.f90)."""
    return 150.0 * 2.0 ** (7 - lmax)


def sim_days_per_hour(steps, seconds, dt=DT):
    return (steps * dt / DAY) / (seconds / 3600.0)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default="adaptive", choices=["adaptive", "uniform"])
    p.add_argument("--lmin", type=int, default=None, help="min level of the adaptive run (default 5)")
    p.add_argument("--level", type=int, default=None, help="max level (default 9 adaptive, 7 uniform)")
    p.add_argument("--nz", type=int, default=None, help="layers (default 32 adaptive, 16 uniform)")
    p.add_argument("--no-extra", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--kernels-only", action="store_true")
    p.add_argument("--wavelets-only", action="store_true")
    p.add_argument("--elliptic-only", action="store_true",
                   help="only the free-surface solve on uniform J5..J<level> (every method, the learned "
                        "preconditioner trained first); each timed solve is an NVTX range named after its method")
    p.add_argument("--ensemble", action="store_true",
                   help="the adaptive mode-split ensemble (RK4_split + adapt) of --members members for --days days")
    p.add_argument("--members", type=int, default=16)
    p.add_argument("--days", type=float, default=1.0)
    p.add_argument("--remap", default="2PPM", choices=["none", "0", "1", "2PPM"],
                   help="--ensemble: the layer remap taken when the relative layer mass drops below 0.9")
    p.add_argument("--learned-layers", action="store_true",
                   help="only the learned network's forward pass on uniform J<level>, layer by layer, with its "
                        "32 -> 32 layer on the tensor cores and on the CUDA cores")
    p.add_argument("--learned-pairs", type=int, default=None, metavar="N",
                   help="--elliptic-only: train the learned preconditioner on N residual/error pairs (8 a "
                        "right-hand side, 50 right-hand sides a batch, one pass) instead of the level's default")
    p.add_argument("--eval-seeds", type=int, default=None,
                   help="--elliptic-only: unseen right-hand sides to evaluate on (default 64 at J8, none below)")
    p.add_argument("--trace", default=None, metavar="PATH",
                   help="record a CUDA kernel timeline of --steps adaptive steps (after --warmup) into PATH "
                        "(Chrome trace) and print its summary instead of the bench line")
    a = p.parse_args()
    adaptive = a.mode == "adaptive" and not (a.kernels_only or a.wavelets_only or a.elliptic_only)
    if a.lmin is None:
        a.lmin = 5
    if a.level is None:
        a.level = 9 if adaptive else 7
    if a.nz is None:
        a.nz = 32 if adaptive else 16
    return a


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = [n for q, n in enumerate(names) if any(r[4 + q].lower().startswith("active") for r in rows)]
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, value, device):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ---------------------------------------------------------------- ours ----
def run_case(level, nz, steps, warmup, seed, device, stream_timing=True, e2e=True, kernels=True, flux_bits=64,
             dt=DT):
    import numpy as np
    import torch

    from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
    from wavetrisk_hydrostatic_b200 import _native as Nt
    from wavetrisk_hydrostatic_b200.model import TriskModel

    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=seed, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    if flux_bits != 64:
        model.flux_precision(flux_bits)
    stream = torch.cuda.ExternalStream(model.stream, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)  # 256 MB > 126 MB L2
    for _ in range(warmup):
        model.rk4(dt, 1)
    model.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(s))           # L2 flush between timed steps, outside the timed region
        ev[s][0].record(stream)
        model.rk4(dt, 1)
        ev[s][1].record(stream)
    model.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    out = {"ms_total": ms, "ms_per_step": ms / steps, "final_state": model.download()}

    if kernels:
        # Per-kernel launch durations of the same stepper, launched kernel by kernel
        # with CUDA events on the handle's stream (same steps, no graph).
        kt = (Nt.C.c_double * 16)()
        nk = Nt.C.c_int(0)
        Nt.check("wt_profile_rk4", Nt.lib().wt_profile_rk4(model.h, dt, steps, kt, Nt.C.byref(nk)))
        names = ["halo_state", "column", "step1", "post_step1", "halo_flux", "trend_rk"]
        out["kernel_ms_per_launch"] = {names[k]: kt[k] for k in range(min(nk.value, len(names))) if kt[k] > 0}

    if e2e:
        NN = g.NN
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        m, t, v = pin((nz, NN)), pin((nz, NN)), pin((nz, 3 * NN))
        m[:] = st["mass"]; t[:] = st["temp"]; v[:] = st["velo"]
        model.rk4_host(dt, 1, m, t, v)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(steps):
            model.rk4_host(dt, 1, m, t, v)
        t1 = time.perf_counter()
        out["e2e_s"] = t1 - t0
        out["h2d_bytes_per_step"] = int(m.nbytes + t.nbytes + v.nbytes)
        out["d2h_bytes_per_step"] = int(m.nbytes + t.nbytes + v.nbytes)
    out["NN"] = g.NN
    out["cells"] = 10 * 4 ** level + 2
    model.close()
    return out


LEARNED_TRAIN = {
    # (right-hand sides, pairs per right-hand side, right-hand sides per batch, Adam passes per batch);
    # --elliptic-only --learned-pairs 20000 trains on 2500 x 8 at J8 (about 2 minutes)
    6: (32, 4, 32, 10),
    7: (64, 4, 32, 6),
    8: (500, 8, 50, 1),    # 4000 residual/error pairs, streamed
}
# hidden activation slope: the identity measured fewer FCG iterations than slope 1/4 at J7 and J8 (5.0 / 6.0
# against 5.1 / 6.75 on 8 unseen right-hand sides, 256 / 512 training pairs)
LEARNED_SLOPE = 1.0


def elliptic_case(lmax, repeats=3, nvtx=False, eval_seeds=None, train=None, slope=LEARNED_SLOPE):
    """Free-surface solve on the uniform hierarchy J5..lmax to relative residual
    1e-10: the reference's FMG and SRJ, the FP64 V-cycle in FP64 refinement
    (plain FP64 multigrid), FP32 V-cycles in FP64 refinement, flexible CG
    without and with the V-cycle, and flexible CG preconditioned by the V-cycle
    plus the learned network (2 -> 32 -> 32 -> 1 channels, its middle layer on
    the tensor cores).  Best of `repeats` device-timed solves (the report's ms)
    from a zero first guess, at a fixed V-cycle schedule and at the schedule the
    autotuner picks for each method; then, with eval_seeds, the mean over that
    many right-hand sides none of the methods was tuned or trained on."""
    import numpy as np

    from wavetrisk_hydrostatic_b200 import Grid
    from wavetrisk_hydrostatic_b200.cases import bathymetry, elliptic_rhs
    from wavetrisk_hydrostatic_b200.model import EllipticSolver, solver_opts

    g = Grid(5, lmax, radius=6371e3)
    levels = [g.level(l) for l in range(5, lmax + 1)]
    S = EllipticSolver(levels, [bathymetry(lv, seed=1) for lv in levels])
    off = S.offsets
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=2)
    S.upload(f=f)
    S.restrict()
    _, fr = S.download()
    out = {"workload": f"Helmholtz free-surface solve, uniform J{lmax} ({10 * 4 ** lmax + 2} cells), "
                       f"hierarchy J5..J{lmax}, seeded bathymetry 500-5000 m, dt 600 s, rel. residual 1e-10"}
    it = dict(ir_max=2000)
    q = len(levels) - 1

    def timed(name, o, key=None):
        best, rep = None, None
        for _ in range(repeats):
            S.upload(u=np.zeros(off[-1]), f=fr)
            if nvtx:
                import torch
                torch.cuda.nvtx.range_push(name)
            rep = S.solve(o)
            if nvtx:
                torch.cuda.nvtx.range_pop()
            best = rep.ms if best is None else min(best, rep.ms)
        r = {"ms": best, "rel_residual": rep.true_rel_residual, "status": rep.status,
             "iterations": rep.iterations[q] if name.startswith("fcg") else rep.outer_iterations}
        if name.startswith("fcg"):
            r.update(restarts=rep.restarts, fallback_at=rep.precond_fallback)
        out[key or name] = r
        return r

    fixed = dict(down_iter=2, up_iter=2, coarse_iter=6)   # the V-cycle fastest for plain FP64 multigrid
    for name, o in (("fmg", solver_opts("fmg", 1e-10, max_vcycle=50, coarse_iter=300)),
                    ("srj", solver_opts("srj", 1e-10, max_srj_iter=4000, coarse_iter=300)),
                    ("mg64", solver_opts("mg64", 1e-10, **fixed)),
                    ("mixed", solver_opts("mixed", 1e-10, **fixed)),
                    ("fcg", solver_opts("fcg", 1e-10, **it)),
                    ("fcg_mg", solver_opts("fcg_mg", 1e-10, **fixed, **it))):
        timed(name, o)
    # every multigrid-based method at the V-cycle schedule the autotuner picks for it (built-in set:
    # down = up in {1, 2, 3} sweeps, coarse in {2, 4, 6, 10, 20}), timed the same way
    tuned = {}

    def tune(name):
        S.upload(u=np.zeros(off[-1]), f=fr)
        o, _ = S.autotune(name, 1e-10, repeats=2, ir_max=2000 if name.startswith("fcg") else 60)
        tuned[name] = o
        timed(name, o, name + "_tuned")["schedule"] = [o.down_iter, o.up_iter, o.coarse_iter]

    for name in ("mg64", "mixed", "fcg_mg"):
        tune(name)
    # the learned preconditioner: trained once, on residual/error pairs of the V-cycle tuned for FCG without
    # it (what that V-cycle leaves is what it learns to correct); training time is reported apart
    n_rhs, cycles, batch, epochs = train or LEARNED_TRAIN.get(lmax, (32, 4, 32, 6))
    d, u_, c = out["fcg_mg_tuned"]["schedule"]
    S.learned_setup(1)
    S.learned_activation(slope)
    tr = S.learned_train(n_rhs=n_rhs, cycles=cycles, epochs=epochs, lr=2e-3, seed=1, down_iter=d, up_iter=u_,
                         coarse_iter=c, batch_rhs=batch)
    out["learned_training"] = {"network": "2 -> 32 -> 32 -> 1, 7 taps, BF16 weights and activations, FP32 "
                                          f"accumulation, activation slope {slope}, 32->32 layer on tcgen05",
                               "pairs": tr.pairs, "adam_steps": tr.steps, "batch_rhs": batch,
                               "pair_schedule": [d, u_, c], "loss_first_epoch": tr.loss_first_epoch,
                               "loss_last_epoch": tr.loss_last_epoch, "ms_generate": tr.ms_generate,
                               "ms_train": tr.ms_train}
    timed("fcg_learned", solver_opts("fcg_learned", 1e-10, **fixed, **it))
    tune("fcg_learned")
    S.learned_tensor_cores(False)                # the same network with its middle layer on the CUDA cores
    timed("fcg_learned", tuned["fcg_learned"], "fcg_learned_tuned_cuda_cores")
    S.learned_tensor_cores(True)
    out["learned_speedup_vs_fp64_mg_tuned"] = out["mg64_tuned"]["ms"] / out["fcg_learned_tuned"]["ms"]
    if eval_seeds:
        # right-hand sides the network never saw (its training ones come from its own seeded generator)
        ev = {name: {"ms": [], "iterations": [], "worst_rel_residual": 0.0, "fallbacks": 0, "failures": 0}
              for name in tuned}
        for sd in range(100, 100 + eval_seeds):
            g2 = np.zeros(off[-1])
            g2[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=sd)
            S.upload(u=np.zeros(off[-1]), f=g2)
            S.restrict()
            _, gr = S.download()
            for name, o in tuned.items():
                S.upload(u=np.zeros(off[-1]), f=gr)
                rep = S.solve(o)
                e = ev[name]
                e["ms"].append(rep.ms)
                e["iterations"].append(rep.iterations[q] if name.startswith("fcg") else rep.outer_iterations)
                e["worst_rel_residual"] = max(e["worst_rel_residual"], rep.true_rel_residual)
                e["fallbacks"] += int(rep.precond_fallback > 0)
                e["failures"] += int(rep.status != 0)
        out["unseen_rhs_eval"] = {"seeds": eval_seeds, **{
            name: {"mean_ms": float(np.mean(e["ms"])), "mean_iterations": float(np.mean(e["iterations"])),
                   "worst_rel_residual": e["worst_rel_residual"], "fallbacks": e["fallbacks"],
                   "failures": e["failures"]} for name, e in ev.items()}}
        ue = out["unseen_rhs_eval"]
        ue["learned_speedup_vs_fp64_mg"] = ue["mg64"]["mean_ms"] / ue["fcg_learned"]["mean_ms"]
        ue["mixed_speedup_vs_fp64_mg"] = ue["mg64"]["mean_ms"] / ue["mixed"]["mean_ms"]
    out["mixed_speedup_vs_fp64_mg"] = out["mg64"]["ms"] / out["mixed"]["ms"]
    out["mixed_speedup_vs_fmg"] = out["fmg"]["ms"] / out["mixed"]["ms"]
    out["learned_speedup_vs_fp64_mg"] = out["mg64"]["ms"] / out["fcg_learned"]["ms"]
    out["learned_speedup_vs_vcycle_fcg"] = out["fcg_mg"]["ms"] / out["fcg_learned"]["ms"]
    out["learned_iterations_vs_vcycle_fcg"] = out["fcg_learned"]["iterations"] / max(1, out["fcg_mg"]["iterations"])
    S.close()
    return out


def workload_config(args, world=1):
    cells = 10 * 4 ** args.level + 2
    if args.mode == "adaptive":
        return {
            "workload": f"adaptive run J{args.lmin}..J{args.level} ({cells} cells at J{args.level}), {args.nz} "
                        f"Boussinesq layers, partially refined patch tree (4x4-node patches) refined level by "
                        f"level at the start as the reference's initialize does and by adapt every step, 4000 m "
                        f"bottom with a seeded Gaussian seamount (2000 m, 50 km), jet + "
                        f"8 seeded Gaussian bumps (300 km, 0.05 m), tol {TOL_AD} thresholds, explicit RK4 "
                        f"dt={dt_adaptive(args.level):g} s, WT_after_step per stage",
            "min_level": args.lmin, "max_level": args.level, "layers": args.nz, "dt_s": dt_adaptive(args.level),
            "tol": TOL_AD,
            "parallelism": f"replicas x{world} (independent ensemble members)" if world > 1 else "single GPU",
            "l2": "flushed (256 MB write) between timed steps, outside the timed region",
        }
    return {
        "workload": f"uniform J{args.level} icosahedral grid ({cells} cells), {args.nz} Boussinesq layers, "
                    f"flat 4000 m bottom, explicit RK4 dt=300 s"
                    + (" (the adaptive J4..J7 16-layer run with every point active)"
                       if (args.level, args.nz) == (7, 16) else ""),
        "level": args.level, "layers": args.nz, "dt_s": DT,
        "parallelism": f"replicas x{world} (independent ensemble members)" if world > 1 else "single GPU",
        "l2": "flushed (256 MB write) between timed steps, outside the timed region",
    }


def wavelet_case(lmin, lmax, nz, repeats=5, device=None):
    """Wavelet transforms of the layered state on the uniform hierarchy
    lmin..lmax: forward_wavelet_transform, inverse_wavelet_transform and
    WT_after_step (wavelets + compression + inverse).  CUDA-event time on the
    handle's stream, best of `repeats`.  Algorithmic bytes of WT_after_step per
    node-layer of the levels above lmin: read scaling and write wavelets of
    5 words, read wavelets and read/write scaling of 5 words = 20 words."""
    import numpy as np
    import torch

    from wavetrisk_hydrostatic_b200 import Grid
    from wavetrisk_hydrostatic_b200.cases import edge_velocity, jet_state, solid_body_rotation
    from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    H = WaveletHierarchy(levels, [np.full(g.NN, -4000.0) for g in levels], nz)
    g = levels[-1]
    st = jet_state(g, nz, seed=3)
    H.upload(lmax, "mass", st["mass"])
    H.upload(lmax, "temp", st["temp"])
    H.upload(lmax, "velo", st["velo"] + edge_velocity(g, solid_body_rotation(0.1))[None, :])
    stream = torch.cuda.ExternalStream(H.stream, device=device)
    out = {"workload": f"wavelet transforms, uniform J{lmin}..J{lmax} hierarchy, {nz} layers (mass, Theta, velocity)"}
    for name, fn in (("forward_ms", H.forward), ("inverse_ms", H.inverse), ("wt_after_step_ms", H.wt_after_step)):
        best = None
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            t = a.elapsed_time(b)
            best = t if best is None else min(best, t)
        out[name] = best
    cells = sum(10 * 4 ** l for l in range(lmin + 1, lmax + 1))
    out["wt_after_step_GBps"] = cells * nz * 20 * 8 / (out["wt_after_step_ms"] / 1e3) / 1e9
    H.close()
    return out


def adaptive_launches(L, need_r=4):
    """Kernels launched by one adaptive step of L levels with a patch tree
    (AdaptiveOcean.step with fixed thresholds once the tree's level_end is the
    top: one graph replay); C = L - 1 parent levels, the same number of levels
    above level_start.
    * RK4, per stage: column, step1 and trend of every level (the levels above
      level_start over their work lists), two scalar and one flux restriction
      and three forward-wavelet kernels per parent level; four inverse kernels
      per parent level after each of the first three stages and after adapt.
    * adapt's mask sequence (init_masks_zero, mask_active, the sweeps with
      refine() of the tree, complete_masks, mask_trsk and 3C + 6 comm_masks).
    * The maps: one seed, need_r dilations and the cut to the tree; per parent
      level seven reconstruct-map launches; three launches per work list (one
      per level above level_start and one per parent level).
    * compress_wavelets of the dropped slots.
    The ncu launch list of one step (profiles/adaptive_J5-J9x32_step_launch_list.md)
    counts 360 for L = 5."""
    C = L - 1
    stage = 12 * L + 12 * C + 12 * C + 16 * C
    masks = C + 3 * L + 13 * C + 4
    maps = 1 + need_r + C + 7 * C + 3 * C + 3 * C
    return stage + masks + maps + C


def algorithmic_bytes_trend_ml(level, nz, n_on=None, n_own=None, n_listed=None):
    """Compulsory bytes of one multi-level trend launch on a level with the
    fused RK sub-step (k_trend_ml, k_trend_ml_list over the level's work list,
    or k_trend_tma<MODE_ML> on the finest level, which stages every input plane
    of a tile, so its traffic is higher).  Every node of [0, n]^2 reads its mask
    and writes dmass and dTheta (2 words a layer); every owned node writes the
    velocity source (3); the n_on nodes with mask_n >= TRSK also read theta,
    qe(3), hflux_mass(3), hflux_Theta(3), Bernoulli and Phi (12 words a layer)
    and len(3), part(6), hex_inv once; every padded node reads the RK base state
    and writes the stage state (5 + 5 words a layer).  Without n_on every node
    counts as active.  n_listed: the work list's owned nodes, which then stand
    for the nodes of [0, n]^2, the owned nodes and the padded nodes alike (the
    list's few ghost-ring slots are left out, so the figure is a lower bound)."""
    n = 2 ** level
    P = n + 4
    NN = 10 * P * P
    inner = 10 * (n + 1) ** 2
    own = 10 * n * n if n_own is None else n_own
    if n_listed is not None:
        inner = own = NN = n_listed
    on = inner if n_on is None else n_on
    return nz * (inner * 2 * 8 + own * 3 * 8 + on * 12 * 8 + NN * 10 * 8) + inner * 4 + on * 10 * 8


def adaptive_states(levels, nz, seed, ph):
    """Initial states of the adaptive run on every level: seamount bathymetry,
    layers following it, jet and bumps (the same seeds on every level)."""
    from wavetrisk_hydrostatic_b200.cases import bump_state, seamount_topography

    return [bump_state(g, nz, seed=seed, ph=ph, topo=seamount_topography(g, seed=seed)) for g in levels]


def adaptive_case(lmin, lmax, nz, steps, warmup, seed, device, e2e=True, profile=True):
    """The adaptive run lmin..lmax (seamount, jet + 8 Gaussian bumps, tol 5e-3
    thresholds of initialize_thresholds_case), its initial grid refined level
    by level as the reference's initialize does, one step = RK4 of the
    hierarchy + adapt (with refine() of the patch tree) + inverse transform.
    CUDA-event time per step on the handle's stream."""
    import numpy as np
    import torch

    from wavetrisk_hydrostatic_b200 import Grid, OceanParams
    from wavetrisk_hydrostatic_b200 import _native as Nt
    from wavetrisk_hydrostatic_b200.adaptive import AdaptiveOcean

    DT_AD = dt_adaptive(lmax)
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = adaptive_states([G.level(lmin - 1)] + levels, nz, seed, ph)
    t_init = time.perf_counter()
    model = AdaptiveOcean(G, lmin, lmax, nz, states[1:], ph, tol=TOL_AD, root_state=states[0])
    t_init = time.perf_counter() - t_init
    del states
    dev = model.dev
    tree_init = tree_summary(model, levels)
    stream = torch.cuda.ExternalStream(dev.stream, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    for _ in range(warmup):
        model.step(DT_AD)
    torch.cuda.synchronize(device)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(s))
        ev[s][0].record(stream)
        torch.cuda.nvtx.range_push("step")   # for an ncu launch list of the timed steps
        model.step(DT_AD)
        torch.cuda.nvtx.range_pop()
        ev[s][1].record(stream)
    torch.cuda.synchronize(device)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    out = {"ms_total": ms, "ms_per_step": ms / steps}
    act = []
    for g, (mn, me) in zip(levels, model.masks()):
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        ii = np.arange(g.n + 1)
        I, J = np.meshgrid(ii, ii, indexing="xy")
        inner = np.concatenate([((d * g.P + J + 2) * g.P + I + 2).ravel() for d in range(10)])
        act.append({"level": g.level, "active_nodes": int(np.count_nonzero(mn[own] >= 8)),
                    "active_edges": int(np.count_nonzero(me[e] >= 8)), "edges": int(e.size),
                    "trsk_nodes_0n": int(np.count_nonzero(mn[inner] >= 2))})
    out["masks"] = act
    out["tree"] = tree_summary(model, levels)
    out["tree_init"] = tree_init
    out["tree"]["init_s"] = round(t_init, 2)
    out["tree"]["init_log"] = [list(x) for x in model.init_log]
    if profile:
        pm = (Nt.C.c_double * 7)()
        pc = (Nt.C.c_int * 7)()
        # NVTX range "roofline_list" for ncu: the profiled step with the timed steps' maps and lists
        torch.cuda.nvtx.range_push("roofline_list")
        Nt.check("wt_profile_rk4_multi", Nt.lib().wt_profile_rk4_multi(dev.h, DT_AD, 1, pm, pc))
        torch.cuda.nvtx.range_pop()
        names = ["step1_top", "step1_coarse", "restrict", "trend_ml_top", "trend_ml_coarse", "rk_sub", "wt_after_step"]
        out["phase_ms"] = {names[p]: pm[p] for p in range(7)}
        out["phase_count_per_step"] = {names[p]: pc[p] for p in range(7)}
        # the roofline kernel timed with every node computed: the timed steps let the
        # finest level's trend leave out the tiles no needed node is in, so there it does
        # less than the algorithmic bytes count (NVTX range "roofline" for ncu)
        dev.skip_inactive(False)
        torch.cuda.nvtx.range_push("roofline")
        Nt.check("wt_profile_rk4_multi", Nt.lib().wt_profile_rk4_multi(dev.h, DT_AD, 1, pm, pc))
        torch.cuda.nvtx.range_pop()
        dev.skip_inactive(True)
        out["phase_ms_dense"] = {names[p]: pm[p] for p in range(7)}
    if e2e:
        # The host keeps what the reference's host holds between steps: the
        # finest level's prognostic state on its existing patches (packed patch
        # by patch, wt_download_tree_state), every level's masks and the finest
        # level's patch bytes.  Each step uploads that state from pinned host
        # buffers, steps, and downloads the new state, the masks and the tree.
        pin = lambda shape, dt=torch.float64: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
        top = levels[-1]
        bufs = dev.tree_state_buffers(alloc=pin)
        mbuf = [{"mask_n": pin(g.NN, torch.int32), "mask_e": pin(3 * g.NN, torch.int32)} for g in levels]
        tbuf = pin(10 * (top.n // model.patch_size) ** 2, torch.uint8)
        ids = dev.FIELDS
        L = Nt.lib()
        dn = [(g.level, k, b[k]) for g, b in reversed(list(zip(levels, mbuf))) for k in ("mask_n", "mask_e")]
        bd = (len(dn), (Nt.C.c_int * len(dn))(*[l for l, _, _ in dn]),
              (Nt.C.c_int * len(dn))(*[ids[k] for _, k, _ in dn]), (Nt.C.c_void_p * len(dn))(*[a.ctypes.data for _, _, a in dn]))
        state = {"n": dev.download_tree_state(bufs)}
        h2d, d2h = [], []
        per_patch = 5 * nz * model.patch_size ** 2 * 8

        def put():
            dev.upload_tree_state(bufs, state["n"])
            h2d.append(state["n"] * per_patch)

        def get():
            state["n"] = dev.download_tree_state(bufs)
            Nt.check("wt_download_fields", L.wt_download_fields(dev.h, *bd))
            Nt.check("wt_tree_download", L.wt_tree_download(dev.h, lmax, tbuf.ctypes.data, None))
            d2h.append(state["n"] * per_patch + sum(a.nbytes for _, _, a in dn) + tbuf.nbytes)

        nsteps_e2e = max(1, steps // 2)
        part = [0.0, 0.0, 0.0]  # upload, step, download (each call returns after its stream)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(nsteps_e2e):
            ta = time.perf_counter()
            put()
            tb = time.perf_counter()
            model.step(DT_AD)
            tc = time.perf_counter()
            get()
            td = time.perf_counter()
            part[0] += tb - ta
            part[1] += tc - tb
            part[2] += td - tc
        t1 = time.perf_counter()
        out["e2e_s"] = t1 - t0
        out["e2e_parts_ms"] = {k: 1e3 * v / nsteps_e2e for k, v in zip(("upload", "step", "download"), part)}
        out["e2e_steps"] = nsteps_e2e
        out["h2d_bytes_per_step"] = int(sum(h2d) / len(h2d))
        out["d2h_bytes_per_step"] = int(sum(d2h) / len(d2h))
    out["cells_finest"] = 10 * 4 ** lmax + 2
    model.close()
    return out


def tree_summary(model, levels):
    """The patch tree after the run: its level_end and, per level, the patches
    that exist out of all and the owned nodes they hold."""
    ps = model.patch_size
    per = []
    nodes = 0
    for g in levels:
        ex = model.patches(g.level)
        st = model.dev.tree_stats(g.level)
        per.append({"level": g.level, "patches": int(ex.sum()), "of": int(ex.size), "needed_owned_nodes": st[3],
                    "owned_nodes": 10 * g.n * g.n})
        nodes += int(ex.sum()) * ps * ps
    dense = sum(10 * g.n * g.n for g in levels)
    return {"level_end": model.level_end(), "patch_size": ps, "levels": per, "tree_nodes": nodes,
            "dense_nodes": dense, "tree_fraction": nodes / dense}


def algorithmic_bytes_trend_rk(level, nz):
    """Compulsory bytes of one k_trend launch (MODE_RK).  Node-layers of the
    computed range [0, n]^2 read theta, qe(3), hflux_mass(3), hflux_Theta(3),
    Bernoulli, Phi and the base mass/temp/velo(3) = 17 words and write the
    stage's mass/temp/velo(3) = 5 words; node-layers of the padded ring only
    read and write the 5 base words; geometry len(3), part(6) and hex_inv is
    read once per node of [0, n]^2."""
    n = 2 ** level
    P = n + 4
    inner = 10 * (n + 1) ** 2
    ring = 10 * P * P - inner
    return nz * (inner * 22 * 8 + ring * 10 * 8) + inner * 10 * 8


def bench_ours(args):
    if args.mode == "uniform":
        return bench_ours_uniform(args)
    import numpy as np
    import torch

    world, rank, local, pg = dist_init(args)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    barrier(pg)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize(device)
    barrier(pg)
    r = adaptive_case(args.lmin, args.level, args.nz, args.steps, args.warmup, seed=1 + rank, device=device)
    torch.cuda.synchronize(device)
    barrier(pg)
    clocks = sampler.stop() if sampler else None
    ms_max = allreduce_max(pg, r["ms_total"], device)
    e2e_max = allreduce_max(pg, r["e2e_s"], device)
    DT_AD = dt_adaptive(args.level)
    value = world * sim_days_per_hour(args.steps, ms_max / 1e3, DT_AD)
    e2e_value = world * sim_days_per_hour(r["e2e_steps"], e2e_max, DT_AD)

    extra = []
    if not args.no_extra and rank == 0 and world == 1:
        for (lv, nz, steps) in [(7, 16, 50), (5, 8, 100), (8, 32, 10)]:
            dtu = DT if lv == 5 else dt_adaptive(lv)   # 300 s is the plain method's; J7, J8 at their CFL step
            rr = run_case(lv, nz, steps, 2, seed=7, device=device, e2e=False, dt=dtu)
            kt = rr["kernel_ms_per_launch"]
            ab = algorithmic_bytes_trend_rk(lv, nz)
            extra.append({
                "workload": f"uniform J{lv} ({rr['cells']} cells), {nz} layers, single-level RK4 dt={dtu:g} s "
                            f"(the fused uniform stepper)",
                "ms_per_step": rr["ms_per_step"], "value": sim_days_per_hour(steps, rr["ms_total"] / 1e3, dtu),
                "unit": "simulated days per wall-clock hour",
                "kernel_ms_per_launch": kt,
                "trend_rk_GBps": ab / (kt["trend_rk"] / 1e3) / 1e9,
                "trend_rk_frac": ab / (kt["trend_rk"] / 1e3) / 1e9 / hbm,
            })
            if lv == 5:   # the reference's CPU-runnable case: the CPU restatement's step on this host beside it
                import oracle
                from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
                g5 = Grid(5, 5, radius=6371e3).level(5)
                ph5 = OceanParams()
                cur = jet_state(g5, nz, seed=7, ph=ph5)
                t_cpu, n_cpu = 0.0, 0
                while n_cpu < 3 or t_cpu < 3.0:
                    t0 = time.perf_counter()
                    m5, t5, v5 = oracle.rk4(g5, nz, ph5, cur, dtu, 1)
                    t_cpu += time.perf_counter() - t0
                    n_cpu += 1
                    cur = dict(cur, mass=m5, temp=t5, velo=v5)
                extra[-1]["cpu_baseline"] = {"ms_per_step": 1e3 * t_cpu / n_cpu,
                                             "value": sim_days_per_hour(n_cpu, t_cpu, dtu),
                                             "cores": oracle.get_threads(), "kind": "port",
                                             "cpu_model": cpu_model(), "sample": f"{n_cpu} RK4 steps"}
            if lv in (7, 8):   # the same run with FP32 flux stencils, error against the FP64 run
                rm = run_case(lv, nz, steps, 2, seed=7, device=device, e2e=False, flux_bits=32, dt=dtu)
                ref, got = rr["final_state"], rm["final_state"]
                err = {k: float(np.abs(got[k] - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-300))
                       for k in ("mass", "temp", "velo")}
                km = rm["kernel_ms_per_launch"]
                extra.append({
                    "workload": f"uniform J{lv}, {nz} layers, RK4 dt={dtu:g} s with the step1 flux stencils in "
                                f"FP32 (WT_TUNE_FLUX_PRECISION=32; FP64 trends, conservation and RK accumulation)",
                    "ms_per_step": rm["ms_per_step"], "value": sim_days_per_hour(steps, rm["ms_total"] / 1e3, dtu),
                    "unit": "simulated days per wall-clock hour",
                    "speedup_vs_fp64": rr["ms_per_step"] / rm["ms_per_step"],
                    "max_rel_error_vs_fp64_after_steps": {"steps": steps, **err},
                    "kernel_ms_per_launch": km,
                    "step1_plus_trend_ms_fp64": kt["step1"] + kt["trend_rk"],
                    "step1_plus_trend_ms_fp32_fluxes": km["step1"] + km["trend_rk"],
                })
        for lmax in (6, 7, 8):
            extra.append(elliptic_case(lmax, eval_seeds=64 if lmax == 8 else None))
        for (lmin, lmax, nzw) in ((5, 7, 16), (5, 8, 32)):
            extra.append(wavelet_case(lmin, lmax, nzw, device=device))

    if rank == 0:
        pm, pc = r["phase_ms"], r["phase_count_per_step"]
        share = {k: pm[k] * pc[k] for k in pm}
        tot = sum(share.values())
        dom = max(share, key=lambda k: share[k])
        # the roofline kernel: the finest level's k_trend_ml_list (its work list
        # = the needed slots), timed in the profiled step that takes the same maps
        listed = r["tree"]["levels"][-1]["needed_owned_nodes"]
        ab = algorithmic_bytes_trend_ml(args.level, args.nz, n_on=r["masks"][-1]["trsk_nodes_0n"], n_listed=listed)
        t_list = pm["trend_ml_top"]
        ach = ab / (t_list / 1e3) / 1e9
        ab_dense = algorithmic_bytes_trend_ml(args.level, args.nz)
        t_dense = r["phase_ms_dense"]["trend_ml_top"]
        traffic = None
        tf = os.path.join(ROOT, "profiles", "trend_ml_list_traffic.json")
        if os.path.exists(tf):
            try:
                tj = json.load(open(tf))
                if tj.get("traffic_per_algorithmic_byte"):   # measured on a smaller case, scaled by the bytes
                    traffic = int(tj["traffic_per_algorithmic_byte"] * ab)
            except Exception:
                traffic = None
        cpu = cpu_baseline(args, quick=True, tree_fraction=r["tree_init"]["tree_fraction"])
        L = args.level - args.lmin + 1
        line = {
            "metric": "sim-days/hour",
            "value": value,
            "unit": "simulated days per wall-clock hour",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded seamount, jet and Gaussian bumps)",
            "config": workload_config(args, world),
            "e2e": {"value": e2e_value, "unit": "simulated days per wall-clock hour",
                    "h2d_bytes_per_step": r["h2d_bytes_per_step"], "d2h_bytes_per_step": r["d2h_bytes_per_step"],
                    "path": "C-ABI wt_upload_tree_state / wt_adaptive_step / wt_download_tree_state + "
                            "wt_download_fields + wt_tree_download, pinned host buffers: the finest level's state "
                            "(every layer) on its existing patches in, that state, every level's masks and the "
                            "finest level's patch bytes out, every step (bytes: averages over the steps)",
                    "parts_ms_per_step": r["e2e_parts_ms"]},
            "gpu_launches": adaptive_launches(L) * args.steps,
            "roofline": {"bound": "hbm", "kernel": "k_trend_ml_list (level_end, over its work list)", "achieved": ach,
                         "peak": hbm, "unit": "GB/s", "frac": ach / hbm, "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes_per_launch": ab, "listed_owned_nodes": listed,
                         "kernel_ms": t_list,
                         "timing": "CUDA events around the kernel's launches in one profiled RK4 step (phase by phase, "
                                   "the same needed-node maps and work lists as the timed steps)",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the same kernel on the "
                                           "J5..J7 x 32 workload, per algorithmic byte, scaled to this launch "
                                           "(profiles/trend_ml_list_traffic.json)" if traffic else None,
                         "dense_tma_kernel": {"kernel": "k_trend_tma<MODE_ML> with every node computed (maps off)",
                                              "ms": t_dense, "algorithmic_bytes": ab_dense,
                                              "achieved_GBps": ab_dense / (t_dense / 1e3) / 1e9,
                                              "frac": ab_dense / (t_dense / 1e3) / 1e9 / hbm},
                         "dominant_phase_by_time": dom,
                         "phase_share": {k: v / tot for k, v in share.items()},
                         "phase_ms_per_occurrence": pm, "phase_count_per_step": pc},
            "masks_after_run": r["masks"],
            "patch_tree": r["tree"],
            "patch_tree_initial": r["tree_init"],
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        if extra:
            line["extra"] = extra
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def bench_ours_uniform(args):
    import torch

    world, rank, local, pg = dist_init(args)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    barrier(pg)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize(device)
    barrier(pg)
    r = run_case(args.level, args.nz, args.steps, args.warmup, seed=1000 + rank, device=device)
    torch.cuda.synchronize(device)
    barrier(pg)
    clocks = sampler.stop() if sampler else None
    ms_max = allreduce_max(pg, r["ms_total"], device)
    e2e_max = allreduce_max(pg, r["e2e_s"], device)
    value = world * sim_days_per_hour(args.steps, ms_max / 1e3)
    e2e_value = world * sim_days_per_hour(args.steps, e2e_max)

    extra = []
    if not args.no_extra and rank == 0 and world == 1:
        for (lv, nz, steps) in [(5, 8, 100), (8, 32, 10)]:
            dtu = DT if lv == 5 else dt_adaptive(lv)
            rr = run_case(lv, nz, steps, 2, seed=7, device=device, e2e=False, dt=dtu)
            kt = rr["kernel_ms_per_launch"]
            ab = algorithmic_bytes_trend_rk(lv, nz)
            extra.append({
                "workload": f"uniform J{lv} ({rr['cells']} cells), {nz} layers, RK4 dt={dtu:g} s",
                "ms_per_step": rr["ms_per_step"], "value": sim_days_per_hour(steps, rr["ms_total"] / 1e3, dtu),
                "kernel_ms_per_launch": kt,
                "trend_rk_GBps": ab / (kt["trend_rk"] / 1e3) / 1e9,
                "trend_rk_frac": ab / (kt["trend_rk"] / 1e3) / 1e9 / hbm,
            })
        for lmax in (6, 7, 8):
            extra.append(elliptic_case(lmax, eval_seeds=64 if lmax == 8 else None))
        for (lmin, lmax, nzw) in ((5, 7, 16), (5, 8, 32)):
            extra.append(wavelet_case(lmin, lmax, nzw, device=device))

    if rank == 0:
        kt = r["kernel_ms_per_launch"]
        dom = max(kt, key=lambda k: kt[k])
        ab = algorithmic_bytes_trend_rk(args.level, args.nz)
        ach = ab / (kt["trend_rk"] / 1e3) / 1e9
        traffic = None
        tf = os.path.join(ROOT, "profiles", "trend_rk_traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get(f"J{args.level}_nz{args.nz}")
            except Exception:
                traffic = None
        cpu = cpu_baseline(args, quick=True, tree_fraction=r["tree_init"]["tree_fraction"])
        line = {
            "metric": "sim-days/hour",
            "value": value,
            "unit": "simulated days per wall-clock hour",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded jet + white-noise free surface)",
            "config": workload_config(args, world),
            "e2e": {"value": e2e_value, "unit": "simulated days per wall-clock hour",
                    "h2d_bytes_per_step": r["h2d_bytes_per_step"], "d2h_bytes_per_step": r["d2h_bytes_per_step"],
                    "path": "wt_rk4_step_host (C-ABI), pinned host buffers, state copied in and out every step"},
            "gpu_launches": 12 * args.steps,
            "roofline": {"bound": "hbm", "kernel": "trend_rk", "achieved": ach, "peak": hbm, "unit": "GB/s",
                         "frac": ach / hbm, "peak_source": peak_src, "traffic": traffic,
                         "dominant_kernel_by_time": dom, "kernel_ms_per_launch": kt},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        if extra:
            line["extra"] = extra
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


# ----------------------------------------------------------- reference ----
def cpu_baseline(args, quick=False, tree_fraction=None):
    """Times the CPU restatement (oracle) on a bounded sample of the workload."""
    if args.mode == "adaptive":
        return cpu_baseline_adaptive(args, quick, tree_fraction)
    import numpy as np

    import oracle
    from oracle.grid import Grid as OGrid
    from wavetrisk_hydrostatic_b200.cases import OceanParams, jet_state

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    g = OGrid(args.level, args.level, radius=6371e3).level(args.level)
    ph = OceanParams()
    st = jet_state(g, args.nz, seed=1, ph=ph)
    oracle.rk4(g, args.nz, ph, st, DT, 1)
    budget = args.cpu_seconds if not quick else min(args.cpu_seconds, 10.0)
    steps, t_used = 0, 0.0
    cur = st
    while t_used < budget:
        t0 = time.perf_counter()
        m, t, v = oracle.rk4(g, args.nz, ph, cur, DT, 1)
        t_used += time.perf_counter() - t0
        cur = dict(st, mass=m, temp=t, velo=v)
        steps += 1
    return {"value": sim_days_per_hour(steps, t_used), "unit": "simulated days per wall-clock hour",
            "cores": oracle.get_threads(), "kind": "port",
            "sample": f"{steps} RK4 steps of the same workload ({t_used:.1f} s of CPU time)"}


def hierarchy_nodes(lmin, lmax):
    return sum(10 * 4 ** l + 2 for l in range(lmin, lmax + 1))


class AdaptiveCpuSampler:
    """CPU restatement (oracle) of the adaptive step, timed on bounded
    samples of the workload.  A sample is one whole adaptive step (multi-level
    trend and RK4 with WT_after_step per stage, adapt's mask sequence,
    compression, inverse transform) with every one of the workload's layers
    on the hierarchy lmin..lmax-2, i.e. the same computation at a quarter of
    the resolution; its time is scaled to lmin..lmax by the ratio of the node
    counts of the two hierarchies (about 16).  The oracle computes every node
    of every level, so its cost per node-layer does not depend on the
    resolution: on 8 threads it measured 0.894, 0.922 and 0.908 us per
    node-layer and step for J5..J6, J5..J7 and J5..J8 with 32 layers.
    Geometry comes from the oracle's own grid builder."""

    def __init__(self, lmin, lmax, nz, seed=1, tree_fraction=None):
        import oracle
        from oracle.grid import Grid as OGrid
        from wavetrisk_hydrostatic_b200.cases import OceanParams

        self.oracle = oracle
        self.threads = os.cpu_count() or 1
        oracle.set_threads(self.threads)
        self.threads = oracle.get_threads()
        self.ph = OceanParams()
        self.lmin, self.lmax, self.nz, self.seed = lmin, lmax, nz, seed
        self.ls = max(lmin + 1, lmax - 2)
        # the reference computes the nodes of its existing patches only: the
        # workload's initial patch tree holds this fraction of the hierarchy's nodes
        self.tree_fraction = oracle_tree_fraction(lmin, lmax, nz, seed) if tree_fraction is None else tree_fraction
        self.dense_scale = hierarchy_nodes(lmin, lmax) / hierarchy_nodes(lmin, self.ls)
        self.scale = self.dense_scale * self.tree_fraction
        G = OGrid(lmin, self.ls, radius=6371e3)
        self.levels = [G.level(l) for l in range(lmin, self.ls + 1)]
        self._setup()

    def _setup(self):
        import numpy as np
        from oracle.wavelet import Hierarchy

        ph, nz = self.ph, self.nz
        states = adaptive_states(self.levels, nz, self.seed, ph)
        self.thr = TOL_AD * np.stack([ph.ref_density * np.full(nz, ph.depth / nz), np.full(nz, 1e16),
                                      np.full(nz, 1.0)])
        H = Hierarchy(self.levels, nz)
        for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
            H.set(self.ls, key, states[-1][name])
        H.forward()
        H.mask_build(self.thr, 0, self.ls)
        H.compress()
        H.inverse()
        for st in states:
            for k in ("mass", "temp", "velo"):
                st.pop(k)
        self.states, self.H = states, H

    def sample(self):
        """One sample: (seconds of the step at lmin..lmax-2, the same scaled to lmin..lmax)."""
        H = self.H
        keys = (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v"))
        t0 = time.perf_counter()
        cur = [dict(self.states[q], **{n: H.field(g.level, k).copy() for n, k in keys})
               for q, g in enumerate(self.levels)]
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in self.levels]
        self.oracle.rk4_multi(self.levels, self.nz, self.ph, cur, masks, dt_adaptive(self.lmax), 1, H=H)
        H.mask_build(self.thr, 0, self.ls)
        H.compress()
        H.inverse()
        t = time.perf_counter() - t0
        return t, t * self.scale

    def describe(self, n, secs):
        return (f"{n} samples, each one whole adaptive step with all {self.nz} layers on the hierarchy "
                f"J{self.lmin}..J{self.ls} ({secs:.1f} s of CPU time in all; the oracle computes every node), "
                f"scaled by the node count x{self.dense_scale:.2f} to J{self.lmin}..J{self.lmax} and by the "
                f"fraction of those nodes in the existing patches of the workload's initial patch tree "
                f"({self.tree_fraction:.4f}), which is what the reference computes; CPU restatement (oracle), "
                f"multi-level trend over the 10 lozenges and wavelets over layers on {self.threads} threads, "
                f"mask sequence on one")


def oracle_tree_fraction(lmin, lmax, nz, seed):
    """The fraction of the hierarchy's owned nodes that lie in existing
    patches after the reference's initial refinement of the workload, from the
    oracle's restatement (oracle/tree.py); the GPU's tree is bit-identical to
    it (tests/test_tree_gpu.py)."""
    import numpy as np

    from oracle.grid import Grid as OGrid
    from oracle.tree import ReferenceInit
    from wavetrisk_hydrostatic_b200.adaptive import patch_size_for
    from wavetrisk_hydrostatic_b200.cases import OceanParams

    ph = OceanParams()
    G = OGrid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin - 1, lmax + 1)]
    ics = {g.level: st for g, st in zip(levels, adaptive_states(levels, nz, seed, ph))}
    thr = TOL_AD * np.stack([ph.ref_density * np.full(nz, ph.depth / nz), np.full(nz, 1e16), np.full(nz, 1.0)])
    ps = patch_size_for(lmin)
    RI = ReferenceInit(levels[0], levels[1:], nz, ics, thr, lmax, ps=ps).run()
    nodes = sum(int(e.sum()) * ps * ps for e in RI.tree.exist.values())
    return nodes / sum(10 * 4 ** l for l in range(lmin, lmax + 1))


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline_adaptive(args, quick=False, tree_fraction=None):
    """The oracle's adaptive step on the same workload: one warm-up sample,
    then samples until the time budget is used (at least two)."""
    S = AdaptiveCpuSampler(args.lmin, args.level, args.nz, tree_fraction=tree_fraction)
    S.sample()
    budget = args.cpu_seconds if not quick else min(args.cpu_seconds, 10.0)
    n, used, est = 0, 0.0, 0.0
    while n < 2 or used < budget:
        t, tf = S.sample()
        n, used, est = n + 1, used + t, est + tf
    return {"value": sim_days_per_hour(n, est, dt_adaptive(args.level)), "unit": "simulated days per wall-clock hour",
            "cores": S.threads, "kind": "port", "sample": S.describe(n, used), "seconds_per_step": est / n,
            "tree_fraction": S.tree_fraction,
            "dense_value": sim_days_per_hour(n, est / S.tree_fraction, dt_adaptive(args.level)),
            "cpu_model": cpu_model(), "host_threads": os.cpu_count()}


def bench_reference(args):
    """The reference arm: the CPU restatement of the path on the host cores,
    on the same workload, metric and config as our arm: --warmup untimed and
    --steps timed samples as AdaptiveCpuSampler describes; value = simulated
    days per hour of the scaled whole-workload steps."""
    world, rank, local, pg = dist_init(args)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    steps = max(1, args.steps)
    if args.mode == "adaptive":
        S = AdaptiveCpuSampler(args.lmin, args.level, args.nz)
        for _ in range(max(1, args.warmup)):
            S.sample()
        used, est = 0.0, 0.0
        for _ in range(steps):
            t, tf = S.sample()
            used, est = used + t, est + tf
        value = sim_days_per_hour(steps, est, dt_adaptive(args.level))
        cb = {"value": value, "unit": "simulated days per wall-clock hour", "cores": S.threads, "kind": "port",
              "sample": S.describe(steps, used), "seconds_per_step": est / steps, "tree_fraction": S.tree_fraction,
              "dense_value": sim_days_per_hour(steps, est / S.tree_fraction, dt_adaptive(args.level)),
              "cpu_model": cpu_model(), "host_threads": os.cpu_count()}
        data = "synthetic (seeded seamount, jet and Gaussian bumps)"
    else:
        cb = cpu_baseline(args)
        data = "synthetic (seeded jet + white-noise free surface)"
    line = {
        "impl": "reference",
        "metric": "sim-days/hour",
        "value": cb["value"],
        "unit": cb["unit"],
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": data,
        "config": workload_config(args, world),
        "note": "CPU restatement of the reference path (no Fortran compiler on the build or GPU hosts)",
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def bench_kernels(args):
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    r = run_case(args.level, args.nz, args.steps, args.warmup, seed=1, device=device, e2e=False, kernels=False)
    print(json.dumps({"workload": f"uniform J{args.level} ({r['cells']} cells), {args.nz} layers, RK4 dt=300 s",
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                      "value": sim_days_per_hour(args.steps, r["ms_total"] / 1e3),
                      "unit": "simulated days per wall-clock hour"}), flush=True)


def bench_trace(args):
    """Kernel timeline of graph-replayed adaptive steps (torch.profiler's CUDA
    activity trace, which sees every kernel of the process with its stream):
    per step the span, the time some kernel is running, and each kernel's
    summed duration.  A profiling aid; its times are not bench values."""
    import collections

    import torch
    from torch.profiler import ProfilerActivity, profile

    from wavetrisk_hydrostatic_b200 import Grid, OceanParams
    from wavetrisk_hydrostatic_b200.adaptive import AdaptiveOcean

    torch.cuda.set_device(0)
    ph = OceanParams()
    G = Grid(args.lmin, args.level, radius=6371e3)
    levels = [G.level(l) for l in range(args.lmin, args.level + 1)]
    states = adaptive_states([G.level(args.lmin - 1)] + levels, args.nz, 1, ph)
    model = AdaptiveOcean(G, args.lmin, args.level, args.nz, states[1:], ph, tol=TOL_AD, root_state=states[0])
    del states
    for _ in range(args.warmup):
        model.step(dt_adaptive(args.level))
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(args.steps):
            model.step(dt_adaptive(args.level))
        torch.cuda.synchronize()
    prof.export_chrome_trace(args.trace)
    ev = [e for e in json.load(open(args.trace))["traceEvents"] if e.get("cat") == "kernel"]
    iv = sorted((e["ts"], e["ts"] + e["dur"]) for e in ev)
    busy, (cs, ce) = 0.0, iv[0]
    for a, b in iv[1:]:
        if a > ce:
            busy += ce - cs
            cs, ce = a, b
        else:
            ce = max(ce, b)
    busy += ce - cs
    span = max(b for _, b in iv) - iv[0][0]
    tot = collections.Counter()
    for e in ev:
        tot[e["name"].split("(")[0].replace("void ", "")] += e["dur"]
    print(json.dumps({"workload": f"adaptive run J{args.lmin}..J{args.level}, {args.nz} layers", "steps": args.steps,
                      "kernels": len(ev), "span_us_per_step": span / args.steps,
                      "busy_us_per_step": busy / args.steps,
                      "kernel_us_per_step": {k: v / args.steps for k, v in tot.most_common()}}), flush=True)
    model.close()


def bench_wavelets(args):
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    print(json.dumps(wavelet_case(args.level - 2, args.level, args.nz, repeats=max(1, args.steps), device=device)),
          flush=True)


def dt_split(lmax):
    """Mode-split step of the ensemble: 4 times the explicit step (the free
    surface's gravity waves are implicit, so the external-wave CFL no longer
    binds).  At 8 times, 2 of the 16 members (one J8, one J9) went unstable
    within the day."""
    return 4.0 * dt_adaptive(lmax)


def ensemble_case(members=16, days=1.0, nz=32, lmin=5, rank=0, world=1, device=None, solver="mixed",
                  remap="2PPM"):
    """The adaptive mode-split ensemble: members with max levels J7, J8, J9
    in turn, each over its own seeded seamount and jet + bumps, J5..J<max> x nz
    layers, stepped by RK4_split (the implicit free surface solved every step)
    + adapt + inverse transform for `days` simulated days, with the layers
    remapped (remap type `remap`, None for none) whenever the smallest relative
    layer mass drops below 0.9, as the reference's time_step does.  Members
    are dealt to ranks (member m on rank m % world); each runs on its own
    handle, one after the other.  CUDA-event time of the steps (set-up
    excluded, the min-mass tests and remaps included)."""
    import numpy as np
    import torch

    from wavetrisk_hydrostatic_b200 import Grid, OceanParams
    from wavetrisk_hydrostatic_b200.adaptive import ModeSplitOcean
    from wavetrisk_hydrostatic_b200.model import solver_opts

    ph = OceanParams()
    mine = [m for m in range(members) if m % world == rank]
    lmax_of = {m: (7, 8, 9)[m % 3] for m in range(members)}
    G = Grid(lmin, max(lmax_of[m] for m in mine) if mine else lmin, radius=6371e3)
    out = []
    for m in mine:
        lmax = lmax_of[m]
        levels = [G.level(l) for l in range(lmin, lmax + 1)]
        states = adaptive_states([G.level(lmin - 1)] + levels, nz, 100 + m, ph)
        root_state, states = states[0], states[1:]
        g = levels[-1]
        own = g.owned
        area = 1.0 / g.hex_inv[own]

        def total_mass(m):   # area-weighted total mass of the finest level's layers (means included)
            return float(np.sum((states_mean + m[:, own]) * area[None, :]))

        states_mean = states[-1]["mean_m"][:, own]
        mass0 = total_mass(states[-1]["mass"])
        dt = dt_split(lmax)
        steps = int(round(days * DAY / dt))
        model = ModeSplitOcean(G, lmin, lmax, nz, states, dt, ph, tol=TOL_AD, root_state=root_state,
                               solver=solver_opts(solver, 1e-9, down_iter=2, up_iter=2, coarse_iter=6),
                               remap=remap)
        del states
        stream = torch.cuda.ExternalStream(model.dev.stream, device=device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its, unconverged = [], 0
        torch.cuda.synchronize(device)
        a.record(stream)
        for _ in range(steps):
            rep = model.step()
            its.append(rep.outer_iterations)
            unconverged += int(rep.status != 0)
        b.record(stream)
        torch.cuda.synchronize(device)
        ms = a.elapsed_time(b)
        mass = model.dev.download(lmax, "mass")
        velo = model.dev.download(lmax, "velo")
        eta = model.dev.free_surface(lmax)
        mn = model.masks()[-1][0]
        out.append({"member": m, "levels": [lmin, lmax], "dt_s": dt, "steps": steps, "ms": ms,
                    "ms_per_step": ms / max(1, steps), "status": model.dev.status(),
                    "solver_unconverged_steps": unconverged, "remaps": model.remaps,
                    "last_min_mass": model.min_mass,
                    "solver_mean_iterations": float(np.mean(its)) if its else 0.0,
                    "finite": bool(np.isfinite(mass).all() and np.isfinite(velo).all() and np.isfinite(eta).all()),
                    "max_abs_velocity": float(np.abs(velo[:, np.concatenate([np.nonzero(g.owned)[0] + e * g.NN
                                                                           for e in range(3)])]).max()),
                    "rel_total_mass_change": (total_mass(mass) - mass0) / mass0,
                    "active_fraction_finest": float(np.count_nonzero(mn[g.owned] >= 12)) / int(g.owned.sum())})
        model.close()
    return out


def learned_layers_case(lmax, reps=20):
    """The learned network's forward pass on uniform J<lmax>, layer by layer
    (mean device time over reps launches on a seeded residual), with the
    32 -> 32 layer on the tensor cores and on the CUDA cores.  Layer 2 per
    node: 2 * 224 * 32 flops; algorithmic bytes 64 (the node's own BF16 input
    row, the six tap rows being other nodes' rows) + 64 (output) + 28 (7 tap
    indices).  At J9 the activations (168 MB each) exceed the 126 MB L2."""
    import numpy as np

    from wavetrisk_hydrostatic_b200 import Grid
    from wavetrisk_hydrostatic_b200.cases import bathymetry
    from wavetrisk_hydrostatic_b200.model import EllipticSolver

    g = Grid(5, lmax, radius=6371e3)
    levels = [g.level(l) for l in range(5, lmax + 1)]
    S = EllipticSolver(levels, [bathymetry(lv, seed=1) for lv in levels])
    ns = S.learned_setup(1)
    S.learned_activation(LEARNED_SLOPE)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    hbm, tc = float(peaks["hbm_gbs"]), float(peaks["bf16_tflops"])
    out = {"workload": f"learned preconditioner forward pass, uniform J{lmax} ({ns} nodes), 2 -> 32 -> 32 -> 1 "
                       f"channels, 7 taps, BF16 activations", "nodes": ns}
    flops2, bytes2 = 2.0 * 224 * 32 * ns, (64 + 64 + 28) * ns
    for name, on in (("tensor_cores", True), ("cuda_cores", False)):
        S.learned_tensor_cores(on)
        ms = S.learned_layer_times(reps)
        out[name] = {"layer_ms": ms, "layer2_TFLOPs": flops2 / (ms[1] / 1e3) / 1e12,
                     "layer2_GBps": bytes2 / (ms[1] / 1e3) / 1e9}
        out[name]["layer2_frac_of_measured_hbm"] = out[name]["layer2_GBps"] / hbm
        out[name]["layer2_frac_of_measured_bf16"] = out[name]["layer2_TFLOPs"] / tc
    out["layer2_speedup_tensor_vs_cuda_cores"] = out["cuda_cores"]["layer_ms"][1] / out["tensor_cores"]["layer_ms"][1]
    S.close()
    return out


def bench_ensemble(args):
    """--ensemble: the 16-member mode-split ensemble for --days simulated days
    on N GPUs (members dealt to ranks, no collective on the data path); the
    line's value is member-days per hour of the slowest rank."""
    import torch

    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(device)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=device)
    res = ensemble_case(args.members, args.days, args.nz if args.nz else 32, rank=rank, world=world, device=device,
                        remap=None if args.remap == "none" else args.remap)
    ms = sum(r["ms"] for r in res)
    if world > 1:
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        allres = [None] * world
        dist.all_gather_object(allres, res)
        res = [r for part in allres for r in part]
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": "ensemble member-days per hour", "value": args.members * args.days / (ms / 3.6e6),
                          "unit": "simulated member-days per wall-clock hour", "n_gpus": world,
                          "ms_total_slowest_rank": ms, "scaling": "strong",
                          "config": {"workload": f"{args.members}-member adaptive mode-split ensemble, J5..J7/J8/J9 "
                                                 f"in turn x {args.nz or 32} layers, seeded seamount + jet + bumps, "
                                                 f"RK4_split + adapt + inverse transform, layers remapped "
                                                 f"({args.remap}) below relative mass 0.9, {args.days} "
                                                 f"simulated day(s)",
                                     "dtype": "f64"},
                          "members": res}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        bench_reference(args)
    elif args.kernels_only:
        bench_kernels(args)
    elif args.trace:
        bench_trace(args)
    elif args.wavelets_only:
        bench_wavelets(args)
    elif args.ensemble:
        bench_ensemble(args)
    elif args.learned_layers:
        print(json.dumps(learned_layers_case(args.level)), flush=True)
    elif args.elliptic_only:
        tr = None if args.learned_pairs is None else (max(1, args.learned_pairs // 8), 8, 50, 1)
        ev = args.eval_seeds if args.eval_seeds is not None else (64 if args.level == 8 else None)
        print(json.dumps(elliptic_case(args.level, nvtx=True, eval_seeds=ev, train=tr)))
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
