"""Benchmark: particle-steps/s of the full PIC-MCC step (rhs -> Poisson -> E -> sort -> MCC ->
push+deposit) on the 2048x2048 aperture-plate workload, one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config 4]

Prints ONE JSON line (rank 0).  Timing: CUDA events on the library's own stream, barrier +
synchronize on both sides, max over ranks.  The particle arrays (8.4 GB per species) are far
larger than L2, so no L2 flush is needed between steps.  Weak scaling for N > 1: the particles
are decomposed over the ranks as the reference does (load_part.f90:96), each rank holding one
GPU's workload at Nm / N, and the int64 charge accumulators are summed with one NCCL
all-reduce per step (exact, order-free); Poisson is solved replicated.

``--impl reference`` runs and times the CPU restatement of the same routines (OpenMP, all host
cores) on a bounded sample of the same workload: the configuration at its own particles per
cell on a smaller box (``--cpu-cells``), every phase measured and nothing scaled.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_PARTICLE_STEP = 40  # X, Y, VX, VY, VZ read + written by the fused push/deposit
PERM_BYTES_PER_PARTICLE = 4   # the push after a sort also reads the sort's permutation


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic_per_particle():
    """DRAM bytes per pushed particle of k_push_deposit from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "push_deposit_ncu.md")
    try:
        m = re.search(r"dram_bytes_per_particle\s*=\s*([0-9.]+)", open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms from before the warm-up
    (nvidia-smi takes a moment to start) and kept for the timed region only (its timestamps)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        t = time.time()
        while time.time() - t < 10.0 and os.path.getsize(self.path) == 0:   # first sample written
            time.sleep(0.05)

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self) -> dict:
        import datetime
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [[f.strip() for f in l.split(",")] for l in open(self.path).read().strip().splitlines()
                if l.count(",") >= 9]
        os.unlink(self.path)

        def stamp(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                return None
        inside = [r for r in rows if stamp(r) is not None and self.t0 is not None and self.t0 <= stamp(r) <= self.t1]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in inside if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in inside for k in range(4) if "Active" in r[6 + k] and "Not" not in r[6 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside)}


# ------------------------------------------------------------------------------------------
def sample_case(config: int, cells: int):
    """The bounded CPU sample of a workload: the same configuration (deck, walls, fields, its own
    particles per cell) on a box of `cells` cells along x, the aspect ratio kept."""
    from jd_lepic_b200 import configs
    full = configs.make_case(config)
    if cells >= full.nx:
        return full, full
    ny = max(16, cells * full.ny // full.nx)
    return full, configs.make_case(config, nx=cells, ny=ny)


def cpu_particles(case, spp, seed: int) -> dict:
    """Initial particles of a case for the CPU restatement: the load profile (uniform, or the
    Gaussian by rejection) outside the wall cells, Maxwellian velocities at vt0."""
    rng = np.random.default_rng(seed)
    n = case.n_particles
    L = case.nx * case.dx
    pts = []
    while sum(len(p) for p in pts) < n:
        x = rng.random(2 * n) * L
        y = rng.random(2 * n) * case.ny * case.dy
        if case.profile == 1:
            r2 = (x - 0.5 * L) ** 2 + (y - 0.5 * case.ny * case.dy) ** 2
            dens = case.n_floor + (case.n_peak - case.n_floor) * np.exp(-r2 / (2 * case.sigma ** 2))
            keep = rng.random(2 * n) * case.n_peak <= dens
            x, y = x[keep], y[keep]
        ix = (x / case.dx).astype(int) + 1
        iy = (y / case.dy).astype(int) + 1
        b = case.bcnd
        wall = (b[iy, ix] >= 1) & (b[iy, ix + 1] >= 1) & (b[iy + 1, ix + 1] >= 1) & (b[iy + 1, ix] >= 1)
        pts.append(np.stack([x[~wall], y[~wall]], 1))
    xy = np.concatenate(pts)[:n]
    parts = {}
    for s in range(spp.ntype):
        p = np.zeros((n, 6))
        p[:, :2] = xy
        p[:, 3:] = rng.normal(0, spp.vt0[s] / np.sqrt(2), (n, 3))
        parts[s] = p
    return parts


def cpu_baseline(config: int, cells: int, steps: int, warmup: int, nthreads: int) -> dict:
    """The step restated on the CPU (the oracle port: FP64, OpenMP over `nthreads` host threads,
    the reference's loop structure), run and timed as it is on a bounded sample of the workload
    (sample_case): calc_rhs, the reference's FP64 V-cycles stopped on the same relative L2
    residual as the device (1e-8; the L1 tolerance of mode-0 configurations), calc_Efield,
    part_sorting and collisions at their 1-in-10 cadence (main.f90:479-480), the mover and the
    deposit.  Every phase is measured; nothing is scaled."""
    from oracle import oracle as O
    from jd_lepic_b200 import deck as dk
    from jd_lepic_b200.simulation import species_params
    full, case = sample_case(config, cells)
    spp = species_params(case, dk.read_reactions(case.deck_text, case.ngas))
    sim = O.OracleSimulation(case, nthreads=nthreads, particles=cpu_particles(case, spp, case.seed), seed=123456)
    l2 = case.poisson_mode != 0
    eps = 1e-8 if l2 else case.eps
    it = 1
    for _ in range(warmup):
        sim.step(it, eps, l2)
        it += 1
    done = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        done += sum(sim.np_tot)
        sim.step(it, eps, l2)
        it += 1
    t = time.perf_counter() - t0
    return {"value": done / t, "unit": "particle-steps/s", "cores": nthreads, "kind": "port",
            "ms_per_step": t / steps * 1e3,
            "sample": (f"{full.name} at its {case.ppc} particles per cell on a {case.nx}x{case.ny}-cell box "
                       f"({case.n_particles} particles per species; the full workload is {full.nx}x{full.ny}, "
                       f"{full.n_particles} per species): {steps} steps after {warmup}, every phase measured, "
                       f"Poisson to {'relative L2 ' if l2 else 'L1 '}{eps:g}")}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from jd_lepic_b200 import configs
    full = configs.make_case(args.config)
    nt = host_threads()
    t0 = time.perf_counter()
    cb = cpu_baseline(args.config, args.cpu_cells, args.steps, args.warmup, nt)
    wall = time.perf_counter() - t0
    line = {"metric": "particle-steps/s per PIC step (push+deposit+MCC+sort+Poisson to 1e-8)",
            "value": cb["value"], "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": full.name, "particles_per_species": full.n_particles, "grid": [full.nx, full.ny],
                       "poisson": "the reference's multigrid (FP64) on the CPU, relative L2 residual 1e-8",
                       "sample": cb["sample"]},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line))
    return 0


def learned_compare(args, sim, lib, ctx, capi, stream, it, eps, pois, one_step_fn):
    import torch
    import ctypes as C
    cfg = capi.LepicCnnConfig(enable_training=1, warmup_solves=10 ** 9, steps_warmup=args.learn_train_steps,
                              train_every=1, steps_after=args.learn_train_steps, crop=args.learn_crop,
                              batch=args.learn_batch, lr=C.c_float(args.learn_lr), seed=11)
    sim.check(lib.lepic_gpu_cnn_configure(ctx, C.byref(cfg)), "cnn_configure")

    def timed(fn):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    t_train = timed(lambda: [one_step_fn(it + k, False, capi.POISSON_LEARNED) for k in range(args.learn_steps)])
    it += args.learn_steps
    cfg_off = capi.LepicCnnConfig(**{f: getattr(cfg, f) for f, _ in cfg._fields_})
    cfg_off.enable_training = 0
    rows = []
    for k in range(args.learn_ab):
        sim.check(lib.lepic_gpu_calc_rhs(ctx, None), "calc_rhs")
        phi_prev = sim.grid(capi.GRID_PHI)
        row = {}
        for name, m in (("fp64_mg", capi.POISSON_FP64_MG_L2), ("mixed_pcg", capi.POISSON_MIXED_IR),
                        ("learned", capi.POISSON_LEARNED), ("learned_train", capi.POISSON_LEARNED)):
            sim.set_phi(phi_prev)
            sim.check(lib.lepic_gpu_cnn_configure(ctx, C.byref(cfg if name == "learned_train" else cfg_off)),
                      "cnn_configure")
            st = capi.LepicSolveStats()
            ms = timed(lambda: sim.check(lib.lepic_gpu_iterative_solver(ctx, None, eps, m, C.byref(st)), "solver"))
            row[name] = {"ms": ms, "cycles": st.cycles, "res_l2_rel": st.res_l2_rel}
            if name == "fp64_mg":
                phi_ref = sim.grid(capi.GRID_PHI)
            if name == "learned":   # the same discrete solution as the FP64 multigrid's
                phi_l = sim.grid(capi.GRID_PHI)
                row[name]["phi_rel_err_vs_fp64"] = float(np.abs(phi_l - phi_ref).max() / np.abs(phi_ref).max())
                cs = capi.LepicCnnStats()
                sim.check(lib.lepic_gpu_cnn_stats(ctx, C.byref(cs)), "cnn_stats")
                row[name]["res_ratio"] = cs.last_res_ratio
                row[name]["accepted"] = cs.last_accepted
        rows.append(row)
        sim.check(lib.lepic_gpu_calc_efield(ctx, None), "efield")
        sim.check(lib.lepic_gpu_push_deposit(ctx, it, None), "push")
        it += 1
    sim.check(lib.lepic_gpu_cnn_configure(ctx, C.byref(cfg_off)), "cnn_configure")
    mean = lambda name, key: float(np.mean([r[name][key] for r in rows]))
    out = {"training_pic_steps": args.learn_steps, "training_ms_total": t_train,
           "train_steps_per_solve": args.learn_train_steps, "crop": args.learn_crop, "batch": args.learn_batch,
           "ab_steps": args.learn_ab}
    for name in ("fp64_mg", "mixed_pcg", "learned", "learned_train"):
        out[name] = {"ms": mean(name, "ms"), "cycles": mean(name, "cycles"),
                     "res_l2_rel_max": max(r[name]["res_l2_rel"] for r in rows)}
    out["learned"]["res_ratio"] = mean("learned", "res_ratio")
    out["learned"]["phi_rel_err_vs_fp64_max"] = max(r["learned"]["phi_rel_err_vs_fp64"] for r in rows)
    out["learned"]["accepted"] = mean("learned", "accepted")
    out["online_training_ms_per_solve"] = out["learned_train"]["ms"] - out["learned"]["ms"]
    out["speedup_learned_vs_fp64_mg"] = out["fp64_mg"]["ms"] / out["learned"]["ms"]
    out["speedup_learned_vs_mixed_pcg"] = out["mixed_pcg"]["ms"] / out["learned"]["ms"]
    pois["learned_ab"] = out
    return it


def sources_measure(args, sim, lib, ctx, stream, it, case):
    """eheating, the heating-region tally, part_injection and part_flux_emitter (the per-step
    particle sources) on the workload's own electron population, each entry point timed with CUDA events on
    the library's stream over args.steps calls after 3 untimed ones.  Heating region: the slit
    0.1 L <= x <= 0.6 L over the full height; nu_h = 5e8 /s (nu*dt*ns_heat = 2e-3 at dt = 1e-12 s,
    ns_heat = 4); 65536 particles injected per species and call (fixed current, uniform slit).
    Algorithmic bytes: heating 8 B per electron slot (X, Y) + 4 B per electron in the region
    (VX, the hole test) + 20 B per heated electron (VY, VZ read, three velocities written);
    the tally 8 B per slot + 12 B per electron in the region."""
    import ctypes as C
    import torch
    from jd_lepic_b200 import _capi as capi, sources as S
    from jd_lepic_b200 import deck as dk
    Lcm, Hcm = case.nx * case.dx * 100.0, case.ny * case.dy * 100.0
    n_inj = 65536
    I_inj = n_inj * dk.QE * sim.sp.Nm[0] / case.dt
    sc = S.source_config(S.SourceDeck(heat_region_cm=(0.1 * Lcm, 0.6 * Lcm, 0.0, Hcm), nu_h=5.0e8, Pabs=(0.0,),
                                      I_inj=I_inj, opt_inj=1, ni0=(1.0, 1.0), ns_heat=4, seed=2024),
                         case.dt, sim.sp.vt0[0])
    sim.set_sources(sc)
    reps = max(3, args.steps)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    n_slots = sim.push_stats()["n_slots"][0]
    t0 = sim.source_tallies()
    heat_ms = timed(lambda: sim.check(lib.lepic_gpu_eheating(ctx, it), "eheating"))
    t1 = sim.source_tallies()
    n_heated = (t1["n_heated"] - t0["n_heated"]) / (t1["n_heat_calls"] - t0["n_heat_calls"])
    tally_ms = timed(lambda: sim.check(lib.lepic_gpu_heating_tally(ctx), "heating_tally"))
    n_in = sum(sim.source_tallies()["Nh"])
    c0 = sim.source_tallies()["n_inj"]
    inj_ms = timed(lambda: sim.check(lib.lepic_gpu_part_injection(ctx, it), "part_injection"))
    c1 = sim.source_tallies()["n_inj"]
    # part_flux_emitter of electrons (THm = 1 eV) from the plasma-side face of the aperture
    # plate at x = 0.8 L, 65536 per call; only on the workloads that have the plate (the
    # emitter reports LEPIC_ERANGE when no wall face lies at xg1)
    i0 = int(round(0.8 * case.nx)) + 1
    emit_ms, e0, e1 = None, 0, 0
    if (case.bcnd[2:case.ny + 1, i0] == 2).any():   # plate nodes inside the box (not a wall row)
        ap = max(5, int(round(40 * case.nx / 2048)))
        Lgrd = case.ny * case.dy - (ap // 2) * case.dy * 3
        js = n_inj * dk.QE * sim.sp.Nm[0] / (case.zmax * Lgrd * case.dt)
        sc.js = js
        sc.ptype_fx, sc.tag_b, sc.ns_Hm, sc.n_holes = 0, -1, 1, 3
        sc.xg1, sc.Lg, sc.Lh = (i0 - 0.5) * case.dx, case.ny * case.dy, (ap // 2) * case.dy
        sc.THm = 1.0
        sim.set_sources(sc)
        e0 = sim.source_tallies()["n_emit"][0]
        emit_ms = timed(lambda: sim.check(lib.lepic_gpu_flux_emitter(ctx, it), "flux_emitter"))
        e1 = sim.source_tallies()["n_emit"][0]
    sim.sync()
    peak, peak_kind = peaks()
    heat_bytes = 8 * n_slots + 4 * n_in + 20 * n_heated
    tally_bytes = 8 * n_slots + 12 * n_in
    heat_gbs = heat_bytes / (heat_ms * 1e-3) / 1e9
    tally_gbs = tally_bytes / (tally_ms * 1e-3) / 1e9
    return {
        "electron_slots": n_slots, "in_region": n_in, "heated_per_call": n_heated,
        "eheating": {"ms": heat_ms, "achieved_gbs": heat_gbs, "frac": heat_gbs / peak,
                     "algorithmic_bytes": heat_bytes, "kernels": "k_eheat + k_finish"},
        "heating_tally": {"ms": tally_ms, "achieved_gbs": tally_gbs, "frac": tally_gbs / peak,
                          "algorithmic_bytes": tally_bytes, "kernels": "k_heat_tally + k_finish"},
        "part_injection": {"ms": inj_ms, "injected_per_call": [(b - a) / (reps + 3) for a, b in zip(c0, c1)],
                           "kernels": "k_inj_plan + k_inject + k_finish"},
        "flux_emitter": ({"ms": emit_ms, "emitted_per_call": (e1 - e0) / (reps + 3), "kernels": "k_emit (one CTA)"}
                         if emit_ms is not None else "no aperture plate in this workload"),
        "peak_gbs": peak, "peak_kind": peak_kind, "calls_timed": reps,
    }


def run_ours(args):
    import torch
    import torch.distributed as dist
    from jd_lepic_b200 import configs, _capi as capi
    from jd_lepic_b200.simulation import GpuSimulation
    import ctypes as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    kw = {"ppc": args.ppc} if args.ppc else {}
    if args.nx:
        kw.update(nx=args.nx, ny=args.nx)
    case = configs.make_case(args.config, **kw)
    # weak scaling with the reference's particle decomposition (load_part.f90:96): the deck's
    # np_cell grows with the ranks, so Nm = n0 Vc / np_cell shrinks by 1/world, and each rank
    # loads np_cell n_cell / world particles (one GPU's workload) with its own seed; the int64
    # all-reduce of rho after each push (calc_rho.f90:71-74) gives every rank the global charge
    case.ppc *= world
    case.nproc_mpi = world
    case.seed = case.seed + 7919 * rank
    sim = GpuSimulation(case, tile=(args.tile, args.tile))
    lib, ctx = sim.lib, sim.ctx
    stream = torch.cuda.ExternalStream(sim.stream_ptr())
    mode = args.mode
    eps = 1e-8

    acc_views = []
    if world > 1:
        for s in range(sim.sp.ntype):
            ptr = C.c_void_p()
            sim.check(lib.lepic_gpu_deposit_grid(ctx, s, C.byref(ptr)), "deposit_grid")
            nn = (case.nx + 3) * (case.ny + 3)

            class _A:
                __cuda_array_interface__ = {"shape": (nn,), "typestr": "<i8", "data": (ptr.value, False),
                                            "version": 3, "stream": sim.stream_ptr()}
            acc_views.append(torch.as_tensor(_A(), device=f"cuda:{local}"))

    def reduce_rho():
        if world > 1:
            with torch.cuda.stream(stream):
                for t in acc_views:
                    dist.all_reduce(t, op=dist.ReduceOp.SUM)

    ev = {}

    def phase(name, it, fn):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        ev.setdefault(name, []).append((it, a, b))

    def one_step(it, timed, solve_mode=None):
        sm = mode if solve_mode is None else solve_mode

        def rec(name, fn):
            if timed:
                phase(name, it, fn)
            else:
                fn()
        rec("rhs", lambda: sim.check(lib.lepic_gpu_calc_rhs(ctx, None), "calc_rhs"))
        rec("poisson", lambda: sim.check(lib.lepic_gpu_iterative_solver(ctx, None, eps, sm, None), "solver"))
        rec("efield", lambda: sim.check(lib.lepic_gpu_calc_efield(ctx, None), "efield"))
        if it % 10 == 1:
            def srt():
                for s in range(sim.sp.ntype):
                    sim.check(lib.lepic_gpu_part_sorting(ctx, s, None), "sort")
            rec("sort", srt)
        if it > 1 and it % 10 == 1:
            rec("mcc", lambda: sim.check(lib.lepic_gpu_collisions(ctx, it, None), "collisions"))
        rec("push_deposit", lambda: sim.check(lib.lepic_gpu_push_deposit(ctx, it, None), "push"))
        rec("allreduce", reduce_rho) if world > 1 else None

    # the mixed solve starts each step from the extrapolation of the last two potentials
    if mode == capi.POISSON_MIXED_IR:
        sim.check(lib.lepic_gpu_set_warm_start(ctx, 1), "set_warm_start")

    # cold solve to a converged phi, then warm-up steps
    clocks = ClockSampler(local)
    clocks.start()
    it = 1
    for _ in range(args.warmup):
        one_step(it, False)
        it += 1
    sim.sync()
    n_start = sum(sim.push_stats()["np_tot"])
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.mark_start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    first_timed = it
    for _ in range(args.steps):
        one_step(it, True)
        it += 1
    t_end.record(stream)
    torch.cuda.synchronize()
    clocks.mark_end()
    sim.sync()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    n_end = sum(sim.push_stats()["np_tot"])
    total_ms = t_start.elapsed_time(t_end)
    if world > 1:
        tt = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    phases = {k: sum(a.elapsed_time(b) for _, a, b in v) for k, v in ev.items()}
    n_avg = 0.5 * (n_start + n_end)
    value = n_avg * args.steps * world / (total_ms * 1e-3)
    push_ms = phases["push_deposit"] / args.steps
    # the push after each sort reads the pending permutation too (lepic_options.sort_defer = 1)
    n_sort_pushes = sum(1 for k in range(first_timed, first_timed + args.steps) if k % 10 == 1)
    bytes_per_launch = (BYTES_PER_PARTICLE_STEP + PERM_BYTES_PER_PARTICLE * n_sort_pushes / args.steps) * n_avg
    peak, peak_kind = peaks()
    achieved = bytes_per_launch / (push_ms * 1e-3) / 1e9
    tpp = profiled_traffic_per_particle()

    # Poisson: plain FP64 multigrid (the reference's V-cycle, stopped on the same L2 criterion)
    # vs FP64 CG preconditioned by the FP32 V-cycle, on the next step's rhs, both from the same
    # warm start (the previous step's phi, as in the time loop) and from a cold start
    sim.check(lib.lepic_gpu_calc_rhs(ctx, None), "calc_rhs")
    phi_save = sim.grid(capi.GRID_PHI)
    phi_cold = np.where(case.bcnd >= 1, case.phi0, 0.0)
    pois = {}
    if mode == capi.POISSON_MIXED_IR:
        # the time loop's start first, while its history is valid: 2 phi_n - phi_(n-1)
        st = capi.LepicSolveStats()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        sim.check(lib.lepic_gpu_iterative_solver(ctx, None, eps, capi.POISSON_MIXED_IR, C.byref(st)), "solver")
        b.record(stream)
        torch.cuda.synchronize()
        pois["mixed_pcg_extrapolated"] = {"ms": a.elapsed_time(b), "cycles": st.cycles, "res_l2_rel": st.res_l2_rel}
    # then both solvers from the previous phi as it is (set_phi forgets the history); a mixed
    # solve first, untimed, when the time loop used another mode: a context's first mixed solve
    # also factors the coarse level's operator (once, on the host)
    for m in (capi.POISSON_MIXED_IR, capi.POISSON_FP64_PCG):
        if m != mode:
            sim.set_phi(phi_save)
            sim.check(lib.lepic_gpu_iterative_solver(ctx, None, eps, m, None), "solver")
    for start, phi0 in (("warm", phi_save), ("cold", phi_cold)):
        for name, m in (("fp64_mg", capi.POISSON_FP64_MG_L2), ("mixed_pcg", capi.POISSON_MIXED_IR),
                        ("fp64_pcg", capi.POISSON_FP64_PCG)):
            sim.set_phi(phi0)
            st = capi.LepicSolveStats()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            sim.check(lib.lepic_gpu_iterative_solver(ctx, None, eps, m, C.byref(st)), "solver")
            b.record(stream)
            torch.cuda.synchronize()
            pois[f"{name}_{start}"] = {"ms": a.elapsed_time(b), "cycles": st.cycles, "res_l2_rel": st.res_l2_rel}
    sim.set_phi(phi_save)
    for start in ("warm", "cold"):
        pois[f"speedup_{start}"] = pois[f"fp64_mg_{start}"]["ms"] / pois[f"mixed_pcg_{start}"]["ms"]
        # the same CG with an FP64 cycle: what the FP32 cycle alone gains
        pois[f"speedup_precision_{start}"] = pois[f"fp64_pcg_{start}"]["ms"] / pois[f"mixed_pcg_{start}"]["ms"]
    if "mixed_pcg_extrapolated" in pois:
        pois["speedup_warm_extrapolated"] = pois["fp64_mg_warm"]["ms"] / pois["mixed_pcg_extrapolated"]["ms"]

    # learned warm start: PIC steps in the learned mode (online training), then an A/B on the
    # following steps -- plain FP64 multigrid, the mixed CG and the learned start, each from the
    # previous step's phi on the same rhs (training off while timed; its cost reported apart)
    if args.learn_steps > 0:
        it = learned_compare(args, sim, lib, ctx, capi, stream, it, eps, pois, one_step)

    # end to end through the C ABI with host buffers: phi exchanged with pinned host memory
    # every step (the Fortran host's array: downloaded after the solve and uploaded again as the
    # next solve's input, both on the copy stream beside the E field and the push) and the
    # particle counters read back
    # (3 untimed steps first: the copy stream, its events and the download snapshot are created
    # at a context's first overlapped copy, and the first mixed solve after the comparison above
    # starts without the extrapolation's history; then 20 timed steps, two sorts among them)
    e2e_steps = min(args.steps, 20)
    nn = (case.nx + 3) * (case.ny + 3)
    phi_host = torch.empty(nn, dtype=torch.float64, pin_memory=True)
    phi_host.copy_(torch.from_numpy(phi_save.ravel()))
    php = C.cast(phi_host.data_ptr(), C.POINTER(C.c_double))
    ps = capi.LepicPushStats()

    def e2e_loop(nsteps):
        nonlocal it
        sim.check(lib.lepic_gpu_stage_solver_input(ctx, php), "stage")   # the first step's input
        for k in range(nsteps):
            sim.check(lib.lepic_gpu_calc_rhs(ctx, None), "calc_rhs")
            sim.check(lib.lepic_gpu_iterative_solver_async(ctx, None, php, eps, mode), "solver")
            sim.check(lib.lepic_gpu_calc_efield(ctx, None), "efield")
            if it % 10 == 1:
                for s in range(sim.sp.ntype):
                    sim.check(lib.lepic_gpu_part_sorting(ctx, s, None), "sort")
            if it > 1 and it % 10 == 1:
                sim.check(lib.lepic_gpu_collisions(ctx, it, None), "collisions")
            if k + 1 < nsteps:   # the next step's input, uploaded beside the push
                sim.check(lib.lepic_gpu_stage_solver_input(ctx, php), "stage")
            sim.check(lib.lepic_gpu_push_deposit(ctx, it, C.byref(ps)), "push")
            reduce_rho()
            it += 1

    e2e_loop(3)
    ne0 = sum(ps.np_tot[:sim.sp.ntype])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    w0 = time.perf_counter()
    e2e_loop(e2e_steps)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - w0
    if world > 1:
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    ne1 = sum(ps.np_tot[:sim.sp.ntype])
    e2e_value = 0.5 * (ne0 + ne1) * e2e_steps * world / e2e_s

    # the deposit alone (charge_deposition over the same particles, as after a load or restart):
    # how much of the fused push+deposit the deposit is; it reads X, Y and VX (the hole test)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(5):
        sim.check(lib.lepic_gpu_charge_deposition(ctx), "charge_deposition")
    b.record(stream)
    torch.cuda.synchronize()
    dep_ms = a.elapsed_time(b) / 5
    n_now = sum(sim.push_stats()["np_tot"])
    deposit_only = {"ms": dep_ms, "particles": n_now, "achieved_gbs": 12.0 * n_now / (dep_ms * 1e-3) / 1e9,
                    "algorithmic_bytes_per_particle": 12, "kernels": "k_push_deposit<MOVE=false> per species"}
    src = sources_measure(args, sim, lib, ctx, stream, it, case) if not args.no_sources else None

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args.config, args.cpu_cells, 5, 2, host_threads())
    line = None
    if rank == 0:
        # kernels of this library launched in the timed steps (memsets/copies not counted), as
        # the ncu launch list shows them: rhs 1, the warm start's extrapolation 1 (mixed mode),
        # Poisson 1 (cooperative), E field 1 (4 with the periodic or Neumann option), push 1 per
        # species; a sort step adds 8 per species
        # (keys, three scan passes, scatter, two segment passes, work items; the records move in
        # the push), a collision step the selection and the collisions per colliding species
        # and the product commit per species
        n_mcc = sum(1 for s in range(sim.sp.ntype) if sim.xs.p_ncol[s] > 0)
        e_launches = 4 if (case.flag_pbc or case.flag_nmn) else 1
        launches = 0
        for t in range(first_timed, first_timed + args.steps):
            launches += 1 + (1 if mode == capi.POISSON_MIXED_IR else 0) + 1 + e_launches + sim.sp.ntype
            if t % 10 == 1:
                launches += 8 * sim.sp.ntype
            if t > 1 and t % 10 == 1:
                launches += 2 * n_mcc + sim.sp.ntype
        line = {
            "metric": "particle-steps/s per PIC step (push+deposit+MCC+sort+Poisson to 1e-8)",
            "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 particles / f64 Poisson residual",
            "data": "synthetic",
            "config": {"workload": case.name, "grid": [case.nx, case.ny],
                       "particles_per_species_per_gpu": case.n_load, "species": sim.sp.ntype,
                       "decomposition": (f"particles split over {world} ranks (load_part.f90:96), np_cell "
                                         f"{case.ppc} in all, Nm = n0 Vc / np_cell, int64 rho all-reduce per step"
                                         if world > 1 else "one rank"),
                       "particles_avg_per_gpu": n_avg, "poisson": {1: "FP64 CG preconditioned by an FP32 V-cycle, relative L2 residual 1e-8, "
                                      "started from 2 phi_(n-1) - phi_(n-2)",
                                   3: "learned warm start + FP64 CG with the FP32 V-cycle, relative L2 "
                                      "residual 1e-8"}.get(mode, "FP64 multigrid"),
                       "l2": "inputs larger than L2 (particle arrays 8.4 GB/species)",
                       "sort_every": 10, "mcc_every": 10, "tile": args.tile},
            "phases_ms_per_step": {k: v / args.steps for k, v in phases.items()},
            "deposit_alone": deposit_only,
            "poisson_compare": pois,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel": "k_push_deposit (both species, incl. accumulator clears)",
                         "algorithmic_bytes_per_particle": bytes_per_launch / n_avg,
                         "traffic": (tpp * n_avg if tpp else None)},
            "cpu_baseline": ({k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")} if cb else None),
            "e2e": {"value": e2e_value, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": 8 * nn, "d2h_bytes_per_step": 8 * nn + C.sizeof(capi.LepicPushStats)},
            "gpu_launches": launches,
            "clocks": clk,
            "sources": src,
        }
        print(json.dumps(line))
    sim.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=4)
    ap.add_argument("--mode", type=int, default=1)
    ap.add_argument("--tile", type=int, default=16)
    ap.add_argument("--cpu-cells", type=int, default=512,
                    help="cells along x of the CPU baseline's sample box (the workload's ppc kept)")
    ap.add_argument("--ppc", type=int, default=0, help="override particles per cell (profiling runs)")
    ap.add_argument("--nx", type=int, default=0, help="override the grid to nx x nx cells (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sources", action="store_true", help="skip the particle-source kernel timings")
    ap.add_argument("--learn-steps", type=int, default=60, help="PIC steps of online training before the A/B")
    ap.add_argument("--learn-ab", type=int, default=4, help="steps of the learned/plain Poisson A/B")
    ap.add_argument("--learn-train-steps", type=int, default=2, help="Adam steps per learned solve")
    ap.add_argument("--learn-crop", type=int, default=256)
    ap.add_argument("--learn-batch", type=int, default=4)
    ap.add_argument("--learn-lr", type=float, default=2e-3)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
