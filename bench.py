#!/usr/bin/env python
"""Benchmark: walker-steps/s and NS iterations/s of the B200 NS walk.

Workload (the batched-replica LJ configuration): 32-atom LJ NPT (eps=sigma=1,
rc=2.5), P=8 runs at pressures log-spaced 0.01-1.0, K=512 walkers each,
n_mcmc_steps=40, galilean (n_reflect=10, step 0.1, weight 4) + volume (step
0.3, weight 1), pressure replica exchange every 10 iterations; uniform-gas
start (cubic cell, V ~ U(0, 8N], fractional coordinates U[0,1)^3) from a
seeded threefry key.  All inputs synthetic.

One step = one launch of 10 NS iterations on all 8 runs (the iterations
between two replica-exchange passes) + the swap pass.  walker-steps/s =
P * (n_cull + n_extra) * n_mcmc_steps * iterations / s.

``--impl reference`` times the reference's algorithm on the host CPU: the
CPU oracle in the reference's own float32 arithmetic (JAX is not installable
here), threaded over the runs.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P_RUNS, K, N, T, R_REFLECT, RE_INTERVAL = 8, 512, 32, 40, 10, 10
PRESSURES = np.logspace(-2, 0, P_RUNS).astype(np.float32)
METRIC = "walker-steps/s"
CONFIG = {
    "workload": "LJ-32 NPT, 8 pressure replicas (0.01-1.0) x 512 walkers, "
                "n_mcmc_steps=40, galilean(n_reflect=10)+volume, RE every 10 iterations",
    "n_runs": P_RUNS, "n_walkers": K, "n_atoms": N, "n_mcmc_steps": T,
    "n_reflect": R_REFLECT, "re_interval": RE_INTERVAL, "n_cull": 1, "n_extra": 0,
    "iterations_per_step": RE_INTERVAL,
}
# per-run atom counts and chemical potentials (the uneven semi-grand workload)
N_LIST = [N] * P_RUNS
MUS = None
RE_ON = True
WORKLOAD = "batched"


def select_workload(name: str) -> None:
    """The default is the batched-replica configuration above.  ``single``:
    one 8-atom LJ NPT run (P = 0.1) of 128 walkers, n_mcmc_steps = 20.
    ``uneven``: 16 semi-grand runs of binary LJ (sigma AA/BB/AB 1/0.88/0.8,
    epsilon 1/0.5/1.5, cutoff 2.5) with atom counts drawn from {16, 24, ..., 96}
    (threefry-seeded), Delta-mu signed-log-spaced in [-2, 2], 1024 walkers,
    species Bernoulli(0.5) from a threefry key, galilean + volume + morph +
    swap, n_mcmc_steps = 40, all runs in one launch.  ``sw``: 4 runs of
    64-atom Stillinger-Weber silicon NPT at 0.1 GPa, 1024 walkers,
    n_mcmc_steps = 40, the LJ move mix with its steps scaled by the SW sigma
    (galilean 0.2 A, volume 2.8 A^3 per atom), uniform gas with V in
    (0, 8 N 20 A^3].  None of these exchanges replicas; a step is 10 NS
    iterations."""
    global P_RUNS, K, N, T, PRESSURES, CONFIG, N_LIST, MUS, RE_ON, WORKLOAD
    global V_PER_ATOM, STEP_SIZES
    WORKLOAD = name
    if name == "batched":
        return
    RE_ON = False
    if name == "single":
        P_RUNS, K, N, T = 1, 128, 8, 20
        N_LIST = [N]
        PRESSURES = np.full(1, 0.1, np.float32)
        desc = ("LJ-8 NPT single run (P=0.1) x 128 walkers, n_mcmc_steps=20, "
                "galilean(n_reflect=10)+volume")
    elif name == "uneven":
        from jaxrens_b200 import prng

        P_RUNS, K, T = 16, 1024, 40
        u = prng.uniform(prng.fold_in(prng.key(96), 0), P_RUNS)
        N_LIST = [int(16 + 8 * np.floor(v * 11)) for v in u]
        N = max(N_LIST)
        PRESSURES = np.full(P_RUNS, 0.1, np.float32)
        dmu = np.concatenate([-np.logspace(np.log10(2.0), -2, 8), np.logspace(-2, np.log10(2.0), 8)])
        MUS = np.stack([np.zeros(P_RUNS), dmu], axis=1).astype(np.float32)
        desc = ("binary LJ semi-grand (Kob-Andersen pair tables), 16 runs with N in "
                "{16..96} x 1024 walkers, Delta-mu in [-2, 2], n_mcmc_steps=40, "
                "galilean(n_reflect=10)+volume+morph+swap")
    elif name in ("sw", "sw_da"):
        from jaxrens_b200.backends import EV_PER_A3_PER_GPA

        P_RUNS, K, N, T = 4, 1024, 64, 40
        N_LIST = [N] * P_RUNS
        PRESSURES = np.full(P_RUNS, 0.1 * EV_PER_A3_PER_GPA, np.float32)
        V_PER_ATOM = 8.0 * 20.0
        STEP_SIZES = (0.2, 2.8)
        desc = ("Stillinger-Weber Si-64 NPT, 4 runs at 0.1 GPa x 1024 walkers, "
                "n_mcmc_steps=40, galilean(n_reflect=10)+volume")
        if name == "sw_da":
            STEP_SIZES = (0.05, 0.5)
            desc = ("Stillinger-Weber Si-64 NPT, 4 runs at 0.1 GPa x 1024 walkers, "
                    "n_mcmc_steps=40, galilean(n_reflect=10, 0.05 A)+volume(0.5 A^3/atom), "
                    "condensed start: diamond cells scaled by up to +-6% in volume, "
                    "atoms displaced uniformly by up to 0.35 A")
    else:
        raise SystemExit(f"unknown workload {name}")
    CONFIG = {"workload": desc, "n_runs": P_RUNS, "n_walkers": K,
              "n_atoms": N_LIST if name == "uneven" else N, "n_mcmc_steps": T,
              "n_reflect": R_REFLECT, "re_interval": None, "n_cull": 1, "n_extra": 0,
              "iterations_per_step": RE_INTERVAL}


V_PER_ATOM = 8.0           # uniform-gas volume bound per atom
STEP_SIZES = (0.1, 0.3)    # galilean, volume
# algorithmic flops per unique pair interaction (triclinic MIC accounting)
FLOPS_EF, FLOPS_E = 61.0, 48.0
# Stillinger-Weber, per pair / triplet inside the cutoff: energy+forces 74 and
# 60, energy only 58 and 12
SW_FLOPS = (74.0, 60.0, 58.0, 12.0)


def condensed_silicon(seed: int, count: int, amp: float = 0.35):
    """``count`` 64-atom silicon cells (2x2x2 conventional diamond cells,
    a = 5.431 A) scaled by (1 + U(-0.06, 0.06))^(1/3) and with every atom
    displaced by U(-amp, amp) A per coordinate: the solid-like walkers of a
    late nested-sampling run (numpy-seeded synthetic data)."""
    rng = np.random.default_rng(seed)
    basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0], [.25, .25, .25],
                      [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    cells = np.array([[i, j, k] for i in range(2) for j in range(2) for k in range(2)])
    x0 = ((cells[:, None, :] + basis[None]).reshape(-1, 3) * 5.431)
    c0 = np.eye(3) * 2 * 5.431
    pos, cel = [], []
    for _ in range(count):
        f = (1.0 + rng.uniform(-0.06, 0.06)) ** (1.0 / 3.0)
        pos.append(x0 * f + rng.uniform(-amp, amp, x0.shape))
        cel.append(c0 * f)
    return np.asarray(pos, np.float32), np.asarray(cel, np.float32)


def build_case(seed: int):
    from jaxrens_b200 import EnsembleTerm, Hamiltonian, build_mwg, create_lj, create_sw, prng
    from jaxrens_b200 import init as jinit
    from jaxrens_b200 import moves as mvs

    if WORKLOAD == "uneven":
        model = create_lj(epsilon=[[1.0, 1.5], [1.5, 0.5]], sigma=[[1.0, 0.8], [0.8, 0.88]],
                          cutoff=2.5)
    elif WORKLOAD in ("sw", "sw_da"):
        model = create_sw()
    else:
        model = create_lj(epsilon=1.0, sigma=1.0, cutoff=2.5)
    H = Hamiltonian(model, [EnsembleTerm(pressure=float(PRESSURES[0]))])
    moves = [mvs.gmc(n_reflect=R_REFLECT, step_size=STEP_SIZES[0], weight=4.0),
             mvs.volume_move(N, step_size=STEP_SIZES[1], weight=1.0)]
    if WORKLOAD == "uneven":
        moves += [mvs.morph_move(2, weight=1.0), mvs.swap_move(2, weight=1.0)]
    init_fn, step, _ = build_mwg(H, moves)
    root = prng.key(seed)
    keys = prng.split(root, P_RUNS + 3)
    pos, cells = [], []
    for r in range(P_RUNS):
        if WORKLOAD == "sw_da":
            p_, c_ = condensed_silicon(seed * 1000 + r, K)
        else:
            p_, c_ = jinit.uniform_gas(keys[r], K, N_LIST[r], V_PER_ATOM * N_LIST[r])
        pos.append(p_)
        cells.append(c_)
    if WORKLOAD == "uneven":
        # species Bernoulli(0.5), walker-major, from one threefry key per run
        tkeys = prng.split(keys[P_RUNS + 2], P_RUNS)
        types = [prng.bernoulli(tkeys[r], K * n, 0.5).astype(np.int32).reshape(K, n)
                 for r, n in enumerate(N_LIST)]
    else:
        types = [np.zeros((K, N), np.int32) for _ in range(P_RUNS)]
    run_keys = prng.split(keys[P_RUNS], P_RUNS)
    return H, init_fn, step, pos, cells, types, run_keys, keys[P_RUNS + 1]


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None
        self.first = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "10"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a while to print its first line: wait for it so
            # that a short timed region still falls inside the sampling
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except (OSError, FileNotFoundError):
            self.proc = None
        self.first = len(self.lines)

    def mark(self) -> None:
        """The timed region starts now: stop() keeps the samples from here."""
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        window = "timed region"
        lines = self.lines[self.first:]
        if not lines:
            # a timed region shorter than the sampling period: the samples
            # just before it (warm-up steps of the same workload)
            lines = self.lines[max(0, self.first - 3):]
            window = "warm-up steps just before the timed region"
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


def fp32_peak_tflops(torch) -> float:
    """Measured FP32 FMA-pipe throughput (probe kernel, best of 5)."""
    from jaxrens_b200 import _lib

    L = _lib.load()
    dev = torch.device("cuda")
    scratch = torch.zeros(148 * 64, dtype=torch.float32, device=dev)
    fl = C.c_double(0.0)
    s = torch.cuda.current_stream().cuda_stream
    blocks = 148 * 8
    _lib.check(L.jr_bench_fma_peak(blocks, 2000, C.c_void_p(scratch.data_ptr()), C.byref(fl), s), "fma")
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check(L.jr_bench_fma_peak(blocks, 2000, C.c_void_p(scratch.data_ptr()), C.byref(fl), s), "fma")
        e1.record()
        e1.synchronize()
        best = max(best, fl.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def rank_seed(seed: int, rank: int) -> int:
    """Each rank owns its own P runs (replicas only: no data-path exchange),
    seeded apart so no two ranks walk the same runs."""
    return seed + 1000 * rank


def max_over_ranks(ms: float, world: int, device) -> float:
    """The job's time is the slowest rank's device time."""
    if world == 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, iters: int, total_ms: float) -> tuple[float, float]:
    """Whole-job walker-steps/s and NS iterations/s: every rank's P runs,
    (n_cull + n_extra) * n_mcmc_steps walker-steps per run iteration."""
    walker_steps = world * P_RUNS * 1 * T * iters
    return walker_steps / (total_ms * 1e-3), world * P_RUNS * iters / (total_ms * 1e-3)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from jaxrens_b200 import _lib, prng
    from jaxrens_b200 import nested_sampling as nsm

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)

    H, init_fn, step, pos, cells, types, run_keys, re_key = build_case(rank_seed(args.seed, rank))
    pr = {"pressure": PRESSURES}
    if MUS is not None:
        pr["chemical_potentials"] = MUS
    ns = nsm.init_ns_parallel(init_fn, pos, types, None, cells, run_keys, ensemble_params=pr)
    re = nsm.InterREManager(RE_INTERVAL, 1, re_key)
    cfg = None
    if args.cluster is not None:
        cfg = _lib.JrLaunchConfig(args.threads, args.tpa, args.cluster, int(args.warp))
    # prologue: leave the random-gas start before measuring (untimed)
    info = nsm.InfoBuffers(ns, step.n_moves, RE_INTERVAL, dead=True)
    for _ in range(args.prologue // RE_INTERVAL):
        nsm.ns_iterate(ns, step, RE_INTERVAL, T, 0, info=info, cfg=cfg)
        if RE_ON:
            re.apply(ns, step)
    torch.cuda.synchronize()
    if args.tune and cfg is None:
        # tuned on the walkers past the prologue, the state the timed steps see
        best = _lib.JrLaunchConfig()
        dims = nsm.make_dims(ns, step, T, 0)
        la = nsm.prior_mass.log_alpha(K, 1)
        params = step.with_evidence(la, float(nsm.prior_mass.iteration_offsets(K, 1)[1][0]))
        sb = nsm.state_buffers(ns)
        _lib.check(_lib.load().jr_autotune(C.byref(dims), C.byref(params), C.byref(sb), 10,
                                           C.byref(best), torch.cuda.current_stream().cuda_stream),
                   "jr_autotune")
        cfg = best
    torch.cuda.synchronize()

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def one_step(record):
        if record is not None:
            record[0].record()
        nsm.ns_iterate(ns, step, RE_INTERVAL, T, 0, info=info, cfg=cfg)
        if record is not None:
            record[1].record()
        if RE_ON:
            re.apply(ns, step)

    # the clock sampler runs from the warm-up on; its samples from the start
    # of the timed region are the ones reported
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        one_step(None)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks.mark()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    # The host enqueues step k+1 while step k runs (no per-step synchronize),
    # so the host-side launch work never leaves the GPU idle inside a step's
    # events; each step's evaluation counts are folded into a device-side
    # flop total outside the events.
    flops_dev = torch.zeros((), dtype=torch.float64, device=dev)      # executed
    flops_ref_dev = torch.zeros((), dtype=torch.float64, device=dev)  # reference accounting
    pairs_dev = torch.tensor([n * (n - 1) / 2.0 for n in N_LIST], dtype=torch.float64, device=dev)
    sw_flops_dev = torch.tensor(SW_FLOPS, dtype=torch.float64, device=dev)
    rounds_dev = torch.zeros((), dtype=torch.float64, device=dev)
    it_start = ns.iteration.clone()
    for k in range(args.steps):
        flush.fill_(float(k))  # evict the (L2-resident) walker state between steps
        evs[k][0].record()
        one_step(ev[k])
        evs[k][1].record()
        rounds_dev += info.rounds.sum(dtype=torch.float64)
        # executed work, counted by the kernel: pairs (and SW triplets)
        # evaluated with forces, then energy-only
        tc = info.term_counts.sum(dim=(0, 1), dtype=torch.float64)
        if WORKLOAD == "sw":
            flops_dev += (tc * sw_flops_dev).sum()
        else:
            flops_dev += tc[0] * FLOPS_EF + tc[2] * FLOPS_E
            # the reference's accounting: n_reflect energy+force evaluations
            # per galilean step, one energy-only per other step
            ne = info.n_evaluations.sum(dim=(0, 2), dtype=torch.float64)
            ng = info.n_grad_evaluations.sum(dim=(0, 2), dtype=torch.float64)
            flops_ref_dev += ((ng * FLOPS_EF + (ne - ng) * FLOPS_E) * pairs_dev).sum()
    torch.cuda.synchronize()
    flops = float(flops_dev.item())
    flops_ref = float(flops_ref_dev.item())
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    iters = int((ns.iteration - it_start)[0].item())
    assert iters == args.steps * RE_INTERVAL
    total_ms = max_over_ranks(total_ms, world, dev)
    value, ns_iters = job_throughput(world, iters, total_ms)
    achieved = flops / (sum(kern_ms) * 1e-3) / 1e12
    peak = fp32_peak_tflops(torch)

    # ---- end to end: host state in, result out, through the public API ----
    e2e = end_to_end(args, ns, step, re, cfg, torch, nsm)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cpu = cpu_baseline(args) if (world == 1 and not args.no_cpu) else None
    traffic = None
    prof = os.path.join(ROOT, "profiles", "ns_iterate_kernel_lj32_8x512.json")
    if WORKLOAD == "batched" and os.path.exists(prof):
        traffic = json.load(open(prof)).get("dram_bytes_per_launch")
    line = {
        "metric": METRIC, "value": value, "unit": "walker-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair terms, f64 accumulation", "data": "synthetic",
        "config": dict(CONFIG),
        "parallelism": f"replicas x{world} GPUs",
        "l2": "flushed (256 MiB write) between timed steps",
        "launch": None if cfg is None else {"threads": cfg.threads, "tpa": cfg.tpa,
                                            "cluster": cfg.cluster,
                                            "warp_walkers": cfg.warp_walkers,
                                            "source": "jr_autotune" if args.tune else "flags"},
        "ns_iters_per_s": ns_iters, "ns_iters_per_s_per_run": ns_iters / (world * P_RUNS),
        "speculation_rounds_per_launch": float(rounds_dev.item()) / (args.steps * P_RUNS),
        "e2e": e2e,
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None, "traffic": traffic,
                     "traffic_unit": "DRAM bytes per ns_iterate_kernel launch (ncu capture)",
                     "peak_source": "measured FP32 FMA probe (jr_bench_fma_peak) on this GPU",
                     "peak_nominal": 148 * 128 * 2 * 1.965e-3,
                     "kernel": "ns_iterate_kernel", "flops_per_step": flops / args.steps,
                     "flops_accounting": "executed: pairs (and triplets) the kernel evaluated, "
                                         "forces only on reflecting galilean steps",
                     "flops_per_step_reference_accounting":
                         (flops_ref / args.steps) if WORKLOAD != "sw" else None},
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


def end_to_end(args, ns, step, re, cfg, torch, nsm):
    """Each step: a pinned-host state -> device (one copy), 10 iterations +
    swap through the public API, per-iteration results (dead energies, log Z)
    -> host.  The host holds n_snap consecutive states of the run and step k
    starts from state k mod n_snap, so the steps sample different trajectories
    (and speculation outcomes) as the device-resident steps do.  Two device
    copies of the state alternate, so the upload of step k+1 (on a copy
    stream) overlaps the walk of step k; every step starts from its own
    upload."""
    import dataclasses

    pop = ns.population
    names_p = ["positions", "direction", "types", "energy", "energy64", "cell", "step_sizes",
               "n_accepted", "n_proposed"]
    names_s = ["rng_key", "log_evidence", "iteration", "emax"]
    fields = [getattr(pop, k) for k in names_p] + [getattr(ns, k) for k in names_s]
    # the whole state in one pinned host buffer and one device buffer (fields
    # 256-byte aligned), so each step uploads it with a single copy; the
    # state the API works on is views into the device buffer
    offs, off = [], 0
    for f in fields:
        off = (off + 255) // 256 * 256
        offs.append(off)
        off += f.numel() * f.element_size()
    bufs = []
    for _ in range(2):
        flat_dev = torch.empty(off, dtype=torch.uint8, device=pop.positions.device)
        views = [flat_dev[o:o + f.numel() * f.element_size()].view(f.dtype).view(f.shape)
                 for f, o in zip(fields, offs)]
        pop_b = dataclasses.replace(pop, **dict(zip(names_p, views[:len(names_p)])))
        ns_b = dataclasses.replace(ns, population=pop_b, **dict(zip(names_s, views[len(names_p):])))
        bufs.append((flat_dev, ns_b))
    h2d = off
    info = nsm.InfoBuffers(bufs[0][1], step.n_moves, RE_INTERVAL, dead=False)
    # consecutive states (one step apart) in pinned host memory, as many as
    # the timed steps up to 32 (128 MB), so the end-to-end mean covers as many
    # trajectories as the device-resident one
    n = max(30, args.steps // 2)
    n_snap = min(n, 32)
    for f, v in zip(fields, [getattr(bufs[0][1].population, k) for k in names_p] +
                    [getattr(bufs[0][1], k) for k in names_s]):
        v.copy_(f)
    flat_host = []
    for _ in range(n_snap):
        h = torch.empty(off, dtype=torch.uint8).pin_memory()
        h.copy_(bufs[0][0])
        flat_host.append(h)
        nsm.ns_iterate(bufs[0][1], step, RE_INTERVAL, T, 0, info=info, cfg=cfg)
        if RE_ON:
            re.apply(bufs[0][1], step)
    out_e = torch.empty((RE_INTERVAL, P_RUNS), dtype=torch.float64).pin_memory()
    out_z = torch.empty((RE_INTERVAL, P_RUNS), dtype=torch.float64).pin_memory()
    d2h = out_e.numel() * 8 + out_z.numel() * 8
    main = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    uploaded = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]

    def upload(k):
        b = k % 2
        with torch.cuda.stream(copy):
            copy.wait_event(consumed[b] if k >= 2 else t0)
            bufs[b][0].copy_(flat_host[k % n_snap], non_blocking=True)
            uploaded[b].record(copy)

    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    upload(0)
    for k in range(n):
        b = k % 2
        if k + 1 < n:
            upload(k + 1)
        main.wait_event(uploaded[b])
        nsm.ns_iterate(bufs[b][1], step, RE_INTERVAL, T, 0, info=info, cfg=cfg)
        if RE_ON:
            re.apply(bufs[b][1], step)
        consumed[b].record(main)
        out_e.copy_(info.emax, non_blocking=True)
        out_z.copy_(info.log_evidence, non_blocking=True)
    t1.record()
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"value": world * P_RUNS * T * RE_INTERVAL * n / (ms * 1e-3), "unit": "walker-steps/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": n,
            "pipeline": "state upload of step k+1 on a copy stream overlaps the walk of step k",
            "inputs": f"{n_snap} consecutive host states of the run, cycled"}


class ReferenceRun:
    """The reference algorithm on host cores: the CPU oracle in the
    reference's float32 op order, the runs threaded, replica exchange every
    ``RE_INTERVAL`` iterations like the GPU arm.  The case is built once and
    walked through the same untimed prologue as the GPU arm; ``iterate(n)``
    advances every run by n NS iterations and returns the seconds it took."""

    def __init__(self, seed: int, threads: int, prologue: int):
        from jaxrens_b200 import prior_mass
        from jaxrens_b200 import nested_sampling as nsm
        from oracle import oracle as O
        from tests._cases import oracle_model, oracle_moves

        H, init_fn, step, pos, cells, types, run_keys, re_key = build_case(seed)
        self.re = nsm.InterREManager(RE_INTERVAL, 1, re_key)
        self.done = 0
        self.O, self.threads = O, threads
        self.model, self.moves = oracle_model(H), oracle_moves(step)
        self.reps = []
        for r in range(P_RUNS):
            mu = None if MUS is None else MUS[r]
            e = np.array([O.energy(self.model, pos[r][k], types[r][k], cells[r][k],
                                   pressure=float(PRESSURES[r]), mu=mu, mode=O.REF32,
                                   forces=False)[0]
                          for k in range(K)])
            self.reps.append(O.Replica(pos[r], types[r], e, cells[r],
                                       np.tile(step.default_step_sizes, (K, 1)), run_keys[r],
                                       pressure=float(PRESSURES[r]), mu=mu))
        self.la = prior_mass.log_alpha(K, 1)
        self.wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
        self.iterate(prologue)  # past the random-gas start, untimed

    def iterate(self, n: int) -> float:
        t0 = time.perf_counter()
        for _ in range(n):
            self.O.ns_step_batched(self.model, self.moves, self.reps, T, self.la, self.wo,
                                   shared_move_key=True, mode=self.O.REF32,
                                   n_threads=self.threads)
            self.done += 1
            if RE_ON and self.done % RE_INTERVAL == 0:
                self.O.re_step(self.reps, self.re.next_swap_key(), 1, mode=self.O.REF32)
        return time.perf_counter() - t0


def host_cpu() -> dict:
    """The host's logical CPU count and model name (from /proc/cpuinfo)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"host_cpus": os.cpu_count(), "cpu_model": model}


def cpu_baseline(args):
    threads = min(os.cpu_count() or 1, P_RUNS)
    dt = ReferenceRun(args.seed, threads, args.prologue).iterate(args.cpu_iters)
    return {"value": P_RUNS * T * args.cpu_iters / dt, "unit": "walker-steps/s",
            "cores": threads, "kind": "port", **host_cpu(),
            "sample": f"{args.cpu_iters} NS iterations x {P_RUNS} runs (after the same "
                      f"{args.prologue}-iteration untimed prologue as the GPU arm), "
                      f"{dt:.1f} s, CPU oracle in the reference's float32 op order"}


def run_reference(args):
    """Reference arm: each step is a bounded sample of the workload (every run
    advanced by cpu_iters / steps NS iterations), warm-up steps untimed."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = min(os.cpu_count() or 1, P_RUNS)
    ref = ReferenceRun(args.seed, threads, args.prologue)
    per_step = max(1, args.cpu_iters // max(1, args.steps))
    for _ in range(args.warmup):
        ref.iterate(per_step)
    dt = sum(ref.iterate(per_step) for _ in range(max(1, args.steps)))
    n_iter = per_step * max(1, args.steps)
    value = P_RUNS * T * n_iter / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "walker-steps/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(CONFIG),
        "parallelism": f"{threads} host threads over runs",
        "cpu_baseline": {"value": value, "unit": "walker-steps/s", "cores": threads,
                         "kind": "port", **host_cpu(),
                         "sample": f"{per_step} NS iterations x {P_RUNS} runs per step, "
                                   f"{dt:.1f} s timed; reference algorithm (CPU oracle, "
                                   "reference float32 op order); JAX is not installable on "
                                   "this image"},
        "e2e": {"value": value, "unit": "walker-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _da_arm(name, ns, step, n_steps, walk, torch):
    """Time n_steps steps of RE_INTERVAL iterations of ``walk(ns)`` (which
    returns the step's info buffers), with an L2 flush between steps; the
    counters summed over the steps."""
    dev = ns.rng_key.device
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(n_steps)]
    M = step.n_moves
    acc = torch.zeros(M, dtype=torch.float64, device=dev)
    prop = torch.zeros(M, dtype=torch.float64, device=dev)
    nev = torch.zeros(M, dtype=torch.float64, device=dev)
    nsur = torch.zeros(M, dtype=torch.float64, device=dev)
    for k in range(n_steps):
        flush.fill_(float(k))
        ev[k][0].record()
        info = walk(ns)
        ev[k][1].record()
        acc += info.n_accepted.sum(dim=(0, 1), dtype=torch.float64)
        prop += info.n_proposed.sum(dim=(0, 1), dtype=torch.float64)
        nev += info.n_evaluations.sum(dim=(0, 1), dtype=torch.float64)
        if getattr(info, "n_surrogate_evaluations", None) is not None:
            nsur += info.n_surrogate_evaluations.sum(dim=(0, 1), dtype=torch.float64)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    ws = n_steps * RE_INTERVAL * P_RUNS * T
    return {"arm": name, "value": ws / (ms * 1e-3), "ms_per_step": ms / n_steps,
            "accepted_steps_per_s": float(acc.sum()) / (ms * 1e-3),
            "acceptance_per_move": (acc / prop).tolist(),
            "exact_evaluations_per_walker_step": float(nev.sum()) / ws,
            "exact_evaluations_per_move_step": (nev / prop).tolist(),
            "surrogate_evaluations_per_walker_step": float(nsur.sum()) / ws,
            "mean_contour_after": float(ns.emax.double().mean())}


def train_kernel_roofline(drv, torch):
    """Achieved bfloat16 tensor throughput of one surrogate training step
    (`jr_sur_train_step`, tcgen05) on the driver's minibatch of ring
    configurations of 64 atoms (and, beside it, on 4096 configurations):
    algorithmic flops = 3 x 2 x 5,184 multiply-adds per atom (forward, and a
    backward of twice the forward) over the batch's atoms, divided by the
    median CUDA-event duration of 20 steps.  The peak is the measured cuBLAS
    bf16 figure of the machine when present, else the 1.59 PFLOP/s fallback."""
    from jaxrens_b200.surrogate import Surrogate

    idx = drv.ring.recent_valid(drv.train_window)
    N = drv.ring.n_atoms_max

    def step_ms(B):
        pick = idx[torch.randint(0, idx.numel(), (B,), generator=drv.gen, device=idx.device)]
        D = Surrogate.descriptors(drv.ring.positions[pick], drv.ring.cell[pick])
        U = drv.ring.energy_u[pick].contiguous()
        rows = torch.arange(B, dtype=torch.int32, device=idx.device)
        times = []
        for _ in range(20):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            drv.sur.train_step(D, U, rows, 0.0)
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b))
        return sorted(times)[len(times) // 2]

    B = drv.batch
    ms = step_ms(B)
    ms_big = step_ms(4096)
    flops = 3 * 2 * 5184 * B * N
    flops_big = 3 * 2 * 5184 * 4096 * N
    peak, source = 1590.0, "fallback 1.59 PFLOP/s bf16"
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            peak = float(json.load(open(path))["bf16_tflops"])
            source = "measured (MEASURED_PEAKS.json bf16_tflops)"
        except (KeyError, ValueError, TypeError):
            pass
    achieved = flops / (ms * 1e-3) / 1e12
    big = flops_big / (ms_big * 1e-3) / 1e12
    return {"bound": "tensor", "kernel": "sur_train_kernel", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
            "batch": B, "ms_per_step": ms, "flops_per_step": flops, "peak_source": source,
            "batch_4096": {"achieved": big, "frac": big / peak, "ms_per_step": ms_big}}


def run_da(args):
    """The Stillinger-Weber workload walked by delayed acceptance on the
    learned surrogate, beside the exact walk from the same state.  After the
    (exact, untimed) prologue the surrogate is bootstrapped from the live
    walkers and the prologue's dead walkers; the timed DA steps include the
    online training (16 Adam steps of 256 ring samples every 200 iterations)
    and its recalibration.  Arms: da (trained), da_untrained (normalisation
    only), exact."""
    import torch

    from jaxrens_b200 import delayed_acceptance as da
    from jaxrens_b200 import nested_sampling as nsm
    from jaxrens_b200.surrogate import Surrogate

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    H, init_fn, step, pos, cells, types, run_keys, _ = build_case(args.seed)
    ns = nsm.init_ns_parallel(init_fn, pos, types, None, cells, run_keys,
                              ensemble_params={"pressure": PRESSURES})
    info = nsm.InfoBuffers(ns, step.n_moves, RE_INTERVAL, dead=True)
    dx, dc = [], []
    for _ in range(args.prologue // RE_INTERVAL):
        nsm.ns_iterate(ns, step, RE_INTERVAL, T, 0, info=info)
        dx.append(info.dead_positions.reshape(-1, N, 3).clone())
        dc.append(info.dead_cell.reshape(-1, 3, 3).clone())
    torch.cuda.synchronize()
    ns_exact, ns_untr = ns.clone(), ns.clone()
    drv = da.DelayedAcceptanceNS(ns, step, n_mcmc_steps=T, ring_capacity=100_000,
                                 train_every=200, train_steps=16, batch=256, lr=1e-3,
                                 bootstrap_steps=600, shift_sigmas=args.shift_sigmas,
                                 seed=args.seed)
    t0 = time.time()
    drv.bootstrap(torch.cat(dx) if dx else None, torch.cat(dc) if dc else None)
    torch.cuda.synchronize()
    boot_s = time.time() - t0
    untr = Surrogate(seed=args.seed + 1)
    untr.in_scale, untr.in_shift = drv.sur.in_scale, drv.sur.in_shift
    untr.out_scale, untr.out_shift = drv.sur.out_scale, drv.sur.out_shift
    untr.tau, untr.contour_shift = drv.sur.tau, drv.sur.contour_shift

    def walk_da(s):
        out = drv.run(RE_INTERVAL, block=RE_INTERVAL)
        return out

    def walk_untr(s):
        return da.ns_iterate_da(s, step, untr, RE_INTERVAL, T)

    def walk_exact(s):
        return nsm.ns_iterate(s, step, RE_INTERVAL, T, 0)

    for _ in range(args.warmup):
        walk_da(ns)
        walk_untr(ns_untr)
        walk_exact(ns_exact)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    arms = [_da_arm("da", ns, step, args.steps, walk_da, torch),
            _da_arm("da_untrained", ns_untr, step, args.steps, walk_untr, torch),
            _da_arm("exact", ns_exact, step, args.steps, walk_exact, torch)]
    clk = clocks.stop()
    # one training round on its own (16 Adam steps and the recalibration),
    # the median of 3 host-timed rounds with the device drained around each
    rounds = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        drv.train(drv.train_steps)
        torch.cuda.synchronize()
        rounds.append((time.perf_counter() - t0) * 1e3)
    train_ms = sorted(rounds)[1]
    tensor = train_kernel_roofline(drv, torch)
    line = {
        "metric": METRIC, "value": arms[0]["value"], "unit": "walker-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": arms[0]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 SW terms, bf16 surrogate products with f32 accumulation",
        "data": "synthetic", "config": dict(CONFIG, walk="delayed acceptance"),
        "l2": "flushed (256 MiB write) between timed steps",
        "surrogate": {"bootstrap_s": boot_s, "train_round_ms": train_ms,
                      "train_every_iterations": drv.train_every,
                      "contour_shift": drv.sur.contour_shift,
                      "tau": drv.sur.tau, "ring_samples": drv.ring.reserved},
        "arms": arms,
        "roofline": tensor,
        "da_over_exact": arms[0]["value"] / arms[2]["value"],
        "clocks": clk,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--prologue", type=int, default=200)
    ap.add_argument("--cpu-iters", type=int, default=None,
                    help="NS iterations of the CPU samples (default: 2000, 200 for sw)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shift-sigmas", type=float, default=0.0,
                    help="sw_da: surrogate contour moved inside by this many robust "
                         "standard deviations of the surrogate's error")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip jr_autotune (by default it picks the launch shape once, "
                         "after the prologue and outside the timed region)")
    ap.add_argument("--cluster", type=int, default=None)
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--tpa", type=int, default=8)
    ap.add_argument("--warp", type=int, default=0)
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "single", "uneven", "sw", "sw_da"],
                    help="batched (default, the headline line), or the single-run, uneven "
                         "semi-grand and Stillinger-Weber configurations")
    args = ap.parse_args()
    select_workload(args.workload)
    if args.cpu_iters is None:
        args.cpu_iters = {"sw": 200, "uneven": 100}.get(args.workload, 2000)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "sw_da":
        run_da(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
