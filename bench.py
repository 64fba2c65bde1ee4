#!/usr/bin/env python
"""Benchmark of the KAOS kinetic particle loop on B200.

Workload (one line per run, rank 0 prints JSON): the precision A/B tube --
L = 4 dipole flux tube from 1000 km to |q| = 1e-3, 256 cells, 3D velocity grid
48x48x64 (geometric), 1e7 O+ macro-ions (seeded synthetic Maxwellian,
T = 0.3 eV, n0 = 1e10 m^-3, H = 300 km), wave heating on (chi = 1.7,
1e-3 eV/s at the base), ion-neutral collisions on, dt = 0.005 s, master
step every 20 steps (boundary removal/injection, ambipolar field, counts and
moments), so that the timed window holds whole master intervals (the
reference's own cadence, the lower-boundary cell transit time over h, is
~2000 steps on this tube).

A "step" is one computational step of every particle of the tube.  The
metric is particle-steps/s (higher is better).  `value` is the mixed-
precision path; the FP64 path is timed beside it (`fp64`).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank advances its own tube
(tubes are independent in the reference: species/tube loops are outermost,
_8_KineticSolver.f90:43-44): weak scaling, no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s, mixed-prec vs FP64 on 1 B200, at stated moment error"
N_PART = 10_000_000
# master-step cadence of the timed runs (the reference's own cadence, the
# lower-boundary cell transit time over h, is ~2000 steps on this tube); a
# 20-step window after the warm-up holds one whole master interval
NDATFAC = 20
# the per-moment error runs: the configuration's 500 steps
ERR_STEPS = 500
# algorithmic bytes per ion-step frozen for the mixed path when its state
# was FP32 (cell + FP32 offset, FP32 velocities and fields, 20 B read + 20 B
# written + 8 B of fields)
FROZEN_MIXED_BYTES = 48

# F_alg: FP64 flop-equivalents of one ion push-step of the reference
# formulation on this tube, counted by the op-counting build of the oracle
# (add 176, mul 554, div 158, sqrt 22, transcendental calls 41; weights
# add/mul 1, div/sqrt 4, transcendental 20).
F_ALG = 2270
FP64_NOMINAL_TFLOPS = 37.0  # B200 FP64, nominal; no FP64 figure is measured


def fp64_pipe_roofline(rate_per_gpu):
    """The FP64 path against the FP64 pipe: ion-steps/s x F_alg."""
    achieved = rate_per_gpu * F_ALG / 1e12
    return {"bound": "fp64", "achieved": achieved, "peak": FP64_NOMINAL_TFLOPS,
            "unit": "TFLOP/s (flop-equivalents)", "frac": achieved / FP64_NOMINAL_TFLOPS,
            "peak_kind": "nominal", "f_alg": F_ALG,
            "weights": "add/mul 1, div/sqrt 4, transcendental call 20"}


def clocks_sampler(stop, out):
    """nvidia-smi clocks during the timed region (one sample per 200 ms)."""
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "200"], stdout=subprocess.PIPE, text=True)
    except Exception:
        return
    dev = os.environ.get("LOCAL_RANK", "0")
    while not stop.is_set():
        line = p.stdout.readline()
        if not line:
            break
        f = [x.strip() for x in line.split(",")]
        if f and f[0] == dev:
            out.append(f)
    p.terminate()


def summarize_clocks(samples):
    if not samples:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
    mx = [float(s[2]) for s in samples if s[2].replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[k] for s in samples for k in range(4)
                      if len(s) > 5 + k and s[5 + k].lower().startswith("active")})
    return {"sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None, "reasons": reasons}


def with_clocks(fn, *a):
    """fn(*a) with nvidia-smi clocks sampled while it runs; returns (result,
    clocks summary)."""
    stop, samples = threading.Event(), []
    th = threading.Thread(target=clocks_sampler, args=(stop, samples), daemon=True)
    th.start()
    try:
        r = fn(*a)
    finally:
        stop.set()
        th.join(timeout=5)
    return r, summarize_clocks(samples)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_workload(precision, n_part=N_PART, heating=True, collisions=True,
                   ndatfac=NDATFAC):
    from kaos_b200 import grids
    mi, spec, tube, vg = grids.config_c2(n_particles=n_part, heating=heating,
                                         collisions=collisions,
                                         precision=precision, ndatfac=ndatfac)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=20261203)
    return mi, spec, tube, vg, (q, vpar, v1, v2)


def bytes_per_particle_step(mixed, heating, collisions):
    """Algorithmic HBM bytes per ion per ordinary step (reads + writes).
    `collisions`: the charge exchange converts ions in this interval (an
    idle interval -- no converting cell, no ENA -- stores no Qindk1 or k4
    point at its ordinary steps)."""
    if mixed:  # FP64 state: cell coordinate, V||, (Vperp1, Vperp2); FP32 AEA, AG
        rd, wr = 8 + 8 + 16 + 8, 8 + 8 + (16 if heating else 0)
        if collisions:  # Qindk1 + q at k4 (FP32) written for the charge exchange
            wr += 8
    else:      # rho, z, V||, Vperp1, Vperp2, AEA, AG (8 B) + Qindk1 (4 B)
        rd, wr = 7 * 8 + 4, (5 if heating else 3) * 8 + 4
        if collisions:  # q, rho, z at k4
            wr += 24
    if heating:  # the 64-bit ion id keys the Philox stream of the kicks
        rd += 8
    return rd + wr


def profiled_traffic(name):
    """DRAM bytes per ion-step of a push kernel from its committed ncu
    summary (the `traffic_bytes_per_ion:` line), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_ion:"):
                    return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


# master steps between two compactions of the ion arrays in the library
COMPACT_EVERY = 8


def graph_warmup(args, ndatfac):
    """Warm-up steps of a run replayed from CUDA graphs: every kind of step
    graph (run lengths, master and next-master steps, both ENA and both ion
    buffer parities, the compacting master step of each) is captured before
    the timed steps, which then only replay -- through two compactions and
    three more master intervals; at least --warmup."""
    return max(args.warmup, (2 * COMPACT_EVERY + 3) * ndatfac)


def run_ours(args, precision, graph=False, ndatfac=NDATFAC, steps=None):
    from kaos_b200 import build as kbuild
    from kaos_b200.lib import Solver
    kbuild.build()
    steps = args.steps if steps is None else steps
    mi, spec, tube, vg, init = build_workload(precision, args.particles,
                                              heating=not args.no_heating,
                                              collisions=args.collisions,
                                              ndatfac=ndatfac)
    s = Solver(mi, [tube], vg)
    t0 = time.perf_counter()
    s.load(0, *init)
    t_load = time.perf_counter() - t0
    s.set_graph(graph)
    if args.launch:
        s.set_launch(*(int(x) for x in args.launch.split(",")))
    s.step(graph_warmup(args, ndatfac) if graph else args.warmup)
    n0, _ = s.count()
    # --- device-timed region: K steps in one call (CUDA events on the
    # library's stream; inputs 0.5-1 GB > L2, so no explicit flush) --------
    s.step(steps)
    ms, launches = s.timing()
    pms, pl = s.push_timing()  # events around each push launch
    n1, ne = s.count()
    nmean = 0.5 * (n0 + n1)
    value = nmean * steps / (ms * 1e-3)
    push_ms = pms / max(pl, 1)
    return dict(value=value, ms=ms, launches=launches, n=nmean, push_ms=push_ms,
                t_load=t_load, solver=s, init=init, tube=tube, mi=mi,
                launch=s.launch(), enas=ne)


def run_large(args, precision, steps):
    """The large single tube (L=6, 512 cells, 64x64x96, 1e8 O+ with a kappa
    tail, generated on the device), mixed or FP64 path, steps replayed from
    CUDA graphs."""
    from kaos_b200 import grids
    from kaos_b200.lib import Solver
    mi, spec, tube, vg = grids.config_c3(args.large_particles, precision=precision,
                                         ndatfac=NDATFAC)
    s = Solver(mi, [tube], vg)
    s.init_particles(0, tube._counts, seed=20261203, **grids.C3_TAIL)
    s.set_graph(True)
    if args.launch:
        s.set_launch(*(int(x) for x in args.launch.split(",")))
    s.step(graph_warmup(args, mi.ndatfac))
    n0, _ = s.count()
    s.step(steps)
    ms, _ = s.timing()
    n1, _ = s.count()
    launch = s.launch()
    s.close()
    n = 0.5 * (n0 + n1)
    return dict(value=n * steps / (ms * 1e-3), ms=ms / steps, n=n, launch=launch)


def run_batched(args, precision, steps):
    """Batched uneven tubes (256 tubes, L in [2, 8], 64-512 cells, 1e4-1e6
    ions each, ~5.7e7 in all, heating on) advancing together: one launch
    per kernel over the (tube, chunk) work items, steps replayed from CUDA
    graphs, the autotuner's launch shape."""
    from kaos_b200 import grids
    from kaos_b200.lib import Solver
    mi, specs, tubes, vg = grids.config_c4(args.batched_tubes, precision=precision,
                                           ndatfac=NDATFAC)
    s = Solver(mi, tubes, vg)
    for k, t in enumerate(tubes):
        s.init_particles(k, t._counts, seed=20261203 + k)
    s.set_graph(True)
    if args.launch:
        s.set_launch(*(int(x) for x in args.launch.split(",")))
    s.step(graph_warmup(args, mi.ndatfac))
    n0 = sum(s.count(k)[0] for k in range(len(tubes)))
    s.step(steps)
    ms, _ = s.timing()
    n1 = sum(s.count(k)[0] for k in range(len(tubes)))
    launch = s.launch()
    s.close()
    n = 0.5 * (n0 + n1)
    return dict(value=n * steps / (ms * 1e-3), ms=ms / steps, n=n, launch=launch,
                ntubes=len(tubes))


def run_c5(args, precision, steps):
    """Two species plus neutral products, batched: 64 tubes (L 3-7, 256
    cells) with O+ and H+ as two entries each (2e7 ions), charge exchange
    with an H exosphere producing ENAs, ENA moments, and the 0.5 km/s E x B
    drift: after every master interval each entry's tables are regenerated
    on its new L-shell on the host and queued with kaos_update_tube (applied
    at the next master step).  Device time of the steps only; steps replayed
    from CUDA graphs except the master steps that apply a move."""
    from kaos_b200 import grids
    from kaos_b200.lib import Solver
    mi, specs, tubes, vg, evg = grids.config_c5(precision=precision, ndatfac=NDATFAC)
    s = Solver(mi, tubes, vg)
    s.set_ena_grid(evg)
    for k, t in enumerate(tubes):
        s.init_particles(k, t._counts, seed=20261203 + k)
    s.set_graph(True)
    if args.launch:
        s.set_launch(*(int(x) for x in args.launch.split(",")))
    Ls = [sp.L for sp in specs]
    cur = list(tubes)  # each entry's tables on its current L-shell
    nd = mi.ndatfac

    def intervals(n):
        ms = 0.0
        for _ in range(n):
            s.step(nd)
            ms += s.timing()[0]
            for k in range(len(tubes)):  # E x B drift to the next L-shell
                Ls[k] += grids.conv_c5_dl(nd, mi.h)
                cur[k] = grids.moved_tube(specs[k], mi, cur[k], Ls[k])
                s.update_tube(k, cur[k])
        return ms
    intervals(2 * COMPACT_EVERY + 3)  # warm-up: every step graph captured
    cnt = lambda i: sum(s.count(k)[i] for k in range(len(tubes)))
    n0 = cnt(0)
    nint = max(1, steps // nd)
    ms = intervals(nint)
    n1, ne = cnt(0), cnt(1)
    launch = s.launch()
    s.close()
    n = 0.5 * (n0 + n1)
    return dict(value=n * nint * nd / (ms * 1e-3), ms=ms / (nint * nd), n=n, enas=ne,
                steps=nint * nd, launch=launch, entries=len(tubes))


MOMENT_NAMES = ("M0", "M1par", "M1perp1", "M1perp2", "M2", "M2par", "M2perp1",
                "M2perp2", "Nq", "EAmag", "nuPoi")


def moment_ids():
    from kaos_b200 import model_input as M
    return {"M0": M.KAOS_M0, "M1par": M.KAOS_M1PAR, "M1perp1": M.KAOS_M1PERP1,
            "M1perp2": M.KAOS_M1PERP2, "M2": M.KAOS_M2, "M2par": M.KAOS_M2PAR,
            "M2perp1": M.KAOS_M2PERP1, "M2perp2": M.KAOS_M2PERP2, "Nq": M.KAOS_NQ,
            "EAmag": M.KAOS_EAMAG, "nuPoi": M.KAOS_NUPOI}


def moment_errors(a, b):
    """Norm-wise relative difference max|a - b| / max|b| per moment (a, b:
    objects with .moments(selector))."""
    out = {}
    for k, m in moment_ids().items():
        x, y = a.moments(m), b.moments(m)
        scale = float(np.max(np.abs(y)))
        out[k] = float(np.max(np.abs(x - y)) / scale) if scale > 0 else 0.0
    return out


def error_run(args, heating, collisions, n_part, with_oracle=False, mixed_prec=None):
    """The mixed path (KAOS_PREC_MIXED, or the precision mode given) against
    the FP64 path (and, on a small sample, the FP64 oracle) over the
    configuration's 500 steps from the same ions and random streams: the
    error of every moment at every master step from step 100 on (maximum
    over those steps) and at the last one."""
    from kaos_b200 import grids
    from kaos_b200.lib import Solver
    from kaos_b200.model_input import KAOS_PREC_FP64, KAOS_PREC_MIXED
    mixed = KAOS_PREC_MIXED if mixed_prec is None else mixed_prec
    runs = {}
    init = None
    for prec in (KAOS_PREC_FP64, mixed):
        mi, spec, tube, vg = grids.config_c2(n_particles=n_part, heating=heating,
                                             collisions=collisions, precision=prec,
                                             ndatfac=NDATFAC)
        init = grids.initial_particles(tube, spec, mi, seed=20261203)
        s = Solver(mi, [tube], vg)
        s.load(0, *init)
        runs[prec] = s
    orc = None
    if with_oracle:
        from oracle.oracle import Oracle
        mi, spec, tube, vg = grids.config_c2(n_particles=n_part, heating=heating,
                                             collisions=collisions,
                                             precision=KAOS_PREC_FP64, ndatfac=NDATFAC)
        orc = Oracle(mi, tube, vg)
        orc.load(*init)
    worst = {k: 0.0 for k in MOMENT_NAMES}
    worst_o = {k: 0.0 for k in MOMENT_NAMES}
    done, last, last_o = 0, None, None
    while done < ERR_STEPS:
        k = NDATFAC if done else 1
        k = min(k, ERR_STEPS - done)
        for s in runs.values():
            s.step(k)
        if orc is not None:
            orc.step(k)
        done += k
        if done < 100 or done % NDATFAC:
            continue
        last = moment_errors(runs[mixed], runs[KAOS_PREC_FP64])
        worst = {m: max(worst[m], last[m]) for m in MOMENT_NAMES}
        if orc is not None:
            last_o = moment_errors(runs[mixed], orc)
            worst_o = {m: max(worst_o[m], last_o[m]) for m in MOMENT_NAMES}
    for s in runs.values():
        s.close()
    out = {"ions": n_part, "steps": ERR_STEPS, "master_every": NDATFAC,
           "vs_fp64_max_over_master_steps_from_100": worst,
           "vs_fp64_at_last_step": last}
    if orc is not None:
        out["vs_oracle_max_over_master_steps_from_100"] = worst_o
        out["vs_oracle_at_last_step"] = last_o
    return out


def moment_error_block(args):
    """Every moment of the mixed path against the FP64 path on the full
    tube (1e7 ions), with heating and collisions on (the timed workload) and
    off, and against the FP64 oracle on a 2e4-ion sample of the tube."""
    from kaos_b200.model_input import KAOS_PREC_MIXED_K64
    on = error_run(args, True, True, args.particles)
    off = error_run(args, False, False, args.particles)
    orc = error_run(args, True, True, 20000, with_oracle=True)
    k64 = error_run(args, True, True, args.particles, mixed_prec=KAOS_PREC_MIXED_K64)
    def mx(d):
        return max(d.values())
    return {"heating_collisions_on": on, "heating_collisions_off": off,
            "oracle_sample": orc,
            "max_vs_fp64_on": mx(on["vs_fp64_max_over_master_steps_from_100"]),
            "max_vs_fp64_off": mx(off["vs_fp64_max_over_master_steps_from_100"]),
            "max_vs_oracle_sample": mx(orc["vs_oracle_max_over_master_steps_from_100"]),
            "kick64_heating_collisions_on": k64,
            "max_vs_fp64_on_kick64": mx(k64["vs_fp64_max_over_master_steps_from_100"]),
            "definition": "max over cells |m_mixed - m_ref| / max over cells |m_ref|, "
                          "per moment, at every master step from step 100 to 500"}


def run_e2e(args, precision, launch):
    """Same metric through the public C-ABI with host buffers: the initial
    particle arrays go from pinned host memory to the device once (amortised
    per step), every step reads all the per-cell moments back to the host
    (kaos_get_moments_all, into pinned memory),
    and the final ion state comes back into pinned host memory.  The push
    launch shape is the one the autotuner chose for the device-timed run."""
    from kaos_b200.lib import Solver
    import torch
    mi, spec, tube, vg, init = build_workload(precision, args.particles,
                                              heating=not args.no_heating,
                                              collisions=args.collisions)
    s = Solver(mi, [tube], vg)
    s.set_launch(*launch)
    K = args.steps

    def pinned(n, dtype):
        return torch.empty(n, dtype=dtype, pin_memory=True).numpy()
    src = []
    for a in init:
        b = pinned(len(a), torch.float64)
        b[:] = a
        src.append(b)
    cap = tube.capacity
    out = {k: pinned(cap, torch.float64) for k in ("q", "vpar", "vperp1", "vperp2")}
    out["qind"] = pinned(cap, torch.int32)
    from kaos_b200.model_input import KAOS_NMOMENTS
    mom = torch.empty((KAOS_NMOMENTS, tube.nq), dtype=torch.float64,
                      pin_memory=True).numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.load(0, *src)
    t1 = time.perf_counter()
    h2d = sum(a.nbytes for a in src)
    d2h = 0
    for _ in range(K):
        s.step(1)
        d2h += s.moments_all(out=mom).nbytes
    t2 = time.perf_counter()
    p = s.state(out=out)
    d2h += sum(v.nbytes for v in p.values())
    t3 = time.perf_counter()
    dt = t3 - t0
    n = len(p["q"])
    s.close()
    return dict(value=n * K / dt, h2d=h2d / K, d2h=d2h / K,
                phases_ms={"load": 1e3 * (t1 - t0), "steps": 1e3 * (t2 - t1),
                           "state": 1e3 * (t3 - t2)})


def workload_config(args, n_ions):
    """The `config` object of both arms' lines (same workload)."""
    return {"workload": "precision A/B tube: L=4, 256 cells, 3D grid 48x48x64, "
                        f"{int(n_ions)} O+ per GPU, heating "
                        f"{'off' if args.no_heating else 'on'}, collisions "
                        f"{'on' if args.collisions else 'off'}, dt 5 ms, "
                        f"master step every {NDATFAC} steps",
            "master_step_every": NDATFAC,
            "l2": "inputs > L2 (particle arrays 1-1.5 GB); no flush",
            "parallelism": f"tube per GPU x{args.gpus}"}


def cpu_baseline(args, sample_particles=20000, sample_steps=NDATFAC):
    """The CPU oracle (FP64 restatement of the reference loop, direct
    binning) on a bounded sample of the same workload, one host thread, over
    one whole master interval; beside it the literal reference algorithm
    (O(Nq Nv Np) counting, IonParticleCountsSub _8_3_1_...:311-357) on the
    plain FP64 configuration, on all host cores and on one."""
    from oracle.oracle import Oracle
    from kaos_b200 import grids
    from kaos_b200.model_input import KAOS_PREC_FP64
    mi, spec, tube, vg = grids.config_c2(n_particles=sample_particles,
                                         heating=not args.no_heating,
                                         collisions=args.collisions,
                                         precision=KAOS_PREC_FP64, ndatfac=NDATFAC)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=20261203)
    o = Oracle(mi, tube, vg)
    o.load(q, vpar, v1, v2)
    o.step(NDATFAC)
    t0 = time.perf_counter()
    o.step(sample_steps)
    dt = time.perf_counter() - t0
    n, _ = o.count()
    out = dict(value=n * sample_steps / dt, unit="particle-steps/s", cores=1,
               kind="port",
               sample=f"{n} O+ of the same tube x {sample_steps} steps holding one "
                      "master step (oracle, direct binning, 1 thread)")
    out["literal_c1"] = literal_baseline()
    out["literal_c1_1core"] = literal_baseline(cores=1)
    return out


def _literal_worker(job, barrier, out):
    """One host core: the oracle with the reference's literal counting loops
    on its own sample of the plain FP64 configuration (master step every 20
    steps), timed over one master interval."""
    seed, npart, steps = job
    from oracle.oracle import Oracle
    from kaos_b200 import grids
    mi, spec, tube, vg = grids.config_c1(n_particles=npart)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=seed)
    o = Oracle(mi, tube, vg)
    o.set_literal(True)
    o.load(q, vpar, v1, v2)
    o.step(1)
    n0, _ = o.count()
    barrier.wait()
    t0 = time.time()
    o.step(steps)
    t1 = time.time()
    n1, _ = o.count()
    out.put((0.5 * (n0 + n1) * steps, t0, t1))


def parallel_oracle(worker, jobs):
    """Run one oracle job per host core (spawned processes, started
    together); all particle-steps / the span from the first start to the
    last end."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier, out = ctx.Barrier(len(jobs)), ctx.Queue()
    procs = [ctx.Process(target=worker, args=(j, barrier, out)) for j in jobs]
    for p in procs:
        p.start()
    res = [out.get(timeout=900) for _ in procs]
    for p in procs:
        p.join()
    work = sum(r[0] for r in res)
    span = max(r[2] for r in res) - min(r[1] for r in res)
    return work / span, span


def literal_baseline(npart=10000, steps=20, cores=None):
    """The literal reference algorithm on `cores` host cores (default all)."""
    cores = len(os.sched_getaffinity(0)) if cores is None else cores
    jobs = [(20261203 + k, npart, steps) for k in range(cores)]
    v, span = parallel_oracle(_literal_worker, jobs)
    return {"value": v, "unit": "particle-steps/s", "cores": cores,
            "kind": "port", "algorithm": "literal O(Nq Nv Np) counting",
            "sample": f"plain FP64 configuration (L=4, 128 cells, 2D grid 64x32): "
                      f"{cores} processes x {npart} O+ x {steps} steps (steps 2-21, "
                      "master step at 20)", "span_s": span}


def _reference_worker(job, barrier, out):
    """One host core: the oracle on its own seeded sample of the workload;
    all workers start their timed steps together."""
    seed, npart, warmup, steps, heating, collisions = job
    from oracle.oracle import Oracle
    from kaos_b200 import grids
    from kaos_b200.model_input import KAOS_PREC_FP64
    mi, spec, tube, vg = grids.config_c2(n_particles=npart, heating=heating,
                                         collisions=collisions,
                                         precision=KAOS_PREC_FP64, ndatfac=NDATFAC)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=seed)
    o = Oracle(mi, tube, vg)
    o.load(q, vpar, v1, v2)
    o.step(warmup)
    n0, _ = o.count()
    barrier.wait()
    t0 = time.time()
    o.step(steps)
    t1 = time.time()
    n1, _ = o.count()
    out.put((0.5 * (n0 + n1) * steps, t0, t1))


def reference_arm(args):
    """--impl reference: the CPU restatement of the reference loop (the
    reference itself is Fortran+MPI and cannot be built in this image) on
    every host core: one process per core, each advancing its own bounded
    sample of the workload over the same steps and cadence; throughput =
    all particle-steps / the span from the first start to the last end."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    npart = 20000
    cores = len(os.sched_getaffinity(0))
    jobs = [(20261203 + k, npart, args.warmup, args.steps, not args.no_heating,
             args.collisions) for k in range(cores)]
    v, span = parallel_oracle(_reference_worker, jobs)
    return {
        "impl": "reference", "metric": METRIC, "value": v,
        "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * span / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, N_PART),
        "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": cores,
                         "kind": "port",
                         "sample": f"{cores} processes x {npart} O+ of the tube x "
                                   f"{args.steps} steps after {args.warmup}, oracle "
                                   "FP64, direct binning (faster than the reference's "
                                   "literal counting loops)"},
        "e2e": {"value": v, "unit": "particle-steps/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=N_PART)
    ap.add_argument("--no-heating", action="store_true")
    ap.add_argument("--no-collisions", dest="collisions", action="store_false")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--kick64", action="store_true",
                    help="with --only mixed: time the mixed path with the heating kick "
                         "in FP64 (precision mode KAOS_PREC_MIXED_K64)")
    ap.add_argument("--large-particles", type=int, default=100_000_000,
                    help="ions of the large single-tube line (0: skip it)")
    ap.add_argument("--batched-tubes", type=int, default=256,
                    help="tubes of the batched uneven-tube line (0: skip it)")
    ap.add_argument("--c5", type=int, default=1,
                    help="1: time the two-species/ENA/convection batch (0: skip it)")
    ap.add_argument("--only", default="all",
                    choices=["all", "mixed", "large", "cadence1", "batched", "c5"],
                    help="mixed: time the mixed path alone; large: the large single "
                         "tube's mixed path alone; cadence1: the mixed path with every "
                         "step a master step (all for profiling)")
    ap.add_argument("--launch", default=None,
                    help="fixed push launch shape CHUNK,MODE instead of the autotuner "
                         "(CHUNK ions per work item 1024/2048/4096; MODE bit 0 persistent "
                         "grid, bits 1-2 mixed push register budget 0: 64, 1: 80, "
                         "2: 72 with 128-thread blocks)")
    args = ap.parse_args()
    if args.impl == "reference":
        line = reference_arm(args)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    import torch
    if args.only == "cadence1":
        from kaos_b200.model_input import KAOS_PREC_MIXED
        r = run_ours(args, KAOS_PREC_MIXED, graph=True, ndatfac=1)
        r["solver"].close()
        print(json.dumps({"cadence1_mixed": r["value"], "ms_per_step": r["ms"] / args.steps,
                          "push_ms": r["push_ms"], "steps": args.steps,
                          "launch": r["launch"]}), flush=True)
        return
    if args.only == "c5":
        from kaos_b200.model_input import KAOS_PREC_MIXED
        c = run_c5(args, KAOS_PREC_MIXED, args.steps)
        print(json.dumps({"c5_mixed": c["value"], "ms_per_step": c["ms"], "n": c["n"],
                          "enas": c["enas"], "steps": c["steps"], "launch": c["launch"]}),
              flush=True)
        return
    if args.only == "batched":
        from kaos_b200.model_input import KAOS_PREC_MIXED
        b32 = run_batched(args, KAOS_PREC_MIXED, args.steps)
        print(json.dumps({"batched_mixed": b32["value"], "ms_per_step": b32["ms"],
                          "n": b32["n"], "tubes": b32["ntubes"], "steps": args.steps,
                          "launch": b32["launch"]}), flush=True)
        return
    if args.only == "large":
        from kaos_b200.model_input import KAOS_PREC_MIXED
        l32 = run_large(args, KAOS_PREC_MIXED, args.steps)
        print(json.dumps({"large_mixed": l32["value"], "ms_per_step": l32["ms"],
                          "n": l32["n"], "steps": args.steps, "launch": l32["launch"]}),
              flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from kaos_b200.model_input import KAOS_PREC_FP64, KAOS_PREC_MIXED, KAOS_PREC_MIXED_K64
    full = args.only == "all"
    # FP64 path first (reported beside the headline)
    r64 = run_ours(args, KAOS_PREC_FP64) if full else None
    stop = threading.Event()
    samples = []
    th = threading.Thread(target=clocks_sampler, args=(stop, samples), daemon=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    th.start()
    r32 = run_ours(args, KAOS_PREC_MIXED_K64 if (args.kick64 and not full)
                   else KAOS_PREC_MIXED)
    torch.cuda.synchronize()
    stop.set()
    if full:
        r64["solver"].close()
    r32["solver"].close()
    # error of every moment of the mixed path against the FP64 path and the
    # FP64 oracle (same ions, same random streams), master steps 100-500
    moment_error = moment_error_block(args) if full else None
    # the mixed path with the heating kick in FP64 (KAOS_PREC_MIXED_K64: the
    # variant whose moments keep the FP64 path's bins with heating on)
    rk = None
    if full:
        rk = run_ours(args, KAOS_PREC_MIXED_K64)
        rk["solver"].close()
    # the same steps replayed from CUDA graphs, and at cadence 1 (every step
    # a master step: removal/injection, fields, counts and moments each step)
    rg = rc1 = None
    if full:
        rg = run_ours(args, KAOS_PREC_MIXED, graph=True)
        rg["solver"].close()
        rc1 = run_ours(args, KAOS_PREC_MIXED, graph=True, ndatfac=1,
                       steps=min(args.steps, 50))
        rc1["solver"].close()
    ms = r32["ms"]
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * r32["n"] * args.steps / (ms * 1e-3)
    # (this tube's exosphere forms no ENA: its intervals are idle)
    cx_active = args.collisions and r32["enas"] > 0
    mixed_bytes = bytes_per_particle_step(True, not args.no_heating, cx_active)
    achieved = mixed_bytes * r32["n"] / (r32["push_ms"] * 1e-3) / 1e9
    achieved_frozen = FROZEN_MIXED_BYTES * r32["n"] / (r32["push_ms"] * 1e-3) / 1e9
    peak, peak_kind = peaks()
    e2e = None
    if not args.skip_e2e and full:  # before the large tube's allocations
        e2e = run_e2e(args, KAOS_PREC_MIXED, r32["launch"])
    large = None
    if full and args.large_particles > 0:
        lsteps = min(args.steps, 100)
        l32, lclk = with_clocks(run_large, args, KAOS_PREC_MIXED, lsteps)
        l64 = run_large(args, KAOS_PREC_FP64, lsteps)
        large = {"workload": "large single tube: L=6, 512 cells 800 km to the equator, "
                             f"3D grid 64x64x96, {int(l32['n'])} O+ (90 % 0.3 eV Maxwellian "
                             "+ 10 % kappa=3 5 eV tail, generated on the device), heating "
                             "and collisions on, LB injection from the Maxwellian flux, dt 5 ms",
                 "steps": lsteps, "mixed": l32["value"] * world,
                 "mixed_ms_per_step": l32["ms"], "fp64": l64["value"] * world,
                 "fp64_ms_per_step": l64["ms"],
                 "mixed_over_fp64": l32["value"] / l64["value"],
                 "push_launch": l32["launch"], "mixed_clocks": lclk,
                 "note": "both paths replayed from CUDA graphs"}
    batched = None
    if full and args.batched_tubes > 0:
        bsteps = min(args.steps, 100)
        b32, bclk = with_clocks(run_batched, args, KAOS_PREC_MIXED, bsteps)
        b64 = run_batched(args, KAOS_PREC_FP64, bsteps)
        batched = {"workload": f"{b32['ntubes']} batched uneven tubes: L uniform in [2, 8], "
                               "64-512 cells, 1e4-1e6 O+ each (log-uniform), "
                               f"{int(b32['n'])} in all, n0 1e9-1e11 m^-3, T 0.1-1 eV, "
                               "shared 3D grid 48x48x64, heating 1e-4-1e-2 eV/s, dt 5 ms",
                   "steps": bsteps, "mixed": b32["value"] * world,
                   "mixed_ms_per_step": b32["ms"], "fp64": b64["value"] * world,
                   "fp64_ms_per_step": b64["ms"],
                   "mixed_over_fp64": b32["value"] / b64["value"],
                   "push_launch": b32["launch"], "mixed_clocks": bclk,
                   "note": "one launch per kernel over (tube, chunk) work items; "
                           "both paths replayed from CUDA graphs"}
    species = None
    if full and args.c5:
        try:
            c32, cclk = with_clocks(run_c5, args, KAOS_PREC_MIXED, min(args.steps, 100))
            c64 = run_c5(args, KAOS_PREC_FP64, min(args.steps, 100))
            species = {"workload": "64 tubes (L 3-7, 256 cells), O+ and H+ at 4:1 density as "
                                   f"{c32['entries']} entries, {int(c32['n'])} ions, charge "
                                   "exchange with an H exosphere (1e16 m^-3 at the base: "
                                   "the per-cell Poisson mean at 1e11 forms no ENA; "
                                   "scale height 1000 km) to "
                                   f"{c32['enas']} ENAs, ENA moments on 48x48x64, E x B "
                                   "drift 0.5 km/s (tables regenerated each master interval), "
                                   "dt 5 ms",
                       "steps": c32["steps"], "mixed": c32["value"] * world,
                       "mixed_ms_per_step": c32["ms"], "fp64": c64["value"] * world,
                       "fp64_ms_per_step": c64["ms"],
                       "mixed_over_fp64": c32["value"] / c64["value"],
                       "push_launch": c32["launch"], "mixed_clocks": cclk,
                       "note": "ion-steps per second of device time (host table "
                               "regeneration excluded); CUDA graphs except the master "
                               "steps that apply a move"}
        except Exception as e:  # reported, never fatal to the bench line
            species = {"error": f"{type(e).__name__}: {e}"}
    cpu = cpu_baseline(args) if (rank == 0 and world == 1 and full) else None
    tpi = profiled_traffic("k_push32_mixed_c2.md")
    traffic = None if tpi is None else tpi * r32["n"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": dict(workload_config(args, r32["n"]), **{
                "precision": "mixed: FP32 arithmetic (forces, RK stages, heating) on FP64 "
                             "state (cell coordinate, V||, Vperp pair), FP64 quartic / "
                             "renormalisation / reductions",
                "push_launch": {"ions_per_item": r32["launch"][0],
                                "persistent": bool(r32["launch"][1] & 1),
                                "registers": (64, 80, 72)[(r32["launch"][1] >> 1) & 3],
                                "master_step_registers":
                                    ((64, 80, 72)[(r32["launch"][1] >> 1) & 3],
                                     64, 80, 72)[(r32["launch"][1] >> 3) & 3],
                                "threads_per_block": 128 if r32["launch"][1] & 4 else 256,
                                "chosen_by": "fixed" if args.launch else "autotuner"}}),
            "fp64": None if not full else {
                "value": r64["value"] * world, "ms_per_step": r64["ms"] / args.steps,
                "push_ms": r64["push_ms"]},
            "mixed_over_fp64": value / (r64["value"] * world) if full else None,
            "fp64_roofline": fp64_pipe_roofline(r64["value"]) if full else None,
            "mixed_push_ms": r32["push_ms"],
            "kick64": None if not full else {
                "value": rk["value"] * world, "ms_per_step": rk["ms"] / args.steps,
                "push_ms": rk["push_ms"],
                "over_fp64": rk["value"] / r64["value"],
                "push_launch": rk["launch"],
                "moment_error_vs_fp64_max": moment_error["max_vs_fp64_on_kick64"],
                "note": "precision mode KAOS_PREC_MIXED_K64: the mixed path with the "
                        "heating kick in FP64 (the FP64 path's formula and draw), "
                        "same workload; its moment error is in "
                        "moment_error_vs_fp64.kick64_heating_collisions_on"},
            "large": large,
            "batched": batched,
            "species_ena_convection": species,
            "moment_error_vs_fp64": moment_error,
            "graph": None if not full else {
                "value": rg["value"] * world, "ms_per_step": rg["ms"] / args.steps,
                "push_launch": rg["launch"],
                "warmup_steps": graph_warmup(args, NDATFAC),
                "note": "mixed path, steps replayed from CUDA graphs (a warm-up through "
                        "two compactions and three more master intervals captures every "
                        "step graph before timing)"},
            "cadence1": None if not full else {
                "value": rc1["value"] * world,
                "ms_per_step": rc1["ms"] / min(args.steps, 50),
                "steps": min(args.steps, 50),
                "note": "mixed path, every step a master step, CUDA graphs"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_push32 (mixed push), average over the timed "
                                   "window's launches (ordinary and master steps)",
                         "bytes_per_particle": mixed_bytes,
                         "frozen_bytes_per_particle": FROZEN_MIXED_BYTES,
                         "achieved_at_frozen_bytes": achieved_frozen,
                         "frac_at_frozen_bytes": achieved_frozen / peak,
                         "bytes_note": "the mixed state is FP64 (cell coordinate, V||, "
                                       "Vperp pair: 32 B read + 32 B written) so that every "
                                       "moment matches the FP64 path; the frozen 48 B "
                                       "counted the earlier FP32 state; Qindk1 and the k4 "
                                       "point (8 B) are stored only in intervals whose "
                                       "charge exchange converts ions (none here: the "
                                       "exosphere forms no ENA)"
                                       if not cx_active else
                                       "the mixed state is FP64 (cell coordinate, V||, "
                                       "Vperp pair: 32 B read + 32 B written) so that every "
                                       "moment matches the FP64 path; the frozen 48 B "
                                       "counted the earlier FP32 state",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "per ion of a 6e6-ion launch, scaled to this launch"},
            "cpu_baseline": cpu,
            "e2e": None if e2e is None else {
                "value": e2e["value"] * world, "unit": "particle-steps/s",
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                "phases_ms": e2e["phases_ms"]},
            "gpu_launches": r32["launches"],
            "clocks": summarize_clocks(samples),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
