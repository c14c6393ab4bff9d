#!/usr/bin/env python
"""Throughput of the euler3D residual-and-update path on B200, in cell-iterations/s.

Workload (the second-order configuration): the 80^3 hexahedron bump channel
split into 6 tetrahedra per hexahedron (3,072,000 tetrahedra), cut into 16
x-slab topology blocks that all live on one GPU; least-squares gradients,
Venkatakrishnan limiter (K = 5), Roe flux, Mach 0.7, alpha 1.25 deg, 5-stage
Runge-Kutta, CFL 1.5; FP32 flux/gradient/limiter arithmetic with the FP64
conserved state and FP64 norm / force reductions.  The mesh is synthetic
(seedless deterministic generator, euler3d_b200.meshgen) and goes through the
reference's file formats (SU2 blocks + .top topology + input deck).

A step is one outer iteration of the solver over every cell of every block
(5 RK stages, local time step, residual norms, wall forces, inter-block halo).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one per GPU, launched by torchrun): the
path has no inter-GPU exchange when all blocks of a case live on one GPU.
``--mode blocks`` instead splits the one case's 16 blocks over the N ranks
(the reference's MPI distribution; the connexion halo crosses GPUs through
NCCL once per outer iteration) and reports strong scaling.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "cell-iters/s"
UNIT = "cell-iterations/s"
WORKLOAD = dict(n=80, blocks=16, order=2, flux="roe", gradient="leastsquares", limiter="venkatakrishnan", k=5.0,
                omega=2.16e-16, mach=0.7, aoa_deg=1.25, cfl=1.5, stages=5)
REFDRIVER = os.path.join(HERE, "oracle", "_ref", "e3d_refdriver")
RENUMBER = "none+boundary_last"  # device cell order of the channel workload (the library's default)
# the warm-start surrogate trained on the seeded channel sweep (python -m euler3d_b200.sweep train --out ...)
WARM_DATA = os.path.join(HERE, "euler3d_b200", "data", "warmstart_channel_ausm1.npz")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_case(directory: str, n: int, blocks: int) -> str:
    from euler3d_b200 import meshgen as mg

    w = WORKLOAD
    deck = mg.Deck(topology="", cfl=w["cfl"], stages=w["stages"], mach=w["mach"], aoa_deg=w["aoa_deg"],
                   max_iter=1000000, criterion=-15.0, flux=w["flux"], order=w["order"], gradient=w["gradient"],
                   limiter=w["limiter"], omega=w["omega"], k=w["k"])
    return mg.write_case(directory, n, blocks, deck=deck)


# the swept-wing configuration: AUSM + least squares + Venkatakrishnan (K = 5), M 0.8, alpha 3
WING_SCHEME = dict(order=2, flux="ausm", gradient="leastsquares", limiter="venkatakrishnan", omega=2.16e-16, k=5.0,
                   mach=0.8, aoa_deg=3.0, cfl=1.5, stages=5)
# body-fitted mesh: O-grid points around each section x layers off the wall x spanwise stations
# (wing, beyond the tip): 256 x 80 x (112 + 48) hexahedra, 6 tetrahedra each
WING_DIMS = (256, 80, 112, 48)
# the earlier Delaunay mesh (--wing-mesh delaunay): seeded points, staircase wall
WING_DELAUNAY_SCHEME = dict(WING_SCHEME, limiter="barthjespersen")
WING_POINTS = 3_800_000


def wing_case(a, td):
    """The swept-wing case: an existing directory (--mesh-dir) or a fresh one."""
    from euler3d_b200 import meshgen as mg
    from euler3d_b200 import wingmesh as wm

    delaunay = a.wing_mesh == "delaunay"
    w = WING_DELAUNAY_SCHEME if delaunay else WING_SCHEME
    if a.mesh_dir and os.path.exists(os.path.join(a.mesh_dir, "wing.deck")):
        case_dir = a.mesh_dir
    else:
        case_dir = a.mesh_dir or os.path.join(td, "wing")
        deck = mg.Deck(topology="", max_iter=1000000, criterion=-15.0, **w)
        if delaunay:
            wm.write_wing_case(case_dir, WING_POINTS, n_blocks=16, seed=5, deck=deck)
        else:
            wm.write_body_fitted_wing_case(case_dir, *WING_DIMS, n_blocks=16, deck=deck)
    scheme = (f"{w['gradient']} + {w['limiter']} (K = {w['k']:g}) + {w['flux']}, M {w['mach']}, alpha "
              f"{w['aoa_deg']}, {w['stages']}-stage RK, CFL {w['cfl']}")
    if delaunay:
        mesh = (f"in a farfield box, seeded Delaunay tetrahedra (seed 5, {WING_POINTS:,} points requested), wall "
                f"left by the removed interior tetrahedra")
    else:
        ni, nj, nkw, nko = WING_DIMS
        mesh = (f"in a tunnel box (inlet/outlet farfield, sides symmetry), body-fitted: O-grid sections of {ni} x "
                f"{nj} hexahedra, {nkw} + {nko} spanwise stations, rounded tip, 6 tetrahedra per hexahedron")
    cfg = {"workload": f"swept trapezoidal wing (NACA 4-digit 12 %, 30 deg sweep, taper 0.56) {mesh}; 16 x-slab "
                       f"blocks on one GPU, Morton-ordered cells; {scheme}",
           "blocks": 16,
           "arithmetic": "fp32 fluxes/gradients/limiters, fp64 conserved state and reductions"
           if a.precision == "fp32" else "fp64 throughout (reference arithmetic)",
           "l2": "working set (many GB) far larger than the 126 MB L2; no flush needed"}
    return os.path.join(case_dir, "wing.deck"), case_dir, cfg


def fp32_error_report(td):
    """The FP32 variant's error against the FP64 path, which is the reference's
    arithmetic bit for bit: the 20^3 x 6 (48,000-tet) first-order Roe case, M 0.5,
    500 iterations, and the first 20 iterations of the 3.07M-tet second-order
    workload's own scheme on a 20^3 x 6 mesh in 4 blocks."""
    import numpy as np

    from euler3d_b200 import api
    from euler3d_b200 import meshgen as mg

    out = {}
    cases = {"bump20_o1_roe_500it": (20, 1, dict(order=1, flux="roe", mach=0.5, aoa_deg=0.0), 500),
             "bump20b4_o2_ls_venk_roe_20it": (20, 4, dict(order=2, flux="roe", gradient="leastsquares",
                                                          limiter="venkatakrishnan", k=5.0, mach=0.7,
                                                          aoa_deg=1.25), 20)}
    for name, (n, nb, deck, iters) in cases.items():
        path = mg.write_case(os.path.join(td, "err_" + name), n, nb, deck=mg.Deck(topology="", **deck))
        case = api.Case(path)
        res = {}
        for prec in ("fp64", "fp32"):
            s = api.Solver(case, precision=prec, hist_capacity=iters + 16)
            s.iterate(iters)
            res[prec] = (s.history(), [s.get(b, "prim") for b in range(case.n_blocks)])
            s.close()
        h64, p64 = res["fp64"]
        h32, p32 = res["fp32"]
        scale = np.array([1.0, 0.7 * 1.4 ** 0.5, 0.7 * 1.4 ** 0.5, 0.7 * 1.4 ** 0.5, 1.0])  # freestream magnitudes
        dev = max(float(np.max(np.abs(a.reshape(5, -1) - b.reshape(5, -1)) / scale[:, None])) for a, b in zip(p32, p64))
        out[name] = {"iterations": iters,
                     "max_abs_ro_conv_decades": float(np.max(np.abs(h32["conv"][:, 0] - h64["conv"][:, 0]))),
                     "cl_rel": float(abs(h32["cl"][-1] - h64["cl"][-1]) / abs(h64["cl"][-1])),
                     "cd_rel": float(abs(h32["cd"][-1] - h64["cd"][-1]) / abs(h64["cd"][-1])),
                     "max_cell_state_dev": dev,
                     "note": "state deviation scaled by freestream density, speed and pressure"}
        case.close()
    return out


def workload_config(n, blocks, precision):
    w = WORKLOAD
    cells = 6 * n ** 3
    # bytes the reconstruction pass must touch per launch: about 16 + 50 b per
    # tet (states, neighbour ids, least-squares weights, r-vectors, face states)
    mb = cells * (16 + 50 * (4 if precision == "fp32" else 8)) / 1e6
    l2 = (f"each stage pass touches about {mb:,.0f} MB, more than the 126 MB L2; no flush needed" if mb > 126
          else f"each stage pass touches about {mb:,.1f} MB, less than the 126 MB L2: a test size, not a bench number")
    return {"workload": f"bump channel {n}^3 hex x 6 tets ({cells:,} tets), {blocks} slab blocks on one GPU, "
                        f"{w['gradient']} + {w['limiter']} (K={w['k']:g}) + {w['flux']}, M {w['mach']}, "
                        f"alpha {w['aoa_deg']}, {w['stages']}-stage RK, CFL {w['cfl']}",
            "cells": cells, "blocks": blocks,
            "arithmetic": "fp32 fluxes/gradients/limiters, fp64 conserved state and reductions"
            if precision == "fp32" else "fp64 throughout (reference arithmetic)",
            "l2": l2}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        self.marks = []

    def mark(self, tag):
        self.marks.append((tag, time.time()))

    def stop(self):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        return rows

    @staticmethod
    def summarize(rows):
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------ CPU baselines
def run_refdriver(deck: str, blocks: str, iters: int, warmup: int, cwd: str):
    out = subprocess.run([REFDRIVER, deck, "--iters", str(iters), "--warmup", str(warmup), "--blocks", blocks,
                          "--quiet"], cwd=cwd, capture_output=True, text=True, check=True, timeout=3600)
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_baseline_single(deck: str, case_dir: str):
    """The reference CPU solver on one host core over a bounded sample: block 0
    of the 16 (192,000 cells) for 2 outer iterations (about 10 s of CPU work)."""
    if os.path.exists(REFDRIVER):
        with tempfile.TemporaryDirectory() as wd:
            _link_case(case_dir, wd)
            r = run_refdriver(os.path.basename(deck), "0:1", 3, 1, wd)
        return {"value": r["cell_iters_per_s"], "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"block 0 ({r['cells']:,} cells) of the same workload, {r['iters']} outer iteration(s) "
                          "after 1 warm-up, reference solver compiled from its sources (serial, -O2), 1 core"}
    # fallback: the C restatement of the path (pinned bitwise to the reference)
    sys.path.insert(0, os.path.join(HERE, "tests"))
    from oracle_c import OracleBlock, OracleCase, params_from_deck

    from euler3d_b200.api import Case

    case = Case(deck)
    ob = OracleBlock.from_case(case, 0)
    oc = OracleCase([ob], params_from_deck(case.deck))
    oc.iterate(1)
    t = time.perf_counter()
    oc.iterate(1)
    dt = time.perf_counter() - t
    return {"value": ob.n_real / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"block 0 ({ob.n_real:,} cells), 1 outer iteration after 1 warm-up, C restatement, 1 core"}


def _link_case(case_dir: str, wd: str):
    for name in os.listdir(case_dir):
        if name.endswith((".su2", ".top", ".deck")):
            os.symlink(os.path.join(case_dir, name), os.path.join(wd, name))
    os.makedirs(os.path.join(wd, "bin"), exist_ok=True)


def run_reference_arm(a, rank: int):
    """The reference's own CPU solver, all host cores: one process per block
    range, as the reference distributes blocks over MPI ranks
    (MPI/src/BlockCommunicator.cpp:20-39); a step is one outer iteration over
    every block.  Bounded: at most 5 timed steps after at most 1 warm-up."""
    if rank != 0:
        return 0
    if a.workload != "channel":
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm times the default workload; the "
                                                             f"{a.workload} line carries its own cpu_baseline"}))
        return 0
    n, blocks = a.n, a.blocks
    if not os.path.exists(REFDRIVER):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/e3d_refdriver was not built (the "
                                                             "reference sources were absent when build() ran)"}))
        return 0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    procs = max(1, min(cores, blocks))
    steps = max(1, min(a.steps, 5))
    warm = min(max(a.warmup, 0), 1)
    with tempfile.TemporaryDirectory() as td:
        case_dir = os.path.join(td, "case")
        deck = make_case(case_dir, n, blocks)
        per = [blocks // procs + (1 if i < blocks % procs else 0) for i in range(procs)]
        starts = [sum(per[:i]) for i in range(procs)]
        jobs = []
        for i in range(procs):
            wd = os.path.join(td, f"p{i}")
            os.makedirs(wd)
            _link_case(case_dir, wd)
            cmd = [REFDRIVER, os.path.basename(deck), "--iters", str(warm + steps), "--warmup", str(warm),
                   "--blocks", f"{starts[i]}:{starts[i] + per[i]}", "--quiet"]
            jobs.append(subprocess.Popen(cmd, cwd=wd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        res = []
        for j in jobs:
            out, _ = j.communicate(timeout=3600)
            if j.returncode != 0:
                raise RuntimeError("reference driver failed")
            res.append(json.loads(out.strip().splitlines()[-1]))
    cells = sum(r["cells"] for r in res)
    t = max(r["solve_s"] for r in res)
    value = cells * steps / t
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 1000.0 * t / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(n, blocks, "fp64"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                             "sample": f"{steps} outer iteration(s) of all {blocks} blocks after {warm} warm-up, "
                                       f"{procs} processes x 1 thread each owning a contiguous block range "
                                       "(no inter-process halo), reference solver compiled from its sources"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ ranks
def combine_ranks(local_ms: float, cells: int, steps: int, world: int, dist=None, device="cpu") -> dict:
    """Replicas: every rank advances its own copy of the workload; the job's
    time is the slowest rank's device time (max over ranks), and the job
    processed world x cells x steps cell-iterations."""
    import torch

    t = torch.tensor([local_ms], dtype=torch.float64, device=device)
    if world > 1 and dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    return {"ms": ms, "value": world * cells * steps / (ms / 1000.0)}


# ------------------------------------------------------------------ our arm
# ------------------------------------------------------------------ sweep workloads
POLAR_SCHEME = dict(order=2, flux="ausm", gradient="greengauss", limiter="barthjespersen", omega=2.16e-16, stages=5,
                    cfl=1.5)


def _ref_sample(decks, iters, procs):
    """The reference solver (oracle driver, fast face builder) on `procs`
    cases at once, `iters` iterations each: aggregate cell-iterations/s."""
    if not os.path.exists(REFDRIVER):
        return None
    jobs = []
    t0 = time.perf_counter()
    for d in decks[:procs]:
        jobs.append(subprocess.Popen([REFDRIVER, os.path.basename(d), "--iters", str(iters), "--warmup", "0",
                                      "--blocks", "0:1", "--quiet"],
                                     cwd=os.path.dirname(d), stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                     text=True))
    total = 0.0
    slow = 0.0
    for j in jobs:
        out, _ = j.communicate()
        r = json.loads(out.strip().splitlines()[-1])
        total += r["cells"] * r["iters"]
        slow = max(slow, r["solve_s"])
    return {"value": total / slow, "unit": UNIT, "cores": len(jobs), "kind": "reference",
            "sample": f"{len(jobs)} cases of the sweep run concurrently (one process and core each), {iters} "
                      f"iterations each, reference solver compiled from its sources (-O2, fast face builder); "
                      f"aggregate = sum(cells x iterations) / slowest solve time",
            "wall_s": time.perf_counter() - t0}


def warmstart_bounded(n_cases: int = 4, n_max: int = 32) -> dict:
    """Time to an 8-order density drop, bounded to fit the default run: the
    first `n_cases` held-out cases of the warm-start sweep with at most n_max^3
    x 6 tetrahedra, solved by the plain FP64 drop-in path case after case and
    by one batch with the committed surrogate's warm start (FP32 to -5, then
    FP32 in difference form on an FP64 base).  The same per-case stop rule and reference residual as
    `--workload warmstart`, on fewer and smaller cases."""
    from euler3d_b200 import api
    from euler3d_b200 import sweep as sw

    if not os.path.exists(WARM_DATA):
        return {"unavailable": f"{os.path.relpath(WARM_DATA, HERE)} missing"}
    specs = [p for p in sw.polar_specs(sw.HELD_OUT_SEED, 32, n_range=(25, 60), prefix="test") if p.n <= n_max]
    specs = specs[:n_cases]
    crit, max_iter = -8.0, 200000
    with tempfile.TemporaryDirectory() as td:
        decks = sw.write_cases(td, specs, sw.WARM_SCHEME, sides="channel", processes=1)
        cases = [api.Case(d) for d in decks]
        m, info = sw.load_surrogate(WARM_DATA)
        learned = sw.solve_batched(cases, crit, max_iter, surrogate=m)
        plain = [sw.solve_plain(c, crit, max_iter) for c in cases]
        m.close()
        for c in cases:
            c.close()
    t_plain = sum(p["wall_s"] for p in plain)
    dcl = max(abs(l["cl"] - p["cl"]) / max(abs(p["cl"]), 1e-2) for l, p in zip(learned["cases"], plain))
    dcd = max(abs(l["cd"] - p["cd"]) / max(abs(p["cd"]), 1e-2) for l, p in zip(learned["cases"], plain))
    return {"metric": "time to 1e-8 density-residual drop (s)", "unit": "s", "higher_is_better": False,
            "cases": [dict(n=p.n, mach=round(p.mach, 4), aoa_deg=round(p.aoa_deg, 4)) for p in specs],
            "cells": sum(p["cells"] for p in plain), "plain_s": t_plain, "batched_learned_s": learned["wall_s"],
            "speedup": t_plain / learned["wall_s"], "iters_plain": [p["reached"] for p in plain],
            "iters_learned": [c["reached"] for c in learned["cases"]], "max_rel_dcl": dcl, "max_rel_dcd": dcd,
            "phases": learned["phases"], "surrogate": {k: info.get(k) for k in ("cases", "train_seed", "loss")},
            "workload": "held-out channel cases of the warm-start sweep (seed 2000, n <= %d), first-order AUSM, "
                        "5-stage RK, CFL 1.5; plain = FP64 drop-in path case after case (e3d_solve, check every 50)"
                        % n_max}


def run_sweep_workload(a, rank, world):
    import torch

    from euler3d_b200 import api
    from euler3d_b200 import sweep as sw

    if world > 1 and rank != 0:
        return 0  # the sweep workloads are single-GPU measurements
    torch.cuda.set_device(0)
    small = a.scale == "small"
    nr = (10, 16) if small else (25, 60)
    clocks = ClockSampler(0)
    with tempfile.TemporaryDirectory() as td:
        if a.workload == "polar":
            specs = sw.polar_specs(3, 16 if small else 64, n_range=nr)
            t0 = time.time()
            decks = sw.write_cases(td, specs, POLAR_SCHEME, sides="farfield")
            cases = [api.Case(d) for d in decks]
            log(f"[bench] {len(cases)} cases written and loaded in {time.time() - t0:.1f}s")
            cells = sum(c.block_info(0).n_real for c in cases)
            warm, steps = max(3, a.warmup), max(1, a.steps)
            forms = {}
            for form in ("persistent", "per-pass", None):
                if form:
                    os.environ["E3D_BATCH_FORM"] = form
                else:
                    os.environ.pop("E3D_BATCH_FORM", None)
                b = api.Batch(cases, precision="fp32", hist_capacity=max(4096, warm + steps + 64))
                b.solve_batch(warm, -1e300, iters_per_launch=warm)  # autotune + warm-up iterations
                torch.cuda.synchronize()
                if form is None:
                    clocks.mark("start")
                _, ms = b.solve_batch(warm + steps, -1e300, iters_per_launch=steps)
                if form is None:
                    clocks.mark("end")
                forms[form or "autotuned"] = {"value": cells * steps / (ms / 1e3), "ms": ms, "tuning": b.tuning()}
                b.close()
            value, ms = forms["autotuned"]["value"], forms["autotuned"]["ms"]
            # plain: the same iterations case after case through the single-case path
            plain = {}
            for prec in ("fp32", "fp64"):
                tot = 0.0
                for c in cases:
                    s = api.Solver(c, precision=prec)
                    s.iterate(warm)
                    tot += s.iterate_timed(steps)
                    s.close()
                plain[prec] = {"value": cells * steps / (tot / 1e3), "ms": tot}
            cpu = None if a.no_cpu_baseline else _ref_sample(
                sorted(decks, key=lambda d: os.path.getsize(d.replace(".deck", ".su2"))), 2,
                min(len(decks), os.cpu_count() or 1))
            line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warm,
                    "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f32", "data": "synthetic",
                    "config": {"workload": f"polar sweep: {len(cases)} bump channels n~U{{{nr[0]}..{nr[1]}}} "
                                           f"(seed 3), Mach U[0.3,0.8], alpha U[-2,6]; AUSM + Green-Gauss + "
                                           f"Barth-Jespersen, order 2, 5-stage RK, CFL 1.5; all cases in one "
                                           f"batch, form and tiles autotuned",
                               "cells": cells, "cases": len(cases),
                               "arithmetic": "fp32 fluxes/gradients/limiters, fp64 conserved state and reductions",
                               "l2": "working set far larger than the 126 MB L2"},
                    "forms": forms, "plain_per_case": plain, "batched_vs_plain_fp32": value / plain["fp32"]["value"],
                    "batched_vs_plain_fp64": value / plain["fp64"]["value"], "cpu_baseline": cpu,
                    "clocks": ClockSampler.summarize(clocks.stop())}
        else:
            t0 = time.time()
            need_train = a.retrain or small or not os.path.exists(WARM_DATA)
            tr_specs = sw.polar_specs(1000, 24 if small else 200, n_range=nr, prefix="train") if need_train else []
            te_specs = sw.polar_specs(2000, 8 if small else 32, n_range=nr, prefix="test")
            decks = sw.write_cases(td, tr_specs + te_specs, sw.WARM_SCHEME, sides="channel")
            cases = [api.Case(d) for d in decks]
            train, test = cases[:len(tr_specs)], cases[len(tr_specs):]
            log(f"[bench] {len(cases)} cases written and loaded in {time.time() - t0:.1f}s")
            crit, max_iter = -8.0, 200000
            if need_train:
                m, tinfo = sw.train_surrogate(train, seed=1000, criterion=-4.0, steps=40000 if not small else 5000)
            else:  # the surrogate trained on the same 200 cases, committed (python -m euler3d_b200.sweep train)
                m, tinfo = sw.load_surrogate(WARM_DATA)
                tinfo = dict(tinfo, source=os.path.relpath(WARM_DATA, HERE))
            log(f"[bench] surrogate: {tinfo}")
            clocks.mark("start")
            learned = sw.solve_batched(test, crit, max_iter, surrogate=m)
            log(f"[bench] batched + learned: {learned['wall_s']:.2f}s {learned['phases']}")
            batched = sw.solve_batched(test, crit, max_iter, surrogate=None)
            log(f"[bench] batched: {batched['wall_s']:.2f}s {batched['phases']}")
            plain = []
            for c in test:
                plain.append(sw.solve_plain(c, crit, max_iter))
                log(f"[bench] plain case {len(plain)}: {plain[-1]}")
            clocks.mark("end")
            t_plain = sum(p["wall_s"] for p in plain)
            cells = sum(p["cells"] for p in plain)
            dcl = max(abs(l["cl"] - p["cl"]) / max(abs(p["cl"]), 1e-2) for l, p in zip(learned["cases"], plain))
            dcd = max(abs(l["cd"] - p["cd"]) / max(abs(p["cd"]), 1e-2) for l, p in zip(learned["cases"], plain))
            line = {"metric": "time to 1e-8 density-residual drop (s)", "value": learned["wall_s"], "unit": "s",
                    "n_gpus": 1, "steps": len(test), "warmup": 0, "ms_per_step": None, "higher_is_better": False,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                    "config": {"workload": f"{len(test)} held-out channel cases n~U{{{nr[0]}..{nr[1]}}} (seed 2000), "
                                           f"Mach U[0.3,0.8], alpha U[-2,6], first-order AUSM, 5-stage RK, CFL 1.5; "
                                           f"surrogate trained on {len(train)} cases (seed 1000)",
                               "cells": cells, "criterion": crit},
                    "plain_s": t_plain, "batched_s": batched["wall_s"], "speedup_learned": t_plain / learned["wall_s"],
                    "speedup_batched_only": t_plain / batched["wall_s"],
                    "iters_plain": [p["reached"] for p in plain],
                    "iters_learned": [c["reached"] for c in learned["cases"]],
                    "iters_batched": [c["reached"] for c in batched["cases"]],
                    "max_rel_dcl": dcl, "max_rel_dcd": dcd,
                    "learned": {k: v for k, v in learned.items() if k != "cases"},
                    "batched": {k: v for k, v in batched.items() if k != "cases"},
                    "surrogate": tinfo, "clocks": ClockSampler.summarize(clocks.stop())}
    print(json.dumps(line))
    return 0


def run_block_sharded(a, rank: int, world: int, local: int) -> int:
    """The channel case with its blocks split over the ranks (euler3d_b200.shard):
    every rank advances its block range, the connexion halo crosses ranks
    after every outer iteration (NCCL all-to-all on the solver stream; no
    exchange at N = 1), and the job's time is the slowest rank's device time
    over the K iterations (CUDA events on the solver stream)."""
    import datetime

    import torch
    import torch.distributed as dist

    from euler3d_b200 import _lib as L
    from euler3d_b200 import shard
    from euler3d_b200.api import Case

    torch.cuda.set_device(local)
    timeout = datetime.timedelta(seconds=120)
    if world > 1:
        dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", local))
    else:
        import socket

        so = socket.socket()
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
        so.close()
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=timeout)
    warm, steps = max(3, a.warmup), max(1, a.steps)
    with tempfile.TemporaryDirectory() as td:
        case = Case(make_case(td, a.n, a.blocks))
        cfg = workload_config(a.n, a.blocks, a.precision)
        cfg["cell_order"] = a.renumber
        run = shard.Sharded(case, precision=a.precision, device=local, renumber=a.renumber,
                            hist_capacity=max(4096, steps + warm + 64))
        s = run.solver
        cells_all = sum(case.block_info(b).n_real for b in range(case.n_blocks))
        cells_mine = sum(info.n_real for info in s._info)
        clocks = ClockSampler(local)
        run.iterate(warm)
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks.mark("start")
        e0.record(run.stream)
        run.step(steps)
        e1.record(run.stream)
        e1.synchronize()
        clocks.mark("end")
        run.gather()
        ms_t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64)
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX, group=run.ctrl)
        ms = float(ms_t.item())
        hist = run.history()
        assert all(abs(x) < 1e300 for x in hist["rms"][:, 0]), "non-finite residual"
        halo = int(s.send_counts.sum() + s.recv_counts.sum())
        launches = (s.launches_per_iteration() + 2) * steps
        # end to end through the public API with host buffers: every step
        # imports this rank's solver state from pinned host memory, runs one
        # sharded iteration (halo exchange and norm gather included) and
        # exports the state back
        nbytes = s.state_bytes()
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        lib = L.lib()
        L.check(lib.e3d_state_export(s._h, C.c_void_p(host.data_ptr()), nbytes))
        e2e_steps = max(3, a.e2e_steps)
        dist.barrier()
        te = time.perf_counter()
        for _ in range(e2e_steps):
            L.check(lib.e3d_state_import(s._h, C.c_void_p(host.data_ptr()), nbytes))
            run.iterate(1)
            L.check(lib.e3d_state_export(s._h, C.c_void_p(host.data_ptr()), nbytes))
        te_t = torch.tensor([time.perf_counter() - te], dtype=torch.float64)
        dist.all_reduce(te_t, op=dist.ReduceOp.MAX, group=run.ctrl)
        e2e = {"value": cells_all * e2e_steps / float(te_t.item()), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": e2e_steps,
               "path": "e3d_state_import (pinned host) + one sharded iteration (halo exchange, norm gather) + "
                       "e3d_state_export, host wall clock, max over ranks"}
        kt = s.time_kernels(min(steps, 10))
        dom = max((k for k in kt if k["bytes_per_launch"]), key=lambda k: k["total_ms"])
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = dom["bytes_per_launch"] / (dom["total_ms"] / dom["launches"] / 1000.0) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "kernel": dom["name"],
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "note": "rank 0's blocks"}
        cl = ClockSampler.summarize(clocks.stop())
        line = {"metric": METRIC, "value": cells_all * steps / (ms / 1000.0), "unit": UNIT, "n_gpus": world,
                "steps": steps, "warmup": warm, "ms_per_step": ms / steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32" if a.precision == "fp32" else "f64",
                "data": "synthetic", "config": dict(cfg, parallelism=f"blocks{world}", cells=cells_all,
                                                    rank0_cells=cells_mine, rank0_halo_entries=halo,
                                                    transport=run.transport),
                "roofline": roofline, "cpu_baseline": None, "e2e": e2e, "gpu_launches": launches, "clocks": cl,
                "final": {"iterations": int(len(hist["iter"])), "ro_conv": float(hist["conv"][-1, 0]),
                          "cl": float(hist["cl"][-1]), "cd": float(hist["cd"][-1])}}
        if rank == 0:
            print(json.dumps(line))
        run.close()
        case.close()
    dist.barrier(group=None)
    dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--blocks", type=int, default=WORKLOAD["blocks"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["channel", "polar", "warmstart", "wing"], default="channel",
                    help="channel: the 3.07M-tet second-order case (default); polar: 64-case batched sweep "
                         "throughput; warmstart: time to an 8-order drop, batched + learned vs plain; wing: the "
                         "~20M-tet swept wing")
    ap.add_argument("--wing-mesh", choices=["body-fitted", "delaunay"], default="body-fitted",
                    help="wing: the body-fitted structured mesh (conforming wall; default) or the seeded Delaunay "
                         "point cloud")
    ap.add_argument("--mesh-dir", default=None,
                    help="wing: a directory holding wing.deck (written by euler3d_b200.wingmesh); generated "
                         "into a temporary directory when absent")
    ap.add_argument("--scale", choices=["full", "small"], default="full",
                    help="small: the same sweep workloads on 10^3..16^3 meshes (quick checks)")
    ap.add_argument("--renumber", default=RENUMBER,
                    choices=[f"{b}{s}" for b in ("none", "rcm", "morton", "shuffle") for s in ("", "+boundary_last")],
                    help="device order of each block's real cells (e3d_options.renumber)")
    ap.add_argument("--no-error-report", action="store_true",
                    help="channel, fp32: skip the FP32-vs-FP64 error report (profiling runs)")
    ap.add_argument("--retrain", action="store_true",
                    help="warmstart: solve the 200 training cases and train the surrogate again instead of "
                         "loading the committed one")
    ap.add_argument("--warm-cases", type=int, default=4,
                    help="channel: held-out cases of the bounded time-to-8-orders comparison (0: skip)")
    ap.add_argument("--fp64-steps", type=int, default=50,
                    help="channel, fp32: also time this many steps of the FP64 bitwise drop-in path (0: skip)")
    ap.add_argument("--mode", choices=["replicas", "blocks"], default="replicas",
                    help="channel, N GPUs: N independent copies of the case (weak scaling, default), or the case's "
                         "blocks split over the N ranks with the halo exchanged every iteration (strong scaling)")
    a = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference_arm(a, rank)
    if a.workload not in ("channel", "wing"):
        return run_sweep_workload(a, rank, world)
    if a.mode == "blocks":
        return run_block_sharded(a, rank, world, local)

    import torch
    import torch.distributed as dist

    from euler3d_b200 import _lib as L
    from euler3d_b200.api import Case, Solver

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    warm = max(3, a.warmup)
    steps = max(1, a.steps)
    with tempfile.TemporaryDirectory() as td:
        t0 = time.time()
        if a.workload == "wing":
            deck, case_dir, cfg = wing_case(a, td)
        else:
            deck, case_dir = make_case(td, a.n, a.blocks), td
            cfg = workload_config(a.n, a.blocks, a.precision)
        cfg["cell_order"] = a.renumber
        t1 = time.time()
        case = Case(deck)
        t2 = time.time()
        s = Solver(case, precision=a.precision, device=local, hist_capacity=max(4096, a.steps + 64),
                   renumber=a.renumber)
        t3 = time.time()
        log(f"[bench] rank {rank}: mesh gen {t1 - t0:.1f}s, case load {t2 - t1:.1f}s, solver setup {t3 - t2:.1f}s, "
            f"device bytes {s.device_bytes() / 1e9:.2f} GB")
        cells = sum(case.block_info(b).n_real for b in range(case.n_blocks))
        cfg["cells"] = cells
        clocks = ClockSampler(local)
        s.iterate(warm)
        s.sync()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks.mark("start")
        ms = s.iterate_timed(steps)  # CUDA events on the solver stream around the K graph launches
        clocks.mark("end")
        torch.cuda.synchronize()
        comb = combine_ranks(ms, cells, steps, world, dist if world > 1 else None, device="cuda")
        ms, value = comb["ms"], comb["value"]
        hist = s.history()
        assert all(abs(x) < 1e300 for x in hist["rms"][:, 0]), "non-finite residual"
        launches = s.launches_per_iteration() * steps

        # per-kernel device times (eager launches with events between kernels)
        kt = s.time_kernels(min(steps, 10))
        dom = max((k for k in kt if k["bytes_per_launch"]), key=lambda k: k["total_ms"])
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        peak = peaks.get("hbm_gbs", 6650.0)
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        achieved = dom["bytes_per_launch"] / (dom["total_ms"] / dom["launches"] / 1000.0) / 1e9
        traffic = None
        try:
            tr = json.load(open(os.path.join(HERE, "profiles", "ncu_traffic.json")))
            traffic = tr.get(f"{a.precision}:{dom['name']}") if a.workload == "channel" else None
        except Exception:
            pass
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "kernel": dom["name"], "peak_source": peak_src,
                    "bytes_per_launch": dom["bytes_per_launch"],
                    "launch_ms": dom["total_ms"] / dom["launches"],
                    "kernels": {k["name"]: {"launches": k["launches"], "ms": k["total_ms"],
                                            "gbs": (k["bytes_per_launch"] / (k["total_ms"] / k["launches"] / 1000.0)
                                                    / 1e9) if k["bytes_per_launch"] else None} for k in kt}}

        # end to end through the C ABI with host buffers: every step imports the
        # solver state from pinned host memory, runs one outer iteration and
        # exports the state back (plus the iteration record)
        nbytes = s.state_bytes()
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        lib = L.lib()
        L.check(lib.e3d_state_export(s._h, C.c_void_p(host.data_ptr()), nbytes))
        e2e_steps = max(3, a.e2e_steps)
        rec = (L.IterRecord * 1)()
        n_hist = C.c_int()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        te = time.perf_counter()
        for _ in range(e2e_steps):
            L.check(lib.e3d_state_import(s._h, C.c_void_p(host.data_ptr()), nbytes))
            L.check(lib.e3d_iterate(s._h, 1))
            L.check(lib.e3d_state_export(s._h, C.c_void_p(host.data_ptr()), nbytes))
            L.check(lib.e3d_history_length(s._h, C.byref(n_hist)))
            L.check(lib.e3d_history(s._h, n_hist.value - 1, 1, C.cast(rec, C.c_void_p)))
        te = time.perf_counter() - te
        t_e = torch.tensor([te], device="cuda", dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t_e, op=dist.ReduceOp.MAX)
        e2e = {"value": world * cells * e2e_steps / float(t_e.item()), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes + C.sizeof(L.IterRecord), "steps": e2e_steps,
               "path": "e3d_state_import (pinned host) + e3d_iterate(1) + e3d_state_export + e3d_history, "
                       "host wall clock"}
        rows = clocks.stop()
        # samples whose timestamps fall in the timed region (nvidia-smi prints no
        # timestamp in this query: keep all samples of the measured run)
        cl = ClockSampler.summarize(rows)

        # the FP64 bitwise drop-in path (the reference's arithmetic) on the same
        # workload, timed the same way: its own solver, warm-up, CUDA events
        fp64_path = None
        if a.precision == "fp32" and a.workload == "channel" and a.fp64_steps > 0:
            s64 = Solver(case, precision="fp64", device=local, hist_capacity=max(4096, a.fp64_steps + 64),
                         renumber=a.renumber)
            s64.iterate(warm)
            s64.sync()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            ms64 = s64.iterate_timed(a.fp64_steps)
            torch.cuda.synchronize()
            c64 = combine_ranks(ms64, cells, a.fp64_steps, world, dist if world > 1 else None, device="cuda")
            kt64 = s64.time_kernels(5)
            fp64_path = {"value": c64["value"], "unit": UNIT, "ms_per_step": c64["ms"] / a.fp64_steps,
                         "steps": a.fp64_steps, "warmup": warm, "dtype": "f64",
                         "note": "the drop-in path: every array bit for bit the reference's",
                         "kernels_gbs": {k["name"]: (k["bytes_per_launch"] / (k["total_ms"] / k["launches"] / 1000.0)
                                                     / 1e9) if k["bytes_per_launch"] else None for k in kt64}}
            s64.close()
        warm8 = None
        if rank == 0 and world == 1 and a.workload == "channel" and a.warm_cases > 0:
            s.close()  # frees the workload's device memory before the sweep
            warm8 = warmstart_bounded(a.warm_cases)
        fp32_err = None
        if rank == 0 and a.precision == "fp32" and a.workload == "channel" and not a.no_error_report:
            fp32_err = fp32_error_report(td)
        cpu = None
        if rank == 0 and world == 1 and not a.no_cpu_baseline:
            try:
                cpu = cpu_baseline_single(deck, case_dir)
            except Exception as e:  # reported, not fatal: the GPU number stands
                cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if a.precision == "fp32" else "f64", "data": "synthetic",
            "config": dict(cfg, parallelism=f"replicas{world}"),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": cl,
            "final": {"iterations": int(len(hist["iter"])), "ro_conv": float(hist["conv"][-1, 0]),
                      "cl": float(hist["cl"][-1]), "cd": float(hist["cd"][-1])},
            "fp32_vs_fp64": fp32_err, "fp64_path": fp64_path, "time_to_8_orders": warm8}
    if rank == 0:
        print(json.dumps(line))
    s.close()
    case.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
