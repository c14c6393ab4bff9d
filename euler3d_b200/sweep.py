"""Mach/alpha polar sweeps: seeded case lists, the plain per-case solve, and the
batched + learned solve (every case in one batch, surrogate warm start, FP32
until the FP32 rounding floor, then FP64 to the target drop).

The reference runs one case per process (Solver/src/Solver.cpp:76-97 loops a
single mesh until PostProcessing.cpp:77 finds ro_convergence_ <= criterion);
a sweep there is many such runs.  The plain arm here is that same loop on the
GPU, case after case, through the FP64 drop-in path.  The batched arm solves
the same discrete equations: per case it stops at the same density drop,
measured from the same reference residual (the freestream start's first
iteration), so both reach the same converged Cl/Cd.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import api
from . import meshgen as mg


@dataclass
class CaseSpec:
    name: str
    n: int           # hexahedra per side (6 n^3 tetrahedra)
    mach: float
    aoa_deg: float


def polar_specs(seed: int, count: int, n_range=(25, 60), mach_range=(0.3, 0.8), aoa_range=(-2.0, 6.0),
                prefix="case") -> list[CaseSpec]:
    """Seeded sweep: n ~ U{n_range}, Mach ~ U[mach_range], alpha ~ U[aoa_range] (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    n = rng.integers(n_range[0], n_range[1] + 1, count)
    mach = rng.uniform(mach_range[0], mach_range[1], count)
    aoa = rng.uniform(aoa_range[0], aoa_range[1], count)
    return [CaseSpec(f"{prefix}{seed}_{i}", int(n[i]), float(mach[i]), float(aoa[i])) for i in range(count)]


def _write_one(args):
    directory, spec, scheme, sides = args
    d = mg.Deck(topology="", mach=spec.mach, aoa_deg=spec.aoa_deg, max_iter=1000000, criterion=-15.0, **scheme)
    return mg.write_case(os.path.join(directory, spec.name), spec.n, 1, prefix=spec.name, deck=d, sides=sides)


def write_cases(directory: str, specs: list[CaseSpec], scheme: dict, sides: str = "farfield",
                processes: int | None = None) -> list[str]:
    """Write every case (SU2 block, .top, deck) in parallel; returns the deck paths in spec order.

    Worker processes are started with 'spawn', so this is safe after CUDA has
    been initialised in the calling process."""
    jobs = [(directory, s, scheme, sides) for s in specs]
    procs = processes or min(len(jobs), os.cpu_count() or 1, 32)
    if procs <= 1:
        return [_write_one(j) for j in jobs]
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(_write_one, jobs, chunksize=1)


def _first_below(conv: np.ndarray, level: float) -> int | None:
    hit = np.nonzero(conv <= level)[0]
    return int(hit[0]) + 1 if hit.size else None


def solve_plain(case: api.Case, criterion: float, max_iter: int, check_every: int = 50,
                precision: str = "fp64") -> dict:
    """The reference's loop on the GPU for one case: freestream start, fused
    iterations until the density drop reaches `criterion`."""
    s = api.Solver(case, precision=precision, hist_capacity=max(4096, check_every * 4))
    t0 = time.perf_counter()
    s.solve(max_iter, criterion, check_every)
    wall = time.perf_counter() - t0
    h = s.history()
    c = h["conv"][:, 0]
    out = dict(iters=len(c), reached=_first_below(c, criterion), wall_s=wall, cl=float(h["cl"][-1]),
               cd=float(h["cd"][-1]), cells=sum(case.block_info(b).n_real for b in range(case.n_blocks)))
    s.close()
    return out


def solve_batched(cases: list[api.Case], criterion: float, max_iter: int, surrogate: api.Surrogate | None = None,
                  switch_at: float | None = -5.0, iters_per_launch: int = 50, stall_window: int = 400,
                  fp64: str = "auto") -> dict:
    """All cases in one batch: one freestream iteration (the reference residual
    of each case's drop), the surrogate's warm start when given, FP32
    iterations to `switch_at` (below a 4-order drop, a case whose FP32
    residual has stopped falling for `stall_window` iterations, its FP32
    rounding floor, also moves on),
    then the finishing phase to `criterion` (`fp64`: "fp64-fma" for the FP64
    kernels built with fused multiply-add, "fp64" for the bit-identical ones,
    "fp32-delta" for FP32 iterations in difference form on an FP64 base,
    "auto" for the difference form where the scheme has it (first-order AUSM
    on tetrahedra; the fastest form there) and contracted FP64 elsewhere); each
    case leaves the work list once it gets there."""
    t0 = time.perf_counter()
    b = api.Batch(cases, precision="fp32" if switch_at is not None else "fp64",
                  hist_capacity=max(4096, iters_per_launch * 4))
    if switch_at is None and fp64 in ("fp64-fma", "auto"):
        fp64 = "fp64-fma"
        api.set_precision(b, fp64)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    b.solve_batch(1, -1e300, iters_per_launch=1)
    fallback = 0
    t_warm = 0.0
    if surrogate is not None:
        tw = time.perf_counter()
        fallback = surrogate.warm_start(b)
        t_warm = time.perf_counter() - tw
    phases = []
    if switch_at is not None:
        tp = time.perf_counter()
        # stall detection only near the floor: the early transient of a freestream
        # start has plateaus of its own
        b.solve_batch(max_iter, max(switch_at, -4.0), iters_per_launch=iters_per_launch)
        b.solve_batch(max_iter, switch_at, iters_per_launch=iters_per_launch, stall_window=stall_window)
        phases.append(dict(precision="fp32", to=switch_at, wall_s=time.perf_counter() - tp, tuning=b.tuning()))
        tp = time.perf_counter()
        if fp64 == "auto":
            try:
                api.set_precision(b, "fp32-delta")
                fp64 = "fp32-delta"
            except L.E3DError as e:
                if e.code != L.ERRORS_BY_NAME["E3D_ERR_ARG"]:
                    raise
                fp64 = "fp64-fma"
                api.set_precision(b, fp64)
        else:
            api.set_precision(b, fp64)
        phases.append(dict(precision="switch", wall_s=time.perf_counter() - tp))
    tp = time.perf_counter()
    b.solve_batch(max_iter, criterion, iters_per_launch=iters_per_launch)
    phases.append(dict(precision=fp64 if switch_at is not None else "fp64", to=criterion,
                       wall_s=time.perf_counter() - tp, tuning=b.tuning()))
    wall = time.perf_counter() - t0
    per_case = []
    for c in range(len(cases)):
        h = b.case_history(c)
        cv = h["conv"][:, 0]
        per_case.append(dict(iters=len(cv), reached=_first_below(cv, criterion), cl=float(h["cl"][-1]),
                             cd=float(h["cd"][-1])))
    b.close()
    return dict(wall_s=wall, setup_s=t_setup, warm_s=t_warm, fallback=fallback, phases=phases, cases=per_case)


def train_surrogate(cases: list[api.Case], seed: int, criterion: float = -4.0, max_iter: int = 200000,
                    steps: int = 40000, batch: int = 32768, lr: float = 3e-3, iters_per_launch: int = 200,
                    group: int = 64, stall_window: int = 3000) -> tuple[api.Surrogate, dict]:
    """Solves the training cases in batches of `group` (FP32, freestream start)
    to `criterion`, adds every real cell's converged state to the surrogate's
    sample store, and trains it."""
    m = api.Surrogate(seed=seed, gamma=1.4)
    t0 = time.perf_counter()
    cell_iters = 0
    for g0 in range(0, len(cases), group):
        part = cases[g0:g0 + group]
        b = api.Batch(part, precision="fp32", hist_capacity=max(4096, iters_per_launch * 4))
        b.solve_batch(max_iter, criterion, iters_per_launch=iters_per_launch, stall_window=stall_window)
        for c, case in enumerate(part):
            cell_iters += int(b.case_history(c)["conv"].shape[0]) * sum(
                case.block_info(k).n_real for k in range(case.n_blocks))
        m.add_solution(b)
        b.close()
    t_solve = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss, hist = m.train(steps, batch=batch, lr=lr)
    t_train = time.perf_counter() - t0
    return m, dict(samples=m.n_samples, solve_s=t_solve, train_s=t_train, loss=loss,
                   loss_first=float(np.mean(hist[:20])), cell_iters=cell_iters)


def save_surrogate(m: api.Surrogate, path: str, info: dict) -> None:
    """Trained parameters and input/output normalisation, with how they were made."""
    params, norm = m.get_params()
    np.savez_compressed(path, params=params, norm=norm, info=np.array(json.dumps(info)))


def load_surrogate(path: str, gamma: float = 1.4, device: int = -1) -> tuple[api.Surrogate, dict]:
    z = np.load(path)
    m = api.Surrogate(seed=0, gamma=gamma, device=device)
    m.set_params(z["params"], z["norm"])
    return m, json.loads(str(z["info"]))


# The warm-start workload: first-order AUSM on the channel variant of the bump
# mesh (z planes and top SYMMETRY, inlet and outlet FARFIELD), where every case
# of the sweep's Mach/alpha range converges to an 8-order drop.
WARM_SCHEME = dict(order=1, flux="ausm", stages=5, cfl=1.5)
TRAIN_SEED, HELD_OUT_SEED = 1000, 2000


def train_warmstart(out: str, n_cases: int = 200, n_range=(25, 60), steps: int = 40000,
                    workdir: str | None = None) -> dict:
    """Solves the seeded training sweep, trains the surrogate on the converged
    states and writes it to `out` (see save_surrogate)."""
    import tempfile

    with tempfile.TemporaryDirectory(dir=workdir) as td:
        specs = polar_specs(TRAIN_SEED, n_cases, n_range=n_range, prefix="train")
        decks = write_cases(td, specs, WARM_SCHEME, sides="channel")
        cases = [api.Case(d) for d in decks]
        m, info = train_surrogate(cases, seed=TRAIN_SEED, criterion=-4.0, steps=steps)
        info.update(scheme=WARM_SCHEME, train_seed=TRAIN_SEED, cases=n_cases, n_range=list(n_range))
        save_surrogate(m, out, info)
        for c in cases:
            c.close()
    return info


# The swept-wing configuration's warm start: the surrogate learns converged
# states of a coarse body-fitted wing over Mach and alpha and warm-starts the
# fine mesh.  Its inputs (cell centre, distance to the wall, Mach, alpha) do
# not depend on the mesh, so a surrogate trained on one resolution applies to
# another of the same geometry.
WING_SCHEME = dict(order=2, flux="ausm", gradient="leastsquares", limiter="venkatakrishnan", k=5.0,
                   omega=2.16e-16, stages=5, cfl=1.5)
WING_TRAIN_SEED = 3000


def wing_points(seed: int, count: int, mach_range=(0.5, 0.85), aoa_range=(0.0, 5.0)) -> list[tuple[float, float]]:
    """Seeded (Mach, alpha) points, uniform in both (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    mach = rng.uniform(mach_range[0], mach_range[1], count)
    aoa = rng.uniform(aoa_range[0], aoa_range[1], count)
    return [(round(float(m), 4), round(float(a), 4)) for m, a in zip(mach, aoa)]


def write_wing_cases(directory: str, dims: tuple, points: list[tuple[float, float]], scheme: dict = WING_SCHEME,
                     n_blocks: int = 1) -> list[str]:
    """One body-fitted wing mesh (dims: ni, nj, nk_wing, nk_out) and one deck
    per (Mach, alpha) point, all naming the same topology; returns the decks."""
    from . import wingmesh as wm

    def deck(m, a):
        return mg.Deck(topology="wing.top", mach=m, aoa_deg=a, max_iter=1000000, criterion=-15.0, **scheme)

    first, _ = wm.write_body_fitted_wing_case(directory, *dims, n_blocks=n_blocks, deck=deck(*points[0]))
    decks = [first]
    for i, (m, a) in enumerate(points[1:], 1):
        path = os.path.join(directory, f"wing_{i}.deck")
        mg.write_deck(path, deck(m, a))
        decks.append(path)
    return decks


# the wing's time to an 8-order drop runs first-order AUSM (the second-order
# scheme has no 8-order drop on airfoil and wing meshes)
WING_WARM_SCHEME = dict(order=1, flux="ausm", stages=5, cfl=1.5)


def wing_warmstart(n_train: int = 32, train_dims=(64, 20, 24, 8), target_dims=(128, 40, 48, 16), mach: float = 0.8,
                   aoa: float = 3.0, criterion: float = -8.0, out: str | None = None,
                   workdir: str | None = None) -> dict:
    """Trains the surrogate on n_train coarse wings (seeded Mach/alpha, solved
    to -4 in FP32), then times the target wing from freestream to `criterion`:
    plain (FP64 drop-in path) against learned (warm start, FP32 to its floor,
    FP64 with contraction to the criterion)."""
    import tempfile

    rec = dict(n_train=n_train, train_dims=list(train_dims), target_dims=list(target_dims), mach=mach, aoa=aoa,
               criterion=criterion, scheme=WING_WARM_SCHEME)
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        pts = wing_points(WING_TRAIN_SEED, n_train)
        cases = [api.Case(d) for d in write_wing_cases(os.path.join(td, "train"), train_dims, pts,
                                                        scheme=WING_WARM_SCHEME)]
        m, info = train_surrogate(cases, seed=WING_TRAIN_SEED, criterion=-4.0, steps=40000, group=16)
        rec["train"] = info
        if out:
            save_surrogate(m, out, dict(info, points=pts, dims=list(train_dims), scheme=WING_WARM_SCHEME))
        target = api.Case(write_wing_cases(os.path.join(td, "target"), target_dims, [(mach, aoa)],
                                           scheme=WING_WARM_SCHEME)[0])
        rec["plain"] = solve_plain(target, criterion, 1000000, check_every=100)
        rec["learned"] = solve_batched([target], criterion, 1000000, surrogate=m)
        rec["speedup"] = rec["plain"]["wall_s"] / rec["learned"]["wall_s"]
        for c in cases + [target]:
            c.close()
    return rec


def finishing_forms(n: int = 48, count: int = 8, iters: int = 300, depth_cases: int = 2,
                    depth: float = -11.0) -> dict:
    """The finishing phase's three forms on one batch of `count` channel cases
    (n^3 x 6 tets each, first-order AUSM, per-pass form for all three): device
    ms per iteration of FP32, FP32 in difference form and FP64 with
    contraction, each after 100 warm-up iterations; then `depth_cases` of them
    from freestream to `depth`, once in contracted FP64 and once FP32 to -5
    followed by the difference form (iterations needed, converged Cl/Cd)."""
    import tempfile

    specs = polar_specs(HELD_OUT_SEED, count, n_range=(n, n), prefix="test")
    rec = dict(n=n, cases=count, iters=iters, scheme=WARM_SCHEME, forms={})
    old_form = os.environ.get("E3D_BATCH_FORM")
    os.environ["E3D_BATCH_FORM"] = "per-pass"
    try:
        with tempfile.TemporaryDirectory() as td:
            cases = [api.Case(d) for d in write_cases(td, specs, WARM_SCHEME, sides="channel")]
            cells = sum(c.block_info(b).n_real for c in cases for b in range(c.n_blocks))
            rec["cells"] = cells
            b = api.Batch(cases, precision="fp32", hist_capacity=4096)
            it = 1
            b.solve_batch(it, -1e300, iters_per_launch=1)
            for form in ("fp32", "fp32-delta", "fp64-fma"):
                if form != "fp32":
                    api.set_precision(b, form)
                it += 100
                b.solve_batch(it, -1e300, iters_per_launch=50)
                it += iters
                _, ms = b.solve_batch(it, -1e300, iters_per_launch=100)
                rec["forms"][form] = dict(ms_per_iter=ms / iters, cell_iters_per_s=cells * iters / (ms / 1e3))
            b.close()
            sub = cases[:depth_cases]
            if sub:
                a = solve_batched(sub, depth, 200000, switch_at=None, fp64="fp64-fma")
                d = solve_batched(sub, depth, 200000, switch_at=-5.0, fp64="fp32-delta")
                rec["depth"] = dict(level=depth, fp64_fma=a, fp32_then_delta=d,
                                    max_rel_dcl=max(abs(x["cl"] - y["cl"]) / abs(y["cl"])
                                                    for x, y in zip(d["cases"], a["cases"])),
                                    max_rel_dcd=max(abs(x["cd"] - y["cd"]) / abs(y["cd"])
                                                    for x, y in zip(d["cases"], a["cases"])))
            for c in cases:
                c.close()
    finally:
        if old_form is None:
            os.environ.pop("E3D_BATCH_FORM", None)
        else:
            os.environ["E3D_BATCH_FORM"] = old_form
    return rec


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Warm-start surrogates: train on the seeded channel sweep, time "
                                             "the swept wing's drop with and without one, or time the finishing "
                                             "phase's forms.")
    ap.add_argument("command", choices=["train", "wing", "finishing"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--cases", type=int, default=None)
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--n", type=int, default=48, help="finishing: hexahedra per side of each case")
    ap.add_argument("--iters", type=int, default=300, help="finishing: timed iterations per form")
    ap.add_argument("--depth-cases", type=int, default=2, help="finishing: cases of the depth check (0: none)")
    a = ap.parse_args(argv)
    if a.command == "train":
        if not a.out:
            ap.error("train needs --out")
        info = train_warmstart(a.out, n_cases=a.cases or 200, steps=a.steps)
    elif a.command == "wing":
        info = wing_warmstart(n_train=a.cases or 32, out=a.out)
    else:
        info = finishing_forms(n=a.n, count=a.cases or 8, iters=a.iters, depth_cases=a.depth_cases)
    print(json.dumps(info))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
