"""Python face of the B200 residual/update path.

Two layers over the C ABI (include/e3d.h):

* ``Case`` / ``Solver``: load the reference's deck + topology + SU2 blocks,
  create a device-resident solver, run fused outer iterations, read results.
* Strategy classes with the reference's names and call structure
  (FluxScheme/RoeScheme/AusmScheme, Gradient/GreenGauss/LeastSquares,
  Limiter/BarthJespersen/Venkatakrishnan, Interpolation/FirstOrder/SecondOrder,
  Timestep, Updater, ResidualCalculator, RungeKutta, ReferenceSolver), selected
  by the same strings (Solver/src/ResidualCalculator.cpp:72-95,
  Solver/src/SecondOrder.cpp:50-61).  Each method launches the matching
  granular kernel on a device-resident ``Block``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L

_ARRAYS_ALL5 = ("prim", "limiter")
_ARRAYS_REAL5 = ("conv_res", "diss_res", "w0")
_ARRAYS_REAL1 = ("dt", "spectral_radius")


class Case:
    """Host case: the reference's Interface + CompleteMesh after InitializeMyBlocks."""

    def __init__(self, deck_path: str, workdir: str | None = None):
        lib = L.lib()
        h = C.c_void_p()
        wd = workdir if workdir is not None else os.path.dirname(os.path.abspath(deck_path))
        L.check(lib.e3d_case_load(deck_path.encode(), wd.encode(), C.byref(h)))
        self._h = h
        n = C.c_int()
        L.check(lib.e3d_case_n_blocks(h, C.byref(n)))
        self.n_blocks = n.value
        d = L.DeckInfo()
        L.check(lib.e3d_case_deck(h, C.byref(d)))
        self.deck = d

    def block_info(self, b: int) -> L.BlockInfo:
        info = L.BlockInfo()
        L.check(L.lib().e3d_case_block_info(self._h, b, C.byref(info)))
        return info

    def get(self, b: int, name: str) -> np.ndarray:
        lib = L.lib()
        n = C.c_int64()
        f64 = name in ("face_normal", "face_area", "face_center", "r_left", "r_right", "cell_volume",
                       "cell_center", "ls_weights", "node_xyz")
        fn = lib.e3d_case_get_f64 if f64 else lib.e3d_case_get_i32
        L.check(fn(self._h, b, name.encode(), None, C.byref(n)))
        out = np.empty(n.value, dtype=np.float64 if f64 else np.int32)
        L.check(fn(self._h, b, name.encode(), L.ptr(out), C.byref(n)))
        return out

    def cell_order(self, b: int, mode: str) -> np.ndarray:
        """order[i] = file index of the real cell a solver with renumber=mode places i-th."""
        n = self.block_info(b).n_real
        out = np.empty(n, dtype=np.int32)
        L.check(L.lib().e3d_case_cell_order(self._h, b, L.RENUMBER[mode], L.ptr(out), n))
        return out

    def close(self):
        if getattr(self, "_h", None):
            L.lib().e3d_case_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Device-resident solver over every block of a case."""

    def __init__(self, case: Case, precision: str = "fp64", carry_w0: int = -1, use_graph: bool = True,
                 device: int = -1, stream: int | None = None, hist_capacity: int = 4096,
                 renumber: str = "none+boundary_last"):
        lib = L.lib()
        o = L.Options()
        lib.e3d_default_options(C.byref(o))
        o.precision = L.FP32 if precision == "fp32" else L.FP64
        o.carry_w0 = carry_w0
        o.use_graph = 1 if use_graph else 0
        o.device = device
        o.stream = stream
        o.hist_capacity = hist_capacity
        o.renumber = L.RENUMBER[renumber]
        h = C.c_void_p()
        L.check(lib.e3d_solver_create(case._h, C.byref(o), C.byref(h)))
        self._h = h
        self.case = case
        self.precision = precision
        self.n_blocks = case.n_blocks
        self._info = [case.block_info(b) for b in range(case.n_blocks)]

    # ---- fused outer iterations
    def iterate(self, n: int) -> None:
        L.check(L.lib().e3d_iterate(self._h, n))

    def solve(self, max_iter: int, criterion: float, check_every: int = 1) -> int:
        done = C.c_int()
        L.check(L.lib().e3d_solve(self._h, max_iter, criterion, check_every, C.byref(done)))
        return done.value

    def iterate_timed(self, n: int) -> float:
        """n outer iterations; returns their device time in ms (CUDA events)."""
        ms = C.c_double()
        L.check(L.lib().e3d_iterate_timed(self._h, n, C.byref(ms)))
        return ms.value

    def state_bytes(self) -> int:
        n = C.c_int64()
        L.check(L.lib().e3d_state_bytes(self._h, C.byref(n)))
        return n.value

    def export_state(self, buf) -> None:
        """Copy the whole solver state into ``buf`` (numpy uint8 array or any
        object exposing a writable buffer address via ``.ctypes.data``)."""
        L.check(L.lib().e3d_state_export(self._h, C.c_void_p(buf.ctypes.data), buf.nbytes))

    def import_state(self, buf) -> None:
        L.check(L.lib().e3d_state_import(self._h, C.c_void_p(buf.ctypes.data), buf.nbytes))

    def sync(self) -> None:
        L.check(L.lib().e3d_solver_sync(self._h))

    def history(self) -> dict[str, np.ndarray]:
        lib = L.lib()
        n = C.c_int()
        L.check(lib.e3d_history_length(self._h, C.byref(n)))
        recs = (L.IterRecord * max(1, n.value))()
        if n.value:
            L.check(lib.e3d_history(self._h, 0, n.value, C.cast(recs, C.c_void_p)))
        r = recs[:n.value]
        return {
            "iter": np.array([x.iter for x in r], dtype=np.int64),
            "rms": np.array([list(x.rms) for x in r]).reshape(-1, 5),
            "conv": np.array([list(x.conv) for x in r]).reshape(-1, 5),
            "cl": np.array([x.cl for x in r]), "cd": np.array([x.cd for x in r]),
            "cmx": np.array([x.cmx for x in r]), "cmy": np.array([x.cmy for x in r]),
            "cmz": np.array([x.cmz for x in r]),
        }

    # ---- state
    def _len(self, b: int, name: str) -> int:
        if not 0 <= b < self.n_blocks:
            return 0  # the C ABI reports the bad block index
        i = self._info[b]
        if name in _ARRAYS_ALL5:
            return 5 * i.n_all
        if name == "grad":
            return 15 * i.n_all
        if name in _ARRAYS_REAL5:
            return 5 * i.n_real
        if name in _ARRAYS_REAL1:
            return i.n_real
        raise KeyError(name)

    def get(self, b: int, name: str) -> np.ndarray:
        out = np.empty(self._len(b, name), dtype=np.float64)
        L.check(L.lib().e3d_state_get(self._h, b, name.encode(), L.ptr(out), out.size))
        return out

    def set(self, b: int, name: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        L.check(L.lib().e3d_state_set(self._h, b, name.encode(), L.ptr(a), a.size))

    def flow_data(self) -> np.ndarray:
        out = np.empty(10 * self.n_blocks, dtype=np.float64)
        L.check(L.lib().e3d_flow_data(self._h, L.ptr(out), out.size))
        return out.reshape(self.n_blocks, 10)

    def device_bytes(self) -> int:
        n = C.c_int64()
        L.check(L.lib().e3d_solver_device_bytes(self._h, C.byref(n)))
        return n.value

    def launches_per_iteration(self) -> int:
        n = C.c_int()
        L.check(L.lib().e3d_launches_per_iteration(self._h, C.byref(n)))
        return n.value

    def time_kernels(self, n_iter: int) -> list[dict]:
        rows = C.c_int()
        names = C.create_string_buffer(1024)
        launches = np.zeros(32, dtype=np.int32)
        ms = np.zeros(32)
        by = np.zeros(32)
        L.check(L.lib().e3d_time_kernels(self._h, n_iter, names, 1024, L.ptr(launches), L.ptr(ms), L.ptr(by), 32,
                                         C.byref(rows)))
        nm = names.value.decode().split(",")
        return [{"name": nm[i], "launches": int(launches[i]), "total_ms": float(ms[i]),
                 "bytes_per_launch": float(by[i])} for i in range(rows.value)]

    def close(self):
        if getattr(self, "_h", None):
            L.lib().e3d_solver_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch(Solver):
    """Several cases advanced together (one device arena, persistent kernel)."""

    def __init__(self, cases: list, precision: str = "fp32", use_graph: bool = True, device: int = -1,
                 hist_capacity: int = 4096, renumber: str = "none+boundary_last"):
        lib = L.lib()
        o = L.Options()
        lib.e3d_default_options(C.byref(o))
        o.precision = L.FP32 if precision == "fp32" else L.FP64
        o.use_graph = 1 if use_graph else 0
        o.device = device
        o.hist_capacity = hist_capacity
        o.renumber = L.RENUMBER[renumber]
        arr = (C.c_void_p * len(cases))(*[c._h.value for c in cases])
        h = C.c_void_p()
        L.check(lib.e3d_batch_create(arr, len(cases), C.byref(o), C.byref(h)))
        self._h = h
        self.cases = cases
        self.case = cases[0]
        self.precision = precision
        self.n_blocks = sum(c.n_blocks for c in cases)
        self._info = [c.block_info(b) for c in cases for b in range(c.n_blocks)]

    def solve_batch(self, max_iter: int, criterion: float, iters_per_launch: int = 10, stall_window: int = 0):
        """Returns (iterations needed per case, device ms of the whole solve)."""
        done = np.zeros(len(self.cases), dtype=np.int32)
        ms = C.c_double()
        L.check(L.lib().e3d_batch_solve(self._h, max_iter, criterion, iters_per_launch, stall_window, L.ptr(done),
                                        C.byref(ms)))
        return done, ms.value

    def case_history(self, c: int) -> dict[str, np.ndarray]:
        lib = L.lib()
        n = C.c_int()
        L.check(lib.e3d_case_history_length(self._h, c, C.byref(n)))
        recs = (L.IterRecord * max(1, n.value))()
        if n.value:
            L.check(lib.e3d_case_history(self._h, c, 0, n.value, C.cast(recs, C.c_void_p)))
        r = recs[:n.value]
        return {"iter": np.array([x.iter for x in r]), "rms": np.array([list(x.rms) for x in r]).reshape(-1, 5),
                "conv": np.array([list(x.conv) for x in r]).reshape(-1, 5), "cl": np.array([x.cl for x in r]),
                "cd": np.array([x.cd for x in r])}

    def tuning(self) -> dict:
        t, g, ms, fc = C.c_int(), C.c_int(), C.c_double(), C.c_int()
        L.check(L.lib().e3d_batch_tuning(self._h, C.byref(t), C.byref(g), C.byref(ms), C.byref(fc)))
        return {"tile_cells": t.value, "grid": g.value, "mode": "per-pass" if g.value == 0 else "persistent",
                "ms_per_iter": ms.value, "from_cache": bool(fc.value)}


def set_precision(solver: Solver, precision: str) -> None:
    """Switch an FP32 solver (or batch) in place: to FP64 ("fp64", or "fp64-fma" for batch
    solves with the FP64 kernels built with fused multiply-add), or to "fp32-delta", FP32
    batch solves in difference form (an FP64 base state and FP32 differences, the base
    residual in FP64), which fall below the FP32 floor (first-order AUSM, tetrahedra)."""
    code = {"fp64": L.FP64, "fp64-fma": L.FP64_FMA, "fp32": L.FP32, "fp32-delta": L.FP32_DELTA}[precision]
    L.check(L.lib().e3d_solver_set_precision(solver._h, code))
    solver.precision = precision if precision in ("fp32", "fp32-delta") else "fp64"


def cell_features(solver: Solver) -> np.ndarray:
    """Surrogate inputs of every real cell, [n_real_total, 8] float32 (x, y, z, wall distance, Mach, alpha, 0, 0)."""
    n = sum(i.n_real for i in solver._info)
    out = np.empty((n, 8), dtype=np.float32)
    L.check(L.lib().e3d_cell_features(solver._h, L.ptr(out), out.size))
    return out


class Surrogate:
    """The per-cell warm-start MLP (6 -> 128 -> 128 -> 128 -> 5, GELU, BF16 weights, FP32 accumulation)."""

    N_PARAMS, N_NORM = L.SURROGATE_PARAMS, L.SURROGATE_NORM

    def __init__(self, seed: int = 0, gamma: float = 1.4, device: int = -1):
        h = C.c_void_p()
        L.check(L.lib().e3d_surrogate_create(device, seed, gamma, C.byref(h)))
        self._h = h

    def add_solution(self, solver: Solver) -> None:
        L.check(L.lib().e3d_surrogate_add_solution(self._h, solver._h))

    def add_samples(self, features: np.ndarray, states: np.ndarray) -> None:
        f = np.ascontiguousarray(features[:, :6], dtype=np.float32)
        w = np.ascontiguousarray(states[:, :5], dtype=np.float32)
        L.check(L.lib().e3d_surrogate_add_samples(self._h, L.ptr(f), L.ptr(w), f.shape[0]))

    @property
    def n_samples(self) -> int:
        n = C.c_int64()
        L.check(L.lib().e3d_surrogate_sample_count(self._h, C.byref(n)))
        return n.value

    def clear(self) -> None:
        L.check(L.lib().e3d_surrogate_clear(self._h))

    def train(self, steps: int, batch: int = 16384, lr: float = 2e-3) -> tuple[float, np.ndarray]:
        hist = np.zeros(max(1, steps), dtype=np.float32)
        loss = C.c_double()
        L.check(L.lib().e3d_surrogate_train(self._h, steps, batch, lr, L.ptr(hist), C.byref(loss)))
        return loss.value, hist[:steps]

    def gradient(self, features: np.ndarray, states: np.ndarray) -> tuple[float, np.ndarray]:
        f = np.ascontiguousarray(features[:, :6], dtype=np.float32)
        w = np.ascontiguousarray(states[:, :5], dtype=np.float32)
        g = np.zeros(self.N_PARAMS, dtype=np.float32)
        loss = C.c_double()
        L.check(L.lib().e3d_surrogate_gradient(self._h, L.ptr(f), L.ptr(w), f.shape[0], L.ptr(g), C.byref(loss)))
        return loss.value, g

    def predict(self, features: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(features[:, :6], dtype=np.float32)
        out = np.zeros((f.shape[0], 5), dtype=np.float32)
        L.check(L.lib().e3d_surrogate_predict(self._h, L.ptr(f), f.shape[0], L.ptr(out)))
        return out

    def get_params(self) -> tuple[np.ndarray, np.ndarray]:
        p = np.zeros(self.N_PARAMS, dtype=np.float32)
        n = np.zeros(self.N_NORM, dtype=np.float32)
        L.check(L.lib().e3d_surrogate_get_params(self._h, L.ptr(p), L.ptr(n)))
        return p, n

    def set_params(self, params: np.ndarray | None = None, norm: np.ndarray | None = None) -> None:
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        n = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        L.check(L.lib().e3d_surrogate_set_params(self._h, None if p is None else L.ptr(p),
                                                 None if n is None else L.ptr(n)))

    def warm_start(self, solver: Solver) -> int:
        n = C.c_int()
        L.check(L.lib().e3d_warm_start(solver._h, self._h, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            L.lib().e3d_surrogate_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------------
# Strategy classes with the reference's names.  A ``Block`` is one block of a
# device-resident solver (the reference's Block*); methods launch one kernel.
class Block:
    def __init__(self, solver: Solver, block_id: int):
        self.solver = solver
        self.block_id_ = block_id

    @property
    def _h(self):
        return self.solver._h


class FluxScheme:
    """Solver/head/FluxScheme.h:9-23."""

    _scheme = None

    def __init__(self, gamma: float):
        self.gamma_ = gamma
        self.current_beta_ = 1.0

    def computeFluxConv(self, block: Block) -> None:
        L.check(L.lib().e3d_flux_conv(block._h, block.block_id_, self._scheme))

    def computeFluxDiss(self, block: Block) -> None:
        L.check(L.lib().e3d_flux_diss(block._h, block.block_id_, self._scheme, self.current_beta_))


class RoeScheme(FluxScheme):
    """Central flux + Roe dissipation (FluxScheme.cpp:16-211, RoeScheme.cpp:12-311)."""

    _scheme = L.FLUX["roe"]


class AusmScheme(FluxScheme):
    """Liou-Steffen AUSM (AusmScheme.cpp:12-243, :647-871)."""

    _scheme = L.FLUX["ausm"]


class Gradient:
    _kind = None

    def computeGradients(self, block: Block) -> None:
        L.check(L.lib().e3d_gradients(block._h, block.block_id_, self._kind))


class GreenGauss(Gradient):
    _kind = L.GRAD["greengauss"]


class LeastSquares(Gradient):
    _kind = L.GRAD["leastsquares"]


class Limiter:
    _kind = None
    omega_ = 0.0
    k_ = 0.0

    def computeLimiters(self, block: Block) -> None:
        L.check(L.lib().e3d_limiters(block._h, block.block_id_, self._kind, self.omega_, self.k_))


class BarthJespersen(Limiter):
    _kind = L.LIM["barthjespersen"]

    def __init__(self, omega: float):
        self.omega_ = omega


class Venkatakrishnan(Limiter):
    _kind = L.LIM["venkatakrishnan"]

    def __init__(self, k: float):
        self.k_ = k


class Interpolation:
    def computeInterpolation(self, block: Block) -> None:
        raise NotImplementedError


class FirstOrder(Interpolation):
    """No reconstruction (FirstOrder.cpp:12-15)."""

    def computeInterpolation(self, block: Block) -> None:
        return None


class SecondOrder(Interpolation):
    """Gradient then limiter (SecondOrder.cpp:20-61): 'leastsquares' else
    Green-Gauss; 'venkatakrishnan' else Barth-Jespersen."""

    def __init__(self, gradient_choice: str, limiter_choice: str, omega: float, k: float):
        self.gradient_ = LeastSquares() if gradient_choice == "leastsquares" else GreenGauss()
        self.limiter_ = Venkatakrishnan(k) if limiter_choice == "venkatakrishnan" else BarthJespersen(omega)

    def computeInterpolation(self, block: Block) -> None:
        self.gradient_.computeGradients(block)
        self.limiter_.computeLimiters(block)


class NoSmoother:
    def smoothResidual(self, block: Block) -> None:
        return None


class CentralIrsSmoother:
    """CentralIrsSmoother.cpp:12-166: one Jacobi step of central implicit residual smoothing."""

    def smoothResidual(self, block: Block) -> None:
        L.check(L.lib().e3d_smooth_residual(block.solver._h, block.block_id_))


RK_TABLES = {  # Solver/src/RungeKutta.cpp:23-68
    1: ([1.0], [1.0]),
    2: ([0.6, 1.0], [1.0, 0.0]),
    3: ([0.6, 0.6, 1.0], [1.0, 0.0, 0.0]),
    4: ([0.25, 1.0 / 3.0, 0.5, 1.0], [1.0, 0.5, 0.0, 0.0]),
    5: ([0.2742, 0.2067, 0.5020, 0.5142, 1.0], [1.0, 0.0, 0.56, 0.0, 0.44]),
}


class ResidualCalculator:
    """ResidualCalculator.cpp:24-95."""

    def __init__(self, gamma, beta_rk, interpolation_choice, gradient_choice, limiter_choice,
                 flux_scheme_choice, residual_smoother_choice, omega, k):
        self.current_stage_ = 0
        self.beta_rk_ = list(beta_rk)
        self.interpolation_ = (SecondOrder(gradient_choice, limiter_choice, omega, k)
                               if interpolation_choice == 2 else FirstOrder())
        if flux_scheme_choice == "roe":
            self.flux_scheme_ = RoeScheme(gamma)
        elif flux_scheme_choice == "ausm":
            self.flux_scheme_ = AusmScheme(gamma)
        else:
            raise ValueError(f"unknown flux scheme {flux_scheme_choice!r} (roe|ausm)")
        self.residual_smoother_ = CentralIrsSmoother() if residual_smoother_choice else NoSmoother()

    def computeResidual(self, block: Block) -> None:
        self.interpolation_.computeInterpolation(block)
        self.flux_scheme_.computeFluxConv(block)
        self.flux_scheme_.current_beta_ = self.beta_rk_[self.current_stage_]
        # the reference guard `beta > (10^-16)` is an integer XOR (== -6): always true
        self.flux_scheme_.computeFluxDiss(block)
        self.residual_smoother_.smoothResidual(block)


class Updater:
    """Updater.cpp:12-88."""

    def __init__(self, gamma, alpha_rk):
        self.gamma_ = gamma
        self.alpha_rk_ = list(alpha_rk)
        self.current_stage_ = 0

    def updateInternalBlock(self, block: Block) -> None:
        L.check(L.lib().e3d_update_internal(block._h, block.block_id_, self.alpha_rk_[self.current_stage_]))

    def updateBoundary(self, block: Block) -> None:
        L.check(L.lib().e3d_update_boundary(block._h, block.block_id_))


class Timestep:
    """Timestep.cpp:26-148."""

    def __init__(self, gamma, cfl):
        self.gamma_ = gamma
        self.cfl_ = cfl

    def computeSpectralRadius(self, block: Block) -> None:
        L.check(L.lib().e3d_spectral_radius(block._h, block.block_id_))

    def computeTimestep(self, block: Block) -> None:
        L.check(L.lib().e3d_timestep(block._h, block.block_id_))


class RungeKutta:
    """RungeKutta.cpp:15-94."""

    def __init__(self, gamma, stage_number, interpolation_choice, gradient_choice, limiter_choice,
                 flux_scheme_choice, residual_smoother_choice, omega, k):
        if stage_number not in RK_TABLES:
            raise ValueError("Invalid number of RK stages")
        self.stage_number_ = stage_number
        alpha, beta = RK_TABLES[stage_number]
        self.updater_ = Updater(gamma, alpha)
        self.residual_calculator_ = ResidualCalculator(gamma, beta, interpolation_choice, gradient_choice,
                                                       limiter_choice, flux_scheme_choice,
                                                       residual_smoother_choice, omega, k)

    def computeRungeKutta(self, block: Block) -> None:
        for s in range(self.stage_number_):
            self.residual_calculator_.current_stage_ = s
            self.residual_calculator_.computeResidual(block)
            self.updater_.current_stage_ = s
            self.updater_.updateInternalBlock(block)
            self.updater_.updateBoundary(block)


def save_w0(block: Block) -> None:
    """Solver::saveW0 (Solver.cpp:161-210)."""
    L.check(L.lib().e3d_save_w0(block._h, block.block_id_))


def halo(solver: Solver) -> None:
    """BlockCommunicator::updateBoundaries (MPI/src/BlockCommunicator.cpp:66-270)."""
    L.check(L.lib().e3d_halo(solver._h))


class ReferenceSolver:
    """Solver::solve (Solver.cpp:36-98) sequenced call by call through the strategy
    objects, block after block, on the device.  ``iterate`` runs n outer
    iterations and returns the per-block flow data after each one."""

    def __init__(self, solver: Solver):
        d = solver.case.deck
        self.solver = solver
        self.timestep_ = Timestep(d.gamma, d.cfl)
        grad = "leastsquares" if d.gradient == L.GRAD["leastsquares"] else "greengauss"
        lim = "venkatakrishnan" if d.limiter == L.LIM["venkatakrishnan"] else "barthjespersen"
        flux = {0: "roe", 1: "ausm"}[d.flux]
        self.runge_kutta_ = RungeKutta(d.gamma, d.stages, d.order, grad, lim, flux, bool(d.smoothing),
                                       d.omega, d.k)
        self.blocks = [Block(solver, b) for b in range(solver.n_blocks)]
        self._started = False

    def iterate(self, n: int) -> list[np.ndarray]:
        if not self._started:
            halo(self.solver)
            self._started = True
        out = []
        for _ in range(n):
            for b in self.blocks:
                save_w0(b)
                self.timestep_.computeSpectralRadius(b)
                self.timestep_.computeTimestep(b)
                self.runge_kutta_.computeRungeKutta(b)
            out.append(self.solver.flow_data())
            halo(self.solver)
        return out
