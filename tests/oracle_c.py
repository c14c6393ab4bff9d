"""ctypes driver for the C restatement oracle (oracle/libe3d_oracle.so) and for
the same source built as a model of the FP32 variant (oracle/libe3d_oracle32.so).

Test infrastructure: used by tests/ and by bench.py's CPU-baseline leg only.
Blocks are assembled from per-block geometry arrays (the reference's own, from
a golden dump, or the host library's, which tests pin bitwise to them).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "oracle", "libe3d_oracle.so")
LIB32 = os.path.join(REPO, "oracle", "libe3d_oracle32.so")

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


class OBlock(C.Structure):
    _fields_ = [("n_real", C.c_int), ("n_all", C.c_int), ("n_faces", C.c_int),
                ("face_cells", IP), ("face_normal", DP), ("face_area", DP), ("face_center", DP), ("r_left", DP),
                ("r_right", DP), ("cell_face_ptr", IP), ("cell_faces", IP), ("cell_cells", IP), ("cell_volume", DP),
                ("ls_weights", DP), ("n_markers", C.c_int), ("n_real_boundaries", C.c_int), ("marker_kind", IP),
                ("marker_size", IP), ("marker_cells", IP), ("n_wall_faces", C.c_int), ("wall_faces", IP),
                ("prim", DP), ("conv_res", DP), ("diss_res", DP), ("w0", DP), ("grad", DP), ("limiter", DP),
                ("dt", DP), ("spectral_radius", DP)]


class OParams(C.Structure):
    _fields_ = [("gamma", C.c_double), ("cfl", C.c_double), ("mach", C.c_double), ("aoa_deg", C.c_double),
                ("cmac", C.c_double), ("omega", C.c_double), ("k", C.c_double), ("stages", C.c_int),
                ("order", C.c_int), ("flux", C.c_int), ("gradient", C.c_int), ("limiter", C.c_int),
                ("smoothing", C.c_int)]


class OConn(C.Structure):
    _fields_ = [("dest_block", C.c_int), ("origin_block", C.c_int), ("n", C.c_int), ("dest_cells", IP),
                ("origin_cells", IP)]


_libs: dict = {}


def lib(fp32: bool = False):
    """The FP64 oracle, or (fp32=True) the model of the FP32 variant."""
    path = LIB32 if fp32 else LIB
    if path not in _libs:
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C oracle oracle`")
        _libs[path] = C.CDLL(path)
        _libs[path].e3d_oracle_set_noise.argtypes = [C.c_ulonglong]
    return _libs[path]


def _p(a, t):
    return a.ctypes.data_as(t)


class OracleBlock:
    """One block: geometry arrays + owned FP64 state in the reference layouts."""

    GEO = ("face_cells", "face_normal", "face_area", "face_center", "r_left", "r_right", "cell_face_ptr",
           "cell_faces", "cell_cells", "cell_volume", "ls_weights", "marker_kind", "marker_size", "marker_cells",
           "wall_faces")

    def __init__(self, geo: dict, n_real: int, n_all: int, n_faces: int, n_real_boundaries: int):
        self.a = {}
        for k in self.GEO:
            dt = np.float64 if k in ("face_normal", "face_area", "face_center", "r_left", "r_right", "cell_volume",
                                     "ls_weights") else np.int32
            self.a[k] = np.ascontiguousarray(geo[k], dtype=dt)
        self.prim = np.zeros(5 * n_all)
        self.conv_res = np.zeros(5 * n_all)
        self.diss_res = np.zeros(5 * n_all)
        self.w0 = np.zeros(5 * n_all)
        self.grad = np.zeros(15 * n_all)
        self.limiter = np.zeros(5 * n_all)
        self.dt = np.zeros(n_real)
        self.spectral_radius = np.zeros(n_real)
        a = self.a
        self.s = OBlock(n_real, n_all, n_faces, _p(a["face_cells"], IP), _p(a["face_normal"], DP),
                        _p(a["face_area"], DP), _p(a["face_center"], DP), _p(a["r_left"], DP), _p(a["r_right"], DP),
                        _p(a["cell_face_ptr"], IP), _p(a["cell_faces"], IP), _p(a["cell_cells"], IP),
                        _p(a["cell_volume"], DP), _p(a["ls_weights"], DP), len(a["marker_kind"]), n_real_boundaries,
                        _p(a["marker_kind"], IP), _p(a["marker_size"], IP), _p(a["marker_cells"], IP),
                        len(a["wall_faces"]), _p(a["wall_faces"], IP), _p(self.prim, DP), _p(self.conv_res, DP),
                        _p(self.diss_res, DP), _p(self.w0, DP), _p(self.grad, DP), _p(self.limiter, DP),
                        _p(self.dt, DP), _p(self.spectral_radius, DP))
        self.n_real, self.n_all = n_real, n_all

    @classmethod
    def from_golden(cls, g, b: int) -> "OracleBlock":
        cnt = g[f"init.b{b}.counts"]
        geo = {k: g[f"init.b{b}.{k}"] for k in cls.GEO if k != "cell_face_ptr"}
        nf = g[f"init.b{b}.cell_nfaces"]
        geo["cell_face_ptr"] = np.concatenate([[0], np.cumsum(nf)]).astype(np.int32)
        return cls(geo, int(cnt[0]), int(cnt[1]), int(cnt[2]), int(cnt[3]))

    @classmethod
    def from_case(cls, case, b: int) -> "OracleBlock":
        info = case.block_info(b)
        geo = {k: case.get(b, k) for k in cls.GEO}
        return cls(geo, info.n_real, info.n_all, info.n_faces, info.n_real_boundaries)


def params_from_deck(d) -> OParams:
    """d: a DeckInfo from the C ABI or a dict of meshgen.Deck fields."""
    get = (lambda k: d[k]) if isinstance(d, dict) else (lambda k: getattr(d, k))
    if isinstance(d, dict):
        flux = {"roe": 0, "ausm": 1}[d["flux"]]
        grad = 1 if d["gradient"] == "leastsquares" else 0
        lim = 1 if d["limiter"] == "venkatakrishnan" else 0
    else:
        flux, grad, lim = d.flux, d.gradient, d.limiter
    return OParams(get("gamma"), get("cfl"), get("mach"), get("aoa_deg"), get("cmac"), get("omega"), get("k"),
                   get("stages"), get("order"), flux, grad, lim, int(bool(get("smoothing"))))


class OracleCase:
    """All blocks of a case plus the connexion lists; runs outer iterations."""

    def __init__(self, blocks: list[OracleBlock], params: OParams, connexions: list[tuple] = (), fp32: bool = False,
                 noise_seed: int = 0):
        self.fp32 = fp32
        self.noise_seed = noise_seed
        self.blocks = blocks
        self.p = params
        self.arr = (OBlock * len(blocks))(*[b.s for b in blocks])
        self._conn_keep = []
        cs = []
        for dest, origin, dcells, ocells in connexions:
            d = np.ascontiguousarray(dcells, dtype=np.int32)
            o = np.ascontiguousarray(ocells, dtype=np.int32)
            self._conn_keep += [d, o]
            cs.append(OConn(dest, origin, len(d), _p(d, IP), _p(o, IP)))
        self.conns = (OConn * max(1, len(cs)))(*cs)
        self.n_conn = len(cs)
        self.rms0 = (C.c_double * 5)()
        self.have_rms0 = C.c_int(0)
        self.iters = 0
        for i in range(len(blocks)):
            lib(fp32).e3d_oracle_init_state(C.byref(self.arr[i]), C.byref(self.p))

    def iterate(self, n: int) -> np.ndarray:
        hist = np.zeros((n, 15))
        L = lib(self.fp32)
        if self.fp32:
            L.e3d_oracle_set_noise(self.noise_seed)  # restarts the seeded sequence
            if self.iters:
                raise ValueError("the FP32 model runs its iterations in one call (seeded noise sequence)")
        rc = L.e3d_oracle_iterate(self.arr, len(self.blocks), self.conns, self.n_conn, C.byref(self.p), n,
                                  self.iters, self.rms0, C.byref(self.have_rms0), _p(hist, DP))
        if self.fp32:
            L.e3d_oracle_set_noise(0)
        assert rc == 0
        self.iters += n
        return hist

    def call(self, fn: str, b: int, *args) -> None:
        getattr(lib(self.fp32), "e3d_oracle_" + fn)(C.byref(self.arr[b]), *args)


def connexions_from_topology(path: str, n_real: list[int]) -> list[tuple]:
    """Parses a .top file the way the reference does (CompleteMesh.cpp:170-292)."""
    lines = open(path).read().split("\n")
    nb = int(lines[0].split()[1])
    pos = 1 + nb
    entries = {}
    while pos < len(lines) and lines[pos].strip():
        idx = int(lines[pos].split()[1])
        gc = int(lines[pos + 1].split()[1])
        m = int(lines[pos + 2].split()[1])
        pos += 3
        marks = []
        for _ in range(m):
            origin = int(lines[pos].split()[1])
            k = int(lines[pos + 1].split()[1])
            cells = [int(x) for x in lines[pos + 2:pos + 2 + k]]
            pos += 2 + k
            marks.append((origin, cells))
        entries[idx] = (gc, marks)
    out = []
    for b in range(nb):
        if b not in entries:
            continue
        count, marks = entries[b]
        for origin, cells in marks:
            dest = list(range(count, count + len(cells)))
            count += len(cells)
            out.append((b, origin, dest, cells))
    return out


def case_oracle(case, top_path: str, fp32: bool = False, noise_seed: int = 0) -> OracleCase:
    blocks = [OracleBlock.from_case(case, b) for b in range(case.n_blocks)]
    return OracleCase(blocks, params_from_deck(case.deck),
                      connexions_from_topology(top_path, [b.n_real for b in blocks]), fp32=fp32,
                      noise_seed=noise_seed)
