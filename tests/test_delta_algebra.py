"""The difference-form AUSM face flux (euler3d_b200/csrc/delta.cu), restated
in float32 numpy, against the float64 difference of the reference's AUSM
face flux (AusmScheme.cpp:12-243, 716-871; the same expressions as
physics.cuh's flux_ausm_conv / flux_ausm_diss).  Host only: this checks the
algebra the kernel uses, not the kernel (tests/test_delta_gpu.py runs that).

Bar: the float32 difference form's error, relative to the size of the flux
change, stays at float32 rounding (measured about 1e-6; bound 1e-5) for state
changes from 1e-2 down to 1e-7 of the state, also across the AUSM branch
points (|M| = 1 and the |M| <= 0.25 dissipation fix).  Subtracting two float32
fluxes instead loses the change at the small end (measured 4e-5, 3e-3, 0.3
and 3.8 of the change at 1e-2, 1e-4, 1e-6 and 1e-7): that is the FP32 floor
the difference form removes.
"""
import numpy as np

F = np.float32
G, GR = 1.4, 1.4 / 0.4


def ausm64(L, R, n, nn):
    """Reference AUSM face flux (convective, dissipative) in float64."""
    def side(q):
        r, u, v, w, p = q
        H = 0.5 * (u * u + v * v + w * w) + GR * p / r
        V = u * n[0] + v * n[1] + w * n[2]
        c = np.sqrt(G * p / r)
        return r, u, v, w, p, H, V / c, c
    rL, uL, vL, wL, pL, HL, ML, cL = side(L)
    rR, uR, vR, wR, pR, HR, MR, cR = side(R)
    if ML <= -1.0:
        pLp, MLp = 0.0, 0.0
    elif ML < 1.0:
        pLp, MLp = pL * 0.25 * (ML + 1.0) ** 2 * (2.0 - ML), 0.25 * (ML + 1.0) ** 2
    else:
        pLp, MLp = pL, ML
    if MR <= -1.0:
        pRm, MRm = pR, MR
    elif MR < 1.0:
        pRm, MRm = pR * 0.25 * (1.0 - MR) ** 2 * (2.0 + MR), -0.25 * (MR - 1.0) ** 2
    else:
        pRm, MRm = 0.0, 0.0
    M = MLp + MRm
    FL = np.array([rL * cL, rL * uL * cL, rL * vL * cL, rL * wL * cL, rL * HL * cL])
    FR = np.array([rR * cR, rR * uR * cR, rR * vR * cR, rR * wR * cR, rR * HR * cR])
    fc = 0.5 * M * (FL + FR) * nn
    fc[1:4] += np.asarray(n) * (pLp + pRm) * nn
    Mf = M if abs(M) > 0.25 else (M * M + 0.0625) / 0.5
    fd = 0.5 * abs(Mf) * (FR - FL) * nn
    return fc, fd


def dcell(b, d):
    """delta.cu dcell: face-independent quantities as base value + difference (float32)."""
    r, u, v, w, p = (F(x) for x in b)
    dr, du, dv, dw, dp = (F(x) for x in d)
    qq = u * u + v * v + w * w
    dqq = du * (F(2) * u + du) + dv * (F(2) * v + dv) + dw * (F(2) * w + dw)
    pr = p * (F(1) / r)
    dpr = (dp - pr * dr) / (r + dr)
    H, dH = F(0.5) * qq + F(GR) * pr, F(0.5) * dqq + F(GR) * dpr
    x, x1 = F(G) * pr, F(G) * (pr + dpr)
    ic, ic1 = F(1) / np.sqrt(x), F(1) / np.sqrt(x1)
    c, c1 = x * ic, x1 * ic1
    dc = F(G) * dpr / (c + c1)
    F1, dF1 = r * c, dr * c1 + r * dc
    return dict(u=u, v=v, w=w, p=p, du=du, dv=dv, dw=dw, dp=dp, H=H, dH=dH, dc=dc, ic=ic, ic1=ic1, F1=F1, dF1=dF1)


def piecewise(x, d, lo, hi, i0, i1, piece):
    if i0 == i1:
        return piece(i0, x, d)
    acc, x0, rest = F(0), x, d
    step = 1 if i1 > i0 else -1
    for i in range(i0, i1, step):
        bp = (lo if i == 0 else hi) if step == 1 else (hi if i == 2 else lo)
        e = F(bp) - x0
        acc += piece(i, x0, e)
        rest -= e
        x0 = F(bp)
    return acc + piece(i1, x0, rest)


def split_piece(M):
    return 0 if M <= -1 else (1 if M < 1 else 2)


def fix_piece(M):
    return 0 if M < -0.25 else (1 if M <= 0.25 else 2)


def side_flux(s):
    Fv = [s["F1"], s["F1"] * s["u"], s["F1"] * s["v"], s["F1"] * s["w"], s["F1"] * s["H"]]
    dF = [s["dF1"], s["dF1"] * (s["u"] + s["du"]) + s["F1"] * s["du"],
          s["dF1"] * (s["v"] + s["dv"]) + s["F1"] * s["dv"],
          s["dF1"] * (s["w"] + s["dw"]) + s["F1"] * s["dw"],
          s["dF1"] * (s["H"] + s["dH"]) + s["F1"] * s["dH"]]
    return Fv, dF


def ausm_delta32(bL, dL, bR, dR, n, nn):
    """delta.cu ausm_delta_face<true> in float32."""
    L, R = dcell(bL, dL), dcell(bR, dR)
    nx, ny, nz, nn = F(n[0]), F(n[1]), F(n[2]), F(nn)

    def mach(s):
        V = s["u"] * nx + s["v"] * ny + s["w"] * nz
        dV = s["du"] * nx + s["dv"] * ny + s["dw"] * nz
        M = V * s["ic"]
        return M, (dV - M * s["dc"]) * s["ic1"]
    LM, LdM = mach(L)
    RM, RdM = mach(R)
    iL0, iL1 = split_piece(LM), split_piece(LM + LdM)
    MLp = [F(0), F(0.25) * (LM + 1) * (LM + 1), LM][iL0]
    PLp = [F(0), F(0.25) * (LM + 1) * (LM + 1) * (F(2) - LM), F(1)][iL0]
    dMLp = piecewise(LM, LdM, -1, 1, iL0, iL1,
                     lambda i, x, e: [F(0), F(0.25) * e * (F(2) * (x + 1) + e), e][i])
    dPLp = piecewise(LM, LdM, -1, 1, iL0, iL1,
                     lambda i, x, e: F(0.25) * e * (F(3) - F(3) * x * x - F(3) * x * e - e * e) if i == 1 else F(0))
    iR0, iR1 = split_piece(RM), split_piece(RM + RdM)
    MRm = [RM, F(-0.25) * (RM - 1) * (RM - 1), F(0)][iR0]
    PRm = [F(1), F(0.25) * (F(1) - RM) * (F(1) - RM) * (F(2) + RM), F(0)][iR0]
    dMRm = piecewise(RM, RdM, -1, 1, iR0, iR1,
                     lambda i, x, e: [e, F(-0.25) * e * (F(2) * (x - 1) + e), F(0)][i])
    dPRm = piecewise(RM, RdM, -1, 1, iR0, iR1,
                     lambda i, x, e: F(0.25) * e * (F(-3) + F(3) * x * x + F(3) * x * e + e * e) if i == 1 else F(0))
    M, dM = MLp + MRm, dMLp + dMRm
    dpLp = L["dp"] * (PLp + dPLp) + L["p"] * dPLp
    dpRm = R["dp"] * (PRm + dPRm) + R["p"] * dPRm
    FL, dFL = side_flux(L)
    FR, dFR = side_flux(R)
    h = F(0.5) * nn
    fc = [h * (dM * (FL[k] + FR[k] + dFL[k] + dFR[k]) + M * (dFL[k] + dFR[k])) for k in range(5)]
    dps = (dpLp + dpRm) * nn
    fc[1] += nx * dps
    fc[2] += ny * dps
    fc[3] += nz * dps
    j0, j1 = fix_piece(M), fix_piece(M + dM)
    aM = [-M, (M * M + F(0.0625)) * F(2), M][j0]
    daM = piecewise(M, dM, -0.25, 0.25, j0, j1, lambda i, x, e: [-e, F(2) * e * (F(2) * x + e), e][i])
    fd = [h * (daM * (FR[k] - FL[k] + dFR[k] - dFL[k]) + aM * (dFR[k] - dFL[k])) for k in range(5)]
    return np.array(fc, dtype=np.float64), np.array(fd, dtype=np.float64)


def _state(rng, mach, along=None):
    """A primitive state (rho, u, v, w, p) moving at `mach` sound speeds, in a
    random direction or along the unit vector `along` (normal Mach = mach)."""
    r, p = rng.uniform(0.8, 1.2), rng.uniform(0.6, 0.8)
    c = np.sqrt(G * p / r)
    e = rng.normal(size=3) if along is None else along
    u = mach * c * e / np.linalg.norm(e)
    return np.array([r, u[0], u[1], u[2], p])


def _faces(rng, count, mach_range, aligned=False):
    out = []
    for _ in range(count):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        a = n if aligned else None
        out.append((_state(rng, rng.uniform(*mach_range), a), _state(rng, rng.uniform(*mach_range), a), n,
                    rng.uniform(0.5, 2.0)))
    return out


def _rel_errors(faces, rng, scale, naive=False):
    worst = 0.0
    for bL, bR, n, nn in faces:
        dL = rng.normal(size=5) * scale * np.abs(bL).clip(0.1)
        dR = rng.normal(size=5) * scale * np.abs(bR).clip(0.1)
        # the base the kernel sees is float32; its float64 value is the reference point
        bL32, bR32 = bL.astype(np.float32).astype(np.float64), bR.astype(np.float32).astype(np.float64)
        dL32, dR32 = dL.astype(np.float32).astype(np.float64), dR.astype(np.float32).astype(np.float64)
        c1, d1 = ausm64(bL32 + dL32, bR32 + dR32, n.astype(np.float32).astype(np.float64), float(F(nn)))
        c0, d0 = ausm64(bL32, bR32, n.astype(np.float32).astype(np.float64), float(F(nn)))
        exact = np.concatenate([c1 - c0, d1 - d0])
        if naive:  # two float32 fluxes subtracted: what the plain FP32 variant resolves
            qa = [x.astype(np.float32) for x in (bL32 + dL32, bR32 + dR32)]
            qb = [x.astype(np.float32) for x in (bL32, bR32)]
            ca, da = ausm64(*[x.astype(np.float64) for x in qa], n, nn)
            cb, db = ausm64(*[x.astype(np.float64) for x in qb], n, nn)
            got = np.concatenate([ca.astype(np.float32) - cb.astype(np.float32),
                                  da.astype(np.float32) - db.astype(np.float32)]).astype(np.float64)
        else:
            fc, fd = ausm_delta32(bL32, dL32, bR32, dR32, n, nn)
            got = np.concatenate([fc, fd])
        worst = max(worst, np.max(np.abs(got - exact)) / max(np.max(np.abs(exact)), 1e-300))
    return worst


def test_difference_form_error_scales_with_the_flux_change():
    rng = np.random.default_rng(11)
    faces = _faces(rng, 300, (0.0, 0.9))
    for scale in (1e-2, 1e-4, 1e-6, 1e-7):
        assert _rel_errors(faces, rng, scale) < 1e-5, scale
    # the plain float32 difference of two fluxes has lost the change at the small end
    assert _rel_errors(faces, rng, 1e-7, naive=True) > 0.5


def _pieces(q, n):
    r, u, v, w, p = q
    M = (u * n[0] + v * n[1] + w * n[2]) / np.sqrt(G * p / r)
    return split_piece(M)


def test_difference_form_across_the_branch_points():
    rng = np.random.default_rng(12)
    # states moving along the face normal at a normal Mach number just either
    # side of 1 (split branches) and of 0.25 (the interface Mach number there is
    # near the normal one, at the dissipation fix), changed by about as much
    scale = 1e-3
    faces = (_faces(rng, 300, (1 - 2 * scale, 1 + 2 * scale), aligned=True)
             + _faces(rng, 300, (0.25 - 2 * scale, 0.25 + 2 * scale), aligned=True))
    assert _rel_errors(faces, rng, scale) < 1e-5
    # the sample does cross the branch points: count faces whose left state's split changes
    crossed = 0
    for bL, bR, n, nn in faces[:300]:
        dL = rng.normal(size=5) * scale * np.abs(bL).clip(0.1)
        crossed += _pieces(bL, n) != _pieces(bL + dL, n)
    assert crossed > 20
