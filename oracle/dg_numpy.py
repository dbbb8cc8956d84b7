"""Test infrastructure only: CPU restatement (numpy, FP64) of the reference's
hot path for entropy variables on periodic blocks. It is the checker of the
CUDA path and is never called by the product.

Parity of this restatement is pinned against the golden fixtures produced by
the reference solver itself (tests/golden/make_golden.py, oracle/_ref).

Follows, function by function:
  volume_residual   ElementClass::VolumeResidual            src/ElementClass.cpp:3809-4443
  face traces       TPSAG{I,J,K}                              include/TensorProductSolAndGrad[IJK]Face.hpp
  interior faces    FluxesInternalFace                        src/FluxesFace.cpp:220-343
                    InviscidFluxesFace (entropy branch)       src/FluxesFace.cpp:694-975
                    ViscousFluxesFace, PenAndSymFluxesSymmVar src/FluxesFace.cpp:1152-1651
  face residuals    I/J/KFaceResiduals + neighbour sums       src/ElementClass.cpp:2582-3404,
                                                              src/SolverClass.cpp:3616-3732
  mass solve        CG_EntropyVarMassMatrix                   src/CG_MassMatrix.cpp:250-504
  time step         ElementClass::ComputeTimeStep             src/ElementClass.cpp:1522-1644
  nodal gradients   ComputeVelocityGradientsNodalDOFs         src/ElementClass.cpp:1647-1795
  SGS models        CWALEModel / CVremanModel::EddyViscosity  src/SGSModel.cpp:35-202
  Runge-Kutta       ExecuteTimeSynchronizationStep stages     src/SolverClass.cpp:2368-2396
The metric-index behaviour of the reference (gradient and symmetrizing-flux
transforms take the metric of point l = variable index) is reproduced when
compat=True.

Arrays: state U[e, v, k, j, i] (modal, K per axis); integration-point data
[e, ..., k, j, i] (M per axis); face data [e, ..., slow, fast].
"""
from __future__ import annotations

import dataclasses

import numpy as np

GAM = 1.4
GM1 = GAM - 1.0
FHF_LAM = GAM / 0.72
FHF_TURB = GAM / 0.90          # turbulent Prandtl number 0.9
LAM_OVER_MU = -2.0 / 3.0
EPS_SMALL = 1e-30
SGS_NONE, SGS_WALE, SGS_VREMAN = 0, 1, 2


@dataclasses.dataclass
class Disc:
    """Operators and geometry (the shapes of include/vcp3d_b200.h)."""
    K: int
    M: int
    leg: np.ndarray          # [K, M]
    dleg: np.ndarray         # [K, M]
    face: np.ndarray         # [2, K]
    dface: np.ndarray        # [2, K]
    w: np.ndarray            # [M]
    legdof: np.ndarray       # [K, K]
    center: np.ndarray       # [K^3]
    vol: np.ndarray          # [nE, 10, M^3]
    fmet: np.ndarray         # [nE, 6, 13, M^2]
    scal: np.ndarray         # [nE, 15]
    nbr: np.ndarray          # [nE, 6]
    mu: float
    tau_num: float           # (p+1)^2 * relative penalty
    theta: float
    riemann: int             # 0 Roe, 1 Ismail-Roe
    p_ref: float
    u_ref: float
    rho_ref: float
    cfl: float
    n_poly: int
    sgs: int = SGS_NONE      # subgrid-scale model
    fbody: tuple = None      # body force per unit volume / p_ref, or None
    dlegdof: np.ndarray = None   # [K, K] basis derivative at the 1-D nodal DOFs
    vmd: np.ndarray = None       # [nE, 10, K^3] metric terms at the nodal DOFs


# ---------------------------------------------------------------------------
# Tensor contractions along one axis of [e, v, a2, a1, a0].
# ---------------------------------------------------------------------------
def _ax(x, op, axis):
    """Apply op[c, o] along the given array axis (contracting c)."""
    y = np.tensordot(x, op, axes=([axis], [0]))
    return np.moveaxis(y, -1, axis)


def vol_interp(U, leg, dleg):
    """TPSAGV: value and parametric derivatives (r=i, s=j, t=k) at the Gauss points."""
    tK = _ax(U, leg, 2)
    tJ = _ax(tK, leg, 3)
    val = _ax(tJ, leg, 4)
    dr = _ax(tJ, dleg, 4)
    ds = _ax(_ax(tK, dleg, 3), leg, 4)
    dt = _ax(_ax(_ax(U, dleg, 2), leg, 3), leg, 4)
    return val, dr, ds, dt


def vol_project(F, opk, opj, opi):
    """TPAVR: sum_m op(k,m) ... F at points -> DOFs (op given as [K, M], used transposed)."""
    return _ax(_ax(_ax(F, opk.T, 2), opj.T, 3), opi.T, 4)


def entropy_to_prim(V):
    V4Inv = 1.0 / V[4]
    u, v, w = -V4Inv * V[1], -V4Inv * V[2], -V4Inv * V[3]
    eKin = 0.5 * (u * u + v * v + w * w)
    s = GAM - GM1 * (V[0] - V[4] * eKin)
    rho = (-V[4] * np.exp(s)) ** (-1.0 / GM1)
    p = -rho * V4Inv
    return rho, u, v, w, p, eKin


def _weights3(w):
    """mIntWeights[k][j][i] = (w_i w_j) w_k (StandardElementClass::DataStandardElement)."""
    return (w[None, None, :] * w[None, :, None]) * w[:, None, None]


def _cart_grad(dr, ds, dt, met, off, compat):
    """Parametric -> Cartesian gradients; met[e, q, pt]; off = index of dr/dx.

    Volume metric: off = 1 (dr/dx at 1, dr/dy at 2, ..., dt/dz at 9).
    Face metric:   off = 4.
    dr, ds, dt: [e, 5, P]. compat: variable n uses the metric of point n.
    """
    if compat:
        # Fewer than 5 points (faces with M = 2): variable 4 reads the padding,
        # a copy of point 0 (src/ElementClass.cpp:1163-1173).
        idx = [n if n < met.shape[2] else 0 for n in range(5)]
        m = met[:, off:off + 9, idx][:, :, :, None]     # [e, 9, n, 1]
    else:
        m = met[:, off:off + 9, None, :]                 # [e, 9, 1, P]
    gx = dr * m[:, 0] + ds * m[:, 3] + dt * m[:, 6]
    gy = dr * m[:, 1] + ds * m[:, 4] + dt * m[:, 7]
    gz = dr * m[:, 2] + ds * m[:, 5] + dt * m[:, 8]
    return gx, gy, gz


def eddy_viscosity(model, length, rho, G):
    """Dynamic eddy viscosity of the WALE (C_w = 0.325) or Vreman (c = 0.07)
    model, src/SGSModel.cpp:35-202. G[i][j] = d u_i / d x_j, length = the
    element's LES length scale (broadcastable against rho)."""
    if model == SGS_NONE:
        return np.zeros_like(rho)
    if model == SGS_WALE:
        lw = 0.325 * length
        S = [[0.5 * (G[i][j] + G[j][i]) for j in range(3)] for i in range(3)]
        G2 = [[G[i][0] * G[0][j] + G[i][1] * G[1][j] + G[i][2] * G[2][j] for j in range(3)]
              for i in range(3)]
        Sd = [[0.5 * (G2[i][j] + G2[j][i]) for j in range(3)] for i in range(3)]
        tr = (Sd[0][0] + Sd[1][1] + Sd[2][2]) / 3.0
        for i in range(3):
            Sd[i][i] = Sd[i][i] - tr
        sumS = (S[0][0] ** 2 + S[1][1] ** 2 + S[2][2] ** 2
                + 2.0 * (S[0][1] ** 2 + S[0][2] ** 2 + S[1][2] ** 2))
        sumSd = (Sd[0][0] ** 2 + Sd[1][1] ** 2 + Sd[2][2] ** 2
                 + 2.0 * (Sd[0][1] ** 2 + Sd[0][2] ** 2 + Sd[1][2] ** 2))
        sd32 = sumSd * np.sqrt(sumSd)
        denom = sumS * sumS * np.sqrt(sumS) + np.sqrt(sd32 * sumSd)
        return rho * (lw * lw) * sd32 / np.maximum(denom, EPS_SMALL)
    # Vreman: alpha = G with its trace removed from the diagonal.
    tr = (G[0][0] + G[1][1] + G[2][2]) / 3.0
    a = [[G[i][j] - (tr if i == j else 0.0) for j in range(3)] for i in range(3)]
    l2 = length * length
    b = [[l2 * (a[i][0] * a[j][0] + a[i][1] * a[j][1] + a[i][2] * a[j][2]) for j in range(3)]
         for i in range(3)]
    B = (b[0][0] * b[1][1] - b[0][1] ** 2 + b[0][0] * b[2][2] - b[0][2] ** 2
         + b[1][1] * b[2][2] - b[1][2] ** 2)
    B = np.maximum(B, 0.0)
    denom = sum(a[i][j] ** 2 for i in range(3) for j in range(3))
    return rho * 0.07 * np.sqrt(B / np.maximum(denom, EPS_SMALL))


def volume_residual(U, d: Disc, compat=True):
    """Volume part of the residual and the CG point data (src/ElementClass.cpp:3809-4443)."""
    nE, M = U.shape[0], d.M
    MD = M ** 3
    val, dr, ds, dt = vol_interp(U, d.leg, d.dleg)
    V = val.reshape(nE, 5, MD)
    gx, gy, gz = _cart_grad(dr.reshape(nE, 5, MD), ds.reshape(nE, 5, MD),
                            dt.reshape(nE, 5, MD), d.vol, 1, compat)
    rho, u, v, w, p, eKin = entropy_to_prim(V.transpose(1, 0, 2))
    ov1mg = -1.0 / GM1
    V4Inv = 1.0 / V[:, 4]
    rE = -p * ov1mg + rho * eKin
    dudx, dudy, dudz = [-V4Inv * (g[:, 1] + u * g[:, 4]) for g in (gx, gy, gz)]
    dvdx, dvdy, dvdz = [-V4Inv * (g[:, 2] + v * g[:, 4]) for g in (gx, gy, gz)]
    dwdx, dwdy, dwdz = [-V4Inv * (g[:, 3] + w * g[:, 4]) for g in (gx, gy, gz)]
    fact = -V4Inv * V4Inv * ov1mg
    dedx, dedy, dedz = gx[:, 4] * fact, gy[:, 4] * fact, gz[:, 4] * fact
    W3 = _weights3(d.w).reshape(MD)
    J = d.vol[:, 0]
    weight = -J * W3
    eddy = eddy_viscosity(d.sgs, d.scal[:, 3:4], rho, [[dudx, dudy, dudz], [dvdx, dvdy, dvdz],
                                                       [dwdx, dwdy, dwdz]])
    mu = d.mu + eddy
    ru, rv, rw = rho * u, rho * v, rho * w
    div = LAM_OVER_MU * (dudx + dvdy + dwdz)
    txx, tyy, tzz = mu * (2 * dudx + div), mu * (2 * dvdy + div), mu * (2 * dwdz + div)
    txy, txz, tyz = mu * (dudy + dvdx), mu * (dudz + dwdx), mu * (dvdz + dwdy)
    kq = d.mu * FHF_LAM + eddy * FHF_TURB
    qx, qy, qz = -kq * dedx, -kq * dedy, -kq * dedz
    fx = [ru, ru * u - txx + p, rv * u - txy, rw * u - txz,
          (rE + p) * u - (u * txx + v * txy + w * txz - qx)]
    fy = [rv, ru * v - txy, rv * v - tyy + p, rw * v - tyz,
          (rE + p) * v - (u * txy + v * tyy + w * tyz - qy)]
    fz = [rw, ru * w - txz, rv * w - tyz, rw * w - tzz + p,
          (rE + p) * w - (u * txz + v * tyz + w * tzz - qz)]
    vm = d.vol
    F = []
    for q in range(3):
        m1, m2, m3 = (weight * vm[:, 1 + 3 * q + c] for c in range(3))
        F.append(np.stack([fx[n] * m1 + fy[n] * m2 + fz[n] * m3 for n in range(5)], axis=1)
                 .reshape(nE, 5, M, M, M))
    R = (vol_project(F[0], d.leg, d.leg, d.dleg) + vol_project(F[1], d.leg, d.dleg, d.leg)
         + vol_project(F[2], d.dleg, d.leg, d.leg))
    if d.fbody is not None:
        # Body force: -J w (f, u . f) on momentum and energy (src/ElementClass.cpp:4495-4533).
        fx, fy, fz = d.fbody
        S = np.stack([weight * fx, weight * fy, weight * fz,
                      weight * (u * fx + v * fy + w * fz)], axis=1).reshape(nE, 4, M, M, M)
        R[:, 1:] = R[:, 1:] + vol_project(S, d.leg, d.leg, d.leg)
    cg = dict(rho=rho, u=u, v=v, w=w, p=p, rE=rE, eKin=eKin, JW=J * W3, eddy_max=eddy.max())
    return R, cg


def face_traces(U, d: Disc):
    """Value and (dr, ds, dt) on the six faces of every element, [e, 5, slow, fast]."""
    out = []
    for f in range(6):
        dd, g = f // 2, f % 2
        nax = 4 - dd                       # array axis of the face-normal index
        bn = np.moveaxis(np.tensordot(U, d.face[g], axes=([nax], [0])), 0, 0)
        bnd = np.tensordot(U, d.dface[g], axes=([nax], [0]))
        val = _ax(_ax(bn, d.leg, 3), d.leg, 2)
        dS = _ax(_ax(bn, d.leg, 3), d.dleg, 2)
        dF = _ax(_ax(bn, d.dleg, 3), d.leg, 2)
        dN = _ax(_ax(bnd, d.leg, 3), d.leg, 2)
        if dd == 0:
            out.append((val, dN, dF, dS))
        elif dd == 1:
            out.append((val, dF, dN, dS))
        else:
            out.append((val, dF, dS, dN))
    return out


def _face_prim(V):
    """Primitive variables as in InviscidFluxesFace (note 0.5*V4*|v|^2)."""
    V4Inv = 1.0 / V[4]
    u, v, w = -V4Inv * V[1], -V4Inv * V[2], -V4Inv * V[3]
    vt2 = u * u + v * v + w * w
    s = GAM - GM1 * (V[0] - 0.5 * V[4] * vt2)
    rho = (-V[4] * np.exp(s)) ** (-1.0 / GM1)
    return rho, u, v, w, -V4Inv * rho, vt2


def _logmean_F(zeta):
    f = (zeta - 1.0) / (zeta + 1.0)
    u = f * f
    series = 1.0 + u / 3.0 + u * u / 5.0 + u * u * u / 7.0 + u * u * u * u / 9.0
    with np.errstate(divide="ignore", invalid="ignore"):
        exact = np.log(zeta) / (2.0 * f)
    return np.where(u < 0.01, series, exact)


def ismail_roe(VL, VR, nx, ny, nz, area):
    """Entropy branch of InviscidFluxesFace, Ismail-Roe (src/FluxesFace.cpp:813-975)."""
    rL, uL, vL, wL, pL, _ = _face_prim(VL)
    rR, uR, vR, wR, pR, _ = _face_prim(VR)
    dV = [VR[n] - VL[n] for n in range(5)]
    z0L, z0R = np.sqrt(rL / pL), np.sqrt(rR / pR)
    z4L, z4R = np.sqrt(rL * pL), np.sqrt(rR * pR)
    z0A, z4A = 0.5 * (z0L + z0R), 0.5 * (z4L + z4R)
    z1A, z2A, z3A = 0.5 * (uL * z0L + uR * z0R), 0.5 * (vL * z0L + vR * z0R), 0.5 * (wL * z0L + wR * z0R)
    z0Log = z0A / _logmean_F(z0L / z0R)
    z4Log = z4A / _logmean_F(z4L / z4R)
    inv = 1.0 / z0A
    rA = z0A * z4Log
    p1 = inv * z4A
    p2 = 0.5 * ((GAM + 1) / GAM * z4Log / z0Log + GM1 / GAM * p1)
    uA, vA, wA = inv * z1A, inv * z2A, inv * z3A
    vn = uA * nx + vA * ny + wA * nz
    kin = 0.5 * (uA * uA + vA * vA + wA * wA)
    a2 = GAM * p2 / rA
    a = np.sqrt(a2)
    H = a2 / GM1 + kin
    E = H - p2 / rA
    abv1 = rA * (uA * dV[1] + vA * dV[2] + wA * dV[3])
    abv2 = abv1 + rA * (dV[0] + H * dV[4])
    dr = abv1 + rA * (dV[0] + E * dV[4])
    dru, drv, drw = uA * abv2 + p2 * dV[1], vA * abv2 + p2 * dV[2], wA * abv2 + p2 * dV[3]
    drE = H * abv1 + rA * E * (dV[0] + H * dV[4]) + p2 * kin * dV[4]
    lam1 = np.abs(vn + a) * 0.5 * (1 + 1.0 / 6.0)
    lam2 = np.abs(vn - a) * 0.5 * (1 + 1.0 / 6.0)
    lam3 = np.abs(vn) * 0.5
    b1, b2 = 0.5 * (lam1 + lam2), 0.5 * (lam1 - lam2)
    b3 = b1 - lam3
    b4 = GM1 * (kin * dr - uA * dru - vA * drv - wA * drw + drE)
    b5 = nx * dru + ny * drv + nz * drw - vn * dr
    b6 = b3 * b4 / a2 + b2 * b5 / a
    b7 = b2 * b4 / a + b3 * b5
    f = [rA * vn - (lam3 * dr + b6),
         rA * vn * uA + p1 * nx - (lam3 * dru + uA * b6 + nx * b7),
         rA * vn * vA + p1 * ny - (lam3 * drv + vA * b6 + ny * b7),
         rA * vn * wA + p1 * nz - (lam3 * drw + wA * b6 + nz * b7),
         rA * vn * H - (lam3 * drE + H * b6 + vn * b7)]
    return [fi * area for fi in f]


def roe(VL, VR, nx, ny, nz, halfArea):
    """Entropy branch of InviscidFluxesFace, Roe with entropy fix (src/FluxesFace.cpp:694-809)."""
    rL, uL, vL, wL, pL, v2L = _face_prim(VL)
    rR, uR, vR, wR, pR, v2R = _face_prim(VR)
    rEL, rER = pL / GM1 + 0.5 * rL * v2L, pR / GM1 + 0.5 * rR * v2R
    dr, dru, drv, drw, drE = rR - rL, rR * uR - rL * uL, rR * vR - rL * vL, rR * wR - rL * wL, rER - rEL
    zL, zR = np.sqrt(rL), np.sqrt(rR)
    t = 1.0 / (zL + zR)
    uA, vA, wA = t * (zL * uL + zR * uR), t * (zL * vL + zR * vR), t * (zL * wL + zR * wR)
    H = t * ((rEL + pL) / zL + (rER + pR) / zR)
    alpha = 0.5 * (uA * uA + vA * vA + wA * wA)
    a2 = np.abs(GM1 * (H - alpha))
    a = np.sqrt(a2)
    vn = uA * nx + vA * ny + wA * nz
    l1, l2, l3 = np.abs(vn + a), np.abs(vn - a), np.abs(vn)
    t = 0.001 * np.maximum(l1, l2)
    l1, l2, l3 = np.maximum(l1, t), np.maximum(l2, t), np.maximum(l3, t)
    b1, b2 = 0.5 * (l1 + l2), 0.5 * (l1 - l2)
    b3 = b1 - l3
    b4 = GM1 * (alpha * dr - uA * dru - vA * drv - wA * drw + drE)
    b5 = nx * dru + ny * drv + nz * drw - vn * dr
    b6 = b3 * b4 / a2 + b2 * b5 / a
    b7 = b2 * b4 / a + b3 * b5
    vnL, vnR = uL * nx + vL * ny + wL * nz, uR * nx + vR * ny + wR * nz
    pa = halfArea * (pL + pR)
    return [halfArea * (rL * vnL + rR * vnR - (l3 * dr + b6)),
            halfArea * (rL * uL * vnL + rR * uR * vnR - (l3 * dru + uA * b6 + nx * b7)) + pa * nx,
            halfArea * (rL * vL * vnL + rR * vR * vnR - (l3 * drv + vA * b6 + ny * b7)) + pa * ny,
            halfArea * (rL * wL * vnL + rR * wR * vnR - (l3 * drw + wA * b6 + nz * b7)) + pa * nz,
            halfArea * (rEL * vnL + rER * vnR + pL * vnL + pR * vnR
                        - (l3 * drE + H * b6 + vn * b7))]


def viscous_face(VL, VR, gx, gy, gz, nnx, nny, nnz, wf, area, mu_lam, tau, theta, f,
                 sgs=SGS_NONE, len_les=None):
    """ViscousFluxesFace + PenAndSymFluxesSymmVar (src/FluxesFace.cpp:1152-1651), entropy
    variables; the eddy viscosity of the averaged state when an SGS model is used.
    Updates f in place; returns Cartesian symmetrizing fluxes and the eddy viscosity."""
    V = [0.5 * (VL[n] + VR[n]) for n in range(5)]
    V4Inv = 1.0 / V[4]
    u, v, w = -V4Inv * V[1], -V4Inv * V[2], -V4Inv * V[3]
    du = [-V4Inv * (g[1] + u * g[4]) for g in (gx, gy, gz)]
    dv = [-V4Inv * (g[2] + v * g[4]) for g in (gx, gy, gz)]
    dw = [-V4Inv * (g[3] + w * g[4]) for g in (gx, gy, gz)]
    if sgs != SGS_NONE:
        rho = (-V[4] * np.exp(GAM - GM1 * (V[0] - V[4] * 0.5 * (u * u + v * v + w * w)))) \
            ** (-1.0 / GM1)
        eddy = eddy_viscosity(sgs, len_les, rho, [du, dv, dw])
    else:
        eddy = np.zeros_like(u)
    mu = mu_lam + eddy
    fe = V4Inv * V4Inv / GM1
    de = [fe * g[4] for g in (gx, gy, gz)]
    dV = [VL[n] - VR[n] for n in range(5)]
    pOvRho = -V4Inv
    A = wf * area
    nx, ny, nz = A * nnx, A * nny, A * nnz
    div = LAM_OVER_MU * (du[0] + dv[1] + dw[2])
    txx, tyy, tzz = mu * (2 * du[0] + div), mu * (2 * dv[1] + div), mu * (2 * dw[2] + div)
    txy, txz, tyz = mu * (du[1] + dv[0]), mu * (du[2] + dw[0]), mu * (dv[2] + dw[1])
    kq = mu_lam * FHF_LAM + eddy * FHF_TURB
    qx, qy, qz = -kq * de[0], -kq * de[1], -kq * de[2]
    f[1] = f[1] - (txx * nx + txy * ny + txz * nz)
    f[2] = f[2] - (txy * nx + tyy * ny + tyz * nz)
    f[3] = f[3] - (txz * nx + tyz * ny + tzz * nz)
    f[4] = f[4] - ((u * txx + v * txy + w * txz - qx) * nx + (u * txy + v * tyy + w * tyz - qy) * ny
                   + (u * txz + v * tyz + w * tzz - qz) * nz)
    lam, lp1, lp2 = LAM_OVER_MU, LAM_OVER_MU + 1, LAM_OVER_MU + 2
    e = pOvRho / GM1
    ff = pOvRho * wf * area * mu
    abvE = u * u + v * v + w * w + (mu_lam * FHF_LAM + eddy * FHF_TURB) / mu * e
    un = u * nnx + v * nny + w * nnz
    dVn = dV[1] * nnx + dV[2] * nny + dV[3] * nnz
    tt = tau * ff
    am = lp1 * (dVn + un * dV[4])
    f[1] = f[1] + tt * (am * nnx + dV[1] + u * dV[4])
    f[2] = f[2] + tt * (am * nny + dV[2] + v * dV[4])
    f[3] = f[3] + tt * (am * nnz + dV[3] + w * dV[4])
    f[4] = f[4] + tt * (lp1 * un * dVn + u * dV[1] + v * dV[2] + w * dV[3] + (abvE + lp1 * un * un) * dV[4])
    sc = 0.5 * theta * ff
    nx, ny, nz = sc * nnx, sc * nny, sc * nnz
    d1, d2, d3, d4 = dV[1], dV[2], dV[3], dV[4]
    K11 = (lp2, u * lp2, v, w, abvE + u * u * lp1)
    K22 = (u, lp2, v * lp2, w, abvE + v * v * lp1)
    K33 = (u, v, lp2, w * lp2, abvE + w * w * lp1)
    z = np.zeros_like(d1)
    sx = [z, -(lp2 * d1 + K11[1] * d4) * nx - (lam * d2 + v * lam * d4) * ny - (lam * d3 + w * lam * d4) * nz,
          -(d2 + v * d4) * nx - (d1 + u * d4) * ny,
          -(d3 + w * d4) * nx - (d1 + u * d4) * nz,
          -(K11[1] * d1 + v * d2 + w * d3 + K11[4] * d4) * nx - (v * d1 + u * lam * d2 + u * v * lp1 * d4) * ny
          - (w * d1 + u * lam * d3 + u * w * lp1 * d4) * nz]
    sy = [z, -(d2 + v * d4) * nx - (d1 + u * d4) * ny,
          -(lam * d1 + u * lam * d4) * nx - (lp2 * d2 + K22[2] * d4) * ny - (lam * d3 + w * lam * d4) * nz,
          -(d3 + w * d4) * ny - (d2 + v * d4) * nz,
          -(v * lam * d1 + u * d2 + u * v * lp1 * d4) * nx - (u * d1 + K22[2] * d2 + w * d3 + K22[4] * d4) * ny
          - (w * d2 + v * lam * d3 + v * w * lp1 * d4) * nz]
    sz = [z, -(d3 + w * d4) * nx - (d1 + u * d4) * nz,
          -(d3 + w * d4) * ny - (d2 + v * d4) * nz,
          -(lam * d1 + u * lam * d4) * nx - (lam * d2 + v * lam * d4) * ny - (lp2 * d3 + K33[3] * d4) * nz,
          -(w * lam * d1 + u * d3 + u * w * lp1 * d4) * nx - (w * lam * d2 + v * d3 + v * w * lp1 * d4) * ny
          - (u * d1 + v * d2 + K33[3] * d3 + K33[4] * d4) * nz]
    return sx, sy, sz, eddy


def _face_expand(B, d: Disc, dd, g, q):
    """One TPR*F distribution of face data B[e, 5, slow, fast] into [e, 5, k, j, i].
    q = -1: normal flux; q = 0, 1, 2: symmetrizing flux of parametric direction r, s, t."""
    fast_q = 1 if dd == 0 else 0
    slow_q = 1 if dd == 2 else 2
    opS = d.dleg if q == slow_q else d.leg
    opF = d.dleg if q == fast_q else d.leg
    vec = d.dface[g] if q == dd else d.face[g]
    t = _ax(_ax(B, opS.T, 2), opF.T, 3)             # [e, 5, K(slow), K(fast)]
    if dd == 0:   # (k, j), normal i
        return t[:, :, :, :, None] * vec[None, None, None, None, :]
    if dd == 1:   # (k, i), normal j
        return t[:, :, :, None, :] * vec[None, None, None, :, None]
    return t[:, :, None, :, :] * vec[None, None, :, None, None]   # (j, i), normal k


def face_residual(U, d: Disc, compat=True):
    """Interior-face contributions (all faces periodic/interior)."""
    nE = U.shape[0]
    M2 = d.M * d.M
    tr = face_traces(U, d)
    R = np.zeros_like(U)
    own_min, nb_max = [], []
    for dd in range(3):
        L = d.nbr[:, 2 * dd]
        if np.any(L < 0):
            raise NotImplementedError("boundary faces are not restated")
        trR = [a.reshape(nE, 5, M2) for a in tr[2 * dd]]
        trL = [a[L].reshape(nE, 5, M2) for a in tr[2 * dd + 1]]
        fmR = d.fmet[:, 2 * dd]
        fmL = d.fmet[L, 2 * dd + 1]
        gxL, gyL, gzL = _cart_grad(trL[1], trL[2], trL[3], fmL, 4, compat)
        gxR, gyR, gzR = _cart_grad(trR[1], trR[2], trR[3], fmR, 4, compat)
        gx, gy, gz = 0.5 * (gxL + gxR), 0.5 * (gyL + gyR), 0.5 * (gzL + gzR)
        VL = [trL[0][:, n] for n in range(5)]
        VR = [trR[0][:, n] for n in range(5)]
        wf = (d.w[None, :] * d.w[:, None]).reshape(M2)   # w_fast * w_slow
        nx, ny, nz, area = fmL[:, 0], fmL[:, 1], fmL[:, 2], fmL[:, 3]
        if d.riemann == 1:
            f = ismail_roe(VL, VR, nx, ny, nz, wf * area)
        else:
            f = roe(VL, VR, nx, ny, nz, 0.5 * wf * area)
        lenScale = np.minimum(d.scal[:, dd], d.scal[L, dd])
        tau = d.tau_num / lenScale[:, None]
        len_les = 0.5 * (d.scal[:, 3] + d.scal[L, 3])[:, None]
        sx, sy, sz, _ = viscous_face(VL, VR, [gx[:, n] for n in range(5)],
                                     [gy[:, n] for n in range(5)], [gz[:, n] for n in range(5)],
                                     nx, ny, nz, wf, area, d.mu, tau, d.theta, f, d.sgs, len_les)
        flux = np.stack(f, axis=1)
        SX, SY, SZ = np.stack(sx, axis=1), np.stack(sy, axis=1), np.stack(sz, axis=1)

        def param(fm):
            if compat:
                m = fm[:, 4:13, [n if n < M2 else 0 for n in range(5)]][:, :, :, None]
            else:
                m = fm[:, 4:13, None, :]
            return [SX * m[:, 3 * q] + SY * m[:, 3 * q + 1] + SZ * m[:, 3 * q + 2] for q in range(3)]

        symL, symR = param(fmL), param(fmR)
        sh = (nE, 5, d.M, d.M)
        cR = _face_expand((-flux).reshape(sh), d, dd, 0, -1)
        cL = _face_expand(flux.reshape(sh), d, dd, 1, -1)
        for q in range(3):
            cR = cR + _face_expand(symR[q].reshape(sh), d, dd, 0, q)
            cL = cL + _face_expand(symL[q].reshape(sh), d, dd, 1, q)
        own_min.append(cR)
        toL = np.empty_like(cL)
        toL[L] = cL
        nb_max.append(toL)
    for c in own_min:
        R += c
    for c in nb_max:
        R += c
    return R


def _dvdu(U, d: Disc):
    """Preconditioner dV/dU * 8/vol at the element centre (src/CG_MassMatrix.cpp:313-361)."""
    V = np.einsum("l,evl->ve", d.center, U.reshape(U.shape[0], 5, -1))
    rho, u, v, w, p, eKin = entropy_to_prim(V)
    JacInv = 8.0 / d.scal[:, 5]
    pInv = 1.0 / p
    a1 = GM1 * rho * pInv * pInv
    a2 = eKin * a1
    D = np.empty((U.shape[0], 5, 5))
    D[:, 0, 0] = GAM / GM1 / rho + a2 * eKin
    D[:, 0, 1] = D[:, 1, 0] = -u * a2
    D[:, 0, 2] = D[:, 2, 0] = -v * a2
    D[:, 0, 3] = D[:, 3, 0] = -w * a2
    D[:, 0, 4] = D[:, 4, 0] = a2 - pInv
    D[:, 1, 1] = a1 * u * u + pInv
    D[:, 1, 2] = D[:, 2, 1] = a1 * u * v
    D[:, 1, 3] = D[:, 3, 1] = a1 * u * w
    D[:, 1, 4] = D[:, 4, 1] = -a1 * u
    D[:, 2, 2] = a1 * v * v + pInv
    D[:, 2, 3] = D[:, 3, 2] = a1 * v * w
    D[:, 2, 4] = D[:, 4, 2] = -a1 * v
    D[:, 3, 3] = a1 * w * w + pInv
    D[:, 3, 4] = D[:, 4, 3] = -a1 * w
    D[:, 4, 4] = a1
    return D * JacInv[:, None, None]


def mass_solve(Rraw, U, cg, d: Disc, max_iter=100):
    """Flexible PCG on the entropy-variable mass matrix, per element
    (src/CG_MassMatrix.cpp:250-504). Returns (solution, iterations per element)."""
    nE, K, M = U.shape[0], d.K, d.M
    r = Rraw.reshape(nE, 5, -1).copy()
    x = np.zeros_like(r)
    rInit = np.abs(r).max(axis=(1, 2))
    active = rInit * (8.0 / d.scal[:, 5]) > 1e-10
    D = _dvdu(U, d)
    z = np.einsum("eab,ebl->eal", D, r)
    p = z.copy()
    rho, u, v, w, pr, rE, eKin, JW = (cg[k] for k in ("rho", "u", "v", "w", "p", "rE", "eKin", "JW"))
    ru, rv, rw, rH = rho * u, rho * v, rho * w, rE + pr
    A = np.array([[rho, ru, rv, rw, rE], [ru, ru * u + pr, ru * v, ru * w, rH * u],
                  [rv, ru * v, rv * v + pr, rv * w, rH * v], [rw, ru * w, rv * w, rw * w + pr, rH * w],
                  [rE, rH * u, rH * v, rH * w, rE * rH / rho + pr * eKin]])   # [5, 5, e, P]
    iters = np.zeros(nE, dtype=int)
    todo = active.copy()
    for it in range(max_iter + 1):
        if not todo.any():
            break
        if it == max_iter:
            raise RuntimeError("CG did not converge in 100 iterations")
        dotrz = np.sum(r * z, axis=(1, 2))
        pI = _ax(_ax(_ax(p.reshape(nE, 5, K, K, K), d.leg, 2), d.leg, 3), d.leg, 4).reshape(nE, 5, -1)
        q = JW[:, None, :] * pI
        pI = np.einsum("abep,ebp->eap", A, q).reshape(nE, 5, M, M, M)
        Ap = vol_project(pI, d.leg, d.leg, d.leg).reshape(nE, 5, -1)
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha = np.where(todo, dotrz / np.sum(p * Ap, axis=(1, 2)), 0.0)
        x = x + alpha[:, None, None] * p
        r = r - alpha[:, None, None] * Ap
        iters += todo
        done = np.abs(r).max(axis=(1, 2)) < 1e-10 * rInit
        todo = todo & ~done
        z = np.einsum("eab,ebl->eal", D, r)
        with np.errstate(divide="ignore", invalid="ignore"):
            beta = np.where(todo, -alpha * np.sum(z * Ap, axis=(1, 2)) / dotrz, 0.0)
        p = np.where(todo[:, None, None], beta[:, None, None] * p + z, p)
    return x.reshape(U.shape), iters


def residual(U, d: Disc, compat=True):
    """Full residual: returns (raw residual, residual after the mass solve, CG iterations)."""
    Rv, cg = volume_residual(U, d, compat)
    Rraw = Rv + face_residual(U, d, compat)
    res, iters = mass_solve(Rraw, U, cg, d)
    return Rraw, res, iters


def time_step(U, d: Disc):
    """Global CFL time step (ElementClass::ComputeTimeStep, src/ElementClass.cpp:1522-1644)."""
    V = _ax(_ax(_ax(U, d.legdof, 2), d.legdof, 3), d.legdof, 4).reshape(U.shape[0], 5, -1)
    rho, u, v, w, p, _ = entropy_to_prim(V.transpose(1, 0, 2))
    rho, u, v, w, p = rho * d.rho_ref, u * d.u_ref, v * d.u_ref, w * d.u_ref, p * d.p_ref
    sc = d.scal
    li, lj, lk = 1.0 / sc[:, 0:1], 1.0 / sc[:, 1:2], 1.0 / sc[:, 2:3]
    muDim = d.mu * d.p_ref / d.u_ref
    radVisNu = max(max(1.0, 2.0 + LAM_OVER_MU), FHF_LAM) * (li * li + lj * lj + lk * lk)
    if d.sgs != SGS_NONE:
        eddy = _nodal_eddy_viscosity(U, d, rho, u, v, w, p)
        radVisTurb = max(max(1.0, 2.0 + LAM_OVER_MU), FHF_TURB) * (li * li + lj * lj + lk * lk)
        radVis = (1.0 / rho * (muDim * radVisNu + eddy * radVisTurb)).max(axis=1)
    else:
        radVis = (1.0 / rho * muDim * radVisNu).max(axis=1)
    a = np.sqrt(np.abs(GAM * p / rho))
    vI = u * sc[:, 6:7] + v * sc[:, 7:8] + w * sc[:, 8:9]
    vJ = u * sc[:, 9:10] + v * sc[:, 10:11] + w * sc[:, 11:12]
    vK = u * sc[:, 12:13] + v * sc[:, 13:14] + w * sc[:, 14:15]
    radInv = ((np.abs(vI) + a) * li + (np.abs(vJ) + a) * lj + (np.abs(vK) + a) * lk).max(axis=1)
    f1 = [2.0, 6.0, 12.0, 20.0, 28.0, 38.0, 50.0, 64.0, 80.0, 98.0]
    f2 = [6.0, 36.0, 150.0, 420.0, 980.0, 1975.0, 3575.0, 7000.0, 14000.0, 28000.0]
    dt = d.cfl * d.u_ref / (f1[d.n_poly] * radInv + f2[d.n_poly] * radVis)
    return float(dt.min())


def _nodal_eddy_viscosity(U, d: Disc, rho, u, v, w, p):
    """Eddy viscosity in the nodal DOFs from the dimensional primitive variables
    (ComputeVelocityGradientsNodalDOFs, entropy branch, src/ElementClass.cpp:1647-1795,
    then EddyViscosity with the element's LES length scale)."""
    nE = U.shape[0]
    _, dr, ds, dt = vol_interp(U, d.legdof, d.dlegdof)
    dr, ds, dt = (a.reshape(nE, 5, -1) for a in (dr, ds, dt))
    uRefInv = 1.0 / d.u_ref
    un, vn, wn = u * uRefInv, v * uRefInv, w * uRefInv
    V4Inv = -p * uRefInv * uRefInv / rho
    comp = []
    for c, vel in ((1, un), (2, vn), (3, wn)):
        comp.append([-V4Inv * (g[:, c] + vel * g[:, 4]) for g in (dr, ds, dt)])
    m = d.vmd
    G = [[d.u_ref * (comp[i][0] * m[:, 1 + j] + comp[i][1] * m[:, 4 + j] + comp[i][2] * m[:, 7 + j])
          for j in range(3)] for i in range(3)]
    return eddy_viscosity(d.sgs, d.scal[:, 3:4], rho, G)


LS_A = [0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0]
LS_B = [1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
        2277821191437.0 / 14882151754819.0]


def run(U, d: Disc, n_steps, scheme="ssprk3", compat=True):
    """n_steps time steps from U (the residual of U is evaluated first, as the
    reference main program does). Returns (state, dt history)."""
    U = U.copy()
    _, res, _ = residual(U, d, compat)
    hist = []
    for _ in range(n_steps):
        dt = time_step(U, d)
        hist.append(dt)
        if scheme == "ssprk3":
            U0 = U.copy()
            for a, b in ((1.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0)):
                U = (1.0 - a) * U + a * U0 - (b * dt) * res
                _, res, _ = residual(U, d, compat)
        else:
            dU = np.zeros_like(U)
            for a, b in zip(LS_A, LS_B):
                dU = a * dU - dt * res
                U = U + b * dU
                _, res, _ = residual(U, d, compat)
    return U, np.array(hist)


def from_discretization(disc, params) -> Disc:
    """Builds the restatement's inputs from the library's set-up arrays
    (vcp3d_open_b200.solver.Discretization and capi.Params)."""
    K, M = params.n_poly + 1, params.n_int_1d
    return Disc(K=K, M=M, leg=disc.leg_int, dleg=disc.dleg_int, face=disc.leg_face,
                dface=disc.dleg_face, w=disc.w_int, legdof=disc.leg_dofs,
                center=disc.basis_center, vol=disc.vol_metric, fmet=disc.face_metric,
                scal=disc.elem_scalars, nbr=disc.neighbors.astype(np.int64), mu=params.mu,
                tau_num=float((params.n_poly + 1) ** 2) * params.rel_penalty,
                theta=params.theta_sym, riemann=params.riemann, p_ref=params.p_ref,
                u_ref=params.u_ref, rho_ref=params.rho_ref, cfl=params.cfl,
                n_poly=params.n_poly, sgs=params.sgs_model, dlegdof=disc.dleg_dofs,
                vmd=disc.vol_metric_dofs,
                fbody=(tuple(1.0 / params.p_ref * f for f in params.body_force)
                       if any(params.body_force) else None))
