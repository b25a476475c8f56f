"""CA-GMRES(s, t) oracle in numpy / scipy-LAPACK.

TEST INFRASTRUCTURE ONLY (see oracle/oracle.py).  Restates KSP_pCAGMRES
(src/pcagmres.f90:1557-2518) of the reference with its helpers:

* basis: s preconditioned products per block, monomial or Newton
  (calc_NewtonBasisVec, pcagmres.f90:1480-1552; calc_NewtonBasis, :586-611);
* block classical Gram-Schmidt of the new block against the previous Q
  (calc_gemm_dot / CAGMRES_GEMM, pcagmres.f90:2109-2141, 1052-1080);
* R-only QR of the block (QRDecomposition_, src/QRDecomposition.f90:1331-1552):
  TSQR (Householder R), Cholesky QR or Cholesky QR2, then Q = V R^-1 (calcQ_VRinv_);
* the Hessenberg matrix rebuilt from R, the change-of-basis matrix B and R^-1
  (calc_HessenbergMatrix, pcagmres.f90:879-1052), Givens rotations with the residual
  history (GivensRotations, :190-242) and the update x += M^-1 Q y (update_xVec);
* Ritz values of the leading Hessenberg block (DHSEQR in the reference; LAPACK's
  DGEEV here gives the same eigenvalues) ordered by modified Leja ordering
  (src/LejaOrdering.f90:18-322), used as Newton shifts from the second block on.

One deliberate simplification, identical in exact arithmetic: Q is formed for every
block, including the last block of a cycle where the reference keeps R only and corrects
the update with R^-1 (update_xVec_cagmres, pcagmres.f90:1338-1478).

SpMV and the preconditioner are the C oracle's (oracle/parcel_oracle.cpp).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
from scipy.linalg import lapack

import oracle as _orc

MONOMIAL, NEWTON = 0, 1
QR_MGS, QR_CGS, QR_TSQR, QR_CHOL, QR_CHOL2 = 1, 2, 3, 4, 5


def _chol_upper(G):
    R, info = lapack.dpotrf(G, lower=0, clean=1)
    if info != 0:
        raise np.linalg.LinAlgError(f"dpotrf info {info}")
    return np.triu(R)


def _trinv_upper(R):
    Ri, info = lapack.dtrtri(np.array(R, order="F"), lower=0)
    if info != 0:
        raise np.linalg.LinAlgError(f"dtrtri info {info}")
    return np.triu(Ri)


def qr_r_only(V, flag):
    """R factor of the n x c panel V (columns are V[:, j])."""
    if V.shape[1] == 1 or flag in (QR_MGS, QR_CGS):
        flag = QR_CHOL2
    if flag == QR_TSQR and V.shape[0] > V.shape[1] and V.shape[0] > 64:
        R = np.linalg.qr(V, mode="r")
        # TSQR_Ronly_ (QRDecomposition.f90:887-1002) flips rows to a positive diagonal
        sg = np.where(np.diag(R) < 0.0, -1.0, 1.0)
        return R * sg[:, None]
    if flag == QR_CHOL:
        return _chol_upper(V.T @ V)
    R1 = _chol_upper(V.T @ V)
    Q1 = V @ _trinv_upper(R1)
    R2 = _chol_upper(Q1.T @ Q1)
    return R2 @ R1


def newton_basis(s, B1, er, ei):
    """calc_NewtonBasis (pcagmres.f90:586-611), B1 is (s+1) x s, updated in place."""
    i = 1
    while i <= s:
        if i == s:
            B1[i - 1, i - 1] = er[i - 1]
        elif abs(ei[i - 1]) == 0.0:
            B1[i - 1, i - 1] = er[i - 1]
        else:
            B1[i - 1, i - 1] = er[i - 1]
            B1[i, i] = er[i - 1]
            B1[i - 1, i] = -ei[i - 1] * ei[i - 1]
            i += 1
        i += 1


def leja(er, ei):
    """modified_leja_ordering (src/LejaOrdering.f90:100-322) on the first len(er) values."""
    n = len(er)
    er = list(er)
    ei = list(ei)
    for i in range(1, n):             # stable insertion sort, descending modulus
        j = i
        while j > 0 and np.sqrt(er[j - 1] ** 2 + ei[j - 1] ** 2) < np.sqrt(er[j] ** 2 + ei[j] ** 2):
            er[j], er[j - 1] = er[j - 1], er[j]
            ei[j], ei[j - 1] = ei[j - 1], ei[j]
            j -= 1
    ptmp = [1.0] * n
    mu = [1.0] * n
    theta_r = [0.0] * n
    theta_i = [0.0] * n
    outlist = [0] * n
    C = 1.0
    if ei[0] > 0.0:
        theta_r[0], theta_i[0] = er[0], ei[0]
        theta_r[1], theta_i[1] = er[1], ei[1]
        outlist[0], outlist[1] = 0, 1
        L = 2
    else:
        theta_r[0], theta_i[0] = er[0], 0.0
        outlist[0] = 0
        L = 1

    def mprod(tr_, ti_, L_):
        out = 1.0
        vals = []
        for j in range(0, L_ - 1):
            a = tr_ - theta_r[j]
            b = ti_ - theta_i[j]
            vals.append(np.sqrt(a * a + b * b) ** mu[outlist[j]])
        for v in vals:
            out = out * v
        return out

    while L < n:
        Cold = C
        for j in range(0, L - 1):
            a = theta_r[L - 1] - theta_r[j]
            b = theta_i[L - 1] - theta_i[j]
            ptmp[j + 1] = np.sqrt(a * a + b * b) ** (mu[outlist[j]] / L)
        C = 1.0
        for j in range(n):
            C = C * ptmp[j]
        f = C / Cold
        for j in range(n):
            er[j] = er[j] / f
            ei[j] = ei[j] / f
            theta_r[j] = theta_r[j] / f
            theta_i[j] = theta_i[j] / f
        tmp = [0.0] * n
        for j in range(n):
            if j not in outlist[:L]:
                tmp[j] = mprod(er[j], ei[j], L)
        mx = abs(tmp[0])
        k = 0
        for j in range(1, n):
            if abs(tmp[j]) > mx:
                mx = abs(tmp[j])
                k = j
        if abs(ei[k]) > 0.0:
            if ei[k] < 0.0:
                theta_r[L], theta_i[L] = er[k - 1], ei[k - 1]
                theta_r[L + 1], theta_i[L + 1] = er[k], ei[k]
                outlist[L], outlist[L + 1] = k - 1, k
            else:
                theta_r[L], theta_i[L] = er[k], ei[k]
                theta_r[L + 1], theta_i[L + 1] = er[k + 1], ei[k + 1]
                outlist[L], outlist[L + 1] = k, k + 1
            L += 2
        else:
            theta_r[L], theta_i[L] = er[k], 0.0
            outlist[L] = k
            L += 1
    return (np.array([t * C for t in theta_r]), np.array([t * C for t in theta_i]))


def givens(Hg, i, co, si, ze):
    """GivensRotations (pcagmres.f90:190-242) on column i (1-based); Hg (m+1) x m."""
    col = Hg[:, i - 1]
    for k in range(1, i):
        t1 = col[k - 1] * co[k - 1] - col[k] * si[k - 1]
        t2 = col[k - 1] * si[k - 1] + col[k] * co[k - 1]
        col[k - 1], col[k] = t1, t2
    t = col[i] / 1.0 - 300.0 if col[i - 1] == 0.0 else col[i] / col[i - 1]
    co[i - 1] = 1.0 / np.sqrt(1.0 + t * t)
    si[i - 1] = -co[i - 1] * t
    t1 = co[i - 1] * ze[i - 1] - si[i - 1] * ze[i]
    t2 = si[i - 1] * ze[i - 1] + co[i - 1] * ze[i]
    ze[i - 1], ze[i] = t1, t2
    col[i - 1] = co[i - 1] * col[i - 1] - si[i - 1] * col[i]
    col[i] = 0.0


def hessenberg_update(s, t, k, B1, H, R1, Rk, BRup, hk_pre):
    """calc_HessenbergMatrix (pcagmres.f90:879-1052).  Returns the new hk_pre."""
    if k == 1:
        Rinv = _trinv_upper(R1[:s, :s])
        RB = R1 @ B1
        Hes = RB @ Rinv
        H[: s + 1, :s] = Hes
        return Hes[s, s - 1]
    s1 = s * (k - 1)
    Rt0 = np.zeros((s + 1, s + 1))
    Rt0[0, :] = BRup[s1, :]
    Rt0[1:, 1:] = Rk
    BRu = BRup[:s1, :]
    BR = BRup[:s1, :s]
    Rinv = _trinv_upper(Rt0[:s, :s])
    BlockHes = H[:s1, :s1]
    X = -(BlockHes @ BR) + (BRu @ B1)
    H[:s1, s1:s1 + s] = X @ Rinv
    bk = B1[s, s - 1]
    rho_tilde = Rt0[s - 1, s - 1]
    rho = Rt0[s, s]
    hk = rho / rho_tilde * bk
    H[s * k, s * k - 1] = hk
    Hss = (Rt0[:s, :s] @ B1[:s, :s]) @ Rinv
    for i in range(s):
        Hss[i, s - 1] = Hss[i, s - 1] + bk / rho_tilde * Rt0[i, s]
    e1 = np.zeros((s, s))
    e1[0, :] = BR[s1 - 1, :] * hk_pre
    Hss = Hss - e1 @ Rinv
    H[s1:s1 + s, s1:s1 + s] = Hss
    return hk


def pcagmres(A, b, x0=None, *, precon=None, s=4, t=1, basis=MONOMIAL, qrflag=QR_CHOL, itrmax=1000,
             rtolmax=1e-8, abstolmax=0.0, **pre):
    """Returns (x, reshistory[:niter], niter, iret)."""
    M = A if isinstance(A, _orc.Matrix) else _orc.Matrix(A)
    n = M.n
    P = precon if precon is not None else (_orc.Precon(M, **pre) if pre.get("ipreflag", 0) else (lambda v: v.copy()))
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    st = s * t
    hist = np.zeros(itrmax + st + 2)
    B1 = np.zeros((s + 1, s))
    for i in range(s):
        B1[i + 1, i] = 1.0
    er = np.zeros(st)
    ei = np.zeros(st)
    bnorm = np.sqrt(np.dot(b, b))
    iflag_exit = -1
    iflag_basis = -1
    itr0 = 0
    itr = 1
    while itr <= itrmax:
        itr0 = itr
        co = np.zeros(st + 1)
        si = np.zeros(st + 1)
        ze = np.zeros(st + 1)
        H = np.zeros((st + 1, st))
        Hg = np.zeros((st + 1, st))
        hk_pre = 0.0
        r = b - _orc.spmv(M, x)
        rnorm = np.sqrt(np.dot(r, r))
        if rnorm < abstolmax or rnorm / bnorm < rtolmax:
            break
        if itr == 1:
            hist[0] = rnorm / bnorm
        ze[0] = -rnorm
        V = np.zeros((n, s + 1))
        Q = np.zeros((n, st + 1))
        V[:, 0] = (-1.0 / rnorm) * r
        mm = 0
        R1 = Rk = BRup = None
        for k in range(1, t + 1):
            if basis == NEWTON and iflag_basis == 1:
                newton_basis(s, B1, er, ei)
            for i in range(1, s + 1):
                pv = P(V[:, i - 1])
                w = _orc.spmv(M, pv)
                if iflag_basis == 1 and basis == NEWTON:
                    if i != 1:
                        # The reference adds +B1(i-1,i) V_{i-2} (calc_NewtonBasisVec), while its
                        # Hessenberg (calc_HessenbergMatrix) takes the basis relation with
                        # B1(i-1,i) as stored; the two agree only with the opposite sign here,
                        # which is the real form of a complex shift pair.  The oracle uses the
                        # consistent sign (identical when every shift is real).
                        alpha = -B1[i - 1, i - 1]
                        beta = -B1[i - 2, i - 1]
                        w = alpha * V[:, i - 1] + beta * V[:, i - 2] + 1.0 * w
                    else:
                        alpha = -B1[i - 1, i - 1]
                        w = alpha * V[:, i - 1] + 1.0 * w
                V[:, i] = w
            if k == 1:
                R1 = qr_r_only(V, qrflag)
                Q[:, : s + 1] = V @ _trinv_upper(R1)
            else:
                s1 = s * (k - 1) + 1
                BRup = Q[:, :s1].T @ V
                for c in range(1, s + 1):
                    acc = V[:, c].copy()
                    for j in range(s1):
                        acc = acc - Q[:, j] * BRup[j, c]
                    V[:, c] = acc
                Rk = qr_r_only(V[:, 1:], qrflag)
                Q[:, s1:s1 + s] = V[:, 1:] @ _trinv_upper(Rk)
            hk_pre = hessenberg_update(s, t, k, B1, H, R1, Rk, BRup, hk_pre)
            if k != t:
                V = np.zeros((n, s + 1))
                V[:, 0] = Q[:, s * k]
            Hg[:, s * (k - 1):s * k] = H[:, s * (k - 1):s * k]
            for i in range(s * (k - 1) + 1, s * k + 1):
                mm = i
                givens(Hg, i, co, si, ze)
                rnorm = abs(ze[i])
                itr0 = i + (itr - 1) + 1
                hist[itr0 - 1] = rnorm / bnorm
                if rnorm / bnorm < rtolmax or i + (itr - 1) + 1 == itrmax:
                    iflag_exit = 1
                    break
            if iflag_exit == 1:
                break
            if basis == NEWTON:
                iflag_basis = 1
                ev = sla.eigvals(H[: s * k, : s * k])
                wr, wi = leja(ev.real, ev.imag)
                er[: s * k] = wr
                ei[: s * k] = wi
        # update_xVec: y = Hg^-1 ze over mm columns, x += M^-1 Q y
        y = np.zeros(mm)
        for i in range(mm, 0, -1):
            v = ze[i - 1]
            for j in range(mm, i, -1):
                v = v - Hg[i - 1, j - 1] * y[j - 1]
            d = Hg[i - 1, i - 1]
            y[i - 1] = v / 1.0e-300 if d == 0.0 else v / d
        v0 = Q[:, :mm] @ y
        x = P(v0) + x
        if iflag_exit == 1:
            break
        itr += st
    niter = min(itrmax, itr0)
    iret = 1 if itrmax <= itr else 0
    return x, hist[:niter].copy(), niter, iret
