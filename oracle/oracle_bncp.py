"""TEST INFRASTRUCTURE (the oracle), not the product: only tests/, smoke() and bench.py's CPU legs
may use it, as the checker.

numpy restatement of the batched exact-cone NCP and its fixed-branch sensitivity:
  - pgs: projected Gauss-Seidel lambda_c <- proj_K(lambda_c - rho_c (u_c + Gamma(u_c))),
    rho_c = 1/lambda_max(G_cc) (the sweep of src/motion_engine/ncp/ncp_gpu.py:485-568 on the
    Delassus operator), stopping on the natural residual (ncp_ref.natural_residual,
    src/motion_engine/ncp/ncp_ref.py:224-234);
  - classify: open / stick / slip (ncp_ref.classify, :251-274);
  - active_system: the fixed-branch residual Jacobian and parameter maps (ncp_ref._active_system,
    :786-842);
  - sensitivity: -A^-1 [Bmu Bb] (ncp_ref.sensitivity, :907-959), NaN for a singular branch
    (smallest LU pivot below 1e-12 max|A|) or a branch boundary;
  - vjp: (A^-T g) mapped by -Bb^T and -Bmu^T.
"""
import numpy as np


def proj(z, mu):
    zn, zt = z[0], np.hypot(z[1], z[2])
    if zt <= mu * zn:
        return z.copy()
    if mu * zt <= -zn:
        return np.zeros(3)
    s = (zn + mu * zt) / (1.0 + mu * mu)
    f = mu * s / zt
    return np.array([s, f * z[1], f * z[2]])


def _rho(G, nc):
    return np.array([1.0 / np.linalg.eigvalsh(G[3 * c:3 * c + 3, 3 * c:3 * c + 3]).max() for c in range(nc)])


def residual(lam, G, b, mu, rho=None):
    nc = len(mu)
    rho = _rho(G, nc) if rho is None else rho
    u = G @ lam + b
    r = 0.0
    for c in range(nc):
        sl = slice(3 * c, 3 * c + 3)
        s = u[sl].copy()
        s[0] += mu[c] * np.hypot(u[3 * c + 1], u[3 * c + 2])
        r = max(r, float(np.abs(lam[sl] - proj(lam[sl] - rho[c] * s, mu[c])).max()))
    return r


def pgs(G, b, mu, iters=5000, tol=1e-14, check=10, warm=None):
    G, b, mu = (np.asarray(x, np.float64) for x in (G, b, mu))
    nc = len(mu)
    lam = np.zeros(3 * nc) if warm is None else np.array(warm, np.float64)
    rho = _rho(G, nc)
    for it in range(iters):
        if check > 0 and it % check == 0 and residual(lam, G, b, mu, rho) < tol:
            return lam, it
        for c in range(nc):
            sl = slice(3 * c, 3 * c + 3)
            u = b[sl] + G[sl] @ lam
            s = u.copy()
            s[0] += mu[c] * np.hypot(u[1], u[2])
            lam[sl] = proj(lam[sl] - rho[c] * s, mu[c])
    return lam, iters


def classify(lam, mu, tol_lam=1e-10, tol_rel=1e-6):
    nc = len(mu)
    L = np.asarray(lam).reshape(nc, 3)
    scale = max(float(np.abs(L).max()) if nc else 0.0, 1e-30)
    out = np.zeros(nc, np.int32)
    for c in range(nc):
        ln, lt = L[c, 0], np.hypot(L[c, 1], L[c, 2])
        if ln <= tol_lam + tol_rel * scale:
            out[c] = 0
        elif lt >= mu[c] * ln * (1.0 - tol_rel) - tol_lam:
            out[c] = 2
        else:
            out[c] = 1
    return out


def active_system(lam, G, b, mu, labels):
    n = len(b)
    nc = n // 3
    u = G @ lam + b
    A, Bmu, Bb = np.zeros((n, n)), np.zeros((n, nc)), np.zeros((n, n))
    boundary = False
    for c in range(nc):
        i = 3 * c
        if labels[c] == 0:
            A[i:i + 3, i:i + 3] = np.eye(3)
            boundary |= abs(u[i]) < 1e-9
        elif labels[c] == 1:
            A[i:i + 3] = G[i:i + 3]
            Bb[i:i + 3, i:i + 3] = np.eye(3)
        else:
            A[i] = G[i]
            Bb[i, i] = 1.0
            s = u[i + 1:i + 3]
            ns = float(np.linalg.norm(s))
            if ns < 1e-14:
                boundary, ns = True, 1e-14
            sh = s / ns
            P = (np.eye(2) - np.outer(sh, sh)) / ns
            A[i + 1:i + 3] = mu[c] * lam[i] * (P @ G[i + 1:i + 3])
            A[i + 1:i + 3, i] += mu[c] * sh
            A[i + 1, i + 1] += 1.0
            A[i + 2, i + 2] += 1.0
            Bb[i + 1:i + 3, i + 1:i + 3] = mu[c] * lam[i] * P
            Bmu[i + 1:i + 3, c] = lam[i] * sh
        ln, lt = lam[i], np.hypot(lam[i + 1], lam[i + 2])
        sc = max(abs(ln), 1e-12)
        boundary |= labels[c] == 1 and abs(lt - mu[c] * ln) < 1e-7 * mu[c] * sc
        boundary |= labels[c] != 0 and ln < 1e-9
    return A, Bmu, Bb, bool(boundary)


def _singular(A):
    """LU with partial pivoting: a pivot below 1e-12 max|A| marks the branch singular."""
    M = A.copy()
    n = len(M)
    amax = np.abs(A).max() if n else 0.0
    for k in range(n):
        p = k + int(np.argmax(np.abs(M[k:, k])))
        if not abs(M[p, k]) > 1e-12 * amax:
            return True
        M[[k, p]] = M[[p, k]]
        M[k + 1:, k] /= M[k, k]
        M[k + 1:, k + 1:] -= np.outer(M[k + 1:, k], M[k, k + 1:])
    return False


def sensitivity(lam, G, b, mu):
    """(dlam/dmu, dlam/db, labels, status): status bit 1 singular, bit 2 boundary."""
    labels = classify(lam, mu)
    A, Bmu, Bb, bnd = active_system(lam, G, b, mu, labels)
    status = (1 if _singular(A) else 0) | (2 if bnd else 0)
    n, nc = len(b), len(mu)
    if status:
        return np.full((n, nc), np.nan), np.full((n, n), np.nan), labels, status
    X = -np.linalg.solve(A, np.hstack([Bmu, Bb]))
    return X[:, :nc], X[:, nc:], labels, status


def vjp(lam, G, b, mu, glam):
    dmu, db, _, _ = sensitivity(lam, G, b, mu)
    return db.T @ glam, dmu.T @ glam
