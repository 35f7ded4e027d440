"""Oracle (test infrastructure): qd3Dsolver's LOBPCG wrappers restated on the CPU.

The iteration itself is the third-party `scipy.sparse.linalg.lobpcg` (scipy 1.18.1 in this
image; the reference pins no version), called exactly the way the reference calls it
(eigensolvers.py:247-248, 352-353): largest=False, retResidualNormsHistory=True, warnings
suppressed. Everything around that call restates eigensolvers.py line for line in meaning:

  residual_norms     eigensolvers.py:76-87
  rayleigh_quotients eigensolvers.py:90-101
  certify            eigensolvers.py:104-114
  hermiticity_error  eigensolvers.py:117-135
  solve_lowest       eigensolvers.py:200-268 (block = k + max(2, k//2), seeded X0 padding)
  folded_operator    eigensolvers.py:301-310
  solve_interior     eigensolvers.py:313-372 (X0 = rng.standard_normal + 1j * second draw)
  solve_lowest_hole  eigensolvers.py:375-386
"""
import time
import warnings

import numpy as np
import scipy.sparse.linalg as spla


def residual_norms(A, E, V):
    V = np.asarray(V)
    Vn = V / np.linalg.norm(V, axis=0)
    return np.linalg.norm(A @ Vn - Vn * np.asarray(E)[None, :], axis=0)


def rayleigh_quotients(A, V):
    V = np.asarray(V)
    AV = A @ V
    return (np.einsum('ij,ij->j', V.conj(), AV).real
            / np.einsum('ij,ij->j', V.conj(), V).real)


def certify(A, E, V, tol=1e-6):
    res = residual_norms(A, E, V)
    rq = rayleigh_quotients(A, V)
    return res, rq, bool(np.all(res < tol))


def hermiticity_error(A, n_probe=8, seed=0):
    rng = np.random.default_rng(seed)
    n = A.shape[0]
    worst = 0.0
    for _ in range(n_probe):
        x = rng.standard_normal(n)
        y = rng.standard_normal(n)
        if np.iscomplexobj(A) or getattr(A, 'dtype', None) == np.complex128:
            x = x + 1j * rng.standard_normal(n)
            y = y + 1j * rng.standard_normal(n)
        x /= np.linalg.norm(x)
        y /= np.linalg.norm(y)
        worst = max(worst, abs(np.vdot(y, A @ x) - np.vdot(A @ y, x)))
    return worst


def start_block(n, block, seed, complex_=True):
    """The seeded starting block of eigensolvers.py:344-347 (and :230-234)."""
    rng = np.random.default_rng(seed)
    X0 = rng.standard_normal((n, block))
    if complex_:
        X0 = X0 + 1j * rng.standard_normal((n, block))
    return X0


def folded_operator(A, sigma):
    n = A.shape[0]

    def apply(x):
        y = A @ x - sigma * x
        return A @ y - sigma * y

    return spla.LinearOperator((n, n), matvec=apply, matmat=apply, dtype=A.dtype)


def solve_interior(A, k=4, sigma=0.0, M=None, tol=1e-8, maxiter=3000, extra=None, seed=0,
                   X0=None):
    """Folded-spectrum LOBPCG, returns (E, V, info) like eigensolvers.solve_interior."""
    F = folded_operator(A, sigma)
    n = A.shape[0]
    if extra is None:
        extra = max(2, k // 2)
    block = min(k + extra, n)
    if X0 is None:
        X0 = start_block(n, block, seed, np.iscomplexobj(A) or A.dtype == np.complex128)
    t0 = time.time()
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        mu, V, hist = spla.lobpcg(F, X0, M=M, largest=False, tol=tol, maxiter=maxiter,
                                  retResidualNormsHistory=True, verbosityLevel=0)
    dt = time.time() - t0
    E = rayleigh_quotients(A, V)
    order = np.argsort(np.abs(E - sigma))
    E, V = E[order][:k], V[:, order][:, :k]
    order2 = np.argsort(E)
    E, V = E[order2], V[:, order2]
    res = residual_norms(A, E, V)
    return E, V, dict(time=dt, iterations=len(hist), residuals=res,
                      converged=bool(res.max() < 1e-6), mu=mu)


def solve_lowest(A, k=4, M=None, X0=None, tol=1e-8, maxiter=2000, extra=None, seed=0):
    n = A.shape[0]
    if extra is None:
        extra = max(2, k // 2)
    block = min(k + extra, n)
    cplx = np.iscomplexobj(A) or A.dtype == np.complex128
    if X0 is None:
        X0 = start_block(n, block, seed, cplx)
    elif X0.shape[1] < block:
        rng = np.random.default_rng(seed)
        pad = rng.standard_normal((n, block - X0.shape[1]))
        if cplx:
            pad = pad + 1j * rng.standard_normal((n, block - X0.shape[1]))
        X0 = np.hstack([X0, pad])
    t0 = time.time()
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        E, V, hist = spla.lobpcg(A, X0, M=M, largest=False, tol=tol, maxiter=maxiter,
                                 retResidualNormsHistory=True, verbosityLevel=0)
    dt = time.time() - t0
    order = np.argsort(E)
    E, V = E[order], V[:, order]
    res_all = residual_norms(A, E, V)
    gap = (E[k] - E[k - 1]) if len(E) > k else np.nan
    return E[:k], V[:, :k], dict(time=dt, iterations=len(hist), residuals=res_all[:k],
                                 residuals_all=res_all, block=block, gap_to_next=gap,
                                 converged=bool(res_all[:k].max() < 1e-6))
