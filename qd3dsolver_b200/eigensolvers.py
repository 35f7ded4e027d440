"""Drop-in for qd3Dsolver's `eigensolvers` on the B200: LOBPCG with every block op on the GPU.

Same signatures, defaults and return conventions as the reference (eigensolvers.py):
  solve_interior(A, k=4, sigma=0.0, M=None, tol=1e-8, maxiter=3000, extra=None, seed=0,
                 verbose=True, certify_tol=1e-6)                       eigensolvers.py:313-372
  solve_lowest(A, k=4, M=None, X0=None, tol=1e-8, maxiter=2000, extra=None, seed=0,
               verbose=True, certify_tol=1e-6)                          eigensolvers.py:200-268
  solve_lowest_hole(A, k=4, **kw)                                       eigensolvers.py:375-386
  residual_norms, rayleigh_quotients, certify, hermiticity_error        eigensolvers.py:76-135
  folded_operator                                                       eigensolvers.py:301-310

`A` is the operator returned by `qd3dsolver_b200.kp_pryor.confined_hamiltonian`. The starting
block is drawn on the host with NumPy exactly as the reference draws it, so a GPU solve and the
reference's SciPy solve start from the same vectors. E is float64 ascending, V a complex128
NumPy array (n, k) with orthonormal columns, info carries time, iterations, residuals and
converged, plus `status` (converged / maxiter / cholesky_breakdown / eigh_breakdown /
nonfinite) and the folded Ritz values `mu`.
"""
import ctypes
import time

import numpy as np
import scipy.sparse.linalg as spla

from . import _lib
from ._lib import check, lib
from .kp_pryor import KPOperator


def _torch():
    import torch
    return torch


def _require_op(A):
    if not isinstance(A, KPOperator):
        raise TypeError("A must be the device operator from "
                        "qd3dsolver_b200.kp_pryor.confined_hamiltonian")
    return A


def start_block(n, block, seed, complex_=True):
    """X0 exactly as eigensolvers.py:344-347 draws it (same generator, same order)."""
    rng = np.random.default_rng(seed)
    X0 = rng.standard_normal((n, block))
    if complex_:
        X0 = X0 + 1j * rng.standard_normal((n, block))
    return X0


def _to_device(X):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(X, dtype=np.complex128)).cuda()


def _device_residuals(A, Vd, E=None):
    """(Rayleigh quotients, residual norms) of H for the columns of the device block Vd."""
    torch = _torch()
    k = Vd.shape[1]
    need = int(lib().qdkp_residuals_workspace_size(A.handle, k))
    ws = torch.empty(need, dtype=torch.uint8, device=Vd.device)
    rq = np.empty(k)
    res = np.empty(k)
    Ein = None if E is None else np.ascontiguousarray(E, dtype=np.float64)
    stream = torch.cuda.current_stream(Vd.device).cuda_stream
    check(lib().qdkp_residuals(A.handle, Vd.data_ptr(), Vd.stride(0), k,
                               Ein.ctypes.data if Ein is not None else None,
                               rq.ctypes.data, res.ctypes.data, ws.data_ptr(), ws.numel(),
                               stream), 'qdkp_residuals')
    return rq, res


def lobpcg_device(A, X0, folded, sigma=0.0, tol=None, maxiter=20, restart_control=20,
                  verbosity=0, time_hx=False):
    """scipy.sparse.linalg.lobpcg(A or (A - sigma)^2, X0, largest=False) on the GPU.

    Returns (lambda, V_device, residual_history, info_dict)."""
    torch = _torch()
    A = _require_op(A)
    X0d = X0 if hasattr(X0, 'data_ptr') else _to_device(X0)
    n, block = X0d.shape
    if n < 5 * block:
        return _dense_device(A, X0d, folded, sigma)
    prm = _lib.LobpcgParams(block=block, folded=int(bool(folded)), sigma=float(sigma),
                            tol=float(tol) if tol else 0.0, maxiter=int(maxiter),
                            restart_control=int(restart_control), precision=_lib.C128,
                            verbosity=int(verbosity), time_hx=int(bool(time_hx)))
    need = int(lib().qdkp_lobpcg_workspace_size(A.handle, ctypes.byref(prm)))
    if need == 0:
        raise ValueError(f"block size {block} is outside the supported range [1, 24]")
    ws = torch.empty(need, dtype=torch.uint8, device=X0d.device)
    V = torch.empty((n, block), dtype=torch.complex128, device=X0d.device)
    lam = np.empty(block)
    hist = np.zeros((maxiter + 3, block))
    info = _lib.LobpcgInfo()
    stream = torch.cuda.current_stream(X0d.device).cuda_stream
    check(lib().qdkp_lobpcg_solve(A.handle, ctypes.byref(prm), X0d.data_ptr(), lam.ctypes.data,
                                  V.data_ptr(), hist.ctypes.data, ctypes.byref(info),
                                  ws.data_ptr(), ws.numel(), stream), 'qdkp_lobpcg_solve')
    rows = info.iterations
    return lam, V, hist[:rows], dict(iterations=rows, best_iteration=info.best_iteration,
                                     status=_lib.LOBPCG_STATUS.get(info.status, 'unknown'),
                                     explicit_gram=bool(info.explicit_gram),
                                     hx_applications=int(info.hx_applications),
                                     hx_launches=int(info.hx_launches),
                                     hx_seconds=float(info.hx_seconds),
                                     hx_bytes=float(info.hx_bytes),
                                     solver_seconds=info.seconds)


def _dense_device(A, X0d, folded, sigma):
    """scipy's lobpcg on a problem smaller than five block widths: it warns and solves the dense
    eigenproblem instead (lobpcg.py:455-489). Here the dense A (or (A - sigma)^2) is formed on the
    GPU by applying the device operator to the identity, and its lowest `block` pairs come from
    the device's dense Hermitian solver; no iterations, an empty history."""
    import warnings
    torch = _torch()
    n, block = X0d.shape
    warnings.warn(f"The problem size {n} minus the constraints size 0 is too small relative to "
                  f"the block size {block}. Using a dense eigensolver instead of LOBPCG "
                  f"iterations. No output of the history of the iterations.", UserWarning,
                  stacklevel=3)
    eye = torch.eye(n, dtype=torch.complex128, device=X0d.device)
    D = torch.empty((n, n), dtype=torch.complex128, device=X0d.device)
    mode = _lib.APPLY_FOLDED if folded else _lib.APPLY_PLAIN
    for c0 in range(0, n, 24):
        c1 = min(n, c0 + 24)
        D[:, c0:c1] = A.apply(eye[:, c0:c1].contiguous(), sigma=sigma if folded else 0.0,
                              mode=mode)
    D = 0.5 * (D + D.conj().T)
    w, Vf = torch.linalg.eigh(D)
    lam = w[:block].cpu().numpy()
    V = Vf[:, :block].contiguous()
    return lam, V, np.zeros((0, block)), dict(iterations=0, best_iteration=0, status='converged',
                                              explicit_gram=False, hx_applications=n,
                                              hx_launches=(n + 23) // 24, hx_seconds=0.0,
                                              hx_bytes=0.0, solver_seconds=0.0, dense=True)


# ------------------------------------------------------------------------------------------
# Verification layer (eigensolvers.py:76-135)
# ------------------------------------------------------------------------------------------

def residual_norms(A, E, V):
    """||A v_i - E_i v_i|| on normalised columns (eV)."""
    if isinstance(A, KPOperator):
        Vd = V if hasattr(V, 'data_ptr') else _to_device(V)
        return _device_residuals(A, Vd, np.asarray(E, dtype=float))[1]
    V = np.asarray(V)
    Vn = V / np.linalg.norm(V, axis=0)
    return np.linalg.norm(A @ Vn - Vn * np.asarray(E)[None, :], axis=0)


def rayleigh_quotients(A, V):
    if isinstance(A, KPOperator):
        Vd = V if hasattr(V, 'data_ptr') else _to_device(V)
        return _device_residuals(A, Vd)[0]
    V = np.asarray(V)
    AV = A @ V
    return (np.einsum('ij,ij->j', V.conj(), AV).real / np.einsum('ij,ij->j', V.conj(), V).real)


def certify(A, E, V, tol=1e-6, label='', verbose=True):
    res = residual_norms(A, E, V)
    rq = rayleigh_quotients(A, V)
    drift = np.abs(rq - np.asarray(E))
    ok = bool(np.all(res < tol))
    if verbose:
        tag = f"[{label}] " if label else ""
        print(f"{tag}max residual {res.max():.3e} eV, max |Ritz - Rayleigh| {drift.max():.3e} eV"
              f"  -> {'OK' if ok else 'NOT CONVERGED at tol=%.0e' % tol}")
    return res, rq, ok


def hermiticity_error(A, n_probe=8, seed=0):
    rng = np.random.default_rng(seed)
    n = A.shape[0]
    worst = 0.0
    for _ in range(n_probe):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        x /= np.linalg.norm(x)
        y /= np.linalg.norm(y)
        worst = max(worst, abs(np.vdot(y, A @ x) - np.vdot(A @ y, x)))
    return worst


def folded_operator(A, sigma):
    """(A - sigma)^2 as a LinearOperator; applied on the GPU in one call per block."""
    A = _require_op(A)
    n = A.shape[0]

    def apply(x):
        x2 = np.asarray(x).reshape(n, -1)
        y = A.apply_host(x2, sigma=sigma, mode=_lib.APPLY_FOLDED)
        return y.reshape(np.shape(x))

    return spla.LinearOperator((n, n), matvec=apply, matmat=apply, dtype=np.complex128)


# ------------------------------------------------------------------------------------------
# Solvers
# ------------------------------------------------------------------------------------------

def solve_interior(A, k=4, sigma=0.0, M=None, tol=1e-8, maxiter=3000, extra=None, seed=0,
                   verbose=True, certify_tol=1e-6, return_device=False, time_hx=False):
    """Eigenpairs of A closest to sigma by folded-spectrum LOBPCG on the GPU."""
    A = _require_op(A)
    if M is not None:
        raise NotImplementedError("preconditioned LOBPCG is not built on the device "
                                  "(the reference's hot-path callers pass M=None)")
    n = A.shape[0]
    if extra is None:
        extra = max(2, k // 2)
    block = min(k + extra, n)
    X0 = start_block(n, block, seed, True)
    t0 = time.time()
    mu, Vd, hist, dinfo = lobpcg_device(A, X0, folded=True, sigma=sigma, tol=tol,
                                        maxiter=maxiter, time_hx=time_hx)
    rq, _ = _device_residuals(A, Vd)
    order = np.argsort(np.abs(rq - sigma))[:k]
    E = rq[order]
    order2 = np.argsort(E)
    sel = order[order2]
    E = E[order2]
    Vk = Vd[:, list(sel)].contiguous()
    _, res = _device_residuals(A, Vk, E)
    dt = time.time() - t0
    if verbose:
        print(f"  folded LOBPCG (B200): {dt:.1f}s, {len(hist)} iterations, block {block}, "
              f"sigma = {sigma:.4f} eV, max residual {res.max():.2e} eV")
        if res.max() > certify_tol:
            print(f"  WARNING: residual exceeds {certify_tol:.0e} eV -- the folded problem is "
                  f"badly conditioned; move sigma closer to the wanted states or raise maxiter.")
    info = dict(dinfo)
    info.update(time=dt, iterations=len(hist), residuals=res,
                converged=bool(res.max() < certify_tol), mu=mu, residual_history=hist)
    V = Vk if return_device else Vk.cpu().numpy()
    return E, V, info


def solve_lowest(A, k=4, M=None, X0=None, tol=1e-8, maxiter=2000, extra=None, seed=0,
                 verbose=True, certify_tol=1e-6, return_device=False):
    """Algebraically lowest k eigenpairs of A by LOBPCG on the GPU."""
    A = _require_op(A)
    if M is not None:
        raise NotImplementedError("preconditioned LOBPCG is not built on the device")
    n = A.shape[0]
    if extra is None:
        extra = max(2, k // 2)
    block = min(k + extra, n)
    if X0 is None:
        X0 = start_block(n, block, seed, True)
    elif X0.shape[1] < block:
        rng = np.random.default_rng(seed)
        pad = rng.standard_normal((n, block - X0.shape[1]))
        pad = pad + 1j * rng.standard_normal((n, block - X0.shape[1]))
        X0 = np.hstack([X0, pad])
    t0 = time.time()
    lam, Vd, hist, dinfo = lobpcg_device(A, X0, folded=False, tol=tol, maxiter=maxiter)
    order = np.argsort(lam)
    E = lam[order]
    Vd = Vd[:, list(order)].contiguous()
    _, res_all = _device_residuals(A, Vd, E)
    dt = time.time() - t0
    E_k, res_k = E[:k], res_all[:k]
    gap = (E[k] - E[k - 1]) if len(E) > k else np.nan
    if verbose:
        print(f"  LOBPCG (B200): {dt:.1f}s, {len(hist)} iterations, block {block}, max residual "
              f"on the wanted {k}: {res_k.max():.2e} eV; gap to next Ritz value {gap*1e3:.2f} meV")
    info = dict(dinfo)
    info.update(time=dt, iterations=len(hist), residuals=res_k, residuals_all=res_all,
                block=block, gap_to_next=gap, converged=bool(res_k.max() < certify_tol),
                residual_history=hist)
    Vk = Vd[:, :k].contiguous()
    return E_k, (Vk if return_device else Vk.cpu().numpy()), info


def solve_lowest_hole(A, k=4, **kwargs):
    """Hole states at the top of the spectrum: solve -A for the bottom, negate back
    (eigensolvers.py:375-386). -A is a second device operator with the sign flipped."""
    negA = _require_op(A).negated()
    try:
        E, V, info = solve_lowest(negA, k=k, **kwargs)
    finally:
        negA.close()
    return -E[::-1], V[:, ::-1].copy() if isinstance(V, np.ndarray) else V.flip(1), info
