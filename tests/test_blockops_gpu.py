"""The tall-skinny block products of the LOBPCG iteration on the B200, against numpy: Gram
matrices A^H B and Ritz updates A C, for complex128 blocks (FP64 tensor-core MMA) and complex64
blocks (split-precision TF32 tensor-core MMA, FP32 accumulation, FP64 partial sums)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(1000, 12, 12), (37_123, 36, 24), (5_000, 36, 36), (999, 7, 5), (300_000, 12, 12),
          (2_048, 24, 12)]


def _dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a.astype(dtype))).cuda()


@pytest.mark.parametrize('prec', ['c128', 'c64'])
def test_block_gram(prec):
    import torch
    from qd3dsolver_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(3)
    dt = np.complex128 if prec == 'c128' else np.complex64
    code = _lib.C128 if prec == 'c128' else _lib.C64
    for n, P, Q in SHAPES:
        A = rng.standard_normal((n, P)) + 1j * rng.standard_normal((n, P))
        B = rng.standard_normal((n, Q)) + 1j * rng.standard_normal((n, Q))
        A, B = A.astype(dt).astype(np.complex128), B.astype(dt).astype(np.complex128)
        ref = A.conj().T @ B
        dA, dB = _dev(A, dt), _dev(B, dt)
        ws = torch.empty(int(L.qdkp_block_gram_workspace_size(P, Q)), dtype=torch.uint8,
                         device='cuda')
        out = np.empty((P, Q), dtype=np.complex128)
        _lib.check(L.qdkp_block_gram(dA.data_ptr(), P, P, dB.data_ptr(), Q, Q, n, code,
                                     out.ctypes.data, ws.data_ptr(), ws.numel(), None),
                   'qdkp_block_gram')
        # error relative to |A|^H |B| (the scale of the summed products)
        scale = (np.abs(A).T @ np.abs(B)).max()
        err = np.abs(out - ref).max() / scale
        assert err < (1e-14 if prec == "c128" else 1e-6), (n, P, Q, err)


@pytest.mark.parametrize('prec', ['c128', 'c64'])
def test_block_update(prec):
    import torch
    from qd3dsolver_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(4)
    dt = np.complex128 if prec == 'c128' else np.complex64
    code = _lib.C128 if prec == 'c128' else _lib.C64
    for n, P, q in [(1000, 24, 12), (37_123, 12, 12), (999, 7, 5), (300_001, 36, 12)]:
        A = (rng.standard_normal((n, P)) + 1j * rng.standard_normal((n, P))).astype(dt)
        C = rng.standard_normal((P, q)) + 1j * rng.standard_normal((P, q))
        ref = A.astype(np.complex128) @ C
        dA = _dev(A, dt)
        dY = torch.empty((n, q), dtype=dA.dtype, device='cuda')
        ws = torch.empty(int(L.qdkp_block_update_workspace_size(P, q)), dtype=torch.uint8,
                         device='cuda')
        Cc = np.ascontiguousarray(C)
        _lib.check(L.qdkp_block_update(dA.data_ptr(), P, P, Cc.ctypes.data, q, n,
                                       dY.data_ptr(), q, code, ws.data_ptr(), ws.numel(), None),
                   'qdkp_block_update')
        Y = dY.cpu().numpy().astype(np.complex128)
        scale = (np.abs(A).astype(float) @ np.abs(C)).max()
        err = np.abs(Y - ref).max() / scale
        assert err < (1e-14 if prec == "c128" else 1e-6), (n, P, q, err)
        # in place on the input block (the engine's X = X Cx, R = R U): first q columns
        if P >= q:
            dA2 = _dev(A, dt)
            Cq = np.ascontiguousarray(C)
            _lib.check(L.qdkp_block_update(dA2.data_ptr(), P, P, Cq.ctypes.data, q, n,
                                           dA2.data_ptr(), P, code, ws.data_ptr(), ws.numel(),
                                           None), 'qdkp_block_update')
            Y2 = dA2.cpu().numpy()[:, :q].astype(np.complex128)
            assert np.abs(Y2 - ref).max() / scale < (1e-14 if prec == "c128" else 1e-6)


def _pencil(rng, n, kind):
    """Hermitian A and positive definite B (or None) shaped like LOBPCG's Rayleigh-Ritz pencils:
    'pairs': a spectrum of exactly degenerate pairs (Kramers-like) with a general B; 'folded': a
    cluster of small eigenvalues (a folded spectrum near sigma) under large ones, with a general B;
    'random': Gaussian Hermitian with B = None."""
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    if kind == 'pairs':
        lam = np.repeat(1e-3 * np.arange(n // 2 + 1) * (1 + 0.1 * (np.arange(n // 2 + 1) % 3)), 2)[:n]
    elif kind == 'folded':
        lam = np.concatenate([np.sort(rng.uniform(1e-5, 1e-2, n // 3)),
                              rng.uniform(1.0, 100.0, n - n // 3)])
    else:
        X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        return (X + X.conj().T) / 2, None
    A = (Q * lam) @ Q.conj().T
    A = (A + A.conj().T) / 2
    Gm = np.eye(n) + 0.3 / np.sqrt(n) * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    return A, Gm.conj().T @ Gm


@pytest.mark.parametrize('n', [12, 24, 36, 48, 72])
def test_block_eigh(n):
    """The Rayleigh-Ritz eigensolve against scipy.linalg.eigh, for all pairs (Householder + QL)
    and for the wanted smallest pairs only (multisection + inverse iteration): eigenvalues,
    residuals and B-orthonormality, on degenerate-pair, folded and random pencils."""
    import scipy.linalg as sl
    from qd3dsolver_b200 import _lib
    L = _lib.lib()
    import torch
    rng = np.random.default_rng(n)
    ws = torch.empty(int(L.qdkp_block_eigh_workspace_size(n)), dtype=torch.uint8, device='cuda')
    for kind in ('pairs', 'folded', 'random'):
        A, B = _pencil(rng, n, kind)
        wref = sl.eigh(A, B, eigvals_only=True)
        anorm = np.abs(wref).max()
        for nwant in sorted({n, max(1, n // 3), n // 2}):
            w = np.zeros(n)
            V = np.zeros((n, n), dtype=np.complex128)
            Ac = np.ascontiguousarray(A)
            Bc = None if B is None else np.ascontiguousarray(B)
            _lib.check(L.qdkp_block_eigh(Ac.ctypes.data, None if Bc is None else Bc.ctypes.data,
                                         n, nwant, w.ctypes.data, V.ctypes.data, ws.data_ptr(),
                                         ws.numel(), None), 'qdkp_block_eigh')
            Bm = np.eye(n) if B is None else B
            Vk, wk = V[:, :nwant], w[:nwant]
            assert np.all(np.diff(wk) >= 0), (kind, nwant)
            assert np.abs(wk - wref[:nwant]).max() <= 1e-12 * anorm, (kind, nwant)
            res = np.linalg.norm(A @ Vk - (Bm @ Vk) * wk, axis=0).max() / anorm
            orth = np.abs(Vk.conj().T @ Bm @ Vk - np.eye(nwant)).max()
            assert res < 1e-13, (kind, nwant, res)
            assert orth < 1e-12, (kind, nwant, orth)


def test_block_eigh_not_positive_definite():
    import torch
    from qd3dsolver_b200 import _lib
    L = _lib.lib()
    n = 24
    A = np.eye(n, dtype=np.complex128)
    B = -np.eye(n, dtype=np.complex128)
    ws = torch.empty(int(L.qdkp_block_eigh_workspace_size(n)), dtype=torch.uint8, device='cuda')
    w = np.zeros(n)
    V = np.zeros((n, n), dtype=np.complex128)
    for nwant in (n, 8):
        rc = L.qdkp_block_eigh(A.ctypes.data, B.ctypes.data, n, nwant, w.ctypes.data,
                               V.ctypes.data, ws.data_ptr(), ws.numel(), None)
        assert rc == -5, rc                       # QDKP_ERR_NUMERIC
