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
