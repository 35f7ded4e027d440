"""The allocation-free folded apply, checked against the workspace-taking entry point.

qdkp_apply_folded_noalloc serves callers that cannot allocate device memory when they apply the
operator (bindings without a device allocator, contexts where cudaMalloc's implicit
synchronisation is not allowed). It must give the same (H - sigma)^2 X as
qdkp_apply(..., QDKP_APPLY_FOLDED, workspace) on consecutive calls, and refuse blocks larger
than its fixed scratch. This file is collected last so that a stop at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _operator():
    from qd3dsolver_b200 import kp_pryor as kpg
    z = np.load(os.path.join(GOLDEN, 'solve_cases.npz'))
    with open(os.path.join(GOLDEN, 'solve_cases.json')) as fh:
        meta = json.load(fh)
    f = {k[3:]: z[k] for k in z.files if k.startswith('f8_')}
    st = {k: f[k] for k in ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')}
    return kpg.confined_hamiltonian(kpg.GridOperators(tuple(meta['shape']), float(z['h'])), f,
                                    8, strain=st)


def _call_noalloc(L, H, X, Y, sigma, prec, stream):
    return L.qdkp_apply_folded_noalloc(H.handle, X.data_ptr(), X.stride(0), Y.data_ptr(),
                                       Y.stride(0), X.shape[1], sigma, prec, stream)


def test_noalloc_folded_matches_workspace_apply_twice():
    import torch
    from qd3dsolver_b200 import _lib
    L = _lib.lib()
    H = _operator()
    n = H.shape[0]
    stream = torch.cuda.current_stream().cuda_stream
    gen = torch.Generator(device='cuda').manual_seed(11)
    for dtype, prec, tol in ((torch.complex128, _lib.C128, 1e-13),
                             (torch.complex64, _lib.C64, 1e-6)):
        for call, (m, sigma) in enumerate(((6, 1.0585), (3, 0.2856))):   # two calls in a row
            X = torch.randn((n, m), dtype=dtype, device='cuda', generator=gen)
            Y = torch.empty_like(X)
            Yref = torch.empty_like(X)
            ws = torch.empty_like(X)
            rc = L.qdkp_apply(H.handle, X.data_ptr(), m, Yref.data_ptr(), m, m, sigma,
                              _lib.APPLY_FOLDED, prec, ws.data_ptr(),
                              ws.numel() * ws.element_size(), stream)
            assert rc == 0, L.qdkp_last_error()
            rc = _call_noalloc(L, H, X, Y, sigma, prec, stream)
            assert rc == 0, L.qdkp_last_error()
            torch.cuda.synchronize()
            err = ((Y - Yref).abs().max() / Yref.abs().max()).item()
            assert err < tol, (dtype, call, err)


def test_noalloc_rejects_blocks_beyond_the_scratch():
    import torch
    from qd3dsolver_b200 import _lib
    L = _lib.lib()
    H = _operator()
    n = H.shape[0]
    cap = L.qdkp_apply_folded_noalloc_max_elems(_lib.C128)
    assert cap == (64 << 20) // 16
    m = cap // n + 1                                    # one column more than fits
    X = torch.zeros((n, m), dtype=torch.complex128, device='cuda')
    Y = torch.empty_like(X)
    rc = _call_noalloc(L, H, X, Y, 0.5, _lib.C128, torch.cuda.current_stream().cuda_stream)
    assert rc == -4
    assert b'exceed the fixed scratch' in L.qdkp_last_error()


def test_noalloc_folded_matches_the_oracle():
    """The allocation-free folded apply against the oracle's own (H - sigma)^2 X (the restated
    CSR pinned to the reference's H @ X), complex128 to 1e-13, complex64 to single precision."""
    import torch
    from qd3dsolver_b200 import _lib
    from oracle import kp_operator as ko
    L = _lib.lib()
    H = _operator()
    z = np.load(os.path.join(GOLDEN, 'solve_cases.npz'))
    with open(os.path.join(GOLDEN, 'solve_cases.json')) as fh:
        meta = json.load(fh)
    f = {k[3:]: z[k] for k in z.files if k.startswith('f8_')}
    Ho = ko.confined_hamiltonian(tuple(meta['shape']), float(z['h']), f, 8, strain=True)
    n = H.shape[0]
    rng = np.random.default_rng(12)
    sigma = 0.8123
    Xh = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    S = Ho @ Xh - sigma * Xh
    ref = Ho @ S - sigma * S
    stream = torch.cuda.current_stream().cuda_stream
    for dtype, prec, tol in ((torch.complex128, _lib.C128, 1e-13), (torch.complex64, _lib.C64, 4e-6)):
        X = torch.from_numpy(Xh).to(dtype).cuda()
        Y = torch.empty_like(X)
        assert _call_noalloc(L, H, X, Y, sigma, prec, stream) == 0, L.qdkp_last_error()
        torch.cuda.synchronize()
        err = np.abs(Y.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err < tol, (dtype, err)
    H.close()

