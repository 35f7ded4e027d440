"""Failure statuses, injected on the host (no GPU fault, trap or hang is involved).

The reference's failure behaviour is scipy's: a rank-deficient start block raises "Linearly
dependent initial approximations" (scipy lobpcg.py:628-635), a residual that blows up restarts
or stops the loop, and eigensolvers.py reports convergence through `info` instead of raising
(eigensolvers.py:243-248). Here every solve carries a status:
  * a NaN in a coefficient field      -> 'nonfinite' (plain and served), others unaffected;
  * a start block with repeated columns -> the same error as scipy;
  * a sigma inside a dense continuum  -> 'maxiter' at the request's budget, while the solves
    sharing the engine finish exactly as they do alone;
  * a zero-extent grid                -> QDKP_ERR_ARG (tests/test_abi.py, no GPU needed).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _small(nan_site=None):
    from qd3dsolver_b200 import kp_pryor as kpg
    z = np.load(os.path.join(GOLDEN, 'solve_cases.npz'))
    with open(os.path.join(GOLDEN, 'solve_cases.json')) as fh:
        meta = json.load(fh)
    f = {k[3:]: np.array(z[k]) for k in z.files if k.startswith('f8_')}
    if nan_site is not None:
        f['Ec'].reshape(-1)[nan_site] = np.nan
    st = {k: f[k] for k in ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')}
    H = kpg.confined_hamiltonian(kpg.GridOperators(tuple(meta['shape']), float(z['h'])), f, 8,
                                 strain=st)
    return H, meta


def test_nan_field_gives_nonfinite_status_plain_and_served():
    from qd3dsolver_b200 import eigensolvers as eg, serving
    Hbad, meta = _small(nan_site=123)
    Hok, _ = _small()
    sig = meta['interior_cb']['sigma']
    E, V, info = eg.solve_interior(Hbad, k=4, sigma=sig, tol=1e-9, maxiter=50, verbose=False)
    assert info['status'] == 'nonfinite' and not info['converged']
    good = lambda: serving.Request(Hok, k=4, sigma=sig, tol=1e-9, maxiter=4000, tag='ok')
    bad = serving.Request(Hbad, k=4, sigma=sig, tol=1e-9, maxiter=4000, tag='nan')
    mix = serving.solve_batch([bad, good()], max_slots=2, ticks_per_poll=4)
    alone = serving.solve_batch([good()], max_slots=1, ticks_per_poll=4)[0]
    assert mix[0].result['status'] == 'nonfinite' and not mix[0].result['converged']
    assert mix[1].result['status'] == 'converged'
    assert mix[1].result['iterations'] == alone.result['iterations']
    assert np.abs(mix[1].result['E'] - alone.result['E']).max() <= 1e-12


def test_rank_deficient_start_block_is_refused_like_scipy():
    from qd3dsolver_b200 import eigensolvers as eg, serving, _lib
    H, meta = _small()
    n = H.shape[0]
    X0 = eg.start_block(n, 6, 0)
    X0[:, 3] = X0[:, 1]                                    # a repeated column
    with pytest.raises(_lib.QdkpError, match='Linearly dependent initial approximations'):
        eg.solve_lowest(H, k=4, X0=X0, tol=1e-9, maxiter=50, verbose=False)
    import torch
    eng = serving.Engine(2)
    r = serving.Request(H, k=4, sigma=meta['interior_cb']['sigma'], tol=1e-9, maxiter=50)
    with pytest.raises(_lib.QdkpError):
        eng.admit(r, X0=torch.from_numpy(X0).cuda())
    eng.close()


def test_continuum_sigma_retires_at_maxiter_without_delaying_others():
    """A folded request centred deep in the conduction continuum of the b = 10 nm pyramid runs to
    its iteration budget and retires with status maxiter; a bound-state request sharing the
    engine finishes with the same iterations and eigenvalues as alone."""
    from qd3dsolver_b200 import kp_pryor as kpg, serving, workloads as wl
    w = wl.fig4_from_fixture(os.path.join(GOLDEN, 'fig4_b10_fields.npz'))
    f = w.fields
    H = kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                 strain={k: f[k] for k in wl.STRAIN_KEYS})
    cont = serving.Request(H, k=8, sigma=2.2, tol=1e-9, maxiter=150, tag='continuum')
    good = lambda: serving.Request(H, k=8, sigma=w.sigma['cb'], tol=1e-8, maxiter=8000, tag='cb')
    mix = serving.solve_batch([cont, good()], max_slots=2, ticks_per_poll=8)
    alone = serving.solve_batch([good()], max_slots=1, ticks_per_poll=8)[0]
    assert mix[0].result['status'] == 'maxiter' and not mix[0].result['converged']
    assert mix[0].result['iterations'] <= 150 + 3
    assert mix[1].result['status'] == 'converged'
    assert mix[1].result['iterations'] == alone.result['iterations']
    assert np.abs(mix[1].result['E'] - alone.result['E']).max() <= 1e-12
    H.close()
