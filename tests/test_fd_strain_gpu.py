"""The inhomogeneous FD elasticity solve on the B200 (qdkp_fd_strain through fields.solve_strain_fd)
against the reference's own elasticity_fd.solve_strain_fd: the small cases of
tests/golden/make_fd_golden.py and the FD strain of all seven Fig-4 environments
(tests/golden/make_fig4_golden.py), which the reference built with the same function."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')
# both solves stop at ||r|| / ||f|| < 1e-10: the fields agree to the CG tolerance times the
# operator's conditioning, far below the 1e-6 the band edges need
TOL = 1e-8


def _meta():
    with open(os.path.join(GOLDEN, 'fd_strain_cases.json')) as fh:
        return json.load(fh)


def _err(st, ref):
    scale = max(np.abs(ref[k]).max() for k in STRAIN)
    return max(np.abs(getattr(st, k) - ref[k]).max() for k in STRAIN) / scale


def test_fd_strain_reference_cases():
    from qd3dsolver_b200 import fields
    meta = _meta()
    arr = np.load(os.path.join(GOLDEN, 'fd_strain_cases.npz'))
    for c in meta['cases']:
        t = c['tag']
        st, tot = fields.solve_strain_fd(arr[f'{t}_mask'], c['eps_star'], c['C_dot'],
                                         c['C_matrix'], c['h'], tol=c['tol'], return_total=True)
        ref = {k: arr[f'{t}_{k}'] for k in STRAIN}
        assert _err(st, ref) < TOL, (t, _err(st, ref))
        assert st.cg_converged and st.cg_modes_dropped == c['modes_dropped'] == 1
        assert abs(st.cg_iterations - c['iterations']) <= 1, (t, st.cg_iterations, c['iterations'])
        # total = elastic + the eigenstrain inside the dot on the diagonal
        off = -c['eps_star'] * arr[f'{t}_mask']
        assert np.abs(tot.exx - st.exx - off).max() < 1e-14
        assert np.abs(tot.exy - st.exy).max() == 0.0


@pytest.mark.parametrize('base', [6, 8, 10, 12, 14, 16, 18])
def test_fd_strain_fig4_environments(base):
    from qd3dsolver_b200 import fields
    f = _meta()['fig4']
    fx = np.load(os.path.join(GOLDEN, f'fig4_b{base}_fields.npz'))
    st = fields.solve_strain_fd(fx['mask'], f['eps_star'], f['C_dot'], f['C_matrix'], f['h'],
                                tol=f['tol'])
    ref = {k: fx[k] for k in STRAIN}
    assert st.cg_converged
    assert _err(st, ref) < TOL, (base, _err(st, ref))


def test_fd_strain_unconverged_raises():
    """require_converged: a capped iteration count raises like the reference
    (elasticity_fd.py:328-341); with require_converged=False the field comes back flagged."""
    from qd3dsolver_b200 import fields
    f = _meta()['fig4']
    fx = np.load(os.path.join(GOLDEN, 'fig4_b6_fields.npz'))
    with pytest.raises(RuntimeError, match='did not converge'):
        fields.solve_strain_fd(fx['mask'], f['eps_star'], f['C_dot'], f['C_matrix'], f['h'],
                               tol=1e-10, maxiter=2)
    st = fields.solve_strain_fd(fx['mask'], f['eps_star'], f['C_dot'], f['C_matrix'], f['h'],
                                tol=1e-10, maxiter=2, require_converged=False)
    assert not st.cg_converged and st.cg_iterations == 2 and st.cg_residual > 1e-10


def test_fig4_environment_fd_strain_matches_reference_fields():
    """workloads.fig4_environment(strain='fd') with this package's Pryor Table I constants and
    eigenstrain reproduces the reference environment's FD strain (pryor_fig4.py:115)."""
    from qd3dsolver_b200 import workloads as wl
    fx = np.load(os.path.join(GOLDEN, 'fig4_b10_fields.npz'))
    w = wl.fig4_environment(10.0, strain='fd')
    assert w.mask.shape == fx['mask'].shape and np.array_equal(w.mask, fx['mask'])
    scale = max(np.abs(fx[k]).max() for k in STRAIN)
    err = max(np.abs(w.fields[k] - fx[k]).max() for k in STRAIN) / scale
    assert err < TOL, err
    # and the band edges and sigmas built from it (Bir-Pikus shifts, piezo potential)
    for k in ('Ec', 'Ev'):
        assert np.abs(w.fields[k] - fx[k]).max() < 1e-8, k
    assert abs(w.sigma['cb'] - float(fx['sigma_e'])) < 1e-8
    assert abs(w.sigma['vb'] - float(fx['sigma_h'])) < 1e-8
