"""Fourier strain and the piezo potential on the GPU (qdkp_fourier_strain, qdkp_piezo_potential)
against the reference's own strain_fourier.solve_strain and piezoelectric.potential outputs
(tests/golden/inputs_cases.*: an InAs pyramid in GaAs and an InGaSb lens in InAs), and against
the pinned host restatement on the 48x48x36 pyramid (odd and even extents both covered)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize('tag', ['pyr', 'lens'])
def test_strain_and_potential_match_the_reference(tag):
    from qd3dsolver_b200 import fields, workloads as wl
    z = np.load(os.path.join(GOLDEN, 'inputs_cases.npz'))
    with open(os.path.join(GOLDEN, 'inputs_cases.json')) as fh:
        meta = json.load(fh)
    c = meta['cases'][tag]
    mat = wl.material(c['matrix'])
    dot = wl.alloy(*c['dot']) if isinstance(c['dot'], list) else wl.material(c['dot'])
    mask = z[f'{tag}_mask']
    st = fields.solve_strain(mask, c['misfit'], mat['C11'], mat['C12'], mat['C44'], c['h'])
    for k in STRAIN:
        assert _rel(getattr(st, k), z[f'{tag}_{k}']) < 1e-12, k
    e14 = np.where(mask, dot['e14'], mat['e14'])
    phi = fields.potential(st, e14, mat['eps_R'], c['h'])
    assert _rel(phi, z[f'{tag}_phi']) < 1e-11
    phin = fields.potential(st, e14, mat['eps_R'], c['h'], sign=-1.0)
    assert _rel(phin, -z[f'{tag}_phi']) < 1e-11


def test_strain_on_the_48x48x36_and_odd_grids():
    from qd3dsolver_b200 import fields, workloads as wl
    w = wl.config1()
    mat = wl.material('GaAs')
    eps = wl.misfit(wl.material('InAs'), mat)
    st = fields.solve_strain(w.mask, eps, mat['C11'], mat['C12'], mat['C44'], w.h)
    for k in STRAIN:
        assert _rel(getattr(st, k), w.fields[k]) < 1e-12, k
    rng = np.random.default_rng(9)
    mask = rng.random((9, 7, 11)) < 0.3
    ref = wl.solve_strain(mask, eps, mat['C11'], mat['C12'], mat['C44'], 0.6)
    st = fields.solve_strain(mask, eps, mat['C11'], mat['C12'], mat['C44'], 0.6)
    for k in STRAIN:
        assert _rel(getattr(st, k), ref[k]) < 1e-12, k
    e14 = np.where(mask, -0.045, -0.16)
    assert _rel(fields.potential(st, e14, 12.9, 0.6), wl.piezo_potential(ref, e14, 12.9, 0.6)) < 1e-11
