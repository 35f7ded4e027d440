"""The host input producers of qd3dsolver_b200.workloads against the reference's own outputs.

tests/golden/inputs_cases.* were written by the reference itself (make_inputs_golden.py): its
material tables and alloy rule, masks, homogeneous Fourier strain, piezo potential, band-edge
fields, material fields and the exact valence edge / hole_sigma, on an InAs pyramid in GaAs and an
In(0.45)Ga(0.55)Sb lens in InAs. The restatement must reproduce them to rounding.
"""
import json
import os

import numpy as np
import pytest

from qd3dsolver_b200 import workloads as wl

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


@pytest.fixture(scope='module')
def golden():
    z = np.load(os.path.join(GOLDEN, 'inputs_cases.npz'))
    with open(os.path.join(GOLDEN, 'inputs_cases.json')) as fh:
        meta = json.load(fh)
    return z, meta


def _close(a, b, rtol=1e-12):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= rtol * scale


def test_material_tables_and_alloys(golden):
    _, meta = golden
    for name in ('GaAs', 'InAs', 'GaSb', 'InSb'):
        m = wl.material(name)
        for k, v in meta['materials'][name].items():
            assert m[k] == pytest.approx(v, rel=1e-12, abs=1e-15), (name, k)
    for key, (sysname, x) in {'InGaSb(0.45)': ('InGaSb', 0.45), 'InAsSb(0.3)': ('InAsSb', 0.3),
                              'InGaSb(1.0)': ('InGaSb', 1.0)}.items():
        m = wl.alloy(sysname, x)
        for k, v in meta['materials'][key].items():
            assert m[k] == pytest.approx(v, rel=1e-12, abs=1e-15), (key, k)


def test_pryor_table(golden):
    _, meta = golden
    for name, ref in meta['pryor'].items():
        ours = wl.PRYOR_TABLE_I[name]
        for k, v in ours.items():
            assert v == pytest.approx(ref[k], rel=1e-12, abs=1e-15), (name, k)


@pytest.mark.parametrize('tag', ['pyr', 'lens'])
def test_fields_of_a_dot(golden, tag):
    z, meta = golden
    c = meta['cases'][tag]
    shape, h = tuple(c['shape']), c['h']
    dot = wl.alloy(*c['dot']) if isinstance(c['dot'], list) else wl.material(c['dot'])
    mat = wl.material(c['matrix'])
    cx = wl.centered_axis(shape[0], h)
    cz = (np.arange(shape[2]) - c['z_offset_cells'] + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    mask = (wl.pyramid_mask(X, Y, Z, 4.0) if tag == 'pyr' else wl.lens_mask(X, Y, Z, 2.6, 1.4))
    assert np.array_equal(mask, z[f'{tag}_mask'])
    eps = wl.misfit(dot, mat)
    assert eps == pytest.approx(c['misfit'], rel=1e-13)
    st = wl.solve_strain(mask, eps, mat['C11'], mat['C12'], mat['C44'], h)
    for k in STRAIN:
        assert _close(st[k], z[f'{tag}_{k}']), k
    e14 = np.where(mask, dot['e14'], mat['e14'])
    phi = wl.piezo_potential(st, e14, mat['eps_R'], h)
    assert _close(phi, z[f'{tag}_phi'], 1e-11)
    Ec, Ev = wl.band_edge_fields(mask, st['exx'] + st['eyy'] + st['ezz'], dot, mat)
    Ec, Ev = Ec - phi, Ev - phi
    assert _close(Ec, z[f'{tag}_Ec']) and _close(Ev, z[f'{tag}_Ev'])
    f8 = wl.material_fields(mask, dot, mat, Ev, Ec, 8)
    for k in ('gamma1', 'gamma2', 'gamma3', 'P0', 'delta_so', 'b', 'd', 'a_c', 'a_v'):
        assert _close(f8[k], z[f'{tag}_f8_{k}']), k
    f6 = wl.material_fields(mask, dot, mat, Ev, Ec, 6)
    for k in ('gamma1', 'gamma2', 'gamma3'):
        assert _close(f6[k], z[f'{tag}_f6_{k}']), k
    v1 = wl.local_valence_edge(Ev, st, f8['b'], f8['d'], f8['delta_so'])
    assert _close(v1, z[f'{tag}_v1'], 1e-12)
    assert wl.hole_sigma(Ev, st, f8['b'], f8['d'], f8['delta_so'], mask) == \
        pytest.approx(c['sigma_h'], abs=1e-12)
    assert float(Ec[mask].min()) == pytest.approx(c['sigma_e'], abs=1e-12)


def test_48x48x36_pyramid_fields_match_the_reference():
    """The 48x48x36 pyramid workload (workloads.config1) against the per-field sums, sigmas and
    dot volume the reference recorded for the same geometry (make_config1_golden.py)."""
    with open(os.path.join(GOLDEN, 'config1_iterates.json')) as fh:
        ref = json.load(fh)
    w = wl.config1()
    assert list(w.shape) == ref['shape'] and int(w.mask.sum()) == ref['mask_cells']
    assert w.sigma['cb'] == pytest.approx(ref['sigma_e'], abs=1e-12)
    assert w.sigma['vb'] == pytest.approx(ref['sigma_h'], abs=1e-12)
    for k, v in ref['field_sums'].items():
        scale = float(np.abs(w.fields[k]).sum())
        assert abs(float(np.sum(w.fields[k])) - v) <= 1e-12 * scale + 1e-12, k
