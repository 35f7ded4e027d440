"""The sigma providers on the GPU (qdkp_local_band_edges): kp_pryor.local_band_edges and
kp_pryor.hole_sigma (kp_pryor.py:156-191, 469-531) against the reference's own values.

  * the exact valence-band top inside the dot of every Fig-4 environment the reference built
    (sigma_h of tests/golden/fig4_b*.json / _fields.npz);
  * the per-site v1 field and hole_sigma of the input fixtures (tests/golden/inputs_cases.*),
    through the drop-in functions with the reference's signatures.
"""
import glob
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def test_hole_sigma_of_every_fig4_environment():
    from qd3dsolver_b200 import kp_pryor as kpg, workloads as wl
    paths = sorted(glob.glob(os.path.join(GOLDEN, 'fig4_b*_fields.npz')))
    assert paths
    for p in paths:
        w = wl.fig4_from_fixture(p)
        f = w.fields
        H = kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                     strain={k: f[k] for k in STRAIN})
        e = H.band_edges(mask=w.mask, levels=True)
        assert e['top_v1'] == pytest.approx(w.sigma['vb'], abs=1e-12), p
        assert e['kramers'] < 1e-12
        v1 = wl.local_valence_edge(f['Ev'], f, f['b'], f['d'], f['delta_so'])
        assert np.abs(e['v1'] - v1).max() < 1e-12
        assert np.all(e['v1'] >= e['v2'] - 1e-15) and np.all(e['v2'] >= e['v3'] - 1e-15)
        H.close()


@pytest.mark.parametrize('tag', ['pyr', 'lens'])
def test_drop_in_local_band_edges_and_hole_sigma(tag):
    from qd3dsolver_b200 import kp_pryor as kpg
    z = np.load(os.path.join(GOLDEN, 'inputs_cases.npz'))
    with open(os.path.join(GOLDEN, 'inputs_cases.json')) as fh:
        meta = json.load(fh)['cases'][tag]
    st = {k: z[f'{tag}_{k}'] for k in STRAIN}
    Ev, Ec, mask = z[f'{tag}_Ev'], z[f'{tag}_Ec'], z[f'{tag}_mask']
    b, d, dso = (z[f'{tag}_f8_{k}'] for k in ('b', 'd', 'delta_so'))
    e = kpg.local_band_edges(st, Ev, Ec, dso, 0.0, 0.0, b, d, hydrostatic_applied=True)
    assert np.abs(e['v1'] - z[f'{tag}_v1']).max() < 1e-12
    assert np.array_equal(e['cb'], Ec) and e['kramers'] < 1e-12
    sig = kpg.hole_sigma(Ev, st, b, d, dso, inside_mask=mask)
    assert sig == pytest.approx(meta['sigma_h'], abs=1e-12)
    assert kpg.hole_sigma(Ev, st, b, d, dso, inside_mask=mask, margin=0.01) == \
        pytest.approx(meta['sigma_h'] + 0.01, abs=1e-12)
