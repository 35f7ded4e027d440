"""The six-band hole route on the GPU against the reference's own heterostructure.six_band_holes
(eigsh 'LA' on the six-band operator) and valence_edge_top, on an InAs lens in GaAs
(tests/golden/make_sixband_golden.py)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


@pytest.fixture(scope='module')
def env():
    from qd3dsolver_b200 import workloads as wl
    z = np.load(os.path.join(GOLDEN, 'sixband_fields.npz'))
    with open(os.path.join(GOLDEN, 'sixband.json')) as fh:
        ref = json.load(fh)
    e = dict(mask=z['mask'], h=ref['h'], dot=wl.material(ref['dot']),
             matrix=wl.material(ref['matrix']), Ev=z['Ev'], Ec=z['Ec'],
             strain={k: z[k] for k in STRAIN})
    return e, ref


def test_valence_edge_top(env):
    from qd3dsolver_b200 import heterostructure as hs
    e, ref = env
    assert hs.valence_edge_top(e) == pytest.approx(ref['top'], abs=1e-12)
    rep = hs.valence_edge_top(e, reduce='mean', erode=1, report=True)
    assert rep['top_raw_max'] == pytest.approx(ref['top'], abs=1e-12)
    assert rep['n_interior'] < rep['n_mask']


@pytest.mark.parametrize('k', [4, 8])
def test_six_band_holes_match_the_reference(env, k):
    from qd3dsolver_b200 import heterostructure as hs
    e, ref = env
    r = hs.six_band_holes(e, k=k, tol=1e-9, verbose=False)
    rk = ref[f'k{k}']
    assert r['n_spurious'] == rk['n_spurious'] and r['n_bands'] == 6
    assert len(r['E']) == len(rk['E'])
    assert np.abs(np.asarray(r['E']) - np.asarray(rk['E'])).max() < 1e-7
    assert np.all(np.diff(r['E']) <= 1e-12)                       # descending, like the reference
    assert np.abs(np.asarray(r['loc']) - np.asarray(rk['loc'])).max() < 1e-5
    assert r['V'].shape == (6 * e['mask'].size, len(rk['E']))
