import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA B200 and the built libqdkp.so')


@pytest.fixture(scope='session')
def operator_cases():
    """The reference's own H @ X on small grids for every confined_hamiltonian flag."""
    z = np.load(os.path.join(GOLDEN, 'operator_cases.npz'))
    keys = sorted({k.split('_')[0] for k in z.files})
    cases = []
    for key in keys:
        meta = z[key + '_meta']
        fields = {k[len(key) + 1:]: z[k] for k in z.files
                  if k.startswith(key + '_') and k[len(key) + 1:] not in ('meta', 'h', 'X', 'Y')}
        cases.append(dict(name=key, shape=tuple(int(v) for v in meta[:3]), n_bands=int(meta[3]),
                          hole=bool(meta[4]), strain=bool(meta[5]), hydro=bool(meta[6]),
                          interband=bool(meta[7]), nnz=int(meta[8]), h=float(z[key + '_h']),
                          fields=fields, X=z[key + '_X'], Y=z[key + '_Y']))
    return cases
