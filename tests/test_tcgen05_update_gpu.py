"""The complex64 block updates on the tcgen05 pipeline (QDKP_C64_UPDATE=tcgen05): the kernel is
chosen once per process, so the existing update, engine and Fig-4 counting-rule tests run again
in a child process that selects it, and a direct check compares it with the default split-TF32
mma.sync kernel on the same inputs."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHECK = r'''
import numpy as np, torch, sys
sys.path.insert(0, sys.argv[1])
from qd3dsolver_b200 import _lib
L = _lib.lib()
rng = np.random.default_rng(11)
out = {}
for n, P, q in [(84_640, 36, 12), (300_001, 72, 24), (999, 7, 5), (129, 3, 1)]:
    A = (rng.standard_normal((n, P)) + 1j * rng.standard_normal((n, P))).astype(np.complex64)
    C = np.ascontiguousarray(rng.standard_normal((P, q)) + 1j * rng.standard_normal((P, q)))
    dA = torch.from_numpy(A).cuda()
    dY = torch.empty((n, q), dtype=torch.complex64, device='cuda')
    ws = torch.empty(int(L.qdkp_block_update_workspace_size(P, q)), dtype=torch.uint8, device='cuda')
    _lib.check(L.qdkp_block_update(dA.data_ptr(), P, P, C.ctypes.data, q, n, dY.data_ptr(), q,
                                   _lib.C64, ws.data_ptr(), ws.numel(), None), 'qdkp_block_update')
    out[f'{n}_{P}_{q}'] = dY.cpu().numpy()
np.savez(sys.argv[2], **out)
'''


def _run_check(env_value, path):
    env = dict(os.environ, QDKP_C64_UPDATE=env_value)
    r = subprocess.run([sys.executable, '-c', _CHECK, ROOT, path], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(path)


def test_tcgen05_and_mma_updates_agree(tmp_path):
    """Both kernels against each other and against the FP64 product, on the engine's shapes
    (three 12-column blocks, 24-column blocks split into three, ragged sizes)."""
    a = _run_check('tcgen05', str(tmp_path / 'tc.npz'))
    b = _run_check('mma', str(tmp_path / 'mma.npz'))
    rng = np.random.default_rng(11)
    for n, P, q in [(84_640, 36, 12), (300_001, 72, 24), (999, 7, 5), (129, 3, 1)]:
        A = (rng.standard_normal((n, P)) + 1j * rng.standard_normal((n, P))).astype(np.complex64)
        C = rng.standard_normal((P, q)) + 1j * rng.standard_normal((P, q))
        ref = A.astype(np.complex128) @ C
        scale = (np.abs(A).astype(float) @ np.abs(C)).max()
        key = f'{n}_{P}_{q}'
        assert np.abs(a[key] - ref).max() / scale < 1e-6, key
        assert np.abs(b[key] - ref).max() / scale < 1e-6, key
        assert np.abs(a[key] - b[key]).max() / scale < 2e-6, key


def test_engine_and_update_tests_on_tcgen05():
    """The block-update tests, the engine's alone-equals-mix and single-solve tests and the served
    mixed form's counting rule on the Fig-4 fixtures, with the tcgen05 updates."""
    env = dict(os.environ, QDKP_C64_UPDATE='tcgen05')
    r = subprocess.run([sys.executable, '-m', 'pytest', '-q', '-x', '-m', 'gpu', '-p', 'no:cacheprovider',
                        'tests/test_blockops_gpu.py::test_block_update',
                        'tests/test_engine_gpu.py', 'tests/test_fig4_gpu.py::test_served_mixed_passes_the_counting_rule'],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
