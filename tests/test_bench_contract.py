"""bench.py's reference arm keeps its JSON contract (runs on the host cores; no GPU needed).

The reference arm times the reference's CPU algorithm (scipy LOBPCG on the restated CSR
operator) on a bounded sample of the Fig-4 sweep and prints one JSON line with the same metric,
unit and direction as the GPU arm, plus `impl`, `cpu_baseline` and a zero-copy `e2e` block.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, 'bench.py', '--impl', 'reference', '--steps', '1',
                          '--warmup', '3'], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d['impl'] == 'reference'
    assert d['unit'] == 'eigenpairs/s' and d['higher_is_better'] is True
    assert d['value'] > 0 and d['steps'] == 1 and d['warmup'] >= 3 and d['n_gpus'] == 1
    assert d['metric'].startswith('converged k')
    cb = d['cpu_baseline']
    assert cb['kind'] in ('reference', 'port') and cb['cores'] >= 1 and cb['sample']
    assert cb['value'] == d['value'] and cb['unit'] == d['unit']
    e2e = d['e2e']
    assert e2e['value'] == d['value'] and e2e['unit'] == d['unit']
    assert e2e['h2d_bytes_per_step'] == 0 and e2e['d2h_bytes_per_step'] == 0
    assert 'workload' in d['config']
