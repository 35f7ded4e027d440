"""Build libqdkp.so (sm_100a) in-tree with nvcc.

    python -m qd3dsolver_b200.build [--verbose-ptxas]

Compiles every .cu file of qd3dsolver_b200/csrc into qd3dsolver_b200/libqdkp.so. Objects go to
qd3dsolver_b200/_build/ and are reused while their source and headers are unchanged; objects of
superseded sources are removed after a successful link.
"""
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
BUILD = os.path.join(PKG, '_build')
LIB = os.path.join(PKG, 'libqdkp.so')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
         '-I', os.path.join(ROOT, 'include')]


def _headers_digest():
    h = hashlib.sha1()
    for d in (CSRC, os.path.join(ROOT, 'include')):
        for f in sorted(os.listdir(d)):
            if f.endswith(('.cuh', '.h')):
                with open(os.path.join(d, f), 'rb') as fh:
                    h.update(fh.read())
    return h.hexdigest()[:12]


def build(verbose_ptxas=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_digest()
    objs, jobs = [], []
    for f in sorted(os.listdir(CSRC)):
        if not f.endswith('.cu'):
            continue
        src = os.path.join(CSRC, f)
        with open(src, 'rb') as fh:
            dig = hashlib.sha1(fh.read() + hdr.encode() + ' '.join(FLAGS).encode()).hexdigest()[:16]
        obj = os.path.join(BUILD, f"{f[:-3]}-{dig}.o")
        objs.append(obj)
        if os.path.exists(obj) and not force and not verbose_ptxas:
            continue
        cmd = [NVCC] + ARCH + FLAGS + ['-c', src, '-o', obj]
        if verbose_ptxas:
            cmd += ['-Xptxas', '-v']
        jobs.append((f, cmd))

    def compile_one(job):
        return job[0], subprocess.run(job[1], capture_output=True, text=True)

    # one nvcc per source file, in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f, r in ex.map(compile_one, jobs):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {f}:\n{r.stdout}\n{r.stderr}")
            if verbose_ptxas:
                sys.stderr.write(f"== {f}\n" + r.stderr)
    tmp = LIB + '.tmp'
    cmd = [NVCC] + ARCH + ['-shared', '-o', tmp] + objs + ['-lcudart', '-lcufft']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    # objects of earlier sources or headers are never reused: keep only this build's
    keep = {os.path.basename(o) for o in objs}
    for f in os.listdir(BUILD):
        if f.endswith('.o') and f not in keep:
            os.remove(os.path.join(BUILD, f))
    return LIB


if __name__ == '__main__':
    print(build(verbose_ptxas='--verbose-ptxas' in sys.argv, force='--force' in sys.argv))
