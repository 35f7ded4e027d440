"""Run the reference's own eight-band folded LOBPCG on the 48x48x36 InAs/GaAs pyramid workload
and write its eigenvalues, residuals and gauge-invariant state summaries as golden fixtures.

This imports the reference package read-only from REFERENCE_DIR (default /root/reference), so it
only runs where the reference is mounted. It is the generator of `config1_<band>.json`; nothing
on the GPU side reads the reference at run time.

Workload (48x48x36 at h = 0.5 nm, 24x24x18 nm GaAs box):
  * x/y from qdsolver_core.centered_axis(48, 0.5); z at cell centres (k - 12 + 0.5) * h, i.e.
    6 nm of GaAs below the wetting layer.
  * 0.5 nm InAs wetting slab (0 <= z < 0.5, one grid plane) plus a {101} pyramid of base 10 nm,
    height 5 nm standing on it (z_base = 0.5).
  * materials.py (0 K) InAs in GaAs, strain_fourier.solve_strain with the GaAs elastic constants,
    materials.band_edge_fields(zero='matrix_vb'), no piezoelectric potential.
  * sigma_e = Ec[mask].min(), sigma_h = kp_pryor.hole_sigma(...) (pryor_fig4.py:135-138).
  * eigensolvers.solve_interior(H, k=8, sigma, tol=1e-7, maxiter=8000)
    (pryor_fig4.bound_states defaults, pryor_fig4.py:196-205), seed 0.

Usage: python tests/golden/make_config1_oracle.py cb|vb [--save-vectors DIR]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

REFERENCE_DIR = os.environ.get('REFERENCE_DIR', '/root/reference')
HERE = os.path.dirname(os.path.abspath(__file__))


def build(ref):
    qd, kp, kpc, sf, mt = (ref[k] for k in ('qd', 'kp', 'kpc', 'sf', 'mt'))
    h = 0.5
    cx = qd.centered_axis(48, h)
    cz = (np.arange(36) - 12 + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    dot, mat = mt.kp_params(mt.MATERIALS['InAs']), mt.kp_params(mt.MATERIALS['GaAs'])
    mask = qd.pyramid_mask(X, Y, Z, 10.0, z_base=0.5) | ((Z >= 0) & (Z < 0.5))
    st = sf.solve_strain(mask, mt.misfit(dot, mat), mat['C11'], mat['C12'], mat['C44'], h)
    Ec, Ev = mt.band_edge_fields(mask, st.trace, dot, mat)
    ops = kpc.GridOperators(mask.shape, h)
    f = kp.material_fields(mask, dot, mat, Ev, Ec, 8)
    H = kp.confined_hamiltonian(ops, f, 8, strain=st)
    sig_e = float(Ec[mask].min())
    sig_h = kp.hole_sigma(Ev, st, np.where(mask, dot['b'], mat['b']),
                          np.where(mask, dot['d'], mat['d']),
                          np.where(mask, dot['delta_so'], mat['delta_so']), inside_mask=mask)
    return H, mask, f, st, sig_e, float(sig_h)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('band', choices=('cb', 'vb'))
    ap.add_argument('--save-vectors', default=None)
    ap.add_argument('--maxiter', type=int, default=8000)
    ap.add_argument('--tol', type=float, default=1e-7)
    a = ap.parse_args()

    sys.path.insert(0, REFERENCE_DIR)
    import qdsolver_core as qd, kp_pryor as kp, kp_confined as kpc
    import strain_fourier as sf, materials as mt, eigensolvers as eig
    ref = dict(qd=qd, kp=kp, kpc=kpc, sf=sf, mt=mt)

    t0 = time.time()
    H, mask, f, st, sig_e, sig_h = build(ref)
    t_build = time.time() - t0
    sigma = sig_e if a.band == 'cb' else sig_h
    E, V, info = eig.solve_interior(H, k=8, sigma=sigma, tol=a.tol, maxiter=a.maxiter,
                                    verbose=False)
    n = mask.size
    rho = (np.abs(V.reshape(8, n, -1)) ** 2).sum(axis=0)          # (N, k)
    loc = (rho[mask.ravel()].sum(axis=0) / rho.sum(axis=0)).tolist()
    pairs = np.sort(E).reshape(-1, 2)
    out = dict(band=a.band, sigma=sigma, sigma_e=sig_e, sigma_h=sig_h, k=8, block=12,
               tol=a.tol, maxiter=a.maxiter, seed=0,
               E=E.tolist(), residuals=info['residuals'].tolist(),
               iterations=int(info['iterations']), seconds=float(info['time']),
               build_seconds=t_build, converged=bool(info['converged']),
               loc=loc, kramers_split=float(np.abs(np.diff(pairs, axis=1)).max()),
               nnz=int(H.nnz), n=int(H.shape[0]),
               cpu_count=os.cpu_count(),
               openblas_threads=os.environ.get('OPENBLAS_NUM_THREADS'))
    with open(os.path.join(HERE, f'config1_{a.band}.json'), 'w') as fh:
        json.dump(out, fh, indent=1)
    if a.save_vectors:
        os.makedirs(a.save_vectors, exist_ok=True)
        np.save(os.path.join(a.save_vectors, f'config1_{a.band}_V.npy'), V)
    print(json.dumps({k: out[k] for k in ('band', 'E', 'iterations', 'seconds')}))


if __name__ == '__main__':
    main()
