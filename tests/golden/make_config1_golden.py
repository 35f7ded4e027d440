"""Golden fixture on the 48x48x36 InAs/GaAs pyramid operator: the reference's own first LOBPCG
iterations, for an iterate-by-iterate check of the GPU solver at this size.

The folded solve on this grid does not converge in either implementation (the GaAs barrier's
finite-difference spectrum has a spurious band through sigma at h = 0.5 nm with the materials.py
parameters; tests/test_spurious_band.py pins it), so the fixture records a truncated run: the
reference builds the operator and calls scipy's lobpcg exactly as eigensolvers.solve_interior
does (eigensolvers.py:340-353: block 12, X0 from default_rng(0), folded operator, largest=False)
with maxiter = ITERATIONS, and the residual-norm history and the Ritz values are saved for both
bands. Also saved: the structural facts a user of the workload checks (sigma_e, sigma_h, nnz,
per-field sums of the coefficient fields, used to confirm that the host input producers of the
benchmark build the same fields).

Workload (48x48x36 at h = 0.5 nm, 24x24x18 nm GaAs box):
  * x/y from qdsolver_core.centered_axis(48, 0.5); z at cell centres (k - 12 + 0.5) * h, i.e.
    6 nm of GaAs below the wetting layer.
  * 0.5 nm InAs wetting slab (0 <= z < 0.5, one grid plane) plus a {101} pyramid of base 10 nm,
    height 5 nm standing on it (z_base = 0.5).
  * materials.py (0 K) InAs in GaAs, strain_fourier.solve_strain with the GaAs elastic constants,
    materials.band_edge_fields(zero='matrix_vb'), no piezoelectric potential.
  * sigma_e = Ec[mask].min(), sigma_h = kp_pryor.hole_sigma(...) (pryor_fig4.py:135-138).

Writes config1_iterates.json next to this file.
Usage: python tests/golden/make_config1_golden.py --reference DIR [--iterations 6]
"""
import argparse
import json
import os
import sys
import time
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIELD_KEYS = ('gamma1', 'gamma2', 'gamma3', 'P0', 'Ec', 'Ev', 'delta_so', 'b', 'd')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def build(qd, kp, kpc, sf, mt):
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
    ap.add_argument('--reference', required=True, help='directory of the qd3Dsolver sources')
    ap.add_argument('--iterations', type=int, default=6)
    a = ap.parse_args()
    sys.path.insert(0, os.path.abspath(a.reference))
    import qdsolver_core as qd, kp_pryor as kp, kp_confined as kpc
    import strain_fourier as sf, materials as mt, eigensolvers as eig
    import scipy.sparse.linalg as spla

    t0 = time.time()
    H, mask, f, st, sig_e, sig_h = build(qd, kp, kpc, sf, mt)
    t_build = time.time() - t0
    sums = {k: float(np.sum(f[k])) for k in FIELD_KEYS}
    sums.update({k: float(np.sum(getattr(st, k))) for k in STRAIN})
    out = dict(shape=[48, 48, 36], h=0.5, nnz=int(H.nnz), n=int(H.shape[0]), sigma_e=sig_e,
               sigma_h=sig_h, mask_cells=int(mask.sum()), field_sums=sums, block=12, seed=0,
               iterations=a.iterations, build_seconds=t_build)
    n, block = H.shape[0], 12
    for band, sigma in (('cb', sig_e), ('vb', sig_h)):
        rng = np.random.default_rng(0)                      # eigensolvers.py:344-347
        X0 = rng.standard_normal((n, block)) + 1j * rng.standard_normal((n, block))
        F = eig.folded_operator(H, sigma)
        t0 = time.time()
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            lam, _, hist = spla.lobpcg(F, X0, largest=False, tol=1e-7, maxiter=a.iterations,
                                       retResidualNormsHistory=True)
        dt = time.time() - t0
        out[band] = dict(sigma=sigma, mu=np.real(np.asarray(lam)).tolist(),
                         residual_history=np.abs(np.asarray(hist)).tolist(), seconds=dt,
                         seconds_per_iteration=dt / (a.iterations + 1))
        print(band, f"{dt:.1f}s", flush=True)
    out['cpu_count'] = os.cpu_count()
    out['openblas_threads'] = os.environ.get('OPENBLAS_NUM_THREADS')
    with open(os.path.join(HERE, 'config1_iterates.json'), 'w') as fh:
        json.dump(out, fh, indent=1)


if __name__ == '__main__':
    main()
