"""Generate the small golden fixtures from the reference itself (run where it is mounted).

operator_cases.npz -- for several grids (including 1-cell and 2-cell extents) and every flag of
    kp_pryor.confined_hamiltonian (n_bands 8/6/4, hole_convention, strain on/off,
    include_hydrostatic, interband_strain), the 15 coefficient fields (+ a_c, a_v), a seeded
    complex block X and Y = H @ X computed with the reference's CSR, plus its nnz.
solve_cases.npz / solve_cases.json -- a small InAs/GaAs pyramid (16x16x12 at h = 1.0 nm) solved
    by the reference's eigensolvers.solve_interior (cb and vb, k = 4) and solve_lowest on the
    4-band hole operator (hole_convention=True, k = 4): eigenvalues, residuals, iterations.

Usage: python tests/golden/make_golden.py --reference DIR
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIELD_KEYS = ('gamma1', 'gamma2', 'gamma3', 'P0', 'Ec', 'Ev', 'delta_so', 'b', 'd',
              'exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx', 'a_c', 'a_v')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def physical_fields(shape, h, rng, ref):
    """A random dot (40% fill) with reference strain and band edges; returns a function giving
    the reference's material fields for a band count (P0 = 0 where the model has none)."""
    kp, sf, mt = ref['kp'], ref['sf'], ref['mt']
    mask = rng.random(shape) < 0.4
    dot, mat = mt.kp_params(mt.MATERIALS['InAs']), mt.kp_params(mt.MATERIALS['GaAs'])
    st = sf.solve_strain(mask, mt.misfit(dot, mat), mat['C11'], mat['C12'], mat['C44'], h)
    Ec, Ev = mt.band_edge_fields(mask, st.trace, dot, mat)

    def fields(nb):
        f = kp.material_fields(mask, dot, mat, Ev, Ec, nb)
        f.setdefault('P0', np.zeros(shape))
        for k in STRAIN:
            f[k] = getattr(st, k)
        return f
    return fields, st


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help='directory of the qd3Dsolver sources')
    sys.path.insert(0, os.path.abspath(ap.parse_args().reference))
    import qdsolver_core as qd, kp_pryor as kp, kp_confined as kpc
    import strain_fourier as sf, materials as mt, eigensolvers as eig
    ref = dict(qd=qd, kp=kp, sf=sf, mt=mt)
    rng = np.random.default_rng(20261203)

    cases = {}
    shapes = [(5, 6, 7), (2, 2, 2), (1, 3, 4), (4, 1, 3), (3, 4, 1), (9, 7, 8)]
    flags = [  # n_bands, hole_convention, strain, include_hydrostatic, interband_strain
        (8, False, True, False, True), (8, False, False, False, True),
        (8, False, True, False, False), (8, False, True, True, True),
        (6, False, True, False, True), (6, True, True, False, True),
        (4, False, True, False, True), (4, True, False, False, True)]
    idx = 0
    for shape in shapes:
        h = float(rng.choice([0.375, 0.5, 1.0]))
        fields, st = physical_fields(shape, h, rng, ref)
        for (nb, hc, use_strain, ih, ib) in flags:
            if shape == (9, 7, 8) and nb != 8:
                continue
            fb = fields(nb)
            H = kp.confined_hamiltonian(kpc.GridOperators(shape, h), fb, nb, hole_convention=hc,
                                        strain=st if use_strain else None,
                                        include_hydrostatic=ih, interband_strain=ib)
            n = H.shape[0]
            m = 3
            X = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
            Y = H @ X
            key = f"c{idx:02d}"
            cases[key + '_meta'] = np.array([shape[0], shape[1], shape[2], nb, int(hc),
                                             int(use_strain), int(ih), int(ib), H.nnz])
            cases[key + '_h'] = np.array(h)
            for k in FIELD_KEYS:
                cases[key + '_' + k] = np.asarray(fb[k], dtype=float)
            cases[key + '_X'] = X
            cases[key + '_Y'] = Y
            idx += 1
    np.savez_compressed(os.path.join(HERE, 'operator_cases.npz'), **cases)
    print('operator cases', idx)

    # ---- small solves -------------------------------------------------------------------
    h = 1.0
    cx = qd.centered_axis(16, h)
    cz = (np.arange(12) - 4 + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    dot, mat = mt.kp_params(mt.MATERIALS['InAs']), mt.kp_params(mt.MATERIALS['GaAs'])
    mask = qd.pyramid_mask(X, Y, Z, 8.0)
    st = sf.solve_strain(mask, mt.misfit(dot, mat), mat['C11'], mat['C12'], mat['C44'], h)
    Ec, Ev = mt.band_edge_fields(mask, st.trace, dot, mat)
    f8 = kp.material_fields(mask, dot, mat, Ev, Ec, 8)
    f4 = kp.material_fields(mask, dot, mat, Ev, Ec, 4)
    H8 = kp.confined_hamiltonian(kpc.GridOperators(mask.shape, h), f8, 8, strain=st)
    H4 = kp.confined_hamiltonian(kpc.GridOperators(mask.shape, h), f4, 4, strain=st,
                                 hole_convention=True)
    sig_e = float(Ec[mask].min())
    sig_h = float(kp.hole_sigma(Ev, st, np.where(mask, dot['b'], mat['b']),
                                np.where(mask, dot['d'], mat['d']),
                                np.where(mask, dot['delta_so'], mat['delta_so']),
                                inside_mask=mask))
    out = {}
    arrays = dict(mask=mask, h=np.array(h))
    for k in FIELD_KEYS:
        arrays['f8_' + k] = np.asarray(f8[k] if k in f8 else getattr(st, k), dtype=float)
        arrays['f4_' + k] = np.asarray(f4[k] if k in f4
                                       else (getattr(st, k) if k in STRAIN else 0.0 * Ec),
                                       dtype=float)
    for band, sig in (('cb', sig_e), ('vb', sig_h)):
        E, V, info = eig.solve_interior(H8, k=4, sigma=sig, tol=1e-9, maxiter=4000,
                                        verbose=False)
        out['interior_' + band] = dict(sigma=sig, k=4, tol=1e-9, maxiter=4000, E=E.tolist(),
                                       residuals=info['residuals'].tolist(),
                                       iterations=int(info['iterations']))
    E, V, info = eig.solve_lowest(H4, k=4, tol=1e-9, maxiter=4000, verbose=False)
    out['lowest_4band_hole'] = dict(k=4, tol=1e-9, maxiter=4000, E=E.tolist(),
                                    residuals=info['residuals'].tolist(),
                                    iterations=int(info['iterations']),
                                    gap_to_next=float(info['gap_to_next']))
    out['shape'] = list(mask.shape)
    out['nnz8'] = int(H8.nnz)
    np.savez_compressed(os.path.join(HERE, 'solve_cases.npz'), **arrays)
    with open(os.path.join(HERE, 'solve_cases.json'), 'w') as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps({k: v for k, v in out.items() if isinstance(v, dict)}, indent=1)[:2000])


if __name__ == '__main__':
    main()
