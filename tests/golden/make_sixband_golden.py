"""Golden fixture for the six-band hole route (heterostructure.six_band_holes,
heterostructure.py:800-894), run where the reference is mounted.

Environment: an InAs lens (radius 5 nm, height 3 nm, qdsolver_core.lens_mask) in GaAs on a
20x20x14 grid at h = 1.0 nm, materials.py parameters, homogeneous Fourier strain with the matrix
elastic constants, materials.band_edge_fields. The reference's six_band_holes (eigsh 'LA' on the
six-band operator, band-edge filter at valence_edge_top, localisation) is run for k = 4 and 8.
Writes sixband_fields.npz and sixband.json next to this file.
Usage: python tests/golden/make_sixband_golden.py --reference DIR
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help='directory of the qd3Dsolver sources')
    sys.path.insert(0, os.path.abspath(ap.parse_args().reference))
    import qdsolver_core as qd, strain_fourier as sf, materials as mt, heterostructure as hs
    h = 1.0
    cx = qd.centered_axis(20, h)
    cz = (np.arange(14) - 4 + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    mask = qd.lens_mask(X, Y, Z, 5.0, 3.0)
    dot, mat = mt.kp_params(mt.MATERIALS['InAs']), mt.kp_params(mt.MATERIALS['GaAs'])
    st = sf.solve_strain(mask, mt.misfit(dot, mat), mat['C11'], mat['C12'], mat['C44'], h)
    Ec, Ev = mt.band_edge_fields(mask, st.trace, dot, mat)
    env = dict(mask=mask, h=h, dot=dot, matrix=mat, Ev=Ev, Ec=Ec, strain=st)
    out = dict(grid=list(mask.shape), h=h, dot='InAs', matrix='GaAs', z_offset_cells=4,
               lens=dict(radius=5.0, height=3.0), top=hs.valence_edge_top(env))
    for k in (4, 8):
        r = hs.six_band_holes(env, k=k, tol=1e-10, verbose=False)
        out[f'k{k}'] = dict(E=np.asarray(r['E']).tolist(), loc=np.asarray(r['loc']).tolist(),
                            n_spurious=int(r['n_spurious']))
    arrays = dict(mask=mask, Ev=Ev, Ec=Ec, **{k: np.asarray(getattr(st, k)) for k in STRAIN})
    np.savez_compressed(os.path.join(HERE, 'sixband_fields.npz'), **arrays)
    with open(os.path.join(HERE, 'sixband.json'), 'w') as fh:
        json.dump(out, fh, indent=1)


if __name__ == '__main__':
    main()
