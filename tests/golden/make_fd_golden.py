"""Golden fixtures for the inhomogeneous FD elasticity solve (elasticity_fd.solve_strain_fd).

Runs the reference's own solve_strain_fd on small periodic grids (a sphere, an ellipsoidal lens
and a box; InAs in GaAs with the constants pryor_fig4 uses, and one case with the dot softer in
shear) and records the elastic strain fields, the CG iteration count, the relative residual and
the preconditioner's dropped modes. The Fig-4 environments' FD strain (fig4_b*_fields.npz) came
from the same function with pryor_fig4's EPS_STAR, C_DOT and C_MAT, which are recorded here too.

Writes fd_strain_cases.npz and fd_strain_cases.json next to this file.
Usage: python tests/golden/make_fd_golden.py --reference DIR
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def masks():
    out = {}
    x, y, z = np.meshgrid(np.arange(12), np.arange(10), np.arange(9), indexing='ij')
    out['sphere_12x10x9'] = ((x - 5.5) ** 2 + (y - 4.5) ** 2 + (z - 4.0) ** 2) <= 3.2 ** 2
    x, y, z = np.meshgrid(np.arange(16), np.arange(16), np.arange(12), indexing='ij')
    out['lens_16x16x12'] = (((x - 7.5) / 5.5) ** 2 + ((y - 7.5) / 5.5) ** 2 + ((z - 4.0) / 2.5) ** 2) <= 1.0
    m = np.zeros((9, 11, 7), dtype=bool)
    m[3:6, 2:8, 2:5] = True
    out['box_9x11x7'] = m
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help="the reference's source directory")
    args = ap.parse_args()
    sys.path.insert(0, os.path.abspath(args.reference))
    import elasticity_fd as ef
    import pryor_fig4 as f4

    cases = []
    arrays = {}
    soft = (f4.C_DOT[0], f4.C_DOT[1], 0.6 * f4.C_DOT[2])
    specs = [('sphere_12x10x9', 1.0, f4.C_DOT), ('lens_16x16x12', 0.5, f4.C_DOT),
             ('box_9x11x7', 0.75, f4.C_DOT), ('sphere_12x10x9', 0.6, soft)]
    mk = masks()
    for i, (name, h, cdot) in enumerate(specs):
        mask = mk[name]
        st = ef.solve_strain_fd(mask, f4.EPS_STAR, cdot, f4.C_MAT, h, tol=1e-10)
        tag = f'c{i}'
        arrays[f'{tag}_mask'] = mask
        for k in STRAIN:
            arrays[f'{tag}_{k}'] = np.asarray(getattr(st, k), dtype=float)
        cases.append(dict(tag=tag, mask=name, shape=list(mask.shape), h=h, eps_star=f4.EPS_STAR,
                          C_dot=list(cdot), C_matrix=list(f4.C_MAT), tol=1e-10,
                          iterations=int(st.cg_iterations), residual=float(st.cg_residual),
                          converged=bool(st.cg_converged), modes_dropped=int(st.cg_modes_dropped)))
        print(tag, name, h, st.cg_iterations, st.cg_residual, st.cg_modes_dropped, flush=True)
    np.savez_compressed(os.path.join(HERE, 'fd_strain_cases.npz'), **arrays)
    with open(os.path.join(HERE, 'fd_strain_cases.json'), 'w') as fh:
        json.dump(dict(cases=cases, fig4=dict(eps_star=f4.EPS_STAR, C_dot=list(f4.C_DOT),
                                              C_matrix=list(f4.C_MAT), h=1.0, tol=1e-10)),
                  fh, indent=1)


if __name__ == '__main__':
    main()
