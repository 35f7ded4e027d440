"""Golden fixture for the host input producers (run where the reference is mounted).

The benchmark and the batched workloads build their coefficient fields with
qd3dsolver_b200.workloads, a restatement of the reference's host layers. This script records what
the reference itself computes for small grids, so that a CPU test can pin the restatement:

  materials      materials.MATERIALS / kp_params / alloy('InGaSb', x) / alloy('InAsSb', x),
                 misfit (materials.py:258-332, 513-553); pryor1998.PRYOR_TABLE_I (53-84)
  geometry       qdsolver_core.centered_axis, pyramid_mask, lens_mask, spherical_cap_mask
  strain         strain_fourier.solve_strain (176-235), matrix elastic constants
  piezo          piezoelectric.potential (86-99)
  band edges     materials.band_edge_fields (556-586, zero='matrix_vb')
  fields         kp_pryor.material_fields (564-593), n_bands = 8 and 6
  sigma          kp_pryor.local_band_edges (469-531) 'v1' and hole_sigma (156-191)

Cases: an InAs pyramid in GaAs (16x16x12, h = 0.5 nm) and an In(0.45)Ga(0.55)Sb lens in InAs
(14x14x10, h = 0.6 nm), each with the piezo potential folded into both band edges.
Writes inputs_cases.npz and inputs_cases.json next to this file.
Usage: python tests/golden/make_inputs_golden.py --reference DIR
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')
MAT_KEYS = ('delta_so', 'Ep', 'gamma1L', 'gamma2L', 'gamma3L', 'VBO', 'a_c', 'a_v', 'b', 'd',
            'C11', 'C12', 'C44', 'e14', 'eps_R', 'Eg', 'a0')


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help='directory of the qd3Dsolver sources')
    sys.path.insert(0, os.path.abspath(ap.parse_args().reference))
    import qdsolver_core as qd, kp_pryor as kp, strain_fourier as sf, piezoelectric as pz
    import materials as mt, pryor1998 as pr

    meta = {'materials': {}, 'pryor': {}, 'cases': {}}
    for name in ('GaAs', 'InAs', 'GaSb', 'InSb'):
        m = mt.kp_params(mt.MATERIALS[name])
        meta['materials'][name] = {k: float(m[k]) for k in MAT_KEYS}
    for sysname, x in (('InGaSb', 0.45), ('InAsSb', 0.3), ('InGaSb', 1.0)):
        m = mt.alloy(sysname, x)
        meta['materials'][f'{sysname}({x})'] = {k: float(m[k]) for k in MAT_KEYS}
    for name, m in pr.PRYOR_TABLE_I.items():
        meta['pryor'][name] = {k: float(v) for k, v in m.items() if isinstance(v, (int, float))}

    arrays = {}
    cases = (('pyr', 'InAs', 'GaAs', (16, 16, 12), 0.5),
             ('lens', ('InGaSb', 0.45), 'InAs', (14, 14, 10), 0.6))
    for tag, dot_name, mat_name, shape, h in cases:
        dot = mt.kp_params(mt.alloy(*dot_name) if isinstance(dot_name, tuple)
                           else mt.MATERIALS[dot_name])
        mat = mt.kp_params(mt.MATERIALS[mat_name])
        cx = qd.centered_axis(shape[0], h)
        cz = (np.arange(shape[2]) - 3 + 0.5) * h
        X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
        if tag == 'pyr':
            mask = qd.pyramid_mask(X, Y, Z, 4.0, z_base=0.0)
        else:
            mask = qd.lens_mask(X, Y, Z, 2.6, 1.4, z_base=0.0)
        eps = mt.misfit(dot, mat)
        st = sf.solve_strain(mask, eps, mat['C11'], mat['C12'], mat['C44'], h)
        e14 = np.where(mask, dot['e14'], mat['e14'])
        phi = pz.potential(st, e14, mat['eps_R'], h)
        Ec, Ev = mt.band_edge_fields(mask, st.trace, dot, mat)
        Ec, Ev = Ec - phi, Ev - phi
        f8 = kp.material_fields(mask, dot, mat, Ev, Ec, n_bands=8)
        f6 = kp.material_fields(mask, dot, mat, Ev, Ec, n_bands=6)
        b = np.where(mask, dot['b'], mat['b'])
        d = np.where(mask, dot['d'], mat['d'])
        dso = np.where(mask, dot['delta_so'], mat['delta_so'])
        v1 = kp.local_band_edges(st, Ev, Ec, dso, 0.0, 0.0, b, d, hydrostatic_applied=True)['v1']
        sig_h = kp.hole_sigma(Ev, st, b, d, dso, inside_mask=mask)
        arrays[f'{tag}_mask'] = mask
        for k in STRAIN:
            arrays[f'{tag}_{k}'] = np.asarray(getattr(st, k), dtype=float)
        arrays[f'{tag}_phi'] = phi
        arrays[f'{tag}_Ec'] = Ec
        arrays[f'{tag}_Ev'] = Ev
        arrays[f'{tag}_v1'] = v1
        for k in ('gamma1', 'gamma2', 'gamma3', 'P0', 'delta_so', 'b', 'd', 'a_c', 'a_v'):
            arrays[f'{tag}_f8_{k}'] = np.asarray(f8[k], dtype=float)
        for k in ('gamma1', 'gamma2', 'gamma3'):
            arrays[f'{tag}_f6_{k}'] = np.asarray(f6[k], dtype=float)
        meta['cases'][tag] = dict(dot=dot_name, matrix=mat_name, shape=list(shape), h=h,
                                  misfit=float(eps), sigma_h=float(sig_h),
                                  sigma_e=float(Ec[mask].min()), z_offset_cells=3)
    np.savez_compressed(os.path.join(HERE, 'inputs_cases.npz'), **arrays)
    with open(os.path.join(HERE, 'inputs_cases.json'), 'w') as fh:
        json.dump(meta, fh, indent=1)


if __name__ == '__main__':
    main()
