"""Drop-in for qd3Dsolver's six-band hole route on the GPU (heterostructure.py:800-952).

  valence_edge_top(env, reduce='max', erode=0, report=False)
      the k = 0 top of the local valence band inside the island (the per-site valence levels come
      from the device kernel behind kp_pryor.local_band_edges)
  six_band_holes(env, k=8, tol=1e-8, maxiter=20000, verbose=True)
      hole states from the six-band (valence-only) operator: the largest algebraic eigenvalues,
      found as the lowest of -H by the device LOBPCG (the reference uses eigsh 'LA'), with the
      reference's margin of extra states, its filter of states above the island's valence top,
      and the device localisation of each state.

`env` carries the reference's keys: mask, h, dot, matrix (material parameter dicts with the
materials.py keys), Ev, Ec (band-edge fields) and strain (a StrainTensor-like object or a dict of
the six components). Returns the reference's dict (E descending, V, inside, loc, top, n_bands,
n_spurious, seconds) with V a host array.
"""
import time

import numpy as np

from . import eigensolvers as eg, kp_pryor as kp, post, workloads as wl


def _pick(env, key):
    m = env['mask']
    return np.where(m, env['dot'][key], env['matrix'][key])


def valence_edge_top(env, reduce='max', erode=0, report=False):
    if reduce not in ('max', 'mean'):
        raise ValueError(f"reduce must be 'max' or 'mean', got {reduce!r}")
    m = np.asarray(env['mask'], dtype=bool)
    sel = m
    if erode:
        from scipy.ndimage import binary_erosion
        eroded = binary_erosion(m, iterations=int(erode))
        if eroded.any():
            sel = eroded
    edges = kp.local_band_edges(env['strain'], env['Ev'], np.zeros_like(np.asarray(env['Ev'])),
                                _pick(env, 'delta_so'), 0.0, 0.0, _pick(env, 'b'),
                                _pick(env, 'd'), hydrostatic_applied=True)
    v1 = edges['v1']
    top = float(v1[sel].max() if reduce == 'max' else v1[sel].mean())
    if not report:
        return top
    return dict(top=top, top_max=float(v1[sel].max()), top_mean=float(v1[sel].mean()),
                top_raw_max=float(v1[m].max()), interior_std=float(v1[sel].std()),
                n_interior=int(sel.sum()), n_mask=int(m.sum()), reduce=reduce)


def six_band_holes(env, k=8, tol=1e-8, maxiter=20000, verbose=True):
    m, h = np.asarray(env['mask'], dtype=bool), env['h']
    fields = wl.material_fields(m, env['dot'], env['matrix'], env['Ev'], env['Ec'], n_bands=6)
    H = kp.confined_hamiltonian(kp.GridOperators(m.shape, h), fields, n_bands=6,
                                strain=env['strain'])
    try:
        nb = H.shape[0] // m.size
        top = valence_edge_top(env)
        t0 = time.time()
        n_solve = min(max(2 * k, k + 8), H.shape[0] - 2)
        E, V, info = eg.solve_lowest_hole(H, k=n_solve, tol=tol, maxiter=maxiter, verbose=False,
                                          return_device=True)
        order = np.argsort(-E)
        E = E[order]
        V = V[:, list(order)].contiguous()
        inside = post.state_summary(H, V, m)['loc']
        keep = E <= top + 1e-6
        n_spurious = int((~keep).sum())
        idx = np.flatnonzero(keep)[:k]
        E, inside = E[idx], inside[idx]
        V = V[:, list(idx)].cpu().numpy()
        if verbose:
            print(f"  six-band vb (B200): {H.shape[0]:,} unknowns, {time.time() - t0:.1f}s, "
                  f"island valence top = {top:.4f} eV")
            if n_spurious:
                print(f"    discarded {n_spurious} eigenvalue(s) above the band edge "
                      f"(interface artifacts); check convergence in h")
            for j, (e, f) in enumerate(zip(E, inside)):
                print(f"    h{j}: E = {e:+.4f} eV, confinement {(top - e) * 1e3:6.1f} meV, "
                      f"{f * 100:5.1f}% inside the dot")
        return dict(E=E, V=V, inside=inside, loc=inside, top=top, n_bands=nb,
                    n_spurious=n_spurious, seconds=time.time() - t0,
                    status=info.get('status'), iterations=info.get('iterations'))
    finally:
        H.close()
