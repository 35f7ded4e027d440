"""Oracle (test infrastructure): gauge-invariant post-processing of eigenvectors.

localization   pryor_fig4.py:179-193 -- fraction of sum_bands |psi|^2 inside the dot mask.
kramers_levels pryor_fig4.py:222-236 -- pair the sorted spectrum, report the worst
               within-pair splitting.
"""
import numpy as np


def localization(V, mask, n_bands=8):
    V = np.asarray(V)
    n = mask.size
    rho = (np.abs(V.reshape(n_bands, n, -1)) ** 2).sum(axis=0)
    return rho[mask.ravel()].sum(axis=0) / rho.sum(axis=0)


def kramers_levels(E, loc):
    E = np.asarray(E)
    n = len(E) // 2 * 2
    pairs = E[:n].reshape(-1, 2)
    worst = float(np.abs(np.diff(pairs, axis=1)).max()) if n else 0.0
    return pairs.mean(axis=1), np.asarray(loc)[:n].reshape(-1, 2).mean(axis=1), worst


def pair_densities(V, n_sites, n_bands=8):
    """Sum over bands and over each Kramers pair of |psi|^2 -- invariant under the U(2) gauge
    freedom within a degenerate pair, so it is what GPU and oracle vectors are compared by."""
    V = np.asarray(V)
    k = V.shape[1] // 2 * 2
    rho = (np.abs(V[:, :k].reshape(n_bands, n_sites, k)) ** 2).sum(axis=0)
    return rho.reshape(n_sites, k // 2, 2).sum(axis=2)
