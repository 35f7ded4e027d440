"""Why the 48x48x36 (h = 0.5 nm) and 128x128x96 (h = 0.375 nm) pyramid workloads do not converge.

The finite-difference bulk symbol of the discretised eight-band operator along [100] is read off
the oracle CSR (the restatement of kp_pryor.confined_hamiltonian pinned to the reference's own
H @ X): a plane wave exp(i k x) u_j, constant in y and z, applied on an (n, 3, 3) grid of uniform
GaAs gives H_FD(k) u_j at the central site. With the materials.py parameters the eight-band
modified Luttinger parameters of GaAs are negative (gamma2 = -0.88, gamma3 = -0.01), and the top
valence-derived pair of the FD spectrum rises through the gap at the zone edge k = pi/h:

    h = 1.0 nm: 0.28 eV     h = 0.5 nm: 1.37 eV     h = 0.375 nm: 2.51 eV

so at h = 0.5 nm the GaAs barrier has grid-scale states at the conduction target sigma_e
(1.008 eV) and at the valence target sigma_h of the 48x48x36 pyramid, and at h = 0.375 nm across
the whole 1.519 eV gap: folded LOBPCG around either sigma sits in a dense spurious continuum.
With Pryor's Table I parameters at h = 1.0 nm (the Fig-4 sweep, where the reference converges)
the same band tops out at 0.009 eV, below every sigma_h of that sweep.
"""
import numpy as np
import pytest

from oracle import kp_operator as ko
from qd3dsolver_b200 import workloads as wl


def _params(table, name):
    m = wl.material(name) if table == 'materials' else dict(wl.PRYOR_TABLE_I[name])
    g1, g2, g3 = wl.modified_luttinger(m)
    return dict(g1=g1, g2=g2, g3=g3, Ep=m['Ep'], Eg=m['Eg'], dso=m['delta_so'])


def fd_bands_100(p, h, nk=49, n=12):
    """Eigenvalues (nk, 8) of the FD bulk symbol H_FD(k) for k in [0, pi/h] along [100]."""
    shape = (n, 3, 3)
    N = n * 9
    one = np.ones(shape)
    f = dict(gamma1=p['g1'] * one, gamma2=p['g2'] * one, gamma3=p['g3'] * one,
             P0=np.sqrt(p['Ep'] * wl.G) * one, Ec=p['Eg'] * one, Ev=0.0 * one,
             delta_so=p['dso'] * one, b=0.0 * one, d=0.0 * one)
    H = ko.confined_hamiltonian(shape, h, f, 8, strain=False)
    site = int(np.ravel_multi_index((n // 2, 1, 1), shape))
    ks = np.linspace(0.0, np.pi / h, nk)
    out = []
    for k in ks:
        ph = np.exp(1j * k * np.arange(n) * h)
        wave = np.repeat(ph, 9)                      # constant over (y, z); x slowest
        V = np.zeros((8 * N, 8), dtype=complex)
        for j in range(8):
            V[j * N:(j + 1) * N, j] = wave
        Y = H @ V
        Hk = np.array([[Y[i * N + site, j] for j in range(8)] for i in range(8)]) / ph[n // 2]
        assert np.abs(Hk - Hk.conj().T).max() < 1e-10
        out.append(np.linalg.eigvalsh(Hk))
    return ks, np.array(out)


def test_fd_symbol_at_k0_is_the_band_edges():
    """At k = 0 the symbol is the bulk band-edge matrix: SO pair at -Delta, HH/LH at 0, CB at Eg."""
    for table in ('materials', 'pryor'):
        p = _params(table, 'GaAs')
        _, E = fd_bands_100(p, 0.5, nk=2)
        np.testing.assert_allclose(E[0], [-p['dso']] * 2 + [0.0] * 4 + [p['Eg']] * 2, atol=1e-12)


@pytest.mark.parametrize('h, top', [(1.0, 0.282), (0.5, 1.369), (0.375, 2.513)])
def test_materials_gaas_spurious_band_rises_through_the_gap(h, top):
    p = _params('materials', 'GaAs')
    assert p['g2'] < -0.8 and p['g3'] < 0.0
    ks, E = fd_bands_100(p, h)
    spur = E[:, 5]                                    # top valence-derived pair (ascending order)
    assert abs(spur.max() - top) < 2e-3
    assert np.argmax(spur) == len(ks) - 1            # at the zone edge k = pi/h
    assert E[:, 6].min() == pytest.approx(p['Eg'], abs=1e-9)   # the CB itself stays above Eg


def test_spurious_band_covers_the_solve_targets_of_the_pyramid_workloads():
    """h = 0.5: above sigma_e and sigma_h of the 48x48x36 pyramid; h = 0.375: above the whole
    GaAs gap, hence above any sigma of the 128x128x96 pyramid."""
    p = _params('materials', 'GaAs')
    w = wl.config1()
    top_05 = fd_bands_100(p, 0.5)[1][:, 5].max()
    assert top_05 > w.sigma['cb'] > w.sigma['vb']
    assert w.sigma['cb'] == pytest.approx(1.00784, abs=2e-4)
    top_0375 = fd_bands_100(p, 0.375)[1][:, 5].max()
    assert top_0375 > p['Eg']


def test_pryor_table_gaas_stays_below_the_fig4_hole_targets():
    p = _params('pryor', 'GaAs')
    top = fd_bands_100(p, 1.0)[1][:, 5].max()
    assert top < 0.01
    # sigma_h of the Fig-4 sweep is ~0.41-0.45 eV (e.g. 0.428 eV at b = 10 nm)
    assert top < 0.4
