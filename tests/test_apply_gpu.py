"""H.X on the B200 against the reference's own H @ X (golden fixtures) and the oracle CSR."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(c):
    from qd3dsolver_b200 import kp_pryor as kpg
    f = c['fields']
    strain = {k: f[k] for k in ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')} if c['strain'] else None
    return kpg.confined_hamiltonian(kpg.GridOperators(c['shape'], c['h']), f, c['n_bands'],
                                    hole_convention=c['hole'], strain=strain,
                                    include_hydrostatic=c['hydro'],
                                    interband_strain=c['interband'])


def test_apply_c128_matches_reference_fixtures(operator_cases):
    """complex128 H.X equals the reference CSR product to 1e-13 relative, every flag/grid."""
    for c in operator_cases:
        H = _build(c)
        assert H.shape == (c['X'].shape[0],) * 2
        Y = H @ c['X']
        err = np.abs(Y - c['Y']).max() / np.abs(c['Y']).max()
        assert err < 1e-13, (c['name'], c['shape'], c['n_bands'], err)
        y1 = H @ c['X'][:, 1]
        assert np.abs(y1 - c['Y'][:, 1]).max() / np.abs(c['Y']).max() < 1e-13


def test_apply_c64_within_single_precision(operator_cases):
    import torch
    from qd3dsolver_b200 import _lib
    for c in operator_cases[::3]:
        H = _build(c)
        X = torch.from_numpy(c['X'].astype(np.complex64)).cuda()
        Y = H.apply(X).cpu().numpy()
        err = np.abs(Y - c['Y']).max() / np.abs(c['Y']).max()
        assert err < 2e-6, (c['name'], err)


def test_c64_column_layouts(operator_cases):
    """complex64 blocks with even, odd and strided column layouts (the staged kernel copies
    16-byte pairs of columns only when the leading dimension and width are even)."""
    import torch
    rng = np.random.default_rng(5)
    for c in [c for c in operator_cases if c['n_bands'] == 8][:6]:
        H = _build(c)
        n = H.shape[0]
        for m, ld in ((4, 4), (3, 3), (4, 6), (5, 7)):
            X = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
            ref = H @ X
            big = torch.zeros((n, ld), dtype=torch.complex64, device='cuda')
            big[:, :m] = torch.from_numpy(X.astype(np.complex64)).cuda()
            Y = H.apply(big[:, :m]).cpu().numpy()
            err = np.abs(Y - ref).max() / np.abs(ref).max()
            assert err < 2e-6, (c['name'], m, ld, err)


def test_shifted_and_folded_modes(operator_cases):
    import torch
    from qd3dsolver_b200 import _lib
    c = operator_cases[0]
    H = _build(c)
    sigma = 0.731
    X = c['X']
    Xt = torch.from_numpy(X).cuda()
    Ys = H.apply(Xt, sigma=sigma, mode=_lib.APPLY_SHIFTED).cpu().numpy()
    ref = c['Y'] - sigma * X
    assert np.abs(Ys - ref).max() / np.abs(ref).max() < 1e-13
    Yf = H.apply(Xt, sigma=sigma, mode=_lib.APPLY_FOLDED).cpu().numpy()
    ref2 = (H @ ref) - sigma * ref
    assert np.abs(Yf - ref2).max() / np.abs(ref2).max() < 1e-13
    # strided (leading dimension > m) input
    big = torch.zeros((X.shape[0], 5), dtype=torch.complex128, device='cuda')
    big[:, 1:4] = Xt
    Y2 = H.apply(big[:, 1:4]).cpu().numpy()
    assert np.abs(Y2 - c['Y']).max() / np.abs(c['Y']).max() < 1e-13


def test_diagonal_matches_oracle(operator_cases):
    from oracle import kp_operator as ko
    for c in operator_cases[:8]:
        H = _build(c)
        Ho = ko.confined_hamiltonian(c['shape'], c['h'], c['fields'], c['n_bands'],
                                     hole_convention=c['hole'], strain=c['strain'],
                                     include_hydrostatic=c['hydro'],
                                     interband_strain=c['interband'])
        d = H.diagonal()
        do = Ho.diagonal()
        if c['hydro']:
            continue
        assert np.abs(d - do).max() <= 1e-12 * np.abs(do).max()


def test_config1_operator_against_oracle():
    """Full 48x48x36 pyramid operator: device H.X vs the oracle CSR on a seeded block."""
    from qd3dsolver_b200 import workloads as wl, kp_pryor as kpg
    from oracle import kp_operator as ko
    w = wl.config1()
    f = w.fields
    H = kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                 strain={k: f[k] for k in wl.STRAIN_KEYS})
    Ho = ko.confined_hamiltonian(w.shape, w.h, f, 8, strain=True)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((w.n, 4)) + 1j * rng.standard_normal((w.n, 4))
    Y = H @ X
    Yo = Ho @ X
    assert np.abs(Y - Yo).max() / np.abs(Yo).max() < 1e-13
    assert Ho.nnz <= H.nnz <= Ho.nnz * (1 + 1e-4)   # structural count bounds scipy's


def test_every_tile_shape_matches_reference(operator_cases):
    """Each staged tile shape and the direct kernel reproduce the reference H @ X (the
    autotuner may pick any of them)."""
    import torch
    from qd3dsolver_b200 import _lib
    cases = [c for c in operator_cases if c['n_bands'] == 8]
    for c in cases[:10]:
        H = _build(c)
        for tile in list(range(_lib.TILE_COUNT)) + [_lib.TILE_DIRECT]:
            # the TMA shapes are complex64 only; on these small grids they fall back
            H.set_tile(tile if tile < _lib.TILE_TMA0 else _lib.TILE_DIRECT, _lib.C128)
            H.set_tile(tile, _lib.C64)
            Y = H @ c['X']
            err = np.abs(Y - c['Y']).max() / np.abs(c['Y']).max()
            assert err < 1e-13, (c['name'], tile, err)
            X32 = torch.from_numpy(c['X'].astype(np.complex64)).cuda()
            e32 = np.abs(H.apply(X32).cpu().numpy() - c['Y']).max() / np.abs(c['Y']).max()
            assert e32 < 2e-6, (c['name'], tile, e32)


def test_autotuner_keeps_a_valid_choice():
    from qd3dsolver_b200 import _lib, workloads as wl
    import torch
    w = wl.fig4_environment(6.0)
    from qd3dsolver_b200 import kp_pryor as kpg
    f = w.fields
    H = kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                 strain={k: f[k] for k in wl.STRAIN_KEYS})
    secs = H.tune(12, torch.complex128, reps=2)
    assert len(secs) == _lib.TILE_TMA0 + 1 and all(v > 0 for v in secs.values())
    best = min(secs, key=secs.get)
    assert H.get_tile(_lib.C128) == best
    secs = H.tune(12, torch.complex64, reps=2)       # the TMA shapes that fit this grid too
    assert any(t >= _lib.TILE_TMA0 for t in secs) and all(v > 0 for v in secs.values())
    assert H.get_tile(_lib.C64) == min(secs, key=secs.get)
    H.close()


def _fixture_operator(name):
    import os
    from qd3dsolver_b200 import kp_pryor as kpg, workloads as wl
    w = wl.fig4_from_fixture(os.path.join(os.path.dirname(__file__), 'golden', name))
    f = w.fields
    return w, kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                       strain={k: f[k] for k in wl.STRAIN_KEYS})


def test_tma_tiles_match_oracle():
    """The complex64 TMA tile shapes on grids their tensor maps fit (the reference's b = 10 nm
    Fig-4 fields, 27x27x22): against the oracle CSR for plain, shifted and folded modes, column
    counts that fill a CTA's columns exactly or leave a partial chunk, and strided blocks."""
    import torch
    from qd3dsolver_b200 import _lib
    from oracle import kp_operator as ko
    w, H = _fixture_operator('fig4_b10_fields.npz')
    Ho = ko.confined_hamiltonian(w.shape, w.h, w.fields, 8, strain=True)
    n = H.shape[0]
    rng = np.random.default_rng(3)
    Xall = rng.standard_normal((n, 24)) + 1j * rng.standard_normal((n, 24))
    Yall = Ho @ Xall
    sigma = 0.4281
    ran = 0
    for tile in range(_lib.TILE_TMA0, _lib.TILE_COUNT):
        H.set_tile(tile, _lib.C64)
        for m in (4, 6, 12, 24):
            X = torch.from_numpy(Xall[:, :m].astype(np.complex64)).cuda()
            ref = Yall[:, :m]
            Y = H.apply(X).cpu().numpy()
            err = np.abs(Y - ref).max() / np.abs(ref).max()
            assert err < 2e-6, (tile, m, err)
            ran += 1
        X = torch.from_numpy(Xall[:, :12].astype(np.complex64)).cuda()
        refs = Yall[:, :12] - sigma * Xall[:, :12]
        Ys = H.apply(X, sigma=sigma, mode=_lib.APPLY_SHIFTED).cpu().numpy()
        assert np.abs(Ys - refs).max() / np.abs(refs).max() < 2e-6, tile
        reff = Ho @ refs - sigma * refs
        Yf = H.apply(X, sigma=sigma, mode=_lib.APPLY_FOLDED).cpu().numpy()
        assert np.abs(Yf - reff).max() / np.abs(reff).max() < 4e-6, tile
        # a block inside a wider, even leading dimension; and an odd one (falls back)
        for ld in (16, 15):
            big = torch.zeros((n, ld), dtype=torch.complex64, device='cuda')
            big[:, 2:10] = torch.from_numpy(Xall[:, :8].astype(np.complex64)).cuda()
            Y = H.apply(big[:, 2:10]).cpu().numpy()
            assert np.abs(Y - Yall[:, :8]).max() / np.abs(Yall[:, :8]).max() < 2e-6, (tile, ld)
    assert ran >= 12
    fault = __import__('ctypes').c_int(-1)
    assert _lib.lib().qdkp_device_fault(torch.cuda.current_device(), 1, fault) == 0
    assert fault.value == 0
    H.close()


def test_tma_tiles_on_the_48x48x36_operator():
    """Every TMA tile shape on the 48x48x36 pyramid operator (m = 12 and 24) equals the
    complex128 direct kernel (itself pinned to the reference) to single precision."""
    import torch
    from qd3dsolver_b200 import _lib, workloads as wl, kp_pryor as kpg
    w = wl.config1()
    f = w.fields
    H = kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                 strain={k: f[k] for k in wl.STRAIN_KEYS})
    H.set_tile(_lib.TILE_DIRECT, _lib.C128)
    g = torch.Generator(device='cuda').manual_seed(5)
    for m in (12, 24):
        X = torch.randn((H.shape[0], m), dtype=torch.complex128, device='cuda', generator=g)
        ref = H.apply(X)
        X32 = X.to(torch.complex64)
        for tile in range(_lib.TILE_TMA0, _lib.TILE_COUNT):
            H.set_tile(tile, _lib.C64)
            Y = H.apply(X32).to(torch.complex128)
            err = ((Y - ref).abs().max() / ref.abs().max()).item()
            assert err < 2e-6, (tile, m, err)
    H.close()
