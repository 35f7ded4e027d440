"""Host-side input producers for the eight-band eigensolve: materials, dot geometry, strain,
piezoelectric potential and the per-site coefficient fields the device operator consumes.

In qd3Dsolver these are the L1/L2 host layers (qdsolver_core.py, materials.py,
strain_fourier.py, piezoelectric.py, kp_pryor.material_fields / hole_sigma). They stay on the
CPU here as well; this module restates the parts the seeded synthetic workloads need so that the
same inputs can be produced where the reference is not installed:

  materials at 0 K         materials.py:150-175 (_LATTICE, _VARSHNI, _FIXED), set_temperature
                           materials.py:277-303, alloy materials.py:306-332
  geometry                 qdsolver_core.centered_axis 149-162, pyramid_mask 359-369,
                           spherical_cap_mask 209-229, lens_mask 200-206, dash_mask 288-325,
                           island_grid 238-272
  homogeneous strain       strain_fourier.solve_strain 176-235 (one FFT, cubic Christoffel
                           inverse, elastic = total - eigenstrain)
  piezo potential          piezoelectric.polarization/charge_density/potential 59-99
  band edges               materials.band_edge_fields 556-586, misfit 518
  coefficient fields       kp_pryor.material_fields 564-593, modified_luttinger 194-206,
                           kane_P0 209-213
  valence-edge sigma       kp_pryor.local_band_edges 469-531 / hole_sigma 156-191

Deviation, stated where it is used: qd3Dsolver's materials table has no In(x)Ga(1-x)As alloy
(materials.py:209-222). `alloy('InGaAs', x)` interpolates linearly (Vegard, zero bowing) between
InAs and GaAs, which is what the batched-dot workload asks for.
"""
import numpy as np

G = 0.0380998                                   # eV nm^2, qdsolver_core.py:19
E_CHARGE = 1.602176634e-19                      # C, poisson_solver.py:25
EPS0 = 8.8541878128e-12                         # F/m, poisson_solver.py:26
POISSON_CONST = E_CHARGE * 1e9 / EPS0           # V nm, poisson_solver.py:30
CHARGE_UNIT = 1.0 / (E_CHARGE * 1e18)           # piezoelectric.py:50

FIELD_KEYS = ('gamma1', 'gamma2', 'gamma3', 'P0', 'Ec', 'Ev', 'delta_so', 'b', 'd',
              'exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')
STRAIN_KEYS = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')

# --------------------------------------------------------------------------------------------
# Materials at T = 0 K (Vurgaftman, Meyer & Ram-Mohan 2001 values as tabulated by qd3Dsolver)
# --------------------------------------------------------------------------------------------

_A300 = {'GaAs': (5.65325, 3.88e-5), 'InAs': (6.05830, 2.74e-5),
         'GaSb': (6.09590, 4.72e-5), 'InSb': (6.47940, 3.48e-5)}
_EG0 = {'GaAs': 1.519, 'InAs': 0.417, 'GaSb': 0.812, 'InSb': 0.235}
_TABLE = {
    #        delta_so Ep    g1L   g2L   g3L   VBO    a_c    a_v    b     d     C11     C12    C44    e14    eps_R
    'GaAs': (0.341, 28.8, 6.98, 2.06, 2.93, -0.80, -7.17, -1.16, -2.0, -4.8, 122.10, 56.60, 60.00, -0.160, 12.9),
    'InAs': (0.390, 21.5, 20.0, 8.50, 9.20, -0.59, -5.08, -1.00, -1.8, -3.6, 83.29, 45.26, 39.59, -0.045, 15.15),
    'GaSb': (0.760, 27.0, 13.4, 4.70, 6.00, -0.03, -7.50, -0.80, -2.0, -4.7, 88.42, 40.26, 43.22, -0.130, 15.7),
    'InSb': (0.810, 23.3, 34.8, 15.5, 16.5, 0.00, -6.94, -0.36, -2.0, -4.7, 68.47, 37.35, 31.11, -0.070, 16.8),
}
_KEYS = ('delta_so', 'Ep', 'gamma1L', 'gamma2L', 'gamma3L', 'VBO', 'a_c', 'a_v', 'b', 'd',
         'C11', 'C12', 'C44', 'e14', 'eps_R')
_ALLOYS = {
    # name: (x = 1 parent, x = 0 parent, bowing)
    'InGaSb': ('InSb', 'GaSb', {'Eg': 0.415, 'delta_so': 0.10}),
    'InAsSb': ('InSb', 'InAs', {'Eg': 0.67, 'delta_so': 1.20}),
    'InGaAs': ('InAs', 'GaAs', {}),                   # Vegard: deviation, see module docstring
}


def material(name):
    """Parameters of one binary at 0 K: a0 = a(300 K) - 300 da/dT, Eg = Varshni Eg(0)."""
    a300, dadT = _A300[name]
    m = dict(zip(_KEYS, _TABLE[name]))
    m.update(name=name, a0=a300 + dadT * (0.0 - 300.0), Eg=_EG0[name])
    return m


def alloy(system, x):
    """P(x) = x P_A + (1-x) P_B - C x (1-x) over every tabulated key (materials.py:306-332)."""
    if not 0.0 <= x <= 1.0:
        raise ValueError(f"composition x must be in [0, 1], got {x}")
    pa, pb, bow = _ALLOYS[system]
    A, B = material(pa), material(pb)
    out = {k: x * A[k] + (1 - x) * B[k] - bow.get(k, 0.0) * x * (1 - x)
           for k in _KEYS + ('Eg', 'a0')}
    out.update(name=f"{system}({x:.3f})", system=system, x=x)
    return out


def misfit(dot, matrix):
    return (matrix['a0'] - dot['a0']) / dot['a0']


# --------------------------------------------------------------------------------------------
# Geometry
# --------------------------------------------------------------------------------------------

def centered_axis(n, h):
    return (np.arange(n) - (n - 1) / 2.0) * h


def pyramid_mask(X, Y, Z, base, z_base=0.0):
    zz = Z - z_base
    half = base / 2.0
    return (zz >= 0.0) & (np.abs(X) < half - zz) & (np.abs(Y) < half - zz)


def spherical_cap_mask(X, Y, Z, base_radius, height, z_base=0.0):
    R = (base_radius ** 2 + height ** 2) / (2.0 * height)
    zz = Z - z_base
    return (zz >= 0.0) & (X ** 2 + Y ** 2 + (zz - (height - R)) ** 2 <= R ** 2)


def lens_mask(X, Y, Z, base_radius, height, z_base=0.0):
    zz = Z - z_base
    return (zz >= 0.0) & ((X ** 2 + Y ** 2) / base_radius ** 2 + (zz / height) ** 2 < 1.0)


def dash_mask(X, Y, Z, length, width, height, contact_angle_deg=54.7356, z_base=0.0):
    tan_t = np.tan(np.deg2rad(contact_angle_deg))
    if width > length or height > (width / 2.0) * tan_t:
        raise ValueError("dash: need length >= width and a non-negative top facet")
    zz = Z - z_base
    inset = zz / tan_t
    return ((zz >= 0.0) & (zz <= height) & (np.abs(X) <= length / 2.0 - inset)
            & (np.abs(Y) <= width / 2.0 - inset))


# --------------------------------------------------------------------------------------------
# Strain (homogeneous anisotropic elasticity by one FFT) and piezoelectric potential
# --------------------------------------------------------------------------------------------

def _kgrid(shape, h):
    ks = [2 * np.pi * np.fft.fftfreq(n, d=h) for n in shape]
    return np.meshgrid(*ks, indexing='ij')


def solve_strain(mask, eps_star, C11, C12, C44, h):
    """Elastic strain of an inclusion with dilatational eigenstrain -eps_star in a cubic matrix.

    u_k = -i eps_T (C11 + 2 C12) chi_k K(k)^-1 k with K_ik = C_ijkl k_j k_l (cubic), the k = 0
    mode dropped; strain = symmetric gradient of u; elastic = total - eps_T chi on the diagonal.
    Returns a dict of the six tensor components (tensor shear convention).
    """
    chi = np.ascontiguousarray(mask, dtype=float)
    eps_T = -float(eps_star)
    chi_k = np.fft.fftn(chi)
    KX, KY, KZ = _kgrid(chi.shape, h)
    cs = C12 + C44
    k11 = C11 * KX * KX + C44 * (KY * KY + KZ * KZ)
    k22 = C11 * KY * KY + C44 * (KX * KX + KZ * KZ)
    k33 = C11 * KZ * KZ + C44 * (KX * KX + KY * KY)
    k12, k13, k23 = cs * KX * KY, cs * KX * KZ, cs * KY * KZ
    c11 = k22 * k33 - k23 * k23
    c12 = k13 * k23 - k12 * k33
    c13 = k12 * k23 - k13 * k22
    c22 = k11 * k33 - k13 * k13
    c23 = k12 * k13 - k11 * k23
    c33 = k11 * k22 - k12 * k12
    det = k11 * c11 + k12 * c12 + k13 * c13
    inv = np.zeros_like(det)
    np.divide(1.0, det, out=inv, where=det != 0.0)
    i11, i12, i13, i22, i23, i33 = (c * inv for c in (c11, c12, c13, c22, c23, c33))
    pref = -1j * eps_T * (C11 + 2 * C12) * chi_k
    ux = pref * (i11 * KX + i12 * KY + i13 * KZ)
    uy = pref * (i12 * KX + i22 * KY + i23 * KZ)
    uz = pref * (i13 * KX + i23 * KY + i33 * KZ)

    def back(a):
        return np.fft.ifftn(a).real

    off = eps_T * chi
    return dict(exx=back(1j * KX * ux) - off, eyy=back(1j * KY * uy) - off,
                ezz=back(1j * KZ * uz) - off,
                exy=back(0.5j * (KY * ux + KX * uy)), eyz=back(0.5j * (KZ * uy + KY * uz)),
                ezx=back(0.5j * (KX * uz + KZ * ux)))


def piezo_potential(strain, e14, eps_r, h, sign=1.0):
    """First-order zincblende piezo potential (V): P = 2 e14 (eyz, ezx, exy), rho = -div P,
    spectral Poisson eps_r k^2 phi = rho * POISSON_CONST with k = 0 dropped."""
    P = (2.0 * e14 * strain['eyz'] * sign, 2.0 * e14 * strain['ezx'] * sign,
         2.0 * e14 * strain['exy'] * sign)
    KX, KY, KZ = _kgrid(P[0].shape, h)
    div = (1j * KX * np.fft.fftn(P[0]) + 1j * KY * np.fft.fftn(P[1])
           + 1j * KZ * np.fft.fftn(P[2]))
    rho = -np.fft.ifftn(div).real * CHARGE_UNIT
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    inv = np.zeros_like(k2)
    np.divide(1.0, k2, out=inv, where=k2 != 0.0)
    return np.fft.ifftn(np.fft.fftn(rho) * POISSON_CONST * inv / eps_r).real


def band_edge_fields(mask, trace, dot, matrix):
    """(Ec, Ev) with the hydrostatic shift, zero at the unstrained matrix valence edge."""
    ref = matrix['VBO']
    Ev0 = np.where(mask, dot['VBO'] - ref, matrix['VBO'] - ref)
    Ec0 = Ev0 + np.where(mask, dot['Eg'], matrix['Eg'])
    a_c = np.where(mask, dot['a_c'], matrix['a_c'])
    a_v = np.where(mask, dot['a_v'], matrix['a_v'])
    return Ec0 + a_c * trace, Ev0 - a_v * trace


def modified_luttinger(m):
    shift = m['Ep'] / (3 * m['Eg'] + m['delta_so'])
    return m['gamma1L'] - shift, m['gamma2L'] - 0.5 * shift, m['gamma3L'] - 0.5 * shift


def material_fields(mask, dot, matrix, Ev, Ec, n_bands=8):
    """Per-site coefficient fields (kp_pryor.material_fields): modified Luttinger parameters and
    P0 = sqrt(Ep G) for 8 bands, the unmodified gamma^L for 6 / 4 bands."""
    def pick(key):
        return np.where(mask, dot[key], matrix[key])

    if n_bands == 8:
        gd, gm = modified_luttinger(dot), modified_luttinger(matrix)
        g1, g2, g3 = (np.where(mask, a, b) for a, b in zip(gd, gm))
        P0 = np.where(mask, np.sqrt(dot['Ep'] * G), np.sqrt(matrix['Ep'] * G))
    else:
        g1, g2, g3 = pick('gamma1L'), pick('gamma2L'), pick('gamma3L')
        P0 = np.zeros(mask.shape)
    return dict(gamma1=g1, gamma2=g2, gamma3=g3, P0=P0, delta_so=pick('delta_so'),
                Ev=Ev, Ec=Ec, b=pick('b'), d=pick('d'), a_c=pick('a_c'), a_v=pick('a_v'))


def local_valence_edge(Ev, strain, b, d, delta_so):
    """Largest k = 0 eigenvalue of the 6x6 valence block per site (kp_pryor.local_band_edges
    with Ec = 0, a_c = a_v = 0, hydrostatic already applied): the v1 field."""
    sq3, sq2, sq32 = np.sqrt(3.0), np.sqrt(2.0), np.sqrt(1.5)
    q = -(b / 2.0) * (strain['exx'] + strain['eyy'] - 2.0 * strain['ezz'])
    r = (sq3 / 2.0) * b * (strain['exx'] - strain['eyy']) - 1j * d * strain['exy']
    s = -d * (strain['ezx'] - 1j * strain['eyz'])
    P = -np.asarray(Ev, dtype=float)
    shp = np.broadcast_shapes(q.shape, P.shape)
    H = np.zeros(shp + (6, 6), dtype=complex)
    # rows/cols 2..7 of Pryor's table at k = 0 (U = V = 0): upper triangle then adjoint
    up = {(0, 0): -P + q, (0, 1): -np.conj(s), (0, 2): r, (0, 4): sq32 * s, (0, 5): -sq2 * q,
          (1, 1): -P - q, (1, 3): r, (1, 4): -sq2 * r, (1, 5): s / sq2,
          (2, 2): -P - q, (2, 3): np.conj(s), (2, 4): np.conj(s) / sq2, (2, 5): sq2 * np.conj(r),
          (3, 3): -P + q, (3, 4): sq2 * q, (3, 5): sq32 * np.conj(s),
          (4, 4): -P - delta_so, (5, 5): -P - delta_so}
    for (i, j), v in up.items():
        H[..., i, j] = v
        if i != j:
            H[..., j, i] = np.conj(v)
    return np.linalg.eigvalsh(H)[..., 5]


def hole_sigma(Ev, strain, b, d, delta_so, mask, margin=0.0):
    return float(np.max(local_valence_edge(Ev, strain, b, d, delta_so)[mask])) + margin


# --------------------------------------------------------------------------------------------
# Workloads
# --------------------------------------------------------------------------------------------

class Workload:
    """Everything one eigensolve needs on the host: grid, fields, mask, sigma per band."""

    def __init__(self, name, shape, h, fields, mask, sigma_e, sigma_h, k, meta=None):
        self.name, self.shape, self.h = name, tuple(shape), float(h)
        self.fields, self.mask = fields, mask
        self.sigma = {'cb': float(sigma_e), 'vb': float(sigma_h)}
        self.k = int(k)
        self.meta = meta or {}

    @property
    def n_sites(self):
        return int(np.prod(self.shape))

    @property
    def n(self):
        return 8 * self.n_sites


def build_environment(name, mask, h, dot, matrix, piezo=False, k=8, sigma_e_outside=False,
                      meta=None, device=False, strain='fourier'):
    """Strain, band edges, coefficient fields and both sigmas of one dot. device=True runs the
    strain, the piezo potential and the valence-edge sigma on the GPU (qd3dsolver_b200.fields,
    kp_pryor.hole_sigma); the same arithmetic, for batches whose host preparation would
    otherwise take minutes. strain='fd' (device only) is the inhomogeneous FD elasticity with the
    dot's and the matrix's own constants at tol 1e-10, as heterostructure.build computes it
    (heterostructure.py:284-291); 'fourier' the homogeneous solution with the matrix's."""
    if strain not in ('fourier', 'fd'):
        raise ValueError("strain must be 'fourier' or 'fd'")
    if strain == 'fd' and not device:
        raise ValueError("strain='fd' runs on the device only (device=True)")
    if device:
        from . import fields as dfields, kp_pryor as kpd
        if strain == 'fd':
            sd = dfields.solve_strain_fd(mask, misfit(dot, matrix),
                                         (dot['C11'], dot['C12'], dot['C44']),
                                         (matrix['C11'], matrix['C12'], matrix['C44']), h,
                                         tol=1e-10)
        else:
            sd = dfields.solve_strain(mask, misfit(dot, matrix), matrix['C11'], matrix['C12'],
                                      matrix['C44'], h)
        st = sd.as_dict()
    else:
        st = solve_strain(mask, misfit(dot, matrix), matrix['C11'], matrix['C12'], matrix['C44'], h)
    trace = st['exx'] + st['eyy'] + st['ezz']
    Ec, Ev = band_edge_fields(mask, trace, dot, matrix)
    if piezo:
        e14 = np.where(mask, dot['e14'], matrix['e14'])
        phi = (dfields.potential(st, e14, matrix['eps_R'], h) if device
               else piezo_potential(st, e14, matrix['eps_R'], h))
        Ec, Ev = Ec - phi, Ev - phi
    f = material_fields(mask, dot, matrix, Ev, Ec, 8)
    f.update(st)
    sig_e = float(Ec[~mask].min()) if sigma_e_outside else float(Ec[mask].min())
    if device:
        sig_h = kpd.hole_sigma(Ev, st, f['b'], f['d'], f['delta_so'], inside_mask=mask)
    else:
        sig_h = hole_sigma(Ev, st, f['b'], f['d'], f['delta_so'], mask)
    return Workload(name, mask.shape, h, f, mask, sig_e, sig_h, k, meta)


def pyramid_in_box(nxy, nz, h, base, z_below, wetting=0.5, dot='InAs', matrix='GaAs',
                   piezo=False, k=8, name='pyramid'):
    """Square {101} pyramid on a wetting slab: x/y from centered_axis, z at cell centres with
    the slab bottom `z_below` nm above the box floor; slab [0, wetting), pyramid base at z =
    wetting."""
    cx = centered_axis(nxy, h)
    kz0 = int(round(z_below / h))
    cz = (np.arange(nz) - kz0 + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    mask = pyramid_mask(X, Y, Z, base, z_base=wetting) | ((Z >= 0) & (Z < wetting))
    dm = dot if isinstance(dot, dict) else material(dot)
    mm = matrix if isinstance(matrix, dict) else material(matrix)
    return build_environment(name, mask, h, dm, mm, piezo=piezo, k=k,
                             meta=dict(base=base, wetting=wetting, piezo=piezo))


def config1():
    """48x48x36 at h = 0.5 nm: InAs {101} pyramid (base 10, height 5 nm) on a 0.5 nm InAs
    wetting slab in a 24x24x18 nm GaAs box, Fourier strain, no piezo, 4 Kramers pairs/band."""
    return pyramid_in_box(48, 36, 0.5, 10.0, 6.0, name='pyramid48x48x36_h0.5', k=8)


def config2():
    """128x128x96 at h = 0.375 nm: the same pyramid scaled to base 18 / height 9 nm in a
    48x48x36 nm box, with the first-order piezoelectric potential, 8 Kramers pairs/band.
    The 0.5 nm wetting slab is not a multiple of h; on cell-centred z it covers 1 plane."""
    return pyramid_in_box(128, 96, 0.375, 18.0, 12.0, piezo=True, k=16,
                          name='pyramid128x128x96_h0.375')


def random_dot(rng, h=0.5, n_min=32, n_max=96, pairs=(2, 8), family='InGaAs/GaAs', device=False):
    """One seeded dot of the batched-dot family: In(x)Ga(1-x)As (x ~ U[0.6, 1]) pyramid or
    spherical cap in GaAs, base 6-20 nm, aspect 0.2-0.5, 2-8 Kramers pairs."""
    x = rng.uniform(0.6, 1.0)
    shape_kind = 'pyramid' if rng.random() < 0.5 else 'cap'
    base = rng.uniform(6.0, 20.0)
    aspect = rng.uniform(0.2, 0.5)
    npairs = int(rng.integers(pairs[0], pairs[1] + 1))
    height = base * (0.5 if shape_kind == 'pyramid' else aspect)
    pad = max(3.0, 0.35 * base)
    nxy = int(np.clip(round((base + 2 * pad) / h), n_min, n_max)) // 2 * 2
    nz = int(np.clip(round((height + 2 * pad) / h), n_min, int(n_max * 0.75))) // 2 * 2
    cx = centered_axis(nxy, h)
    kz0 = int(round(min(pad, nz * h / 2 - height / 2) / h))
    cz = (np.arange(nz) - kz0 + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    if shape_kind == 'pyramid':
        mask = pyramid_mask(X, Y, Z, base)
    else:
        mask = spherical_cap_mask(X, Y, Z, base / 2.0, height)
    dot = alloy('InGaAs', x)
    return build_environment(f"{shape_kind}_x{x:.2f}_b{base:.1f}_{nxy}x{nxy}x{nz}", mask, h,
                             dot, material('GaAs'), k=2 * npairs,
                             meta=dict(x=x, kind=shape_kind, base=base, height=height),
                             device=device, strain='fd' if device else 'fourier')


def antimonide_request(rng, n_min=32, n_max=128, pairs=(2, 8), device=False):
    """One request of the antimonide serving stream: an InSb or In(x)Ga(1-x)Sb
    (x ~ U[0.3, 1.0]) lens or dash in InAs, radius 3-15 nm, h ~ U[0.4, 0.6] nm, grid 32^3 to
    128^3, 2-8 Kramers pairs, the conduction or the valence band with sigma as
    heterostructure.eight_band_states sets it (heterostructure.py:978-985: the matrix minimum
    of Ec for cb, the exact valence top inside the dot for vb), first-order piezo potential.

    Choices the stream leaves open, fixed here: half the dots are InSb and half the alloy; a
    lens has height / radius ~ U[0.3, 0.6]; a dash has length 2 r, width ~ U[0.5, 1] x length
    and the height of a lens of the same radius, capped by its facets. Strain: with device=True
    the inhomogeneous FD elasticity, as the reference's heterostructure.build computes it; on the
    host the homogeneous Fourier solution with the matrix's elastic constants.
    Returns (Workload, band)."""
    insb = rng.random() < 0.5
    x = 1.0 if insb else rng.uniform(0.3, 1.0)
    kind = 'lens' if rng.random() < 0.5 else 'dash'
    r = rng.uniform(3.0, 15.0)
    h = rng.uniform(0.4, 0.6)
    hgt = r * rng.uniform(0.3, 0.6)
    npairs = int(rng.integers(pairs[0], pairs[1] + 1))
    band = 'cb' if rng.random() < 0.5 else 'vb'
    pad = max(3.0, 0.5 * r)
    n_xy = int(np.clip(round((2 * r + 2 * pad) / h), n_min, n_max)) // 2 * 2
    n_z = int(np.clip(round((hgt + 2 * pad) / h), n_min, n_max)) // 2 * 2
    cx = centered_axis(n_xy, h)
    kz0 = int(round(min(pad, n_z * h / 2 - hgt / 2) / h))
    cz = (np.arange(n_z) - kz0 + 0.5) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    if kind == 'lens':
        mask = lens_mask(X, Y, Z, r, hgt)
    else:
        length = 2 * r
        width = length * rng.uniform(0.5, 1.0)
        cap = (width / 2.0) * np.tan(np.deg2rad(54.7356))
        mask = dash_mask(X, Y, Z, length, width, min(hgt, 0.95 * cap))
    dot = alloy('InGaSb', x)
    w = build_environment(f"{kind}_{'InSb' if insb else f'InGaSb{x:.2f}'}_r{r:.1f}_h{h:.2f}_"
                          f"{n_xy}x{n_xy}x{n_z}", mask, h, dot, material('InAs'), piezo=True,
                          k=2 * npairs, sigma_e_outside=True,
                          meta=dict(x=x, kind=kind, radius=r, height=hgt, band=band),
                          device=device, strain='fd' if device else 'fourier')
    return w, band


# --------------------------------------------------------------------------------------------
# Pryor (1998) InAs/GaAs benchmark: the reference's Fig-4 sweep (pryor_fig4.py)
# --------------------------------------------------------------------------------------------

#: Pryor's Table I (pryor1998.py:53-84): Luttinger, gap, spin-orbit, Ep, deformation
#: potentials (Pryor's a_v sign), piezo e14, eps_R, elastic constants, lattice constant and the
#: unstrained valence offset.
PRYOR_TABLE_I = {
    'InAs': dict(gamma1L=19.67, gamma2L=8.37, gamma3L=9.29, Eg=0.418, delta_so=0.38, Ep=22.2,
                 a_c=-6.66, a_v=0.66, b=-1.8, d=-3.6, e14=0.045, eps_R=15.15,
                 C11=83.29, C12=45.26, C44=39.59, a0=6.0583, E_vbo=0.085),
    'GaAs': dict(gamma1L=6.85, gamma2L=2.1, gamma3L=2.9, Eg=1.519, delta_so=0.33, Ep=25.7,
                 a_c=-9.3, a_v=0.7, b=-2.0, d=-5.4, e14=0.159, eps_R=15.15,
                 C11=121.1, C12=54.8, C44=60.4, a0=5.6532, E_vbo=0.0),
}
#: Island base widths of the Fig-4 sweep (pryor_fig4.py:71).
FIG4_SIZES = (6.0, 8.0, 10.0, 12.0, 14.0, 16.0, 18.0)


def fig4_grid(base, h=1.0, pad=8.0):
    """pryor_fig4.clean_grid: odd, mirror-symmetric x/y axis, island base on a grid plane."""
    nx = int(round(2 * (base / 2 + pad) / h)) // 2 * 2 + 1
    kz0 = int(round(pad / h))
    nz = kz0 + int(round((base / 2 + pad) / h)) + 1
    cx = centered_axis(nx, h)
    cz = (np.arange(nz) - kz0) * h
    X, Y, Z = np.meshgrid(cx, cx, cz, indexing='ij')
    return pyramid_mask(X, Y, Z, base)


def fig4_environment(base, h=1.0, pad=8.0, piezo=True, strain='fourier'):
    """Pryor's b-nm pyramid (Table I parameters, first-order piezo potential applied as
    U = -phi to both edges, sigma_e = Ec[dot].min(), sigma_h = exact valence edge), as
    pryor_fig4.environment builds it (pryor_fig4.py:109-153).

    strain='fd': the inhomogeneous FD elasticity with the dot's and the matrix's constants at
    tol 1e-10, as the reference computes it (pryor_fig4.py:115), on the device
    (fields.solve_strain_fd). strain='fourier' (host): the homogeneous Fourier solution with
    GaAs elastic constants (strain_fourier.solve_strain), a stated deviation.
    """
    dot, mat = PRYOR_TABLE_I['InAs'], PRYOR_TABLE_I['GaAs']
    pyr = fig4_grid(base, h, pad)
    eps_star = (mat['a0'] - dot['a0']) / dot['a0']
    if strain == 'fd':
        from . import fields as dfields
        st = dfields.solve_strain_fd(pyr, eps_star, (dot['C11'], dot['C12'], dot['C44']),
                                     (mat['C11'], mat['C12'], mat['C44']), h,
                                     tol=1e-10).as_dict()
    elif strain == 'fourier':
        st = solve_strain(pyr, eps_star, mat['C11'], mat['C12'], mat['C44'], h)
    else:
        raise ValueError("strain must be 'fourier' or 'fd'")
    trace = st['exx'] + st['eyy'] + st['ezz']
    Ev0 = np.where(pyr, dot['E_vbo'], mat['E_vbo'])
    Ec0 = Ev0 + np.where(pyr, dot['Eg'], mat['Eg'])
    a_c = np.where(pyr, dot['a_c'], mat['a_c'])
    a_v = np.where(pyr, dot['a_v'], mat['a_v'])
    Ec, Ev = Ec0 + a_c * trace, Ev0 - a_v * trace
    if piezo:
        phi = piezo_potential(st, np.where(pyr, dot['e14'], mat['e14']), mat['eps_R'], h)
        Ec, Ev = Ec - phi, Ev - phi
    f = material_fields(pyr, dot, mat, Ev, Ec, 8)
    f.update(st)
    sig_e = float(Ec[pyr].min())
    sig_h = hole_sigma(Ev, st, f['b'], f['d'], f['delta_so'], pyr)
    return Workload(f"fig4_b{base:g}_h{h:g}", pyr.shape, h, f, pyr, sig_e, sig_h, 8,
                    meta=dict(base=base, pad=pad, piezo=piezo))


def fig4_from_fixture(path):
    """Workload from a saved field fixture (reference-built fields, e.g. FD strain)."""
    z = np.load(path)
    mask = z['mask']
    f = {k: z[k] for k in FIELD_KEYS}
    return Workload(f"fixture:{path.rsplit('/', 1)[-1]}", mask.shape, float(z['h']), f, mask,
                    float(z['sigma_e']), float(z['sigma_h']), 8)
