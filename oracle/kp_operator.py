"""Oracle (test infrastructure): the discretised Pryor eight-band k.p operator as a SciPy CSR.

A CPU restatement of what qd3Dsolver builds in `kp_pryor.confined_hamiltonian`
(kp_pryor.py:363-466) on top of the central-difference machinery of `kp_confined`
(kp_confined.py:58-183, GridOperators 398-454, scheme 'central', hard walls). It is the checker
for the CUDA H.X kernel, never part of the product path.

Operator summary (h = grid spacing, G = hbar^2/2m0 = 0.0380998 eV nm^2, qdsolver_core.py:19):
  D_a        Hermitian central difference -i/(2h)(x[p+a] - x[p-a]), truncated at the walls
             (kp_confined.py:58-85).
  k2_a(al)   three-point face-averaged second derivative; off-diagonal -(al_p+al_q)/(2h^2),
             diagonal = sum of the face terms plus al_p/h^2 for each box face p touches
             (the "ghost wall", kp_confined.py:88-143).
  cross(al,a,b) = (D_a diag(al) D_b + D_b diag(al) D_a)/2 (kp_confined.py:146-183).
  symf(f, D) = (diag(f) D + D diag(f))/2 (kp_pryor.py:434-446).
  A = Ec + G sum_a k2_a(1); P = -Ev + G sum_a k2_a(g1); Q = G(k2x+k2y-2k2z)(g2) + Q_eps;
  R = G(-sqrt3 (k2x-k2y)(g2) + 2i sqrt3 cross(g3,x,y)) + R_eps;
  S = 2 sqrt3 G (cross(g3,z,x) - i cross(g3,z,y)) + S_eps   (kp_pryor.py:410-424);
  U = symf(P0, Dz)/sqrt3 - u_s, V = (symf(P0,Dx) - i symf(P0,Dy))/sqrt6 - v_s
  (kp_pryor.py:430-454); Bir-Pikus shear terms kp_pryor.py:111-113.
  The 8x8 upper triangle is Pryor's table (kp_pryor.py:244-301), completed by the adjoint
  (kp_pryor.py:216-241); n_bands = 6 / 4 take rows/cols 2..7 / 2..5 (kp_pryor.py:70) and
  hole_convention negates those sub-models (kp_pryor.py:239-240, 464).

Vectors are band-major: index = band * N + site, site in C order (x slowest, z fastest).
"""
import numpy as np
import scipy.sparse as sp

G = 0.0380998                       # eV nm^2, qdsolver_core.py:19
SQ2, SQ3, SQ32, SQ6 = np.sqrt(2.0), np.sqrt(3.0), np.sqrt(1.5), np.sqrt(6.0)
BAND_RANGE = {8: (0, 8), 6: (2, 8), 4: (2, 6)}          # kp_pryor.py:70
FIELD_KEYS = ('gamma1', 'gamma2', 'gamma3', 'P0', 'Ec', 'Ev', 'delta_so', 'b', 'd',
              'exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def _flat_pairs(shape, axis):
    """Flat indices (here, next) of every pair of neighbours along `axis`."""
    idx = np.arange(int(np.prod(shape))).reshape(shape)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[axis] = slice(0, shape[axis] - 1)
    hi[axis] = slice(1, shape[axis])
    return idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel(), tuple(lo), tuple(hi)


def first_derivative(shape, axis, h):
    """k_axis = -i d/daxis as a Hermitian central difference, hard walls (kp_confined.py:58-85)."""
    n = int(np.prod(shape))
    here, nxt, _, _ = _flat_pairs(shape, axis)
    c = -1j / (2.0 * h)
    rows = np.concatenate([here, nxt])
    cols = np.concatenate([nxt, here])
    vals = np.concatenate([np.full(here.size, c), np.full(here.size, -c)])
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n), dtype=complex)


def second_derivative(alpha, h, axis):
    """d/da(alpha d/da) with face averages and the hard-wall ghost term
    (kp_confined.py:99-142, non-periodic branch)."""
    shape = alpha.shape
    n = alpha.size
    here, nxt, lo, hi = _flat_pairs(shape, axis)
    t = (0.5 * (alpha[lo] + alpha[hi]) / h ** 2).ravel()
    diag = np.zeros(shape)
    diag[lo] += t.reshape(alpha[lo].shape)
    diag[hi] += t.reshape(alpha[hi].shape)
    first = [slice(None)] * 3
    last = [slice(None)] * 3
    first[axis] = 0
    last[axis] = shape[axis] - 1
    diag[tuple(first)] += alpha[tuple(first)] / h ** 2
    diag[tuple(last)] += alpha[tuple(last)] / h ** 2
    rows = np.concatenate([here, nxt, np.arange(n)])
    cols = np.concatenate([nxt, here, np.arange(n)])
    vals = np.concatenate([-t, -t, diag.ravel()])
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n), dtype=complex)


class Grid:
    """Shape, spacing and the three first-derivative operators of one grid."""

    def __init__(self, shape, h):
        self.shape = tuple(int(s) for s in shape)
        self.h = float(h)
        self.D = [first_derivative(self.shape, a, self.h) for a in range(3)]

    def k2(self, alpha, axis):
        return second_derivative(np.asarray(alpha, dtype=float), self.h, axis)

    def cross(self, alpha, a, b):
        Al = sp.diags(np.asarray(alpha, dtype=float).ravel())
        return (self.D[a] @ Al @ self.D[b] + self.D[b] @ Al @ self.D[a]) / 2.0


def _diag(v):
    return sp.diags(np.asarray(v).ravel().astype(complex))


def _symf(f, D):
    F = _diag(f)
    return (F @ D + D @ F) / 2.0


def bir_pikus(e, b, d):
    """(Q_eps, R_eps, S_eps), kp_pryor.py:111-113."""
    q = -(b / 2.0) * (e['exx'] + e['eyy'] - 2.0 * e['ezz'])
    r = (SQ3 / 2.0) * b * (e['exx'] - e['eyy']) - 1j * d * e['exy']
    s = -d * (e['ezx'] - 1j * e['eyz'])
    return q, r, s


def pryor_upper(A, P, Q, R, S, U, V, Dl, adj):
    """Pryor's 8x8 upper triangle (kp_pryor.py:249-300) as {(row, col): operator}.
    Band order CB+, CB-, LH+, HH+, HH-, LH-, SO+, SO- (kp_pryor.py:66)."""
    return {
        (0, 0): A, (0, 2): adj(V), (0, 4): SQ3 * V, (0, 5): -SQ2 * U, (0, 6): -U,
        (0, 7): SQ2 * adj(V),
        (1, 1): A, (1, 2): -SQ2 * U, (1, 3): -SQ3 * adj(V), (1, 5): -V, (1, 6): SQ2 * V,
        (1, 7): U,
        (2, 2): -P + Q, (2, 3): -adj(S), (2, 4): R, (2, 6): SQ32 * S, (2, 7): -SQ2 * Q,
        (3, 3): -P - Q, (3, 5): R, (3, 6): -SQ2 * R, (3, 7): S / SQ2,
        (4, 4): -P - Q, (4, 5): adj(S), (4, 6): adj(S) / SQ2, (4, 7): SQ2 * adj(R),
        (5, 5): -P + Q, (5, 6): SQ2 * Q, (5, 7): SQ32 * adj(S),
        (6, 6): -P - Dl,
        (7, 7): -P - Dl,
    }


def confined_hamiltonian(shape, h, fields, n_bands=8, hole_convention=False, strain=True,
                         include_hydrostatic=False, interband_strain=True):
    """The confined k.p Hamiltonian (eV) as CSR, same matrix as kp_pryor.confined_hamiltonian.

    `fields` maps the keys of FIELD_KEYS (plus a_c, a_v when include_hydrostatic) to arrays of
    `shape`. `strain=False` drops every strain term, as the reference does for strain=None.
    """
    grid = Grid(shape, h)
    n = int(np.prod(grid.shape))
    f = {k: np.asarray(v, dtype=float) for k, v in fields.items()}
    ones = np.ones(grid.shape)

    A = _diag(f['Ec']) + G * (grid.k2(ones, 0) + grid.k2(ones, 1) + grid.k2(ones, 2))
    P = -_diag(f['Ev']) + G * (grid.k2(f['gamma1'], 0) + grid.k2(f['gamma1'], 1)
                               + grid.k2(f['gamma1'], 2))
    Q = G * (grid.k2(f['gamma2'], 0) + grid.k2(f['gamma2'], 1) - 2 * grid.k2(f['gamma2'], 2))
    R = G * (-SQ3 * (grid.k2(f['gamma2'], 0) - grid.k2(f['gamma2'], 1))
             + 2j * SQ3 * grid.cross(f['gamma3'], 0, 1))
    S = 2 * SQ3 * G * (grid.cross(f['gamma3'], 2, 0) - 1j * grid.cross(f['gamma3'], 2, 1))
    Dl = _diag(f['delta_so'])
    if strain:
        q, r, s = bir_pikus(f, f['b'], f['d'])
        Q = Q + _diag(q)
        R = R + _diag(r)
        S = S + _diag(s)
        if include_hydrostatic:
            tr = f['exx'] + f['eyy'] + f['ezz']
            A = A + _diag(f['a_c'] * tr)
            P = P + _diag(f['a_v'] * tr)

    zero = sp.csr_matrix((n, n), dtype=complex)
    if n_bands == 8:
        P0 = f['P0']
        Dx, Dy, Dz = grid.D
        U = _symf(P0, Dz) / SQ3
        V = (_symf(P0, Dx) - 1j * _symf(P0, Dy)) / SQ6
        if strain and interband_strain:
            u = (_symf(P0 * f['ezx'], Dx) + _symf(P0 * f['eyz'], Dy)
                 + _symf(P0 * f['ezz'], Dz)) / SQ3
            v = (_symf(P0 * (f['exx'] - 1j * f['exy']), Dx)
                 + _symf(P0 * (f['exy'] - 1j * f['eyy']), Dy)
                 + _symf(P0 * (f['ezx'] - 1j * f['eyz']), Dz)) / SQ6
            U, V = U - u, V - v
    else:
        U = V = zero

    def adj(M):
        return M.conj().T

    up = pryor_upper(A, P, Q, R, S, U, V, Dl, adj)
    lo_b, hi_b = BAND_RANGE[n_bands]
    m = hi_b - lo_b
    rows = [[None] * m for _ in range(m)]
    for i in range(m):
        for j in range(i, m):
            rows[i][j] = up.get((i + lo_b, j + lo_b), zero)
    for i in range(m):
        for j in range(i):
            rows[i][j] = adj(rows[j][i])
    if hole_convention and n_bands != 8:
        rows = [[-blk for blk in r] for r in rows]
    return sp.bmat(rows, format='csr')


def nnz_estimate(H):
    return int(H.nnz)
