"""CPU restatement of qd3Dsolver's inhomogeneous FD elasticity (elasticity_fd.py) -- TEST
INFRASTRUCTURE ONLY (the checker of the device solve; nothing in the product imports it).

The reference minimises the discretised strain energy of trilinear (Q1) hexahedral elements with
2x2x2 Gauss quadrature on a periodic grid (elasticity_fd.py:1-73): displacements on nodes,
materials and strain on elements, element i spanning nodes i + c for the eight corners c. Its
solve is preconditioned CG on the stiffness system with the exact inverse of the volume-averaged
homogeneous operator applied in Fourier space (elasticity_fd.py:211-271, 366-419), and the strain
is the trilinear gradient at the element centres (elasticity_fd.py:343-362).

This restatement applies the operator as a 27-point stencil per node whose 3x3 coefficient
blocks are sums of the element stiffness blocks of the eight elements around the node
(an equivalent regrouping of elasticity_fd.py:243-267), and uses real FFTs for the
preconditioner (the symbol is Hermitian in k, so the result is the real part the reference
takes). Parity: tests/golden/make_fd_golden.py records the reference's own solves.
"""
import itertools

import numpy as np

CORNERS = np.array(list(itertools.product([0, 1], repeat=3)))          # (8, 3)
SIGNS = 2.0 * CORNERS - 1.0
GAUSS = np.array(list(itertools.product([-1.0, 1.0], repeat=3))) / np.sqrt(3.0)
OFFSETS = np.array(list(itertools.product([-1, 0, 1], repeat=3)))       # (27, 3)


def shape_gradients(h, xi):
    """dN_n / dx_d at local points xi (npts, 3) of the cube [-1, 1]^3 with side h: shape
    (npts, 8, 3), N_n = prod_d (1 + s_nd xi_d) / 2 (elasticity_fd.py:90-106)."""
    xi = np.atleast_2d(xi)
    f = 0.5 * (1.0 + SIGNS[None] * xi[:, None, :])                     # (npts, 8, 3)
    g = np.empty(f.shape)
    for d in range(3):
        o = [e for e in range(3) if e != d]
        g[:, :, d] = 0.5 * SIGNS[None, :, d] * f[:, :, o[0]] * f[:, :, o[1]]
    return g * (2.0 / h)


def cubic_stiffness(C11, C12, C44):
    """C_ijkl of a cubic crystal (elasticity_fd.py:109-123)."""
    e = np.eye(3)
    C = C12 * e[:, :, None, None] * e[None, None, :, :]
    C = C + C44 * (e[:, None, :, None] * e[None, :, None, :] + e[:, None, None, :] * e[None, :, :, None])
    for i in range(3):
        C[i, i, i, i] += C11 - C12 - 2.0 * C44
    return C


def element_arrays(C11, C12, C44, h):
    """K[a, b, j, l] = sum_g w detJ C_ijkl G[g,a,i] G[g,b,k] and W[a, j] = sum_g w detJ G[g,a,j]
    (elasticity_fd.py:126-153; unit Gauss weights, detJ = (h/2)^3)."""
    G = shape_gradients(h, GAUSS)
    w = (h / 2.0) ** 3
    K = w * np.einsum('ijkl,gai,gbk->abjl', cubic_stiffness(C11, C12, C44), G, G)
    return K, w * G.sum(axis=0)


def roll(a, shift):
    return np.roll(a, shift, axis=(-3, -2, -1))


def apply(U, chi, K_m, K_d):
    """F[p]_j = sum over the elements e = p - c_a around node p of
    sum_{b,l} K_{mat(e)}[a,b,j,l] U_l[e + c_b] (elasticity_fd.py:243-267), grouped by the node
    offset d = c_b - c_a."""
    F = np.zeros_like(U)
    for d in OFFSETS:
        Ud = roll(U, tuple(-d))                                           # U[p + d]
        for a in range(8):
            b = CORNERS[a] + d
            if np.any(b < 0) or np.any(b > 1):
                continue
            bi = int(b[0] * 4 + b[1] * 2 + b[2])
            mat = roll(chi, tuple(CORNERS[a]))                          # chi[p - c_a]
            Km, dK = K_m[a, bi], K_d[a, bi] - K_m[a, bi]
            for j in range(3):
                for l in range(3):
                    if Km[j, l] != 0.0 or dK[j, l] != 0.0:
                        F[j] += (Km[j, l] + dK[j, l] * mat) * Ud[l]
    return F


def symbol_inverse(K, shape):
    """Exact inverse of the homogeneous stencil's symbol S(k)_jl = sum_{a,b} K[a,b,j,l]
    exp(i k.(c_b - c_a)) on the rfft half-spectrum, zero where the block is singular by the
    reference's scale-free test: tr/3 > 1e-12 max(tr/3) and |det| > 1e-9 (tr/3)^3
    (elasticity_fd.py:156-208). Returns (Sinv (nx, ny, nz//2+1, 3, 3), modes dropped on the full
    spectrum)."""
    nx, ny, nz = shape
    kx = 2 * np.pi * np.fft.fftfreq(nx)
    ky = 2 * np.pi * np.fft.fftfreq(ny)
    kz = 2 * np.pi * np.fft.fftfreq(nz)
    KX, KY, KZ = np.meshgrid(kx, ky, kz, indexing='ij')
    S = np.zeros((nx, ny, nz, 3, 3), dtype=complex)
    for a in range(8):
        for b in range(8):
            d = CORNERS[b] - CORNERS[a]
            S += K[a, b][None, None, None] * np.exp(1j * (d[0] * KX + d[1] * KY + d[2] * KZ))[..., None, None]
    tr = np.trace(S, axis1=-2, axis2=-1).real / 3.0
    det = np.abs(np.linalg.det(S))
    good = (tr > 1e-12 * tr.max()) & (det > 1e-9 * np.maximum(tr, 0.0) ** 3)
    inv = np.zeros_like(S)
    inv[good] = np.linalg.inv(S[good])
    return inv[:, :, :nz // 2 + 1], int(good.size - good.sum())


def precondition(R, Sinv):
    nz = R.shape[-1]
    Rk = np.fft.rfftn(R, axes=(-3, -2, -1))
    Uk = np.einsum('...jl,l...->j...', Sinv, Rk)
    return np.fft.irfftn(Uk, s=R.shape[-3:], axes=(-3, -2, -1))


def pcg(F, Aop, Minv, tol, maxiter):
    """Preconditioned CG with the mean of each component projected out (elasticity_fd.py:366-419).
    Returns (U, iterations, relative residual, breakdown reason or None)."""
    def project(V):
        return V - V.mean(axis=(-3, -2, -1), keepdims=True)
    F = project(F)
    U = np.zeros_like(F)
    R = F.copy()
    Z = Minv(R)
    P = Z.copy()
    rz = float(np.vdot(R, Z).real)
    fn = float(np.linalg.norm(F))
    if fn == 0.0:
        return U, 0, 0.0, None
    if rz <= 0.0:
        return project(U), 0, 1.0, 'preconditioner not positive definite'
    rel, why, it = 1.0, None, 0
    for it in range(1, maxiter + 1):
        AP = Aop(P)
        pap = float(np.vdot(P, AP).real)
        if pap <= 0:
            why = 'non-positive curvature'
            break
        alpha = rz / pap
        U += alpha * P
        R -= alpha * AP
        rel = float(np.linalg.norm(R)) / fn
        if rel < tol:
            break
        Z = Minv(R)
        rzn = float(np.vdot(R, Z).real)
        if rzn <= 0.0:
            why = 'preconditioner lost positive definiteness'
            break
        P = Z + (rzn / rz) * P
        rz = rzn
    return project(U), it, rel, why


def solve_strain_fd(mask, eps_star, C_dot, C_matrix, h, tol=1e-10, maxiter=2000):
    """Elastic strain (exx, eyy, ezz, exy, eyz, ezx) of an inclusion with its own elastic
    constants, plus (iterations, relative residual, converged, modes dropped)
    (elasticity_fd.py:275-363)."""
    chi = np.asarray(mask, dtype=float)
    eps_T = -float(eps_star)
    K_d, W_d = element_arrays(*C_dot, h)
    K_m, _ = element_arrays(*C_matrix, h)
    Sinv, dropped = symbol_inverse(K_m + chi.mean() * (K_d - K_m), chi.shape)
    bulk = eps_T * (C_dot[0] + 2.0 * C_dot[1]) * chi
    F = np.zeros((3,) + chi.shape)
    for a in range(8):
        for j in range(3):
            F[j] += W_d[a, j] * roll(bulk, tuple(CORNERS[a]))
    U, it, rel, why = pcg(F, lambda V: apply(V, chi, K_m, K_d), lambda R: precondition(R, Sinv),
                          tol, maxiter)
    G0 = shape_gradients(h, np.zeros(3))[0]
    grad = np.zeros((3, 3) + chi.shape)
    for n in range(8):
        Un = roll(U, tuple(-CORNERS[n]))
        for i in range(3):
            grad[i] += G0[n, i] * Un
    off = eps_T * chi
    strain = dict(exx=grad[0, 0] - off, eyy=grad[1, 1] - off, ezz=grad[2, 2] - off,
                  exy=0.5 * (grad[0, 1] + grad[1, 0]), eyz=0.5 * (grad[1, 2] + grad[2, 1]),
                  ezx=0.5 * (grad[2, 0] + grad[0, 2]))
    converged = rel < tol and why is None and dropped <= 1
    return strain, dict(iterations=it, residual=rel, converged=converged, modes_dropped=dropped)
