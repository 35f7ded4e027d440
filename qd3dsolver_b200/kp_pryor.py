"""Drop-in for qd3Dsolver's `kp_pryor.confined_hamiltonian` backed by the B200 library.

`confined_hamiltonian(ops, fields, n_bands=8, hole_convention=False, strain=None,
include_hydrostatic=False, interband_strain=True)` takes the reference's arguments
(kp_pryor.py:363-364) and returns a `KPOperator`: a scipy `LinearOperator` whose coefficient
fields live on the GPU and whose `@` runs the matrix-free CUDA stencil instead of a CSR product.
It provides everything the reference's callers use on `H` (shape, nnz, dtype, `H @ X` for 1-D
and 2-D arrays, `diagonal()`), plus device-side application on torch tensors for the solvers.
"""
import ctypes

import numpy as np
import scipy.sparse.linalg as spla

from . import _lib
from ._lib import check, lib

G = 0.0380998                      # eV nm^2, qdsolver_core.py:19
FIELD_ORDER = ('gamma1', 'gamma2', 'gamma3', 'P0', 'Ec', 'Ev', 'delta_so', 'b', 'd',
               'exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')
STRAIN_KEYS = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')
BAND_LABELS_8 = ['CB+1/2', 'CB-1/2', 'LH+1/2', 'HH+3/2', 'HH-3/2', 'LH-1/2', 'SO+1/2', 'SO-1/2']
BAND_SLICES = {8: slice(0, 8), 6: slice(2, 8), 4: slice(2, 6)}


class GridOperators:
    """Grid description with the interface of kp_confined.GridOperators (kp_confined.py:
    398-454) that the device operator needs: shape, h, periodic, scheme. No CSR is built."""

    SCHEMES = ('central',)

    def __init__(self, shape, h, periodic=False, scheme='central'):
        if scheme not in self.SCHEMES:
            raise ValueError(f"scheme must be one of {self.SCHEMES}, got {scheme!r}")
        self.shape = tuple(int(s) for s in shape)
        self.h = float(h)
        self.periodic = bool(periodic)
        self.scheme = scheme


def _strain_dict(strain):
    if strain is None:
        return None
    if isinstance(strain, dict):
        return {k: np.asarray(strain[k], dtype=float) for k in STRAIN_KEYS}
    return {k: np.asarray(getattr(strain, k), dtype=float) for k in STRAIN_KEYS}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.QdkpError("the qdkp operator needs a CUDA device; none is visible")
    return torch


class KPOperator(spla.LinearOperator):
    """Device-resident eight- (or six-/four-) band k.p operator."""

    def __init__(self, shape, h, n_bands, flags, fields, device=None):
        torch = _torch()
        self.grid_shape = tuple(int(s) for s in shape)
        self.h = float(h)
        self.n_bands = int(n_bands)
        self.flags = int(flags)
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.n_sites = int(np.prod(self.grid_shape))
        n = self.n_bands * self.n_sites
        super().__init__(dtype=np.dtype(np.complex128), shape=(n, n))
        self._fields = {k: np.ascontiguousarray(fields[k], dtype=np.float64).ravel()
                        if fields.get(k) is not None else None for k in FIELD_ORDER}
        ptrs = (ctypes.c_void_p * len(FIELD_ORDER))(
            *[v.ctypes.data if v is not None else None for v in
              (self._fields[k] for k in FIELD_ORDER)])
        h_ = ctypes.c_void_p()
        nx, ny, nz = self.grid_shape
        check(lib().qdkp_operator_create(nx, ny, nz, self.h, self.n_bands, self.flags, ptrs,
                                         self.device, ctypes.byref(h_)),
              'qdkp_operator_create')
        self._handle = h_
        nnz = ctypes.c_int64()
        check(lib().qdkp_operator_info(h_, None, None, None, None, None, ctypes.byref(nnz)),
              'qdkp_operator_info')
        self._nnz = int(nnz.value)
        self._ws = None

    # -- lifetime ---------------------------------------------------------------------------
    def close(self):
        if getattr(self, '_handle', None) is not None and self._handle.value:
            lib().qdkp_operator_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if self._handle is None:
            raise _lib.QdkpError("operator has been closed")
        return self._handle

    # -- what the reference's callers use on H ----------------------------------------------
    @property
    def nnz(self):
        """Structural nonzero count of the CSR the reference would assemble."""
        return self._nnz

    def diagonal(self):
        """diag(H), the Jacobi preconditioner input (eigensolvers.py:154)."""
        f = {k: (v.reshape(self.grid_shape) if v is not None else np.zeros(self.grid_shape))
             for k, v in self._fields.items()}
        h2 = self.h ** 2
        dk = []
        for key in ('gamma1', 'gamma2'):
            a = f[key]
            out = []
            for ax in range(3):
                d = np.zeros(self.grid_shape)
                n = self.grid_shape[ax]
                lo = [slice(None)] * 3
                hi = [slice(None)] * 3
                lo[ax] = slice(0, n - 1)
                hi[ax] = slice(1, n)
                t = 0.5 * (a[tuple(lo)] + a[tuple(hi)]) / h2
                d[tuple(lo)] += t
                d[tuple(hi)] += t
                for edge in (0, n - 1):
                    sl = [slice(None)] * 3
                    sl[ax] = edge
                    d[tuple(sl)] += a[tuple(sl)] / h2
                out.append(d)
            dk.append(out)
        A = f['Ec'] + 6 * G / h2
        P = -f['Ev'] + G * (dk[0][0] + dk[0][1] + dk[0][2])
        Q = G * (dk[1][0] + dk[1][1] - 2 * dk[1][2])
        if self.flags & _lib.STRAIN:
            Q = Q - (f['b'] / 2.0) * (f['exx'] + f['eyy'] - 2.0 * f['ezz'])
        bands = [A, A, -P + Q, -P - Q, -P - Q, -P + Q, -P - f['delta_so'], -P - f['delta_so']]
        sl = BAND_SLICES[self.n_bands]
        d = np.concatenate([b.ravel() for b in bands[sl]])
        if (self.flags & _lib.HOLE_CONVENTION) and self.n_bands != 8:
            d = -d
        if self.flags & _lib.NEGATE:
            d = -d
        return d.astype(np.complex128)

    def tocsc(self):
        raise NotImplementedError("KPOperator is matrix-free: ILU preconditioning "
                                  "(eigensolvers.ilu_preconditioner) needs the CSR path")

    def __sub__(self, other):
        raise NotImplementedError("KPOperator is matrix-free: form shifts with "
                                  "apply(..., sigma=...) instead of H - sigma * I")

    def _adjoint(self):
        return self                                       # Hermitian by construction

    # -- host application (scipy LinearOperator protocol) ------------------------------------
    def _matvec(self, x):
        return self._matmat(np.asarray(x).reshape(-1, 1)).reshape(-1)

    def _matmat(self, X):
        return self.apply_host(X)

    def apply_host(self, X, sigma=0.0, mode=_lib.APPLY_PLAIN):
        torch = _torch()
        X = np.ascontiguousarray(X, dtype=np.complex128)
        if X.ndim != 2 or X.shape[0] != self.shape[0]:
            raise ValueError(f"expected an ({self.shape[0]}, m) block, got {X.shape}")
        m = X.shape[1]
        need = int(lib().qdkp_apply_host_workspace_size(self.handle, m, mode))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=f'cuda:{self.device}')
        Y = np.empty_like(X)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        check(lib().qdkp_apply_host(self.handle, X.ctypes.data, Y.ctypes.data, m, float(sigma),
                                    mode, self._ws.data_ptr(), self._ws.numel(), stream),
              'qdkp_apply_host')
        return Y

    # -- device application -------------------------------------------------------------------
    def apply(self, X, sigma=0.0, mode=_lib.APPLY_PLAIN, out=None, workspace=None):
        """Y = H X, (H - sigma) X or (H - sigma)^2 X for a CUDA tensor X of shape (n, m),
        complex128 or complex64 (row stride may exceed m)."""
        torch = _torch()
        if X.dim() != 2 or X.shape[0] != self.shape[0] or X.stride(1) != 1:
            raise ValueError("X must be an (n, m) CUDA tensor with unit column stride")
        prec = {torch.complex128: _lib.C128, torch.complex64: _lib.C64}.get(X.dtype)
        if prec is None:
            raise TypeError("X must be complex128 or complex64")
        m = X.shape[1]
        Y = torch.empty_like(X, memory_format=torch.contiguous_format) if out is None else out
        ws_ptr, ws_bytes = None, 0
        if mode == _lib.APPLY_FOLDED:
            if workspace is None:
                workspace = torch.empty_like(X, memory_format=torch.contiguous_format)
            ws_ptr, ws_bytes = workspace.data_ptr(), workspace.numel() * workspace.element_size()
        stream = torch.cuda.current_stream(X.device).cuda_stream
        check(lib().qdkp_apply(self.handle, X.data_ptr(), X.stride(0), Y.data_ptr(),
                               Y.stride(0), m, float(sigma), mode, prec, ws_ptr, ws_bytes, stream),
              'qdkp_apply')
        return Y

    def set_tile(self, tile, precision=_lib.C128):
        """Force the H.X kernel for this operator and precision: a staged tile shape
        0..TILE_COUNT-1 (TILE_TMA0.. are the complex64 TMA shapes), TILE_DIRECT, or TILE_AUTO
        (heuristic)."""
        check(lib().qdkp_operator_set_tile(self.handle, precision, int(tile)),
              'qdkp_operator_set_tile')

    def get_tile(self, precision=_lib.C128):
        t = ctypes.c_int()
        check(lib().qdkp_operator_get_tile(self.handle, precision, ctypes.byref(t)),
              'qdkp_operator_get_tile')
        return t.value

    def tune(self, m, dtype=None, reps=5):
        """Autotune the H.X kernel for (n, m) blocks of `dtype` (complex128 by default): time
        every staged tile shape and the direct kernel on a random block, keep the fastest for
        this operator. Returns {tile: seconds per launch}."""
        torch = _torch()
        dtype = dtype or torch.complex128
        prec = {torch.complex128: _lib.C128, torch.complex64: _lib.C64}[dtype]
        dev = f'cuda:{self.device}'
        X = torch.randn(self.shape[0], m, dtype=dtype, device=dev)
        Y = torch.empty_like(X)
        secs = (ctypes.c_double * (_lib.TILE_COUNT + 1))()
        stream = torch.cuda.current_stream(dev).cuda_stream
        check(lib().qdkp_operator_tune(self.handle, X.data_ptr(), m, Y.data_ptr(), m, m, prec,
                                       int(reps), secs, stream), 'qdkp_operator_tune')
        tiles = list(range(_lib.TILE_COUNT)) + [_lib.TILE_DIRECT]
        return {t: secs[i] for i, t in enumerate(tiles) if secs[i] >= 0}

    def band_edges(self, mask=None, levels=False):
        """k = 0 valence levels of every site from this operator's own fields (Ev with the
        hydrostatic shift, strain, b, d, delta_so): returns dict(top_v1 = max v1 over `mask`
        (hole_sigma with margin 0), kramers = largest in-pair splitting, and with levels=True
        v1, v2, v3 as grid-shaped host arrays)."""
        torch = _torch()
        dev = f'cuda:{self.device}'
        md = None
        if mask is not None:
            md = torch.from_numpy(np.ascontiguousarray(
                np.asarray(mask, dtype=bool).ravel()).view(np.uint8).copy()).to(dev)
            if md.numel() != self.n_sites:
                raise ValueError("mask must have one entry per grid site")
        lv = torch.empty(3 * self.n_sites, dtype=torch.float64, device=dev) if levels else None
        need = int(lib().qdkp_local_band_edges_workspace_size(self.handle))
        ws = torch.empty(need, dtype=torch.uint8, device=dev)
        top, split = ctypes.c_double(), ctypes.c_double()
        stream = torch.cuda.current_stream(dev).cuda_stream
        check(lib().qdkp_local_band_edges(self.handle, md.data_ptr() if md is not None else None,
                                          lv.data_ptr() if lv is not None else None,
                                          ctypes.byref(top), ctypes.byref(split), ws.data_ptr(),
                                          ws.numel(), stream), 'qdkp_local_band_edges')
        out = dict(top_v1=top.value, kramers=split.value)
        if levels:
            v = lv.cpu().numpy().reshape(3, *self.grid_shape)
            out.update(v1=v[0], v2=v[1], v3=v[2])
        return out

    def norm2_estimate(self, iters=30, seed=0):
        """||H||_2 from `iters` power iterations on a seeded complex vector (a lower bound that
        converges from below; used to form relative residuals ||Hv - Ev|| / (||H||_2 ||v||))."""
        torch = _torch()
        g = torch.Generator(device=f'cuda:{self.device}').manual_seed(seed)
        x = torch.randn((self.shape[0], 1), dtype=torch.complex128,
                        device=f'cuda:{self.device}', generator=g)
        x /= x.norm()
        lam = 0.0
        for _ in range(iters):
            y = self.apply(x)
            lam = float(y.norm())
            if lam == 0.0:
                break
            x = y / lam
        return lam

    def negated(self):
        """-H as a second device operator (same fields, sign flipped in the stencil)."""
        f = {k: (v.reshape(self.grid_shape) if v is not None else None)
             for k, v in self._fields.items()}
        return KPOperator(self.grid_shape, self.h, self.n_bands, self.flags ^ _lib.NEGATE, f,
                          self.device)

    def update_diagonal(self, Ec=None, Ev=None):
        """Swap in new Ec / Ev fields (Hartree or potential updates) without re-uploading."""
        a = np.ascontiguousarray(Ec, dtype=np.float64).ravel() if Ec is not None else None
        b = np.ascontiguousarray(Ev, dtype=np.float64).ravel() if Ev is not None else None
        check(lib().qdkp_operator_update_diagonal(self.handle,
                                                  a.ctypes.data if a is not None else None,
                                                  b.ctypes.data if b is not None else None),
              'qdkp_operator_update_diagonal')
        if a is not None:
            self._fields['Ec'] = a
        if b is not None:
            self._fields['Ev'] = b


def confined_hamiltonian(ops, fields, n_bands=8, hole_convention=False, strain=None,
                         include_hydrostatic=False, interband_strain=True):
    """Device-resident replacement of kp_pryor.confined_hamiltonian (kp_pryor.py:363-466).

    `ops` is anything with `.shape` and `.h` (kp_confined.GridOperators or this module's
    GridOperators); only hard walls and the 'central' scheme exist on the device.
    """
    if getattr(ops, 'periodic', False):
        raise NotImplementedError("periodic grids are only used for bulk validation and are "
                                  "not built on the device")
    if getattr(ops, 'scheme', 'central') != 'central':
        raise NotImplementedError("only the default 'central' cross-term scheme is built")
    if n_bands not in BAND_SLICES:
        raise ValueError("n_bands must be 8, 6 or 4")
    shape = tuple(int(s) for s in ops.shape)
    st = _strain_dict(strain)
    f = {k: np.asarray(fields[k], dtype=float) for k in
         ('gamma1', 'gamma2', 'gamma3', 'delta_so', 'Ev', 'Ec')}
    for k, v in f.items():
        if v.shape != shape:
            f[k] = np.broadcast_to(v, shape).copy()
    f['P0'] = np.asarray(fields['P0'], dtype=float) if n_bands == 8 else None
    flags = 0
    if hole_convention:
        flags |= _lib.HOLE_CONVENTION
    if st is not None:
        flags |= _lib.STRAIN
        if interband_strain and n_bands == 8:
            flags |= _lib.INTERBAND_STRAIN
        f['b'] = np.asarray(fields['b'], dtype=float)
        f['d'] = np.asarray(fields['d'], dtype=float)
        f.update(st)
        if include_hydrostatic:
            # A + a_c Tr(eps) and P + a_v Tr(eps) (kp_pryor.py:425-428); P = -Ev + ...
            tr = st['exx'] + st['eyy'] + st['ezz']
            f['Ec'] = f['Ec'] + np.asarray(fields['a_c']) * tr
            f['Ev'] = f['Ev'] - np.asarray(fields['a_v']) * tr
    for k in list(f):
        if f[k] is not None and f[k].shape != shape:
            f[k] = np.broadcast_to(f[k], shape).copy()
    return KPOperator(shape, ops.h, n_bands, flags, f)


def _edge_operator(strain, Ev, delta_so, b, d):
    """A device operator carrying only the fields the k = 0 valence block reads."""
    st = _strain_dict(strain)
    arrs = [np.asarray(Ev, dtype=float), np.asarray(delta_so, dtype=float),
            np.asarray(b, dtype=float), np.asarray(d, dtype=float)] + list(st.values())
    shape = np.broadcast_shapes(*[a.shape for a in arrs])
    grid = shape if len(shape) == 3 else (int(np.prod(shape)) if shape else 1, 1, 1)

    def g(a):
        return np.broadcast_to(np.asarray(a, dtype=float), shape).reshape(grid).copy()
    zero = np.zeros(grid)
    f = dict(gamma1=zero, gamma2=zero, gamma3=zero, P0=zero, Ec=zero, Ev=g(Ev),
             delta_so=g(delta_so), b=g(b), d=g(d))
    f.update({k: g(v) for k, v in st.items()})
    return KPOperator(grid, 1.0, 8, _lib.STRAIN, f), shape


def local_band_edges(strain, Ev, Ec, delta_so, a_c, a_v, b, d, hydrostatic_applied=False):
    """kp_pryor.local_band_edges (kp_pryor.py:469-531) on the GPU: dict(cb, v1, v2, v3,
    kramers) with v1 >= v2 >= v3 the Kramers-paired k = 0 valence levels. Same arguments and
    broadcasting; `strain` is a StrainTensor-like object or a dict of the six components."""
    st = _strain_dict(strain)
    tr = st['exx'] + st['eyy'] + st['ezz']
    Ev_s = np.asarray(Ev, dtype=float) if hydrostatic_applied else np.asarray(Ev) - a_v * tr
    Ec_s = np.asarray(Ec, dtype=float) if hydrostatic_applied else np.asarray(Ec) + a_c * tr
    H, shape = _edge_operator(st, Ev_s, delta_so, b, d)
    try:
        e = H.band_edges(levels=True)
    finally:
        H.close()
    return dict(cb=np.broadcast_to(Ec_s, shape).copy(), v1=e['v1'].reshape(shape),
                v2=e['v2'].reshape(shape), v3=e['v3'].reshape(shape), kramers=e['kramers'])


def hole_sigma(Ev_field, strain, b_field, d_field, delta_so_field, inside_mask=None,
               margin=0.0, hydrostatic_applied=True):
    """kp_pryor.hole_sigma (kp_pryor.py:156-191) on the GPU: the exact local valence-band top,
    max of v1 inside the mask, plus `margin`."""
    st = _strain_dict(strain)
    Ev_s = np.asarray(Ev_field, dtype=float)
    if not hydrostatic_applied:
        raise NotImplementedError("hole_sigma passes a_v = 0, so hydrostatic_applied=False "
                                  "does not change the result; pass the shifted Ev")
    H, shape = _edge_operator(st, Ev_s, delta_so_field, b_field, d_field)
    try:
        mask = None if inside_mask is None else np.broadcast_to(inside_mask, shape)
        top = H.band_edges(mask=mask)['top_v1']
    finally:
        H.close()
    return float(top) + margin

