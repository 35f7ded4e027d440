"""Host-input producers on the GPU: drop-ins for strain_fourier.solve_strain,
elasticity_fd.solve_strain_fd and piezoelectric.potential (strain_fourier.py:142-235,
elasticity_fd.py:275-419, piezoelectric.py:59-99).

  solve_strain(inside_mask, eps_star, C11, C12, C44, h)        -> StrainTensor (elastic strain)
  solve_strain_fd(inside_mask, eps_star, C_dot, C_matrix, h)   -> FDStrainTensor (elastic strain
                                                                  with cg_iterations, cg_residual,
                                                                  cg_converged, cg_modes_dropped)
  potential(strain, e14, eps_r, h, sign=+1.0)                  -> phi (volts)

Same arguments, conventions and periodic cell as the reference; the transforms, the stencils, the
CG iteration and the spectral algebra run on the device (qdkp_fourier_strain, qdkp_fd_strain,
qdkp_piezo_potential). Results are host NumPy
arrays, or device tensors with device=True.
"""
import ctypes

import numpy as np

from ._lib import FdInfo, check, lib

COMPONENTS = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def _torch():
    import torch
    if not torch.cuda.is_available():
        from ._lib import QdkpError
        raise QdkpError("the device field producers need a CUDA device; none is visible")
    return torch


class StrainTensor:
    """The six components (tensor shear convention) and the trace, like
    strain_fourier.StrainTensor (strain_fourier.py:84-139)."""

    def __init__(self, exx, eyy, ezz, exy, eyz, ezx):
        self.exx, self.eyy, self.ezz, self.exy, self.eyz, self.ezx = exx, eyy, ezz, exy, eyz, ezx

    @property
    def trace(self):
        return self.exx + self.eyy + self.ezz

    def as_dict(self):
        return {k: getattr(self, k) for k in COMPONENTS}


def _ws(torch, nbytes, device):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def solve_strain(inside_mask, eps_star, C11, C12, C44, h, device=False):
    torch = _torch()
    mask = np.ascontiguousarray(np.asarray(inside_mask, dtype=bool))
    if mask.ndim != 3:
        raise ValueError("inside_mask must be a 3-D grid")
    nx, ny, nz = mask.shape
    dev = torch.device('cuda', torch.cuda.current_device())
    md = torch.from_numpy(mask.view(np.uint8).copy()).to(dev)
    out = torch.empty((6,) + mask.shape, dtype=torch.float64, device=dev)
    ws = _ws(torch, lib().qdkp_fourier_strain_workspace_size(nx, ny, nz), dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    check(lib().qdkp_fourier_strain(nx, ny, nz, float(h), md.data_ptr(), float(eps_star),
                                    float(C11), float(C12), float(C44), out.data_ptr(),
                                    ws.data_ptr(), ws.numel(), stream), 'qdkp_fourier_strain')
    parts = out if device else out.cpu().numpy()
    return StrainTensor(*[parts[i] for i in range(6)])


class FDStrainTensor(StrainTensor):
    """A StrainTensor with how the iterative FD solve went (elasticity_fd.py:76-87):
    cg_iterations, cg_residual, cg_converged, cg_modes_dropped (1 = only the k = 0 rigid
    translation, the legitimate one)."""

    cg_iterations = 0
    cg_residual = 0.0
    cg_converged = False
    cg_modes_dropped = 0


_BREAKDOWN = {1: 'preconditioner is not positive definite',
              2: 'non-positive curvature p.Ap',
              3: 'preconditioner lost positive definiteness'}


def solve_strain_fd(inside_mask, eps_star, C_dot, C_matrix, h, tol=1e-10, maxiter=2000,
                    verbose=False, return_total=False, require_converged=True, device=False):
    """Elastic strain of an inclusion with its own cubic constants C_dot = (C11, C12, C44) in a
    matrix with C_matrix, by the reference's Q1 finite-element energy minimisation
    (elasticity_fd.solve_strain_fd, elasticity_fd.py:275-363): same arguments, conventions and
    errors (RuntimeError when require_converged and the CG did not converge cleanly). Returns the
    elastic FDStrainTensor, or (elastic, total) with return_total."""
    torch = _torch()
    mask = np.ascontiguousarray(np.asarray(inside_mask, dtype=bool))
    if mask.ndim != 3:
        raise ValueError("inside_mask must be a 3-D grid")
    nx, ny, nz = mask.shape
    dev = torch.device('cuda', torch.cuda.current_device())
    md = torch.from_numpy(mask.view(np.uint8).copy()).to(dev)
    out = torch.empty((6,) + mask.shape, dtype=torch.float64, device=dev)
    tot = torch.empty((6,) + mask.shape, dtype=torch.float64, device=dev) if return_total else None
    ws = _ws(torch, lib().qdkp_fd_strain_workspace_size(nx, ny, nz), dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    cd = (ctypes.c_double * 3)(*[float(c) for c in C_dot])
    cm = (ctypes.c_double * 3)(*[float(c) for c in C_matrix])
    info = FdInfo()
    check(lib().qdkp_fd_strain(nx, ny, nz, float(h), md.data_ptr(), float(eps_star), cd, cm,
                               float(tol), int(maxiter), out.data_ptr(),
                               tot.data_ptr() if tot is not None else None, ctypes.byref(info),
                               ws.data_ptr(), ws.numel(), stream), 'qdkp_fd_strain')
    if verbose:
        print(f"    CG {info.iterations:4d}  ||r||/||f|| = {info.residual:.3e}")
    if require_converged and not info.converged:
        why = []
        if info.breakdown:
            why.append(f"CG broke down at iteration {info.iterations} ({_BREAKDOWN[info.breakdown]})")
        if info.residual >= tol:
            why.append(f"residual {info.residual:.2e} did not reach tol {tol:.0e} in "
                       f"{info.iterations} iterations")
        if info.modes_dropped > 1:
            why.append(f"preconditioner dropped {info.modes_dropped} wavevectors (only k = 0, "
                       "i.e. 1, is legitimate)")
        raise RuntimeError(f"strain solve did not converge on grid {mask.shape}: "
                           + "; ".join(why))
    parts = out if device else out.cpu().numpy()
    elastic = FDStrainTensor(*[parts[i] for i in range(6)])
    elastic.cg_iterations, elastic.cg_residual = int(info.iterations), float(info.residual)
    elastic.cg_converged, elastic.cg_modes_dropped = bool(info.converged), int(info.modes_dropped)
    if not return_total:
        return elastic
    tp = tot if device else tot.cpu().numpy()
    return elastic, StrainTensor(*[tp[i] for i in range(6)])


def potential(strain, e14, eps_r, h, sign=+1.0, device=False):
    torch = _torch()
    comps = [getattr(strain, k) if not isinstance(strain, dict) else strain[k] for k in COMPONENTS]
    dev = torch.device('cuda', torch.cuda.current_device())
    S = torch.stack([c if hasattr(c, 'data_ptr') else torch.from_numpy(np.asarray(c, dtype=float))
                     for c in comps]).to(dev, torch.float64).contiguous()
    shape = tuple(S.shape[1:])
    if len(shape) != 3:
        raise ValueError("strain components must be 3-D grids")
    e = (np.array(np.broadcast_to(np.asarray(e14, dtype=float), shape))
         if not hasattr(e14, 'data_ptr') else e14)
    E = (e14 if hasattr(e14, 'data_ptr') else torch.from_numpy(np.ascontiguousarray(e))).to(
        dev, torch.float64).contiguous()
    phi = torch.empty(shape, dtype=torch.float64, device=dev)
    nx, ny, nz = shape
    ws = _ws(torch, lib().qdkp_piezo_potential_workspace_size(nx, ny, nz), dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    check(lib().qdkp_piezo_potential(nx, ny, nz, float(h), S.data_ptr(), E.data_ptr(),
                                     float(eps_r), float(sign), phi.data_ptr(), ws.data_ptr(),
                                     ws.numel(), stream), 'qdkp_piezo_potential')
    return phi if device else phi.cpu().numpy()
