"""Post-processing of eigenstates on the GPU: the drop-in for pryor_fig4's localisation and
Kramers pairing (pryor_fig4.localization, pryor_fig4.py:179-193; kramers_levels, 222-236).

  localization(V, pyr)              -> loc per column, computed by the device reduction
                                       (qdkp_state_summary) whether V is on the host or the GPU
  kramers_levels(E, loc, split_tol) -> (levels, level localisation, worst splitting), the
                                       reference's pairing of consecutive entries
  state_summary(H, V, mask, E)      -> both in one device pass (what serving attaches to each
                                       result)
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib


def _torch():
    import torch
    return torch


def _device_mask(mask, device):
    """A device uint8 copy of a grid-shaped bool mask (a device tensor is used as it is)."""
    if hasattr(mask, 'data_ptr'):
        return mask
    m = np.ascontiguousarray(np.asarray(mask, dtype=bool).ravel()).view(np.uint8)
    return _torch().from_numpy(m.copy()).to(f'cuda:{device}')


def state_summary(H, V, mask, E=None):
    """Localisation of every column of V (device (n, k) complex128/complex64 tensor, or a host
    array) in the dot `mask` (grid-shaped bool array or a device uint8 tensor of n_sites), and,
    given the energies E in the column order, the Kramers levels of consecutive pairs.
    Returns dict(loc, levels, level_loc, kramers_split)."""
    torch = _torch()
    if not hasattr(V, 'data_ptr'):
        V = torch.from_numpy(np.ascontiguousarray(V, dtype=np.complex128)).to(f'cuda:{H.device}')
    if V.dim() != 2 or V.shape[0] != H.shape[0] or V.stride(1) != 1:
        raise ValueError("V must be an (n, k) block with unit column stride")
    prec = {torch.complex128: _lib.C128, torch.complex64: _lib.C64}.get(V.dtype)
    if prec is None:
        raise TypeError("V must be complex128 or complex64")
    k = V.shape[1]
    md = _device_mask(mask, H.device)
    if md.numel() != H.n_sites:
        raise ValueError(f"mask has {md.numel()} sites, the operator {H.n_sites}")
    need = int(lib().qdkp_state_summary_workspace_size(H.handle, k))
    if need == 0:
        raise ValueError("k must be in [1, 128]")
    ws = torch.empty(need, dtype=torch.uint8, device=V.device)
    loc = np.empty(k)
    Ein = None if E is None else np.ascontiguousarray(E, dtype=np.float64)
    npair = k // 2
    levels, lloc, worst = np.empty(max(npair, 1)), np.empty(max(npair, 1)), ctypes.c_double()
    stream = torch.cuda.current_stream(V.device).cuda_stream
    check(lib().qdkp_state_summary(H.handle, V.data_ptr(), V.stride(0), k, prec, md.data_ptr(),
                                   Ein.ctypes.data if Ein is not None else None, loc.ctypes.data,
                                   levels.ctypes.data, lloc.ctypes.data, ctypes.byref(worst),
                                   ws.data_ptr(), ws.numel(), stream), 'qdkp_state_summary')
    out = dict(loc=loc)
    if Ein is not None:
        out.update(levels=levels[:npair], level_loc=lloc[:npair], kramers_split=worst.value)
    return out


def localization(V, pyr, H=None):
    """pryor_fig4.localization: fraction of sum_bands |psi|^2 inside the dot, per column.
    `H` is the device operator the states belong to (needed for the grid); V host or device."""
    if H is None:
        raise TypeError("localization on the GPU needs the operator H the states belong to")
    return state_summary(H, V, pyr)['loc']


def kramers_levels(E, loc, split_tol=1e-4):
    """pryor_fig4.kramers_levels: (level energies, mean localisation per level, largest
    within-pair splitting in eV) of the spectrum paired as given."""
    E = np.asarray(E)
    n = len(E) // 2 * 2
    pairs = E[:n].reshape(-1, 2)
    lvl = pairs.mean(axis=1)
    worst = float(np.abs(np.diff(pairs, axis=1)).max()) if n else 0.0
    lloc = np.asarray(loc)[:n].reshape(-1, 2).mean(axis=1)
    return lvl, lloc, worst
