"""ctypes binding of libqdkp.so (the C ABI declared in include/qdkp.h).

The library is loaded from this package directory. There is no CPU fallback: if the shared
object is missing or fails to load, every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libqdkp.so')

QDKP_OK = 0
HOLE_CONVENTION, STRAIN, INTERBAND_STRAIN, NEGATE = 1, 2, 4, 8
C128, C64 = 0, 1
APPLY_PLAIN, APPLY_SHIFTED, APPLY_FOLDED = 0, 1, 2
TILE_AUTO, TILE_DIRECT, TILE_COUNT = -1, -2, 17
TILE_TMA0 = 4                     # first TMA tile shape (complex64)
TILE_TMA2 = 12                    # first producer-warp TMA tile shape (complex64)
LOBPCG_STATUS = {0: 'converged', 1: 'maxiter', 2: 'cholesky_breakdown',
                 3: 'eigh_breakdown', 4: 'nonfinite'}


class QdkpError(RuntimeError):
    pass


class LobpcgParams(ctypes.Structure):
    _fields_ = [('block', ctypes.c_int), ('folded', ctypes.c_int), ('sigma', ctypes.c_double),
                ('tol', ctypes.c_double), ('maxiter', ctypes.c_int),
                ('restart_control', ctypes.c_int), ('precision', ctypes.c_int),
                ('verbosity', ctypes.c_int), ('time_hx', ctypes.c_int),
                ('stall_iterations', ctypes.c_int)]


class FdInfo(ctypes.Structure):
    _fields_ = [('iterations', ctypes.c_int), ('residual', ctypes.c_double),
                ('modes_dropped', ctypes.c_int), ('breakdown', ctypes.c_int),
                ('converged', ctypes.c_int)]


class LobpcgInfo(ctypes.Structure):
    _fields_ = [('iterations', ctypes.c_int), ('best_iteration', ctypes.c_int),
                ('status', ctypes.c_int), ('explicit_gram', ctypes.c_int),
                ('best_mean_residual', ctypes.c_double), ('seconds', ctypes.c_double),
                ('hx_applications', ctypes.c_int64), ('hx_launches', ctypes.c_int64),
                ('hx_seconds', ctypes.c_double), ('hx_bytes', ctypes.c_double)]


_lib = None

_SIGNATURES = {
    'qdkp_last_error': (ctypes.c_char_p, []),
    'qdkp_kernel_launches': (ctypes.c_int64, []),
    'qdkp_version': (ctypes.c_char_p, []),
    'qdkp_operator_create': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    'qdkp_operator_update_diagonal': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_void_p]),
    'qdkp_operator_info': (ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 4
                           + [ctypes.POINTER(ctypes.c_int64)] * 2),
    'qdkp_operator_destroy': (ctypes.c_int, [ctypes.c_void_p]),
    'qdkp_structural_nnz': (ctypes.c_int64, [ctypes.c_int] * 5),
    'qdkp_apply': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                  ctypes.c_void_p]),
    'qdkp_apply_folded_noalloc_max_elems': (ctypes.c_size_t, [ctypes.c_int]),
    'qdkp_apply_folded_noalloc': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                 ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                                 ctypes.c_double, ctypes.c_int, ctypes.c_void_p]),
    'qdkp_operator_set_tile': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    'qdkp_operator_get_tile': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int)]),
    'qdkp_operator_tune': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                          ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p]),
    'qdkp_device_fault': (ctypes.c_int, [ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int)]),
    'qdkp_apply_host_workspace_size': (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int,
                                                         ctypes.c_int]),
    'qdkp_apply_host': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_lobpcg_workspace_size': (ctypes.c_size_t, [ctypes.c_void_p,
                                                     ctypes.POINTER(LobpcgParams)]),
    'qdkp_lobpcg_solve': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LobpcgParams),
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.POINTER(LobpcgInfo),
                                         ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_engine_create': (ctypes.c_int, [ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    'qdkp_engine_destroy': (ctypes.c_int, [ctypes.c_void_p]),
    'qdkp_engine_slot_workspace_size': (ctypes.c_size_t, [ctypes.c_void_p,
                                                          ctypes.POINTER(LobpcgParams)]),
    'qdkp_engine_admit': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.POINTER(LobpcgParams), ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_int)]),
    'qdkp_engine_step': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    'qdkp_engine_set_graphs': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    'qdkp_engine_poll': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    'qdkp_engine_retire': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.POINTER(LobpcgInfo), ctypes.c_void_p]),
    'qdkp_block_gram_workspace_size': (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    'qdkp_block_gram': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                       ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_fd_strain_workspace_size': (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    'qdkp_fd_strain': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(FdInfo),
                                      ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_block_eigh_workspace_size': (ctypes.c_size_t, [ctypes.c_int]),
    'qdkp_block_eigh': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_block_update_workspace_size': (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    'qdkp_block_update': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                         ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_residuals_workspace_size': (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int]),
    'qdkp_residuals': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                      ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.c_void_p]),
    'qdkp_state_summary_workspace_size': (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int]),
    'qdkp_state_summary': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_local_band_edges_workspace_size': (ctypes.c_size_t, [ctypes.c_void_p]),
    'qdkp_local_band_edges': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_fourier_strain_workspace_size': (ctypes.c_size_t, [ctypes.c_int] * 3),
    'qdkp_fourier_strain': (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_void_p]
                            + [ctypes.c_double] * 4 + [ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_size_t, ctypes.c_void_p]),
    'qdkp_piezo_potential_workspace_size': (ctypes.c_size_t, [ctypes.c_int] * 3),
    'qdkp_piezo_potential': (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.c_double,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                             ctypes.c_void_p]),
}

# Every symbol include/qdkp.h declares (checked by the CPU test suite).
EXPORTS = tuple(_SIGNATURES)


def lib():
    """Load libqdkp.so once; raise if it is absent (there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QdkpError(f"{LIB_PATH} is missing: build it with "
                            f"`python -m qd3dsolver_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc, what):
    if rc != QDKP_OK:
        msg = lib().qdkp_last_error().decode(errors='replace')
        raise QdkpError(f"{what} failed ({rc}): {msg}")
