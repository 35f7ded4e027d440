"""Served form: many eight-band solves resident on one GPU, advanced together by the batched
LOBPCG engine (qdkp_engine_* in include/qdkp.h).

The reference solves one operator at a time (eigensolvers.solve_interior, eigensolvers.py:
313-372); here every request keeps its LOBPCG state (X, AX, P, AP, Ritz values) in a device
slot, one tick advances every running slot by one iteration, finished slots are retired (final
Rayleigh-Ritz, same post-processing as solve_interior) and their memory is reused for requests
that arrive later. Admission checks free HBM before a slot's workspace is allocated.

  Engine(max_slots)                  -- the device engine
  Request(H, k, sigma, ...)          -- one solve (folded around sigma, or extremal)
  solve_batch(requests)              -- continuous batching over a list, all present at t = 0
  serve(requests, arrivals)          -- requests that arrive over time; p50 / p99 latency

Mixed precision (Request(precision='mixed')): a request first iterates in complex64 (H.X on
the packed FP32 stencil, tall blocks in complex64, every Gram, Cholesky and Rayleigh-Ritz matrix
in FP64) down to `mixed_tol`, above the complex64 rounding floor of the folded residual; its
Ritz block is then promoted to a complex128 slot (re-orthonormalised, Rayleigh-Ritz in FP64)
that iterates to `tol`. Results, selection and residuals are the complex128 ones.
"""
import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib
from . import post
from .eigensolvers import start_block, _device_residuals
from .kp_pryor import KPOperator


def _torch():
    import torch
    return torch


@dataclass
class Request:
    H: KPOperator
    k: int = 4
    sigma: float = 0.0
    tol: float = 1e-8
    maxiter: int = 3000
    extra: int = None
    seed: int = 0
    folded: bool = True
    tag: object = None
    precision: str = 'c128'        # 'c128', or 'mixed' (complex64 search, complex128 finish)
    mixed_tol: float = 1e-4        # residual at which a mixed request leaves complex64
    mixed_stall: int = 30          # ... or after this many iterations without a new best
    mask: object = None            # dot mask (grid-shaped bool): results carry localisation and
                                   # Kramers levels (pryor_fig4.localization / kramers_levels)
    # filled in by the engine
    slot: int = -1
    t_arrive: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    result: dict = field(default=None)
    phase: str = 'c128'            # precision of the slot the request occupies
    iters_done: int = 0            # iterations of finished phases (scipy's count)
    ticks: dict = field(default_factory=dict)   # iterations run per phase

    @property
    def block(self):
        extra = max(2, self.k // 2) if self.extra is None else self.extra
        return min(self.k + extra, self.H.shape[0])


class Engine:
    """The batched engine on one device: admit, step, poll, retire."""

    def __init__(self, max_slots=64, device=None, graphs=True):
        torch = _torch()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.max_slots = int(max_slots)
        h = ctypes.c_void_p()
        check(lib().qdkp_engine_create(self.max_slots, self.device, ctypes.byref(h)),
              'qdkp_engine_create')
        self._h = h
        if not graphs:
            check(lib().qdkp_engine_set_graphs(self._h, 0), 'qdkp_engine_set_graphs')
        self._slots = {}       # slot -> (request, workspace, X0)
        self.ticks = 0

    def close(self):
        if getattr(self, '_h', None) is not None and self._h.value:
            lib().qdkp_engine_destroy(self._h)
            self._h = None
        self._slots.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    def _params(self, r, phase=None):
        phase = phase or ('c64' if r.precision == 'mixed' else 'c128')
        stall = 0
        if phase == 'c64':
            tol, prec = max(float(r.mixed_tol), float(r.tol or 0.0)), _lib.C64
            stall = int(r.mixed_stall)
        else:
            tol, prec = (float(r.tol) if r.tol else 0.0), _lib.C128
        maxiter = max(1, int(r.maxiter) - int(sum(r.ticks.values())))
        return _lib.LobpcgParams(block=r.block, folded=int(r.folded), sigma=float(r.sigma),
                                 tol=tol, maxiter=maxiter, restart_control=20, precision=prec,
                                 verbosity=0, time_hx=0, stall_iterations=stall)

    def workspace_bytes(self, r):
        prm = self._params(r)
        return int(lib().qdkp_engine_slot_workspace_size(r.H.handle, ctypes.byref(prm)))

    def free(self):
        return self.max_slots - len(self._slots)

    def can_admit(self, r, reserve_bytes=256 << 20):
        """A free slot and enough free HBM for the slot's workspace (plus a reserve)."""
        if not self.free():
            return False
        free_b, _ = _torch().cuda.mem_get_info(self.device)
        return free_b >= self.workspace_bytes(r) + reserve_bytes

    def admit(self, r, X0=None, phase=None):
        """Give request r a slot. X0 (device, n x block complex128) defaults to the seeded start
        block of solve_interior; `phase` ('c64' / 'c128') defaults to the request's first."""
        torch = _torch()
        phase = phase or ('c64' if r.precision == 'mixed' else 'c128')
        prm = self._params(r, phase)
        need = int(lib().qdkp_engine_slot_workspace_size(r.H.handle, ctypes.byref(prm)))
        if need == 0:
            raise ValueError(f"block {r.block} outside [1, 24]")
        ws = torch.empty(need, dtype=torch.uint8, device=f'cuda:{self.device}')
        if X0 is None:
            X0 = torch.from_numpy(start_block(r.H.shape[0], r.block, r.seed, True)).to(ws.device)
        r.phase = phase
        slot = ctypes.c_int()
        check(lib().qdkp_engine_admit(self._h, r.H.handle, ctypes.byref(prm), X0.data_ptr(),
                                      ws.data_ptr(), need, self.stream, ctypes.byref(slot)),
              'qdkp_engine_admit')
        r.slot = slot.value
        r.t_admit = time.perf_counter()
        self._slots[r.slot] = (r, ws, X0)
        return r.slot

    def step(self, ticks=1):
        check(lib().qdkp_engine_step(self._h, int(ticks), self.stream), 'qdkp_engine_step')
        self.ticks += ticks

    def poll(self):
        state = (ctypes.c_int * self.max_slots)()
        status = (ctypes.c_int * self.max_slots)()
        iters = (ctypes.c_int * self.max_slots)()
        check(lib().qdkp_engine_poll(self._h, state, status, iters, self.stream),
              'qdkp_engine_poll')
        self._iters = list(iters)
        self._status = list(status)
        return list(state), list(status), list(iters)

    def promote(self, slot):
        """A stopped complex64 slot: its final Ritz block becomes the start block of a
        complex128 slot for the same request. Returns the new slot."""
        torch = _torch()
        r, ws, X0 = self._slots.pop(slot)
        V = torch.empty((r.H.shape[0], r.block), dtype=torch.complex128, device=ws.device)
        lam = np.empty(r.block)
        info = _lib.LobpcgInfo()
        check(lib().qdkp_engine_retire(self._h, slot, lam.ctypes.data, V.data_ptr(), None,
                                       ctypes.byref(info), self.stream), 'qdkp_engine_retire')
        r.iters_done += int(info.iterations)
        del ws, X0
        return self.admit(r, X0=V, phase='c128')

    def finish(self, slot):
        """Retire a stopped slot, or promote it if it ended a complex64 phase; returns the new
        slot id for a promotion, else None."""
        r = self._slots[slot][0]
        r.ticks[r.phase] = r.ticks.get(r.phase, 0) + int(getattr(self, '_iters', [0] * (slot + 1))[slot])
        nonfinite = getattr(self, '_status', [0] * (slot + 1))[slot] == 4
        if r.phase == 'c64' and not nonfinite:          # a NaN search is not promoted
            return self.promote(slot)
        self.retire(slot)
        return None

    def retire(self, slot, certify_tol=1e-6):
        """Final Rayleigh-Ritz, then solve_interior's selection (k nearest sigma, ascending)
        or solve_lowest's (k lowest) with residual norms of H."""
        torch = _torch()
        r, ws, X0 = self._slots.pop(slot)
        m = r.block
        V = torch.empty((r.H.shape[0], m), dtype=torch.complex128, device=ws.device)
        lam = np.empty(m)
        info = _lib.LobpcgInfo()
        check(lib().qdkp_engine_retire(self._h, slot, lam.ctypes.data, V.data_ptr(), None,
                                       ctypes.byref(info), self.stream), 'qdkp_engine_retire')
        if r.folded:
            rq, _ = _device_residuals(r.H, V)
            order = np.argsort(np.abs(rq - r.sigma))[:r.k]
            E = rq[order]
            o2 = np.argsort(E)
            sel, E = order[o2], E[o2]
        else:
            sel = np.argsort(lam)[:r.k]
            E = lam[sel]
        Vk = V[:, list(sel)].contiguous()
        _, res = _device_residuals(r.H, Vk, E)
        r.t_done = time.perf_counter()
        r.result = dict(E=E, V=Vk, residuals=res, iterations=r.iters_done + info.iterations,
                        ticks=dict(r.ticks), mu=lam,
                        status=_lib.LOBPCG_STATUS.get(info.status, 'unknown'),
                        converged=bool(res.max() < certify_tol))
        if r.mask is not None:
            r.result.update(post.state_summary(r.H, Vk, r.mask, E))
        del ws, X0
        return r


def solve_batch(requests, max_slots=64, ticks_per_poll=8, engine=None):
    """Run every request through the engine with continuous batching: slots free up as solves
    finish and the next requests are admitted. Returns the requests with `.result` filled."""
    own = engine is None
    eng = Engine(max_slots) if own else engine
    pending = list(requests)
    running = {}
    t0 = time.perf_counter()
    for r in pending:
        r.t_arrive = t0
    try:
        while pending or running:
            while pending and eng.can_admit(pending[0]):
                r = pending.pop(0)
                running[eng.admit(r)] = r
            if not running:
                raise RuntimeError("cannot admit any request: not enough free HBM")
            eng.step(ticks_per_poll)
            state, status, iters = eng.poll()
            for s in [s for s in running if state[s] == 0]:
                r = running.pop(s)
                s2 = eng.finish(s)
                if s2 is not None:
                    running[s2] = r
    finally:
        if own:
            eng.close()
    return requests


def serve(requests, arrivals, max_slots=64, ticks_per_poll=8):
    """Requests arriving at `arrivals` seconds (relative to the start): admitted as soon as they
    have arrived and a slot plus HBM are free. Returns (requests, stats) with p50 / p99 latency
    (arrival to result) and converged eigenpairs per second."""
    eng = Engine(max_slots)
    order = np.argsort(arrivals)
    queue = [(float(arrivals[i]), requests[i]) for i in order]
    running = {}
    t0 = time.perf_counter()
    try:
        while queue or running:
            now = time.perf_counter() - t0
            while queue and queue[0][0] <= now and eng.can_admit(queue[0][1]):
                ta, r = queue.pop(0)
                r.t_arrive = t0 + ta
                running[eng.admit(r)] = r
            if not running:
                time.sleep(min(0.001, max(0.0, queue[0][0] - now)))
                continue
            eng.step(ticks_per_poll)
            state, status, iters = eng.poll()
            for s in [s for s in running if state[s] == 0]:
                r = running.pop(s)
                s2 = eng.finish(s)
                if s2 is not None:
                    running[s2] = r
    finally:
        eng.close()
    wall = time.perf_counter() - t0
    lat = np.array([r.t_done - r.t_arrive for r in requests])
    pairs = sum(int((r.result['residuals'] <= 1e-6).sum()) for r in requests)
    return requests, dict(wall=wall, eigenpairs=pairs, eigenpairs_per_s=pairs / wall,
                          p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)))
