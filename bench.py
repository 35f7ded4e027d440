"""Benchmark: converged eight-band k.p eigenpairs per second on the B200.

Headline workload ("fig4 sweep"): the reference's own Fig-4 benchmark (pryor_fig4.sweep), with
the coefficient fields the reference itself builds (committed fixtures tests/golden/fig4_b*.npz:
Pryor Table I parameters, FD-elasticity strain, first-order piezo potential, sigma_e and sigma_h
from pryor_fig4.environment). InAs {101} pyramids of base b = 6, 8, ..., 18 nm in GaAs at
h = 1.0 nm with 8 nm padding (grids 23x23x20 to 35x35x26, 84,640 to 254,800 unknowns); for every
size both bands, folded-spectrum LOBPCG with k = 8, block 12, seed 0 (pryor_fig4.bound_states).
One step = the 14 solves. An eigenpair counts only if it passes all three checks against the
reference's own solve of the same fields (tests/golden/fig4_b*.json):
  |E - E_ref| <= 1e-6 eV, Kramers partner within 1e-7 eV, ||Hv - Ev|| / (||H||_2 ||v||) <= 1e-8.

This sweep stands in for the 48x48x36 (h = 0.5 nm) and 128x128x96 (h = 0.375 nm) pyramid
workloads, on which neither implementation converges: with the materials.py parameters the GaAs
barrier's finite-difference spectrum has a spurious band through sigma (tests/test_spurious_band.py).
Those two operators are measured by fixed-iteration legs instead (key `baseline_configs`:
seconds per LOBPCG iteration of the plain complex128 drop-in, the served complex128 engine and
the complex64 phase of the served mixed form; the CPU oracle on the 48x48x36 operator), and the
128x128x96 operator carries the H.X roofline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form plain]

Under torchrun (N > 1) every rank solves its own copy of the sweep (weak scaling, no
collective on the data path); the elapsed time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
sys.path.insert(0, ROOT)

METRIC = "converged k·p eigenpairs/s at 1e-6 eV, served vs plain; p50/p99; H·X HBM GB/s"
SIZES = (6.0, 8.0, 10.0, 12.0, 14.0, 16.0, 18.0)
BANDS = ('cb', 'vb')
K, BLOCK, MAXITER = 8, 12, 8000
TOL = 1e-8                 # folded-residual tolerance: tight enough for the relative-residual rule
E_TOL, SPLIT_TOL, REL_TOL = 1e-6, 1e-7, 1e-8
CPU_FULL_BASE = 6.0        # the CPU baseline solves this size to convergence (both bands)


def dist_env():
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return ws, rank, local


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
            p = json.load(fh)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.device), f'--query-gpu={self.FIELDS}',
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ''
        sm, mx, reasons = [], [], set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(mx), 'samples': len(sm),
                'reasons': sorted(reasons)}


# ----------------------------------------------------------------------------------------------
# Workload and the parity check of every counted eigenpair
# ----------------------------------------------------------------------------------------------

def load_sweep():
    """The seven Fig-4 environments as the reference built them, and its own solves of them."""
    from qd3dsolver_b200 import workloads as wl
    wls, refs = [], {}
    for b in SIZES:
        w = wl.fig4_from_fixture(os.path.join(GOLDEN, f'fig4_b{int(b)}_fields.npz'))
        w.name = f'fig4_b{int(b)}'
        w.meta['base'] = b
        with open(os.path.join(GOLDEN, f'fig4_b{int(b)}.json')) as fh:
            refs[b] = json.load(fh)
        wls.append(w)
    return wls, refs


def checked_pairs(E, res, ref_band, hnorm):
    """Eigenpairs of one solve that pass the three checks against the reference's solve of the
    same operator and band. Returns (count, worst |dE|, worst relative residual, worst split)."""
    E = np.asarray(E, dtype=float)
    res = np.asarray(res, dtype=float)
    o = np.argsort(E)
    E, res = E[o], res[o]
    refE = np.asarray(ref_band['E'], dtype=float)
    n = len(E)
    dE = np.array([np.abs(refE - e).min() for e in E])
    rel = res / hnorm
    split = np.full(n, np.inf)
    for i in range(n - n % 2):
        split[i] = abs(E[i] - E[i ^ 1])
    ok = (dE <= E_TOL) & (rel <= REL_TOL) & (split <= SPLIT_TOL)
    return int(ok.sum()), float(dE.max()), float(rel.max()), float(split[:n - n % 2].max())


def score(results, refs):
    """results: {(b, band): (E, residuals)} -> (pairs, parity summary)."""
    pairs, worst = 0, dict(abs_dE=0.0, rel_residual=0.0, kramers_split=0.0)
    for (b, band), (E, res) in results.items():
        c, de, rl, sp = checked_pairs(E, res, refs[b][band], refs[b]['H_norm2'])
        pairs += c
        worst['abs_dE'] = max(worst['abs_dE'], de)
        worst['rel_residual'] = max(worst['rel_residual'], rl)
        worst['kramers_split'] = max(worst['kramers_split'], sp)
    return pairs, worst


def make_operator(w):
    from qd3dsolver_b200 import kp_pryor as kpg, workloads as wl
    f = w.fields
    return kpg.confined_hamiltonian(kpg.GridOperators(w.shape, w.h), f, 8,
                                    strain={k: f[k] for k in wl.STRAIN_KEYS})


def flush_l2(torch, device):
    buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    buf.fill_(1.0)
    del buf


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


# ----------------------------------------------------------------------------------------------
# H.X roofline on the 128x128x96 operator
# ----------------------------------------------------------------------------------------------

def hx_roofline(torch, device, w2, launches=10):
    """H.X on the 128x128x96 operator, block 24 (inputs and outputs far larger than L2): the
    autotuner times every kernel / tile, then the chosen one is timed with CUDA events around
    `launches` launches on the launching stream. Algorithmic bytes per launch:
    N (15 s_f + 2 * 8 * m * s_c)."""
    from qd3dsolver_b200 import _lib
    H = make_operator(w2)
    out = {}
    stream = torch.cuda.current_stream(device)
    for dt, name, sf, sc in ((torch.complex128, 'c128', 8, 16), (torch.complex64, 'c64', 4, 8)):
        secs = H.tune(24, dt, reps=3)
        X = torch.randn(H.shape[0], 24, dtype=dt, device=device)
        Y = torch.empty_like(X)
        for _ in range(3):
            H.apply(X, out=Y)
        torch.cuda.synchronize(device)
        e0, e1 = _events(torch)
        e0.record(stream)
        for _ in range(launches):
            H.apply(X, out=Y)
        e1.record(stream)
        torch.cuda.synchronize(device)
        t = e0.elapsed_time(e1) * 1e-3 / launches
        byts = H.n_sites * (15 * sf + 2 * 8 * 24 * sc)
        prec = _lib.C128 if name == 'c128' else _lib.C64
        tile = H.get_tile(prec)
        label = ('direct' if tile == _lib.TILE_DIRECT else
                 f'TMA tile {tile}' if tile >= _lib.TILE_TMA0 else f'staged tile {tile}')
        out[name] = {'ms': t * 1e3, 'GBps': byts / t / 1e9, 'bytes': byts, 'launches': launches,
                     'kernel': label,
                     'tuner_GBps': {str(k): byts / v / 1e9 for k, v in secs.items()}}
        del X, Y
    H.close()
    return out


def hx_traffic():
    """DRAM bytes per 128x128x96 complex64 H.X launch from the committed ncu summary (a capture of
    the same kernel on a smaller grid, scaled by sites: traffic grows with the sites processed)."""
    p = os.path.join(ROOT, 'profiles', 'kp_apply_traffic.json')
    try:
        with open(p) as fh:
            return json.load(fh).get('dram_bytes_per_launch_128x128x96_c64_m24')
    except Exception:
        return None


# ----------------------------------------------------------------------------------------------
# Fixed-iteration legs on the 48x48x36 and 128x128x96 pyramid operators
# ----------------------------------------------------------------------------------------------

def fixed_iteration_legs(torch, device, wl1, wl2, iters):
    """Seconds per LOBPCG iteration on the two pyramid operators (block 12 / 24, seed-0 start
    blocks, both bands, never converging within `iters`): the plain complex128 drop-in (one solve
    at a time, (t(iters) - t(2)) / (iters - 2) per band), and the served engine with both bands
    resident (complex128 slots, and the complex64 phase of the mixed form), `iters` ticks."""
    from qd3dsolver_b200 import eigensolvers as eg, serving
    legs = {}
    for w, block in ((wl1, 12), (wl2, 24)):
        H = make_operator(w)
        n = H.shape[0]
        k = block * 2 // 3
        leg = {'grid': 'x'.join(map(str, w.shape)), 'h_nm': w.h, 'unknowns': n, 'block': block,
               'k': k, 'iterations_timed': iters,
               'sigma_eV': {b: w.sigma[b] for b in BANDS}}
        X0 = torch.from_numpy(eg.start_block(n, block, 0)).to(device)
        plain = {}
        for band in BANDS:
            ts = {}
            for it in (2, iters):
                torch.cuda.synchronize(device)
                e0, e1 = _events(torch)
                e0.record()
                eg.lobpcg_device(H, X0, folded=True, sigma=w.sigma[band], tol=1e-30, maxiter=it)
                e1.record()
                torch.cuda.synchronize(device)
                ts[it] = e0.elapsed_time(e1) * 1e-3
            plain[band] = (ts[iters] - ts[2]) / (iters - 2)
        leg['plain_c128_s_per_iteration'] = plain
        plain_rate = 2.0 / (plain['cb'] + plain['vb'])      # iterations / s, one solve at a time
        leg['plain_c128_iterations_per_s'] = plain_rate
        for form, prec in (('served_c128', 'c128'), ('served_mixed_c64_phase', 'mixed')):
            eng = serving.Engine(2, device=device.index)
            reqs = [serving.Request(H, k=k, sigma=w.sigma[b], tol=1e-30, maxiter=iters + 10,
                                    precision=prec, mixed_tol=1e-30, mixed_stall=0)
                    for b in BANDS]
            for r in reqs:
                eng.admit(r, X0=X0)
            eng.step(1)                     # first tick of this slot layout: graph capture
            torch.cuda.synchronize(device)
            e0, e1 = _events(torch)
            e0.record()
            eng.step(iters)
            e1.record()
            torch.cuda.synchronize(device)
            dt = e0.elapsed_time(e1) * 1e-3
            eng.poll()
            eng.close()
            del reqs
            leg[form + '_s_per_tick'] = dt / iters
            leg[form + '_iterations_per_s'] = 2.0 * iters / dt       # both bands advance a tick
            leg[form + '_vs_plain'] = (2.0 * iters / dt) / plain_rate
        legs[w.name] = leg
        H.close()
        del X0
        torch.cuda.empty_cache()
    return legs


# ----------------------------------------------------------------------------------------------
# Batched uneven dots and the antimonide serving stream
# ----------------------------------------------------------------------------------------------

def guarded(leg, *args):
    """A side leg whose failure is reported in its own key instead of ending the run."""
    import traceback
    try:
        return leg(*args)
    except Exception as e:                              # noqa: BLE001 -- reported, not hidden
        traceback.print_exc(file=sys.stderr)
        return {'error': f'{type(e).__name__}: {e}'[:300]}


def fd_strain_leg(torch, w2):
    """The inhomogeneous FD elasticity (fields.solve_strain_fd, the reference's
    elasticity_fd.solve_strain_fd) on the 128x128x96 pyramid: InAs dot in GaAs with Pryor's
    Table I constants, tol 1e-10, timed on the device (one warm-up solve first)."""
    from qd3dsolver_b200 import fields, workloads as wl
    dot, mat = wl.PRYOR_TABLE_I['InAs'], wl.PRYOR_TABLE_I['GaAs']
    eps_star = (mat['a0'] - dot['a0']) / dot['a0']
    args = (w2.mask, eps_star, (dot['C11'], dot['C12'], dot['C44']),
            (mat['C11'], mat['C12'], mat['C44']), w2.h)
    fields.solve_strain_fd(*args, tol=1e-10, device=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = fields.solve_strain_fd(*args, tol=1e-10, device=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {'grid': 'x'.join(map(str, w2.shape)), 'sites': int(np.prod(w2.shape)),
            'seconds': dt, 'iterations': st.cg_iterations, 'residual': st.cg_residual,
            'converged': st.cg_converged, 'modes_dropped': st.cg_modes_dropped,
            'ms_per_iteration': dt / max(st.cg_iterations, 1) * 1e3}


def batched_dots_leg(torch, device, ndots, budget):
    """64 seeded In(x)Ga(1-x)As/GaAs dots (x ~ U[0.6, 1], pyramid or spherical cap, base 6-20 nm,
    h = 0.5 nm, grids 32^3 to 96x96x72, 2-8 Kramers pairs; seed 1), bands alternating cb / vb,
    each solve given `budget` iterations. With the materials.py GaAs barrier at h = 0.5 nm none of
    them converges (the spurious band of tests/test_spurious_band.py), so the leg reports
    iteration throughput: the served engine (mixed precision, all dots admitted by free HBM
    into one continuous batch whose ticks replay as CUDA graphs) against the plain complex128
    drop-in solving them one by one, on the same requests and budget."""
    from qd3dsolver_b200 import eigensolvers as eg, serving, workloads as wl
    rng = np.random.default_rng(1)
    t0 = time.perf_counter()
    dots = [wl.random_dot(rng, device=True) for _ in range(ndots)]
    t_prep = time.perf_counter() - t0
    ops = [make_operator(w) for w in dots]
    bands = [BANDS[i % 2] for i in range(ndots)]

    def reqs():
        return [serving.Request(H, k=w.k, sigma=w.sigma[b], tol=1e-8, maxiter=budget,
                                precision='mixed', tag=i)
                for i, (w, H, b) in enumerate(zip(dots, ops, bands))]
    serving.solve_batch(reqs()[:2], max_slots=2)                 # warm: kernels, graph paths
    torch.cuda.synchronize(device)
    e0, e1 = _events(torch)
    e0.record()
    served = serving.solve_batch(reqs(), max_slots=ndots, ticks_per_poll=8)
    e1.record()
    torch.cuda.synchronize(device)
    t_served = e0.elapsed_time(e1) * 1e-3
    it_s = sum(r.result['iterations'] for r in served)
    un_s = sum(r.result['iterations'] * r.H.shape[0] for r in served)
    e0, e1 = _events(torch)
    e0.record()
    it_p = un_p = 0
    for w, H, b in zip(dots, ops, bands):
        X0 = eg.start_block(H.shape[0], min(w.k + max(2, w.k // 2), 24), 0)
        _, _, hist, info = eg.lobpcg_device(H, X0, folded=True, sigma=w.sigma[b], tol=1e-8,
                                            maxiter=budget)
        it_p += info['iterations']
        un_p += info['iterations'] * H.shape[0]
    e1.record()
    torch.cuda.synchronize(device)
    t_plain = e0.elapsed_time(e1) * 1e-3
    sizes = [w.n for w in dots]
    out = {'dots': ndots, 'seed': 1, 'iterations_budget': budget,
           'unknowns_min_max': [min(sizes), max(sizes)],
           'k_min_max': [min(w.k for w in dots), max(w.k for w in dots)],
           'host_preparation_s': t_prep,
           'served_mixed': {'seconds': t_served, 'iterations': it_s,
                            'iterations_per_s': it_s / t_served,
                            'unknown_iterations_per_s': un_s / t_served,
                            'statuses': sorted({r.result['status'] for r in served}),
                            'converged': sum(bool(r.result['converged']) for r in served)},
           'plain_c128': {'seconds': t_plain, 'iterations': it_p,
                          'iterations_per_s': it_p / t_plain,
                          'unknown_iterations_per_s': un_p / t_plain}}
    out['served_vs_plain_unknown_iterations'] = (out['served_mixed']['unknown_iterations_per_s'] /
                                                 out['plain_c128']['unknown_iterations_per_s'])
    for H in ops:
        H.close()
    return out


def antimonide_stream_leg(torch, device, nreq, budget):
    """A prefix of the seeded (seed 2) antimonide request stream: InSb / In(x)Ga(1-x)Sb lens or
    dash dots in InAs, radius 3-15 nm, h 0.4-0.6 nm, grids 32^3 to 128^3, 2-8 Kramers pairs, cb
    or vb with sigma as heterostructure.eight_band_states sets it, each with an iteration
    budget (broken-gap valence targets sit in the matrix conduction continuum and end at it).
    The requests are first solved as one batch to measure the engine's capacity; then the same
    requests arrive by a Poisson process at 80% of that capacity and are served with
    continuous batching (admission by free HBM). An eigenpair counts when its request
    converged, its relative residual ||Hv - Ev|| / ||H||_2 is <= 1e-8 (||H||_2 by power
    iteration) and its Kramers partner is within 1e-7 eV."""
    from qd3dsolver_b200 import serving, workloads as wl
    rng = np.random.default_rng(2)
    t0 = time.perf_counter()
    items = [wl.antimonide_request(rng, device=True) for _ in range(nreq)]
    t_prep = time.perf_counter() - t0
    ops = [make_operator(w) for w, _ in items]
    norms = [H.norm2_estimate() for H in ops]

    def reqs():
        return [serving.Request(H, k=w.k, sigma=w.sigma[b], tol=1e-8, maxiter=budget,
                                precision='mixed', tag=(i, b), mask=w.mask)
                for i, ((w, b), H) in enumerate(zip(items, ops))]
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    serving.solve_batch(reqs(), max_slots=nreq, ticks_per_poll=8)
    t_batch = time.perf_counter() - t0
    rate = 0.8 * nreq / t_batch
    rr = reqs()
    arrivals = np.cumsum(np.random.default_rng(3).exponential(1.0 / rate, size=nreq))
    _, stats = serving.serve(rr, arrivals, max_slots=nreq, ticks_per_poll=8)
    counted = 0
    for r, hn in zip(rr, norms):
        res = r.result
        if res['status'] != 'converged':
            continue
        E = np.asarray(res['E'])
        ok = (np.asarray(res['residuals']) / hn) <= REL_TOL
        o = np.argsort(E)
        split = np.full(len(E), np.inf)
        for i in range(len(E) - len(E) % 2):
            split[o[i]] = abs(E[o[i]] - E[o[i ^ 1]])
        counted += int((ok & (split <= SPLIT_TOL)).sum())
    st = [r.result['status'] for r in rr]
    return {'requests': nreq, 'of_stream': 2000, 'seed': 2, 'iterations_budget': budget,
            'host_preparation_s': t_prep, 'batch_seconds': t_batch, 'rate_per_s': rate,
            'statuses': {k: st.count(k) for k in sorted(set(st))},
            'bands': {b: sum(1 for _, bb in items if bb == b) for b in BANDS},
            'unknowns_min_max': [min(w.n for w, _ in items), max(w.n for w, _ in items)],
            'eigenpairs_checked': counted, 'eigenpairs_checked_per_s': counted / stats['wall'],
            **stats}


# ----------------------------------------------------------------------------------------------
# CPU: the oracle (scipy LOBPCG on the oracle CSR), timed on the host cores
# ----------------------------------------------------------------------------------------------

def _oracle_operator(w):
    from oracle import kp_operator as ko
    t0 = time.perf_counter()
    Hc = ko.confined_hamiltonian(w.shape, w.h, w.fields, 8, strain=True)
    return Hc, time.perf_counter() - t0


def cpu_seconds_per_iteration(Hc, sigma, block=BLOCK, lo=1, hi=3):
    """Folded scipy LOBPCG from the seed-0 start block: (t(hi) - t(lo)) / (hi - lo)."""
    import warnings
    import scipy.sparse.linalg as spla
    from oracle import eigensolvers as oe
    X0 = oe.start_block(Hc.shape[0], block, 0)
    F = oe.folded_operator(Hc, sigma)
    ts = {}
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        for it in (lo, hi):
            t0 = time.perf_counter()
            spla.lobpcg(F, X0.copy(), largest=False, tol=1e-30, maxiter=it)
            ts[it] = time.perf_counter() - t0
    return max(ts[hi] - ts[lo], 1e-9) / (hi - lo)


def cpu_child(args):
    """Host-core work run in a child process beside the GPU legs: --cpu-solve B BAND runs the
    oracle's complete folded solve of one Fig-4 solve (what pryor_fig4.bound_states runs, at the
    reference's tol 1e-7); --cpu-sample B1,B2,.. times CSR assembly and seconds per iteration of
    both bands of those sizes."""
    wls, refs = load_sweep()
    byb = {w.meta['base']: w for w in wls}
    if args.cpu_solve:
        from oracle import eigensolvers as oe
        b, band = float(args.cpu_solve[0]), args.cpu_solve[1]
        w = byb[b]
        Hc, t_asm = _oracle_operator(w)
        t0 = time.perf_counter()
        E, V, info = oe.solve_interior(Hc, k=K, sigma=w.sigma[band], tol=1e-7, maxiter=MAXITER)
        t = time.perf_counter() - t0
        print(json.dumps({'base': b, 'band': band, 'assembly_s': t_asm, 'solve_s': t,
                          'iterations': int(info['iterations']),
                          'max_residual_eV': float(np.max(info['residuals']))}))
        return
    out = {}
    for b in (float(x) for x in args.cpu_sample.split(',')):
        w = byb[b]
        Hc, t_asm = _oracle_operator(w)
        out[str(b)] = {'assembly_s': t_asm, **{band: cpu_seconds_per_iteration(Hc, w.sigma[band])
                                               for band in BANDS}}
    print(json.dumps(out))


def start_cpu_children():
    env = dict(os.environ, OPENBLAS_NUM_THREADS='1', OMP_NUM_THREADS='1',
               CUDA_VISIBLE_DEVICES='')
    me = os.path.abspath(__file__)
    procs = [subprocess.Popen([sys.executable, me, '--cpu-solve', str(CPU_FULL_BASE), band],
                              stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                              env=env) for band in BANDS]
    rest = ','.join(str(b) for b in SIZES if b != CPU_FULL_BASE)
    procs.append(subprocess.Popen([sys.executable, me, '--cpu-sample', rest],
                                  stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                                  env=env))
    return procs


def finish_cpu_children(procs, refs, timeout=900):
    try:
        outs = [json.loads(p.communicate(timeout=timeout)[0].strip().splitlines()[-1])
                for p in procs]
    except Exception as e:                     # a child that failed or ran out of time
        for p in procs:
            if p.poll() is None:
                p.kill()
        return {'value': None, 'unavailable': f'CPU baseline child failed: {e!r}'[:200]}
    full, sample = outs[:2], outs[2]
    total = 0.0
    detail = {}
    for f in full:
        total += f['assembly_s'] / 2 + f['solve_s']
        detail[f"b{int(f['base'])}_{f['band']}"] = {'solve_s': f['solve_s'],
                                                    'iterations': f['iterations']}
    for bs, s in sample.items():
        b = float(bs)
        for band in BANDS:
            it = refs[b][band]['iterations']
            total += s['assembly_s'] / 2 + s[band] * it
            detail[f"b{int(b)}_{band}"] = {'s_per_iteration': s[band], 'iterations': it}
    return {'value': len(SIZES) * len(BANDS) * K / total, 'unit': 'eigenpairs/s', 'cores': 3,
            'kind': 'port',
            'sample': f'oracle (scipy LOBPCG on the oracle CSR, single-threaded SpMM): complete '
                      f'folded solves of b = {int(CPU_FULL_BASE)} nm cb and vb at the '
                      f'reference\'s tol 1e-7, each in its own process; for b = 8..18 nm CSR '
                      f'assembly plus seconds per iteration of both bands, times the reference\'s '
                      f'own iteration counts of those solves (tests/golden/fig4_b*.json); three '
                      f'single-threaded processes beside the GPU run',
            'sweep_seconds_estimate': total, 'solves': detail}


def cpu_config1(w1):
    """The oracle on the 48x48x36 pyramid operator: CSR assembly and seconds per folded LOBPCG
    iteration of each band (block 12)."""
    Hc, t_asm = _oracle_operator(w1)
    return {'assembly_s': t_asm,
            's_per_iteration': {band: cpu_seconds_per_iteration(Hc, w1.sigma[band])
                                for band in BANDS},
            'openblas_threads': os.environ.get('OPENBLAS_NUM_THREADS'),
            'cpu_count': os.cpu_count()}


# ----------------------------------------------------------------------------------------------
# The GPU arm
# ----------------------------------------------------------------------------------------------

def run_ours(args):
    ws, rank, local = dist_env()
    children = start_cpu_children() if (rank == 0 and ws == 1 and not args.no_cpu) else None
    import torch
    from qd3dsolver_b200 import eigensolvers as eg, _lib, serving, workloads as wl
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    lib = _lib.lib()
    wls, refs = load_sweep()
    ops = [make_operator(w) for w in wls]
    torch.cuda.synchronize(device)

    def served_step():
        reqs = [serving.Request(H, k=K, sigma=w.sigma[band], tol=args.tol, maxiter=MAXITER,
                                tag=(w.meta['base'], band), precision=args.precision,
                                mixed_tol=args.mixed_tol)
                for w, H in zip(wls, ops) for band in BANDS]
        t0 = time.perf_counter()
        serving.solve_batch(reqs, max_slots=len(reqs), ticks_per_poll=args.ticks_per_poll)
        return dict(lat=[r.t_done - t0 for r in reqs],
                    res={r.tag: (r.result['E'], r.result['residuals']) for r in reqs},
                    iters={r.tag: r.result['iterations'] for r in reqs},
                    ticks={r.tag: r.result['ticks'] for r in reqs},
                    hx_s=0.0, hx_b=0.0, hx_n=0)

    def plain_step(time_hx=False):
        lat, res, iters = [], {}, {}
        hx_s = hx_b = 0.0
        hx_n = 0
        for w, H in zip(wls, ops):
            for band in BANDS:
                t0 = time.perf_counter()
                E, V, info = eg.solve_interior(H, k=K, sigma=w.sigma[band], tol=args.tol,
                                               maxiter=MAXITER, verbose=False,
                                               return_device=True, time_hx=time_hx)
                lat.append(time.perf_counter() - t0)
                res[(w.meta['base'], band)] = (E, info['residuals'])
                hx_s += info['hx_seconds']
                hx_b += info['hx_bytes']
                hx_n += info['hx_launches']
                iters[(w.meta['base'], band)] = info['iterations']
        return dict(lat=lat, res=res, hx_s=hx_s, hx_b=hx_b, hx_n=hx_n, iters=iters)

    step_fn = served_step if args.form == 'served' else (lambda: plain_step(time_hx=True))
    for _ in range(args.warmup):
        step_fn()
    flush_l2(torch, device)
    sampler = ClockSampler(local)
    if rank == 0:
        sampler.start()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(device)
    l0 = lib.qdkp_kernel_launches()
    steps = []
    t_start = time.perf_counter()
    for s in range(args.steps):
        e0, e1 = _events(torch)
        e0.record()
        r = step_fn()
        e1.record()
        torch.cuda.synchronize(device)
        r['ms'] = e0.elapsed_time(e1)
        steps.append(r)
        if s + 1 < args.steps:
            flush_l2(torch, device)
    torch.cuda.synchronize(device)
    wall = time.perf_counter() - t_start
    launches = lib.qdkp_kernel_launches() - l0
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop() if rank == 0 else None
    total_ms = sum(r['ms'] for r in steps)
    pairs, parity = 0, None
    for r in steps:
        p, parity_s = score(r['res'], refs)
        pairs += p
        parity = parity_s if parity is None else {k: max(parity[k], v) for k, v in parity_s.items()}
    if ws > 1:
        total_ms, pairs = combine_ranks(total_ms, pairs, device)
    value = pairs / (total_ms * 1e-3)
    lat = sorted(x for r in steps for x in r['lat'])
    hx_s = sum(r['hx_s'] for r in steps)
    hx_b = sum(r['hx_b'] for r in steps)
    hx_n = sum(r['hx_n'] for r in steps)

    plain = None
    if args.form == 'served' and rank == 0 and not args.no_plain:
        # the plain c128 single-solve form on the same 14 solves, and its H.X launch timings
        torch.cuda.synchronize(device)
        e0, e1 = _events(torch)
        e0.record()
        rp = plain_step(time_hx=True)
        e1.record()
        torch.cuda.synchronize(device)
        plain_ms = e0.elapsed_time(e1)
        pp, pparity = score(rp['res'], refs)
        plain = {'value': pp / (plain_ms * 1e-3), 'unit': 'eigenpairs/s',
                 'ms_per_step': plain_ms, 'eigenpairs_checked': pp, 'parity': pparity,
                 'iterations': {f"b{int(b)}_{band}": it for (b, band), it in rp['iters'].items()},
                 'latency_s': {'p50': sorted(rp['lat'])[len(rp['lat']) // 2],
                               'p99': sorted(rp['lat'])[-1]}}
        hx_s, hx_b, hx_n = rp['hx_s'], rp['hx_b'], rp['hx_n']

    # ---- e2e: the public API with host buffers (fields and X0 up, E and V down) -------------
    e2e = None
    if rank == 0 and not args.no_e2e:
        torch.cuda.synchronize(device)
        h2d = d2h = 0
        t0 = time.perf_counter()
        hops = [make_operator(w) for w in wls]          # uploads the 15 fields from the host
        h2d += sum(15 * w.n_sites * 8 for w in wls)
        res = {}
        if args.form == 'served':
            reqs = [serving.Request(H, k=K, sigma=w.sigma[band], tol=args.tol, maxiter=MAXITER,
                                    precision=args.precision, mixed_tol=args.mixed_tol,
                                    tag=(w.meta['base'], band))
                    for w, H in zip(wls, hops) for band in BANDS]
            serving.solve_batch(reqs, max_slots=len(reqs), ticks_per_poll=args.ticks_per_poll)
            for r in reqs:                               # X0 drawn on the host and uploaded
                h2d += r.H.shape[0] * r.block * 16
                V = r.result['V'].cpu().numpy()
                d2h += V.nbytes + r.result['E'].nbytes
                res[r.tag] = (r.result['E'], r.result['residuals'])
        else:
            for w, H in zip(wls, hops):
                for band in BANDS:
                    E, V, info = eg.solve_interior(H, k=K, sigma=w.sigma[band], tol=args.tol,
                                                   maxiter=MAXITER, verbose=False)
                    h2d += H.shape[0] * BLOCK * 16
                    d2h += V.nbytes + E.nbytes
                    res[(w.meta['base'], band)] = (E, info['residuals'])
        for H in hops:
            H.close()
        torch.cuda.synchronize(device)
        e2e_t = time.perf_counter() - t0
        e2e_pairs, _ = score(res, refs)
        e2e = {'value': e2e_pairs / e2e_t, 'unit': 'eigenpairs/s', 'h2d_bytes_per_step': h2d,
               'd2h_bytes_per_step': d2h, 'seconds_per_step': e2e_t,
               'eigenpairs_checked': e2e_pairs,
               'path': 'confined_hamiltonian + ' + ('serving.solve_batch' if args.form == 'served'
                                                    else 'eigensolvers.solve_interior')}

    # ---- serving: requests arriving over time (Poisson, seed 2), p50 / p99 latency ---------
    stream = None
    if rank == 0 and args.form == 'served' and not args.no_stream:
        rng = np.random.default_rng(2)
        reqs = [serving.Request(H, k=K, sigma=w.sigma[band], tol=args.tol, maxiter=MAXITER,
                                precision=args.precision, mixed_tol=args.mixed_tol,
                                tag=(w.meta['base'], band))
                for _ in range(2) for w, H in zip(wls, ops) for band in BANDS]
        rng.shuffle(reqs)
        # mean arrival rate: ~80 % of the batch throughput measured above
        rate = 0.8 * (value / K)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
        _, stats = serving.serve(reqs, arrivals, max_slots=len(SIZES) * len(BANDS),
                                 ticks_per_poll=args.ticks_per_poll)
        sp = sum(checked_pairs(r.result['E'], r.result['residuals'], refs[r.tag[0]][r.tag[1]],
                               refs[r.tag[0]]['H_norm2'])[0] for r in reqs)
        stream = dict(requests=len(reqs), rate_per_s=rate, eigenpairs_checked=sp,
                      eigenpairs_checked_per_s=sp / stats['wall'], **stats)

    for H in ops:
        H.close()
    del ops
    torch.cuda.empty_cache()
    big = None
    if rank == 0 and not (args.no_config2 and args.no_fixed):
        w1, w2 = wl.config1(), wl.config2()
        w1.name, w2.name = 'pyramid_48x48x36_h0.5', 'pyramid_128x128x96_h0.375'
        hx2 = None if args.no_config2 else hx_roofline(torch, device, w2)
        legs = None if args.no_fixed else fixed_iteration_legs(torch, device, w1, w2,
                                                               args.fixed_iterations)
        fd = None if args.no_config2 else guarded(fd_strain_leg, torch, w2)
        big = dict(hx2=hx2, legs=legs, w1=w1, fd=fd)
    dots = (guarded(batched_dots_leg, torch, device, args.dots, args.dot_budget)
            if (rank == 0 and not args.no_dots) else None)
    stream5 = (guarded(antimonide_stream_leg, torch, device, args.stream5, args.stream5_budget)
               if (rank == 0 and not args.no_stream5) else None)
    cpu = finish_cpu_children(children, refs) if children else None
    if cpu is not None and big is not None and big['legs'] is not None:
        c1 = cpu_config1(big['w1'])
        leg = big['legs'][big['w1'].name]
        c1['iterations_per_s'] = 2.0 / sum(c1['s_per_iteration'].values())
        leg['cpu_oracle'] = c1
        leg['plain_c128_vs_cpu'] = leg['plain_c128_iterations_per_s'] / c1['iterations_per_s']
    if rank == 0:
        peak, peak_kind = peaks()
        achieved = hx_b / hx_s / 1e9 if hx_s > 0 else None
        rl = None
        hx2 = big['hx2'] if big else None
        if hx2:
            c = hx2['c64']
            rl = {'kernel': f"kp_apply (H.X, {c['kernel']}, complex64, 128x128x96, 24 columns)",
                  'bound': 'hbm', 'achieved': c['GBps'], 'peak': peak, 'unit': 'GB/s',
                  'frac': c['GBps'] / peak, 'peak_source': f'{peak_kind} hbm_gbs',
                  'traffic': hx_traffic(), 'algorithmic_bytes_per_launch': c['bytes'],
                  'avg_launch_us': c['ms'] * 1e3, 'launches': c['launches'],
                  'where': 'CUDA events around 10 launches on the launching stream after the '
                           'timed steps; inputs and outputs 4.8 GB (> L2)'}
        out = {
            'metric': METRIC, 'value': value, 'unit': 'eigenpairs/s', 'n_gpus': ws,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': ('c64+c128' if (args.form == 'served' and args.precision == 'mixed')
                      else 'c128'),
            'data': 'synthetic inputs built by the reference (committed fixtures)',
            'config': {'workload': 'fig4 sweep, reference-built fields: InAs/GaAs pyramids '
                                   'b=6..18 nm, h=1.0 nm, Pryor Table I, FD strain + piezo, cb+vb, '
                                   'k=8, block 12, maxiter 8000 (pryor_fig4.sweep); stands in for '
                                   'the 48x48x36 / 128x128x96 pyramids, which converge in neither '
                                   'implementation (see baseline_configs)',
                       'form': (('served: batched engine, 14 solves resident, continuous '
                                 'batching, CUDA-graph ticks, ' +
                                 ('complex64 search to 1e-4 then complex128 finish (FP64 '
                                  'Gram/Cholesky/Rayleigh-Ritz throughout)'
                                  if args.precision == 'mixed' else 'complex128'))
                                if args.form == 'served' else
                                'plain c128 single-solve drop-in (solve_interior)'),
                       'tol': args.tol,
                       'counted': 'eigenpairs with |E-E_ref|<=1e-6 eV, Kramers split<=1e-7 eV, '
                                  '||Hv-Ev||/||H||_2<=1e-8 against the reference\'s own solves',
                       'solves_per_step': len(SIZES) * len(BANDS),
                       'eigenpairs_per_step': len(SIZES) * len(BANDS) * K,
                       'l2': 'flushed between timed steps (256 MB write); per-solve blocks '
                             '16-49 MB x ~10 reuse L2 within a solve',
                       'parallelism': f'replicas x{ws}'},
            'eigenpairs_checked_per_step': pairs / args.steps / ws,
            'parity': parity,
            'latency_s': {'p50': lat[len(lat) // 2], 'p99': lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                          'per': 'solve'},
            'iterations': {f"b{int(b)}_{band}": it for (b, band), it in steps[-1]['iters'].items()},
            'ticks_per_phase': ({f"b{int(b)}_{band}": t for (b, band), t in steps[-1]['ticks'].items()}
                                if 'ticks' in steps[-1] else None),
            'roofline': rl,
            'roofline_plain_step': {'kernel': 'kp_apply (H.X, complex128, every launch of the '
                                              'plain-form step, CUDA events)',
                                    'bound': 'hbm',
                                    'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                                    'frac': (achieved / peak) if achieved else None,
                                    'peak_source': f'{peak_kind} hbm_gbs',
                                    'launches': hx_n, 'avg_launch_us': hx_s / max(hx_n, 1) * 1e6,
                                    'algorithmic_bytes_per_launch': hx_b / max(hx_n, 1)},
            'plain': plain,
            'served_vs_plain': (value / plain['value']) if plain and plain['value'] else None,
            'serving_stream': stream,
            'baseline_configs': big['legs'] if big else None,
            'batched_dots': dots,
            'antimonide_stream': stream5,
            'hx_config2': hx2,
            'fd_strain_config2': big['fd'] if big else None,
            'cpu_baseline': cpu,
            'e2e': e2e,
            'clocks': clocks,
            'gpu_launches': launches,
            'gpu_launches_per_step': launches / args.steps,
            'wall_s_timed': wall,
        }
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def combine_ranks(total_ms, pairs, device):
    """Whole-job numbers of a replica run: elapsed time is the max over ranks (device-timed on
    each), converged eigenpairs the sum over ranks."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(total_ms)], dtype=torch.float64, device=device)
    p = torch.tensor([float(pairs)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    return float(t.item()), float(p.item())


# ----------------------------------------------------------------------------------------------
# Profiling aids
# ----------------------------------------------------------------------------------------------

def hx_probe(args):
    """A few H.X launches on the 48x48x36 or 128x128x96 operator (prints one JSON line)."""
    import torch
    from qd3dsolver_b200 import workloads as wl, _lib
    w = wl.config1() if args.hx_grid == '48' else wl.config2()
    H = make_operator(w)
    dt = torch.complex128 if args.hx_dtype == 'c128' else torch.complex64
    if args.hx_tile is not None:
        H.set_tile(args.hx_tile, _lib.C128 if args.hx_dtype == 'c128' else _lib.C64)
    X = torch.randn(H.shape[0], args.hx_m, dtype=dt, device='cuda')
    Y = torch.empty_like(X)
    for _ in range(args.hx_launches):
        H.apply(X, out=Y)
    torch.cuda.synchronize()
    print(json.dumps({'hx_probe': w.name, 'm': args.hx_m, 'dtype': args.hx_dtype,
                      'tile': args.hx_tile, 'launches': args.hx_launches}))
    H.close()


def engine_probe(args):
    """The served engine on the 14 sweep solves for a fixed number of ticks, with direct kernel
    launches (no graph), so that a profiler sees every kernel of a tick (prints one JSON line)."""
    import torch
    from qd3dsolver_b200 import serving
    wls, _ = load_sweep()
    keep = set(args.probe_solves.split(',')) if args.probe_solves else None
    pairs = [(w, band) for w in wls for band in BANDS
             if keep is None or f"b{int(w.meta['base'])}_{band}" in keep]
    ops = {w.name: make_operator(w) for w, _ in pairs}
    if args.probe_plain:
        # the plain drop-in, one solve after the other, each for --probe-ticks iterations
        from qd3dsolver_b200 import eigensolvers as eg
        for w, band in pairs:
            H = ops[w.name]
            X0 = torch.from_numpy(eg.start_block(H.shape[0], BLOCK, 0)).cuda()
            eg.lobpcg_device(H, X0, folded=True, sigma=w.sigma[band], tol=1e-30,
                             maxiter=args.probe_ticks)
        torch.cuda.synchronize()
    else:
        eng = serving.Engine(len(pairs), graphs=False)
        for w, band in pairs:
            eng.admit(serving.Request(ops[w.name], k=K, sigma=w.sigma[band], tol=TOL,
                                      maxiter=MAXITER, precision=args.precision))
        eng.step(args.probe_ticks)
        torch.cuda.synchronize()
        eng.close()
    print(json.dumps({'engine_probe': len(pairs), 'ticks': args.probe_ticks,
                      'precision': args.precision, 'plain': bool(args.probe_plain)}))
    for H in ops.values():
        H.close()


def tick_probe(args):
    """Latency of one resident solve: wall-clock milliseconds per engine tick (CUDA-graph
    replay, 64 ticks after 8, complex64 and complex128 slots) and per plain drop-in iteration
    ((t(40) - t(5)) / 35), on the chosen sweep solves' valence bands (prints one JSON line)."""
    import torch
    from qd3dsolver_b200 import eigensolvers as eg, serving
    wls, _ = load_sweep()
    keep = (args.probe_solves or 'b6_vb,b10_vb,b18_vb').split(',')
    out = {}
    for w in wls:
        for band in BANDS:
            tag = f"b{int(w.meta['base'])}_{band}"
            if tag not in keep:
                continue
            H = make_operator(w)
            X0 = torch.from_numpy(eg.start_block(H.shape[0], BLOCK, 0)).cuda()
            ts = {}
            for it in (5, 40):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                eg.lobpcg_device(H, X0, folded=True, sigma=w.sigma[band], tol=1e-30, maxiter=it)
                torch.cuda.synchronize()
                ts[it] = time.perf_counter() - t0
            rec = {'rows': H.shape[0], 'plain_ms_per_iteration': (ts[40] - ts[5]) / 35 * 1e3}
            for prec, name in (('mixed', 'c64'), ('c128', 'c128')):
                eng = serving.Engine(2, graphs=True)
                eng.admit(serving.Request(H, k=K, sigma=w.sigma[band], tol=1e-30, maxiter=10 ** 6,
                                          precision=prec))
                eng.step(8)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                eng.step(64)
                torch.cuda.synchronize()
                rec[f'{name}_ms_per_tick'] = (time.perf_counter() - t0) / 64 * 1e3
                eng.close()
            out[tag] = rec
            H.close()
    print(json.dumps({'tick_probe': out}))


# ----------------------------------------------------------------------------------------------
# The reference arm: the reference's CPU algorithm on the host cores
# ----------------------------------------------------------------------------------------------

def run_reference(args):
    """Each step samples one sweep size (in turn): the oracle's CSR assembly and seconds per
    folded scipy-LOBPCG iteration of both bands. The value is the sweep's eigenpairs/s from those
    samples and the reference's own iteration counts of the 14 solves (sizes a short run did not
    sample are scaled from the sampled ones by CSR nonzeros). After the steps, the 48x48x36
    pyramid operator is sampled the same way."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    wls, refs = load_sweep()
    samples = {}
    step_s = []
    for s in range(args.warmup + args.steps):
        w = wls[s % len(wls)]
        t0 = time.perf_counter()
        Hc, t_asm = _oracle_operator(w)
        samples[w.meta['base']] = dict(asm=t_asm, nnz=Hc.nnz, **{
            band: cpu_seconds_per_iteration(Hc, w.sigma[band]) for band in BANDS})
        step_s.append(time.perf_counter() - t0)
    fit = {k: np.mean([v[k] / v['nnz'] for v in samples.values()]) for k in ('asm',) + BANDS}
    total = 0.0
    for w in wls:
        b = w.meta['base']
        smp = samples.get(b) or {k: fit[k] * refs[b]['nnz'] for k in ('asm',) + BANDS}
        for band in BANDS:
            total += smp['asm'] / 2 + smp[band] * refs[b][band]['iterations']
    value = len(SIZES) * len(BANDS) * K / total
    ms = statistics.mean(step_s[args.warmup:]) * 1e3
    c1 = None
    if not args.no_fixed:
        from qd3dsolver_b200 import workloads as wl
        c1 = cpu_config1(wl.config1())
        c1['iterations_per_s'] = 2.0 / sum(c1['s_per_iteration'].values())
    threads = os.environ.get('OPENBLAS_NUM_THREADS') or str(os.cpu_count())
    out = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'eigenpairs/s',
           'n_gpus': ws, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms,
           'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128',
           'data': 'synthetic inputs built by the reference (committed fixtures)',
           'config': {'workload': 'fig4 sweep, reference-built fields (same as the ours arm)',
                      'form': 'scipy LOBPCG on the CSR operator (the reference algorithm '
                              'restated in oracle/)'},
           'cpu_baseline': {'value': value, 'unit': 'eigenpairs/s', 'cores': int(threads),
                            'kind': 'port',
                            'sample': 'per step one sweep size in turn: oracle CSR assembly + '
                                      'seconds per folded LOBPCG iteration of cb and vb '
                                      '((t(3) - t(1)) / 2); times the reference\'s own '
                                      'iteration counts of the 14 solves; CSR SpMM '
                                      'single-threaded, BLAS on all cores',
                            'sizes_sampled': sorted(samples)},
           'baseline_configs': {'pyramid_48x48x36_h0.5': {'cpu_oracle': c1}} if c1 else None,
           'e2e': {'value': value, 'unit': 'eigenpairs/s', 'h2d_bytes_per_step': 0,
                   'd2h_bytes_per_step': 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=2)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', choices=('ours', 'reference'), default='ours')
    ap.add_argument('--tol', type=float, default=TOL)
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline')
    ap.add_argument('--no-config2', action='store_true', help='skip the 128x128x96 H.X timing')
    ap.add_argument('--no-fixed', action='store_true',
                    help='skip the fixed-iteration legs on the pyramid operators')
    ap.add_argument('--fixed-iterations', type=int, default=20)
    ap.add_argument('--no-dots', action='store_true', help='skip the 64-dot batched leg')
    ap.add_argument('--dots', type=int, default=64)
    ap.add_argument('--dot-budget', type=int, default=20)
    ap.add_argument('--no-stream5', action='store_true', help='skip the antimonide stream leg')
    ap.add_argument('--stream5', type=int, default=12, help='requests of the antimonide stream')
    ap.add_argument('--stream5-budget', type=int, default=150)
    ap.add_argument('--form', choices=('served', 'plain'), default='served')
    ap.add_argument('--no-plain', action='store_true', help='skip the plain-form comparison')
    ap.add_argument('--no-e2e', action='store_true', help='skip the host-buffer end-to-end run')
    ap.add_argument('--no-stream', action='store_true', help='skip the Poisson-arrival run')
    ap.add_argument('--hx-probe', action='store_true',
                    help='only run a few H.X launches on a pyramid operator (profiling)')
    ap.add_argument('--hx-grid', choices=('48', '128'), default='48')
    ap.add_argument('--hx-m', type=int, default=12)
    ap.add_argument('--hx-dtype', choices=('c128', 'c64'), default='c128')
    ap.add_argument('--hx-tile', type=int, default=None)
    ap.add_argument('--hx-launches', type=int, default=3)
    ap.add_argument('--engine-probe', action='store_true',
                    help='only run the served engine for --probe-ticks ticks (profiling)')
    ap.add_argument('--probe-ticks', type=int, default=20)
    ap.add_argument('--probe-solves', default=None,
                    help='comma-separated solves of the probe (e.g. b10_vb); default all 14')
    ap.add_argument('--tick-probe', action='store_true',
                    help='only time lone-slot ticks and plain iterations (latency)')
    ap.add_argument('--probe-plain', action='store_true',
                    help='probe the plain drop-in (one solve after the other) instead')
    ap.add_argument('--ticks-per-poll', type=int, default=16)
    ap.add_argument('--mixed-tol', type=float, default=1e-4,
                    help='residual at which a mixed-precision solve leaves complex64')
    ap.add_argument('--precision', choices=('mixed', 'c128'), default='mixed',
                    help='served form: complex64 search + complex128 finish, or complex128 only')
    ap.add_argument('--cpu-solve', nargs=2, default=None, help=argparse.SUPPRESS)
    ap.add_argument('--cpu-sample', default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.cpu_solve or args.cpu_sample:
        cpu_child(args)
    elif args.hx_probe:
        hx_probe(args)
    elif args.engine_probe:
        engine_probe(args)
    elif args.tick_probe:
        tick_probe(args)
    elif args.impl == 'reference':
        run_reference(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
