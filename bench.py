"""Benchmark: batched Bloch-periodic kinetic operator + restrict/interpolate.

Workload (one "step"): 256 complex128 wave functions on a 96^3 periodic
grid, Bloch phases at k = (0.25, 0, 0.1), kinetic operator -1/2 Laplacian
(nn = 3, 19 points) applied to the whole batch, then Transformer restrict
(order 3, 96^3 -> 48^3) and interpolate (48^3 -> 96^3) of the same batch.
Inputs are N(0,1) + i N(0,1) from a fixed seed (synthetic).

Metric: FD-stencil GB/s = algorithmic bytes per step / device time, with
algorithmic bytes = every input read once + every output written once
(apply 32 B per point, restrict and interpolate 18 B per fine point).
Arrays are 3.6 GB each, far larger than L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank runs its own batch
(independent replicas, weak scaling); rank 0 prints the JSON line with the
whole-job GB/s over the max of the per-rank device times.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NBANDS = 256
N = (96, 96, 96)
CELL = (96 * 0.2 / 0.52917721,) * 3
KPT = (0.25, 0.0, 0.1)
METRIC = 'FD-stencil GB/s (kinetic nn=3 apply + restrict + interpolate)'
WORKLOAD = ('kinetic -0.5*Lap nn=3 on 256 complex128 96^3 periodic, Bloch '
            'k=(0.25,0,0.1) + Transformer restrict/interpolate nn=3')


def set_batch(nb):
    global NBANDS
    NBANDS = int(nb)


def algorithmic_bytes(nb=None):
    nb = NBANDS if nb is None else nb
    pts = nb * N[0] * N[1] * N[2]
    apply_b = 32 * pts
    restrict_b = 16 * pts + 16 * pts // 8
    interp_b = 16 * pts // 8 + 16 * pts
    return apply_b, restrict_b, interp_b


def measured_peak():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


def ncu_traffic():
    """DRAM bytes per apply launch from the committed ncu summary."""
    path = os.path.join(ROOT, 'profiles', 'fd_apply_c128_96cube.txt')
    try:
        for line in open(path):
            if line.startswith('dram_bytes_per_launch_full_batch:'):
                return float(line.split(':')[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed
    region (every 200 ms)."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,'
         'clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--id={self.index}',
                 f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                 '-lms', '200'], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        for l in getattr(self, 'lines', []):
            f = [x.strip() for x in l.split(',')]
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        return {'sm_mhz': float(np.median(sm)) if sm else None,
                'sm_max_mhz': smax, 'reasons': sorted(reasons),
                'samples': len(sm)}


def make_batch(nb, seed=0):
    rng = np.random.default_rng(seed)
    shape = (nb,) + N
    a = np.empty(shape, complex)
    a.real = rng.standard_normal(shape)
    a.imag = rng.standard_normal(shape)
    return a


# --------------------------------------------------------------- CPU sides
CPU_SAMPLE = 16   # wave functions per CPU step (bounded sample)


def cpu_step_child(nb, reps):
    """Run inside a fresh process: time the reference's own C core
    (oracle/_ref) on `nb` wave functions, `reps` times; print JSON."""
    from oracle import gpaw_layer as L
    kind = 'reference' if L._REF is not None else 'port'
    gd = L.GridDescriptor(N, CELL, 1)
    gd2 = gd.coarsen()
    ph = gd.phase_factor_cd(KPT)
    kin = L.Laplace(gd, -0.5, 3, complex)
    rst = L.Transformer(gd, gd2, 3, complex)
    itp = L.Transformer(gd2, gd, 3, complex)
    a = make_batch(nb, seed=1)
    b = np.empty_like(a)
    c = np.empty((nb,) + tuple(gd2.n_c), complex)
    d = np.empty_like(a)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        kin.apply(a, b, ph)
        rst.apply(a, c, phases=ph)
        itp.apply(c, d, phases=ph)
        times.append(time.perf_counter() - t0)
    print(json.dumps({'kind': kind, 'times': times, 'nb': nb}))


def cpu_measure(nb=CPU_SAMPLE, reps=3):
    cores = len(os.sched_getaffinity(0))
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), CUDA_VISIBLE_DEVICES='')
    out = subprocess.run(
        [sys.executable, os.path.abspath(__file__), '--_cpu-child', str(nb),
         str(reps)], env=env, capture_output=True, text=True, check=True,
        cwd=ROOT).stdout
    r = json.loads(out.strip().splitlines()[-1])
    t = float(np.median(r['times']))
    gbs = sum(algorithmic_bytes(nb)) / t / 1e9
    return {'value': gbs, 'unit': 'GB/s', 'cores': cores, 'kind': r['kind'],
            'sample': f'{nb} of {NBANDS} wave functions per step, median of '
                      f'{reps} steps ({t * 1e3:.1f} ms each), OpenMP over the '
                      f'batch with {cores} threads'}


# ------------------------------------------ CPU baselines of the Poisson path
def _c4_geometry(count, seed=0):
    """Sides and Gaussian counts of the C4 batch (the same draws as
    gpaw_b200.batch.c4_grids and poisson_c4)."""
    sides = np.random.default_rng(seed).choice(np.arange(32, 129, 8),
                                               size=(count, 3))
    rng = np.random.default_rng(1)
    ngs = [int(rng.integers(4, 17)) for _ in range(count)]
    return sides, ngs


def _c4_cpu_one(i):
    """One C4 grid solved by the reference's C core (oracle/_ref) to
    1e-10 relative residual; returns its V-cycle count."""
    from oracle import gpaw_layer as L
    from gpaw_b200.workloads import (BOHR, eps_for_relative_residual,
                                     gaussian_density, random_gaussians)
    sides, ngs = _c4_geometry(i + 1)
    h = 0.18 / BOHR
    Nc = tuple(int(x) for x in sides[i])
    gd = L.GridDescriptor(Nc, tuple(x * h for x in Nc), 0)
    rng = np.random.default_rng(100 + i)
    rho = gaussian_density(gd, *random_gaussians(gd, ngs[i], rng))
    rho = rho - rho.sum() / rho.size
    ps = L.FDPoissonSolver(nn=3, eps=eps_for_relative_residual(rho, gd),
                           maxiter=400)
    ps.set_grid_descriptor(gd)
    return ps.solve_neutral(gd.zeros(), rho)


def cpu_poisson_child(which, arg):
    """Fresh process: the reference's C core on a Poisson configuration;
    prints JSON.  c1: two solves (OMP threads from the environment), the
    potential saved to `arg` (.npy).  c4: the first `arg` grids of the C4
    batch over a pool of single-threaded processes, one per core."""
    from oracle import gpaw_layer as L
    kind = 'reference' if L._REF is not None else 'port'
    if which == 'c1':
        from gpaw_b200.workloads import BOHR, c1_density, neutralize
        h = 0.2 / BOHR
        gd = L.GridDescriptor((64, 64, 64), (64 * h,) * 3, 0)
        rho = neutralize(c1_density(gd), gd)
        ps = L.FDPoissonSolver(nn=3, eps=2e-10)
        ps.set_grid_descriptor(gd)
        times = []
        for _ in range(2):
            phi = gd.zeros()
            t0 = time.perf_counter()
            n = ps.solve_neutral(phi, rho)
            times.append(time.perf_counter() - t0)
        np.save(arg, phi)
        print(json.dumps({'kind': kind, 'times': times, 'niter': n}))
    else:
        import multiprocessing as mp
        count = int(arg)
        cores = len(os.sched_getaffinity(0))
        t0 = time.perf_counter()
        with mp.get_context('spawn').Pool(cores) as pool:
            ns = pool.map(_c4_cpu_one, range(count), chunksize=1)
        t = time.perf_counter() - t0
        print(json.dumps({'kind': kind, 'seconds': t, 'grids': count,
                          'workers': cores, 'vcycles': ns}))


def cpu_poisson(which, arg, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads),
               CUDA_VISIBLE_DEVICES='')
    out = subprocess.run(
        [sys.executable, os.path.abspath(__file__), '--_cpu-poisson-child',
         which, str(arg)], env=env, capture_output=True, text=True,
        check=True, cwd=ROOT).stdout
    return json.loads(out.strip().splitlines()[-1])


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    steps, warm = args.steps, args.warmup
    cb = cpu_measure(CPU_SAMPLE, reps=max(1, min(steps, 3)))
    line = {'metric': METRIC, 'value': cb['value'], 'unit': 'GB/s',
            'n_gpus': int(os.environ.get('WORLD_SIZE', '1')),
            'steps': steps, 'warmup': warm,
            'ms_per_step': sum(algorithmic_bytes(CPU_SAMPLE)) /
            (cb['value'] * 1e9) * 1e3,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'c128', 'data': 'synthetic',
            'config': {'workload': WORKLOAD, 'batch': NBANDS,
                       'grid': list(N), 'sample_batch': CPU_SAMPLE},
            'impl': 'reference', 'cpu_baseline': cb,
            'e2e': {'value': cb['value'], 'unit': 'GB/s',
                    'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- Poisson
def reference_gpu_c2(dev, kin, rst, itp, x, y, c, z, ph, nb, reps=5):
    """The reference's own GPU kernels (c/gpu/kernels, compiled for sm_100a
    from its sources into oracle/_ref by `make -C oracle gpu`) on the same
    C2 step, timed with CUDA events on the same stream: the GPU baseline
    beside this library's kernels.  Each call pastes the batch, block by
    block of 16 grids, into the reference's padded buffer, copies the
    periodic halos with their phases and runs its kernel, as its
    single-domain GPU path does.  Also the largest relative difference of
    its outputs from this library's (the reference's GPU kernels sum in
    their own order)."""
    import ctypes as C
    import torch
    path = os.path.join(ROOT, 'oracle', '_ref', 'libgpaw_ref_gpu.so')
    if not os.path.exists(path):
        return {'unavailable': 'oracle/_ref/libgpaw_ref_gpu.so not built'}
    lib = C.CDLL(path)
    vp, lp, dp = C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_double)
    lib.refgpu_operator_new.restype = vp
    lib.refgpu_operator_new.argtypes = [dp, lp, C.c_int, C.c_int, lp, lp,
                                        C.c_int]
    lib.refgpu_operator_apply.argtypes = [vp, vp, vp, C.c_int, dp]
    lib.refgpu_transformer_new.restype = vp
    lib.refgpu_transformer_new.argtypes = [lp, lp, C.c_int, lp, lp, lp, lp,
                                           C.c_int, C.c_int]
    lib.refgpu_transformer_apply.argtypes = [vp, vp, vp, C.c_int, dp]

    def longs(a):
        a = np.ascontiguousarray(np.asarray(a).ravel(), np.int64)
        return a, a.ctypes.data_as(lp)

    def dbls(a):
        a = np.ascontiguousarray(np.asarray(a, float).ravel())
        return a, a.ctypes.data_as(dp)

    keep = []
    co, co_p = dbls(kin.coef_p)
    of, of_p = longs(kin.offset_p)
    sz, sz_p = longs(kin.gd.n_c)
    ne, ne_p = longs(kin.gd.neighbor_cd)
    keep += [co, of, sz, ne]
    hop = lib.refgpu_operator_new(co_p, of_p, len(kin.coef_p), int(kin.mp),
                                  sz_p, ne_p, 0)

    def transformer(t):
        si, si_p = longs(t.gdin.n_c)
        so, so_p = longs(t.gdout.n_c)
        pa, pa_p = longs(t.pad_cd)
        npd, npd_p = longs(t.neighborpad_cd)
        sk, sk_p = longs(t.skip_cd)
        nbr, nbr_p = longs(t.gdin.neighbor_cd)
        keep.extend([si, so, pa, npd, sk, nbr])
        return lib.refgpu_transformer_new(si_p, so_p, 2 * t.nn, pa_p, npd_p,
                                          sk_p, nbr_p, 0, int(t.interpolate))

    hr, hi = transformer(rst), transformer(itp)
    if not (hop and hr and hi):
        return {'unavailable': 'reference GPU objects could not be built'}
    phv, ph_p = dbls(np.column_stack([np.asarray(ph).real.ravel(),
                                      np.asarray(ph).imag.ravel()]))
    keep.append(phv)
    ry, rc, rz = torch.empty_like(y), torch.empty_like(c), torch.empty_like(z)
    calls = {
        'apply': lambda: lib.refgpu_operator_apply(
            hop, vp(x.data_ptr()), vp(ry.data_ptr()), nb, ph_p),
        'restrict': lambda: lib.refgpu_transformer_apply(
            hr, vp(x.data_ptr()), vp(rc.data_ptr()), nb, ph_p),
        'interpolate': lambda: lib.refgpu_transformer_apply(
            hi, vp(c.data_ptr()), vp(rz.data_ptr()), nb, ph_p)}
    ab, rb, ib = algorithmic_bytes(nb)
    nbytes = {'apply': ab, 'restrict': rb, 'interpolate': ib}
    out = {'how': 'reference c/gpu/kernels for sm_100a, blocks of 16 '
                  'grids, paste + halo copies + kernel per block'}
    st = torch.cuda.current_stream()
    for k, f in calls.items():
        if f() != 0:
            return {'unavailable': f'reference GPU {k} failed'}
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            f()
        e1.record(st)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        out[k] = {'ms': t * 1e3, 'gbs': nbytes[k] / t / 1e9}
    # ours on the same inputs (the step just ran: y, c, z hold them)
    kin.apply(x, y, ph)
    rst.apply(x, c, phases=ph)
    itp.apply(c, z, phases=ph)
    for k, (a, b) in {'apply': (ry, y), 'restrict': (rc, c),
                      'interpolate': (rz, z)}.items():
        out[k]['max_rel_diff_vs_ours'] = float((a - b).abs().max() /
                                               b.abs().max())
    return out


def poisson_c1(dev, nsolve=20, cpu=True):
    """64^3 zero-BC FDPoissonSolver (nn = 3, Jacobi, reference schedule),
    h = 0.2 A, 8 Gaussians: solves/s at the reference's eps = 2e-10 and at
    the eps that gives 1e-10 relative residual."""
    import torch
    from gpaw_b200 import FDPoissonSolver, GridDescriptor
    from gpaw_b200.workloads import (BOHR, c1_density,
                                     eps_for_relative_residual, neutralize)
    h = 0.2 / BOHR
    gd = GridDescriptor((64, 64, 64), (64 * h,) * 3, 0, device=dev)
    rho = neutralize(c1_density(gd), gd)
    rho_d = torch.from_numpy(rho).to(dev)
    rnorm = float(np.sqrt((rho * rho).sum()))
    out = {'grid': [64, 64, 64], 'h_angstrom': 0.2, 'precision': 'fp64'}
    for tag, eps in (('eps_2e-10', 2e-10),
                     ('rel_1e-10', eps_for_relative_residual(rho, gd))):
        ps = FDPoissonSolver(nn=3, relax='J', eps=eps)
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        ps.solve_neutral(phi, rho_d)          # warm-up (builds the graph)
        times = []
        for _ in range(nsolve):
            phi.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            n = ps.solve_neutral(phi, rho_d)
            times.append(time.perf_counter() - t0)
        r = torch.empty_like(phi)
        n2 = torch.zeros(1, dtype=torch.float64, device=dev)
        ps.operators[0].residual(phi, rho_d, r, None, 1.0, n2)
        rel = float(np.sqrt(n2.item())) / rnorm
        t = float(np.median(times))
        out[tag] = {'eps': eps, 'vcycles': n, 'ms_per_solve': t * 1e3,
                    'solves_per_s': 1.0 / t, 'rel_residual': rel,
                    'p50_ms': t * 1e3,
                    'p99_ms': float(np.percentile(times, 99)) * 1e3}
        if tag == 'eps_2e-10' and cpu:
            out[tag]['cpu_reference'] = c1_cpu(phi.cpu().numpy(), n)
    return out


def c1_apply(dev, reps=50):
    """The C1 stand-alone apply: one FDOperator.apply of the Poisson
    solver's Laplacian (nn = 3, scaled by -1/(4 pi)) on a seeded N(0,1)
    float64 array of the 64^3 zero-boundary grid (63^3 unknowns).  The
    array (4 MB) fits in L2, so L2 is flushed (a 256 MB write) before every
    timed launch; each launch is timed on its own with CUDA events.  Also
    reported: the same launch back to back with the array L2-resident."""
    import torch
    from gpaw_b200 import GridDescriptor, Laplace
    from gpaw_b200.workloads import BOHR
    h = 0.2 / BOHR
    gd = GridDescriptor((64, 64, 64), (64 * h,) * 3, 0, device=dev)
    op = Laplace(gd, -0.25 / np.pi, 3)
    rng = np.random.default_rng(0)
    a = torch.from_numpy(rng.standard_normal(tuple(gd.n_c))).to(dev)
    b = torch.empty_like(a)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream()
    for _ in range(5):
        op.apply(a, b)
    # The host takes longer to issue a launch through the Python API than
    # the kernel runs, so a short device-side wait is queued in front of
    # each timed region: the events then bracket the kernel's device time
    # instead of the host's launch latency.
    hold = int(2e-4 * 1.9e9)           # about 0.2 ms of SM cycles
    cold = []
    for _ in range(reps):
        flush.fill_(1)
        torch.cuda._sleep(hold)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        op.apply(a, b)
        e1.record(st)
        e1.synchronize()
        cold.append(e0.elapsed_time(e1) / 1e3)
    torch.cuda._sleep(hold * 20)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        op.apply(a, b)
    e1.record(st)
    e1.synchronize()
    hot = e0.elapsed_time(e1) / 1e3 / reps
    t = float(np.median(cold))
    nbytes = 16 * a.numel()
    peak, _ = measured_peak()
    return {'grid': [63, 63, 63], 'dtype': 'f64', 'nn': 3,
            'us': t * 1e6, 'gbs': nbytes / t / 1e9,
            'frac': nbytes / t / 1e9 / peak,
            'us_l2_resident': hot * 1e6, 'gbs_l2_resident': nbytes / hot / 1e9,
            'how': 'median of %d launches, L2 flushed before each, a device '
                   'wait queued ahead so that the events time the kernel, '
                   'not the host launch' % reps}


def c1_cpu(phi_gpu, n_gpu):
    """The same C1 solve by the reference's C core on the host cores (one
    thread and all threads, the better reported) and the GPU potential's
    max error against it."""
    import tempfile
    cores = len(os.sched_getaffinity(0))
    best = None
    fd, path = tempfile.mkstemp(suffix='.npy')
    os.close(fd)
    try:
        for threads in sorted({1, cores}):
            r = cpu_poisson('c1', path, threads)
            t = float(min(r['times']))
            if best is None or t < best['ms_per_solve'] / 1e3:
                phi_cpu = np.load(path)
                err = float(np.abs(phi_gpu - phi_cpu).max() /
                            np.abs(phi_cpu).max())
                best = {'ms_per_solve': t * 1e3, 'solves_per_s': 1.0 / t,
                        'threads': threads, 'cores': cores,
                        'kind': r['kind'], 'vcycles': r['niter'],
                        'same_vcycles_as_gpu': r['niter'] == n_gpu,
                        'max_rel_err_gpu_vs_cpu': err}
    finally:
        os.unlink(path)
    return best


def poisson_c3(dev, nsolve=5, which=('fp64', 'mixed4', 'mixed6')):
    """192^3 zero-BC, h = 0.18 A, 64 Gaussians: plain FP64 V-cycle with the
    reference schedule (7 grids) versus FP32 V-cycles in FP64 defect
    correction, both to 1e-10 relative residual.  The mixed solver runs
    with the stated 4 levels (2 + 2 smoothing sweeps); a 6-level variant is
    reported beside it (coarsest grid 5^3 instead of 23^3)."""
    import torch
    from gpaw_b200 import FDPoissonSolver, GridDescriptor, MixedPoissonSolver
    from gpaw_b200.workloads import (BOHR, c3_density,
                                     eps_for_relative_residual, neutralize)
    h = 0.18 / BOHR
    gd = GridDescriptor((192, 192, 192), (192 * h,) * 3, 0, device=dev)
    rho = neutralize(c3_density(gd, 64), gd)
    rho_d = torch.from_numpy(rho).to(dev)
    rnorm = float(np.sqrt((rho * rho).sum()))
    fp64 = FDPoissonSolver(nn=3, relax='J',
                           eps=eps_for_relative_residual(rho, gd))
    fp64.set_grid_descriptor(gd)
    mixed4 = MixedPoissonSolver(nn=3, tol=1e-10, levels=4)
    mixed4.set_grid_descriptor(gd)
    mixed6 = MixedPoissonSolver(nn=3, tol=1e-10, levels=6)
    mixed6.set_grid_descriptor(gd)
    out = {'grid': [192, 192, 192], 'h_angstrom': 0.18, 'gaussians': 64}
    phis = {}
    for tag, ps in (('fp64_reference_schedule', fp64),
                    ('mixed_4_levels', mixed4),
                    ('mixed_6_levels', mixed6)):
        if {'fp64_reference_schedule': 'fp64', 'mixed_4_levels': 'mixed4',
                'mixed_6_levels': 'mixed6'}[tag] not in which:
            continue
        phi = gd.zeros()
        ps.solve_neutral(phi, rho_d)      # warm-up (builds the graph)
        times = []
        for _ in range(nsolve):
            phi.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            n = ps.solve_neutral(phi, rho_d)
            times.append(time.perf_counter() - t0)
        r = torch.empty_like(phi)
        n2 = torch.zeros(1, dtype=torch.float64, device=dev)
        fp64.operators[0].residual(phi, rho_d, r, None, 1.0, n2)
        t = float(np.median(times))
        phis[tag] = phi
        out[tag] = {'vcycles': n, 'ms_per_solve': t * 1e3,
                    'solves_per_s': 1.0 / t,
                    'rel_residual': float(np.sqrt(n2.item())) / rnorm}
    if len(phis) < 3:
        return out
    b = phis['fp64_reference_schedule']
    for lv in (4, 6):
        a = phis[f'mixed_{lv}_levels']
        out[f'mixed_{lv}_levels']['max_rel_diff_vs_fp64'] = float(
            (a - b).abs().max() / b.abs().max())
        out[f'speedup_mixed_{lv}_over_fp64'] = (
            out[f'mixed_{lv}_levels']['solves_per_s'] /
            out['fp64_reference_schedule']['solves_per_s'])
    return out


def mixed_vcycle_trace(dev, levels=4, reps=5):
    """Per-kernel device times of one mixed-precision V-cycle on the C3 grid
    (the 4-level FP32 V-cycle inside its FP64 defects), launched kernel by
    kernel through gb_mixed_vcycle_eager under the library's kernel trace;
    mean over `reps` V-cycles."""
    import ctypes as C
    import torch
    from gpaw_b200 import GridDescriptor, MixedPoissonSolver, _lib
    from gpaw_b200.workloads import BOHR, c3_density, neutralize
    h = 0.18 / BOHR
    gd = GridDescriptor((192, 192, 192), (192 * h,) * 3, 0, device=dev)
    rho = torch.from_numpy(neutralize(c3_density(gd, 64), gd)).to(dev)
    ps = MixedPoissonSolver(nn=3, tol=1e-10, levels=levels)
    ps.set_grid_descriptor(gd)
    phi = gd.zeros()
    ps.solve_neutral(phi, rho)          # builds the graph, sets attributes
    phi.zero_()
    lib = _lib.load()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (ps._h.h, C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()),
            st)
    _lib.check(lib.gb_mixed_vcycle_eager(*args))
    torch.cuda.synchronize()
    with _lib.KernelTrace() as tr:
        for _ in range(reps):
            _lib.check(lib.gb_mixed_vcycle_eager(*args))
    per = {}
    for label, ms in tr.intervals:
        if label == 'end of defect':
            continue
        per.setdefault(label, []).append(ms)
    rows = sorted(((k, float(np.sum(v)) / reps) for k, v in per.items()),
                  key=lambda kv: -kv[1])
    return {'levels': levels, 'grid': [192, 192, 192],
            'ms_per_vcycle_with_defects': sum(v for _, v in rows),
            'kernels_ms': [[k, round(v, 4)] for k, v in rows]}


def poisson_c4(dev, count=512, precisions=('mixed', 'fp64'), cpu=True):
    """512 zero-BC grids, every side from {32, 40, ..., 128}, each with 4-16
    seeded Gaussians (C3 distributions), solved to 1e-10 relative residual:
    every solve enqueued on one of 16 streams, one synchronisation."""
    import torch
    from gpaw_b200.batch import PoissonBatch, c4_grids
    from gpaw_b200.workloads import neutral_density_device
    gds = c4_grids(count, seed=0, device=dev)
    rng = np.random.default_rng(1)
    rhos = [neutral_density_device(gd, int(rng.integers(4, 17)), 100 + i)
            for i, gd in enumerate(gds)]
    npts = sum(int(np.prod(gd.n_c)) for gd in gds)
    out = {'grids': count, 'points': npts,
           'sides': '{32,40,...,128} per axis, zero BC, h = 0.18 A'}
    for prec in precisions:
        t0 = time.perf_counter()
        batch = PoissonBatch(gds, tol=1e-10, precision=prec, nstreams=16)
        phis = [gd.zeros() for gd in gds]
        batch.prepare(rhos)
        batch.solve(phis, rhos)                # warm-up: builds the graphs
        setup = time.perf_counter() - t0
        for p in phis:
            p.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n = batch.solve(phis, rhos)
        t = time.perf_counter() - t0
        out[prec] = {'solves_per_s': count / t, 'seconds': t,
                     'vcycles_mean': float(np.mean(n)),
                     'vcycles_max': int(np.max(n)), 'setup_s': setup}
        del batch
    if 'mixed' in out and 'fp64' in out:
        out['speedup_mixed_over_fp64'] = (out['mixed']['solves_per_s'] /
                                          out['fp64']['solves_per_s'])
    if cpu:
        cores = len(os.sched_getaffinity(0))
        ncpu = min(count, cores)
        r = cpu_poisson('c4', ncpu, 1)
        out['cpu_reference'] = {
            'solves_per_s': r['grids'] / r['seconds'], 'kind': r['kind'],
            'sample': f'first {r["grids"]} grids of the batch, FP64 '
                      f'reference schedule to 1e-10, {r["workers"]} '
                      f'single-threaded processes',
            'cores': r['workers'], 'vcycles_mean': float(np.mean(r['vcycles']))}
    return out


# Algorithmic bytes per fine grid point of each kernel of the fd_precond
# sequence (gpaw/preconditioner.py:74-93 as gb_fd_precond fuses it), for
# float64 data of 8 B: level 1 has 1/8 of the fine points, level 2 1/64.
PRECOND_BYTES_PER_FINE_PT = {
    'restrict0': 8 + 2 * 8 / 8,            # R in; r1, d1 out
    'kin1 q1 = K1': 3 * 8 / 8,              # d1, r1 in; q1 out
    'restrict1': 8 / 8 + 2 * 8 / 64,        # q1 in; r2, d2 out
    'kin2': 3 * 8 / 64,                     # d2, r2 in; q2 out
    'interp2': 8 / 64 + 2 * 8 / 8,          # q2, d1 in; d1 out
    'kin1 q1 = d1': 3 * 8 / 8,              # d1, r1 in; q1 out
    'interp1': 8 / 8 + 8,                   # q1 in; q0 out
    'kin0': 3 * 8,                          # q0, R in; d0 out
}


def _precond_key(label):
    for k in PRECOND_BYTES_PER_FINE_PT:
        if label.startswith(k):
            return k
    return label


def precond_c4(dev, nbands=128):
    """Preconditioner (gpaw/preconditioner.py) on 128 float64 band residuals,
    112^3 periodic (Gamma point), kinetic operator nn = 3: time per call,
    the black-box figure (R in, d0 out: 16 B/pt) and the per-kernel times
    and bytes of the executed sequence (the library's kernel trace)."""
    import torch
    from gpaw_b200 import GridDescriptor, Laplace, Preconditioner
    from gpaw_b200._lib import KernelTrace
    from gpaw_b200.workloads import BOHR
    N = (112, 112, 112)
    gd = GridDescriptor(N, (112 * 0.18 / BOHR,) * 3, 1, device=dev)
    pc = Preconditioner(gd, Laplace(gd, -0.5, 3), float, block=nbands)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    R = torch.randn((nbands,) + N, dtype=torch.float64, device=dev,
                    generator=g)
    out = torch.empty_like(R)
    for _ in range(2):
        pc(R, None, out=out)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record()
    for _ in range(reps):
        pc(R, None, out=out)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    with KernelTrace() as tr:
        for _ in range(reps):
            pc(R, None, out=out)
    per = {}
    for label, ms in tr.intervals:
        per.setdefault(_precond_key(label), []).append(ms)
    npts = R.numel()
    kernels = []
    seq_bytes = 0.0
    for k, bpp in PRECOND_BYTES_PER_FINE_PT.items():
        ms = float(np.mean(per.get(k, [float('nan')])))
        nb = bpp * npts
        seq_bytes += nb
        kernels.append({'kernel': k, 'ms': ms, 'bytes': nb,
                        'gbs': nb / ms / 1e6})
    ksum = sum(k['ms'] for k in kernels) / 1e3
    return {'bands': nbands, 'grid': list(N), 'ms_per_call': t * 1e3,
            'blackbox_gbs': 16 * npts / t / 1e9,
            'sequence_bytes': seq_bytes,
            'sequence_gbs': seq_bytes / t / 1e9,
            'kernel_sum_ms': ksum * 1e3, 'kernels': kernels}


def weighted_fd(dev, reps=10, cpu=True):
    """The solvation solver's weighted operator (WeightedFDOperator: nn = 3
    Laplacian and the three Gradients weighted by eps and its gradient,
    gpaw/old/solvation/poisson.py:80-85) on one 192^3 zero-BC float64 grid:
    apply and one weighted-Jacobi sweep, GB/s of the algorithmic bytes
    (apply: in + out + 4 weights = 48 B/pt; sweep: phi in + rho + phi out
    + 4 weights = 56 B/pt).  Arrays total 0.5 GB, larger than L2."""
    import torch
    from gpaw_b200 import Gradient, GridDescriptor, Laplace
    from gpaw_b200.wfd_operators import WeightedFDOperator
    N = (192, 192, 192)
    gd = GridDescriptor(N, (N[0] * 0.18 / 0.52917721,) * 3, 0, device=dev)
    scale = -0.25 / np.pi
    ops = [Laplace(gd, scale, 3)] + [Gradient(gd, v, scale, 3)
                                     for v in range(3)]
    wop = WeightedFDOperator(ops)
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    shape = tuple(int(n) for n in gd.n_c)
    eps = 1.0 + 77.0 * torch.rand(shape, dtype=torch.float64, device=dev,
                                  generator=g)
    w = [eps] + [torch.randn(shape, dtype=torch.float64, device=dev,
                             generator=g) for _ in range(3)]
    wop.set_weights(w)
    x = torch.randn(shape, dtype=torch.float64, device=dev, generator=g)
    y = torch.empty_like(x)
    rho = torch.randn(shape, dtype=torch.float64, device=dev, generator=g)
    npts = x.numel()
    out = {'grid': list(N), 'operators': 'Laplace nn=3 + 3 Gradients nn=3',
           'weights': 4}

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    t = timed(lambda: wop.apply(x, y))
    out['apply'] = {'ms': t * 1e3, 'gbs': 48 * npts / t / 1e9}
    t = timed(lambda: wop.relax(2, x, rho, 2, 2.0 / 3.0)) / 2
    out['jacobi_sweep'] = {'ms': t * 1e3, 'gbs': 56 * npts / t / 1e9}
    if cpu:
        # the reference's WOperator on the host (one grid: its OpenMP
        # region splits the batch, so one thread works) and the GPU
        # result's max error against it
        from oracle import gpaw_layer as L
        be = 'ref' if L._REF is not None else 'port'
        gdo = L.GridDescriptor(N, gd.cell_cv, 0)
        wo = L.WeightedFDOperator([L.FDOperator(op.coef_p, op.offset_pc, gdo,
                                                be=be) for op in ops], be=be)
        wo.set_weights([a.cpu().numpy() for a in w])
        xin = x.cpu().numpy()
        ref = np.zeros_like(xin)
        wop.apply(x, y)
        got = y.cpu().numpy()
        ts = []
        for _ in range(2):
            t0 = time.perf_counter()
            wo.apply(xin, ref)
            ts.append(time.perf_counter() - t0)
        t = min(ts)
        out['cpu_reference'] = {
            'apply_ms': t * 1e3, 'gbs': 48 * npts / t / 1e9, 'threads': 1,
            'kind': 'reference' if be == 'ref' else 'port',
            'max_rel_err_gpu_vs_cpu': float(np.abs(got - ref).max() /
                                            np.abs(ref).max())}
    out['poisson_dielectric_64'] = weighted_poisson(dev, cpu=cpu)
    return out


def weighted_poisson(dev, nsolve=5, cpu=True):
    """WeightedFDPoissonSolver (gpaw/old/solvation/poisson.py:75-124) on the
    C1 grid (64^3 zero BC, h = 0.2 A) with a dielectric of 1 inside a
    sphere and 80 outside, to the reference's eps = 2e-10: ms per solve,
    V-cycles, and the reference's C core (WOperator + Transformer, one
    host thread) on the same solve with the GPU potential's max error."""
    import torch
    from gpaw_b200 import Gradient, GridDescriptor, Laplace
    from gpaw_b200.solvation import WeightedFDPoissonSolver
    from gpaw_b200.workloads import BOHR, c1_density, neutralize
    h = 0.2 / BOHR
    N = (64, 64, 64)
    cell = (64 * h,) * 3
    gd = GridDescriptor(N, cell, 0, device=dev)
    rho = neutralize(c1_density(gd), gd)
    x = np.stack([a.cpu().numpy() if hasattr(a, 'cpu') else a
                  for a in gd.get_grid_point_coordinates()]) - 32 * h
    w2 = (8 * h) ** 2
    g = np.exp(-(x**2).sum(0) / w2)
    arrays = [80.0 - 79.0 * g] + [79.0 * g * 2.0 * x[c] / w2 for c in range(3)]

    class Dielectric:
        eps_gradeps = [torch.from_numpy(a).to(dev) for a in arrays]

    ps = WeightedFDPoissonSolver(nn=3, eps=2e-10)
    ps.set_grid_descriptor(gd)
    ps.set_dielectric(Dielectric())
    ps.restrict_op_weights()
    rho_d = torch.from_numpy(rho).to(dev)
    phi = gd.zeros()
    ps.solve_neutral(phi, rho_d)
    times = []
    for _ in range(nsolve):
        phi.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n = ps.solve_neutral(phi, rho_d)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    out = {'grid': list(N), 'eps': 2e-10, 'vcycles': n, 'ms_per_solve': t * 1e3,
           'solves_per_s': 1.0 / t}
    if cpu:
        from oracle import gpaw_layer as L
        be = 'ref' if L._REF is not None else 'port'
        gdo = L.GridDescriptor(N, cell, 0)

        def stencils(g_, scale, nn):
            gp = GridDescriptor(tuple(g_.N_c), cell, 0, device=dev)
            ops = [Laplace(gp, scale, nn)] + [Gradient(gp, j, scale, nn)
                                              for j in range(3)]
            return [(op.coef_p, op.offset_pc) for op in ops]

        wo = L.WeightedFDPoissonSolver(stencils, nn=3, eps=2e-10, be=be)
        wo.set_grid_descriptor(gdo)
        wo.set_dielectric(arrays)
        wo.restrict_op_weights()
        phi_o = gdo.zeros()
        t0 = time.perf_counter()
        n_o = wo.solve_neutral(phi_o, rho)
        tc = time.perf_counter() - t0
        got = phi.cpu().numpy()
        out['cpu_reference'] = {
            'ms_per_solve': tc * 1e3, 'threads': 1,
            'kind': 'reference' if be == 'ref' else 'port', 'vcycles': n_o,
            'same_vcycles_as_gpu': n_o == n,
            'max_rel_err_gpu_vs_cpu': float(np.abs(got - phi_o).max() /
                                            np.abs(phi_o).max())}
    return out


def serving_c5(dev, rates=(50, 100, 200, 500, 1000, 2000), count=1000,
               warm_count=200):
    """Poisson-arrival stream of mixed-precision Poisson solves (to 1e-10)
    and nn = 3 stencil applications, grid sides log-uniform in [24, 160]
    (multiples of 8), admitted against a 16 GB budget, 8 slots, three
    resident solvers per shape; `count` requests per rate, after an
    untimed pass of `warm_count` requests at the same rate."""
    from gpaw_b200.serving import Server, latency_stats, make_requests
    # every shape of the stream has resident solvers (graphs captured)
    # before serving starts; the loop never builds one while it serves
    import gc
    import torch
    gc.collect()
    torch.cuda.empty_cache()        # what earlier sections left cached
    srv = Server(hbm_budget=16 << 30, nslots=8, device=dev, grow=False)
    srv.warm([(s, s, s) for s in range(24, 161, 8)], per_shape=3)
    # one untimed burst at the highest rate first: every slot stream and
    # resident solver has run before any timed stream
    burst = make_requests(max(rates), 4 * warm_count, seed=99)
    srv.run(burst, {r.rid: srv.host_input(r) for r in burst})
    out = {'slots': 8, 'hbm_budget_gb': 16, 'requests_per_rate': count}
    for lam in rates:
        warm = make_requests(lam, warm_count, seed=10_000 + lam)
        srv.run(warm, {r.rid: srv.host_input(r) for r in warm})
        reqs = make_requests(lam, count, seed=lam)
        inputs = {r.rid: srv.host_input(r) for r in reqs}
        srv.run(reqs, inputs)
        st = latency_stats(reqs)
        st['poisson_vcycles_mean'] = float(np.mean(
            [r.niter for r in reqs if r.kind == 'poisson'] or [0]))
        out[f'lambda_{lam}'] = st
    # anisotropic stream: every axis draws its own side (18^3 possible
    # shapes), so solvers are built on demand while serving and the least
    # recently used are evicted under the budget; warmed by an untimed
    # stream of other draws
    del srv
    gc.collect()
    torch.cuda.empty_cache()
    srv = Server(hbm_budget=16 << 30, nslots=8, device=dev, grow=True)
    warm = make_requests(200, 300, seed=7, anisotropic=True)
    srv.run(warm, {r.rid: srv.host_input(r) for r in warm})
    aniso = {'requests_per_rate': 500}
    for lam in (50, 200, 1000):
        reqs = make_requests(lam, 500, seed=20_000 + lam, anisotropic=True)
        inputs = {r.rid: srv.host_input(r) for r in reqs}
        b0, e0 = srv.built, srv.evicted
        srv.run(reqs, inputs)
        st = latency_stats(reqs)
        st['solvers_built'] = srv.built - b0
        st['solvers_evicted'] = srv.evicted - e0
        aniso[f'lambda_{lam}'] = st
    out['anisotropic'] = aniso
    return out


def serving_subprocess():
    out = subprocess.run(
        [sys.executable, os.path.abspath(__file__), '--poisson-only', 'c5'],
        capture_output=True, text=True, check=True, cwd=ROOT,
        env=dict(os.environ)).stdout
    return json.loads(out.strip().splitlines()[-1])


# ---------------------------------------------------------------- GPU side
def run_gpu(args):
    import torch
    import torch.distributed as dist

    from gpaw_b200 import GridDescriptor, Laplace, Transformer
    from gpaw_b200.replicas import max_over_ranks

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(
            seconds=120), device_id=dev)

    # CPU baseline before any heavy GPU work (rank 0, N = 1 only)
    cpu_base = cpu_measure() if (rank == 0 and world == 1 and
                                 not args.no_cpu) else None

    gd = GridDescriptor(N, CELL, 1, device=dev)
    gd2 = gd.coarsen()
    ph = gd.phase_factor_cd(KPT)
    kin = Laplace(gd, -0.5, 3, complex)
    rst = Transformer(gd, gd2, 3, complex)
    itp = Transformer(gd2, gd, 3, complex)

    host = make_batch(NBANDS, seed=rank)
    x = torch.from_numpy(host).to(dev)
    y = torch.empty_like(x)
    c = torch.empty((NBANDS,) + tuple(gd2.n_c), dtype=torch.complex128,
                    device=dev)
    z = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    # z-block depths of the three kernels picked by timing (autotuner)
    from gpaw_b200 import autotune
    depth = {'apply': autotune.tune_operator(kin, x, y, ph, reps=2)[0],
             'restrict': autotune.tune_transformer(rst, x, c, ph, reps=2)[0],
             'interpolate': autotune.tune_transformer(itp, c, z, ph,
                                                      reps=2)[0]}

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        kin.apply(x, y, ph)
        if ev is not None:
            ev[1].record(stream)
        rst.apply(x, c, phases=ph)
        if ev is not None:
            ev[2].record(stream)
        itp.apply(c, z, phases=ph)
        if ev is not None:
            ev[3].record(stream)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
           for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t_end.record(stream)
        barrier()
    elapsed = t_start.elapsed_time(t_end) / 1e3
    apply_s = [e[0].elapsed_time(e[1]) / 1e3 for e in evs]
    rst_s = [e[1].elapsed_time(e[2]) / 1e3 for e in evs]
    itp_s = [e[2].elapsed_time(e[3]) / 1e3 for e in evs]
    if world > 1:
        elapsed = max_over_ranks(elapsed, device=dev)

    ab, rb, ib = algorithmic_bytes()
    per_step = ab + rb + ib
    value = world * per_step * args.steps / elapsed / 1e9

    # end-to-end through the public API: pinned host in, results back out,
    # streamed in chunks of bands with the copies overlapped (StepPipeline)
    e2e = None
    if not args.no_e2e:
        from gpaw_b200.pipeline import StepPipeline
        hin = torch.from_numpy(host).pin_memory()
        hy = torch.empty(y.shape, dtype=y.dtype).pin_memory()
        hz = torch.empty(z.shape, dtype=z.dtype).pin_memory()
        hc = torch.empty(c.shape, dtype=c.dtype).pin_memory()
        e_steps = max(1, min(3, args.steps))
        pipe = StepPipeline(kin, rst, itp, chunk=32, device=dev)
        pipe.run(hin, hy, hc, hz, ph)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e_steps):
            pipe.run(hin, hy, hc, hz, ph)
        stream.wait_stream(pipe.s_out)
        e1.record(stream)
        barrier()
        et = e0.elapsed_time(e1) / 1e3
        if world > 1:
            et = max_over_ranks(et, device=dev)
        e2e = {'value': world * per_step * e_steps / et / 1e9, 'unit': 'GB/s',
               'h2d_bytes_per_step': int(x.numel() * 16),
               'd2h_bytes_per_step': int((y.numel() + c.numel() +
                                          z.numel()) * 16),
               'how': 'gpaw_b200.pipeline.StepPipeline, chunks of 32 bands, '
                      'copy-in / compute / copy-out overlapped'}

    peak, peak_src = measured_peak()
    apply_t = float(np.mean(apply_s))
    achieved = ab / apply_t / 1e9
    rst_t = float(np.mean(rst_s))
    itp_t = float(np.mean(itp_s))
    line = {
        'metric': METRIC, 'value': value, 'unit': 'GB/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': elapsed / args.steps * 1e3,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'c128', 'data': 'synthetic',
        'config': {'workload': WORKLOAD, 'batch': NBANDS, 'grid': list(N),
                   'parallelism': f'replicas x{world}',
                   'l2': 'inputs 3.6 GB per array, larger than L2 (no flush)',
                   'z_block_depth': {k: (v or 'auto') for k, v in depth.items()}},
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                     'unit': 'GB/s', 'frac': achieved / peak,
                     'traffic': ncu_traffic(), 'kernel': 'fd apply c128',
                     'peak_source': peak_src},
        'gpu_launches': 3 * args.steps,
        'clocks': clk.summary(),
        'e2e': e2e,
        'cpu_baseline': cpu_base,
    }
    ref_gpu = None
    if (rank == 0 or world == 1) and not args.no_ref_gpu:
        ref_gpu = reference_gpu_c2(dev, kin, rst, itp, x, y, c, z, ph, NBANDS)
    detail = {'c2': {'kernels_ms': {'apply': apply_t * 1e3,
                                    'restrict': rst_t * 1e3,
                                    'interpolate': itp_t * 1e3},
                     'kernels_gbs': {'apply': achieved,
                                     'restrict': rb / rst_t / 1e9,
                                     'interpolate': ib / itp_t / 1e9}}}
    if ref_gpu is not None:
        detail['c2']['reference_gpu'] = ref_gpu
    # FD Hamiltonian local part on the same batch: kin(psi) + v psi fused
    if (rank == 0 or world == 1) and not args.no_ham:
        from gpaw_b200 import FDHamiltonian
        ham = FDHamiltonian(gd, kin_stencil=3, dtype=complex)
        vt = torch.randn(tuple(gd.n_c), dtype=torch.float64, device=dev)
        ham.apply_local_potential(vt, x, y, ph)
        h0 = torch.cuda.Event(enable_timing=True)
        h1 = torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for _ in range(5):
            ham.apply_local_potential(vt, x, y, ph)
        h1.record(stream)
        torch.cuda.synchronize()
        ht = h0.elapsed_time(h1) / 1e3 / 5
        hb = ab + vt.numel() * 8
        detail['c2']['hamiltonian'] = {
            'what': 'kin(psi) + v psi, 256 x 96^3 complex128, one kernel',
            'ms': ht * 1e3, 'gbs': hb / ht / 1e9,
            'vs_apply_alone': ht / apply_t}
    # CPU references of the Poisson path: rank 0 at N = 1 only.  The
    # Poisson, batch and serving sections are single-GPU configurations:
    # they run at N = 1 (the scaling runs time the C2 step alone).
    cpu_ok = not args.no_cpu and rank == 0 and world == 1
    single = world == 1
    if not args.no_poisson and single:
        detail['c1'] = poisson_c1(dev, cpu=cpu_ok)
        detail['c1']['apply'] = c1_apply(dev)
        detail['c3'] = poisson_c3(dev)
        detail['wfd'] = weighted_fd(dev, cpu=cpu_ok)
    if not args.no_batch and single:
        detail['c4'] = poisson_c4(dev, cpu=cpu_ok)
        detail['pc'] = precond_c4(dev)
    if not args.no_serving and single:
        # in a fresh process: the host-driven loop's latencies should not
        # depend on what this process did before (measured: they do)
        detail['c5'] = serving_subprocess()
    line['configs'] = summarize(detail, peak)
    if args.detail and rank == 0:
        with open(args.detail, 'w') as f:
            json.dump({'line': line, 'detail': detail}, f, indent=1)
    if rank == 0:
        print(json.dumps(line, separators=(',', ':')), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _g(x, digits=4):
    """Round for the compact summary."""
    if x is None:
        return None
    if isinstance(x, bool) or isinstance(x, int):
        return x
    return float(f'{x:.{digits}g}')


def summarize(d, peak):
    """A compact per-configuration summary (a few hundred bytes) of the
    detailed results, so that the figure of every configuration fits the
    end of the JSON line."""
    out = {}
    c2 = d.get('c2')
    if c2:
        k = c2['kernels_gbs']
        out['c2'] = {'gbs': {n: _g(v) for n, v in k.items()},
                     'frac': {n: _g(v / peak, 3) for n, v in k.items()}}
        if 'hamiltonian' in c2:
            out['c2']['ham_gbs'] = _g(c2['hamiltonian']['gbs'])
        rg = c2.get('reference_gpu')
        if rg and 'apply' in rg:
            out['c2']['ref_gpu_gbs'] = {n: _g(rg[n]['gbs']) for n in k}
            out['c2']['ours_over_ref_gpu'] = {n: _g(k[n] / rg[n]['gbs'], 3)
                                              for n in k}
        elif rg:
            out['c2']['ref_gpu'] = rg.get('unavailable')
    c1 = d.get('c1')
    if c1:
        a = c1['apply']
        e = c1['eps_2e-10']
        r = c1['rel_1e-10']
        out['c1'] = {'apply_us': _g(a['us']), 'apply_gbs': _g(a['gbs']),
                     'apply_frac': _g(a['frac'], 3),
                     'apply_us_l2': _g(a['us_l2_resident']),
                     'solve_ms': _g(e['ms_per_solve']), 'vc': e['vcycles'],
                     'solves_s': _g(e['solves_per_s']),
                     'rel1e-10_ms': _g(r['ms_per_solve']),
                     'rel1e-10_vc': r['vcycles']}
        cr = e.get('cpu_reference')
        if cr:
            out['c1']['cpu_ms'] = _g(cr['ms_per_solve'])
            out['c1']['cpu_err'] = _g(cr['max_rel_err_gpu_vs_cpu'], 2)
    c3 = d.get('c3')
    if c3:
        f = c3['fp64_reference_schedule']
        m4, m6 = c3['mixed_4_levels'], c3['mixed_6_levels']
        out['c3'] = {'fp64_ms': _g(f['ms_per_solve']), 'fp64_vc': f['vcycles'],
                     'mixed4_ms': _g(m4['ms_per_solve']),
                     'mixed4_vc': m4['vcycles'],
                     'speedup4': _g(c3['speedup_mixed_4_over_fp64'], 3),
                     'mixed6_ms': _g(m6['ms_per_solve']),
                     'speedup6': _g(c3['speedup_mixed_6_over_fp64'], 3),
                     'rel_res4': _g(m4['rel_residual'], 2),
                     'diff4': _g(m4['max_rel_diff_vs_fp64'], 2)}
    c4 = d.get('c4')
    if c4:
        out['c4'] = {'mixed_sps': _g(c4['mixed']['solves_per_s']),
                     'fp64_sps': _g(c4['fp64']['solves_per_s']),
                     'speedup': _g(c4['speedup_mixed_over_fp64'], 3),
                     'setup_s': _g(c4['mixed']['setup_s'], 3)}
        if 'cpu_reference' in c4:
            out['c4']['cpu_sps'] = _g(c4['cpu_reference']['solves_per_s'], 3)
    pc = d.get('pc')
    if pc:
        out['pc'] = {'ms': _g(pc['ms_per_call']),
                     'bb_gbs': _g(pc['blackbox_gbs']),
                     'seq_gbs': _g(pc['sequence_gbs']),
                     'k_ms_gbs': [[k['kernel'].split(' ')[0], _g(k['ms'], 3),
                                   _g(k['gbs'], 3)] for k in pc['kernels']]}
    wfd = d.get('wfd')
    if wfd:
        out['wfd'] = {'apply_gbs': _g(wfd['apply']['gbs']),
                      'jac_gbs': _g(wfd['jacobi_sweep']['gbs']),
                      'diel_ms': _g(wfd['poisson_dielectric_64']['ms_per_solve'])}
    c5 = d.get('c5')
    if c5:
        out['c5'] = {'n': c5['requests_per_rate'],
                     'thr_p50_p99': {k.split('_')[1]: [
                         _g(v['throughput_per_s']), _g(v['p50_ms'], 3),
                         _g(v['p99_ms'], 3)]
                         for k, v in c5.items() if k.startswith('lambda_')}}
        an = c5.get('anisotropic')
        if an:
            out['c5']['aniso_thr_p50_p99_built'] = {k.split('_')[1]: [
                _g(v['throughput_per_s']), _g(v['p50_ms'], 3),
                _g(v['p99_ms'], 3), v['solvers_built']]
                for k, v in an.items() if k.startswith('lambda_')}
    return out


def relaunch_with_ranks(args):
    """`bench.py --gpus N` outside torchrun: start N ranks (one process per
    GPU) under torch.distributed.run on this node and return its exit
    status."""
    import socket
    with socket.socket() as sk:
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1',
           f'--nproc-per-node={args.gpus}', '--master-addr=127.0.0.1',
           f'--master-port={port}', os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd, cwd=ROOT).returncode


def main():
    if len(sys.argv) > 1 and sys.argv[1] == '--_cpu-child':
        cpu_step_child(int(sys.argv[2]), int(sys.argv[3]))
        return
    if len(sys.argv) > 1 and sys.argv[1] == '--_cpu-poisson-child':
        cpu_poisson_child(sys.argv[2], sys.argv[3])
        return
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=10)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='gpaw_b200')
    p.add_argument('--no-cpu', action='store_true')
    p.add_argument('--no-e2e', action='store_true')
    p.add_argument('--no-poisson', action='store_true')
    p.add_argument('--no-batch', action='store_true')
    p.add_argument('--no-serving', action='store_true')
    p.add_argument('--no-ham', action='store_true',
                   help='skip the fused Hamiltonian section')
    p.add_argument('--no-ref-gpu', action='store_true',
                   help="skip timing the reference's own GPU kernels")
    p.add_argument('--poisson-only', default=None,
                   choices=['c1', 'c3', 'c4', 'pc', 'c5', 'wfd', 'c1a', 'c3m',
                            'c3f', 'c3trace'],
                   help='run one Poisson configuration only (profiling)')
    p.add_argument('--batch', type=int, default=NBANDS,
                   help='wave functions per step (profiling runs only)')
    p.add_argument('--detail', default=None,
                   help='also write every measured figure to this JSON file')
    args = p.parse_args()
    set_batch(args.batch)
    if (args.gpus > 1 and 'WORLD_SIZE' not in os.environ and
            not args.poisson_only):
        sys.exit(relaunch_with_ranks(args))
    if args.poisson_only:
        import torch
        dev = torch.device('cuda', 0)
        if args.poisson_only in ('c1', 'c3'):
            f = poisson_c1 if args.poisson_only == 'c1' else poisson_c3
            r = f(dev, nsolve=max(1, args.steps))
        elif args.poisson_only == 'c3trace':
            r = mixed_vcycle_trace(dev)
        elif args.poisson_only in ('c3m', 'c3f'):
            # one solver of C3 alone (profiling): the 4-level mixed solver
            # or the FP64 reference schedule
            r = poisson_c3(dev, nsolve=max(1, args.steps),
                           which=('mixed4',) if args.poisson_only == 'c3m'
                           else ('fp64',))
        else:
            r = {'c4': poisson_c4, 'pc': precond_c4, 'c5': serving_c5,
                 'wfd': weighted_fd, 'c1a': c1_apply}[args.poisson_only](dev)
        print(json.dumps(r), flush=True)
    elif args.impl == 'reference':
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
