"""
Benchmark of the B200 split-Richardson iteration (voxel-iterations per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload spheres3d] [--n|--size 128]

Workload (default): 3D vector Maxwell, isotropic, complex64, 128^3 grid, 200 seeded spheres, 12-voxel absorbing
ramp, x-polarised Gaussian sheet source (macromax_b200.workloads.spheres_3d).  A step is one iteration
d = chi [G (chi E + s') - E] with the divergence guard and update, on inputs resident in HBM; the working set
(two field buffers, work buffer, source and chi: 208 MB) is larger than the 126 MB L2, so nothing is flushed
between steps.  ``e2e`` is one full solve to the workload's residue through the public API from host numpy arrays
(host->device copies of chi, source and initial field and the device->host copy of the solution inside the timed
region).  ``--impl reference`` times the reference package's own Solution on its torch backend with CPU tensors
(all host threads), or the numpy oracle where the package is absent.
Multi-GPU: the path does not shard a single grid, so N > 1 runs N independent replicas (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'voxel-iterations/s (split-Richardson iteration)'
# inner (complex64) stop rule of the batched mixed-precision solve: tight enough that every sampled source is within
# 1e-7 relative L2 of its FP64 solution when the outer residue is below 1e-8
MIXED_INNER_RTOL = 5e-5
UNIT = 'voxel-it/s'


def word_bytes(dtype) -> int:
    return 16 if np.dtype(dtype) == np.complex128 else 8


def algorithmic_bytes(nvox: int, c: int, m: int, dtype, batch: int = 1) -> float:
    """Compulsory traffic of one iteration: sizeof(word) (8c + 2m/B) per voxel-RHS."""
    return word_bytes(dtype) * (8 * c + 2 * m / batch) * nvox * batch


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,clocks.mem')

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        try:
            proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.QUERY}',
                                     '--format=csv,noheader,nounits', '-lms', '200'],
                                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        try:
            while not self._stop.is_set():
                line = proc.stdout.readline()
                if not line:
                    break
                self.samples.append([x.strip() for x in line.split(',')])
        finally:
            proc.terminate()

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._thread.join(timeout=3)

    def summary(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace('.', '').isdigit()]
        smax = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = set()
        for s in self.samples:
            for i, nme in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith('active'):
                    reasons.add(nme)
        mem = [float(s[9]) for s in self.samples if len(s) > 9 and s[9].replace('.', '').isdigit()]
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': max(smax) if smax else None,
                'reasons': sorted(reasons), 'samples': len(self.samples),
                'mem_mhz': statistics.median(mem) if mem else None}


def make_workload(args):
    from macromax_b200 import workloads
    if args.workload == 'spheres3d':
        return workloads.spheres_3d(n=args.n)
    if args.workload == 'disks2d':
        return workloads.disks_2d(n=args.n)
    if args.workload == 'design3d':
        return workloads.design_3d(n=args.n)
    if args.workload == 'voronoi3d':
        return workloads.voronoi_3d(n=args.n)
    raise SystemExit(f'unknown workload {args.workload}')


def dist_setup(args):
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = 'nccl' if args.impl == 'ours' else 'gloo'
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def cpu_oracle_rate(wl, dtype, iters: int, workers: int):
    """Oracle (reference algorithm, numpy/pocketfft) voxel-iterations/s on the host, over ``iters`` iterations."""
    from oracle import mmoracle as mo
    mo.set_fft_workers(workers)
    sol = mo.from_workload(wl, dtype)
    sol.advance()  # warm-up iteration
    t0 = time.perf_counter()
    for _ in range(iters):
        sol.advance()
    dt = time.perf_counter() - t0
    return int(np.prod(wl['shape'])) * iters / dt, dt


def cpu_torch_rate(wl, dtype, iters: int):
    """The same iteration with torch CPU tensors (the reference's torch backend form): voxel-iterations/s."""
    import torch
    from oracle import mmoracle as mo
    from oracle.torch_cpu import TorchCPUIteration
    it = TorchCPUIteration(mo.from_workload(wl, dtype))
    it.advance()  # warm-up iteration
    t0 = time.perf_counter()
    for _ in range(iters):
        it.advance()
    dt = time.perf_counter() - t0
    return int(np.prod(wl['shape'])) * iters / dt, dt, torch.get_num_threads()


def reference_package_rates(wl, iters: int):
    """The reference package's own Solution (python/macromax/solver.py) on its NumPy and torch-CPU backends, on the
    same workload and host cores: voxel-iterations/s over ``iters`` iterations after one warm-up iteration, and the
    set-up time.  None where the package is not present (it is read from baseline/_ref)."""
    import torch
    from oracle.refimport import import_reference, reference_available
    if not reference_available():
        return None
    mm = import_reference()
    out = {}
    nvox = int(np.prod(wl['shape']))
    for name, cfg in (('numpy', {'type': 'numpy'}), ('torch_cpu', {'type': 'torch', 'device': 'cpu'})):
        mm.backend.config(cfg)
        grid = mm.Grid(shape=wl['shape'], step=wl['step'])
        t0 = time.perf_counter()
        sol = mm.Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                          source_distribution=wl['source'], bound=mm.bound.Bound(grid, thickness=wl['bound_thickness']),
                          dtype=np.complex64)
        t1 = time.perf_counter()
        it = iter(sol)
        next(it)  # warm-up iteration
        t2 = time.perf_counter()
        for _ in range(iters):
            next(it)
        dt = time.perf_counter() - t2
        # numpy.fft runs on one thread; torch uses its intra-op thread pool
        out[name] = {'value': nvox * iters / dt, 'unit': UNIT, 'setup_s': t1 - t0, 'kind': 'reference',
                     'cores': 1 if name == 'numpy' else torch.get_num_threads(),
                     'sample': f'{iters} iterations of the reference package\'s Solution on its {name} backend '
                               f'after one warm-up iteration ({dt:.1f} s)'}
        del sol, it
    mm.backend.config({'type': 'numpy'})
    return out


def reference_package_arm(wl, steps: int, warmup: int):
    """The reference package's own Solution (python/macromax/solver.py:1049-1098) on its torch backend with CPU
    tensors and all host threads -- the fastest of its host backends on this workload -- one iteration per step after
    ``warmup`` untimed iterations.  Returns (voxel-iterations/s, seconds, threads, set-up seconds), or None where the
    package is not present (it is read from baseline/_ref)."""
    import torch
    from oracle.refimport import import_reference, reference_available
    if not reference_available():
        return None
    torch.set_num_threads(os.cpu_count() or 1)
    mm = import_reference()
    mm.backend.config({'type': 'torch', 'device': 'cpu'})
    try:
        grid = mm.Grid(shape=wl['shape'], step=wl['step'])
        t0 = time.perf_counter()
        sol = mm.Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                          source_distribution=wl['source'], bound=mm.bound.Bound(grid, thickness=wl['bound_thickness']),
                          dtype=np.complex64)
        setup = time.perf_counter() - t0
        it = iter(sol)
        for _ in range(warmup):
            next(it)
        t0 = time.perf_counter()
        for _ in range(steps):
            next(it)
        dt = time.perf_counter() - t0
    finally:
        mm.backend.config({'type': 'numpy'})
    return int(np.prod(wl['shape'])) * steps / dt, dt, torch.get_num_threads(), setup


def bench_reference(args, wl, rank, world, pg):
    """--impl reference: the reference's own iteration on the host cores, one iteration per step -- the reference
    package's Solution on its torch-CPU backend with all host threads, or, where the package is absent, the numpy
    oracle (its NumPy backend's algorithm) with all host threads in scipy.fft."""
    dtype = np.complex64
    cores = os.cpu_count() or 1
    if rank != 0:
        return
    got = None
    try:
        got = reference_package_arm(wl, args.steps, args.warmup)
    except Exception as e:  # report and fall back to the restatement
        print(f'reference package arm unavailable ({type(e).__name__}: {e}); timing the numpy oracle', file=sys.stderr)
    if got is not None:
        value, dt, threads, setup = got
        cpu = {'value': value, 'unit': UNIT, 'cores': threads, 'kind': 'reference',
               'sample': f"{args.steps} iterations of the reference package's Solution on its torch backend with CPU "
                         f'tensors ({threads} threads) after {args.warmup} warm-up iterations; set-up {setup:.2f} s '
                         'not timed'}
    else:
        from oracle import mmoracle as mo
        mo.set_fft_workers(cores)
        sol = mo.from_workload(wl, dtype)
        for _ in range(args.warmup):
            sol.advance()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sol.advance()
        dt = time.perf_counter() - t0
        value = int(np.prod(wl['shape'])) * args.steps / dt
        cpu = {'value': value, 'unit': UNIT, 'cores': cores, 'kind': 'port',
               'sample': f'{args.steps} iterations of the numpy oracle on the full workload, '
                         f'scipy.fft pocketfft with {cores} workers'}
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * dt / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c64', 'data': 'synthetic (seeded generator)',
        'config': config_of(args, wl, world),
        'cpu_baseline': cpu,
        'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def config_of(args, wl, world=1):
    c = 3 if np.asarray(wl['source']).ndim > len(wl['shape']) and np.asarray(wl['source']).shape[0] == 3 else 1
    chi = 'isotropic chi' if np.asarray(wl['epsilon']).ndim == len(wl['shape']) else '3x3 anisotropic chi'
    return {'workload': f"{wl['name']}: {'x'.join(map(str, wl['shape']))} grid, {c}-component field, "
                        f"{chi}, complex64, 1 RHS", 'grid': list(wl['shape']), 'components': c,
            'batch': 1, 'l2': 'working set > L2 (no flush needed)', 'parallelism': f'replicas x{world}'}


def bench_ours(args, wl, rank, world, local, pg):
    import torch
    from macromax_b200 import Bound, Grid, Solution
    from macromax_b200 import _native as nat
    torch.cuda.set_device(local)
    dtype = np.complex64
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=bound, dtype=dtype)
    eng = sol._engine
    nvox = eng.N
    c = eng.ncomp
    # stored chi words per voxel: 1, 6 (a symmetric 3x3, the algorithmic figure's m) or 9
    m = {nat.MMX_CHI_SCALAR: 1, nat.MMX_CHI_SYM6: 6}.get(eng.chi_kind, 9)
    tuned = None
    if args.variant >= 0:
        from macromax_b200 import autotune
        autotune.set_variant(eng, args.variant)
        tuned = {'variant': args.variant, 'pinned': True}
    elif args.autotune:
        from macromax_b200 import autotune
        tuned = autotune.tune(eng, iters=10, use_cache=False)
    # every step is a real iteration: the stop rule is disabled for the timed run
    st = eng.read_state()
    st['rtol'] = -1.0
    st['maxiter'] = np.inf
    st['active'] = 1
    eng.write_state(st)
    stream = torch.cuda.current_stream()
    chunk = max(1, min(args.chunk, args.steps))
    nchunks, rem = divmod(args.steps, chunk)
    eng.iterate(args.warmup) if args.warmup > 1 else eng.iterate(1)  # warm-up steps (one captured graph)
    # capture the timed chunk's graphs outside the timed region: the timed chunks continue the warm-up's solve, so
    # with the fused epilogue each starts from the first pass that the previous chunk left in the work buffer
    eng.prepare_graph(chunk)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        # a short device sleep ahead of the start event, so that the first graph is already queued when the timed
        # region begins: the host's launch latency stays out of the device-timed steps (the e2e figure keeps it)
        torch.cuda._sleep(2_000_000)
        start.record(stream)
        for _ in range(nchunks):
            eng.iterate(chunk, cont=True)
        for _ in range(rem):
            eng.iterate(1)
        stop.record(stream)
        torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    ms = start.elapsed_time(stop)
    if pg is not None:
        from macromax_b200.distributed import max_over_ranks
        ms = max_over_ranks(ms, device='cuda')
    ms_per_step = ms / args.steps
    value = world * nvox * args.steps / (ms / 1e3)
    st = eng.read_state()
    assert np.all(st['status'] == 0) and np.all(st['iteration'] >= args.steps), 'iteration did not run'
    launches_per_iter = len_passes(wl, tuned['variant'] if tuned else 0)
    alg = algorithmic_bytes(nvox, c, m, dtype)
    peaks = load_peaks()
    achieved = alg / (ms_per_step / 1e3) / 1e9
    roof = {'bound': 'hbm', 'achieved': achieved, 'peak': peaks['hbm_gbs'], 'unit': 'GB/s',
            'frac': achieved / peaks['hbm_gbs'], 'traffic': traffic_per_iteration(wl, tuned['variant'] if tuned else 0),
            'peak_source': peaks['source'],
            'unit_of_launch': f'one iteration = {launches_per_iter} pass kernels (CUDA graph chunks of {chunk})',
            'algorithmic_bytes': alg, 'bytes_per_voxel': alg / nvox}
    sol._engine.close()
    e2e = e2e_solve(wl, dtype, tuned['variant'] if tuned else None) if rank == 0 and not args.no_e2e else None
    # the GPU measurements run before the host baseline, whose FFT worker threads would compete with the host side
    # of the timed GPU solves
    secondary = run_secondary(args) if rank == 0 and args.secondary != 'none' else None
    cpu = None
    if rank == 0 and not args.no_cpu:
        rate, dt = cpu_oracle_rate(wl, dtype, args.cpu_iters, os.cpu_count() or 1)
        cpu = {'value': rate, 'unit': UNIT, 'cores': os.cpu_count() or 1, 'kind': 'port',
               'sample': f'{args.cpu_iters} iterations of the numpy oracle on the full workload ({dt:.1f} s), '
                         f'scipy.fft with {os.cpu_count()} workers'}
        if np.asarray(wl['epsilon']).ndim == len(wl['shape']):  # isotropic: the torch-CPU form as well
            trate, tdt, threads = cpu_torch_rate(wl, dtype, args.cpu_iters)
            cpu['torch_cpu'] = {'value': trate, 'unit': UNIT, 'cores': threads, 'kind': 'port',
                                'sample': f'{args.cpu_iters} iterations with torch CPU tensors on the full workload '
                                          f'({tdt:.1f} s), {threads} threads'}
        try:
            ref_pkg = reference_package_rates(wl, 3)
        except Exception as e:  # the reference package is optional here; its absence or failure is reported
            ref_pkg = {'unavailable': f'{type(e).__name__}: {e}'[:200]}
        if ref_pkg is not None:
            cpu['reference_package'] = ref_pkg
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms_per_step, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'c64', 'data': 'synthetic (seeded generator)',
            'config': config_of(args, wl, world),
            'roofline': roof, 'cpu_baseline': cpu, 'e2e': e2e, 'clocks': clocks.summary(),
            # with the fused epilogue a graph chunk continues from the previous one; a single iteration (mmx_iterate)
            # starts with the plain first pass
            'gpu_launches': launches_per_iter * args.steps + (rem if fused_epilogue(
                wl, tuned['variant'] if tuned else 0) else 0),
            'kernel_variant': tuned,
            'timed_region': (f'{args.steps} iterations as CUDA-graph chunks of {chunk} on one stream between CUDA '
                             'events, continuing the warm-up solve; the first chunk is queued behind a 1 ms device '
                             'sleep, so the host launch '
                             'latency is not timed (e2e includes it)'),
        }
        if secondary is not None:
            line['secondary'] = secondary
        print(json.dumps(line), flush=True)


def traffic_per_iteration(wl, variant=0):
    """DRAM bytes of one iteration of this workload and kernel variant from the committed ncu capture (or None)."""
    path = os.path.join(ROOT, 'profiles', 'traffic.json')
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d[wl['name']]['variants'][str(int(variant))]['dram_bytes_per_iteration'])
    except (OSError, ValueError, KeyError, TypeError):
        return None


def run_secondary(args):
    """
    The other configurations (seconds, device-timed by synchronisation around whole solves):
      - 2D scalar 256^2 disks in complex128 to 1e-6 or 500 iterations, set-up included;
      - 3D anisotropic 192^3 Voronoi grains, complex64 inner iterations with FP64 defect correction, to 1e-8;
      - a magnetic medium (the reference test suite's negative-index plate, 128^2) to residue 1e-3;
      - the full scattering matrix of a 512 x 256 slab (254 columns in batched solves);
      - the standalone transform mmx_fftn (BackEnd.ft) of three 128^3 complex64 fields;
      - batched mixed precision (2D scalar slab, 512^2 grid, 256 plane-wave sources) to residue 1e-8, with the error
        of 8 seeded sources against FP64 solutions, against the plain complex64 per-source loop (one Solution per
        source for all 256 sources, to 1e-5: single precision cannot reach 1e-8), each on the kernel variant the
        autotuner picks for it (chosen before the timed solves); and the uneven batch
        64 x 128^2 + 32 x 256^2 + 8 x 384^2 to 1e-8;
      - adjoint gradient (3D scalar design problem, 128^3, 32 sources): forward + adjoint solve in complex64 to 1e-6
        (on the kernel variant the autotuner picks for a batch of the same problem), and in mixed precision to
        1e-10, each gradient's error against the same gradient from FP64 solves.
    """
    import torch
    from macromax_b200 import Bound, Grid, Solution, adjoint, workloads
    from macromax_b200 import _native as nat
    from macromax_b200.mixed import MixedSolution
    out = {}
    wl = workloads.correlated_slab_2d(n=512, nb_modes=256)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    t0 = time.perf_counter()
    ms = MixedSolution(grid, wl['source'], wl['epsilon'], bound=bound, vacuum_wavelength=wl['wavelength'])
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    tuned_batch = ms.tune()  # the inner iteration's kernel variant, chosen before the timed solve
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    ms.solve(rtol=1e-8, inner_rtol=MIXED_INNER_RTOL)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    mixed_s = t2 - t1
    res = float(ms.residues.max())
    inner = ms.total_inner_iterations
    outer = [float(np.max(r)) for r in ms.outer_residues]
    sample = np.sort(np.random.default_rng(11).choice(256, 8, replace=False))
    x_sample = ms.E[sample]  # FP64 solutions of the sampled sources
    ms.close()
    # their error against FP64 solutions: the device complex128 iteration (the path pinned to the reference's iterates
    # at 1e-10) to residue 1e-12
    errs = []
    for k, b in enumerate(sample):
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'][b], bound=bound, dtype=np.complex128)
        sol.solve(None, rtol=1e-12, maxiter=200000)
        ref = sol.E
        errs.append(float(np.linalg.norm((x_sample[k] - ref).ravel()) / np.linalg.norm(ref.ravel())))
        sol._engine.close()
    # the plain complex64 loop: one Solution per source, every one of the 256 sources, to 1e-5 (single precision
    # alone does not reach 1e-8), on the kernel variant the autotuner picks for one source of this problem
    from macromax_b200 import autotune
    seq = 0.0
    its = 0
    tuned_single = None
    for b in range(256):
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'][b], bound=bound, dtype=np.complex64)
        if tuned_single is None:  # (the trials restore the fields and the state)
            tuned_single = autotune.tune(sol._engine, iters=10, use_cache=False)
        else:
            autotune.set_variant(sol._engine, tuned_single['variant'])
        torch.cuda.synchronize()
        a = time.perf_counter()
        sol.solve(None, rtol=1e-5, maxiter=100000)
        torch.cuda.synchronize()
        seq += time.perf_counter() - a
        its += sol.iteration
        sol._engine.close()
    out['batched_mixed_slab2d_512x256'] = {
        'time_to_1e-8_s': mixed_s, 'max_residue': res, 'setup_s': t1 - t0, 'inner_iterations': inner,
        'inner_rtol': MIXED_INNER_RTOL, 'outer_residues_max': outer,
        'error_vs_fp64_solution': {'max': max(errs), 'sources': [int(b) for b in sample], 'errors': errs,
                                   'reference': 'device complex128 iteration to residue 1e-12'},
        'plain_c64_loop_to_1e-5_s (all 256 sources)': seq, 'plain_iterations_per_source': its / 256,
        'speedup_vs_plain_loop': seq / mixed_s,
        'kernel_variant': {'batched_inner': tuned_batch, 'plain_loop': tuned_single},
        'voxel_iterations_per_s': 256 * 512 * 512 * inner / mixed_s}
    torch.cuda.empty_cache()
    # the uneven batch of the same material class: 64 x 128^2, 32 x 256^2 and 8 x 384^2 sources to 1e-8, all
    # members' inner solves in one graph per chunk
    from macromax_b200.mixed import MixedUnevenSolution
    members = []
    for n_, b_, seed_ in ((128, 64, 41), (256, 32, 42), (384, 8, 43)):
        w_ = workloads.correlated_slab_2d(n=n_, nb_modes=b_, seed=seed_, slab_px=n_ // 4)
        g_ = Grid(shape=w_['shape'], step=w_['step'])
        members.append(MixedSolution(g_, w_['source'], w_['epsilon'], bound=Bound(g_, thickness=w_['bound_thickness']),
                                     vacuum_wavelength=w_['wavelength']))
    mu = MixedUnevenSolution(members)
    torch.cuda.synchronize()
    a = time.perf_counter()
    mu.solve(rtol=1e-8)
    torch.cuda.synchronize()
    uneven_s = time.perf_counter() - a
    work = sum(m.inner.engine.N * int(sum(np.sum(i) for i in m.inner_iterations)) for m in members)
    out['uneven_mixed_slab2d_64x128^2_32x256^2_8x384^2'] = {
        'time_to_1e-8_s': uneven_s, 'max_residue': float(max(m.residues.max() for m in members)),
        'outer_steps': [len(m.outer_residues) for m in members],
        'voxel_rhs_iterations_per_s': work / uneven_s}
    mu.close()
    # 2D scalar Helmholtz, complex128 (the reference NumPy backend's configuration): 256^2 disks to 1e-6 or 500
    # iterations, including the set-up, second of two runs
    wl = workloads.disks_2d(n=256)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    for rep in range(2):
        torch.cuda.synchronize()
        a = time.perf_counter()
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                       dtype=np.complex128)
        sol.solve(None, rtol=1e-6, maxiter=500)
        E = sol.E
        b = time.perf_counter()
        sol._engine.close()
    out['disks2d_256_c128'] = {'time_to_solution_s (set-up included)': b - a, 'iterations': int(sol.iteration),
                               'residue': float(sol.residue), 'voxel_iterations_per_s': 256 ** 2 * sol.iteration / (b - a)}
    del E
    # 3D anisotropic vector Maxwell, 192^3 Voronoi grains: complex64 inner iterations + FP64 defect correction to 1e-8
    wl = workloads.voronoi_3d(n=192)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    torch.cuda.synchronize()
    a = time.perf_counter()
    ms = MixedSolution(grid, wl['source'], wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                       vacuum_wavelength=wl['wavelength'])
    torch.cuda.synchronize()
    b = time.perf_counter()
    # the inner iteration's kernel variant: the plain 3x3-chi passes or the fused epilogue (timed trials on the
    # problem's own sources, then restored)
    tuned3 = ms.tune(iters=10, candidates=(0, nat.MMX_VARIANT_FUSED_EPILOGUE))
    torch.cuda.synchronize()
    b = time.perf_counter()
    ms.solve(rtol=1e-8)
    torch.cuda.synchronize()
    c = time.perf_counter()
    out['anisotropic_voronoi3d_192_mixed'] = {
        'setup_s': b - a, 'time_to_1e-8_s': c - b, 'max_residue': float(ms.residues.max()),
        'inner_iterations': ms.total_inner_iterations, 'outer_steps': len(ms.outer_residues),
        'voxel_iterations_per_s': 192 ** 3 * ms.total_inner_iterations / (c - b), 'kernel_variant': tuned3}
    # error against an FP64 solution: the plain complex128 iteration on the device (the path pinned to the reference's
    # iterates at 1e-10) run to residue 1e-11 (the FP64 numpy oracle would take hours at this size)
    x64 = ms.E[0]
    ms.close()
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'], source_distribution=wl['source'],
                   bound=Bound(grid, thickness=wl['bound_thickness']), dtype=np.complex128)
    torch.cuda.synchronize()
    a = time.perf_counter()
    sol.solve(None, rtol=1e-11, maxiter=20000)
    torch.cuda.synchronize()
    b = time.perf_counter()
    ref = sol.E
    out['anisotropic_voronoi3d_192_mixed']['error_vs_fp64_solution'] = float(
        np.linalg.norm((x64 - ref).ravel()) / np.linalg.norm(ref.ravel()))
    out['anisotropic_voronoi3d_192_mixed']['fp64_reference'] = {
        'iterations': int(sol.iteration), 'residue': float(sol.residue), 'seconds': b - a}
    sol._engine.close()
    del x64, ref
    # magnetic medium: the reference test suite's negative-index plate (128^2, complex64) to residue 1e-3
    from macromax_b200 import LinearBound, solve
    wavelength, k0 = 500e-9, 2 * np.pi / 500e-9
    grid = Grid(shape=(128, 128), step=wavelength / 4)
    rz = np.array([[np.cos(np.pi / 6), -np.sin(np.pi / 6), 0], [np.sin(np.pi / 6), np.cos(np.pi / 6), 0], [0, 0, 1]])
    kin = rz * k0 @ np.array([1, 0, 0])
    cur = np.exp(1j * (kin[0] * grid[0] + kin[1] * grid[1]))
    sp = grid.shape[0] - int(2e-6 / grid.step[0])
    cur[:sp, :] = 0
    cur[sp + 1:, :] = 0
    cur = cur * np.exp(-0.5 * ((grid[1] - grid[1].ravel()[grid.shape[0] // 3]) / 2.5e-6) ** 2)
    cur = cur[np.newaxis] * (rz @ np.array([0, 1, 1j]) / np.sqrt(2))[:, np.newaxis, np.newaxis]
    n = 1 + (-1.5 - 1) * np.ones(grid[1].shape) * (np.abs(grid[0]) < 2.5e-6)
    for _ in range(2):  # the first solve loads the kernels and captures its iteration graphs: the second is timed
        torch.cuda.synchronize()
        a = time.perf_counter()
        sol = solve(grid, vacuum_wavelength=wavelength, current_density=cur, refractive_index=n,
                    bound=LinearBound(grid, thickness=2e-6, max_extinction_coefficient=0.5),
                    callback=None, rtol=1e-3, maxiter=1e4, dtype=np.complex64)
        torch.cuda.synchronize()
        b = time.perf_counter()
    out['magnetic_negative_index_plate_128'] = {'time_to_1e-3_s (set-up included)': b - a,
                                                'iterations': int(sol.iteration), 'residue': float(sol.residue)}
    sol.close()
    # standalone transform (BackEnd.ft): mmx_fftn forward of three 128^3 complex64 fields, graph-replayed
    import ctypes
    from macromax_b200 import _native as nat
    plan = nat.Plan((128, 128, 128), 1, 1, nat.MMX_C64)
    x = torch.randn(3 * 128 ** 3, dtype=torch.complex64, device='cuda')
    y = torch.empty_like(x)

    def fft():
        nat.call('mmx_fftn', plan.handle, nat.device_ptr(x), nat.device_ptr(y), 3, 0,
                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    fft()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(20):
            fft()
    g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / 200
    out['fftn_128^3_x3_c64'] = {'us_per_transform': t * 1e6,
                                'GB_per_s (3 passes, each reading and writing the fields)': 6 * x.numel() * 8 / t / 1e9}
    del g, x, y
    plan.close()
    # scattering matrix: every column of a 512 x 256 grid holding a 128-px layer of the correlated-disorder slab
    # across axis 0, periodic across, absorbing 32-px layers at both ends of axis 0
    from macromax_b200.matrix import ScatteringMatrix
    wl = workloads.correlated_slab_2d(n=512)
    start = (512 - 128) // 2
    eps = np.ones((512, 256), dtype=np.complex128)
    eps[start:start + 128, :] = wl['epsilon'][16:272, start:start + 128].T
    grid = Grid(shape=(512, 256), step=wl['step'])
    thickness = np.zeros((2, 1))
    thickness[0, 0] = 32 * wl['step']
    sm = ScatteringMatrix(grid, vectorial=False, vacuum_wavelength=wl['wavelength'], epsilon=eps,
                          bound=LinearBound(grid, thickness=thickness, max_extinction_coefficient=0.25),
                          dtype=np.complex64)
    torch.cuda.synchronize()
    a = time.perf_counter()
    _ = sm._solution  # set-up (preconditioner) of the shared material
    torch.cuda.synchronize()
    b = time.perf_counter()
    S = np.asarray(sm)
    c = time.perf_counter()
    tm = getattr(sm, 'timing', {'modes_s': float('nan'), 'solve_s': float('nan')})
    out['scattering_matrix_slab2d_512x256'] = {
        'columns': int(S.shape[1]), 'setup_s': b - a, 'columns_s': c - b,
        'solves_s': tm['solve_s'], 'mode_synthesis_and_detection_on_device_s': tm['modes_s'],
        'other_host_s': (c - b) - tm['solve_s'] - tm['modes_s']}
    del S, sm
    # adjoint: one small untimed pass first, so that the first use of torch's autograd and indexing kernels (about
    # 1 s of one-time loading) is not counted in the timed forward / backward
    wl = workloads.design_3d(n=32, nb_sources=2)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    eps = torch.tensor(wl['epsilon'], dtype=torch.complex64, device='cuda', requires_grad=True)
    E = adjoint.solve(eps, torch.tensor(wl['source'], dtype=torch.complex64, device='cuda'), grid,
                      2 * np.pi / wl['wavelength'], bound=Bound(grid, thickness=wl['bound_thickness']), rtol=1e-3)
    (-(E[:, 0][(slice(None),) + wl['patch']].abs() ** 2).sum()).backward()
    torch.cuda.synchronize()
    wl = workloads.design_3d(n=128, nb_sources=32)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    k0 = 2 * np.pi / wl['wavelength']
    eps = torch.tensor(wl['epsilon'], dtype=torch.complex64, device='cuda', requires_grad=True)
    src = torch.tensor(wl['source'], dtype=torch.complex64, device='cuda')
    # the pass-kernel variant of both solves: the autotuner's choice on a batch of the same problem, before timing
    from macromax_b200 import autotune
    from macromax_b200.batch import BatchSolution
    tb = BatchSolution(grid, wl['source'], wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                       wavenumber=k0, dtype=np.complex64)
    tuned_adj = autotune.tune(tb.engine, iters=10, use_cache=False)
    tb.close()
    del tb
    stats = {}
    torch.cuda.synchronize()
    a = time.perf_counter()
    E = adjoint.solve(eps, src, grid, k0, bound=Bound(grid, thickness=wl['bound_thickness']), rtol=1e-6,
                      maxiter=100000, stats=stats, variant=tuned_adj['variant'])
    torch.cuda.synchronize()
    b = time.perf_counter()
    loss = -(E[:, 0][(slice(None),) + wl['patch']].abs() ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    c = time.perf_counter()
    fi, ai = stats['forward_iterations'], stats['adjoint_iterations']
    solve_s = stats['forward_solve_s'] + stats['adjoint_solve_s']
    g32 = eps.grad.detach().to(torch.complex128).cpu().numpy()
    del E, loss, eps, src
    torch.cuda.empty_cache()
    out['adjoint_design3d_128x32'] = {
        'forward_s': b - a, 'backward_s': c - b, 'forward_iterations_max': int(fi.max()),
        'adjoint_iterations_max': int(ai.max()),
        'voxel_iterations_per_s': 128 ** 3 * (int(fi.sum()) + int(ai.sum())) / (c - a),
        'solve_s (forward + adjoint iterations only)': solve_s,
        'solve_voxel_iterations_per_s': 128 ** 3 * (int(fi.sum()) + int(ai.sum())) / solve_s,
        'gradient_error_vs_fp64_adjoint': adjoint_fp64_error(wl, g32), 'kernel_variant': tuned_adj}
    del g32
    torch.cuda.empty_cache()
    # the same gradient with both solves in mixed precision (complex64 inner iterations, FP64 defect correction to
    # residue 1e-10): accurate beyond what complex64 solves reach
    eps = torch.tensor(wl['epsilon'], dtype=torch.complex64, device='cuda', requires_grad=True)
    src = torch.tensor(wl['source'], dtype=torch.complex64, device='cuda')
    stats = {}
    torch.cuda.synchronize()
    a = time.perf_counter()
    E = adjoint.solve(eps, src, grid, k0, bound=Bound(grid, thickness=wl['bound_thickness']), rtol=1e-10,
                      stats=stats, precision='mixed')
    loss = -(E[:, 0][(slice(None),) + wl['patch']].abs() ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    b = time.perf_counter()
    gm = eps.grad.detach().to(torch.complex128).cpu().numpy()
    del E, loss, eps, src
    torch.cuda.empty_cache()
    out['adjoint_design3d_128x32']['mixed_precision'] = {
        'forward_and_backward_s': b - a, 'forward_inner_iterations': int(stats['forward_iterations'][0]),
        'adjoint_inner_iterations': int(stats['adjoint_iterations'][0]),
        'gradient_error_vs_fp64_adjoint': adjoint_fp64_error(wl, gm)}
    return out


def adjoint_fp64_error(wl, g32):
    """Relative L2 error of a complex64 adjoint gradient dL/d eps (loss -sum |E|^2 over the detector patch, summed over
    the sources) against the same adjoint-state gradient from FP64 solves (complex64 inner iterations with FP64
    defect correction to residue 1e-11): forward fields E, adjoint fields nu for the sources conj(dL/dE), gradient
    conj(sum_b nu_b E_b) k0^2 -- over the whole grid and over the design region."""
    from macromax_b200 import Bound, Grid
    from macromax_b200.mixed import MixedSolution
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    k0 = 2 * np.pi / wl['wavelength']
    fwd = MixedSolution(grid, wl['source'], wl['epsilon'], bound=bound, vacuum_wavelength=wl['wavelength'])
    fwd.solve(rtol=1e-11)
    E = fwd.E
    fwd.close()
    dLdE = np.zeros_like(E)
    idx = (slice(None), 0) + tuple(wl['patch'])
    dLdE[idx] = -2 * E[idx]
    adj = MixedSolution(grid, np.conj(dLdE), wl['epsilon'], bound=bound, vacuum_wavelength=wl['wavelength'])
    adj.solve(rtol=1e-11)
    nu = adj.E
    adj.close()
    g64 = np.conj(np.sum(nu[:, 0] * E[:, 0], axis=0)) * k0 ** 2
    d = tuple(wl['design'])
    return {'grid': float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
            'design_region': float(np.linalg.norm(g32[d] - g64[d]) / np.linalg.norm(g64[d])),
            'reference': 'FP64 forward and adjoint solves (mixed precision) to residue 1e-11'}


def len_passes(wl, variant=0) -> int:
    """Pass kernels per iteration: one per axis and direction (2 ndim - 1); 3 for a 3D grid on the plane passes;
    with the fused epilogue the first pass becomes a repair pass (the same count; one extra prologue per chunk)."""
    d = len(wl['shape'])
    iso = np.asarray(wl['epsilon']).ndim == d
    if d == 3 and (variant or 0) & 8 and tuple(wl['shape'][1:]) == (128, 128) and iso:
        return 3
    return 1 if d == 1 else 2 * d - 1


def fused_epilogue(wl, variant=0) -> bool:
    """Whether the plan runs the fused epilogue: isotropic chi, or a 3x3 chi on 192-sample rows of a vector field."""
    d = len(wl['shape'])
    if d < 2 or not (variant or 0) & 16 or (variant or 0) & 8:
        return False
    iso = np.asarray(wl['epsilon']).ndim == d
    return iso or int(wl['shape'][-1]) == 192


def e2e_solve(wl, dtype, variant=None):
    """One full solve to the workload's residue through the public API from host arrays (host->device copies of
    chi and source, the field started at zero on the device as the reference's Solution starts it, device->host
    copy of the solution), on the kernel variant ``variant`` (the autotuner's choice for this problem class; None:
    the plan's default).  A first, untimed solve captures the iteration graphs."""
    import torch
    from macromax_b200 import Bound, Grid, Solution, autotune
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=bound, dtype=dtype)
    eng = sol._engine
    if variant is not None:
        autotune.set_variant(eng, int(variant))
    chi_host = eng.chi.cpu().numpy()
    src_host = eng.sources.cpu().numpy()
    pin = [torch.from_numpy(a).pin_memory() for a in (chi_host, src_host)]
    out_pin = torch.empty((eng.ncomp, eng.N), dtype=eng.torch_dtype, pin_memory=True)  # the result's host buffer
    result = None
    for timed in (False, True):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.chi.copy_(pin[0], non_blocking=True)
        eng.sources.copy_(pin[1], non_blocking=True)
        eng.fields.zero_()
        eng.reset_update_norm()
        eng.reset_alpha()
        st = eng.run(float(wl['rtol']), float(wl['maxiter']))
        out_pin.copy_(eng.current(st)[0])
        torch.cuda.synchronize()
        out = out_pin.numpy()
        dt = time.perf_counter() - t0
        iters = int(st['iteration'][0])
        h2d = sum(int(p.numel() * p.element_size()) for p in pin)
        if timed:
            result = {'value': eng.N * iters / dt, 'unit': UNIT, 'h2d_bytes_per_step': h2d,
                      'd2h_bytes_per_step': int(out.nbytes), 'iterations': iters, 'seconds': dt,
                      'residue': float(st['residue'][0]), 'kernel_variant': autotune.get_variant(eng),
                      'step': f"one solve to residue {wl['rtol']} from host arrays (time to residual)"}
    sol._engine.close()
    # time to residual including the set-up, as a user runs it: Solution from host arrays (host FP64 preconditioner
    # with its objective on the device, plan, graph captures), solve, field read back
    for timed in (False, True):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'], bound=bound, dtype=dtype)
        if variant is not None:
            autotune.set_variant(sol._engine, int(variant))
        sol.solve(None, rtol=float(wl['rtol']), maxiter=float(wl['maxiter']))
        E = sol.E
        dt = time.perf_counter() - t0
        if timed:
            result['time_to_residual_with_setup_s'] = dt
            result['with_setup_iterations'] = int(sol.iteration)
        sol._engine.close()
        del E
    return result


def load_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            d = json.load(f)
        return {'hbm_gbs': float(d['hbm_gbs']), 'source': 'measured (MEASURED_PEAKS.json)'}
    except (OSError, KeyError, ValueError):
        return {'hbm_gbs': 6650.0, 'source': 'fallback 6.65 TB/s'}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=400)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='spheres3d')
    # --size: the same option under torchrun, whose own parser takes --n for an abbreviation of its options
    ap.add_argument('--n', '--size', dest='n', type=int, default=128)
    ap.add_argument('--cpu-iters', type=int, default=6)
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--chunk', type=int, default=50, help='iterations per captured CUDA graph in the timed region')
    ap.add_argument('--secondary', default='batched', choices=['none', 'batched'])
    ap.add_argument('--autotune', type=int, default=1, help='time the kernel variants first and use the fastest')
    ap.add_argument('--variant', type=int, default=-1,
                    help='pin the kernel variant (MMX_VARIANT_* flags) instead of autotuning')
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = make_workload(args)
    rank, world, local, pg = dist_setup(args)
    try:
        if args.impl == 'reference':
            bench_reference(args, wl, rank, world, pg)
        else:
            bench_ours(args, wl, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == '__main__':
    main()
