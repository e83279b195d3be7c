"""
Autotuner for the kernel variant of an iteration plan.

For one problem class -- (grid shape, components, chi kind, batch, precision, GPU) -- it times a few iterations of
every kernel variant the plan offers (``mmx_plan_set_variant``: compile-time register-staged passes, shared-memory
staged passes, strided passes staged by bulk tensor (TMA) copies, the epilogue fused with the next prologue,
persistent double-buffered prologue/epilogue, plane passes over the two inner axes of a 3D grid,
runtime-length kernels) with CUDA events and keeps the
fastest.  Results are cached in a JSON file (``$MACROMAX_B200_TUNE_CACHE`` or
``~/.cache/macromax_b200/autotune.json``), so a problem class is measured once per machine.  The trial iterations
run on copies of the engine's fields and state, which are restored afterwards, so tuning leaves the solve
untouched.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from . import _native as nat

CANDIDATES = (0, nat.MMX_VARIANT_FUSED_EPILOGUE, nat.MMX_VARIANT_TMA,
              nat.MMX_VARIANT_TMA | nat.MMX_VARIANT_FUSED_EPILOGUE, nat.MMX_VARIANT_PLANE,
              nat.MMX_VARIANT_SHARED_STAGED, nat.MMX_VARIANT_PERSISTENT,
              nat.MMX_VARIANT_SHARED_STAGED | nat.MMX_VARIANT_PERSISTENT, nat.MMX_VARIANT_GENERIC)


def cache_path() -> str:
    return os.environ.get('MACROMAX_B200_TUNE_CACHE',
                          os.path.join(os.path.expanduser('~'), '.cache', 'macromax_b200', 'autotune.json'))


def problem_key(engine) -> str:
    name = torch.cuda.get_device_name(engine.device)
    return (f"{'x'.join(map(str, engine.shape))}|c{engine.ncomp}|chi{engine.chi_kind}|b{engine.batch}|"
            f"p{engine.precision}|{name}")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(d):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + '.tmp'
        with open(tmp, 'w') as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def set_variant(engine, flags: int):
    nat.call('mmx_plan_set_variant', engine.plan.handle, int(flags))


def get_variant(engine) -> int:
    return int(nat.load().mmx_plan_get_variant(engine.plan.handle))


def tune(engine, iters: int = 20, use_cache: bool = True, candidates=CANDIDATES) -> dict:
    """Pick and apply the fastest variant for ``engine``; returns {'variant', 'us_per_iteration', 'trials'}.

    The trials run the engine's own right-hand sides.  A trial counts only if every right-hand side took all its
    timed iterations: an engine whose sources and fields are zero (0 / 0 residue) stops at once and would time empty
    launches, so it raises ``RuntimeError`` instead (set its sources first)."""
    key = problem_key(engine)
    cache = _load() if use_cache else {}
    if use_cache and key in cache:
        set_variant(engine, cache[key]['variant'])
        return cache[key]
    fields = engine.fields.clone()
    state = engine.state.clone()
    st = engine.read_state()
    st['rtol'] = -1.0
    st['maxiter'] = np.inf
    st['active'] = 1
    engine.write_state(st)
    trials = {}
    stream = torch.cuda.current_stream()
    for flags in candidates:
        try:
            set_variant(engine, flags)
            engine.iterate(2)  # capture + warm up
            engine.prepare_graph(iters)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            before = engine.read_state()['iteration'].copy()
            a.record(stream)
            engine.iterate(iters)
            b.record(stream)
            torch.cuda.synchronize()
            after = engine.read_state()
            if not np.all(after['iteration'] - before == iters):
                continue  # some right-hand side stopped: the time is not that of full iterations
            trials[str(flags)] = a.elapsed_time(b) * 1e3 / iters
        except nat.NativeError:
            continue
    if not trials:
        engine.fields.copy_(fields)
        engine.state.copy_(state)
        raise RuntimeError('autotune: no variant ran its iterations on every right-hand side '
                           '(zero sources, or a diverging state?)')
    best = min(trials, key=trials.get)
    engine.fields.copy_(fields)
    engine.state.copy_(state)
    set_variant(engine, int(best))
    result = {'variant': int(best), 'us_per_iteration': trials[best], 'trials': trials}
    if use_cache:
        cache = _load()
        cache[key] = result
        _save(cache)
    return result
