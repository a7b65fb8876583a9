"""The oracle on several basins at once, in spawned worker processes.

TEST INFRASTRUCTURE ONLY: used by tests/ (full-size parity against the
oracle) and by bench.py's CPU legs (the timed CPU baseline and the accuracy
check of the timed run), never by the product path.

A basin is named by a spec `(name, kwargs)`: `name` is a case constructor of
`shygpu.cases` and `kwargs` its arguments; a constructor that returns a list
gives its first case.  Workers build their own cases from the specs (the
generators are seeded, so every process builds the same basin) and are
started with `spawn`, so a parent that already holds a CUDA context can use
them.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
_PATHS = [str(HERE), str(HERE.parent / "shyfemcm-ismar_b200")]

STATE_FIELDS = ("znv", "utlnv", "vtlnv", "hdknv", "wlnv", "tempv", "saltv", "conzv")


def _paths():
    for p in _PATHS:
        if p not in sys.path:
            sys.path.insert(0, p)


def build_case(spec):
    _paths()
    from shygpu import cases
    name, kw = spec
    c = getattr(cases, name)(**kw)
    return c[0] if isinstance(c, list) else c


def _state_worker(args):
    spec, nsteps, fields = args
    _paths()
    import shyref
    case = build_case(spec)
    m = shyref.OracleModel(case)
    t0 = time.perf_counter()
    m.run(nsteps)
    secs = time.perf_counter() - t0
    st = m.state()
    i = m.info()
    return {"state": {k: st[k] for k in fields}, "volume": i.volume, "dtime": i.dtime,
            "krylov_iters": i.krylov_iters, "seconds": secs}


def _timing_worker(args):
    specs, nsteps, warm = args
    _paths()
    import shyref
    models, units = [], 0
    for spec in specs:
        c = build_case(spec)
        models.append(shyref.OracleModel(c))
        units += c["nkn"] * c["nlv"]
    for m in models:
        m.run(warm)
    t0 = time.perf_counter()
    for m in models:
        m.run(nsteps)
    return units * nsteps, time.perf_counter() - t0


def pool(nproc):
    return mp.get_context("spawn").Pool(nproc)


def run_states(specs, nsteps, fields=STATE_FIELDS, nproc=None, wait=True):
    """Each spec's basin advanced `nsteps` from its initial state, one worker
    per basin.  Returns [{"state", "volume", "dtime", "krylov_iters",
    "seconds"}] in spec order, or (pool, AsyncResult) with wait=False (the
    caller calls .get() and then closes the pool)."""
    p = pool(nproc or min(len(specs), os.cpu_count() or 1))
    r = p.map_async(_state_worker, [(s, nsteps, tuple(fields)) for s in specs], chunksize=1)
    if not wait:
        return p, r
    try:
        return r.get()
    finally:
        p.close()
        p.join()


def deal(sizes, nbins):
    """Largest first, each to the least-loaded bin: index lists per bin."""
    bins = [[] for _ in range(nbins)]
    load = [0] * nbins
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        b = load.index(min(load))
        bins[b].append(i)
        load[b] += sizes[i]
    return [b for b in bins if b]


def time_steps(specs, sizes, nsteps, warm, nproc):
    """The basins of `specs` dealt over `nproc` processes by size, each
    process advancing its basins `warm` untimed and `nsteps` timed steps.
    Returns (node*layer*steps, slowest process's seconds, processes)."""
    groups = deal(sizes, nproc)
    with pool(len(groups)) as p:
        res = p.map(_timing_worker, [([specs[i] for i in g], nsteps, warm) for g in groups], chunksize=1)
    return sum(r[0] for r in res), max(r[1] for r in res), len(groups)
