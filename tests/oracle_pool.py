"""The CPU oracle spread over the host's cores: the checker of the full-size
parity tests.  TEST INFRASTRUCTURE ONLY (imported by tests/).

The oracle's J and K are sums over independent pieces of the reference's loop,
so they split exactly:

* molecules: over bra shells I = offset (mod stride)
  (oracle_fourindex_eri_sample), summed over every offset;
* lattices: over the (Q1,Q2) cell-pair tickets that MYID/NUMPROCS hand each
  rank (src/pfourindexdirect.f90:224-240), summed over every rank -- exactly
  the caller's MPI_ALLREDUCE (:757-758).

Workers are started with the 'spawn' method (a pool forked from a process
that already holds a CUDA context can hang); each receives the system and the
density once, through the pool initialiser.
"""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np

_STATE = {}


def _init(sysm, pp, ph):
    _STATE['args'] = (sysm, pp, ph)


def _mol_piece(job):
    import oracle
    stride, offset = job
    sysm, pp, _ = _STATE['args']
    return oracle.fourindex_eri_sample(sysm, pp, stride, offset)


def _lat_piece(job):
    import oracle
    myid, numprocs = job
    sysm, pp, ph = _STATE['args']
    return oracle.fourindex_eri(sysm, pp, ph, myid=myid, numprocs=numprocs)


def workers() -> int:
    return max(1, min(os.cpu_count() or 1, 64))


def fourindex_eri(sysm, pp: np.ndarray, ph=None, nproc: int = None):
    """(C_C, X_C) of the whole build from the oracle, computed in parallel."""
    nproc = nproc or workers()
    ctx = mp.get_context('spawn')
    if sysm.ncell1 == 1 and ph is None:
        stride = 4 * nproc       # small pieces: the bra shells' costs differ by orders of magnitude
        jobs, fn = [(stride, o) for o in range(stride)], _mol_piece
    else:
        jobs, fn = [(r, 4 * nproc) for r in range(4 * nproc)], _lat_piece
    with ctx.Pool(nproc, initializer=_init, initargs=(sysm, pp, ph)) as pool:
        parts = pool.map(fn, jobs, chunksize=1)
    c = np.sum([p[0] for p in parts], axis=0)
    x = np.sum([p[1] for p in parts], axis=0)
    return c, x
