"""The multi-rank Fock build on the host (gloo, two ranks, CPU).

The reference splits the (Q1,Q2) cell pairs over MPI ranks by its TICKET round
robin and sums J/K with MPI_ALLREDUCE (src/pfourindexdirect.f90:224-240,
757-758); the library takes the same myid/numprocs in pfe_args and bench.py
sums the ranks' C_C/X_C with one all-reduce.  Here two gloo ranks each build
their share with the oracle (which follows the reference's TICKET loop) and
sum it with torch.distributed.all_reduce, as the bench's N > 1 path does with
NCCL; the sum equals the one-rank build of a translational chain and of a
helical chain to rounding, and each rank's share is a proper part of it.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _decks():
    from polymer_b200 import geometry, inputdeck
    chain = inputdeck.make_deck([1, 1], [[0, 0, 0], [1.4, 0, 0]], '6-31Gss', period=(4.0, 0, 0),
                                kpoints=(4, 0, 0), cutoff1=2, cutoff2=3, inttol=1e-10)
    helix = geometry.polyethylene_deck('STO-3G', cutoff1=1, cutoff2=2, kpoints=4)
    return {'chain': chain, 'helix': helix}


def _inputs(name):
    import oracle
    from polymer_b200 import scf, system
    s = system.build_system(_decks()[name], oracle.onee)
    rng = np.random.default_rng(3)
    n = s.basis.npgs
    a = rng.normal(size=(s.ncell1, n, n)) * 0.01
    pp = a + a.transpose(0, 2, 1)
    ph = scf.rotate(scf.HostState(s), torch.tensor(pp))
    return s, pp, (ph.numpy() if ph is not None else None)


def _rank(rank, world, port, name, out_path):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    import datetime
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        s, pp, ph = _inputs(name)
        c, x = oracle.fourindex_eri(s, pp, ph, myid=rank, numprocs=world)
        share = float(np.abs(c).max())
        tc, tx = torch.tensor(c), torch.tensor(x)
        dist.all_reduce(tc)
        dist.all_reduce(tx)
        if rank == 0:
            np.savez(out_path, c=tc.numpy(), x=tx.numpy(), share0=share)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('name', ['chain', 'helix'])
def test_rank_shares_sum_to_the_full_build(name, tmp_path):
    import oracle
    out = str(tmp_path / 'sum.npz')
    mp.spawn(_rank, args=(2, _free_port(), name, out), nprocs=2, join=True)
    got = np.load(out)
    s, pp, ph = _inputs(name)
    c, x = oracle.fourindex_eri(s, pp, ph)
    scale = float(np.abs(c).max())
    assert float(np.abs(got['c'] - c).max()) <= 1e-12 * scale
    assert float(np.abs(got['x'] - x).max()) <= 1e-12 * float(np.abs(x).max())
    assert 0.0 < float(got['share0'])          # rank 0 computed a non-empty share
    assert float(np.abs(got['c'] - c).max()) < float(got['share0'])
