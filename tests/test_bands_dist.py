"""Row bands across ranks, on CPU with gloo (world sizes 2 and 3): the halo
exchange (cellato_b200.bands.exchange_halos, the code the GPU ranks run over
NCCL) and the whole band decomposition -- exchange, then K generations per
band -- against the oracle on the global grid.  The per-band stepping here
is the oracle on the padded band (test infrastructure); on GPUs it is
cb2_band_pass."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _exchange_worker(rank, world, port, ghost, band, k, out):
    _init(rank, world, port)
    from cellato_b200.bands import exchange_halos
    P, words = 2, 3
    t = torch.full((P, band + 2 * ghost, words), -1, dtype=torch.int32)
    for p in range(P):
        for r in range(band):
            t[p, ghost + r, :] = (rank * 1000 + r) * 10 + p
    exchange_halos(t, ghost, band, k, rank, world)
    up, down = (rank - 1) % world, (rank + 1) % world
    ok = True
    for p in range(P):
        for j in range(k):
            ok &= bool((t[p, ghost - k + j] == (up * 1000 + band - k + j) * 10 + p).all())
            ok &= bool((t[p, ghost + band + j] == (down * 1000 + j) * 10 + p).all())
    out[rank] = int(ok)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_halos_gloo(world):
    out = mp.Manager().dict()
    mp.spawn(_exchange_worker, args=(world, _free_port(), 4, 6, 3, out), nprocs=world, join=True)
    assert [out[r] for r in range(world)] == [1] * world


def _bands_worker(rank, world, port, automaton, x, rows, steps, k, ghost, out):
    _init(rank, world, port)
    from cellato_b200.bands import exchange_halos
    from oracle import oracle as O
    probs = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}[automaton]
    P = O.PLANES[automaton]
    cells = O.init_cells(x, rows, 99, O.thresholds(probs))
    band = rows // world
    row0 = rank * band
    idx = [(row0 - ghost + i) % rows for i in range(band + 2 * ghost)]
    padded = cells[idx]
    planes = torch.from_numpy(O.pack("bit_planes", padded, P, 32).view(np.int32).reshape(P, band + 2 * ghost, x // 32).copy())
    left = steps
    while left > 0:
        kk = min(k, left)
        exchange_halos(planes, ghost, band, kk, rank, world)
        cur = O.unpack("bit_planes", planes.numpy().view(np.uint8).reshape(-1), x, band + 2 * ghost, P, 32)
        nxt = O.run_standard(automaton, cur, kk)  # ghost rows beyond kk are junk, never used
        new = torch.from_numpy(O.pack("bit_planes", nxt, P, 32).view(np.int32).reshape(P, band + 2 * ghost, x // 32))
        planes[:, ghost:ghost + band] = new[:, ghost:ghost + band]
        left -= kk
    mine = O.unpack("bit_planes", planes[:, ghost:ghost + band].contiguous().numpy().view(np.uint8).reshape(-1),
                    x, band, P, 32)
    gathered = [torch.zeros_like(torch.from_numpy(mine)) for _ in range(world)]
    dist.all_gather(gathered, torch.from_numpy(mine.copy()))
    if rank == 0:
        full = np.concatenate([g.numpy() for g in gathered], axis=0)
        out["ok"] = bool((full == O.run_standard(automaton, cells, steps)).all())
    dist.destroy_process_group()


@pytest.mark.parametrize("world,automaton", [(2, 0), (3, 1), (2, 2)])
def test_band_decomposition_matches_global_oracle(world, automaton):
    out = mp.Manager().dict()
    mp.spawn(_bands_worker, args=(world, _free_port(), automaton, 64, 24 * world, 21, 4, 5, out), nprocs=world,
             join=True)
    assert out["ok"]
