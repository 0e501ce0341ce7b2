"""One grid split into row bands across ranks (one GPU per rank).

Rank r of W owns global rows [r*B, (r+1)*B) of a grid W*B rows tall (torus),
stored with ``ghost`` extra rows above and below: planes of shape
(P, B + 2*ghost, X/32) int32.  A pass of K <= ghost generations needs the K
rows next to the band from the neighbouring ranks, so every pass is

    exchange_halos(...)   K rows up and K rows down (one send/recv pair each
                          way, contiguous rows; NCCL over NVLink on GPUs,
                          gloo on CPU tensors)
    cb2_band_pass(...)    the strip kernels on the band rows only

The grid shards with one exchange step per pass and no other communication;
the seeded input and the checksum are defined on the global grid, so a band
run reproduces the single-grid run cell for cell.
"""
from __future__ import annotations

import ctypes
from fractions import Fraction

import torch
import torch.distributed as dist

from . import _abi
from ._abi import check, lib
from .grid import automaton_id, automaton_info, plan, thresholds

GHOST = 32  # rows kept on each side: the largest temporal depth


def exchange_halos(planes: torch.Tensor, ghost: int, band_rows: int, k: int, rank: int, world: int,
                   group=None) -> None:
    """Fills the k ghost rows next to the band: the rows above it get the last
    k band rows of rank-1, the rows below it the first k band rows of rank+1
    (torus).  `planes` is (P, band_rows + 2*ghost, words) on this rank."""
    if not 0 < k <= ghost or band_rows < k:
        raise ValueError(f"halo of {k} rows needs 0 < k <= ghost ({ghost}) and k <= band rows ({band_rows})")
    first = planes[:, ghost:ghost + k, :]
    last = planes[:, ghost + band_rows - k:ghost + band_rows, :]
    top_ghost = planes[:, ghost - k:ghost, :]
    bottom_ghost = planes[:, ghost + band_rows:ghost + band_rows + k, :]
    if world == 1:
        top_ghost.copy_(last)
        bottom_ghost.copy_(first)
        return
    up, down = (rank - 1) % world, (rank + 1) % world
    send_last, send_first = last.contiguous(), first.contiguous()
    recv_top, recv_bottom = torch.empty_like(send_last), torch.empty_like(send_first)
    # Posting order matters when up == down (two ranks): per peer, messages
    # match in order, so both ranks send [last, first] and receive
    # [from up -> top ghost, from down -> bottom ghost].
    ops = [dist.P2POp(dist.isend, send_last, down, group), dist.P2POp(dist.isend, send_first, up, group),
           dist.P2POp(dist.irecv, recv_top, up, group), dist.P2POp(dist.irecv, recv_bottom, down, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    top_ghost.copy_(recv_top)
    bottom_ghost.copy_(recv_bottom)


def _planes(t: torch.Tensor):
    P = t.shape[0]
    stride = t.stride(0) * t.element_size()
    return (ctypes.c_void_p * P)(*[t.data_ptr() + p * stride for p in range(P)])


class BandGrid:
    """This rank's band of a grid of ``global_rows`` rows split over ``world`` ranks."""

    def __init__(self, automaton, x_size: int, global_rows: int, rank: int = 0, world: int = 1, ghost: int = GHOST,
                 group=None, device=None):
        if global_rows % world:
            raise ValueError(f"{global_rows} rows do not split evenly over {world} ranks")
        self.automaton = automaton_id(automaton)
        self.name, self.P, self.states = automaton_info(self.automaton)
        self.x_size, self.global_rows = int(x_size), int(global_rows)
        self.rank, self.world, self.ghost, self.group = rank, world, ghost, group
        self.band = global_rows // world
        if self.band < ghost:
            raise ValueError(f"bands of {self.band} rows are thinner than the {ghost} ghost rows")
        self.row0 = rank * self.band
        self.rows_total = self.band + 2 * ghost
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        shape = (self.P, self.rows_total, self.x_size // 32)
        self.bufs = [torch.zeros(shape, dtype=torch.int32, device=self.device) for _ in range(2)]
        self.cur = 0
        self.time_step = 0
        self.seed = 42  # random seed of stochastic rules (run_params::seed)

    @property
    def planes(self) -> torch.Tensor:
        return self.bufs[self.cur]

    def fill_random(self, seed: int, probs=None, stream=None) -> None:
        thr = thresholds(probs if probs is not None else [Fraction(1, self.states)] * self.states)
        arr = (ctypes.c_uint64 * max(1, len(thr)))(*[int(v) for v in thr])
        check(lib.cb2_fill_random_planes(self.automaton, _planes(self.planes), self.x_size, self.rows_total,
                                         self.row0 - self.ghost, self.global_rows, seed, arr, len(thr),
                                         _stream(stream)), "band fill")
        self.time_step = 0

    def plan_k(self, temporal_steps: int = 0) -> int:
        k = temporal_steps or plan(self.automaton, self.x_size, self.band)["temporal_steps"]
        return min(k, self.ghost)

    def run(self, steps: int, temporal_steps: int = 0, tile_rows: int = 0, stream=None) -> int:
        """Advances `steps` generations; returns the number of passes."""
        k_main = self.plan_k(temporal_steps)
        t = _abi.tuning(0, tile_rows, 0, 0)
        left, passes = steps, 0
        while left > 0:
            k = k_main
            while k > left:
                k //= 2
            exchange_halos(self.planes, self.ghost, self.band, k, self.rank, self.world, self.group)
            check(lib.cb2_band_pass_at(self.automaton, _planes(self.bufs[self.cur]),
                                       _planes(self.bufs[1 - self.cur]), self.x_size, self.rows_total, self.ghost,
                                       self.band, k, self.time_step + (steps - left), self.seed,
                                       self.row0 - self.ghost, self.global_rows, ctypes.byref(t), _stream(stream)),
                  "band pass")
            self.cur ^= 1
            left -= k
            passes += 1
        self.time_step += steps
        return passes

    def local_checksum(self, values=None, stream=None) -> list[int]:
        out = (ctypes.c_uint64 * 16)()
        if values is None:
            vp, nv = None, 0
        else:
            vals = (ctypes.c_int64 * len(values))(*[int(v) for v in values])
            vp, nv = vals, len(values)
        check(lib.cb2_checksum_planes(self.automaton, _planes(self.planes), self.x_size, self.rows_total, self.ghost,
                                      self.band, self.row0, self.global_rows, vp, nv, out, _stream(stream)),
              "band checksum")
        return [int(v) for v in out]

    def checksum(self, values=None) -> list[int]:
        """The global grid's 16 tile sums (sum of every band's share)."""
        local = torch.tensor(self.local_checksum(values), dtype=torch.int64, device=self.device)
        if self.world > 1:
            dist.all_reduce(local, group=self.group)
        return [int(v) for v in local.tolist()]

    def band_planes_host(self) -> torch.Tensor:
        """The band's rows (without ghosts) as a host tensor (P, band, words)."""
        return self.planes[:, self.ghost:self.ghost + self.band, :].cpu()


def _stream(stream):
    if stream is None:
        return None
    return stream if isinstance(stream, int) else int(stream.cuda_stream)
