"""One grid split into row bands across ranks (one GPU per rank).

Rank r of W owns global rows [r*B, (r+1)*B) of a grid W*B rows tall (torus),
stored with ``ghost`` extra rows above and below: planes of shape
(P, B + 2*ghost, X/32) int32.  A pass of K <= ghost generations needs the K
rows next to the band from the neighbouring ranks.  Every pass is

    post_halos(...)       K rows up and K rows down (one send/recv pair each
                          way, contiguous rows; NCCL over NVLink on GPUs,
                          gloo on CPU tensors), posted without waiting
    interior pass         band rows K .. B-K-1, which read band rows only,
                          while the exchange is in flight
    finish()              the received rows land in the ghost rows
    two edge passes       the K rows at each edge of the band

with pass depths from cb2_band_schedule (the same schedule cb2_band_run
follows for C and C++ hosts).  The grid shards with one exchange step per
pass and no other communication; the seeded input and the checksum are
defined on the global grid, so a band run reproduces the single-grid run cell
for cell.
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


def post_halos(planes: torch.Tensor, ghost: int, band_rows: int, k: int, rank: int, world: int, group=None):
    """Posts the halo exchange for a pass of k generations and returns a
    function that completes it: once called, the k rows above the band hold
    the last k band rows of rank-1 and the k rows below it the first k band
    rows of rank+1 (torus).  `planes` is (P, band_rows + 2*ghost, words).
    On GPUs the sends and receives run on NCCL's stream, ordered after the
    work already on the current stream; finish() makes the current stream
    wait for them, so work enqueued in between overlaps the exchange."""
    if not 0 < k <= ghost or band_rows < k:
        raise ValueError(f"halo of {k} rows needs 0 < k <= ghost ({ghost}) and k <= band rows ({band_rows})")
    first = planes[:, ghost:ghost + k, :]
    last = planes[:, ghost + band_rows - k:ghost + band_rows, :]
    top_ghost = planes[:, ghost - k:ghost, :]
    bottom_ghost = planes[:, ghost + band_rows:ghost + band_rows + k, :]
    if world == 1:
        def finish_local():
            top_ghost.copy_(last)
            bottom_ghost.copy_(first)
        return finish_local
    up, down = (rank - 1) % world, (rank + 1) % world
    send_last, send_first = last.contiguous(), first.contiguous()
    recv_top, recv_bottom = torch.empty_like(send_last), torch.empty_like(send_first)
    # Posting order matters when up == down (two ranks): per peer, messages
    # match in order, so both ranks send [last, first] and receive
    # [from up -> top ghost, from down -> bottom ghost].
    ops = [dist.P2POp(dist.isend, send_last, down, group), dist.P2POp(dist.isend, send_first, up, group),
           dist.P2POp(dist.irecv, recv_top, up, group), dist.P2POp(dist.irecv, recv_bottom, down, group)]
    reqs = dist.batch_isend_irecv(ops)

    def finish():
        for req in reqs:
            req.wait()
        top_ghost.copy_(recv_top)
        bottom_ghost.copy_(recv_bottom)
    return finish


def exchange_halos(planes: torch.Tensor, ghost: int, band_rows: int, k: int, rank: int, world: int,
                   group=None) -> None:
    """post_halos followed at once by its completion."""
    post_halos(planes, ghost, band_rows, k, rank, world, group)()


def schedule(steps: int, temporal_steps: int, ghost: int = GHOST) -> list[int]:
    """Depths of the passes of a band run (cb2_band_schedule): passes of
    min(temporal_steps, ghost), then the remainder's binary digits."""
    n = check(lib.cb2_band_schedule(steps, temporal_steps, ghost, None, 0), "band schedule")
    depths = (ctypes.c_int * max(1, n))()
    check(lib.cb2_band_schedule(steps, temporal_steps, ghost, depths, n), "band schedule")
    return list(depths[:n])


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
        """Advances `steps` generations; returns the number of passes.  With a
        `stream`, the exchange's copies and the passes are all ordered on it."""
        t = _abi.tuning(0, tile_rows, 0, 0)
        depths = schedule(steps, self.plan_k(temporal_steps), self.ghost)
        if self.device.type == "cuda":
            s = stream if isinstance(stream, torch.cuda.Stream) or stream is None else \
                torch.cuda.ExternalStream(int(stream))
            with torch.cuda.stream(s if s is not None else torch.cuda.current_stream(self.device)):
                self._passes(depths, t, torch.cuda.current_stream(self.device).cuda_stream)
        else:
            self._passes(depths, t, None)
        self.time_step += steps
        return len(depths)

    def _passes(self, depths, tuning, stream) -> None:
        g, B = self.ghost, self.band
        t0 = self.time_step
        for k in depths:
            finish = post_halos(self.planes, g, B, k, self.rank, self.world, self.group)
            src, dst = self.bufs[self.cur], self.bufs[1 - self.cur]
            if self.world > 1 and B >= 3 * k:
                self._pass(src, dst, g + k, B - 2 * k, k, t0, tuning, stream)  # needs no ghost row
                finish()
                self._pass(src, dst, g, k, k, t0, tuning, stream)
                self._pass(src, dst, g + B - k, k, k, t0, tuning, stream)
            else:
                finish()
                self._pass(src, dst, g, B, k, t0, tuning, stream)
            self.cur ^= 1
            t0 += k

    def _pass(self, src: torch.Tensor, dst: torch.Tensor, row_first: int, rows_out: int, k: int, time_step: int,
              tuning, stream) -> None:
        """k generations of planes rows [row_first, row_first + rows_out) from
        src into dst (the strip kernels; reads k rows beyond them)."""
        check(lib.cb2_band_pass_at(self.automaton, _planes(src), _planes(dst), self.x_size, self.rows_total,
                                   row_first, rows_out, k, time_step, self.seed, self.row0 - self.ghost,
                                   self.global_rows, ctypes.byref(tuning), stream), "band pass")

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
        # uint64 sums (modulo 2^64, as the reference's standard grid sums
        # them) travel as two's-complement int64.
        signed = [v - (1 << 64) if v >= 1 << 63 else v for v in self.local_checksum(values)]
        local = torch.tensor(signed, dtype=torch.int64, device=self.device)
        if self.world > 1:
            dist.all_reduce(local, group=self.group)
        return [int(v) & ((1 << 64) - 1) for v in local.tolist()]

    def band_planes_host(self) -> torch.Tensor:
        """The band's rows (without ghosts) as a host tensor (P, band, words)."""
        return self.planes[:, self.ghost:self.ghost + self.band, :].cpu()


def _stream(stream):
    if stream is None:
        return None
    return stream if isinstance(stream, int) else int(stream.cuda_stream)
