"""The reference's traverser / run_params / experiment surface over the B200 backend.

Mirrors, for Python callers and the tests:
  * ``RunParams``      experiments/run_params.hpp:10-43 (same field names)
  * ``Traverser``      the Traverser concept: ``is_CUDA``, ``init(grid, params)``,
                       ``run(steps, callback)``, ``fetch_result()``
                       (traversers/cuda/simple.hpp:25-104, cpu/simple.hpp:19-95)
  * ``run_experiment`` experiment_manager::run_experiment(params, initial_state)
                       (experiments/experiment_manager.hpp:43-93)
The C++ drop-in for the reference's own catalog is
``include/cellato_b200/traverser.hpp``.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .grid import AUTOMATA, DeviceGrid, HostGrid, automaton_id

DEVICE = "CUDA"
TRAVERSER = "b200"


@dataclasses.dataclass
class RunParams:
    automaton: str = "game-of-life"
    device: str = DEVICE
    traverser: str = TRAVERSER
    evaluator: str = "bit_planes"
    layout: str = "bit_planes"
    reference_impl: str = "none"
    x_size: int = 0
    y_size: int = 0
    steps: int = 0
    word_size: int = 64
    x_tile_size: int = 0
    y_tile_size: int = 0
    temporal_steps: int = 0        # 0 = autotuned / heuristic
    temporal_tile_size_y: int = 0  # output rows per warp strip, 0 = automatic
    rounds: int = 1
    warmup_rounds: int = 0
    seed: int = 42
    cuda_block_size_x: int = 32
    cuda_block_size_y: int = 8
    words_per_lane: int = 0
    levels_per_warp: int = 0
    rows_per_step: int = 0

    def csv_line(self) -> str:
        f = self
        return ",".join(str(v) for v in (
            f.automaton, f.device, f.traverser, f.evaluator, f.layout,
            f.reference_impl if f.reference_impl != "none" else "", f.x_size, f.y_size, f.steps, f.rounds,
            f.warmup_rounds, f.x_tile_size, f.y_tile_size, f.cuda_block_size_x, f.cuda_block_size_y, f.seed,
            f.word_size, f.temporal_steps, f.temporal_tile_size_y))

    @staticmethod
    def csv_header() -> str:
        return ("automaton,device,traverser,evaluator,layout,reference_impl,x_size,y_size,steps,rounds,"
                "warmup_rounds,x_tile_size,y_tile_size,cuda_block_size_x,cuda_block_size_y,seed,word_size,"
                "temporal_steps,temporal_tile_size_y")


class Traverser:
    """B200 traverser: the grid lives on the device between init and fetch_result."""

    is_CUDA = True

    def __init__(self):
        self._grid: DeviceGrid | None = None
        self._layout = "bit_planes"
        self._word_bits = 64
        self._params = RunParams()

    def init(self, grid: HostGrid, params: RunParams) -> None:
        if params.temporal_steps not in (0, 1, 2, 4, 8, 16, 32):
            raise ValueError(f"Invalid --temporal_steps {params.temporal_steps}: use 1, 2, 4, 8, 16 or 32")
        self._params = params
        self._layout, self._word_bits = grid.layout, grid.word_bits
        self._grid = DeviceGrid(grid.automaton, grid.x_size, grid.y_size)
        self._grid.upload(grid)

    def run(self, steps: int, callback=None, stream=None) -> None:
        if self._grid is None:
            raise RuntimeError("run() before init()")
        p = self._params
        if callback is None:
            self._grid.run(steps, p.temporal_steps, p.temporal_tile_size_y, p.words_per_lane, p.levels_per_warp,
                           stream=stream, rows_per_step=p.rows_per_step)
            return
        # Callback after every chunk with the host grid, like temporal.cuh:230-232.
        chunk = p.temporal_steps or 1
        callback(0, self._grid.download(self._layout, self._word_bits, stream))
        done = 0
        while done < steps:
            n = min(chunk, steps - done)
            self._grid.run(n, n if n in (1, 2, 4, 8, 16, 32) else 0, p.temporal_tile_size_y, p.words_per_lane,
                           p.levels_per_warp if n == chunk else 0, stream=stream,
                           rows_per_step=p.rows_per_step if n == chunk else 0)
            done += n
            callback(done, self._grid.download(self._layout, self._word_bits, stream))

    def fetch_result(self, stream=None) -> HostGrid:
        """Host grid of the final generation; frees the device copy (simple.cuh:81-89)."""
        if self._grid is None:
            raise RuntimeError("fetch_result() before init()")
        out = self._grid.download(self._layout, self._word_bits, stream)
        self._grid.close()
        self._grid = None
        return out


def run_experiment(params: RunParams, initial_state: np.ndarray) -> dict:
    """experiment_manager::run_experiment: warm-up + measured rounds, CUDA-event
    timing of traverser.run, checksum of each measured round's result."""
    import torch

    aut = automaton_id(params.automaton)
    cells = np.ascontiguousarray(initial_state, dtype=np.uint8).reshape(params.y_size, params.x_size)
    standard = HostGrid.from_cells(aut, cells)
    host = standard if params.layout == "standard" else standard.to_layout(params.layout, params.word_size)
    times, checksums = [], []
    stream = torch.cuda.current_stream()
    for r in range(params.warmup_rounds + params.rounds):
        t = Traverser()
        t.init(host, params)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        t.run(params.steps, stream=stream)
        stop.record(stream)
        stop.synchronize()
        result = t.fetch_result(stream)
        if r >= params.warmup_rounds:
            times.append(start.elapsed_time(stop))
            checksums.append(result.get_checksum())
    mean = sum(times) / len(times)
    std = math.sqrt(sum((t - mean) ** 2 for t in times) / len(times))
    cells_total = params.x_size * params.y_size
    per_cell_ps = mean * 1e9 / cells_total / params.steps if cells_total and params.steps else 0.0
    same = all(c == checksums[0] for c in checksums)
    csv = (f"{params.csv_line()},{mean:.6f},{per_cell_ps:.6f},{std:.6f},{'true' if same else 'false'},"
           f"{checksums[0]}")
    return {"execution_times_ms": times, "checksums": checksums, "average_time_ms": mean,
            "average_time_per_cell_ps": per_cell_ps, "std_time_ms": std, "rounds_had_same_checksums": same,
            "csv_line": csv}


__all__ = ["RunParams", "Traverser", "run_experiment", "AUTOMATA"]
