"""Python view of the library's device grids and the reference's host layouts.

``DeviceGrid`` owns a ``cb2_grid`` (P bit-planes on the GPU, double-buffered).
``HostGrid`` is the host image of a grid in one of the reference's layouts
(standard, bit_array, bit_planes, tiled_bit_planes), byte-for-byte what the
reference grid classes store (memory/*_grid.hpp).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from fractions import Fraction

import numpy as np

from . import _abi
from ._abi import check, lib

def _registry() -> dict[str, int]:
    out = {}
    for i in range(lib.cb2_automaton_count()):
        name = ctypes.c_char_p()
        check(lib.cb2_automaton_info(i, ctypes.byref(name), None, None), "automaton info")
        out[name.value.decode()] = i
    return out


# Every registered automaton by name: the hand-written networks (0-2), then the
# lowered DSL automata (bundled, examples, "<name>:dsl" twins).
AUTOMATA = _registry()
NAMES = {v: k for k, v in AUTOMATA.items()}


def automaton_id(automaton) -> int:
    if isinstance(automaton, int):
        return automaton
    return check(lib.cb2_automaton_lookup(automaton.encode()), "automaton lookup")


def automaton_info(automaton) -> tuple[str, int, int]:
    """(name, bit-planes, states) of an automaton given by id or name."""
    a = automaton_id(automaton)
    name = ctypes.c_char_p()
    planes = ctypes.c_int()
    states = ctypes.c_int()
    check(lib.cb2_automaton_info(a, ctypes.byref(name), ctypes.byref(planes), ctypes.byref(states)))
    return name.value.decode(), planes.value, states.value


def state_values(automaton) -> list[int]:
    """State value of each dictionary index (what the reference's checksum sums)."""
    a = automaton_id(automaton)
    n = check(lib.cb2_automaton_values(a, None, 0), "automaton values")
    arr = (ctypes.c_int64 * n)()
    check(lib.cb2_automaton_values(a, arr, n), "automaton values")
    return [int(v) for v in arr]


def thresholds(probs) -> np.ndarray:
    """Cumulative state probabilities (dictionary-index order) as 53-bit integer thresholds.

    State s is drawn with probability probs[s]; the device generator compares
    53 uniform bits against these integers, so the stream is exact and
    reproducible on any host.
    """
    fr = [p if isinstance(p, Fraction) else Fraction(str(p)) for p in probs]
    if abs(sum(fr) - 1) > Fraction(1, 10**12):  # decimal floats such as 1/3 sum to 1 only within rounding
        raise ValueError(f"probabilities sum to {float(sum(fr))}, not 1")
    out, cum = [], Fraction(0)
    for p in fr[:-1]:
        cum += p
        out.append(int(cum * (1 << 53)))
    return np.array(out, dtype=np.uint64)


def layout_bytes(automaton, layout: str, word_bits: int, x_size: int, y_size: int) -> int:
    return check(lib.cb2_layout_bytes(automaton_id(automaton), _abi.LAYOUTS[layout], word_bits, x_size, y_size),
                 "layout size")


def _stream_handle(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)  # torch.cuda.Stream


@dataclass
class HostGrid:
    """Host image of a grid in a reference layout."""

    automaton: int
    layout: str
    word_bits: int
    x_size: int
    y_size: int
    data: np.ndarray  # uint8 view of the image bytes

    def __post_init__(self):
        self.automaton = automaton_id(self.automaton)  # a name or an id
        need = layout_bytes(self.automaton, self.layout, self.word_bits, self.x_size, self.y_size)
        self.data = np.ascontiguousarray(self.data).view(np.uint8).reshape(-1)
        if self.data.nbytes != need:
            raise ValueError(f"{self.layout} image of {self.data.nbytes} bytes, expected {need}")

    @classmethod
    def empty(cls, automaton, layout: str, word_bits: int, x_size: int, y_size: int) -> "HostGrid":
        n = layout_bytes(automaton, layout, word_bits, x_size, y_size)
        return cls(automaton_id(automaton), layout, word_bits, x_size, y_size, np.zeros(n, dtype=np.uint8))

    @classmethod
    def from_cells(cls, automaton, cells: np.ndarray) -> "HostGrid":
        """Standard layout (one uint8 dictionary index per cell) from a (y, x) array."""
        c = np.ascontiguousarray(cells, dtype=np.uint8)
        y, x = c.shape
        return cls(automaton_id(automaton), "standard", 8, x, y, c.reshape(-1))

    def cells(self) -> np.ndarray:
        """(y, x) uint8 dictionary indexes; only for the standard layout."""
        if self.layout != "standard":
            raise ValueError("cells() needs the standard layout; use to_standard()")
        if self.word_bits == 8:
            return self.data.reshape(self.y_size, self.x_size)
        return self.data.view(np.uint32).reshape(self.y_size, self.x_size).astype(np.uint8)

    def to_layout(self, layout: str, word_bits: int) -> "HostGrid":
        """Converts through the device (upload in this layout, download in the other)."""
        with DeviceGrid(self.automaton, self.x_size, self.y_size) as g:
            g.upload(self)
            return g.download(layout, word_bits)

    def to_standard(self) -> "HostGrid":
        return self if (self.layout == "standard" and self.word_bits == 8) else self.to_layout("standard", 8)

    def get_checksum(self) -> str:
        """The reference's 16-tile checksum string (memory/standard_grid.hpp:182-218)."""
        with DeviceGrid(self.automaton, self.x_size, self.y_size) as g:
            g.upload(self)
            return g.checksum_str()


class DeviceGrid:
    """A device-resident grid (``cb2_grid``)."""

    def __init__(self, automaton, x_size: int, y_size: int):
        self.automaton = automaton_id(automaton)
        self.name, self.planes, self.states = automaton_info(self.automaton)
        self.x_size, self.y_size = int(x_size), int(y_size)
        h = ctypes.c_void_p()
        check(lib.cb2_grid_create(self.automaton, self.x_size, self.y_size, ctypes.byref(h)), "grid create")
        self._h = h

    # context manager / lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib.cb2_grid_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # data movement ----------------------------------------------------------------------------
    def upload(self, host: HostGrid, stream=None) -> None:
        if host.automaton != self.automaton or host.x_size != self.x_size or host.y_size != self.y_size:
            raise ValueError("host grid does not match this device grid")
        check(lib.cb2_grid_upload(self._h, _abi.LAYOUTS[host.layout], host.word_bits,
                                  host.data.ctypes.data_as(ctypes.c_void_p), host.data.nbytes,
                                  _stream_handle(stream)), "upload")

    def upload_async(self, host: HostGrid, stream=None) -> None:
        """upload() enqueued on `stream` without waiting (cb2_grid_upload_async):
        `host` must stay unchanged until the stream has passed the copy."""
        if host.automaton != self.automaton or host.x_size != self.x_size or host.y_size != self.y_size:
            raise ValueError("host grid does not match this device grid")
        check(lib.cb2_grid_upload_async(self._h, _abi.LAYOUTS[host.layout], host.word_bits,
                                        host.data.ctypes.data_as(ctypes.c_void_p), host.data.nbytes,
                                        _stream_handle(stream)), "upload")

    def download_async(self, out: np.ndarray, layout: str = "bit_planes", word_bits: int = 64, stream=None) -> None:
        """download() into `out` enqueued on `stream` without waiting
        (cb2_grid_download_async): `out` is written when the stream passes the copy."""
        n = layout_bytes(self.automaton, layout, word_bits, self.x_size, self.y_size)
        buf = out.view(np.uint8).reshape(-1)
        if buf.nbytes != n:
            raise ValueError(f"output buffer of {buf.nbytes} bytes, expected {n}")
        check(lib.cb2_grid_download_async(self._h, _abi.LAYOUTS[layout], word_bits,
                                          buf.ctypes.data_as(ctypes.c_void_p), n, _stream_handle(stream)),
              "download")

    def upload_cells(self, cells: np.ndarray, stream=None) -> None:
        self.upload(HostGrid.from_cells(self.automaton, cells), stream)

    def download(self, layout: str = "standard", word_bits: int = 8, stream=None, out: np.ndarray | None = None
                 ) -> HostGrid:
        n = layout_bytes(self.automaton, layout, word_bits, self.x_size, self.y_size)
        buf = np.empty(n, dtype=np.uint8) if out is None else out.view(np.uint8).reshape(-1)
        if buf.nbytes != n:
            raise ValueError(f"output buffer of {buf.nbytes} bytes, expected {n}")
        check(lib.cb2_grid_download(self._h, _abi.LAYOUTS[layout], word_bits, buf.ctypes.data_as(ctypes.c_void_p),
                                    n, _stream_handle(stream)), "download")
        return HostGrid(self.automaton, layout, word_bits, self.x_size, self.y_size, buf)

    def cells(self, stream=None) -> np.ndarray:
        return self.download("standard", 8, stream).cells()

    def fill_random(self, seed: int, probs=None, thr: np.ndarray | None = None, stream=None) -> None:
        if thr is None:
            if probs is None:  # uniform over the dictionary
                probs = [Fraction(1, self.states)] * self.states
            thr = thresholds(probs)
        t = np.ascontiguousarray(thr, dtype=np.uint64)
        check(lib.cb2_grid_fill_random(self._h, seed, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(t),
                                       _stream_handle(stream)), "fill_random")

    # the hot path -----------------------------------------------------------------------------
    def run(self, steps: int, temporal_steps: int = 0, tile_rows: int = 0, words_per_lane: int = 0,
            levels_per_warp: int = 0, stream=None, rows_per_step: int = 0) -> None:
        t = _abi.tuning(temporal_steps, tile_rows, words_per_lane, levels_per_warp, rows_per_step)
        check(lib.cb2_grid_run(self._h, steps, ctypes.byref(t), _stream_handle(stream)), "run")

    def checksum(self, values=None, stream=None) -> list[int]:
        out = (ctypes.c_uint64 * 16)()
        if values is None:
            check(lib.cb2_grid_checksum(self._h, None, 0, out, _stream_handle(stream)), "checksum")
        else:
            v = np.ascontiguousarray(values, dtype=np.int64)
            check(lib.cb2_grid_checksum(self._h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(v), out,
                                        _stream_handle(stream)), "checksum")
        return [int(x) for x in out]

    def checksum_str(self, values=None, stream=None) -> str:
        return "-".join(str(v) for v in self.checksum(values, stream))

    def planes_ptrs(self) -> list[int]:
        arr = (ctypes.c_void_p * 8)()
        n = ctypes.c_int()
        check(lib.cb2_grid_planes(self._h, arr, ctypes.byref(n), None))
        return [arr[i] for i in range(n.value)]

    @property
    def time_step(self) -> int:
        return int(lib.cb2_grid_time_step(self._h))

    @time_step.setter
    def time_step(self, t: int) -> None:
        check(lib.cb2_grid_set_time_step(self._h, t), "set time_step")

    def set_seed(self, seed: int) -> None:
        """Random seed of stochastic rules (run_params::seed, default 42)."""
        check(lib.cb2_grid_set_seed(self._h, seed), "set seed")


class Batch:
    """Many device grids advanced together by one persistent kernel (``cb2_batch``).

    ``steps[i]`` generations for ``grids[i]`` per run.  The grids stay owned
    by the caller and must outlive the batch.
    """

    def __init__(self, grids: list[DeviceGrid], steps: list[int], temporal_steps: int = 0, tile_rows: int = 0,
                 spin_limit: int = 0, stall_task: int = -1):
        if len(grids) != len(steps) or not grids:
            raise ValueError("grids and steps must be non-empty lists of the same length")
        self.grids = list(grids)
        self.steps = [int(s) for s in steps]
        handles = (ctypes.c_void_p * len(grids))(*[g.handle for g in grids])
        st = np.ascontiguousarray(self.steps, dtype=np.int64)
        opts = _abi.BatchOpts(temporal_steps, tile_rows, spin_limit, stall_task)
        h = ctypes.c_void_p()
        check(lib.cb2_batch_create(handles, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(grids),
                                   ctypes.byref(opts), ctypes.byref(h)), "batch create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.cb2_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, stream=None) -> None:
        check(lib.cb2_batch_run(self._h, _stream_handle(stream)), "batch run")

    def wait(self, stream=None) -> None:
        check(lib.cb2_batch_wait(self._h, _stream_handle(stream)), "batch")

    def run_per_grid(self, stream=None) -> None:
        check(lib.cb2_batch_run_per_grid(self._h, _stream_handle(stream)), "per-grid run")

    def info(self) -> dict:
        tasks = ctypes.c_int64()
        cells = ctypes.c_double()
        ctas = ctypes.c_int()
        check(lib.cb2_batch_info(self._h, ctypes.byref(tasks), ctypes.byref(cells), ctypes.byref(ctas)))
        return {"tasks": tasks.value, "cell_updates": cells.value, "persistent_ctas": ctas.value}


def plan(automaton, x_size: int, y_size: int, temporal_steps: int = 0, tile_rows: int = 0,
         words_per_lane: int = 0, levels_per_warp: int = 0, rows_per_step: int = 0) -> dict:
    """The plan (temporal depth, strip height, lane width, levels per warp, rows per step) a run would use."""
    want = _abi.tuning(temporal_steps, tile_rows, words_per_lane, levels_per_warp, rows_per_step)
    got = _abi.Tuning()
    check(lib.cb2_plan(automaton_id(automaton), x_size, y_size, ctypes.byref(want), ctypes.byref(got)), "plan")
    return got.as_dict()


def run_bit_planes(automaton, a_planes: list[int], b_planes: list[int], x_size: int, y_size: int, steps: int,
                   temporal_steps: int = 0, tile_rows: int = 0, words_per_lane: int = 0, levels_per_warp: int = 0,
                   stream=None, rows_per_step: int = 0) -> bool:
    """Advances caller-owned device planes; returns True if the result is in ``b_planes``."""
    a = (ctypes.c_void_p * len(a_planes))(*a_planes)
    b = (ctypes.c_void_p * len(b_planes))(*b_planes)
    t = _abi.tuning(temporal_steps, tile_rows, words_per_lane, levels_per_warp, rows_per_step)
    res = ctypes.c_int()
    check(lib.cb2_run_bit_planes(automaton_id(automaton), a, b, x_size, y_size, steps, ctypes.byref(t),
                                 _stream_handle(stream), ctypes.byref(res)), "run_bit_planes")
    return bool(res.value)


def variants(automaton) -> list[tuple[int, int, int, int]]:
    """The instantiated strip kernels as (temporal_steps, words_per_lane, levels_per_warp, rows_per_step)."""
    a = automaton_id(automaton)
    n = check(lib.cb2_variants(a, None, 0), "variants")
    arr = (_abi.Tuning * n)()
    check(lib.cb2_variants(a, arr, n), "variants")
    return [(t.temporal_steps, t.words_per_lane, t.levels_per_warp, t.rows_per_step) for t in arr]


def autotune(automaton, x_size: int, y_size: int, budget_ms: float = 0.0) -> dict:
    best = _abi.Tuning()
    check(lib.cb2_autotune(automaton_id(automaton), x_size, y_size, budget_ms, ctypes.byref(best)), "autotune")
    return best.as_dict()


def tuning_load(path: str) -> int:
    return check(lib.cb2_tuning_load(path.encode()), "tuning load")


def tuning_save(path: str) -> int:
    return check(lib.cb2_tuning_save(path.encode()), "tuning save")


def measure_lop3_peak() -> float:
    v = ctypes.c_double()
    check(lib.cb2_measure_lop3_peak(ctypes.byref(v)), "lop3 peak")
    return v.value


def network_ops(automaton) -> tuple[float, float]:
    alu = ctypes.c_double()
    shf = ctypes.c_double()
    check(lib.cb2_network_ops(automaton_id(automaton), ctypes.byref(alu), ctypes.byref(shf)))
    return alu.value, shf.value
