"""ctypes access to the test-only checkers.  TEST INFRASTRUCTURE ONLY.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module; the product package never does.

* ``libcellato_oracle.so`` -- the C restatement of Cellato's hot path
  (``cellato_oracle.c``), each function citing the reference file it follows.
* ``_ref/libcellato_ref.so`` -- Cellato's own CPU traverser compiled from the
  reference headers (``ref_shim.cpp``); present wherever ``make -C oracle``
  ran with the reference sources available, and shipped prebuilt otherwise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from fractions import Fraction

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "libcellato_oracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libcellato_ref.so")

AUTOMATA = {"game-of-life": 0, "wire": 1, "excitable": 2}
PLANES = {0: 1, 1: 2, 2: 3}
LAYOUTS = {"standard": 0, "bit_array": 1, "bit_planes": 2, "tiled_bit_planes": 3}

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i64 = ctypes.c_int64

_oracle = None
_ref = None


def build() -> None:
    """Compile the checkers (the reference shim only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.orc_planes.argtypes = [ctypes.c_int]
        lib.orc_splitmix64.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        lib.orc_splitmix64.restype = ctypes.c_uint64
        lib.orc_init_cells.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint64, _u64p, ctypes.c_int]
        lib.orc_step_standard.argtypes = [ctypes.c_int, _i64, _i64, _u8p, _u8p]
        lib.orc_run_standard.argtypes = [ctypes.c_int, _i64, _i64, _i64, _u8p]
        lib.orc_step_bit_planes.argtypes = [ctypes.c_int, _i64, _i64, _u32p, _u32p]
        lib.orc_run_bit_planes.argtypes = [ctypes.c_int, _i64, _i64, _i64, _u32p]
        lib.orc_checksum.argtypes = [_u8p, _i64, _i64, _i64p, _u64p]
        lib.orc_checksum_planes.argtypes = [_u32p, _i64, _i64, ctypes.c_int, _i64p, _u64p]
        lib.orc_init_bit_planes.argtypes = [_u32p, _i64, _i64, ctypes.c_int, ctypes.c_uint64, _u64p, ctypes.c_int]
        lib.orc_init_bit_planes_rows.argtypes = [_u32p, _i64, _i64, ctypes.c_int, ctypes.c_uint64, _u64p,
                                                 ctypes.c_int, _i64, _i64]
        for name in ("orc_pack_bit_planes", "orc_unpack_bit_planes"):
            getattr(lib, name).argtypes = [_u8p, _i64, _i64, ctypes.c_int, _u8p]
        for name in ("orc_pack_bit_array", "orc_unpack_bit_array", "orc_pack_tiled", "orc_unpack_tiled"):
            getattr(lib, name).argtypes = [_u8p, _i64, _i64, ctypes.c_int, ctypes.c_int, _u8p]
        lib.orc_sample_ratio.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _u64p, ctypes.c_int, ctypes.c_uint64,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        lib.orc_sample_ratio.restype = ctypes.c_uint64
        _oracle = lib
    return _oracle


def sample_ratio(num: int, den: int, words, active: int | None = None, lane_bits: int = 64) -> tuple[int, int]:
    """Exact Bernoulli(num/den) per lane from scripted random words (digit j =
    words[j]), as core/probability.hpp:27-87; returns (lanes set, words used),
    words used = -1 when the words ran out."""
    w = np.ascontiguousarray(np.array([int(v) for v in words] or [0], dtype=np.uint64))
    used = ctypes.c_int()
    mask = (1 << lane_bits) - 1
    r = _lib().orc_sample_ratio(num, den, _p(w, _u64p), len(words), mask if active is None else active, lane_bits,
                                ctypes.byref(used))
    return int(r), used.value


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _reflib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_SO} is not built (run `make -C oracle` where the reference sources exist)")
        lib = ctypes.CDLL(REF_SO)
        lib.ref_run.argtypes = [ctypes.c_int] * 6 + [_u8p, _u8p, ctypes.c_char_p, ctypes.c_int]
        lib.ref_pack.argtypes = [ctypes.c_int] * 5 + [_u8p, _u8p, ctypes.c_size_t]
        lib.ref_bench.argtypes = [ctypes.c_int] * 7 + [_u8p]
        lib.ref_bench.restype = ctypes.c_double
        lib.ref_run_seeded.argtypes = [ctypes.c_int] * 7 + [_u8p, _u8p, ctypes.c_char_p, ctypes.c_int]
        lib.ref_automaton_id.argtypes = [ctypes.c_char_p]
        lib.ref_bench_planes64.argtypes = [ctypes.c_int] * 5 + [_u64p]
        lib.ref_bench_planes64.restype = ctypes.c_double
        lib.ref_run_planes64.argtypes = [ctypes.c_int] * 5 + [_u64p, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                                              ctypes.POINTER(_u64p), ctypes.c_int]
        _ref = lib
    return _ref


def _p(a: np.ndarray, t):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def thresholds(probs) -> np.ndarray:
    """Cumulative state probabilities (dictionary-index order) as exact 53-bit integer thresholds."""
    fr = [Fraction(str(p)) if not isinstance(p, Fraction) else p for p in probs]
    total = sum(fr)
    if abs(total - 1) > Fraction(1, 10**12):  # decimal floats such as 1/3 sum to 1 only within rounding
        raise ValueError(f"probabilities sum to {float(total)}, not 1")
    out, cum = [], Fraction(0)
    for p in fr[:-1]:
        cum += p
        out.append(int(cum * (1 << 53)))
    return np.array(out, dtype=np.uint64)


def init_cells(x: int, y: int, seed: int, thr: np.ndarray) -> np.ndarray:
    cells = np.empty(x * y, dtype=np.uint8)
    thr = np.ascontiguousarray(thr, dtype=np.uint64)
    _lib().orc_init_cells(_p(cells, _u8p), x * y, seed, _p(thr, _u64p), len(thr))
    return cells.reshape(y, x)


def splitmix64(seed: int, index: int) -> int:
    return int(_lib().orc_splitmix64(seed, index))


def run_standard(automaton: int, cells: np.ndarray, steps: int) -> np.ndarray:
    c = np.ascontiguousarray(cells, dtype=np.uint8).copy()
    y, x = c.shape
    rc = _lib().orc_run_standard(automaton, x, y, steps, _p(c, _u8p))
    if rc:
        raise ValueError(f"orc_run_standard failed ({rc})")
    return c


def run_bit_planes(automaton: int, planes: np.ndarray, x: int, y: int, steps: int) -> np.ndarray:
    """planes: uint32 array of P*y*(x/32) words (plane-major)."""
    p = np.ascontiguousarray(planes, dtype=np.uint32).copy()
    rc = _lib().orc_run_bit_planes(automaton, x, y, steps, _p(p, _u32p))
    if rc:
        raise ValueError(f"orc_run_bit_planes failed ({rc})")
    return p


def checksum(cells: np.ndarray, values=None) -> list[int]:
    c = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = c.shape
    vals = np.arange(256, dtype=np.int64) if values is None else np.ascontiguousarray(values, dtype=np.int64)
    out = np.zeros(16, dtype=np.uint64)
    _lib().orc_checksum(_p(c, _u8p), x, y, _p(vals, _i64p), _p(out, _u64p))
    return [int(v) for v in out]


def checksum_str(cells: np.ndarray, values=None) -> str:
    return "-".join(str(v) for v in checksum(cells, values))


def init_bit_planes(x: int, y: int, planes: int, seed: int, thr: np.ndarray, threads: int = 1) -> np.ndarray:
    """init_cells written straight into bit planes: uint32 array (planes, y, x/32),
    generated by `threads` host threads over row ranges."""
    out = np.empty((planes, y, x // 32), dtype=np.uint32)
    thr = np.ascontiguousarray(thr, dtype=np.uint64)
    lib = _lib()
    threads = max(1, min(threads, y))
    bounds = [y * t // threads for t in range(threads + 1)]

    def rows(t):
        return lib.orc_init_bit_planes_rows(_p(out, _u32p), x, y, planes, seed, _p(thr, _u64p), len(thr),
                                            bounds[t], bounds[t + 1] - bounds[t])
    if threads == 1:
        rcs = [rows(0)]
    else:
        from concurrent.futures import ThreadPoolExecutor  # ctypes releases the GIL during the calls
        with ThreadPoolExecutor(threads) as pool:
            rcs = list(pool.map(rows, range(threads)))
    if any(rcs):
        raise ValueError(f"orc_init_bit_planes_rows failed ({rcs})")
    return out


def checksum_planes(planes: np.ndarray, x: int, y: int, n_planes: int, values=None) -> list[int]:
    """The 16-tile checksum computed from bit planes (any word size: the bytes are the same)."""
    w = np.ascontiguousarray(planes).view(np.uint32)
    assert w.size == n_planes * y * x // 32
    vals = np.arange(256, dtype=np.int64) if values is None else np.ascontiguousarray(values, dtype=np.int64)
    out = np.zeros(16, dtype=np.uint64)
    _lib().orc_checksum_planes(_p(w, _u32p), x, y, n_planes, _p(vals, _i64p), _p(out, _u64p))
    return [int(v) for v in out]


def pack(layout: str, cells: np.ndarray, planes: int, word_bits: int) -> np.ndarray:
    c = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = c.shape
    lib = _lib()
    if layout == "bit_planes":
        out = np.zeros(planes * y * x // 8, dtype=np.uint8)
        rc = lib.orc_pack_bit_planes(_p(c, _u8p), x, y, planes, _p(out, _u8p))
    elif layout == "bit_array":
        cpw = word_bits // planes
        out = np.zeros((x * y // cpw) * (word_bits // 8), dtype=np.uint8)
        rc = lib.orc_pack_bit_array(_p(c, _u8p), x, y, planes, word_bits, _p(out, _u8p))
    elif layout == "tiled_bit_planes":
        out = np.zeros(planes * y * x // 8, dtype=np.uint8)
        rc = lib.orc_pack_tiled(_p(c, _u8p), x, y, planes, word_bits, _p(out, _u8p))
    else:
        raise ValueError(layout)
    if rc:
        raise ValueError(f"pack {layout} failed ({rc})")
    return out


def unpack(layout: str, data: np.ndarray, x: int, y: int, planes: int, word_bits: int) -> np.ndarray:
    d = np.ascontiguousarray(data).view(np.uint8)
    cells = np.empty((y, x), dtype=np.uint8)
    lib = _lib()
    if layout == "bit_planes":
        rc = lib.orc_unpack_bit_planes(_p(d, _u8p), x, y, planes, _p(cells, _u8p))
    elif layout == "bit_array":
        rc = lib.orc_unpack_bit_array(_p(d, _u8p), x, y, planes, word_bits, _p(cells, _u8p))
    elif layout == "tiled_bit_planes":
        rc = lib.orc_unpack_tiled(_p(d, _u8p), x, y, planes, word_bits, _p(cells, _u8p))
    else:
        raise ValueError(layout)
    if rc:
        raise ValueError(f"unpack {layout} failed ({rc})")
    return cells


# ---- the reference itself (oracle/_ref) ------------------------------------------------------

def ref_run(automaton: int, cells: np.ndarray, steps: int, layout: str = "standard", word_bits: int = 64):
    """Reference CPU simple traverser; returns (final cells, checksum string)."""
    c = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = c.shape
    out = np.empty_like(c)
    buf = ctypes.create_string_buffer(1024)
    rc = _reflib().ref_run(automaton, LAYOUTS[layout], word_bits, x, y, steps, _p(c, _u8p), _p(out, _u8p), buf, 1024)
    if rc:
        raise ValueError(f"ref_run failed ({rc})")
    return out, buf.value.decode()


def ref_automaton(name: str) -> int:
    """The reference shim's id of the automaton called `name` (config::name)."""
    i = _reflib().ref_automaton_id(name.encode())
    if i < 0:
        raise KeyError(name)
    return i


def ref_run_named(name: str, cells: np.ndarray, steps: int, seed: int = 42, layout: str = "standard",
                  word_bits: int = 64):
    """Reference CPU simple traverser for any automaton the shim knows, with the
    run's random seed; returns (final cells, checksum string)."""
    c = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = c.shape
    out = np.empty_like(c)
    buf = ctypes.create_string_buffer(1024)
    rc = _reflib().ref_run_seeded(ref_automaton(name), LAYOUTS[layout], word_bits, x, y, steps, seed, _p(c, _u8p),
                                  _p(out, _u8p), buf, 1024)
    if rc:
        raise ValueError(f"ref_run_seeded failed ({rc})")
    return out, buf.value.decode()


def ref_pack(automaton: int, layout: str, cells: np.ndarray, word_bits: int) -> np.ndarray:
    c = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = c.shape
    out = np.zeros(x * y, dtype=np.uint8)  # packed layouts never exceed one byte per cell
    n = _reflib().ref_pack(automaton, LAYOUTS[layout], word_bits, x, y, _p(c, _u8p), _p(out, _u8p), out.nbytes)
    if n < 0:
        raise ValueError(f"ref_pack failed ({n})")
    return out[:n].copy()


def ref_run_planes64(automaton: int, planes: np.ndarray, x: int, y: int, steps: int, checkpoints=(), seed: int = 42,
                     report_every: int = 0):
    """Reference CPU simple traverser, bit_planes layout, 64-bit words, over
    caller-given planes (uint64 (P, y, x/64), or any array of those bytes).
    Returns (final planes, {checkpoint: planes after that generation})."""
    p = np.ascontiguousarray(planes).view(np.uint64).copy()
    cps = [int(c) for c in checkpoints if 0 < int(c) < steps]
    snaps = [np.empty_like(p) for _ in cps]
    cp_arr = (ctypes.c_int * max(1, len(cps)))(*cps)
    snap_ptrs = (_u64p * max(1, len(cps)))(*[_p(s_, _u64p) for s_ in snaps])
    rc = _reflib().ref_run_planes64(automaton, x, y, steps, seed, _p(p, _u64p), cp_arr, len(cps), snap_ptrs,
                                    report_every)
    if rc:
        raise ValueError(f"ref_run_planes64 failed ({rc})")
    out = dict(zip(cps, snaps))
    if steps in [int(c) for c in checkpoints]:
        out[steps] = p
    return p, out


def ref_bench_planes64(automaton: int, planes: np.ndarray, x: int, y: int, steps: int, threads: int) -> float:
    """Seconds taken by the slowest of `threads` host threads, each running the
    reference CPU traverser (bit_planes, 64-bit words) on its band of y/threads
    rows of the grid held in `planes` (any array of the plane bytes)."""
    p = np.ascontiguousarray(planes).view(np.uint64)
    s = _reflib().ref_bench_planes64(automaton, x, y, steps, threads, _p(p, _u64p))
    if s < 0:
        raise RuntimeError(f"ref_bench_planes64 failed ({s})")
    return float(s)


def ref_bench(automaton: int, cells: np.ndarray, steps: int, threads: int, layout: str = "bit_planes",
              word_bits: int = 64) -> float:
    """Seconds taken by the slowest of `threads` independent reference traversers."""
    c = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = c.shape
    s = _reflib().ref_bench(automaton, LAYOUTS[layout], word_bits, x, y, steps, threads, _p(c, _u8p))
    if s < 0:
        raise RuntimeError("ref_bench failed")
    return float(s)
