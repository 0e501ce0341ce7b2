"""ctypes binding of the C-ABI in ``include/cellato_b200.h``.

The library ``libcellato_b200.so`` is built in-tree (``__graft_entry__.build()``
or ``make -C cellato_b200/csrc``).  There is no fallback: if the library is
missing, importing this module raises ``ImportError``.

Status codes become the exception types the reference raises for the same
conditions: ``CudaError`` for CUDA failures (traversers/cuda_utils.cuh:37-47),
``ValueError`` for invalid arguments (std::invalid_argument), ``LookupError``
for unknown names, ``MemoryError`` for exhausted device memory and
``TimeoutError`` for bounded device waits that gave up.
"""
from __future__ import annotations

import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcellato_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "cellato_b200.h")

CB2_OK = 0
CB2_EINVAL = -1
CB2_ECUDA = -2
CB2_ENOMEM = -3
CB2_ESTATE = -4
CB2_ETIMEOUT = -5
CB2_ENOTFOUND = -6

LAYOUT_STANDARD = 0
LAYOUT_BIT_ARRAY = 1
LAYOUT_BIT_PLANES = 2
LAYOUT_TILED_BIT_PLANES = 3
LAYOUTS = {
    "standard": LAYOUT_STANDARD,
    "bit_array": LAYOUT_BIT_ARRAY,
    "bit_planes": LAYOUT_BIT_PLANES,
    "tiled_bit_planes": LAYOUT_TILED_BIT_PLANES,
}


class CudaError(RuntimeError):
    """A CUDA runtime call inside the library failed."""


class StateError(ValueError):
    """A cell value is not an index of the automaton's state dictionary."""


class Tuning(ctypes.Structure):
    _fields_ = [("temporal_steps", ctypes.c_int), ("tile_rows", ctypes.c_int), ("words_per_lane", ctypes.c_int),
                ("levels_per_warp", ctypes.c_int), ("rows_per_step", ctypes.c_int)]

    def as_dict(self):
        return {"temporal_steps": self.temporal_steps, "tile_rows": self.tile_rows,
                "words_per_lane": self.words_per_lane, "levels_per_warp": self.levels_per_warp,
                "rows_per_step": self.rows_per_step}


class BatchOpts(ctypes.Structure):
    _fields_ = [("temporal_steps", ctypes.c_int), ("tile_rows", ctypes.c_int), ("spin_limit", ctypes.c_longlong),
                ("stall_task", ctypes.c_int)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("memory_budget", ctypes.c_size_t), ("max_active", ctypes.c_int), ("chunk_steps", ctypes.c_int),
                ("temporal_steps", ctypes.c_int), ("tile_rows", ctypes.c_int), ("per_request", ctypes.c_int),
                ("task_capacity", ctypes.c_int), ("spin_limit", ctypes.c_longlong),
                ("fail_alloc_at", ctypes.c_longlong), ("round_cells", ctypes.c_double),
                ("direct_cells", ctypes.c_longlong)]


class Request(ctypes.Structure):
    _fields_ = [("automaton", ctypes.c_int), ("x_size", ctypes.c_int64), ("y_size", ctypes.c_int64),
                ("steps", ctypes.c_int64), ("seed", ctypes.c_uint64), ("n_thresholds", ctypes.c_int),
                ("thresholds", ctypes.c_uint64 * 31), ("host_cells", ctypes.c_void_p),
                ("host_result", ctypes.c_void_p)]


class RequestStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("error", ctypes.c_int), ("steps_done", ctypes.c_int64),
                ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("checksum", ctypes.c_uint64 * 16)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("rounds", ctypes.c_int64), ("cell_updates", ctypes.c_double), ("used_bytes", ctypes.c_int64),
                ("budget_bytes", ctypes.c_int64), ("now_s", ctypes.c_double), ("plan_s", ctypes.c_double),
                ("wait_s", ctypes.c_double), ("tasks", ctypes.c_int64)]


REQ_QUEUED, REQ_ACTIVE, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_vpp = ctypes.POINTER(ctypes.c_void_p)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_tp = ctypes.POINTER(Tuning)
# cb2_halo_exchange_fn: (user, buffer, k, stream) -> status
HALO_EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p)

# name -> (restype, argtypes)
_SIGNATURES = {
    "cb2_abi_version": (ctypes.c_int, []),
    "cb2_last_error": (ctypes.c_char_p, []),
    "cb2_automaton_lookup": (ctypes.c_int, [ctypes.c_char_p]),
    "cb2_automaton_info": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "cb2_automaton_count": (ctypes.c_int, []),
    "cb2_automaton_fingerprint": (ctypes.c_int, [ctypes.c_int, _u64p]),
    "cb2_automaton_values": (ctypes.c_int, [ctypes.c_int, _i64p, ctypes.c_int]),
    "cb2_run_bit_planes": (ctypes.c_int, [ctypes.c_int, _vpp, _vpp, _i64, _i64, _i64, _tp, _vp,
                                          ctypes.POINTER(ctypes.c_int)]),
    "cb2_run_bit_planes_at": (ctypes.c_int, [ctypes.c_int, _vpp, _vpp, _i64, _i64, _i64, _i64, ctypes.c_uint64, _tp,
                                             _vp, ctypes.POINTER(ctypes.c_int)]),
    "cb2_run_bit_planes_in_place": (ctypes.c_int, [ctypes.c_int, _vpp, _i64, _i64, _i64, _i64, ctypes.c_uint64, _tp,
                                                    _vp]),
    "cb2_band_pass": (ctypes.c_int, [ctypes.c_int, _vpp, _vpp, _i64, _i64, _i64, _i64, ctypes.c_int, _tp, _vp]),
    "cb2_band_pass_at": (ctypes.c_int, [ctypes.c_int, _vpp, _vpp, _i64, _i64, _i64, _i64, ctypes.c_int, _i64,
                                        ctypes.c_uint64, _i64, _i64, _tp, _vp]),
    "cb2_band_schedule": (_i64, [_i64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _i64]),
    "cb2_band_run": (ctypes.c_int, [ctypes.c_int, _vpp, _vpp, _i64, _i64, ctypes.c_int, _i64, _i64, ctypes.c_uint64,
                                    _i64, _i64, _tp, HALO_EXCHANGE_FN, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int)]),
    "cb2_fill_random_planes": (ctypes.c_int, [ctypes.c_int, _vpp, _i64, _i64, _i64, _i64, ctypes.c_uint64, _u64p,
                                              ctypes.c_int, _vp]),
    "cb2_checksum_planes": (ctypes.c_int, [ctypes.c_int, _vpp, _i64, _i64, _i64, _i64, _i64, _i64, _i64p,
                                           ctypes.c_int, _u64p, _vp]),
    "cb2_grid_create": (ctypes.c_int, [ctypes.c_int, _i64, _i64, ctypes.POINTER(_vp)]),
    "cb2_grid_destroy": (ctypes.c_int, [_vp]),
    "cb2_grid_upload": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "cb2_grid_download": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "cb2_grid_upload_async": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "cb2_grid_download_async": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "cb2_layout_bytes": (_i64, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64, _i64]),
    "cb2_grid_fill_random": (ctypes.c_int, [_vp, ctypes.c_uint64, _u64p, ctypes.c_int, _vp]),
    "cb2_grid_run": (ctypes.c_int, [_vp, _i64, _tp, _vp]),
    "cb2_grid_checksum": (ctypes.c_int, [_vp, _i64p, ctypes.c_int, _u64p, _vp]),
    "cb2_grid_planes": (ctypes.c_int, [_vp, _vpp, ctypes.POINTER(ctypes.c_int), _i64p]),
    "cb2_grid_time_step": (_i64, [_vp]),
    "cb2_grid_set_seed": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "cb2_grid_set_time_step": (ctypes.c_int, [_vp, _i64]),
    "cb2_batch_create": (ctypes.c_int, [_vpp, _i64p, ctypes.c_int, ctypes.POINTER(BatchOpts), ctypes.POINTER(_vp)]),
    "cb2_batch_destroy": (ctypes.c_int, [_vp]),
    "cb2_batch_run": (ctypes.c_int, [_vp, _vp]),
    "cb2_batch_wait": (ctypes.c_int, [_vp, _vp]),
    "cb2_batch_run_per_grid": (ctypes.c_int, [_vp, _vp]),
    "cb2_batch_info": (ctypes.c_int, [_vp, _i64p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "cb2_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOpts), ctypes.POINTER(_vp)]),
    "cb2_server_submit": (ctypes.c_int, [_vp, ctypes.POINTER(Request), _i64p]),
    "cb2_server_status": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(RequestStatus)]),
    "cb2_server_wait": (ctypes.c_int, [_vp, _i64, ctypes.c_double]),
    "cb2_server_drain": (ctypes.c_int, [_vp, ctypes.c_double]),
    "cb2_server_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ServerStats)]),
    "cb2_server_destroy": (ctypes.c_int, [_vp]),
    "cb2_autotune": (ctypes.c_int, [ctypes.c_int, _i64, _i64, ctypes.c_double, _tp]),
    "cb2_tuning_load": (ctypes.c_int, [ctypes.c_char_p]),
    "cb2_tuning_save": (ctypes.c_int, [ctypes.c_char_p]),
    "cb2_plan": (ctypes.c_int, [ctypes.c_int, _i64, _i64, _tp, _tp]),
    "cb2_variants": (ctypes.c_int, [ctypes.c_int, _tp, ctypes.c_int]),
    "cb2_measure_lop3_peak": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double)]),
    "cb2_network_ops": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double)]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; g.build()'` "
                          "or `make -C cellato_b200/csrc` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    msg = lib.cb2_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str = "") -> int:
    """Raise the exception matching a negative status code; return rc otherwise."""
    if rc >= 0:
        return rc
    msg = last_error()
    text = f"{what}: {msg}" if what else msg
    if rc == CB2_ECUDA:
        raise CudaError(text)
    if rc == CB2_ESTATE:
        raise StateError(text)
    if rc == CB2_ENOMEM:
        raise MemoryError(text)
    if rc == CB2_ETIMEOUT:
        raise TimeoutError(text)
    if rc == CB2_ENOTFOUND:
        raise LookupError(text)
    raise ValueError(text)


def declared_symbols() -> list[str]:
    """Function names the public header declares (for the ABI export test)."""
    with open(HEADER_PATH) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(cb2_[a-z0-9_]+)\s*\(", text)))


def tuning(temporal_steps: int = 0, tile_rows: int = 0, words_per_lane: int = 0, levels_per_warp: int = 0,
           rows_per_step: int = 0) -> Tuning:
    return Tuning(temporal_steps, tile_rows, words_per_lane, levels_per_warp, rows_per_step)
