"""cellato_b200 -- B200 (sm_100a) bit-plane traverser backend for the Cellato DSL.

The compute path is ``libcellato_b200.so`` (hand-written CUDA for sm_100a
behind the C-ABI in ``include/cellato_b200.h``); this package is a thin
ctypes layer over it that mirrors the reference's traverser, grid and
run_params surface.  Importing it without the built library raises.
"""
from ._abi import CudaError, StateError, last_error
from .grid import (AUTOMATA, Batch, DeviceGrid, HostGrid, autotune, automaton_id, automaton_info, layout_bytes,
                   measure_lop3_peak, network_ops, plan, run_bit_planes, thresholds, tuning_load, tuning_save,
                   variants)
from .serve import Server
from .traverser import RunParams, Traverser, run_experiment

__all__ = [
    "AUTOMATA", "Batch", "CudaError", "DeviceGrid", "HostGrid", "RunParams", "Server", "StateError", "Traverser", "autotune",
    "automaton_id", "automaton_info", "last_error", "layout_bytes", "measure_lop3_peak", "network_ops", "plan",
    "run_bit_planes", "run_experiment", "thresholds", "tuning_load", "tuning_save", "variants",
]
