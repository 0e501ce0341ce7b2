"""Python view of the serving loop (``cb2_server``): continuous batching of
simulation requests with admission by device-memory budget."""
from __future__ import annotations

import ctypes
from fractions import Fraction

import numpy as np

from . import _abi
from ._abi import check, lib
from .grid import automaton_id, automaton_info, thresholds

STATES = {_abi.REQ_QUEUED: "queued", _abi.REQ_ACTIVE: "active", _abi.REQ_DONE: "done", _abi.REQ_FAILED: "failed"}


class Server:
    """One server thread on the current device.  ``per_request=True`` runs the
    plain one-request-at-a-time path with the same interface."""

    def __init__(self, memory_budget: int = 0, max_active: int = 0, chunk_steps: int = 0, temporal_steps: int = 0,
                 tile_rows: int = 0, per_request: bool = False, task_capacity: int = 0, spin_limit: int = 0,
                 fail_alloc_at: int = 0, round_cells: float = 0.0, direct_cells: int = 0):
        opts = _abi.ServerOpts(memory_budget, max_active, chunk_steps, temporal_steps, tile_rows, int(per_request),
                               task_capacity, spin_limit, fail_alloc_at, round_cells, direct_cells)
        h = ctypes.c_void_p()
        check(lib.cb2_server_create(ctypes.byref(opts), ctypes.byref(h)), "server create")
        self._h = h
        self._keep = {}  # host buffers that must outlive their requests

    def close(self):
        if getattr(self, "_h", None):
            lib.cb2_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, automaton, x_size: int, y_size: int, steps: int, seed: int = 0, probs=None,
               cells: np.ndarray | None = None, want_cells: bool = False) -> int:
        """Queues a request; returns its id.  Input: ``cells`` (uint8 indexes,
        shape (y, x)) or the seeded generator with ``probs`` (default uniform)."""
        a = automaton_id(automaton)
        req = _abi.Request()
        req.automaton, req.x_size, req.y_size, req.steps, req.seed = a, x_size, y_size, steps, seed
        keep = []
        if cells is not None:
            c = np.ascontiguousarray(cells, dtype=np.uint8)
            if c.shape != (y_size, x_size):
                raise ValueError("cells must have shape (y_size, x_size)")
            keep.append(c)
            req.host_cells = c.ctypes.data
        else:
            if probs is None:
                states = automaton_info(a)[2]
                probs = [Fraction(1, states)] * states
            t = thresholds(probs)
            req.n_thresholds = len(t)
            for i, v in enumerate(t):
                req.thresholds[i] = int(v)
        out = None
        if want_cells:
            out = np.zeros((y_size, x_size), dtype=np.uint8)
            keep.append(out)
            req.host_result = out.ctypes.data
        rid = ctypes.c_int64()
        check(lib.cb2_server_submit(self._h, ctypes.byref(req), ctypes.byref(rid)), "submit")
        self._keep[rid.value] = (keep, out)
        return rid.value

    def status(self, rid: int) -> dict:
        st = _abi.RequestStatus()
        check(lib.cb2_server_status(self._h, rid, ctypes.byref(st)), "status")
        return {"state": STATES[st.state], "error": st.error, "steps_done": st.steps_done, "submit_s": st.submit_s,
                "admit_s": st.admit_s, "done_s": st.done_s, "checksum": [int(v) for v in st.checksum]}

    def wait(self, rid: int, timeout_s: float = 600.0) -> dict:
        check(lib.cb2_server_wait(self._h, rid, timeout_s), f"request {rid}")
        return self.status(rid)

    def result_cells(self, rid: int) -> np.ndarray | None:
        return self._keep.get(rid, (None, None))[1]

    def drain(self, timeout_s: float = 600.0) -> None:
        check(lib.cb2_server_drain(self._h, timeout_s), "drain")

    def stats(self) -> dict:
        s = _abi.ServerStats()
        check(lib.cb2_server_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}
