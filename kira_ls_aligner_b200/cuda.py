"""Drop-in mirror of kira-ls-aligner's GPU backend (src/cuda/).

* ``CudaJob`` / ``CudaResult`` / ``CudaBackend``  -- src/cuda/backend.rs:13-262
* ``is_available``                                -- src/cuda/mod.rs:39-49
* ``dispatcher.start/dispatch/is_active/stop``    -- src/cuda/dispatcher.rs:20-104

``CudaBackend.run_batch`` keeps the reference's argument meaning, result
sentinels and error behaviour (ReadTooLong before any device work, errors as
exceptions of the CudaError family) but ships only phase 0 of the pre-shifted
window: the kernel derives the other bit phases itself.
"""
from __future__ import annotations

import queue
import threading
from dataclasses import dataclass
from typing import Optional, Sequence

from . import _abi as A
from .runtime import (CudaError, DriverError, GpuContext, NoDevice, NotBuilt, ReadTooLong,
                      RuntimeFailure, is_available)

READ_BYTES_MAX = A.READ_BYTES_MAX

__all__ = ["CudaJob", "CudaResult", "CudaBackend", "CudaError", "NotBuilt", "DriverError",
           "RuntimeFailure", "NoDevice", "ReadTooLong", "is_available", "dispatcher",
           "READ_BYTES_MAX"]


@dataclass
class CudaJob:
    """One read against its padded reference window (backend.rs:13-26)."""
    read_packed: bytes
    read_nucs: int
    ref_shifted: Sequence[bytes]
    ref_nucs: int
    max_mismatches: int


@dataclass
class CudaResult:
    """backend.rs:28-35: shift -1 when rejected; second None when absent."""
    shift: int
    mismatches: int
    second_mismatches: Optional[int]


class CudaBackend:
    """GPU sieve backend; hold one per worker thread (backend.rs:42-59)."""

    def __init__(self, device: int = 0):
        self._ctx = GpuContext(device)

    @classmethod
    def new(cls, device: int = 0) -> "CudaBackend":
        return cls(device)

    def run_batch(self, jobs: Sequence[CudaJob]) -> list:
        """Process a batch of jobs in one launch (backend.rs:95-249)."""
        if not jobs:
            return []
        for j in jobs:
            if len(j.read_packed) > READ_BYTES_MAX:
                raise ReadTooLong(
                    f"read too long for the CUDA backend ({len(j.read_packed)} > "
                    f"{READ_BYTES_MAX} bytes packed)", len(j.read_packed), READ_BYTES_MAX)
            l0 = len(j.ref_shifted[0])
            if any(len(p) != l0 for p in j.ref_shifted):
                raise RuntimeFailure("ref_shifted phases have different lengths")
        out = self._ctx.sieve_batch(list(jobs))
        return [CudaResult(int(s), int(m), None if sec == A.INT32_MAX else int(sec))
                for s, m, sec in out]

    def release_buffers(self) -> None:
        self._ctx.close()

    @property
    def context(self) -> GpuContext:
        return self._ctx


class _Dispatcher:
    """Single GPU worker thread behind a channel (dispatcher.rs:20-104)."""

    def __init__(self):
        self._lock = threading.Lock()
        self._state = None  # (queue, thread)

    def start(self, device: int = 0) -> None:
        with self._lock:
            if self._state is not None:
                return
            q: "queue.Queue" = queue.Queue()

            def worker():
                try:
                    backend = CudaBackend(device)
                except CudaError as e:  # dispatcher.rs:33-43: every request gets the error
                    while True:
                        item = q.get()
                        if item is None:
                            return
                        item[1].put(DriverError(f"GPU worker thread is dead: {e}"))
                while True:
                    item = q.get()
                    if item is None:
                        backend.release_buffers()
                        return
                    jobs, reply = item
                    try:
                        reply.put(backend.run_batch(jobs))
                    except CudaError as e:
                        reply.put(e)

            t = threading.Thread(target=worker, name="kira-cuda-dispatch", daemon=True)
            t.start()
            self._state = (q, t)

    def dispatch(self, jobs: Sequence[CudaJob]):
        """Blocking submit; None on any error (the caller then takes its CPU path)."""
        if not jobs:
            return []
        with self._lock:
            st = self._state
            if st is None:
                return None
            reply: "queue.Queue" = queue.Queue()
            st[0].put((list(jobs), reply))
        r = reply.get()
        return None if isinstance(r, Exception) else r

    def is_active(self) -> bool:
        with self._lock:
            return self._state is not None

    def stop(self) -> None:
        with self._lock:
            st, self._state = self._state, None
        if st is not None:
            st[0].put(None)
            st[1].join()


dispatcher = _Dispatcher()
