"""Batched time loop: many independent solves advanced by one graph launch per step.

Each member is a :class:`~lssph.simulation.Simulation`; the batch launches every phase
kernel of a time step once for all members of the same kind, so a step of 64 small
solves costs about as many launches as a step of one.  Members compute exactly what
``Simulation.step`` computes for them alone (bit-identical), stop at their own steady
state or error, and may join or leave between calls (continuous batching).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import LssphError, check, iptr
from .simulation import Simulation


class Batch:
    """An ``lssph_batch``: members in the order they were added."""

    def __init__(self):
        self._lib = _abi.load()
        b = C.c_void_p()
        check(self._lib.lssph_batch_create(C.byref(b)))
        self._b = b
        self.members: list[Simulation] = []

    def close(self) -> None:
        if getattr(self, "_b", None):
            self._lib.lssph_batch_destroy(self._b)
            self._b = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self) -> int:
        return len(self.members)

    def _chk(self, status: int) -> int:
        if status == _abi.OK:
            return status
        msg = self._lib.lssph_batch_error(self._b) or b""
        raise LssphError(status, msg.decode(errors="replace"))

    def add(self, sim: Simulation) -> int:
        """Add a solve; returns its member index."""
        self._chk(self._lib.lssph_batch_add(self._b, sim._h))
        self.members.append(sim)
        return len(self.members) - 1

    def remove(self, sim: Simulation) -> None:
        self._chk(self._lib.lssph_batch_remove(self._b, sim._h))
        self.members = [m for m in self.members if m is not sim]

    def step(self, nsteps: int = 1, raise_on_error: bool = True) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Advance every member nsteps steps.

        Returns (status, steady, steps): per-member status codes, the 1-based step within
        this call at which each member reached a steady state (0 = not reached), and the
        steps each member actually advanced (fewer once it stopped).  With raise_on_error,
        a member error raises LssphError after the call.
        """
        n = len(self.members)
        status = np.zeros(n, dtype=np.int32)
        steady = np.zeros(n, dtype=np.int32)
        steps = np.zeros(n, dtype=np.int32)
        rc = self._lib.lssph_batch_step(self._b, int(nsteps), iptr(status) if n else None,
                                        iptr(steady) if n else None, iptr(steps) if n else None)
        if rc == _abi.E_CUDA or (raise_on_error and rc != _abi.OK):
            self._chk(rc)
        return status, steady, steps

    def launch(self, nsteps: int = 1) -> None:
        """Start a step call; the host is free until wait().  No add/remove meanwhile."""
        self._chk(self._lib.lssph_batch_launch(self._b, int(nsteps)))

    def wait(self, raise_on_error: bool = True) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Finish the call started by launch(); returns what step() returns."""
        n = len(self.members)
        status = np.zeros(n, dtype=np.int32)
        steady = np.zeros(n, dtype=np.int32)
        steps = np.zeros(n, dtype=np.int32)
        rc = self._lib.lssph_batch_wait(self._b, iptr(status) if n else None, iptr(steady) if n else None,
                                        iptr(steps) if n else None)
        if rc == _abi.E_CUDA or (raise_on_error and rc != _abi.OK):
            self._chk(rc)
        return status, steady, steps

    def last_step_stats(self) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_int64()
        self._chk(self._lib.lssph_batch_last_step_stats(self._b, C.byref(ms), C.byref(n)))
        return ms.value, n.value
