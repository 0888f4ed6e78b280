"""Asynchronous, double-buffered q-file snapshots of a resident run.

The reference writes a snapshot every ``iomod`` steps from inside its time loop
(src/main.f90:78-103 calling mpi_snapshot, src/mpi_io.f90:339-497) and waits for the file.
Here ``write()`` only queues work: on the run's stream the device transforms u, v, w, p to
the physical grid (``lsb_snapshot_async``) and copies them into one of two pinned host
buffers, and a writer thread waits for that copy, converts to the file's float32 layout
and writes the file, while the caller keeps stepping.  The second buffer lets the next
snapshot be queued while the previous file is still being written; a third write waits
for the oldest buffer's file to be done.

    w = SnapshotWriter(solver, "out/", stream)     # the solver runs on ``stream``
    for n in range(nsteps // iomod):
        solver.step(iomod)
        w.write(isum=(n + 1) * iomod, t=..., dt=...)
    w.close()                                      # waits for every file
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import formats


class SnapshotWriter:
    def __init__(self, solver, directory: str, stream=None, name: str = "q{isum:05d}.dat",
                 alloc=None, record_event=None):
        """``stream``: a torch CUDA stream the solver is put on (its events order the copies);
        ``alloc(n)`` / ``record_event()`` replace the pinned buffers and CUDA events (tests)."""
        c = solver.cfg
        self.solver = solver
        self.shape = (4, c.nzp, c.ny, c.nx)
        self.dims = (c.nx, c.ny, c.nzp)
        self.dir = directory
        self.name = name
        n = int(np.prod(self.shape))
        if alloc is None or record_event is None:
            import torch
            if stream is None:
                raise ValueError("a CUDA stream is needed to order the copies")
            solver.set_stream(stream.cuda_stream)
            alloc = alloc or (lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True))

            def record_event():
                ev = torch.cuda.Event()
                ev.record(stream)
                return ev
        self._record = record_event
        self.buf = [alloc(n) for _ in range(2)]
        self.busy = [None, None]
        self.next = 0
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.paths = []
        os.makedirs(directory, exist_ok=True)

    @staticmethod
    def _addr(b) -> int:
        return b.data_ptr() if hasattr(b, "data_ptr") else b.ctypes.data

    @staticmethod
    def _view(b) -> np.ndarray:
        return b.numpy() if hasattr(b, "numpy") and not isinstance(b, np.ndarray) else b

    def write(self, isum: int, t: float, dt: float):
        """Queue the snapshot of the run's current state; returns the future of its file."""
        i = self.next
        self.next ^= 1
        if self.busy[i] is not None:
            self.busy[i].result()          # the writer is done with this buffer
        self.solver.snapshot_async(self._addr(self.buf[i]))
        ev = self._record()
        path = os.path.join(self.dir, self.name.format(isum=isum))
        self.paths.append(path)
        self.busy[i] = self.pool.submit(self._job, i, ev, path, isum, t, dt)
        return self.busy[i]

    def _job(self, i, ev, path, isum, t, dt) -> str:
        ev.synchronize()
        q = self._view(self.buf[i]).reshape(self.shape)
        nx, ny, nzp = self.dims
        T = np.zeros(self.shape[1:])   # temperature is identically zero (not carried)
        formats.write_snapshot(path, formats.Snapshot(isum, t, dt, nx, ny, nzp, ny, q[0], q[1], q[2], T, q[3]))
        return path

    def close(self):
        for f in self.busy:
            if f is not None:
                f.result()
        self.pool.shutdown(wait=True)
