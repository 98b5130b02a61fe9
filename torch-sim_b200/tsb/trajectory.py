"""Trajectory reporting from the persistent fused MD kernel.

The reference's ``TrajectoryReporter`` (torch_sim/trajectory.py:69-461) is called
by the runner on the host every step and writes HDF5 through PyTables.  A
persistent kernel never returns to the host between steps, so here the kernel
itself writes every ``state_frequency``-th step into a device frame buffer
(positions as float32, the reference's default ``coerce_to_float32``, and each
system's potential energy; ``tsb_fused_md_ex``), and the host drains it:

* the run is split into chunks of ``frames_per_chunk * state_frequency`` steps;
* two device frame buffers alternate, so chunk k+1 runs while chunk k's frames
  are copied into pinned host memory on a side stream;
* a writer thread appends the frames per system; ``close()`` writes one NumPy
  ``.npz`` file per system (``positions [frames, n, 3]``, ``potential_energy
  [frames]``, ``step``, ``atomic_numbers``, ``masses``, ``cell``, ``pbc``) --
  HDF5 needs PyTables or h5py, which this package does not depend on.
"""

from __future__ import annotations

import queue
import threading

import numpy as np
import torch


class FusedTrajectory:
    def __init__(self, runner, filenames, *, state_frequency: int = 100,
                 frames_per_chunk: int = 10) -> None:
        self.runner = runner
        n_sys = runner.n_sys
        if isinstance(filenames, (str, bytes)):
            filenames = [filenames]
        if len(filenames) != n_sys:
            raise ValueError(f"need one filename per system ({n_sys}), got {len(filenames)}")
        self.filenames = list(filenames)
        self.every = int(state_frequency)
        self.fpc = int(frames_per_chunk)
        if self.every < 1 or self.fpc < 1:
            raise ValueError("state_frequency and frames_per_chunk must be >= 1")
        dev, n = runner.dev, runner.n
        self.dev_x = [torch.empty((self.fpc, n, 3), dtype=torch.float32, device=dev)
                      for _ in range(2)]
        self.dev_e = [torch.empty((self.fpc, n_sys), dtype=torch.float64, device=dev)
                      for _ in range(2)]
        self.host_x = [torch.empty((self.fpc, n, 3), dtype=torch.float32).pin_memory()
                       for _ in range(2)]
        self.host_e = [torch.empty((self.fpc, n_sys), dtype=torch.float64).pin_memory()
                       for _ in range(2)]
        self.copy_stream = torch.cuda.Stream(dev)
        self.copied = [torch.cuda.Event() for _ in range(2)]
        self.host_free = [threading.Event() for _ in range(2)]
        for e in self.host_free:
            e.set()
        bounds = torch.bincount(runner.sys_idx, minlength=n_sys).cumsum(0).cpu().numpy()
        self.lo = np.concatenate([[0], bounds[:-1]])
        self.hi = bounds
        self.frames_x = [[] for _ in range(n_sys)]
        self.frames_e = [[] for _ in range(n_sys)]
        self.steps: list[int] = []
        self.step0 = 0
        self._q: queue.Queue = queue.Queue()
        self._writer = threading.Thread(target=self._drain, daemon=True)
        self._writer.start()

    def _drain(self):
        while True:
            item = self._q.get()
            if item is None:
                return
            b, n_frames, first_step = item
            self.copied[b].synchronize()
            x = self.host_x[b][:n_frames].numpy()
            e = self.host_e[b][:n_frames].numpy()
            for s in range(len(self.filenames)):
                self.frames_x[s].append(x[:, self.lo[s]:self.hi[s]].copy())
                self.frames_e[s].append(e[:, s].copy())
            self.steps.extend(first_step + self.every * k for k in range(n_frames))
            self.host_free[b].set()

    def run(self, n_steps: int):
        """Advance the runner by n_steps, recording a frame every state_frequency steps."""
        r = self.runner
        main = torch.cuda.current_stream(r.dev)
        done, b = 0, 0
        chunk = self.every * self.fpc
        used = [False, False]
        while done < n_steps:
            steps = min(chunk, n_steps - done)
            n_frames = steps // self.every
            if used[b]:  # the copy out of this device buffer (two chunks ago) is done
                main.wait_event(self.copied[b])
            r.launch(steps, frames=(self.dev_x[b], self.dev_e[b], self.every))
            if n_frames:
                ev = torch.cuda.Event()
                ev.record(main)
                self.host_free[b].wait()  # the writer is done with this pinned buffer
                self.host_free[b].clear()
                with torch.cuda.stream(self.copy_stream):
                    self.copy_stream.wait_event(ev)
                    self.host_x[b][:n_frames].copy_(self.dev_x[b][:n_frames], non_blocking=True)
                    self.host_e[b][:n_frames].copy_(self.dev_e[b][:n_frames], non_blocking=True)
                    self.copied[b].record(self.copy_stream)
                used[b] = True
                self._q.put((b, n_frames, self.step0 + done + self.every))
            done += steps
            b ^= 1
        self.step0 += n_steps
        return r

    def close(self, state=None):
        """Wait for the writer and write one .npz per system."""
        self._q.put(None)
        self._writer.join()
        r = self.runner
        st = state if state is not None else r.state
        z = st.atomic_numbers.cpu().numpy()
        masses = st.masses.double().cpu().numpy()
        cell = st.cell.double().cpu().numpy()
        pbc = np.broadcast_to(np.asarray(st.pbc.cpu() if torch.is_tensor(st.pbc) else st.pbc),
                              (len(self.filenames), 3))
        for s, fn in enumerate(self.filenames):
            lo, hi = self.lo[s], self.hi[s]
            pos = (np.concatenate(self.frames_x[s]) if self.frames_x[s]
                   else np.zeros((0, hi - lo, 3), np.float32))
            pe = np.concatenate(self.frames_e[s]) if self.frames_e[s] else np.zeros(0)
            np.savez(fn, positions=pos, potential_energy=pe, step=np.asarray(self.steps),
                     atomic_numbers=z[lo:hi], masses=masses[lo:hi], cell=cell[s], pbc=pbc[s])
