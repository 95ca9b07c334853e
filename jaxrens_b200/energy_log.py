"""The ``.energies`` dead-point log (``io/energy_log.py:24-104``).

Header ``n_walkers n_cull n_dof 0.0 n_atoms``; one row ``iteration energy
volume`` (``%.10e``) per dead point, ``n_cull`` rows per iteration in
descending energy, the volume ``|det(cell)|`` of the dead walker's own cell
(``cli/monitor.py`` energy logging).  Energies are written as the float32
values the reference's ``MCState.energy`` holds.

``EnergyLogCallback`` is the bulk writer for ``run_loop``: the walk kernel
leaves a whole launch's dead points in its info buffers, so the callback
copies them to the host once per launch instead of once per iteration.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np


@dataclass
class EnergyLog:
    iterations: np.ndarray
    energies: np.ndarray
    volumes: np.ndarray
    n_walkers: int
    n_cull: int
    n_atoms: int
    n_dof: int


class EnergyLogger:
    """Writes and reads one run's ``.energies`` file."""

    def __init__(self, path, n_walkers: int, n_cull: int = 1, n_dof: int = 0, n_atoms: int = 0,
                 mode: str = "w"):
        self.path = Path(path)
        self.n_walkers, self.n_cull, self.n_dof, self.n_atoms = n_walkers, n_cull, n_dof, n_atoms
        self._mode = mode
        self._file = None

    def write_header(self) -> None:
        self.path.parent.mkdir(parents=True, exist_ok=True)
        skip = self._mode == "a" and self.path.exists() and self.path.stat().st_size > 0
        self._file = open(self.path, self._mode)
        if not skip:
            self._file.write(f"{self.n_walkers} {self.n_cull} {self.n_dof} 0.0 {self.n_atoms}\n")
            self._file.flush()

    def write_entry(self, iteration: int, energy: float, volume: float = 0.0) -> None:
        if self._file is None:
            self.write_header()
        self._file.write(f"{iteration} {energy:.10e} {volume:.10e}\n")

    def write_entries(self, iterations, energies, volumes) -> None:
        """Many rows at once (one flush)."""
        if self._file is None:
            self.write_header()
        self._file.write("".join(f"{int(i)} {float(e):.10e} {float(v):.10e}\n"
                                 for i, e, v in zip(iterations, energies, volumes)))
        self._file.flush()

    def close(self) -> None:
        if self._file is not None:
            self._file.close()
            self._file = None

    @staticmethod
    def read(path) -> EnergyLog:
        with open(path) as f:
            h = f.readline().split()
            rows = [ln.split() for ln in f if len(ln.split()) >= 2]
        return EnergyLog(np.array([int(r[0]) for r in rows]),
                         np.array([float(r[1]) for r in rows]),
                         np.array([float(r[2]) if len(r) > 2 else 0.0 for r in rows]),
                         int(h[0]), int(h[1]), int(h[4]) if len(h) > 4 else 0, int(h[2]))


def dead_point_rows(first_iteration: int, dead_energy, dead_cell):
    """Rows of ``n_iter`` iterations for one run: ``dead_energy`` ``(n_iter,
    n_cull)`` float64 and ``dead_cell`` ``(n_iter, n_cull, 3, 3)`` float32 ->
    (iterations, float32 energies, volumes), descending energy per iteration."""
    e = np.asarray(dead_energy, np.float64)
    c = np.asarray(dead_cell, np.float32)
    n_iter, n_cull = e.shape
    its = np.repeat(np.arange(first_iteration, first_iteration + n_iter), n_cull)
    ens = e.astype(np.float32).reshape(-1).astype(np.float64)
    vols = np.abs(np.linalg.det(c.reshape(-1, 3, 3))).astype(np.float64)
    return its, ens, vols


class EnergyLogCallback:
    """``run_loop`` callback writing every run's ``.energies`` in bulk, one
    device-to-host copy per launch (``on_launch``)."""

    def __init__(self, paths, n_walkers: int, n_cull: int = 1, n_atoms: int = 0, n_dof: int = 0):
        self.loggers = [EnergyLogger(p, n_walkers, n_cull, n_dof, n_atoms) for p in paths]

    def on_launch(self, first_iteration: int, info, n_keep: int) -> None:
        e = info.dead_energy[:n_keep].detach().cpu().numpy()
        c = info.dead_cell[:n_keep].detach().cpu().numpy()
        if info.n_cull == 1:
            e = e[:, :, None]
            c = c[:, :, None]
        for r, lg in enumerate(self.loggers):
            lg.write_entries(*dead_point_rows(first_iteration, e[:, r], c[:, r]))

    def close(self) -> None:
        for lg in self.loggers:
            lg.close()
