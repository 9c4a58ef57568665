"""Host side of a dB/dt inversion step around the adjoint gradient.

The reference has no inversion code in source form (its inversion module
ships only as compiled objects), so this is the caller the adjoint path
serves: a per-cell log-conductivity model on a regular inversion grid, the
receiver gates of the ``.field2`` output (linear interpolation between the
output rows that bracket each gate time, interp_lin, src/FETD_UTILITY.f90:21-31,
as in src/FETD_FWD.f90:1625-1640) and the least-squares misfit of dB/dt at
those gates, with its derivative with respect to the output rows, which is
what ``FetdGPU.adjoint`` takes.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence, Tuple

import numpy as np


@dataclass
class InversionGrid:
    """A regular grid of cells: ``shape`` = (nx, ny, nz) over ``box`` =
    ((x0, x1), (y0, y1), (z0, z1)) in metres (z > 0 is depth, the reference's
    convention)."""
    shape: Tuple[int, int, int]
    box: Tuple[Tuple[float, float], Tuple[float, float], Tuple[float, float]]

    @property
    def ncell(self) -> int:
        return int(np.prod(self.shape))

    def cell_of_points(self, X: np.ndarray) -> np.ndarray:
        """0-based cell of each point ((nx*ny + ...) ordering: x slowest), -1 outside."""
        idx, inside = [], np.ones(len(X), dtype=bool)
        for a in range(3):
            lo, hi = self.box[a]
            k = np.floor((X[:, a] - lo) / (hi - lo) * self.shape[a]).astype(np.int64)
            inside &= (k >= 0) & (k < self.shape[a])
            idx.append(np.clip(k, 0, self.shape[a] - 1))
        cell = (idx[0] * self.shape[1] + idx[1]) * self.shape[2] + idx[2]
        return np.where(inside, cell, -1)

    def tet_cells(self, nod_cor: np.ndarray, tet_vex: np.ndarray) -> np.ndarray:
        """Cell of each tet by its centroid (tet_vex 1-based), -1 outside."""
        return self.cell_of_points(nod_cor[tet_vex - 1].mean(axis=1))


def lognormal_cells(ncell: int, median: float, sd_decades: float, seed: int) -> np.ndarray:
    """Per-cell conductivities: log10(sigma) ~ N(log10(median), sd_decades^2), seeded."""
    rng = np.random.default_rng(seed)
    return median * 10.0 ** (sd_decades * rng.standard_normal(ncell))


def sigma_with_cells(sig_tet: np.ndarray, tet_cell: np.ndarray, cell_sigma: np.ndarray) -> np.ndarray:
    """sig_tet with every tet inside the grid set to its cell's conductivity."""
    out = np.array(sig_tet, dtype=np.float64, copy=True)
    m = tet_cell >= 0
    out[m] = cell_sigma[tet_cell[m]]
    return out


def gate_matrix(times: np.ndarray, gates: Sequence[float]) -> np.ndarray:
    """W (gates x rows) with gate values = W @ rows: the gate between rows i-1
    and i (the first row whose time reaches the gate) is the straight line
    through them evaluated at the gate time.  A gate at or before the first
    row's time is extrapolated from the first two rows (the library's gate
    loop reaches it again at the second row); a gate after the last row stays
    zero (never reached)."""
    times = np.asarray(times, dtype=np.float64)
    W = np.zeros((len(gates), len(times)))
    for g, tg in enumerate(gates):
        i = int(np.searchsorted(times, tg, side="left"))
        if i >= len(times):
            continue
        if i == 0:
            if len(times) < 2:
                W[g, 0] = 1.0
                continue
            i = 1
        t1, t2 = times[i - 1], times[i]
        w = (tg - t1) / (t2 - t1)
        W[g, i - 1] = 1.0 - w
        W[g, i] = w
    return W


def dbdt_misfit(fields: np.ndarray, times: np.ndarray, gates: Sequence[float], d_obs: np.ndarray,
                component: int = 5) -> Tuple[float, np.ndarray]:
    """J = 1/2 sum over gates and receivers of (d_pred - d_obs)^2 for one
    field component (5 = dB_z/dt) of the output rows ``fields`` (rows, nrec, 9),
    and dJ/dfields in the same layout (the adjoint's input).  d_obs: (gates, nrec)."""
    W = gate_matrix(times, gates)
    pred = W @ fields[:, :, component]
    res = pred - d_obs
    J = 0.5 * float(np.sum(res * res))
    dJ = np.zeros_like(fields)
    dJ[:, :, component] = W.T @ res
    return J, dJ
