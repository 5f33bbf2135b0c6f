"""Row-strip decomposition of one basin over several domains (ranks).

The reference decomposes its basin over a 2-D MPI process grid in
mpi_array_boundary_definition (Control/init_arrays.f90:21-88) and exchanges
one halo row or column per field update with syncborder_real8
(Modules/mod_mpi_parallel_tools.f90:179-252).  The B200 path uses a 1 x P
grid of row strips (one strip per GPU): strip_bounds() applies the
reference's formula for p_size = (1, P), split_basin() cuts a global Basin
into the strips' local arrays (each with its two-row halo from the global
arrays) and gather_state() reassembles the state from the strips.
"""
from __future__ import annotations

from dataclasses import replace
from typing import List

import numpy as np

from .grid import Basin, Bounds


def strip_bounds(b: Bounds, nranks: int) -> List[Bounds]:
    """Local bounds of the strips of a 1 x nranks process grid, south to
    north: Control/init_arrays.f90:59-70 with p_size(2) = nranks (locn rows
    each, the last strip takes the rest); x is not split."""
    if nranks < 1:
        raise ValueError("nranks < 1")
    ny = b.bnd_y2 - b.bnd_y1 + 1                 # global array rows
    locn = (ny - 4) // nranks
    if locn < 1:
        raise ValueError(f"{ny - 4} interior rows cannot be split over {nranks} strips")
    out = []
    for k in range(nranks):
        ny_start = locn * k + b.bnd_y1 + 2
        ny_end = ny_start + locn - 1 if k < nranks - 1 else b.bnd_y2 - 2
        out.append(replace(b, ny_start=ny_start, ny_end=ny_end, bnd_y1=ny_start - 2, bnd_y2=ny_end + 2))
    return out


def _rows(a: np.ndarray, g: Bounds, lb: Bounds) -> np.ndarray:
    return np.asfortranarray(a[:, lb.bnd_y1 - g.bnd_y1: lb.bnd_y2 - g.bnd_y1 + 1].copy(order="F"))


def split_basin(basin: Basin, nranks: int) -> List[Basin]:
    """Local Basins of the strips: every array restricted to the strip's
    rows bnd_y1..bnd_y2 (interior and two halo rows each side, taken from
    the global arrays)."""
    g = basin.bounds
    out = []
    for lb in strip_bounds(g, nranks):
        def cut(d):
            return {k: _rows(v, g, lb) for k, v in d.items()}
        loc = Basin(lb, basin.consts, cut(basin.masks), cut(basin.metrics),
                    None if basin.rlh_s is None else _rows(basin.rlh_s, g, lb),
                    None if basin.hhq_rest is None else _rows(basin.hhq_rest, g, lb),
                    cut(basin.depths), cut(basin.state), cut(basin.means), cut(basin.forcing),
                    cut(basin.scratch),
                    None if basin.taux is None else _rows(basin.taux, g, lb),
                    None if basin.tauy is None else _rows(basin.tauy, g, lb),
                    basin.dt, dict(basin.info, strip=len(out), strips=nranks))
        out.append(loc)
    return out


def gather_state(strips: List[Basin], glob: Basin, groups=("state",)) -> Basin:
    """Copy the strips' interior rows (and the outer halo rows of the first
    and last strip) of the given groups into a copy of the global Basin."""
    out = glob.copy()
    g = glob.bounds
    n = len(strips)
    for k, s in enumerate(strips):
        lb = s.bounds
        r0 = lb.bnd_y1 if k == 0 else lb.ny_start
        r1 = lb.bnd_y2 if k == n - 1 else lb.ny_end
        for grp in groups:
            for name, arr in getattr(s, grp).items():
                getattr(out, grp)[name][:, r0 - g.bnd_y1: r1 - g.bnd_y1 + 1] = \
                    arr[:, r0 - lb.bnd_y1: r1 - lb.bnd_y1 + 1]
    return out
