"""Row-strip decomposition of one basin over several domains (ranks).

The reference decomposes its basin over a 2-D MPI process grid in
mpi_array_boundary_definition (Control/init_arrays.f90:21-88) and exchanges
one halo row or column per field update with syncborder_real8
(Modules/mod_mpi_parallel_tools.f90:179-252).  The B200 path uses a 1 x P
grid of row strips (one strip per GPU): strip_bounds() applies the
reference's formula for p_size = (1, P), split_basin() cuts a global Basin
into the strips' local arrays (each with its halo rows from the global
arrays: two, or 2k where a strip advances k substeps per exchange) and
gather_state() reassembles the state from the strips.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Dict, List

import numpy as np

from .grid import Basin, Bounds


def strip_bounds(b: Bounds, nranks: int, halo: int = 2) -> List[Bounds]:
    """Local bounds of the strips of a 1 x nranks process grid, south to
    north: Control/init_arrays.f90:59-70 with p_size(2) = nranks (locn rows
    each, the last strip takes the rest); x is not split.  `halo` rows (an
    even number >= 2; the reference's 2, or 2k for a strip that advances k
    substeps per exchange) on the sides shared with another strip, 2 on
    the basin's edges."""
    if nranks < 1:
        raise ValueError("nranks < 1")
    if halo < 2 or halo % 2:
        raise ValueError("halo must be an even number >= 2")
    ny = b.bnd_y2 - b.bnd_y1 + 1                 # global array rows
    locn = (ny - 4) // nranks
    if locn < 1:
        raise ValueError(f"{ny - 4} interior rows cannot be split over {nranks} strips")
    if nranks > 1 and halo > locn:
        raise ValueError(f"a halo of {halo} rows exceeds the strips' {locn} rows")
    out = []
    for k in range(nranks):
        ny_start = locn * k + b.bnd_y1 + 2
        ny_end = ny_start + locn - 1 if k < nranks - 1 else b.bnd_y2 - 2
        hs = halo if k > 0 else 2
        hn = halo if k < nranks - 1 else 2
        out.append(replace(b, ny_start=ny_start, ny_end=ny_end, bnd_y1=ny_start - hs, bnd_y2=ny_end + hn))
    return out


def _rows(a: np.ndarray, g: Bounds, lb: Bounds) -> np.ndarray:
    return np.asfortranarray(a[:, lb.bnd_y1 - g.bnd_y1: lb.bnd_y2 - g.bnd_y1 + 1].copy(order="F"))


def split_basin(basin: Basin, nranks: int, halo: int = 2) -> List[Basin]:
    """Local Basins of the strips: every array restricted to the strip's
    rows bnd_y1..bnd_y2 (interior and halo rows, taken from the global
    arrays; see strip_bounds for the halo widths)."""
    g = basin.bounds
    out = []
    for lb in strip_bounds(g, nranks, halo):
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


def stacked_strip(parts: Dict[int, Basin], nstack: int, rank: int, halo: int = 2) -> Basin:
    """Strip `rank` of a basin made of `nstack` basins of equal size stacked
    along y (basin q's interior rows follow basin q-1's): the local Basin of
    strip_bounds(global, nstack, halo)[rank], whose interior is basin
    `rank`'s interior, with its halo rows taken from the neighbouring basins'
    interior rows (or from basin `rank`'s own halo rows at the stack's
    edges).  `parts` holds basins rank-1, rank and rank+1 (those that
    exist), each finalized on its own: every row of the stack carries the
    values of the one basin that owns it, so neighbouring strips hold the
    same values in the rows they share.  The state is basin `rank`'s (and
    its neighbours' in the halo rows)."""
    own = parts[rank]
    b = own.bounds
    ny = b.ny
    glob = replace(b, ny_end=b.ny_start + nstack * ny - 1, bnd_y2=b.ny_start + nstack * ny + 1,
                   nn=b.nnn + nstack * ny - 1)
    lb = strip_bounds(glob, nstack, halo)[rank]
    rows = np.arange(lb.bnd_y1, lb.bnd_y2 + 1)
    # global row n -> (basin, that basin's row): the interior rows of basin
    # q are nnn + q*ny .. nnn + (q+1)*ny - 1; rows below the stack's first
    # interior row belong to basin 0, rows above its last to basin nstack-1
    q = np.clip((rows - glob.ny_start) // ny, 0, nstack - 1)
    src = rows - q * ny

    def take(get):
        out = np.zeros((b.shape[0], len(rows)), dtype=get(own).dtype, order="F")
        for i, (qq, r) in enumerate(zip(q, src)):
            out[:, i] = get(parts[int(qq)])[:, r - b.bnd_y1]
        return out

    def group(name):
        return {k: take(lambda p, k=k: getattr(p, name)[k]) for k in getattr(own, name)}

    loc = Basin(lb, own.consts, group("masks"), group("metrics"), take(lambda p: p.rlh_s),
                take(lambda p: p.hhq_rest), group("depths"), group("state"), group("means"),
                group("forcing"), group("scratch"),
                None if own.taux is None else take(lambda p: p.taux),
                None if own.tauy is None else take(lambda p: p.tauy),
                own.dt, dict(own.info, strip=rank, strips=nstack, stacked=True))
    return loc
