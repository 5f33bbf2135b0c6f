"""Domain bounds, constants and the basin container (Fortran layout).

Every 2-D field is a numpy array in Fortran order with shape
(bnd_x2-bnd_x1+1, bnd_y2-bnd_y1+1): element [m-bnd_x1, n-bnd_y1] is the
reference's f(m, n).  Masks are float32 0/1 (the reference's real(4)
masks), everything else float64.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

MASKS = ("lu", "luu", "luh", "lcu", "lcv", "llu", "llv")
METRICS = ("dx", "dy", "dxt", "dyt", "dxh", "dyh", "dxb", "dyb")
DEPTHS = ("hhq_e", "hhqp_e", "hhqn_e", "hhu_e", "hhup_e", "hhun_e",
          "hhv_e", "hhvp_e", "hhvn_e", "hhh_e", "hhhp_e", "hhhn_e")
STATE = ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e", "ssh_e", "sshp_e")
MEANS = ("ubrtr_i", "vbrtr_i", "ssh4gradx", "ssh4grady")
FORCING = ("RHSx", "RHSy", "wflux", "mu", "mu4", "rdis")
SCRATCH = ("vort", "str_t2d", "str_s2d", "fx", "fy",
           "RHSx_adv", "RHSy_adv", "RHSx_dif", "RHSy_dif")


@dataclass(frozen=True)
class Bounds:
    """Local domain bounds (Modules/mod_mpi_parallel_tools.f90:7-15) plus the
    global significant area and periodicity (Inc/basinpar.fi:4-14)."""

    nx_start: int
    nx_end: int
    ny_start: int
    ny_end: int
    bnd_x1: int
    bnd_x2: int
    bnd_y1: int
    bnd_y2: int
    mmm: int
    mm: int
    nnn: int
    nn: int
    periodicity_x: int = 0
    periodicity_y: int = 0

    @classmethod
    def serial(cls, nx_sig: int, ny_sig: int, periodicity_x: int = 0,
               periodicity_y: int = 0) -> "Bounds":
        """One domain of nx_sig x ny_sig significant points, as
        non_mpi_array_boundary_definition (Control/init_arrays.f90:2-17) sets
        it with mmm = nnn = 3: interior 3..nx_sig+2, arrays 1..nx_sig+4."""
        if nx_sig < 1 or ny_sig < 1:
            raise ValueError("empty basin")
        mmm, nnn = 3, 3
        mm, nn = mmm + nx_sig - 1, nnn + ny_sig - 1
        return cls(mmm, mm, nnn, nn, mmm - 2, mm + 2, nnn - 2, nn + 2,
                   mmm, mm, nnn, nn, periodicity_x, periodicity_y)

    @property
    def shape(self):
        return (self.bnd_x2 - self.bnd_x1 + 1, self.bnd_y2 - self.bnd_y1 + 1)

    @property
    def nx(self) -> int:
        return self.nx_end - self.nx_start + 1

    @property
    def ny(self) -> int:
        return self.ny_end - self.ny_start + 1

    def zeros(self, dtype=np.float64) -> np.ndarray:
        return np.zeros(self.shape, dtype=dtype, order="F")

    def sl(self, m0: int, m1: int, n0: int, n1: int):
        """numpy index of the inclusive Fortran range (m0:m1, n0:n1)."""
        return (slice(m0 - self.bnd_x1, m1 - self.bnd_x1 + 1),
                slice(n0 - self.bnd_y1, n1 - self.bnd_y1 + 1))

    @property
    def interior(self):
        return self.sl(self.nx_start, self.nx_end, self.ny_start, self.ny_end)

    def astuple(self):
        return dataclasses.astuple(self)


@dataclass(frozen=True)
class Consts:
    """Compile-time constants of Inc/basinpar.fi:3,46,76-77."""

    time_smooth: float = 0.05
    free_fall_acc: float = 9.8
    ref_den: float = 1025.0
    full_free_surface: int = 1


@dataclass
class Basin:
    """Everything the barotropic step reads: masks, metrics, Coriolis,
    rest depth, forcing, the external-mode state and its depth arrays."""

    bounds: Bounds
    consts: Consts = field(default_factory=Consts)
    masks: Dict[str, np.ndarray] = field(default_factory=dict)
    metrics: Dict[str, np.ndarray] = field(default_factory=dict)
    rlh_s: Optional[np.ndarray] = None
    hhq_rest: Optional[np.ndarray] = None
    depths: Dict[str, np.ndarray] = field(default_factory=dict)
    state: Dict[str, np.ndarray] = field(default_factory=dict)
    means: Dict[str, np.ndarray] = field(default_factory=dict)
    forcing: Dict[str, np.ndarray] = field(default_factory=dict)
    scratch: Dict[str, np.ndarray] = field(default_factory=dict)
    taux: Optional[np.ndarray] = None
    tauy: Optional[np.ndarray] = None
    dt: float = 0.0
    info: Dict[str, object] = field(default_factory=dict)

    def fill_defaults(self) -> "Basin":
        """Zero-initialise every array that is not set yet, as
        model_grid_allocate / ocean_variables_allocate do
        (Control/init_arrays.f90:154-171, :356-410)."""
        b = self.bounds
        for k in MASKS:
            self.masks.setdefault(k, b.zeros(np.float32))
        for k in METRICS:
            self.metrics.setdefault(k, b.zeros())
        if self.rlh_s is None:
            self.rlh_s = b.zeros()
        if self.hhq_rest is None:
            self.hhq_rest = b.zeros()
        for group, names in ((self.depths, DEPTHS), (self.state, STATE),
                             (self.means, MEANS), (self.forcing, FORCING),
                             (self.scratch, SCRATCH)):
            for k in names:
                group.setdefault(k, b.zeros())
        return self

    def copy(self) -> "Basin":
        def cp(d):
            return {k: v.copy(order="F") for k, v in d.items()}
        return Basin(self.bounds, self.consts, cp(self.masks), cp(self.metrics),
                     None if self.rlh_s is None else self.rlh_s.copy(order="F"),
                     None if self.hhq_rest is None else self.hhq_rest.copy(order="F"),
                     cp(self.depths), cp(self.state), cp(self.means), cp(self.forcing),
                     cp(self.scratch),
                     None if self.taux is None else self.taux.copy(order="F"),
                     None if self.tauy is None else self.tauy.copy(order="F"),
                     self.dt, dict(self.info))

    @property
    def cells(self) -> int:
        return self.bounds.nx * self.bounds.ny
