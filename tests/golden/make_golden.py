"""Golden regression fixtures for the barotropic step.

Each case is one small seeded basin: every input of barotropic_dynamics
(masks, metrics, Coriolis, rest depth, external depths, state, forcing)
and every output after `calls` calls of barotropic_dynamics(tau, nstep,
ksw4) on the CPU oracle (state, time means, depths).  The fixtures pin the
oracle against accidental change and give the CUDA paths a fixed target
that needs no oracle build.  No Fortran compiler exists in this image, so
they are produced by the oracle (a restatement of
Function/vel_ssh.f90:379-679), not by the reference itself.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from inmsom_elfs_b200 import basins                                   # noqa: E402
from inmsom_elfs_b200.grid import (DEPTHS, FORCING, MASKS, MEANS, METRICS,  # noqa: E402
                                   STATE, Basin, Bounds, Consts)

def _bump(b: Bounds, lu: np.ndarray, amp: float, m0: float, n0: float, sigma: float) -> np.ndarray:
    m = np.arange(b.bnd_x1, b.bnd_x2 + 1, dtype=np.float64)[:, None]
    n = np.arange(b.bnd_y1, b.bnd_y2 + 1, dtype=np.float64)[None, :]
    f = amp * np.exp(-((m - m0) ** 2 + (n - n0) ** 2) / (2.0 * sigma ** 2))
    return np.asfortranarray(np.where(lu > 0.5, f, 0.0))


def _channel(nx: int, ny: int, spacing: float = 5.0e3, depth: float = 1000.0,
             dt: float = 12.0, seed: int = 11) -> Basin:
    """Zonally periodic channel: land walls at the first and last interior
    rows, lu copied across the periodic halo as the reference's mask set-up
    does, random depth, zonal wind."""
    rng = np.random.default_rng(seed)
    b = Bounds.serial(nx, ny, periodicity_x=1)
    basin = Basin(b, Consts())
    lu = b.zeros(np.float32)
    lu[b.sl(b.nx_start, b.nx_end, b.ny_start + 1, b.ny_end - 1)] = 1.0
    lu[b.sl(b.mmm - 1, b.mmm - 1, b.bnd_y1, b.bnd_y2)] = lu[b.sl(b.mm, b.mm, b.bnd_y1, b.bnd_y2)]
    lu[b.sl(b.mm + 1, b.mm + 1, b.bnd_y1, b.bnd_y2)] = lu[b.sl(b.mmm, b.mmm, b.bnd_y1, b.bnd_y2)]
    basin.masks["lu"] = lu
    basins.uniform_metrics(basin, spacing)
    basin.rlh_s = np.full(b.shape, 1.0e-4, order="F")
    h = depth * (0.7 + 0.3 * rng.random(b.shape))
    basin.hhq_rest = np.asfortranarray(np.where(lu > 0.5, h, 0.0))
    basin.taux = np.full(b.shape, 0.1, order="F")
    basin.tauy = b.zeros()
    basin.forcing["mu"] = np.full(b.shape, 500.0, order="F")
    basin.forcing["rdis"] = np.full(b.shape, 1.0e-6, order="F")
    basin.dt = dt
    basin.info.update(workload="periodic_channel", nx=nx, ny=ny, seed=seed)
    return basin.fill_defaults()


def _regional_biharmonic(nx: int, ny: int) -> Basin:
    """Regional coastline with non-uniform viscosity, biharmonic viscosity,
    Rayleigh drag and a water flux: every forcing array is 2-D."""
    basin = basins.regional_basin(nx=nx, ny=ny, seed=5)
    b = basin.bounds
    rng = np.random.default_rng(6)
    basin.forcing["mu"] = np.asfortranarray(500.0 + 1000.0 * rng.random(b.shape))
    basin.forcing["mu4"] = np.full(b.shape, 2.0e7, order="F")
    basin.forcing["rdis"] = np.asfortranarray(1.0e-6 * (1.0 + rng.random(b.shape)))
    basin.forcing["wflux"] = np.asfortranarray(1.0e-2 * rng.standard_normal(b.shape))
    return basin


def _cases():
    """name -> (basin builder, ssh bump amplitude, tau in dt units, nstep, ksw4, calls)."""
    return {
        "beta_plane_28x24": (lambda: basins.beta_plane_basin(n=28, ny=24, nbumps=3, bump_sigma=3.0),
                             0.2, 3, 3, 0, 2),
        "spherical_rotated_24x20": (lambda: basins.spherical_basin(nx=24, ny=20, rotation_on_lat=30.0),
                                    0.1, 2, 2, 0, 2),
        "regional_biharmonic_32x28": (lambda: _regional_biharmonic(32, 28), 0.05, 4, 4, 1, 2),
        "periodic_channel_30x16": (lambda: _channel(30, 16), 0.1, 3, 3, 0, 2),
    }


CASE_NAMES = tuple(_cases())


def case_path(name: str) -> Path:
    return HERE / f"{name}.npz"


def load_case(name: str):
    """(basin with every input set, params dict, expected outputs dict
    keyed 'group.name')."""
    z = np.load(case_path(name))
    bt = [int(x) for x in z["bounds"]]
    b = Bounds(*bt)
    cf = z["consts"]
    basin = Basin(b, Consts(float(cf[0]), float(cf[1]), float(cf[2]), int(cf[3])))
    for key in z.files:
        if not key.startswith("in."):
            continue
        _, grp, name = key.split(".", 2)
        arr = np.asfortranarray(z[key])
        if grp == "grid":
            setattr(basin, name, arr)
        else:
            getattr(basin, grp)[name] = arr
    basin.fill_defaults()
    p = z["params"]
    params = dict(tau=float(p[0]), nstep=int(p[1]), ksw4=int(p[2]), calls=int(p[3]))
    expected = {k[4:]: z[k] for k in z.files if k.startswith("out.")}
    return basin, params, expected


def _save(name: str, basin: Basin, params: dict, out: Basin) -> None:
    b = basin.bounds
    arrays = {
        "bounds": np.array(b.astuple(), dtype=np.int64),
        "consts": np.array([basin.consts.time_smooth, basin.consts.free_fall_acc,
                            basin.consts.ref_den, basin.consts.full_free_surface]),
        "params": np.array([params["tau"], params["nstep"], params["ksw4"], params["calls"]]),
        "in.grid.rlh_s": basin.rlh_s,
        "in.grid.hhq_rest": basin.hhq_rest,
    }
    for grp, names in (("masks", MASKS), ("metrics", METRICS), ("depths", DEPTHS),
                       ("state", STATE), ("forcing", FORCING)):
        for k in names:
            arrays[f"in.{grp}.{k}"] = getattr(basin, grp)[k]
    for grp, names in (("state", STATE), ("means", MEANS), ("depths", DEPTHS)):
        for k in names:
            arrays[f"out.{grp}.{k}"] = getattr(out, grp)[k]
    np.savez_compressed(case_path(name), **arrays)


def make(names=None) -> None:
    from oracle import oracle as ora
    ora.load()
    for name, (builder, amp, tau_dt, nstep, ksw4, calls) in _cases().items():
        if names and name not in names:
            continue
        basin = builder()
        basins.finalize(basin, ora.OracleBackend())
        b, lu = basin.bounds, basin.masks["lu"]
        bump = _bump(b, lu, amp, b.nx_start + 0.4 * b.nx, b.ny_start + 0.55 * b.ny, 0.15 * b.nx)
        basin.state["ssh_e"] = bump.copy(order="F")
        basin.state["sshp_e"] = (0.98 * bump).copy(order="F")
        ora.hh_init_external(basin)
        params = dict(tau=tau_dt * basin.dt, nstep=nstep, ksw4=ksw4, calls=calls)
        assert basins.cfl_number(basin) < 1.0, name
        out = basin.copy()
        for _ in range(calls):
            ora.barotropic_dynamics(out, params["tau"], nstep, ksw4)
        _save(name, basin, params, out)
        size = case_path(name).stat().st_size
        print(f"{name}: {b.nx}x{b.ny}, tau={params['tau']}, nstep={nstep}, ksw4={ksw4}, "
              f"calls={calls}, {size} bytes")


if __name__ == "__main__":
    make(sys.argv[1:] or None)
