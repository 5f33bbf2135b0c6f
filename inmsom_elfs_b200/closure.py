"""Learned subgrid momentum closure for coarse grids: training data from
coarse-grained fine runs of the same GPU solver, training with the
library's MLP kernels, and the a-posteriori comparison with the plain
Laplacian viscosity.

The reference has no counterpart; its coarse-grid answer is the Laplacian
lateral viscosity of uv_diff2 (Function/vel_ssh.f90:117-184), which the
plain coarse run keeps.

Workload: a double-gyre basin with a meandering meridional ridge on an
r-times finer grid (the truth) and on the coarse grid.  The land mask of the
fine grid is the coarse one refined, so every coarse cell is r x r fine
cells.  Coarse graining (``coarsen``): SSH is the block mean; u on a coarse
east face is the mean of the r fine u on that face, v likewise on the north
face, so the coarse fluxes are the fine ones.

Training pair for a time t of the fine run (coarse step D = r * fine step):
the coarse state (levels t and t - D) coarse-grained from the fine run, the
network's 45 features of it, and the velocity tendency the coarse step
misses, a = (CG(fine at t + D) - coarse step) / (2 D) on ocean u and v
points (the coarse step is a leap-frog step over 2 D).  The closure run
adds y * out_scale as a momentum tendency, re-evaluated every `every`
coarse steps (inmsom_run_closure).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import time
from dataclasses import dataclass
from typing import Callable, Dict, Optional

import numpy as np

from . import _lib
from .basins import _y_of_rows, finalize, uniform_metrics
from .grid import Basin, Bounds, Consts


@dataclass
class ClosureConfig:
    n_coarse: int = 512            # coarse interior points per side
    factor: int = 4                # fine points per coarse point and side
    spacing_fine: float = 2.0e3    # m
    depth: float = 4000.0          # m
    ridge_rms: float = 300.0       # m, over the basin
    tau0: float = 0.1              # N/m^2
    f0: float = 1.0e-4
    beta: float = 2.0e-11
    drag: float = 1.0e-6           # 1/s
    visc_fine: float = 50.0        # m^2/s, the truth
    visc_plain: float = 1000.0     # m^2/s, the plain coarse run
    visc_base: float = 0.0         # m^2/s, kept by the closure run
    dt_fine: float = 3.0           # s
    seed: int = 2

    @property
    def dt_coarse(self) -> float:
        return self.dt_fine * self.factor


def _ridge_depth(cfg: ClosureConfig, x: np.ndarray, y: np.ndarray, L: float) -> np.ndarray:
    """Rest depth at (x, y) (m from the south-west corner): cfg.depth minus a
    meridional ridge whose axis and crest height meander with y."""
    rng = np.random.default_rng(cfg.seed)
    k = rng.integers(1, 4, size=3)
    ph = rng.uniform(0, 2 * math.pi, size=6)
    s = y / L
    axis = L * (0.5 + 0.04 * sum(np.sin(2 * math.pi * k[i] * s + ph[i]) for i in range(3)))
    crest = 1.0 + 0.3 * np.sin(2 * math.pi * 2 * s + ph[3]) + 0.15 * np.sin(2 * math.pi * 5 * s + ph[4])
    w = L / 40.0
    return crest * np.exp(-0.5 * ((x - axis) / w) ** 2)


def closure_basins(cfg: ClosureConfig, backend, which=("fine", "plain", "base")) -> Dict[str, Basin]:
    """The fine basin and the coarse basins (plain viscosity and the
    closure run's base viscosity), derived masks and wind forcing by
    `backend` (finalize); `which` selects the ones built."""
    r, nc = cfg.factor, cfg.n_coarse
    nf = nc * r
    dxf, dxc = cfg.spacing_fine, cfg.spacing_fine * r
    L = nf * dxf
    cb, fb = Bounds.serial(nc, nc), Bounds.serial(nf, nf)
    lu_c = cb.zeros(np.float32)
    lu_c[cb.sl(cb.nx_start + 1, cb.nx_end - 1, cb.ny_start + 1, cb.ny_end - 1)] = 1.0
    lu_f = fb.zeros(np.float32)
    lu_f[fb.interior] = np.kron(lu_c[cb.interior], np.ones((r, r), np.float32))
    # ridge on the fine T points, coarse depth = block mean (the blocks are
    # all ocean or all land)
    xf = (np.arange(nf) + 0.5) * dxf
    ridge = _ridge_depth(cfg, xf[:, None], xf[None, :], L)
    ocean_f = lu_f[fb.interior] > 0.5
    ridge *= cfg.ridge_rms / math.sqrt(float(np.mean(ridge[ocean_f] ** 2)))
    hf = np.where(ocean_f, cfg.depth - ridge, 0.0)
    hc = hf.reshape(nc, r, nc, r).mean(axis=(1, 3))
    out = {}
    for name, b, dx, lu, h, visc, dt in (("fine", fb, dxf, lu_f, hf, cfg.visc_fine, cfg.dt_fine),
                                          ("plain", cb, dxc, lu_c, hc, cfg.visc_plain, cfg.dt_coarse),
                                          ("base", cb, dxc, lu_c, hc, cfg.visc_base, cfg.dt_coarse)):
        if name not in which:
            continue
        basin = Basin(b, Consts())
        basin.masks["lu"] = lu.copy(order="F")
        uniform_metrics(basin, dx)
        yh = _y_of_rows(b, dx, 0.5)
        basin.rlh_s = np.asfortranarray(np.broadcast_to(cfg.f0 + cfg.beta * yh[None, :], b.shape).copy())
        hr = b.zeros()
        hr[b.interior] = h
        basin.hhq_rest = hr
        yt = _y_of_rows(b, dx, 0.0)
        basin.taux = np.asfortranarray(np.broadcast_to(cfg.tau0 * np.cos(math.pi * yt / L)[None, :],
                                                       b.shape).copy())
        basin.tauy = b.zeros()
        basin.forcing["mu"] = np.full(b.shape, visc, order="F")
        basin.forcing["rdis"] = np.full(b.shape, cfg.drag, order="F")
        basin.dt = dt
        basin.info.update(workload=f"closure_{name}", n=b.nx, spacing=dx, visc=visc)
        basin.fill_defaults()
        out[name] = finalize(basin, backend)
    return out


def coarsen(fb: Bounds, cb: Bounds, r: int, u: np.ndarray, v: np.ndarray, ssh: np.ndarray):
    """Coarse (u, v, ssh) arrays (zero outside the interior) of fine ones."""
    nc = cb.nx
    fi = fb.interior
    U, V, S = u[fi], v[fi], ssh[fi]
    out = []
    for a in (U[r - 1::r, :].reshape(nc, nc, r).mean(axis=2),
              V[:, r - 1::r].reshape(nc, r, nc).mean(axis=1),
              S.reshape(nc, r, nc, r).mean(axis=(1, 3))):
        z = cb.zeros()
        z[cb.interior] = a
        out.append(z)
    return out


def kinetic_energy(b: Bounds, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """0.5 |u|^2 on the T points of the interior (face values averaged)."""
    i0, i1, j0, j1 = b.nx_start - b.bnd_x1, b.nx_end - b.bnd_x1 + 1, b.ny_start - b.bnd_y1, b.ny_end - b.bnd_y1 + 1
    uu = 0.5 * (u[i0:i1, j0:j1] ** 2 + u[i0 - 1:i1 - 1, j0:j1] ** 2)
    vv = 0.5 * (v[i0:i1, j0:j1] ** 2 + v[i0:i1, j0 - 1:j1 - 1] ** 2)
    return 0.5 * (uu + vv)


def cell_order(a: np.ndarray, b: Bounds) -> np.ndarray:
    """Interior values in the feature row order (n - ny_start) * nx + (m - nx_start)."""
    return np.ascontiguousarray(a[b.interior].T).ravel()


def make_norm(basin: Basin, u: np.ndarray, v: np.ndarray, ssh: np.ndarray, out_scale) -> _lib.CClosureNorm:
    """Feature normalisation from the ocean points of a state."""
    b = basin.bounds
    ocean = basin.masks["lu"][b.interior] > 0.5
    norm = _lib.CClosureNorm()
    for k, f in enumerate((u, v, ssh, basin.hhq_rest, basin.rlh_s)):
        x = f[b.interior][ocean]
        sd = float(x.std())
        norm.mean[k] = float(x.mean())
        norm.inv_std[k] = 1.0 / sd if sd > 0 else 1.0
    norm.out_scale[0], norm.out_scale[1] = float(out_scale[0]), float(out_scale[1])
    return norm


def _set_state(basin: Basin, cur, prev) -> None:
    st = basin.state
    st["ubrtr_e"][...], st["vbrtr_e"][...], st["ssh_e"][...] = cur
    st["ubrtrp_e"][...], st["vbrtrp_e"][...], st["sshp_e"][...] = prev


def _rmse(a: np.ndarray, b: np.ndarray, mask: np.ndarray) -> float:
    return float(np.sqrt(np.mean((a[mask] - b[mask]) ** 2)))


class ClosureStudy:
    """Truth run, training set, training and evaluation on one GPU."""

    def __init__(self, cfg: ClosureConfig, device: int = 0, log: Callable[[str], None] = print):
        import torch
        from .solver import BarotropicSolver, GpuBackend
        self.torch = torch
        self.cfg = cfg
        self.log = log
        self.dev = torch.device("cuda", device)
        self.basins = closure_basins(cfg, GpuBackend(device))
        self.fine = BarotropicSolver(self.basins["fine"], device)
        self.fine.load_state()
        self.base = BarotropicSolver(self.basins["base"], device)
        self.t_fine = 0          # fine substeps run
        self.norm: Optional[_lib.CClosureNorm] = None
        self.net = None
        self.x = self.t = None

    # ---------------------------------------------------------------- truth
    def advance_fine(self, nsub: int) -> None:
        while nsub > 0:
            k = min(nsub, 100_000)
            self.fine.run_substeps(k, self.cfg.dt_fine)
            nsub -= k
            self.t_fine += k

    def fine_coarse_state(self):
        """Coarse (u, v, ssh) of the fine run's current level."""
        self.fine.sync_to_host()
        fb, cb = self.basins["fine"].bounds, self.basins["base"].bounds
        st = self.basins["fine"].state
        return coarsen(fb, cb, self.cfg.factor, st["ubrtr_e"], st["vbrtr_e"], st["ssh_e"])

    def triplet(self, gap: int):
        """Coarse states at t - D, t, t + D, the fine run ending at t + D
        after `gap` fine substeps before t - D."""
        r = self.cfg.factor
        self.advance_fine(gap)
        s0 = self.fine_coarse_state()
        self.advance_fine(r)
        s1 = self.fine_coarse_state()
        self.advance_fine(r)
        s2 = self.fine_coarse_state()
        return s0, s1, s2

    def spinup(self, days: float) -> None:
        n = int(round(days * 86400.0 / self.cfg.dt_fine)) // 100 * 100
        t0 = time.time()
        self.advance_fine(n)
        vol, en = self.fine.diag()
        self.log(f"closure: spin-up {days:g} days ({n} fine substeps) in {time.time() - t0:.1f} s, "
                 f"energy {en:.4e}")

    # ------------------------------------------------------------- training
    def collect(self, snapshots: int, gap: int) -> Dict[str, float]:
        """Training set of `snapshots` coarse states `gap` fine substeps
        apart: features on the device, normalised targets."""
        torch = self.torch
        cfg, cb = self.cfg, self.basins["base"].bounds
        bb = self.basins["base"]
        ncell = cb.nx * cb.ny
        lcu = bb.masks["lcu"] > 0.5
        lcv = bb.masks["lcv"] > 0.5
        self.x = torch.empty((snapshots * ncell, 48), dtype=torch.bfloat16, device=self.dev)
        tgt = np.zeros((snapshots, ncell, 2), np.float32)
        D = cfg.dt_coarse
        t0 = time.time()
        for s in range(snapshots):
            s0, s1, s2 = self.triplet(gap if s else 0)
            if self.norm is None:
                self.norm = make_norm(bb, *s1, out_scale=(1.0, 1.0))
            _set_state(bb, s1, s0)
            self.base.load_state()
            self.base.closure_features(self.norm, self.x[s * ncell:(s + 1) * ncell].data_ptr())
            self.base.run_substeps(1, D)
            self.base.sync_to_host()
            au = np.where(lcu, (s2[0] - bb.state["ubrtr_e"]) / (2 * D), 0.0)
            av = np.where(lcv, (s2[1] - bb.state["vbrtr_e"]) / (2 * D), 0.0)
            tgt[s, :, 0] = cell_order(au, cb)
            tgt[s, :, 1] = cell_order(av, cb)
        valid = np.concatenate([cell_order(lcu.astype(np.float32), cb), cell_order(lcv.astype(np.float32), cb)])
        su = float(np.sqrt(np.sum(tgt[:, :, 0] ** 2) / max(1.0, snapshots * valid[:ncell].sum())))
        sv = float(np.sqrt(np.sum(tgt[:, :, 1] ** 2) / max(1.0, snapshots * valid[ncell:].sum())))
        self.norm.out_scale[0], self.norm.out_scale[1] = su, sv
        tgt[:, :, 0] /= su
        tgt[:, :, 1] /= sv
        self.t = torch.from_numpy(tgt.reshape(-1, 2)).to(self.dev)
        self.log(f"closure: {snapshots} training states in {time.time() - t0:.1f} s, "
                 f"tendency rms u {su:.3e} v {sv:.3e} m/s^2")
        return {"snapshots": snapshots, "gap_fine_substeps": gap, "rms_tendency_u": su, "rms_tendency_v": sv}

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0,
              holdout: float = 0.1) -> Dict[str, float]:
        """Adam on random batches of the first (1 - holdout) of the states;
        returns the training and held-out losses (MSE of normalised
        targets: 1 - R^2 when the network is useless)."""
        from .mlp import MLP
        torch = self.torch
        n = self.x.shape[0]
        ncell = self.basins["base"].bounds.nx * self.basins["base"].bounds.ny
        ntrain = int(round((1.0 - holdout) * n / ncell)) * ncell
        self.net = MLP(seed=seed, device=self.dev.index or 0)
        xt, tt = self.x[:ntrain], self.t[:ntrain]
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        losses = self.net.train(xt, tt, steps, batch=batch, lr=lr, seed=seed + 1, log_every=max(1, steps // 10))
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        res = {"train_steps": steps, "batch": batch, "lr": lr, "train_ms": ms,
               "train_loss": losses[-1][1] if losses else float("nan")}
        m = (n - ntrain) // 128 * 128
        if m > 0:
            res["heldout_loss"] = float(self.net.loss_grad(self.x[ntrain:ntrain + m], self.t[ntrain:ntrain + m])[-1].item())
        self.log(f"closure: trained {steps} steps x {batch} in {ms / 1e3:.1f} s: " +
                 ", ".join(f"{k} {v:.4f}" for k, v in res.items() if k.endswith("loss")))
        return res

    # ----------------------------------------------------------- evaluation
    def evaluate(self, gap: int, steps: int, records: int, every: int,
                 extra_plain: Optional[Dict[str, float]] = None) -> Dict[str, object]:
        """From the coarse-grained fine state `gap` fine substeps on, run
        the plain coarse model, the base model without and with the closure
        for `steps` coarse steps; SSH and KE RMSE against the coarse-grained
        truth at `records` times, and the device time of each run."""
        from .solver import BarotropicSolver
        cfg = self.cfg
        cb = self.basins["base"].bounds
        r = cfg.factor
        s0 = self.triplet(gap)[0:2]
        runs = {"plain": self.basins["plain"], "base": self.basins["base"]}
        for name, visc in (extra_plain or {}).items():
            b = self.basins["plain"].copy()
            b.forcing["mu"][...] = visc
            runs[name] = b
        sol = {}
        for name, b in runs.items():
            _set_state(b, s0[1], s0[0])
            sol[name] = BarotropicSolver(b, self.fine.device) if name != "base" else self.base
            sol[name].load_state()
        cl = self.basins["base"].copy()
        _set_state(cl, s0[1], s0[0])
        sol["closure"] = BarotropicSolver(cl, self.fine.device)
        sol["closure"].load_state()
        bas = dict(runs, closure=cl)
        ocean = self.basins["base"].masks["lu"][cb.interior] > 0.5
        per = steps // records
        per -= per % every
        ssh_err = {k: [] for k in sol}
        ke_err = {k: [] for k in sol}
        ms = {k: 0.0 for k in sol}
        alive = {k: True for k in sol}
        truth_ssh_rms = []
        for rec in range(records):
            self.advance_fine(r * per)
            tu, tv, ts = self.fine_coarse_state()
            tke = kinetic_energy(cb, tu, tv)
            truth_ssh_rms.append(float(np.sqrt(np.mean(ts[cb.interior][ocean] ** 2))))
            for k, s in sol.items():
                if not alive[k]:
                    continue
                try:
                    if k == "closure":
                        ms[k] += s.run_closure(per, cfg.dt_coarse, every, self.net.params.data_ptr(),
                                               self.net.wbf16.data_ptr(), self.norm)
                    else:
                        ms[k] += s.run_substeps(per, cfg.dt_coarse)
                    s.sync_to_host()
                except _lib.InmsomError as e:
                    self.log(f"closure: run {k} stopped at record {rec}: {e}")
                    alive[k] = False
                    continue
                st = bas[k].state
                if not np.all(np.isfinite(st["ssh_e"])):
                    alive[k] = False
                    continue
                ssh_err[k].append(_rmse(st["ssh_e"][cb.interior], ts[cb.interior], ocean))
                ke_err[k].append(_rmse(kinetic_energy(cb, st["ubrtr_e"], st["vbrtr_e"]), tke, ocean))
        for k, s in sol.items():
            if s is not self.base:
                s.close()
        out = {"steps": per * records, "records": records, "every": every,
               "truth_ssh_rms_m": float(np.mean(truth_ssh_rms))}
        for k in sol:
            ok = alive[k] and len(ssh_err[k]) == records
            out[k] = {"stable": ok,
                      "ssh_rmse_m": float(np.mean(ssh_err[k])) if ok else None,
                      "ke_rmse": float(np.mean(ke_err[k])) if ok else None,
                      "ssh_rmse_final_m": ssh_err[k][-1] if ok else None,
                      "ms": ms[k]}
        if out["plain"]["stable"] and out["closure"]["stable"]:
            out["ssh_rmse_reduction"] = 1.0 - out["closure"]["ssh_rmse_m"] / out["plain"]["ssh_rmse_m"]
            out["ke_rmse_reduction"] = 1.0 - out["closure"]["ke_rmse"] / out["plain"]["ke_rmse"]
            out["time_ratio"] = out["closure"]["ms"] / out["plain"]["ms"]
        self.log("closure: evaluation " + ", ".join(
            f"{k}: ssh {v['ssh_rmse_m']} ke {v['ke_rmse']} ms {v['ms']:.1f}" for k, v in out.items()
            if isinstance(v, dict)))
        return out

    def close(self) -> None:
        self.fine.close()
        self.base.close()


def run_study(cfg: ClosureConfig, spinup_days: float, snapshots: int, gap: int, train_steps: int,
              eval_gap: int, eval_steps: int, records: int, every: int, batch: int = 65536,
              lr: float = 1e-3, extra_plain: Optional[Dict[str, float]] = None,
              log: Callable[[str], None] = print) -> Dict[str, object]:
    st = ClosureStudy(cfg, log=log)
    try:
        st.spinup(spinup_days)
        res = {"config": dataclasses.asdict(cfg), "spinup_days": spinup_days}
        res["data"] = st.collect(snapshots, gap)
        res["train"] = st.train(train_steps, batch=batch, lr=lr)
        res["eval"] = st.evaluate(eval_gap, eval_steps, records, every, extra_plain)
        return res
    finally:
        st.close()
