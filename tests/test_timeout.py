"""The bounded waits of the fused kernel, made to run out.

The reference has no wait to bound: its failure path stops the program
(Control/dyncall.f90:452-516).  Every mbarrier wait of the fused kernel
gives up after a bounded number of polls; the CTA then sets a status bit,
waits (bounded) for the copies it did issue and returns, and the call
returns INMSOM_ETIMEOUT.  The test hook inmsom_test_hold_copy makes one work
item withhold the copies of one of its input rows -- nothing else sets that
row's barrier, so the wait for it runs out -- with a short poll limit.  No
fault, trap or endless loop is involved, and the context computes the
oracle's result again once the hook is cleared.
"""
import numpy as np
import pytest

from conftest import rel_err
from inmsom_elfs_b200 import _lib, basins

pytestmark = pytest.mark.gpu

POLLS = 4096


def _basin(ora):
    b = basins.beta_plane_basin(n=300, ny=200, seed=14)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    return b


@pytest.mark.parametrize("item,ring_row", [(0, 0), (5, 4), (40, 100)])
def test_run_substeps_times_out_then_recovers(gpu, ora, item, ring_row):
    b = _basin(ora)
    bo, bg = b.copy(), b.copy()
    lib = _lib.load()
    with gpu.BarotropicSolver(bg, resident=True) as s:
        assert s.path()[0] == 1
        s.load_state()
        assert lib.inmsom_test_hold_copy(s._ctx, item, ring_row, POLLS) == _lib.OK
        for nsub in (1, 4):                     # a plain launch, then a replayed graph
            rc = lib.inmsom_run_substeps(s._ctx, nsub, b.dt, None, None)
            assert rc == _lib.ETIMEOUT, rc
            assert b"timed out" in lib.inmsom_gpu_last_error()
        assert lib.inmsom_test_hold_copy(s._ctx, -1, 0, 0) == _lib.OK
        s.load_state()                          # the host still holds the start state
        ora.run_substeps(bo, 10, b.dt)
        s.run_substeps(10, b.dt)
        s.sync_to_host()
    for k in ("ssh_e", "ubrtr_e", "vbrtr_e", "sshp_e", "ubrtrp_e", "vbrtrp_e"):
        assert rel_err(bg.state[k], bo.state[k]) <= 1e-12, k


def test_drop_in_call_times_out_then_recovers(gpu, ora):
    # the time-mean substeps of barotropic_dynamics(tau, nstep) run the
    # kernel's other variants
    b = _basin(ora)
    bo, bg = b.copy(), b.copy()
    lib = _lib.load()
    with gpu.BarotropicSolver(bg) as s:
        assert lib.inmsom_test_hold_copy(s._ctx, 7, 3, POLLS) == _lib.OK
        with pytest.raises(_lib.InmsomError, match="timed out"):
            s.barotropic_dynamics(3 * b.dt, 3)
        assert lib.inmsom_test_hold_copy(s._ctx, -1, 0, 0) == _lib.OK
        # the timed-out call left the resident state undefined; the host
        # arrays still hold the start state (the call copied nothing out)
        s.sync_from_host(_lib.SYNC_STATE)
        for _ in range(3):
            ora.barotropic_dynamics(bo, 3 * b.dt, 3)
            s.barotropic_dynamics(3 * b.dt, 3)
        s.sync_to_host()                        # the resident state to the host arrays
    for k in ("ssh_e", "ubrtr_e", "vbrtr_e"):
        assert rel_err(bg.state[k], bo.state[k]) <= 1e-12, k
    for k in ("ubrtr_i", "vbrtr_i"):
        assert rel_err(bg.means[k], bo.means[k]) <= 1e-12, k


def test_hold_hook_argument_checks():
    lib = _lib.load()
    assert lib.inmsom_test_hold_copy(None, 0, 0, 0) == _lib.EARG
