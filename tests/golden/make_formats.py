"""Golden regression fixture for the on-disk formats.

One seeded case of the checkpoint that ocpwrite writes
(Control/output.f90:1454-1847): the bytes of its 30 files (FP64 and FP32
field files of ten pairs, their GrADS descriptors), produced by the
restatement in oracle/dstd_oracle.py from seeded host arrays; and the
outputs of ctl_file_read on two of the descriptors.  The fixture pins the
restatement and the library against accidental change.  No Fortran
compiler exists in this image, so the bytes come from the restatement, not
from the reference itself.

    python tests/golden/make_formats.py       # rewrites tests/golden/formats_checkpoint.npz
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from inmsom_elfs_b200.grid import Bounds                              # noqa: E402
from oracle import dstd_oracle as od                                  # noqa: E402

NZ = 3
PATH = "cp"          # the descriptors name their data files without the path
AXES = dict(xt=[27.5], xu=[27.25], yt=[40.9], yv=[40.775], dxst=0.5, dyst=0.25, calendar=1,
            date=(2003, 2, 28, 18, 30), tstep=3600.0)


def case():
    """Bounds, masks, z, zw and the state of the fixture (seed 2024)."""
    rng = np.random.default_rng(2024)
    b = Bounds.serial(7, 5, periodicity_x=1)
    sh = b.shape
    st = {}
    for name in ("tt", "ttp", "ss", "ssp", "uu", "uup", "vv", "vvp"):
        st[name] = np.asfortranarray(rng.standard_normal(sh + (NZ,)))
    for name in ("q2", "q2p", "q2l", "q2lp"):
        st[name] = np.asfortranarray(rng.random(sh + (NZ + 1,)) * 1e-4)
    for name in ("ssh_i", "sshp_i", "ssh_e", "sshp_e", "ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e"):
        st[name] = np.asfortranarray(rng.standard_normal(sh))
    masks = {k: np.asfortranarray((rng.random(sh) > 0.3).astype(np.float32)) for k in ("lu", "llu", "llv")}
    z = np.array([0.05, 0.3, 0.75])
    zw = np.array([0.0, 0.1, 0.5, 1.0])
    return b, masks, z, zw, st


def main():
    b, masks, z, zw, st = case()
    files = od.ocpwrite_files(PATH, b, NZ, masks, z, zw, AXES, st)
    out = {}
    for name, content in files.items():
        out["file:" + name] = np.frombuffer(content.encode() if isinstance(content, str) else content, np.uint8)
    for ctl in ("cptt.ctl", "cpube.ctl"):
        r = od.ctl_read(files[ctl])
        for k, v in r.items():
            out[f"read:{ctl}:{k}"] = np.asarray(v if not isinstance(v, list) or not v or not isinstance(v[0], str)
                                                else "\n".join(v))
    np.savez_compressed(HERE / "formats_checkpoint.npz", **out)
    print(f"{len(files)} files, {sum(len(v) for k, v in out.items() if k.startswith('file:'))} bytes")


if __name__ == "__main__":
    main()
