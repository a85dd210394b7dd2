"""Force-matching tables of CUBE's two-level PM.

The fine table wfxyzf.3.ascii holds the short-range force of the fine level on
a 16^3 grid of offsets, format (3i4,3e16.8), read as fk_table(i,j,k,1:3) with
the index check of kernel_f.f90:14-22.  The coarse table wfxyzc.2.ascii holds
the 4^3 corner correction of the coarse kernel, read as ck_table(1:3,i,j,k)
(kernel_c.f90:31-39).  Both files are the reference's data tables, shipped
unchanged in cube_nufluid_b200/data/.
"""
from __future__ import annotations

import os

import numpy as np

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def read_fine_table(path: str | None = None, nf_cutoff: int = 16) -> np.ndarray:
    """Returns fk_table as float32 [3][k][j][i] (C order; == Fortran fk_table(i,j,k,d))."""
    path = path or os.path.join(DATA_DIR, "wfxyzf.3.ascii")
    out = np.zeros((3, nf_cutoff, nf_cutoff, nf_cutoff), dtype=np.float32)
    with open(path) as f:
        for k in range(nf_cutoff):
            for j in range(nf_cutoff):
                for i in range(nf_cutoff):
                    parts = f.readline().split()
                    ii, jj, kk = int(parts[0]), int(parts[1]), int(parts[2])
                    if (ii, jj, kk) != (i + 1, j + 1, k + 1):
                        raise ValueError(f"fine kernel table out of order at {ii} {jj} {kk}")
                    for d in range(3):
                        out[d, k, j, i] = np.float32(float(parts[3 + d]))
    return out


def read_coarse_table(path: str | None = None) -> np.ndarray:
    """Returns ck_table as float32 [k][j][i][3] (C order; == Fortran ck_table(d,i,j,k))."""
    path = path or os.path.join(DATA_DIR, "wfxyzc.2.ascii")
    out = np.zeros((4, 4, 4, 3), dtype=np.float32)
    with open(path) as f:
        for k in range(4):
            for j in range(4):
                for i in range(4):
                    parts = f.readline().split()
                    for d in range(3):
                        out[k, j, i, d] = np.float32(float(parts[3 + d]))
    return out
