"""Writes na196_profile.npz, the Na196 Thomas-Fermi profile the reference's
collision runs sample from (ref/fortran/data/hm1.dat: 1001 radius quantiles;
rhoinit.dat: rmax then 1001 densities on [0, rmax]; read as
src/initial.jl:143-158 does).  Run once where the reference is checked out,
with the reference's ref/fortran/data directory as the argument:

    python vlasov.jl_b200/data/make_profile.py <reference>/ref/fortran/data
"""
import sys
from pathlib import Path

import numpy as np


def read(dirpath: Path):
    with open(dirpath / "hm1.dat") as f:
        n = int(f.readline())
        q = np.array([float(f.readline()) for _ in range(n)])
    with open(dirpath / "rhoinit.dat") as f:
        n = int(f.readline())
        rmax = float(f.readline())
        rho = np.array([float(f.readline()) for _ in range(n)])
    return q, rho, rmax


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_profile.py <reference>/ref/fortran/data")
    src = Path(sys.argv[1])
    q, rho, rmax = read(src)
    out = Path(__file__).resolve().parent / "na196_profile.npz"
    np.savez(out, quantiles=q, density=rho, rmax=rmax)
    print(f"wrote {out}: {len(q)} quantiles (max {q.max():.3f}), {len(rho)} densities, rmax {rmax}")
