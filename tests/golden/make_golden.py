"""Regenerate the golden fixtures in this directory from the reference's own
data files.  Run in a checkout that has the reference project at
``$ADGA_REFERENCE`` (default /root/reference); the fixtures are committed, so
the tests never need the reference at run time.

* umatrix_example.npz   -- documentation/examples/umatrix (Kanamori U=5,
                           V=3.5, J=0.75, 3 bands) parsed as U_ijkl; the
                           golden vector for create_u.
* srvo3_hk_digest.npz   -- shape, k-point sample and checksums of
                           srvo3-testdata/srvo3_k20.hk read with an
                           independent numpy parser; pins the .hk reader.
"""
import os
import sys
from pathlib import Path

import numpy as np

REF = Path(os.environ.get("ADGA_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent


def umatrix():
    rows = np.loadtxt(REF / "documentation/examples/umatrix", skiprows=1)
    nd = int(round(len(rows) ** 0.25))
    U = np.zeros((nd,) * 4)
    for i, j, k, l, v in rows:
        U[int(i) - 1, int(j) - 1, int(k) - 1, int(l) - 1] = v
    np.savez(OUT / "umatrix_example.npz", Umat=U, U=5.0, V=3.5, J=0.75)


def hk_digest():
    path = REF / "srvo3-testdata/srvo3_k20.hk"
    with open(path) as fh:
        head = fh.readline().split()
        nkp, nd = int(head[0]), int(head[1])
        data = np.array(fh.read().split(), dtype=float)
    per = 3 + nd * 2 * nd
    data = data.reshape(nkp, per)
    kd = data[:, :3]
    h = data[:, 3:].reshape(nkp, nd, nd, 2)
    hk = h[..., 0] + 1j * h[..., 1]            # [k, i, j]
    pick = np.array([0, 1, 19, 400, 4321, nkp - 1])
    np.savez(OUT / "srvo3_hk_digest.npz", nkp=nkp, ndim=nd, kpick=pick, k_data=kd[pick],
             hk_pick=hk[pick], hk_sum=hk.sum(), hk_abs_sum=np.abs(hk).sum(),
             trace_mean=np.trace(hk, axis1=1, axis2=2).mean())


if __name__ == "__main__":
    if not REF.exists():
        sys.exit(f"reference not found at {REF}")
    umatrix()
    hk_digest()
    print("fixtures written to", OUT)
