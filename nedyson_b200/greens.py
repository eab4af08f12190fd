"""Host-side contour Green's function in the reference's packed storage.

Mirror of ``NEdyson::green_func`` (reference src/greens.h:17-112,
src/greens.cpp:34-195).  The four components are numpy arrays of nao x nao
row-major complex128 blocks:

* ``les`` -- upper triangle, block (i, j), i <= j, at ``j*(j+1)/2 + i``
  (so the column G^<(., T) is contiguous);
* ``ret`` -- lower triangle, block (i, j), j <= i, at ``i*(i+1)/2 + j``
  (so the row G^R(T, .) is contiguous);
* ``tv``  -- block (t, m) at ``t*(ntau+1) + m``;
* ``mat`` -- block m.

The same layout is used in device memory, so host <-> device copies of a time
slice are single contiguous ranges.  Indices are 64-bit (Python ints / numpy
int64), which removes the reference's ``int`` overflow for nt*(nt+1)/2*nao^2
beyond 2^31.
"""
from __future__ import annotations

import numpy as np


def tri(n: int) -> int:
    """Number of blocks in a packed triangle with time indices 0..n."""
    return (n + 1) * (n + 2) // 2


class HostGF:
    def __init__(self, nt: int, ntau: int, nao: int, sig: int = -1):
        if nao <= 0 or nt < -1 or ntau < 0 or sig * sig != 1:
            raise ValueError("green_func: bad sizes (greens.cpp:35)")
        self.nt, self.ntau, self.nao, self.sig = int(nt), int(ntau), int(nao), int(sig)
        shp = (nao, nao)
        nn = max(nt, -1)
        self.les = np.zeros((tri(nn) if nt >= 0 else 0,) + shp, np.complex128)
        self.ret = np.zeros((tri(nn) if nt >= 0 else 0,) + shp, np.complex128)
        self.tv = np.zeros((max(nt + 1, 0), ntau + 1) + shp, np.complex128)
        self.mat = np.zeros((ntau + 1,) + shp, np.complex128)

    # index helpers (greens.cpp:177-195)
    @staticmethod
    def lesidx(i: int, j: int) -> int:
        assert 0 <= i <= j
        return j * (j + 1) // 2 + i

    @staticmethod
    def retidx(i: int, j: int) -> int:
        assert 0 <= j <= i
        return i * (i + 1) // 2 + j

    def lesblk(self, i, j):
        return self.les[self.lesidx(i, j)]

    def retblk(self, i, j):
        return self.ret[self.retidx(i, j)]

    def les_col(self, t):
        """G^<(0..t, t) -- contiguous."""
        return self.les[self.lesidx(0, t):self.lesidx(0, t) + t + 1]

    def ret_row(self, t):
        """G^R(t, 0..t) -- contiguous."""
        return self.ret[self.retidx(t, 0):self.retidx(t, 0) + t + 1]

    def get_dm(self, t: int) -> np.ndarray:
        """greens.h:68-74: rho = i*sig*G^<(t,t), or -G^M(beta) for t = -1."""
        if t == -1:
            return -self.mat[self.ntau].copy()
        return 1j * self.sig * self.lesblk(t, t)

    def set_tstp_zero(self, t: int) -> None:
        if t == -1:
            self.mat[:] = 0
            return
        self.ret_row(t)[:] = 0
        self.les_col(t)[:] = 0
        self.tv[t] = 0

    def copy(self) -> "HostGF":
        g = HostGF(self.nt, self.ntau, self.nao, self.sig)
        g.les[:] = self.les
        g.ret[:] = self.ret
        g.tv[:] = self.tv
        g.mat[:] = self.mat
        return g

    def nbytes(self) -> int:
        return self.les.nbytes + self.ret.nbytes + self.tv.nbytes + self.mat.nbytes
