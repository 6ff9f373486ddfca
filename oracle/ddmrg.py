"""CPU restatement of tensor-tools' dense (no-QN) tensors and two-site DMRG.

TEST INFRASTRUCTURE ONLY -- the parity oracle; see ``oracle/qtensor.py``.

Follows:
* dtensor index tags (size, name, type, level): dtensor/dtensor_index.h:34-60;
* ``dtensor::operator*`` (contract shared tags; result = this's free indices,
  then A's): dtensor/dtensor.cpp:300-368; ``contract``: :397-430 (positional);
  ``diagonal(type)``: :511-571; vector ops: :792-849;
* dense ``svd``/``svd_bond``: dtensor/dtensor_op.cpp:86-211.  CTF's
  ``svd(U,S,VT,K,threshold)`` is restated as: thin dgesvd, keep at most K
  values, and when ``cutoff > 0`` keep only singular values > cutoff.  That
  threshold rule lives inside CTF (not vendored) and is unpinned;
* MPS product state with DBL_EPSILON off the chosen spin: mps/tt.cpp:225-262;
  ``rc``/``position``/``normalize``: mps/tt.cpp:575-795;
* dense Heisenberg MPO (D=5): models/hams/Heisenberg.cpp:185-208 with
  ``addOperators`` :72-148;
* ``big_dtensor`` product/diagonal/size: dtensor/big_dtensor.cpp:23-161;
* ``buildEnv``/``updateSite``/``updateEnv``/``dmrg`` (dense schedule):
  algos/dmrg/dmrg.cpp:24-51, 228-295, 466-486, 591-646.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import scipy.linalg as sla

from .davidson import tensor_davidson, DavidsonStats
from .qdmrg import spin_op
from .qtensor import Link, Site, All

MoveFromLeft, MoveFromRight = 0, 1
DBL_EPS = np.finfo(np.float64).eps


@dataclass
class DIndex:
    size: int
    name: str
    type: int = Link
    level: int = 0

    def tag(self):
        return (self.size, self.name, self.type, self.level)

    def copy(self):
        return DIndex(self.size, self.name, self.type, self.level)

    def similar(self, other: "DIndex", typ: int = All) -> bool:
        return (self.size == other.size and self.name == other.name
                and (self.type == other.type or typ == All)
                and (self.type == typ or typ == All)
                and (self.level == other.level + 1 or self.level + 1 == other.level))


class DTensor:
    def __init__(self, idx: Optional[List[DIndex]] = None, data: Optional[np.ndarray] = None):
        self.idx = [i.copy() for i in (idx or [])]
        if data is None and idx:
            data = np.zeros([i.size for i in self.idx])
        self.data = data
        self.initted = data is not None

    @property
    def rank(self):
        return len(self.idx)

    def copy(self):
        return DTensor([i.copy() for i in self.idx], None if self.data is None else self.data.copy())

    def prime(self, inc=1):
        for i in self.idx:
            i.level += inc

    def scale(self, c):
        self.data *= c

    def norm(self):
        return float(np.sqrt(np.sum(self.data * self.data)))

    def normalize(self):
        r = self.norm()
        self.data = self.data / r
        return r

    def add(self, A: "DTensor", c=1.0):
        self.data += c * _align(A, self)

    def inner_product(self, A: "DTensor"):
        return float(np.sum(self.data * _align(A, self)))

    def contract(self, A: "DTensor"):
        # positional: both operands use this tensor's labels (dtensor.cpp:397-430)
        return float(np.sum(self.data * A.data))

    def diagonal(self, typ: int) -> "DTensor":
        new_idx = [ix for i, ix in enumerate(self.idx)
                   if not any(ix.similar(jx, typ) for jx in self.idx)]
        pairs = []
        for i in range(self.rank):
            for j in range(i + 1, self.rank):
                if self.idx[i].similar(self.idx[j], typ):
                    keep = i if self.idx[i].level < self.idx[j].level else j
                    new_idx.append(self.idx[keep])
                    pairs.append((i, j))
                    break
        if len(new_idx) == self.rank:
            return self.copy()
        # einsum with primes ignored: repeated letters take the diagonal
        letters = {}
        def lab(ix):
            key = (ix.size, ix.name, ix.type)
            if key not in letters:
                letters[key] = chr(ord("a") + len(letters))
            return letters[key]
        src = "".join(lab(ix) for ix in self.idx)
        dst = "".join(lab(ix) for ix in new_idx)
        return DTensor(new_idx, np.einsum(src + "->" + dst, self.data).copy())


def _align(A: DTensor, like: DTensor) -> np.ndarray:
    perm = [ [ix.tag() for ix in A.idx].index(t.tag()) for t in like.idx ]
    return np.transpose(A.data, perm)


def dcontract(A: DTensor, B: DTensor) -> DTensor:
    """dtensor::operator* (dtensor/dtensor.cpp:300-368)."""
    if A.initted and not B.initted:
        return A.copy()
    if B.initted and not A.initted:
        return B.copy()
    atags = [ix.tag() for ix in A.idx]
    btags = [ix.tag() for ix in B.idx]
    a_ax, b_ax = [], []
    for i, t in enumerate(atags):
        if t in btags:
            a_ax.append(i)
            b_ax.append(btags.index(t))
    idx = [ix for i, ix in enumerate(A.idx) if i not in a_ax] + \
          [ix for j, ix in enumerate(B.idx) if j not in b_ax]
    return DTensor(idx, np.tensordot(A.data, B.data, axes=(a_ax, b_ax)))


def dsvd(A: DTensor, left: List[DIndex], right: List[DIndex], direction: int,
         cutoff: float = 0.0, K: int = 0):
    """dtensor/dtensor_op.cpp:120-211; returns (U, V, S)."""
    tags = [ix.tag() for ix in A.idx]
    perm = [tags.index(ix.tag()) for ix in left] + [tags.index(ix.tag()) for ix in right]
    r = int(np.prod([ix.size for ix in left]))
    c = int(np.prod([ix.size for ix in right]))
    mA = np.transpose(A.data, perm).reshape((r, c), order="F")
    if r == 1 and c == 2:
        d = float(np.sqrt(np.sum(mA * mA)))
        Um = np.ones((1, 1))
        s = np.array([d])
    else:
        Um, s, _ = sla.svd(mA, full_matrices=False, lapack_driver="gesvd")
        keep = s.size
        if K:
            keep = min(keep, K)
        if cutoff > 0:
            keep = min(keep, int(np.sum(s > cutoff)))
        keep = max(keep, 1)
        Um, s = Um[:, :keep], s[:keep]
    k = s.size
    mid = DIndex(k, "dsvdmid", Link, 0)
    if direction == MoveFromLeft:
        U = DTensor(list(left) + [mid], Um.reshape([ix.size for ix in left] + [k], order="F"))
        Vm = Um.T @ mA
        if r == 1 and c == 2:
            Vm = mA.copy()
        V = DTensor([mid] + list(right), Vm.reshape([k] + [ix.size for ix in right], order="F"))
    else:
        if r == 1 and c == 2:
            Vm = mA / s[0] if s[0] != 0 else np.full((1, 2), 1.0 / np.sqrt(2.0))
        else:
            _, _, Vt = sla.svd(mA, full_matrices=False, lapack_driver="gesvd")
            Vm = Vt[:k, :]
        V = DTensor([mid] + list(right), Vm.reshape([k] + [ix.size for ix in right], order="F"))
        Um2 = mA @ Vm.T
        U = DTensor(list(left) + [mid], Um2.reshape([ix.size for ix in left] + [k], order="F"))
    S = DTensor([mid], s.copy())
    return U, V, S


def dsvd_bond(combined: DTensor, A_left: DTensor, A_right: DTensor, mid: DIndex,
              direction: int, cutoff: float = 0.0, K: int = 0):
    """dtensor/dtensor_op.cpp:86-115."""
    t = mid.tag()
    right = [ix for ix in A_right.idx if ix.tag() != t]
    left = [ix for ix in A_left.idx if ix.tag() != t]
    U, V, S = dsvd(combined, left, right, direction, cutoff, K)
    newmid = mid.copy()
    newmid.size = S.data.size
    U.idx[-1] = newmid.copy()
    V.idx[0] = newmid.copy()
    return U, V, S


class DMPS:
    def __init__(self, L: int, product_state: List[int], mid: int = 1, d: int = 2):
        self.length, self.id, self.d = L, mid, d
        self.bond_dims = [1] * (L + 1)
        self.A = []
        for i in range(L):
            idx = [DIndex(1, self.link_name(i)), DIndex(d, "Site%d" % i, Site),
                   DIndex(1, self.link_name(i + 1))]
            data = np.full((1, d, 1), DBL_EPS)
            data[0, product_state[i], 0] = 1.0
            self.A.append(DTensor(idx, data))
        self.center = -1

    def link_name(self, i):
        return "ID%dLink%d" % (self.id, i)

    def _move_left(self, c):
        ln = self.link_name(c)
        left = [ix for ix in self.A[c].idx if ix.name == ln]
        right = [ix for ix in self.A[c].idx if ix.name != ln]
        mid = left[0].copy()
        U, V, S = dsvd(self.A[c], left, right, MoveFromRight)
        mid.size = S.data.size
        self.bond_dims[c] = mid.size
        V.idx[0] = mid.copy()
        self.A[c] = V
        self.A[c - 1] = dcontract(self.A[c - 1], U)
        self.A[c - 1].idx[-1] = mid.copy()
        return S

    def rc(self):
        for i in range(self.length - 1, 0, -1):
            self._move_left(i)
        self.center = 0

    def position(self, site: int):
        if self.center == -1:
            self.rc()
        while self.center != site:
            c = self.center
            if c > site:
                self._move_left(c)
                self.center -= 1
            else:
                ln = self.link_name(c + 1)
                right = [ix for ix in self.A[c].idx if ix.name == ln]
                left = [ix for ix in self.A[c].idx if ix.name != ln]
                mid = right[0].copy()
                U, V, S = dsvd(self.A[c], left, right, MoveFromLeft)
                mid.size = S.data.size
                self.bond_dims[c + 1] = mid.size
                U.idx[-1] = mid.copy()
                self.A[c] = U
                self.A[c + 1] = dcontract(V, self.A[c + 1])
                self.A[c + 1].idx[0] = mid.copy()
                self.center += 1

    def normalize(self):
        nm = self.A[self.center].norm()
        self.A[self.center].data = self.A[self.center].data / nm


class DMPO:
    """Dense Heisenberg MPO, D=5 (models/hams/Heisenberg.cpp:185-208)."""

    def __init__(self, L: int, mid: int = 2, dh=None, tE: float = 0.0, D: int = 5):
        self.length, self.id = L, mid
        self.A = []
        for i in range(L):
            dl = 1 if i == 0 else D
            dr = 1 if i == L - 1 else D
            idx = [DIndex(dl, "ID%dLink%d" % (mid, i)), DIndex(2, "Site%d" % i, Site, 0),
                   DIndex(2, "Site%d" % i, Site, 1), DIndex(dr, "ID%dLink%d" % (mid, i + 1))]
            self.A.append(DTensor(idx, np.zeros((dl, 2, 2, dr))))
        for site in range(L):
            last = site == L - 1
            if site > 0:
                self._add(site, 0, 0, "Id", 1.0)
            if not last:
                self._add(site, 1, 1, "Id", 1.0)
            if dh is not None:
                self._add(site, 1, 0, "Sz", dh[site])
            if tE != 0:
                self._add(site, 1, 0, "Id", -tE / L)
            if site > 0:
                self._add(site, 2, 0, "Sz", 1.0)
            if not last:
                self._add(site, 1, 2, "Sz", 1.0)
            if site > 0:
                self._add(site, 3, 0, "S+", 1.0)
            if not last:
                self._add(site, 1, 3, "S-", 0.5)
            if site > 0:
                self._add(site, 4, 0, "S-", 1.0)
            if not last:
                self._add(site, 1, 4, "S+", 0.5)

    def _add(self, site, r, c, op, val):
        """addOperators (models/hams/Heisenberg.cpp:72-148): element (r,k,b,c) is
        written (not accumulated) with val*<b|op|k>; site 0 drops the row."""
        W = self.A[site].data
        rr = 0 if site == 0 else r
        for k in range(2):
            for b in range(2):
                W[rr, k, b, c] = val * spin_op(b, op, k)


class BigDTensor:
    """big_dtensor (dtensor/big_dtensor.{h,cpp}): MPO tensors kept separately."""

    def __init__(self):
        self.L = self.R = None
        self.mid = []
        self._size = 0

    def setLeft(self, L):
        self.L = L

    def setRight(self, R):
        self.R = R

    def addMid(self, W):
        self.mid.append(W)

    def product(self, v: DTensor) -> DTensor:
        res = DTensor()
        if self.L is not None:
            res = dcontract(self.L, v)
        for m in self.mid:
            res = dcontract(res, m) if res.rank > 0 else dcontract(v, m)
        if self.R is not None:
            res = dcontract(res, self.R)
        res.prime(-1)
        return res

    def expec(self, v):
        return self.product(v).contract(v)

    def diagonal(self) -> DTensor:
        res = DTensor()
        if self.L is not None:
            res = self.L.diagonal(Link)
        for m in self.mid:
            res = dcontract(res, m.diagonal(Site))
        if self.R is not None:
            res = dcontract(res, self.R.diagonal(Link))
        return res

    def size(self):
        if self._size == 0:
            self._size = 1
            for T in (self.L, self.R):
                if T is not None:
                    for ix in T.idx:
                        if ix.level > 0:
                            self._size *= ix.size
        for m in self.mid:
            for ix in m.idx:
                if ix.type == Site:
                    self._size *= ix.size
        return self._size


def _dboundary(psi_idx: DIndex, h_idx: DIndex) -> DTensor:
    a = psi_idx.copy()
    a.level += 1
    return DTensor([a, h_idx.copy(), psi_idx.copy()], np.ones((a.size, h_idx.size, psi_idx.size)))


def denv_step(env: DTensor, A: DTensor, W: DTensor) -> DTensor:
    t1 = A.copy()
    t1.prime()
    return dcontract(dcontract(dcontract(t1, env), W), A)


def dbuild_env(psi: DMPS, H: DMPO):
    L = psi.length
    TR = [None] * L
    TL = [None] * L
    TL[0] = _dboundary(psi.A[0].idx[0], H.A[0].idx[0])
    TR[L - 1] = _dboundary(psi.A[L - 1].idx[-1], H.A[L - 1].idx[-1])
    for i in range(L - 1, 0, -1):
        TR[i - 1] = denv_step(TR[i], psi.A[i], H.A[i])
    return TR, TL


def dupdate_site(psi, H, TR, TL, site, direction, max_bd, cutoff, search_space_size,
                 max_restart, log=None):
    """algos/dmrg/dmrg.cpp:228-295."""
    A = BigDTensor()
    if direction == MoveFromLeft:
        l, r = site, site + 1
    else:
        l, r = site - 1, site
    A.setLeft(TL[l])
    A.addMid(H.A[l])
    A.addMid(H.A[r])
    A.setRight(TR[r])
    x = dcontract(psi.A[l], psi.A[r])
    stats = DavidsonStats()
    energy = tensor_davidson(A, x, search_space_size, max_restart, 1e-12, "S", stats=stats)
    ln = psi.link_name(r)
    mid = [ix for ix in psi.A[l].idx if ix.name == ln][0]
    U, V, S = dsvd_bond(x, psi.A[l], psi.A[r], mid, direction, cutoff, max_bd)
    psi.A[l], psi.A[r] = U, V
    psi.bond_dims[r] = S.data.size
    psi.center = r if direction == MoveFromLeft else l
    if log is not None:
        log.energies.append(energy)
        log.matvecs += stats.matvecs
    return energy


def dupdate_env(psi, H, TR, TL, site, direction):
    if direction == MoveFromLeft:
        TL[site + 1] = denv_step(TL[site], psi.A[site], H.A[site])
    else:
        TR[site - 1] = denv_step(TR[site], psi.A[site], H.A[site])


def ddmrg(psi: DMPS, H: DMPO, num_sweeps: int, max_bd: List[int], cutoff: List[float],
          max_restart: List[int], sweep_logs: Optional[list] = None) -> float:
    """Dense schedule overload (algos/dmrg/dmrg.cpp:591-646): no per-sweep normalize."""
    from .qdmrg import SweepLog
    L = H.length
    psi.position(0)
    psi.normalize()
    TR, TL = dbuild_env(psi, H)
    energy = 0.0
    for sweep in range(num_sweeps):
        lbd = sweep % len(max_bd)
        lc = sweep % len(cutoff)
        lmr = sweep % len(max_restart)
        slog = SweepLog() if sweep_logs is not None else None
        for l in range(2 * sweep, 2 * (sweep + 1)):
            direction = MoveFromLeft if l % 2 == 0 else MoveFromRight
            for i in range(L - 1):
                site = i if direction == MoveFromLeft else L - 1 - i
                energy = dupdate_site(psi, H, TR, TL, site, direction, max_bd[lbd], cutoff[lc],
                                      3, max_restart[lmr], slog)
                dupdate_env(psi, H, TR, TL, site, direction)
        if sweep_logs is not None:
            slog.bond_dims = list(psi.bond_dims)
            sweep_logs.append(slog)
    psi.position(0)
    psi.normalize()
    return energy
