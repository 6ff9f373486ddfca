"""CPU restatement of tensor-tools' U(1) MPS/MPO objects and two-site DMRG.

TEST INFRASTRUCTURE ONLY -- the parity oracle; see ``oracle/qtensor.py``.

Follows:
* qMPS product state and link-QN enumeration: mps/qtt.cpp:205-311;
* spin-1/2 sites: models/sites/spinhalf.{h,cpp} (Dn=0, Up=1, QN -1/+1);
* hand-written Heisenberg qMPO (D=5 as sectors (-2,1),(0,3),(+2,1)):
  models/hams/Heisenberg.cpp:333-402 with ``addOperators`` :152-196;
* ``big_qtensor`` product/expec/size: qtensor/big_qtensor.{h,cpp};
* ``position``/``normalize``: mps/qtt.cpp:899-994;
* ``buildEnv``/``updateSite``/``updateEnv``/``dmrg`` (schedule overload):
  algos/dmrg/dmrg.cpp:56-85, 300-372, 491-509, 702-755.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from .qtensor import QIndex, QTensor, Inward, Outward, Link, Site, qn, qadd, contract
from .qsvd import svd, svd_bond, MoveFromLeft, MoveFromRight, TruncInfo, calc_entropy
from .davidson import tensor_davidsonIT, DavidsonStats

SPIN_PHY_QN = [qn(-1), qn(+1)]  # Dn, Up (models/sites/spinhalf.h:26-32)


def spin_op(bra: int, op: str, ket: int) -> float:
    """spinhalf::d_bra_op_ket (models/sites/spinhalf.cpp:23-46)."""
    Dn, Up = 0, 1
    if op in ("Id", "I"):
        return 1.0 if ket == bra else 0.0
    if op == "Sz":
        if ket == Dn and bra == Dn:
            return -0.5
        if ket == Up and bra == Up:
            return 0.5
        return 0.0
    if op == "Sx":
        return 0.5 if ket != bra else 0.0
    if op in ("S+", "Sp"):
        return 1.0 if (ket == Dn and bra == Up) else 0.0
    if op in ("S-", "Sm"):
        return 1.0 if (ket == Up and bra == Dn) else 0.0
    raise ValueError(op)


class QMPS:
    """qTensorTrain<double,1> built from a product string (mps/qtt.cpp:58-80, 205-311)."""

    def __init__(self, L: int, product_state: List[int], mid: int = 1,
                 phy_qn=SPIN_PHY_QN):
        self.length = L
        self.id = mid
        self.phy_qn = list(phy_qn)
        self.totalQ = (0, 0)
        for s in product_state:
            self.totalQ = qadd(self.totalQ, self.phy_qn[s])
        self.bond_dims = [1] * (L + 1)
        link_qn = [set() for _ in range(L + 1)]
        link_qn[0].add((0, 0))
        link_qn[L].add(self.totalQ)
        for j in range(1, L):
            for q in link_qn[j - 1]:
                for p in self.phy_qn:
                    link_qn[j].add(qadd(q, p))
        for j in range(L - 1, 0, -1):
            rm = [q for q in link_qn[j]
                  if not any(qadd(q, p) in link_qn[j + 1] for p in self.phy_qn)]
            for q in rm:
                link_qn[j].discard(q)
        self.A: List[QTensor] = []
        pref = "ID%dLink" % self.id
        for i in range(L):
            T = QTensor([QIndex(Inward, pref + str(i), Link, 0),
                         QIndex(Inward, "Site" + str(i), Site, 0),
                         QIndex(Outward, pref + str(i + 1), Link, 0)])
            for q in sorted(link_qn[i]):
                T.idx[0].add_qn(q, 1)
            for p in self.phy_qn:
                T.idx[1].add_qn(p, 1)
            for q in sorted(link_qn[i + 1]):
                T.idx[2].add_qn(q, 1)
            T.init_block()
            self.A.append(T)
        last = (0, 0)
        for i in range(L):
            p = self.phy_qn[product_state[i]]
            key = (last, p, qadd(last, p))
            last = qadd(last, p)
            self.A[i].blocks[self.A[i].bid[key]][...] = 1.0
        self.center = L - 1

    def link_name(self, i: int) -> str:
        return "ID%dLink%d" % (self.id, i)

    def position(self, site: int) -> float:
        """mps/qtt.cpp:932-994 (center is never -1 for product states)."""
        S = None
        while self.center != site:
            c = self.center
            if c > site:
                ln = self.link_name(c)
                left = [ix for ix in self.A[c].idx if ix.name == ln]
                right = [ix for ix in self.A[c].idx if ix.name != ln]
                mid = left[0]
                U, V, S = svd(self.A[c], left, right, MoveFromRight)
                self.bond_dims[c] = S.total_size()
                self.A[c] = V
                V.idx[0].name = mid.name
                V.idx[0].level = mid.level
                self.A[c - 1] = contract(self.A[c - 1], U)
                self.A[c - 1].idx[-1].name = mid.name
                self.A[c - 1].idx[-1].level = mid.level
                self.center -= 1
            else:
                ln = self.link_name(c + 1)
                right = [ix for ix in self.A[c].idx if ix.name == ln]
                left = [ix for ix in self.A[c].idx if ix.name != ln]
                mid = right[0]
                U, V, S = svd(self.A[c], left, right, MoveFromLeft)
                self.bond_dims[c + 1] = S.total_size()
                self.A[c] = U
                U.idx[-1].name = mid.name
                U.idx[-1].level = mid.level
                self.A[c + 1] = contract(V, self.A[c + 1])
                self.A[c + 1].idx[0].name = mid.name
                self.A[c + 1].idx[0].level = mid.level
                self.center += 1
        return 0.0 if S is None else calc_entropy(S)

    def normalize(self) -> None:
        """mps/qtt.cpp:899-909 (centre form)."""
        nm = self.A[self.center].norm()
        self.A[self.center].div(nm)


class QMPO:
    """Hand-written Heisenberg qMPO (models/hams/Heisenberg.cpp:333-402)."""

    def __init__(self, L: int, mid: int = 2, dh: Optional[List[float]] = None,
                 tE: float = 0.0, phy_qn=SPIN_PHY_QN):
        self.length = L
        self.id = mid
        self.phy_qn = list(phy_qn)
        self.A: List[QTensor] = []
        pref = "ID%dLink" % self.id
        for i in range(L):
            T = QTensor([QIndex(Inward, pref + str(i), Link, 0),
                         QIndex(Outward, "Site" + str(i), Site, 0),
                         QIndex(Inward, "Site" + str(i), Site, 1),
                         QIndex(Outward, pref + str(i + 1), Link, 0)])
            if i == 0:
                T.idx[0].add_qn(qn(0), 1)
            else:
                T.idx[0].add_qn(qn(0), 3)
                T.idx[0].add_qn(qn(-2), 1)
                T.idx[0].add_qn(qn(2), 1)
            for p in self.phy_qn:
                T.idx[1].add_qn(p, 1)
            for p in self.phy_qn:
                T.idx[2].add_qn(p, 1)
            if i == L - 1:
                T.idx[3].add_qn(qn(0), 1)
            else:
                T.idx[3].add_qn(qn(0), 3)
                T.idx[3].add_qn(qn(-2), 1)
                T.idx[3].add_qn(qn(2), 1)
            T.init_block()
            self.A.append(T)
        for site in range(L):
            last = site == L - 1
            if site > 0:
                self._add(site, 0, 0, "Id", 1.0, 0, 0)
            if not last:
                self._add(site, 1, 1, "Id", 1.0, 0, 0)
            if dh is not None:
                self._add(site, 1, 0, "Sz", dh[site], 0, 0)
            if tE != 0:
                self._add(site, 1, 0, "Id", -tE / L, 0, 0)
            if site > 0:
                self._add(site, 2, 0, "Sz", 1.0, 0, 0)
            if not last:
                self._add(site, 1, 2, "Sz", 1.0, 0, 0)
            if site > 0:
                self._add(site, 0, 0, "S+", 1.0, -2, 0)
                self._add(site, 0, 0, "S-", 1.0, 2, 0)
            if not last:
                self._add(site, 1, 0, "S-", 0.5, 0, -2)
                self._add(site, 1, 0, "S+", 0.5, 0, 2)

    def _add(self, site, r, c, op, val, Qi, Qo):
        """addOperators for qMPO (models/hams/Heisenberg.cpp:152-196)."""
        T = self.A[site]
        added = False
        for k in range(2):
            for b in range(2):
                key = (qn(Qi), self.phy_qn[k], self.phy_qn[b], qn(Qo))
                if key in T.bid:
                    added = True
                    blk = T.blocks[T.bid[key]]
                    rr = 0 if site == 0 else r
                    # column-major offset s0*r + s3*c with unit site dims
                    blk[rr, 0, 0, c] = val * spin_op(b, op, k)
        assert added


class BigQTensor:
    """big_qtensor (qtensor/big_qtensor.{h,cpp}); ``mid`` is pre-contracted."""

    def __init__(self):
        self.L = None
        self.R = None
        self.mid = QTensor()
        self._size = 0
        self.flops = 0

    def setLeft(self, L):
        self.L = L

    def setRight(self, R):
        self.R = R

    def addMid(self, W):
        self.mid = contract(self.mid, W)

    def product(self, v: QTensor) -> QTensor:
        """((L*v)*mid)*R then prime(-1) (qtensor/big_qtensor.cpp:23-40)."""
        res = QTensor()
        if self.L is not None:
            res = contract(self.L, v)
        res = contract(res, self.mid) if res.rank > 0 else contract(v, self.mid)
        if self.R is not None:
            res = contract(res, self.R)
        res.prime(-1)
        return res

    def expec(self, v: QTensor) -> float:
        return self.product(v).contract(v)

    def size(self) -> int:
        """Sector-count product, re-multiplied by mid on each call (:96-118)."""
        if self._size == 0:
            self._size = 1
            if self.L is not None:
                for ix in self.L.idx:
                    if ix.level > 0:
                        self._size *= ix.size()
            if self.R is not None:
                for ix in self.R.idx:
                    if ix.level > 0:
                        self._size *= ix.size()
        for ix in self.mid.idx:
            if ix.type == Site:
                self._size *= ix.size()
        return self._size


def _boundary(psi_idx: QIndex, h_idx: QIndex) -> QTensor:
    T = QTensor([psi_idx, h_idx, psi_idx])
    T.idx[0].level += 1  # primeLink
    T.idx[0].arrow = Outward if T.idx[0].arrow == Inward else Inward
    T.init_block()
    T.set_one()
    T.dag()
    return T


def env_step(env: QTensor, A: QTensor, W: QTensor) -> QTensor:
    """((A^dag' * env) * W) * A (algos/dmrg/dmrg.cpp:491-509)."""
    t1 = A.copy()
    t1.dag()
    t1.prime()
    t4 = contract(t1, env)
    t5 = contract(t4, W)
    return contract(t5, A)


def build_env(psi: QMPS, H: QMPO):
    """algos/dmrg/dmrg.cpp:56-85."""
    L = psi.length
    TR: List[Optional[QTensor]] = [None] * L
    TL: List[Optional[QTensor]] = [None] * L
    TL[0] = _boundary(psi.A[0].idx[0], H.A[0].idx[0])
    TR[L - 1] = _boundary(psi.A[L - 1].idx[-1], H.A[L - 1].idx[-1])
    for i in range(L - 1, 0, -1):
        TR[i - 1] = env_step(TR[i], psi.A[i], H.A[i])
    return TR, TL


class SweepLog:
    def __init__(self):
        self.energies = []
        self.trunc = []
        self.cut_gaps = []
        self.randomized = []
        self.step_matvecs = []
        self.bond_dims = []
        self.entropy = []
        self.matvecs = 0
        self.heff_flops = 0


def update_site(psi: QMPS, H: QMPO, TR, TL, site: int, direction: int, max_bd: int,
                cutoff: float, search_space_size: int, max_restart: int,
                rng: np.random.Generator, log: Optional[SweepLog] = None) -> float:
    """algos/dmrg/dmrg.cpp:300-372."""
    stats = DavidsonStats()
    A = BigQTensor()
    if direction == MoveFromLeft:
        l, r = site, site + 1
    else:
        l, r = site - 1, site
    A.setLeft(TL[l])
    A.addMid(H.A[l])
    A.addMid(H.A[r])
    A.setRight(TR[r])
    x = contract(psi.A[l], psi.A[r])
    energy = tensor_davidsonIT(A, x, search_space_size, max_restart, 1e-12, "S",
                               rng=rng, stats=stats)
    ln = psi.link_name(r)
    mid = [ix for ix in psi.A[l].idx if ix.name == ln][0]
    info = TruncInfo()
    U, V, S = svd_bond(x, psi.A[l], psi.A[r], mid, direction, cutoff, max_bd, info)
    psi.A[l], psi.A[r] = U, V
    psi.bond_dims[r] = S.total_size()
    psi.center = r if direction == MoveFromLeft else l
    if log is not None:
        log.energies.append(energy)
        log.trunc.append((info.trunc_err, info.kept, tuple(info.kept_per_sector)))
        log.cut_gaps.append(min(info.cut_gap, info.cutoff_margin))
        log.randomized.append(stats.randomized)
        log.step_matvecs.append(stats.matvecs)
        log.matvecs += stats.matvecs
        mid_bond = (site == psi.length // 2 - 1) if direction == MoveFromLeft else (site == psi.length // 2)
        if mid_bond:
            log.entropy.append(calc_entropy(S))
    return energy


def update_env(psi: QMPS, H: QMPO, TR, TL, site: int, direction: int) -> None:
    """algos/dmrg/dmrg.cpp:491-509."""
    if direction == MoveFromLeft:
        TL[site + 1] = env_step(TL[site], psi.A[site], H.A[site])
    else:
        TR[site - 1] = env_step(TR[site], psi.A[site], H.A[site])


def dmrg(psi: QMPS, H: QMPO, num_sweeps: int, max_bd: List[int], cutoff: List[float],
         max_restart: List[int], seed: int = 12345, log: Optional[SweepLog] = None,
         sweep_logs: Optional[list] = None) -> float:
    """Schedule overload (algos/dmrg/dmrg.cpp:702-755)."""
    L = H.length
    search_space_size = 3
    psi.position(0)
    psi.normalize()
    TR, TL = build_env(psi, H)
    rng = np.random.default_rng(seed)
    energy = 0.0
    for sweep in range(num_sweeps):
        lbd = sweep % len(max_bd)
        lc = sweep % len(cutoff)
        lmr = sweep % len(max_restart)
        slog = SweepLog() if sweep_logs is not None else log
        for l in range(2 * sweep, 2 * (sweep + 1)):
            direction = MoveFromLeft if l % 2 == 0 else MoveFromRight
            for i in range(L - 1):
                site = i if direction == MoveFromLeft else L - 1 - i
                energy = update_site(psi, H, TR, TL, site, direction, max_bd[lbd], cutoff[lc],
                                     search_space_size, max_restart[lmr], rng, slog)
                update_env(psi, H, TR, TL, site, direction)
        if sweep_logs is not None:
            slog.bond_dims = list(psi.bond_dims)
            sweep_logs.append(slog)
        psi.normalize()
    psi.position(0)
    return energy


def neel(L: int) -> List[int]:
    """Neel string of project/main.cpp:159-164: even sites Dn, odd sites Up."""
    return [0 if i % 2 == 0 else 1 for i in range(L)]
