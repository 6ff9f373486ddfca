"""CPU restatement of tensor-tools' block-sparse U(1) tensor (``qtensor``).

TEST INFRASTRUCTURE ONLY.  This module is the parity oracle for the CUDA
path.  Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or as the timed CPU baseline -- never as the product.

Parity status: the reference cannot be compiled here (CTF, MPI, HDF5, Eigen
and ScaLAPACK are absent) and ships no golden vectors for this path, so this
restatement is pinned by exact-diagonalisation known answers (``oracle/ed.py``)
and by the structural invariants the reference asserts; bit-level parity with
CTF's own contraction order is unpinned.

Every function cites the reference routine it follows (paths relative to the
reference project root).  Conventions kept from the reference:

* ``QN`` is a pair of ints (``QN_t_2``, util/QN.h:79-127); a spin-1/2 site
  carries (2Sz, 0).  Ordering is lexicographic (util/QN.h:100-104).
* An index carries arrow (0 = Inward, 1 = Outward), name, type (0 = Link,
  1 = Site), prime level and a QN-sorted sector list
  (qtensor/qtensor_index.h:35-66).  Two indices pair in a contraction when
  their tags match after flipping one arrow (qtensor/qtensor.cpp:540-555).
* Block data is an ndarray whose axes follow the tensor's index order.  When
  blocks are flattened into matrices (SVD) the linearisation is column-major,
  first index fastest, as CTF's ``slice`` does (qtensor/qtensor_op.cpp:1229-1246).
"""
from __future__ import annotations

import copy as _copy
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

Inward, Outward = 0, 1
Link, Site, All = 0, 1, 2

QN = Tuple[int, int]


def qn(x: int, y: int = 0) -> QN:
    """QN_t_2 constructed from an int (util/QN.h:85): (x, 0)."""
    return (int(x), int(y))


def qadd(a: QN, b: QN) -> QN:
    return (a[0] + b[0], a[1] + b[1])


def qsub(a: QN, b: QN) -> QN:
    return (a[0] - b[0], a[1] - b[1])


QZERO: QN = (0, 0)


@dataclass
class QIndex:
    """qtensor_index (qtensor/qtensor_index.h:35-118)."""

    arrow: int
    name: str
    type: int = Link
    level: int = 0
    qns: List[Tuple[QN, int]] = field(default_factory=list)

    def add_qn(self, q: QN, dim: int) -> None:
        # addQN keeps the sector list sorted by QN (sortQN via setTag, :47-55)
        self.qns.append((q, int(dim)))
        self.qns.sort(key=lambda p: p[0])

    def size(self) -> int:
        """Number of QN sectors (qtensor_index::size, :62) -- not the dimension."""
        return len(self.qns)

    def qn(self, i: int) -> QN:
        return self.qns[i][0]

    def qdim(self, i: int) -> int:
        return self.qns[i][1]

    def dim(self) -> int:
        return sum(d for _, d in self.qns)

    def tag(self):
        """Hash key equivalent to ``tag()`` (:66): arrow, level, name, type, sectors."""
        return (self.arrow, self.level, self.name, self.type, tuple(self.qns))

    def tag_no_arrow(self):
        return (self.level, self.name, self.type, tuple(self.qns))

    def dagged(self) -> "QIndex":
        r = self.copy()
        r.arrow = Outward if self.arrow == Inward else Inward
        return r

    def copy(self) -> "QIndex":
        return QIndex(self.arrow, self.name, self.type, self.level, list(self.qns))

    def __eq__(self, other):  # qtensor_index::operator== (qtensor/qtensor_index.cpp:85-87)
        return self.tag() == other.tag()


class QTensor:
    """qtensor<double> (qtensor/qtensor.h:47-164) with dense numpy blocks."""

    def __init__(self, idx: List[QIndex] | None = None):
        self.idx: List[QIndex] = [i.copy() for i in (idx or [])]
        self.blocks: List[np.ndarray] = []
        self.bqn: List[Tuple[QN, ...]] = []
        self.bqi: List[Tuple[int, ...]] = []
        self.bqd: List[Tuple[int, ...]] = []
        self.bid: Dict[Tuple[QN, ...], int] = {}
        self.initted = False

    @property
    def rank(self) -> int:
        return len(self.idx)

    def copy(self) -> "QTensor":
        r = QTensor()
        r.idx = [i.copy() for i in self.idx]
        r.blocks = [b.copy() for b in self.blocks]
        r.bqn = list(self.bqn)
        r.bqi = list(self.bqi)
        r.bqd = list(self.bqd)
        r.bid = dict(self.bid)
        r.initted = self.initted
        return r

    # --- construction -----------------------------------------------------
    def init_block(self) -> None:
        """Enumerate all legal sector combinations (qtensor/qtensor.cpp:301-345).

        Combination i decodes with the first index fastest; a combination is
        legal when sum(Inward qn) - sum(Outward qn) == 0.
        """
        if self.rank > 0 and not self.initted:
            stride = [1]
            for ix in self.idx:
                stride.append(ix.size() * stride[-1])
            for i in range(stride[-1]):
                pos, qns, qds = [], [], []
                tot = QZERO
                for j, ix in enumerate(self.idx):
                    p = (i // stride[j]) % ix.size()
                    pos.append(p)
                    qns.append(ix.qn(p))
                    qds.append(ix.qdim(p))
                    tot = qadd(tot, ix.qn(p)) if ix.arrow == Inward else qsub(tot, ix.qn(p))
                if tot == QZERO:
                    self._append_block(tuple(qns), tuple(pos), tuple(qds),
                                       np.zeros(qds, dtype=np.float64))
        self.initted = True

    def _append_block(self, q, qi, qd, data) -> int:
        self.blocks.append(data)
        self.bqn.append(tuple(q))
        self.bqi.append(tuple(qi))
        self.bqd.append(tuple(qd))
        self.bid[tuple(q)] = len(self.blocks) - 1
        return len(self.blocks) - 1

    def set_one(self) -> None:  # :399-405
        for b in self.blocks:
            b[...] = 1.0

    def set_zero(self) -> None:
        for b in self.blocks:
            b[...] = 0.0

    def set_random(self, rng: np.random.Generator) -> None:
        """``setRandom`` (:381-388): CTF fill_random(0,1) per block; seeded here."""
        for b in self.blocks:
            b[...] = rng.random(b.shape)

    # --- index manipulation -------------------------------------------------
    def prime(self, inc: int = 1) -> None:
        for ix in self.idx:
            ix.level += inc

    def dag(self) -> None:
        for ix in self.idx:
            ix.arrow = Outward if ix.arrow == Inward else Inward

    # --- vector ops (qtensor/qtensor.cpp:1031-1179, 1606-1647) --------------
    def scale(self, c: float) -> None:  # operator*= (:1031-1040)
        for b in self.blocks:
            b *= c

    def div(self, c: float) -> None:  # operator/= multiplies by 1/c (:1046-1055)
        inv = 1.0 / c
        for b in self.blocks:
            b *= inv

    def norm(self) -> float:  # :1606-1616
        return float(np.sqrt(sum(float(np.sum(b * b)) for b in self.blocks)))

    def normalize(self) -> float:  # :1638-1647
        r = self.norm()
        inv = 1.0 / r
        for b in self.blocks:
            b *= inv
        return r

    def add(self, A: "QTensor", c: float = 1.0) -> None:
        """``add`` (:1127-1156): matching blocks accumulate, missing ones are inserted."""
        assert A.rank == self.rank
        for key, aid in A.bid.items():
            tid = self.bid.get(key)
            if tid is not None:
                self.blocks[tid] += c * A.blocks[aid]
            else:
                self._append_block(A.bqn[aid], A.bqi[aid], A.bqd[aid], c * A.blocks[aid])

    def inner_product(self, A: "QTensor") -> float:
        """``inner_product`` (:1161-1179): sum over this tensor's blocks present in A."""
        res = 0.0
        for key, tid in self.bid.items():
            aid = A.bid.get(key)
            if aid is not None:
                res += float(np.sum(self.blocks[tid] * A.blocks[aid]))
        return res

    def contract(self, A: "QTensor") -> float:
        """``contract`` (:1095-1119): full contraction over blocks common to both."""
        return self.inner_product(A)

    def total_size(self) -> int:
        return int(sum(b.size for b in self.blocks))


def _tag(ix: QIndex):
    return ix.tag()


def contract(A: QTensor, B: QTensor) -> QTensor:
    """``qtensor::operator*`` (qtensor/qtensor.cpp:523-734), restated step by step.

    Output blocks are created for every (left tuple, right tuple) with equal
    mid-QN -- also when no block pair contributes (:689-694) -- in the order
    mid-QN ascending, right tuple ascending, left tuple ascending.
    """
    assert A.initted or B.initted
    if A.initted and not B.initted:
        return A.copy()
    if B.initted and not A.initted:
        return B.copy()
    marker: Dict[tuple, int] = {}
    pairs: List[Tuple[int, int]] = []
    for i, ix in enumerate(A.idx):
        marker[_tag(ix)] = i
    for i, ix in enumerate(B.idx):
        tp = ix.dagged()
        if _tag(tp) not in marker:
            marker[_tag(ix)] = i
        else:
            pairs.append((marker[_tag(tp)], i))
            marker[_tag(tp)] = -1
            marker[_tag(ix)] = -1
    A_perm = [i for i in range(A.rank) if marker[_tag(A.idx[i])] != -1] + [p[0] for p in pairs]
    B_perm = [p[1] for p in pairs] + [i for i in range(B.rank) if marker[_tag(B.idx[i])] != -1]
    Aix = [A.idx[p] for p in A_perm]
    Bix = [B.idx[p] for p in B_perm]
    nrep = len(pairs)
    nA = A.rank - nrep

    A_bid = {tuple(A.bqn[i][A_perm[j]] for j in range(A.rank)): i for i in range(len(A.blocks))}
    B_bid = {tuple(B.bqn[i][B_perm[j]] for j in range(B.rank)): i for i in range(len(B.blocks))}

    res = QTensor(Aix[:nA] + Bix[nrep:])
    res.initted = True
    mid_set = set()
    left_qi: Dict[QN, set] = {}
    mid_qi: Dict[QN, set] = {}
    right_qi: Dict[QN, set] = {}
    for i in range(len(A.blocks)):
        m = QZERO
        lq = []
        for j in range(nA):
            lq.append(A.bqi[i][A_perm[j]])
            q = A.bqn[i][A_perm[j]]
            m = qadd(m, q) if Aix[j].arrow == Inward else qsub(m, q)
        mid_set.add(m)
        left_qi.setdefault(m, set()).add(tuple(lq))
    for i in range(len(B.blocks)):
        m = QZERO
        rq = []
        for j in range(nrep, B.rank):
            rq.append(B.bqi[i][B_perm[j]])
            q = B.bqn[i][B_perm[j]]
            m = qsub(m, q) if Bix[j].arrow == Inward else qadd(m, q)
        mq = tuple(B.bqi[i][B_perm[j]] for j in range(nrep))
        right_qi.setdefault(m, set()).add(tuple(rq))
        mid_qi.setdefault(m, set()).add(mq)

    a_axes = [A_perm[nA + t] for t in range(nrep)]
    b_axes = [B_perm[t] for t in range(nrep)]
    for m in sorted(mid_set):
        for rq in sorted(right_qi.get(m, ())):
            for lq in sorted(left_qi.get(m, ())):
                qi = tuple(lq) + tuple(rq)
                qd = tuple(Aix[t].qdim(lq[t]) for t in range(nA)) + \
                    tuple(Bix[nrep + t].qdim(rq[t]) for t in range(len(rq)))
                qns = tuple(Aix[t].qn(lq[t]) for t in range(nA)) + \
                    tuple(Bix[nrep + t].qn(rq[t]) for t in range(len(rq)))
                C = np.zeros(qd, dtype=np.float64)
                for mq in sorted(mid_qi.get(m, ())):
                    akey = qns[:nA] + tuple(Aix[nA + t].qn(mq[t]) for t in range(nrep))
                    bkey = tuple(Bix[t].qn(mq[t]) for t in range(nrep)) + qns[nA:]
                    ai = A_bid.get(akey)
                    bi = B_bid.get(bkey)
                    if ai is not None and bi is not None:
                        C += np.tensordot(A.blocks[ai], B.blocks[bi], axes=(a_axes, b_axes))
                res._append_block(qns, qi, qd, C)
    return res


def flops_of_contract(A: QTensor, B: QTensor) -> int:
    """Sum of 2*m*n*k over the block pairs ``contract`` multiplies (:714-722)."""
    total = 0
    marker: Dict[tuple, int] = {}
    pairs = []
    for i, ix in enumerate(A.idx):
        marker[_tag(ix)] = i
    for i, ix in enumerate(B.idx):
        tp = ix.dagged()
        if _tag(tp) not in marker:
            marker[_tag(ix)] = i
        else:
            pairs.append((marker[_tag(tp)], i))
            marker[_tag(tp)] = -1
            marker[_tag(ix)] = -1
    a_ax = [p[0] for p in pairs]
    b_ax = [p[1] for p in pairs]
    b_by_mid: Dict[tuple, List[int]] = {}
    for j in range(len(B.blocks)):
        b_by_mid.setdefault(tuple(B.bqn[j][t] for t in b_ax), []).append(j)
    for i in range(len(A.blocks)):
        key = tuple(A.bqn[i][t] for t in a_ax)
        for j in b_by_mid.get(key, ()):
            m = A.blocks[i].size
            k = int(np.prod([A.bqd[i][t] for t in a_ax])) if a_ax else 1
            n = B.blocks[j].size // k
            total += 2 * (m // k) * n * k
    return total


def to_dense(T: QTensor) -> np.ndarray:
    """Scatter the blocks into a dense array over the full index dimensions."""
    offs = []
    for ix in T.idx:
        o, acc = [], 0
        for _, d in ix.qns:
            o.append(acc)
            acc += d
        offs.append(o)
    out = np.zeros([ix.dim() for ix in T.idx])
    for b, qi in zip(T.blocks, T.bqi):
        sl = tuple(slice(offs[j][qi[j]], offs[j][qi[j]] + b.shape[j]) for j in range(T.rank))
        out[sl] += b
    return out


def deepcopy(T: QTensor) -> QTensor:
    return _copy.deepcopy(T)
