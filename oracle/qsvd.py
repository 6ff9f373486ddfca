"""CPU restatement of tensor-tools' block SVD with truncation (``svd``/``svd_bond``).

TEST INFRASTRUCTURE ONLY -- the parity oracle; see ``oracle/qtensor.py``.

Follows qtensor/qtensor_op.cpp:1097-1453 (``svd``) and :1506-1544
(``svd_bond(combined, ...)``).  The per-sector SVD is LAPACK ``dgesvd``
(scipy), standing in for CTF's ScaLAPACK ``pdgesvd`` (:1269); the 1x2
workaround of :1247-1267 is kept.  Sorting of singular values breaks ties by
(sector, position), where the reference's ``std::sort`` (:1290) leaves them
unspecified.
"""
from __future__ import annotations

from typing import List

import numpy as np
import scipy.linalg as sla

from .qtensor import QIndex, QTensor, Inward, Outward, qadd, qsub, QZERO

MoveFromLeft, MoveFromRight = 0, 1


class TruncInfo:
    def __init__(self):
        self.trunc_err = 0.0
        self.kept = 0
        self.kept_per_sector = []
        self.sector_qn = []
        self.svals = []
        # how close the cut came to going the other way: the relative gap
        # between the last kept and the first dropped singular value, and the
        # relative margin of the discarded weight against the cutoff
        self.cut_gap = float("inf")
        self.cutoff_margin = float("inf")


def find_index_permutation(frm: List[QIndex], to: List[QIndex]) -> List[int]:
    """qtensor/qtensor_index_op.cpp:23-37."""
    perm = []
    for t in to:
        for j, f in enumerate(frm):
            if t == f:
                perm.append(j)
                break
    assert len(perm) == len(to)
    return perm


def _sector_svd(mA: np.ndarray, K: int):
    """CTF Matrix::svd(U,S,V,K,0) stand-in: rank-K thin SVD via dgesvd."""
    U, s, Vt = sla.svd(mA, full_matrices=False, lapack_driver="gesvd")
    if K and K < s.size:
        U, s, Vt = U[:, :K], s[:K], Vt[:K, :]
    return U, s, Vt


def svd(A: QTensor, left: List[QIndex], right: List[QIndex], direction: int,
        cutoff: float = 0.0, K: int = 0, info: TruncInfo | None = None):
    """qtensor/qtensor_op.cpp:1097-1453; returns (U, V, S)."""
    new_idx = list(left) + list(right)
    perm = find_index_permutation(A.idx, new_idx)
    A_bid = {tuple(A.bqn[i][perm[j]] for j in range(A.rank)): i for i in range(len(A.blocks))}
    mid_set = set()
    l_qi, r_qi = {}, {}
    nl = len(left)
    for i in range(len(A.blocks)):
        m = QZERO
        lq, rq = [], []
        for j in range(nl):
            q = A.bqn[i][perm[j]]
            m = qadd(m, q) if left[j].arrow == Inward else qsub(m, q)
            lq.append(A.bqi[i][perm[j]])
        for j in range(len(right)):
            rq.append(A.bqi[i][perm[j + nl]])
        mid_set.add(m)
        l_qi.setdefault(m, set()).add(tuple(lq))
        r_qi.setdefault(m, set()).add(tuple(rq))
    mid_Q = sorted(mid_set)
    l_keys, l_sizes, r_keys, r_sizes = {}, {}, {}, {}
    mid_dim = []
    for q in mid_Q:
        l_keys[q], l_sizes[q], r_keys[q], r_sizes[q] = [], [], [], []
        for lq in sorted(l_qi[q]):
            l_keys[q].append(tuple(left[j].qn(lq[j]) for j in range(nl)))
            l_sizes[q].append(int(np.prod([left[j].qdim(lq[j]) for j in range(nl)])))
        for rq in sorted(r_qi[q]):
            r_keys[q].append(tuple(right[j].qn(rq[j]) for j in range(len(right))))
            r_sizes[q].append(int(np.prod([right[j].qdim(rq[j]) for j in range(len(right))])))
        mid_dim.append(min(sum(l_sizes[q]), sum(r_sizes[q])))

    mU, mV, mS = [], [], []
    S_and_idx = []
    nm = 0.0
    for ii, q in enumerate(mid_Q):
        rows, cols = sum(l_sizes[q]), sum(r_sizes[q])
        mA = np.zeros((rows, cols))
        r0 = 0
        for i, lk in enumerate(l_keys[q]):
            c0 = 0
            for j, rk in enumerate(r_keys[q]):
                # missing combination would alias block 0 in the reference
                # (operator[] default-inserts 0, :1238); every DMRG x has them all
                b = A.blocks[A_bid[lk + rk]]
                mA[r0:r0 + l_sizes[q][i], c0:c0 + r_sizes[q][j]] = \
                    b.reshape(l_sizes[q][i], r_sizes[q][j], order="F")
                c0 += r_sizes[q][j]
            r0 += l_sizes[q][i]
        if rows == 1 and cols == 2:  # ScaLAPACK workaround, :1247-1267
            U = np.ones((1, 1))
            d = float(np.sqrt(np.sum(mA * mA)))
            s = np.array([d])
            Vt = mA / d if d != 0.0 else np.full((1, 2), 1.0 / np.sqrt(2.0))
        else:
            U, s, Vt = _sector_svd(mA, K)
        if direction == MoveFromLeft:
            Vt = s[:, None] * Vt
        else:
            U = U * s[None, :]
        mU.append(U)
        mV.append(Vt)
        mS.append(s)
        for j, sv in enumerate(s):
            S_and_idx.append((float(sv), ii, j))
            nm += float(sv) * float(sv)
    # global descending sort; ties broken by (sector, position)
    S_and_idx.sort(key=lambda t: (-t[0], t[1], t[2]))
    new_dim = [0] * len(mid_Q)
    cumsum = 0.0
    acc = 0
    prev_disc = 1.0
    for sv, ii, _ in S_and_idx:  # :1291-1300
        prev_disc = 1 - cumsum
        cumsum += sv * sv / nm
        if sv == 0.0 and cutoff != 0.0:
            break
        new_dim[ii] += 1
        acc += 1
        if (1 - cumsum < cutoff and cutoff != 0.0) or (acc >= K and K != 0):
            break
    if info is not None:
        if 0 < acc < len(S_and_idx) and S_and_idx[acc - 1][0] > 0.0:
            s_last, s_next = S_and_idx[acc - 1][0], S_and_idx[acc][0]
            info.cut_gap = (s_last - s_next) / s_last
        if cutoff != 0.0 and acc > 0:
            info.cutoff_margin = min(abs(prev_disc - cutoff), abs((1 - cumsum) - cutoff)) / cutoff
        info.trunc_err = max(1 - cumsum, 0.0)
        info.kept = acc
        info.kept_per_sector = [d for d in new_dim]
        info.sector_qn = list(mid_Q)
        info.svals = [s for s in mS]

    midCut = QIndex(Outward, "svdmid")
    for ii, q in enumerate(mid_Q):
        if new_dim[ii] > 0:
            midCut.add_qn(q, new_dim[ii])
    U_t = QTensor(list(left) + [midCut.copy()])
    V_t = QTensor([midCut.dagged()] + list(right))
    S_t = QTensor([midCut.copy()])
    U_t.initted = V_t.initted = S_t.initted = True
    mid_num = 0
    for ii, q in enumerate(mid_Q):
        nd = new_dim[ii]
        if nd == 0:
            continue
        r0 = 0
        for lq, lk, ls in zip(sorted(l_qi[q]), l_keys[q], l_sizes[q]):
            qd = tuple(left[j].qdim(lq[j]) for j in range(nl)) + (nd,)
            data = mU[ii][r0:r0 + ls, :nd].reshape(qd, order="F")
            U_t._append_block(lk + (q,), tuple(lq) + (mid_num,), qd, data.copy())
            r0 += ls
        c0 = 0
        for rq, rk, rs in zip(sorted(r_qi[q]), r_keys[q], r_sizes[q]):
            qd = (nd,) + tuple(right[j].qdim(rq[j]) for j in range(len(right)))
            data = mV[ii][:nd, c0:c0 + rs].reshape(qd, order="F")
            V_t._append_block((q,) + rk, (mid_num,) + tuple(rq), qd, data.copy())
            c0 += rs
        S_t._append_block((q,), (mid_num,), (nd,), mS[ii][:nd].copy())
        mid_num += 1
    return U_t, V_t, S_t


def svd_bond(combined: QTensor, A_left: QTensor, A_right: QTensor, mid: QIndex,
             direction: int, cutoff: float = 0.0, K: int = 0,
             info: TruncInfo | None = None):
    """qtensor/qtensor_op.cpp:1506-1544: returns (new A_left, new A_right, S)."""
    dag_mid = mid.dagged()
    left = [ix for ix in A_left.idx if ix.tag() != mid.tag()]
    right = [ix for ix in A_right.idx if ix.tag() != dag_mid.tag()]
    U, V, S = svd(combined, left, right, direction, cutoff, K, info)
    u = U.idx[-1]
    u.name, u.type, u.level = mid.name, mid.type, mid.level
    v = V.idx[0]
    v.name, v.type, v.level = dag_mid.name, dag_mid.type, dag_mid.level
    return U, V, S


def calc_entropy(S: QTensor, cutoff: float = 1e-24) -> float:
    """calcEntropy (qtensor/qtensor.h:166-173): -sum s^2 ln s^2 over s > cutoff."""
    ent = 0.0
    for b in S.blocks:
        for sv in b.ravel():
            if sv > cutoff:
                ent += -(sv * sv) * np.log(sv * sv)
    return ent
