"""CPU restatement of tensor-tools' AutoMPO, lattices and AutoMPO -> MPO builders.

TEST INFRASTRUCTURE ONLY -- the parity oracle; see ``oracle/qtensor.py``.

Follows:
* term accumulator (operators kept in site order, zero coefficients dropped,
  repeated operator lists summed, terms ordered by operator list):
  models/hams/AutoMPO.cpp:178-201, 247-257, 366-393;
* lattices: models/lattice/square.h:25-103, models/lattice/triangular.h:25-64
  (1-based sites, y fastest);
* finite-state MPO construction: models/hams/Heisenberg.cpp:213-330 (dense)
  and :412-635 (qMPO).  As in the build, a string state sits only on the
  links its term crosses, states inside a charge sector are ordered IL, HL,
  then by first operator, a string's link charge is the divergence of its
  first operator, and coincident elements are summed.  None of this changes
  the operator: the checks pin it against exact diagonalisation.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from .qtensor import QIndex, QTensor, Inward, Outward, Link, Site, qn
from .qdmrg import QMPO, SPIN_PHY_QN, spin_op
from .ddmrg import DIndex, DTensor, DMPO

SPIN_DIV = {"Sz": 0, "Id": 0, "I": 0, "S+": 2, "Sp": 2, "S-": -2, "Sm": -2}


class AutoMPO:
    """AutoMPO::add / Accumulator semantics over a dict keyed by operator list."""

    def __init__(self):
        self._terms: Dict[Tuple[Tuple[int, str], ...], float] = {}

    def add(self, *args):
        """``add(coef, "S+", i, "S-", j)``: numbers before an operator name
        multiply the coefficient, the int after a name is its site."""
        coef, ops, pending = 1.0, [], None
        for a in args:
            if isinstance(a, str):
                if pending is not None:
                    raise ValueError("Invalid input to AutoMPO (two strings in a row?)")
                pending = a
            elif pending is not None:
                i = int(a)
                k = 0
                while k < len(ops) and ops[k][0] <= i:
                    k += 1
                ops.insert(k, (i, pending))
                pending = None
            else:
                coef *= float(a)
        if pending is not None:
            raise ValueError("Invalid input to AutoMPO (missing site number?)")
        if not ops:
            raise ValueError("No operators in HTerm")
        if coef == 0.0:
            return
        key = tuple(ops)
        self._terms[key] = self._terms.get(key, 0.0) + coef

    def terms(self) -> List[Tuple[float, Tuple[Tuple[int, str], ...]]]:
        """(coef, ((site, op), ...)) in LessNoCoef order: length, then (site, op)."""
        keys = sorted(self._terms, key=lambda k: (len(k), k))
        return [(self._terms[k], k) for k in keys]


def square_lattice(Nx: int, Ny: int, yperiodic: bool = False):
    yperiodic = yperiodic and Ny > 2
    out = []
    for n in range(1, Nx * Ny + 1):
        x, y = (n - 1) // Ny + 1, (n - 1) % Ny + 1
        if x < Nx:
            out.append((n, n + Ny, 0, x, y, x + 1, y))
        if Ny > 1:
            if y < Ny:
                out.append((n, n + 1, 0, x, y, x, y + 1))
            if yperiodic and y == 1:
                out.append((n, n + Ny - 1, 0, x, y, x, y + Ny))
    assert len(out) == 2 * Nx * Ny - Ny + (0 if yperiodic else -Nx)
    return out


def square_next_neighbor(Nx: int, Ny: int, yperiodic: bool = False):
    yperiodic = yperiodic and Ny > 2
    out = []
    for n in range(1, Nx * Ny + 1):
        x, y = (n - 1) // Ny + 1, (n - 1) % Ny + 1
        if x < Nx:
            out.append((n, n + Ny, 1, x, y, x + 1, y))
        if Ny > 1:
            if y < Ny:
                out.append((n, n + 1, 1, x, y, x, y + 1))
            if yperiodic and y == 1:
                out.append((n, n + Ny - 1, 1, x, y, x, y + Ny))
        if x < Nx and Ny > 1:
            if y < Ny:
                out.append((n, n + Ny + 1, 2, x, y, x + 1, y + 1))
            if y > 1:
                out.append((n, n + Ny - 1, 2, x, y, x + 1, y - 1))
            if yperiodic and y == Ny:
                out.append((n, n + 1, 2, x, Ny, x + 1, 1))
            if yperiodic and y == 1:
                out.append((n, n + 2 * Ny - 1, 2, x, 1, x + 1, Ny))
    return out


def snake_relabel(bonds, Nx: int, Ny: int):
    """Bonds of a column-major square lattice (site n = (x-1) Ny + y, the
    reference's numbering, models/lattice/square.h:25-103) relabelled to snake
    order: column x runs y = 1..Ny when x is odd and Ny..1 when x is even.
    Coordinates and types are kept; the smaller site comes first.  The
    reference has no snake order; the configuration of the J1-J2 cylinder
    asks for it."""
    def snake(n):
        x, y = (n - 1) // Ny + 1, (n - 1) % Ny + 1
        return (x - 1) * Ny + (y if x % 2 == 1 else Ny + 1 - y)
    out = []
    for s1, s2, t, x1, y1, x2, y2 in bonds:
        a, b = snake(s1), snake(s2)
        if a > b:
            a, b, x1, y1, x2, y2 = b, a, x2, y2, x1, y1
        out.append((a, b, t, x1, y1, x2, y2))
    return out


def triangular_lattice(Nx: int, Ny: int, yperiodic: bool = True):
    yperiodic = yperiodic and Ny > 2
    N = Nx * Ny
    out = []
    for n in range(1, N + 1):
        x, y = (n - 1) // Ny + 1, (n - 1) % Ny + 1
        if x < Nx:
            out.append((n, n + Ny, 0, 0, 0, 0, 0))
        if Ny > 1:
            if n + 1 <= N and (y < Ny or yperiodic):
                out.append((n, n + 1, 0, 0, 0, 0, 0))
            if yperiodic and y == 1:
                out.append((n, n + Ny - 1, 0, 0, 0, 0, 0))
            if x < Nx and y < Ny:
                out.append((n, n + Ny + 1, 0, 0, 0, 0, 0))
    assert len(out) == 3 * N - 2 * Ny + (0 if yperiodic else -2 * Nx + 1)
    return out


def links(ampo: AutoMPO, N: int, with_charges: bool):
    """Per link n: ordered states (kind, first_op, q) with kind 0 IL, 1 HL, 2 string."""
    for _, ops in ampo.terms():
        if len(ops) > 2:
            raise ValueError("terms with more than two operators are not supported")
        if len(ops) == 2 and ops[0][0] == ops[1][0]:
            raise ValueError("two operators on one site are not supported")
        for i, _ in ops:
            if not 0 <= i < N:
                raise ValueError("operator site out of range")
    basis = [[] for _ in range(N + 1)]
    for n in range(N + 1):
        if n < N:
            basis[n].append((0, None, 0))
        if n >= 1:
            basis[n].append((1, None, 0))
    for _, ops in ampo.terms():
        if len(ops) != 2:
            continue
        first = ops[0]
        q = SPIN_DIV[first[1]] if with_charges else 0
        for n in range(first[0] + 1, ops[1][0] + 1):
            if not any(s[0] == 2 and s[1] == first for s in basis[n]):
                basis[n].append((2, first, q))
    # zero charge first, then ascending; Python's sort is stable
    return [sorted(b, key=lambda s: (s[2] != 0, s[2])) for b in basis]


def _sectors(link):
    secs, pos = [], []
    for s in link:
        if not secs or secs[-1][0] != s[2]:
            secs.append([s[2], 0])
        pos.append(secs[-1][1])
        secs[-1][1] += 1
    return secs, pos


def _entries(ampo: AutoMPO, lk, i: int):
    """(row, col, op, value) rules of one site, in the build's order."""
    rows, cols = lk[i], lk[i + 1]
    out = []
    for r, rs in enumerate(rows):
        for c, cs in enumerate(cols):
            if cs[0] == 2 and cs[1][0] == i and rs[0] == 0:
                out.append((r, c, cs[1][1], 1.0))
            if rs[0] == cs[0] and (rs[0] != 2 or rs[1] == cs[1]):
                out.append((r, c, "Id", 1.0))
    il = [r for r, s in enumerate(rows) if s[0] == 0]
    hl = [c for c, s in enumerate(cols) if s[0] == 1]
    for coef, ops in ampo.terms():
        if ops[-1][0] != i:
            continue
        if len(ops) == 2:
            r = [k for k, s in enumerate(rows) if s[0] == 2 and s[1] == ops[0]][0]
            out.append((r, hl[0], ops[1][1], coef))
        else:
            out.append((il[0], hl[0], ops[0][1], coef))
    return out


def build_qmpo(ampo: AutoMPO, N: int, mid: int = 2) -> QMPO:
    lk = links(ampo, N, True)
    H = QMPO.__new__(QMPO)
    H.length, H.id, H.phy_qn, H.A = N, mid, list(SPIN_PHY_QN), []
    pref = "ID%dLink" % mid
    for i in range(N):
        T = QTensor([QIndex(Inward, pref + str(i), Link, 0),
                     QIndex(Outward, "Site" + str(i), Site, 0),
                     QIndex(Inward, "Site" + str(i), Site, 1),
                     QIndex(Outward, pref + str(i + 1), Link, 0)])
        lsec, lpos = _sectors(lk[i])
        rsec, rpos = _sectors(lk[i + 1])
        for q, d in lsec:
            T.idx[0].add_qn(qn(q), d)
        for p in H.phy_qn:
            T.idx[1].add_qn(p, 1)
        for p in H.phy_qn:
            T.idx[2].add_qn(p, 1)
        for q, d in rsec:
            T.idx[3].add_qn(qn(q), d)
        T.init_block()
        for r, c, op, val in _entries(ampo, lk, i):
            for k in range(2):
                for b in range(2):
                    v = val * spin_op(b, op, k)
                    if v == 0.0:
                        continue
                    key = (qn(lk[i][r][2]), H.phy_qn[k], H.phy_qn[b], qn(lk[i + 1][c][2]))
                    if key not in T.bid:
                        raise ValueError("term %s does not conserve the U(1) charge" % op)
                    T.blocks[T.bid[key]][lpos[r], 0, 0, rpos[c]] += v
        H.A.append(T)
    return H


def build_dmpo(ampo: AutoMPO, N: int, mid: int = 2) -> DMPO:
    lk = links(ampo, N, False)
    H = DMPO.__new__(DMPO)
    H.length, H.id, H.A = N, mid, []
    for i in range(N):
        dl, dr = len(lk[i]), len(lk[i + 1])
        W = np.zeros((dl, 2, 2, dr))
        for r, c, op, val in _entries(ampo, lk, i):
            for k in range(2):
                for b in range(2):
                    W[r, k, b, c] += val * spin_op(b, op, k)
        idx = [DIndex(dl, "ID%dLink%d" % (mid, i)), DIndex(2, "Site%d" % i, Site, 0),
               DIndex(2, "Site%d" % i, Site, 1), DIndex(dr, "ID%dLink%d" % (mid, i + 1))]
        H.A.append(DTensor(idx, W))
    return H


def mpo_matrix(W: Sequence[np.ndarray]) -> np.ndarray:
    """Dense 2^N x 2^N operator of an MPO given as (left, ket, bra, right)
    arrays; row/column index = sum_i s_i 2^i (site 0 least significant),
    rows are bras.  Small N only."""
    acc = W[0][0]  # (ket0, bra0, right)
    kets, bras = 1, 1
    acc = acc.reshape(2, 2, -1)
    for A in W[1:]:
        # acc: (K, B, w) ; A: (w, k, b, w')
        acc = np.einsum("KBw,wkbv->kKbBv", acc, A)
        kets, bras = kets * 2, bras * 2
        acc = acc.reshape(acc.shape[0] * acc.shape[1], acc.shape[2] * acc.shape[3], -1)
    M = acc[:, :, 0]  # (ket, bra) with the last site most significant
    return M.T


def term_matrix(N: int, terms) -> np.ndarray:
    """Dense 2^N operator of sum_t coef_t prod_j op_j(site_j), same ordering."""
    def op1(op):
        return np.array([[spin_op(b, op, k) for k in range(2)] for b in range(2)])
    H = np.zeros((2 ** N, 2 ** N))
    for coef, ops in terms:
        mats = [np.eye(2)] * N
        for i, op in ops:
            mats = list(mats)
            mats[i] = op1(op) @ mats[i]
        M = np.array([[1.0]])
        for i in range(N):
            M = np.kron(mats[i], M)
        H += coef * M
    return H
