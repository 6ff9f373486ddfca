"""Exact diagonalisation known answers for spin-1/2 chains.

TEST INFRASTRUCTURE ONLY -- pins the DMRG oracle (``oracle/qdmrg.py``,
``oracle/ddmrg.py``) with exact ground energies in a fixed total-Sz sector.
The reference has no test suite or golden vectors for this path; these
energies are the known answers the restatement is checked against.

H = sum_bonds J (Sx Sx + Sy Sy + delta Sz Sz) + sum_i h_i Sz_i, built as a
sparse matrix over the basis states with the requested number of up spins.
"""
from __future__ import annotations

from itertools import combinations
from typing import List, Optional, Sequence, Tuple

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def sector_basis(L: int, n_up: int) -> np.ndarray:
    states = []
    for ups in combinations(range(L), n_up):
        s = 0
        for u in ups:
            s |= 1 << u
        states.append(s)
    return np.array(sorted(states), dtype=np.int64)


def xxz_hamiltonian(L: int, bonds: Sequence[Tuple[int, int, float]], n_up: int,
                    delta: float = 1.0, h: Optional[Sequence[float]] = None):
    basis = sector_basis(L, n_up)
    index = {int(s): i for i, s in enumerate(basis)}
    rows, cols, vals = [], [], []
    for a, s in enumerate(basis):
        s = int(s)
        diag = 0.0
        for (i, j, J) in bonds:
            si = 0.5 if (s >> i) & 1 else -0.5
            sj = 0.5 if (s >> j) & 1 else -0.5
            diag += J * delta * si * sj
            if si != sj:
                t = s ^ ((1 << i) | (1 << j))
                rows.append(index[t])
                cols.append(a)
                vals.append(0.5 * J)
        if h is not None:
            for i in range(L):
                diag += h[i] * (0.5 if (s >> i) & 1 else -0.5)
        rows.append(a)
        cols.append(a)
        vals.append(diag)
    n = len(basis)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def ground_energy(L: int, bonds: Sequence[Tuple[int, int, float]], n_up: Optional[int] = None,
                  delta: float = 1.0, h: Optional[Sequence[float]] = None) -> float:
    if n_up is None:
        n_up = L // 2
    H = xxz_hamiltonian(L, bonds, n_up, delta, h)
    if H.shape[0] <= 400:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    w = spla.eigsh(H, k=1, which="SA", tol=1e-14, maxiter=100000)[0]
    return float(w[0])


def chain_bonds(L: int, J: float = 1.0) -> List[Tuple[int, int, float]]:
    return [(i, i + 1, J) for i in range(L - 1)]


_OP_ACTION = {
    # op -> {ket bit: (bra bit, amplitude)} for spin-1/2 (Dn = 0, Up = 1)
    "Id": {0: (0, 1.0), 1: (1, 1.0)},
    "Sz": {0: (0, -0.5), 1: (1, 0.5)},
    "Sx": {0: (1, 0.5), 1: (0, 0.5)},
    "S+": {0: (1, 1.0)},
    "S-": {1: (0, 1.0)},
}


def terms_hamiltonian(L: int, terms, n_up: Optional[int] = None):
    """Sparse H = sum_t coef_t prod_j op_j(site_j) for terms given as
    (coef, ((site, op), ...)); over the full 2^L space, or the sector with
    n_up up spins when every term conserves Sz."""
    basis = np.arange(2 ** L, dtype=np.int64) if n_up is None else sector_basis(L, n_up)
    index = {int(s): i for i, s in enumerate(basis)}
    rows, cols, vals = [], [], []
    for a, s in enumerate(basis):
        s = int(s)
        for coef, ops in terms:
            t, amp = s, coef
            for i, op in reversed(ops):
                act = _OP_ACTION[op].get((t >> i) & 1)
                if act is None:
                    amp = 0.0
                    break
                t = (t & ~(1 << i)) | (act[0] << i)
                amp *= act[1]
            if amp == 0.0:
                continue
            if t not in index:
                raise ValueError("term leaves the Sz sector")
            rows.append(index[t])
            cols.append(a)
            vals.append(amp)
    n = len(basis)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def terms_ground_energy(L: int, terms, n_up: Optional[int] = None) -> float:
    H = terms_hamiltonian(L, terms, n_up)
    if H.shape[0] <= 400:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    return float(spla.eigsh(H, k=1, which="SA", tol=1e-14, maxiter=100000)[0][0])
