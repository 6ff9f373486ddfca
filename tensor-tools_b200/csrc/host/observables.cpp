// Overlaps, MPO expectation values and Sz correlators (qMPS and dense MPS).
#include "observables.h"

#include <stdexcept>

namespace ttb {

namespace {

tt_ctx* bound_ctx() {
  if (!rt().ctx) throw std::runtime_error("observables: no device context bound");
  return rt().ctx;
}

// psi_i^dagger with its link indices primed (t1 of mps/observables.cpp:386,419)
qtensor bra_tensor(const qtensor& A) {
  qtensor t = A;
  t.dag();
  for (auto& ix : t.idx_set)
    if (ix.type() == Link) ix.prime();
  return t;
}

// ones over (a, b), daggered: the closing tensors of observables.cpp:423-428,432-437
qtensor ends(const qtensor_index& a, const qtensor_index& b) {
  qtensor e({a, b});
  e.initBlock();
  e.setOne();
  e.dag();
  return e;
}

int site_axis(const qtensor& A) {
  for (unsigned k = 0; k < A.rank; ++k)
    if (A.idx_set[k].type() == Site) return (int)k;
  throw std::runtime_error("measure_sz: MPS tensor without a site index");
}

// Sz applied to the physical mode: every block carries one spin sector of
// dimension 1, so Sz is a constant factor (2Sz / 2) per block.
qtensor apply_sz(const qtensor& A) {
  qtensor t = A;
  int s = site_axis(A);
  for (unsigned b = 0; b < t.blocks.size(); ++b) {
    const BlockMeta& bm = t.blocks[b];
    if (bm.qd[s] != 1) throw std::runtime_error("measure_sz: spin-1/2 sites expected");
    double f = 0.5 * (double)bm.qn[s].a;
    check(tt_vec_scale_mode(bound_ctx(), bm.size, 1, 1, &f, t.block_ptr(b)), "apply Sz");
  }
  return t;
}

void check_pair(unsigned La, unsigned Lb) {
  if (La != Lb || La < 2) throw std::runtime_error("observables: length mismatch");
}

}  // namespace

double psiphi(const qMPS& psi, const qMPS& phi) {
  // mps/observables.cpp:415-450
  check_pair(psi.length, phi.length);
  qtensor acc;
  double res = 0.0;
  for (unsigned i = 0; i < psi.length; ++i) {
    qtensor t1 = bra_tensor(psi.A[i]);
    const qtensor& t2 = phi.A[i];
    if (i == 0) {
      acc = (ends(t1.idx_set[0], t2.idx_set[0]) * t1) * t2;
    } else {
      acc = (t1 * acc) * t2;
    }
    if (i == psi.length - 1) res = acc.contract(ends(t1.idx_set.back(), t2.idx_set.back()));
  }
  return res;
}

double psiHphi(const qMPS& psi, const qMPO& H, const qMPS& phi) {
  // mps/observables.cpp:64-103
  check_pair(psi.length, phi.length);
  check_pair(psi.length, H.length);
  qtensor acc;
  double res = 0.0;
  for (unsigned i = 0; i < psi.length; ++i) {
    qtensor t1 = psi.A[i];
    t1.dag();
    t1.prime();
    const qtensor& t2 = H.A[i];
    const qtensor& t3 = phi.A[i];
    if (i == 0) {
      qtensor le({t1.idx_set[0], t2.idx_set[0], t3.idx_set[0]});
      le.initBlock();
      le.setOne();
      le.dag();
      acc = ((le * t1) * t2) * t3;
    } else {
      acc = ((acc * t1) * t2) * t3;
    }
    if (i == psi.length - 1) {
      qtensor re({t1.idx_set.back(), t2.idx_set.back(), t3.idx_set.back()});
      re.initBlock();
      re.setOne();
      re.dag();
      res = acc.contract(re);
    }
  }
  return res;
}

void measure_sz(const qMPS& psi, std::vector<double>& sz, std::vector<double>& szsz) {
  const unsigned L = psi.length;
  if (L < 2) throw std::runtime_error("measure_sz: need at least two sites");
  std::vector<qtensor> bra(L), zket(L);
  for (unsigned i = 0; i < L; ++i) {
    bra[i] = bra_tensor(psi.A[i]);
    zket[i] = apply_sz(psi.A[i]);
  }
  // EL[i]: sites < i contracted (bond i); ER[i]: sites >= i contracted (bond i)
  std::vector<qtensor> EL(L + 1), ER(L + 1);
  EL[0] = ends(bra[0].idx_set[0], psi.A[0].idx_set[0]);
  for (unsigned i = 0; i < L; ++i) EL[i + 1] = (bra[i] * EL[i]) * psi.A[i];
  ER[L] = ends(bra[L - 1].idx_set.back(), psi.A[L - 1].idx_set.back());
  for (unsigned i = L; i-- > 0;) ER[i] = (bra[i] * ER[i + 1]) * psi.A[i];
  double nrm2 = EL[L].contract(ER[L]);
  if (!(nrm2 > 0.0)) throw std::runtime_error("measure_sz: <psi|psi> is not positive");
  sz.assign(L, 0.0);
  szsz.assign((size_t)L * L, 0.0);
  for (unsigned i = 0; i < L; ++i) {
    qtensor C = (bra[i] * EL[i]) * zket[i];
    sz[i] = C.contract(ER[i + 1]) / nrm2;
    szsz[(size_t)i * L + i] = 0.25;
    for (unsigned j = i + 1; j < L; ++j) {
      qtensor D = bra[j] * C;
      double v = (D * zket[j]).contract(ER[j + 1]) / nrm2;
      szsz[(size_t)i * L + j] = v;
      szsz[(size_t)j * L + i] = v;
      if (j + 1 < L) C = D * psi.A[j];
    }
  }
}

// ---- dense MPS ------------------------------------------------------------------
namespace {

tt_ctx* dense_ctx() {
  if (!rt().ctx) throw std::runtime_error("observables: no device context bound");
  return rt().ctx;
}

dtensor dbra(const dtensor& A) {
  dtensor t = A;
  for (auto& ix : t.idx_set)
    if (ix.type == Link) ix.prime();
  return t;
}

dtensor dends(const dtensor_index& a, const dtensor_index& b) {
  dtensor e({a, b});
  e.setOne();
  return e;
}

dtensor dapply_sz(const dtensor& A) {
  dtensor t = A;
  int s = -1;
  for (unsigned k = 0; k < t.rank; ++k)
    if (t.idx_set[k].type == Site) s = (int)k;
  if (s < 0 || t.idx_set[s].size != 2) throw std::runtime_error("measure_sz: spin-1/2 site index expected");
  int64_t inner = 1, outer = 1;
  for (int k = 0; k < s; ++k) inner *= t.idx_set[k].size;
  for (unsigned k = s + 1; k < t.rank; ++k) outer *= t.idx_set[k].size;
  const double f[2] = {-0.5, 0.5};  // Dn, Up
  check(tt_vec_scale_mode(dense_ctx(), inner, 2, outer, f, t.data->get()), "apply Sz");
  return t;
}

}  // namespace

double psiphi(const MPS& psi, const MPS& phi) {
  // mps/observables.cpp:382-413
  check_pair(psi.length, phi.length);
  dtensor acc;
  double res = 0.0;
  for (unsigned i = 0; i < psi.length; ++i) {
    dtensor t1 = dbra(psi.A[i]);
    const dtensor& t2 = phi.A[i];
    if (i == 0)
      acc = (dends(t1.idx_set[0], t2.idx_set[0]) * t1) * t2;
    else
      acc = (t1 * acc) * t2;
    if (i == psi.length - 1) res = acc.inner_product(dends(t1.idx_set.back(), t2.idx_set.back()));
  }
  return res;
}

double psiHphi(const MPS& psi, const MPO& H, const MPS& phi) {
  // mps/observables.cpp:25-62
  check_pair(psi.length, phi.length);
  check_pair(psi.length, H.length);
  dtensor acc;
  double res = 0.0;
  for (unsigned i = 0; i < psi.length; ++i) {
    dtensor t1 = psi.A[i];
    t1.prime();
    const dtensor& t2 = H.A[i];
    const dtensor& t3 = phi.A[i];
    if (i == 0) {
      dtensor le({t1.idx_set[0], t2.idx_set[0], t3.idx_set[0]});
      le.setOne();
      acc = ((le * t1) * t2) * t3;
    } else {
      acc = ((acc * t1) * t2) * t3;
    }
    if (i == psi.length - 1) {
      dtensor re({t1.idx_set.back(), t2.idx_set.back(), t3.idx_set.back()});
      re.setOne();
      res = acc.inner_product(re);
    }
  }
  return res;
}

void measure_sz(const MPS& psi, std::vector<double>& sz, std::vector<double>& szsz) {
  const unsigned L = psi.length;
  if (L < 2) throw std::runtime_error("measure_sz: need at least two sites");
  std::vector<dtensor> bra(L), zket(L);
  for (unsigned i = 0; i < L; ++i) {
    bra[i] = dbra(psi.A[i]);
    zket[i] = dapply_sz(psi.A[i]);
  }
  std::vector<dtensor> EL(L + 1), ER(L + 1);
  EL[0] = dends(bra[0].idx_set[0], psi.A[0].idx_set[0]);
  for (unsigned i = 0; i < L; ++i) EL[i + 1] = (bra[i] * EL[i]) * psi.A[i];
  ER[L] = dends(bra[L - 1].idx_set.back(), psi.A[L - 1].idx_set.back());
  for (unsigned i = L; i-- > 0;) ER[i] = (bra[i] * ER[i + 1]) * psi.A[i];
  double nrm2 = EL[L].inner_product(ER[L]);
  if (!(nrm2 > 0.0)) throw std::runtime_error("measure_sz: <psi|psi> is not positive");
  sz.assign(L, 0.0);
  szsz.assign((size_t)L * L, 0.0);
  for (unsigned i = 0; i < L; ++i) {
    dtensor C = (bra[i] * EL[i]) * zket[i];
    sz[i] = C.inner_product(ER[i + 1]) / nrm2;
    szsz[(size_t)i * L + i] = 0.25;
    for (unsigned j = i + 1; j < L; ++j) {
      dtensor D = bra[j] * C;
      double v = (D * zket[j]).inner_product(ER[j + 1]) / nrm2;
      szsz[(size_t)i * L + j] = v;
      szsz[(size_t)j * L + i] = v;
      if (j + 1 < L) C = D * psi.A[j];
    }
  }
}

}  // namespace ttb
