// Block SVD with truncation (qtensor/qtensor_op.cpp:1097-1453) and svd_bond
// (:1506-1544), as a density-matrix eigendecomposition on the GPU:
//
//   MoveFromLeft : rho_q = X_q X_q^T  -> U = eigenvectors,  V = U^T X_q (= S V^T)
//   MoveFromRight: rho_q = X_q^T X_q  -> V = eigenvectors,  U = X_q V   (= U S)
//
// so the side that must be orthonormal comes straight out of the FP64
// Jacobi eigensolver and the side that absorbs S is one grouped GEMM, as the
// reference absorbs S into V (left-to-right) or U (right-to-left) at
// :1274-1278.  Singular values are sqrt(|lambda|); the global sort and the
// discarded-weight rule of :1290-1300 run on the host over the few thousand
// values.  Ties are broken by (sector, position).  The 1x2 ScaLAPACK
// workaround of :1247-1267 is reproduced by the eigensolver's 1x2 mode.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>

#include "qtensor.h"

namespace ttb {

namespace {

tt_ctx* ctx() {
  if (!rt().ctx) throw std::runtime_error("ttb: no device context bound");
  return rt().ctx;
}

std::vector<int64_t> cm_strides(const std::vector<int>& qd) {
  std::vector<int64_t> s(qd.size(), 1);
  for (size_t i = 1; i < qd.size(); ++i) s[i] = s[i - 1] * qd[i - 1];
  return s;
}

// fill `n` modes of a pair from axis lists
struct Ax {
  int64_t dim, s1, s2;
};
int fill_modes(const std::vector<Ax>& ax, int32_t* dims, int64_t* st1, int64_t* st2) {
  std::vector<Ax> r;
  for (auto& a : ax)
    if (a.dim != 1) {
      if (!r.empty() && a.s1 == r.back().s1 * r.back().dim && (!st2 || a.s2 == r.back().s2 * r.back().dim)) {
        r.back().dim *= a.dim;
        continue;
      }
      r.push_back(a);
    }
  if (r.size() > TT_MAX_MODES) throw std::runtime_error("svd: too many modes");
  for (size_t i = 0; i < r.size(); ++i) {
    dims[i] = (int32_t)r[i].dim;
    st1[i] = r[i].s1;
    if (st2) st2[i] = r[i].s2;
  }
  return (int)r.size();
}

struct Sector {
  QN q;
  std::vector<std::vector<unsigned>> lq, rq;  // tuples in set order
  std::vector<int64_t> lsz, rsz, loff, roff;  // sizes and offsets inside the sector matrix
  int64_t rows = 0, cols = 0;
  int64_t g = 0;        // Gram dimension
  int64_t g_off = 0, w_off = 0;
  int nvals = 0;        // singular values returned by the per-sector SVD
  int keep = 0;
};

// rho_q += weight / tr(P P^T) * (P P^T)_q over the sectors of the decomposition
void add_noise(const NoiseTerm& nz, const std::vector<Sector>& sec, const std::vector<qtensor_index>& left,
               const std::vector<qtensor_index>& right, int direction, int64_t gtot, const DevPtr& G) {
  const qtensor& P = *nz.P;
  const std::vector<qtensor_index>& side = direction == MoveFromLeft ? left : right;
  const unsigned ns = (unsigned)side.size();
  // the axes of P that carry the kept side's indices (matched by name and type)
  std::vector<int> row_ax(ns, -1);
  for (unsigned j = 0; j < ns; ++j)
    for (unsigned a = 0; a < P.rank; ++a)
      if (P.idx_set[a].name() == side[j].name() && P.idx_set[a].type() == side[j].type() &&
          P.idx_set[a].sectors() == side[j].sectors())
        row_ax[j] = (int)a;
  for (int a : row_ax)
    if (a < 0) throw std::runtime_error("svd noise: perturbation lacks an index of the kept side");
  std::vector<unsigned> col_ax;
  for (unsigned a = 0; a < P.rank; ++a)
    if (std::find(row_ax.begin(), row_ax.end(), (int)a) == row_ax.end()) col_ax.push_back(a);
  // blocks by (row tuple, column tuple)
  std::map<std::vector<unsigned>, std::map<std::vector<unsigned>, unsigned>> by_row;
  for (unsigned b = 0; b < P.blocks.size(); ++b) {
    std::vector<unsigned> rq, cq;
    for (int a : row_ax) rq.push_back(P.blocks[b].qi[a]);
    for (unsigned a : col_ax) cq.push_back(P.blocks[b].qi[a]);
    by_row[rq][cq] = b;
  }
  std::vector<tt_out_block> outs;
  std::vector<tt_block_pair> pairs;
  for (const Sector& s : sec) {
    if (s.g == 0 || (direction == MoveFromRight && s.rows == 1 && s.cols == 2)) continue;
    const auto& tup = direction == MoveFromLeft ? s.lq : s.rq;
    const auto& off = direction == MoveFromLeft ? s.loff : s.roff;
    const auto& sz = direction == MoveFromLeft ? s.lsz : s.rsz;
    for (size_t i = 0; i < tup.size(); ++i) {
      auto ri = by_row.find(tup[i]);
      if (ri == by_row.end()) continue;
      for (size_t j = 0; j < tup.size(); ++j) {
        auto rj = by_row.find(tup[j]);
        if (rj == by_row.end()) continue;
        int ob = -1;
        for (auto& kv : ri->second) {
          auto cj = rj->second.find(kv.first);
          if (cj == rj->second.end()) continue;
          const BlockMeta& bi = P.blocks[kv.second];
          const BlockMeta& bj = P.blocks[cj->second];
          if (ob < 0) {
            outs.push_back(tt_out_block{s.g_off + off[i] + s.g * off[j], (int32_t)sz[i], (int32_t)sz[j],
                                        (int32_t)s.g});
            ob = (int)outs.size() - 1;
          }
          auto si = cm_strides(bi.qd), sj = cm_strides(bj.qd);
          tt_block_pair p;
          std::memset(&p, 0, sizeof(p));
          p.out_block = ob;
          p.a_off = bi.off;
          p.b_off = bj.off;
          std::vector<Ax> ax;
          for (int a : row_ax) ax.push_back({bi.qd[a], si[a], 0});
          p.n_m = fill_modes(ax, p.m_dims, p.a_m_stride, nullptr);
          ax.clear();
          for (unsigned a : col_ax) ax.push_back({bi.qd[a], si[a], sj[a]});
          p.n_k = fill_modes(ax, p.k_dims, p.a_k_stride, p.b_k_stride);
          ax.clear();
          for (int a : row_ax) ax.push_back({bj.qd[a], sj[a], 0});
          p.n_n = fill_modes(ax, p.n_dims, p.b_n_stride, nullptr);
          pairs.push_back(p);
        }
      }
    }
  }
  if (outs.empty()) return;
  // rho_P written block by block into a zeroed buffer of the same layout as G
  DevPtr GP = dev_alloc(gtot);
  GP->zero();
  validate_pairs(outs, pairs, P.arena, P.arena, gtot);
  tt_plan* plan = nullptr;
  check(tt_contract_plan(ctx(), outs.data(), (int)outs.size(), pairs.data(), (int)pairs.size(), TT_PREC_FP64,
                         &plan),
        "svd noise plan");
  PlanHandle ph(plan);
  check(tt_contract_exec(ctx(), plan, P.data->get(), P.data->get(), GP->get(), 1.0), "svd noise gram");
  // tr(rho_P): the diagonals of its sector blocks
  std::vector<tt_copy_desc> diag;
  int64_t nd = 0;
  for (const Sector& s : sec) {
    if (s.g == 0) continue;
    tt_copy_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_modes = 1;
    d.dims[0] = (int32_t)s.g;
    d.src_off = s.g_off;
    d.src_stride[0] = s.g + 1;
    d.dst_off = nd;
    d.dst_stride[0] = 1;
    diag.push_back(d);
    nd += s.g;
  }
  DevPtr D = dev_alloc(std::max<int64_t>(nd, 2));
  D->zero();
  check(tt_strided_copy_batched(ctx(), diag.data(), (int)diag.size(), GP->get(), D->get()), "svd noise trace");
  std::vector<double> dh((size_t)nd);
  check(tt_memcpy_d2h(ctx(), dh.data(), D->get(), sizeof(double) * dh.size()), "svd noise trace");
  double tr = 0.0;
  for (double v : dh) tr += v;
  if (!(tr > 0.0)) return;
  check(tt_vec_axpy(ctx(), gtot, nz.weight / tr, GP->get(), G->get()), "svd noise add");
}

}  // namespace

void svd(const qtensor& A, const std::vector<qtensor_index>& left,
         const std::vector<qtensor_index>& right, qtensor& U, qtensor& V, qtensor& S,
         int direction, double cutoff, unsigned K, TruncInfo* info, const NoiseTerm* noise) {
  S = qtensor();
  std::vector<qtensor_index> new_idx(left);
  new_idx.insert(new_idx.end(), right.begin(), right.end());
  std::vector<unsigned> perm = find_index_permutation(A.idx_set, new_idx);
  const unsigned nl = (unsigned)left.size(), nr = (unsigned)right.size();
  std::unordered_map<QNKey, unsigned, QNKeyHash> A_id;
  for (unsigned i = 0; i < A.blocks.size(); ++i) {
    QNKey k(A.rank);
    for (unsigned j = 0; j < A.rank; ++j) k[j] = A.blocks[i].qn[perm[j]].pack();
    A_id[k] = i;
  }
  std::set<QN> mid_set;
  std::map<QN, std::set<std::vector<unsigned>>> l_qi, r_qi;
  for (unsigned i = 0; i < A.blocks.size(); ++i) {
    QN m(0, 0);
    std::vector<unsigned> lq, rq;
    for (unsigned j = 0; j < nl; ++j) {
      if (left[j].arrow() == Inward) m += A.blocks[i].qn[perm[j]]; else m -= A.blocks[i].qn[perm[j]];
      lq.push_back(A.blocks[i].qi[perm[j]]);
    }
    for (unsigned j = 0; j < nr; ++j) rq.push_back(A.blocks[i].qi[perm[j + nl]]);
    mid_set.insert(m);
    l_qi[m].insert(lq);
    r_qi[m].insert(rq);
  }
  std::vector<Sector> sec;
  int64_t gtot = 0, wtot = 0;
  for (const QN& q : mid_set) {
    Sector s;
    s.q = q;
    for (auto& lq : l_qi[q]) {
      int64_t sz = 1;
      for (unsigned j = 0; j < nl; ++j) sz *= left[j].qdim(lq[j]);
      s.lq.push_back(lq);
      s.loff.push_back(s.rows);
      s.lsz.push_back(sz);
      s.rows += sz;
    }
    for (auto& rq : r_qi[q]) {
      int64_t sz = 1;
      for (unsigned j = 0; j < nr; ++j) sz *= right[j].qdim(rq[j]);
      s.rq.push_back(rq);
      s.roff.push_back(s.cols);
      s.rsz.push_back(sz);
      s.cols += sz;
    }
    s.g = direction == MoveFromLeft ? s.rows : s.cols;
    s.g_off = gtot;
    s.w_off = wtot;
    gtot += s.g * s.g;
    wtot += s.g;
    s.nvals = (int)std::min(s.rows, s.cols);
    if (K != 0 && (int64_t)K < s.nvals) s.nvals = (int)K;
    sec.push_back(std::move(s));
  }
  auto block_of = [&](const Sector& s, size_t i, size_t j) -> int {
    QNKey k(A.rank);
    for (unsigned t = 0; t < nl; ++t) k[t] = left[t].qn(s.lq[i][t]).pack();
    for (unsigned t = 0; t < nr; ++t) k[nl + t] = right[t].qn(s.rq[j][t]).pack();
    auto it = A_id.find(k);
    return it == A_id.end() ? -1 : (int)it->second;
  };
  // axes of an X block split into left / right, with strides
  auto left_axes = [&](unsigned b, std::vector<Ax>& out, int which, const std::vector<int64_t>* other) {
    const BlockMeta& bm = A.blocks[b];
    auto st = cm_strides(bm.qd);
    out.clear();
    for (unsigned j = 0; j < nl; ++j) out.push_back({bm.qd[perm[j]], st[perm[j]], other ? (*other)[j] : 0});
    (void)which;
  };
  auto right_axes = [&](unsigned b, std::vector<Ax>& out, const std::vector<int64_t>* other) {
    const BlockMeta& bm = A.blocks[b];
    auto st = cm_strides(bm.qd);
    out.clear();
    for (unsigned j = 0; j < nr; ++j) out.push_back({bm.qd[perm[nl + j]], st[perm[nl + j]], other ? (*other)[j] : 0});
  };

  // ---- Gram matrices on the GPU --------------------------------------
  DevPtr G = dev_alloc(std::max<int64_t>(gtot, 1));
  DevPtr Z = dev_alloc(std::max<int64_t>(gtot, 1));
  DevPtr W = dev_alloc(std::max<int64_t>(wtot, 1));
  std::vector<tt_out_block> outs;
  std::vector<tt_block_pair> pairs;
  std::vector<tt_eig_problem> probs;
  std::vector<tt_copy_desc> pack12;
  int64_t pack_off = 0;
  for (auto& s : sec) {
    tt_eig_problem ep;
    std::memset(&ep, 0, sizeof(ep));
    ep.g_off = s.g_off;
    ep.w_off = s.w_off;
    ep.n = (int32_t)s.g;
    if (direction == MoveFromRight && s.rows == 1 && s.cols == 2) {
      // the reference's 1x2 path: pack (a, b) contiguously
      ep.flags = TT_EIG_ROW_1X2;
      ep.a_off = pack_off;
      for (size_t j = 0; j < s.rq.size(); ++j) {
        int b = block_of(s, 0, j);
        if (b < 0) continue;
        tt_copy_desc d;
        std::memset(&d, 0, sizeof(d));
        d.n_modes = 1;
        d.dims[0] = (int32_t)s.rsz[j];
        d.src_off = A.blocks[b].off;
        d.src_stride[0] = 1;  // 1 row: block elements are the row in column-major order
        d.dst_off = pack_off + s.roff[j];
        d.dst_stride[0] = 1;
        pack12.push_back(d);
      }
      pack_off += 2;
      probs.push_back(ep);
      continue;
    }
    probs.push_back(ep);
    if (direction == MoveFromLeft) {
      for (size_t i = 0; i < s.lq.size(); ++i)
        for (size_t j = 0; j < s.lq.size(); ++j) {
          tt_out_block ob{s.g_off + s.loff[i] + s.g * s.loff[j], (int32_t)s.lsz[i], (int32_t)s.lsz[j],
                          (int32_t)s.g};
          outs.push_back(ob);
          for (size_t r = 0; r < s.rq.size(); ++r) {
            int bi = block_of(s, i, r), bj = block_of(s, j, r);
            if (bi < 0 || bj < 0) continue;
            tt_block_pair p;
            std::memset(&p, 0, sizeof(p));
            p.out_block = (int32_t)outs.size() - 1;
            p.a_off = A.blocks[bi].off;
            p.b_off = A.blocks[bj].off;
            std::vector<Ax> ax;
            left_axes(bi, ax, 0, nullptr);
            p.n_m = fill_modes(ax, p.m_dims, p.a_m_stride, nullptr);
            auto stj = cm_strides(A.blocks[bj].qd);
            std::vector<int64_t> kb;
            for (unsigned t = 0; t < nr; ++t) kb.push_back(stj[perm[nl + t]]);
            right_axes(bi, ax, &kb);
            p.n_k = fill_modes(ax, p.k_dims, p.a_k_stride, p.b_k_stride);
            left_axes(bj, ax, 0, nullptr);
            p.n_n = fill_modes(ax, p.n_dims, p.b_n_stride, nullptr);
            pairs.push_back(p);
          }
        }
    } else {
      for (size_t i = 0; i < s.rq.size(); ++i)
        for (size_t j = 0; j < s.rq.size(); ++j) {
          tt_out_block ob{s.g_off + s.roff[i] + s.g * s.roff[j], (int32_t)s.rsz[i], (int32_t)s.rsz[j],
                          (int32_t)s.g};
          outs.push_back(ob);
          for (size_t l = 0; l < s.lq.size(); ++l) {
            int bi = block_of(s, l, i), bj = block_of(s, l, j);
            if (bi < 0 || bj < 0) continue;
            tt_block_pair p;
            std::memset(&p, 0, sizeof(p));
            p.out_block = (int32_t)outs.size() - 1;
            p.a_off = A.blocks[bi].off;
            p.b_off = A.blocks[bj].off;
            std::vector<Ax> ax;
            right_axes(bi, ax, nullptr);
            p.n_m = fill_modes(ax, p.m_dims, p.a_m_stride, nullptr);
            auto stj = cm_strides(A.blocks[bj].qd);
            std::vector<int64_t> kb;
            for (unsigned t = 0; t < nl; ++t) kb.push_back(stj[perm[t]]);
            left_axes(bi, ax, 0, &kb);
            p.n_k = fill_modes(ax, p.k_dims, p.a_k_stride, p.b_k_stride);
            right_axes(bj, ax, nullptr);
            p.n_n = fill_modes(ax, p.n_dims, p.b_n_stride, nullptr);
            pairs.push_back(p);
          }
        }
    }
  }
  DevPtr packed;
  if (!pack12.empty()) {
    packed = dev_alloc(pack_off);
    packed->zero();
    check(tt_strided_copy_batched(ctx(), pack12.data(), (int)pack12.size(), A.data->get(), packed->get()),
          "svd pack 1x2");
  }
  if (!outs.empty()) {
    validate_pairs(outs, pairs, A.arena, A.arena, gtot);
    tt_plan* plan = nullptr;
    check(tt_contract_plan(ctx(), outs.data(), (int)outs.size(), pairs.data(), (int)pairs.size(),
                           TT_PREC_FP64, &plan),
          "svd gram plan");
    PlanHandle ph(plan);
    check(tt_contract_exec(ctx(), plan, A.data->get(), A.data->get(), G->get(), 1.0), "svd gram");
  }
  if (noise && noise->P && noise->weight > 0.0 && gtot > 0) add_noise(*noise, sec, left, right, direction, gtot, G);
  // phase 1: tridiagonal form and every eigenvalue; vectors only once the
  // truncation below has fixed how many states each sector keeps
  DevPtr Tt = dev_alloc(std::max<int64_t>(3 * wtot, 1));
  check(tt_sym_eigvals_batched(ctx(), probs.data(), (int)probs.size(), G->get(), Tt->get(), W->get(),
                               packed ? packed->get() : nullptr),
        "svd eigenvalues");
  std::vector<double> w((size_t)std::max<int64_t>(wtot, 1));
  check(tt_memcpy_d2h(ctx(), w.data(), W->get(), sizeof(double) * (size_t)wtot), "svd eigenvalues");

  // ---- truncation (:1290-1300) -----------------------------------------
  struct SV {
    double s;
    unsigned sec, pos;
  };
  std::vector<SV> all;
  double nm = 0.0;
  std::vector<std::vector<double>> svals(sec.size());
  for (unsigned ii = 0; ii < sec.size(); ++ii) {
    for (int j = 0; j < sec[ii].nvals; ++j) {
      double sv = std::sqrt(std::fabs(w[(size_t)(sec[ii].w_off + j)]));
      svals[ii].push_back(sv);
      all.push_back({sv, ii, (unsigned)j});
      nm += sv * sv;
    }
  }
  std::stable_sort(all.begin(), all.end(), [](const SV& a, const SV& b) {
    if (a.s != b.s) return a.s > b.s;
    if (a.sec != b.sec) return a.sec < b.sec;
    return a.pos < b.pos;
  });
  std::vector<unsigned> new_dim(sec.size(), 0);
  double cumsum = 0.0;
  unsigned long acc = 0;
  for (auto& e : all) {
    cumsum += e.s * e.s / nm;
    if (e.s == 0.0 && cutoff != 0.0) break;
    new_dim[e.sec] += 1;
    acc += 1;
    if ((1 - cumsum < cutoff && cutoff != 0.0) || (acc >= K && K != 0)) break;
  }
  if (info) {
    info->gram_max = 0;
    for (auto& s : sec) info->gram_max = std::max<int>(info->gram_max, (int)s.g);
    info->trunc_err = std::max(1 - cumsum, 0.0);
    info->kept = (unsigned)acc;
    info->sector_qn.clear();
    info->kept_per_sector.clear();
    for (unsigned ii = 0; ii < sec.size(); ++ii) {
      info->sector_qn.push_back(sec[ii].q);
      info->kept_per_sector.push_back(new_dim[ii]);
    }
  }

  // phase 2: eigenvectors of the kept states only
  {
    std::vector<int> nvec(sec.size());
    for (unsigned ii = 0; ii < sec.size(); ++ii) nvec[ii] = (int)new_dim[ii];
    DevPtr work = dev_alloc(std::max<int64_t>(3 * gtot, 1));
    check(tt_sym_eigvecs_batched(ctx(), probs.data(), (int)probs.size(), nvec.data(), G->get(), Tt->get(),
                                 W->get(), Z->get(), work->get(), packed ? packed->get() : nullptr),
          "svd eigenvectors");
  }

  // ---- U, V, S structure (:1302-1438) ----------------------------------
  qtensor_index midCut(Outward, "svdmid", Link, 0);
  for (unsigned ii = 0; ii < sec.size(); ++ii)
    if (new_dim[ii] > 0) midCut.addQN(sec[ii].q, new_dim[ii]);
  std::vector<qtensor_index> U_idx(left);
  U_idx.push_back(midCut);
  qtensor_index midDag = midCut;
  midDag.dag();
  std::vector<qtensor_index> V_idx{midDag};
  V_idx.insert(V_idx.end(), right.begin(), right.end());
  U = qtensor(U_idx);
  V = qtensor(V_idx);
  S = qtensor(std::vector<qtensor_index>{midCut});
  U._initted = V._initted = S._initted = true;
  std::vector<std::vector<unsigned>> ublk(sec.size()), vblk(sec.size());
  unsigned mid_num = 0;
  for (unsigned ii = 0; ii < sec.size(); ++ii) {
    unsigned nd = new_dim[ii];
    if (nd == 0) continue;
    const Sector& s = sec[ii];
    for (auto& lq : s.lq) {
      std::vector<QN> qn;
      std::vector<unsigned> qi;
      std::vector<int> qd;
      for (unsigned j = 0; j < nl; ++j) {
        qn.push_back(left[j].qn(lq[j]));
        qi.push_back(lq[j]);
        qd.push_back((int)left[j].qdim(lq[j]));
      }
      qn.push_back(s.q);
      qi.push_back(mid_num);
      qd.push_back((int)nd);
      ublk[ii].push_back(U.add_block_meta(qn, qi, qd));
    }
    for (auto& rq : s.rq) {
      std::vector<QN> qn{s.q};
      std::vector<unsigned> qi{mid_num};
      std::vector<int> qd{(int)nd};
      for (unsigned j = 0; j < nr; ++j) {
        qn.push_back(right[j].qn(rq[j]));
        qi.push_back(rq[j]);
        qd.push_back((int)right[j].qdim(rq[j]));
      }
      vblk[ii].push_back(V.add_block_meta(qn, qi, qd));
    }
    S.add_block_meta({s.q}, {mid_num}, {(int)nd});
    ++mid_num;
  }
  U.allocate(false);
  V.allocate(false);
  S.allocate(false);

  // ---- fill U, V on the GPU ---------------------------------------------
  std::vector<tt_copy_desc> copies;
  std::vector<tt_out_block> pouts;
  std::vector<tt_block_pair> ppairs;
  for (unsigned ii = 0; ii < sec.size(); ++ii) {
    unsigned nd = new_dim[ii];
    if (nd == 0) continue;
    const Sector& s = sec[ii];
    if (direction == MoveFromLeft) {
      // U block (l_i, q) = Z_q[rows of l_i, 0:nd]
      for (size_t i = 0; i < s.lq.size(); ++i) {
        const BlockMeta& ub = U.blocks[ublk[ii][i]];
        tt_copy_desc d;
        std::memset(&d, 0, sizeof(d));
        d.n_modes = 2;
        d.dims[0] = (int32_t)s.lsz[i];
        d.dims[1] = (int32_t)nd;
        d.src_off = s.g_off + s.loff[i];
        d.src_stride[0] = 1;
        d.src_stride[1] = s.g;
        d.dst_off = ub.off;
        d.dst_stride[0] = 1;
        d.dst_stride[1] = s.lsz[i];
        copies.push_back(d);
      }
      // V block (q, r_j) = sum_i Z_q[rows of l_i, 0:nd]^T X(l_i, r_j)
      for (size_t j = 0; j < s.rq.size(); ++j) {
        const BlockMeta& vb = V.blocks[vblk[ii][j]];
        pouts.push_back(tt_out_block{vb.off, (int32_t)nd, (int32_t)s.rsz[j], (int32_t)nd});
        for (size_t i = 0; i < s.lq.size(); ++i) {
          int b = block_of(s, i, j);
          if (b < 0) continue;
          tt_block_pair p;
          std::memset(&p, 0, sizeof(p));
          p.out_block = (int32_t)pouts.size() - 1;
          p.a_off = s.g_off + s.loff[i];
          p.b_off = A.blocks[b].off;
          p.n_m = 1;
          p.m_dims[0] = (int32_t)nd;
          p.a_m_stride[0] = s.g;
          std::vector<Ax> ax;
          auto st = cm_strides(A.blocks[b].qd);
          ax.clear();
          int64_t run = 1;
          for (unsigned t = 0; t < nl; ++t) {
            ax.push_back({A.blocks[b].qd[perm[t]], run, st[perm[t]]});
            run *= A.blocks[b].qd[perm[t]];
          }
          p.n_k = fill_modes(ax, p.k_dims, p.a_k_stride, p.b_k_stride);
          right_axes((unsigned)b, ax, nullptr);
          p.n_n = fill_modes(ax, p.n_dims, p.b_n_stride, nullptr);
          ppairs.push_back(p);
        }
      }
    } else {
      // V block (q, r_j) = Z_q[cols of r_j, 0:nd]^T
      for (size_t j = 0; j < s.rq.size(); ++j) {
        const BlockMeta& vb = V.blocks[vblk[ii][j]];
        tt_copy_desc d;
        std::memset(&d, 0, sizeof(d));
        d.n_modes = 2;
        d.dims[0] = (int32_t)nd;
        d.dims[1] = (int32_t)s.rsz[j];
        d.src_off = s.g_off + s.roff[j];
        d.src_stride[0] = s.g;
        d.src_stride[1] = 1;
        d.dst_off = vb.off;
        d.dst_stride[0] = 1;
        d.dst_stride[1] = nd;
        copies.push_back(d);
      }
      // U block (l_i, q) = sum_j X(l_i, r_j) Z_q[cols of r_j, 0:nd]
      for (size_t i = 0; i < s.lq.size(); ++i) {
        const BlockMeta& ubm = U.blocks[ublk[ii][i]];
        pouts.push_back(tt_out_block{ubm.off, (int32_t)s.lsz[i], (int32_t)nd, (int32_t)s.lsz[i]});
        for (size_t j = 0; j < s.rq.size(); ++j) {
          int b = block_of(s, i, j);
          if (b < 0) continue;
          tt_block_pair p;
          std::memset(&p, 0, sizeof(p));
          p.out_block = (int32_t)pouts.size() - 1;
          p.a_off = A.blocks[b].off;
          p.b_off = s.g_off + s.roff[j];
          std::vector<Ax> ax;
          left_axes((unsigned)b, ax, 0, nullptr);
          p.n_m = fill_modes(ax, p.m_dims, p.a_m_stride, nullptr);
          auto st = cm_strides(A.blocks[b].qd);
          ax.clear();
          int64_t run = 1;
          for (unsigned t = 0; t < nr; ++t) {
            ax.push_back({A.blocks[b].qd[perm[nl + t]], st[perm[nl + t]], run});
            run *= A.blocks[b].qd[perm[nl + t]];
          }
          p.n_k = fill_modes(ax, p.k_dims, p.a_k_stride, p.b_k_stride);
          p.n_n = 1;
          p.n_dims[0] = (int32_t)nd;
          p.b_n_stride[0] = s.g;
          ppairs.push_back(p);
        }
      }
    }
  }
  double* Ud = U.data->get();
  double* Vd = V.data->get();
  if (direction == MoveFromLeft) {
    if (!copies.empty())
      check(tt_strided_copy_batched(ctx(), copies.data(), (int)copies.size(), Z->get(), Ud), "svd U");
    if (!pouts.empty()) {
      validate_pairs(pouts, ppairs, gtot, A.arena, V.arena);
      tt_plan* plan = nullptr;
      check(tt_contract_plan(ctx(), pouts.data(), (int)pouts.size(), ppairs.data(), (int)ppairs.size(),
                             TT_PREC_FP64, &plan),
            "svd V plan");
      PlanHandle ph(plan);
      check(tt_contract_exec(ctx(), plan, Z->get(), A.data->get(), Vd, 1.0), "svd V");
    }
  } else {
    if (!copies.empty())
      check(tt_strided_copy_batched(ctx(), copies.data(), (int)copies.size(), Z->get(), Vd), "svd V");
    if (!pouts.empty()) {
      validate_pairs(pouts, ppairs, A.arena, gtot, U.arena);
      tt_plan* plan = nullptr;
      check(tt_contract_plan(ctx(), pouts.data(), (int)pouts.size(), ppairs.data(), (int)ppairs.size(),
                             TT_PREC_FP64, &plan),
            "svd U plan");
      PlanHandle ph(plan);
      check(tt_contract_exec(ctx(), plan, A.data->get(), Z->get(), Ud, 1.0), "svd U");
    }
  }
  // S values
  std::vector<double> hs;
  for (unsigned ii = 0; ii < sec.size(); ++ii)
    for (unsigned j = 0; j < new_dim[ii]; ++j) hs.push_back(svals[ii][j]);
  if (!hs.empty()) check(tt_memcpy_h2d(ctx(), S.data->get(), hs.data(), sizeof(double) * hs.size()), "svd S");
  // no synchronisation: the caller orders later work on the same stream
}

void svd_bond(const qtensor& combined, qtensor& A_left, qtensor& A_right, const qtensor_index& mid,
              qtensor& S, int direction, double cutoff, unsigned long K, TruncInfo* info, const NoiseTerm* noise) {
  qtensor U, V;
  qtensor_index dag_mid = mid;
  dag_mid.dag();
  std::vector<qtensor_index> left, right;
  for (auto& ix : A_left.idx_set)
    if (!ix.same_tag(mid)) left.push_back(ix);
  for (auto& ix : A_right.idx_set)
    if (!ix.same_tag(dag_mid)) right.push_back(ix);
  svd(combined, left, right, U, V, S, direction, cutoff, (unsigned)K, info, noise);
  qtensor_index& u = U.idx_set.back();
  u.rename(mid.name());
  u.retype(mid.type());
  u.prime((int)mid.level() - (int)u.level());
  qtensor_index& v = V.idx_set[0];
  v.rename(dag_mid.name());
  v.retype(dag_mid.type());
  v.prime((int)dag_mid.level() - (int)v.level());
  A_right = std::move(V);
  A_left = std::move(U);
}

}  // namespace ttb
