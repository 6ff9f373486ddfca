// big_qtensor, device-resident tensor_davidsonIT, qMPS/qMPO and the U(1)
// two-site DMRG driver (see dmrg_q.h for the reference lines followed).
#include "dmrg_q.h"
#include "observables.h"

#include <cuda_profiler_api.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>

namespace ttb {

namespace {

tt_ctx* ctx() {
  if (!rt().ctx) throw std::runtime_error("ttb: no device context bound");
  return rt().ctx;
}

// Tensor sharing another tensor's device data (indices may then be primed or
// dagged without copying the blocks).
qtensor shallow(const qtensor& T) {
  qtensor r;
  r.idx_set = T.idx_set;
  r.rank = T.rank;
  r.blocks = T.blocks;
  r.block_id = T.block_id;
  r.data = T.data;
  r.arena = T.arena;
  r._initted = T._initted;
  return r;
}

}  // namespace

// ---- DIAG -------------------------------------------------------------------
void DIAG(int n, double* M, double* evals) {
  // cyclic Jacobi on a copy; eigenvectors accumulated in V (column-major)
  std::vector<double> A(M, M + (size_t)n * n), V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i + (size_t)n * i] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[i + (size_t)n * j]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, fro = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        fro += a(i, j) * a(i, j);
        if (i != j) off += a(i, j) * a(i, j);
      }
    if (off <= 1e-32 * fro || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a(p, q);
        if (apq == 0.0) continue;
        double tau = (a(q, q) - a(p, p)) / (2.0 * apq);
        double t = (tau >= 0.0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A J
          double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- J^T A
          double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        a(p, q) = a(q, p) = 0.0;
        for (int k = 0; k < n; ++k) {
          double vkp = V[k + (size_t)n * p], vkq = V[k + (size_t)n * q];
          V[k + (size_t)n * p] = c * vkp - s * vkq;
          V[k + (size_t)n * q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
  for (int j = 0; j < n; ++j) {
    evals[j] = a(order[j], order[j]);
    for (int i = 0; i < n; ++i) M[i + (size_t)n * j] = V[i + (size_t)n * order[j]];
  }
}

// ---- big_qtensor --------------------------------------------------------------
qtensor big_qtensor::product(qtensor& v) {
  qtensor res;
  if (L_) res = (*L_) * v;
  if (res.rank > 0) res = res * mid_; else res = v * mid_;
  if (R_) res = res * (*R_);
  res.prime(-1);
  return res;
}

double big_qtensor::expec(qtensor& v) {
  qtensor res = product(v);
  return res.contract(v);
}

size_t big_qtensor::size() const {
  if (size_ == 0) {
    size_ = 1;
    if (L_)
      for (auto& ix : L_->idx_set)
        if (ix.level() > 0) size_ *= ix.size();
    if (R_)
      for (auto& ix : R_->idx_set)
        if (ix.level() > 0) size_ *= ix.size();
  }
  for (auto& ix : mid_.idx_set)
    if (ix.type() == Site) size_ *= ix.size();
  return size_;
}

// ---- the Krylov block layout and the fused product engine -----------------
namespace {

using Presence = std::vector<uint8_t>;

// The intermediates T1 = L x and T2 = T1 (W1 W2) of the H_eff*x products: a
// gigabyte each at bond dimension 3072.  The bound context keeps one buffer
// per intermediate between Davidson calls and only grows it (12.5% headroom),
// so consecutive calls do not hand gigabytes back to the pool and map them
// again.
static DevPtr heff_scratch(int which, int64_t n) {
  DevPtr& buf = rt().heff_scratch[which];
  if (!buf || buf->size() < n) {
    buf.reset();  // back to the pool before the larger one is taken
    buf = dev_alloc(n + n / 8);
  }
  return buf;
}

class ProductEngine {
 public:
  ~ProductEngine() {
    std::sort(kept_.begin(), kept_.end());
    kept_.erase(std::unique(kept_.begin(), kept_.end()), kept_.end());
    for (tt_plan* p : kept_) tt_plan_release_packed(ctx(), p);
  }
  ProductEngine(const ProductEngine&) = delete;
  ProductEngine& operator=(const ProductEngine&) = delete;
  ProductEngine(big_qtensor& A, const qtensor& x) : A_(A), x_(x) {
    if (!A_.left() || !A_.right()) throw std::runtime_error("tensor_davidsonIT: L and R must be set");
    // the block set: x's blocks, then the blocks the product adds, until closed
    for (unsigned b = 0; b < x.blocks.size(); ++b) add_block(x.blocks[b]);
    qtensor out;
    for (int it = 0; it < 8; ++it) {
      out = structure(Presence(ublocks.size(), 1));
      bool grew = false;
      for (unsigned b = 0; b < out.blocks.size(); ++b)
        if (uid.find(out.key_of(b)) == uid.end()) {
          add_block(out.blocks[b]);
          grew = true;
        }
      if (!grew) break;
    }
    // final layout: the product's own output blocks at their output offsets
    // (so the cached *R plan writes straight into the Krylov vectors), then
    // any block of the set the product does not produce
    std::vector<BlockMeta> set = std::move(ublocks);
    ublocks.clear();
    uid.clear();
    n = 0;
    for (unsigned b = 0; b < out.blocks.size(); ++b) add_block(out.blocks[b]);
    for (auto& b : set) {
      QNKey k(b.qn.size());
      for (size_t j = 0; j < b.qn.size(); ++j) k[j] = b.qn[j].pack();
      if (uid.find(k) == uid.end()) add_block(b);
    }
    build_plans(out.arena);
  }

  int64_t n = 0;
  std::vector<BlockMeta> ublocks;
  std::unordered_map<QNKey, unsigned, QNKeyHash> uid;
  double flops = 0.0;
  double part_flops[3] = {0.0, 0.0, 0.0};  // L*x, *mid, *R
  double mid_bytes = 0.0;                  // algorithmic bytes of *mid

  Presence x_presence() const {
    Presence p(ublocks.size(), 0);
    for (unsigned b = 0; b < x_.blocks.size(); ++b) p[uid.at(x_.key_of(b))] = 1;
    return p;
  }

  // x's blocks copied into their places of the layout; the rest is zeroed
  void pack(const qtensor& x, double* dst) const {
    check(tt_memset_zero(ctx(), dst, sizeof(double) * (size_t)n), "pack zero");
    std::vector<tt_copy_desc> d;
    for (unsigned b = 0; b < x.blocks.size(); ++b) {
      const BlockMeta& u = ublocks[uid.at(x.key_of(b))];
      if (u.size != x.blocks[b].size || x.blocks[b].off + x.blocks[b].size > x.arena || u.off + u.size > n)
        throw std::runtime_error("pack: block does not fit the Krylov layout");
      tt_copy_desc c;
      std::memset(&c, 0, sizeof(c));
      c.n_modes = 1;
      c.dims[0] = (int32_t)u.size;
      c.src_off = x.blocks[b].off;
      c.dst_off = u.off;
      c.src_stride[0] = 1;
      c.dst_stride[0] = 1;
      d.push_back(c);
    }
    for (size_t i = 0; i < d.size(); i += 65535)
      check(tt_strided_copy_batched(ctx(), d.data() + i, (int)std::min<size_t>(65535, d.size() - i),
                                    x.data->get(), dst),
            "pack");
  }

  // y = H_eff * v on the whole layout (absent blocks of v are zero).  L and
  // R stay fixed through a Davidson call, so in the tensor-core form their
  // packed tiles are kept in the plans from the first product of the call to
  // the engine's end (~ProductEngine releases them).
  // The precision each contraction of a product runs in.  Under an automatic
  // precision the middle contraction (bandwidth-bound: T1 read, T2 written,
  // k and n the MPO link widths) stays FP64, and L*x and *R above
  // kTensorCoreFlops run on the tensor cores without consulting the cost
  // model, whose choice for them flipped between updates at bond dimension
  // 3072 although the tensor-core form was 4x faster there every time.
  static constexpr double kTensorCoreFlops = 2e10;
  static int part_precision(int precision, int part, double flops) {
    const bool automatic = precision == TT_PREC_TF32_AUTO || precision == TT_PREC_TF32X3_AUTO;
    if (!automatic) return precision;
    if (part == 1) return TT_PREC_FP64;
    if (flops >= kTensorCoreFlops) return precision == TT_PREC_TF32_AUTO ? TT_PREC_TF32 : TT_PREC_TF32X3;
    return precision;
  }

  // ev (optional): four events recorded before L*x, after it, after *mid and after *R
  void apply(const double* v, double* y, int precision = TT_PREC_FP64, void* const* ev = nullptr) {
    if (ev) check(tt_event_record(ctx(), ev[0]), "event");
    if (tt_plan* p = c1_->plan_for(part_precision(precision, 0, part_flops[0]), 1)) {  // L kept through the call
      check(tt_contract_exec_keep(ctx(), p, L_data(), v, i1_->get(), 1.0, 1 | 8), "heff L*v");
      kept_.push_back(p);
    }
    if (ev) check(tt_event_record(ctx(), ev[1]), "event");
    if (tt_plan* p = c2_->plan_for(part_precision(precision, 1, part_flops[1])))
      check(tt_contract_exec(ctx(), p, i1_->get(), A_.mid().data->get(), i2_->get(), 1.0), "heff *mid");
    if (ev) check(tt_event_record(ctx(), ev[2]), "event");
    if (tt_plan* p = c3_->plan_for(part_precision(precision, 2, part_flops[2]), 2)) {  // and so is R
      check(tt_contract_exec_keep(ctx(), p, i2_->get(), A_.right()->data->get(), y, 1.0, 2 | 4), "heff *R");
      kept_.push_back(p);
    }
    if (ev) check(tt_event_record(ctx(), ev[3]), "event");
    for (auto& r : zero_ranges_)
      check(tt_memset_zero(ctx(), y + r.first, sizeof(double) * (size_t)r.second), "heff zero");
  }

  // block presence of product(v) given the presence of v (structure only)
  Presence product_presence(const Presence& p) {
    auto it = pcache_.find(p);
    if (it != pcache_.end()) return it->second;
    qtensor out = structure(p);
    Presence r(ublocks.size(), 0);
    for (unsigned b = 0; b < out.blocks.size(); ++b) r[uid.at(out.key_of(b))] = 1;
    pcache_[p] = r;
    return r;
  }

  // the caller's tensor with the blocks present in `p`, data in `d`
  qtensor materialize(const Presence& p, DevPtr d) const {
    qtensor t(x_.idx_set);
    t._initted = true;
    for (unsigned b = 0; b < ublocks.size(); ++b)
      if (p[b]) {
        unsigned id = t.add_block_meta(ublocks[b].qn, ublocks[b].qi, ublocks[b].qd);
        t.blocks[id].off = ublocks[b].off;
      }
    t.data = d;
    t.arena = n;
    return t;
  }

 private:
  big_qtensor& A_;
  const qtensor& x_;
  std::shared_ptr<const CachedContraction> c1_, c2_, c3_;
  DevPtr i1_, i2_;
  std::vector<std::pair<int64_t, int64_t>> zero_ranges_;
  std::map<Presence, Presence> pcache_;
  std::vector<tt_plan*> kept_;  // plans holding a packed L or R of this call

  const double* L_data() const { return A_.left()->data->get(); }

  void add_block(const BlockMeta& b) {
    BlockMeta m = b;
    m.off = n;
    n += m.size;
    QNKey k(m.qn.size());
    for (size_t j = 0; j < m.qn.size(); ++j) k[j] = m.qn[j].pack();
    uid[k] = (unsigned)ublocks.size();
    ublocks.push_back(std::move(m));
  }

  qtensor meta(const Presence& p) const {
    qtensor t(x_.idx_set);
    t._initted = true;
    for (unsigned b = 0; b < ublocks.size(); ++b)
      if (p[b]) {
        unsigned id = t.add_block_meta(ublocks[b].qn, ublocks[b].qi, ublocks[b].qd);
        t.blocks[id].off = ublocks[b].off;
      }
    t.arena = n;
    return t;
  }

  // product(v) structure for the block set `p` (metadata only; cached)
  qtensor structure(const Presence& p) const {
    qtensor v = meta(p);
    auto c1 = contract_cached(*A_.left(), v, false);
    auto c2 = contract_cached(c1->cs.C, A_.mid(), false);
    auto c3 = contract_cached(c2->cs.C, *A_.right(), false);
    qtensor out = c3->cs.C;
    out.prime(-1);
    return out;
  }

  void build_plans(int64_t produced_size) {
    qtensor v = meta(Presence(ublocks.size(), 1));
    c1_ = contract_cached(*A_.left(), v, false);
    c2_ = contract_cached(c1_->cs.C, A_.mid(), false);
    c3_ = contract_cached(c2_->cs.C, *A_.right(), false);
    const qtensor& o = c3_->cs.C;
    for (unsigned i = 0; i < x_.rank; ++i)
      if (o.idx_set.size() != x_.rank || o.idx_set[i].level() != x_.idx_set[i].level() + 1 ||
          o.idx_set[i].name() != x_.idx_set[i].name() || o.idx_set[i].arrow() != x_.idx_set[i].arrow() ||
          o.idx_set[i].sectors() != x_.idx_set[i].sectors())
        throw std::runtime_error("product: H_eff*x index order differs from x");
    // the product output must sit exactly at the start of the layout
    if (o.arena != produced_size || o.blocks.size() > ublocks.size())
      throw std::runtime_error("product: output layout mismatch");
    for (unsigned b = 0; b < o.blocks.size(); ++b)
      if (o.blocks[b].off != ublocks[b].off || o.blocks[b].qn != ublocks[b].qn)
        throw std::runtime_error("product: output layout mismatch");
    for (unsigned u = (unsigned)o.blocks.size(); u < ublocks.size(); ++u)
      zero_ranges_.push_back({ublocks[u].off, ublocks[u].size});
    flops = c1_->cs.flops + c2_->cs.flops + c3_->cs.flops;
    part_flops[0] = c1_->cs.flops;
    part_flops[1] = c2_->cs.flops;
    part_flops[2] = c3_->cs.flops;
    {
      // algorithmic bytes of the middle contraction: its distinct A and B
      // blocks read once, its C blocks written once
      std::unordered_map<int64_t, int64_t> ua, ub;
      for (const tt_block_pair& q : c2_->cs.pairs) {
        int64_t m = 1, k = 1, nn = 1;
        for (int i = 0; i < q.n_m; ++i) m *= q.m_dims[i];
        for (int i = 0; i < q.n_k; ++i) k *= q.k_dims[i];
        for (int i = 0; i < q.n_n; ++i) nn *= q.n_dims[i];
        ua[q.a_off] = m * k;
        ub[q.b_off] = k * nn;
      }
      int64_t el = 0;
      for (auto& kv : ua) el += kv.second;
      for (auto& kv : ub) el += kv.second;
      for (const tt_out_block& o : c2_->cs.outs) el += (int64_t)o.m * o.n;
      mid_bytes = 8.0 * (double)el;
    }
    i1_ = heff_scratch(0, std::max<int64_t>(c1_->cs.C.arena, 2));
    i2_ = heff_scratch(1, std::max<int64_t>(c2_->cs.C.arena, 2));
  }
};

struct KVec {
  DevPtr d;
  Presence p;
};

double read1(double* d) {
  double h;
  check(tt_memcpy_d2h(ctx(), &h, d, sizeof(double)), "d2h");
  return h;
}

}  // namespace

// Precision of one Davidson call's H_eff*x products.  The mixed-precision
// products carry a relative error of about 1e-7, so the residual never reaches
// the loop's tolerance (1e-12) and every iteration adds a direction; in a
// two-site space small enough for the Krylov vectors to exhaust it (the chain
// ends: size() over-counts the U(1) sector), those directions are product
// noise and the Ritz vector goes wrong.  Tiny problems therefore run their
// products in FP64, where they are launch-bound anyway.
constexpr int64_t kMixedMinDim = 4096;
static int davidson_precision(int64_t dim) {
  return dim <= kMixedMinDim ? TT_PREC_FP64 : rt().heff_precision;
}

// ---- tensor_davidsonIT -----------------------------------------------------
// Device-resident form: every iteration is enqueued up front and the loop's
// decisions run in the tt_dav_* control kernels, so the whole call
// synchronises once; a Gram-Schmidt failure is refilled on the device
// (tt_dav_gs_refill).  Returns false (x untouched apart from its
// normalisation) only if the control state reports an unexpected end; the
// host loop below then redoes the call.
static bool davidson_device(big_qtensor& A, qtensor& x, int max_restart, double tol, DavidsonStats* stats,
                            double& lambda_out) {
  int maxsize = (int)A.size();
  int actual_maxiter = std::min(max_restart, maxsize - 1);
  if (actual_maxiter < 0 || actual_maxiter + 2 > TT_DAV_MAX || x.arena == 0) return false;
  if (!rt().dav) check(tt_dav_state_create(ctx(), &rt().dav), "davidson state");
  tt_dav_state* st = rt().dav;
  double *coef_x = nullptr, *coef_q = nullptr;
  check(tt_dav_coefficients(st, &coef_x, &coef_q), "davidson coefficients");
  const int* refill_flag = nullptr;
  check(tt_dav_refill_flag(st, &refill_flag), "davidson refill flag");
  std::vector<DevBuf> refill_ranges;  // element ranges of each iteration's possible refill
  // x /= |x| on the device (tensor_davidson.cpp:205-206)
  check(tt_vec_nrm2(ctx(), x.arena, x.data->get(), scalar_slot(0)), "norm");
  check(tt_vec_scal_inv_dev(ctx(), x.arena, scalar_slot(0), x.data->get()), "normalize");
  auto tb0 = std::chrono::steady_clock::now();
  ProductEngine eng(A, x);
  const int prec = davidson_precision(eng.n);
  // A Krylov space cannot outgrow the vector.  size() (kept from the
  // reference) multiplies the full dimensions of every primed index, which for
  // a U(1) two-site problem at the chain ends over-counts the sector by orders
  // of magnitude (768 against 6); the loop would then try to extend a complete
  // basis, and a random refill orthogonalised against it leaves a round-off
  // remainder that can pass the 1e-10 test and enter as a near-duplicate
  // direction (Ritz value ~2 lambda).  In FP64 the residual reaches the
  // tolerance before the basis is complete, so the cap does not bind there.
  maxsize = (int)std::min<int64_t>(maxsize, eng.n);
  actual_maxiter = std::min(max_restart, maxsize - 1);
  auto tb1 = std::chrono::steady_clock::now();
  if (stats) stats->t_engine = std::chrono::duration<double>(tb1 - tb0).count();
  const int64_t n = eng.n;
  const int nsz = actual_maxiter + 2;
  std::vector<KVec> v(nsz), va(nsz), xs(nsz);
  auto newvec = [&]() {
    KVec k;
    k.d = dev_alloc(n);
    return k;
  };
  auto por = [](Presence a, const Presence& b) {
    for (size_t i = 0; i < a.size(); ++i) a[i] |= b[i];
    return a;
  };
  std::vector<std::array<void*, 4>> evs;  // per product: before L*x, after L*x, after *mid, after *R
  auto product = [&](const KVec& in) {
    KVec out = newvec();
    std::array<void*, 4> e{nullptr, nullptr, nullptr, nullptr};
    for (auto& x : e) check(tt_event_create(ctx(), &x), "event");
    eng.apply(in.d->get(), out.d->get(), prec, e.data());
    evs.push_back(e);
    out.p = eng.product_presence(in.p);
    return out;
  };
  auto lincomb = [&](KVec& y, const std::vector<const double*>& vs, const double* coef, double scale, int acc) {
    check(tt_vec_lincomb_dev(ctx(), n, (int)vs.size(), vs.data(), coef, scale, acc, y.d->get()), "lincomb");
  };
  const int kQnormSlot = 24, kNormSlot = 20;
  v[0] = newvec();
  eng.pack(x, v[0].d->get());
  v[0].p = eng.x_presence();
  va[0] = product(v[0]);
  {
    const double* p0 = v[0].d->get();
    check(tt_vec_multidot(ctx(), n, 1, &p0, va[0].d->get(), scalar_slot(0)), "initial energy");
  }
  check(tt_dav_begin(ctx(), st, scalar_slot(0)), "davidson begin");
  for (int ii = 0; ii < actual_maxiter + 1; ++ii) {
    const int ni = ii + 1;
    KVec q = newvec();
    if (ii == 0) {
      lincomb(q, {va[0].d->get(), v[0].d->get()}, coef_q, 1.0, 0);
      q.p = por(va[0].p, v[0].p);
    } else {
      check(tt_dav_ritz(ctx(), st, ii), "davidson ritz");
      KVec xn = newvec();
      std::vector<const double*> vv, vq;
      Presence px(v[0].p.size(), 0), pq(v[0].p.size(), 0);
      for (int k = 0; k <= ii; ++k) {
        vv.push_back(v[k].d->get());
        px = por(px, v[k].p);
        vq.push_back(va[k].d->get());
        pq = por(pq, va[k].p);
      }
      check(tt_vec_ritz_residual_dev(ctx(), n, ii + 1, vv.data(), vq.data(), coef_x, coef_q, xn.d->get(),
                                     q.d->get()),
            "ritz vector and residual");
      xn.p = px;
      q.p = por(pq, px);
      xs[ii] = xn;
    }
    check(tt_vec_nrm2(ctx(), n, q.d->get(), scalar_slot(kQnormSlot)), "residual norm");
    check(tt_dav_converged(ctx(), st, ii, actual_maxiter, tol, scalar_slot(kQnormSlot)), "davidson test");
    v[ni] = q;
    if (ii == actual_maxiter) break;
    // one Gram-Schmidt pass (:285-320) with device-side overlaps and norm
    std::vector<const double*> vs;
    for (int k = 0; k < ni; ++k) {
      vs.push_back(v[k].d->get());
      v[ni].p = por(v[ni].p, v[k].p);
    }
    check(tt_vec_multidot(ctx(), n, ni, vs.data(), v[ni].d->get(), scalar_slot(0)), "GS overlaps");
    check(tt_vec_project_nrm2_dev(ctx(), n, ni, vs.data(), scalar_slot(0), v[ni].d->get(), scalar_slot(kNormSlot)),
          "GS update and norm");
    {
      // Gram-Schmidt failure (:298-316) handled on the device: a random
      // refill on the blocks of v[ni-1] and one more projection, both no-ops
      // unless the norm just computed is below 1e-10
      std::vector<int64_t> ranges;
      for (unsigned b = 0; b < eng.ublocks.size(); ++b)
        if (v[ni - 1].p[b]) {
          ranges.push_back(eng.ublocks[b].off);
          ranges.push_back(eng.ublocks[b].off + eng.ublocks[b].size);
        }
      refill_ranges.emplace_back((int64_t)ranges.size() + 1);  // one int64 per 8-byte slot
      int64_t* dr = reinterpret_cast<int64_t*>(refill_ranges.back().get());
      if (!ranges.empty()) check(tt_memcpy_h2d(ctx(), dr, ranges.data(), sizeof(int64_t) * ranges.size()), "ranges");
      check(tt_dav_gs_refill(ctx(), st, ii, ni, maxsize, n, vs.data(), v[ni].d->get(), (int)ranges.size() / 2, dr,
                             rt().rng_counter++, scalar_slot(kNormSlot), scalar_slot(0)),
            "GS refill");
      check(tt_vec_project_nrm2_dev_if(ctx(), n, ni, vs.data(), scalar_slot(0), v[ni].d->get(),
                                       scalar_slot(kNormSlot), refill_flag),
            "GS refill projection");
    }
    check(tt_vec_scal_inv_dev(ctx(), n, scalar_slot(kNormSlot), v[ni].d->get()), "GS scale");
    va[ni] = product(v[ni]);
    vs.push_back(v[ni].d->get());
    check(tt_vec_multidot(ctx(), n, ni + 1, vs.data(), va[ni].d->get(), scalar_slot(0)), "M row");
    check(tt_dav_add_row(ctx(), st, ii, scalar_slot(0), scalar_slot(kNormSlot)), "davidson row");
  }
  tt_dav_result res;
  check(tt_dav_read(ctx(), st, &res), "davidson read");  // the call's one synchronisation
  if (res.final_ii == -2 || !res.done) {
    for (auto& e : evs)
      for (void* x : e) tt_event_destroy(x);
    return false;
  }
  const int f = res.final_ii;
  if (f >= 1) x = eng.materialize(xs[f].p, xs[f].d);
  x.normalize();
  double heff_ms = 0.0;
  for (size_t i = 0; i < evs.size(); ++i) {
    if ((int)i <= f) {  // products of the iterations that ran: the initial one and f more
      for (int k = 0; k < 3; ++k) {
        float ms = 0.f;
        check(tt_event_elapsed_ms(evs[i][k], evs[i][k + 1], &ms), "event");
        heff_ms += ms;
        rt().heff_part_ms[k] += ms;
        rt().heff_part_flops[k] += eng.part_flops[k];
      }
      rt().heff_mid_bytes += eng.mid_bytes;
    }
    for (void* x : evs[i]) tt_event_destroy(x);
  }
  rt().last_heff_ms = heff_ms;
  double lambda = res.lambda;
  if (prec != TT_PREC_FP64 && rt().energy_fp64) {
    KVec y = newvec();
    const KVec& xf = f >= 1 ? xs[f] : v[0];
    eng.apply(xf.d->get(), y.d->get(), TT_PREC_FP64);
    check(tt_vec_dot(ctx(), n, xf.d->get(), y.d->get(), scalar_slot(0)), "fp64 energy");
    lambda = read1(scalar_slot(0));
  }
  if (stats) {
    stats->matvecs = f + 1;
    stats->heff_flops = (f + 1) * eng.flops;
    stats->iters = res.iters;
    stats->randomized = res.randomized;
  }
  rt().dav_refills += res.randomized;
  if (stats) {
    stats->t_loop = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb1).count();
  }
  lambda_out = lambda;
  return true;
}

static double davidson_host(big_qtensor& A, qtensor& x, int m, int max_restart, double tol, char mode,
                            DavidsonStats* stats);

double tensor_davidsonIT(big_qtensor& A, qtensor& x, int m, int max_restart, double tol, char mode,
                         DavidsonStats* stats) {
  if (!(m >= 1 && max_restart >= 1 && tol > 0)) throw std::runtime_error("tensor_davidsonIT: bad arguments");
  if (rt().dav_device) {
    double lambda = 0.0;
    if (davidson_device(A, x, max_restart, tol, stats, lambda)) return lambda;
    rt().dav_fallbacks++;
    if (stats) *stats = DavidsonStats();
  }
  return davidson_host(A, x, m, max_restart, tol, mode, stats);
}

// Host-controlled form: the loop's decisions read scalars back every iteration.
static double davidson_host(big_qtensor& A, qtensor& x, int m, int max_restart, double tol, char mode,
                            DavidsonStats* stats) {
  (void)m;
  (void)mode;
  if (!(m >= 1 && max_restart >= 1 && tol > 0)) throw std::runtime_error("tensor_davidsonIT: bad arguments");
  double x_norm = x.norm();
  x *= 1.0 / x_norm;
  int maxsize = (int)A.size();
  int actual_maxiter = std::min(max_restart, maxsize - 1);
  if (actual_maxiter + 2 > 16)
    throw std::runtime_error("tensor_davidsonIT: at most 14 iterations (16 Krylov vectors) are supported");
  auto tb0 = std::chrono::steady_clock::now();
  ProductEngine eng(A, x);
  const int prec = davidson_precision(eng.n);
  // A Krylov space cannot outgrow the vector.  size() (kept from the
  // reference) multiplies the full dimensions of every primed index, which for
  // a U(1) two-site problem at the chain ends over-counts the sector by orders
  // of magnitude (768 against 6); the loop would then try to extend a complete
  // basis, and a random refill orthogonalised against it leaves a round-off
  // remainder that can pass the 1e-10 test and enter as a near-duplicate
  // direction (Ritz value ~2 lambda).  In FP64 the residual reaches the
  // tolerance before the basis is complete, so the cap does not bind there.
  maxsize = (int)std::min<int64_t>(maxsize, eng.n);
  actual_maxiter = std::min(max_restart, maxsize - 1);
  if (rt().profile) check(tt_ctx_synchronize(ctx()), "sync");
  auto tb1 = std::chrono::steady_clock::now();
  if (stats) stats->t_engine = std::chrono::duration<double>(tb1 - tb0).count();
  const int64_t n = eng.n;
  const int nsz = actual_maxiter + 2;
  std::vector<KVec> v(nsz), va(nsz);
  auto newvec = [&]() {
    KVec k;
    k.d = dev_alloc(n);
    return k;
  };
  // events bracket every product; their times are read once, at the end
  std::vector<std::pair<void*, void*>> evs;
  std::vector<bool> ev_kept;
  auto product = [&](const KVec& in) {
    KVec out = newvec();
    std::pair<void*, void*> e{nullptr, nullptr};
    check(tt_event_create(ctx(), &e.first), "event");
    check(tt_event_create(ctx(), &e.second), "event");
    check(tt_event_record(ctx(), e.first), "event");
    eng.apply(in.d->get(), out.d->get(), prec);
    check(tt_event_record(ctx(), e.second), "event");
    evs.push_back(e);
    ev_kept.push_back(true);
    out.p = eng.product_presence(in.p);
    return out;
  };
  auto count_product = [&]() {
    if (stats) {
      stats->matvecs++;
      stats->heff_flops += eng.flops;
    }
  };
  auto nrm = [&](const KVec& a) {
    check(tt_vec_nrm2(ctx(), n, a.d->get(), scalar_slot(0)), "norm");
    return read1(scalar_slot(0));
  };
  auto multidot = [&](const std::vector<const double*>& xs, const double* y) {
    std::vector<double> r(xs.size());
    check(tt_vec_multidot(ctx(), n, (int)xs.size(), xs.data(), y, scalar_slot(0)), "multidot");
    check(tt_memcpy_d2h(ctx(), r.data(), scalar_slot(0), sizeof(double) * r.size()), "d2h");
    return r;
  };
  auto por = [](Presence a, const Presence& b) {
    for (size_t i = 0; i < a.size(); ++i) a[i] |= b[i];
    return a;
  };
  // coefficients for linear combinations live in scalar slots kCoefSlot..+15
  auto lincomb = [&](KVec& y, const std::vector<const double*>& xs, const std::vector<double>& c,
                     bool accumulate) {
    if (xs.size() != c.size() || xs.size() > 16) throw std::runtime_error("lincomb: 1..16 vectors");
    check(tt_memcpy_h2d(ctx(), scalar_slot(kCoefSlot), c.data(), sizeof(double) * c.size()), "coef h2d");
    check(tt_vec_lincomb_dev(ctx(), n, (int)xs.size(), xs.data(), scalar_slot(kCoefSlot), 1.0, accumulate ? 1 : 0,
                             y.d->get()),
          "lincomb");
  };

  std::vector<double> M((size_t)nsz * nsz, 0.0), Mnext((size_t)nsz * nsz, 0.0), evals(nsz, 0.0);
  double last_lambda = 1000.0;
  const double Approx0 = 1e-12;
  v[0] = newvec();
  eng.pack(x, v[0].d->get());
  v[0].p = eng.x_presence();
  va[0] = product(v[0]);
  count_product();
  double initEn = multidot({v[0].d->get()}, va[0].d->get())[0];
  double lambda = 0.0;
  KVec xv;  // the Ritz vector once an iteration has produced one
  bool have_x = false;
  for (int ii = 0; ii < actual_maxiter + 1; ++ii) {
    const int ni = ii + 1;
    KVec q = newvec();
    if (ii == 0) {
      lambda = initEn;
      M[0] = lambda;
      Mnext[0] = lambda;
      // q = va[0] - lambda v[0]
      lincomb(q, {va[0].d->get(), v[0].d->get()}, {1.0, -lambda}, false);
      q.p = por(va[0].p, v[0].p);
    } else {
      for (int mi = 0; mi < ni; ++mi)
        for (int mj = 0; mj <= mi; ++mj) {
          Mnext[mj + mi * (ni + 1)] = M[mj + mi * ni];
          Mnext[mi + mj * (ni + 1)] = M[mi + mj * ni];
        }
      DIAG(ni, M.data(), evals.data());
      lambda = evals[0];
      const double sgn = (M[0] < 0.0) ? -1.0 : 1.0;  // sign stabilisation (:265-268)
      KVec xn = newvec();
      std::vector<const double*> xs;
      std::vector<double> c;
      Presence px(v[0].p.size(), 0), pq(v[0].p.size(), 0);
      for (int k = 0; k <= ii; ++k) {
        xs.push_back(v[k].d->get());
        c.push_back(sgn * M[k]);
        px = por(px, v[k].p);
      }
      lincomb(xn, xs, c, false);
      xn.p = px;
      // q = sum_k M[k] va[k] - lambda x  (same sign flip)
      xs.clear();
      c.clear();
      for (int k = 0; k <= ii; ++k) {
        xs.push_back(va[k].d->get());
        c.push_back(sgn * M[k]);
        pq = por(pq, va[k].p);
      }
      xs.push_back(xn.d->get());
      c.push_back(-lambda);
      lincomb(q, xs, c, false);
      q.p = por(pq, px);
      xv = xn;
      have_x = true;
    }
    double qnorm = nrm(q);
    bool converged = (qnorm < tol && std::fabs(lambda - last_lambda) < tol) || qnorm < std::max(Approx0, tol * 1e-3);
    last_lambda = lambda;
    if (stats) stats->iters = ii;
    v[ni] = q;
    if (qnorm < 1e-20 || (converged && ii >= 1) || ii == actual_maxiter) break;
    // Gram-Schmidt, one pass, random refill on failure (:285-320).  The
    // overlaps never leave the device; the new vector's norm is read together
    // with the next row of M, because its product is issued right away (and
    // discarded in the rare case that the orthogonalisation failed).
    const int Npass = 1;
    const int kNormSlot = 20;
    int pass = 1, tot_pass = 0;
    bool done = false;
    std::vector<double> row;
    while (pass <= Npass) {
      ++tot_pass;
      std::vector<const double*> vs;
      for (int k = 0; k < ni; ++k) vs.push_back(v[k].d->get());
      check(tt_vec_multidot(ctx(), n, ni, vs.data(), v[ni].d->get(), scalar_slot(0)), "GS overlaps");
      check(tt_vec_lincomb_dev(ctx(), n, ni, vs.data(), scalar_slot(0), -1.0, 1, v[ni].d->get()), "GS update");
      for (int k = 0; k < ni; ++k) v[ni].p = por(v[ni].p, v[k].p);
      check(tt_vec_nrm2(ctx(), n, v[ni].d->get(), scalar_slot(kNormSlot)), "GS norm");
      check(tt_vec_scal_inv_dev(ctx(), n, scalar_slot(kNormSlot), v[ni].d->get()), "GS scale");
      KVec va_new = product(v[ni]);
      std::vector<const double*> vs2(vs);
      vs2.push_back(v[ni].d->get());
      check(tt_vec_multidot(ctx(), n, ni + 1, vs2.data(), va_new.d->get(), scalar_slot(0)), "M row");
      std::vector<double> h(kNormSlot + 1);
      check(tt_memcpy_d2h(ctx(), h.data(), scalar_slot(0), sizeof(double) * h.size()), "d2h");
      double qnrm = h[kNormSlot];
      if (qnrm >= 1e-10) {
        va[ni] = va_new;
        count_product();
        row.assign(h.begin(), h.begin() + ni + 1);
        ++pass;
        continue;
      }
      ev_kept.back() = false;  // the speculative product is discarded
      {
        KVec r = newvec();
        r.p = v[ni - 1].p;
        std::vector<int64_t> ranges;
        for (unsigned b = 0; b < eng.ublocks.size(); ++b)
          if (r.p[b]) {
            ranges.push_back(eng.ublocks[b].off);
            ranges.push_back(eng.ublocks[b].off + eng.ublocks[b].size);
          }
        DevBuf dr((int64_t)ranges.size() + 1);  // one int64 per 8-byte slot
        check(tt_memcpy_h2d(ctx(), dr.get(), ranges.data(), sizeof(int64_t) * ranges.size()), "ranges");
        check(tt_vec_fill_random(ctx(), n, r.d->get(), (int)ranges.size() / 2, (const int64_t*)dr.get(),
                                 rt().rng_counter++),
              "random refill");
        check(tt_ctx_synchronize(ctx()), "sync");
        v[ni] = r;
        if (stats) stats->randomized++;
        qnrm = nrm(v[ni]);
        --pass;
        if (ni >= maxsize || tot_pass > Npass * 3) {
          done = true;
          break;
        }
      }
      check(tt_vec_scal(ctx(), n, 1.0 / qnrm, v[ni].d->get()), "scale");
      ++pass;
    }
    if (done) break;
    std::swap(M, Mnext);
    const int l = ni;
    for (int k = 0; k < ni + 1; ++k) {
      M[l + k * (ni + 1)] = row[k];
      M[k + l * (ni + 1)] = row[k];
    }
  }
  const KVec& xfin = have_x ? xv : v[0];
  if (have_x) {
    x = eng.materialize(xv.p, xv.d);
  }
  x.normalize();  // synchronises: every recorded event has completed
  if (prec != TT_PREC_FP64 && rt().energy_fp64) {
    // mixed precision: the reported energy is the FP64 Rayleigh quotient of
    // the final (normalised) vector, its error second order in the vector's
    KVec y = newvec();
    eng.apply(xfin.d->get(), y.d->get(), TT_PREC_FP64);
    check(tt_vec_dot(ctx(), n, xfin.d->get(), y.d->get(), scalar_slot(0)), "fp64 energy");
    lambda = read1(scalar_slot(0));
  }
  double heff_ms = 0.0;
  for (size_t i = 0; i < evs.size(); ++i) {
    float ms = 0.f;
    if (ev_kept[i]) {
      check(tt_event_elapsed_ms(evs[i].first, evs[i].second, &ms), "event");
      heff_ms += ms;
    }
    tt_event_destroy(evs[i].first);
    tt_event_destroy(evs[i].second);
  }
  rt().last_heff_ms = heff_ms;
  if (stats) stats->t_loop = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb1).count();
  return lambda;
}

// ---- spin-1/2 sites and MPS/MPO construction ------------------------------
double spin_half_op(unsigned bra, const std::string& op, unsigned ket) {
  const unsigned Dn = 0, Up = 1;
  if (op == "Id" || op == "I") return ket == bra ? 1.0 : 0.0;
  if (op == "Sz") {
    if (ket == Dn && bra == Dn) return -0.5;
    if (ket == Up && bra == Up) return 0.5;
    return 0.0;
  }
  if (op == "Sx") return ket != bra ? 0.5 : 0.0;
  if (op == "S+" || op == "Sp") return (ket == Dn && bra == Up) ? 1.0 : 0.0;
  if (op == "S-" || op == "Sm") return (ket == Up && bra == Dn) ? 1.0 : 0.0;
  throw std::runtime_error("spinhalf: unsupported operator " + op);
}

qMPS make_product_qmps(unsigned L, const std::vector<QN>& phy_qn, const std::vector<unsigned>& state,
                       unsigned id) {
  if (state.size() != L || L < 3) throw std::runtime_error("make_product_qmps: bad length");
  qMPS psi;
  psi.length = L;
  psi.id = id;
  psi.phy_qn = phy_qn;
  psi.bond_dims.assign(L + 1, 1);
  QN tot(0, 0);
  for (unsigned s : state) tot += phy_qn.at(s);
  psi.totalQ = tot;
  std::vector<std::set<QN>> link(L + 1);
  link[0].insert(QN(0, 0));
  link[L].insert(tot);
  for (unsigned j = 1; j < L; ++j)
    for (const QN& q : link[j - 1])
      for (const QN& p : phy_qn) link[j].insert(q + p);
  for (unsigned j = L - 1; j > 0; --j) {
    std::vector<QN> rm;
    for (const QN& q : link[j]) {
      bool ok = false;
      for (const QN& p : phy_qn)
        if (link[j + 1].count(q + p)) { ok = true; break; }
      if (!ok) rm.push_back(q);
    }
    for (auto& q : rm) link[j].erase(q);
  }
  for (unsigned i = 0; i < L; ++i) {
    qtensor T({qtensor_index(Inward, psi.link_name(i), Link, 0),
               qtensor_index(Inward, "Site" + std::to_string(i), Site, 0),
               qtensor_index(Outward, psi.link_name(i + 1), Link, 0)});
    for (const QN& q : link[i]) T.idx_set[0].addQN(q, 1);
    for (const QN& p : phy_qn) T.idx_set[1].addQN(p, 1);
    for (const QN& q : link[i + 1]) T.idx_set[2].addQN(q, 1);
    T.initBlock();
    psi.A.push_back(std::move(T));
  }
  QN last(0, 0);
  for (unsigned i = 0; i < L; ++i) {
    QN p = phy_qn[state[i]];
    QNKey k{last.pack(), p.pack(), (last + p).pack()};
    last += p;
    int b = psi.A[i].find_block(k);
    if (b < 0) throw std::runtime_error("make_product_qmps: product block missing");
    double one = 1.0;
    psi.A[i].set_block((unsigned)b, &one);
  }
  psi.center = (int)L - 1;
  return psi;
}

qMPO make_heisenberg_qmpo(unsigned L, const double* dh, double tE, unsigned id) {
  qMPO H;
  H.length = L;
  H.id = id;
  H.phy_qn = {QN(-1), QN(1)};
  std::string pref = "ID" + std::to_string(id) + "Link";
  std::vector<std::vector<std::vector<double>>> host(L);
  for (unsigned i = 0; i < L; ++i) {
    qtensor T({qtensor_index(Inward, pref + std::to_string(i), Link, 0),
               qtensor_index(Outward, "Site" + std::to_string(i), Site, 0),
               qtensor_index(Inward, "Site" + std::to_string(i), Site, 1),
               qtensor_index(Outward, pref + std::to_string(i + 1), Link, 0)});
    if (i == 0) {
      T.idx_set[0].addQN(QN(0), 1);
    } else {
      T.idx_set[0].addQN(QN(0), 3);
      T.idx_set[0].addQN(QN(-2), 1);
      T.idx_set[0].addQN(QN(2), 1);
    }
    for (auto& p : H.phy_qn) T.idx_set[1].addQN(p, 1);
    for (auto& p : H.phy_qn) T.idx_set[2].addQN(p, 1);
    if (i == L - 1) {
      T.idx_set[3].addQN(QN(0), 1);
    } else {
      T.idx_set[3].addQN(QN(0), 3);
      T.idx_set[3].addQN(QN(-2), 1);
      T.idx_set[3].addQN(QN(2), 1);
    }
    T.initBlock();
    host[i].resize(T.blocks.size());
    for (unsigned b = 0; b < T.blocks.size(); ++b) host[i][b].assign((size_t)T.blocks[b].size, 0.0);
    H.A.push_back(std::move(T));
  }
  // addOperators for qMPO (models/hams/Heisenberg.cpp:152-196)
  auto add = [&](unsigned site, unsigned r, unsigned c, const std::string& op, double val, int Qi, int Qo) {
    qtensor& T = H.A[site];
    bool added = false;
    for (unsigned k = 0; k < 2; ++k)
      for (unsigned b = 0; b < 2; ++b) {
        QNKey key{QN(Qi).pack(), H.phy_qn[k].pack(), H.phy_qn[b].pack(), QN(Qo).pack()};
        int blk = T.find_block(key);
        if (blk < 0) continue;
        added = true;
        const BlockMeta& bm = T.blocks[blk];
        int64_t s3 = (int64_t)bm.qd[0] * bm.qd[1] * bm.qd[2];
        int64_t off = (site == 0) ? s3 * c : (int64_t)r + s3 * c;
        host[site][blk][(size_t)off] = val * spin_half_op(b, op, k);
      }
    if (!added) throw std::runtime_error("heisenberg qMPO: operator block missing");
  };
  for (unsigned site = 0; site < L; ++site) {
    bool last = site == L - 1;
    if (site > 0) add(site, 0, 0, "Id", 1.0, 0, 0);
    if (!last) add(site, 1, 1, "Id", 1.0, 0, 0);
    if (dh) add(site, 1, 0, "Sz", dh[site], 0, 0);
    if (tE != 0) add(site, 1, 0, "Id", -tE / L, 0, 0);
    if (site > 0) add(site, 2, 0, "Sz", 1.0, 0, 0);
    if (!last) add(site, 1, 2, "Sz", 1.0, 0, 0);
    if (site > 0) add(site, 0, 0, "S+", 1.0, -2, 0);
    if (site > 0) add(site, 0, 0, "S-", 1.0, 2, 0);
    if (!last) add(site, 1, 0, "S-", 0.5, 0, -2);
    if (!last) add(site, 1, 0, "S+", 0.5, 0, 2);
  }
  for (unsigned i = 0; i < L; ++i)
    for (unsigned b = 0; b < H.A[i].blocks.size(); ++b) H.A[i].set_block(b, host[i][b].data());
  return H;
}

// ---- canonical centre ------------------------------------------------------
double qMPS::position(int site) {
  // mps/qtt.cpp:932-994
  if (center == -1) {
    center = (int)length - 1;  // rc(): sweep the centre from the right end
    while (center > 0) position(center - 1);
  }
  qtensor U, V, S;
  bool moved = false;
  while (center != site) {
    std::vector<qtensor_index> left, right;
    qtensor_index mid;
    if (center > site) {
      std::string ln = link_name((unsigned)center);
      for (auto& ix : A[center].idx_set) {
        if (ix.name() == ln) { left.push_back(ix); mid = ix; } else right.push_back(ix);
      }
      svd(A[center], left, right, U, V, S, MoveFromRight);
      bond_dims[center] = (unsigned)S.total_size();
      A[center] = std::move(V);
      A[center].idx_set[0].rename(mid.name());
      A[center].idx_set[0].prime((int)mid.level() - (int)A[center].idx_set[0].level());
      A[center - 1] = A[center - 1] * U;
      A[center - 1].idx_set.back().rename(mid.name());
      A[center - 1].idx_set.back().prime((int)mid.level() - (int)A[center - 1].idx_set.back().level());
      --center;
    } else {
      std::string ln = link_name((unsigned)center + 1);
      for (auto& ix : A[center].idx_set) {
        if (ix.name() == ln) { right.push_back(ix); mid = ix; } else left.push_back(ix);
      }
      svd(A[center], left, right, U, V, S, MoveFromLeft);
      bond_dims[center + 1] = (unsigned)S.total_size();
      A[center] = std::move(U);
      A[center].idx_set.back().rename(mid.name());
      A[center].idx_set.back().prime((int)mid.level() - (int)A[center].idx_set.back().level());
      A[center + 1] = V * A[center + 1];
      A[center + 1].idx_set[0].rename(mid.name());
      A[center + 1].idx_set[0].prime((int)mid.level() - (int)A[center + 1].idx_set[0].level());
      ++center;
    }
    moved = true;
  }
  if (!moved) return 0.0;
  return calcEntropy(S);
}

void qMPS::normalize() {
  // mps/qtt.cpp:899-909 (centre form)
  double nm = A[center].norm();
  A[center] /= nm;
}

// ---- environments, site update, sweep ---------------------------------------
static qtensor boundary(const qtensor_index& psi_ix, const qtensor_index& h_ix) {
  qtensor T({psi_ix, h_ix, psi_ix});
  T.idx_set[0].prime();  // primeLink
  T.idx_set[0].dag();
  T.initBlock();
  T.setOne();
  T.dag();
  return T;
}

qtensor env_step(const qtensor& env, const qtensor& Ai, const qtensor& W) {
  qtensor t1 = shallow(Ai);
  t1.conj();
  t1.dag();
  t1.prime();
  qtensor t4 = t1 * env;
  qtensor t5 = t4 * W;
  return t5 * Ai;
}

void buildEnv(qMPS& psi, qMPO& H, std::vector<qtensor>& TR, std::vector<qtensor>& TL) {
  // algos/dmrg/dmrg.cpp:56-85
  const unsigned L = psi.length;
  TL[0] = boundary(psi.A[0].idx_set[0], H.A[0].idx_set[0]);
  TR[L - 1] = boundary(psi.A[L - 1].idx_set.back(), H.A[L - 1].idx_set.back());
  for (unsigned i = L - 1; i > 0; --i) TR[i - 1] = env_step(TR[i], psi.A[i], H.A[i]);
}

StepEvents::~StepEvents() {
  for (void* e : ev)
    if (e) tt_event_destroy(e);
}
void StepEvents::record(int i) {
  if (!ev[i]) check(tt_event_create(ctx(), &ev[i]), "step event");
  check(tt_event_record(ctx(), ev[i]), "step event");
}

void updateSite(qMPS& psi, qMPO& H, std::vector<qtensor>& TR, std::vector<qtensor>& TL, unsigned site,
                double& energy, int direction, int max_bd, double cutoff, char mode, int search_space_size,
                int max_restart, DmrgLog* log, double noise) {
  // algos/dmrg/dmrg.cpp:300-372
  unsigned l, r;
  if (direction == MoveFromLeft) { l = site; r = site + 1; } else { l = site - 1; r = site; }
  auto t0 = std::chrono::steady_clock::now();
  std::shared_ptr<StepEvents> events;
  if (log) {
    events = std::make_shared<StepEvents>();
    events->record(0);
  }
  big_qtensor A;
  A.setLeft(&TL[l]);
  A.addMid(&H.A[l]);
  A.addMid(&H.A[r]);
  A.setRight(&TR[r]);
  qtensor x = psi.A[l] * psi.A[r];
  DavidsonStats st;
  energy = tensor_davidsonIT(A, x, search_space_size, max_restart, 1e-12, mode, &st);
  if (rt().profile) check(tt_ctx_synchronize(ctx()), "sync");
  auto t1 = std::chrono::steady_clock::now();
  if (events) events->record(1);
  std::string ln = psi.link_name(r);
  qtensor_index mid;
  for (auto& ix : psi.A[l].idx_set)
    if (ix.name() == ln) { mid = ix; break; }
  qtensor S;
  TruncInfo info;
  if (noise > 0.0) {
    // density-matrix perturbation from the half of H_eff on the kept side:
    // (TL W1) x left to right, x (W2 TR) right to left
    qtensor P = direction == MoveFromLeft ? (TL[l] * x) * H.A[l] : (x * H.A[r]) * TR[r];
    NoiseTerm nt;
    nt.P = &P;
    nt.weight = noise;
    svd_bond(x, psi.A[l], psi.A[r], mid, S, direction, cutoff, (unsigned long)max_bd, &info, &nt);
  } else {
    svd_bond(x, psi.A[l], psi.A[r], mid, S, direction, cutoff, (unsigned long)max_bd, &info);
  }
  if (rt().profile) check(tt_ctx_synchronize(ctx()), "sync");  // the SVD's asynchronous tail counts as SVD
  auto t2 = std::chrono::steady_clock::now();
  if (events) events->record(2);
  psi.bond_dims[r] = (unsigned)S.total_size();
  psi.center = (int)(direction == MoveFromLeft ? r : l);
  if (log) {
    StepLog s;
    s.site = (int)site;
    s.direction = direction;
    s.energy = energy;
    s.trunc_err = info.trunc_err;
    s.kept = info.kept;
    s.matvecs = st.matvecs;
    s.randomized = st.randomized;
    s.heff_flops = st.heff_flops;
    s.sector_qn = info.sector_qn;
    s.kept_per_sector = info.kept_per_sector;
    s.gram_max = info.gram_max;
    s.t_davidson = std::chrono::duration<double>(t1 - t0).count();
    s.t_engine = st.t_engine;
    s.t_svd = std::chrono::duration<double>(t2 - t1).count();
    s.events = std::move(events);
    log->steps.push_back(std::move(s));
    log->heff_flops += st.heff_flops;
    log->heff_seconds += rt().last_heff_ms * 1e-3;
    bool mid_bond = direction == MoveFromLeft ? (site == psi.length / 2 - 1) : (site == psi.length / 2);
    if (mid_bond) log->entropy.push_back(calcEntropy(S));
  }
}

void updateEnv(qMPS& psi, qMPO& H, std::vector<qtensor>& TR, std::vector<qtensor>& TL, unsigned site,
               int direction) {
  // algos/dmrg/dmrg.cpp:491-509; contractions at the environment precision
  PrecisionScope prec(rt().env_precision);
  if (direction == MoveFromLeft)
    TL[site + 1] = env_step(TL[site], psi.A[site], H.A[site]);
  else
    TR[site - 1] = env_step(TR[site], psi.A[site], H.A[site]);
}

void dmrg_prepare(qMPS& psi, qMPO& H, DmrgState& st, DmrgLog* log) {
  const unsigned L = H.length;
  psi.position(0);
  psi.normalize();
  st.TR.assign(L, qtensor());
  st.TL.assign(L, qtensor());
  buildEnv(psi, H, st.TR, st.TL);
  st.envs_built = true;
  st.sweeps_done = 0;
  big_qtensor A;  // initial energy of the one-site problem (dmrg.cpp:716-723)
  A.setLeft(&st.TL[0]);
  A.addMid(&H.A[0]);
  A.setRight(&st.TR[0]);
  double e = A.expec(psi.A[0]);
  if (log) log->initial_energy = e;
}

// After a two-site update at `site` the orthogonality centre has moved past
// it: left-to-right, TR[site] will be rebuilt before it is read again;
// right-to-left, TL[site].  Releasing them keeps only the environments on the
// live side of the centre (TL[0..c], TR[c..L-1]) -- half of the 2L the
// reference holds -- so bond dimension 3072 on the 96-site cylinder fits in
// HBM.  Boundaries (TL[0], TR[L-1]) are never released.
static void release_stale(DmrgState& st, unsigned site, int direction, unsigned L) {
  if (direction == MoveFromLeft && site > 0 && site < L - 1) st.TR[site] = qtensor();
  if (direction == MoveFromRight && site > 0 && site < L - 1) st.TL[site] = qtensor();
}

double dmrg_walk(qMPS& psi, qMPO& H, DmrgState& st, int to, int max_bd, double cutoff, int max_restart,
                 DmrgLog* log) {
  const int L = (int)H.length;
  if (!st.envs_built) throw std::runtime_error("dmrg_walk: environments not built");
  if (to < 0 || to >= L) throw std::runtime_error("dmrg_walk: target site out of range");
  double energy = 0.0;
  while (st.pos != to) {
    const int direction = to > st.pos ? MoveFromLeft : MoveFromRight;
    const unsigned site = (unsigned)st.pos;
    updateSite(psi, H, st.TR, st.TL, site, energy, direction, max_bd, cutoff, 'S', 3, max_restart, log, st.noise);
    auto te0 = std::chrono::steady_clock::now();
    updateEnv(psi, H, st.TR, st.TL, site, direction);
    release_stale(st, site, direction, (unsigned)L);
    if (log && !log->steps.empty()) {
      if (log->steps.back().events) log->steps.back().events->record(3);
      if (rt().profile) check(tt_ctx_synchronize(ctx()), "sync");
      log->steps.back().t_env = std::chrono::duration<double>(std::chrono::steady_clock::now() - te0).count();
    }
    st.pos += direction == MoveFromLeft ? 1 : -1;
  }
  return energy;
}

double dmrg_sweep(qMPS& psi, qMPO& H, DmrgState& st, int max_bd, double cutoff, int max_restart,
                  DmrgLog* log) {
  const unsigned L = H.length;
  if (st.pos != 0) throw std::runtime_error("dmrg_sweep: the orthogonality centre must be at site 0");
  double energy = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  for (int half = 0; half < 2; ++half) {
    int direction = half == 0 ? MoveFromLeft : MoveFromRight;
    for (unsigned i = 0; i < L - 1; ++i) {
      unsigned site = direction == MoveFromLeft ? i : L - 1 - i;
      // the sweep's energy (its last step) is evaluated in FP64 in mixed precision
      rt().energy_fp64 = half == 1 && i == L - 2;
      const bool prof = rt().profile_step == (int)(half * (L - 1) + i);
      if (prof) cudaProfilerStart();
      updateSite(psi, H, st.TR, st.TL, site, energy, direction, max_bd, cutoff, 'S', 3, max_restart, log, st.noise);
      rt().energy_fp64 = false;
      auto te0 = std::chrono::steady_clock::now();
      updateEnv(psi, H, st.TR, st.TL, site, direction);
      release_stale(st, site, direction, L);
      if (prof) {
        check(tt_ctx_synchronize(ctx()), "sync");
        cudaProfilerStop();
      }
      if (log && !log->steps.empty()) {
        if (log->steps.back().events) log->steps.back().events->record(3);
        if (rt().profile) check(tt_ctx_synchronize(ctx()), "sync");
        log->steps.back().t_env =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - te0).count();
      }
    }
  }
  psi.normalize();
  if (rt().env_precision != TT_PREC_FP64) {
    // environments built in mixed precision bias the Ritz value to first
    // order in their error, while the state itself keeps FP64 quality: the
    // sweep energy is <psi|H|psi> / <psi|psi> contracted in FP64
    PrecisionScope prec(TT_PREC_FP64);
    energy = psiHphi(psi, H, psi) / psiphi(psi, psi);
  }
  check(tt_ctx_synchronize(ctx()), "sweep sync");
  auto t1 = std::chrono::steady_clock::now();
  if (log) {
    log->sweep_energy.push_back(energy);
    log->sweep_seconds.push_back(std::chrono::duration<double>(t1 - t0).count());
  }
  st.sweeps_done++;
  return energy;
}

void dmrg_finish(qMPS& psi) { psi.position(0); }

double dmrg(qMPS& psi, qMPO& H, int num_sweeps, const std::vector<int>& max_bd,
            const std::vector<double>& cutoff, const std::vector<int>& max_restart, DmrgLog* log) {
  DmrgState st;
  dmrg_prepare(psi, H, st, log);
  double energy = 0.0;
  for (int sweep = 0; sweep < num_sweeps; ++sweep) {
    int lbd = sweep % (int)max_bd.size();
    int lc = sweep % (int)cutoff.size();
    int lmr = sweep % (int)max_restart.size();
    energy = dmrg_sweep(psi, H, st, max_bd[lbd], cutoff[lc], max_restart[lmr], log);
  }
  dmrg_finish(psi);
  return energy;
}

}  // namespace ttb
