// extern "C" object API (include/tt_dmrg.h) over the C++ host mirror.
#include <cstring>
#include <exception>
#include <string>

#include "../../../include/tt_dmrg.h"
#include <cuda_runtime.h>

#include "../host/dmrg_q.h"

namespace tt {
void set_error(const std::string& msg);
}

struct tt_qtensor {
  ttb::qtensor t;
};
struct tt_bigq {
  ttb::qtensor L, R;
  ttb::big_qtensor op;
};
struct tt_qmps {
  ttb::qMPS psi;
};
struct tt_qmpo {
  ttb::qMPO H;
};
struct tt_qdmrg {
  tt_qmps* psi = nullptr;
  tt_qmpo* H = nullptr;
  ttb::DmrgState st;
  ttb::DmrgLog log;
};

#define TT_GUARD(...)                                       \
  try {                                                     \
    __VA_ARGS__;                                            \
    return TT_OK;                                           \
  } catch (const ttb::tt_error& e) {                        \
    tt::set_error(e.what());                                \
    return e.code;                                          \
  } catch (const std::bad_alloc& e) {                       \
    tt::set_error("host allocation failed");                \
    return TT_ERR_OOM;                                      \
  } catch (const std::exception& e) {                       \
    tt::set_error(e.what());                                \
    return TT_ERR_INVALID;                                  \
  }

#define TT_ARG(cond)                                        \
  do {                                                      \
    if (!(cond)) {                                          \
      tt::set_error("invalid argument: " #cond);            \
      return TT_ERR_INVALID;                                \
    }                                                       \
  } while (0)

namespace {

ttb::qtensor_index make_index(const tt_index_desc& d) {
  ttb::qtensor_index ix(d.arrow == 0 ? ttb::Inward : ttb::Outward, d.name ? d.name : "",
                        d.type == 0 ? ttb::Link : ttb::Site, (unsigned)d.level);
  for (int i = 0; i < d.n_sectors; ++i) ix.addQN(ttb::QN(d.qn[2 * i], d.qn[2 * i + 1]), (unsigned)d.qdim[i]);
  return ix;
}

tt_qtensor* wrap(ttb::qtensor&& t) {
  tt_qtensor* h = new tt_qtensor();
  h->t = std::move(t);
  return h;
}

}  // namespace

extern "C" {

int tt_dmrg_bind(tt_ctx* ctx) {
  TT_ARG(ctx);
  TT_GUARD(ttb::bind_context(ctx));
}

int tt_dmrg_unbind(void) { TT_GUARD(ttb::unbind_context()); }

int tt_dmrg_set_profile_step(int step) { TT_GUARD(ttb::rt().profile_step = step); }

int tt_dmrg_set_davidson(int device_control) { TT_GUARD(ttb::rt().dav_device = device_control != 0); }

int tt_dmrg_davidson_fallbacks(int64_t* n) {
  TT_ARG(n);
  TT_GUARD(*n = ttb::rt().dav_fallbacks);
}

int tt_dmrg_davidson_refills(int64_t* n) {
  TT_ARG(n);
  TT_GUARD(*n = ttb::rt().dav_refills);
}

int tt_dmrg_set_precision(int op, int heff, int env) {
  auto ok = [](int p) { return p >= TT_PREC_FP64 && p <= TT_PREC_TF32X3_AUTO; };
  TT_ARG(ok(op) && ok(heff) && ok(env));
  TT_GUARD({
    ttb::rt().precision = op;
    ttb::rt().heff_precision = heff;
    ttb::rt().env_precision = env;
  });
}

int tt_dmrg_set_profiling(int on) { TT_GUARD(ttb::rt().profile = on != 0); }

int tt_dmrg_heff_parts(double* ms, double* flops, double* mid_bytes) {
  TT_ARG(ms && flops && mid_bytes);
  TT_GUARD({
    for (int k = 0; k < 3; ++k) {
      ms[k] = ttb::rt().heff_part_ms[k];
      flops[k] = ttb::rt().heff_part_flops[k];
    }
    *mid_bytes = ttb::rt().heff_mid_bytes;
  });
}

int tt_dmrg_planning_counters(double* t_structure, int64_t* n_structure, double* t_plan, int64_t* n_plan) {
  TT_GUARD({
    if (t_structure) *t_structure = ttb::rt().t_structure;
    if (n_structure) *n_structure = ttb::rt().n_structure;
    if (t_plan) *t_plan = ttb::rt().t_plan;
    if (n_plan) *n_plan = ttb::rt().n_plan;
  });
}

int tt_dmrg_cache_stats(int64_t* entries, int64_t* plan_bytes, int64_t* evictions, int64_t* evicted) {
  TT_GUARD({ ttb::contraction_cache_stats(entries, plan_bytes, evictions, evicted); });
}

// ---- qtensor -------------------------------------------------------------
int tt_qtensor_create(int rank, const tt_index_desc* idx, tt_qtensor** out) {
  TT_ARG(out && rank >= 0 && (rank == 0 || idx));
  TT_GUARD({
    std::vector<ttb::qtensor_index> v;
    for (int i = 0; i < rank; ++i) v.push_back(make_index(idx[i]));
    *out = wrap(ttb::qtensor(v));
  });
}

int tt_qtensor_init_blocks(tt_qtensor* t) {
  TT_ARG(t);
  TT_GUARD(t->t.initBlock());
}

int tt_qtensor_set_blocks(tt_qtensor* t, int n_blocks, const int32_t* qi) {
  TT_ARG(t && n_blocks >= 0 && (n_blocks == 0 || qi));
  TT_GUARD({
    ttb::qtensor& T = t->t;
    T.blocks.clear();
    T.block_id.clear();
    for (int b = 0; b < n_blocks; ++b) {
      std::vector<ttb::QN> qn;
      std::vector<unsigned> pos;
      std::vector<int> qd;
      for (unsigned j = 0; j < T.rank; ++j) {
        int p = qi[(size_t)b * T.rank + j];
        if (p < 0 || p >= (int)T.idx_set[j].size()) throw std::runtime_error("set_blocks: sector out of range");
        pos.push_back((unsigned)p);
        qn.push_back(T.idx_set[j].qn(p));
        qd.push_back((int)T.idx_set[j].qdim(p));
      }
      T.add_block_meta(qn, pos, qd);
    }
    T.allocate(true);
    T._initted = true;
  });
}

int tt_qtensor_destroy(tt_qtensor* t) {
  TT_GUARD(delete t);
}

int tt_qtensor_copy(const tt_qtensor* t, tt_qtensor** out) {
  TT_ARG(t && out);
  TT_GUARD(*out = wrap(ttb::qtensor(t->t)));
}

int tt_qtensor_rank(const tt_qtensor* t, int* rank) {
  TT_ARG(t && rank);
  TT_GUARD(*rank = (int)t->t.rank);
}

int tt_qtensor_index(const tt_qtensor* t, int i, int32_t* arrow, int32_t* type, int32_t* level,
                     int32_t* n_sectors, char* name_buf, int name_cap, int32_t* qn, int32_t* qdim, int cap) {
  TT_ARG(t && i >= 0 && i < (int)t->t.rank);
  TT_GUARD({
    const ttb::qtensor_index& ix = t->t.idx_set[i];
    if (arrow) *arrow = (int32_t)ix.arrow();
    if (type) *type = (int32_t)ix.type();
    if (level) *level = (int32_t)ix.level();
    if (n_sectors) *n_sectors = (int32_t)ix.size();
    if (name_buf && name_cap > 0) {
      std::strncpy(name_buf, ix.name().c_str(), (size_t)name_cap - 1);
      name_buf[name_cap - 1] = 0;
    }
    for (int s = 0; s < (int)ix.size() && s < cap; ++s) {
      if (qn) { qn[2 * s] = ix.qn(s).a; qn[2 * s + 1] = ix.qn(s).b; }
      if (qdim) qdim[s] = (int32_t)ix.qdim(s);
    }
  });
}

int tt_qtensor_num_blocks(const tt_qtensor* t, int* n) {
  TT_ARG(t && n);
  TT_GUARD(*n = (int)t->t.blocks.size());
}

int tt_qtensor_block_info(const tt_qtensor* t, int b, int32_t* qn, int32_t* qi, int32_t* qd, int64_t* size) {
  TT_ARG(t && b >= 0 && b < (int)t->t.blocks.size());
  TT_GUARD({
    const ttb::BlockMeta& m = t->t.blocks[b];
    for (unsigned j = 0; j < t->t.rank; ++j) {
      if (qn) { qn[2 * j] = m.qn[j].a; qn[2 * j + 1] = m.qn[j].b; }
      if (qi) qi[j] = (int32_t)m.qi[j];
      if (qd) qd[j] = m.qd[j];
    }
    if (size) *size = m.size;
  });
}

int tt_qtensor_find_block(const tt_qtensor* t, const int32_t* qn, int* b) {
  TT_ARG(t && qn && b);
  TT_GUARD({
    ttb::QNKey k(t->t.rank);
    for (unsigned j = 0; j < t->t.rank; ++j) k[j] = ttb::QN(qn[2 * j], qn[2 * j + 1]).pack();
    *b = t->t.find_block(k);
  });
}

int tt_qtensor_get_block(const tt_qtensor* t, int b, double* host) {
  TT_ARG(t && host && b >= 0 && b < (int)t->t.blocks.size());
  TT_GUARD({
    std::vector<double> v = t->t.get_block((unsigned)b);
    std::memcpy(host, v.data(), sizeof(double) * v.size());
  });
}

int tt_qtensor_set_block(tt_qtensor* t, int b, const double* host) {
  TT_ARG(t && host && b >= 0 && b < (int)t->t.blocks.size());
  TT_GUARD(t->t.set_block((unsigned)b, host));
}

int tt_qtensor_prime(tt_qtensor* t, int inc) {
  TT_ARG(t);
  TT_GUARD(t->t.prime(inc));
}

int tt_qtensor_dag(tt_qtensor* t) {
  TT_ARG(t);
  TT_GUARD(t->t.dag());
}

int tt_qtensor_contract(const tt_qtensor* A, const tt_qtensor* B, tt_qtensor** C) {
  TT_ARG(A && B && C);
  TT_GUARD({
    ttb::qtensor r = A->t * B->t;
    tt_ctx_synchronize(ttb::rt().ctx);
    *C = wrap(std::move(r));
  });
}

int tt_qtensor_norm(const tt_qtensor* t, double* out) {
  TT_ARG(t && out);
  TT_GUARD(*out = t->t.norm());
}

int tt_qtensor_scale(tt_qtensor* t, double c) {
  TT_ARG(t);
  TT_GUARD(t->t *= c);
}

int tt_qtensor_add(tt_qtensor* y, const tt_qtensor* x, double c) {
  TT_ARG(y && x);
  TT_GUARD(y->t.add(x->t, c));
}

int tt_qtensor_inner_product(const tt_qtensor* a, const tt_qtensor* b, double* out) {
  TT_ARG(a && b && out);
  TT_GUARD(*out = a->t.inner_product(b->t));
}

int tt_qtensor_svd(const tt_qtensor* A, int nleft, const int* left_axes, int direction, double cutoff,
                   unsigned K, tt_qtensor** U, tt_qtensor** V, tt_qtensor** S, double* trunc_err,
                   unsigned* kept) {
  TT_ARG(A && U && V && S && nleft > 0 && nleft < (int)A->t.rank && left_axes);
  TT_ARG(direction == MoveFromLeft || direction == MoveFromRight);
  TT_GUARD({
    std::vector<ttb::qtensor_index> left, right;
    std::vector<bool> used(A->t.rank, false);
    for (int i = 0; i < nleft; ++i) {
      if (left_axes[i] < 0 || left_axes[i] >= (int)A->t.rank) throw std::runtime_error("svd: bad axis");
      left.push_back(A->t.idx_set[left_axes[i]]);
      used[left_axes[i]] = true;
    }
    for (unsigned i = 0; i < A->t.rank; ++i)
      if (!used[i]) right.push_back(A->t.idx_set[i]);
    ttb::qtensor u, v, s;
    ttb::TruncInfo info;
    ttb::svd(A->t, left, right, u, v, s, direction, cutoff, K, &info);
    *U = wrap(std::move(u));
    *V = wrap(std::move(v));
    *S = wrap(std::move(s));
    if (trunc_err) *trunc_err = info.trunc_err;
    if (kept) *kept = info.kept;
  });
}

int tt_qtensor_svd_bond(const tt_qtensor* combined, tt_qtensor* A_left, tt_qtensor* A_right, int mid_axis,
                        int direction, double cutoff, unsigned long K, tt_qtensor** S, double* trunc_err,
                        unsigned* kept) {
  TT_ARG(combined && A_left && A_right && mid_axis >= 0 && mid_axis < (int)A_left->t.rank);
  TT_GUARD({
    ttb::qtensor s;
    ttb::TruncInfo info;
    ttb::qtensor_index mid = A_left->t.idx_set[mid_axis];
    ttb::svd_bond(combined->t, A_left->t, A_right->t, mid, s, direction, cutoff, K, &info);
    if (S) *S = wrap(std::move(s));
    if (trunc_err) *trunc_err = info.trunc_err;
    if (kept) *kept = info.kept;
  });
}

int tt_qtensor_svd_bond_sectors(const tt_qtensor* combined, tt_qtensor* A_left, tt_qtensor* A_right,
                                int mid_axis, int direction, double cutoff, unsigned long K, tt_qtensor** S,
                                double* trunc_err, unsigned* kept, int* n_sectors, int32_t* qn,
                                uint32_t* kept_per_sector, int cap) {
  TT_ARG(combined && A_left && A_right && mid_axis >= 0 && mid_axis < (int)A_left->t.rank && n_sectors &&
         cap >= 0 && (cap == 0 || (qn && kept_per_sector)));
  TT_GUARD({
    ttb::qtensor s;
    ttb::TruncInfo info;
    ttb::qtensor_index mid = A_left->t.idx_set[mid_axis];
    ttb::svd_bond(combined->t, A_left->t, A_right->t, mid, s, direction, cutoff, K, &info);
    if (S) *S = wrap(std::move(s));
    if (trunc_err) *trunc_err = info.trunc_err;
    if (kept) *kept = info.kept;
    *n_sectors = (int)info.sector_qn.size();
    for (int j = 0; j < *n_sectors && j < cap; ++j) {
      qn[2 * j] = info.sector_qn[j].a;
      qn[2 * j + 1] = info.sector_qn[j].b;
      kept_per_sector[j] = info.kept_per_sector[j];
    }
  });
}

int tt_qtensor_env_update(const tt_qtensor* env, const tt_qtensor* A, const tt_qtensor* W, tt_qtensor** out) {
  TT_ARG(env && A && W && out);
  TT_GUARD({
    ttb::PrecisionScope prec(ttb::rt().env_precision);
    *out = wrap(ttb::env_step(env->t, A->t, W->t));
  });
}

// ---- big_qtensor ---------------------------------------------------------------
int tt_bigq_create(const tt_qtensor* L, const tt_qtensor* W1, const tt_qtensor* W2, const tt_qtensor* R,
                   tt_bigq** out) {
  TT_ARG(L && W1 && R && out);
  TT_GUARD({
    tt_bigq* h = new tt_bigq();
    h->L = L->t;
    h->R = R->t;
    h->op.setLeft(&h->L);
    h->op.addMid(const_cast<ttb::qtensor*>(&W1->t));
    if (W2) h->op.addMid(const_cast<ttb::qtensor*>(&W2->t));
    h->op.setRight(&h->R);
    *out = h;
  });
}

int tt_bigq_product(tt_bigq* op, const tt_qtensor* v, tt_qtensor** out) {
  TT_ARG(op && v && out);
  TT_GUARD({
    ttb::qtensor x = v->t;
    ttb::qtensor r = op->op.product(x);
    *out = wrap(std::move(r));
  });
}

int tt_bigq_size(tt_bigq* op, uint64_t* size) {
  TT_ARG(op && size);
  TT_GUARD(*size = (uint64_t)op->op.size());
}

int tt_bigq_davidson(tt_bigq* op, tt_qtensor* x, int max_restart, double tol, double* eval, int* matvecs) {
  TT_ARG(op && x && eval);
  TT_GUARD({
    ttb::DavidsonStats st;
    *eval = ttb::tensor_davidsonIT(op->op, x->t, 3, max_restart, tol, 'S', &st);
    if (matvecs) *matvecs = st.matvecs;
  });
}

int tt_bigq_destroy(tt_bigq* op) { TT_GUARD(delete op); }

// ---- MPS / MPO -----------------------------------------------------------------
int tt_qmps_product_spinhalf(int L, const int* state, unsigned id, tt_qmps** out) {
  TT_ARG(L >= 3 && state && out);
  TT_GUARD({
    std::vector<unsigned> st(state, state + L);
    for (unsigned s : st)
      if (s > 1) throw std::runtime_error("spin-1/2 product state entries must be 0 (Dn) or 1 (Up)");
    tt_qmps* h = new tt_qmps();
    h->psi = ttb::make_product_qmps((unsigned)L, {ttb::QN(-1), ttb::QN(1)}, st, id);
    *out = h;
  });
}

int tt_qmps_destroy(tt_qmps* psi) { TT_GUARD(delete psi); }

int tt_qmps_length(const tt_qmps* psi, int* L) {
  TT_ARG(psi && L);
  TT_GUARD(*L = (int)psi->psi.length);
}

int tt_qmps_bond_dims(const tt_qmps* psi, int* out) {
  TT_ARG(psi && out);
  TT_GUARD({
    for (size_t i = 0; i < psi->psi.bond_dims.size(); ++i) out[i] = (int)psi->psi.bond_dims[i];
  });
}

int tt_qmps_center(const tt_qmps* psi, int* center) {
  TT_ARG(psi && center);
  TT_GUARD(*center = psi->psi.center);
}

int tt_qmps_position(tt_qmps* psi, int site) {
  TT_ARG(psi && site >= 0 && site < (int)psi->psi.length);
  TT_GUARD(psi->psi.position(site));
}

int tt_qmps_tensor(const tt_qmps* psi, int i, tt_qtensor** out) {
  TT_ARG(psi && out && i >= 0 && i < (int)psi->psi.length);
  TT_GUARD(*out = wrap(ttb::qtensor(psi->psi.A[i])));
}

int tt_qmps_data_size(const tt_qmps* psi, int64_t* n) {
  TT_ARG(psi && n);
  TT_GUARD({
    int64_t s = 0;
    for (auto& A : psi->psi.A) s += A.total_size();
    *n = s;
  });
}

int tt_qmps_get_data(const tt_qmps* psi, double* host) {
  TT_ARG(psi && host);
  TT_GUARD({
    int64_t pos = 0;
    for (auto& A : psi->psi.A)
      for (auto& b : A.blocks) {
        ttb::check(tt_memcpy_d2h(ttb::rt().ctx, host + pos, A.data->get() + b.off, sizeof(double) * (size_t)b.size),
                   "qmps get");
        pos += b.size;
      }
  });
}

int tt_qmps_set_data(tt_qmps* psi, const double* host) {
  TT_ARG(psi && host);
  TT_GUARD({
    int64_t pos = 0;
    for (auto& A : psi->psi.A)
      for (auto& b : A.blocks) {
        ttb::check(tt_memcpy_h2d(ttb::rt().ctx, A.data->get() + b.off, host + pos, sizeof(double) * (size_t)b.size),
                   "qmps set");
        pos += b.size;
      }
    ttb::check(tt_ctx_synchronize(ttb::rt().ctx), "qmps set");
  });
}

namespace {
// blocks of sites [first, last) in block order; one asynchronous copy per run
// of blocks that are back to back in the arena, one synchronisation in all
int copy_sites(const tt_qmps* psi, int first, int last, double* host, const double* src_host) {
  TT_ARG(psi && (host || src_host) && first >= 0 && first <= last && last <= (int)psi->psi.length);
  TT_GUARD({
    tt_ctx* ctx = ttb::rt().ctx;
    if (!ctx) throw std::runtime_error("no device context bound");
    cudaStream_t st = nullptr;
    ttb::check(tt_ctx_stream(ctx, reinterpret_cast<void**>(&st)), "stream");
    int64_t pos = 0;
    for (int i = first; i < last; ++i) {
      const ttb::qtensor& A = psi->psi.A[i];
      size_t b = 0;
      while (b < A.blocks.size()) {
        size_t e = b + 1;  // extend the run while the next block follows in the arena
        while (e < A.blocks.size() && A.blocks[e].off == A.blocks[e - 1].off + A.blocks[e - 1].size) ++e;
        const int64_t n = A.blocks[e - 1].off + A.blocks[e - 1].size - A.blocks[b].off;
        double* dev = A.data->get() + A.blocks[b].off;
        const cudaError_t rc =
            host ? cudaMemcpyAsync(host + pos, dev, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st)
                 : cudaMemcpyAsync(dev, src_host + pos, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, st);
        if (rc != cudaSuccess) throw ttb::tt_error(TT_ERR_CUDA, std::string("site copy: ") + cudaGetErrorString(rc));
        pos += n;
        b = e;
      }
    }
    ttb::check(tt_ctx_synchronize(ctx), "site copy");
  });
}
}  // namespace

int tt_qmps_sites_size(const tt_qmps* psi, int first, int last, int64_t* n) {
  TT_ARG(psi && n && first >= 0 && first <= last && last <= (int)psi->psi.length);
  TT_GUARD({
    int64_t s = 0;
    for (int i = first; i < last; ++i) s += psi->psi.A[i].total_size();
    *n = s;
  });
}

int tt_qmps_get_sites(const tt_qmps* psi, int first, int last, double* host) {
  return copy_sites(psi, first, last, host, nullptr);
}

int tt_qmps_set_sites(tt_qmps* psi, int first, int last, const double* host) {
  return copy_sites(psi, first, last, nullptr, host);
}

int tt_qmpo_heisenberg(int L, const double* dh, double tE, unsigned id, tt_qmpo** out) {
  TT_ARG(L >= 3 && out);
  TT_GUARD({
    tt_qmpo* h = new tt_qmpo();
    h->H = ttb::make_heisenberg_qmpo((unsigned)L, dh, tE, id);
    *out = h;
  });
}

int tt_qmpo_destroy(tt_qmpo* H) { TT_GUARD(delete H); }

int tt_qmpo_tensor(const tt_qmpo* H, int i, tt_qtensor** out) {
  TT_ARG(H && out && i >= 0 && i < (int)H->H.length);
  TT_GUARD(*out = wrap(ttb::qtensor(H->H.A[i])));
}

// ---- DMRG ------------------------------------------------------------------------
int tt_qdmrg_create(tt_qmps* psi, tt_qmpo* H, tt_qdmrg** out) {
  TT_ARG(psi && H && out && psi->psi.length == H->H.length);
  TT_GUARD({
    tt_qdmrg* r = new tt_qdmrg();
    r->psi = psi;
    r->H = H;
    try {
      ttb::dmrg_prepare(psi->psi, H->H, r->st, &r->log);
    } catch (...) {
      delete r;
      throw;
    }
    *out = r;
  });
}

int tt_qdmrg_set_noise(tt_qdmrg* run, double noise) {
  TT_ARG(run && noise >= 0.0);
  TT_GUARD(run->st.noise = noise);
}

int tt_qdmrg_sweep(tt_qdmrg* run, int max_bd, double cutoff, int max_restart, double* energy) {
  TT_ARG(run && max_restart >= 1);
  TT_GUARD({
    double e = ttb::dmrg_sweep(run->psi->psi, run->H->H, run->st, max_bd, cutoff, max_restart, &run->log);
    if (energy) *energy = e;
  });
}

int tt_qdmrg_walk(tt_qdmrg* run, int to_site, int max_bd, double cutoff, int max_restart, double* energy) {
  TT_ARG(run && max_restart >= 1 && to_site >= 0 && to_site < (int)run->H->H.length);
  TT_GUARD({
    double e = ttb::dmrg_walk(run->psi->psi, run->H->H, run->st, to_site, max_bd, cutoff, max_restart, &run->log);
    if (energy) *energy = e;
  });
}

int tt_qdmrg_position(const tt_qdmrg* run, int* site) {
  TT_ARG(run && site);
  TT_GUARD(*site = run->st.pos);
}

int tt_qdmrg_finish(tt_qdmrg* run) {
  TT_ARG(run);
  TT_GUARD(ttb::dmrg_finish(run->psi->psi));
}

int tt_qdmrg_destroy(tt_qdmrg* run) { TT_GUARD(delete run); }

int tt_qdmrg_run(tt_qmps* psi, tt_qmpo* H, int nsweeps, const int* maxm, int n_maxm, const double* cutoff,
                 int n_cutoff, const int* max_restart, int n_mr, double* energy, tt_qdmrg** log_out) {
  TT_ARG(psi && H && maxm && cutoff && max_restart && n_maxm > 0 && n_cutoff > 0 && n_mr > 0);
  TT_GUARD({
    tt_qdmrg* r = nullptr;
    int rc = tt_qdmrg_create(psi, H, &r);
    if (rc != TT_OK) return rc;
    double e = 0.0;
    for (int s = 0; s < nsweeps; ++s) {
      rc = tt_qdmrg_sweep(r, maxm[s % n_maxm], cutoff[s % n_cutoff], max_restart[s % n_mr], &e);
      if (rc != TT_OK) {
        delete r;
        return rc;
      }
    }
    ttb::dmrg_finish(psi->psi);
    if (energy) *energy = e;
    if (log_out) *log_out = r; else delete r;
  });
}

int tt_qdmrg_num_steps(const tt_qdmrg* run, int* n) {
  TT_ARG(run && n);
  TT_GUARD(*n = (int)run->log.steps.size());
}

int tt_qdmrg_step(const tt_qdmrg* run, int i, int* site, int* direction, double* energy, double* trunc_err,
                  unsigned* kept, int* matvecs, double* heff_flops) {
  TT_ARG(run && i >= 0 && i < (int)run->log.steps.size());
  TT_GUARD({
    const ttb::StepLog& s = run->log.steps[i];
    if (site) *site = s.site;
    if (direction) *direction = s.direction;
    if (energy) *energy = s.energy;
    if (trunc_err) *trunc_err = s.trunc_err;
    if (kept) *kept = s.kept;
    if (matvecs) *matvecs = s.matvecs;
    if (heff_flops) *heff_flops = s.heff_flops;
  });
}

int tt_qdmrg_step_sectors(const tt_qdmrg* run, int i, int* n, int32_t* qn, uint32_t* kept, int cap) {
  TT_ARG(run && n && i >= 0 && i < (int)run->log.steps.size());
  TT_GUARD({
    const ttb::StepLog& s = run->log.steps[i];
    *n = (int)s.sector_qn.size();
    for (int j = 0; j < *n && j < cap; ++j) {
      if (qn) { qn[2 * j] = s.sector_qn[j].a; qn[2 * j + 1] = s.sector_qn[j].b; }
      if (kept) kept[j] = s.kept_per_sector[j];
    }
  });
}

int tt_qdmrg_step_profile(const tt_qdmrg* run, int i, int* gram_max, double* t_davidson, double* t_svd,
                          double* t_env, double* t_engine) {
  TT_ARG(run && i >= 0 && i < (int)run->log.steps.size());
  TT_GUARD({
    const ttb::StepLog& s = run->log.steps[i];
    if (gram_max) *gram_max = s.gram_max;
    if (t_davidson) *t_davidson = s.t_davidson;
    if (t_svd) *t_svd = s.t_svd;
    if (t_env) *t_env = s.t_env;
    if (t_engine) *t_engine = s.t_engine;
  });
}

int tt_qdmrg_step_device_ms(const tt_qdmrg* run, int i, double* davidson, double* svd, double* env,
                            double* gap) {
  TT_ARG(run && i >= 0 && i < (int)run->log.steps.size());
  TT_GUARD({
    auto span = [](void* a, void* b) -> double {
      if (!a || !b) return -1.0;
      float ms = 0.0f;
      ttb::check(tt_event_elapsed_ms(a, b, &ms), "step event");
      return (double)ms;
    };
    const auto& ev = run->log.steps[i].events;
    void* e[4] = {nullptr, nullptr, nullptr, nullptr};
    if (ev)
      for (int k = 0; k < 4; ++k) e[k] = ev->ev[k];
    void* prev_end = nullptr;
    if (i > 0 && run->log.steps[i - 1].events) prev_end = run->log.steps[i - 1].events->ev[3];
    if (davidson) *davidson = span(e[0], e[1]);
    if (svd) *svd = span(e[1], e[2]);
    if (env) *env = span(e[2], e[3]);
    if (gap) *gap = span(prev_end, e[0]);
  });
}

int tt_qdmrg_stats(const tt_qdmrg* run, double* heff_flops, double* heff_seconds, double* initial_energy) {
  TT_ARG(run);
  TT_GUARD({
    if (heff_flops) *heff_flops = run->log.heff_flops;
    if (heff_seconds) *heff_seconds = run->log.heff_seconds;
    if (initial_energy) *initial_energy = run->log.initial_energy;
  });
}

int tt_qdmrg_env(const tt_qdmrg* run, int which, int i, tt_qtensor** out) {
  TT_ARG(run && out && (which == 0 || which == 1) && i >= 0 && i < (int)run->st.TL.size());
  TT_GUARD({
    const ttb::qtensor& T = which == 0 ? run->st.TL[i] : run->st.TR[i];
    if (!T._initted) throw std::runtime_error("environment not built for this site");
    *out = wrap(ttb::qtensor(T));
  });
}

int tt_qdmrg_num_sweeps(const tt_qdmrg* run, int* n) {
  TT_ARG(run && n);
  TT_GUARD(*n = (int)run->log.sweep_energy.size());
}

int tt_qdmrg_sweep_info(const tt_qdmrg* run, int i, double* energy, double* seconds) {
  TT_ARG(run && i >= 0 && i < (int)run->log.sweep_energy.size());
  TT_GUARD({
    if (energy) *energy = run->log.sweep_energy[i];
    if (seconds) *seconds = run->log.sweep_seconds[i];
  });
}

}  // extern "C"

// ---- dense path ------------------------------------------------------------------
#include "../host/dmrg_d.h"

struct tt_dmps {
  ttb::MPS psi;
};
struct tt_dmpo {
  ttb::MPO H;
};

extern "C" {

int tt_dmps_product_spinhalf(int L, const int* state, unsigned id, tt_dmps** out) {
  TT_ARG(L >= 3 && state && out);
  TT_GUARD({
    std::vector<unsigned> st(state, state + L);
    tt_dmps* h = new tt_dmps();
    h->psi = ttb::make_product_mps((unsigned)L, st, id);
    *out = h;
  });
}

int tt_dmps_destroy(tt_dmps* psi) { TT_GUARD(delete psi); }

int tt_dmps_bond_dims(const tt_dmps* psi, int* out) {
  TT_ARG(psi && out);
  TT_GUARD({
    for (size_t i = 0; i < psi->psi.bond_dims.size(); ++i) out[i] = (int)psi->psi.bond_dims[i];
  });
}

int tt_dmps_length(const tt_dmps* psi, int* L) {
  TT_ARG(psi && L);
  TT_GUARD(*L = (int)psi->psi.length);
}

int tt_dmpo_heisenberg(int L, const double* dh, double tE, unsigned id, tt_dmpo** out) {
  TT_ARG(L >= 3 && out);
  TT_GUARD({
    tt_dmpo* h = new tt_dmpo();
    h->H = ttb::make_heisenberg_mpo((unsigned)L, dh, tE, id);
    *out = h;
  });
}

int tt_dmpo_destroy(tt_dmpo* H) { TT_GUARD(delete H); }

int tt_ddmrg_run(tt_dmps* psi, tt_dmpo* H, int nsweeps, const int* maxm, int n_maxm, const double* cutoff,
                 int n_cutoff, const int* max_restart, int n_mr, double* energy, double* sweep_energy,
                 int* step_kept) {
  TT_ARG(psi && H && maxm && cutoff && max_restart && n_maxm > 0 && n_cutoff > 0 && n_mr > 0 && nsweeps >= 0);
  TT_ARG(psi->psi.length == H->H.length);
  TT_GUARD({
    ttb::DenseDmrgLog log;
    double e = ttb::dmrg(psi->psi, H->H, nsweeps, std::vector<int>(maxm, maxm + n_maxm),
                         std::vector<double>(cutoff, cutoff + n_cutoff),
                         std::vector<int>(max_restart, max_restart + n_mr), &log);
    if (energy) *energy = e;
    if (sweep_energy)
      for (size_t i = 0; i < log.sweep_energy.size(); ++i) sweep_energy[i] = log.sweep_energy[i];
    if (step_kept)
      for (size_t i = 0; i < log.steps.size(); ++i) step_kept[i] = (int)log.steps[i].kept;
  });
}

}  // extern "C"

// ---- AutoMPO and lattices (host-side; only the MPO builders touch the device) ----
#include "../host/autompo.h"

struct tt_autompo {
  ttb::AutoMPO a;
};

extern "C" {

int tt_autompo_create(tt_autompo** out) {
  TT_ARG(out);
  TT_GUARD(*out = new tt_autompo());
}

int tt_autompo_destroy(tt_autompo* a) { TT_GUARD(delete a); }

int tt_autompo_add(tt_autompo* a, double coef, int nops, const char* const* ops, const int* sites) {
  TT_ARG(a && nops > 0 && ops && sites);
  for (int j = 0; j < nops; ++j) TT_ARG(ops[j] && sites[j] >= 0);
  TT_GUARD({
    ttb::HTerm t;
    for (int j = 0; j < nops; ++j) t.add(ops[j], sites[j]);
    t.coef *= coef;
    a->a.add(t);
  });
}

int tt_autompo_size(const tt_autompo* a, int* n) {
  TT_ARG(a && n);
  TT_GUARD(*n = a->a.size());
}

int tt_autompo_term(const tt_autompo* a, int k, double* coef, int* nops, char* names, int* sites, int cap) {
  TT_ARG(a && k >= 0 && k < a->a.size() && cap >= 0);
  TT_GUARD({
    auto it = a->a.terms().begin();
    std::advance(it, k);
    if (coef) *coef = it->coef;
    if (nops) *nops = it->Nops();
    for (int j = 0; j < it->Nops() && j < cap; ++j) {
      if (names) {
        std::strncpy(names + 16 * j, it->ops[j].op.c_str(), 15);
        names[16 * j + 15] = '\0';
      }
      if (sites) sites[j] = it->ops[j].i;
    }
  });
}

int tt_autompo_link_dims(const tt_autompo* a, int N, int with_charges, int* dims) {
  TT_ARG(a && N >= 2 && dims);
  TT_GUARD({
    auto links = ttb::automp_links(a->a, (unsigned)N, with_charges != 0);
    for (int n = 0; n <= N; ++n) dims[n] = (int)links[n].states.size();
  });
}

int tt_qmpo_from_autompo(const tt_autompo* a, int N, unsigned id, tt_qmpo** out) {
  TT_ARG(a && N >= 2 && out);
  TT_GUARD({
    tt_qmpo* h = new tt_qmpo();
    try {
      h->H = ttb::build_qmpo(a->a, (unsigned)N, id);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int tt_dmpo_from_autompo(const tt_autompo* a, int N, unsigned id, tt_dmpo** out) {
  TT_ARG(a && N >= 2 && out);
  TT_GUARD({
    tt_dmpo* h = new tt_dmpo();
    try {
      h->H = ttb::build_mpo(a->a, (unsigned)N, id);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int tt_dmpo_tensor(const tt_dmpo* H, int i, int64_t* dims, double* data, int64_t cap) {
  TT_ARG(H && dims && i >= 0 && i < (int)H->H.length);
  TT_GUARD({
    const ttb::dtensor& T = H->H.A[i];
    int64_t n = 1;
    for (int j = 0; j < 4; ++j) {
      dims[j] = T.idx_set[j].size;
      n *= dims[j];
    }
    if (data) {
      if (cap < n) throw std::runtime_error("tt_dmpo_tensor: buffer too small");
      std::vector<double> h = T.get();
      std::memcpy(data, h.data(), sizeof(double) * (size_t)n);
    }
  });
}

int tt_lattice(int kind, int Nx, int Ny, int yperiodic, tt_lattice_bond* bonds, int cap, int* n_bonds) {
  TT_ARG(Nx >= 1 && Ny >= 1 && n_bonds && cap >= 0 && (bonds || cap == 0));
  TT_GUARD({
    std::vector<ttb::LatticeBond> g;
    const bool snake = (kind & TT_LATTICE_SNAKE) != 0;
    kind &= ~TT_LATTICE_SNAKE;
    if (snake && kind == TT_LATTICE_TRIANGULAR)
      throw std::runtime_error("tt_lattice: snake order needs a square lattice");
    if (kind == TT_LATTICE_SQUARE)
      g = ttb::square_lattice(Nx, Ny, yperiodic != 0);
    else if (kind == TT_LATTICE_SQUARE_NEXT_NEIGHBOR)
      g = ttb::square_next_neighbor(Nx, Ny, yperiodic != 0);
    else if (kind == TT_LATTICE_TRIANGULAR)
      g = ttb::triangular_lattice(Nx, Ny, yperiodic != 0);
    else
      throw std::runtime_error("tt_lattice: unknown lattice kind");
    if (snake) ttb::snake_relabel(g, Nx, Ny);
    *n_bonds = (int)g.size();
    for (int j = 0; j < (int)g.size() && j < cap; ++j)
      bonds[j] = tt_lattice_bond{g[j].s1, g[j].s2, g[j].type, g[j].x1, g[j].y1, g[j].x2, g[j].y2};
  });
}

}  // extern "C"

// ---- observables ------------------------------------------------------------------
#include "../host/observables.h"

namespace {
template <class Psi>
void copy_sz(const Psi& psi, double* sz, double* szsz) {
  std::vector<double> a, b;
  ttb::measure_sz(psi, a, b);
  if (sz) std::memcpy(sz, a.data(), sizeof(double) * a.size());
  if (szsz) std::memcpy(szsz, b.data(), sizeof(double) * b.size());
}
}  // namespace

extern "C" {

int tt_qmps_overlap(const tt_qmps* psi, const tt_qmps* phi, double* out) {
  TT_ARG(psi && phi && out);
  TT_GUARD(*out = ttb::psiphi(psi->psi, phi->psi));
}

int tt_qmps_expectation(const tt_qmps* psi, const tt_qmpo* H, const tt_qmps* phi, double* out) {
  TT_ARG(psi && H && phi && out);
  TT_GUARD(*out = ttb::psiHphi(psi->psi, H->H, phi->psi));
}

int tt_qmps_measure_sz(const tt_qmps* psi, double* sz, double* szsz) {
  TT_ARG(psi);
  TT_GUARD(copy_sz(psi->psi, sz, szsz));
}

int tt_dmps_overlap(const tt_dmps* psi, const tt_dmps* phi, double* out) {
  TT_ARG(psi && phi && out);
  TT_GUARD(*out = ttb::psiphi(psi->psi, phi->psi));
}

int tt_dmps_expectation(const tt_dmps* psi, const tt_dmpo* H, const tt_dmps* phi, double* out) {
  TT_ARG(psi && H && phi && out);
  TT_GUARD(*out = ttb::psiHphi(psi->psi, H->H, phi->psi));
}

int tt_dmps_measure_sz(const tt_dmps* psi, double* sz, double* szsz) {
  TT_ARG(psi);
  TT_GUARD(copy_sz(psi->psi, sz, szsz));
}

}  // extern "C"

// ---- checkpoints -------------------------------------------------------------------
#include "../host/checkpoint.h"

extern "C" {

int tt_qmps_save(const tt_qmps* psi, const char* fn, const char* wfn) {
  TT_ARG(psi && fn && *fn);
  TT_GUARD(ttb::save(psi->psi, fn, wfn ? wfn : ""));
}

int tt_qmps_load(const char* fn, const char* data_prefix, tt_qmps** out) {
  TT_ARG(fn && out);
  TT_GUARD({
    ttb::qMPS p = ttb::load_qmps(fn, data_prefix ? data_prefix : "");
    tt_qmps* h = new tt_qmps();
    h->psi = std::move(p);
    *out = h;
  });
}

int tt_dmps_save(const tt_dmps* psi, const char* fn, const char* wfn) {
  TT_ARG(psi && fn && *fn);
  TT_GUARD(ttb::save(psi->psi, fn, wfn ? wfn : ""));
}

int tt_dmps_load(const char* fn, const char* data_prefix, tt_dmps** out) {
  TT_ARG(fn && out);
  TT_GUARD({
    ttb::MPS p = ttb::load_mps(fn, data_prefix ? data_prefix : "");
    tt_dmps* h = new tt_dmps();
    h->psi = std::move(p);
    *out = h;
  });
}

}  // extern "C"
