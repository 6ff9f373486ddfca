// Dense path: dtensor, big_dtensor, dense SVD, restarted Davidson, dense DMRG
// (reference lines in dmrg_d.h).  Every dense contraction is one grouped-GEMM
// pair over strided modes; plans depend only on shapes and are cached.
#include "dmrg_d.h"
#include "observables.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>

namespace ttb {

namespace {

tt_ctx* ctx() {
  if (!rt().ctx) throw std::runtime_error("ttb: no device context bound");
  return rt().ctx;
}

std::vector<int64_t> strides_of(const std::vector<dtensor_index>& idx) {
  std::vector<int64_t> s(idx.size(), 1);
  for (size_t i = 1; i < idx.size(); ++i) s[i] = s[i - 1] * idx[i - 1].size;
  return s;
}

double read1(double* d) {
  double h;
  check(tt_memcpy_d2h(ctx(), &h, d, sizeof(double)), "d2h");
  return h;
}

struct Ax {
  int64_t dim, s1, s2;
};
int put_modes(const std::vector<Ax>& ax, int32_t* dims, int64_t* st1, int64_t* st2) {
  std::vector<Ax> r;
  for (auto& a : ax)
    if (a.dim != 1) {
      if (!r.empty() && a.s1 == r.back().s1 * r.back().dim && (!st2 || a.s2 == r.back().s2 * r.back().dim)) {
        r.back().dim *= a.dim;
        continue;
      }
      r.push_back(a);
    }
  if (r.size() > TT_MAX_MODES) throw std::runtime_error("dtensor: too many modes");
  for (size_t i = 0; i < r.size(); ++i) {
    dims[i] = (int32_t)r[i].dim;
    st1[i] = r[i].s1;
    if (st2) st2[i] = r[i].s2;
  }
  return (int)r.size();
}

// A plan for C(M x N) = A(M x K) B(K x N) with the given strided views; cached
// by the complete pair description (dense blocks start at offset 0).
std::shared_ptr<PlanHandle> dense_plan(const tt_block_pair& p, int64_t M, int64_t N, int64_t a_size,
                                       int64_t b_size, int64_t ldc, int precision = TT_PREC_FP64) {
  std::vector<int64_t> key;
  key.push_back(precision);
  key.push_back(M);
  key.push_back(N);
  key.push_back(ldc);
  key.push_back(p.n_m);
  key.push_back(p.n_k);
  key.push_back(p.n_n);
  key.push_back(p.a_off);
  key.push_back(p.b_off);
  for (int i = 0; i < p.n_m; ++i) { key.push_back(p.m_dims[i]); key.push_back(p.a_m_stride[i]); }
  for (int i = 0; i < p.n_k; ++i) {
    key.push_back(p.k_dims[i]);
    key.push_back(p.a_k_stride[i]);
    key.push_back(p.b_k_stride[i]);
  }
  for (int i = 0; i < p.n_n; ++i) { key.push_back(p.n_dims[i]); key.push_back(p.b_n_stride[i]); }
  auto& cache = rt().dense_plans;
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  std::vector<tt_out_block> outs{tt_out_block{0, (int32_t)M, (int32_t)N, (int32_t)ldc}};
  std::vector<tt_block_pair> pairs{p};
  validate_pairs(outs, pairs, a_size, b_size, ldc * std::max<int64_t>(N, 1));
  tt_plan* h = nullptr;
  check(tt_contract_plan(ctx(), outs.data(), 1, pairs.data(), 1, precision, &h), "dense plan");
  auto ph = std::make_shared<PlanHandle>(h);
  if (cache.size() > 4096) cache.clear();
  cache[key] = ph;
  return ph;
}

}  // namespace

// ---- dtensor ----------------------------------------------------------------
dtensor::dtensor(const std::vector<dtensor_index>& idx, bool zero) : idx_set(idx), rank((unsigned)idx.size()) {
  size = 1;
  for (auto& i : idx_set) size *= i.size;
  data = dev_alloc(size);
  if (zero) data->zero();
  _initted = true;
}

dtensor::dtensor(const dtensor& o) : idx_set(o.idx_set), rank(o.rank), size(o.size), _initted(o._initted) {
  if (o.data) {
    data = dev_alloc(size);
    check(tt_memcpy_d2d(ctx(), data->get(), o.data->get(), sizeof(double) * (size_t)size), "dtensor copy");
  }
}

dtensor& dtensor::operator=(const dtensor& o) {
  if (this != &o) {
    dtensor t(o);
    *this = std::move(t);
  }
  return *this;
}

void dtensor::setOne() {
  std::vector<double> h((size_t)size, 1.0);
  set(h.data());
}

std::vector<double> dtensor::get() const {
  std::vector<double> h((size_t)size);
  check(tt_memcpy_d2h(ctx(), h.data(), data->get(), sizeof(double) * h.size()), "dtensor get");
  return h;
}

void dtensor::set(const double* host) {
  check(tt_memcpy_h2d(ctx(), data->get(), host, sizeof(double) * (size_t)size), "dtensor set");
  check(tt_ctx_synchronize(ctx()), "sync");
}

dtensor& dtensor::operator*=(double c) {
  check(tt_vec_scal(ctx(), size, c, data->get()), "scale");
  return *this;
}

dtensor& dtensor::operator/=(double c) { return (*this) *= (1.0 / c); }

double dtensor::norm() const {
  check(tt_vec_nrm2(ctx(), size, data->get(), scalar_slot(0)), "norm");
  return read1(scalar_slot(0));
}

double dtensor::normalize() {
  double r = norm();
  (*this) /= r;
  return r;
}

// A's data laid out in this tensor's index order (indices matched by tag)
static DevPtr aligned(const dtensor& self, const dtensor& A) {
  bool same = A.rank == self.rank;
  for (unsigned i = 0; same && i < self.rank; ++i) same = self.idx_set[i].same_tag(A.idx_set[i]);
  if (same) return A.data;
  std::vector<int64_t> sA = strides_of(A.idx_set), sT = strides_of(self.idx_set);
  tt_copy_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n_modes = (int32_t)self.rank;
  if (self.rank > TT_MAX_MODES) throw std::runtime_error("dtensor: rank too large");
  for (unsigned j = 0; j < self.rank; ++j) {
    int src = -1;
    for (unsigned i = 0; i < A.rank; ++i)
      if (A.idx_set[i].same_tag(self.idx_set[j])) src = (int)i;
    if (src < 0) throw std::runtime_error("dtensor: index sets differ");
    d.dims[j] = (int32_t)self.idx_set[j].size;
    d.src_stride[j] = sA[src];
    d.dst_stride[j] = sT[j];
  }
  DevPtr tmp = dev_alloc(self.size);
  check(tt_strided_copy_batched(ctx(), &d, 1, A.data->get(), tmp->get()), "dtensor align");
  return tmp;
}

void dtensor::add(const dtensor& A, double c) {
  DevPtr a = aligned(*this, A);
  check(tt_vec_axpy(ctx(), size, c, a->get(), data->get()), "axpy");
}

double dtensor::inner_product(const dtensor& A) const {
  DevPtr a = aligned(*this, A);
  check(tt_vec_dot(ctx(), size, data->get(), a->get(), scalar_slot(0)), "dot");
  return read1(scalar_slot(0));
}

double dtensor::contract(const dtensor& A) const {
  if (A.size != size) throw std::runtime_error("dtensor::contract: size mismatch");
  check(tt_vec_dot(ctx(), size, data->get(), A.data->get(), scalar_slot(0)), "dot");
  return read1(scalar_slot(0));
}

dtensor dtensor::diagonal(index_type type) const {
  // dtensor.cpp:511-571: indices without a similar partner, then for every
  // similar pair the one with the lower prime level; primes are ignored when
  // labelling, so a pair reads the diagonal
  std::vector<dtensor_index> nidx;
  std::vector<std::vector<unsigned>> srcs;  // original axes behind each new axis
  for (unsigned i = 0; i < rank; ++i) {
    bool shared = false;
    for (unsigned j = 0; j < rank; ++j)
      if (idx_set[i].similar(idx_set[j], type)) { shared = true; break; }
    if (!shared) {
      nidx.push_back(idx_set[i]);
      srcs.push_back({i});
    }
  }
  for (unsigned i = 0; i < rank; ++i)
    for (unsigned j = i + 1; j < rank; ++j)
      if (idx_set[i].similar(idx_set[j], type)) {
        nidx.push_back(idx_set[i].level < idx_set[j].level ? idx_set[i] : idx_set[j]);
        srcs.push_back({i, j});
        break;
      }
  if (nidx.size() == rank) return dtensor(*this);
  dtensor D(nidx, false);
  std::vector<int64_t> s = strides_of(idx_set), sD = strides_of(nidx);
  tt_copy_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n_modes = (int32_t)nidx.size();
  for (size_t a = 0; a < nidx.size(); ++a) {
    d.dims[a] = (int32_t)nidx[a].size;
    d.dst_stride[a] = sD[a];
    for (unsigned o : srcs[a]) d.src_stride[a] += s[o];
  }
  check(tt_strided_copy_batched(ctx(), &d, 1, data->get(), D.data->get()), "diagonal");
  return D;
}

dtensor operator*(const dtensor& A, const dtensor& B) {
  // dtensor.cpp:300-368: indices whose tag appears in both are summed
  if (A._initted && !B._initted) return A;
  if (B._initted && !A._initted) return B;
  std::vector<int> pa(A.rank, -1), pb(B.rank, -1);
  for (unsigned i = 0; i < A.rank; ++i)
    for (unsigned j = 0; j < B.rank; ++j)
      if (pb[j] < 0 && A.idx_set[i].same_tag(B.idx_set[j])) {
        pa[i] = (int)j;
        pb[j] = (int)i;
        break;
      }
  std::vector<dtensor_index> cidx;
  for (unsigned i = 0; i < A.rank; ++i)
    if (pa[i] < 0) cidx.push_back(A.idx_set[i]);
  for (unsigned j = 0; j < B.rank; ++j)
    if (pb[j] < 0) cidx.push_back(B.idx_set[j]);
  if (cidx.empty()) throw std::runtime_error("dtensor operator*: full contraction to a scalar is not supported");
  std::vector<int64_t> sA = strides_of(A.idx_set), sB = strides_of(B.idx_set);
  std::vector<Ax> mm, km, nm;
  int64_t M = 1, N = 1;
  for (unsigned i = 0; i < A.rank; ++i) {
    if (pa[i] < 0) {
      mm.push_back({A.idx_set[i].size, sA[i], 0});
      M *= A.idx_set[i].size;
    } else {
      km.push_back({A.idx_set[i].size, sA[i], sB[pa[i]]});
    }
  }
  for (unsigned j = 0; j < B.rank; ++j)
    if (pb[j] < 0) {
      nm.push_back({B.idx_set[j].size, sB[j], 0});
      N *= B.idx_set[j].size;
    }
  tt_block_pair p;
  std::memset(&p, 0, sizeof(p));
  p.n_m = put_modes(mm, p.m_dims, p.a_m_stride, nullptr);
  p.n_k = put_modes(km, p.k_dims, p.a_k_stride, p.b_k_stride);
  p.n_n = put_modes(nm, p.n_dims, p.b_n_stride, nullptr);
  dtensor C(cidx, false);
  auto plan = dense_plan(p, M, N, A.size, B.size, std::max<int64_t>(M, 1), rt().precision);
  check(tt_contract_exec(ctx(), plan->get(), A.data->get(), B.data->get(), C.data->get(), 1.0), "dense contract");
  return C;
}

// ---- dense SVD ----------------------------------------------------------------
void dsvd(const dtensor& A, const std::vector<dtensor_index>& left, const std::vector<dtensor_index>& right,
          dtensor& U, dtensor& V, dtensor& S, int direction, double cutoff, unsigned long K) {
  std::vector<int64_t> sA = strides_of(A.idx_set);
  auto axis_of = [&](const dtensor_index& ix) {
    for (unsigned i = 0; i < A.rank; ++i)
      if (A.idx_set[i].same_tag(ix)) return i;
    throw std::runtime_error("dsvd: index not in tensor");
  };
  int64_t r = 1, c = 1;
  std::vector<Ax> lax, rax;  // (dim, stride in A, running stride in the r x c matrix)
  for (auto& ix : left) {
    lax.push_back({ix.size, sA[axis_of(ix)], r});
    r *= ix.size;
  }
  for (auto& ix : right) {
    rax.push_back({ix.size, sA[axis_of(ix)], c});
    c *= ix.size;
  }
  const bool fl = direction == MoveFromLeft;
  const int64_t g = fl ? r : c;
  DevPtr G = dev_alloc(g * g), Z = dev_alloc(g * g), W = dev_alloc(g), T = dev_alloc(3 * g);
  tt_eig_problem ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.n = (int32_t)g;
  DevPtr packed;
  const bool row12 = r == 1 && c == 2;
  if (row12 && !fl) {
    ep.flags = TT_EIG_ROW_1X2;
    packed = dev_alloc(2);
    tt_copy_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_modes = 0;
    int nm = 0;
    for (auto& a : rax)
      if (a.dim != 1) {
        d.dims[nm] = (int32_t)a.dim;
        d.src_stride[nm] = a.s1;
        d.dst_stride[nm] = a.s2;
        ++nm;
      }
    d.n_modes = nm;
    check(tt_strided_copy_batched(ctx(), &d, 1, A.data->get(), packed->get()), "dsvd pack");
  } else {
    // Gram matrix: rows (left) x rows, or cols (right) x cols
    tt_block_pair p;
    std::memset(&p, 0, sizeof(p));
    std::vector<Ax> m_ax = fl ? lax : rax, k_ax = fl ? rax : lax;
    std::vector<Ax> mm, km, nm;
    for (auto& a : m_ax) mm.push_back({a.dim, a.s1, 0});
    for (auto& a : k_ax) km.push_back({a.dim, a.s1, a.s1});
    for (auto& a : m_ax) nm.push_back({a.dim, a.s1, 0});
    p.n_m = put_modes(mm, p.m_dims, p.a_m_stride, nullptr);
    p.n_k = put_modes(km, p.k_dims, p.a_k_stride, p.b_k_stride);
    p.n_n = put_modes(nm, p.n_dims, p.b_n_stride, nullptr);
    auto plan = dense_plan(p, g, g, A.size, A.size, g);
    check(tt_contract_exec(ctx(), plan->get(), A.data->get(), A.data->get(), G->get(), 1.0), "dsvd gram");
  }
  check(tt_sym_eigvals_batched(ctx(), &ep, 1, G->get(), T->get(), W->get(), packed ? packed->get() : nullptr),
        "dsvd eigenvalues");
  std::vector<double> w((size_t)g);
  check(tt_memcpy_d2h(ctx(), w.data(), W->get(), sizeof(double) * w.size()), "dsvd d2h");
  const int64_t nvals = std::min(r, c);
  int64_t keep = nvals;
  if (!row12) {
    if (K) keep = std::min<int64_t>(keep, (int64_t)K);
    if (cutoff > 0) {
      int64_t above = 0;
      for (int64_t i = 0; i < nvals; ++i)
        if (std::sqrt(std::fabs(w[(size_t)i])) > cutoff) ++above;
      keep = std::min(keep, above);
    }
    keep = std::max<int64_t>(keep, 1);
  }
  int nv = (int)keep;
  DevPtr work = dev_alloc(3 * g * g);
  check(tt_sym_eigvecs_batched(ctx(), &ep, 1, &nv, G->get(), T->get(), W->get(), Z->get(), work->get(),
                               packed ? packed->get() : nullptr),
        "dsvd eigenvectors");
  dtensor_index mid(keep, "dsvdmid", Link, 0);
  std::vector<dtensor_index> uidx(left), vidx{mid};
  uidx.push_back(mid);
  vidx.insert(vidx.end(), right.begin(), right.end());
  U = dtensor(uidx, false);
  V = dtensor(vidx, false);
  if (fl) {
    // U = Z[:, :keep] (same column-major layout); V = Z^T A
    check(tt_memcpy_d2d(ctx(), U.data->get(), Z->get(), sizeof(double) * (size_t)(r * keep)), "dsvd U");
    tt_block_pair p;
    std::memset(&p, 0, sizeof(p));
    std::vector<Ax> mm{{keep, r, 0}}, km, nm;
    for (auto& a : lax) km.push_back({a.dim, a.s2, a.s1});
    for (auto& a : rax) nm.push_back({a.dim, a.s1, 0});
    p.n_m = put_modes(mm, p.m_dims, p.a_m_stride, nullptr);
    p.n_k = put_modes(km, p.k_dims, p.a_k_stride, p.b_k_stride);
    p.n_n = put_modes(nm, p.n_dims, p.b_n_stride, nullptr);
    auto plan = dense_plan(p, keep, c, g * g, A.size, keep);
    check(tt_contract_exec(ctx(), plan->get(), Z->get(), A.data->get(), V.data->get(), 1.0), "dsvd V");
  } else {
    // V = Z[:, :keep]^T; U = A V^T
    tt_copy_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_modes = 2;
    d.dims[0] = (int32_t)keep;
    d.dims[1] = (int32_t)c;
    d.src_stride[0] = c;
    d.src_stride[1] = 1;
    d.dst_stride[0] = 1;
    d.dst_stride[1] = keep;
    check(tt_strided_copy_batched(ctx(), &d, 1, Z->get(), V.data->get()), "dsvd V");
    tt_block_pair p;
    std::memset(&p, 0, sizeof(p));
    std::vector<Ax> mm, km, nm{{keep, c, 0}};
    for (auto& a : lax) mm.push_back({a.dim, a.s1, 0});
    for (auto& a : rax) km.push_back({a.dim, a.s1, a.s2});
    p.n_m = put_modes(mm, p.m_dims, p.a_m_stride, nullptr);
    p.n_k = put_modes(km, p.k_dims, p.a_k_stride, p.b_k_stride);
    p.n_n = put_modes(nm, p.n_dims, p.b_n_stride, nullptr);
    auto plan = dense_plan(p, r, keep, A.size, g * g, r);
    check(tt_contract_exec(ctx(), plan->get(), A.data->get(), Z->get(), U.data->get(), 1.0), "dsvd U");
  }
  S = dtensor(std::vector<dtensor_index>{mid}, false);
  std::vector<double> s((size_t)keep);
  for (int64_t i = 0; i < keep; ++i) s[(size_t)i] = std::sqrt(std::fabs(w[(size_t)i]));
  S.set(s.data());
}

void dsvd_bond(const dtensor& combined, dtensor& A_left, dtensor& A_right, dtensor_index& mid, dtensor& S,
               int direction, double cutoff, unsigned long K) {
  // dtensor_op.cpp:86-115
  std::vector<dtensor_index> left, right;
  for (auto& ix : A_right.idx_set)
    if (!ix.same_tag(mid)) right.push_back(ix);
  for (auto& ix : A_left.idx_set)
    if (!ix.same_tag(mid)) left.push_back(ix);
  dtensor U, V;
  dsvd(combined, left, right, U, V, S, direction, cutoff, K);
  mid.size = S.size;
  A_right = std::move(V);
  A_right.idx_set[0] = mid;
  A_left = std::move(U);
  A_left.idx_set.back() = mid;
}

// ---- big_dtensor --------------------------------------------------------------
dtensor big_dtensor::product(dtensor& v) {
  dtensor res;
  if (L_) res = (*L_) * v;
  for (auto* m : mid_) res = res.rank > 0 ? res * (*m) : v * (*m);
  if (R_) res = res * (*R_);
  res.prime(-1);
  return res;
}

double big_dtensor::expec(dtensor& v) {
  dtensor r = product(v);
  return r.contract(v);
}

dtensor big_dtensor::diagonal() {
  dtensor res;
  if (L_) res = L_->diagonal(Link);
  for (auto* m : mid_) {
    dtensor dm = m->diagonal(Site);
    res = res * dm;
  }
  if (R_) {
    dtensor dR = R_->diagonal(Link);
    res = res * dR;
  }
  return res;
}

size_t big_dtensor::size() const {
  if (size_ == 0) {
    size_ = 1;
    for (dtensor* T : {L_, R_})
      if (T)
        for (auto& ix : T->idx_set)
          if (ix.level > 0) size_ *= (size_t)ix.size;
  }
  for (auto* m : mid_)
    for (auto& ix : m->idx_set)
      if (ix.type == Site) size_ *= (size_t)ix.size;
  return size_;
}

// ---- restarted Davidson (tensor_davidson.cpp:74-184) ----------------------------
double tensor_davidson(big_dtensor& A, dtensor& x, int m, int max_restart, double tol, char mode,
                       DavidsonStats* stats) {
  if (!(m >= 1 && max_restart >= 1 && tol > 0)) throw std::runtime_error("tensor_davidson: bad arguments");
  std::vector<dtensor> v(m), va(m);
  dtensor D = A.diagonal();
  std::vector<double> M((size_t)(m + 1) * (m + 1), 0.0), Mnext((size_t)(m + 1) * (m + 1), 0.0), evals(m, 0.0);
  double eval = 0.0, r_norm = 0.0;
  dtensor u, ua, r;
  for (int i = 0; i < max_restart; ++i) {
    for (int j = 0; j < m; ++j) {
      v[j] = x;
      for (int k = j - 1; k >= 0; --k) {
        double alpha = v[k].inner_product(v[j]);
        v[j].add(v[k], -alpha);
      }
      v[j].normalize();
      va[j] = A.product(v[j]);
      if (stats) stats->matvecs++;
      int l = j;
      for (int k = 0; k < j + 1; ++k) {
        M[l + k * (j + 1)] = va[l].inner_product(v[k]);
        M[k + l * (j + 1)] = M[l + k * (j + 1)];
      }
      for (int k = 0; k < j + 1; ++k)
        for (int l2 = 0; l2 <= k; ++l2) {
          Mnext[l2 + k * (j + 2)] = M[l2 + k * (j + 1)];
          Mnext[k + l2 * (j + 2)] = M[k + l2 * (j + 1)];
        }
      if (j > 0) {
        DIAG(j + 1, M.data(), evals.data());
        const bool low = mode == 'S';
        eval = low ? evals[0] : evals[j];
        for (int k = 0; k < j + 1; ++k) {
          double coef = low ? M[k] : M[k + j * (j + 1)];
          if (k == 0) {
            u = v[k];
            u *= coef;
            ua = va[k];
            ua *= coef;
          } else {
            u.add(v[k], coef);
            ua.add(va[k], coef);
          }
        }
      } else {
        eval = M[0];
        u = v[0];
        ua = va[0];
      }
      ua.add(u, -eval);
      r = ua;
      r_norm = r.norm();
      if (j < m - 1) {
        x = r;
        // elemWiseDivide (tensor_davidson.cpp:25-36)
        DevPtr d = aligned(x, D);
        check(tt_vec_precondition(ctx(), x.size, x.data->get(), d->get(), eval), "precondition");
        x.normalize();
      }
      std::swap(M, Mnext);
    }
    x = u;
    if (stats) stats->iters++;
    if (r_norm < tol) break;
  }
  return eval;
}

// ---- MPS / MPO ----------------------------------------------------------------
MPS make_product_mps(unsigned L, const std::vector<unsigned>& state, unsigned id) {
  // mps/tt.cpp:225-262: 1 on the chosen spin, DBL_EPSILON elsewhere
  if (state.size() != L || L < 3) throw std::runtime_error("make_product_mps: bad length");
  MPS psi;
  psi.length = L;
  psi.id = id;
  psi.bond_dims.assign(L + 1, 1);
  for (unsigned i = 0; i < L; ++i) {
    dtensor T({dtensor_index(1, psi.link_name(i)), dtensor_index(2, "Site" + std::to_string(i), Site),
               dtensor_index(1, psi.link_name(i + 1))},
              false);
    double h[2] = {DBL_EPSILON, DBL_EPSILON};
    if (state[i] > 1) throw std::runtime_error("make_product_mps: spin-1/2 states are 0 or 1");
    h[state[i]] = 1.0;
    T.set(h);
    psi.A.push_back(std::move(T));
  }
  psi.center = -1;
  return psi;
}

MPO make_heisenberg_mpo(unsigned L, const double* dh, double tE, unsigned id) {
  // models/hams/Heisenberg.cpp:185-208 with addOperators :72-148 (D = 5)
  MPO H;
  H.length = L;
  H.id = id;
  std::string pref = "ID" + std::to_string(id) + "Link";
  std::vector<std::vector<double>> host(L);
  std::vector<std::vector<int64_t>> dims(L);
  for (unsigned i = 0; i < L; ++i) {
    int64_t dl = i == 0 ? 1 : 5, dr = i == L - 1 ? 1 : 5;
    dims[i] = {dl, dr};
    host[i].assign((size_t)(dl * 4 * dr), 0.0);
    H.A.emplace_back(std::vector<dtensor_index>{dtensor_index(dl, pref + std::to_string(i)),
                                                dtensor_index(2, "Site" + std::to_string(i), Site, 0),
                                                dtensor_index(2, "Site" + std::to_string(i), Site, 1),
                                                dtensor_index(dr, pref + std::to_string(i + 1))},
                     false);
  }
  auto add = [&](unsigned site, unsigned r, unsigned c, const std::string& op, double val) {
    int64_t dl = dims[site][0];
    for (unsigned k = 0; k < 2; ++k)
      for (unsigned b = 0; b < 2; ++b) {
        int64_t rr = site == 0 ? 0 : r;
        host[site][(size_t)(rr + dl * (k + 2 * (b + 2 * (int64_t)c)))] = val * spin_half_op(b, op, k);
      }
  };
  for (unsigned site = 0; site < L; ++site) {
    bool last = site == L - 1;
    if (site > 0) add(site, 0, 0, "Id", 1.0);
    if (!last) add(site, 1, 1, "Id", 1.0);
    if (dh) add(site, 1, 0, "Sz", dh[site]);
    if (tE != 0) add(site, 1, 0, "Id", -tE / L);
    if (site > 0) add(site, 2, 0, "Sz", 1.0);
    if (!last) add(site, 1, 2, "Sz", 1.0);
    if (site > 0) add(site, 3, 0, "S+", 1.0);
    if (!last) add(site, 1, 3, "S-", 0.5);
    if (site > 0) add(site, 4, 0, "S-", 1.0);
    if (!last) add(site, 1, 4, "S+", 0.5);
  }
  for (unsigned i = 0; i < L; ++i) H.A[i].set(host[i].data());
  return H;
}

double MPS::position(int site) {
  // mps/tt.cpp:575-612 (rc) and :739-795
  auto move_left = [&](int c) {
    std::string ln = link_name((unsigned)c);
    std::vector<dtensor_index> left, right;
    dtensor_index mid;
    for (auto& ix : A[c].idx_set) {
      if (ix.name == ln) { left.push_back(ix); mid = ix; } else right.push_back(ix);
    }
    dtensor U, V, S;
    dsvd(A[c], left, right, U, V, S, MoveFromRight);
    mid.size = S.size;
    bond_dims[c] = (unsigned)S.size;
    A[c] = std::move(V);
    A[c].idx_set[0] = mid;
    A[c - 1] = A[c - 1] * U;
    A[c - 1].idx_set.back() = mid;
  };
  if (center == -1) {
    for (int i = (int)length - 1; i > 0; --i) move_left(i);
    center = 0;
  }
  if (center == site) return 0.0;
  while (center != site) {
    if (center > site) {
      move_left(center);
      --center;
    } else {
      std::string ln = link_name((unsigned)center + 1);
      std::vector<dtensor_index> left, right;
      dtensor_index mid;
      for (auto& ix : A[center].idx_set) {
        if (ix.name == ln) { right.push_back(ix); mid = ix; } else left.push_back(ix);
      }
      dtensor U, V, S;
      dsvd(A[center], left, right, U, V, S, MoveFromLeft);
      mid.size = S.size;
      bond_dims[center + 1] = (unsigned)S.size;
      A[center] = std::move(U);
      A[center].idx_set.back() = mid;
      A[center + 1] = V * A[center + 1];
      A[center + 1].idx_set[0] = mid;
      ++center;
    }
  }
  return 0.0;
}

void MPS::normalize() {
  double nm = A[center].norm();
  A[center] /= nm;
}

// ---- environments and the sweep ------------------------------------------------
static dtensor dboundary(const dtensor_index& psi_ix, const dtensor_index& h_ix) {
  dtensor_index a = psi_ix;
  a.prime();  // primeLink
  dtensor T({a, h_ix, psi_ix}, false);
  T.setOne();
  return T;
}

static dtensor denv_step(const dtensor& env, const dtensor& Ai, const dtensor& W) {
  dtensor t1;
  t1.idx_set = Ai.idx_set;
  t1.rank = Ai.rank;
  t1.size = Ai.size;
  t1.data = Ai.data;  // shares the data: only the indices are primed
  t1._initted = true;
  t1.prime();
  dtensor t4 = t1 * env;
  dtensor t5 = t4 * W;
  return t5 * Ai;
}

double dmrg(MPS& psi, MPO& H, int num_sweeps, const std::vector<int>& max_bd, const std::vector<double>& cutoff,
            const std::vector<int>& max_restart, DenseDmrgLog* log) {
  const unsigned L = H.length;
  psi.position(0);
  psi.normalize();
  std::vector<dtensor> TR(L), TL(L);
  TL[0] = dboundary(psi.A[0].idx_set[0], H.A[0].idx_set[0]);
  TR[L - 1] = dboundary(psi.A[L - 1].idx_set.back(), H.A[L - 1].idx_set.back());
  for (unsigned i = L - 1; i > 0; --i) TR[i - 1] = denv_step(TR[i], psi.A[i], H.A[i]);
  double energy = 0.0;
  for (int sweep = 0; sweep < num_sweeps; ++sweep) {
    int lbd = sweep % (int)max_bd.size(), lc = sweep % (int)cutoff.size(), lmr = sweep % (int)max_restart.size();
    for (int half = 0; half < 2; ++half) {
      int direction = half == 0 ? MoveFromLeft : MoveFromRight;
      for (unsigned i = 0; i < L - 1; ++i) {
        unsigned site = direction == MoveFromLeft ? i : L - 1 - i;
        unsigned l = direction == MoveFromLeft ? site : site - 1, r = l + 1;
        big_dtensor A;
        A.setLeft(&TL[l]);
        A.addMid(&H.A[l]);
        A.addMid(&H.A[r]);
        A.setRight(&TR[r]);
        dtensor x = psi.A[l] * psi.A[r];
        DavidsonStats st;
        // mixed-precision products only where the two-site space is large
        // enough that the Krylov vectors cannot exhaust it (their relative
        // error of about 1e-7 keeps the residual above the tolerance, and in
        // an exhausted space the extra directions are product noise)
        const int heff_prec = x.size <= 4096 ? TT_PREC_FP64 : rt().heff_precision;
        {
          PrecisionScope prec(heff_prec);
          energy = tensor_davidson(A, x, 3, max_restart[lmr], 1e-12, 'S', &st);
        }
        if (heff_prec != TT_PREC_FP64 && half == 1 && i == L - 2) {
          // mixed precision: the sweep's energy is the FP64 Rayleigh quotient
          dtensor y = A.product(x);
          energy = x.inner_product(y) / x.inner_product(x);
        }
        dtensor_index mid;
        for (auto& ix : psi.A[l].idx_set)
          if (ix.name == psi.link_name(r)) { mid = ix; break; }
        dtensor S;
        dsvd_bond(x, psi.A[l], psi.A[r], mid, S, direction, cutoff[lc], (unsigned long)max_bd[lbd]);
        psi.bond_dims[r] = (unsigned)S.size;
        psi.center = (int)(direction == MoveFromLeft ? r : l);
        {
          PrecisionScope prec(rt().env_precision);
          if (direction == MoveFromLeft)
            TL[site + 1] = denv_step(TL[site], psi.A[site], H.A[site]);
          else
            TR[site - 1] = denv_step(TR[site], psi.A[site], H.A[site]);
        }
        if (log) log->steps.push_back(DenseStepLog{(int)site, direction, st.matvecs, energy, (unsigned)S.size});
      }
    }
    if (rt().env_precision != TT_PREC_FP64) {
      // mixed-precision environments bias the Ritz value to first order: the
      // sweep energy is <psi|H|psi> / <psi|psi> contracted in FP64
      PrecisionScope prec(TT_PREC_FP64);
      energy = psiHphi(psi, H, psi) / psiphi(psi, psi);
    }
    if (log) {
      log->sweep_energy.push_back(energy);
      log->sweep_bond_dims.push_back(psi.bond_dims);
    }
  }
  psi.position(0);
  psi.normalize();
  return energy;
}

}  // namespace ttb
