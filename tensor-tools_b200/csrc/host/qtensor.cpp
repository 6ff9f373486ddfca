// Host mirror of qtensor: block structure on the host, numbers on the GPU.
#include "qtensor.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <sstream>

namespace ttb {

// ---- runtime ------------------------------------------------------------
Runtime& rt() {
  static thread_local Runtime r;
  return r;
}

void check(int status, const char* what) {
  if (status != TT_OK) {
    std::string msg = std::string(what) + ": " + tt_get_last_error();
    throw tt_error(status, msg);
  }
}

static void drop_dav_state() {
  if (rt().dav) tt_dav_state_destroy(rt().ctx, rt().dav);
  rt().dav = nullptr;
}

void bind_context(tt_ctx* c) {
  clear_contraction_cache();  // cached plans belong to the previous context
  rt().dense_plans.clear();
  rt().scalars.reset();
  rt().heff_scratch[0].reset();
  rt().heff_scratch[1].reset();
  drop_dav_state();
  rt().ctx = c;
  if (c) rt().scalars = std::make_shared<DevBuf>(kScalarSlots);
}
void unbind_context() {
  clear_contraction_cache();
  rt().dense_plans.clear();
  rt().scalars.reset();
  rt().heff_scratch[0].reset();
  rt().heff_scratch[1].reset();
  drop_dav_state();
  rt().ctx = nullptr;
}
double* scalar_slot(int i) { return rt().scalars->get() + i; }

static tt_ctx* ctx() {
  if (!rt().ctx) throw std::runtime_error("ttb: no device context bound (tt_dmrg_bind)");
  return rt().ctx;
}

DevBuf::DevBuf(int64_t n) : n_(n) {
  void* p = nullptr;
  check(tt_device_alloc(ctx(), sizeof(double) * (size_t)std::max<int64_t>(n, 2), &p), "device alloc");
  p_ = static_cast<double*>(p);
}
DevBuf::~DevBuf() {
  if (p_ && rt().ctx) tt_device_free(rt().ctx, p_);
}
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    if (p_ && rt().ctx) tt_device_free(rt().ctx, p_);
    p_ = o.p_;
    n_ = o.n_;
    o.p_ = nullptr;
    o.n_ = 0;
  }
  return *this;
}
void DevBuf::zero() {
  if (n_ > 0) check(tt_memset_zero(ctx(), p_, sizeof(double) * (size_t)n_), "memset");
}
DevPtr dev_alloc(int64_t n) { return std::make_shared<DevBuf>(n); }

PlanHandle::~PlanHandle() {
  if (p_ && rt().ctx) tt_plan_destroy(rt().ctx, p_);
}

// ---- qtensor_index --------------------------------------------------------
void qtensor_index::addQN(QN q, unsigned dim) {
  qn_.push_back({q, dim});
  std::stable_sort(qn_.begin(), qn_.end(),
                   [](const std::pair<QN, unsigned>& x, const std::pair<QN, unsigned>& y) {
                     return x.first < y.first;
                   });
}
int64_t qtensor_index::dim() const {
  int64_t d = 0;
  for (auto& p : qn_) d += p.second;
  return d;
}
std::string qtensor_index::tag_string() const {
  std::ostringstream s;
  s << (arrow_ == Inward ? "in " : "out ") << level_ << " " << name_ << " " << type_ << " ";
  for (auto& p : qn_) s << "qn" << p.first.a << "," << p.first.b << "qdim" << p.second << " ";
  return s.str();
}

// ---- qtensor ----------------------------------------------------------------
qtensor::qtensor(const qtensor& o)
    : idx_set(o.idx_set), rank(o.rank), blocks(o.blocks), block_id(o.block_id), arena(o.arena),
      _initted(o._initted) {
  if (o.data) {
    data = dev_alloc(o.arena);
    check(tt_memcpy_d2d(ctx(), data->get(), o.data->get(), sizeof(double) * (size_t)o.arena), "copy");
  }
}

qtensor& qtensor::operator=(const qtensor& o) {
  if (this != &o) {
    qtensor tmp(o);
    *this = std::move(tmp);
  }
  return *this;
}

QNKey qtensor::key_of(unsigned b) const {
  QNKey k(rank);
  for (unsigned j = 0; j < rank; ++j) k[j] = blocks[b].qn[j].pack();
  return k;
}

int qtensor::find_block(const QNKey& k) const {
  auto it = block_id.find(k);
  return it == block_id.end() ? -1 : (int)it->second;
}

unsigned qtensor::add_block_meta(std::vector<QN> qn, std::vector<unsigned> qi, std::vector<int> qd) {
  BlockMeta b;
  b.size = 1;
  for (int d : qd) b.size *= d;
  b.qn = std::move(qn);
  b.qi = std::move(qi);
  b.qd = std::move(qd);
  blocks.push_back(std::move(b));
  unsigned id = (unsigned)blocks.size() - 1;
  block_id[key_of(id)] = id;
  return id;
}

void qtensor::allocate(bool zero) {
  int64_t off = 0;
  for (auto& b : blocks) {
    b.off = off;
    off += b.size;
  }
  arena = off;
  data = dev_alloc(arena);
  if (zero) data->zero();
}

int64_t qtensor::total_size() const {
  int64_t s = 0;
  for (auto& b : blocks) s += b.size;
  return s;
}

void qtensor::initBlock() {
  // qtensor.cpp:301-345: all sector combinations, first index fastest
  if (rank > 0 && !_initted) {
    std::vector<uint64_t> stride(rank + 1, 1);
    for (unsigned i = 0; i < rank; ++i) stride[i + 1] = stride[i] * idx_set[i].size();
    for (uint64_t i = 0; i < stride[rank]; ++i) {
      std::vector<unsigned> pos(rank);
      std::vector<int> qds(rank);
      std::vector<QN> qns(rank);
      QN tot(0, 0);
      for (unsigned j = 0; j < rank; ++j) {
        pos[j] = (unsigned)((i / stride[j]) % idx_set[j].size());
        qns[j] = idx_set[j].qn(pos[j]);
        qds[j] = (int)idx_set[j].qdim(pos[j]);
        if (idx_set[j].arrow() == Inward) tot += qns[j]; else tot -= qns[j];
      }
      if (tot == QN(0, 0)) add_block_meta(qns, pos, qds);
    }
    allocate(true);
  }
  _initted = true;
}

void qtensor::setZero() {
  if (data) data->zero();
}

void qtensor::setOne() {
  std::vector<double> ones((size_t)arena, 1.0);
  check(tt_memcpy_h2d(ctx(), data->get(), ones.data(), sizeof(double) * ones.size()), "setOne");
}

void qtensor::setRandom() {
  if (arena == 0) return;
  std::vector<int64_t> ranges;
  for (auto& b : blocks) {
    ranges.push_back(b.off);
    ranges.push_back(b.off + b.size);
  }
  // sort ranges by begin for the device-side binary search
  std::vector<std::pair<int64_t, int64_t>> r;
  for (size_t i = 0; i < ranges.size(); i += 2) r.push_back({ranges[i], ranges[i + 1]});
  std::sort(r.begin(), r.end());
  std::vector<int64_t> flat;
  for (auto& p : r) { flat.push_back(p.first); flat.push_back(p.second); }
  void* d = nullptr;
  check(tt_device_alloc(ctx(), sizeof(int64_t) * flat.size(), &d), "alloc");
  check(tt_memcpy_h2d(ctx(), d, flat.data(), sizeof(int64_t) * flat.size()), "h2d");
  check(tt_vec_fill_random(ctx(), arena, data->get(), (int)r.size(), (const int64_t*)d,
                           rt().rng_counter++),
        "setRandom");
  tt_ctx_synchronize(ctx());
  tt_device_free(ctx(), d);
}

qtensor& qtensor::operator*=(double c) {
  if (arena) check(tt_vec_scal(ctx(), arena, c, data->get()), "scale");
  return *this;
}

qtensor& qtensor::operator/=(double c) {
  return (*this) *= (1.0 / c);
}

static double read_scalar(double* d) {
  double h = 0.0;
  check(tt_memcpy_d2h(ctx(), &h, d, sizeof(double)), "d2h");
  return h;
}

double qtensor::norm() const {
  if (arena == 0) return 0.0;
  check(tt_vec_nrm2(ctx(), arena, data->get(), scalar_slot(0)), "norm");
  return read_scalar(scalar_slot(0));
}

double qtensor::normalize() {
  double r = norm();
  (*this) *= (1.0 / r);
  return r;
}

// Copy of A's blocks placed at this tensor's offsets (blocks matched by QN
// key in each tensor's own index order, as block_id_by_qn_str does); blocks
// of this tensor that A lacks are zero.  Index permutations between the two
// are applied by tag.
static DevPtr aligned_copy(const qtensor& self, const qtensor& A) {
  DevPtr tmp = dev_alloc(self.arena);
  tmp->zero();
  std::vector<unsigned> perm(self.rank);  // self axis j <- A axis perm[j]
  for (unsigned j = 0; j < self.rank; ++j) {
    perm[j] = self.rank;
    for (unsigned i = 0; i < A.rank; ++i)
      if (A.idx_set[i].level() == self.idx_set[j].level() && A.idx_set[i].name() == self.idx_set[j].name() &&
          A.idx_set[i].type() == self.idx_set[j].type() && A.idx_set[i].sectors() == self.idx_set[j].sectors()) {
        perm[j] = i;
        break;
      }
    if (perm[j] == self.rank) perm[j] = j;
  }
  std::vector<tt_copy_desc> descs;
  for (unsigned b = 0; b < A.blocks.size(); ++b) {
    int t = self.find_block(A.key_of(b));
    if (t < 0) continue;
    const BlockMeta& ab = A.blocks[b];
    const BlockMeta& tb = self.blocks[t];
    tt_copy_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_modes = (int)self.rank;
    d.src_off = ab.off;
    d.dst_off = tb.off;
    std::vector<int64_t> sA(A.rank, 1), sT(self.rank, 1);
    for (unsigned i = 1; i < A.rank; ++i) sA[i] = sA[i - 1] * ab.qd[i - 1];
    for (unsigned i = 1; i < self.rank; ++i) sT[i] = sT[i - 1] * tb.qd[i - 1];
    for (unsigned j = 0; j < self.rank; ++j) {
      d.dims[j] = tb.qd[j];
      d.dst_stride[j] = sT[j];
      d.src_stride[j] = sA[perm[j]];
    }
    if (d.n_modes > TT_MAX_MODES) throw std::runtime_error("aligned_copy: rank too large");
    descs.push_back(d);
  }
  for (size_t i = 0; i < descs.size(); i += 65535) {
    int n = (int)std::min<size_t>(65535, descs.size() - i);
    check(tt_strided_copy_batched(ctx(), descs.data() + i, n, A.data->get(), tmp->get()), "aligned copy");
  }
  return tmp;
}

static bool same_layout(const qtensor& a, const qtensor& b) {
  if (a.arena != b.arena || a.blocks.size() != b.blocks.size() || a.rank != b.rank) return false;
  for (unsigned i = 0; i < a.rank; ++i)
    if (!a.idx_set[i].same_tag(b.idx_set[i])) return false;
  for (size_t i = 0; i < a.blocks.size(); ++i)
    if (a.blocks[i].off != b.blocks[i].off || a.blocks[i].qn != b.blocks[i].qn) return false;
  return true;
}

void qtensor::add(const qtensor& A, double c) {
  // qtensor.cpp:1127-1156: matching blocks accumulate, missing ones are inserted
  if (A.rank != rank) throw std::runtime_error("add: rank mismatch");
  std::vector<unsigned> missing;
  for (unsigned b = 0; b < A.blocks.size(); ++b)
    if (find_block(A.key_of(b)) < 0) missing.push_back(b);
  if (!missing.empty()) {
    int64_t old = arena;
    int64_t off = arena;
    for (unsigned b : missing) {
      unsigned id = add_block_meta(A.blocks[b].qn, A.blocks[b].qi, A.blocks[b].qd);
      blocks[id].off = off;
      off += blocks[id].size;
    }
    DevPtr nd = dev_alloc(off);
    nd->zero();
    if (old) check(tt_memcpy_d2d(ctx(), nd->get(), data->get(), sizeof(double) * (size_t)old), "grow");
    data = nd;
    arena = off;
  }
  if (same_layout(*this, A)) {
    check(tt_vec_axpy(ctx(), arena, c, A.data->get(), data->get()), "axpy");
  } else {
    DevPtr tmp = aligned_copy(*this, A);
    check(tt_vec_axpy(ctx(), arena, c, tmp->get(), data->get()), "axpy");
  }
}

double qtensor::inner_product(const qtensor& A) const {
  // qtensor.cpp:1161-1179: sum over this tensor's blocks that A also has
  if (arena == 0) return 0.0;
  if (same_layout(*this, A)) {
    check(tt_vec_dot(ctx(), arena, data->get(), A.data->get(), scalar_slot(0)), "dot");
  } else {
    DevPtr tmp = aligned_copy(*this, A);
    check(tt_vec_dot(ctx(), arena, data->get(), tmp->get(), scalar_slot(0)), "dot");
  }
  return read_scalar(scalar_slot(0));
}

double qtensor::contract(const qtensor& A) const { return inner_product(A); }

std::vector<double> qtensor::get_block(unsigned b) const {
  std::vector<double> h((size_t)blocks.at(b).size);
  check(tt_memcpy_d2h(ctx(), h.data(), block_ptr(b), sizeof(double) * h.size()), "get_block");
  return h;
}

void qtensor::set_block(unsigned b, const double* host) {
  check(tt_memcpy_h2d(ctx(), block_ptr(b), host, sizeof(double) * (size_t)blocks.at(b).size), "set_block");
  check(tt_ctx_synchronize(ctx()), "sync");
}

// ---- contraction ----------------------------------------------------------
namespace {

struct Mode {
  int64_t dim;
  int64_t s1, s2;  // strides in the one or two operands that carry the mode
};

// drop unit modes and merge adjacent modes that are contiguous in every operand
std::vector<Mode> simplify(std::vector<Mode> m, bool two) {
  std::vector<Mode> r;
  for (auto& x : m)
    if (x.dim != 1) r.push_back(x);
  std::vector<Mode> out;
  for (auto& x : r) {
    if (!out.empty()) {
      Mode& y = out.back();
      bool c1 = x.s1 == y.s1 * y.dim;
      bool c2 = !two || x.s2 == y.s2 * y.dim;
      if (c1 && c2) {
        y.dim *= x.dim;
        continue;
      }
    }
    out.push_back(x);
  }
  return out;
}

std::vector<int64_t> colmajor_strides(const std::vector<int>& qd) {
  std::vector<int64_t> s(qd.size(), 1);
  for (size_t i = 1; i < qd.size(); ++i) s[i] = s[i - 1] * qd[i - 1];
  return s;
}

}  // namespace

static void contract_structure_impl(const qtensor& A, const qtensor& B, ContractStructure& out) {
  // mark repeated indices (qtensor.cpp:540-555)
  std::vector<std::pair<qtensor_index, int>> marker;
  auto find = [&](const qtensor_index& ix) -> int* {
    for (auto& m : marker)
      if (m.first.same_tag(ix)) return &m.second;
    return nullptr;
  };
  auto put = [&](const qtensor_index& ix, int v) {
    int* p = find(ix);
    if (p) *p = v; else marker.push_back({ix, v});
  };
  std::vector<std::pair<unsigned, unsigned>> idx_pair;
  for (unsigned i = 0; i < A.rank; ++i) put(A.idx_set[i], (int)i);
  for (unsigned i = 0; i < B.rank; ++i) {
    qtensor_index tp = B.idx_set[i];
    tp.dag();
    int* hit = find(tp);
    if (!hit) {
      put(B.idx_set[i], (int)i);
    } else {
      idx_pair.push_back({(unsigned)*hit, i});
      *hit = -1;
      put(B.idx_set[i], -1);
    }
  }
  std::vector<unsigned> A_perm, B_perm;
  for (unsigned i = 0; i < A.rank; ++i)
    if (*find(A.idx_set[i]) != -1) A_perm.push_back(i);
  for (auto& p : idx_pair) {
    A_perm.push_back(p.first);
    B_perm.push_back(p.second);
  }
  for (unsigned i = 0; i < B.rank; ++i)
    if (*find(B.idx_set[i]) != -1) B_perm.push_back(i);
  if (A_perm.size() != A.rank || B_perm.size() != B.rank)
    throw std::runtime_error("operator*: inconsistent index pairing");
  const unsigned nrep = (unsigned)idx_pair.size();
  const unsigned nA = A.rank - nrep;
  std::vector<qtensor_index> Aix(A.rank), Bix(B.rank);
  for (unsigned i = 0; i < A.rank; ++i) Aix[i] = A.idx_set[A_perm[i]];
  for (unsigned i = 0; i < B.rank; ++i) Bix[i] = B.idx_set[B_perm[i]];

  std::unordered_map<QNKey, unsigned, QNKeyHash> A_id, B_id;
  for (unsigned i = 0; i < A.blocks.size(); ++i) {
    QNKey k(A.rank);
    for (unsigned j = 0; j < A.rank; ++j) k[j] = A.blocks[i].qn[A_perm[j]].pack();
    A_id[k] = i;
  }
  for (unsigned i = 0; i < B.blocks.size(); ++i) {
    QNKey k(B.rank);
    for (unsigned j = 0; j < B.rank; ++j) k[j] = B.blocks[i].qn[B_perm[j]].pack();
    B_id[k] = i;
  }
  std::vector<qtensor_index> res_idx;
  for (unsigned i = 0; i < nA; ++i) res_idx.push_back(Aix[i]);
  for (unsigned i = nrep; i < B.rank; ++i) res_idx.push_back(Bix[i]);
  if (res_idx.empty()) throw std::runtime_error("operator*: full contraction to a scalar is not supported");
  out.C = qtensor(res_idx);
  out.a_size = A.arena;
  out.b_size = B.arena;
  out.C._initted = true;
  out.outs.clear();
  out.pairs.clear();
  out.flops = 0.0;

  std::set<QN> mid_set;
  std::map<QN, std::set<std::vector<unsigned>>> left_qi, mid_qi, right_qi;
  for (unsigned i = 0; i < A.blocks.size(); ++i) {
    QN m(0, 0);
    std::vector<unsigned> lq;
    for (unsigned j = 0; j < nA; ++j) {
      lq.push_back(A.blocks[i].qi[A_perm[j]]);
      if (Aix[j].arrow() == Inward) m += A.blocks[i].qn[A_perm[j]]; else m -= A.blocks[i].qn[A_perm[j]];
    }
    mid_set.insert(m);
    left_qi[m].insert(lq);
  }
  for (unsigned i = 0; i < B.blocks.size(); ++i) {
    QN m(0, 0);
    std::vector<unsigned> rq, mq;
    for (unsigned j = nrep; j < B.rank; ++j) {
      rq.push_back(B.blocks[i].qi[B_perm[j]]);
      if (Bix[j].arrow() == Inward) m -= B.blocks[i].qn[B_perm[j]]; else m += B.blocks[i].qn[B_perm[j]];
    }
    for (unsigned j = 0; j < nrep; ++j) mq.push_back(B.blocks[i].qi[B_perm[j]]);
    right_qi[m].insert(rq);
    mid_qi[m].insert(mq);
  }

  // output blocks in the reference's order; C offsets back to back
  int64_t coff = 0;
  for (const QN& q : mid_set) {
    const auto& rset = right_qi[q];
    const auto& lset = left_qi[q];
    const auto& mset = mid_qi[q];
    for (const auto& rq : rset) {
      for (const auto& lq : lset) {
        std::vector<QN> qn;
        std::vector<unsigned> qi;
        std::vector<int> qd;
        int64_t M = 1, N = 1;
        for (unsigned i = 0; i < lq.size(); ++i) {
          qi.push_back(lq[i]);
          qd.push_back((int)Aix[i].qdim(lq[i]));
          qn.push_back(Aix[i].qn(lq[i]));
          M *= qd.back();
        }
        for (unsigned i = 0; i < rq.size(); ++i) {
          qi.push_back(rq[i]);
          qd.push_back((int)Bix[nrep + i].qdim(rq[i]));
          qn.push_back(Bix[nrep + i].qn(rq[i]));
          N *= qd.back();
        }
        unsigned cid = out.C.add_block_meta(qn, qi, qd);
        out.C.blocks[cid].off = coff;
        tt_out_block ob;
        ob.c_off = coff;
        ob.m = (int32_t)M;
        ob.n = (int32_t)N;
        ob.ldc = (int32_t)std::max<int64_t>(M, 1);
        coff += M * N;
        out.outs.push_back(ob);
        for (const auto& mq : mset) {
          QNKey ak(A.rank), bk(B.rank);
          for (unsigned i = 0; i < nA; ++i) ak[i] = qn[i].pack();
          for (unsigned i = 0; i < nrep; ++i) {
            ak[nA + i] = Aix[nA + i].qn(mq[i]).pack();
            bk[i] = Bix[i].qn(mq[i]).pack();
          }
          for (unsigned i = 0; i < rq.size(); ++i) bk[nrep + i] = qn[nA + i].pack();
          auto ait = A_id.find(ak);
          auto bit = B_id.find(bk);
          if (ait == A_id.end() || bit == B_id.end()) continue;
          const BlockMeta& ab = A.blocks[ait->second];
          const BlockMeta& bb = B.blocks[bit->second];
          std::vector<int64_t> sA = colmajor_strides(ab.qd), sB = colmajor_strides(bb.qd);
          std::vector<Mode> mm, km, nm;
          for (unsigned j = 0; j < nA; ++j) mm.push_back({ab.qd[A_perm[j]], sA[A_perm[j]], 0});
          int64_t K = 1;
          for (auto& p : idx_pair) {
            km.push_back({ab.qd[p.first], sA[p.first], sB[p.second]});
            K *= ab.qd[p.first];
          }
          for (unsigned j = nrep; j < B.rank; ++j) nm.push_back({bb.qd[B_perm[j]], sB[B_perm[j]], 0});
          mm = simplify(mm, false);
          km = simplify(km, true);
          nm = simplify(nm, false);
          if (mm.size() > TT_MAX_MODES || km.size() > TT_MAX_MODES || nm.size() > TT_MAX_MODES)
            throw std::runtime_error("operator*: too many non-contiguous modes");
          tt_block_pair bp;
          std::memset(&bp, 0, sizeof(bp));
          bp.out_block = (int32_t)out.outs.size() - 1;
          bp.a_off = ab.off;
          bp.b_off = bb.off;
          bp.n_m = (int32_t)mm.size();
          bp.n_k = (int32_t)km.size();
          bp.n_n = (int32_t)nm.size();
          for (size_t i = 0; i < mm.size(); ++i) { bp.m_dims[i] = (int32_t)mm[i].dim; bp.a_m_stride[i] = mm[i].s1; }
          for (size_t i = 0; i < km.size(); ++i) {
            bp.k_dims[i] = (int32_t)km[i].dim;
            bp.a_k_stride[i] = km[i].s1;
            bp.b_k_stride[i] = km[i].s2;
          }
          for (size_t i = 0; i < nm.size(); ++i) { bp.n_dims[i] = (int32_t)nm[i].dim; bp.b_n_stride[i] = nm[i].s1; }
          out.pairs.push_back(bp);
          out.flops += 2.0 * (double)M * (double)N * (double)K;
        }
      }
    }
  }
  out.C.arena = coff;
}

void validate_pairs(const std::vector<tt_out_block>& outs, const std::vector<tt_block_pair>& pairs,
                    int64_t a_size, int64_t b_size, int64_t c_size) {
  for (const auto& o : outs) {
    if (o.m < 0 || o.n < 0 || o.ldc < std::max(o.m, 1) || o.c_off < 0)
      throw tt_error(TT_ERR_INVALID, "contraction: bad output block");
    if (o.m > 0 && o.n > 0 && o.c_off + (int64_t)(o.m - 1) + (int64_t)o.ldc * (o.n - 1) >= c_size)
      throw tt_error(TT_ERR_INVALID, "contraction: output block outside C");
  }
  for (const auto& p : pairs) {
    if (p.out_block < 0 || p.out_block >= (int)outs.size())
      throw tt_error(TT_ERR_INVALID, "contraction: pair without output block");
    int64_t amax = p.a_off, bmax = p.b_off, m = 1, n = 1;
    for (int i = 0; i < p.n_m; ++i) { amax += (int64_t)(p.m_dims[i] - 1) * p.a_m_stride[i]; m *= p.m_dims[i]; }
    for (int i = 0; i < p.n_k; ++i) {
      amax += (int64_t)(p.k_dims[i] - 1) * p.a_k_stride[i];
      bmax += (int64_t)(p.k_dims[i] - 1) * p.b_k_stride[i];
    }
    for (int i = 0; i < p.n_n; ++i) { bmax += (int64_t)(p.n_dims[i] - 1) * p.b_n_stride[i]; n *= p.n_dims[i]; }
    for (int i = 0; i < p.n_m; ++i) if (p.a_m_stride[i] < 0 || p.m_dims[i] < 1) throw tt_error(TT_ERR_INVALID, "contraction: bad m mode");
    for (int i = 0; i < p.n_k; ++i) if (p.a_k_stride[i] < 0 || p.b_k_stride[i] < 0 || p.k_dims[i] < 1) throw tt_error(TT_ERR_INVALID, "contraction: bad k mode");
    for (int i = 0; i < p.n_n; ++i) if (p.b_n_stride[i] < 0 || p.n_dims[i] < 1) throw tt_error(TT_ERR_INVALID, "contraction: bad n mode");
    if (p.a_off < 0 || p.b_off < 0 || amax >= a_size || bmax >= b_size)
      throw tt_error(TT_ERR_INVALID, "contraction: block pair reaches outside its operand");
    if (m != outs[p.out_block].m || n != outs[p.out_block].n)
      throw tt_error(TT_ERR_INVALID, "contraction: pair shape differs from its output block");
  }
}

void contract_structure(const qtensor& A, const qtensor& B, ContractStructure& out) {
  auto t0 = std::chrono::steady_clock::now();
  contract_structure_impl(A, B, out);
  rt().t_structure += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  rt().n_structure++;
}

namespace {

void serialize(const qtensor& T, std::vector<int64_t>& k) {
  k.push_back(T.rank);
  for (const auto& ix : T.idx_set) {
    k.push_back(((int64_t)ix.arrow() << 40) | ((int64_t)ix.type() << 32) | ix.level());
    k.push_back((int64_t)ix.name().size());
    int64_t w = 0;
    int nb = 0;
    for (char ch : ix.name()) {
      w = (w << 8) | (unsigned char)ch;
      if (++nb == 8) { k.push_back(w); w = 0; nb = 0; }
    }
    if (nb) k.push_back(w);
    k.push_back((int64_t)ix.size());
    for (const auto& s : ix.sectors()) {
      k.push_back(s.first.pack());
      k.push_back(s.second);
    }
  }
  k.push_back((int64_t)T.blocks.size());
  k.push_back(T.arena);
  for (const auto& b : T.blocks) {
    for (const QN& q : b.qn) k.push_back(q.pack());
    for (int d : b.qd) k.push_back(d);
    for (unsigned i : b.qi) k.push_back(i);
    k.push_back(b.off);
  }
}

struct CacheEntry {
  std::vector<int64_t> key;
  std::shared_ptr<CachedContraction> val;
};
struct ContractionCache {
  std::unordered_map<uint64_t, std::vector<CacheEntry>> map;
  size_t entries = 0;
  int64_t plan_bytes = 0;  // device bytes held by the cached plans
  uint64_t clock = 0;      // lookups so far (least recently used entries go first)
  int64_t evictions = 0, evicted = 0;
};
ContractionCache& cache() {
  static thread_local ContractionCache c;
  return c;
}
constexpr size_t kCacheMax = 16384;
// Plans hold device tables; at large bond dimension every step brings new
// block structures, so the cache is also bounded by the device bytes its
// plans hold.  Over either bound the least recently used entries are dropped
// until both are below 3/4 of it: clearing everything made every structure
// of the next steps a cold miss (a second of host planning per block step at
// bond dimension 3072).  Dropping an entry frees only plans nobody else holds
// (a Davidson call keeps its own references).
constexpr int64_t kCachePlanBytesMax = (int64_t)8 << 30;

void evict_lru() {
  ContractionCache& c = cache();
  std::vector<std::pair<uint64_t, std::pair<uint64_t, size_t>>> all;  // (last use, (hash, index))
  for (auto& kv : c.map)
    for (size_t i = 0; i < kv.second.size(); ++i) all.push_back({kv.second[i].val->last_use, {kv.first, i}});
  std::sort(all.begin(), all.end());
  std::unordered_map<uint64_t, std::vector<size_t>> drop;
  size_t entries = c.entries;
  int64_t bytes = c.plan_bytes;
  for (auto& e : all) {
    if (entries <= kCacheMax * 3 / 4 && bytes <= kCachePlanBytesMax * 3 / 4) break;
    const CacheEntry& ce = c.map[e.second.first][e.second.second];
    bytes -= ce.val->plan_bytes;
    entries--;
    drop[e.second.first].push_back(e.second.second);
  }
  for (auto& kv : drop) {
    auto& bucket = c.map[kv.first];
    std::sort(kv.second.rbegin(), kv.second.rend());
    for (size_t i : kv.second) bucket.erase(bucket.begin() + (long)i);
    if (bucket.empty()) c.map.erase(kv.first);
  }
  c.evictions++;
  c.evicted += (int64_t)(c.entries - entries);
  c.entries = entries;
  c.plan_bytes = bytes;
}

}  // namespace

void clear_contraction_cache() {
  cache().map.clear();
  cache().entries = 0;
  cache().plan_bytes = 0;
}

size_t contraction_cache_size() { return cache().entries; }
void contraction_cache_stats(int64_t* entries, int64_t* plan_bytes, int64_t* evictions, int64_t* evicted) {
  if (entries) *entries = (int64_t)cache().entries;
  if (plan_bytes) *plan_bytes = cache().plan_bytes;
  if (evictions) *evictions = cache().evictions;
  if (evicted) *evicted = cache().evicted;
}

std::shared_ptr<const CachedContraction> contract_cached(const qtensor& A, const qtensor& B, bool need_plan) {
  std::vector<int64_t> key;
  key.reserve(64 + 8 * (A.blocks.size() + B.blocks.size()) * (A.rank + B.rank));
  serialize(A, key);
  key.push_back(-1);
  serialize(B, key);
  uint64_t h = 1469598103934665603ull;
  for (int64_t v : key) h = (h ^ (uint64_t)v) * 1099511628211ull;
  auto& bucket = cache().map[h];
  std::shared_ptr<CachedContraction> val;
  for (auto& e : bucket)
    if (e.key == key) {
      val = e.val;
      break;
    }
  if (!val) {
    if (cache().entries >= kCacheMax || cache().plan_bytes >= kCachePlanBytesMax) {
      evict_lru();
      return contract_cached(A, B, need_plan);
    }
    val = std::make_shared<CachedContraction>();
    contract_structure(A, B, val->cs);
    cache().map[h].push_back(CacheEntry{std::move(key), val});
    cache().entries++;
  }
  val->last_use = ++cache().clock;
  if (need_plan) val->plan_for(rt().precision);
  return val;
}

tt_plan* CachedContraction::plan_for(int precision, int keep) const {
  if (precision < TT_PREC_FP64 || precision > TT_PREC_TF32X3_AUTO) throw std::runtime_error("plan_for: bad precision");
  if (cs.outs.empty()) return nullptr;
  if (!plans[precision]) {
    plans[precision] = make_plan(cs, precision, keep);
    int64_t b = 0;
    if (tt_plan_device_bytes(plans[precision]->get(), &b) == TT_OK) {
      cache().plan_bytes += b;
      plan_bytes += b;
    }
  }
  return plans[precision]->get();
}

PrecisionScope::PrecisionScope(int p) : saved(rt().precision) { rt().precision = p; }
PrecisionScope::~PrecisionScope() { rt().precision = saved; }

std::shared_ptr<PlanHandle> make_plan(const ContractStructure& cs, int precision, int keep) {
  auto t0 = std::chrono::steady_clock::now();
  struct Acc {
    std::chrono::steady_clock::time_point t0;
    ~Acc() {
      rt().t_plan += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      rt().n_plan++;
    }
  } acc{t0};
  validate_pairs(cs.outs, cs.pairs, cs.a_size, cs.b_size, cs.C.arena);
  tt_plan* p = nullptr;
  check(tt_contract_plan_keep(ctx(), cs.outs.data(), (int)cs.outs.size(), cs.pairs.data(), (int)cs.pairs.size(),
                              precision, keep, &p),
        "contract plan");
  return std::make_shared<PlanHandle>(p);
}

qtensor operator*(const qtensor& A, const qtensor& B) {
  if (!A._initted && !B._initted) throw std::runtime_error("operator*: both operands uninitialised");
  if (A._initted && !B._initted) return qtensor(A);
  if (B._initted && !A._initted) return qtensor(B);
  auto cc = contract_cached(A, B, false);
  qtensor C = cc->cs.C;  // metadata only (C has no data yet)
  C.data = dev_alloc(C.arena);
  if (tt_plan* p = cc->plan_for(rt().precision))
    check(tt_contract_exec(ctx(), p, A.data->get(), B.data->get(), C.data->get(), 1.0), "contract exec");
  return C;
}

std::vector<unsigned> find_index_permutation(const std::vector<qtensor_index>& from,
                                             const std::vector<qtensor_index>& to) {
  std::vector<unsigned> perm;
  for (size_t i = 0; i < to.size(); ++i)
    for (size_t j = 0; j < from.size(); ++j)
      if (to[i] == from[j]) {
        perm.push_back((unsigned)j);
        break;
      }
  if (perm.size() != to.size()) throw std::runtime_error("find_index_permutation: index not found");
  return perm;
}

double calcEntropy(const qtensor& S, double cutoff) {
  double e = 0.0;
  for (unsigned b = 0; b < S.blocks.size(); ++b)
    for (double s : S.get_block(b))
      if (s > cutoff) e += -(s * s) * std::log(s * s);
  return e;
}

}  // namespace ttb
