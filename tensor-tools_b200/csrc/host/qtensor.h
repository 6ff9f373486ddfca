// Host mirror of tensor-tools' U(1) block-sparse tensor (qtensor) whose block
// data lives in one device arena and whose arithmetic goes through the C ABI
// (include/tt_b200.h).  Block structure, sector order and the rules that
// create, match and drop blocks restate the reference exactly; only the
// numbers move to the GPU.
//
// Reference: util/QN.h:79-127 (QN_t_2), qtensor/qtensor_index.h:35-118,
// qtensor/qtensor.h:47-164, qtensor/qtensor.cpp (initBlock :301-345,
// operator* :523-734, vector ops :1031-1179,1606-1647),
// qtensor/qtensor_op.cpp:1097-1544 (svd, svd_bond).
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../../include/tt_b200.h"

namespace ttb {

// ---- runtime ------------------------------------------------------------
class DevBuf;
struct Runtime {
  tt_ctx* ctx = nullptr;
  uint64_t rng_counter = 0x5eed;
  std::shared_ptr<DevBuf> scalars;  // 16 device doubles for reductions
  // intermediates of the H_eff*x products (L x and L x W1 W2), kept between
  // Davidson calls and only grown
  std::shared_ptr<DevBuf> heff_scratch[2];
  double last_heff_ms = 0.0;        // device time of the last Davidson's H_eff*x launches
  double heff_part_ms[3] = {0.0, 0.0, 0.0};     // device-resident Davidson: L*x, *mid, *R times
  double heff_part_flops[3] = {0.0, 0.0, 0.0};  // and their algorithmic flops
  double heff_mid_bytes = 0.0;                  // algorithmic bytes of the *mid contractions
  bool profile = false;             // synchronise between step phases to time them
  // host-side planning counters (always on; cheap)
  double t_structure = 0.0;         // seconds in contract_structure
  double t_plan = 0.0;              // seconds in plan creation (validation + tt_contract_plan)
  int64_t n_structure = 0, n_plan = 0;
  // plans of dense (single-block) contractions, keyed by their pair description
  std::map<std::vector<int64_t>, std::shared_ptr<class PlanHandle>> dense_plans;
  // precision of qtensor operator* (TT_PREC_FP64 unless a mixed-precision sweep
  // is updating environments); H_eff products take theirs from the sweep
  int precision = TT_PREC_FP64;
  // precisions of a DMRG sweep: H_eff*x in Davidson and the environment
  // updates; GS, Rayleigh-Ritz and the SVD always run in FP64
  int heff_precision = TT_PREC_FP64;
  int env_precision = TT_PREC_FP64;
  bool energy_fp64 = false;  // set by the sweep driver for its last step
  // device-resident Davidson control state (created on first use)
  ::tt_dav_state* dav = nullptr;
  bool dav_device = true;    // run tensor_davidsonIT's control on the device
  int64_t dav_fallbacks = 0; // device-resident calls redone by the host loop
  int64_t dav_refills = 0;   // Gram-Schmidt failures refilled on the device
  int profile_step = -1;      // two-site step of a sweep bracketed by the CUDA profiler range
};
Runtime& rt();
// Bind / unbind the device context used by every host object on this thread.
void bind_context(tt_ctx* ctx);
void unbind_context();
// Device scalars: slots [0, 32) receive reductions, [32, 64) hold the
// coefficients of linear combinations (at most 16 vectors each).
constexpr int kScalarSlots = 64;
constexpr int kCoefSlot = 32;
double* scalar_slot(int i);
// Host-side bounds check of a contraction before it is planned: every
// element a pair can address lies inside its operand (sizes in doubles).
void validate_pairs(const std::vector<tt_out_block>& outs, const std::vector<tt_block_pair>& pairs,
                    int64_t a_size, int64_t b_size, int64_t c_size);
// Failure of a C-ABI call, carrying its TT_ERR_* status.
struct tt_error : std::runtime_error {
  int code;
  tt_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void check(int status, const char* what);  // throws tt_error on failure

// Owning device allocation (stream-ordered pool of the current context).
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(int64_t n_doubles);
  ~DevBuf();
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept;
  double* get() const { return p_; }
  int64_t size() const { return n_; }
  void zero();

 private:
  double* p_ = nullptr;
  int64_t n_ = 0;
};
using DevPtr = std::shared_ptr<DevBuf>;
DevPtr dev_alloc(int64_t n_doubles);

// ---- quantum numbers (QN_t_2) --------------------------------------------
struct QN {
  int32_t a = 0, b = 0;
  QN() = default;
  QN(int32_t x, int32_t y = 0) : a(x), b(y) {}
  QN operator+(const QN& o) const { return QN(a + o.a, b + o.b); }
  QN operator-(const QN& o) const { return QN(a - o.a, b - o.b); }
  QN& operator+=(const QN& o) { a += o.a; b += o.b; return *this; }
  QN& operator-=(const QN& o) { a -= o.a; b -= o.b; return *this; }
  bool operator==(const QN& o) const { return a == o.a && b == o.b; }
  bool operator!=(const QN& o) const { return !(*this == o); }
  bool operator<(const QN& o) const { return a < o.a || (a == o.a && b < o.b); }
  int64_t pack() const { return ((int64_t)a << 32) | (uint32_t)b; }
};

enum arrow_type { Inward = 0, Outward = 1 };
enum index_type { Link = 0, Site = 1, All = 2 };
#define MoveFromLeft 0
#define MoveFromRight 1

using QNKey = std::vector<int64_t>;
struct QNKeyHash {
  size_t operator()(const QNKey& k) const {
    uint64_t h = 1469598103934665603ull;
    for (int64_t v : k) { h ^= (uint64_t)v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); }
    return (size_t)h;
  }
};

// ---- qtensor_index --------------------------------------------------------
class qtensor_index {
 public:
  qtensor_index() = default;
  qtensor_index(arrow_type a, std::string name, index_type t = Link, unsigned level = 0)
      : arrow_(a), name_(std::move(name)), type_(t), level_(level) {}
  void addQN(QN q, unsigned dim);            // keeps sectors sorted by QN
  unsigned size() const { return (unsigned)qn_.size(); }  // number of sectors
  QN qn(unsigned i) const { return qn_.at(i).first; }
  unsigned qdim(unsigned i) const { return qn_.at(i).second; }
  int64_t dim() const;
  arrow_type arrow() const { return arrow_; }
  const std::string& name() const { return name_; }
  index_type type() const { return type_; }
  unsigned level() const { return level_; }
  void rename(const std::string& n) { name_ = n; }
  void retype(index_type t) { type_ = t; }
  void prime(int inc = 1) { level_ = (unsigned)((int)level_ + inc); }
  void dag() { arrow_ = arrow_ == Inward ? Outward : Inward; }
  void resize(unsigned i, unsigned d) { qn_.at(i).second = d; }
  const std::vector<std::pair<QN, unsigned>>& sectors() const { return qn_; }
  // tag(): arrow, level, name, type and sector list (qtensor_index.h:66)
  bool same_tag(const qtensor_index& o) const {
    return arrow_ == o.arrow_ && level_ == o.level_ && type_ == o.type_ && name_ == o.name_ &&
           qn_ == o.qn_;
  }
  bool same_tag_dagged(const qtensor_index& o) const {
    return arrow_ != o.arrow_ && level_ == o.level_ && type_ == o.type_ && name_ == o.name_ &&
           qn_ == o.qn_;
  }
  bool operator==(const qtensor_index& o) const { return same_tag(o); }
  std::string tag_string() const;

 private:
  arrow_type arrow_ = Inward;
  std::string name_;
  index_type type_ = Link;
  unsigned level_ = 0;
  std::vector<std::pair<QN, unsigned>> qn_;
};

// ---- qtensor ----------------------------------------------------------------
struct BlockMeta {
  std::vector<QN> qn;
  std::vector<unsigned> qi;
  std::vector<int> qd;
  int64_t off = 0;   // element offset inside the arena
  int64_t size = 0;
};

class qtensor {
 public:
  qtensor() = default;
  explicit qtensor(const std::vector<qtensor_index>& idx) : idx_set(idx), rank((unsigned)idx.size()) {}
  qtensor(const qtensor& o);             // deep copy (device to device)
  qtensor(qtensor&& o) noexcept = default;
  qtensor& operator=(const qtensor& o);
  qtensor& operator=(qtensor&& o) noexcept = default;

  std::vector<qtensor_index> idx_set;
  unsigned rank = 0;
  std::vector<BlockMeta> blocks;
  std::unordered_map<QNKey, unsigned, QNKeyHash> block_id;
  DevPtr data;
  int64_t arena = 0;          // elements in the arena
  bool _initted = false;

  void initBlock();           // all legal blocks, zero filled
  void setZero();
  void setOne();
  void setRandom();           // uniform(0,1) in every block (seeded counter RNG)
  void prime(int inc = 1) { for (auto& i : idx_set) i.prime(inc); }
  void dag() { for (auto& i : idx_set) i.dag(); }
  void conj() {}
  int64_t total_size() const;
  double* block_ptr(unsigned b) const { return data->get() + blocks[b].off; }
  QNKey key_of(unsigned b) const;
  int find_block(const QNKey& k) const;
  // append block metadata; data offsets assigned by allocate()
  unsigned add_block_meta(std::vector<QN> qn, std::vector<unsigned> qi, std::vector<int> qd);
  void allocate(bool zero);   // lay blocks out back to back and allocate the arena

  // vector ops (qtensor.cpp:1031-1179, 1606-1647)
  qtensor& operator*=(double c);
  qtensor& operator/=(double c);
  void add(const qtensor& A, double c = 1.0);
  double inner_product(const qtensor& A) const;
  double contract(const qtensor& A) const;
  double norm() const;
  double normalize();

  // host copies of block data (column-major, first index fastest)
  std::vector<double> get_block(unsigned b) const;
  void set_block(unsigned b, const double* host);
};

// C = A * B (qtensor.cpp:523-734)
qtensor operator*(const qtensor& A, const qtensor& B);

// metadata-only contraction: structure of A*B and the GEMM pair list
struct ContractStructure {
  qtensor C;                            // idx_set + blocks (no data)
  std::vector<tt_out_block> outs;
  std::vector<tt_block_pair> pairs;
  double flops = 0.0;
  int64_t a_size = 0, b_size = 0;       // operand arenas (doubles), for validation
};
void contract_structure(const qtensor& A, const qtensor& B, ContractStructure& out);

// Cached form: the structure of A*B (and, on first use, its device plan) is
// kept in a per-thread cache keyed by the complete block metadata of both
// operands (index tags, block QNs, dims and arena offsets), compared exactly.
// DMRG repeats the same contractions sweep after sweep once the bond
// dimensions settle, so steady-state sweeps plan nothing.
struct CachedContraction {
  ContractStructure cs;
  // device plans by requested precision (TT_PREC_FP64 ... TT_PREC_TF32X3_AUTO),
  // built on first use; null when cs has no output blocks
  mutable std::shared_ptr<class PlanHandle> plans[TT_PREC_TF32X3_AUTO + 1];
  // keep: the operands (bit 0 A, bit 1 B) the caller keeps packed across
  // execs, a hint for the automatic precision (see tt_contract_plan_keep)
  tt_plan* plan_for(int precision, int keep = 0) const;
  mutable uint64_t last_use = 0;    // cache clock of its last lookup
  mutable int64_t plan_bytes = 0;   // device bytes its plans hold
};
// need_plan builds the plan of rt().precision right away.
std::shared_ptr<const CachedContraction> contract_cached(const qtensor& A, const qtensor& B,
                                                         bool need_plan);
void clear_contraction_cache();
size_t contraction_cache_size();
// entries, device bytes of their plans, eviction rounds and entries evicted
void contraction_cache_stats(int64_t* entries, int64_t* plan_bytes, int64_t* evictions, int64_t* evicted);

// A cached contraction plan on the device.
class PlanHandle {
 public:
  PlanHandle() = default;
  explicit PlanHandle(tt_plan* p) : p_(p) {}
  ~PlanHandle();
  PlanHandle(const PlanHandle&) = delete;
  PlanHandle& operator=(const PlanHandle&) = delete;
  tt_plan* get() const { return p_; }
 private:
  tt_plan* p_ = nullptr;
};
std::shared_ptr<PlanHandle> make_plan(const ContractStructure& cs, int precision = TT_PREC_FP64, int keep = 0);

// Scoped change of rt().precision, the precision of operator* contractions.
struct PrecisionScope {
  int saved;
  explicit PrecisionScope(int p);
  ~PrecisionScope();
};

// ---- block SVD (qtensor_op.cpp:1097-1544) ---------------------------------
struct TruncInfo {
  double trunc_err = 0.0;
  unsigned kept = 0;
  int gram_max = 0;
  std::vector<QN> sector_qn;
  std::vector<unsigned> kept_per_sector;
};
// Density-matrix perturbation ("noise", White, PRB 72, 180403 (2005)): the
// density matrix of the kept side becomes rho + weight * rho_P / tr(rho_P),
// rho_P = P P^T over the rows of P that carry the kept side's indices (found
// by name; other axes are summed), restricted to the QN sectors of A.  The
// kept basis diagonalises the perturbed rho; the other factor is still the
// projection of A itself.  No counterpart in the reference.
struct NoiseTerm {
  const qtensor* P = nullptr;
  double weight = 0.0;
};
void svd(const qtensor& A, const std::vector<qtensor_index>& left,
         const std::vector<qtensor_index>& right, qtensor& U, qtensor& V, qtensor& S,
         int direction, double cutoff = 0.0, unsigned K = 0, TruncInfo* info = nullptr,
         const NoiseTerm* noise = nullptr);
void svd_bond(const qtensor& combined, qtensor& A_left, qtensor& A_right,
              const qtensor_index& mid, qtensor& S, int direction, double cutoff = 0.0,
              unsigned long K = 0, TruncInfo* info = nullptr, const NoiseTerm* noise = nullptr);
double calcEntropy(const qtensor& S, double cutoff = 1e-24);

// permutation from -> to (qtensor_index_op.cpp:23-37)
std::vector<unsigned> find_index_permutation(const std::vector<qtensor_index>& from,
                                             const std::vector<qtensor_index>& to);

}  // namespace ttb
