// Host mirror of tensor-tools' dense path: dtensor, big_dtensor, the dense
// SVD, the restarted preconditioned Davidson and the dense DMRG schedule.
//
// Reference: dtensor/dtensor_index.h:34-60 (tags: size, name, type, level;
// no arrows), dtensor/dtensor.cpp:300-368 (operator*), :397-430 (contract),
// :511-571 (diagonal), :792-849 (vector ops); dtensor/big_dtensor.cpp:23-161;
// dtensor/dtensor_op.cpp:86-211 (svd_bond, svd); linalg/tensor_davidson.cpp
// :25-36 (elemWiseDivide), :74-184 (tensor_davidson); mps/tt.cpp:174-262,
// 575-795; models/hams/Heisenberg.cpp:72-148,185-208; algos/dmrg/dmrg.cpp
// :24-51,228-295,466-486,591-646.
#pragma once

#include <string>
#include <vector>

#include "dmrg_q.h"

namespace ttb {

struct dtensor_index {
  int64_t size = 1;
  std::string name;
  index_type type = Link;
  unsigned level = 0;
  dtensor_index() = default;
  dtensor_index(int64_t s, std::string n, index_type t = Link, unsigned l = 0)
      : size(s), name(std::move(n)), type(t), level(l) {}
  bool same_tag(const dtensor_index& o) const {
    return size == o.size && name == o.name && type == o.type && level == o.level;
  }
  // dtensor_index::similar(A, type) (dtensor/dtensor_index.h:55-57)
  bool similar(const dtensor_index& o, index_type t) const {
    return size == o.size && name == o.name && (type == o.type || t == All) && (type == t || t == All) &&
           (level == o.level + 1 || level + 1 == o.level);
  }
  void prime(int inc = 1) { level = (unsigned)((int)level + inc); }
};

class dtensor {
 public:
  dtensor() = default;
  explicit dtensor(const std::vector<dtensor_index>& idx, bool zero = true);
  dtensor(const dtensor& o);
  dtensor(dtensor&& o) noexcept = default;
  dtensor& operator=(const dtensor& o);
  dtensor& operator=(dtensor&& o) noexcept = default;

  std::vector<dtensor_index> idx_set;
  unsigned rank = 0;
  int64_t size = 0;
  DevPtr data;
  bool _initted = false;

  void prime(int inc = 1) { for (auto& i : idx_set) i.prime(inc); }
  void dag() {}
  void conj() {}
  void setOne();
  dtensor& operator*=(double c);
  dtensor& operator/=(double c);
  void add(const dtensor& A, double c = 1.0);
  double inner_product(const dtensor& A) const;
  double contract(const dtensor& A) const;  // positional (dtensor.cpp:397-430)
  double norm() const;
  double normalize();
  dtensor diagonal(index_type type) const;
  std::vector<double> get() const;
  void set(const double* host);
};

dtensor operator*(const dtensor& A, const dtensor& B);

// dense svd (dtensor_op.cpp:120-211) with the rule CTF's svd(K, threshold)
// is restated as: at most K values, and when cutoff > 0 only values > cutoff
// (at least one).  U (MoveFromLeft) or V (MoveFromRight) are the orthonormal
// eigenvectors of the Gram matrix; the other factor is V = U^T A / U = A V^T.
void dsvd(const dtensor& A, const std::vector<dtensor_index>& left, const std::vector<dtensor_index>& right,
          dtensor& U, dtensor& V, dtensor& S, int direction, double cutoff = 0.0, unsigned long K = 0);
void dsvd_bond(const dtensor& combined, dtensor& A_left, dtensor& A_right, dtensor_index& mid, dtensor& S,
               int direction, double cutoff = 0.0, unsigned long K = 0);

class big_dtensor {
 public:
  void setLeft(dtensor* L) { L_ = L; }
  void setRight(dtensor* R) { R_ = R; }
  void addMid(dtensor* m) { mid_.push_back(m); }
  dtensor product(dtensor& v);
  dtensor diagonal();
  double expec(dtensor& v);
  size_t size() const;

 private:
  dtensor* L_ = nullptr;
  dtensor* R_ = nullptr;
  std::vector<dtensor*> mid_;
  mutable size_t size_ = 0;
};

// restarted, diagonal-preconditioned Davidson (tensor_davidson.cpp:74-184)
double tensor_davidson(big_dtensor& A, dtensor& x, int m, int max_restart, double tol, char mode = 'S',
                       DavidsonStats* stats = nullptr);

struct MPS {
  unsigned length = 0, phy_dim = 2, id = 1;
  int center = -1;
  std::vector<unsigned> bond_dims;
  std::vector<dtensor> A;
  std::string link_name(unsigned i) const { return "ID" + std::to_string(id) + "Link" + std::to_string(i); }
  double position(int site);
  void normalize();
};
struct MPO {
  unsigned length = 0, phy_dim = 2, id = 2;
  std::vector<dtensor> A;
};
MPS make_product_mps(unsigned L, const std::vector<unsigned>& state, unsigned id = 1);
MPO make_heisenberg_mpo(unsigned L, const double* dh = nullptr, double tE = 0.0, unsigned id = 2);

struct DenseStepLog {
  int site = 0, direction = 0, matvecs = 0;
  double energy = 0.0;
  unsigned kept = 0;
};
struct DenseDmrgLog {
  std::vector<DenseStepLog> steps;
  std::vector<double> sweep_energy;
  std::vector<std::vector<unsigned>> sweep_bond_dims;
};
// schedule overload (algos/dmrg/dmrg.cpp:591-646): no per-sweep normalize
double dmrg(MPS& psi, MPO& H, int num_sweeps, const std::vector<int>& max_bd, const std::vector<double>& cutoff,
            const std::vector<int>& max_restart, DenseDmrgLog* log = nullptr);

}  // namespace ttb
