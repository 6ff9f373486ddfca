// AutoMPO term accumulator, lattice bond lists and the MPO builders that turn a
// sum of one- and two-site spin-1/2 terms into a dense MPO or a U(1) qMPO.
//
// Interface follows models/hams/AutoMPO.h:41-218 (SiteTerm, HTerm, AutoMPO with
// the `ampo += coef, "op", i, "op", j;` accumulator) and
// models/lattice/{latticebond,square,triangular}.h; the builders follow the
// finite-state construction of models/hams/Heisenberg.cpp:213-330 (dense) and
// :412-635 (qMPO).  Differences from the reference, all of which leave the
// operator H unchanged:
//   * a link carries a string state only while the term actually crosses it
//     (first.i < n <= last.i); the reference also adds it at link last.i+1 and
//     for one-site terms, where the state is a dead end that adds zero rows;
//   * within a charge sector the states are ordered IL, HL, then strings by
//     their first operator (site, name); sectors are ordered 0 first, then by
//     ascending charge (the reference's sort);
//   * a string state's link charge is the divergence of its first operator for
//     both the index sector list and the block placement;
//   * elements are accumulated, where the reference's CTF write overwrites
//     (identical whenever no two terms share an MPO element).
#pragma once

#include <set>
#include <string>
#include <vector>

#include "dmrg_d.h"
#include "dmrg_q.h"

namespace ttb {

struct SiteTerm {
  std::string op;
  int i = -1;
  SiteTerm() = default;
  SiteTerm(std::string o, int site) : op(std::move(o)), i(site) {}
  bool operator==(const SiteTerm& o) const { return op == o.op && i == o.i; }
  bool operator!=(const SiteTerm& o) const { return !(*this == o); }
  bool operator<(const SiteTerm& o) const { return i != o.i ? i < o.i : op < o.op; }
};

struct HTerm {
  double coef = 1.0;
  std::vector<SiteTerm> ops;
  // Insert keeping site order; an operator on an already-used site goes after
  // the existing ones (models/hams/AutoMPO.cpp:178-201, spin operators only).
  void add(const std::string& op, int i, double x = 1.0);
  int Nops() const { return (int)ops.size(); }
  const SiteTerm& first() const { return ops.front(); }
  const SiteTerm& last() const { return ops.back(); }
};

// Order on operator lists only (models/hams/AutoMPO.cpp:247-257).
struct LessNoCoef {
  bool operator()(const HTerm& a, const HTerm& b) const;
};

class AutoMPO {
 public:
  using storage = std::set<HTerm, LessNoCoef>;

  // Comma accumulator (models/hams/AutoMPO.cpp:259-364): numbers multiply the
  // coefficient, a string names an operator, and the int after it its site.
  class Accumulator {
   public:
    Accumulator(AutoMPO* pa, double x) : pa_(pa), coef_(x) {}
    Accumulator(AutoMPO* pa, const char* op) : pa_(pa), op_(op), state_op_(true) {}
    Accumulator(AutoMPO* pa, const std::string& op) : pa_(pa), op_(op), state_op_(true) {}
    Accumulator(const Accumulator&) = delete;
    ~Accumulator() noexcept(false);
    Accumulator& operator,(double x);
    Accumulator& operator,(int i);
    Accumulator& operator,(const char* op);
    Accumulator& operator,(const std::string& op);

   private:
    AutoMPO* pa_;
    double coef_ = 1.0;
    std::string op_;
    bool state_op_ = false;
    HTerm term_;
  };

  Accumulator operator+=(double x) { return Accumulator(this, x); }
  Accumulator operator+=(int x) { return Accumulator(this, (double)x); }
  Accumulator operator+=(const char* op) { return Accumulator(this, op); }
  Accumulator operator+=(const std::string& op) { return Accumulator(this, op); }

  // Adds a term; zero coefficients are dropped and a repeated operator list
  // sums into the existing coefficient (models/hams/AutoMPO.cpp:366-393).
  void add(HTerm t);
  const storage& terms() const { return terms_; }
  int size() const { return (int)terms_.size(); }
  void reset() { terms_.clear(); }

 private:
  storage terms_;
};

// Lattice bonds with 1-based site numbers, y fastest: n = (x-1)*Ny + y
// (models/lattice/latticebond.h, square.h:25-103, triangular.h:25-64).
// type is 0 when unset, else the bond class ("1" nearest, "2" next nearest).
struct LatticeBond {
  int s1 = 0, s2 = 0, type = 0;
  double x1 = 0, y1 = 0, x2 = 0, y2 = 0;
};
std::vector<LatticeBond> square_lattice(int Nx, int Ny, bool yperiodic);
std::vector<LatticeBond> square_next_neighbor(int Nx, int Ny, bool yperiodic);
std::vector<LatticeBond> triangular_lattice(int Nx, int Ny, bool yperiodic);
// snake site order (column x runs upward when odd, downward when even)
void snake_relabel(std::vector<LatticeBond>& g, int Nx, int Ny);

// Charge carried by a spin-1/2 operator in units of 2Sz (models/sites/spinhalf.cpp:95-106).
int spin_half_div(const std::string& op);

// Finite-state MPO layout shared by both builders: per link n = 0..N the
// ordered states and the (charge, count) sector list.
struct AutoMPOLink {
  struct State {
    int kind = 0;  // 0: IL (identity so far), 1: HL (complete term), 2: open string
    SiteTerm st;
    int q = 0;
    int pos = 0;   // position inside its charge sector
    int gpos = 0;  // position in the whole link
  };
  std::vector<State> states;
  std::vector<std::pair<int, int>> sectors;  // (charge, count)
};
std::vector<AutoMPOLink> automp_links(const AutoMPO& ampo, unsigned N, bool with_charges);

qMPO build_qmpo(const AutoMPO& ampo, unsigned N, unsigned id = 2);
MPO build_mpo(const AutoMPO& ampo, unsigned N, unsigned id = 2);

}  // namespace ttb
