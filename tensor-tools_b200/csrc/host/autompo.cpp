// AutoMPO accumulator, lattices and the dense / U(1) MPO builders.
#include "autompo.h"

#include <algorithm>
#include <exception>
#include <map>
#include <stdexcept>

namespace ttb {

// ---- terms -------------------------------------------------------------------
void HTerm::add(const std::string& op, int i, double x) {
  // models/hams/AutoMPO.cpp:178-201
  if (!op.empty() && op.front() == 'C')
    throw std::runtime_error("AutoMPO: fermionic operators are not supported by the spin-1/2 builders");
  auto it = ops.begin();
  while (it != ops.end() && it->i <= i) ++it;
  coef *= x;
  ops.insert(it, SiteTerm(op, i));
}

bool LessNoCoef::operator()(const HTerm& a, const HTerm& b) const {
  if (a.ops.size() != b.ops.size()) return a.ops.size() < b.ops.size();
  for (size_t j = 0; j < a.ops.size(); ++j)
    if (a.ops[j] != b.ops[j]) return a.ops[j] < b.ops[j];
  return false;
}

void AutoMPO::add(HTerm t) {
  if (t.coef == 0.0) return;
  if (t.ops.empty()) throw std::runtime_error("AutoMPO: term without operators");
  auto it = terms_.find(t);
  if (it == terms_.end()) {
    terms_.insert(std::move(t));
  } else {
    HTerm nt = t;
    nt.coef += it->coef;
    terms_.erase(it);
    terms_.insert(std::move(nt));
  }
}

AutoMPO::Accumulator::~Accumulator() noexcept(false) {
  if (std::uncaught_exceptions() > 0) return;
  if (state_op_) throw std::runtime_error("Invalid input to AutoMPO (missing site number?)");
  if (term_.ops.empty()) throw std::runtime_error("No operators in HTerm");
  term_.coef *= coef_;
  pa_->add(term_);
}

AutoMPO::Accumulator& AutoMPO::Accumulator::operator,(double x) {
  coef_ *= x;
  return *this;
}

AutoMPO::Accumulator& AutoMPO::Accumulator::operator,(int i) {
  if (state_op_) {
    term_.add(op_, i);
    state_op_ = false;
    op_.clear();
  } else {
    coef_ *= (double)i;
  }
  return *this;
}

AutoMPO::Accumulator& AutoMPO::Accumulator::operator,(const char* op) { return operator,(std::string(op)); }

AutoMPO::Accumulator& AutoMPO::Accumulator::operator,(const std::string& op) {
  if (state_op_) throw std::runtime_error("Invalid input to AutoMPO (two strings in a row?)");
  op_ = op;
  state_op_ = true;
  return *this;
}

// ---- lattices ------------------------------------------------------------------
static LatticeBond bond(int s1, int s2, double x1, double y1, double x2, double y2, int type = 0) {
  LatticeBond b;
  b.s1 = s1, b.s2 = s2, b.type = type, b.x1 = x1, b.y1 = y1, b.x2 = x2, b.y2 = y2;
  return b;
}

std::vector<LatticeBond> square_lattice(int Nx, int Ny, bool yperiodic) {
  // models/lattice/square.h:25-58
  yperiodic = yperiodic && Ny > 2;
  int N = Nx * Ny;
  int nbond = 2 * N - Ny + (yperiodic ? 0 : -Nx);
  std::vector<LatticeBond> g;
  for (int n = 1; n <= N; ++n) {
    int x = (n - 1) / Ny + 1, y = (n - 1) % Ny + 1;
    if (x < Nx) g.push_back(bond(n, n + Ny, x, y, x + 1, y));
    if (Ny > 1) {
      if (y < Ny) g.push_back(bond(n, n + 1, x, y, x, y + 1));
      if (yperiodic && y == 1) g.push_back(bond(n, n + Ny - 1, x, y, x, y + Ny));
    }
  }
  if ((int)g.size() != nbond) throw std::runtime_error("Square latt wrong number of bonds");
  return g;
}

std::vector<LatticeBond> square_next_neighbor(int Nx, int Ny, bool yperiodic) {
  // models/lattice/square.h:60-103
  yperiodic = yperiodic && Ny > 2;
  int N = Nx * Ny;
  std::vector<LatticeBond> g;
  for (int n = 1; n <= N; ++n) {
    int x = (n - 1) / Ny + 1, y = (n - 1) % Ny + 1;
    if (x < Nx) g.push_back(bond(n, n + Ny, x, y, x + 1, y, 1));
    if (Ny > 1) {
      if (y < Ny) g.push_back(bond(n, n + 1, x, y, x, y + 1, 1));
      if (yperiodic && y == 1) g.push_back(bond(n, n + Ny - 1, x, y, x, y + Ny, 1));
    }
    if (x < Nx && Ny > 1) {
      if (y < Ny) g.push_back(bond(n, n + Ny + 1, x, y, x + 1, y + 1, 2));
      if (y > 1) g.push_back(bond(n, n + Ny - 1, x, y, x + 1, y - 1, 2));
      if (yperiodic && y == Ny) g.push_back(bond(n, n + 1, x, Ny, x + 1, 1, 2));
      if (yperiodic && y == 1) g.push_back(bond(n, n + 2 * Ny - 1, x, 1, x + 1, Ny, 2));
    }
  }
  return g;
}

// Snake (boustrophedon) site order on an Nx x Ny lattice: column x runs
// y = 1..Ny when x is odd and y = Ny..1 when x is even, so consecutive sites
// along the chain are always lattice neighbours.  The reference numbers
// sites column by column (n = (x-1) Ny + y); this relabels a bond list built
// in that order, keeping every bond's coordinates and type and putting the
// smaller site first.
void snake_relabel(std::vector<LatticeBond>& g, int Nx, int Ny) {
  auto snake = [&](int n) {
    const int x = (n - 1) / Ny + 1, y = (n - 1) % Ny + 1;
    return (x - 1) * Ny + ((x & 1) ? y : Ny + 1 - y);
  };
  (void)Nx;
  for (LatticeBond& b : g) {
    int a = snake(b.s1), c = snake(b.s2);
    if (a > c) {
      std::swap(a, c);
      std::swap(b.x1, b.x2);
      std::swap(b.y1, b.y2);
    }
    b.s1 = a;
    b.s2 = c;
  }
}

std::vector<LatticeBond> triangular_lattice(int Nx, int Ny, bool yperiodic) {
  // models/lattice/triangular.h:25-64 (no coordinates recorded)
  yperiodic = yperiodic && Ny > 2;
  int N = Nx * Ny;
  int nbond = 3 * N - 2 * Ny + (yperiodic ? 0 : -2 * Nx + 1);
  std::vector<LatticeBond> g;
  auto plain = [&](int a, int b) {
    LatticeBond l;
    l.s1 = a, l.s2 = b;
    g.push_back(l);
  };
  for (int n = 1; n <= N; ++n) {
    int x = (n - 1) / Ny + 1, y = (n - 1) % Ny + 1;
    if (x < Nx) plain(n, n + Ny);
    if (Ny > 1) {
      if (n + 1 <= N && (y < Ny || yperiodic)) plain(n, n + 1);
      if (yperiodic && y == 1) plain(n, n + Ny - 1);
      if (x < Nx && y < Ny) plain(n, n + Ny + 1);
    }
  }
  if ((int)g.size() != nbond) throw std::runtime_error("Triangular lattice wrong number of bonds");
  return g;
}

// ---- MPO builders ----------------------------------------------------------------
int spin_half_div(const std::string& op) {
  if (op == "Sz" || op == "Id" || op == "I") return 0;
  if (op == "S+" || op == "Sp") return 2;
  if (op == "S-" || op == "Sm") return -2;
  throw std::runtime_error("spinhalf: operator " + op + " has no definite U(1) charge");
}

static void check_terms(const AutoMPO& ampo, unsigned N) {
  for (const HTerm& t : ampo.terms()) {
    if (t.Nops() > 2) throw std::runtime_error("AutoMPO: terms with more than two operators are not supported");
    for (const SiteTerm& s : t.ops)
      if (s.i < 0 || s.i >= (int)N) throw std::runtime_error("AutoMPO: operator site out of range");
    if (t.Nops() == 2 && t.first().i == t.last().i)
      throw std::runtime_error("AutoMPO: two operators on one site are not supported");
  }
}

std::vector<AutoMPOLink> automp_links(const AutoMPO& ampo, unsigned N, bool with_charges) {
  check_terms(ampo, N);
  std::vector<std::vector<AutoMPOLink::State>> basis(N + 1);
  for (unsigned n = 0; n <= N; ++n) {
    if (n < N) basis[n].push_back({0, SiteTerm("IL", 0), 0});
    if (n >= 1) basis[n].push_back({1, SiteTerm("HL", 0), 0});
  }
  // Terms are visited in the accumulator's order, which sorts two-operator
  // terms by their first operator: strings enter each link in (site, op) order.
  for (const HTerm& t : ampo.terms()) {
    if (t.Nops() != 2) continue;
    int q = with_charges ? spin_half_div(t.first().op) : 0;
    for (int n = t.first().i + 1; n <= t.last().i; ++n) {
      auto& bn = basis[n];
      bool has = std::any_of(bn.begin(), bn.end(), [&](const AutoMPOLink::State& s) {
        return s.kind == 2 && s.st == t.first();
      });
      if (!has) bn.push_back({2, t.first(), q});
    }
  }
  std::vector<AutoMPOLink> links(N + 1);
  for (unsigned n = 0; n <= N; ++n) {
    auto& bn = basis[n];
    std::stable_sort(bn.begin(), bn.end(), [](const AutoMPOLink::State& a, const AutoMPOLink::State& b) {
      if (a.q == 0 && b.q != 0) return true;
      if (b.q == 0 && a.q != 0) return false;
      return a.q < b.q;
    });
    AutoMPOLink& L = links[n];
    for (size_t k = 0; k < bn.size(); ++k) {
      AutoMPOLink::State s = bn[k];
      if (L.sectors.empty() || L.sectors.back().first != s.q) L.sectors.push_back({s.q, 0});
      s.pos = L.sectors.back().second++;
      s.gpos = (int)k;
      L.states.push_back(s);
    }
  }
  return links;
}

namespace {
// One MPO element rule application: (row state, column state, op, coefficient).
struct Entry {
  int r, c;  // state numbers in links[i] / links[i+1]
  std::string op;
  double val;
};

std::vector<Entry> site_entries(const std::vector<const HTerm*>& ending, const std::vector<AutoMPOLink>& links,
                                unsigned i) {
  // models/hams/Heisenberg.cpp:296-328 (dense) / :585-633 (qMPO): start a
  // string from IL, pass IL/HL/strings through with Id, close a string into HL
  // with the last operator and the coefficient, put one-site terms on IL -> HL.
  std::vector<Entry> out;
  const auto& rows = links[i].states;
  const auto& cols = links[i + 1].states;
  int il = -1, hl = -1;
  std::map<SiteTerm, int> row_of;
  for (int r = 0; r < (int)rows.size(); ++r) {
    if (rows[r].kind == 0) il = r;
    if (rows[r].kind == 2) row_of[rows[r].st] = r;
  }
  for (int c = 0; c < (int)cols.size(); ++c)
    if (cols[c].kind == 1) hl = c;
  for (int r = 0; r < (int)rows.size(); ++r)
    for (int c = 0; c < (int)cols.size(); ++c) {
      const auto& rs = rows[r];
      const auto& cs = cols[c];
      if (cs.kind == 2 && cs.st.i == (int)i && rs.kind == 0) out.push_back({r, c, cs.st.op, 1.0});
      if (rs.kind == cs.kind && (rs.kind != 2 || rs.st == cs.st)) out.push_back({r, c, "Id", 1.0});
    }
  for (const HTerm* t : ending) {
    if (t->Nops() == 2) {
      auto it = row_of.find(t->first());
      if (it == row_of.end() || hl < 0) throw std::runtime_error("AutoMPO: internal string bookkeeping error");
      out.push_back({it->second, hl, t->last().op, t->coef});
    } else {
      if (il < 0 || hl < 0) throw std::runtime_error("AutoMPO: internal link bookkeeping error");
      out.push_back({il, hl, t->first().op, t->coef});
    }
  }
  return out;
}

// Terms that close on each site: two-operator terms by their last site and
// one-operator terms by their site, in the accumulator's order.
std::vector<std::vector<const HTerm*>> terms_ending(const AutoMPO& ampo, unsigned N) {
  std::vector<std::vector<const HTerm*>> e(N);
  for (const HTerm& t : ampo.terms()) e[t.last().i].push_back(&t);
  return e;
}
}  // namespace

qMPO build_qmpo(const AutoMPO& ampo, unsigned N, unsigned id) {
  if (N < 2) throw std::runtime_error("build_qmpo: need at least two sites");
  auto links = automp_links(ampo, N, true);
  auto ending = terms_ending(ampo, N);
  qMPO H;
  H.length = N;
  H.id = id;
  H.phy_qn = {QN(-1), QN(1)};
  std::string pref = "ID" + std::to_string(id) + "Link";
  for (unsigned i = 0; i < N; ++i) {
    qtensor T({qtensor_index(Inward, pref + std::to_string(i), Link, 0),
               qtensor_index(Outward, "Site" + std::to_string(i), Site, 0),
               qtensor_index(Inward, "Site" + std::to_string(i), Site, 1),
               qtensor_index(Outward, pref + std::to_string(i + 1), Link, 0)});
    for (auto& s : links[i].sectors) T.idx_set[0].addQN(QN(s.first), s.second);
    for (auto& p : H.phy_qn) T.idx_set[1].addQN(p, 1);
    for (auto& p : H.phy_qn) T.idx_set[2].addQN(p, 1);
    for (auto& s : links[i + 1].sectors) T.idx_set[3].addQN(QN(s.first), s.second);
    T.initBlock();
    std::vector<std::vector<double>> host(T.blocks.size());
    for (size_t b = 0; b < T.blocks.size(); ++b) host[b].assign((size_t)T.blocks[b].size, 0.0);
    for (const Entry& e : site_entries(ending[i], links, i)) {
      const auto& rs = links[i].states[e.r];
      const auto& cs = links[i + 1].states[e.c];
      for (unsigned k = 0; k < 2; ++k)
        for (unsigned b = 0; b < 2; ++b) {
          double v = e.val * spin_half_op(b, e.op, k);
          if (v == 0.0) continue;
          QNKey key{QN(rs.q).pack(), H.phy_qn[k].pack(), H.phy_qn[b].pack(), QN(cs.q).pack()};
          int blk = T.find_block(key);
          if (blk < 0) throw std::runtime_error("build_qmpo: term " + e.op + " does not conserve the U(1) charge");
          const BlockMeta& bm = T.blocks[blk];
          int64_t s3 = (int64_t)bm.qd[0] * bm.qd[1] * bm.qd[2];
          host[blk][(size_t)(rs.pos + s3 * cs.pos)] += v;
        }
    }
    for (size_t b = 0; b < T.blocks.size(); ++b) T.set_block((unsigned)b, host[b].data());
    H.A.push_back(std::move(T));
  }
  return H;
}

MPO build_mpo(const AutoMPO& ampo, unsigned N, unsigned id) {
  if (N < 2) throw std::runtime_error("build_mpo: need at least two sites");
  auto links = automp_links(ampo, N, false);
  auto ending = terms_ending(ampo, N);
  MPO H;
  H.length = N;
  H.id = id;
  std::string pref = "ID" + std::to_string(id) + "Link";
  for (unsigned i = 0; i < N; ++i) {
    int64_t dl = (int64_t)links[i].states.size(), dr = (int64_t)links[i + 1].states.size();
    std::vector<double> host((size_t)(dl * 4 * dr), 0.0);
    for (const Entry& e : site_entries(ending[i], links, i)) {
      int64_t r = links[i].states[e.r].gpos, c = links[i + 1].states[e.c].gpos;
      for (unsigned k = 0; k < 2; ++k)
        for (unsigned b = 0; b < 2; ++b) host[(size_t)(r + dl * (k + 2 * (b + 2 * c)))] += e.val * spin_half_op(b, e.op, k);
    }
    H.A.emplace_back(std::vector<dtensor_index>{dtensor_index(dl, pref + std::to_string(i)),
                                                dtensor_index(2, "Site" + std::to_string(i), Site, 0),
                                                dtensor_index(2, "Site" + std::to_string(i), Site, 1),
                                                dtensor_index(dr, pref + std::to_string(i + 1))},
                     false);
    H.A.back().set(host.data());
  }
  return H;
}

}  // namespace ttb
