// Host mirror of tensor-tools' big_qtensor, tensor_davidsonIT, qMPS/qMPO and
// the U(1) two-site DMRG driver.
//
// Reference: qtensor/big_qtensor.{h,cpp}; linalg/tensor_davidson.cpp:193-347;
// linalg/lapack_wrapper.cpp:40-54 (DIAG); mps/qtt.cpp:205-355,899-994;
// models/hams/Heisenberg.cpp:333-402; algos/dmrg/dmrg.cpp:56-85,300-372,
// 491-509,702-755.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "qtensor.h"

namespace ttb {

// ---- DIAG: small symmetric eigenproblem (dsyev('V','U') semantics) -------
// In place on the column-major n x n array M: eigenvalues ascending in
// evals, eigenvectors in the columns of M.  Cyclic Jacobi in FP64.
void DIAG(int n, double* M, double* evals);

// ---- big_qtensor ---------------------------------------------------------
class big_qtensor {
 public:
  void setLeft(qtensor* L) { L_ = L; }
  void setRight(qtensor* R) { R_ = R; }
  void addMid(qtensor* W) { mid_ = mid_ * (*W); }  // pre-contracts W1*W2 (big_qtensor.h:56)
  qtensor product(qtensor& v);                     // ((L*v)*mid)*R, prime(-1)
  double expec(qtensor& v);
  size_t size() const;                             // sector-count product quirk
  qtensor* left() const { return L_; }
  qtensor* right() const { return R_; }
  const qtensor& mid() const { return mid_; }

 private:
  qtensor* L_ = nullptr;
  qtensor* R_ = nullptr;
  qtensor mid_;
  mutable size_t size_ = 0;
};

// ---- statistics -----------------------------------------------------------
struct DavidsonStats {
  int matvecs = 0;
  int iters = 0;
  int randomized = 0;
  double heff_flops = 0.0;   // algorithmic flops of the H_eff*x products
  double t_engine = 0.0;     // host seconds: Krylov layout + product plans
  double t_loop = 0.0;       // host seconds: the iterations
};

// tensor_davidsonIT for big_qtensor (linalg/tensor_davidson.cpp:193-347).
double tensor_davidsonIT(big_qtensor& A, qtensor& x, int m, int max_restart, double tol,
                         char mode = 'S', DavidsonStats* stats = nullptr);

// ---- MPS / MPO --------------------------------------------------------------
struct qMPS {
  unsigned length = 0;
  unsigned id = 1;
  std::vector<QN> phy_qn;
  QN totalQ;
  int center = -1;
  std::vector<unsigned> bond_dims;
  std::vector<qtensor> A;
  std::string link_name(unsigned i) const { return "ID" + std::to_string(id) + "Link" + std::to_string(i); }
  double position(int site);
  void normalize();
};
struct qMPO {
  unsigned length = 0;
  unsigned id = 2;
  std::vector<QN> phy_qn;
  std::vector<qtensor> A;
};

// Product state (mps/qtt.cpp:58-80, 205-311).
qMPS make_product_qmps(unsigned L, const std::vector<QN>& phy_qn, const std::vector<unsigned>& state,
                       unsigned id = 1);
// Hand-written spin-1/2 Heisenberg qMPO (models/hams/Heisenberg.cpp:333-402),
// with optional site fields dh (Sz) and energy shift tE.
qMPO make_heisenberg_qmpo(unsigned L, const double* dh = nullptr, double tE = 0.0, unsigned id = 2);
// Spin-1/2 operator matrix element <bra|op|ket> (models/sites/spinhalf.cpp:23-46).
double spin_half_op(unsigned bra, const std::string& op, unsigned ket);

// ---- DMRG ---------------------------------------------------------------
// Stream events at the phase boundaries of a logged two-site step: Davidson
// start, SVD start, environment start, environment end.  Their differences
// are the device-stream spans of the phases (gaps in which the device waited
// for the host included).
struct StepEvents {
  void* ev[4] = {nullptr, nullptr, nullptr, nullptr};
  StepEvents() = default;
  StepEvents(const StepEvents&) = delete;
  StepEvents& operator=(const StepEvents&) = delete;
  ~StepEvents();
  void record(int i);  // creates the event on first use
};
struct StepLog {
  int site = 0;
  int direction = 0;
  double energy = 0.0;
  double trunc_err = 0.0;
  unsigned kept = 0;
  int matvecs = 0;
  int randomized = 0;
  double heff_flops = 0.0;
  std::vector<QN> sector_qn;
  std::vector<unsigned> kept_per_sector;
  int gram_max = 0;          // largest per-sector density matrix of the SVD
  double t_davidson = 0.0;   // host wall seconds of the phases of this step
  double t_svd = 0.0;
  double t_env = 0.0;
  double t_engine = 0.0;     // part of t_davidson: Krylov layout and product plans
  std::shared_ptr<StepEvents> events;
};
struct DmrgLog {
  std::vector<StepLog> steps;
  std::vector<double> sweep_energy;
  std::vector<double> sweep_seconds;
  std::vector<double> entropy;
  double initial_energy = 0.0;
  double heff_flops = 0.0;
  double heff_seconds = 0.0;  // device time of the H_eff*x launches (event-timed)
};

// One environment step ((A^dag' env) W) A, for a left or a right environment
// alike (algos/dmrg/dmrg.cpp:56-85 and :491-509 apply it site by site).
qtensor env_step(const qtensor& env, const qtensor& Ai, const qtensor& W);
void buildEnv(qMPS& psi, qMPO& H, std::vector<qtensor>& TR, std::vector<qtensor>& TL);
void updateSite(qMPS& psi, qMPO& H, std::vector<qtensor>& TR, std::vector<qtensor>& TL, unsigned site,
                double& energy, int direction, int max_bd, double cutoff, char mode,
                int search_space_size, int max_restart, DmrgLog* log, double noise = 0.0);
void updateEnv(qMPS& psi, qMPO& H, std::vector<qtensor>& TR, std::vector<qtensor>& TL, unsigned site,
               int direction);
// dmrg schedule overload (algos/dmrg/dmrg.cpp:702-755)
double dmrg(qMPS& psi, qMPO& H, int num_sweeps, const std::vector<int>& max_bd,
            const std::vector<double>& cutoff, const std::vector<int>& max_restart, DmrgLog* log = nullptr);

// State kept between sweeps when sweeps are driven one at a time.
struct DmrgState {
  std::vector<qtensor> TR, TL;
  bool envs_built = false;
  int sweeps_done = 0;
  double noise = 0.0;  // density-matrix perturbation of the following sweeps (0: the reference's update)
  int pos = 0;         // orthogonality centre between calls (0 after dmrg_prepare and after every sweep)
};
// One full sweep (L->R then R->L) of the schedule overload, starting from a
// state prepared by dmrg_prepare (position(0), normalize, buildEnv).
void dmrg_prepare(qMPS& psi, qMPO& H, DmrgState& st, DmrgLog* log);
double dmrg_sweep(qMPS& psi, qMPO& H, DmrgState& st, int max_bd, double cutoff, int max_restart,
                  DmrgLog* log);
void dmrg_finish(qMPS& psi);
// Two-site updates that move the orthogonality centre from st.pos to `to`:
// left-to-right updates of sites pos .. to-1 when to > pos, right-to-left
// updates of sites pos .. to+1 when to < pos, each followed by its
// environment update -- the same step as inside a sweep.  A block of
// mid-chain updates at a settled bond dimension (walk to the middle once,
// then back and forth over a few bonds) is the unit the benchmark times.
// Returns the last step's energy; st.pos becomes `to`.
double dmrg_walk(qMPS& psi, qMPO& H, DmrgState& st, int to, int max_bd, double cutoff, int max_restart,
                 DmrgLog* log);

}  // namespace ttb
