/*
 * tt_dmrg.h -- object-level C ABI of the B200 two-site DMRG inner loop.
 *
 * Handles wrap the C++ host classes that mirror tensor-tools' interface; a
 * foreign-language binding of that interface (ctypes, cgo, JNI ...) binds
 * these.  Every call returns TT_OK (0) or a TT_ERR_* code from tt_b200.h;
 * tt_get_last_error() explains the last failure of the calling thread.
 * Objects are bound to the context passed to tt_dmrg_bind on this thread.
 *
 * Reference interfaces replaced (paths relative to the tensor-tools tree):
 *   tt_qtensor_*             qtensor<T> and qtensor_index    qtensor/qtensor.h:47-164,
 *                                                            qtensor/qtensor_index.h:35-118
 *   tt_qtensor_init_blocks   qtensor<T>::initBlock           qtensor/qtensor.cpp:301-345
 *   tt_qtensor_contract      qtensor<T>::operator*           qtensor/qtensor.cpp:523-734
 *   tt_qtensor_norm/scale/add/inner_product
 *                            norm / operator*= / add / inner_product
 *                                                            qtensor/qtensor.cpp:1031-1179,1606-1647
 *   tt_qtensor_svd           svd(A,left,right,U,V,S,dir,cutoff,K)
 *                                                            qtensor/qtensor_op.cpp:1097-1453
 *   tt_qtensor_svd_bond      svd_bond(combined,...)          qtensor/qtensor_op.cpp:1506-1544
 *   tt_qtensor_svd_bond_sectors  the same, with the kept count of every mid-QN sector
 *   tt_qtensor_env_update    TL[i+1] / TR[i-1] = ((A^dag' env) W) A
 *                                                            algos/dmrg/dmrg.cpp:56-85,491-509
 *   tt_bigq_*                big_qtensor<T> setLeft/addMid/setRight/product/size
 *                                                            qtensor/big_qtensor.{h,cpp}
 *   tt_bigq_davidson         tensor_davidsonIT               linalg/tensor_davidson.cpp:193-347
 *   tt_qmps_product_spinhalf qMPS(sites, product string)     mps/qtt.cpp:58-80,205-311
 *   tt_qmpo_heisenberg       Heisenberg<T>::buildHam(qMPO&)  models/hams/Heisenberg.cpp:333-402
 *   tt_qmps_position         qTensorTrain::position          mps/qtt.cpp:932-994
 *   tt_qdmrg_*               buildEnv / updateSite / updateEnv / dmrg (schedule overload)
 *                                                            algos/dmrg/dmrg.cpp:56-85,300-372,
 *                                                            491-509,702-755
 *   tt_qmps_overlap / tt_dmps_overlap
 *                            psiphi(qMPS&, qMPS&) / psiphi(MPS&, MPS&)
 *                                                            mps/observables.cpp:382-450
 *   tt_qmps_expectation / tt_dmps_expectation
 *                            psiHphi(psi, H, phi)            mps/observables.cpp:25-103
 *   tt_qmps_measure_sz / tt_dmps_measure_sz
 *                            <Sz_i>, <Sz_i Sz_j> (no reference counterpart; the
 *                            reference offers only psiHphi / psiphi)
 *   tt_qmps_save / tt_qmps_load, tt_dmps_save / tt_dmps_load
 *                            qTensorTrain::save/load, TensorTrain::save/load
 *                                                            mps/qtt.cpp:678-771, mps/tt.cpp,
 *                                                            dtensor/dtensor.cpp:610-713
 *   tt_autompo_*             AutoMPO, HTerm, SiteTerm         models/hams/AutoMPO.{h,cpp}
 *   tt_qmpo_from_autompo     Heisenberg<T>::buildHam(AutoMPO&, qMPO&)
 *                                                            models/hams/Heisenberg.cpp:412-635
 *   tt_dmpo_from_autompo     Heisenberg<T>::buildHam(AutoMPO&, MPO&)
 *                                                            models/hams/Heisenberg.cpp:213-330
 *   tt_lattice               squareLattice / squareNextNeighbor / triangularLattice
 *                                                            models/lattice/square.h:25-103,
 *                                                            models/lattice/triangular.h:25-64
 *   tt_ddmrg_*               the dense dtensor / big_dtensor path and its dmrg
 *                                                            dtensor/dtensor.cpp, dtensor/big_dtensor.cpp,
 *                                                            dtensor/dtensor_op.cpp,
 *                                                            algos/dmrg/dmrg.cpp:24-51,228-295,
 *                                                            466-486,591-646
 */
#ifndef TT_DMRG_H
#define TT_DMRG_H

#include <stddef.h>
#include <stdint.h>

#include "tt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tt_qtensor tt_qtensor;
typedef struct tt_bigq tt_bigq;
typedef struct tt_qmps tt_qmps;
typedef struct tt_qmpo tt_qmpo;
typedef struct tt_qdmrg tt_qdmrg;

/* arrow: 0 Inward, 1 Outward; type: 0 Link, 1 Site; qn: 2 ints per sector */
typedef struct {
  int32_t arrow;
  int32_t type;
  int32_t level;
  int32_t n_sectors;
  const char* name;
  const int32_t* qn;
  const int32_t* qdim;
} tt_index_desc;

int tt_dmrg_bind(tt_ctx* ctx);
int tt_dmrg_unbind(void);
/* on != 0: synchronise between the phases of each two-site step so that
 * tt_qdmrg_step_profile reports per-phase times (slower; off by default) */
int tt_dmrg_set_profiling(int on);
/* Per-thread totals over the device-resident Davidson calls' H_eff*x
 * products: device milliseconds and algorithmic flops of L*x, *mid and *R
 * (ms[0..2], flops[0..2], event-timed on the library stream) and the
 * algorithmic bytes of the *mid contractions (distinct operand blocks read
 * once, the output written once). */
int tt_dmrg_heff_parts(double* ms, double* flops, double* mid_bytes);
/* host-side planning counters of this thread: seconds and calls spent in
 * block-structure computation and in contraction-plan creation */
int tt_dmrg_planning_counters(double* t_structure, int64_t* n_structure, double* t_plan, int64_t* n_plan);
/* this thread's contraction cache (block structures and plans keyed by the
 * operands' structure): entries, device bytes of their plans' tables, and
 * how often least-recently-used entries were evicted (rounds, entries) */
int tt_dmrg_cache_stats(int64_t* entries, int64_t* plan_bytes, int64_t* evictions, int64_t* evicted);

/* Precisions (TT_PREC_*) on this thread: op -- qtensor/dtensor contractions
 * (operator*); heff -- the H_eff*x products inside Davidson; env -- the
 * environment updates of a sweep.  Gram-Schmidt, the Rayleigh-Ritz problem,
 * the SVD and the two-site tensor stay FP64; with heff != TT_PREC_FP64 the
 * last step of every sweep re-evaluates its energy with an FP64 product. */
int tt_dmrg_set_precision(int op, int heff, int env);
/* Davidson control on this thread: 1 (default) runs tensor_davidsonIT's
 * decisions on the device and synchronises once per call (a Gram-Schmidt
 * failure is refilled on the device); 0 always uses the host loop.
 * tt_dmrg_davidson_fallbacks counts device calls redone by the host loop. */
int tt_dmrg_set_davidson(int device_control);
int tt_dmrg_davidson_fallbacks(int64_t* n);
/* Gram-Schmidt failures of the device-resident loop refilled on the device
 * (random refill and re-orthogonalisation, linalg/tensor_davidson.cpp:298-316) */
int tt_dmrg_davidson_refills(int64_t* n);
/* Diagnostics: bracket two-site step `step` (0 .. 2L-3) of every following
 * U(1) sweep with cudaProfilerStart/Stop, so a profiler started with its
 * capture off sees that step only; -1 (default) disables. */
int tt_dmrg_set_profile_step(int step);

/* ---- qtensor ------------------------------------------------------------- */
int tt_qtensor_create(int rank, const tt_index_desc* idx, tt_qtensor** out);
int tt_qtensor_init_blocks(tt_qtensor* t);
/* explicit block list: qi holds n_blocks*rank sector positions; blocks are
 * zero-filled, laid out in the given order (blocks created by the
 * reference's contraction or SVD need not be all legal combinations) */
int tt_qtensor_set_blocks(tt_qtensor* t, int n_blocks, const int32_t* qi);
int tt_qtensor_destroy(tt_qtensor* t);
int tt_qtensor_copy(const tt_qtensor* t, tt_qtensor** out);
int tt_qtensor_rank(const tt_qtensor* t, int* rank);
/* name copied into name_buf (NUL-terminated); qn/qdim need 2*cap / cap ints */
int tt_qtensor_index(const tt_qtensor* t, int i, int32_t* arrow, int32_t* type, int32_t* level,
                     int32_t* n_sectors, char* name_buf, int name_cap, int32_t* qn, int32_t* qdim, int cap);
int tt_qtensor_num_blocks(const tt_qtensor* t, int* n);
int tt_qtensor_block_info(const tt_qtensor* t, int b, int32_t* qn, int32_t* qi, int32_t* qd, int64_t* size);
/* b = -1 when no block has these QNs (2*rank ints, in the tensor's index order) */
int tt_qtensor_find_block(const tt_qtensor* t, const int32_t* qn, int* b);
int tt_qtensor_get_block(const tt_qtensor* t, int b, double* host);
int tt_qtensor_set_block(tt_qtensor* t, int b, const double* host);
int tt_qtensor_prime(tt_qtensor* t, int inc);
int tt_qtensor_dag(tt_qtensor* t);
int tt_qtensor_contract(const tt_qtensor* A, const tt_qtensor* B, tt_qtensor** C);
int tt_qtensor_norm(const tt_qtensor* t, double* out);
int tt_qtensor_scale(tt_qtensor* t, double c);
int tt_qtensor_add(tt_qtensor* y, const tt_qtensor* x, double c);
int tt_qtensor_inner_product(const tt_qtensor* a, const tt_qtensor* b, double* out);
/* left_axes: the nleft axes of A forming the row index (in order); the rest
 * (in A's order) form the column index.  Outputs are new handles. */
int tt_qtensor_svd(const tt_qtensor* A, int nleft, const int* left_axes, int direction, double cutoff,
                   unsigned K, tt_qtensor** U, tt_qtensor** V, tt_qtensor** S, double* trunc_err,
                   unsigned* kept);
/* svd_bond(combined, A_left, A_right, mid = A_left's axis mid_axis, ...): replaces A_left, A_right */
int tt_qtensor_svd_bond(const tt_qtensor* combined, tt_qtensor* A_left, tt_qtensor* A_right, int mid_axis,
                        int direction, double cutoff, unsigned long K, tt_qtensor** S, double* trunc_err,
                        unsigned* kept);
/* svd_bond as above, also reporting the mid-QN sectors of the SVD in
 * ascending QN order: *n_sectors of them (sectors that keep no state
 * included), their QNs as pairs qn[2j], qn[2j+1] and their kept counts (the
 * first `cap` are written).  The truncation log of svd
 * (qtensor/qtensor_op.cpp:1290-1330) reports the same per-sector counts. */
int tt_qtensor_svd_bond_sectors(const tt_qtensor* combined, tt_qtensor* A_left, tt_qtensor* A_right,
                                int mid_axis, int direction, double cutoff, unsigned long K, tt_qtensor** S,
                                double* trunc_err, unsigned* kept, int* n_sectors, int32_t* qn,
                                uint32_t* kept_per_sector, int cap);
/* One environment update, the step of buildEnv and updateEnv
 * (algos/dmrg/dmrg.cpp:56-85 q buildEnv, :491-509 q updateEnv): out =
 * ((A^dag' * env) * W) * A, contracted by index tags, so the same call
 * extends a left environment TL[i] -> TL[i+1] with site i or a right one
 * TR[i] -> TR[i-1].  Contractions run at the precision set by
 * tt_dmrg_set_precision for environments.  *out is a new handle. */
int tt_qtensor_env_update(const tt_qtensor* env, const tt_qtensor* A, const tt_qtensor* W, tt_qtensor** out);

/* ---- big_qtensor and Davidson --------------------------------------------- */
/* W2 may be NULL (one-site operator).  L, W1, W2, R are copied. */
int tt_bigq_create(const tt_qtensor* L, const tt_qtensor* W1, const tt_qtensor* W2, const tt_qtensor* R,
                   tt_bigq** out);
int tt_bigq_product(tt_bigq* op, const tt_qtensor* v, tt_qtensor** out);
int tt_bigq_size(tt_bigq* op, uint64_t* size);
/* tensor_davidsonIT(op, x, 3, max_restart, tol, 'S'); x is updated in place */
int tt_bigq_davidson(tt_bigq* op, tt_qtensor* x, int max_restart, double tol, double* eval, int* matvecs);
int tt_bigq_destroy(tt_bigq* op);

/* ---- U(1) MPS / MPO / DMRG --------------------------------------------------- */
/* spin-1/2 sites: state[i] = 0 (Dn) or 1 (Up) */
int tt_qmps_product_spinhalf(int L, const int* state, unsigned id, tt_qmps** out);
int tt_qmps_destroy(tt_qmps* psi);
int tt_qmps_length(const tt_qmps* psi, int* L);
int tt_qmps_bond_dims(const tt_qmps* psi, int* out);       /* L+1 entries */
int tt_qmps_center(const tt_qmps* psi, int* center);
int tt_qmps_position(tt_qmps* psi, int site);
/* copy of site tensor i as a new handle */
int tt_qmps_tensor(const tt_qmps* psi, int i, tt_qtensor** out);
/* block data of all site tensors, site by site and block by block (the
 * block structure stays on the host): size in doubles, device -> host and
 * host -> device (host buffers should be pinned for full bandwidth) */
int tt_qmps_data_size(const tt_qmps* psi, int64_t* n);
int tt_qmps_get_data(const tt_qmps* psi, double* host);
int tt_qmps_set_data(tt_qmps* psi, const double* host);
/* The same for the site tensors [first, last) only (their blocks in order):
 * one asynchronous copy per contiguous run of blocks and one synchronisation,
 * so a pinned host buffer moves at full bandwidth.  The reference keeps its
 * qMPS in (distributed) host memory (mps/qtt.h:124-129). */
int tt_qmps_sites_size(const tt_qmps* psi, int first, int last, int64_t* n);
int tt_qmps_get_sites(const tt_qmps* psi, int first, int last, double* host);
int tt_qmps_set_sites(tt_qmps* psi, int first, int last, const double* host);
/* dh: L site fields (may be NULL), tE: energy shift */
int tt_qmpo_heisenberg(int L, const double* dh, double tE, unsigned id, tt_qmpo** out);
int tt_qmpo_destroy(tt_qmpo* H);
int tt_qmpo_tensor(const tt_qmpo* H, int i, tt_qtensor** out);

/* Step-wise driver: create = position(0), normalize, buildEnv, initial energy. */
int tt_qdmrg_create(tt_qmps* psi, tt_qmpo* H, tt_qdmrg** out);
/* one full sweep (L->R, R->L, normalize) with this sweep's schedule entries */
/* Noise for the following sweeps: the kept side's density matrix of every
 * truncation becomes rho + noise * rho_P / tr(rho_P), rho_P the reduced
 * density matrix of (half of H_eff) x (White, PRB 72, 180403 (2005)); the
 * reference has no noise term, 0 restores its update exactly. */
int tt_qdmrg_set_noise(tt_qdmrg* run, double noise);
int tt_qdmrg_sweep(tt_qdmrg* run, int max_bd, double cutoff, int max_restart, double* energy);
int tt_qdmrg_finish(tt_qdmrg* run);                          /* psi.position(0) */
/* Two-site updates (the sweep's step: updateSite + updateEnv,
 * algos/dmrg/dmrg.cpp:300-372,491-509) moving the orthogonality centre from
 * its current site to to_site: left to right when to_site is larger, right to
 * left when smaller.  A sweep needs the centre at site 0 (where
 * tt_qdmrg_create and every sweep leave it).  *energy: the last step's. */
int tt_qdmrg_walk(tt_qdmrg* run, int to_site, int max_bd, double cutoff, int max_restart, double* energy);
int tt_qdmrg_position(const tt_qdmrg* run, int* site);
int tt_qdmrg_destroy(tt_qdmrg* run);
/* whole schedule overload dmrg(psi, H, nsweeps, maxm[], cutoff[], max_restart[]);
 * log_out (may be NULL) receives the run record (destroy with tt_qdmrg_destroy) */
int tt_qdmrg_run(tt_qmps* psi, tt_qmpo* H, int nsweeps, const int* maxm, int n_maxm, const double* cutoff,
                 int n_cutoff, const int* max_restart, int n_mr, double* energy, tt_qdmrg** log_out);
int tt_qdmrg_num_steps(const tt_qdmrg* run, int* n);
int tt_qdmrg_step(const tt_qdmrg* run, int i, int* site, int* direction, double* energy, double* trunc_err,
                  unsigned* kept, int* matvecs, double* heff_flops);
int tt_qdmrg_step_sectors(const tt_qdmrg* run, int i, int* n, int32_t* qn, uint32_t* kept, int cap);
/* per-step profile: largest sector density matrix of the SVD and host wall
 * seconds of the Davidson, SVD and environment-update phases */
int tt_qdmrg_step_profile(const tt_qdmrg* run, int i, int* gram_max, double* t_davidson, double* t_svd,
                          double* t_env, double* t_engine);
/* per-step device-stream spans in milliseconds, from events recorded on the
 * library stream at the phase boundaries: Davidson, SVD, environment update,
 * and the span from the previous logged step's end to this step's start
 * (gap; negative for the first step).  A span includes any time in which the
 * device waited for the host.  Waits for the step's last event. */
int tt_qdmrg_step_device_ms(const tt_qdmrg* run, int i, double* davidson, double* svd, double* env,
                            double* gap);
int tt_qdmrg_stats(const tt_qdmrg* run, double* heff_flops, double* heff_seconds, double* initial_energy);
/* copy of the left (which = 0, TL[i]) or right (which = 1, TR[i]) environment.
 * Only the environments on the live side of the orthogonality centre c are
 * kept (TL[0..c], TR[c..L-1], plus the boundaries): the others are released
 * as the centre passes them and come back empty (rank 0) until rebuilt. */
int tt_qdmrg_env(const tt_qdmrg* run, int which, int i, tt_qtensor** out);
int tt_qdmrg_num_sweeps(const tt_qdmrg* run, int* n);
int tt_qdmrg_sweep_info(const tt_qdmrg* run, int i, double* energy, double* seconds);

/* ---- dense (no QN) MPS / MPO / DMRG ------------------------------------------ */
typedef struct tt_dmps tt_dmps;
typedef struct tt_dmpo tt_dmpo;
/* MPS(sites, product string): 1 on the chosen spin, DBL_EPSILON elsewhere */
int tt_dmps_product_spinhalf(int L, const int* state, unsigned id, tt_dmps** out);
int tt_dmps_destroy(tt_dmps* psi);
int tt_dmps_bond_dims(const tt_dmps* psi, int* out);  /* L+1 entries */
int tt_dmps_length(const tt_dmps* psi, int* L);
/* hand-written Heisenberg MPO, bond dimension 5 */
int tt_dmpo_heisenberg(int L, const double* dh, double tE, unsigned id, tt_dmpo** out);
int tt_dmpo_destroy(tt_dmpo* H);
/* dmrg(MPS&, MPO&, nsweeps, maxm[], cutoff[], max_restart[]); sweep_energy
 * (nsweeps entries) and step_kept (2*(L-1)*nsweeps entries) may be NULL */
int tt_ddmrg_run(tt_dmps* psi, tt_dmpo* H, int nsweeps, const int* maxm, int n_maxm, const double* cutoff,
                 int n_cutoff, const int* max_restart, int n_mr, double* energy, double* sweep_energy,
                 int* step_kept);

/* ---- observables ----------------------------------------------------------------- */
/* <psi|phi> and <psi|H|phi> (unnormalised, as the reference) */
int tt_qmps_overlap(const tt_qmps* psi, const tt_qmps* phi, double* out);
int tt_qmps_expectation(const tt_qmps* psi, const tt_qmpo* H, const tt_qmps* phi, double* out);
/* <Sz_i> (L entries) and <Sz_i Sz_j> (L*L, row-major, symmetric), normalised
 * by <psi|psi>; either output may be NULL */
int tt_qmps_measure_sz(const tt_qmps* psi, double* sz, double* szsz);
int tt_dmps_overlap(const tt_dmps* psi, const tt_dmps* phi, double* out);
int tt_dmps_expectation(const tt_dmps* psi, const tt_dmpo* H, const tt_dmps* phi, double* out);
int tt_dmps_measure_sz(const tt_dmps* psi, double* sz, double* szsz);

/* ---- checkpoints ------------------------------------------------------------------ */
/* Metadata to fn + ".ttmps" (text: MPS attributes, indices, per-block sector
 * tuples and byte offsets); block data, dense column-major doubles back to
 * back in site and block order, to wfn (NULL: fn + "__T.bin"). */
int tt_qmps_save(const tt_qmps* psi, const char* fn, const char* wfn);
/* fn: the ".ttmps" file; data_prefix (may be NULL) is prepended to the
 * recorded raw file name */
int tt_qmps_load(const char* fn, const char* data_prefix, tt_qmps** out);
int tt_dmps_save(const tt_dmps* psi, const char* fn, const char* wfn);
int tt_dmps_load(const char* fn, const char* data_prefix, tt_dmps** out);

/* ---- AutoMPO and lattices ------------------------------------------------------ */
typedef struct tt_autompo tt_autompo;
int tt_autompo_create(tt_autompo** out);
int tt_autompo_destroy(tt_autompo* a);
/* ampo += coef, ops[0], sites[0], ...: operators are kept in site order, a zero
 * coefficient is dropped and a repeated operator list sums its coefficient */
int tt_autompo_add(tt_autompo* a, double coef, int nops, const char* const* ops, const int* sites);
int tt_autompo_size(const tt_autompo* a, int* n);
/* term k in the accumulator's order (operator lists sorted by length, then by
 * (site, name)); op names are copied NUL-terminated into names[16*j] for
 * j < min(*nops, cap), and their sites into sites[j] */
int tt_autompo_term(const tt_autompo* a, int k, double* coef, int* nops, char* names, int* sites, int cap);
/* MPO bond dimensions of the finite-state layout for N sites (N+1 entries);
 * with_charges selects the U(1) layout, which needs Sz / S+ / S- / Id only */
int tt_autompo_link_dims(const tt_autompo* a, int N, int with_charges, int* dims);
int tt_qmpo_from_autompo(const tt_autompo* a, int N, unsigned id, tt_qmpo** out);
int tt_dmpo_from_autompo(const tt_autompo* a, int N, unsigned id, tt_dmpo** out);
/* dims (4 entries) and, when data is not NULL, the column-major values of the
 * dense MPO tensor on site i (left link, ket site, bra site, right link) */
int tt_dmpo_tensor(const tt_dmpo* H, int i, int64_t* dims, double* data, int64_t cap);

enum { TT_LATTICE_SQUARE = 0, TT_LATTICE_SQUARE_NEXT_NEIGHBOR = 1, TT_LATTICE_TRIANGULAR = 2 };
/* OR'd into a square kind: snake site order (column x runs y = 1..Ny when x is
 * odd, Ny..1 when x is even); the reference numbers sites column by column
 * only (models/lattice/square.h:25-103), so this is a relabelling of the same
 * bonds with the smaller site first */
enum { TT_LATTICE_SNAKE = 0x100 };
/* 1-based sites, y fastest; type 0 unset, 1 nearest, 2 next-nearest neighbour;
 * coordinates are 0 where the reference records none (triangular) */
typedef struct {
  int s1, s2, type;
  double x1, y1, x2, y2;
} tt_lattice_bond;
/* writes min(*n_bonds, cap) bonds; *n_bonds is the full count */
int tt_lattice(int kind, int Nx, int Ny, int yperiodic, tt_lattice_bond* bonds, int cap, int* n_bonds);

#ifdef __cplusplus
}
#endif
#endif /* TT_DMRG_H */
