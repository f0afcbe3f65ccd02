/*
 * admp_b200 -- C ABI of the B200 (sm_100a) electrostatics hot path that sits
 * behind torch-admp's CoulombForceModule / QEqForceModule / TorchNeighborList.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer owned by the caller, except the
 *    arguments documented as "host".  `stream` is a cudaStream_t (void* here so
 *    this header needs no CUDA include).  Work is stream-ordered; entry points
 *    that must return a size to the host (the neighbour-list count and the QEq
 *    solver's convergence result) synchronise that stream.
 *  - `dtype` selects the element type of the floating-point arrays:
 *    ADMP_F64 (double) or ADMP_F32 (float).  Energies, virial-type reductions
 *    and the CG dot products are always double.
 *  - Gradient outputs ACCUMULATE (+=) into caller-zeroed buffers; NULL skips
 *    that output.  Energies accumulate into double buffers.
 *  - Index arrays (`pairs`) are int64 as produced by the reference
 *    (row-major [npairs, 2]).
 *  - Errors are never raised on the device: kernels record the first bad
 *    index / non-finite value in an error word that the entry point reads
 *    back, and return a status code.  admp_last_error_message() describes it.
 *  - Scratch memory is passed in by the caller (`workspace`); the
 *    *_workspace_size() queries give the bytes needed.  No entry point
 *    allocates device memory.
 */
#ifndef ADMP_B200_H_
#define ADMP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADMP_ABI_VERSION 1

/* status codes */
#define ADMP_OK 0
#define ADMP_ERR_BAD_ARG 1           /* shape / argument error (ValueError in the reference) */
#define ADMP_ERR_CUTOFF_TOO_LARGE 2  /* nblist.py:620-660 check_cutoff */
#define ADMP_ERR_NOT_CONVERGED 3     /* CG hit max_iter (qeq.py:1261-1262 "did not converge") */
#define ADMP_ERR_WORKSPACE 4         /* workspace too small */
#define ADMP_ERR_CUDA 5              /* CUDA runtime error */
#define ADMP_ERR_BAD_INDEX 6         /* pair index outside [0, natoms) */
#define ADMP_ERR_CAPACITY 7          /* output capacity too small */
#define ADMP_ERR_NONFINITE 8         /* NaN/Inf in positions or box */
#define ADMP_ERR_MESH 9              /* unsupported mesh size */

/* dtype codes */
#define ADMP_F64 0
#define ADMP_F32 1

/* pair-term modes for admp_pair_energy */
#define ADMP_PAIR_EWALD 0    /* erfc(kappa r) q_i q_j / r          pme.py:312-349 */
#define ADMP_PAIR_OBC 1      /* q_i q_j / r, safe_inverse 1e-8     pme.py:529-561 */
#define ADMP_PAIR_DAMPING 2  /* -erfc(r / 2 eta_ij) q_i q_j / r    qeq.py:60-129  */

/* flags for admp_atom_terms */
#define ADMP_TERM_SELF 1          /* pme.py:448-461 */
#define ADMP_TERM_NON_NEUTRAL 2   /* pme.py:463-493 */
#define ADMP_TERM_SLAB 4          /* pme.py:495-527 (axis in bits 8..9) */
#define ADMP_TERM_DAMP_SELF 8     /* qeq.py:121-126 */
#define ADMP_TERM_SITE 16         /* qeq.py:159-209 */

int admp_abi_version(void);
const char* admp_status_string(int status);
/* Human-readable detail of the last non-OK status on this host thread. */
const char* admp_last_error_message(void);
/* Synchronous device-error checks (default on): entry points that launch
 * kernels with index checks synchronise `stream` and report a bad index as a
 * status.  With checks off, errors stay recorded on the device until
 * admp_check_errors() (which always synchronises) reads and clears them. */
void admp_set_sync_checks(int on);
int admp_check_errors(void* stream);
/* Number of kernels this library has launched (all entry points). */
long long admp_launch_count(void);
/* Kernel profiler: when enabled (capacity > 0 event pairs; 0 disables) the
 * hot kernels are bracketed by CUDA events on their launch stream and tagged
 * with their algorithmic bytes.  admp_profile_read fills per-kernel totals
 * (index order: spread, fft_z_fwd, fft_y_fwd, fft_x_green, fft_y_inv,
 * fft_z_inv, gather, pair_ef, csr_spmv, neighbors, cg_vector, tc_z_fwd,
 * tc_y_fwd, tc_x, tc_y_inv, tc_z_inv; the tc_* entries are the FP32 CG
 * matvec's mesh passes on the tensor cores, the fft_* ones the shared-memory
 * FFT passes). */
#define ADMP_PROFILE_KERNELS 16
int admp_profile_enable(int capacity);
int admp_profile_read(double* ms, long long* launches, double* bytes, int n);

/* ------------------------------------------------------------------------ */
/* Reciprocal-space PME.                                                     */
/* Replaces CoulombForceModule._forward_pbc_reciprocal (pme.py:351-446) with  */
/* recip.spread_charges / setup_kpts / _coeff_k_1 (recip.py:216-308,          */
/* pme.py:661-683) and the autograd backward through them (utils.py:85-112). */
/* nframes systems of `natoms` each; kmesh is HOST [nframes*3].               */
/* Outputs per frame: energy (+=), dE/dpos [nf,N,3], dE/dq [nf,N],            */
/* dE/dbox [nf,3,3] (all optional, accumulated).                              */
/* ------------------------------------------------------------------------ */
size_t admp_pme_recip_workspace_size(int dtype, int nframes, const int* kmesh);
int admp_pme_recip(int dtype, int nframes, int natoms, const int* kmesh, const void* pos,
                   const void* box, const void* q, double kappa, double ke, double* energy,
                   void* dE_dpos, void* dE_dq, void* dE_dbox, void* workspace,
                   size_t workspace_bytes, void* stream);

/* Variant of admp_pme_recip that allocates nothing and takes no workspace,  */
/* for callers that cannot allocate device memory when they call (e.g. a    */
/* plugin inside an MD engine that owns all device memory, or a step loop   */
/* that must not trigger cudaMalloc's device-wide synchronisation).  It has */
/* no counterpart in the reference.  Its scratch is a fixed 16 MiB array in */
/* the library's device memory (admp_pme_recip_noalloc_max_scratch()), held */
/* by every GPU that loads the library until exit; calls needing more       */
/* scratch than that (admp_pme_recip_workspace_size) return               */
/* ADMP_ERR_WORKSPACE.  The first call on a device looks up the array's     */
/* device address (cudaGetSymbolAddress); with CUDA's lazy module loading   */
/* that first lookup also loads the library's module, which is when the    */
/* array itself is created (a device allocation that may synchronise).  So  */
/* make one call (or a warm-up call) per device before the region that must */
/* not allocate, and before any stream capture.  The looked-up address is   */
/* cached per device and is not valid after cudaDeviceReset.  All calls     */
/* share the array: calls that overlap on the GPU race.                     */
size_t admp_pme_recip_noalloc_max_scratch(void);
int admp_pme_recip_noalloc(int dtype, int nframes, int natoms, const int* kmesh, const void* pos,
                           const void* box, const void* q, double kappa, double ke, double* energy,
                           void* dE_dpos, void* dE_dq, void* dE_dbox, void* stream);

/* ------------------------------------------------------------------------ */
/* Pair terms over a caller pair list.                                       */
/* Replaces _forward_pbc_real (pme.py:312-349), _forward_obc (pme.py:529-561) */
/* and the pair part of GaussianDampingForceModule (qeq.py:104-119).          */
/* pairs [nf,P,2] int64, ds [nf,P], buffer_scales [nf,P] (dtype), q [nf,N],   */
/* eta [nf,N] (damping only).  Outputs (all accumulated): energy [nf],       */
/* dE/dds [nf,P], dE/dq [nf,N], dE/deta [nf,N].                               */
/* ------------------------------------------------------------------------ */
int admp_pair_energy(int dtype, int mode, int nframes, int natoms, long long npairs,
                     const long long* pairs, const void* ds, const void* buffer_scales,
                     const void* q, const void* eta, double kappa, double ke, double* energy,
                     void* dE_dds, void* dE_dq, void* dE_deta, void* stream);

/* ------------------------------------------------------------------------ */
/* Per-atom terms: Ewald self (pme.py:448-461), non-neutral correction        */
/* (pme.py:463-493), slab correction (pme.py:495-527), damping self energy    */
/* (qeq.py:121-126) and site energy chi q + hardness q^2 (qeq.py:159-209).    */
/* `terms` (optional) receives [nf][5] = self, non_neutral, slab, damp_self,  */
/* site.  pos/box are needed for SLAB / NON_NEUTRAL, eta for DAMP_SELF,       */
/* chi/hardness for SITE.  Gradients accumulate.                              */
/* ------------------------------------------------------------------------ */
int admp_atom_terms(int dtype, int flags, int nframes, int natoms, const void* pos, const void* box,
                    const void* q, const void* eta, const void* chi, const void* hardness,
                    double kappa, double ke, double* energy, double* terms, void* dE_dq,
                    void* dE_dpos, void* dE_dbox, void* dE_deta, void* dE_dchi, void* dE_dhard,
                    void* stream);

/* ------------------------------------------------------------------------ */
/* Pair distances ds = |pbc_shift(r_i - r_j)| (nblist.py:517-551,            */
/* spatial.py:15-36) or |r_j - r_i| without a box (pbc = 0), and their       */
/* backward (gradient of a loss w.r.t. positions and box given dL/dds).       */
/* ------------------------------------------------------------------------ */
int admp_pair_distances(int dtype, int pbc, int natoms, long long npairs, const long long* pairs,
                        const void* pos, const void* box, void* ds, void* stream);
int admp_pair_distances_backward(int dtype, int pbc, int natoms, long long npairs,
                                 const long long* pairs, const void* pos, const void* box,
                                 const void* grad_ds, void* grad_pos, void* grad_box, void* stream);

/* ------------------------------------------------------------------------ */
/* Cell-list neighbour list: TorchNeighborList.forward (nblist.py:304-445,   */
/* 472-490) incl. check_cutoff (nblist.py:620-660).  Full list (both         */
/* orders), 0.01 < r < rc with a box, r < rc without.  Two phases:            */
/*   admp_nblist_count  -> *npairs (host), synchronises `stream`;            */
/*   admp_nblist_fill   -> pairs [npairs,2] int64 sorted by (i, j) and        */
/*                         buffer_scales [npairs] int64 (1 if i < j).         */
/* The same workspace must be passed to both calls.                           */
/* ------------------------------------------------------------------------ */
size_t admp_nblist_workspace_size(int natoms);
int admp_nblist_count(int dtype, int pbc, int natoms, const void* pos, const void* box,
                      double cutoff, void* workspace, size_t workspace_bytes, long long* npairs,
                      void* stream);
int admp_nblist_fill(int dtype, int pbc, int natoms, const void* pos, const void* box,
                     double cutoff, void* workspace, size_t workspace_bytes, long long* pairs,
                     long long* buffer_scales, long long capacity, void* stream);

/* ------------------------------------------------------------------------ */
/* Neighbour list over periodic images for any cutoff, including rc above   */
/* half the box: replaces dp_nblist (nblist.py:33-93) with its               */
/* make_extended_pairs / make_local_pairs / make_ds (nblist.py:140-240).    */
/* Pairs (i, j, n) with |r_j - r_i + n.B| <= rc: first every i < j image    */
/* (buffer scale 1), then every self image (i, i, n != 0) (scale 1/2).      */
/* nnei >= 0 keeps each atom's nnei nearest images, as the per-atom `sel`   */
/* truncation of the list dp_nblist is built from (ties at the nnei-th      */
/* distance are all kept); nnei < 0 keeps all.  Two phases, one workspace:  */
/*   admp_image_nblist_count -> *n_ij, *n_ii (host; synchronises `stream`), */
/*                              *n_truncated = atoms that hit nnei;         */
/*   admp_image_nblist_fill  -> pairs [n_ij+n_ii, 2] int64 (i-major), and   */
/*                              shifts [n_ij+n_ii, 3] int32 image vectors n.*/
/* pbc = 0 (box may be NULL): plain pairs within rc, no images.             */
/* Pair distances and their backward for pairs with image shifts:           */
/* ds = |r_j - r_i + n.B|; the box gradient is sum_p n_p (x) dL/d(dr_p).     */
/* ------------------------------------------------------------------------ */
size_t admp_image_nblist_workspace_size(int natoms);
int admp_image_nblist_count(int dtype, int pbc, int natoms, const void* pos, const void* box,
                            double cutoff, int nnei, void* workspace, size_t workspace_bytes,
                            long long* n_ij, long long* n_ii, int* n_truncated, void* stream);
int admp_image_nblist_fill(int dtype, int pbc, int natoms, const void* pos, const void* box,
                           double cutoff, void* workspace, size_t workspace_bytes, long long* pairs,
                           int* shifts, long long capacity, void* stream);
int admp_image_pair_distances(int dtype, int natoms, long long npairs, const long long* pairs,
                              const int* shifts, const void* pos, const void* box, void* ds,
                              void* stream);
int admp_image_pair_distances_backward(int dtype, int natoms, long long npairs,
                                       const long long* pairs, const int* shifts, const void* pos,
                                       const void* box, const void* grad_ds, void* grad_pos,
                                       void* grad_box, void* stream);

/* ------------------------------------------------------------------------ */
/* Matrix-free projected CG solve of the QEq charges: replaces               */
/* pgrad_optimize / QEqForceModule.solve_pgrad (qeq.py:609-712, 1117-1270)   */
/* and the quadratic / LBFGS minimisers (qeq.py:1273-1527).  Minimises       */
/* E(q) = site + Coulomb(PME) + damping subject to C q = b with linear CG    */
/* (E is quadratic in q); stops when ||P grad||_2 / N < tol (qeq.py:1516).   */
/*   flags: ADMP_QEQ_* below; kmesh HOST [3]; C [n_const, N] dtype;           */
/*   b HOST [n_const] (double); q in: initial guess, out: solution.           */
/*   rhs_shift: optional [N] added to chi (electrode potential b-vector).     */
/* Returns ADMP_ERR_NOT_CONVERGED (q still written) when max_iter is hit.    */
/* ------------------------------------------------------------------------ */
#define ADMP_QEQ_KSPACE 1
#define ADMP_QEQ_RSPACE 2
#define ADMP_QEQ_DAMPING 4
#define ADMP_QEQ_SLAB 8         /* slab axis in bits 8..9 */
#define ADMP_QEQ_PROJECT_Q0 16  /* project the initial guess onto C q = b first */
size_t admp_qeq_workspace_size(int dtype, int natoms, long long npairs, const int* kmesh,
                               int n_const);
int admp_qeq_solve(int dtype, int flags, int natoms, const int* kmesh, const void* pos,
                   const void* box, long long npairs, const long long* pairs, const void* ds,
                   const void* buffer_scales, const void* chi, const void* hardness,
                   const void* eta, const void* rhs_shift, double kappa, double ke, int n_const,
                   const void* C, const double* b, void* q, double tol, int max_iter,
                   int* iters, double* resid, void* workspace, size_t workspace_bytes,
                   void* stream);

/* Several frames of the same atom count in one solve (the differentiation */
/* batch: jittered frames of one system, and the implicit adjoint of their   */
/* charges).  The reference solves one frame per pgrad_optimize call          */
/* (qeq.py:1117-1270); per frame the arithmetic and the stopping rule are the */
/* same as admp_qeq_solve.  Frame f holds atoms [f N, (f+1) N) of pos, chi,   */
/* hardness, eta, rhs_shift and q, box f, and mesh kmesh[3f .. 3f+2] (HOST    */
/* [nframes, 3]); pairs index atoms over all frames (frame f's pairs use     */
/* indices f N + i); C [n_const, N] and b (HOST [n_const]) are shared by      */
/* every frame.  iters, resid: HOST [nframes] or NULL.  nframes <= 256.       */
size_t admp_qeq_frames_workspace_size(int dtype, int nframes, int natoms, long long npairs,
                                      const int* kmesh, int n_const);
int admp_qeq_solve_frames(int dtype, int flags, int nframes, int natoms, const int* kmesh,
                          const void* pos, const void* box, long long npairs,
                          const long long* pairs, const void* ds, const void* buffer_scales,
                          const void* chi, const void* hardness, const void* eta,
                          const void* rhs_shift, double kappa, double ke, int n_const,
                          const void* C, const double* b, void* q, double tol, int max_iter,
                          int* iters, double* resid, void* workspace, size_t workspace_bytes,
                          void* stream);

/* Hessian-vector product of the same quadratic form (dE/dq at p minus at   */
/* 0): out [N] = H p.  Used by the implicit adjoint of the charge solve.      */
int admp_qeq_hvp(int dtype, int flags, int natoms, const int* kmesh, const void* pos,
                 const void* box, long long npairs, const long long* pairs, const void* ds,
                 const void* buffer_scales, const void* hardness, const void* eta, double kappa,
                 double ke, const void* p, void* out, void* workspace, size_t workspace_bytes,
                 void* stream);

/* admp_qeq_hvp for nframes frames at once (the layout of                     */
/* admp_qeq_solve_frames; workspace from admp_qeq_frames_workspace_size):    */
/* out [nframes, N] = H_f p_f.  The dense Hessian of matinv_optimize /       */
/* calc_hessian (qeq.py:460-515, 1620-1670) is built from these, one batch   */
/* of unit vectors (frames of the same geometry) per call, instead of one    */
/* autograd pass per column.                                                 */
int admp_qeq_hvp_frames(int dtype, int flags, int nframes, int natoms, const int* kmesh,
                        const void* pos, const void* box, long long npairs,
                        const long long* pairs, const void* ds, const void* buffer_scales,
                        const void* hardness, const void* eta, double kappa, double ke,
                        const void* p, void* out, void* workspace, size_t workspace_bytes,
                        void* stream);

/* ------------------------------------------------------------------------ */
/* Batched serving.  Many independent systems (PME energy+forces requests or */
/* QEq solves) run per launch; their state lives in caller-owned pools so a   */
/* scheduler can admit new systems and retire finished ones between CG        */
/* iterations.  There is no reference counterpart: the reference evaluates   */
/* one system per Python call (CoulombForceModule.forward, pgrad_optimize);   */
/* the per-system arithmetic is the same as the entry points above (FP32 or  */
/* FP64 bulk, double reductions), with the total-charge constraint.          */
/* ------------------------------------------------------------------------ */
#define ADMP_SYS_PME 0
#define ADMP_SYS_QEQ 1

typedef struct admp_sys {
  int natoms;          /* atoms of the system */
  int atom_off;        /* first atom in the per-atom pools */
  int slot;            /* index into the per-slot pools (box, energy, CG state) */
  int kind;            /* ADMP_SYS_PME or ADMP_SYS_QEQ */
  int kmesh[3];
  int pad;
  long long pair_off;  /* first entry in the pair pools */
  long long pair_cap;  /* entries reserved for this system's neighbour rows */
  long long green_off; /* QEq: first element of its cached Green's function in pools->green
                        * (K0*K1*(K2/2+1) elements); unused for PME systems */
  double kappa;
  double rcut;
} admp_sys;

typedef struct admp_pools {
  /* per atom (dtype) */
  void* pos;           /* [A,3] */
  void* q;             /* [A]   charges; QEq warm start in, solution out */
  void* chi;           /* [A]   QEq electronegativity */
  void* hardness;      /* [A] */
  void* eta;           /* [A]   Gaussian widths */
  void* force;         /* [A,3] forces out */
  void* frac;          /* [A]   float4 (F32) / double4 (F64) scratch */
  long long* pstart;   /* [A]   first pair entry of the atom's row */
  int* pcnt;           /* [A]   row length */
  int* cell_of;        /* [A]   scratch */
  int* sorted;         /* [A]   scratch */
  /* per pair */
  int* col;            /* [P]   neighbour atom (pool index) */
  void* coef;          /* [P]   QEq real-space matrix entries (dtype) */
  /* per slot */
  void* box;           /* [S,3,3] */
  double* energy;      /* [S] */
  void* cg_state;      /* [S] x admp_serve_slot_state_bytes() */
  int* slot_info;      /* [S,4]: done, iterations, status, pairs needed */
  /* CG vectors per atom */
  double* cg_x;
  double* cg_r;
  double* cg_diag;
  double* cg_z;
  double* cg_chi;
  double* cg_hx;
  void* cg_p;          /* dtype */
  void* cg_hp;         /* dtype */
  /* per-launch scratch */
  void* mesh;          long long mesh_cap;   /* dtype elements */
  void* spec;          long long spec_cap;   /* complex elements */
  double* acc;         int acc_cap;          /* systems (32 doubles each) */
  int* cells;          long long cells_cap;  /* ints */
  void* sys_scratch;   long long sys_scratch_bytes;
  void* green;         long long green_cap;  /* dtype: cached Green's functions of QEq slots */
  /* optional double copies used only for the neighbour decisions of FP32
   * pools (which pairs lie inside rc), so the pair set equals the FP64 one */
  double* pos64;       /* [A,3] or NULL */
  double* box64;       /* [S,3,3] or NULL */
  void* frac64;        /* [A] double4 scratch, needed with pos64 */
  int flags;           /* reserved, 0 */
  double* slot_resid;  /* optional [S]: ||P grad||_2 / N of each QEq slot's latest iterate */
} admp_pools;

size_t admp_serve_slot_state_bytes(void);
size_t admp_serve_sys_scratch_bytes(int nsys);
size_t admp_serve_cells_needed(const admp_sys* sys, int nsys);
/* neighbour rows of the listed systems: atom a of a system gets the row slot
 * col[pair_off + a * (pair_cap / natoms) ..] (pstart, pcnt); slot_info[.,2]
 * gets the status (cutoff too large, non-finite input, or ADMP_ERR_CAPACITY
 * when a row outgrew its slot) and slot_info[.,3] the pair entries the system
 * needs after an overflow (natoms x longest row), else 0.                  */
int admp_serve_neighbors(int dtype, const admp_pools* pools, const admp_sys* sys, int nsys, void* stream);
/* energy [slot] and forces of the listed systems at the charges in pools->q:
 * PME systems: Ewald real + reciprocal + self + non-neutral (pme.py:261-310);
 * QEq systems: additionally Gaussian damping and site terms (qeq.py:408-458). */
int admp_serve_energy_forces(int dtype, const admp_pools* pools, const admp_sys* sys, int nsys, double ke,
                             void* stream);
/* QEq CG state of the listed systems from the warm start in pools->q. */
int admp_serve_qeq_init(int dtype, const admp_pools* pools, const admp_sys* sys, int nsys, double tol,
                        int max_iter, double ke, void* stream);
/* niter CG iterations of the listed systems (converged ones are skipped);
 * slot_info[.,0..1] get done flags and iteration counts. */
int admp_serve_qeq_iterate(int dtype, const admp_pools* pools, const admp_sys* sys, int nsys, int niter,
                           double tol, int max_iter, double ke, void* stream);
/* copy the CG solution into pools->q */
int admp_serve_qeq_finish(int dtype, const admp_pools* pools, const admp_sys* sys, int nsys, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ADMP_B200_H_ */
