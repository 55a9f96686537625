/* sdpa_b200 C ABI: the drop-in boundary of the B200 SDP solver.
 *
 * Plain C types only (no C++ or torch types), int status codes (0 = success,
 * negative = error; see SDPAB_E*), explicit CUDA stream handles passed as
 * void*.  Two families:
 *
 *  1. Whole-problem handle API mirroring the reference's public C++ class
 *     SDPA (sdpa_call.h:91-267): create, read .dat-s / parameter files or
 *     input elements, initializeSolve, solve, result getters.  The C++ class
 *     of the same shape is declared in sdpa_call.h of this directory; these
 *     functions are its C binding for FFI callers (ctypes, MEX, cgo ...).
 *
 *  2. Batched API: thousands of small SDPs (one SDP block, or several SDP
 *     blocks and LP blocks per instance) solved by one persistent
 *     kernel launch (no counterpart in the reference, which solves one problem
 *     per process; its per-problem semantics are those of SDPA::solve,
 *     sdpa_solve.cpp:59-233).
 *
 * Index conventions of the batched API: entries are 0-based (row, col) with
 * row <= col (upper triangle, as SDPA stores them, sdpa_struct.h:82-139);
 * matrix 0 of an instance is F0 as written in the .dat-s file (the solver
 * negates it to C = -F0 like IO::setElement, sdpa_io.cpp:511), matrices
 * 1..m are F_1..F_m.  Results follow the reference's getters: xvec is
 * getResultXVec (sdpa_call.cpp:668-671), X is getResultXMat (the solver's
 * internal Z, :673-694), Y is getResultYMat (internal X, :696-717),
 * primal/dual objectives are getPrimalObj / getDualObj (:719-729), phase is
 * getPhaseValue's code (:769-786).
 */
#ifndef SDPA_B200_H
#define SDPA_B200_H

#if defined(__GNUC__)
#define SDPAB_API __attribute__((visibility("default")))
#else
#define SDPAB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SDPAB_OK 0
#define SDPAB_EINVAL (-1)      /* invalid argument */
#define SDPAB_ECUDA (-2)       /* CUDA runtime error (message via sdpab_last_error) */
#define SDPAB_ESIZE (-3)       /* instance larger than the configured limits */
#define SDPAB_ENODEV (-4)      /* no CUDA device */
#define SDPAB_ESTATE (-5)      /* call out of order (e.g. solve before input) */
#define SDPAB_EIO (-6)         /* file could not be opened or parsed */

/* Phase codes: SDPA::PhaseType order (sdpa_call.h:95-96). */
#define SDPAB_noINFO 0
#define SDPAB_pFEAS 1
#define SDPAB_dFEAS 2
#define SDPAB_pdFEAS 3
#define SDPAB_pdINF 4
#define SDPAB_pFEAS_dINF 5
#define SDPAB_pINF_dFEAS 6
#define SDPAB_pdOPT 7
#define SDPAB_pUNBD 8
#define SDPAB_dUNBD 9

/* Solver parameters, the ten numeric fields of the reference's Parameter
 * (sdpa_parts.h; param.sdpa lines 1-10, read by Parameter::readFile,
 * sdpa_parts.cpp:231-263). */
typedef struct sdpab_params {
  int maxIteration;
  double epsilonStar, lambdaStar, omegaStar, lowerBound, upperBound;
  double betaStar, betaBar, gammaStar, epsilonDash;
} sdpab_params;

/* Fills p with Parameter::setDefaultParameter(type) (sdpa_parts.cpp:182-224):
 * 0 = PARAMETER_DEFAULT, 1 = UNSTABLE_BUT_FAST, 2 = STABLE_BUT_SLOW. */
SDPAB_API int sdpab_default_params(int type, sdpab_params* p);

/* Reads the ten numeric lines of a param.sdpa file
 * (replaces Parameter::readFile, sdpa_parts.cpp:231-263). */
SDPAB_API int sdpab_read_params(const char* path, sdpab_params* p);

/* Last error message of the calling thread (static storage). */
SDPAB_API const char* sdpab_last_error(void);

/* Library version string. */
SDPAB_API const char* sdpab_version(void);

/* ------------------------------------------------------- whole-problem API */

/* Opaque handle of one problem: a C binding of the drop-in C++ class SDPA
 * (sdpa_call.h in this directory), for FFI callers.  The solve is the
 * host-driven CUDA solver: any number of SDP blocks plus LP blocks. */
typedef struct sdpab_sdpa sdpab_sdpa;

typedef struct sdpab_sdpa_info_t {
  double primal_obj, dual_obj;       /* getPrimalObj / getDualObj */
  double primal_error, dual_error;   /* getPrimalError / getDualError */
  double mu, duality_gap;            /* getMu / getDualityGap */
  double solve_seconds;              /* getSolveTime */
  int iterations;                    /* getIteration */
  int phase;                         /* getPhaseValue code */
  int m, nblock;                     /* getConstraintNumber / getBlockNumber */
} sdpab_sdpa_info_t;

/* new SDPA() / delete (sdpa_call.cpp:38-55) */
SDPAB_API sdpab_sdpa* sdpab_sdpa_new(void);
SDPAB_API void sdpab_sdpa_free(sdpab_sdpa* h);
/* setParameter* (sdpa_call.cpp:62-143) from the ten numeric parameters */
SDPAB_API int sdpab_sdpa_set_params(sdpab_sdpa* h, const sdpab_params* prm);
/* SDPA::readInput (sdpa_call.cpp:897-944); sparse_type: 0 AUTO (by the
 * ".dat-s" suffix), 1 SPARSE, 2 DENSE */
SDPAB_API int sdpab_sdpa_read_input(sdpab_sdpa* h, const char* path, int sparse_type);
/* SDPA::setInitPoint(true) + SDPA::readInit (sdpa_call.cpp:946-991) */
SDPAB_API int sdpab_sdpa_read_init(sdpab_sdpa* h, const char* path, int sparse_type);
/* SDPA::readParameter (sdpa_call.cpp:993-1003) */
SDPAB_API int sdpab_sdpa_read_param(sdpab_sdpa* h, const char* path);
/* inputConstraintNumber / inputBlockNumber / inputBlockSize / inputBlockType /
 * inputCVec / inputElement (sdpa_call.cpp:245-341) for nnz 1-based entries
 * (k = 0 is F0) followed by initializeUpperTriangle */
SDPAB_API int sdpab_sdpa_input_problem(sdpab_sdpa* h, int m, int nblock, const int* block_struct,
                                       const double* c, long long nnz, const int* k, const int* l,
                                       const int* i, const int* j, const double* v);
/* setInitPoint(true) + inputInitXVec / inputInitXMat / inputInitYMat
 * (sdpa_call.cpp:148-159, :343-434); X[l], Y[l] dense column-major per SDP
 * block, a vector per LP block */
SDPAB_API int sdpab_sdpa_set_init(sdpab_sdpa* h, const double* xvec, const double* const* X,
                                  const double* const* Y);
/* Precision of the solve (no reference counterpart): SDPAB_PREC_FP64, or
 * SDPAB_PREC_MIXED = FP32 products and FP32 Schur Cholesky with FP64
 * iterative refinement of dy while the relative complementarity gap
 * nDim * mu / max(1, (|objP| + |objD|) / 2) >= mu_switch (0 = 1e-2), FP64
 * after. */
SDPAB_API int sdpab_sdpa_set_precision(sdpab_sdpa* h, int mode, double mu_switch);
/* Bound on the polls of every wait in the mixed mode's tensor-core pipelines
 * (no reference counterpart; < 0: the default bound).  A pipeline that gives
 * up makes that iteration use the FP64 Schur factor or the SIMT products; a
 * small bound exercises that fall-back in tests. */
SDPAB_API int sdpab_sdpa_set_tc_wait(sdpab_sdpa* h, long long polls);
/* Tensor-core pipelines that gave up during the last solve (their
 * iterations fell back as above). */
SDPAB_API int sdpab_sdpa_tc_timeouts(sdpab_sdpa* h, int* out);
/* SDPA::initializeSolve + SDPA::solve (sdpa_solve.cpp:10-43, :59-233) */
SDPAB_API int sdpab_sdpa_solve(sdpab_sdpa* h);
/* scalar getters (sdpa_call.cpp:719-847) */
SDPAB_API int sdpab_sdpa_info(sdpab_sdpa* h, sdpab_sdpa_info_t* out);
/* The constraint order of the host-driven solver's Schur factorisation (no
 * counterpart in the reference, which leaves the order to MUMPS when it
 * takes its sparse path, Chordal::ordering_bMat, sdpa_chordal.cpp:365-524).
 * Problems of two or more SDP blocks and at least 512 constraints are put in
 * a minimum-degree order of the constraint groups (constraints sharing an
 * SDP block or an LP coordinate) when that leaves fewer 128 x 128 tile pairs
 * in the symbolic factorisation than the caller's order; results always
 * come back in the caller's order (SDPAB_ORDER=natural in the environment
 * keeps the caller's order).  Host only, no device work: order[position] =
 * constraint (0-based), pairs[0] / pairs[1] = the symbolic tile pairs in the
 * caller's / the returned order.  Entries as for sdpab_sdpa_input_problem. */
SDPAB_API int sdpab_constraint_order(int m, int nblock, const int* block_struct, long long nnz, const int* k,
                                     const int* l, const int* i, const int* j, int* order, long long* pairs);

/* Device seconds per solver phase (the reference's ComputeTime categories,
 * sdpa_parts.h:48-86): out8 = rMat+gVec, bMat, Cholesky, solves, dX/dZ,
 * step length, update (inverses), residuals. */
SDPAB_API int sdpab_sdpa_phase_times(sdpab_sdpa* h, double* out8);
/* Schur factorisation of the last solve (no counterpart in the reference,
 * whose choice between the dense and the MUMPS sparse factorisation is
 * internal, Chordal::ordering_bMat, sdpa_chordal.cpp:365-524): *sparse = 1
 * when the factorisation skipped the 128 x 128 tiles its symbolic pattern
 * leaves zero; pairs[0] / pairs[1] = trailing tile pairs updated / of the
 * dense factorisation.  SDPAB_SCHUR=dense or =sparse in the environment
 * forces the mode. */
SDPAB_API int sdpab_sdpa_schur_pattern(sdpab_sdpa* h, int* sparse, long long* pairs);
/* getResultXVec (sdpa_call.cpp:668-671), copied into out[m] */
SDPAB_API int sdpab_sdpa_get_xvec(sdpab_sdpa* h, double* out);
/* getResultXMat (which = 0) / getResultYMat (which = 1) of block l
 * (sdpa_call.cpp:673-717), copied into out */
SDPAB_API int sdpab_sdpa_get_block(sdpab_sdpa* h, int l, int which, double* out);
/* getBlockSize / getBlockType (sdpa_call.cpp:813-847) */
SDPAB_API int sdpab_sdpa_block_size(sdpab_sdpa* h, int l, int* size, int* is_sdp);
/* SDPA::getDimacsError (IO::computeDimacs, sdpa_io.cpp:775-813): err7[1..6];
 * the norms, X . Z and the minimum eigenvalues are computed on the GPU. */
SDPAB_API int sdpab_sdpa_dimacs(sdpab_sdpa* h, double* err7);
/* Minimum eigenvalue of a symmetric n x n matrix (DEVICE pointer, column-major,
 * lower triangle referenced) into *out (host), computed on the GPU: the
 * dsyev minimum of Lal::getMinEigenValue (sdpa_linear.cpp:145-182) that
 * IO::computeDimacs takes of X and Z.  Synchronises `stream`. */
SDPAB_API int sdpab_min_eigenvalue(int n, const double* A, double* out, void* stream);
/* SDPA::writeInitSparse (sdpa_call.cpp:1199-1220) */
SDPAB_API int sdpab_sdpa_write_init(sdpab_sdpa* h, const char* path);
/* SDPA::copyCurrentToInit (sdpa_call.cpp:1238-1245) + setInitPoint(true) */
SDPAB_API int sdpab_sdpa_copy_current_to_init(sdpab_sdpa* h);

/* ------------------------------------------------ learned warm start (MPNN) */

/* No counterpart in the reference.  A 3-layer message-passing network over
 * the MaxCut graph predicts, per node, r_i = 4 x_i / d_i (x = SDPA's x
 * vector, d = weighted degree); the batched solver turns the proposed x into
 * a strictly interior start (SDPAB_INIT_DUAL).  BF16 weights, FP32
 * accumulation, hand-written forward / backward / Adam kernels; all pointers
 * are device pointers. */
#define SDPAB_MPNN_HIDDEN 64
#define SDPAB_MPNN_FEATURES 8
#define SDPAB_MPNN_LAYERS 3

typedef struct sdpab_graph_batch {
  int num_nodes;           /* nodes of all graphs of the batch */
  long long num_edges;     /* directed edges (each undirected edge twice) */
  const int* rowptr;       /* [num_nodes+1] CSR over destination nodes */
  const int* col;          /* [num_edges] source node of each edge */
  const float* aval;       /* [num_edges] a_ij = w_ij / (d_i + 1)  (i destination) */
  const float* aval_t;     /* [num_edges] a_ji for the same (i, j) slot (transpose) */
  const float* feat;       /* [num_nodes * SDPAB_MPNN_FEATURES] node features */
  int mask_count;          /* nodes counted by the loss mask (0 = all) */
} sdpab_graph_batch;

SDPAB_API long long sdpab_mpnn_num_params(void);
/* float counts of the activation and backward scratch buffers for num_nodes */
SDPAB_API long long sdpab_mpnn_act_floats(int num_nodes);
SDPAB_API long long sdpab_mpnn_scratch_floats(int num_nodes);
/* out[num_nodes] = predicted r per node */
SDPAB_API int sdpab_mpnn_forward(const sdpab_graph_batch* g, const unsigned short* weights_bf16, float* act,
                                 float* out, void* stream);
/* loss = sum_i mask_i (r_i - target_i)^2 / count and grads[num_params] */
SDPAB_API int sdpab_mpnn_loss_grad(const sdpab_graph_batch* g, const unsigned short* weights_bf16, float* act,
                                   float* scratch, const float* target, const float* mask, float* grads,
                                   float* loss, void* stream);
/* one Adam step on the FP32 master weights, refreshing the BF16 copy */
SDPAB_API int sdpab_mpnn_adam(float* master, unsigned short* weights_bf16, const float* grads, float* m1,
                              float* m2, int step, float lr, float beta1, float beta2, float eps,
                              float weight_decay, void* stream);
SDPAB_API int sdpab_mpnn_to_bf16(const float* master, unsigned short* weights_bf16, void* stream);
/* proposed SDPA x vector from the network output: x_i = r_i d_i / 4 for nodes
 * with edges, fallback_i for isolated nodes (node order = packed batch order) */
SDPAB_API int sdpab_mpnn_propose_x(int num_nodes, const float* r, const double* degree, const double* fallback,
                                   double* xvec, void* stream);

/* ---------------------------------------------------------------- batched API */

/* Precision modes of the batched solver. */
#define SDPAB_PREC_FP64 0    /* every step in FP64 (the plain path) */
#define SDPAB_PREC_MIXED_SIMT 2   /* host-driven solver: mixed without tensor cores (comparison) */
#define SDPAB_PREC_MIXED 1   /* while nDim * mu / max(1, mean |objective|) >=
                                mixed_switch_gap: the Schur Cholesky in FP32 with FP64
                                iterative refinement of dy (predictor and corrector
                                solves), and bulk products in FP32 (FP32 accumulation;
                                in the batched solver only with mixed_products = 1, else
                                on the FP64 MMA); FP64 residuals, gap, Lanczos step
                                length and factorisations of X and Z; everything FP64
                                once mu falls below that point, and in the batched
                                solver also once an FP32 factor fails or a refinement
                                does not converge in three steps */

typedef struct sdpab_batch {
  int count;                   /* number of instances */
  int nmax, mmax;              /* upper bounds of n and m over the batch */
  const int* n;                /* [count] matrix order (sum of the block orders) */
  const int* m;                /* [count] number of constraints */
  const long long* vec_off;    /* [count] offset of the instance's b / xvec (m doubles) */
  const double* b;             /* c vector of the .dat-s file (b of the internal problem) */
  const long long* mat_off;    /* [count] offset into mat_ptr of the instance's m+2 pointers */
  const long long* mat_ptr;    /* entry ranges: matrix k of instance i is
                                  [mat_ptr[mat_off[i]+k], mat_ptr[mat_off[i]+k+1]) */
  const int* row;              /* entries: 0-based row (row <= col) */
  const int* col;              /* entries: 0-based column */
  const double* val;           /* entries: value as written in the file */
  const long long* dense_off;  /* [count] offset of the instance's n*n blocks in X / Y arrays */
  /* Block structure (optional; NULL nblock = one SDP block of order n, and
   * every Schur entry by formula F3, the fast path for MaxCut-like
   * constraints with one or two entries).  A batch that sets it runs the
   * general solver: block structure, and per constraint the reference's
   * choice between F1 and F3 (sdpa_newton.cpp:515-695); set it (one block of
   * order n is allowed) for constraints with many entries.  An
   * instance's blocks (bLOCKsTRUCT of the .dat-s file: positive = SDP block,
   * negative = LP block of that many diagonal entries; order 1 counts as LP,
   * sdpa_block.cpp:80-91) lie along the diagonal of its n x n matrices,
   * n = sum |size|, in file order; row / col are those global indices.  An
   * entry must lie inside one block, and inside an LP block on its diagonal.
   * X / Y results are the block-diagonal n x n matrices. */
  const int* nblock;           /* [count] number of blocks (1 .. SDPAB_BATCH_MAX_BLOCKS) */
  const int* blk_off;          /* [count] offset of the instance's sizes in blk_size */
  const int* blk_size;         /* signed block orders */
} sdpab_batch;

#define SDPAB_BATCH_MAX_BLOCKS 64  /* blocks per instance in a batch */

#define SDPAB_INIT_NONE 0      /* standard start lambda* I */
#define SDPAB_INIT_POINT 1     /* start from the given (x, X, Y) */
#define SDPAB_INIT_DUAL 2      /* start from a proposed x only (constraints X_ii = b_i, i.e.
                                  F_i = e_i e_i^T): the solver shifts x until
                                  X = sum F_i x_i - F0 is positive definite with margin
                                  init_margin * mean |F0_ii|, and sets
                                  Y = D X^-1 D with unit-scaled diagonal */
#define SDPAB_INIT_FACTOR 3    /* start from a low-rank factor V of the user Y (constraints
                                  X_ii = b_i as for SDPAB_INIT_DUAL; row i of V has norm
                                  sqrt(b_i)), e.g. from sdpab_lowrank_factor.  The solver forms
                                  Y = V V^T, the multipliers x_i = (F0 Y)_ii / b_i and
                                  X = sum F_i x_i - F0, and starts on the central path's
                                  equation Y0 X0 = mu I at
                                    mu = max(init_mu, 3 rho) s,  s = mean |F0_ii|,
                                    rho = |X V|_F / (|V|_F s) (the factor's stationarity
                                    residual, 0 at the optimum),  tau = 0.3 sqrt(mu s):
                                    X0 = X + mu (Y + tau I)^-1 + delta I,  Y0 = mu X0^-1,
                                  delta the first of 0, mu/n, 4 mu/n, 16 mu/n, ... that makes X0
                                  positive definite (x shifted by delta to match).  No
                                  counterpart in the reference, which starts only from a given
                                  point or lambda* I.  Instances not of this form take the
                                  standard start (status 1). */

typedef struct sdpab_batch_init {
  const int* flag;             /* [count] SDPAB_INIT_* per instance */
  const double* xvec;          /* x (vec_off layout), as SDPA::inputInitXVec */
  const double* X;             /* user X (dense_off layout), as inputInitXMat */
  const double* Y;             /* user Y (dense_off layout), as inputInitYMat */
  double init_margin;          /* SDPAB_INIT_DUAL interiority margin (0 = 0.02) */
  const double* V;             /* SDPAB_INIT_FACTOR: instance q's factor, n x rank row-major, at
                                  V + vec_off[q] * rank (may be NULL otherwise) */
  int rank;                    /* columns of V */
  double init_mu;              /* SDPAB_INIT_FACTOR: the smallest start mu relative to
                                  mean |F0_ii| (0 = 3e-6) */
} sdpab_batch_init;

typedef struct sdpab_batch_result {
  double* xvec;                /* [vec_off layout] getResultXVec; may be NULL */
  double* X;                   /* [dense_off layout] getResultXMat(1); may be NULL */
  double* Y;                   /* [dense_off layout] getResultYMat(1); may be NULL */
  double* primal_obj;          /* [count] getPrimalObj */
  double* dual_obj;            /* [count] getDualObj */
  double* mu;                  /* [count] getMu */
  double* primal_error;        /* [count] getPrimalError */
  double* dual_error;          /* [count] getDualError */
  int* iterations;             /* [count] getIteration */
  int* phase;                  /* [count] getPhaseValue code */
  int* status;                 /* [count] 0 ok; 1 warm start not usable (standard start
                                  used); 2 warm-started or mixed-precision solve ended
                                  outside pdOPT and was solved again from the standard
                                  start in FP64 (iterations count both attempts);
                                  <0 instance rejected */
} sdpab_batch_result;

typedef struct sdpab_batch_config {
  int precision;               /* SDPAB_PREC_FP64 or SDPAB_PREC_MIXED */
  int ctas_per_sm;             /* resident solver blocks per SM (0 = 2 of 256 threads,
                                  4 of 128) */
  double mixed_switch_gap;     /* mixed mode: FP64 once nDim * mu / max(1, mean
                                  |objective|) < this (0 = 1e-2) */
  int staging_doubles;         /* shared-memory staging of GEMM tiles and Lanczos
                                  matrices per solver block, in doubles (0 = auto;
                                  raised to the GEMM minimum of 6400) */
  int mixed_products;          /* mixed mode: the n^3 products of the FP32 phase in
                                  FP32 (1) or on the FP64 MMA (0) */
  int block_threads;           /* threads per solver block (one instance in flight
                                  each): 256 (0 = default) or 128; with 128, four
                                  blocks share an SM by default */
  double refine_tol;           /* mixed mode: the FP64 refinement of a solve with the
                                  FP32 Schur factor stops once the correction is below
                                  this times |dy| (0 = 1e-8; three steps at most) */
  int factor_smem;             /* 1: the Schur factorisation runs in shared memory
                                  when the staging area holds it (m (m + 1) + 32
                                  elements), 0: blocked from L2 */
} sdpab_batch_config;

/* Tensor-core lower update C -= P P^T of an M x M FP32 matrix, P M x K
 * (column-major, device pointers), with split-TF32 MMAs (tcgen05) and FP32
 * accumulation: the trailing update of the mixed-precision Schur factor,
 * exposed stand-alone (no counterpart in the reference; the reference's is
 * dsyrk inside rATL_dpotrfL, sdpa_dpotrf.cpp:218-265).  Synchronises
 * `stream`.  Every wait of the MMA pipeline is bounded: wait_polls < 0 keeps
 * the default bound, wait_polls >= 0 gives up after that many polls (for
 * tests of the fall-back: the call then returns SDPAB_ECUDA and leaves the
 * tiles whose block gave up unchanged). */
SDPAB_API long long sdpab_tc_syrk_work_bytes(int M, int K);  /* device scratch of the call below */
SDPAB_API int sdpab_tc_syrk(int M, int K, const float* P, int ldp, float* C, int ldc, void* work,
                            long long wait_polls, void* stream);

/* Tensor-core product C_q = A_q B^T for q < batch, FP64 in and out
 * (column-major device pointers; A_q M x K at A + q sA, B N x K shared, C_q
 * M x N at C + q sC), in split TF32 with FP32 accumulation: the F1 products
 * (X A_j) Z^-1 of the mixed-precision Schur assembly (Z^-1 symmetric, so
 * B = Z^-1), exposed stand-alone (no counterpart in the reference, whose F1
 * products are dgemm calls, sdpa_newton.cpp:885-889).  Synchronises
 * `stream`.  wait_polls as for sdpab_tc_syrk. */
SDPAB_API long long sdpab_tc_gemm_work_bytes(int M, int N, int K, int batch);
SDPAB_API int sdpab_tc_gemm(int M, int N, int K, int batch, const double* A, int lda, long long sA, const double* B,
                            int ldb, double* C, int ldc, long long sC, void* work, long long wait_polls,
                            void* stream);

/* Solves a batch whose arrays (problem, init, result) are all DEVICE pointers,
 * asynchronously on `stream` (a cudaStream_t, NULL = default stream).
 * `order` (device, optional) gives the processing order of the instances;
 * largest-first balances the persistent schedule.  init may be NULL. */
SDPAB_API int sdpab_batch_solve(const sdpab_batch* prob, const sdpab_batch_init* init,
                      const sdpab_params* prm, const sdpab_batch_config* cfg,
                      sdpab_batch_result* res, const int* order, void* stream);

/* Same batch with HOST pointers: copies the inputs to the device, solves,
 * copies the results back and synchronises.  The largest-first order is
 * computed here. */
SDPAB_API int sdpab_batch_solve_host(const sdpab_batch* prob, const sdpab_batch_init* init,
                           const sdpab_params* prm, const sdpab_batch_config* cfg,
                           sdpab_batch_result* res);

/* Batched solve that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc while running, e.g. a
 * process whose own memory pool already holds the device's memory, or a
 * service that must not allocate after start-up because cudaMalloc
 * synchronises the device and may fail under memory pressure.  Arguments are
 * those of sdpab_batch_solve (all DEVICE pointers; the caller owns inputs and
 * outputs), except that it takes no sdpab_batch_config: it always solves in
 * FP64 with the default launch shape.  The solver's scratch is a fixed region of
 * SDPAB_NOALLOC_SCRATCH_BYTES inside this library, held on every GPU that
 * loads it until the process exits; one solver block needs
 * 8 * (14 * nmax^2 + mmax^2) bytes of it (nmax = mmax = 120 fits 19 blocks,
 * the largest accepted size is about nmax = mmax = 528), larger batches run
 * with fewer concurrent blocks, and sizes whose single block does not fit are
 * rejected with SDPAB_ESIZE.  Every call looks up the region's device
 * address on the current device (the first call on a device also loads the
 * module there; make that first call before any stream capture).  Calls
 * share the region (it keeps the last call's contents; the queue
 * counter is cleared each call): calls that overlap on the GPU race. */
#define SDPAB_NOALLOC_SCRATCH_BYTES (32ull * 1024ull * 1024ull)
SDPAB_API int sdpab_batch_solve_noalloc(const sdpab_batch* prob, const sdpab_batch_init* init,
                                        const sdpab_params* prm, sdpab_batch_result* res,
                                        const int* order, void* stream);

/* Low-rank factor for SDPAB_INIT_FACTOR (no counterpart in the reference).
 * For every instance whose constraints are X_ii = b_i (one SDP block, m = n,
 * F_i = e_i e_i^T, b > 0: MaxCut-type relaxations), an approximate solution
 * of the user's dual problem  max <F0, Y>  s.t.  Y_ii = b_i, Y >= 0  in the
 * factored form Y = V V^T (Burer-Monteiro), by block-coordinate ascent over
 * the rows of V (the mixing method of Wang, Chang and Kolter, 2017):
 *   v_i <- sqrt(b_i) g_i / |g_i|,  g_i = sum_{j != i} F0_ij v_j,
 * rows in order, from a seeded pseudo-random V.  Instance q uses
 * r_q = min(rank, ceil(sqrt(2 n_q)) + 1) columns (its other columns are
 * written as 0) and stops when a sweep changes sum_i <v_i, g_i> by at most
 * tol relative, or after max_sweeps sweeps, or, when sweep_work > 0, after
 * sweep_work / (n + L) sweeps (L: the instance's off-diagonal entries of F0,
 * counted in both triangles), which bounds the longest instances' share of
 * the launch.
 *   prob: DEVICE batch; num_entries: length of its row / col / val arrays;
 *   rank: columns of V, 1..32 (0 = ceil(sqrt(2 nmax)) + 1, at most 32);
 *   V: DEVICE, [nvec * rank] doubles (instance q at V + vec_off[q] * rank);
 *   sweeps: DEVICE, [count] ints out: sweeps run, -1 for an instance not of
 *   this form (its V is not written);
 *   order: DEVICE, [count] instance indices in the order warps take them
 *   (largest first balances the launch), or NULL for 0..count-1.
 * Calls on different streams may run concurrently on disjoint instances
 * (each call has its own work-queue counter; the row scratch is per entry).
 * One warp per instance, taken from a work queue; F0's off-diagonal entries are laid out by rows in a
 * library-owned scratch (2 * num_entries entries, kept between calls, freed
 * by sdpab_release_workspace).  SDPAB_ESIZE when one instance's factor does
 * not fit in shared memory (nmax * rank above about 24,000). */
SDPAB_API int sdpab_lowrank_factor(const sdpab_batch* prob, long long num_entries, int rank, int max_sweeps,
                                   double tol, long long sweep_work, unsigned long long seed, double* V,
                                   int* sweeps, const int* order, void* stream);
/* The rank sdpab_lowrank_factor uses for rank = 0. */
SDPAB_API int sdpab_lowrank_default_rank(int nmax);

/* Device memory the batched solver keeps between calls (workspace, staging). */
SDPAB_API long long sdpab_workspace_bytes(void);
/* Frees that memory on the current device. */
SDPAB_API int sdpab_release_workspace(void);

#ifdef __cplusplus
}
#endif

#endif /* SDPA_B200_H */
