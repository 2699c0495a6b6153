/* oos_gpu.h: the C ABI of the B200 implementation of O_o_Solver's numeric hot path: the supernodal multifrontal
 * LDL^T factorisation (positive definite and indefinite), its solves, and the shift-invert block Lanczos built on
 * them.
 *
 * The entry points replace, one for one, the reference's C++ boundary of that path (paths within jcdulas/O_o_Solver):
 *
 *   oosgpu_symbolic_create        the SymbolicFactor a factorisation is given
 *                                 (include/oos/linalg/symbolic/SymbolicFactor.hpp:37-126: firstColumn, columnCount,
 *                                 rows, supernodes().parent)
 *   oosgpu_symbolic_from_partition the row-structure step of SymbolicFactor::analyse
 *                                 (src/linalg/symbolic/SymbolicFactor.cpp:227-290)
 *   oosgpu_factorise              SupernodalFactor::factorise, both pivoting modes
 *                                 (include/oos/linalg/supernodal/SupernodalFactor.hpp:181-183)
 *   oosgpu_factor_panel           SupernodalFactor::panel (SupernodalFactor.hpp:203)
 *   oosgpu_solve                  FactorSolve::solve (include/oos/linalg/supernodal/FactorSolve.hpp:81)
 *   oosgpu_solve_refined          IterativeRefinement (src/linalg/dense/IterativeRefinement.cpp) over the factor
 *   oosgpu_pencil_*               SparsePencil (include/oos/linalg/eigen/SparsePencil.hpp): factorise at a shift
 *                                 (Sturm count), solve, mass product
 *   oosgpu_modes_*                BlockLanczos::solve (src/linalg/eigen/BlockLanczos.cpp:87-244) and its
 *                                 EigenSolution
 *   oosgpu_symmetric_eigen, oosgpu_sturm_verify, oosgpu_shift_next
 *                                 the Lanczos host logic: SmallEigenSolver, SturmCheck, ShiftStrategy
 *
 *
 * Conventions: plain pointers and sizes; `_device` variants take device pointers (the caller's stream order is the
 * handle's stream, oosgpu_factor_stream), the others host pointers (copies included). Every call returns a status
 * (OOSGPU_OK or an error code mapping one of the reference's exceptions) and leaves a message for
 * oosgpu_last_error() on failure. The library owns its device memory; the caller owns every buffer it passes. One
 * handle is used by one thread at a time (no internal locking), as the reference's factor is built by one thread.
 */
#ifndef OOS_GPU_H
#define OOS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: each maps an exception of the reference's boundary. */
enum
{
    OOSGPU_OK = 0,
    OOSGPU_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    OOSGPU_MEMORY_BUDGET = 2,    /* base::MemoryBudgetError (device memory) */
    OOSGPU_SINGULAR = 3,         /* base::SingularityError (zero pivot; ratio test with bail-out >= 0) */
    OOSGPU_CANCELLED = 4,        /* base::OperationCancelledError */
    OOSGPU_CUDA_ERROR = 5,       /* a CUDA runtime error (no counterpart: the reference runs on the CPU) */
    OOSGPU_INTERNAL = 6,         /* base::InternalError */
    OOSGPU_NOT_FACTORISED = 7,   /* std::logic_error: solve before factorise */
    OOSGPU_SOLVER = 8            /* base::SolverError */
};

/* The message of the last failed call on this thread. */
const char* oosgpu_last_error(void);
/* 1 when a CUDA device is usable, 0 otherwise (the library never falls back to the CPU). */
int oosgpu_device_count(void);
/* The eigenvalue solves keep the device buffers of their workspaces and eigenvectors in a process-wide cache once
 * freed (at most 4 GiB), so that later solves allocate nothing. This frees the idle ones of `device` (-1: of every
 * device) and returns the bytes freed: to give the memory back, and before a cudaDeviceReset, after which cached
 * buffers would belong to a destroyed context (destroy every handle first). */
int64_t oosgpu_release_cached_buffers(int device);

/* ---- symbolic structure ---------------------------------------------------------------------------------------- */
typedef struct oosgpu_symbolic oosgpu_symbolic;

/* From the arrays of a reference SymbolicFactor: supernode s owns columns [first_column[s], first_column[s + 1]),
 * its rows below them are rows[row_start[s] .. row_start[s + 1]) ascending, parent[s] = -1 for a root; children
 * before parents. Checked (OOSGPU_INVALID_ARGUMENT). */
int oosgpu_symbolic_create(int32_t dof_count, int32_t supernode_count, const int32_t* first_column,
                           const int32_t* parent, const int64_t* row_start, const int32_t* rows,
                           oosgpu_symbolic** out);
/* From a node graph (sorted symmetric adjacency), node weights (DOFs per node), the final node order and a supernode
 * partition of the positions (first_position: count + 1, parent: count): the row structures R(s) computed as
 * SymbolicFactor::analyse does. */
int oosgpu_symbolic_from_partition(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                                   const int32_t* weights, const int32_t* node_at_position, int32_t supernode_count,
                                   const int32_t* first_position, const int32_t* parent, oosgpu_symbolic** out);
/* sizes[0..7]: dofs, supernodes, row entries, panel values, factor entries, levels, update values, 0;
 * flops: SymbolicFactor::flopCount. */
int oosgpu_symbolic_sizes(const oosgpu_symbolic* symbolic, int64_t sizes[8], double* flops);
/* The solves' chain launches of the symbolic structure's plan, built on the host (no device needed): [0] launches,
 * [1] tasks, [2] ready flags, [3] tasks of the largest launch. Building the plan checks that every chain task is listed
 * after the blocks it waits on (an internal error otherwise). No counterpart in the reference's API. */
int oosgpu_symbolic_solve_chains(const oosgpu_symbolic* symbolic, int64_t counts[4]);
int oosgpu_symbolic_rows(const oosgpu_symbolic* symbolic, int64_t* row_start, int32_t* rows);
void oosgpu_symbolic_destroy(oosgpu_symbolic* symbolic);

/* ---- factorisation --------------------------------------------------------------------------------------------- */
typedef struct oosgpu_factor oosgpu_factor;

/* FactorOptions (SupernodalFactor.hpp:63-97). */
typedef struct
{
    double max_ratio;                /* PivotPolicy::maxRatio (PARAM MaxDiagonalRatio), default 1e7 */
    int32_t bailout;                 /* PivotPolicy::bailout (SingularityBailOut): < 0 continues past flagged pivots */
    const double* reference_diagonal; /* FactorOptions::referenceDiagonal (host, dimension values) or NULL */
    /* FactorOptions::pivoting: 0 PivotingMode::PositiveDefinite, 1 PivotingMode::Indefinite (Bunch-Kaufman 1x1/2x2
     * pivots among each front's candidates, a candidate that cannot be pivoted delayed to the parent front, which
     * grows by it (info->delayed counts them); zero pivots counted in the inertia, not refused; the ratio test is not
     * applied) */
    int32_t pivoting;
    /* FP64 (0), or mixed (1, positive definite mode only): the update matrices of the large fronts by 3xTF32 products
     * on the tcgen05 tensor cores with FP32 accumulation (about FP32 accuracy; refine the solves in FP64). No
     * counterpart in the reference. */
    int32_t precision;
} oosgpu_factor_options;

/* What a factorisation found (SupernodalFactor accessors and PivotDiagnostics). */
typedef struct
{
    int64_t positive;
    int64_t negative;
    int64_t zero;
    int64_t delayed;                /* SupernodalFactor::delayedPivotCount: candidates delayed to a parent front */
    int64_t two_by_two;
    int64_t issue_count;            /* pivots flagged by the ratio test */
    int32_t equation_of_largest;    /* PivotDiagnostics::equationOfLargestRatio */
    int32_t zero_pivot_count;       /* supernodes stopped by a zero pivot (SingularityError) */
    double largest_ratio;
    int32_t issues[16];             /* the first flagged equations, increasing */
    int32_t zero_pivots[16];        /* the first zero-pivot equations, increasing */
    double device_seconds;          /* the factorisation's device time (CUDA events) */
} oosgpu_factor_info;

/* A factor of `symbolic` on CUDA device `device` (the symbolic structure is copied: it may be destroyed after). */
int oosgpu_factor_create(const oosgpu_symbolic* symbolic, int device, oosgpu_factor** out);
void oosgpu_factor_destroy(oosgpu_factor* factor);
/* The CUDA stream (cudaStream_t) the handle runs on. */
void* oosgpu_factor_stream(oosgpu_factor* factor);

/* Factorises the lower-triangle CSC (col_offsets: dimension + 1, rows ascending from the diagonal, values) given in
 * the symbolic factor's equation order. Host arrays. OOSGPU_SINGULAR: a zero pivot, or the ratio test flagged pivots
 * with bailout >= 0 (the info is filled either way). */
int oosgpu_factorise(oosgpu_factor* factor, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                     const double* values, const oosgpu_factor_options* options, oosgpu_factor_info* info);
/* The same on device arrays (stream-ordered on the handle's stream). */
int oosgpu_factorise_device(oosgpu_factor* factor, int32_t dimension, int64_t terms, const int64_t* col_offsets,
                            const int32_t* rows, const double* values, const oosgpu_factor_options* options,
                            oosgpu_factor_info* info);

/* ---- partial factorisation: PartialFactor (include/oos/linalg/supernodal/PartialFactor.hpp:48-112) ------------ */
/* PartialFactor::factorise: the symbolic factor's last supernode is the trailing set (the unit's boundary: the last
 * `trailing` equations, a root with no rows below, alone in its level; the reference's SymbolicFactor with a trailing
 * node count). Every other supernode is factorised in positive definite FP64 mode (options->pivoting 0, precision 0,
 * the ratio test as oosgpu_factorise); the trailing front, assembled from the matrix's boundary entries and its
 * children's update matrices, is K* = K_bb - K_bi K_ii^-1 K_ib, written to schur_complement (host, trailing x
 * trailing, column-major, both triangles). info covers the interior pivots. A partial factor refuses
 * oosgpu_solve (FactorSolve::solve refuses a partial factor too). */
int oosgpu_factorise_partial(oosgpu_factor* factor, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                             const double* values, int32_t trailing, const oosgpu_factor_options* options,
                             double* schur_complement, oosgpu_factor_info* info);
/* PartialFactor::condenseLoads: f* = f_b - K_bi K_ii^-1 f_i of the loads (host, dimension x columns, leading
 * dimension ld) into condensed (host, trailing x columns, leading dimension ld_condensed): the forward sweep over the
 * interior, the trailing rows gathered from the children of the trailing supernode. */
int oosgpu_partial_condense(oosgpu_factor* factor, const double* loads, int64_t ld, int64_t columns, double* condensed,
                            int64_t ld_condensed);
/* PartialFactor::recover: the loads (host, dimension x columns, leading dimension ld) replaced by the solution with
 * the trailing rows given (trailing_values, trailing x columns): u_i = K_ii^-1 (f_i - K_ib u_b), the trailing rows
 * u_b. */
int oosgpu_partial_recover(oosgpu_factor* factor, double* loads_to_solution, int64_t ld, int64_t columns,
                           const double* trailing_values, int64_t ld_trailing);

/* The panel of supernode s (host copies): eliminated columns, rows; values (rows x eliminated, column-major),
 * row equations and the 2x2 subdiagonal (zeros in positive definite mode) when the pointers are not NULL. */
int oosgpu_factor_panel(oosgpu_factor* factor, int32_t s, int64_t* eliminated, int64_t* row_count, double* values,
                        int32_t* rows, double* subdiagonal);

/* No counterpart in the reference: host right-hand sides (dimension x columns, leading dimension ld) copied to the
 * device ahead of their solve, on a copy stream of the handle's own, so that the copy overlaps what the handle does
 * meanwhile. deferred 0: the copy starts now; deferred 1: it starts when the next oosgpu_factorise has queued the
 * upload of its matrix (the two copies share the host link: the matrix first, then the loads while the matrix is
 * factorised). The next oosgpu_solve or oosgpu_solve_refined on host arrays with the same b, ld and columns uses the
 * copy; any other solve drops it. b must stay unchanged (and allocated) until that solve. */
int oosgpu_solve_prefetch(oosgpu_factor* factor, const double* b, int64_t ld, int64_t columns, int32_t deferred);
/* B <- A^-1 B, B column-major dimension x columns (leading dimension ld), host memory. */
int oosgpu_solve(oosgpu_factor* factor, double* b, int64_t ld, int64_t columns);
/* The same on device memory (stream-ordered on the handle's stream). */
int oosgpu_solve_device(oosgpu_factor* factor, double* b, int64_t ld, int64_t columns);
/* The device time of the last solve (CUDA events), seconds. */
double oosgpu_last_solve_seconds(oosgpu_factor* factor);

/* oosgpu_solve_device without allocating: no counterpart in the reference (its solves run in host memory). For
 * callers that cannot call cudaMalloc once running (a fixed device-memory budget handed over at set-up, allocations
 * forbidden afterwards). Its scratch is a fixed 16 MiB device array in the library (2^21 doubles, held on every GPU
 * that loads the library until exit); a factor needing more than that for one right-hand side (equations plus update
 * rows) is refused with OOSGPU_INVALID_ARGUMENT. The first call on a device looks the array's address up; under
 * CUDA's lazy module loading that first call is also when the array and the solve's kernels are loaded onto the
 * device, which takes device memory. So make the first call during set-up, before any stream capture: a call with
 * columns = 0 is enough. Later calls take no device memory. All calls share the array: calls that overlap on the GPU
 * race. The looked-up address, like every handle of this library, does not survive a cudaDeviceReset. */
int oosgpu_solve_device_noalloc(oosgpu_factor* factor, double* b, int64_t ld, int64_t columns);

/* FP64 iterative refinement around the solve (the fixed-precision refinement of LAPACK xPORFS that the reference
 * applies to free bodies, include/oos/linalg/dense/IterativeRefinement.hpp:39-64): X = A^-1 B, then while a column's
 * normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) exceeds `tolerance`,
 * x += A^-1 (b - A x), at most max_steps times. (The relative residual ||b - A x||_2 / ||b||_2 is reported, not
 * tested: on an ill-conditioned stiffness its FP64 floor, about eps ||A|| ||x|| / ||b||, can lie above any useful
 * tolerance whatever the solve.) The residuals use the last factorised matrix (a host matrix's device copy, or the
 * caller's device arrays, which must then outlive the factorisation's use). */
typedef struct
{
    double tolerance;  /* on the normwise backward error; default 1e-10 */
    int32_t max_steps; /* default 10 */
    /* 0: each correction is one solve (classical refinement); k in [1, 12]: each correction solves
     * A^-1-preconditioned A d = r by GMRES with at most k Krylov vectors (GMRES-IR, for a factor less accurate than
     * the matrix's conditioning needs, e.g. the mixed-precision form). No counterpart in the reference. */
    int32_t krylov;
} oosgpu_refine_options;
typedef struct
{
    int32_t steps;         /* corrections made (the most over the column tiles) */
    double residual;       /* the largest final relative residual ||b - A x||_2 / ||b||_2 over the columns */
    double device_seconds; /* device time of the solve and its refinement */
    double backward_error; /* the largest final normwise backward error over the columns */
} oosgpu_refine_info;
/* B (ldb) and X (ldx) column-major, host memory; B is not modified. */
int oosgpu_solve_refined(oosgpu_factor* factor, const double* b, int64_t ldb, double* x, int64_t ldx, int64_t columns,
                         const oosgpu_refine_options* options, oosgpu_refine_info* info);
/* The same on device memory. */
int oosgpu_solve_refined_device(oosgpu_factor* factor, const double* b, int64_t ldb, double* x, int64_t ldx,
                                int64_t columns, const oosgpu_refine_options* options, oosgpu_refine_info* info);

/* ---- measurement (no counterpart in the reference: its RunReport carries stage times only,
 *      include/oos/api/Analyses.hpp:182-199) ---------------------------------------------------------------------- */
/* Brackets every launch of the following factorisations and solve sweeps with CUDA events (enable != 0). */
int oosgpu_factor_profile(oosgpu_factor* factor, int32_t enable);
/* The launches of the last profiled factorisation (which 0) or of the sweeps of the last profiled solve's last column
 * tile (which 1), in launch order: kind (the plan's launch kinds: 0 small fronts, 1 assembly, 2 diagonal blocks,
 * 3 panel rows, 4 panel update, 5 update matrix, 6 forward small, 7 forward gather, 8 forward diagonal, 9 forward
 * update, 10 backward small, 11 backward rows, 12 backward diagonal, 13 backward update, 14-19 the indefinite
 * kinds, 20 diagonal inverses, 21 the mixed update matrix, 22 the sums of split backward products, 23 the
 * diagonal sweep), blocks, first column of the step, device seconds. At most
 * `capacity` are written; *total is how many there are. */
int oosgpu_factor_launch_profile(oosgpu_factor* factor, int32_t which, int64_t capacity, int32_t* kinds,
                                 int32_t* counts, int32_t* k0, double* seconds, int64_t* total);
/* After a profiled factorisation, per launch kind k < kinds (0 small fronts, 1 assembly, 2 diagonal blocks, 3 panel
 * rows, 4 panel update, 5 update-matrix Schur product): device seconds, launches, algorithmic flops and bytes. */
int oosgpu_factor_kernel_stats(oosgpu_factor* factor, int32_t kinds, double* seconds, int64_t* launches,
                               double* flops, double* bytes);
/* counts[0]: kernels one factorisation launches; counts[1]: kernels one solve of `columns` right-hand sides
 * launches. */
int oosgpu_factor_launch_counts(oosgpu_factor* factor, int64_t columns, int64_t counts[2]);

/* ---- kernel choice (no counterpart in the reference: its kernel family is chosen per process, by the CPU's
 *      instruction set, include/oos/linalg/dense/KernelSelection.hpp) ------------------------------------------- */
/* The kernel choice of the launch kinds that have two kernels (the diagonal blocks by 16-column sub-panels or column
 * by column; the extend-add element-wise or staged in shared memory; the update matrix by 64 x 64 tiles or by
 * TMA-fed 128 x 128 tiles). mode 1 (the default): the autotuner, which on the next positive definite FP64
 * factorisation of the handle runs the factorisation twice with each kernel, every launch timed (its shorter time
 * kept), and lets each size
 * class of launch (1, <= 8, <= 148, <= 592, more blocks) keep the faster one. mode 0: the first kernel of each pair;
 * mode 2: the second everywhere. Any call forgets an earlier choice. */
int oosgpu_factor_set_tuning(oosgpu_factor* factor, int32_t mode);
/* The autotuner's choices: per (launch kind, size class), the launches, the seconds of kernel 0 and kernel 1 in the
 * timing factorisations, and the kernel chosen. At most `capacity` records; *total is how many there are (0 before the
 * tuning factorisation). */
int oosgpu_factor_tuning_report(oosgpu_factor* factor, int64_t capacity, int32_t* kinds, int32_t* size_classes,
                                int32_t* launches, double* seconds0, double* seconds1, int32_t* chosen, int64_t* total);

/* ---- shifted pencil: the ShiftedPencil plug-in (include/oos/linalg/eigen/ShiftedPencil.hpp:55-88) as SparsePencil
 *      implements it (include/oos/linalg/eigen/SparsePencil.hpp:29-85) -------------------------------------------- */
typedef struct oosgpu_pencil oosgpu_pencil;

/* K and M: lower CSC of one structure (the symbolic factor's equation order), host arrays, copied. Refused: another
 * dimension (OOSGPU_INVALID_ARGUMENT), a negative or infinite mass diagonal term (OOSGPU_SOLVER). */
int oosgpu_pencil_create(const oosgpu_symbolic* symbolic, int device, int32_t dimension, const int64_t* col_offsets,
                         const int32_t* rows, const double* stiffness, const double* mass, oosgpu_pencil** out);
/* BucklingPencil (include/oos/linalg/eigen/BucklingPencil.hpp:29-72): the pencil K phi = lambda B phi of the stiffness
 * K and the differential stiffness K_d of a preload (B = -K_d), both lower CSC on one pattern in the symbolic factor's
 * order. Its shifted matrices K + sigma K_d are factorised in indefinite mode with the powers-of-two scaling of K; the
 * operator's inner product is K's. oosgpu_modes_solve on it runs BlockLanczos::solveBuckling (BlockLanczos.cpp:90-91):
 * the load factors nearest 0 of either sign in [lower_bound, upper_bound), by increasing magnitude (the positive first
 * on a tie); K must be positive definite (OOSGPU_SOLVER otherwise). */
int oosgpu_pencil_create_buckling(const oosgpu_symbolic* symbolic, int device, int32_t dimension,
                                  const int64_t* col_offsets, const int32_t* rows, const double* stiffness,
                                  const double* differential, oosgpu_pencil** out);
void oosgpu_pencil_destroy(oosgpu_pencil* pencil);
void* oosgpu_pencil_stream(oosgpu_pencil* pencil);
/* ShiftedPencil::factorise: S (K - shift M) S factorised in indefinite mode; info->negative is the Sturm count of the
 * shift, info->zero > 0 a singular shift (returned, not refused). */
int oosgpu_pencil_factorise(oosgpu_pencil* pencil, double shift, oosgpu_factor_info* info);
/* ShiftedPencil::solve: X <- (K - shift M)^-1 X with the last factor, X column-major on the device. */
int oosgpu_pencil_solve_device(oosgpu_pencil* pencil, double* x, int64_t ld, int64_t columns);
/* ShiftedPencil::multiplyMass: Y <- M X, device blocks (a lumped mass by its diagonal). */
int oosgpu_pencil_multiply_mass_device(oosgpu_pencil* pencil, const double* x, int64_t ldx, double* y, int64_t ldy,
                                       int64_t columns);
/* ShiftedPencil::diagonalRayleighBound (min K_ii / M_ii over K_ii, M_ii > 0), SparsePencil::hasDiagonalMass and
 * factorisationCount. */
int oosgpu_pencil_properties(const oosgpu_pencil* pencil, double* rayleigh_bound, int32_t* lumped,
                             int64_t* factorisations);

/* ---- eigenvalue analysis: BlockLanczos::solve (include/oos/linalg/eigen/BlockLanczos.hpp:102-161,
 *      src/linalg/eigen/BlockLanczos.cpp:84-246) over the GPU pencil ------------------------------------------------ */

/* EigenRequest (include/oos/linalg/eigen/EigenRequest.hpp:21-35): every root of [lower, upper] (mode_count 0), or the
 * lowest mode_count roots above lower_bound (and below upper_bound when finite); lower_bound <= 0: from the lowest
 * root. Infinite bounds are +-INFINITY. */
typedef struct oosgpu_eigen_request
{
    double lower_bound;
    double upper_bound;
    int64_t mode_count;
} oosgpu_eigen_request;

/* LanczosOptions (BlockLanczos.hpp:21-64): the block size, the modes one shift converges, the tolerance of
 * ||Op y - theta y||_M <= tol |theta|, the shifts and the thick restarts allowed, the seed of the random starts. */
typedef struct oosgpu_lanczos_options
{
    int64_t block_size;
    int64_t modes_per_shift;
    double convergence_tolerance;
    int64_t maximum_shifts;
    int64_t maximum_restarts;
    uint64_t seed;
} oosgpu_lanczos_options;

/* The reference's defaults (block 7, 40 modes per shift, 1e-10, 40 shifts, 20 restarts, its seed). */
void oosgpu_lanczos_defaults(oosgpu_lanczos_options* options);

typedef struct oosgpu_modes oosgpu_modes;

/* The eigenpairs of `request` (options null: the defaults). Errors as the reference's: OOSGPU_INVALID_ARGUMENT for a
 * request or settings out of range, OOSGPU_SOLVER for a pencil singular at every shift tried, contradicting Sturm
 * counts or unbounded negative roots, OOSGPU_MEMORY_BUDGET when the basis does not fit in device memory. */
int oosgpu_modes_solve(oosgpu_pencil* pencil, const oosgpu_eigen_request* request,
                       const oosgpu_lanczos_options* options, oosgpu_modes** out);
/* The same with the first Lanczos run started from `start` (device memory, dimension x columns, leading dimension ld,
 * columns = the block size) instead of a random block: a learned start block (the predicted modes of a design); the
 * later runs, at other shifts, start from random blocks. start NULL: oosgpu_modes_solve. No counterpart in the
 * reference (LanczosRun::startBlock, LanczosRun.cpp:217-229, draws the block). */
int oosgpu_modes_solve_start(oosgpu_pencil* pencil, const oosgpu_eigen_request* request,
                             const oosgpu_lanczos_options* options, const double* start, int64_t ld, int64_t columns,
                             oosgpu_modes** out);
/* counts: [0] eigenpairs, [1] factorisations, [2] shifts, [3] verified by the Sturm counts, [4] complete (0/1),
 * [5] Lanczos block steps; seconds: [0] wall seconds of the solve, [1] device seconds of its factorisations, then
 * wall seconds of [2] the factorisations, [3] the operator (solves and mass products), [4] the M-orthogonalisation
 * and the basis products, [5] the projected problem. */
int oosgpu_modes_summary(const oosgpu_modes* modes, int64_t counts[6], double seconds[6]);
/* Where a solve's time went. counts: [0] blocks that met a dependent column and were orthonormalised column by column
 * (the reference's MassOrthogonalizer fallback), [1] one-column operator applications that replaced dependent columns;
 * seconds (wall): the parts of seconds[4] of the summary, [0] start blocks, [1] block steps, [2] thick restarts,
 * [3] harvests of converged pairs; then outside the summary's phases, [4] the workspace's set-up, [5] the answer's
 * gathering, [6] the workspace's release. Either may be null. No counterpart in the reference's API. */
int oosgpu_modes_work(const oosgpu_modes* modes, int64_t counts[2], double seconds[7]);
/* The eigenvalues (increasing) and their residual bounds ||Op y - theta y||_M / |theta|. */
int oosgpu_modes_values(const oosgpu_modes* modes, double* eigenvalues, double* residual_bounds);
/* The M-orthonormal eigenvectors, dimension x count, into host memory of leading dimension ld. */
int oosgpu_modes_vectors(const oosgpu_modes* modes, double* vectors, int64_t ld);
/* The eigenvectors in device memory (dimension x count, leading dimension dimension), owned by `modes`. */
const double* oosgpu_modes_vectors_device(const oosgpu_modes* modes);
/* 7 values per shift (ShiftRecord, BlockLanczos.hpp:68-78): shift, purpose (0 lowest bound, 1 lower bound, 2 upper
 * bound, 3 advance, 4 fill gap), Sturm count, Lanczos run (0/1), block steps, restarts, converged pairs. */
int oosgpu_modes_shifts(const oosgpu_modes* modes, double* records);
void oosgpu_modes_destroy(oosgpu_modes* modes);

/* ---- the host logic of the shift-invert Lanczos, exposed for its callers and its tests (no device needed) ---- */

/* SmallEigenSolver over a symmetric p x p matrix (src/linalg/dense/SmallEigenSolver.cpp): eigenvalues increasing,
 * eigenvectors as columns (p x p, leading dimension p), each signed so that its first component of largest magnitude
 * is positive. `a` is read in its lower triangle, column-major with leading dimension ld. */
int oosgpu_symmetric_eigen(const double* a, int64_t p, int64_t ld, double* eigenvalues, double* eigenvectors);
/* SturmCheck::addPoint for each (shift, count) then verify (src/linalg/eigen/SturmCheck.cpp) against the sorted
 * eigenvalues found: result = verified up to, verified count, has mismatch (0/1), mismatch lower, mismatch upper,
 * expected count * 1e6 + found count. */
int oosgpu_sturm_verify(int64_t points, const double* shifts, const int64_t* counts, int64_t values,
                        const double* sorted, double result[6]);
/* ShiftStrategy(request, scale).nextShift (src/linalg/eigen/ShiftStrategy.cpp:121-193): verification in
 * oosgpu_sturm_verify's layout; purpose as in oosgpu_modes_shifts. */
int oosgpu_shift_next(double lower, double upper, int64_t mode_count, double scale, const double verification[6],
                      int64_t values, const double* sorted, int64_t ritz_count, const double* ritz,
                      int64_t shift_count, const double* lanczos_shifts, double* shift, int32_t* purpose);

/* ---- the learned start block's network (no counterpart in the reference) -----------------------------------------
 * A multilayer perceptron inputs -> hidden -> hidden -> outputs, ReLU after each hidden layer, FP32 on the GPU: He
 * initialised from `seed`, trained by full-batch Adam on the mean squared error, every step by this library's kernels.
 * Parameters (flat, oosgpu_mlp_parameter_count floats): W1 (inputs x hidden, row-major), b1, W2 (hidden x hidden), b2,
 * W3 (hidden x outputs), b3. Samples are rows (batch x inputs, batch x outputs, row-major, host). */
typedef struct oosgpu_mlp oosgpu_mlp;
int oosgpu_mlp_create(int32_t inputs, int32_t hidden, int32_t outputs, uint64_t seed, int device, oosgpu_mlp** out);
void oosgpu_mlp_destroy(oosgpu_mlp* mlp);
int64_t oosgpu_mlp_parameter_count(const oosgpu_mlp* mlp);
int oosgpu_mlp_get_parameters(oosgpu_mlp* mlp, float* parameters);
int oosgpu_mlp_set_parameters(oosgpu_mlp* mlp, const float* parameters);
int oosgpu_mlp_predict(oosgpu_mlp* mlp, const float* inputs, int32_t batch, float* outputs);
/* The gradients of the mean squared error (mean over the batch and the outputs) at the current parameters, and the
 * loss; either output may be NULL. */
int oosgpu_mlp_gradients(oosgpu_mlp* mlp, const float* inputs, const float* targets, int32_t batch, float* gradients,
                         float* loss);
/* `epochs` full-batch Adam steps (beta 0.9 / 0.999, epsilon 1e-8) at `rate`; losses (epochs values, or NULL): the loss
 * before each step. */
int oosgpu_mlp_train(oosgpu_mlp* mlp, const float* inputs, const float* targets, int32_t batch, int32_t epochs,
                     float rate, float* losses);

/* ---- model-side helpers (no counterpart in the reference's linalg: they stand in for its assembly and DOF
 *      selection, src/assembly and SymmetricCsc::fromBlocks, src/linalg/sparse/SymmetricCsc.cpp:41) ---------------- */
typedef struct oosgpu_model oosgpu_model;

/* A plate of nx x ny flat-shell quadrilaterals on lx x ly, thickness t, clamped along x = 0, 6 DOFs per node. */
int oosgpu_model_plate(int32_t nx, int32_t ny, double lx, double ly, double thickness, double young, double poisson,
                       double pressure, oosgpu_model** out);
/* A cube of n^3 trilinear hexahedra, clamped on z = 0, lumped mass, 3 DOFs per node. */
int oosgpu_model_hex(int32_t n, double edge, double young, double poisson, double density, oosgpu_model** out);
/* A square skin of n x n flat shells on lx x ly (thickness t), clamped along x = 0, stiffened by `stringers` blades along x
 * (height x thickness section, frame elements on the skin's grid lines y = k ly / (stringers + 1)); 6 DOFs per node. */
int oosgpu_model_stiffened_panel(int32_t n, double lx, double ly, double thickness, double young, double poisson,
                                 int32_t stringers, double blade_height, double blade_thickness, double pressure,
                                 oosgpu_model** out);
/* A rectangular wing box of flat shells of size h (span along y, chord along x, height along z, ribs every rib_pitch),
 * clamped at the root y = 0, lumped mass; thicknesses: 24 zones (upper skin 8 spanwise, lower skin 8, front spar 4,
 * rear spar 4); 6 DOFs per node. */
int oosgpu_model_wing_box(double span, double chord, double height, double rib_pitch, double h,
                          const double* thicknesses, double rib_thickness, double young, double poisson, double density,
                          oosgpu_model** out);
void oosgpu_model_destroy(oosgpu_model* model);
/* sizes[0..3]: free nodes, DOFs per node, adjacency entries, 0 */
int oosgpu_model_sizes(const oosgpu_model* model, int64_t sizes[4]);
/* The node graph (offsets: nodes + 1, neighbours) and coordinates (3 per node); NULL pointers are skipped. */
int oosgpu_model_graph(const oosgpu_model* model, int64_t* offsets, int32_t* neighbours, double* coordinates);
int oosgpu_model_csc_terms(const oosgpu_model* model, const int32_t* node_at_position, int64_t* terms);
/* which: 0 stiffness, 1 lumped mass on the stiffness pattern. */
int oosgpu_model_csc(const oosgpu_model* model, const int32_t* node_at_position, int32_t which, int64_t* col_offsets,
                     int32_t* rows, double* values);
/* The same columns written by the GPU `device` into device arrays (col_offsets: dimension + 1, rows and values:
 * oosgpu_model_csc_terms), from the model's element list: the element matrices, the node blocks and the columns are
 * formed on the device, with the host's arithmetic in the host's order (the same values bit for bit). The role of the
 * reference's StiffnessAssembler and SymmetricCsc::fromBlocks (include/oos/assembly/assemble/StiffnessAssembler.hpp:
 * 21-33, src/linalg/sparse/SymmetricCsc.cpp:41) for this project's workload models. which 1 (lumped mass) copies the
 * host's mass. */
int oosgpu_model_csc_device(const oosgpu_model* model, const int32_t* node_at_position, int32_t which, int32_t device,
                            int64_t* col_offsets, int32_t* rows, double* values);
/* Column 0 the pressure load; columns j >= 1: `points` seeded nodes (splitmix64, seed_base + j) with N(0, sigma)
 * forces on their out-of-plane translation. rhs column-major, leading dimension ld. */
int oosgpu_model_loads(const oosgpu_model* model, const int32_t* node_at_position, int64_t columns,
                       uint64_t seed_base, int32_t points, double sigma, double* rhs, int64_t ld);

#ifdef __cplusplus
}
#endif

#endif
