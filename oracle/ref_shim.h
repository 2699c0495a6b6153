/* C entry points over the reference's own linear algebra (jcdulas/O_o_Solver, modules base + linalg), built from its
 * sources by oracle/Makefile into oracle/_ref/liboos_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker of the GPU path (tests, smoke, the CPU-baseline leg of the
 * benchmark); the product never links or calls it.
 *
 * Every function returns 0 on success, or -1 with a message in the shim's last-error buffer (ref_last_error) when
 * the reference threw. Arrays are caller-owned. */
#ifndef OOS_REF_SHIM_H
#define OOS_REF_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ref_symbolic ref_symbolic;
typedef struct ref_factor ref_factor;

const char* ref_last_error(void);

/* ConstrainedOrdering::order (src/linalg/ordering/ConstrainedOrdering.cpp:28-66) then SymbolicFactor::analyse
 * (src/linalg/symbolic/SymbolicFactor.cpp:167) on a node graph. method: 0 automatic, 1 minimum degree,
 * 2 nested dissection, 3 natural; 4 = the order given in `given_order` (node at each position). amalgamate: 1 the
 * default AmalgamationThresholds, 0 none (fundamental supernodes). coords: 3 doubles per node, or NULL. */
ref_symbolic* ref_analyse(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                          const int32_t* weights, const double* coords, int method, const int32_t* given_order,
                          int amalgamate, int threads);
/* The same with a trailing set of nodes (the boundary of a unit, ordered last in their given order and forming the
 * last supernode: ConstrainedOrdering's trailing nodes, SymbolicFactor::analyse's trailingNodeCount). */
ref_symbolic* ref_analyse_trailing(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                                   const int32_t* weights, const double* coords, int method,
                                   const int32_t* given_order, int amalgamate, int threads,
                                   const int32_t* trailing_nodes, int32_t trailing_count);
void ref_symbolic_free(ref_symbolic* s);

/* sizes[0..9]: nodes, dofs, supernodes, row entries, panel values, factor entries, largest front values,
 * update-stack peak values, trailing dofs, 0 */
void ref_sym_sizes(const ref_symbolic* s, int64_t sizes[10]);
double ref_sym_flops(const ref_symbolic* s);
/* seconds spent in ordering and in analyse */
void ref_sym_times(const ref_symbolic* s, double times[2]);
void ref_sym_node_order(const ref_symbolic* s, int32_t* node_at_position);
void ref_sym_first_columns(const ref_symbolic* s, int32_t* first_column_of_position /* nodes + 1 */);
void ref_sym_supernodes(const ref_symbolic* s, int32_t* first_position /* count + 1 */, int32_t* parent);
void ref_sym_rows(const ref_symbolic* s, int64_t* row_start /* count + 1 */, int32_t* rows);

/* SupernodalFactor::factorise (src/linalg/supernodal/SupernodalFactor.cpp:12-28) on a lower-triangle CSC in the
 * symbolic factor's order. pivoting: 0 positive definite, 1 indefinite. family: -1 automatic (KernelSelection),
 * 0 reference, 1 avx2, 2 avx512. max_ratio/bailout: PivotPolicy (bailout < 0 continues past flagged pivots).
 * seconds[0] = wall time of factorise. */
ref_factor* ref_factorise(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                          const double* values, int pivoting, int family, int threads, double max_ratio, int bailout,
                          double* seconds);
void ref_factor_free(ref_factor* f);
/* info[0..7]: positive, negative, zero, delayed pivots, 2x2 pivots, pivot issue count, equation of largest ratio,
 * kernel kind */
void ref_factor_info(const ref_factor* f, int64_t info[8], double* largest_ratio);
/* The panel of supernode s: eliminated columns, rows; values column-major (rows x eliminated, leading dimension
 * rows) copied into `values` when not NULL, the row equations into `rows`, the 2x2 subdiagonal into `subdiagonal`
 * (eliminated values; zeros in positive definite mode). */
int ref_factor_panel(const ref_factor* f, int32_t s, int64_t* eliminated, int64_t* row_count, double* values,
                     int32_t* rows, double* subdiagonal);
/* FactorSolve::solve (src/linalg/supernodal/FactorSolve.cpp:176-190): B <- A^-1 B in place, B column-major. */
int ref_solve(const ref_factor* f, double* b, int64_t ld, int64_t columns, int threads, double* seconds);

/* SparsePencil + BlockLanczos::solve (src/linalg/eigen/SparsePencil.cpp, BlockLanczos.cpp:87-244): the eigenpairs of
 * K x = lambda M x that the request (lower, upper, mode_count: EigenRequest) asks for. block_size and
 * modes_per_shift: LanczosOptions (0: the default). eigenvalues: up to `capacity`; eigenvectors: dimension x capacity
 * (may be NULL). shifts: up to max_shifts records of (shift, purpose, sturm count, has run, block steps, restarts,
 * converged); counts[0..4]: modes found, factorisations, shift records, verified count, complete. seconds[0]: wall
 * time of the solve. */
int ref_modes(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
              const double* stiffness, const double* mass, double lower, double upper, int64_t mode_count,
              int64_t block_size, int64_t modes_per_shift, int family, int threads, double* eigenvalues,
              int64_t capacity, double* eigenvectors, double* shifts, int64_t max_shifts, int64_t counts[5],
              double* seconds);

/* The same for the buckling pencil (BucklingPencil, BlockLanczos::solveBuckling): K x = lambda (-K_d) x, the load
 * factors nearest 0 of either sign in [lower, upper); `differential` is K_d on the pattern of K. */
int ref_buckling(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                 const double* stiffness, const double* differential, double lower, double upper, int64_t mode_count,
                 int64_t block_size, int64_t modes_per_shift, int family, int threads, double* eigenvalues,
                 int64_t capacity, double* eigenvectors, double* shifts, int64_t max_shifts, int64_t counts[5],
                 double* seconds);

/* SturmCheck::addPoint + verify (src/linalg/eigen/SturmCheck.cpp): result = verifiedUpTo, verifiedCount,
 * hasMismatch, mismatch.lower, mismatch.upper, expected * 1e6 + found. */
int ref_sturm_verify(int64_t points, const double* shifts, const int64_t* counts, int64_t values, const double* sorted,
                     double result[6]);
/* ShiftStrategy(request, scale).nextShift (src/linalg/eigen/ShiftStrategy.cpp:121-193); verification as
 * ref_sturm_verify's result. */
int ref_shift_next(double lower, double upper, int64_t mode_count, double scale, const double verification[6],
                   int64_t values, const double* sorted, int64_t ritz_count, const double* ritz, int64_t shift_count,
                   const double* lanczos_shifts, double* shift, int32_t* purpose);

/* SmallEigenSolver::decompose (src/linalg/dense/SmallEigenSolver.cpp:261-297) of the lower triangle of a, column-major
 * leading dimension ld: eigenvalues increasing, eigenvectors p x p (leading dimension p). */
int ref_symmetric_eigen(const double* a, int64_t p, int64_t ld, double* eigenvalues, double* eigenvectors);

/* pencilScaleOf (src/linalg/eigen/PencilScaling.cpp:64-80): the power-of-two scales of a stiffness CSC. */
int ref_pencil_scale(int32_t dimension, const int64_t* col_offsets, const int32_t* rows, const double* values,
                     double* scale);

/* PartialFactor (src/linalg/supernodal/PartialFactor.cpp:65): the interior of a unit factorised, K* = K_bb -
 * K_bi K_ii^-1 K_ib written to schur_complement (trailing x trailing, column-major, both triangles). NULL on error. */
typedef struct ref_partial ref_partial;
ref_partial* ref_partial_factorise(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets,
                                   const int32_t* rows, const double* values, int family, double* schur_complement);
void ref_partial_free(ref_partial* p);
/* PartialFactor::condenseLoads: f* = f_b - K_bi K_ii^-1 f_i (trailing x columns) of loads (dimension x columns). */
int ref_partial_condense(const ref_partial* p, const double* loads, int64_t columns, double* condensed);
/* PartialFactor::recover: loads (dimension x columns, in place) -> the solution with the trailing rows given. */
int ref_partial_recover(const ref_partial* p, double* loads, int64_t columns, const double* trailing);

#ifdef __cplusplus
}
#endif

#endif
