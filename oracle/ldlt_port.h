/* A plain-C restatement of the reference's positive definite multifrontal LDL^T and its solves (jcdulas/O_o_Solver,
 * src/linalg/supernodal/MultifrontalDriver.cpp, FrontAssembly.cpp, src/linalg/kernels/reference/DenseBlockKernels.cpp,
 * src/linalg/supernodal/FactorSolve.cpp), built by oracle/Makefile into oracle/_ref/libldlt_port.so.
 *
 * TEST INFRASTRUCTURE ONLY: a second, readable checker of the GPU path beside the reference library itself; compiled
 * with -ffp-contract=off so that its factor has the bits of the reference family's (every product rounded before
 * its sum, the same chains). The product never links it. */
#ifndef OOS_LDLT_PORT_H
#define OOS_LDLT_PORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The symbolic structure: supernode s owns columns [first_column[s], first_column[s+1]), its rows below them are
 * rows[row_start[s] .. row_start[s+1]) ascending, parent[s] = -1 at a root; children before parents.
 * panels: sum of c(c + r) values, supernode s at the sum before it, column-major, leading dimension c + r.
 * inertia: positive, negative, zero of D. Returns 0, or 1 + the first zero-pivot equation's supernode count when a
 * pivot is zero or not finite (zero_pivot_equation set to the first such equation), or -1 on a structure error. */
int port_factorise(int32_t dimension, int32_t supernode_count, const int32_t* first_column, const int32_t* parent,
                   const int64_t* row_start, const int32_t* rows, const int64_t* col_offsets, const int32_t* col_rows,
                   const double* values, double* panels, int64_t inertia[3], int32_t* zero_pivot_equation);

/* B <- A^-1 B with the factor of port_factorise (B column-major, leading dimension ld). */
int port_solve(int32_t dimension, int32_t supernode_count, const int32_t* first_column, const int32_t* parent,
               const int64_t* row_start, const int32_t* rows, const double* panels, double* b, int64_t ld,
               int64_t columns);

#ifdef __cplusplus
}
#endif

#endif
