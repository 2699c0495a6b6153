/* Plain-C restatement of the reference's positive definite multifrontal LDL^T and its sweeps; see ldlt_port.h.
 * TEST INFRASTRUCTURE ONLY. */

#include "ldlt_port.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* The position of DOF `row` in the front of supernode s: its columns first, then R(s) (binary search); -1 outside. */
static int64_t position_in_front(int32_t first, int32_t c, const int32_t* r, int64_t rc, int32_t row)
{
    if (row < first)
        return -1;
    if (row < first + c)
        return row - first;
    int64_t lo = 0, hi = rc;
    while (lo < hi)
    {
        const int64_t mid = (lo + hi) / 2;
        if (r[mid] < row)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < rc && r[lo] == row ? c + lo : -1;
}

/* MultifrontalDriver::run in postorder (MultifrontalDriver.cpp:651-702): each supernode's front assembled
 * (FrontAssembly.cpp:166-300: cleared, the matrix's entries of its columns, then its children's update matrices in
 * increasing order) and eliminated by the reference family's unblocked right-looking LDL^T
 * (kernels/reference/DenseBlockKernels.cpp:368-446: l_ik = a_ik / d_k, then a_ij -= l_ik * (l_jk * d_k) for k
 * increasing), its panel stored with zeros above the diagonal and its update matrix kept for its parent. */
int port_factorise(int32_t dimension, int32_t supernode_count, const int32_t* first_column, const int32_t* parent,
                   const int64_t* row_start, const int32_t* rows, const int64_t* col_offsets, const int32_t* col_rows,
                   const double* values, double* panels, int64_t inertia[3], int32_t* zero_pivot_equation)
{
    const int32_t S = supernode_count;
    int64_t* panel_offset = (int64_t*)calloc((size_t)S + 1, sizeof(int64_t));
    double** updates = (double**)calloc((size_t)S, sizeof(double*));
    int32_t* status = (int32_t*)calloc((size_t)S, sizeof(int32_t)); /* 0 done, 1 zero pivot, 2 skipped */
    int32_t* child_head = (int32_t*)malloc((size_t)S * sizeof(int32_t));
    int32_t* child_next = (int32_t*)malloc((size_t)S * sizeof(int32_t));
    int result = 0;
    inertia[0] = inertia[1] = inertia[2] = 0;
    *zero_pivot_equation = -1;
    (void)dimension;
    for (int32_t s = 0; s < S; ++s)
    {
        const int64_t c = first_column[s + 1] - first_column[s];
        const int64_t r = row_start[s + 1] - row_start[s];
        panel_offset[s + 1] = panel_offset[s] + c * (c + r);
        child_head[s] = -1;
    }
    for (int32_t s = S - 1; s >= 0; --s)
        if (parent[s] >= 0)
        {
            child_next[s] = child_head[parent[s]];
            child_head[parent[s]] = s;
        }
    for (int32_t s = 0; s < S && result >= 0; ++s)
    {
        const int32_t first = first_column[s];
        const int64_t c = first_column[s + 1] - first;
        const int64_t r = row_start[s + 1] - row_start[s];
        const int64_t n = c + r;
        const int32_t* rs = rows + row_start[s];
        int skipped = 0;
        for (int32_t ch = child_head[s]; ch >= 0; ch = child_next[ch])
            if (status[ch] != 0)
                skipped = 1;
        if (skipped)
        {
            status[s] = 2;
            for (int32_t ch = child_head[s]; ch >= 0; ch = child_next[ch])
            {
                free(updates[ch]);
                updates[ch] = NULL;
            }
            continue;
        }
        /* The front, whole (n x n, lower triangle used), then split into the panel and the update matrix. */
        double* front = (double*)calloc((size_t)(n * n), sizeof(double));
        for (int64_t j = 0; j < c; ++j)
        {
            const int32_t column = first + (int32_t)j;
            for (int64_t k = col_offsets[column]; k < col_offsets[column + 1]; ++k)
            {
                const int32_t row = col_rows[k];
                const int64_t position = row < column ? -1 : position_in_front(first, (int32_t)c, rs, r, row);
                if (position < 0)
                {
                    result = -1;
                    break;
                }
                front[position + j * n] += values[k];
            }
        }
        for (int32_t ch = child_head[s]; ch >= 0; ch = child_next[ch])
        {
            const int64_t rc = row_start[ch + 1] - row_start[ch];
            const int32_t* crows = rows + row_start[ch];
            int64_t* map = (int64_t*)malloc((size_t)(rc > 0 ? rc : 1) * sizeof(int64_t));
            for (int64_t k = 0; k < rc; ++k)
            {
                map[k] = position_in_front(first, (int32_t)c, rs, r, crows[k]);
                if (map[k] < 0)
                    result = -1;
            }
            const double* u = updates[ch];
            for (int64_t jc = 0; jc < rc && result >= 0; ++jc)
                for (int64_t ic = jc; ic < rc; ++ic)
                    front[map[ic] + map[jc] * n] += u[ic + jc * rc];
            free(map);
            free(updates[ch]);
            updates[ch] = NULL;
        }
        int64_t eliminated = c;
        for (int64_t k = 0; k < c; ++k)
        {
            const double pivot = front[k + k * n];
            if (pivot == 0.0 || !isfinite(pivot))
            {
                eliminated = k;
                break;
            }
            for (int64_t i = k + 1; i < n; ++i)
                front[i + k * n] = front[i + k * n] / pivot;
            for (int64_t j = k + 1; j < n; ++j)
            {
                const double w = front[j + k * n] * pivot;
                for (int64_t i = j; i < n; ++i)
                    front[i + j * n] -= front[i + k * n] * w;
            }
        }
        if (eliminated < c)
        {
            status[s] = 1;
            if (*zero_pivot_equation < 0)
                *zero_pivot_equation = first + (int32_t)eliminated;
            result += 1;
        }
        double* panel = panels + panel_offset[s];
        for (int64_t j = 0; j < c; ++j)
            for (int64_t i = 0; i < n; ++i)
                panel[i + j * n] = i >= j ? front[i + j * n] : 0.0;
        if (status[s] == 0)
        {
            for (int64_t k = 0; k < c; ++k)
            {
                const double d = front[k + k * n];
                inertia[d > 0.0 ? 0 : (d < 0.0 ? 1 : 2)] += 1;
            }
            if (r > 0)
            {
                double* u = (double*)malloc((size_t)(r * r) * sizeof(double));
                for (int64_t j = 0; j < r; ++j)
                    for (int64_t i = j; i < r; ++i)
                        u[i + j * r] = front[(c + i) + (c + j) * n];
                updates[s] = u;
            }
        }
        free(front);
    }
    for (int32_t s = 0; s < S; ++s)
        free(updates[s]);
    free(updates);
    free(status);
    free(child_head);
    free(child_next);
    free(panel_offset);
    return result;
}

/* FactorSolve::solve's three sweeps (FactorSolve.cpp:31-158), column by column: forward over the supernodes in
 * increasing order (x_F <- L11^-1 x_F, q increasing; then x_R -= L21 x_F, terms in increasing q), diagonal
 * (x_j / d_j), backward in decreasing order (x_F -= L21^T x_R, then x_F <- L11^-T x_F from the last row up). */
int port_solve(int32_t dimension, int32_t supernode_count, const int32_t* first_column, const int32_t* parent,
               const int64_t* row_start, const int32_t* rows, const double* panels, double* b, int64_t ld,
               int64_t columns)
{
    (void)parent;
    int64_t* panel_offset = (int64_t*)calloc((size_t)supernode_count + 1, sizeof(int64_t));
    for (int32_t s = 0; s < supernode_count; ++s)
    {
        const int64_t c = first_column[s + 1] - first_column[s];
        const int64_t r = row_start[s + 1] - row_start[s];
        panel_offset[s + 1] = panel_offset[s] + c * (c + r);
    }
    for (int64_t col = 0; col < columns; ++col)
    {
        double* x = b + col * ld;
        for (int32_t s = 0; s < supernode_count; ++s)
        {
            const int32_t f = first_column[s];
            const int64_t c = first_column[s + 1] - f;
            const int64_t r = row_start[s + 1] - row_start[s];
            const int64_t n = c + r;
            const double* l = panels + panel_offset[s];
            const int32_t* rs = rows + row_start[s];
            for (int64_t i = 1; i < c; ++i)
                for (int64_t q = 0; q < i; ++q)
                    x[f + i] -= l[i + q * n] * x[f + q];
            for (int64_t i = 0; i < r; ++i)
                for (int64_t q = 0; q < c; ++q)
                    x[rs[i]] -= l[c + i + q * n] * x[f + q];
        }
        for (int32_t s = 0; s < supernode_count; ++s)
        {
            const int32_t f = first_column[s];
            const int64_t c = first_column[s + 1] - f;
            const int64_t n = c + (row_start[s + 1] - row_start[s]);
            const double* l = panels + panel_offset[s];
            for (int64_t k = 0; k < c; ++k)
                x[f + k] = x[f + k] / l[k + k * n];
        }
        for (int32_t s = supernode_count - 1; s >= 0; --s)
        {
            const int32_t f = first_column[s];
            const int64_t c = first_column[s + 1] - f;
            const int64_t r = row_start[s + 1] - row_start[s];
            const int64_t n = c + r;
            const double* l = panels + panel_offset[s];
            const int32_t* rs = rows + row_start[s];
            for (int64_t q = 0; q < c; ++q)
                for (int64_t i = 0; i < r; ++i)
                    x[f + q] -= l[c + i + q * n] * x[rs[i]];
            for (int64_t i = c - 1; i >= 0; --i)
                for (int64_t q = c - 1; q > i; --q)
                    x[f + i] -= l[q + i * n] * x[f + q];
        }
        for (int64_t i = 0; i < dimension; ++i)
            x[i] = x[i] + 0.0;
    }
    free(panel_offset);
    return 0;
}
