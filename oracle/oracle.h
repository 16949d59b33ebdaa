/* CPU restatement of the reference's supernodal Cholesky path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the
 * checker; the product never links or calls it.
 *
 * It restates, in plain single-threaded C++, the algorithm of
 * Sparse::CholeskyDecomposition<double,int32,int64> of HenrikSchumacher/Tensors
 * (file:line citations are on each function in oracle.cpp).  Its integer
 * outputs are pinned bit-exact, and its floating-point outputs to rounding,
 * against the reference's own code compiled by oracle/Makefile (_ref/).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Supernode strategies, numbered as CholeskyDecomposition.hpp:119-124. */
enum { TB_ORACLE_MAXIMAL = 0, TB_ORACLE_FUNDAMENTAL = 1, TB_ORACLE_AMALGAMATED = 2 };

/* Full symmetric CSR pattern (sorted rows, diagonal present), n rows.
 * perm: perm[i] = original index placed at position i, or NULL for identity. */
void * tb_oracle_analyze( int n, const int64_t * outer, const int32_t * inner,
                          const int32_t * perm, int strategy, int amalgamation_threshold );
void   tb_oracle_destroy( void * h );

int     tb_oracle_sn_count( void * h );
/* Array selectors as in ref_driver.cpp: 0 perm, 1 inverse perm, 2 value
 * permutation, 3 SN_rp, 4 SN_outer, 5 SN_inner, 6 row_to_SN, 7 SN_tri_ptr,
 * 8 SN_rec_ptr, 9 assembly-tree parents, 10 elimination-tree parents,
 * 11 permuted outer, 12 permuted inner, 13 assembly-tree child pointers,
 * 14 assembly-tree child indices. */
int64_t tb_oracle_array_size( void * h, int which );
void    tb_oracle_array_copy( void * h, int which, int64_t * out );

/* Multifrontal numeric factorization; values in the caller's CSR order.
 * Returns 0 on success, 1 if a pivot was not positive. */
int     tb_oracle_factor( void * h, const double * values, double reg );
int64_t tb_oracle_tri_size( void * h );
int64_t tb_oracle_rec_size( void * h );
void    tb_oracle_tri_copy( void * h, double * out );
void    tb_oracle_rec_copy( void * h, double * out );

/* X = alpha * A^{-1} B + beta * X, row-major n x nrhs with leading dims. */
void    tb_oracle_solve( void * h, double alpha, const double * B, int ldB,
                         double beta, double * X, int ldX, int nrhs );
/* Half solves: which = 0 for U^T y = b (lower), 1 for U x = y (upper). */
void    tb_oracle_half_solve( void * h, int which, double alpha, const double * B, int ldB,
                              double beta, double * X, int ldX, int nrhs );
double  tb_oracle_log_det( void * h );

#ifdef __cplusplus
}
#endif
