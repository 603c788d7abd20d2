/*
 * chidg_oracle.h -- CPU FP64 restatement of ChiDG's implicit linear-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: the pytest
 * suite, __graft_entry__.smoke() and the cpu_baseline leg of bench.py call it
 * as the checker.  It is never linked into, loaded by, or used as a fallback
 * for the CUDA product library (chidg_b200/libchidg_gpu.so).
 *
 * Each routine restates one reference routine; the file:line it follows is
 * given beside the implementation in chidg_oracle.cpp.  Parity pinning: the
 * known-answer tests of the reference (test_fgmres.pf, test_fgmres_ref.pf,
 * test_ILU0_mod.pf, test_ILU0_HB_mod.pf, test_chidg_matrix_operator_*mv.pf)
 * are replayed against this library by tests/test_oracle_kat.py from the
 * fixtures in tests/golden/.  Dense b x b block inverses (LAPACK DGETRF +
 * DGETRI in the reference) are only pinned to tolerance against numpy.
 *
 * The pattern arguments use the same conventions as include/chidg_gpu.h:
 *  - elements are numbered 0..nelem-1 (all domains flattened, reference
 *    element order), each with nvars fields x nterms modes and ntime levels;
 *  - the vector is element-major; inside an element it is time-major, then
 *    field, then mode (densevector_t%get_time_start);
 *  - blocks are listed row by row in reference storage order
 *    (lblks in face order XI_MIN..ZETA_MAX,DIAG, then chi_blks, bc_blks,
 *    hb_blks) and stored packed, each column-major nrows x ncols.
 */
#ifndef CHIDG_ORACLE_H
#define CHIDG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_matrix orc_matrix;
typedef struct orc_precon orc_precon;

enum { ORC_BLK_LOCAL = 0, ORC_BLK_CHIMERA = 1, ORC_BLK_BC = 2, ORC_BLK_HB = 3 };
enum { ORC_PRECON_IDENTITY = 0, ORC_PRECON_JACOBI = 1, ORC_PRECON_ILU0 = 2, ORC_PRECON_RASILU0 = 3, ORC_PRECON_HB = 4 };
enum { ORC_OK = 0, ORC_EINVAL = 1, ORC_ESINGULAR = 3 };

typedef struct {
    double tol, rtol;
    int32_t nmax, nkrylov;
    int32_t orthogonalization;   /* 0 = CGS, 1 = MGS */
    int32_t inner_fgmres;
    double inner_tol, inner_rtol;
    int32_t inner_nmax, inner_nkrylov, inner_orthogonalization;
    int32_t use_controller;      /* 1: refresh M only when the matrix stamp changed */
} orc_fgmres_opts;

typedef struct {
    int32_t niter;
    int32_t nrestart;
    double residual_norm;        /* true ||b - A x|| (print_report) */
    double res_estimate;         /* |p(j+1)| at exit */
    double r0norm_initial;
    int32_t nhist;               /* entries written to hist */
} orc_fgmres_result;

orc_matrix* orc_matrix_create(int32_t nelem, int32_t ntime,
                              const int32_t* elem_nvars, const int32_t* elem_nterms,
                              const int32_t* elem_proc, int64_t nblocks,
                              const int32_t* blk_row_elem, const int32_t* blk_row_time,
                              const int32_t* blk_col_elem, const int32_t* blk_col_time,
                              const int32_t* blk_kind);
void    orc_matrix_destroy(orc_matrix*);
int64_t orc_matrix_nvalues(const orc_matrix*);
int64_t orc_matrix_nvec(const orc_matrix*);
int     orc_matrix_set_values(orc_matrix*, const double* packed);
int     orc_matrix_get_values(const orc_matrix*, double* packed);
int     orc_matrix_block_offsets(const orc_matrix*, int64_t* offsets);
int     orc_mv(orc_matrix*, const double* x, double* y);
double  orc_dot(const orc_matrix*, const double* x, const double* y);
double  orc_norm(const orc_matrix*, const double* x);
int     orc_inv(int32_t n, const double* a, double* ainv);
/* Host threads for the data-parallel loops (matrix rows, ILU rows of one
 * dependency level, RAS subdomains, independent Gram-Schmidt dots).  Results
 * are bitwise the same for every thread count: each row, dot or vector entry
 * is computed on one thread in the serial order.  Default 1. */
int     orc_set_threads(int32_t n);
int32_t orc_get_threads(void);

orc_precon* orc_precon_create(orc_matrix*, int32_t kind);
void    orc_precon_destroy(orc_precon*);
int     orc_precon_update(orc_precon*, orc_matrix*);
int     orc_precon_apply(orc_precon*, orc_matrix*, const double* v, double* z);
int     orc_precon_error_elem(const orc_precon*);
/* Factor blocks: for each LOCAL block k of the matrix, LD holds the L block
 * (lower) or the inverted diagonal (diag); other entries are left as zero.
 * Only defined for ILU0 / JACOBI. */
int     orc_precon_get_LD(const orc_precon*, double* packed);

int     orc_fgmres_solve(orc_matrix*, orc_precon*, const double* b, double* x,
                         const orc_fgmres_opts*, orc_fgmres_result*, double* hist, int32_t hist_cap);
void    orc_matrix_touch(orc_matrix*);   /* bump the stamp, as chidg_matrix%store does */
/* chidg_matrix_t%transposed: orc_mv then computes A^T x, ILU0 / Jacobi factor
 * A^T and RASILU0 refuses (ORC_EINVAL), as the reference does. */
int     orc_matrix_set_transposed(orc_matrix*, int32_t transposed);

#ifdef __cplusplus
}
#endif
#endif
