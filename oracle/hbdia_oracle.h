/* Test infrastructure only: a plain-C restatement of the reference's HBDIA
 * hot path, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker.  Nothing in hbdia_b200 links or calls it.
 *
 * Pinned against the reference's own code compiled from its sources
 * (oracle/_ref/libhbdia_ref.so, see oracle/Makefile) and against the golden
 * fixtures in tests/golden/.
 */
#ifndef HBDIA_ORACLE_H
#define HBDIA_ORACLE_H
#include <stdint.h>

typedef struct orc_layout orc_layout;

/* sizes[] layout returned by orc_sizes():
 *  [0] num_blocks (maxNumBlocks)     [1] total kept offsets
 *  [2] value slots (offsets*bw)      [3] COO remainder entries
 *  [4] number of distinct diagonals  [5] histogram length
 *  [6] has_hbdia (0: nothing converted) [7] numRows  [8] numCols
 *  [9] COO row-pointer length (numRows+1, or 0) */
enum { ORC_NSIZES = 10 };

/* convertToHBDIAFormat restated (src/Format/HBDIA.cpp:507-718).
 * is_f32 selects the value type of vals (float when 1, double when 0).
 * Returns 0, or -1 on bad arguments, -2 when storage exceeds 1e11 slots
 * (src/Format/HBDIA.cpp:592-598). */
int orc_convert(const int32_t *rows, const int32_t *cols, const void *vals, int is_f32,
                int64_t nnz, int32_t numRows, int32_t numCols, int32_t blockWidth,
                int32_t threshold, int64_t maxCooEntries, orc_layout **out);
/* The partial-matrix form: offsets col - (row + rowBase). */
int orc_convert_partial(const int32_t *rows, const int32_t *cols, const void *vals, int is_f32,
                        int64_t nnz, int32_t numRows, int32_t numCols, int32_t rowBase, int32_t blockWidth,
                        int32_t threshold, int64_t maxCooEntries, orc_layout **out);
void orc_sizes(const orc_layout *h, int64_t *sizes);
void orc_export(const orc_layout *h, int32_t *offsets, int32_t *blockStart, void *data,
                int32_t *cooRow, int32_t *cooCol, void *cooVal, int32_t *cooRowPtr,
                int32_t *histBlocks, int32_t *histNnz);
void orc_destroy(orc_layout *h);

/* hbdiaSpMV restated: blocked-DIA part (src/Operations/HBDIASpMV.cu:7-74),
 * COO remainder (src/Operations/HBDIASpMV.cpp:36-99) and the merge
 * (src/Operations/HBDIASpMV.cu:77-88).  x and y hold numRows elements. */
void orc_spmv_f64(const orc_layout *h, const double *x, double *y);
void orc_spmv_f32(const orc_layout *h, const float *x, float *y);
/* A partial matrix's rows of y over the global x (numGlobalCols elements). */
void orc_spmv_partial_f64(const orc_layout *h, int32_t numGlobalCols, const double *x, double *y);
/* orc_spmv_f64 with the blocked-DIA values taken from `values` instead. */
void orc_spmv_f64_values(const orc_layout *h, const double *values, double *y, const double *x);

/* Whole-matrix COO SpMV over row-sorted COO, one thread, in the order of
 * cpu_coo_spmv_kernel (src/Operations/HBDIASpMV.cpp:36-99).  Rows without
 * entries are left untouched, as in the reference. */
void orc_coo_spmv_f64(const int32_t *rows, const int32_t *cols, const double *vals,
                      int64_t nnz, const double *x, int32_t numRows, double *y);

/* Seeded benchmark workloads (restated from this library's own generator so
 * that the checker and the reference's CPU arm need no product code):
 * x[i] = lo + (hi - lo) * U[0, 1) from MT19937-64(seed) */
void orc_fill_uniform(double *out, int64_t n, double lo, double hi, uint64_t seed);
/* 27-point stencil on nx*ny*nz (index k*nx*ny + j*nx + i; centre `center`,
 * neighbours `neighbor`) plus floor(frac * stencil entries) extra entries at
 * uniform (row, column) positions outside the stencil, without repeats,
 * values U(lo, hi); row-sorted, each row's stencil entries first.  Call with
 * rows == NULL for the count.  Returns 0, or -1 on bad arguments. */
int orc_workload_stencil27(int32_t nx, int32_t ny, int32_t nz, double center, double neighbor, double frac,
                           double lo, double hi, uint64_t seed, int64_t *nnzOut, int32_t *rows, int32_t *cols,
                           double *vals);

#endif
