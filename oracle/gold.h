/* ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference's FP64 "gold" interpolation path and
 * of its .plt grid reader.  It is the checker that the CUDA product is compared
 * against (tests, __graft_entry__.smoke and bench.py's cpu_baseline only); the
 * product never links, loads or calls it.
 *
 * Pinned against: the reference's known-answer test (surplus.plt, init(),
 * check() in LinearBasis/tests/InterpolateArray/test.cpp:24-215) and
 * bit-for-bit against the reference's own gold kernel compiled in place
 * (oracle/_ref/libref_gold.so) on the same grids and points.
 */
#ifndef SGI_ORACLE_GOLD_H
#define SGI_ORACLE_GOLD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A dense grid as the reference's DataDense holds it
 * (LinearBasis/gold/include/Data.h:252-273), without row padding:
 *   index[n*2*dim + k]       = i (0 when dim k is at level 1)
 *   index[n*2*dim + dim + k] = j
 *   surplus[n*TotalDof + o] */
typedef struct oracle_grid
{
	int dim, nno, TotalDof, Level;
	int* index;
	double* surplus;
} oracle_grid;

/* Reads a .plt file in any of the reference's three layouts (compressed,
 * binary, text).  Returns 0 on success; on failure returns a nonzero code and
 * writes a message to err (the reference prints it and abort()s instead). */
int oracle_plt_read(const char* path, int nagents, oracle_grid* g, char* err, size_t errlen);
void oracle_grid_free(oracle_grid* g);

/* One point: value[0..TotalDof) = sum over nodes of surplus * prod of hats. */
void oracle_interpolate(const oracle_grid* g, const double* x, double* value);

/* npts points (X row-major npts x dim, out npts x TotalDof), OpenMP over
 * points with nthreads threads (<=0: all). */
void oracle_interpolate_batch(const oracle_grid* g, long npts, const double* X, double* out, int nthreads);

/* Gradient of L = sum_p sum_o c[p,o] f_o(x_p):
 *   dx[p*dim + k] = dL/dx_{p,k}
 *   ds[n*TotalDof + o] += dL/dsurplus[n,o]   (accumulated, caller zeroes)
 * Slopes are one-sided at kinks: d/dx (1-|x i - j|) = -i sign(x i - j), with
 * sign(0) = 0.  Single-threaded (ds is a shared accumulator). */
void oracle_gradient(const oracle_grid* g, long npts, const double* X, const double* c,
	double* dx, double* ds);

/* Number of nodes with non-zero weight at x (the "active" count A(x)). */
long oracle_active_count(const oracle_grid* g, const double* x);

/* The seeded synthetic workload, restated (oracle/gen.c): the same grids and
 * points as the product's sgi_gen_adaptive and sgi_gen_points.  The grid's
 * arrays are malloc'd (free with oracle_grid_free).  Return 0 on success. */
int oracle_gen_adaptive(int dim, int nno, int TotalDof, int max_level, double p_dim, unsigned long long seed,
	oracle_grid* g);
int oracle_gen_points(int dim, long npts, int kind, unsigned long long seed, double kink_reject, int max_level,
	double* out);

/* Writes the compressed .plt layout the reference's loaders read. */
int oracle_plt_write(const oracle_grid* g, const char* path);

#ifdef __cplusplus
}
#endif

#endif
