/* ORACLE — test infrastructure only (see gold.h).  Built with
 * -ffp-contract=off so every multiply and add rounds separately, as the
 * reference's gold kernel does when compiled for x86-64 without FMA. */
#include "gold.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define FAIL(...) do { if (err) snprintf(err, errlen, __VA_ARGS__); goto fail; } while (0)

static int read_exact(FILE* f, void* dst, size_t n) { return fread(dst, 1, n, f) == n; }

/* Width of the IA/JA integers in the compressed layout: 1, 2 or 4 bytes,
 * chosen by the column count (LinearBasis/gold/src/Data.cpp:526-548, 550-573). */
static int csr_width(int ncols)
{
	if (ncols <= 255) return 1;
	if (ncols <= 65535) return 2;
	return 4;
}

static uint32_t read_uint(const unsigned char* p, int w)
{
	if (w == 1) return p[0];
	if (w == 2) { uint16_t v; memcpy(&v, p, 2); return v; }
	uint32_t v; memcpy(&v, p, 4); return v;
}

/* One CSR block of the compressed layout (index: gold/src/Data.cpp:49-121,
 * surplus: :123-190): marker, u32 nnz, nnz values of `valsize` bytes,
 * (nno+1) IA deltas and nnz JA column ids of width w.  IA is rebuilt by prefix
 * sum; IA[0] must be 0 and IA must not decrease; JA must be < ncols. */
static int read_csr(FILE* f, const char* marker, int nno, int ncols, size_t valsize,
	void** vals, int** rowptr, uint32_t** cols, uint32_t* nnz_out, char* err, size_t errlen)
{
	char mk[16] = {0};
	size_t ml = strlen(marker);
	int w = csr_width(ncols);
	unsigned char* buf = NULL;
	uint32_t nnz = 0;
	*vals = NULL; *rowptr = NULL; *cols = NULL;
	if (!read_exact(f, mk, ml) || memcmp(mk, marker, ml)) FAIL("Cannot read %s data", marker);
	if (!read_exact(f, &nnz, 4)) FAIL("Cannot read %s nonzeros", marker);
	*vals = malloc(valsize * (nnz ? nnz : 1));
	if (!read_exact(f, *vals, valsize * nnz)) FAIL("Truncated %s values", marker);
	buf = malloc((size_t)w * ((uint32_t)(nno + 1) > nnz ? (uint32_t)(nno + 1) : nnz) + 4);
	if (!read_exact(f, buf, (size_t)w * (nno + 1))) FAIL("Truncated %s IA", marker);
	*rowptr = malloc(sizeof(int) * (nno + 1));
	(*rowptr)[0] = (int)read_uint(buf, w);
	for (int i = 1; i <= nno; i++) (*rowptr)[i] = (int)read_uint(buf + (size_t)w * i, w) + (*rowptr)[i - 1];
	if ((*rowptr)[0] != 0) FAIL("IA[0] must be 0");
	for (int i = 1; i <= nno; i++)
		if ((*rowptr)[i] < (*rowptr)[i - 1]) FAIL("IA must not decrease (IA[%d] < IA[%d])", i, i - 1);
	if ((uint32_t)(*rowptr)[nno] != nnz) FAIL("IA[nno] (%d) != nonzeros (%u)", (*rowptr)[nno], nnz);
	if (!read_exact(f, buf, (size_t)w * nnz)) FAIL("Truncated %s JA", marker);
	*cols = malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
	for (uint32_t k = 0; k < nnz; k++)
	{
		(*cols)[k] = read_uint(buf + (size_t)w * k, w);
		if ((int)(*cols)[k] >= ncols) FAIL("JA[%u] = %u out of column range", k, (*cols)[k]);
	}
	free(buf);
	*nnz_out = nnz;
	return 0;
fail:
	free(buf); free(*vals); free(*rowptr); free(*cols);
	*vals = NULL; *rowptr = NULL; *cols = NULL;
	return 1;
}

/* Level -> hat scale i for the uncompressed layouts: i = 2 << (l - 2)
 * (gold/src/Data.cpp:479).  Level 1 evaluates that shift with count -1, which
 * x86 masks to 31, giving 0: the constant basis function. */
static int level_to_i(int l)
{
	if (l == 1) return 0;
	if (l < 1 || l > 31) return -1;
	return 2 << (l - 2);
}

int oracle_plt_read(const char* path, int nagents, oracle_grid* g, char* err, size_t errlen)
{
	FILE* f = NULL;
	int hdr[4];
	char marker[11] = {0};
	int compressed = 0, binary = 1;
	memset(g, 0, sizeof(*g));

	f = fopen(path, "rb");
	if (!f) FAIL("Error opening file: %s", path);
	if (!read_exact(f, marker, 10)) FAIL("Error reading file: %s", path);
	compressed = !strcmp(marker, "compressed");
	if (!compressed) rewind(f);
	if (!read_exact(f, hdr, sizeof(hdr))) FAIL("Error reading file: %s", path);
	if (!compressed && hdr[0] != nagents)
	{
		/* Not a binary header: reopen as text (gold/src/Data.cpp:383-405). */
		fclose(f);
		f = fopen(path, "r");
		binary = 0;
		if (!f || fscanf(f, "%d %d %d %d", &hdr[0], &hdr[1], &hdr[2], &hdr[3]) != 4)
			FAIL("Error reading file: %s", path);
	}
	g->dim = hdr[0]; g->nno = hdr[1]; g->TotalDof = hdr[2]; g->Level = hdr[3];
	if (g->dim != nagents)
		FAIL("File \"%s\" # of dimensions (%d) mismatches config (%d)", path, g->dim, nagents);
	if (g->nno < 0 || g->TotalDof <= 0 || g->dim <= 0) FAIL("Bad header in %s", path);

	g->index = calloc((size_t)g->nno * 2 * g->dim + 1, sizeof(int));
	g->surplus = calloc((size_t)g->nno * g->TotalDof + 1, sizeof(double));
	if (!g->index || !g->surplus) FAIL("Out of memory");

	if (!compressed)
	{
		int* vals = malloc(sizeof(int) * 2 * g->dim);
		for (int n = 0; n < g->nno; n++)
		{
			int ok = 1;
			if (binary) ok = read_exact(f, vals, sizeof(int) * 2 * g->dim);
			else for (int k = 0; k < 2 * g->dim && ok; k++) ok = fscanf(f, "%d", &vals[k]) == 1;
			if (!ok) { free(vals); FAIL("Error reading file: %s", path); }
			for (int k = 0; k < g->dim; k++)
			{
				int i = level_to_i(vals[k]);
				if (i < 0) { int bad = vals[k]; free(vals); FAIL("Level %d out of range in %s", bad, path); }
				g->index[(size_t)n * 2 * g->dim + k] = i;
				/* j = index - 1, and 0 for the constant function (:485-494). */
				g->index[(size_t)n * 2 * g->dim + g->dim + k] = i ? vals[g->dim + k] - 1 : 0;
			}
			double* s = g->surplus + (size_t)n * g->TotalDof;
			if (binary) ok = read_exact(f, s, sizeof(double) * g->TotalDof);
			else for (int o = 0; o < g->TotalDof && ok; o++) ok = fscanf(f, "%lf", &s[o]) == 1;
			if (!ok) { free(vals); FAIL("Error reading file: %s", path); }
		}
		free(vals);
	}
	else
	{
		void* v = NULL; int* ia = NULL; uint32_t* ja = NULL; uint32_t nnz = 0;
		if (read_csr(f, "index", g->nno, g->dim, 4, &v, &ia, &ja, &nnz, err, errlen)) goto fail;
		/* Compressed pairs are stored already transformed: {u16 i, u16 j}. */
		for (int n = 0; n < g->nno; n++)
			for (int k = ia[n]; k < ia[n + 1]; k++)
			{
				uint16_t pr[2];
				memcpy(pr, (char*)v + 4 * (size_t)k, 4);
				g->index[(size_t)n * 2 * g->dim + ja[k]] = pr[0];
				g->index[(size_t)n * 2 * g->dim + g->dim + ja[k]] = pr[1];
			}
		free(v); free(ia); free(ja);
		if (read_csr(f, "surplus", g->nno, g->TotalDof, 8, &v, &ia, &ja, &nnz, err, errlen)) goto fail;
		for (int n = 0; n < g->nno; n++)
			for (int k = ia[n]; k < ia[n + 1]; k++)
				memcpy(&g->surplus[(size_t)n * g->TotalDof + ja[k]], (char*)v + 8 * (size_t)k, 8);
		free(v); free(ia); free(ja);
	}
	fclose(f);
	return 0;
fail:
	if (f) fclose(f);
	oracle_grid_free(g);
	return 1;
}

void oracle_grid_free(oracle_grid* g)
{
	free(g->index); free(g->surplus);
	g->index = NULL; g->surplus = NULL;
}

/* The reference's gold loop (LinearBasis/gold/src/InterpolateArray.cpp:26-41):
 * nodes in file order; per node the hats of all dims in dim order, multiplied
 * into temp starting from 1.0, skipping the node at the first hat <= 0; then
 * value[o] += temp * surplus[n][o]. */
void oracle_interpolate(const oracle_grid* g, const double* x, double* value)
{
	const int dim = g->dim, TD = g->TotalDof;
	memset(value, 0, sizeof(double) * TD);
	for (int n = 0; n < g->nno; n++)
	{
		const int* ii = g->index + (size_t)n * 2 * dim;
		const int* jj = ii + dim;
		double temp = 1.0;
		int zero = 0;
		for (int k = 0; k < dim; k++)
		{
			double xp = 1.0 - fabs(x[k] * ii[k] - jj[k]);
			if (xp <= 0.0) { zero = 1; break; }
			temp *= xp;
		}
		if (zero) continue;
		const double* s = g->surplus + (size_t)n * TD;
		for (int o = 0; o < TD; o++)
			value[o] += temp * s[o];
	}
}

struct batch_job
{
	const oracle_grid* g;
	long npts, next, chunk;
	const double* X;
	double* out;
	pthread_mutex_t lock;
};

static void* batch_worker(void* arg)
{
	struct batch_job* j = (struct batch_job*)arg;
	for (;;)
	{
		pthread_mutex_lock(&j->lock);
		long p0 = j->next;
		j->next += j->chunk;
		pthread_mutex_unlock(&j->lock);
		if (p0 >= j->npts) break;
		long p1 = p0 + j->chunk < j->npts ? p0 + j->chunk : j->npts;
		for (long p = p0; p < p1; p++)
			oracle_interpolate(j->g, j->X + (size_t)p * j->g->dim, j->out + (size_t)p * j->g->TotalDof);
	}
	return NULL;
}

void oracle_interpolate_batch(const oracle_grid* g, long npts, const double* X, double* out, int nthreads)
{
	if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
	if (nthreads < 1) nthreads = 1;
	struct batch_job j = { g, npts, 0, 4, X, out, PTHREAD_MUTEX_INITIALIZER };
	pthread_t* th = malloc(sizeof(pthread_t) * nthreads);
	for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, batch_worker, &j);
	for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
	free(th);
}

long oracle_active_count(const oracle_grid* g, const double* x)
{
	long cnt = 0;
	for (int n = 0; n < g->nno; n++)
	{
		const int* ii = g->index + (size_t)n * 2 * g->dim;
		const int* jj = ii + g->dim;
		int zero = 0;
		for (int k = 0; k < g->dim && !zero; k++)
			zero = 1.0 - fabs(x[k] * ii[k] - jj[k]) <= 0.0;
		cnt += !zero;
	}
	return cnt;
}

/* Gradient of the gold form (no counterpart in the reference, which has no
 * derivative path).  For an active node with hats h_k (all > 0) the weight is
 * w = prod_k h_k, dw/dx_k = (prod_{m != k} h_m) * (-i_k sign(x_k i_k - j_k)),
 * computed with prefix/suffix products (no division). */
void oracle_gradient(const oracle_grid* g, long npts, const double* X, const double* c,
	double* dx, double* ds)
{
	const int dim = g->dim, TD = g->TotalDof;
	double* h = malloc(sizeof(double) * (dim + 1));
	double* pre = malloc(sizeof(double) * (dim + 1));
	double* suf = malloc(sizeof(double) * (dim + 1));
	for (long p = 0; p < npts; p++)
	{
		const double* x = X + (size_t)p * dim;
		const double* cp = c + (size_t)p * TD;
		double* gx = dx + (size_t)p * dim;
		memset(gx, 0, sizeof(double) * dim);
		for (int n = 0; n < g->nno; n++)
		{
			const int* ii = g->index + (size_t)n * 2 * dim;
			const int* jj = ii + dim;
			int zero = 0;
			for (int k = 0; k < dim && !zero; k++)
			{
				h[k] = 1.0 - fabs(x[k] * ii[k] - jj[k]);
				zero = h[k] <= 0.0;
			}
			if (zero) continue;
			pre[0] = 1.0;
			for (int k = 0; k < dim; k++) pre[k + 1] = pre[k] * h[k];
			suf[dim] = 1.0;
			for (int k = dim - 1; k >= 0; k--) suf[k] = suf[k + 1] * h[k];
			const double w = pre[dim];
			const double* s = g->surplus + (size_t)n * TD;
			double cs = 0.0;
			for (int o = 0; o < TD; o++)
			{
				cs += cp[o] * s[o];
				ds[(size_t)n * TD + o] += cp[o] * w;
			}
			for (int k = 0; k < dim; k++)
			{
				if (!ii[k]) continue;
				double t = x[k] * ii[k] - jj[k];
				double slope = t > 0.0 ? -(double)ii[k] : (t < 0.0 ? (double)ii[k] : 0.0);
				gx[k] += cs * pre[k] * suf[k + 1] * slope;
			}
		}
	}
	free(h); free(pre); free(suf);
}
