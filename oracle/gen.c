/* ORACLE — test infrastructure only.
 *
 * The seeded synthetic workload (adaptive grids, query points) restated in C,
 * so that the timed CPU reference arm can build its grid file and points
 * without loading the product library.  It must produce the same grids and
 * points as the product's generators (sgi_gen_adaptive, sgi_gen_points), which
 * tests/test_oracle.py checks array for array.
 *
 * Random numbers: xoshiro256** (Blackman & Vigna, 2018) seeded through
 * splitmix64; a double takes the top 53 bits of a draw; normals by Box-Muller.
 * Adaptive grid: from the level-1 root, repeatedly take a uniformly random
 * leaf and add its hierarchical children along a random non-empty subset of
 * dimensions (each with probability p_dim; one uniform dimension when none is
 * drawn), skipping children above max_level and nodes already present, until
 * nno nodes exist; nodes are emitted in depth-first preorder of that
 * refinement tree, surplus[n][o] = uniform[-1,1] * 2^(-2 * sum_k (l_k - 1)).
 */
#include "gold.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s[4]; } rng_t;

static void rng_seed(rng_t* r, uint64_t seed)
{
	for (int k = 0; k < 4; k++)
	{
		seed += 0x9e3779b97f4a7c15ull;
		uint64_t z = seed;
		z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
		z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
		r->s[k] = z ^ (z >> 31);
	}
}

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(rng_t* r)
{
	uint64_t* s = r->s;
	const uint64_t out = rotl64(s[1] * 5, 7) * 9, t = s[1] << 17;
	s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
	s[2] ^= t; s[3] = rotl64(s[3], 45);
	return out;
}

static double rng_uniform(rng_t* r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }
static uint64_t rng_below(rng_t* r, uint64_t n) { return (uint64_t)(rng_uniform(r) * (double)n) % n; }

static double rng_normal(rng_t* r)
{
	double u1 = rng_uniform(r), u2 = rng_uniform(r);
	if (u1 < 1e-300) u1 = 1e-300;
	return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

/* One non-constant dimension of a node: level l >= 2, hat centre index j. */
typedef struct { uint16_t dim; uint8_t l; uint16_t j; } comp_t;

typedef struct
{
	comp_t* comps;      /* all nodes' components, node n at [off[n], off[n+1]) */
	size_t ncomps, capcomps;
	uint32_t* off;
	int n, cap;
	int* table;         /* open addressing: node id + 1, 0 = empty */
	size_t tmask;
} store_t;

static uint64_t node_hash(const comp_t* c, int cnt)
{
	uint64_t h = 0x243f6a8885a308d3ull;
	for (int k = 0; k < cnt; k++)
	{
		h ^= ((uint64_t)c[k].dim << 24) | ((uint64_t)c[k].l << 16) | c[k].j;
		h *= 0x100000001b3ull;
		h ^= h >> 31;
	}
	return h;
}

static int node_same(const store_t* st, int n, const comp_t* c, int cnt)
{
	if ((int)(st->off[n + 1] - st->off[n]) != cnt) return 0;
	const comp_t* a = st->comps + st->off[n];
	for (int k = 0; k < cnt; k++)
		if (a[k].dim != c[k].dim || a[k].l != c[k].l || a[k].j != c[k].j) return 0;
	return 1;
}

/* Adds the node if absent; returns its id, or -1 if it was present. */
static int store_add(store_t* st, const comp_t* c, int cnt)
{
	size_t slot = node_hash(c, cnt) & st->tmask;
	while (st->table[slot])
	{
		if (node_same(st, st->table[slot] - 1, c, cnt)) return -1;
		slot = (slot + 1) & st->tmask;
	}
	if (st->ncomps + cnt > st->capcomps)
	{
		st->capcomps = 2 * st->capcomps + cnt;
		st->comps = realloc(st->comps, st->capcomps * sizeof(comp_t));
	}
	memcpy(st->comps + st->ncomps, c, cnt * sizeof(comp_t));
	st->ncomps += cnt;
	st->off[st->n + 1] = (uint32_t)st->ncomps;
	st->table[slot] = st->n + 1;
	return st->n++;
}

int oracle_gen_adaptive(int dim, int nno, int TotalDof, int max_level, double p_dim, unsigned long long seed,
	oracle_grid* g)
{
	memset(g, 0, sizeof(*g));
	if (dim <= 0 || dim > 65535 || nno < 1 || TotalDof <= 0 || max_level < 2 || max_level > 15 ||
		!(p_dim > 0.0 && p_dim <= 1.0))
		return 1;
	store_t st = {0};
	st.cap = nno;
	st.off = calloc((size_t)nno + 1, sizeof(uint32_t));
	size_t tsize = 1;
	while (tsize < (size_t)nno * 2) tsize <<= 1;
	st.table = calloc(tsize, sizeof(int));
	st.tmask = tsize - 1;
	st.capcomps = 1024;
	st.comps = malloc(st.capcomps * sizeof(comp_t));
	/* refinement tree: children in insertion order */
	int* first = malloc(sizeof(int) * nno);
	int* last = malloc(sizeof(int) * nno);
	int* next = malloc(sizeof(int) * nno);
	int* leaves = malloc(sizeof(int) * nno);
	int* chosen = malloc(sizeof(int) * dim);
	comp_t* c = calloc((size_t)dim + 1, sizeof(comp_t));
	int nleaves = 0;
	rng_t rng;
	rng_seed(&rng, seed);
	store_add(&st, c, 0);
	first[0] = last[0] = next[0] = -1;
	leaves[nleaves++] = 0;
	int rc = 0;
	while (st.n < nno)
	{
		if (!nleaves) { rc = 2; goto out; }
		const size_t k = rng_below(&rng, (uint64_t)nleaves);
		const int n = leaves[k];
		leaves[k] = leaves[--nleaves];
		int nch = 0;
		for (int d = 0; d < dim; d++)
			if (rng_uniform(&rng) < p_dim) chosen[nch++] = d;
		if (!nch) chosen[nch++] = (int)rng_below(&rng, (uint64_t)dim);
		for (int q0 = 0; q0 < nch; q0++)
		{
			const int d = chosen[q0];
			const comp_t* b = st.comps + st.off[n];
			const int cnt = (int)(st.off[n + 1] - st.off[n]);
			int pos = -1, l = 1, j = 0;
			for (int q = 0; q < cnt; q++)
				if (b[q].dim == d) { pos = q; l = b[q].l; j = b[q].j; }
			if (l + 1 > max_level) continue;
			int cj[2], nc;
			if (l == 1) { cj[0] = 0; cj[1] = 2; nc = 2; }
			else if (l == 2) { cj[0] = j == 0 ? 1 : 3; nc = 1; }
			else { cj[0] = 2 * j - 1; cj[1] = 2 * j + 1; nc = 2; }
			for (int q = 0; q < nc && st.n < nno; q++)
			{
				/* the parent's components with dimension d replaced or
				 * inserted in dimension order */
				const comp_t nc_ = { (uint16_t)d, (uint8_t)(l + 1), (uint16_t)cj[q] };
				int m = 0;
				if (pos >= 0)
				{
					memcpy(c, b, cnt * sizeof(comp_t));
					c[pos] = nc_;
					m = cnt;
				}
				else
				{
					int ins = 0;
					while (ins < cnt && b[ins].dim < d) ins++;
					memcpy(c, b, ins * sizeof(comp_t));
					c[ins] = nc_;
					memcpy(c + ins + 1, b + ins, (cnt - ins) * sizeof(comp_t));
					m = cnt + 1;
				}
				const int id = store_add(&st, c, m);
				b = st.comps + st.off[n];      /* store_add may move the components */
				if (id < 0) continue;
				first[id] = last[id] = next[id] = -1;
				if (last[n] < 0) first[n] = id;
				else next[last[n]] = id;
				last[n] = id;
				leaves[nleaves++] = id;
			}
			if (st.n >= nno) break;
		}
	}
	/* depth-first preorder of the refinement tree */
	{
		int* order = malloc(sizeof(int) * nno);
		int* stack = malloc(sizeof(int) * nno);
		int no = 0, sp = 0;
		stack[sp++] = 0;
		while (sp)
		{
			const int n = stack[--sp];
			order[no++] = n;
			/* push children in reverse so the first child is visited first */
			int tmp = sp;
			for (int ch = first[n]; ch >= 0; ch = next[ch]) stack[sp++] = ch;
			for (int a = tmp, b2 = sp - 1; a < b2; a++, b2--) { int t = stack[a]; stack[a] = stack[b2]; stack[b2] = t; }
		}
		g->dim = dim; g->nno = nno; g->TotalDof = TotalDof;
		g->index = calloc((size_t)nno * 2 * dim + 1, sizeof(int));
		g->surplus = malloc(sizeof(double) * ((size_t)nno * TotalDof + 1));
		rng_t rs;
		rng_seed(&rs, seed ^ 0x5eed5eed5eed5eedull);
		int maxdepth = 0;
		for (int r = 0; r < nno; r++)
		{
			const int n = order[r];
			int depth = 0;
			for (uint32_t q = st.off[n]; q < st.off[n + 1]; q++)
			{
				const comp_t* cc = st.comps + q;
				g->index[(size_t)r * 2 * dim + cc->dim] = 1 << (cc->l - 1);
				g->index[(size_t)r * 2 * dim + dim + cc->dim] = cc->j;
				depth += cc->l - 1;
			}
			if (depth > maxdepth) maxdepth = depth;
			const double scale = ldexp(1.0, -2 * depth);
			for (int o = 0; o < TotalDof; o++)
				g->surplus[(size_t)r * TotalDof + o] = (2.0 * rng_uniform(&rs) - 1.0) * scale;
		}
		g->Level = maxdepth;
		free(order);
		free(stack);
	}
out:
	free(first); free(last); free(next); free(leaves); free(chosen); free(c);
	free(st.comps); free(st.off); free(st.table);
	return rc;
}

int oracle_gen_points(int dim, long npts, int kind, unsigned long long seed, double kink_reject, int max_level,
	double* out)
{
	if (dim <= 0 || npts < 0 || kind < 0 || kind > 2 || max_level < 1 || max_level > 30) return 1;
	rng_t rng;
	rng_seed(&rng, seed);
	const double cell = ldexp(1.0, -(max_level - 1));
	for (long p = 0; p < npts; p++)
	{
		const int clustered = kind == 1 || (kind == 2 && p >= npts / 2);
		double* x = out + (size_t)p * dim;
		for (long attempt = 0;; attempt++)
		{
			int ok = 1;
			for (int d = 0; d < dim; d++)
			{
				double v = clustered ? 0.5 + 0.05 * rng_normal(&rng) : rng_uniform(&rng);
				v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
				x[d] = v;
				if (kink_reject > 0.0)
				{
					const double r = v / cell;
					if (fabs(r - nearbyint(r)) * cell < kink_reject) ok = 0;
				}
			}
			if (ok) break;
			if (attempt > 1000000) return 2;
		}
	}
	return 0;
}

static void put_uint(FILE* f, uint32_t v, int w, int* ok)
{
	for (int b = 0; b < w; b++)
		if (putc_unlocked((int)((v >> (8 * b)) & 0xffu), f) == EOF) *ok = 0;
}

static int csr_cols_width(int ncols) { return ncols <= 255 ? 1 : (ncols <= 65535 ? 2 : 4); }

/* The compressed .plt layout that the reference's loaders read
 * (LinearBasis/gold/src/Data.cpp:49-190, 322-595): marker "compressed",
 * int32 header {dim, nno, TotalDof, Level}; "index", u32 nnz, nnz pairs
 * {u16 i, u16 j} of the non-constant dimensions, (nno + 1) row counts (the
 * first 0) and nnz dimension ids; "surplus", u32 nnz, nnz doubles whose bit
 * pattern is not zero, (nno + 1) row counts and nnz output ids.  Counts and
 * ids are 1, 2 or 4 bytes wide by the column count (255 / 65535). */
int oracle_plt_write(const oracle_grid* g, const char* path)
{
	const int D = g->dim, TD = g->TotalDof;
	FILE* f = fopen(path, "wb");
	if (!f) return 1;
	setvbuf(f, NULL, _IOFBF, 1 << 22);
	int ok = fwrite("compressed", 1, 10, f) == 10;
	const int hdr[4] = { g->dim, g->nno, g->TotalDof, g->Level };
	ok = ok && fwrite(hdr, sizeof(int), 4, f) == 4;
	/* index block */
	uint32_t nnz = 0;
	for (size_t k = 0; k < (size_t)g->nno * D; k++)
	{
		const size_t n = k / D, d = k % D;
		if (g->index[n * 2 * D + d] || g->index[n * 2 * D + D + d]) nnz++;
	}
	ok = ok && fwrite("index", 1, 5, f) == 5;
	put_uint(f, nnz, 4, &ok);
	for (int n = 0; n < g->nno; n++)
		for (int d = 0; d < D; d++)
		{
			const int i = g->index[(size_t)n * 2 * D + d], j = g->index[(size_t)n * 2 * D + D + d];
			if (!i && !j) continue;
			if (i < 0 || i > 65535 || j < 0 || j > 65535) { fclose(f); return 3; }
			const uint16_t pr[2] = { (uint16_t)i, (uint16_t)j };
			if (fwrite(pr, 2, 2, f) != 2) ok = 0;
		}
	int w = csr_cols_width(D);
	put_uint(f, 0, w, &ok);
	for (int n = 0; n < g->nno; n++)
	{
		uint32_t c = 0;
		for (int d = 0; d < D; d++) c += g->index[(size_t)n * 2 * D + d] || g->index[(size_t)n * 2 * D + D + d];
		put_uint(f, c, w, &ok);
	}
	for (int n = 0; n < g->nno; n++)
		for (int d = 0; d < D; d++)
			if (g->index[(size_t)n * 2 * D + d] || g->index[(size_t)n * 2 * D + D + d]) put_uint(f, (uint32_t)d, w, &ok);
	/* surplus block */
	nnz = 0;
	for (size_t k = 0; k < (size_t)g->nno * TD; k++)
	{
		uint64_t bits;
		memcpy(&bits, g->surplus + k, 8);
		nnz += bits != 0;
	}
	ok = ok && fwrite("surplus", 1, 7, f) == 7;
	put_uint(f, nnz, 4, &ok);
	for (size_t k = 0; k < (size_t)g->nno * TD; k++)
	{
		uint64_t bits;
		memcpy(&bits, g->surplus + k, 8);
		if (bits)
			for (int b = 0; b < 8; b++)
				if (putc_unlocked((int)((bits >> (8 * b)) & 0xffu), f) == EOF) ok = 0;
	}
	w = csr_cols_width(TD);
	put_uint(f, 0, w, &ok);
	for (int n = 0; n < g->nno; n++)
	{
		uint32_t c = 0;
		for (int o = 0; o < TD; o++)
		{
			uint64_t bits;
			memcpy(&bits, g->surplus + (size_t)n * TD + o, 8);
			c += bits != 0;
		}
		put_uint(f, c, w, &ok);
	}
	for (int n = 0; n < g->nno; n++)
		for (int o = 0; o < TD; o++)
		{
			uint64_t bits;
			memcpy(&bits, g->surplus + (size_t)n * TD + o, 8);
			if (bits) put_uint(f, (uint32_t)o, w, &ok);
		}
	if (fclose(f)) ok = 0;
	return ok ? 0 : 2;
}
