// Host layer of the B200 sparse-grid interpolator: grid files, synthetic grids
// and points, the reference-compatible xps/chains form, and the device layout
// (containment tree with skip pointers) that the kernels traverse.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <unordered_set>

#include "sgi_internal.h"

namespace sgi {

static thread_local std::string g_error;

int fail(int code, const char* fmt, ...)
{
	char buf[1024];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	g_error = buf;
	return code;
}

void clear_error() { g_error.clear(); }

} // namespace sgi

using namespace sgi;

extern "C" const char* sgi_last_error(void) { return g_error.c_str(); }

// ============================================================== .plt reading
//
// Three layouts, selected as the reference's DataDense::load selects them
// (LinearBasis/gold/src/Data.cpp:322-405):
//  * "compressed": a 10-byte marker, int32 {dim, nno, TotalDof, Level}, then two
//    CSR blocks, "index" (values {u16 i, u16 j}, already in (i, j) form) and
//    "surplus" (f64 values).  Each block: marker, u32 nnz, values, nno+1 row
//    deltas, nnz column ids; deltas and ids are u8/u16/u32 by column count.
//  * binary: int32 header, then per node 2*dim int32 (levels, then 1-based
//    indices) and TotalDof f64.
//  * text: the same numbers as whitespace-separated text; chosen when the
//    binary header's dim differs from nagents.
// Levels become i = 2^(l-1) (0 for level 1) and j = index - 1 (0 for level 1).

namespace {

struct File
{
	FILE* f = nullptr;
	~File() { if (f) fclose(f); }
	bool read(void* dst, size_t n) { return fread(dst, 1, n, f) == n; }
};

int csr_width(int ncols) { return ncols <= 255 ? 1 : (ncols <= 65535 ? 2 : 4); }

uint32_t get_uint(const unsigned char* p, int w)
{
	if (w == 1) return p[0];
	if (w == 2) { uint16_t v; memcpy(&v, p, 2); return v; }
	uint32_t v; memcpy(&v, p, 4); return v;
}

// Reads one CSR block; calls put(row, col, value_bytes) per nonzero.
template <class Put>
int read_block(File& in, const char* marker, int nno, int ncols, size_t vsize, const char* path, Put put)
{
	size_t ml = strlen(marker);
	char mk[16] = {0};
	if (!in.read(mk, ml) || memcmp(mk, marker, ml))
		return fail(SGI_E_FORMAT, "%s: cannot read %s data", path, marker);
	uint32_t nnz = 0;
	if (!in.read(&nnz, 4)) return fail(SGI_E_FORMAT, "%s: cannot read %s nonzeros", path, marker);
	std::vector<unsigned char> vals((size_t)nnz * vsize);
	if (!in.read(vals.data(), vals.size())) return fail(SGI_E_FORMAT, "%s: truncated %s values", path, marker);
	const int w = csr_width(ncols);
	std::vector<unsigned char> raw((size_t)w * (nno + 1));
	if (!in.read(raw.data(), raw.size())) return fail(SGI_E_FORMAT, "%s: truncated %s row deltas", path, marker);
	std::vector<int64_t> ia(nno + 1);
	ia[0] = get_uint(raw.data(), w);
	if (ia[0] != 0) return fail(SGI_E_FORMAT, "%s: %s IA[0] must be 0", path, marker);
	for (int r = 1; r <= nno; r++) ia[r] = ia[r - 1] + get_uint(raw.data() + (size_t)w * r, w);
	if (ia[nno] != (int64_t)nnz)
		return fail(SGI_E_FORMAT, "%s: %s rows hold %lld nonzeros, header says %u", path, marker,
			(long long)ia[nno], nnz);
	raw.resize((size_t)w * nnz);
	if (!in.read(raw.data(), raw.size())) return fail(SGI_E_FORMAT, "%s: truncated %s columns", path, marker);
	for (int r = 0; r < nno; r++)
		for (int64_t k = ia[r]; k < ia[r + 1]; k++)
		{
			uint32_t c = get_uint(raw.data() + (size_t)w * k, w);
			if ((int)c >= ncols || (int)c < 0)
				return fail(SGI_E_FORMAT, "%s: %s column %u out of range", path, marker, c);
			put(r, (int)c, vals.data() + vsize * k);
		}
	return SGI_OK;
}

int level_to_i(int l)
{
	if (l == 1) return 0;
	if (l < 1 || l > 31) return -1;
	return 1 << (l - 1);
}

} // namespace

extern "C" int sgi_host_grid_read_plt(const char* path, int nagents, sgi_host_grid_t* out)
{
	clear_error();
	if (!path || !out) return fail(SGI_E_INVALID, "null argument");
	*out = nullptr;
	File in;
	in.f = fopen(path, "rb");
	if (!in.f) return fail(SGI_E_FORMAT, "Error opening file: %s", path);
	char marker[11] = {0};
	if (!in.read(marker, 10)) return fail(SGI_E_FORMAT, "Error reading file: %s", path);
	const bool compressed = !strcmp(marker, "compressed");
	if (!compressed) rewind(in.f);
	int hdr[4];
	if (!in.read(hdr, sizeof(hdr))) return fail(SGI_E_FORMAT, "Error reading file: %s", path);
	bool binary = true;
	if (!compressed && hdr[0] != nagents)
	{
		fclose(in.f);
		in.f = fopen(path, "r");
		binary = false;
		if (!in.f || fscanf(in.f, "%d %d %d %d", &hdr[0], &hdr[1], &hdr[2], &hdr[3]) != 4)
			return fail(SGI_E_FORMAT, "Error reading file: %s", path);
	}
	if (hdr[0] != nagents)
		return fail(SGI_E_MISMATCH, "File \"%s\" # of dimensions (%d) mismatches config (%d)", path, hdr[0], nagents);
	if (hdr[0] <= 0 || hdr[1] < 0 || hdr[2] <= 0)
		return fail(SGI_E_FORMAT, "%s: bad header {%d, %d, %d}", path, hdr[0], hdr[1], hdr[2]);
	sgi_host_grid* hg = new (std::nothrow) sgi_host_grid;
	if (!hg) return fail(SGI_E_NOMEM, "out of memory");
	HostGrid& g = hg->g;
	g.dim = hdr[0]; g.nno = hdr[1]; g.TotalDof = hdr[2]; g.Level = hdr[3];
	try
	{
		g.index.assign((size_t)g.nno * 2 * g.dim, 0);
		g.surplus.assign((size_t)g.nno * g.TotalDof, 0.0);
	}
	catch (...) { delete hg; return fail(SGI_E_NOMEM, "out of memory for %d nodes", hdr[1]); }
	int rc = SGI_OK;
	const int D = g.dim, TD = g.TotalDof;
	if (compressed)
	{
		rc = read_block(in, "index", g.nno, D, 4, path, [&](int r, int c, const unsigned char* v)
		{
			uint16_t p[2];
			memcpy(p, v, 4);
			g.index[(size_t)r * 2 * D + c] = p[0];
			g.index[(size_t)r * 2 * D + D + c] = p[1];
		});
		if (rc == SGI_OK)
			rc = read_block(in, "surplus", g.nno, TD, 8, path, [&](int r, int c, const unsigned char* v)
			{
				memcpy(&g.surplus[(size_t)r * TD + c], v, 8);
			});
	}
	else
	{
		std::vector<int> vals(2 * D);
		for (int n = 0; n < g.nno && rc == SGI_OK; n++)
		{
			bool ok = true;
			if (binary) ok = in.read(vals.data(), sizeof(int) * 2 * D);
			else for (int k = 0; k < 2 * D && ok; k++) ok = fscanf(in.f, "%d", &vals[k]) == 1;
			if (!ok) { rc = fail(SGI_E_FORMAT, "Error reading file: %s (node %d)", path, n); break; }
			for (int k = 0; k < D; k++)
			{
				int i = level_to_i(vals[k]);
				if (i < 0) { rc = fail(SGI_E_FORMAT, "%s: level %d out of range", path, vals[k]); break; }
				g.index[(size_t)n * 2 * D + k] = i;
				g.index[(size_t)n * 2 * D + D + k] = i ? vals[D + k] - 1 : 0;
			}
			double* s = &g.surplus[(size_t)n * TD];
			if (binary) ok = in.read(s, sizeof(double) * TD);
			else for (int o = 0; o < TD && ok; o++) ok = fscanf(in.f, "%lf", &s[o]) == 1;
			if (!ok && rc == SGI_OK) rc = fail(SGI_E_FORMAT, "Error reading file: %s (node %d)", path, n);
		}
	}
	if (rc != SGI_OK) { delete hg; return rc; }
	*out = hg;
	return SGI_OK;
}

// ============================================================== .plt writing

namespace {

void put_uint(std::vector<unsigned char>& b, uint32_t v, int w)
{
	unsigned char t[4];
	memcpy(t, &v, 4);
	b.insert(b.end(), t, t + w);
}

} // namespace

extern "C" int sgi_host_grid_write_plt(sgi_host_grid_t hg, const char* path)
{
	clear_error();
	if (!hg || !path) return fail(SGI_E_INVALID, "null argument");
	const HostGrid& g = hg->g;
	const int D = g.dim, TD = g.TotalDof;
	std::vector<unsigned char> b;
	b.reserve((size_t)g.nno * 64 + 1024);
	const char* mk = "compressed";
	b.insert(b.end(), mk, mk + 10);
	int hdr[4] = { g.dim, g.nno, g.TotalDof, g.Level };
	b.insert(b.end(), (unsigned char*)hdr, (unsigned char*)hdr + 16);
	// index block
	{
		std::vector<uint16_t> pairs;
		std::vector<uint32_t> rowcnt(g.nno), cols;
		for (int n = 0; n < g.nno; n++)
			for (int k = 0; k < D; k++)
			{
				int i = g.index[(size_t)n * 2 * D + k], j = g.index[(size_t)n * 2 * D + D + k];
				if (!i && !j) continue;
				if (i < 0 || i > 65535 || j < 0 || j > 65535)
					return fail(SGI_E_RANGE, "node %d dim %d: (i, j) = (%d, %d) does not fit u16", n, k, i, j);
				pairs.push_back((uint16_t)i); pairs.push_back((uint16_t)j);
				cols.push_back(k); rowcnt[n]++;
			}
		const int w = csr_width(D);
		b.insert(b.end(), (const unsigned char*)"index", (const unsigned char*)"index" + 5);
		put_uint(b, (uint32_t)cols.size(), 4);
		b.insert(b.end(), (unsigned char*)pairs.data(), (unsigned char*)(pairs.data() + pairs.size()));
		put_uint(b, 0, w);
		for (int n = 0; n < g.nno; n++) put_uint(b, rowcnt[n], w);
		for (uint32_t c : cols) put_uint(b, c, w);
	}
	// surplus block (entries whose bit pattern is non-zero)
	{
		std::vector<double> vals;
		std::vector<uint32_t> rowcnt(g.nno), cols;
		for (int n = 0; n < g.nno; n++)
			for (int o = 0; o < TD; o++)
			{
				double v = g.surplus[(size_t)n * TD + o];
				uint64_t bits; memcpy(&bits, &v, 8);
				if (!bits) continue;
				vals.push_back(v); cols.push_back(o); rowcnt[n]++;
			}
		const int w = csr_width(TD);
		b.insert(b.end(), (const unsigned char*)"surplus", (const unsigned char*)"surplus" + 7);
		put_uint(b, (uint32_t)vals.size(), 4);
		b.insert(b.end(), (unsigned char*)vals.data(), (unsigned char*)(vals.data() + vals.size()));
		put_uint(b, 0, w);
		for (int n = 0; n < g.nno; n++) put_uint(b, rowcnt[n], w);
		for (uint32_t c : cols) put_uint(b, c, w);
	}
	FILE* f = fopen(path, "wb");
	if (!f) return fail(SGI_E_FORMAT, "cannot create %s", path);
	size_t wrote = fwrite(b.data(), 1, b.size(), f);
	int cl = fclose(f);
	if (wrote != b.size() || cl) return fail(SGI_E_FORMAT, "short write to %s", path);
	return SGI_OK;
}

extern "C" int sgi_host_grid_from_dense(int dim, int nno, int TotalDof, const int* index,
	const double* surplus, sgi_host_grid_t* out)
{
	clear_error();
	if (!out || dim <= 0 || nno < 0 || TotalDof <= 0 || (nno && (!index || !surplus)))
		return fail(SGI_E_INVALID, "bad grid arguments");
	sgi_host_grid* hg = new (std::nothrow) sgi_host_grid;
	if (!hg) return fail(SGI_E_NOMEM, "out of memory");
	hg->g.dim = dim; hg->g.nno = nno; hg->g.TotalDof = TotalDof;
	hg->g.index.assign(index, index + (size_t)nno * 2 * dim);
	hg->g.surplus.assign(surplus, surplus + (size_t)nno * TotalDof);
	*out = hg;
	return SGI_OK;
}

extern "C" int sgi_host_grid_view(sgi_host_grid_t hg, int* dim, int* nno, int* TotalDof,
	const int** index, const double** surplus)
{
	clear_error();
	if (!hg) return fail(SGI_E_INVALID, "null grid");
	if (dim) *dim = hg->g.dim;
	if (nno) *nno = hg->g.nno;
	if (TotalDof) *TotalDof = hg->g.TotalDof;
	if (index) *index = hg->g.index.data();
	if (surplus) *surplus = hg->g.surplus.data();
	return SGI_OK;
}

extern "C" void sgi_host_grid_free(sgi_host_grid_t hg) { delete hg; }

// ============================================================== generators
//
// Random numbers: xoshiro256** (Blackman & Vigna, 2018) seeded through
// splitmix64; doubles take the top 53 bits.

namespace {

struct Rng
{
	uint64_t s[4];
	explicit Rng(uint64_t seed)
	{
		for (int k = 0; k < 4; k++)
		{
			seed += 0x9e3779b97f4a7c15ull;
			uint64_t z = seed;
			z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
			z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
			s[k] = z ^ (z >> 31);
		}
	}
	static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
	uint64_t next()
	{
		uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
		s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
		s[2] ^= t; s[3] = rotl(s[3], 45);
		return r;
	}
	double uniform() { return (next() >> 11) * 0x1.0p-53; }
	uint64_t below(uint64_t n) { return (uint64_t)(uniform() * (double)n) % n; }
	double normal()
	{
		double u1 = uniform(), u2 = uniform();
		if (u1 < 1e-300) u1 = 1e-300;
		return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
	}
};

// A 1-D hierarchical component: level l >= 2 and hat (i, j) = (2^(l-1), j).
struct Comp { uint16_t dim; uint8_t l; uint16_t j; };

// Children of a 1-D component (level 1 has l = 1, j = 0).
int comp_children(int l, int j, int out_j[2])
{
	if (l == 1) { out_j[0] = 0; out_j[1] = 2; return 2; }
	if (l == 2) { out_j[0] = j == 0 ? 1 : 3; return 1; }
	out_j[0] = 2 * j - 1; out_j[1] = 2 * j + 1; return 2;
}

// Nodes as sorted component lists, stored flat, with exact-key hashing.
struct NodeStore
{
	std::vector<uint32_t> off{0};
	std::vector<Comp> comps;
	int size() const { return (int)off.size() - 1; }
	const Comp* begin(int n) const { return comps.data() + off[n]; }
	int count(int n) const { return (int)(off[n + 1] - off[n]); }
	uint64_t hash(int n) const
	{
		uint64_t h = 1469598103934665603ull;
		for (const Comp* c = begin(n), *e = c + count(n); c != e; c++)
		{
			uint64_t v = ((uint64_t)c->dim << 24) | ((uint64_t)c->l << 16) | c->j;
			h = (h ^ v) * 1099511628211ull;
			h ^= h >> 29;
		}
		return h;
	}
	bool equal(int a, int b) const
	{
		if (count(a) != count(b)) return false;
		const Comp* x = begin(a); const Comp* y = begin(b);
		for (int k = 0, e = count(a); k < e; k++)
			if (x[k].dim != y[k].dim || x[k].l != y[k].l || x[k].j != y[k].j) return false;
		return true;
	}
	void push(const std::vector<Comp>& c)
	{
		comps.insert(comps.end(), c.begin(), c.end());
		off.push_back((uint32_t)comps.size());
	}
	void pop() { comps.resize(off[off.size() - 2]); off.pop_back(); }
};

struct NodeHash { const NodeStore* s; size_t operator()(int n) const { return (size_t)s->hash(n); } };
struct NodeEq { const NodeStore* s; bool operator()(int a, int b) const { return s->equal(a, b); } };

// Emit nodes (in `order`) as a dense host grid with random surpluses.
int emit_grid(const NodeStore& st, const std::vector<int>& order, int dim, int TotalDof, uint64_t seed,
	sgi_host_grid_t* out)
{
	sgi_host_grid* hg = new (std::nothrow) sgi_host_grid;
	if (!hg) return fail(SGI_E_NOMEM, "out of memory");
	HostGrid& g = hg->g;
	g.dim = dim; g.nno = (int)order.size(); g.TotalDof = TotalDof;
	try
	{
		g.index.assign((size_t)g.nno * 2 * dim, 0);
		g.surplus.resize((size_t)g.nno * TotalDof);
	}
	catch (...) { delete hg; return fail(SGI_E_NOMEM, "out of memory"); }
	Rng rng(seed ^ 0x5eed5eed5eed5eedull);
	int maxdepth = 0;
	for (int r = 0; r < g.nno; r++)
	{
		int n = order[r], depth = 0;
		for (const Comp* c = st.begin(n), *e = c + st.count(n); c != e; c++)
		{
			g.index[(size_t)r * 2 * dim + c->dim] = 1 << (c->l - 1);
			g.index[(size_t)r * 2 * dim + dim + c->dim] = c->j;
			depth += c->l - 1;
		}
		maxdepth = std::max(maxdepth, depth);
		const double scale = ldexp(1.0, -2 * depth);
		for (int o = 0; o < TotalDof; o++)
			g.surplus[(size_t)r * TotalDof + o] = (2.0 * rng.uniform() - 1.0) * scale;
	}
	g.Level = maxdepth;
	*out = hg;
	return SGI_OK;
}

} // namespace

extern "C" int sgi_gen_regular(int dim, int level, int TotalDof, uint64_t seed, sgi_host_grid_t* out)
{
	clear_error();
	if (!out || dim <= 0 || dim > 65535 || level < 1 || level > 15 || TotalDof <= 0)
		return fail(SGI_E_INVALID, "bad regular-grid arguments");
	// Depth-first over the canonical tree: a node's children refine dimensions
	// d >= its last refined dimension, so every node is generated once.
	NodeStore st;
	std::vector<int> order;
	struct Frame { std::vector<Comp> c; int min_dim; int depth; };
	std::vector<Frame> stack;
	stack.push_back({ {}, 0, 0 });
	while (!stack.empty())
	{
		Frame f = std::move(stack.back());
		stack.pop_back();
		st.push(f.c);
		order.push_back(st.size() - 1);
		if ((size_t)order.size() > (size_t)2000000000) return fail(SGI_E_RANGE, "grid too large");
		if (f.depth >= level - 1) continue;
		std::vector<Frame> kids;
		for (int d = f.min_dim; d < dim; d++)
		{
			int l = 1, j = 0, pos = -1;
			for (size_t k = 0; k < f.c.size(); k++)
				if (f.c[k].dim == d) { l = f.c[k].l; j = f.c[k].j; pos = (int)k; }
			int cj[2];
			int nc = comp_children(l, j, cj);
			for (int q = 0; q < nc; q++)
			{
				Frame kf{ f.c, d, f.depth + 1 };
				Comp nc_{ (uint16_t)d, (uint8_t)(l + 1), (uint16_t)cj[q] };
				if (pos >= 0) kf.c[pos] = nc_;
				else kf.c.push_back(nc_);
				kids.push_back(std::move(kf));
			}
		}
		// push in reverse so children are emitted in (dim, j) order
		for (auto it = kids.rbegin(); it != kids.rend(); ++it) stack.push_back(std::move(*it));
	}
	return emit_grid(st, order, dim, TotalDof, seed, out);
}

extern "C" int sgi_gen_adaptive(int dim, int nno, int TotalDof, int max_level, double p_dim,
	uint64_t seed, sgi_host_grid_t* out)
{
	clear_error();
	if (!out || dim <= 0 || dim > 65535 || nno < 1 || TotalDof <= 0 || max_level < 2 || max_level > 15 ||
		!(p_dim > 0.0 && p_dim <= 1.0))
		return fail(SGI_E_INVALID, "bad adaptive-grid arguments");
	Rng rng(seed);
	NodeStore st;
	st.push({});
	std::unordered_set<int, NodeHash, NodeEq> present(1024, NodeHash{ &st }, NodeEq{ &st });
	present.reserve((size_t)nno * 2);
	present.insert(0);
	std::vector<std::vector<int>> kids(1);
	std::vector<int> leaves{ 0 };
	std::vector<int> chosen;
	std::vector<Comp> c;
	while (st.size() < nno)
	{
		if (leaves.empty()) return fail(SGI_E_RANGE, "no leaf left to refine at %d nodes", st.size());
		size_t k = rng.below(leaves.size());
		int n = leaves[k];
		leaves[k] = leaves.back();
		leaves.pop_back();
		chosen.clear();
		for (int d = 0; d < dim; d++)
			if (rng.uniform() < p_dim) chosen.push_back(d);
		if (chosen.empty()) chosen.push_back((int)rng.below(dim));
		for (int d : chosen)
		{
			const Comp* b = st.begin(n);
			const int cnt = st.count(n);
			int pos = -1, l = 1, j = 0;
			for (int q = 0; q < cnt; q++)
				if (b[q].dim == d) { pos = q; l = b[q].l; j = b[q].j; }
			if (l + 1 > max_level) continue;
			int cj[2];
			const int nc = comp_children(l, j, cj);
			for (int q = 0; q < nc && st.size() < nno; q++)
			{
				c.assign(st.begin(n), st.begin(n) + st.count(n));
				Comp nc_{ (uint16_t)d, (uint8_t)(l + 1), (uint16_t)cj[q] };
				if (pos >= 0) c[pos] = nc_;
				else
				{
					c.push_back(nc_);
					std::sort(c.begin(), c.end(), [](const Comp& a, const Comp& b2) { return a.dim < b2.dim; });
				}
				st.push(c);
				const int id = st.size() - 1;
				if (!present.insert(id).second) { st.pop(); continue; }
				kids[n].push_back(id);
				kids.emplace_back();
				leaves.push_back(id);
			}
			if (st.size() >= nno) break;
		}
	}
	// depth-first preorder of the refinement tree
	std::vector<int> order;
	order.reserve(st.size());
	std::vector<std::pair<int, int>> stack{ { 0, 0 } };
	order.push_back(0);
	while (!stack.empty())
	{
		auto& top = stack.back();
		if (top.second < (int)kids[top.first].size())
		{
			int ch = kids[top.first][top.second++];
			order.push_back(ch);
			stack.push_back({ ch, 0 });
		}
		else stack.pop_back();
	}
	return emit_grid(st, order, dim, TotalDof, seed, out);
}

extern "C" int sgi_gen_points(int dim, long npts, int kind, uint64_t seed, double kink_reject,
	int max_level, double* out)
{
	clear_error();
	if (dim <= 0 || npts < 0 || (npts && !out) || kind < 0 || kind > 2 || max_level < 1 || max_level > 30)
		return fail(SGI_E_INVALID, "bad point arguments");
	Rng rng(seed);
	const double cell = ldexp(1.0, -(max_level - 1));
	for (long p = 0; p < npts; p++)
	{
		const bool clustered = kind == 1 || (kind == 2 && p >= npts / 2);
		double* x = out + (size_t)p * dim;
		for (int attempt = 0;; attempt++)
		{
			bool ok = true;
			for (int d = 0; d < dim; d++)
			{
				double v = clustered ? 0.5 + 0.05 * rng.normal() : rng.uniform();
				v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
				x[d] = v;
				if (kink_reject > 0.0)
				{
					double r = v / cell;
					double dist = fabs(r - nearbyint(r)) * cell;
					if (dist < kink_reject) ok = false;
				}
			}
			if (ok) break;
			if (attempt > 1000000) return fail(SGI_E_RANGE, "kink rejection does not terminate");
		}
	}
	return SGI_OK;
}

// ============================================================ xps / chains
//
// The reference x86 loader's sparse form (LinearBasis/x86/src/Data.cpp:598-951),
// restated.  nfreqs is the most non-empty (i, j) pairs of any row.  For
// frequency f, the f-th non-empty pair of every row (in dimension order) is
// listed column by column (dimension-major, rows ascending); that listing's
// position renumbers the rows ("order"; rows without an f-th pair follow in row
// order).  Rows are first permuted by frequency 0's order.  xps ids are handed
// out in order of first appearance over (f, dimension, position), id 0 being
// the empty pair; chain[r][f] is the id of row r's f-th pair (0 if none).  The
// rows are then sorted by chain[.][0] with std::sort, and each run of equal
// chain[.][f-1] values (except the last run) by chain[.][f]; the surplus rows
// follow.  Pairs are kept as 8-bit i and j, as the reference stores them.

extern "C" int sgi_host_grid_xps_chains(sgi_host_grid_t hg, int* nfreqs_out, int* szxps_out,
	int* xps_out, int* chains_out, int* row_perm_out)
{
	clear_error();
	if (!hg) return fail(SGI_E_INVALID, "null grid");
	const HostGrid& g = hg->g;
	const int D = g.dim, nno = g.nno;
	// rows' non-empty pairs in dimension order
	std::vector<uint32_t> off(nno + 1, 0);
	std::vector<uint32_t> pdim;
	std::vector<uint8_t> pi, pj;
	int nfreqs = 0;
	for (int n = 0; n < nno; n++)
	{
		for (int k = 0; k < D; k++)
		{
			int i = g.index[(size_t)n * 2 * D + k], j = g.index[(size_t)n * 2 * D + D + k];
			if (!i && !j) continue;
			if (i < 0 || i > 255 || j < 0 || j > 255)
				return fail(SGI_E_RANGE, "node %d dim %d: (i, j) = (%d, %d) exceeds the 8-bit pairs of the x86 form",
					n, k, i, j);
			pdim.push_back(k); pi.push_back((uint8_t)i); pj.push_back((uint8_t)j);
		}
		off[n + 1] = (uint32_t)pdim.size();
		nfreqs = std::max(nfreqs, (int)(off[n + 1] - off[n]));
	}
	if (!nfreqs) return fail(SGI_E_FORMAT, "Index array cannot be of all zeros");
	if (D > 65535) return fail(SGI_E_RANGE, "dim %d exceeds the 16-bit xps dimension", D);

	// per frequency: column-major position of each row's f-th pair
	std::vector<std::vector<uint32_t>> trans(nfreqs, std::vector<uint32_t>(nno));
	std::vector<std::vector<uint32_t>> at(nfreqs); // at[f][order] = pair index
	std::vector<uint32_t> colcount(D);
	for (int f = 0; f < nfreqs; f++)
	{
		std::fill(colcount.begin(), colcount.end(), 0);
		for (int n = 0; n < nno; n++)
			if ((int)(off[n + 1] - off[n]) > f) colcount[pdim[off[n] + f]]++;
		std::vector<uint32_t> colstart(D + 1, 0);
		for (int k = 0; k < D; k++) colstart[k + 1] = colstart[k] + colcount[k];
		const uint32_t listed = colstart[D];
		at[f].assign(listed, 0);
		std::vector<uint32_t> fillpos(colstart.begin(), colstart.end() - 1);
		std::vector<char> seen(nno, 0);
		for (int n = 0; n < nno; n++)
			if ((int)(off[n + 1] - off[n]) > f)
			{
				uint32_t q = off[n] + f, pos = fillpos[pdim[q]]++;
				trans[f][n] = pos;
				at[f][pos] = q;
				seen[n] = 1;
			}
		uint32_t last = listed;
		for (int n = 0; n < nno; n++)
			if (!seen[n]) trans[f][n] = last++;
	}
	// xps ids by first appearance
	struct Key { uint32_t v; bool operator==(const Key& o) const { return v == o.v; } };
	struct KeyHash { size_t operator()(const Key& k) const { return k.v * 0x9e3779b1u; } };
	std::unordered_map<uint32_t, uint32_t> ids;
	std::vector<uint32_t> xps_key{ 0 };
	std::vector<std::vector<uint32_t>> temps(nfreqs);
	for (int f = 0; f < nfreqs; f++)
	{
		temps[f].assign(nno, 0);
		for (uint32_t pos = 0; pos < at[f].size(); pos++)
		{
			uint32_t q = at[f][pos];
			uint32_t key = ((uint32_t)pdim[q] << 16) | ((uint32_t)pi[q] << 8) | pj[q];
			auto it = ids.find(key);
			uint32_t id;
			if (it == ids.end()) { id = (uint32_t)xps_key.size(); ids.emplace(key, id); xps_key.push_back(key); }
			else id = it->second;
			temps[f][pos] = id;
		}
	}
	const int szxps = (int)xps_key.size();
	// rows after the first permutation: r1 = trans[0][n]
	std::vector<uint32_t> orig_of(nno);
	for (int n = 0; n < nno; n++) orig_of[trans[0][n]] = n;
	const int W = nfreqs + 1;
	std::vector<uint32_t> vv((size_t)nno * W);
	for (int r = 0; r < nno; r++)
	{
		const int n = orig_of[r];
		for (int f = 0; f < nfreqs; f++)
		{
			uint32_t t = f == 0 ? r : trans[f][n];
			vv[(size_t)r * W + f] = t < temps[f].size() ? temps[f][t] : 0;
		}
		vv[(size_t)r * W + nfreqs] = r;
	}
	// the reference's sort passes, on row indices
	std::vector<uint32_t> perm(nno);
	for (int r = 0; r < nno; r++) perm[r] = r;
	auto key = [&](uint32_t r, int f) { return vv[(size_t)r * W + f]; };
	std::sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return key(a, 0) < key(b, 0); });
	for (int f = 1; f < nfreqs; f++)
	{
		size_t i = 0;
		while (i < perm.size())
		{
			size_t ii = i + 1;
			for (; ii < perm.size(); ii++)
				if (key(perm[ii], f - 1) != key(perm[i], f - 1))
				{
					std::sort(perm.begin() + i, perm.begin() + ii,
						[&](uint32_t a, uint32_t b) { return key(a, f) < key(b, f); });
					break;
				}
			i = ii;
		}
	}
	for (int r = 0; r < nno; r++)
		for (int f = 0; f < nfreqs; f++)
			if (key(perm[r], f) > 65535)
				return fail(SGI_E_RANGE, "Chain index %u is out of the 16-bit chain range", key(perm[r], f));
	if (nfreqs_out) *nfreqs_out = nfreqs;
	if (szxps_out) *szxps_out = szxps;
	if (xps_out)
		for (int k = 0; k < szxps; k++)
		{
			xps_out[3 * k + 0] = (xps_key[k] >> 8) & 0xff;
			xps_out[3 * k + 1] = xps_key[k] & 0xff;
			xps_out[3 * k + 2] = xps_key[k] >> 16;
		}
	if (chains_out)
		for (int r = 0; r < nno; r++)
			for (int f = 0; f < nfreqs; f++)
				chains_out[(size_t)r * nfreqs + f] = (int)key(perm[r], f);
	if (row_perm_out)
		for (int r = 0; r < nno; r++)
			row_perm_out[r] = (int)orig_of[key(perm[r], nfreqs)];
	return SGI_OK;
}

// ============================================================ device layout

namespace sgi {

double coarse_threshold_for(const HostGrid& g)
{
	double m = 0.0;
	for (double v : g.surplus) m = std::max(m, fabs(v));
	static const double rel = []()
	{
		const char* e = getenv("SGI_COARSE_REL");
		return e ? atof(e) : 0x1.0p-16;
	}();
	return m * rel;
}

namespace {

// Open support ((j-1)/i, (j+1)/i) of hat (i, j), i > 0, contains that of (i2, j2).
inline bool interval_contains(int64_t i1, int64_t j1, int64_t i2, int64_t j2)
{
	return (j1 - 1) * i2 <= (j2 - 1) * i1 && (j2 + 1) * i1 <= (j1 + 1) * i2;
}

} // namespace

int build_layout(const HostGrid& g, DeviceLayout& L)
{
	const int D = g.dim, nno = g.nno, TD = g.TotalDof;
	L.rec.assign((size_t)4 * nno, 0);
	L.comps.clear();
	L.lo_index.assign(nno, ~0u);
	std::vector<uint32_t> cptr(nno + 1, 0);
	std::vector<char> dead(nno, 0);
	L.max_comps = 0;
	for (int n = 0; n < nno; n++)
	{
		int cnt = 0;
		for (int k = 0; k < D; k++)
		{
			const int i = g.index[(size_t)n * 2 * D + k], j = g.index[(size_t)n * 2 * D + D + k];
			if (!i && !j) continue;
			if (i < 0 || i > 65535 || j < 0 || j > 65535)
				return fail(SGI_E_RANGE, "node %d dim %d: (i, j) = (%d, %d) outside 0..65535", n, k, i, j);
			if (!i) dead[n] = 1; // 1 - |j| <= 0 everywhere
			L.comps.push_back((uint32_t)k);
			L.comps.push_back((uint32_t)i | ((uint32_t)j << 16));
			cnt++;
		}
		if (cnt > 255) return fail(SGI_E_RANGE, "node %d has %d non-constant dimensions (max 255)", n, cnt);
		L.max_comps = std::max(L.max_comps, cnt);
		cptr[n + 1] = (uint32_t)(L.comps.size() / 2);
	}
	if (D > 65535) return fail(SGI_E_RANGE, "dim %d exceeds 65535", D);
	const uint32_t* C = L.comps.data();
	auto contains = [&](int p, int n) -> bool
	{
		uint32_t a = cptr[p], ae = cptr[p + 1], b = cptr[n], be = cptr[n + 1];
		for (; a < ae; a++)
		{
			const uint32_t d = C[2 * a];
			while (b < be && C[2 * b] < d) b++;
			if (b == be || C[2 * b] != d) return false;
			const uint32_t pa = C[2 * a + 1], pb = C[2 * b + 1];
			if (!interval_contains(pa & 0xffff, pa >> 16, pb & 0xffff, pb >> 16)) return false;
		}
		return true;
	};
	// containment tree over the grid order: parent = deepest enclosing node
	// still open on the stack; a node's subtree ends where it is popped
	std::vector<int> stack, parent(nno, -1);
	std::vector<uint32_t> skip(nno, 0), depth(nno, 0);
	L.tree_depth = 0; L.tree_roots = 0; L.multi_delta = 0;
	for (int n = 0; n < nno; n++)
	{
		if (dead[n]) { skip[n] = n + 1; continue; }
		while (!stack.empty() && !contains(stack.back(), n)) { skip[stack.back()] = n; stack.pop_back(); }
		parent[n] = stack.empty() ? -1 : stack.back();
		if (parent[n] < 0) L.tree_roots++;
		stack.push_back(n);
		depth[n] = (uint32_t)stack.size();
		L.tree_depth = std::max(L.tree_depth, (int)stack.size());
	}
	for (int t : stack) skip[t] = nno;
	L.parent = parent;
	// coarse rows
	L.coarse_threshold = coarse_threshold_for(g);
	L.ncoarse = 0;
	for (int n = 0; n < nno; n++)
	{
		double m = 0.0;
		for (int o = 0; o < TD; o++) m = std::max(m, fabs(g.surplus[(size_t)n * TD + o]));
		if (m >= L.coarse_threshold && m > 0.0) L.lo_index[n] = (uint32_t)L.ncoarse++;
	}
	// records
	L.aux.assign((size_t)2 * nno, 0u);
	for (int n = 0; n < nno; n++)
	{
		const uint32_t cnt = cptr[n + 1] - cptr[n];
		uint32_t flags = 0, ddim = 0, dij = 0;
		if (dead[n]) flags |= NODE_DEAD;
		else
		{
			// delta components: those not identical to the parent's
			int ndelta = 0;
			uint32_t b = parent[n] >= 0 ? cptr[parent[n]] : 0, be = parent[n] >= 0 ? cptr[parent[n] + 1] : 0;
			for (uint32_t a = cptr[n]; a < cptr[n + 1]; a++)
			{
				while (b < be && C[2 * b] < C[2 * a]) b++;
				const bool same = b < be && C[2 * b] == C[2 * a] && C[2 * b + 1] == C[2 * a + 1];
				if (!same) { if (!ndelta) { ddim = C[2 * a]; dij = C[2 * a + 1]; } ndelta++; }
			}
			if (ndelta == 0) flags |= NODE_ALWAYS;
			else if (ndelta > 1) { flags |= NODE_MULTI; L.multi_delta++; }
		}
		if (L.lo_index[n] != ~0u) flags |= NODE_COARSE;
		// the parent's component in the delta dimension
		uint32_t old = 0;
		if (parent[n] >= 0 && !(flags & (NODE_DEAD | NODE_MULTI | NODE_ALWAYS)))
			for (uint32_t b2 = cptr[parent[n]]; b2 < cptr[parent[n] + 1]; b2++)
				if (C[2 * b2] == ddim) old = C[2 * b2 + 1];
		L.aux[2 * (size_t)n + 0] = old;
		L.aux[2 * (size_t)n + 1] = depth[n];
		L.rec[4 * (size_t)n + 0] = skip[n];
		L.rec[4 * (size_t)n + 1] = cptr[n];
		L.rec[4 * (size_t)n + 2] = cnt | flags | (ddim << 16);
		L.rec[4 * (size_t)n + 3] = dij;
	}
	return SGI_OK;
}

int build_descent(const HostGrid& g, const DeviceLayout& L, DescentLayout& D)
{
	const int nno = g.nno;
	// children of every node in index order; index nno collects the roots
	std::vector<uint32_t> kid_ptr(nno + 2, 0), kids;
	for (int n = 0; n < nno; n++)
	{
		if (L.rec[4 * (size_t)n + 2] & NODE_DEAD) continue;
		const int p = L.parent[n] < 0 ? nno : L.parent[n];
		kid_ptr[p + 1]++;
	}
	for (int p = 0; p <= nno; p++) kid_ptr[p + 1] += kid_ptr[p];
	kids.assign(kid_ptr[nno + 1], 0);
	{
		std::vector<uint32_t> fill(kid_ptr.begin(), kid_ptr.end() - 1);
		for (int n = 0; n < nno; n++)
		{
			if (L.rec[4 * (size_t)n + 2] & NODE_DEAD) continue;
			const int p = L.parent[n] < 0 ? nno : L.parent[n];
			kids[fill[p]++] = (uint32_t)n;
		}
	}
	D.a.clear(); D.b.clear(); D.cmin.clear(); D.cmax.clear();
	D.first.assign(nno + 1, 0);
	D.count.assign(nno + 1, 0);
	D.npairs = 0;
	struct Grp { uint32_t L, R, dk, old, ijL, ijR, lo, hi; };
	std::vector<Grp> grp;
	std::vector<std::pair<uint32_t, uint32_t>> simple;   // (delta dim, child)
	for (int p = 0; p <= nno; p++)
	{
		grp.clear();
		simple.clear();
		for (uint32_t a = kid_ptr[p]; a < kid_ptr[p + 1]; a++)
		{
			const uint32_t c = kids[a];
			const uint32_t z = L.rec[4 * (size_t)c + 2];
			if (z & NODE_MULTI) grp.push_back({ c, DESC_NONE, DESC_MULTI << 16, 0u, 0u, 0u, c, c });
			else if (z & NODE_ALWAYS) grp.push_back({ c, DESC_NONE, DESC_ALWAYS << 16, 0u, 0u, 0u, c, c });
			else simple.emplace_back(z >> 16, c);
		}
		// simple children by dimension: exactly two in a dimension with
		// disjoint supports there form a pair, every other one is a singleton
		std::sort(simple.begin(), simple.end());
		for (size_t s = 0; s < simple.size();)
		{
			size_t e = s + 1;
			while (e < simple.size() && simple[e].first == simple[s].first) e++;
			const uint32_t dd = simple[s].first;
			bool paired = false;
			if (e - s == 2)
			{
				const uint32_t c = simple[s].second, c2 = simple[s + 1].second;
				const uint32_t ij = L.rec[4 * (size_t)c + 3], ij2 = L.rec[4 * (size_t)c2 + 3];
				const uint32_t old = L.aux[2 * (size_t)c];
				const int64_t i1 = ij & 0xffff, j1 = ij >> 16, i2 = ij2 & 0xffff, j2 = ij2 >> 16;
				// open supports ((j-1)/i, (j+1)/i): the left one ends where or
				// before the right one starts
				const bool c_left = (j1 + 1) * i2 <= (j2 - 1) * i1;
				const bool c2_left = (j2 + 1) * i1 <= (j1 - 1) * i2;
				if ((c_left || c2_left) && L.aux[2 * (size_t)c2] == old)
				{
					grp.push_back({ c_left ? c : c2, c_left ? c2 : c, dd, old, c_left ? ij : ij2, c_left ? ij2 : ij,
					                std::min(c, c2), std::max(c, c2) });
					D.npairs++;
					paired = true;
				}
			}
			if (!paired)
				for (size_t k = s; k < e; k++)
				{
					const uint32_t c = simple[k].second;
					grp.push_back({ c, DESC_NONE, dd, L.aux[2 * (size_t)c], L.rec[4 * (size_t)c + 3], 0u, c, c });
				}
			s = e;
		}
		std::stable_sort(grp.begin(), grp.end(), [](const Grp& x, const Grp& y) { return x.lo < y.lo; });
		D.first[p] = (uint32_t)D.cmin.size();
		D.count[p] = (uint32_t)grp.size();
		for (const Grp& q : grp)
		{
			D.a.insert(D.a.end(), { q.L, q.R, q.dk, q.old });
			D.b.insert(D.b.end(), { q.ijL, q.ijR });
			D.cmin.push_back(q.lo);
			D.cmax.push_back(q.hi);
		}
	}
	return SGI_OK;
}

} // namespace sgi

extern "C" int sgi_host_grid_descent(sgi_host_grid_t hg, int* ngroups, int* npairs, uint32_t* a, uint32_t* b,
	uint32_t* first, uint32_t* count)
{
	clear_error();
	if (!hg || !ngroups) return fail(SGI_E_INVALID, "null argument");
	DeviceLayout L;
	int rc = build_layout(hg->g, L);
	if (rc) return rc;
	DescentLayout D;
	rc = build_descent(hg->g, L, D);
	if (rc) return rc;
	*ngroups = (int)D.cmin.size();
	if (npairs) *npairs = D.npairs;
	if (a) memcpy(a, D.a.data(), D.a.size() * 4);
	if (b) memcpy(b, D.b.data(), D.b.size() * 4);
	if (first) memcpy(first, D.first.data(), D.first.size() * 4);
	if (count) memcpy(count, D.count.data(), D.count.size() * 4);
	return SGI_OK;
}

extern "C" int sgi_host_grid_tree(sgi_host_grid_t hg, int* skip, int* parent)
{
	clear_error();
	if (!hg) return fail(SGI_E_INVALID, "null grid");
	DeviceLayout L;
	int rc = build_layout(hg->g, L);
	if (rc) return rc;
	for (int n = 0; n < hg->g.nno; n++)
	{
		if (skip) skip[n] = (int)L.rec[4 * (size_t)n];
		if (parent) parent[n] = L.parent[n];
	}
	return SGI_OK;
}
