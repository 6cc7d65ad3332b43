// Device layer of the B200 sparse-grid interpolator (sm_100a).
//
// Grid layout (built by sgi::build_layout): nodes in grid order, each with a
// 16-byte record {skip, comp_ptr, ncomp|flags|delta dim, delta (i, j)} and a
// CSR list of its non-constant components (dim, i, j) in dimension order.
// Every node's support lies inside its tree parent's support, and a node's
// subtree is the index range [n, skip[n]).
//
// Forward kernels: one warp per query point, points pulled from a device work
// counter.  Two walks find a point's active nodes.
//
// Window walk (FP64 form, hit counts, backward, FP32C fallback): the warp
// walks the nodes in windows of 32 consecutive indices:
//   * lane k checks node n0+k against the point with one hat evaluation (the
//     component in which it differs from its parent);
//   * an inclusive max-scan of the skip pointers of failing nodes marks every
//     node inside a failing node's subtree as pruned;
//   * surviving nodes ("hits") get their weight, the product of all their
//     hats in dimension order, from their own lane;
//   * hits are accumulated in index order: all lanes read the node's surplus
//     row (coalesced) and update the TotalDof accumulators they own;
//   * the next window starts after the window or after the largest pruned
//     subtree, whichever is further.
// With nodes in file order, the FP64 form performs the reference gold kernel's
// operations in its order (LinearBasis/gold/src/InterpolateArray.cpp:26-41):
// the same multiplies for the weight and the same multiply-then-add sequence per
// output, so its results are bit-identical to gold's.
//
// Descent walk (FP32C form, fwd_f32d_kernel): the warp keeps a stack of child
// groups of active nodes (left/right child pairs per dimension, see
// sgi::build_descent) and evaluates one group per lane, 32 per step; a hit's
// weight is its parent's times its hat over the parent's hat in that
// dimension, and terms are split by size into FP64 rows (big), FP32 rows
// (fine) and dropped ones (negligible).
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "sgi_internal.h"

using namespace sgi;

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MAXG = 48;       // grids per launch (kernel parameter space)
constexpr int BLOCK = 256;     // threads per block: 8 warps
constexpr int WARPS = BLOCK / 32;
constexpr int PASS = 256;      // outputs per launch pass (TotalDof > 256: several passes)

struct GridDesc
{
	const uint4* rec;
	const uint2* comps;
	const double* s64;
	const float* s32;
	const double* s64c;          // FP64 copies of the coarse rows (FP32C form)
	const uint32_t* coarse_index; // row of node n in s64c, for coarse nodes
	const int* parent;           // tree parent per node (-1 for roots)
	const float* rowmax;         // largest |surplus| of each row (FP32C), or null
	const uint2* aux;            // {parent's component in the delta dim, depth}: FP32C weights
	const uint4* grp_a;          // descent child groups (FP32C): {L, R, d | kind << 16, parent's ij in d}
	const uint2* grp_b;          //   {L's ij in d, R's}
	const uint4* ninfo;          //   per node: {first group, group count, rowmax bits, FP64 copy row or NONE}
	const uint4* s16;            // FP16 rows (FP32C), per 256 outputs in lane order; see build_image
	int depth;                   // containment-tree depth (bounds the descent stack)
	float skip_below;            // FP32C drops fine terms with |w| * rowmax below this
	float big_below;             // FP32C: terms with |w| * rowmax from this up are big (FP64 rows)
	float f16_below;             // FP32C: fine terms with |w| * rowmax below this read the FP16 rows (0: none)
	long long pt_begin;
	int nno;
	int ld;
};

// Nodes of a chunk boundary's ancestor chain kept per grid (depths 1..CHAIN).
constexpr int CHAIN = 31;

struct FwdArgs
{
	GridDesc g[MAXG];
	// ancestor chain of the chunk start per grid: chain[k][d - 1] is the node
	// at depth d whose subtree contains the chunk start, d = 1..chain_len[k]
	uint32_t chain[MAXG][CHAIN];
	int chain_len[MAXG];
	// descent starts of this launch per grid: the child groups of the chain
	// node at depth d that may hold nodes of the chunk (cseg[k][d - 1]), and
	// the tree roots' groups that may (rseg[k]); {first, end}
	uint2 cseg[MAXG][CHAIN];
	uint2 rseg[MAXG];
	const double* x;
	double* out;
	unsigned long long* counter;
	long long npts;
	int ngrids, dim, TD, o_begin;
	// node range of this launch: [chunk_begin, chunk_begin + chunk_len) of
	// every grid; chunk_len 0 means the whole grid
	int chunk_begin, chunk_len;
};

// kernel parameters are limited to 32,764 bytes
static_assert(sizeof(FwdArgs) <= 32764, "FwdArgs exceeds the kernel parameter limit");

// Exact conversion of v < 2^32 to double in the FP64 pipe: the bit pattern
// 0x43300000:v is 2^52 + v, and subtracting 2^52 is exact.
__device__ __forceinline__ double u32_to_double(uint32_t v)
{
	return __dsub_rn(__hiloint2double(0x43300000, (int)v), 4503599627370496.0);
}

__device__ __forceinline__ double hat(double x, uint32_t ij)
{
	// 1 - |x*i - j| with the gold macro's rounding (LinearBasis/include/LinearBasis.h:50);
	// i and j convert exactly, so the result is the same as with (double)i, (double)j
	return __dsub_rn(1.0, fabs(__dsub_rn(__dmul_rn(x, u32_to_double(ij & 0xffffu)), u32_to_double(ij >> 16))));
}

// 1/h for h in (0, 1], to about 2^-44 relative: the approximate FP64
// reciprocal refined by one Newton-Raphson step, r' = r + r(1 - h r).
__device__ __forceinline__ double rcp_weight(double h)
{
	double r;
	asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(h));
	const double e = fma(-h, r, 1.0);
	return fma(r, e, r);
}

__device__ __forceinline__ int find_grid(const FwdArgs& a, long long p)
{
	int gi = 0;
	while (gi + 1 < a.ngrids && a.g[gi + 1].pt_begin <= p) gi++;
	return gi;
}

// Product of a hit node's hats in dimension order (the gold loop's `temp`).
// Components are fetched four at a time, so a node costs one memory round
// trip per four components instead of one per component.
__device__ __forceinline__ double node_weight(const GridDesc& G, const double* xs, uint32_t cptr, uint32_t ncomp)
{
	double w = 1.0;
	for (uint32_t c0 = 0; c0 < ncomp; c0 += 4)
	{
		uint2 cp[4];
#pragma unroll
		for (int q = 0; q < 4; q++)
			cp[q] = c0 + q < ncomp ? __ldg(G.comps + cptr + c0 + q) : make_uint2(0u, 0u);
#pragma unroll
		for (int q = 0; q < 4; q++)
			if (c0 + q < ncomp) w = __dmul_rn(w, hat(xs[cp[q].x], cp[q].y));
	}
	return w;
}

// True when every hat of the node is positive at x (a product test would
// accept an even number of negative hats).
__device__ __forceinline__ bool node_active(const GridDesc& G, const double* xs, uint32_t cptr, uint32_t ncomp)
{
	bool act = true;
	for (uint32_t c0 = 0; c0 < ncomp && act; c0 += 4)
	{
		uint2 cp[4];
#pragma unroll
		for (int q = 0; q < 4; q++)
			cp[q] = c0 + q < ncomp ? __ldg(G.comps + cptr + c0 + q) : make_uint2(0u, 0u);
#pragma unroll
		for (int q = 0; q < 4; q++)
			if (c0 + q < ncomp) act = act && hat(xs[cp[q].x], cp[q].y) > 0.0;
	}
	return act;
}

// Depth of the per-warp weight stack of the incremental form.
constexpr int WPATH = 64;

// Walks nodes [a, b) of one grid for the point whose coordinates are in xs
// (shared memory).  Calls on_hits(mask, n0, w, rec, rowmax) per window; bits
// of mask are hit lanes, lane k's w is the weight of node n0+k, rec its record
// and rowmax its row's largest |surplus| (when the grid descriptor has them).
// A failing lane marks the lanes inside its subtree with a bit mask, and one
// warp OR reduction gives every lane whether an earlier failing node covers
// it; the next window starts at the larger of n0+32 and the largest failing
// skip (one warp max reduction).
// Inside the range a node is reached only when all its ancestors in the range
// are active.  A node whose tree parent lies before `a` ("chunk root") has its
// parent in the chunk start's ancestor chain: bit d of pathmask tells whether
// the chain node at depth d is active (bit 0 stands for the roots' parent),
// and the chunk root is then decided by its delta hat like any other node.
// Chunk roots whose parent is deeper than the chain's clen stored levels are
// checked on all their components.
// Without INCR every hit takes the full product (the FP64 form: gold's
// multiplies in gold's order).
// INCR (FP32C): a hit's weight is its tree parent's weight times its delta
// hat over the parent's hat in that dimension (1 when the parent is constant
// there).  A hit whose parent precedes the window reads the parent's weight
// from wpath[depth - 1], the weight of the last hit one level up, which in
// depth-first order is the parent; hits whose parent is in the same window
// take it from that lane; wpath[0] = 1 stands for the roots' parent.  Chunk
// roots, nodes differing from their parent in several dimensions and nodes
// deeper than the stack take the full product.
template <bool INCR, class OnHits>
__device__ __forceinline__ void traverse(const GridDesc& G, const double* xs, int lane, int a, int b,
	OnHits&& on_hits, double* wpath = nullptr, unsigned pathmask = 1u, int clen = 0)
{
	int n0 = a;
	if (INCR)
	{
		if (lane == 0) wpath[0] = 1.0;
		__syncwarp();
	}
	// the next window's records are fetched before this window's hits are
	// accumulated, so that their latency overlaps the row gathers
	uint4 rn = make_uint4(0u, 0u, 0u, 0u);
	uint2 xn = make_uint2(0u, 0u);
	int pn = -1;
	float mn = 0.f;
	if (n0 + lane < b)
	{
		rn = __ldg(G.rec + n0 + lane);
		if (INCR || a > 0) pn = __ldg(G.parent + n0 + lane);
		if (G.rowmax) mn = __ldg(G.rowmax + n0 + lane);
		if (INCR || a > 0) xn = __ldg(G.aux + n0 + lane);
	}
	while (n0 < b)
	{
		const int idx = n0 + lane;
		const bool valid = idx < b;
		const uint4 r = rn;
		const uint2 ax = xn;
		const float rm = mn;
		const uint32_t ncomp = r.z & 0xffu;
		const bool chunk_root = a > 0 && valid && pn < a;
		bool act = false, full = false;
		double factor = 1.0;
		if (valid)
		{
			// depth of a chunk root's parent: ax.y - 1 (0 for tree roots)
			const bool croot_full = chunk_root && (ax.y == 0u || (int)ax.y - 1 > clen);
			if (r.z & NODE_DEAD) act = false;
			else if ((r.z & NODE_MULTI) || croot_full) { act = node_active(G, xs, r.y, ncomp); full = true; }
			else if (chunk_root && !((pathmask >> (ax.y - 1u)) & 1u)) act = false;
			else if (r.z & NODE_ALWAYS) act = true;
			else
			{
				const double xd = xs[r.z >> 16];
				const double hd = hat(xd, r.w);
				act = hd > 0.0;
				if (INCR && act) factor = ax.x ? hd * rcp_weight(hat(xd, ax.x)) : hd;
			}
			if (INCR && ax.y >= (uint32_t)WPATH) full = true;
		}
		// lanes lane+1 .. skip-n0-1 lie in a failing node's subtree
		const unsigned cover = (valid && !act) ? r.x : 0u;
		unsigned bits = 0u;
		if (cover)
		{
			const int e = min((int)cover - n0, 32);
			bits = (e >= 32 ? FULL : ((1u << e) - 1u)) & ~((2u << lane) - 1u);
		}
		const unsigned pruned = __reduce_or_sync(FULL, bits);
		const bool hit = act && !((pruned >> lane) & 1u);
		const unsigned mask = __ballot_sync(FULL, hit);
		const int nnext = max(n0 + 32, (int)__reduce_max_sync(FULL, cover));
		const int pcur = pn;
		rn = make_uint4(0u, 0u, 0u, 0u);
		pn = -1;
		if (nnext + lane < b)
		{
			rn = __ldg(G.rec + nnext + lane);
			if (INCR || a > 0) pn = __ldg(G.parent + nnext + lane);
			if (G.rowmax) mn = __ldg(G.rowmax + nnext + lane);
			if (INCR || a > 0) xn = __ldg(G.aux + nnext + lane);
		}
		double w = 0.0;
		if (!INCR) w = hit ? node_weight(G, xs, r.y, ncomp) : 0.0;
		else if (mask)
		{
			// hits whose parent precedes the window take its weight from the
			// stack; chains of hits inside the window resolve in shuffle rounds
			if (hit) w = full ? node_weight(G, xs, r.y, ncomp)
			               : (pcur < n0 ? wpath[ax.y - 1] * factor : 0.0);
			const int plane = pcur - n0;                 // parent's lane, if in the window
			bool done = !hit || full || pcur < n0;
			for (int round = 0; round < 32 && __any_sync(FULL, !done); round++)
			{
				const double wp = __shfl_sync(FULL, w, plane >= 0 && plane < 32 ? plane : lane);
				const bool pdone = __shfl_sync(FULL, (int)done, plane >= 0 && plane < 32 ? plane : lane);
				if (!done && pdone) { w = wp * factor; done = true; }
			}
			// the deepest-indexed hit at each depth becomes that depth's entry
			__syncwarp();
			const unsigned same = __match_any_sync(FULL, hit ? ax.y : 0xffffffffu);
			if (hit && ax.y < (uint32_t)WPATH && (31 - __clz(same & mask)) == lane) wpath[ax.y] = w;
			__syncwarp();
		}
		if (mask) on_hits(mask, n0, w, r, rm);
		n0 = nnext;
	}
}

template <class OnHits>
__device__ __forceinline__ void traverse(const GridDesc& G, const double* xs, int lane, OnHits&& on_hits)
{
	traverse<false>(G, xs, lane, 0, G.nno, on_hits);
}

// Activity (bit d of the result; bit 0 set) and, when wpath is given, weight
// (wpath[d]; 0 when inactive) of the chunk start's ancestor chain for the
// point in xs.  Lane d takes the chain node at depth d, whose parent is the
// node at depth d - 1: as in the walk, it is active when its parent is and
// its delta hat is positive, and its weight is the parent's times the delta
// hat over the parent's hat in that dimension (a prefix AND over a ballot and
// a segmented prefix product over the lanes; nodes differing from their
// parent in several dimensions are evaluated on all components and start a
// new segment).  A chunk root's parent is one of these nodes.  Every node
// before the end of the shallowest inactive chain node's subtree is
// inactive, so *start moves there.
// chain_node(d) gives the chain node at depth d + 1, d = 0..len-1.
template <class ChainNode>
__device__ __forceinline__ unsigned chain_state_of(ChainNode&& chain_node, int len, const GridDesc& G,
	const double* xs, int lane, double* wpath, int* start)
{
	if (len == 0) return 1u;
	const bool mine = lane >= 1 && lane <= len;
	bool local = true, multi = false;
	double f = 1.0;
	uint32_t skip = 0u;
	if (mine)
	{
		const uint32_t node = chain_node(lane - 1);
		const uint4 r = __ldg(G.rec + node);
		skip = r.x;
		if (r.z & NODE_MULTI)
		{
			multi = true;
			local = node_active(G, xs, r.y, r.z & 0xffu);
			if (wpath && local) f = node_weight(G, xs, r.y, r.z & 0xffu);
		}
		else if (!(r.z & NODE_ALWAYS))
		{
			const double xd = xs[r.z >> 16];
			const double hd = hat(xd, r.w);
			local = hd > 0.0;
			if (wpath && local)
			{
				const uint32_t old = __ldg(G.aux + node).x;
				f = old ? hd * rcp_weight(hat(xd, old)) : hd;
			}
		}
	}
	// active: every chain node shallower than the first local failure
	const unsigned fails = __ballot_sync(FULL, mine && !local);
	const unsigned upto = fails ? (1u << (__ffs(fails) - 1)) - 1u : FULL;
	const unsigned m = (upto & ((2u << len) - 1u)) | 1u;
	if (wpath)
	{
		double w = mine ? f : 1.0;
		bool seg = multi || lane == 0;
#pragma unroll
		for (int off = 1; off < 32; off <<= 1)
		{
			const double wu = __shfl_up_sync(FULL, w, off);
			const bool su = __shfl_up_sync(FULL, (int)seg, off);
			if (lane >= off && !seg) { w *= wu; seg = su; }
		}
		if (mine) wpath[lane] = ((m >> lane) & 1u) ? w : 0.0;
	}
	const unsigned inactive = ~m & ((2u << len) - 2u);   // depths 1..len
	const uint32_t end = __shfl_sync(FULL, skip, inactive ? __ffs(inactive) - 1 : 0);
	if (inactive) *start = max(*start, (int)end);
	return m;
}

// The chain of this launch's chunk start (kernel parameters) for grid gi.
__device__ __forceinline__ unsigned chain_state(const FwdArgs& a, int gi, const GridDesc& G, const double* xs,
	int lane, double* wpath, int* start)
{
	return chain_state_of([&](int d) { return a.chain[gi][d]; }, a.chain_len[gi], G, xs, lane, wpath, start);
}

// Node range of this launch for grid G.
__device__ __forceinline__ void chunk_of(const FwdArgs& a, const GridDesc& G, int* lo, int* hi)
{
	*lo = a.chunk_begin;
	*hi = a.chunk_len ? (int)min((long long)G.nno, (long long)a.chunk_begin + a.chunk_len) : G.nno;
}

// Loads point p into the warp's shared slot; returns false (after writing NaN
// outputs, as the gold kernel produces for a non-finite coordinate) if any
// coordinate is not finite.
__device__ __forceinline__ bool load_point(const FwdArgs& a, long long p, double* xs, int lane)
{
	bool finite = true;
	for (int k = lane; k < a.dim; k += 32)
	{
		const double v = a.x[(size_t)p * a.dim + k];
		xs[k] = v;
		finite &= isfinite(v);
	}
	__syncwarp();
	return __all_sync(FULL, finite);
}

// Output ownership: with E = 2, lane l owns outputs 64v + 2l + {0, 1} of the
// pass (v < V), so every row read is one coalesced 16-byte (FP64) or 8-byte
// (FP32) load per lane; with E = 1 (TotalDof <= 32) lane l owns output l.
template <int E>
__device__ __forceinline__ int out_col(int v, int lane) { return v * 32 * E + lane * E; }

template <int E>
__device__ __forceinline__ void load_row(const double* row, int o, bool in, double* d)
{
	if (E == 4)
	{
		const double2 t0 = in ? __ldg(reinterpret_cast<const double2*>(row + o)) : make_double2(0.0, 0.0);
		const double2 t1 = in ? __ldg(reinterpret_cast<const double2*>(row + o + 2)) : make_double2(0.0, 0.0);
		d[0] = t0.x; d[1] = t0.y; d[2] = t1.x; d[3] = t1.y;
	}
	else if (E == 2)
	{
		const double2 t = in ? __ldg(reinterpret_cast<const double2*>(row + o)) : make_double2(0.0, 0.0);
		d[0] = t.x; d[1] = t.y;
	}
	else d[0] = in ? __ldg(row + o) : 0.0;
}

template <int E>
__device__ __forceinline__ void load_row(const float* row, int o, bool in, float* d)
{
	if (E == 4)
	{
		const float4 t = in ? __ldg(reinterpret_cast<const float4*>(row + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
		d[0] = t.x; d[1] = t.y; d[2] = t.z; d[3] = t.w;
	}
	else if (E == 2)
	{
		const float2 t = in ? __ldg(reinterpret_cast<const float2*>(row + o)) : make_float2(0.f, 0.f);
		d[0] = t.x; d[1] = t.y;
	}
	else d[0] = in ? __ldg(row + o) : 0.f;
}

// QH: rows in flight per warp.  A window's hits are taken QH at a time in
// index order: their rows are all loaded before the first is added, and the
// adds follow the gold order.  Two rows suit large batches (registers buy
// warps); small batches, whose few warps wait on each row, use more.
template <int V, int E, int QH = 2>
__global__ void __launch_bounds__(BLOCK) fwd_f64_kernel(const __grid_constant__ FwdArgs a)
{
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	double* xs = smem + (threadIdx.x >> 5) * a.dim;
	const bool first = a.chunk_begin == 0;
	for (;;)
	{
		long long p = 0;
		if (lane == 0) p = (long long)atomicAdd(a.counter, 1ull);
		p = __shfl_sync(FULL, p, 0);
		if (p >= a.npts) break;
		const int gi = find_grid(a, p);
		const GridDesc& G = a.g[gi];
		int lo, hi;
		chunk_of(a, G, &lo, &hi);
		if (!first && lo >= hi) continue;   // this grid has no nodes in the chunk
		const bool ok = load_point(a, p, xs, lane);
		if (!ok && !first) continue;        // NaN already written by the first chunk
		unsigned pathmask = 1u;
		if (!first)
		{
			pathmask = chain_state(a, gi, G, xs, lane, nullptr, &lo);
			if (lo >= hi) continue;         // no active node in the chunk: outputs unchanged
		}
		double* dst = a.out + (size_t)p * a.TD + a.o_begin;
		// the running sums continue from the previous chunk, so the adds keep
		// the gold loop's order across chunks
		double acc[V][E];
#pragma unroll
		for (int v = 0; v < V; v++)
#pragma unroll
			for (int e = 0; e < E; e++)
			{
				const int o = out_col<E>(v, lane) + e;
				acc[v][e] = (!first && a.o_begin + o < a.TD) ? __ldcs(dst + o) : 0.0;
			}
		if (ok)
		{
			traverse<false>(G, xs, lane, lo, hi, [&](unsigned mask, int n0, double w, const uint4&, float)
			{
				// QH hits per step, all their rows loaded before any is added, so
				// that each warp keeps QH rows in flight; the adds stay in order
				while (mask)
				{
					int kq[QH];
#pragma unroll
					for (int q = 0; q < QH; q++)
					{
						kq[q] = mask ? __ffs(mask) - 1 : -1;
						if (mask) mask &= mask - 1;
					}
					double sq[QH][V][E];
#pragma unroll
					for (int q = 0; q < QH; q++)
					{
						const double* row = G.s64 + (size_t)(n0 + (kq[q] >= 0 ? kq[q] : kq[0])) * G.ld + a.o_begin;
#pragma unroll
						for (int v = 0; v < V; v++)
						{
							const int o = out_col<E>(v, lane);
							load_row<E>(row, o, kq[q] >= 0 && a.o_begin + o < G.ld, sq[q][v]);
						}
					}
#pragma unroll
					for (int q = 0; q < QH; q++)
					{
						if (kq[q] < 0) break;   // warp-uniform
						const double wq = __shfl_sync(FULL, w, kq[q]);
#pragma unroll
						for (int v = 0; v < V; v++)
#pragma unroll
							for (int e = 0; e < E; e++) acc[v][e] = __dadd_rn(acc[v][e], __dmul_rn(wq, sq[q][v][e]));
					}
				}
			}, nullptr, pathmask, a.chain_len[gi]);
		}
#pragma unroll
		for (int v = 0; v < V; v++)
#pragma unroll
			for (int e = 0; e < E; e++)
			{
				const int o = out_col<E>(v, lane) + e;
				if (a.o_begin + o < a.TD)
					__stcs(dst + o, ok ? acc[v][e] : (G.nno ? __longlong_as_double(0x7ff8000000000000ll) : 0.0));
			}
		__syncwarp();
	}
}

// Per-warp list of fine terms, {row, FP32 weight}: a window's fine hits are
// appended, and the list is drained once it holds 32 or more.
constexpr int FCAP = 64;

// Shared memory per warp of the list form, in doubles: the list, the weight
// stack and the point (rounded up to keep the next warp 16-byte aligned).
__host__ __device__ __forceinline__ int list_stride(int dim) { return FCAP + WPATH + ((dim + 1) & ~1); }

// FP32 + compensated form.  Terms are split by size: a term is "big" when
// |w| * max|s_row| is at least the coarse threshold (2^-16 of the largest
// surplus by default); big terms read the FP64 copy of their row (rows whose
// largest |surplus| reaches the threshold have one) and add with an FP64 FMA.
// The other ("fine") terms, each below the threshold, are appended to a
// per-warp list of {row, FP32 weight} entries and gathered in FP32 in groups
// of Q rows; their FP32 partial sums are added to the outputs' FP64 running
// sums every FLUSH terms.  Fine terms below 2^-42 of the largest surplus are
// dropped before their row is read; in the descent form, fine terms below
// 2^-29 of it read FP16 copies of their rows (see halves_to_float).  The
// running sums also carry the outputs across node chunks.
constexpr int FLUSH = 8;

template <int V, int E, int Q, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) fwd_f32c_kernel(const __grid_constant__ FwdArgs a)
{
	static_assert(FLUSH % Q == 0 || Q % FLUSH == 0, "groups of Q must tile the flush interval");
	static_assert(32 % Q == 0, "groups of Q must tile a window");
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	double* wbase = smem + (threadIdx.x >> 5) * list_stride(a.dim);
	uint2* fl = reinterpret_cast<uint2*>(wbase);
	double* wpath = wbase + FCAP;
	double* xs = wpath + WPATH;
	const bool first = a.chunk_begin == 0;
	for (;;)
	{
		long long p = 0;
		if (lane == 0) p = (long long)atomicAdd(a.counter, 1ull);
		p = __shfl_sync(FULL, p, 0);
		if (p >= a.npts) break;
		const int gi = find_grid(a, p);
		const GridDesc& G = a.g[gi];
		int lo_n, hi_n;
		chunk_of(a, G, &lo_n, &hi_n);
		if (!first && lo_n >= hi_n) continue;   // this grid has no nodes in the chunk
		const bool ok = load_point(a, p, xs, lane);
		if (!ok && !first) continue;            // NaN already written by the first chunk
		unsigned pathmask = 1u;
		if (!first)
		{
			pathmask = chain_state(a, gi, G, xs, lane, wpath, &lo_n);
			if (lo_n >= hi_n) continue;         // no active node in the chunk: outputs unchanged
		}
		double* dst = a.out + (size_t)p * a.TD + a.o_begin;
		double acc[V][E];
#pragma unroll
		for (int v = 0; v < V; v++)
#pragma unroll
			for (int e = 0; e < E; e++)
			{
				const int o = out_col<E>(v, lane) + e;
				acc[v][e] = (!first && a.o_begin + o < a.TD) ? __ldcs(dst + o) : 0.0;
			}
		if (ok)
		{
			const int lcol = a.o_begin + out_col<E>(0, lane);
			const float* s32l = G.s32 + lcol;
			const double* s64l = G.s64c + lcol;
			const uint32_t ld = (uint32_t)G.ld;
			float part[V][E];
#pragma unroll
			for (int v = 0; v < V; v++)
#pragma unroll
				for (int e = 0; e < E; e++) part[v][e] = 0.f;
			int cnt = 0, since = 0;
			auto flush = [&]()
			{
#pragma unroll
				for (int v = 0; v < V; v++)
#pragma unroll
					for (int e = 0; e < E; e++) { acc[v][e] = __dadd_rn(acc[v][e], (double)part[v][e]); part[v][e] = 0.f; }
			};
			// entries [h, hend) of the list, hend - h a multiple of Q
			auto groups = [&](int h, int hend)
			{
				for (; h < hend; h += Q)
				{
					uint2 en[Q];
#pragma unroll
					for (int q = 0; q < Q; q += 2)
					{
						if (q + 1 < Q)
						{
							const uint4 t = *reinterpret_cast<const uint4*>(fl + h + q);
							en[q] = make_uint2(t.x, t.y);
							en[q + 1] = make_uint2(t.z, t.w);
						}
						else en[q] = fl[h + q];
					}
					float sv[Q][V][E];
#pragma unroll
					for (int q = 0; q < Q; q++)
					{
						const float* row = s32l + (size_t)en[q].x * ld;
#pragma unroll
						for (int v = 0; v < V; v++) load_row<E>(row, v * 32 * E, lcol + v * 32 * E < G.ld, sv[q][v]);
					}
#pragma unroll
					for (int v = 0; v < V; v++)
#pragma unroll
						for (int e = 0; e < E; e++)
#pragma unroll
							for (int q = 0; q < Q; q++)
								part[v][e] = __fmaf_rn(__uint_as_float(en[q].y), sv[q][v][e], part[v][e]);
					since += Q;
					if (since >= FLUSH) { flush(); since = 0; }
				}
			};
			traverse<true>(G, xs, lane, lo_n, hi_n, [&](unsigned mask, int n0, double w, const uint4& rec, float rm)
			{
				const bool mine = (mask >> lane) & 1u;
				const float wf = __double2float_rn(w);
				const float bound = fabsf(wf) * rm;
				const bool big = mine && (rec.z & NODE_COARSE) && bound >= G.big_below;
				const bool fine = mine && !big && bound >= G.skip_below;
				unsigned cm = __ballot_sync(FULL, big);
				const unsigned fm = __ballot_sync(FULL, fine);
				if (fine) fl[cnt + __popc(fm & ((1u << lane) - 1u))] = make_uint2((uint32_t)(n0 + lane), __float_as_uint(wf));
				cnt += __popc(fm);
				if (cm)
				{
					const uint32_t ci = big ? __ldg(G.coarse_index + n0 + lane) : 0u;
					// big terms two at a time (two FP64 rows in flight)
					while (cm)
					{
						const int k0 = __ffs(cm) - 1;
						cm &= cm - 1;
						const bool two = cm != 0u;
						const int k1 = two ? __ffs(cm) - 1 : k0;
						if (two) cm &= cm - 1;
						const double w0 = __shfl_sync(FULL, w, k0);
						const double w1 = __shfl_sync(FULL, w, k1);
						const double* row0 = s64l + (size_t)__shfl_sync(FULL, ci, k0) * ld;
						const double* row1 = s64l + (size_t)__shfl_sync(FULL, ci, k1) * ld;
						double s0[V][E], s1[V][E];
#pragma unroll
						for (int v = 0; v < V; v++)
						{
							const bool in = lcol + v * 32 * E < G.ld;
							load_row<E>(row0, v * 32 * E, in, s0[v]);
							load_row<E>(row1, v * 32 * E, in && two, s1[v]);
						}
#pragma unroll
						for (int v = 0; v < V; v++)
#pragma unroll
							for (int e = 0; e < E; e++)
							{
								acc[v][e] = fma(w0, s0[v][e], acc[v][e]);
								if (two) acc[v][e] = fma(w1, s1[v][e], acc[v][e]);
							}
					}
				}
				if (cnt >= 32)
				{
					// all whole groups; the remainder (< Q entries) moves to the front
					__syncwarp();
					const int whole = cnt - cnt % Q;
					groups(0, whole);
					const int rem = cnt - whole;
					uint2 t = make_uint2(0u, 0u);
					if (lane < rem) t = fl[whole + lane];
					__syncwarp();
					if (lane < rem) fl[lane] = t;
					__syncwarp();
					cnt = rem;
				}
			}, wpath, pathmask, a.chain_len[gi]);
			if (cnt)
			{
				// pad to whole groups with weight-0 copies of the first entry
				const int padded = (cnt + Q - 1) / Q * Q;
				__syncwarp();
				const uint32_t r0 = fl[0].x;
				if (lane >= cnt && lane < padded) fl[lane] = make_uint2(r0, 0u);
				__syncwarp();
				groups(0, padded);
			}
			flush();
		}
#pragma unroll
		for (int v = 0; v < V; v++)
#pragma unroll
			for (int e = 0; e < E; e++)
			{
				const int o = out_col<E>(v, lane) + e;
				if (a.o_begin + o < a.TD)
					__stcs(dst + o, ok ? acc[v][e] : (G.nno ? __longlong_as_double(0x7ff8000000000000ll) : 0.0));
			}
		__syncwarp();
	}
}

// ------------------------------------------------------------ descent walk
//
// FP32C form over the descent layout: instead of scanning node windows, the
// warp keeps a stack (shared memory) of pending child-group ranges, each with
// its parent's weight, and evaluates up to 32 groups per step, one per lane.
// A pair group holds the left and right child of its parent in one
// dimension (disjoint supports): the lane tests the left child's hat and, if
// it is zero, the right one's, so at most one child per group is a hit and
// nearly every lane evaluation finds one.  A hit's weight is its parent's
// weight times its hat over the parent's hat in that dimension; a hit with
// children in the launch's node range pushes its own group range.
//
// Stack bound: a step takes B = min(32, SCAP - depth - size) groups (depth =
// the tree's depth), or one group from the top range when that is below 1.
// A step of B groups pushes at most B ranges, so it leaves at most
// SCAP - depth.  Single-group steps push, above the ranges present when they
// began (at most SCAP - depth), a chain of ranges of increasing tree depth
// (each one the children of a node taken from the range below it): at most
// depth of them, so the size never exceeds SCAP.  The starts are at most 32
// ranges (the roots' and one per chain node), which fit while
// depth <= SCAP - 32.  The host selects this kernel only then, and for
// chunked launches only when every chain is complete (depth <= CHAIN + 1).
// SCAP = 96 keeps the shared memory per warp small (what the blocks do not
// take stays L1 cache, which holds re-read surplus rows) while steps of 32
// groups stay the rule: on the d=59, 1M-node grid the stack holds at most
// about 40 ranges.
constexpr int SCAP = 96;

// Shared memory per warp of the descent form, in doubles: the stack (SCAP
// 16-byte entries), the fine-term list (whose first 32 doubles hold the chain
// weights at a chunk start, before any term is listed), the list of fine
// terms read from FP16 rows, and the point.
__host__ __device__ __forceinline__ int desc_stride(int dim) { return 2 * SCAP + 2 * FCAP + ((dim + 1) & ~1); }

// FP16 rows: row n holds its surpluses times 2^k_n as IEEE half precision,
// k_n = 14 - floor(log2(rowmax_n)), so that the row's largest magnitude lies
// in [2^14, 2^15).  Within each block of 256 outputs, lane l's 16 bytes hold
// outputs 128 v + 4 l + e (v = 0, 1; e = 0..3) in that order: the outputs the
// lane owns in the two-by-four output layout, one 16-byte load per row.
// The halves convert to FP32 exactly (one conversion instruction each,
// subnormal halves included), and the term's weight is scaled by
// 2^-k_n = 2^(floor(log2(rowmax_n)) - 14) when it is listed.  The host
// builds FP16 rows only for grids whose largest |surplus| is at least 2^-60,
// so that this scale (rowmax_n >= 2^-42 of it for any listed term) and the
// scaled weight stay normal FP32 numbers.
__device__ __forceinline__ void halves_to_float(uint32_t u, float& lo, float& hi)
{
	asm("{ .reg .b16 l, h; mov.b32 {l, h}, %2; cvt.f32.f16 %0, l; cvt.f32.f16 %1, h; }" : "=f"(lo), "=f"(hi) : "r"(u));
}
__device__ __forceinline__ float f16_weight(float wf, uint32_t rowmax_bits)
{
	return wf * __uint_as_float((((rowmax_bits >> 23) & 0xffu) - 14u) << 23);
}
static_assert(FCAP >= 32, "the chain weights (32 doubles) alias the fine-term list");

__device__ __forceinline__ uint4 pack_seg(uint32_t b, uint32_t e, double w)
{
	return make_uint4(b, e, (uint32_t)__double2loint(w), (uint32_t)__double2hiint(w));
}

template <int V, int E, int Q, int MINB, bool FULLROW>
__global__ void __launch_bounds__(BLOCK, MINB) fwd_f32d_kernel(const __grid_constant__ FwdArgs a)
{
	static_assert(FLUSH % Q == 0 || Q % FLUSH == 0, "groups of Q must tile the flush interval");
	static_assert(32 % Q == 0, "groups of Q must tile a step's hits");
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	double* wbase = smem + (threadIdx.x >> 5) * desc_stride(a.dim);
	uint4* stk = reinterpret_cast<uint4*>(wbase);
	uint2* fl = reinterpret_cast<uint2*>(wbase + 2 * SCAP);
	double* wchain = wbase + 2 * SCAP;     // aliases fl: used before any term is listed
	uint2* fl16 = reinterpret_cast<uint2*>(wbase + 2 * SCAP + FCAP);
	double* xs = wbase + 2 * SCAP + 2 * FCAP;
	// FP16 rows serve launches whose lanes own two blocks of four outputs of
	// full 256-output passes (the layout of the rows)
	constexpr bool F16 = V == 2 && E == 4 && FULLROW;
	constexpr int Q16 = 2 * Q;   // FP16 rows per group: the registers of Q FP32 rows
	// the final padding fills entries below 32 only: a group size that does not
	// divide 32 could pad past them and read stale row indices
	static_assert(32 % Q16 == 0, "groups of Q16 must tile a step's hits");
	const bool first = a.chunk_begin == 0;
	for (;;)
	{
		long long p = 0;
		if (lane == 0) p = (long long)atomicAdd(a.counter, 1ull);
		p = __shfl_sync(FULL, p, 0);
		if (p >= a.npts) break;
		const int gi = find_grid(a, p);
		const GridDesc& G = a.g[gi];
		int lo_n, hi_n;
		chunk_of(a, G, &lo_n, &hi_n);
		if (!first && lo_n >= hi_n) continue;   // this grid has no nodes in the chunk
		const bool ok = load_point(a, p, xs, lane);
		if (!ok && !first) continue;            // NaN already written by the first chunk
		// starts: lane 0 the roots' groups, lane d the groups of the active
		// chain node at depth d (after the first chunk)
		int size = 0;
		if (ok)
		{
			unsigned pathmask = 1u;
			const int len = first ? 0 : a.chain_len[gi];
			if (len)
			{
				int unused = lo_n;
				pathmask = chain_state(a, gi, G, xs, lane, wchain, &unused);
			}
			uint2 seg = make_uint2(0u, 0u);
			double ws = 1.0;
			if (lane == 0) seg = a.rseg[gi];
			else if (lane <= len && ((pathmask >> lane) & 1u)) { seg = a.cseg[gi][lane - 1]; ws = wchain[lane]; }
			const bool push = seg.y > seg.x;
			const unsigned pm = __ballot_sync(FULL, push);
			if (push) stk[__popc(pm & ((1u << lane) - 1u))] = pack_seg(seg.x, seg.y, ws);
			size = __popc(pm);
			__syncwarp();
			if (!first && !size) continue;     // no active start in the chunk: outputs unchanged
		}
		double* dst = a.out + (size_t)p * a.TD + a.o_begin;
		double acc[V][E];
#pragma unroll
		for (int v = 0; v < V; v++)
#pragma unroll
			for (int e = 0; e < E; e++)
			{
				const int o = out_col<E>(v, lane) + e;
				acc[v][e] = (!first && (FULLROW || a.o_begin + o < a.TD)) ? __ldcs(dst + o) : 0.0;
			}
		if (size)
		{
			const int lcol = a.o_begin + out_col<E>(0, lane);
			const float* s32l = G.s32 + lcol;
			const double* s64l = G.s64c + lcol;
			const uint32_t ld = (uint32_t)G.ld;
			const float skip_below = G.skip_below, big_below = G.big_below;
			const float f16_below = F16 && G.s16 ? G.f16_below : 0.f;
			const uint4* s16l = G.s16 + (a.o_begin >> 8) * 32 + lane;
			const uint32_t ld16 = (uint32_t)G.ld >> 3;
			const int room = SCAP - G.depth;        // steps of min(32, room - size) groups
			float part[V][E];
#pragma unroll
			for (int v = 0; v < V; v++)
#pragma unroll
				for (int e = 0; e < E; e++) part[v][e] = 0.f;
			int cnt = 0, cnt16 = 0, since = 0;
			auto flush = [&]()
			{
#pragma unroll
				for (int v = 0; v < V; v++)
#pragma unroll
					for (int e = 0; e < E; e++) { acc[v][e] = __dadd_rn(acc[v][e], (double)part[v][e]); part[v][e] = 0.f; }
			};
			// list entries [h, hend), hend - h a multiple of Q
			auto groups = [&](int h, int hend)
			{
				for (; h < hend; h += Q)
				{
					uint2 en[Q];
#pragma unroll
					for (int q = 0; q < Q; q += 2)
					{
						if (q + 1 < Q)
						{
							const uint4 t = *reinterpret_cast<const uint4*>(fl + h + q);
							en[q] = make_uint2(t.x, t.y);
							en[q + 1] = make_uint2(t.z, t.w);
						}
						else en[q] = fl[h + q];
					}
					float sv[Q][V][E];
#pragma unroll
					for (int q = 0; q < Q; q++)
					{
						const float* row = s32l + (size_t)en[q].x * ld;
#pragma unroll
						for (int v = 0; v < V; v++)
							load_row<E>(row, v * 32 * E, FULLROW || lcol + v * 32 * E < (int)ld, sv[q][v]);
					}
					// two outputs per packed FMA (each output's own rounding
					// and order, as with one FMA per output)
					if constexpr (E % 2 == 0)
					{
#pragma unroll
						for (int v = 0; v < V; v++)
#pragma unroll
							for (int e = 0; e < E; e += 2)
							{
								float2 pp = make_float2(part[v][e], part[v][e + 1]);
#pragma unroll
								for (int q = 0; q < Q; q++)
								{
									const float wq = __uint_as_float(en[q].y);
									pp = __ffma2_rn(make_float2(wq, wq), make_float2(sv[q][v][e], sv[q][v][e + 1]), pp);
								}
								part[v][e] = pp.x;
								part[v][e + 1] = pp.y;
							}
					}
					else
					{
#pragma unroll
						for (int v = 0; v < V; v++)
#pragma unroll
							for (int e = 0; e < E; e++)
#pragma unroll
								for (int q = 0; q < Q; q++)
									part[v][e] = __fmaf_rn(__uint_as_float(en[q].y), sv[q][v][e], part[v][e]);
					}
					since += Q;
					if (since >= FLUSH) { flush(); since = 0; }
				}
			};
			// FP16 list entries [h, hend), hend - h a multiple of Q16
			auto groups16 = [&](int h, int hend)
			{
				for (; h < hend; h += Q16)
				{
					uint2 en[Q16];
#pragma unroll
					for (int q = 0; q < Q16; q += 2)
					{
						const uint4 t = *reinterpret_cast<const uint4*>(fl16 + h + q);
						en[q] = make_uint2(t.x, t.y);
						en[q + 1] = make_uint2(t.z, t.w);
					}
					uint4 hv[Q16];
#pragma unroll
					for (int q = 0; q < Q16; q++) hv[q] = __ldg(s16l + (size_t)en[q].x * ld16);
#pragma unroll
					for (int q = 0; q < Q16; q++)
					{
						const float2 ww = make_float2(__uint_as_float(en[q].y), __uint_as_float(en[q].y));
						float f[8];
						halves_to_float(hv[q].x, f[0], f[1]);
						halves_to_float(hv[q].y, f[2], f[3]);
						halves_to_float(hv[q].z, f[4], f[5]);
						halves_to_float(hv[q].w, f[6], f[7]);
						float2 pp;
						pp = __ffma2_rn(ww, make_float2(f[0], f[1]), make_float2(part[0][0], part[0][1]));
						part[0][0] = pp.x; part[0][1] = pp.y;
						pp = __ffma2_rn(ww, make_float2(f[2], f[3]), make_float2(part[0][2], part[0][3]));
						part[0][2] = pp.x; part[0][3] = pp.y;
						pp = __ffma2_rn(ww, make_float2(f[4], f[5]), make_float2(part[V - 1][0], part[V - 1][1]));
						part[V - 1][0] = pp.x; part[V - 1][1] = pp.y;
						pp = __ffma2_rn(ww, make_float2(f[6], f[7]), make_float2(part[V - 1][2], part[V - 1][3]));
						part[V - 1][2] = pp.x; part[V - 1][3] = pp.y;
					}
					since += Q16;
					if (since >= FLUSH) { flush(); since = 0; }
				}
			};
			while (size > 0)
			{
				const int B = max(1, min(32, room - size));
				// lane k looks at stack entry size - 1 - k (lane 0: the top)
				uint4 e = make_uint4(0u, 0u, 0u, 0u);
				if (lane < size) e = stk[size - 1 - lane];
				const uint32_t cntk = e.y - e.x;
				uint32_t incl = cntk;
#pragma unroll
				for (int off = 1; off < 32; off <<= 1)
				{
					const uint32_t t = __shfl_up_sync(FULL, incl, off);
					if (lane >= off) incl += t;
				}
				const uint32_t take = min((uint32_t)B, __shfl_sync(FULL, incl, 31));
				const uint32_t start = incl - cntk;
				// ranges taken whole leave the stack; the one taken in part
				// (the new top) moves its first group
				const unsigned whole = __ballot_sync(FULL, lane < size && incl <= take);
				if (lane < size && start < take && incl > take) stk[size - 1 - lane].x = e.x + (take - start);
				const unsigned starts = __reduce_or_sync(FULL, (lane < size && start < take) ? (1u << start) : 0u);
				const int k = max(__popc(starts & ((2u << lane) - 1u)) - 1, 0);   // this lane's range
				const uint32_t kb = __shfl_sync(FULL, e.x, k);
				const uint32_t ks = __shfl_sync(FULL, start, k);
				const double wp = __hiloint2double((int)__shfl_sync(FULL, e.w, k), (int)__shfl_sync(FULL, e.z, k));
				size -= __popc(whole);
				// evaluate group kb + lane - ks
				uint32_t c = DESC_NONE;
				double w = 0.0;
				if ((uint32_t)lane < take)
				{
					const uint32_t gidx = kb + (uint32_t)lane - ks;
					const uint4 ga = __ldg(G.grp_a + gidx);
					const uint32_t kind = (ga.z >> 16) & 3u;
					if (kind == DESC_SIMPLE)
					{
						const uint2 gb = __ldg(G.grp_b + gidx);
						const double xd = xs[ga.z & 0xffffu];
						double h = hat(xd, gb.x);
						if (h > 0.0) c = ga.x;
						else if (ga.y != DESC_NONE)
						{
							h = hat(xd, gb.y);
							if (h > 0.0) c = ga.y;
						}
						if (c != DESC_NONE) w = ga.w ? wp * h * rcp_weight(hat(xd, ga.w)) : wp * h;
					}
					else if (kind == DESC_MULTI)
					{
						const uint4 r = __ldg(G.rec + ga.x);
						if (node_active(G, xs, r.y, r.z & 0xffu)) { c = ga.x; w = node_weight(G, xs, r.y, r.z & 0xffu); }
					}
					else { c = ga.x; w = wp; }
					if (c != DESC_NONE && ((int)c < lo_n || (int)c >= hi_n)) c = DESC_NONE;
				}
				const bool hit = c != DESC_NONE;
				uint4 ni = make_uint4(0u, 0u, 0u, DESC_NONE);
				if (hit) ni = __ldg(G.ninfo + c);
				// hits with children in the range push their groups
				const bool pushme = hit && ni.y && (int)c + 1 < hi_n;
				const unsigned pm = __ballot_sync(FULL, pushme);
				// the stack bound keeps size + pushes within SCAP; the test only
				// stops a write past the stack
				const int slot = size + __popc(pm & ((1u << lane) - 1u));
				if (pushme && slot < SCAP) stk[slot] = pack_seg(ni.x, ni.x + ni.y, w);
				size = min(size + __popc(pm), SCAP);
				__syncwarp();
				const unsigned mask = __ballot_sync(FULL, hit);
				if (!mask) continue;
				// big terms (rows with an FP64 copy, |w| * rowmax at or above the
				// threshold) now; fine terms to the list; negligible ones dropped
				const float wf = __double2float_rn(w);
				const float bound = fabsf(wf) * __uint_as_float(ni.z);
				const bool big = hit && ni.w != DESC_NONE && bound >= big_below;
				const bool fine = hit && !big && bound >= skip_below;
				const bool half = fine && bound < f16_below;
				unsigned cm = __ballot_sync(FULL, big);
				const unsigned fm = __ballot_sync(FULL, fine && !half);
				const unsigned hm = __ballot_sync(FULL, half);
				const unsigned below = (1u << lane) - 1u;
				if (fine && !half) fl[cnt + __popc(fm & below)] = make_uint2(c, __float_as_uint(wf));
				if (half) fl16[cnt16 + __popc(hm & below)] = make_uint2(c, __float_as_uint(f16_weight(wf, ni.z)));
				cnt += __popc(fm);
				cnt16 += __popc(hm);
				while (cm)
				{
					const int k0 = __ffs(cm) - 1;
					cm &= cm - 1;
					const bool two = cm != 0u;
					const int k1 = two ? __ffs(cm) - 1 : k0;
					if (two) cm &= cm - 1;
					const double w0 = __shfl_sync(FULL, w, k0);
					const double w1 = __shfl_sync(FULL, w, k1);
					const double* row0 = s64l + (size_t)__shfl_sync(FULL, ni.w, k0) * ld;
					const double* row1 = s64l + (size_t)__shfl_sync(FULL, ni.w, k1) * ld;
					double s0[V][E], s1[V][E];
#pragma unroll
					for (int v = 0; v < V; v++)
					{
						const bool in = FULLROW || lcol + v * 32 * E < (int)ld;
						load_row<E>(row0, v * 32 * E, in, s0[v]);
						load_row<E>(row1, v * 32 * E, in && two, s1[v]);
					}
#pragma unroll
					for (int v = 0; v < V; v++)
#pragma unroll
						for (int e2 = 0; e2 < E; e2++)
						{
							acc[v][e2] = fma(w0, s0[v][e2], acc[v][e2]);
							if (two) acc[v][e2] = fma(w1, s1[v][e2], acc[v][e2]);
						}
				}
				if (cnt >= 32)
				{
					// all whole groups; the remainder (< Q entries) moves to the front
					__syncwarp();
					const int wholeq = cnt - cnt % Q;
					groups(0, wholeq);
					const int rem = cnt - wholeq;
					uint2 t = make_uint2(0u, 0u);
					if (lane < rem) t = fl[wholeq + lane];
					__syncwarp();
					if (lane < rem) fl[lane] = t;
					__syncwarp();
					cnt = rem;
				}
				if (F16 && cnt16 >= 32)
				{
					__syncwarp();
					const int wholeq = cnt16 - cnt16 % Q16;
					groups16(0, wholeq);
					const int rem = cnt16 - wholeq;
					uint2 t = make_uint2(0u, 0u);
					if (lane < rem) t = fl16[wholeq + lane];
					__syncwarp();
					if (lane < rem) fl16[lane] = t;
					__syncwarp();
					cnt16 = rem;
				}
			}
			if (cnt)
			{
				// pad to whole groups with weight-0 copies of the first entry
				const int padded = (cnt + Q - 1) / Q * Q;
				__syncwarp();
				const uint32_t r0 = fl[0].x;
				if (lane >= cnt && lane < padded) fl[lane] = make_uint2(r0, 0u);
				__syncwarp();
				groups(0, padded);
			}
			if (F16 && cnt16)
			{
				const int padded = (cnt16 + Q16 - 1) / Q16 * Q16;
				__syncwarp();
				const uint32_t r0 = fl16[0].x;
				if (lane >= cnt16 && lane < padded) fl16[lane] = make_uint2(r0, 0u);
				__syncwarp();
				groups16(0, padded);
			}
			flush();
		}
#pragma unroll
		for (int v = 0; v < V; v++)
#pragma unroll
			for (int e = 0; e < E; e++)
			{
				const int o = out_col<E>(v, lane) + e;
				if (FULLROW || a.o_begin + o < a.TD)
					__stcs(dst + o, ok ? acc[v][e] : (G.nno ? __longlong_as_double(0x7ff8000000000000ll) : 0.0));
			}
		__syncwarp();
	}
}

// Small batches of the FP64 form (fewer points than resident warps, not
// node-chunked): one warp per (point, block of 32 outputs of the pass), lane
// l owning output 32 * block + l.  Each warp walks the tree itself (the
// blocks of one point walk in parallel) and lists its hits, with their
// gold-order weights, in index order in shared memory; the list is drained
// CDEPTH rows at a time, every lane loading its output of CDEPTH rows before
// the adds, which follow the gold order.  One double per lane per row lets a
// warp keep CDEPTH rows in flight where fwd_f64_kernel, owning up to eight
// outputs per lane, keeps eight (32 rows: 6-9 % faster than 16).
constexpr int CLIST = 128;
constexpr int CDEPTH = 32;

__host__ __device__ __forceinline__ int cols_stride(int dim) { return CLIST + CLIST / 2 + ((dim + 1) & ~1); }

__global__ void __launch_bounds__(BLOCK) fwd_f64_cols_kernel(const __grid_constant__ FwdArgs a)
{
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	double* wbase = smem + (threadIdx.x >> 5) * cols_stride(a.dim);
	double* lw = wbase;
	uint32_t* ln = reinterpret_cast<uint32_t*>(wbase + CLIST);
	double* xs = wbase + CLIST + CLIST / 2;
	const int cols = min(a.TD - a.o_begin, PASS);
	const int ncb = (cols + 31) / 32;
	const long long nitems = a.npts * ncb;
	for (;;)
	{
		long long it = 0;
		if (lane == 0) it = (long long)atomicAdd(a.counter, 1ull);
		it = __shfl_sync(FULL, it, 0);
		if (it >= nitems) break;
		const long long p = it / ncb;
		const int col = (int)(it % ncb) * 32 + lane;
		const bool cin = col < cols;
		const GridDesc& G = a.g[find_grid(a, p)];
		const bool ok = load_point(a, p, xs, lane);
		double acc = 0.0;
		int n = 0;
		// list entries [0, cnt) in order
		auto drain = [&](int cnt)
		{
			for (int b = 0; b < cnt; b += CDEPTH)
			{
				double sv[CDEPTH];
#pragma unroll
				for (int q = 0; q < CDEPTH; q++)
					sv[q] = (b + q < cnt && cin) ? __ldg(G.s64 + (size_t)ln[b + q] * G.ld + a.o_begin + col) : 0.0;
#pragma unroll
				for (int q = 0; q < CDEPTH; q++)
				{
					if (b + q >= cnt) break;   // warp-uniform
					acc = __dadd_rn(acc, __dmul_rn(lw[b + q], sv[q]));
				}
			}
		};
		if (ok)
		{
			traverse<false>(G, xs, lane, 0, G.nno, [&](unsigned mask, int n0, double w, const uint4&, float)
			{
				if ((mask >> lane) & 1u)
				{
					const int pos = n + __popc(mask & ((1u << lane) - 1u));
					ln[pos] = (uint32_t)(n0 + lane);
					lw[pos] = w;
				}
				n += __popc(mask);   // below CLIST - 32 before, below CLIST after
				__syncwarp();
				if (n >= CLIST - 32)
				{
					drain(n);
					n = 0;
					__syncwarp();
				}
			});
			if (n) drain(n);
		}
		if (cin)
			a.out[(size_t)p * a.TD + a.o_begin + col] = ok ? acc : (G.nno ? __longlong_as_double(0x7ff8000000000000ll) : 0.0);
		__syncwarp();
	}
}

// Small FP64 batches in two phases.  A point's walk takes its windows one
// after another, and its warps then wait on their rows a few at a time; with
// few points most of the GPU idles.  Here the walk is spread over many warps
// and the rows are staged in bulk; the arithmetic is the gold kernel's, in
// its order (bit-identical to fwd_f64_kernel).
// Phase 1 (walk_chunks_kernel): one warp per (point, chunk of LCS nodes)
// walks the chunk from its start's ancestor chain (a table built with the
// grid), lists the chunk's hits in index order with their gold-order weights,
// and prefetches their surplus rows into the L2.  For the FP32C form (grid
// descriptors with row maxima) it lists only the terms the FP32C kernels keep
// (big terms, and others whose bound reaches the dropped-term bound); their
// FP64 rows are then added exactly.
// Phase 2 (fwd_f64_list_kernel): one warp per (point, 32 outputs) takes the
// point's hits chunk after chunk, copies the rows of LDEPTH hits into shared
// memory (cp.async, one double per lane per row) and then adds them in order.
constexpr int LCS = 512;                   // nodes per phase-1 chunk
constexpr int LDEPTH = 256;                // rows per phase-2 copy round
constexpr int LBLOCK = 64;                 // phase-2 threads per block
constexpr uint32_t HIT_BAD = 0xffffffffu;  // hit count of a point with a non-finite coordinate

__host__ __device__ __forceinline__ int list_stride() { return LDEPTH * 32 + LDEPTH + LDEPTH / 2; }

struct ListArgs
{
	GridDesc g[MAXG];
	const uint32_t* ctab[MAXG];  // per chunk k, 32 words: {chain length, chain node at depth 1..length}
	long long ibeg[MAXG + 1];    // first (point, chunk) item of each grid; a point's items are consecutive
	int nch[MAXG];               // chunks per grid
	const double* x;
	double* out;
	uint32_t* hcnt;              // hits of item i: hcnt[i] (HIT_BAD for a non-finite point)
	uint32_t* hnode;             //   their nodes and weights at [i * LCS, i * LCS + hcnt[i])
	double* hw;
	long long npts;
	int ngrids, dim, TD;
};
static_assert(sizeof(ListArgs) <= 32764, "ListArgs exceeds the kernel parameter limit");

__device__ __forceinline__ int list_grid(const ListArgs& a, long long p)
{
	int gi = 0;
	while (gi + 1 < a.ngrids && a.g[gi + 1].pt_begin <= p) gi++;
	return gi;
}

__global__ void __launch_bounds__(BLOCK) walk_chunks_kernel(const __grid_constant__ ListArgs a)
{
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	double* xs = smem + warp * a.dim;
	const long long nitems = a.ibeg[a.ngrids];
	for (long long it = (long long)blockIdx.x * WARPS + warp; it < nitems; it += (long long)gridDim.x * WARPS)
	{
		int gi = 0;
		while (gi + 1 < a.ngrids && a.ibeg[gi + 1] <= it) gi++;
		const GridDesc& G = a.g[gi];
		const long long loc = it - a.ibeg[gi];
		const long long p = G.pt_begin + loc / a.nch[gi];
		const int k = (int)(loc % a.nch[gi]);
		bool finite = true;
		for (int d = lane; d < a.dim; d += 32)
		{
			const double v = a.x[(size_t)p * a.dim + d];
			xs[d] = v;
			finite &= isfinite(v);
		}
		__syncwarp();
		uint32_t cnt = HIT_BAD;
		if (__all_sync(FULL, finite))
		{
			cnt = 0;
			const uint32_t* ch = a.ctab[gi] + (size_t)k * 32;
			const int len = (int)__ldg(ch);
			int lo = k * LCS;
			const int hi = min(G.nno, lo + LCS);
			const unsigned pathmask = chain_state_of([&](int d) { return __ldg(ch + 1 + d); }, len, G, xs, lane,
			                                         nullptr, &lo);
			uint32_t* hn = a.hnode + (size_t)it * LCS;
			double* hv = a.hw + (size_t)it * LCS;
			const int rowb = a.TD * 8;
			if (lo < hi)
				traverse<false>(G, xs, lane, lo, hi, [&](unsigned mask, int n0, double w, const uint4& r, float rm)
				{
					bool keep = (mask >> lane) & 1u;
					if (keep && G.rowmax)
					{
						const float bound = fabsf(__double2float_rn(w)) * rm;
						keep = ((r.z & NODE_COARSE) && bound >= G.big_below) || bound >= G.skip_below;
					}
					const unsigned km = __ballot_sync(FULL, keep);
					if (keep)
					{
						const uint32_t pos = cnt + __popc(km & ((1u << lane) - 1u));
						hn[pos] = (uint32_t)(n0 + lane);
						hv[pos] = w;
						const char* row = reinterpret_cast<const char*>(G.s64 + (size_t)(n0 + lane) * G.ld);
						for (int b = 0; b < rowb; b += 128) asm volatile("prefetch.global.L2 [%0];" :: "l"(row + b));
					}
					cnt += __popc(km);
				}, nullptr, pathmask, len);
		}
		if (lane == 0) a.hcnt[it] = cnt;
		__syncwarp();
	}
}

__global__ void __launch_bounds__(LBLOCK) fwd_f64_list_kernel(const __grid_constant__ ListArgs a)
{
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	double* rows = smem + (size_t)warp * list_stride();
	double* ew = rows + LDEPTH * 32;
	uint32_t* en = reinterpret_cast<uint32_t*>(ew + LDEPTH);
	const uint32_t rows_s = (uint32_t)__cvta_generic_to_shared(rows) + lane * 8u;
	const int ncb = (a.TD + 31) / 32;
	const long long nitems = a.npts * ncb;
	for (long long it = (long long)blockIdx.x * (LBLOCK / 32) + warp; it < nitems;
	     it += (long long)gridDim.x * (LBLOCK / 32))
	{
		const long long p = it / ncb;
		const int col = (int)(it % ncb) * 32 + lane;
		const bool cin = col < a.TD;
		const int gi = list_grid(a, p);
		const GridDesc& G = a.g[gi];
		const int nch = a.nch[gi];
		const long long i0 = a.ibeg[gi] + (p - G.pt_begin) * nch;
		const double* src = G.s64 + (cin ? col : 0);
		double acc = 0.0;
		bool ok = true;
		// hits of chunks k0 .. k0 + 31: lane l holds chunk k0 + l's count c and
		// the exclusive prefix excl; t of the group's T hits are taken
		int k0 = -32;
		uint32_t c = 0, excl = 0, T = 0, t = 0;
		for (;;)
		{
			int m = 0;
			while (m < LDEPTH)
			{
				if (t == T)
				{
					k0 += 32;
					if (k0 >= nch) break;
					c = k0 + lane < nch ? __ldg(a.hcnt + i0 + k0 + lane) : 0u;
					if (__any_sync(FULL, c == HIT_BAD)) { ok = false; break; }
					uint32_t incl = c;
#pragma unroll
					for (int off = 1; off < 32; off <<= 1)
					{
						const uint32_t v = __shfl_up_sync(FULL, incl, off);
						if (lane >= off) incl += v;
					}
					T = __shfl_sync(FULL, incl, 31);
					excl = incl - c;
					t = 0;
					continue;
				}
				const uint32_t take = min(T - t, (uint32_t)(LDEPTH - m));
				// list positions of hits t .. t + take - 1 first, then all their
				// loads, then the stores: one round trip for the whole take
				size_t e[LDEPTH / 32];
#pragma unroll
				for (int j = 0; j < LDEPTH / 32; j++)
				{
					const uint32_t h = t + (uint32_t)(j * 32 + lane);
					// the chunk of hit h: the last lane whose prefix is at most h
					int sl = 0;
#pragma unroll
					for (int step = 16; step >= 1; step >>= 1)
					{
						const uint32_t v = __shfl_sync(FULL, excl, sl + step);
						if (v <= h) sl += step;
					}
					const uint32_t es = __shfl_sync(FULL, excl, sl);
					e[j] = (size_t)(i0 + k0 + sl) * LCS + (h - es);
				}
				uint32_t nd[LDEPTH / 32];
				double wv[LDEPTH / 32];
#pragma unroll
				for (int j = 0; j < LDEPTH / 32; j++)
				{
					const bool in = (uint32_t)(j * 32 + lane) < take;
					nd[j] = in ? a.hnode[e[j]] : 0u;
					wv[j] = in ? a.hw[e[j]] : 0.0;
				}
#pragma unroll
				for (int j = 0; j < LDEPTH / 32; j++)
					if ((uint32_t)(j * 32 + lane) < take)
					{
						en[m + j * 32 + lane] = nd[j];
						ew[m + j * 32 + lane] = wv[j];
					}
				m += (int)take;
				t += take;
			}
			if (!ok || m == 0) break;
			__syncwarp();
			if (cin)
			{
				for (int q = 0; q < m; q++)
					asm volatile("cp.async.ca.shared.global [%0], [%1], 8;"
					             :: "r"(rows_s + (uint32_t)q * 256u), "l"(src + (size_t)en[q] * G.ld) : "memory");
			}
			asm volatile("cp.async.wait_all;" ::: "memory");
			__syncwarp();
#pragma unroll 8
			for (int q = 0; q < m; q++) acc = __dadd_rn(acc, __dmul_rn(ew[q], rows[q * 32 + lane]));
			__syncwarp();
		}
		if (cin) a.out[(size_t)p * a.TD + col] = ok ? acc : (G.nno ? __longlong_as_double(0x7ff8000000000000ll) : 0.0);
	}
}

// Active-node count per point (single grid).  With `classes` (a grid
// descriptor of the FP32C form), also the point's terms by the FP32C form's
// classes: classes[4p] big (FP64 row), [4p + 1] fine (FP32 row), [4p + 2]
// fine (FP16 row), [4p + 3] dropped, by the bound |w| * max|s_row| of the
// full-product weight.
template <bool CLASSES>
__global__ void __launch_bounds__(BLOCK) count_kernel(const __grid_constant__ FwdArgs a, long long* counts,
	long long* classes)
{
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	double* xs = smem + (threadIdx.x >> 5) * a.dim;
	for (;;)
	{
		long long p = 0;
		if (lane == 0) p = (long long)atomicAdd(a.counter, 1ull);
		p = __shfl_sync(FULL, p, 0);
		if (p >= a.npts) break;
		const GridDesc& G = a.g[find_grid(a, p)];
		long long cnt = 0, nbig = 0, nfine = 0, nhalf = 0;
		if (load_point(a, p, xs, lane))
			traverse(G, xs, lane, [&](unsigned mask, int, double w, const uint4& r, float rm)
			{
				cnt += __popc(mask);
				if (CLASSES)
				{
					const bool hit = (mask >> lane) & 1u;
					const float bound = fabsf(__double2float_rn(w)) * rm;
					const bool big = hit && (r.z & NODE_COARSE) && bound >= G.big_below;
					const bool fine = hit && !big && bound >= G.skip_below;
					const bool half = fine && bound < G.f16_below;
					nbig += __popc(__ballot_sync(FULL, big));
					nfine += __popc(__ballot_sync(FULL, fine && !half));
					nhalf += __popc(__ballot_sync(FULL, half));
				}
			});
		if (lane == 0)
		{
			if (!CLASSES) counts[p] = cnt;
			else
			{
				classes[4 * p] = nbig;
				classes[4 * p + 1] = nfine;
				classes[4 * p + 2] = nhalf;
				classes[4 * p + 3] = cnt - nbig - nfine - nhalf;
			}
		}
		__syncwarp();
	}
}

// ------------------------------------------------------------------ backward
//
// dL/dx: per point (one warp), for every active node n the scalar
// cs = sum_o gout[p,o] * s[n,o] (warp reduction), then for each component c of
// n, dw/dx_{dim c} = (prod of the other hats) * slope_c, slope = -i sign(x i - j).
// dL/dsurplus: pairs (node, point, weight) are written at per-point offsets
// (exclusive scan of the active counts: no atomics), stably radix-sorted by
// node, and each node's segment is reduced by one warp in point order.

// One (point, weight) pair of the dL/dsurplus reduction, sorted by node with
// its node as the key.
struct PairVal
{
	uint32_t point, pad;
	double w;
};

struct BwdArgs
{
	GridDesc G;
	const double* x;
	const double* gout;
	double* gx;
	const long long* pair_off;   // npts + 1, or null
	uint32_t* pair_node;
	PairVal* pair_val;
	unsigned long long* counter;
	long long npts;
	int dim, TD;
};

template <int R>
__global__ void __launch_bounds__(BLOCK) bwd_points_kernel(const __grid_constant__ BwdArgs a)
{
	extern __shared__ double smem[];
	const int lane = threadIdx.x & 31;
	double* xs = smem + (threadIdx.x >> 5) * 2 * a.dim;
	double* gxs = xs + a.dim;
	const GridDesc& G = a.G;
	for (;;)
	{
		long long p = 0;
		if (lane == 0) p = (long long)atomicAdd(a.counter, 1ull);
		p = __shfl_sync(FULL, p, 0);
		if (p >= a.npts) break;
		for (int k = lane; k < a.dim; k += 32) { xs[k] = a.x[(size_t)p * a.dim + k]; gxs[k] = 0.0; }
		double g[R];
#pragma unroll
		for (int r = 0; r < R; r++)
		{
			const int o = lane + 32 * r;
			g[r] = o < a.TD ? a.gout[(size_t)p * a.TD + o] : 0.0;
		}
		__syncwarp();
		long long woff = a.pair_off ? a.pair_off[p] : 0;
		traverse(G, xs, lane, [&](unsigned mask, int n0, double w, const uint4& rec, float)
		{
			if (a.pair_off)
			{
				const int rank = __popc(mask & ((1u << lane) - 1u));
				if ((mask >> lane) & 1u)
				{
					a.pair_node[woff + rank] = (uint32_t)(n0 + lane);
					a.pair_val[woff + rank] = PairVal{ (uint32_t)p, 0u, w };
				}
				woff += __popc(mask);
			}
			if (!a.gx) return;
			// dx contribution of hit k with cs = sum_o gout[o] * s[node, o]
			auto components = [&](int k, double cs)
			{
				const uint32_t cptr = __shfl_sync(FULL, rec.y, k);
				const uint32_t ncomp = __shfl_sync(FULL, rec.z, k) & 0xffu;
				if (ncomp <= 32)
				{
					// lane c holds component c's hat and slope; the product of the
					// other hats is the exclusive prefix times the exclusive suffix
					// product over the lanes (lanes past ncomp hold 1)
					double h = 1.0, slope = 0.0;
					uint32_t dc = 0;
					if ((uint32_t)lane < ncomp)
					{
						const uint2 cp = __ldg(G.comps + cptr + lane);
						dc = cp.x;
						h = hat(xs[cp.x], cp.y);
						const double t = xs[cp.x] * (double)(cp.y & 0xffffu) - (double)(cp.y >> 16);
						slope = t > 0.0 ? -(double)(cp.y & 0xffffu) : (t < 0.0 ? (double)(cp.y & 0xffffu) : 0.0);
					}
					double pre = h, suf = h;
	#pragma unroll
					for (int off = 1; off < 32; off <<= 1)
					{
						const double u = __shfl_up_sync(FULL, pre, off);
						const double d = __shfl_down_sync(FULL, suf, off);
						if (lane >= off) pre *= u;
						if (lane + off < 32) suf *= d;
					}
					double before = __shfl_up_sync(FULL, pre, 1), after = __shfl_down_sync(FULL, suf, 1);
					if (lane == 0) before = 1.0;
					if (lane == 31) after = 1.0;
					if ((uint32_t)lane < ncomp) gxs[dc] += cs * (before * after) * slope;
				}
				else
					for (uint32_t c = lane; c < ncomp; c += 32)
					{
						const uint2 cp = __ldg(G.comps + cptr + c);
						double others = 1.0;
						for (uint32_t q = 0; q < ncomp; q++)
							if (q != c)
							{
								const uint2 cq = __ldg(G.comps + cptr + q);
								others *= hat(xs[cq.x], cq.y);
							}
						const double t = xs[cp.x] * (double)(cp.y & 0xffffu) - (double)(cp.y >> 16);
						const double slope = t > 0.0 ? -(double)(cp.y & 0xffffu) : (t < 0.0 ? (double)(cp.y & 0xffffu) : 0.0);
						gxs[cp.x] += cs * others * slope;
					}
				__syncwarp();
			};
			// two hits at a time: both rows loaded and reduced together; their
			// dx contributions are added one after the other (they may share
			// dimensions)
			while (mask)
			{
				const int k0 = __ffs(mask) - 1;
				mask &= mask - 1;
				const bool two = mask != 0u;
				const int k1 = two ? __ffs(mask) - 1 : k0;
				if (two) mask &= mask - 1;
				const double* row0 = G.s64 + (size_t)(n0 + k0) * G.ld;
				const double* row1 = G.s64 + (size_t)(n0 + k1) * G.ld;
				double s0[R], s1[R];
#pragma unroll
				for (int r = 0; r < R; r++)
				{
					const int o = lane + 32 * r;
					s0[r] = o < a.TD ? __ldg(row0 + o) : 0.0;
					s1[r] = (two && o < a.TD) ? __ldg(row1 + o) : 0.0;
				}
				double cs0 = 0.0, cs1 = 0.0;
#pragma unroll
				for (int r = 0; r < R; r++) { cs0 = fma(g[r], s0[r], cs0); cs1 = fma(g[r], s1[r], cs1); }
#pragma unroll
				for (int off = 16; off > 0; off >>= 1)
				{
					cs0 += __shfl_xor_sync(FULL, cs0, off);
					cs1 += __shfl_xor_sync(FULL, cs1, off);
				}
				components(k0, cs0);
				if (two) components(k1, cs1);
			}
		});
		if (a.gx)
			for (int k = lane; k < a.dim; k += 32) a.gx[(size_t)p * a.dim + k] = gxs[k];
		__syncwarp();
	}
}

// One warp per node: dL/dsurplus[n, :] = sum over its pairs of w * gout[point, :],
// in sorted (point) order.  The node's pairs are read 32 at a time (lane l
// loads pair q + l) and their gout rows two at a time.
template <int R>
__global__ void __launch_bounds__(BLOCK) bwd_surplus_kernel(const uint32_t* __restrict__ sorted_node,
	const PairVal* __restrict__ sorted_val, long long npairs, const double* __restrict__ gout,
	double* __restrict__ gs, int nno, int TD)
{
	const int lane = threadIdx.x & 31;
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
	for (long long n = warp; n < nno; n += nwarps)
	{
		// segment [lo, e) of node n in the sorted keys
		long long lo = 0, hi = npairs;
		while (lo < hi) { long long m = (lo + hi) >> 1; if (sorted_node[m] < (uint32_t)n) lo = m + 1; else hi = m; }
		long long e = lo, h2 = npairs;
		while (e < h2) { long long m = (e + h2) >> 1; if (sorted_node[m] <= (uint32_t)n) e = m + 1; else h2 = m; }
		double acc[R];
#pragma unroll
		for (int r = 0; r < R; r++) acc[r] = 0.0;
		for (long long q0 = lo; q0 < e; q0 += 32)
		{
			const int m = (int)min(32ll, e - q0);
			PairVal pv{ 0u, 0u, 0.0 };
			if (lane < m) pv = sorted_val[q0 + lane];
			for (int k = 0; k < m; k += 2)
			{
				const bool two = k + 1 < m;
				const double w0 = __shfl_sync(FULL, pv.w, k);
				const double w1 = __shfl_sync(FULL, pv.w, two ? k + 1 : k);
				const double* r0 = gout + (size_t)__shfl_sync(FULL, pv.point, k) * TD;
				const double* r1 = gout + (size_t)__shfl_sync(FULL, pv.point, two ? k + 1 : k) * TD;
				double v0[R], v1[R];
#pragma unroll
				for (int r = 0; r < R; r++)
				{
					const int o = lane + 32 * r;
					v0[r] = o < TD ? r0[o] : 0.0;
					v1[r] = (two && o < TD) ? r1[o] : 0.0;
				}
#pragma unroll
				for (int r = 0; r < R; r++)
				{
					acc[r] = fma(w0, v0[r], acc[r]);
					if (two) acc[r] = fma(w1, v1[r], acc[r]);
				}
			}
		}
#pragma unroll
		for (int r = 0; r < R; r++)
		{
			const int o = lane + 32 * r;
			if (o < TD) gs[(size_t)n * TD + o] = acc[r];
		}
	}
}


// ------------------------------------------------------------ host helpers

thread_local sgi_launch_stats g_stats{};

#define CUDA_TRY(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
	return fail(SGI_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); } while (0)

// Per-device workspace: a ring of work counters (one per launch; a counter is
// reused after 65536 later launches on the device) and staging buffers for
// the host-pointer entry point.
struct DeviceWork
{
	std::mutex mtx;
	unsigned long long* counters = nullptr;
	std::atomic<unsigned> next{0};
	int sms = 0;
	int l2_bytes = 0;
	// host-pointer staging
	double* dx = nullptr; size_t dx_bytes = 0;
	double* dout = nullptr; size_t dout_bytes = 0;
	cudaStream_t stream = nullptr, stream2 = nullptr, copy_in = nullptr, copy_out = nullptr;
	static constexpr int NEV = 8;
	cudaEvent_t ev_in[NEV] = {}, ev_done[NEV] = {};
	// stream-ordered scratch (backward pass, small-batch hit lists): a
	// private pool that keeps freed memory for the next call instead of
	// returning it at every synchronization (as the default pool does), so
	// repeated calls do not map their scratch again.  Created under its own
	// mutex: the host-pointer entry holds mtx while it launches.
	std::mutex pool_mtx;
	std::atomic<cudaMemPool_t> pool{nullptr};
};
constexpr unsigned NCOUNTERS = 1u << 16;

std::mutex g_work_mtx;
std::vector<DeviceWork*> g_work;

int device_work(int dev, DeviceWork** out)
{
	std::lock_guard<std::mutex> lk(g_work_mtx);
	if ((int)g_work.size() <= dev) g_work.resize(dev + 1, nullptr);
	if (!g_work[dev])
	{
		DeviceWork* w = new DeviceWork;
		CUDA_TRY(cudaMalloc(&w->counters, sizeof(unsigned long long) * NCOUNTERS));
		CUDA_TRY(cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, dev));
		CUDA_TRY(cudaDeviceGetAttribute(&w->l2_bytes, cudaDevAttrL2CacheSize, dev));
		g_work[dev] = w;
	}
	*out = g_work[dev];
	return SGI_OK;
}

int scratch_pool(DeviceWork* W, int dev, cudaMemPool_t* out)
{
	if (!W->pool.load())
	{
		std::lock_guard<std::mutex> lk(W->pool_mtx);
		if (!W->pool.load())
		{
			cudaMemPoolProps props{};
			props.allocType = cudaMemAllocationTypePinned;
			props.location.type = cudaMemLocationTypeDevice;
			props.location.id = dev;
			cudaMemPool_t pool = nullptr;
			CUDA_TRY(cudaMemPoolCreate(&pool, &props));
			uint64_t keep = UINT64_MAX;
			CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
			W->pool.store(pool);
		}
	}
	*out = W->pool.load();
	return SGI_OK;
}

// Node-range chunk for the forward launches: grids whose surplus rows exceed
// the L2 are walked in node ranges, all points per range, so that the rows
// each range gathers stay mostly L2-resident.
// Small batches are not chunked.  sgi_set_chunk_rows (or SGI_CHUNK_ROWS at
// start-up) overrides: 0 = no chunks, n > 0 = chunks of n nodes.
std::atomic<int> g_chunk_override{[]() { const char* e = getenv("SGI_CHUNK_ROWS"); return e ? atoi(e) : -1; }()};

int chunk_rows_env() { return g_chunk_override.load(); }

// FP32C variant of the direct entry points (plans time their own): -1 =
// automatic (auto_variant), else the variant sgi_set_fp32c_variant (or
// SGI_FP32C_VARIANT at start-up) fixed.
std::atomic<int> g_variant{[]() { const char* e = getenv("SGI_FP32C_VARIANT"); return e ? atoi(e) : -1; }()};

// The automatic FP32C variant: eight fine rows in flight per warp (2) for a
// batch of fewer than 64 points per SM, whose warps wait on their rows (on a
// 200k-node d=59 grid, 16 / 1,024 / 8,192 points: 242 / 451 / 994 us against
// 327 / 661 / 1,130 us for variant 1), else two rows at 4 blocks per SM (1),
// the faster at a million points.
int auto_variant(int variant, long long npts, int sms)
{
	if (variant >= 0) return variant;
	return npts < (long long)sms * 64 ? 2 : 1;
}

uint32_t float_bits(float f)
{
	uint32_t u;
	memcpy(&u, &f, 4);
	return u;
}

// FP32C kernel variants (fine rows in flight per warp against warps per SM):
// 0 = groups of four rows, at least 3 blocks per SM; 1 = two rows, 4 blocks;
// 2 = eight rows, 2 blocks.  They run the descent walk when every grid of the
// launch allows it (descent_ok), else the window walk; 3-5 force the window
// walk with the settings of 0-2.  Plans time 0-2.
constexpr int NVARIANTS = 3;
constexpr int NVARIANTS_ALL = 6;
template <int V, int E>
void (*f32c_variant(int variant))(FwdArgs)
{
	switch (variant % NVARIANTS)
	{
	case 1: return fwd_f32c_kernel<V, E, 2, 4>;
	case 2: return fwd_f32c_kernel<V, E, 8, 2>;
	default: return fwd_f32c_kernel<V, E, 4, 3>;
	}
}

template <int V, int E, bool FULLROW>
void (*f32d_variant(int variant))(FwdArgs)
{
	switch (variant)
	{
	case 1: return fwd_f32d_kernel<V, E, 2, 4, FULLROW>;
	case 2: return fwd_f32d_kernel<V, E, 8, 2, FULLROW>;
	default: return fwd_f32d_kernel<V, E, 4, 3, FULLROW>;
	}
}

template <int V, int E>
void (*fp32c_kernel(int variant, bool descent, int cols))(FwdArgs)
{
	if (!descent || variant >= NVARIANTS) return f32c_variant<V, E>(variant);
	// a pass whose columns fill every lane's outputs needs no column tests
	return cols == V * 32 * E ? f32d_variant<V, E, true>(variant) : f32d_variant<V, E, false>(variant);
}

// small: a batch of fewer points than resident warps; the FP64 form then
// keeps eight rows in flight per warp (four for eight outputs per lane).
void (*select_fwd(int precision, int ld, int cols, int variant = 0, bool descent = false, bool small = false))(FwdArgs)
{
	const bool f64 = precision == SGI_FP64;
	if (ld <= 32) return f64 ? (small ? fwd_f64_kernel<1, 1, 8> : fwd_f64_kernel<1, 1>) : fp32c_kernel<1, 1>(variant, descent, cols);
	if (cols <= 64) return f64 ? (small ? fwd_f64_kernel<1, 2, 8> : fwd_f64_kernel<1, 2>) : fp32c_kernel<1, 2>(variant, descent, cols);
	// FP32C reads four consecutive outputs per lane (16-byte loads) when rows
	// are a multiple of 128 wide
	const bool e4 = !f64 && ld % 128 == 0;
	if (cols <= 128)
		return f64 ? (small ? fwd_f64_kernel<2, 2, 8> : fwd_f64_kernel<2, 2>)
		           : e4 ? fp32c_kernel<1, 4>(variant, descent, cols) : fp32c_kernel<2, 2>(variant, descent, cols);
	return f64 ? (small ? fwd_f64_kernel<4, 2, 4> : fwd_f64_kernel<4, 2>)
	           : e4 ? fp32c_kernel<2, 4>(variant, descent, cols) : fp32c_kernel<4, 2>(variant, descent, cols);
}

// Dynamic shared memory of a forward launch.
size_t fwd_smem(int precision, int dim, bool descent = false)
{
	if (precision != SGI_FP32C) return (size_t)WARPS * dim * sizeof(double);
	return (size_t)WARPS * (descent ? desc_stride(dim) : list_stride(dim)) * sizeof(double);
}

int pick_R(int cols)
{
	if (cols <= 32) return 1;
	if (cols <= 64) return 2;
	if (cols <= 128) return 4;
	return 8;
}

int chunk_rows(const DeviceWork* W, const sgi_grid* g0, int precision, long long npts, int maxnno);

template <class K>
int occupancy_grid(K kernel, size_t smem, int sms, int* blocks, int block_threads = BLOCK)
{
	int per_sm = 0;
	CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block_threads, smem));
	if (per_sm < 1) return fail(SGI_E_CUDA, "kernel does not fit on an SM (smem %zu)", smem);
	*blocks = per_sm * sms;
	return SGI_OK;
}

} // namespace

// ------------------------------------------------------------- grid object

struct sgi_grid
{
	int device = 0;
	int dim = 0, nno = 0, TD = 0, ld = 0;
	uint4* rec = nullptr;
	uint2* comps = nullptr;
	float* rowmax = nullptr;
	float skip_below = 0.f;      // in use: the larger of skip_floor and the surplus cutoff
	float skip_floor = 0.f;      // FP32C's own negligible-term bound, 2^-42 of max |surplus|
	float f16_floor = 0.f;       // FP32C: fine terms below this bound read the FP16 rows (2^-29 of max |surplus|)
	uint4* s16 = nullptr;        // FP16 rows (see the kernels' description), or null
	uint2* aux = nullptr;
	double* s64 = nullptr;
	float* s32 = nullptr;
	double* s64c = nullptr;
	uint32_t* coarse_index = nullptr;
	int* parent = nullptr;
	// descent layout (FP32C): child groups and per-node group ranges
	uint4* grp_a = nullptr;
	uint2* grp_b = nullptr;
	uint4* ninfo = nullptr;
	// host copy of the containment tree, for the ancestor chains of node
	// chunk boundaries, and of the group ranges and child bounds, for the
	// descent's starts (pmax: running largest child index over a node's groups)
	std::vector<int> parent_h;
	std::vector<uint32_t> skip_h, depth_h;
	std::vector<uint32_t> gfirst_h, gcount_h, gcmin_h, gpmax_h;
	// two-phase small batches: per chunk of LCS nodes, 32 words {length of
	// the chunk start's ancestor chain, chain node at depth 1..length}
	uint32_t* ctab = nullptr;
	int nlch = 0;
	sgi_grid_info info{};
};

namespace {

// Batches below this many points are not node-chunked by default.
constexpr long long CHUNK_MIN_POINTS = 81920;

int chunk_rows(const DeviceWork* W, const sgi_grid* g0, int precision, long long npts, int maxnno)
{
	const int env = chunk_rows_env();
	if (env >= 0) return env >= maxnno ? 0 : env;
	// rows filling half the L2 (the FP32 rows for FP32C): the autotuner's
	// choice for both forms on the d=59, 1M-node, TotalDof=256 workload.
	// Smaller batches read each chunk's rows too few times to pay for every
	// point's set-up per chunk (d=59 grids of 300k and 1M nodes: unchunked is
	// faster up to 64k points, chunked from 96k points up)
	const long long row = (long long)g0->ld * (precision == SGI_FP64 ? 8 : 4);
	const long long rows = std::max(1024ll, (long long)W->l2_bytes / 2 / row);
	if (npts < CHUNK_MIN_POINTS || maxnno <= rows) return 0;
	return (int)rows;
}

void host_plans_forget(const sgi_grid* g);

void free_grid(sgi_grid* g)
{
	if (!g) return;
	host_plans_forget(g);
	int prev = 0;
	cudaGetDevice(&prev);
	cudaSetDevice(g->device);
	cudaFree(g->rec); cudaFree(g->comps); cudaFree(g->s64); cudaFree(g->s32); cudaFree(g->s64c); cudaFree(g->coarse_index);
	cudaFree(g->parent);
	cudaFree(g->rowmax);
	cudaFree(g->aux);
	cudaFree(g->grp_a); cudaFree(g->grp_b); cudaFree(g->ninfo);
	cudaFree(g->ctab);
	cudaFree(g->s16);
	cudaSetDevice(prev);
	delete g;
}

// precision SGI_FP32C also hands the kernel the row maxima for its
// negligible-term test; the FP64 form keeps every term.
GridDesc desc_of(const sgi_grid* g, long long pt_begin, int precision = SGI_FP64)
{
	GridDesc d;
	d.rec = g->rec; d.comps = g->comps;
	d.rowmax = precision == SGI_FP32C ? g->rowmax : nullptr;
	d.aux = g->aux;
	d.skip_below = precision == SGI_FP32C ? g->skip_below : 0.f;
	d.big_below = precision == SGI_FP32C ? (float)g->info.coarse_threshold : 0.f;
	d.s64 = g->s64; d.s32 = g->s32; d.s64c = g->s64c;
	d.coarse_index = g->coarse_index; d.parent = g->parent; d.pt_begin = pt_begin; d.nno = g->nno; d.ld = g->ld;
	d.grp_a = g->grp_a; d.grp_b = g->grp_b; d.ninfo = g->ninfo; d.depth = g->info.tree_depth;
	d.s16 = precision == SGI_FP32C ? g->s16 : nullptr;
	d.f16_below = precision == SGI_FP32C && g->s16 ? g->f16_floor : 0.f;
	return d;
}

struct DeviceGuard
{
	int prev = -1;
	explicit DeviceGuard(int dev) { cudaGetDevice(&prev); cudaSetDevice(dev); }
	~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

} // namespace

extern "C" int sgi_device_count(void)
{
	int n = 0;
	if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
	return n;
}

namespace {

template <class G>
int chain_at(const G* g, int c0, uint32_t* out);

// Everything sgi_grid_create uploads and keeps on the host, built from the
// host grid: the device layout (records, components, containment tree,
// descent groups, chain table), the surplus forms and the host copies the
// launches need.  The layout cache stores it as it is.
struct GridImage
{
	unsigned flags = 0;
	int dim = 0, nno = 0, TD = 0, ld = 0, nlch = 0;
	float skip_floor = 0.f, f16_floor = 0.f;
	std::vector<uint32_t> rec, comps, coarse_index, aux, ctab, grp_a, grp_b, ninfo;
	std::vector<uint16_t> s16;
	std::vector<int> parent;
	std::vector<double> s64, s64c;
	std::vector<float> s32, rowmax;
	std::vector<int> parent_h;
	std::vector<uint32_t> skip_h, depth_h, gfirst_h, gcount_h, gcmin_h, gpmax_h;
	sgi_grid_info info{};
};

// IEEE binary16 bits of v, rounded to nearest (ties to even); |v| < 65504.
uint16_t half_bits(double v)
{
	const uint16_t sign = std::signbit(v) ? 0x8000u : 0u;
	const double a = fabs(v);
	if (a == 0.0) return sign;
	int ex = 0;
	frexp(a, &ex);                                 // a in [2^(ex-1), 2^ex)
	if (ex - 1 >= -14)
	{
		double m = nearbyint(ldexp(a, 11 - ex));   // 11 significant bits, in [1024, 2048]
		int e = ex - 1;
		if (m >= 2048.0) { m = 1024.0; e++; }
		return (uint16_t)(sign | ((e + 15) << 10) | ((int)m - 1024));
	}
	const double q = nearbyint(ldexp(a, 24));     // subnormal: multiples of 2^-24
	return (uint16_t)(sign | (int)q);              // q == 1024 is the smallest normal's bits
}

int build_image(const HostGrid& g, unsigned flags, GridImage& im)
{
	if (g.nno > 0x7fffffff - 64) return fail(SGI_E_RANGE, "too many nodes");
	DeviceLayout L;
	int rc = build_layout(g, L);
	if (rc) return rc;
	im.flags = flags;
	im.dim = g.dim; im.nno = g.nno; im.TD = g.TotalDof;
	// row stride: 32 for TotalDof <= 32 (a lane per output), else a multiple
	// of 64 (a lane per output pair per 64 columns)
	im.ld = g.TotalDof <= 32 ? 32 : (g.TotalDof + 63) / 64 * 64;
	const size_t nrow = (size_t)std::max(g.nno, 1);
	im.rec = L.rec; im.comps = L.comps; im.coarse_index = L.lo_index; im.parent = L.parent; im.aux = L.aux;
	im.parent_h = L.parent;
	im.skip_h.resize(g.nno);
	im.depth_h.resize(g.nno);
	for (int n = 0; n < g.nno; n++) { im.skip_h[n] = L.rec[4 * (size_t)n]; im.depth_h[n] = L.aux[2 * (size_t)n + 1]; }
	if (g.nno > 0)
	{
		im.nlch = (g.nno + LCS - 1) / LCS;
		im.ctab.assign((size_t)im.nlch * 32, 0u);
		for (int k = 0; k < im.nlch; k++)
			im.ctab[(size_t)k * 32] = (uint32_t)chain_at(&im, k * LCS, &im.ctab[(size_t)k * 32 + 1]);
	}
	if (!(flags & SGI_BUILD_NO_FP64))
	{
		im.s64.assign(nrow * im.ld, 0.0);
		for (int n = 0; n < g.nno; n++)
			memcpy(&im.s64[(size_t)n * im.ld], &g.surplus[(size_t)n * g.TotalDof], sizeof(double) * g.TotalDof);
	}
	if (flags & (SGI_BUILD_FP32 | SGI_BUILD_NO_FP64))
	{
		im.s32.assign(nrow * im.ld, 0.f);
		im.s64c.assign((size_t)std::max(L.ncoarse, 1) * im.ld, 0.0);
		for (int n = 0; n < g.nno; n++)
			for (int o = 0; o < g.TotalDof; o++)
			{
				const double v = g.surplus[(size_t)n * g.TotalDof + o];
				im.s32[(size_t)n * im.ld + o] = (float)v;
				if (L.lo_index[n] != ~0u) im.s64c[(size_t)L.lo_index[n] * im.ld + o] = v;
			}
		// row maxima for the FP32C form's negligible-term test: a fine term is
		// dropped when |w| * max|s_row| < 2^-42 * max|s|
		im.rowmax.assign(nrow, 0.f);
		double smax = 0.0;
		for (int n = 0; n < g.nno; n++)
		{
			double m = 0.0;
			for (int o = 0; o < g.TotalDof; o++) m = std::max(m, fabs(g.surplus[(size_t)n * g.TotalDof + o]));
			im.rowmax[n] = (float)(m * (1.0 + 0x1.0p-20));   // rounded up
			smax = std::max(smax, m);
		}
		im.skip_floor = (float)(ldexp(smax, -42));
		// FP16 rows for fine terms whose bound is below 2^-29 * max|s| (each
		// such term then carries at most 2^-11 of its bound, below 2^-40 *
		// max|s|, in rounding: no more than an FP32 row gives the largest fine
		// terms, 2^-24 of a bound below 2^-16 * max|s|), on
		// grids whose passes are all 256 outputs wide (the rows' lane layout)
		// and whose row maxima keep the weight scaling a normal FP32 number
		if (im.ld % 256 == 0 && smax >= 0x1p-60 && smax < 0x1p100)
		{
			static const double f16_rel = []()
			{
				const char* e = getenv("SGI_F16_REL");
				return e ? atof(e) : 0x1.0p-29;
			}();
			im.f16_floor = (float)(smax * f16_rel);
			im.s16.assign(nrow * im.ld, 0u);
			for (int n = 0; n < g.nno; n++)
			{
				if (im.rowmax[n] <= 0.f) continue;
				int ex = 0;
				frexp((double)im.rowmax[n], &ex);          // rowmax in [2^(ex-1), 2^ex)
				const int k = 14 - (ex - 1);
				const double* src = &g.surplus[(size_t)n * g.TotalDof];
				uint16_t* dst = &im.s16[(size_t)n * im.ld];
				for (int o = 0; o < g.TotalDof; o++)
				{
					const int b = o >> 8, r = o & 255, v = r >> 7, l = (r & 127) >> 2, e = r & 3;
					dst[b * 256 + l * 8 + v * 4 + e] = half_bits(ldexp(src[o], k));
				}
			}
		}
		// descent layout: groups, and per node (plus the roots' virtual
		// parent at index nno) {first group, group count, rowmax, FP64 copy row}
		DescentLayout D;
		rc = build_descent(g, L, D);
		if (rc) return rc;
		const size_t ng = D.cmin.size();
		im.ninfo.resize((size_t)4 * (g.nno + 1));
		for (int n = 0; n <= g.nno; n++)
		{
			im.ninfo[4 * (size_t)n + 0] = D.first[n];
			im.ninfo[4 * (size_t)n + 1] = D.count[n];
			im.ninfo[4 * (size_t)n + 2] = n < g.nno ? float_bits(im.rowmax[n]) : 0u;
			im.ninfo[4 * (size_t)n + 3] = n < g.nno ? L.lo_index[n] : DESC_NONE;
		}
		im.grp_a = std::move(D.a);
		im.grp_b = std::move(D.b);
		im.gfirst_h = D.first;
		im.gcount_h = D.count;
		im.gcmin_h = D.cmin;
		im.gpmax_h.resize(ng);
		for (int n = 0; n <= g.nno; n++)
		{
			uint32_t m = 0;
			for (uint32_t q = D.first[n]; q < D.first[n] + D.count[n]; q++) { m = std::max(m, D.cmax[q]); im.gpmax_h[q] = m; }
		}
	}
	sgi_grid_info& I = im.info;
	I.dim = g.dim; I.nno = g.nno; I.TotalDof = g.TotalDof; I.ld = im.ld;
	I.max_comps = L.max_comps; I.tree_depth = L.tree_depth; I.tree_roots = L.tree_roots;
	I.multi_delta = L.multi_delta; I.ncoarse = L.ncoarse; I.comps = (long long)L.comps.size() / 2;
	I.device_bytes = 0; I.coarse_threshold = L.coarse_threshold;
	return SGI_OK;
}

// Uploads an image to `device` (moving its host copies into the grid).
int upload_image(GridImage& im, int device, sgi_grid_t* out)
{
	int ndev = sgi_device_count();
	if (ndev == 0) return fail(SGI_E_NODEVICE, "no CUDA device");
	if (device < 0 || device >= ndev) return fail(SGI_E_INVALID, "device %d out of range (%d devices)", device, ndev);
	DeviceGuard guard(device);
	sgi_grid* d = new sgi_grid;
	d->device = device; d->dim = im.dim; d->nno = im.nno; d->TD = im.TD; d->ld = im.ld;
	long long bytes = 0;
	auto upload = [&](void** dst, const void* src, size_t n) -> int
	{
		cudaError_t e = cudaMalloc(dst, std::max<size_t>(n, 16));
		if (e != cudaSuccess) return fail(SGI_E_NOMEM, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
		bytes += (long long)n;
		if (n && src)
		{
			e = cudaMemcpy(*dst, src, n, cudaMemcpyHostToDevice);
			if (e != cudaSuccess) return fail(SGI_E_CUDA, "cudaMemcpy failed: %s", cudaGetErrorString(e));
		}
		return SGI_OK;
	};
	int rc = upload((void**)&d->rec, im.rec.data(), im.rec.size() * 4);
	if (!rc) rc = upload((void**)&d->comps, im.comps.data(), im.comps.size() * 4);
	if (!rc) rc = upload((void**)&d->coarse_index, im.coarse_index.data(), im.coarse_index.size() * 4);
	if (!rc) rc = upload((void**)&d->parent, im.parent.data(), im.parent.size() * 4);
	if (!rc) rc = upload((void**)&d->aux, im.aux.data(), im.aux.size() * 4);
	if (!rc && im.nno > 0) rc = upload((void**)&d->ctab, im.ctab.data(), im.ctab.size() * 4);
	if (!rc && !im.s16.empty()) rc = upload((void**)&d->s16, im.s16.data(), im.s16.size() * 2);
	if (!rc && !im.s64.empty()) rc = upload((void**)&d->s64, im.s64.data(), im.s64.size() * 8);
	if (!rc && !im.s32.empty())
	{
		rc = upload((void**)&d->s32, im.s32.data(), im.s32.size() * 4);
		if (!rc) rc = upload((void**)&d->s64c, im.s64c.data(), im.s64c.size() * 8);
		if (!rc) rc = upload((void**)&d->rowmax, im.rowmax.data(), im.rowmax.size() * 4);
		if (!rc) rc = upload((void**)&d->grp_a, im.grp_a.data(), im.grp_a.size() * 4);
		if (!rc) rc = upload((void**)&d->grp_b, im.grp_b.data(), im.grp_b.size() * 4);
		if (!rc) rc = upload((void**)&d->ninfo, im.ninfo.data(), im.ninfo.size() * 4);
	}
	if (rc) { free_grid(d); return rc; }
	d->nlch = im.nlch;
	d->skip_floor = d->skip_below = im.skip_floor;
	d->f16_floor = im.f16_floor;
	d->parent_h = std::move(im.parent_h);
	d->skip_h = std::move(im.skip_h);
	d->depth_h = std::move(im.depth_h);
	d->gfirst_h = std::move(im.gfirst_h);
	d->gcount_h = std::move(im.gcount_h);
	d->gcmin_h = std::move(im.gcmin_h);
	d->gpmax_h = std::move(im.gpmax_h);
	d->info = im.info;
	d->info.device_bytes = bytes;
	*out = d;
	return SGI_OK;
}

// ------------------------------------------------------------ layout cache
//
// File: magic, format version, build flags, the .plt's size and modification
// time (ns), then the image's scalars and arrays (element count, then the
// raw elements, in a fixed order), then a 64-bit sum of every 8-byte word
// written before it.  Native byte order: a cache is read back on the machine
// (or an identical one) that wrote it.
constexpr char CACHE_MAGIC[8] = { 'S', 'G', 'I', 'L', 'A', 'Y', 'O', 'T' };
constexpr uint32_t CACHE_VERSION = 3;

struct CacheKey
{
	int64_t size = 0, mtime_ns = 0;
};

int plt_key(const char* path, CacheKey* k)
{
	struct stat st;
	if (stat(path, &st)) return fail(SGI_E_FORMAT, "Error opening file: %s", path);
	k->size = (int64_t)st.st_size;
	k->mtime_ns = (int64_t)st.st_mtim.tv_sec * 1000000000ll + st.st_mtim.tv_nsec;
	return SGI_OK;
}

std::string cache_file(const char* path, const char* cache_path)
{
	return cache_path ? std::string(cache_path) : std::string(path) + ".sgi-layout";
}

struct CacheWriter
{
	FILE* f;
	uint64_t sum = 0;
	bool ok = true;
	std::vector<unsigned char> pend;   // bytes not yet summed (partial word)
	void raw(const void* p, size_t n)
	{
		if (!n) return;
		if (fwrite(p, 1, n, f) != n) ok = false;
		const unsigned char* c = (const unsigned char*)p;
		size_t i = 0;
		if (!pend.empty())
		{
			while (i < n && pend.size() < 8) pend.push_back(c[i++]);
			if (pend.size() < 8) return;
			uint64_t w; memcpy(&w, pend.data(), 8); sum += w; pend.clear();
		}
		for (; i + 8 <= n; i += 8) { uint64_t w; memcpy(&w, c + i, 8); sum += w; }
		while (i < n) pend.push_back(c[i++]);
	}
	template <class T> void val(const T& v) { raw(&v, sizeof(T)); }
	template <class T> void vec(const std::vector<T>& v) { val((uint64_t)v.size()); raw(v.data(), v.size() * sizeof(T)); }
	// the sum with a trailing partial word zero-padded
	uint64_t total()
	{
		uint64_t t = sum;
		if (!pend.empty()) { unsigned char w8[8] = {0}; memcpy(w8, pend.data(), pend.size()); uint64_t w; memcpy(&w, w8, 8); t += w; }
		return t;
	}
};

struct CacheReader
{
	FILE* f;
	uint64_t sum = 0;
	bool ok = true;
	std::vector<unsigned char> pend;
	int64_t left;
	void raw(void* p, size_t n)
	{
		if (!ok || !n) return;
		if ((int64_t)n > left || fread(p, 1, n, f) != n) { ok = false; return; }
		left -= (int64_t)n;
		const unsigned char* c = (const unsigned char*)p;
		size_t i = 0;
		if (!pend.empty())
		{
			while (i < n && pend.size() < 8) pend.push_back(c[i++]);
			if (pend.size() < 8) return;
			uint64_t w; memcpy(&w, pend.data(), 8); sum += w; pend.clear();
		}
		for (; i + 8 <= n; i += 8) { uint64_t w; memcpy(&w, c + i, 8); sum += w; }
		while (i < n) pend.push_back(c[i++]);
	}
	template <class T> void val(T& v) { raw(&v, sizeof(T)); }
	template <class T> void vec(std::vector<T>& v)
	{
		uint64_t n = 0;
		val(n);
		if (!ok || n * sizeof(T) > (uint64_t)left) { ok = false; return; }
		v.resize(n);
		raw(v.data(), n * sizeof(T));
	}
	uint64_t total()
	{
		uint64_t t = sum;
		if (!pend.empty()) { unsigned char w8[8] = {0}; memcpy(w8, pend.data(), pend.size()); uint64_t w; memcpy(&w, w8, 8); t += w; }
		return t;
	}
};

template <class IO, class Image>
void cache_fields(IO& io, Image& im)
{
	io.val(im.dim); io.val(im.nno); io.val(im.TD); io.val(im.ld); io.val(im.nlch); io.val(im.skip_floor);
	io.val(im.f16_floor);
	auto& I = im.info;
	io.val(I.dim); io.val(I.nno); io.val(I.TotalDof); io.val(I.ld); io.val(I.max_comps); io.val(I.tree_depth);
	io.val(I.tree_roots); io.val(I.multi_delta); io.val(I.ncoarse); io.val(I.comps); io.val(I.device_bytes);
	io.val(I.coarse_threshold);
	io.vec(im.rec); io.vec(im.comps); io.vec(im.coarse_index); io.vec(im.aux); io.vec(im.ctab);
	io.vec(im.grp_a); io.vec(im.grp_b); io.vec(im.ninfo); io.vec(im.parent);
	io.vec(im.s64); io.vec(im.s64c); io.vec(im.s32); io.vec(im.rowmax); io.vec(im.s16);
	io.vec(im.parent_h); io.vec(im.skip_h); io.vec(im.depth_h);
	io.vec(im.gfirst_h); io.vec(im.gcount_h); io.vec(im.gcmin_h); io.vec(im.gpmax_h);
}

// Writes the cache through a temporary file renamed into place, so that a
// reader never sees a partial file.
int write_cache(const GridImage& im, const CacheKey& key, const std::string& file)
{
	const std::string tmp = file + ".tmp" + std::to_string((long long)getpid());
	FILE* f = fopen(tmp.c_str(), "wb");
	if (!f) return fail(SGI_E_FORMAT, "cannot create %s", tmp.c_str());
	setvbuf(f, nullptr, _IOFBF, 1 << 22);
	CacheWriter w{ f };
	w.raw(CACHE_MAGIC, 8);
	w.val(CACHE_VERSION); w.val(im.flags); w.val(key.size); w.val(key.mtime_ns);
	cache_fields(w, const_cast<GridImage&>(im));
	const uint64_t sum = w.total();
	w.pend.clear();
	w.val(sum);
	if (fclose(f)) w.ok = false;
	if (!w.ok || rename(tmp.c_str(), file.c_str()))
	{
		unlink(tmp.c_str());
		return fail(SGI_E_FORMAT, "cannot write the layout cache %s", file.c_str());
	}
	return SGI_OK;
}

// True (and the image filled) when `file` is a complete cache of this format
// version for these build flags and this .plt key.
bool read_cache(const std::string& file, unsigned flags, const CacheKey& key, GridImage& im)
{
	FILE* f = fopen(file.c_str(), "rb");
	if (!f) return false;
	setvbuf(f, nullptr, _IOFBF, 1 << 22);
	struct stat st;
	if (fstat(fileno(f), &st)) { fclose(f); return false; }
	CacheReader r{ f };
	r.left = (int64_t)st.st_size;
	char magic[8];
	uint32_t version = 0, fl = 0;
	CacheKey k;
	r.raw(magic, 8);
	r.val(version); r.val(fl); r.val(k.size); r.val(k.mtime_ns);
	bool ok = r.ok && !memcmp(magic, CACHE_MAGIC, 8) && version == CACHE_VERSION && fl == flags &&
		k.size == key.size && k.mtime_ns == key.mtime_ns;
	if (ok)
	{
		cache_fields(r, im);
		const uint64_t sum = r.total();
		r.pend.clear();
		uint64_t stored = 0;
		r.val(stored);
		ok = r.ok && stored == sum && r.left == 0;
	}
	fclose(f);
	if (ok) im.flags = flags;
	return ok;
}

int image_from_plt(const char* path, int nagents, unsigned flags, GridImage& im)
{
	sgi_host_grid_t hg = nullptr;
	int rc = sgi_host_grid_read_plt(path, nagents, &hg);
	if (rc) return rc;
	rc = build_image(hg->g, flags, im);
	sgi_host_grid_free(hg);
	return rc;
}

} // namespace

extern "C" int sgi_grid_create(sgi_host_grid_t hg, int device, unsigned flags, sgi_grid_t* out)
{
	clear_error();
	if (!hg || !out) return fail(SGI_E_INVALID, "null argument");
	*out = nullptr;
	int ndev = sgi_device_count();
	if (ndev == 0) return fail(SGI_E_NODEVICE, "no CUDA device");
	if (device < 0 || device >= ndev) return fail(SGI_E_INVALID, "device %d out of range (%d devices)", device, ndev);
	GridImage im;
	int rc = build_image(hg->g, flags, im);
	if (rc) return rc;
	return upload_image(im, device, out);
}

extern "C" int sgi_grid_load(const char* path, int nagents, int device, unsigned flags, const char* cache_path,
	sgi_grid_t* out, int* hit)
{
	clear_error();
	if (!path || !out) return fail(SGI_E_INVALID, "null argument");
	*out = nullptr;
	if (hit) *hit = 0;
	int ndev = sgi_device_count();
	if (ndev == 0) return fail(SGI_E_NODEVICE, "no CUDA device");
	if (device < 0 || device >= ndev) return fail(SGI_E_INVALID, "device %d out of range (%d devices)", device, ndev);
	CacheKey key;
	int rc = plt_key(path, &key);
	if (rc) return rc;
	const std::string file = cache_file(path, cache_path);
	GridImage im;
	if (read_cache(file, flags, key, im) && im.dim == nagents)
	{
		if (hit) *hit = 1;
		return upload_image(im, device, out);
	}
	im = GridImage{};
	rc = image_from_plt(path, nagents, flags, im);
	if (rc) return rc;
	if (write_cache(im, key, file)) clear_error();   // a cache that cannot be written is not an error
	return upload_image(im, device, out);
}

extern "C" int sgi_grid_cache_write(const char* path, int nagents, unsigned flags, const char* cache_path)
{
	clear_error();
	if (!path) return fail(SGI_E_INVALID, "null argument");
	CacheKey key;
	int rc = plt_key(path, &key);
	if (rc) return rc;
	GridImage im;
	rc = image_from_plt(path, nagents, flags, im);
	if (rc) return rc;
	return write_cache(im, key, cache_file(path, cache_path));
}

extern "C" int sgi_grid_cache_valid(const char* path, int nagents, unsigned flags, const char* cache_path)
{
	clear_error();
	if (!path) return fail(SGI_E_INVALID, "null argument");
	CacheKey key;
	int rc = plt_key(path, &key);
	if (rc) return rc;
	GridImage im;
	return read_cache(cache_file(path, cache_path), flags, key, im) && im.dim == nagents ? 1 : 0;
}

extern "C" int sgi_grid_info_get(sgi_grid_t g, sgi_grid_info* info)
{
	clear_error();
	if (!g || !info) return fail(SGI_E_INVALID, "null argument");
	*info = g->info;
	return SGI_OK;
}

extern "C" void sgi_grid_destroy(sgi_grid_t g) { free_grid(g); }

extern "C" int sgi_grid_set_surplus_cutoff(sgi_grid_t g, double cutoff, double* effective)
{
	clear_error();
	if (!g) return fail(SGI_E_INVALID, "null grid");
	if (!g->s32) return fail(SGI_E_INVALID, "surplus cutoff: the grid has no FP32 form (build with SGI_BUILD_FP32)");
	if (std::isnan(cutoff)) return fail(SGI_E_INVALID, "surplus cutoff is NaN");
	// compared in FP32 with bounds computed in FP32; a cutoff above the FP32
	// range skips every term that is not big
	const float c = cutoff > (double)FLT_MAX ? INFINITY : (float)cutoff;
	g->skip_below = std::max(g->skip_floor, c);
	if (effective) *effective = g->skip_below;
	return SGI_OK;
}

extern "C" int sgi_set_chunk_rows(int rows)
{
	const int prev = g_chunk_override.load();
	g_chunk_override.store(rows < 0 ? -1 : rows);
	return prev;
}

extern "C" int sgi_set_fp32c_variant(int variant)
{
	clear_error();
	if (variant >= NVARIANTS_ALL && variant != SGI_FP32C_AUTO)
		return fail(SGI_E_INVALID, "FP32C variant %d out of range (0..%d, or SGI_FP32C_AUTO)", variant, NVARIANTS_ALL - 1);
	const int prev = g_variant.exchange(variant < 0 || variant == SGI_FP32C_AUTO ? -1 : variant);
	return prev < 0 ? SGI_FP32C_AUTO : prev;
}

extern "C" int sgi_last_launch(sgi_launch_stats* s)
{
	if (!s) return fail(SGI_E_INVALID, "null argument");
	*s = g_stats;
	return SGI_OK;
}

namespace {

int check_set(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets)
{
	if (ngrids < 1 || !grids || !pt_offsets) return fail(SGI_E_INVALID, "empty grid set");
	for (int k = 0; k < ngrids; k++)
	{
		if (!grids[k]) return fail(SGI_E_INVALID, "grid %d is null", k);
		if (grids[k]->device != grids[0]->device) return fail(SGI_E_INVALID, "grids on different devices");
		if (grids[k]->dim != grids[0]->dim)
			return fail(SGI_E_MISMATCH, "state %d has dim %d, state 0 has %d", k, grids[k]->dim, grids[0]->dim);
		if (grids[k]->TD != grids[0]->TD)
			return fail(SGI_E_MISMATCH, "state %d TotalDof (%d) mismatches state 0 (%d)", k, grids[k]->TD, grids[0]->TD);
		if (pt_offsets[k + 1] < pt_offsets[k]) return fail(SGI_E_INVALID, "point offsets decrease at %d", k);
	}
	if (pt_offsets[0] != 0) return fail(SGI_E_INVALID, "pt_offsets[0] must be 0");
	return SGI_OK;
}

// Ancestor chain of a node-chunk start c0: the nodes p < c0 whose subtree
// range [p, skip[p]) reaches past c0, stored by depth (out[d - 1] is the one
// at depth d, d = 1..CHAIN); returns the number stored.  The tree parent of
// every chunk root (a node at or after c0 whose parent precedes c0) is in
// this chain: its range holds both the parent and the chunk root.  The chain
// is the part of the ancestor path of the last live node before c0 that is
// still open at c0; every ancestor of an open node is open, so the stored
// depths run from 1 without gaps.
template <class G>
int chain_at(const G* g, int c0, uint32_t* out)
{
	if (c0 <= 0 || c0 >= g->nno) return 0;
	int q = c0 - 1;
	while (q >= 0 && g->depth_h[q] == 0) q--;   // dead nodes are outside the tree
	uint32_t filled = 0;
	for (; q >= 0; q = g->parent_h[q])
		if (g->skip_h[q] > (uint32_t)c0)
		{
			const uint32_t d = g->depth_h[q];
			if (d >= 1 && d <= (uint32_t)CHAIN) { out[d - 1] = (uint32_t)q; filled |= 1u << (d - 1); }
		}
	// depths 1..len, stopping at a gap (none in a tree; kept as a guard)
	int len = 0;
	while (len < CHAIN && ((filled >> len) & 1u)) len++;
	return len;
}

// Group range of node n (n = nno: the roots' virtual parent) that may hold
// children in [lo, hi): a node's groups are ordered by their smallest child,
// so the range runs from the first group whose running largest child reaches
// lo to the first group whose smallest child is at or past hi (a superset:
// the kernel tests every child against the range).
uint2 group_range(const sgi_grid* g, int n, int lo, int hi)
{
	const uint32_t b = g->gfirst_h[n], e = b + g->gcount_h[n];
	const uint32_t* pm = g->gpmax_h.data();
	const uint32_t* cm = g->gcmin_h.data();
	const uint32_t s = (uint32_t)(std::lower_bound(pm + b, pm + e, (uint32_t)lo) - pm);
	const uint32_t t = (uint32_t)(std::lower_bound(cm + b, cm + e, (uint32_t)hi) - cm);
	return make_uint2(s, std::max(s, t));
}

// Walk starts of a launch over grids[gb .. gb + ng) for the node range set in
// a (chunk_begin, chunk_len): the ancestor chain of the range start and, for
// the descent layout, the group ranges of the chain nodes and of the roots.
void set_starts(FwdArgs& a, const sgi_grid_t* grids, int gb, int ng)
{
	for (int k = 0; k < ng; k++)
	{
		const sgi_grid* g = grids[gb + k];
		a.chain_len[k] = chain_at(g, a.chunk_begin, a.chain[k]);
		a.rseg[k] = make_uint2(0u, 0u);
		if (g->gfirst_h.empty()) continue;
		const int lo = a.chunk_begin;
		const int hi = a.chunk_len ? (int)std::min((long long)g->nno, (long long)a.chunk_begin + a.chunk_len) : g->nno;
		if (lo >= hi) continue;
		a.rseg[k] = group_range(g, g->nno, lo, hi);
		for (int d = 0; d < a.chain_len[k]; d++) a.cseg[k][d] = group_range(g, (int)a.chain[k][d], lo, hi);
	}
}

// The FP32C descent needs every grid of the launch to have its layout and a
// tree shallow enough for the stack bound, and for chunked launches for
// complete ancestor chains.
bool descent_ok(const sgi_grid_t* grids, int gb, int ng, bool chunked)
{
	for (int k = 0; k < ng; k++)
	{
		const sgi_grid* g = grids[gb + k];
		if (!g->grp_a || g->gfirst_h.empty()) return false;
		const int dep = g->info.tree_depth;
		if (dep > SCAP - 32 || (chunked && dep > CHAIN + 1)) return false;
	}
	return true;
}

// Node-chunk size of a launch group (chunk < 0: automatic).
int group_clen(const DeviceWork* W, const sgi_grid_t* grids, int gb, int ng, const long long* pt_offsets,
	int precision, int chunk)
{
	int maxnno = 0;
	for (int k = 0; k < ng; k++) maxnno = std::max(maxnno, grids[gb + k]->nno);
	return chunk < 0 ? chunk_rows(W, grids[0], precision, pt_offsets[gb + ng] - pt_offsets[gb], maxnno)
	                 : (chunk >= maxnno ? 0 : chunk);
}

// Scratch bytes of a launch group's hit lists when it runs the two-phase
// small-batch kernels (FP64, or FP32C on grids that keep their FP64 rows; not
// node-chunked; fewer points than resident warps; lists within
// LIST_SCRATCH_MAX), else 0.
constexpr size_t LIST_SCRATCH_MAX = 256ull << 20;

size_t list_scratch(const DeviceWork* W, const sgi_grid_t* grids, int gb, int ng, const long long* pt_offsets,
	int precision, int clen)
{
	const long long np = pt_offsets[gb + ng] - pt_offsets[gb];
	if ((precision != SGI_FP64 && precision != SGI_FP32C) || clen || np == 0 || np >= (long long)W->sms * WARPS)
		return 0;
	long long items = 0;
	for (int k = 0; k < ng; k++)
	{
		if (!grids[gb + k]->s64) return 0;
		items += (pt_offsets[gb + k + 1] - pt_offsets[gb + k]) * grids[gb + k]->nlch;
	}
	if (items == 0) return 0;
	const size_t bytes = (((size_t)items * 4 + 255) & ~(size_t)255) + (size_t)items * LCS * 12;
	return bytes <= LIST_SCRATCH_MAX ? bytes : 0;
}

// The two launches of a two-phase group; buf holds list_scratch() bytes.
int launch_lists(const DeviceWork* W, const sgi_grid_t* grids, int gb, int ng, const long long* pt_offsets,
	const double* x, double* out, int precision, char* buf, cudaStream_t stream, int* phase2_blocks)
{
	const sgi_grid* g0 = grids[0];
	const long long p0 = pt_offsets[gb];
	ListArgs la;
	memset(&la, 0, sizeof(la));
	long long items = 0;
	for (int k = 0; k < ng; k++)
	{
		const sgi_grid* g = grids[gb + k];
		la.g[k] = desc_of(g, pt_offsets[gb + k] - p0, precision);
		la.ctab[k] = g->ctab;
		la.nch[k] = g->nlch;
		la.ibeg[k] = items;
		items += (pt_offsets[gb + k + 1] - pt_offsets[gb + k]) * g->nlch;
	}
	la.ibeg[ng] = items;
	la.x = x + (size_t)p0 * g0->dim;
	la.out = out + (size_t)p0 * g0->TD;
	la.npts = pt_offsets[gb + ng] - p0;
	la.ngrids = ng; la.dim = g0->dim; la.TD = g0->TD;
	la.hcnt = reinterpret_cast<uint32_t*>(buf);
	la.hnode = reinterpret_cast<uint32_t*>(buf + (((size_t)items * 4 + 255) & ~(size_t)255));
	la.hw = reinterpret_cast<double*>(la.hnode + (size_t)items * LCS);
	const size_t sm1 = (size_t)WARPS * g0->dim * sizeof(double);
	int b1 = 0;
	int rc = occupancy_grid(walk_chunks_kernel, sm1, W->sms, &b1);
	if (rc) return rc;
	b1 = (int)std::min<long long>(b1, (items + WARPS - 1) / WARPS);
	walk_chunks_kernel<<<b1, BLOCK, sm1, stream>>>(la);
	CUDA_TRY(cudaGetLastError());
	const size_t sm2 = (size_t)(LBLOCK / 32) * list_stride() * sizeof(double);
	CUDA_TRY(cudaFuncSetAttribute(fwd_f64_list_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
	int b2 = 0;
	rc = occupancy_grid(fwd_f64_list_kernel, sm2, W->sms, &b2, LBLOCK);
	if (rc) return rc;
	const long long items2 = la.npts * ((g0->TD + 31) / 32);
	b2 = (int)std::min<long long>(b2, (items2 + LBLOCK / 32 - 1) / (LBLOCK / 32));
	fwd_f64_list_kernel<<<b2, LBLOCK, sm2, stream>>>(la);
	CUDA_TRY(cudaGetLastError());
	*phase2_blocks = b2;
	return SGI_OK;
}

// Pool memory handed back on the stream when the scope ends.
struct PoolScratch
{
	char* p = nullptr;
	cudaStream_t s = nullptr;
	~PoolScratch() { if (p) cudaFreeAsync(p, s); }
};

// Launches of one forward call.  chunk < 0: the automatic chunk size; work
// counters come from `counters` (one per launch, in order) when given, else
// from the device workspace's ring.  Two-phase small-batch groups take their
// hit lists from `scratch` when given (plans), else from the device's pool;
// while the stream is being captured without scratch they run the one-phase
// kernels instead.
int launch_forward(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets, const double* x,
	double* out, int precision, cudaStream_t stream, int chunk = -1, unsigned long long* counters = nullptr,
	int* nlaunch = nullptr, int variant = -1, char* scratch = nullptr, size_t scratch_bytes = 0)
{
	if (variant < 0) variant = g_variant.load();   // may stay -1: automatic per launch group
	const sgi_grid* g0 = grids[0];
	DeviceWork* W = nullptr;
	int rc = device_work(g0->device, &W);
	if (rc) return rc;
	if (precision == SGI_FP64) { for (int k = 0; k < ngrids; k++) if (!grids[k]->s64) return fail(SGI_E_INVALID, "grid %d has no FP64 surplus", k); }
	else if (precision == SGI_FP32C) { for (int k = 0; k < ngrids; k++) if (!grids[k]->s32) return fail(SGI_E_INVALID, "grid %d was built without SGI_BUILD_FP32", k); }
	else return fail(SGI_E_INVALID, "unknown precision %d", precision);
	// per warp: the point's coordinates, and for FP32C the term list and the
	// weight stack (window walk) or the group-range stack (descent)
	if (fwd_smem(precision, g0->dim, true) > 200 * 1024) return fail(SGI_E_RANGE, "dim %d too large for shared staging", g0->dim);
	g_stats = sgi_launch_stats{};
	size_t lneed = 0;
	for (int gb = 0; gb < ngrids; gb += MAXG)
	{
		const int ng = std::min(MAXG, ngrids - gb);
		lneed = std::max(lneed, list_scratch(W, grids, gb, ng, pt_offsets, precision,
		                                     group_clen(W, grids, gb, ng, pt_offsets, precision, chunk)));
	}
	PoolScratch pooled;
	char* lbuf = nullptr;
	if (lneed)
	{
		if (scratch) lbuf = scratch_bytes >= lneed ? scratch : nullptr;
		else
		{
			cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
			CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
			if (cap == cudaStreamCaptureStatusNone)
			{
				cudaMemPool_t pool = nullptr;
				rc = scratch_pool(W, g0->device, &pool);
				if (rc) return rc;
				void* pbuf = nullptr;
				if (cudaMallocFromPoolAsync(&pbuf, lneed, pool, stream) == cudaSuccess)
				{
					lbuf = static_cast<char*>(pbuf);
					pooled.p = lbuf;
					pooled.s = stream;
				}
				else cudaGetLastError();   // no room: the one-phase kernels
			}
		}
	}
	int launches = 0;
	for (int gb = 0; gb < ngrids; gb += MAXG)
	{
		const int ng = std::min(MAXG, ngrids - gb);
		const long long p0 = pt_offsets[gb], p1 = pt_offsets[gb + ng];
		if (p1 == p0) continue;
		if (lbuf)
		{
			const int gclen = group_clen(W, grids, gb, ng, pt_offsets, precision, chunk);
			if (list_scratch(W, grids, gb, ng, pt_offsets, precision, gclen))
			{
				int b2 = 0;
				rc = launch_lists(W, grids, gb, ng, pt_offsets, x, out, precision, lbuf, stream, &b2);
				if (rc) return rc;
				launches += 2;
				g_stats.kernels += 2;
				g_stats.grid_blocks = b2;
				g_stats.block_threads = LBLOCK;
				g_stats.points += p1 - p0;
				continue;
			}
		}
		FwdArgs a;
		memset(&a, 0, sizeof(a));
		for (int k = 0; k < ng; k++) a.g[k] = desc_of(grids[gb + k], pt_offsets[gb + k] - p0, precision);
		a.x = x + (size_t)p0 * g0->dim;
		a.out = out + (size_t)p0 * g0->TD;
		a.npts = p1 - p0;
		a.ngrids = ng; a.dim = g0->dim; a.TD = g0->TD;
		int maxnno = 0;
		for (int k = 0; k < ng; k++) maxnno = std::max(maxnno, grids[gb + k]->nno);
		const int clen = group_clen(W, grids, gb, ng, pt_offsets, precision, chunk);
		const int nchunks = clen ? (maxnno + clen - 1) / clen : 1;
		const bool descent = precision == SGI_FP32C && descent_ok(grids, gb, ng, clen > 0);
		const bool small = a.npts < (long long)W->sms * WARPS;
		// small unchunked FP64 batches: one warp per (point, 32 outputs)
		const bool cols_mode = precision == SGI_FP64 && small && clen == 0;
		const size_t smem = cols_mode ? (size_t)WARPS * cols_stride(g0->dim) * sizeof(double)
		                              : fwd_smem(precision, g0->dim, descent);
		for (int ob = 0; ob < g0->TD; ob += PASS)
		for (int c = 0; c < std::max(nchunks, 1); c++)
		{
			a.o_begin = ob;
			a.chunk_begin = c * clen;
			a.chunk_len = clen;
			set_starts(a, grids, gb, ng);
			a.counter = counters ? counters + launches : W->counters + (W->next.fetch_add(1) % NCOUNTERS);
			CUDA_TRY(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream));
			const int cols = std::min(g0->TD - ob, PASS);
			void (*kern)(FwdArgs) = cols_mode ? fwd_f64_cols_kernel
				: select_fwd(precision, g0->ld, cols, auto_variant(variant, a.npts, W->sms), descent, small);
			if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
			int blocks = 0;
			rc = occupancy_grid(kern, smem, W->sms, &blocks);
			if (rc) return rc;
			const long long items = cols_mode ? a.npts * ((cols + 31) / 32) : a.npts;
			const long long need = (items + WARPS - 1) / WARPS;
			if (blocks > need) blocks = (int)need;
			kern<<<blocks, BLOCK, smem, stream>>>(a);
			CUDA_TRY(cudaGetLastError());
			launches++;
			g_stats.kernels++;
			g_stats.grid_blocks = blocks;
			g_stats.block_threads = BLOCK;
		}
		g_stats.points += a.npts;
	}
	if (nlaunch) *nlaunch = launches;
	return SGI_OK;
}

// Launch count of a forward call with chunk size `chunk` >= 0 (as
// launch_forward given the scratch its two-phase groups need), and that
// scratch in *list_bytes.
int count_launches(const DeviceWork* W, int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	int precision, int chunk, size_t* list_bytes)
{
	int n = 0;
	const int passes = (grids[0]->TD + PASS - 1) / PASS;
	*list_bytes = 0;
	for (int gb = 0; gb < ngrids; gb += MAXG)
	{
		const int ng = std::min(MAXG, ngrids - gb);
		if (pt_offsets[gb + ng] == pt_offsets[gb]) continue;
		int maxnno = 0;
		for (int k = 0; k < ng; k++) maxnno = std::max(maxnno, grids[gb + k]->nno);
		const int clen = chunk >= maxnno ? 0 : chunk;
		const size_t lb = list_scratch(W, grids, gb, ng, pt_offsets, precision, clen);
		*list_bytes = std::max(*list_bytes, lb);
		n += lb ? 2 : passes * (clen ? (maxnno + clen - 1) / clen : 1);
	}
	return n;
}

} // namespace

extern "C" int sgi_interpolate(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision, void* stream)
{
	clear_error();
	int rc = check_set(ngrids, grids, pt_offsets);
	if (rc) return rc;
	if (pt_offsets[ngrids] > 0 && (!x || !out)) return fail(SGI_E_INVALID, "null x or out");
	DeviceGuard guard(grids[0]->device);
	return launch_forward(ngrids, grids, pt_offsets, x, out, precision, (cudaStream_t)stream);
}

namespace {
// Host calls of the FP64 form with at most this many points replay a CUDA
// graph kept per call shape (defined with the plans below).
constexpr long long HOST_PLAN_MAX_POINTS = 256;
int host_plan_call(DeviceWork* W, int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, bool* done);
} // namespace

extern "C" int sgi_interpolate_host(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision)
{
	clear_error();
	int rc = check_set(ngrids, grids, pt_offsets);
	if (rc) return rc;
	const long long npts = pt_offsets[ngrids];
	if (npts > 0 && (!x || !out)) return fail(SGI_E_INVALID, "null x or out");
	if (npts == 0) return SGI_OK;
	const sgi_grid* g0 = grids[0];
	DeviceGuard guard(g0->device);
	DeviceWork* W = nullptr;
	rc = device_work(g0->device, &W);
	if (rc) return rc;
	std::lock_guard<std::mutex> lk(W->mtx);
	if (!W->stream)
	{
		CUDA_TRY(cudaStreamCreateWithFlags(&W->stream, cudaStreamNonBlocking));
		CUDA_TRY(cudaStreamCreateWithFlags(&W->copy_in, cudaStreamNonBlocking));
		CUDA_TRY(cudaStreamCreateWithFlags(&W->copy_out, cudaStreamNonBlocking));
		CUDA_TRY(cudaStreamCreateWithFlags(&W->stream2, cudaStreamNonBlocking));
		for (int k = 0; k < DeviceWork::NEV; k++)
		{
			CUDA_TRY(cudaEventCreateWithFlags(&W->ev_in[k], cudaEventDisableTiming));
			CUDA_TRY(cudaEventCreateWithFlags(&W->ev_done[k], cudaEventDisableTiming));
		}
	}
	const int D = g0->dim, TD = g0->TD;
	const size_t xb = (size_t)npts * D * sizeof(double), ob = (size_t)npts * TD * sizeof(double);
	if (W->dx_bytes < xb) { cudaFree(W->dx); W->dx = nullptr; W->dx_bytes = 0; CUDA_TRY(cudaMalloc(&W->dx, xb)); W->dx_bytes = xb; }
	if (W->dout_bytes < ob) { cudaFree(W->dout); W->dout = nullptr; W->dout_bytes = 0; CUDA_TRY(cudaMalloc(&W->dout, ob)); W->dout_bytes = ob; }
	if (precision == SGI_FP64 && npts <= HOST_PLAN_MAX_POINTS)
	{
		bool done = false;
		rc = host_plan_call(W, ngrids, grids, pt_offsets, x, out, &done);
		if (rc || done) return rc;
	}
	// With pinned host buffers the batch is cut into sub-batches whose copies
	// in and out overlap the other sub-batches' kernels (a copy stream each
	// way, and two compute streams that the sub-batches alternate between, so
	// that one sub-batch's launches fill the tails of the other's); with
	// pageable buffers the copies would block the host, so it runs as one.
	cudaPointerAttributes ax{}, ao{};
	const bool pinned = cudaPointerGetAttributes(&ax, x) == cudaSuccess && ax.type == cudaMemoryTypeHost &&
		cudaPointerGetAttributes(&ao, out) == cudaSuccess && ao.type == cudaMemoryTypeHost;
	cudaGetLastError();
	// sub-batches of about 128k points (at most 8): the first sub-batch's copy
	// in and the last one's copy out are all that the kernels do not hide,
	// while every sub-batch repeats all node-chunk launches, whose tails the
	// other compute stream fills (on d=59, 1M nodes, TotalDof 256, 1M
	// points, FP32C: 2 / 3 / 4 / 6 / 8 sub-batches took 114.9 / 106.2 /
	// 106.5 / 109.1 / 113.5 ms on one compute stream, 126.7 / 108.8 / 108.9 /
	// 104.4 / 101.0 ms on two, 102.8 ms for 8 on three; 10, 12 and 16 on two
	// 102.0, 101.5 and 105.5 ms).  With three or more, the first and the last
	// are half the size of the others: their exposed copies shrink while each
	// middle sub-batch's copy out still fits under the next one's kernels.
	const int nsub = !pinned ? 1 : (int)std::min(8ll, std::max(1ll, (npts + 64 * 1024) / (128 * 1024)));
	std::vector<long long> cut(nsub + 1);
	{
		const long long units = nsub >= 3 ? 2ll * nsub - 2 : nsub;   // weights 1, 2, ..., 2, 1
		long long acc = 0;
		cut[0] = 0;
		for (int b = 0; b < nsub; b++)
		{
			acc += (nsub >= 3 && b > 0 && b < nsub - 1) ? 2 : 1;
			cut[b + 1] = npts * acc / units;
		}
	}
	// the node chunks are chosen for the whole batch, so that sub-batches
	// below the chunking threshold are chunked as the batch would be
	int maxnno = 0;
	for (int k = 0; k < ngrids; k++) maxnno = std::max(maxnno, grids[k]->nno);
	const int chunk = chunk_rows(W, g0, precision, npts, maxnno);
	std::vector<sgi_grid_t> sg;
	std::vector<long long> so;
	for (int b = 0; b < nsub; b++)
	{
		const long long P0 = cut[b], P1 = cut[b + 1];
		if (P1 == P0) continue;
		cudaEvent_t ein = W->ev_in[b % DeviceWork::NEV], edone = W->ev_done[b % DeviceWork::NEV];
		CUDA_TRY(cudaMemcpyAsync(W->dx + (size_t)P0 * D, x + (size_t)P0 * D, (size_t)(P1 - P0) * D * sizeof(double),
			cudaMemcpyHostToDevice, W->copy_in));
		CUDA_TRY(cudaEventRecord(ein, W->copy_in));
		cudaStream_t cs = (b & 1) ? W->stream2 : W->stream;
		CUDA_TRY(cudaStreamWaitEvent(cs, ein, 0));
		// the grids overlapping [P0, P1), offsets relative to P0
		sg.clear();
		so.clear();
		for (int k = 0; k < ngrids; k++)
		{
			const long long lo = std::max(P0, pt_offsets[k]), hi = std::min(P1, pt_offsets[k + 1]);
			if (hi <= lo) continue;
			sg.push_back(grids[k]);
			so.push_back(lo - P0);
		}
		so.push_back(P1 - P0);
		rc = launch_forward((int)sg.size(), sg.data(), so.data(), W->dx + (size_t)P0 * D, W->dout + (size_t)P0 * TD,
			precision, cs, chunk);
		if (rc) return rc;
		CUDA_TRY(cudaEventRecord(edone, cs));
		CUDA_TRY(cudaStreamWaitEvent(W->copy_out, edone, 0));
		CUDA_TRY(cudaMemcpyAsync(out + (size_t)P0 * TD, W->dout + (size_t)P0 * TD, (size_t)(P1 - P0) * TD * sizeof(double),
			cudaMemcpyDeviceToHost, W->copy_out));
	}
	CUDA_TRY(cudaStreamSynchronize(W->copy_out));
	CUDA_TRY(cudaStreamSynchronize(W->stream));
	CUDA_TRY(cudaStreamSynchronize(W->stream2));
	return SGI_OK;
}

namespace {

int count_terms(sgi_grid_t g, long long npts, const double* x, long long* counts, long long* classes, void* stream)
{
	DeviceGuard guard(g->device);
	DeviceWork* W = nullptr;
	int rc = device_work(g->device, &W);
	if (rc) return rc;
	FwdArgs a;
	memset(&a, 0, sizeof(a));
	a.g[0] = desc_of(g, 0, classes ? SGI_FP32C : SGI_FP64);
	a.x = x; a.npts = npts; a.ngrids = 1; a.dim = g->dim; a.TD = g->TD;
	a.counter = W->counters + (W->next.fetch_add(1) % NCOUNTERS);
	cudaStream_t s = (cudaStream_t)stream;
	CUDA_TRY(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), s));
	const size_t smem = (size_t)WARPS * g->dim * sizeof(double);
	void (*kern)(FwdArgs, long long*, long long*) = classes ? count_kernel<true> : count_kernel<false>;
	if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int blocks = 0;
	rc = occupancy_grid(kern, smem, W->sms, &blocks);
	if (rc) return rc;
	kern<<<blocks, BLOCK, smem, s>>>(a, counts, classes);
	CUDA_TRY(cudaGetLastError());
	return SGI_OK;
}

} // namespace

extern "C" int sgi_active_count(sgi_grid_t g, long long npts, const double* x, long long* out, void* stream)
{
	clear_error();
	if (!g || npts < 0 || (npts && (!x || !out))) return fail(SGI_E_INVALID, "bad arguments");
	if (!npts) return SGI_OK;
	return count_terms(g, npts, x, out, nullptr, stream);
}

extern "C" int sgi_term_classes(sgi_grid_t g, long long npts, const double* x, long long* out, void* stream)
{
	clear_error();
	if (!g || npts < 0 || (npts && (!x || !out))) return fail(SGI_E_INVALID, "bad arguments");
	if (!g->s32) return fail(SGI_E_INVALID, "term classes: the grid has no FP32 form (build with SGI_BUILD_FP32)");
	if (!npts) return SGI_OK;
	return count_terms(g, npts, x, nullptr, out, stream);
}

extern "C" int sgi_backward(sgi_grid_t g, long long npts, const double* x, const double* gout,
	double* gx, double* gsurplus, void* stream_)
{
	clear_error();
	if (!g || npts < 0 || (npts && (!x || !gout))) return fail(SGI_E_INVALID, "bad arguments");
	if (!g->s64) return fail(SGI_E_INVALID, "grid has no FP64 surplus");
	if (g->TD > 256) return fail(SGI_E_RANGE, "backward supports TotalDof <= 256");
	if (npts > 0xffffffffll) return fail(SGI_E_RANGE, "too many points");
	cudaStream_t stream = (cudaStream_t)stream_;
	DeviceGuard guard(g->device);
	DeviceWork* W = nullptr;
	int rc = device_work(g->device, &W);
	if (rc) return rc;
	g_stats = sgi_launch_stats{};
	if (gsurplus && (npts == 0 || g->nno == 0))
	{
		CUDA_TRY(cudaMemsetAsync(gsurplus, 0, sizeof(double) * (size_t)g->nno * g->TD, stream));
		gsurplus = nullptr;
	}
	if (npts == 0) return SGI_OK;
	const int R = pick_R(g->TD);
	void (*pk)(BwdArgs) = R == 1 ? bwd_points_kernel<1> : R == 2 ? bwd_points_kernel<2> : R == 4 ? bwd_points_kernel<4> : bwd_points_kernel<8>;
	const size_t smem = (size_t)WARPS * 2 * g->dim * sizeof(double);
	if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int blocks = 0;
	rc = occupancy_grid(pk, smem, W->sms, &blocks);
	if (rc) return rc;

	BwdArgs a;
	memset(&a, 0, sizeof(a));
	a.G = desc_of(g, 0);
	a.x = x; a.gout = gout; a.gx = gx; a.npts = npts; a.dim = g->dim; a.TD = g->TD;

	// scratch (stream-ordered allocations from the device's pool)
	cudaMemPool_t pool = nullptr;
	rc = scratch_pool(W, g->device, &pool);
	if (rc) return rc;
	long long* counts = nullptr;
	long long* offs = nullptr;
	uint32_t *pn = nullptr, *node_sorted = nullptr;
	PairVal *pv = nullptr, *val_sorted = nullptr;
	void* tmp = nullptr;
	long long npairs = 0;
	auto cleanup = [&]()
	{
		cudaFreeAsync(counts, stream); cudaFreeAsync(offs, stream); cudaFreeAsync(pn, stream);
		cudaFreeAsync(pv, stream); cudaFreeAsync(val_sorted, stream); cudaFreeAsync(node_sorted, stream);
		cudaFreeAsync(tmp, stream);
	};
#define BWD_TRY(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { cleanup(); \
	return fail(SGI_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); } } while (0)
	if (gsurplus)
	{
		BWD_TRY(cudaMallocFromPoolAsync((void**)&counts, sizeof(long long) * (npts + 1), pool, stream));
		BWD_TRY(cudaMallocFromPoolAsync((void**)&offs, sizeof(long long) * (npts + 1), pool, stream));
		BWD_TRY(cudaMemsetAsync(counts + npts, 0, sizeof(long long), stream));
		rc = sgi_active_count(g, npts, x, counts, stream);
		if (rc) { cleanup(); return rc; }
		size_t tb = 0;
		BWD_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts, offs, npts + 1, stream));
		BWD_TRY(cudaMallocFromPoolAsync(&tmp, tb, pool, stream));
		BWD_TRY(cub::DeviceScan::ExclusiveSum(tmp, tb, counts, offs, npts + 1, stream));
		BWD_TRY(cudaMemcpyAsync(&npairs, offs + npts, sizeof(long long), cudaMemcpyDeviceToHost, stream));
		BWD_TRY(cudaStreamSynchronize(stream));
		cudaFreeAsync(tmp, stream); tmp = nullptr;
		if (npairs > 0x7fffffffll) { cleanup(); return fail(SGI_E_RANGE, "%lld active pairs exceed 2^31", npairs); }
		const size_t np = (size_t)std::max(npairs, 1ll);
		BWD_TRY(cudaMallocFromPoolAsync((void**)&pn, 4 * np, pool, stream));
		BWD_TRY(cudaMallocFromPoolAsync((void**)&pv, sizeof(PairVal) * np, pool, stream));
		a.pair_off = offs; a.pair_node = pn; a.pair_val = pv;
	}
	a.counter = W->counters + (W->next.fetch_add(1) % NCOUNTERS);
	BWD_TRY(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream));
	pk<<<blocks, BLOCK, smem, stream>>>(a);
	BWD_TRY(cudaGetLastError());
	g_stats.kernels++;
	if (gsurplus)
	{
		const size_t np = (size_t)std::max(npairs, 1ll);
		BWD_TRY(cudaMallocFromPoolAsync((void**)&val_sorted, sizeof(PairVal) * np, pool, stream));
		BWD_TRY(cudaMallocFromPoolAsync((void**)&node_sorted, 4 * np, pool, stream));
		// stable radix sort by node: each node's pairs stay in point order
		size_t tb = 0;
		int endbit = 1;
		while (endbit < 32 && (1ll << endbit) <= (long long)g->nno) endbit++;
		BWD_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, pn, node_sorted, pv, val_sorted, (int)npairs, 0, endbit, stream));
		BWD_TRY(cudaMallocFromPoolAsync(&tmp, tb, pool, stream));
		BWD_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, pn, node_sorted, pv, val_sorted, (int)npairs, 0, endbit, stream));
		void (*sk)(const uint32_t*, const PairVal*, long long, const double*, double*, int, int) =
			R == 1 ? bwd_surplus_kernel<1> : R == 2 ? bwd_surplus_kernel<2> : R == 4 ? bwd_surplus_kernel<4> : bwd_surplus_kernel<8>;
		sk<<<W->sms * 8, BLOCK, 0, stream>>>(node_sorted, val_sorted, npairs, gout, gsurplus, g->nno, g->TD);
		BWD_TRY(cudaGetLastError());
		g_stats.kernels += 1;   // and the library's radix sort
	}
	cleanup();
	g_stats.points = npts;
	return SGI_OK;
#undef BWD_TRY
}

// ------------------------------------------------- forward without allocation
//
// sgi_interpolate_noalloc: the work counters of its launches live in this
// fixed array of the module's device image instead of the lazily allocated
// per-device workspace.  Host code must not use the symbol itself as a device
// address; it takes the address from cudaGetSymbolAddress once per device.

static __device__ __align__(256) unsigned long long g_noalloc_counters[SGI_NOALLOC_MAX_LAUNCHES];

namespace {

std::mutex g_noalloc_mtx;
std::vector<unsigned long long*> g_noalloc_addr; // per device; null until set up
std::vector<int> g_noalloc_sms;

// With `dev` current: the array's device address and the SM count, looked up
// on the first call for this device.
int noalloc_setup(int dev, unsigned long long** addr, int* sms)
{
	std::lock_guard<std::mutex> lk(g_noalloc_mtx);
	if ((int)g_noalloc_addr.size() <= dev) { g_noalloc_addr.resize(dev + 1, nullptr); g_noalloc_sms.resize(dev + 1, 0); }
	if (!g_noalloc_addr[dev])
	{
		unsigned long long* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_counters);
		if (e != cudaSuccess) return fail(SGI_E_CUDA, "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
		int n = 0;
		e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		if (e != cudaSuccess) return fail(SGI_E_CUDA, "cudaDeviceGetAttribute failed: %s", cudaGetErrorString(e));
		g_noalloc_sms[dev] = n;
		g_noalloc_addr[dev] = p;
	}
	*addr = g_noalloc_addr[dev];
	*sms = g_noalloc_sms[dev];
	return SGI_OK;
}

} // namespace

extern "C" int sgi_interpolate_noalloc(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision, void* stream_)
{
	clear_error();
	int rc = check_set(ngrids, grids, pt_offsets);
	if (rc) return rc;
	if (pt_offsets[ngrids] > 0 && (!x || !out)) return fail(SGI_E_INVALID, "null x or out");
	if (precision != SGI_FP64 && precision != SGI_FP32C) return fail(SGI_E_INVALID, "unknown precision %d", precision);
	for (int k = 0; k < ngrids; k++)
	{
		if (precision == SGI_FP64 && !grids[k]->s64) return fail(SGI_E_INVALID, "grid %d has no FP64 surplus", k);
		if (precision == SGI_FP32C && !grids[k]->s32) return fail(SGI_E_INVALID, "grid %d was built without SGI_BUILD_FP32", k);
	}
	const sgi_grid* g0 = grids[0];
	const int variant = g_variant.load();   // resolved per group as sgi_interpolate does
	if (fwd_smem(precision, g0->dim, true) > 200 * 1024) return fail(SGI_E_RANGE, "dim %d too large for shared staging", g0->dim);
	// count the launches first: reject before launching anything
	const int passes = (g0->TD + PASS - 1) / PASS;
	long long launches = 0;
	for (int gb = 0; gb < ngrids; gb += MAXG)
		if (pt_offsets[std::min(ngrids, gb + MAXG)] > pt_offsets[gb]) launches += passes;
	if (launches > SGI_NOALLOC_MAX_LAUNCHES)
		return fail(SGI_E_RANGE, "call needs %lld kernel launches; the no-allocation scratch holds work counters "
			"for at most %d (ceil(ngrids/%d) * ceil(TotalDof/%d) launches)", launches, SGI_NOALLOC_MAX_LAUNCHES,
			MAXG, PASS);
	DeviceGuard guard(g0->device);
	cudaStream_t stream = (cudaStream_t)stream_;
	unsigned long long* counters = nullptr;
	int sms = 0;
	rc = noalloc_setup(g0->device, &counters, &sms);
	if (rc) return rc;
	g_stats = sgi_launch_stats{};
	int slot = 0;
	for (int gb = 0; gb < ngrids; gb += MAXG)
	{
		const int ng = std::min(MAXG, ngrids - gb);
		const long long p0 = pt_offsets[gb], p1 = pt_offsets[gb + ng];
		if (p1 == p0) continue;
		FwdArgs a;
		memset(&a, 0, sizeof(a));
		for (int k = 0; k < ng; k++) a.g[k] = desc_of(grids[gb + k], pt_offsets[gb + k] - p0, precision);
		a.x = x + (size_t)p0 * g0->dim;
		a.out = out + (size_t)p0 * g0->TD;
		a.npts = p1 - p0;
		a.ngrids = ng; a.dim = g0->dim; a.TD = g0->TD;
		set_starts(a, grids, gb, ng);   // whole grids: the roots' groups
		// the kernels sgi_interpolate picks for an unchunked launch
		const bool descent = precision == SGI_FP32C && descent_ok(grids, gb, ng, false);
		const bool small = a.npts < (long long)sms * WARPS;
		const bool cols_mode = precision == SGI_FP64 && small;
		const size_t smem = cols_mode ? (size_t)WARPS * cols_stride(g0->dim) * sizeof(double)
		                              : fwd_smem(precision, g0->dim, descent);
		for (int ob = 0; ob < g0->TD; ob += PASS)
		{
			a.o_begin = ob;
			a.counter = counters + slot++;
			CUDA_TRY(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream));
			const int cols = std::min(g0->TD - ob, PASS);
			void (*kern)(FwdArgs) = cols_mode ? fwd_f64_cols_kernel
				: select_fwd(precision, g0->ld, cols, auto_variant(variant, a.npts, sms), descent, small);
			if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
			int blocks = 0;
			rc = occupancy_grid(kern, smem, sms, &blocks);
			if (rc) return rc;
			const long long items = cols_mode ? a.npts * ((cols + 31) / 32) : a.npts;
			const long long need = (items + WARPS - 1) / WARPS;
			if (blocks > need) blocks = (int)need;
			kern<<<blocks, BLOCK, smem, stream>>>(a);
			CUDA_TRY(cudaGetLastError());
			g_stats.kernels++;
			g_stats.grid_blocks = blocks;
			g_stats.block_threads = BLOCK;
		}
		g_stats.points += a.npts;
	}
	return SGI_OK;
}

// ------------------------------------------------------- plans (CUDA graphs)
//
// A plan records every launch of one forward call (work-counter clears and
// chunk launches) into a CUDA graph once and replays it with one
// cudaGraphLaunch.  The chunk size is chosen by timing candidates on the
// caller's own inputs the first time a (dim, largest nno, TotalDof,
// precision, batch size) key is seen.

struct sgi_plan
{
	int device = 0;
	int chunk = 0;
	int variant = 0;
	int launches = 0;
	unsigned long long* counters = nullptr;
	char* scratch = nullptr;          // hit lists of two-phase small-batch groups
	size_t scratch_bytes = 0;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	float tuned_ms = 0.f;
};

namespace {

struct TuneKey
{
	int dim, maxnno, TD, precision;
	long long npts;
	bool operator<(const TuneKey& o) const
	{
		return std::tie(dim, maxnno, TD, precision, npts) < std::tie(o.dim, o.maxnno, o.TD, o.precision, o.npts);
	}
};
std::mutex g_tune_mtx;
struct TuneResult { int chunk, variant; float ms; };
std::map<TuneKey, TuneResult> g_tune;

// Best of three timed calls after a warm-up: single calls of the candidates
// differ by a few percent from run to run, as much as the candidates do.
int time_forward(int ngrids, const sgi_grid_t* grids, const long long* offs, const double* x, double* out,
	int precision, cudaStream_t s, int chunk, int variant, float* ms)
{
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	CUDA_TRY(cudaEventCreate(&e0));
	CUDA_TRY(cudaEventCreate(&e1));
	int rc = launch_forward(ngrids, grids, offs, x, out, precision, s, chunk, nullptr, nullptr, variant);
	for (int r = 0; r < 3 && !rc; r++)
	{
		cudaEventRecord(e0, s);
		rc = launch_forward(ngrids, grids, offs, x, out, precision, s, chunk, nullptr, nullptr, variant);
		if (rc) break;
		cudaEventRecord(e1, s);
		cudaEventSynchronize(e1);
		float t = 0.f;
		cudaEventElapsedTime(&t, e0, e1);
		if (r == 0 || t < *ms) *ms = t;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	return rc;
}

void free_plan(sgi_plan* p)
{
	if (!p) return;
	if (p->exec) cudaGraphExecDestroy(p->exec);
	if (p->graph) cudaGraphDestroy(p->graph);
	if (p->counters) cudaFree(p->counters);
	if (p->scratch) cudaFree(p->scratch);
	delete p;
}

} // namespace

extern "C" int sgi_plan_create(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision, int chunk_rows_req, void* stream_, sgi_plan_t* out_plan)
{
	clear_error();
	if (!out_plan) return fail(SGI_E_INVALID, "null plan");
	*out_plan = nullptr;
	int rc = check_set(ngrids, grids, pt_offsets);
	if (rc) return rc;
	const long long npts = pt_offsets[ngrids];
	if (npts > 0 && (!x || !out)) return fail(SGI_E_INVALID, "null x or out");
	if (precision != SGI_FP64 && precision != SGI_FP32C) return fail(SGI_E_INVALID, "unknown precision %d", precision);
	DeviceGuard guard(grids[0]->device);
	cudaStream_t stream = (cudaStream_t)stream_;
	DeviceWork* W = nullptr;
	rc = device_work(grids[0]->device, &W);
	if (rc) return rc;
	int maxnno = 0;
	for (int k = 0; k < ngrids; k++) maxnno = std::max(maxnno, grids[k]->nno);
	sgi_plan* p = new sgi_plan;
	p->device = grids[0]->device;
	float tuned = 0.f;
	int chunk = chunk_rows_req, variant = 0;
	{
		const TuneKey key{ grids[0]->dim, maxnno, grids[0]->TD, precision, npts };
		bool hit = false;
		if (chunk < 0)
		{
			std::lock_guard<std::mutex> lk(g_tune_mtx);
			auto it = g_tune.find(key);
			if (it != g_tune.end()) { chunk = it->second.chunk; variant = it->second.variant; tuned = it->second.ms; hit = true; }
		}
		if (!hit)
		{
			// candidates: no chunks, and chunks whose rows fill 1/4, 1/2, 3/4, 1
			// and 2 L2s (or the requested chunk); kernel variants for FP32C
			std::vector<int> cand;
			if (chunk >= 0) cand.push_back(chunk);
			else
			{
				const long long row = (long long)grids[0]->ld * (precision == SGI_FP64 ? 8 : 4);
				cand.push_back(0);
				for (double f : { 0.25, 0.5, 0.75, 1.0, 2.0 })
				{
					const long long r = std::max(1024ll, (long long)(W->l2_bytes * f / row));
					if (r < maxnno) cand.push_back((int)r);
				}
			}
			const int nvar = precision == SGI_FP32C ? NVARIANTS : 1;
			chunk = cand[0];
			variant = 0;
			if (cand.size() * nvar > 1)
			{
				float best = 0.f;
				bool first = true;
				for (int c : cand)
					for (int v = 0; v < nvar; v++)
					{
						float ms = 0.f;
						rc = time_forward(ngrids, grids, pt_offsets, x, out, precision, stream, c, v, &ms);
						if (rc) { free_plan(p); return rc; }
						if (first || ms < best) { best = ms; chunk = c; variant = v; first = false; }
					}
				tuned = best;
				if (chunk_rows_req < 0)
				{
					std::lock_guard<std::mutex> lk(g_tune_mtx);
					g_tune[key] = TuneResult{ chunk, variant, tuned };
				}
			}
		}
	}
	p->variant = variant;
	p->chunk = chunk;
	p->tuned_ms = tuned;
	size_t list_bytes = 0;
	p->launches = count_launches(W, ngrids, grids, pt_offsets, precision, chunk, &list_bytes);
	cudaError_t e = cudaMalloc(&p->counters, sizeof(unsigned long long) * std::max(p->launches, 1));
	if (e != cudaSuccess) { free_plan(p); return fail(SGI_E_NOMEM, "cudaMalloc failed: %s", cudaGetErrorString(e)); }
	if (list_bytes)
	{
		e = cudaMalloc(&p->scratch, list_bytes);
		if (e != cudaSuccess) { free_plan(p); return fail(SGI_E_NOMEM, "cudaMalloc failed: %s", cudaGetErrorString(e)); }
		p->scratch_bytes = list_bytes;
	}
	cudaStream_t cs = nullptr;
	e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
	if (e != cudaSuccess) { free_plan(p); return fail(SGI_E_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e)); }
	e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
	if (e == cudaSuccess)
	{
		int n = 0;
		rc = launch_forward(ngrids, grids, pt_offsets, x, out, precision, cs, chunk, p->counters, &n, variant,
		                    p->scratch, p->scratch_bytes);
		cudaGraph_t g = nullptr;
		e = cudaStreamEndCapture(cs, &g);
		p->graph = g;
		if (!rc && e == cudaSuccess && n != p->launches) rc = fail(SGI_E_CUDA, "plan recorded %d launches, expected %d", n, p->launches);
	}
	cudaStreamDestroy(cs);
	if (rc) { free_plan(p); return rc; }
	if (e != cudaSuccess) { free_plan(p); return fail(SGI_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e)); }
	e = cudaGraphInstantiate(&p->exec, p->graph, 0);
	if (e != cudaSuccess) { free_plan(p); return fail(SGI_E_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(e)); }
	*out_plan = p;
	return SGI_OK;
}

extern "C" int sgi_plan_launch(sgi_plan_t p, void* stream)
{
	clear_error();
	if (!p) return fail(SGI_E_INVALID, "null plan");
	DeviceGuard guard(p->device);
	CUDA_TRY(cudaGraphLaunch(p->exec, (cudaStream_t)stream));
	g_stats = sgi_launch_stats{};
	g_stats.kernels = p->launches;
	return SGI_OK;
}

extern "C" int sgi_plan_info(sgi_plan_t p, int* chunk_rows_out, int* variant, int* launches, float* tuned_ms)
{
	clear_error();
	if (!p) return fail(SGI_E_INVALID, "null plan");
	if (variant) *variant = p->variant;
	if (chunk_rows_out) *chunk_rows_out = p->chunk;
	if (launches) *launches = p->launches;
	if (tuned_ms) *tuned_ms = p->tuned_ms;
	return SGI_OK;
}

extern "C" void sgi_plan_destroy(sgi_plan_t p)
{
	if (!p) return;
	DeviceGuard guard(p->device);
	free_plan(p);
}

namespace {

// Small host calls of the FP64 form (the plugin's one point, or one point per
// state, per call) replay a plan over the device's staging buffers, kept per
// call shape (device, grids, point offsets): the call then costs two copies
// and one graph launch instead of the launches' host set-up.  FP64 results
// do not depend on the launch configuration, so they are the same bits as
// the direct launches'.  Entries whose plan would hold more than
// HOST_PLAN_MAX_SCRATCH of hit-list scratch are not kept; at most
// HOST_PLANS_MAX shapes per device are, the least recently used replaced
// first.  An entry goes when one of its grids is destroyed, or when the
// staging buffers it was recorded on are replaced by larger ones.  Evictions
// touch only entries of the calling device, whose workspace mutex the
// caller holds, so no other thread can be replaying them.
struct HostPlanKey
{
	int device;
	std::vector<const sgi_grid*> grids;
	std::vector<long long> offs;
	bool operator<(const HostPlanKey& o) const
	{
		return std::tie(device, grids, offs) < std::tie(o.device, o.grids, o.offs);
	}
};
struct HostPlan
{
	sgi_plan_t plan;
	const double* dx;
	const double* dout;
	unsigned long long used;
};
constexpr size_t HOST_PLANS_MAX = 16;
constexpr size_t HOST_PLAN_MAX_SCRATCH = 32ull << 20;
std::mutex g_hp_mtx;
std::map<HostPlanKey, HostPlan>* g_hp = new std::map<HostPlanKey, HostPlan>();   // kept until exit
unsigned long long g_hp_clock = 0;

void host_plans_forget(const sgi_grid* g)
{
	std::lock_guard<std::mutex> lk(g_hp_mtx);
	for (auto it = g_hp->begin(); it != g_hp->end();)
	{
		if (std::find(it->first.grids.begin(), it->first.grids.end(), g) != it->first.grids.end())
		{
			sgi_plan_destroy(it->second.plan);
			it = g_hp->erase(it);
		}
		else ++it;
	}
}

int host_plan_call(DeviceWork* W, int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, bool* done)
{
	*done = false;
	const int dev = grids[0]->device;
	HostPlanKey key{ dev, std::vector<const sgi_grid*>(grids, grids + ngrids),
	                 std::vector<long long>(pt_offsets, pt_offsets + ngrids + 1) };
	sgi_plan_t p = nullptr;
	{
		std::lock_guard<std::mutex> lk(g_hp_mtx);
		auto it = g_hp->find(key);
		if (it != g_hp->end())
		{
			if (it->second.dx == W->dx && it->second.dout == W->dout)
			{
				p = it->second.plan;
				it->second.used = ++g_hp_clock;
			}
			else
			{
				sgi_plan_destroy(it->second.plan);
				g_hp->erase(it);
			}
		}
	}
	if (!p)
	{
		size_t lb = 0;
		count_launches(W, ngrids, grids, pt_offsets, SGI_FP64, 0, &lb);
		if (lb > HOST_PLAN_MAX_SCRATCH) return SGI_OK;            // the direct launches serve
		if (sgi_plan_create(ngrids, grids, pt_offsets, W->dx, W->dout, SGI_FP64, 0, W->stream, &p) != SGI_OK)
		{
			clear_error();
			return SGI_OK;
		}
		std::lock_guard<std::mutex> lk(g_hp_mtx);
		size_t n = 0;
		auto lru = g_hp->end();
		for (auto it = g_hp->begin(); it != g_hp->end(); ++it)
			if (it->first.device == dev)
			{
				n++;
				if (lru == g_hp->end() || it->second.used < lru->second.used) lru = it;
			}
		if (n >= HOST_PLANS_MAX && lru != g_hp->end())
		{
			sgi_plan_destroy(lru->second.plan);
			g_hp->erase(lru);
		}
		(*g_hp)[key] = HostPlan{ p, W->dx, W->dout, ++g_hp_clock };
	}
	const long long npts = pt_offsets[ngrids];
	const int D = grids[0]->dim, TD = grids[0]->TD;
	CUDA_TRY(cudaMemcpyAsync(W->dx, x, (size_t)npts * D * sizeof(double), cudaMemcpyHostToDevice, W->stream));
	CUDA_TRY(cudaGraphLaunch(p->exec, W->stream));
	CUDA_TRY(cudaMemcpyAsync(out, W->dout, (size_t)npts * TD * sizeof(double), cudaMemcpyDeviceToHost, W->stream));
	CUDA_TRY(cudaStreamSynchronize(W->stream));
	g_stats = sgi_launch_stats{};
	g_stats.kernels = p->launches;
	g_stats.points = npts;
	*done = true;
	return SGI_OK;
}

} // namespace
