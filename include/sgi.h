/*
 * sgi.h — C ABI of the B200 sparse-grid linear-basis interpolator.
 *
 * The hot path of the HDDM LinearBasis postprocessor: for every query point x,
 *
 *     value[o] = sum over grid nodes n of surplus[n][o] * prod_d phi(x_d; i_nd, j_nd)
 *     phi(x; i, j) = max(0, 1 - |x*i - j|)          (i = 0, j = 0: phi = 1)
 *
 * on one GPU.  Plain pointers and sizes only; every entry point returns 0
 * (SGI_OK) or a negative SGI_E* code, with a message for the calling thread in
 * sgi_last_error().  Device pointers are CUDA device (or managed) memory on the
 * grid's device; `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * Which reference interface each entry point replaces is cited per function
 * (paths relative to the reference project apc-llc/hddm-solver-postprocessors).
 * The reference's own plugin exports (getInterpolator, getData, ...) are
 * declared in sgi_plugin.h.
 */
#ifndef SGI_H
#define SGI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SGI_OK             0
#define SGI_E_INVALID     -1   /* bad argument (null pointer, negative size, ...) */
#define SGI_E_MISMATCH    -2   /* DofPerNode / dim mismatch between call and grid */
#define SGI_E_FORMAT      -3   /* malformed or unreadable grid file */
#define SGI_E_RANGE       -4   /* value outside what the device layout encodes */
#define SGI_E_CUDA        -5   /* CUDA runtime error */
#define SGI_E_NOMEM       -6   /* host or device allocation failed */
#define SGI_E_NODEVICE    -7   /* no CUDA device */
#define SGI_E_DEVICE      -8   /* a kernel reported an error through its status word */

/* Message of the last failing call on this thread ("" if none). */
const char* sgi_last_error(void);

/* Number of CUDA devices (0 when none).  Replaces the GPU count of
 * LinearBasis/cuda/src/Devices.cu:13-47 / supported.cpp:13-20. */
int sgi_device_count(void);

/* ---------------------------------------------------------- host grids */
/* A grid in the reference's dense form (LinearBasis/gold/include/Data.h:252):
 * for node n and dimension k, index[n*2*dim + k] = i (0 for level 1) and
 * index[n*2*dim + dim + k] = j; surplus[n*TotalDof + o].  Owned by the
 * library. */
typedef struct sgi_host_grid* sgi_host_grid_t;

/* Read a .plt grid file in any of the reference's layouts (compressed,
 * binary, text); `nagents` is the configured dimension, which the file's
 * header must match.  Replaces DataDense::load's reader,
 * LinearBasis/gold/src/Data.cpp:322-595. */
int sgi_host_grid_read_plt(const char* path, int nagents, sgi_host_grid_t* out);

/* Write the compressed .plt layout (marker "compressed", header, CSR index
 * block of {u16 i, u16 j} pairs, CSR surplus block) that
 * LinearBasis/gold/src/Data.cpp:49-190 reads.  No reference counterpart
 * (the reference only reads). */
int sgi_host_grid_write_plt(sgi_host_grid_t g, const char* path);

/* Wrap caller arrays (copied). */
int sgi_host_grid_from_dense(int dim, int nno, int TotalDof, const int* index,
	const double* surplus, sgi_host_grid_t* out);

/* Views of the arrays (valid until sgi_host_grid_free). */
int sgi_host_grid_view(sgi_host_grid_t g, int* dim, int* nno, int* TotalDof,
	const int** index, const double** surplus);
void sgi_host_grid_free(sgi_host_grid_t g);

/* Synthetic grids (no reference counterpart; the reference's large test grids
 * are not in its tree).  Nodes are emitted in depth-first order of their
 * refinement tree.  Surpluses are uniform[-1,1] * 2^(-2*sum_k(l_k-1)).
 *   regular:  all nodes with sum_k (l_k - 1) <= level - 1
 *   adaptive: from the level-1 root, repeatedly pick a uniformly random leaf
 *             and add all its children along a random non-empty subset of
 *             dimensions (each kept with probability p_dim), skipping children
 *             above max_level, until nno nodes exist. */
int sgi_gen_regular(int dim, int level, int TotalDof, uint64_t seed, sgi_host_grid_t* out);
int sgi_gen_adaptive(int dim, int nno, int TotalDof, int max_level, double p_dim,
	uint64_t seed, sgi_host_grid_t* out);

/* Query points: kind 0 = uniform [0,1]^dim, 1 = N(0.5, 0.05^2) clipped to
 * [0,1], 2 = first half uniform and second half clustered.  If kink_reject > 0,
 * points with any coordinate within kink_reject of a multiple of
 * 2^-(max_level-1) (a superset of every hat's kinks) are redrawn.  out is
 * npts x dim, row-major. */
int sgi_gen_points(int dim, long npts, int kind, uint64_t seed, double kink_reject,
	int max_level, double* out);

/* The reference x86 loader's sparse form of one grid (xps = unique
 * (i, j, dim) triples with id 0 = empty; chains = per-node xps ids,
 * 0-terminated, nfreqs per node; rows reordered).  Reproduces
 * DataSparse::load, LinearBasis/x86/src/Data.cpp:598-951, bit for bit.
 * Call with null arrays first to get nfreqs and szxps.
 *   xps[3*k + {0,1,2}] = i, j, dim      (szxps triples)
 *   chains[n*nfreqs + f]                (nno * nfreqs)
 *   row_perm[r] = input row stored at reordered row r  (nno) */
int sgi_host_grid_xps_chains(sgi_host_grid_t g, int* nfreqs, int* szxps,
	int* xps, int* chains, int* row_perm);

/* The containment tree the kernels walk (for inspection and tests): for node
 * n in grid order, parent[n] is the nearest earlier node whose support holds
 * n's support and that is still open on the depth-first stack (-1 if none),
 * and n's subtree is the index range [n, skip[n]).  No reference counterpart. */
int sgi_host_grid_tree(sgi_host_grid_t g, int* skip, int* parent);

/* The child groups the FP32C descent walks (for inspection and tests).  The
 * tree children of each node are grouped: two children that differ from the
 * node only in the same dimension d, with disjoint supports in d, form a pair
 * (at most one is active at any point, and x_d picks it); every other child is
 * a singleton.  Group g: a[4g..4g+3] = {left child, right child (0xffffffff
 * for a singleton), d | kind << 16, the parent's (i | j << 16) in d (0 when
 * constant)}, b[2g..2g+1] = {left's (i | j << 16) in d, right's}; kind 0 =
 * the children differ from the parent in d only, 1 = the child differs in
 * several dimensions, 2 = the child has the parent's components.  Node n's
 * groups are [first[n], first[n] + count[n]); entry nno lists the tree roots.
 * Call with null arrays first to get ngroups; a is 4*ngroups, b 2*ngroups,
 * first and count nno + 1 entries.  No reference counterpart. */
int sgi_host_grid_descent(sgi_host_grid_t g, int* ngroups, int* npairs, uint32_t* a, uint32_t* b,
	uint32_t* first, uint32_t* count);

/* --------------------------------------------------------- device grids */
typedef struct sgi_grid* sgi_grid_t;

/* Build flags */
#define SGI_BUILD_FP32    0x1u   /* also keep the FP32 surplus (+ FP64 copies of coarse rows) */
#define SGI_BUILD_NO_FP64 0x2u   /* drop the FP64 surplus (FP32 forms only)              */

typedef struct sgi_grid_info
{
	int dim, nno, TotalDof;
	int ld;               /* surplus row stride on the device (elements)          */
	int max_comps;        /* most non-constant dimensions of any node (nfreqs)    */
	int tree_depth;       /* depth of the containment tree                       */
	int tree_roots;       /* nodes without a containing ancestor                  */
	int multi_delta;      /* nodes that differ from their tree parent in >1 dim   */
	int ncoarse;          /* rows with an FP64 copy for FP32C big terms           */
	long long comps;      /* stored (dim, i, j) components                        */
	long long device_bytes;
	double coarse_threshold;
} sgi_grid_info;

/* Upload a grid to `device`.  Nodes keep the host grid's order, so the FP64
 * forward form adds node contributions in file order, as the reference's gold
 * kernel does.  Replaces the device upload of cuda Data::load,
 * LinearBasis/cuda/src/Data.cu:348-949. */
int sgi_grid_create(sgi_host_grid_t g, int device, unsigned flags, sgi_grid_t* out);
int sgi_grid_info_get(sgi_grid_t g, sgi_grid_info* info);
void sgi_grid_destroy(sgi_grid_t g);

/* Load a .plt grid file onto `device` through a cache of its built device
 * layout (the containment tree, descent groups, chain table and surplus
 * forms that sgi_grid_create builds on the host from the file's arrays).
 * cache_path NULL means "<path>.sgi-layout".  When the cache is complete,
 * of this library's format version, built with the same flags and for the
 * same .plt (its size and modification time, to the nanosecond), the layout
 * is read from it and uploaded: the .plt is not parsed and nothing is
 * rebuilt.  Otherwise the .plt is read (nagents checked against its header,
 * as sgi_host_grid_read_plt does), the layout built and uploaded, and the
 * cache written through a temporary file renamed into place (a cache that
 * cannot be written is not an error).  *hit (may be NULL) is 1 when the
 * cache was used.  The result is the grid sgi_grid_create makes from the
 * same file, and computes the same bits.  The cache is a native-byte-order
 * file for this library build; it holds the FP64 surplus rows too, so it is
 * larger than a compressed .plt.  Replaces the parse and the per-load
 * layout work of the reference's Data::load
 * (LinearBasis/gold/src/Data.cpp:322-595, LinearBasis/x86/src/Data.cpp:598-951),
 * which has no cache. */
int sgi_grid_load(const char* path, int nagents, int device, unsigned flags, const char* cache_path,
	sgi_grid_t* out, int* hit);

/* The cache half of sgi_grid_load without a GPU: build the layout of `path`
 * on the host and write its cache (cache_path NULL: "<path>.sgi-layout"). */
int sgi_grid_cache_write(const char* path, int nagents, unsigned flags, const char* cache_path);

/* 1 when the cache of `path` is valid for these flags and nagents (its key,
 * version and checksum match), 0 when sgi_grid_load would rebuild it, or a
 * negative SGI_E_* code (the .plt itself is missing). */
int sgi_grid_cache_valid(const char* path, int nagents, unsigned flags, const char* cache_path);

/* Surplus cutoff of the FP32C form.  The reference parses a surplusCutoff
 * parameter (LinearBasis/cpu/src/parameters.cpp:103-108,
 * LinearBasis/cuda/src/parameters.cpp:110-127) and no kernel reads it; here
 * it skips small terms.  The term of node n at point x is skipped, before its
 * surplus row is read, when its bound |w_n(x)| * max_o |surplus[n][o]| (in
 * FP32) is below `cutoff` (absolute, in surplus units), unless it is a big
 * term (a row with an FP64 copy whose bound reaches coarse_threshold).  Each
 * output then moves from the FP32C result by at most the sum of the bounds of
 * the terms skipped at that point.  cutoff <= 0, the default, keeps the form's
 * own bound of 2^-42 times the largest |surplus|, and so does any cutoff below
 * it.  A cutoff above 2^-29 times the largest |surplus| also leaves no term
 * to the FP16 rows (see SGI_FP32C).  `effective` (may be NULL) receives the
 * bound in use.  Calls and plans made afterwards use it; plans made before
 * keep theirs.  Not to be called
 * while another thread calls with this grid.  The FP64 form ignores it.
 * Returns SGI_E_INVALID for a grid built without SGI_BUILD_FP32. */
int sgi_grid_set_surplus_cutoff(sgi_grid_t g, double cutoff, double* effective);

/* ---------------------------------------------------------- interpolate */
#define SGI_FP64   0   /* plain FP64: node order and rounding of the gold kernel */
#define SGI_FP32C  1   /* FP32 products of small terms, FP64 big terms and sums, FP64 final */
/* SGI_FP32C classes every term of a point by its bound |w| * max|s_row|
 * against the grid's largest |surplus| smax: big (at least 2^-16 smax, on a
 * row with an FP64 copy) reads the FP64 row and adds in FP64; fine reads the
 * FP32 row, multiplies and sums in FP32 and adds the sums to FP64 every eight
 * terms; fine terms below 2^-29 smax read an FP16 copy of the row instead
 * (rows scaled by a power of two per row; grids whose rows are a multiple of
 * 256 outputs wide; the environment variable SGI_F16_REL, read once, sets
 * another fraction of smax); terms below 2^-42 smax are dropped.  Per term the
 * rounding of the row is at most 2^-24 of its bound (FP32), 2^-11 (FP16), in
 * either case below 2^-40 smax, and a dropped term moves an output by at most
 * its bound. */

/* Batched forward over a set of grids sharing dim and TotalDof (a multistate
 * set or a single grid): grid g owns points [pt_offsets[g], pt_offsets[g+1]).
 * x: device, pt_offsets[ngrids] x dim; out: device, pt_offsets[ngrids] x
 * TotalDof.  pt_offsets is HOST memory.  One persistent launch pulls points
 * from a device work queue.  Replaces LinearBasis_cuda_Generic_InterpolateArray
 * (LinearBasis/cuda/src/InterpolateArray.cu:239-267, one point per call) and
 * ..._InterpolateArrayManyMultistate (InterpolateArrayManyMultistate.cu:346-395,
 * one point per state per call).
 * Small batches (fewer points than the GPU holds warps; FP32C only on grids
 * that keep their FP64 rows) walk node chunks in parallel into hit lists,
 * 12 bytes per (point, node), at most 256 MB per call, taken from a
 * per-device stream-ordered pool that keeps freed memory for later calls
 * (plans own theirs); FP32C then adds the FP64 rows of the terms it keeps.
 * While `stream` is being captured outside a plan, or when the lists would
 * not fit, they run the one-phase kernels instead (FP64: same bits). */
int sgi_interpolate(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision, void* stream);

/* Same with HOST x/out: stages through pinned buffers, copies in, launches,
 * copies out and synchronizes — the reference plugin's per-call contract
 * (include/interpolator.h:32-37, host x and value arrays). */
int sgi_interpolate_host(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision);

/* Backward of the FP64 form for one grid: given gout = dL/dvalue (npts x
 * TotalDof, device), writes gx = dL/dx (npts x dim, device; may be NULL) and
 * gsurplus = dL/dsurplus (nno x TotalDof in file row order, device; may be
 * NULL; overwritten).  Weights are recomputed, never stored; dL/dsurplus is
 * reduced without atomics.  Its scratch (about 40 bytes per active
 * (point, node) pair when gsurplus is requested) comes from a per-device
 * memory pool that keeps freed memory for later calls until the process
 * exits.  No reference counterpart. */
int sgi_backward(sgi_grid_t g, long long npts, const double* x, const double* gout,
	double* gx, double* gsurplus, void* stream);

/* Forward without any device allocation.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory: a host solver that hands
 * all device memory to its own pre-reserved arena (an extra cudaMalloc can
 * fail or fragment it), and time-stepping loops that cannot afford
 * cudaMalloc's implicit device synchronization.  sgi_interpolate's work
 * counters live in a workspace that its first call on a device allocates;
 * this variant instead keeps them in a fixed array inside the library's device
 * image, SGI_NOALLOC_MAX_LAUNCHES counters of 8 bytes per device, held by
 * every GPU that loads the library until the process exits.
 *
 * Arguments and results are those of sgi_interpolate (device x and out, host
 * pt_offsets); FP64 results are bit-identical to it.  It launches every grid
 * whole, never in node chunks (each chunk launch would take one more counter
 * from the fixed array): on grids whose surplus rows exceed the L2, which
 * sgi_interpolate walks in chunks for batches of 81,920 points or more, it
 * reads rows from HBM instead of the L2 and is slower, and its FP32C results
 * may differ from sgi_interpolate's in the last bits (the order of the FP64
 * additions differs; both stay within the FP32C tolerance).  Small batches
 * run the one-phase kernels here (sgi_interpolate's two-phase ones need
 * scratch), with the same consequence for FP32C bits.  A call makes
 * ceil(ngrids / 48) * ceil(TotalDof / 256) kernel launches (groups of grids
 * with no points are skipped); a call that would need more than
 * SGI_NOALLOC_MAX_LAUNCHES launches is rejected with SGI_E_RANGE before
 * anything is launched.  The first call on each device looks up the array's
 * device address with that device current; make that first call before any
 * stream capture.  Every call shares the one array and clears the counters it
 * uses on `stream` before each launch, so calls that overlap on the GPU
 * (different streams, or different host threads) race on the counters and
 * must be serialized by the caller.  The call allocates nothing, neither
 * itself nor through CUDA or any library. */
#define SGI_NOALLOC_MAX_LAUNCHES 64
int sgi_interpolate_noalloc(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision, void* stream);

/* Active-node count A(x) per point (device int64 out[npts]); diagnostics. */
int sgi_active_count(sgi_grid_t g, long long npts, const double* x, long long* out, void* stream);

/* The FP32C form's terms per point by class (device int64 out[4 * npts]):
 * out[4p] big terms (rows with an FP64 copy whose bound |w| * max|s_row|
 * reaches the coarse threshold: FP64 row reads), out[4p + 1] fine terms read
 * from FP32 rows, out[4p + 2] fine terms read from FP16 rows, out[4p + 3]
 * terms dropped unread (bound below the grid's negligible-term bound or
 * surplus cutoff).  Bounds use the full-product
 * weight rounded to FP32; the forward kernels build weights incrementally, so
 * a term within rounding of a threshold may fall on the other side there.
 * Diagnostics (the bytes the forward gathers); SGI_E_INVALID for a grid
 * built without SGI_BUILD_FP32.  No reference counterpart. */
int sgi_term_classes(sgi_grid_t g, long long npts, const double* x, long long* out, void* stream);

/* Node-range chunking of the forward launches (process-wide).  A grid whose
 * surplus rows exceed the L2 is walked in chunks of consecutive nodes (rows
 * filling half the L2: FP64 rows for FP64, FP32 rows for FP32C), every point against one chunk per launch, the outputs
 * carried between chunks in FP64 (the FP64 form keeps gold's order and bits).
 * rows < 0: automatic (the default; batches under 81,920 points are not
 * chunked); 0: never chunk; > 0: chunks of `rows` nodes.  Returns the previous
 * setting.  No reference counterpart. */
int sgi_set_chunk_rows(int rows);

/* FP32C kernel variant used by sgi_interpolate, sgi_interpolate_host and
 * sgi_interpolate_noalloc (plans pick their own by timing among 0-2): 0 = four
 * fine surplus rows in flight per warp, 1 = two rows and more warps per SM,
 * 2 = eight rows and fewer warps.  Variants 0-2 walk the tree by descent
 * (child groups, see sgi_host_grid_descent) whenever every grid of a launch
 * allows it (tree depth <= 96, and <= 32 for node-chunked launches), else by
 * node windows; 3-5 are 0-2 with the node-window walk forced.  The variants
 * order the FP64 additions of big terms and of FP32 partial sums differently,
 * so their results may differ in the last bits (all within the FP32C
 * tolerance).  variant < 0 or SGI_FP32C_AUTO restores the default,
 * automatic: 2 for a launch with fewer than 64 points per SM (9,472 on a
 * B200), else 1.  Returns the previous setting
 * (SGI_FP32C_AUTO for automatic), or a negative error code.  No reference
 * counterpart. */
#define SGI_FP32C_AUTO 255
int sgi_set_fp32c_variant(int variant);

/* Plans: one forward call recorded into a CUDA graph and replayed.
 * sgi_plan_create records every launch of sgi_interpolate(ngrids, grids,
 * pt_offsets, x, out, precision) (work-counter clears and node-chunk launches,
 * with work counters, and the hit lists of small batches, owned by the plan)
 * into a graph; sgi_plan_launch replays
 * it on `stream` with one cudaGraphLaunch.  x and out are baked into the
 * graph: later replays read the same x buffer and write the same out buffer.
 * chunk_rows >= 0 fixes the node-chunk size (0 = none); chunk_rows < 0 lets the
 * autotuner choose it: the first time a (dim, largest nno, TotalDof,
 * precision, point count) key is seen, candidate chunk sizes (none, and rows
 * filling 1/4, 1/2, 3/4, 1 and 2 L2s), and for FP32C the kernel variants, are timed
 * on the given inputs (which runs the forward, overwriting out) and the
 * fastest is cached for the process.
 * Replays of one plan must not overlap each other.  No reference counterpart
 * (the reference relaunched per call and JIT-compiled per dimension,
 * LinearBasis/cuda/src/JIT.cpp:223-257). */
typedef struct sgi_plan* sgi_plan_t;
int sgi_plan_create(int ngrids, const sgi_grid_t* grids, const long long* pt_offsets,
	const double* x, double* out, int precision, int chunk_rows, void* stream, sgi_plan_t* plan);
int sgi_plan_launch(sgi_plan_t plan, void* stream);
/* The plan's node-chunk size, FP32C kernel variant (as sgi_set_fp32c_variant),
 * launches per replay and the tuned time of one call (ms). */
int sgi_plan_info(sgi_plan_t plan, int* chunk_rows, int* variant, int* launches, float* tuned_ms);
void sgi_plan_destroy(sgi_plan_t plan);

/* Launch statistics of this thread's last sgi_interpolate/sgi_backward call. */
typedef struct sgi_launch_stats
{
	int kernels;          /* kernels launched by the call                 */
	int grid_blocks;
	int block_threads;
	long long points;
} sgi_launch_stats;
int sgi_last_launch(sgi_launch_stats* s);

#ifdef __cplusplus
}
#endif

#endif /* SGI_H */
