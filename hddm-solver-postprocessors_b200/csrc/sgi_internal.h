// Internal declarations shared by the host layer (sgi_host.cpp), the device
// layer (sgi_device.cu) and the plugin surface (plugin.cpp).
#ifndef SGI_INTERNAL_H
#define SGI_INTERNAL_H

#include <cstdint>
#include <string>
#include <vector>

#include "sgi.h"

namespace sgi {

// Thread-local error message; returns `code` so callers can `return fail(...)`.
int fail(int code, const char* fmt, ...);
void clear_error();

// A grid in the reference's dense form (see sgi.h).
struct HostGrid
{
	int dim = 0, nno = 0, TotalDof = 0, Level = 0;
	std::vector<int> index;      // nno * 2 * dim
	std::vector<double> surplus; // nno * TotalDof
};

// ---------------------------------------------------------------- device layout
//
// Node record, 16 bytes, one per node in grid order:
//   x: skip      index of the first node after this node's subtree
//   y: comp_ptr  first component of this node in `comps`
//   z: ncomp (bits 0-7) | flags (bits 8-15) | dim of the delta component (16-31)
//   w: i (bits 0-15) | j (bits 16-31) of the delta component
// A component is (dim, i, j) packed as uint2 {dim, i | j << 16}; a node's
// components are its non-constant dimensions in increasing dimension order.
enum NodeFlags : uint32_t
{
	NODE_ALWAYS = 1u << 8,  // no components: weight 1 everywhere
	NODE_DEAD   = 1u << 9,  // a component with i = 0, j != 0: weight 0 everywhere
	NODE_MULTI  = 1u << 10, // activity needs all components checked
	NODE_COARSE = 1u << 11, // FP32C keeps an FP64 copy of this node's row
};

struct DeviceLayout
{
	std::vector<uint32_t> rec;   // 4 * nno
	std::vector<uint32_t> comps; // 2 * ncomps
	std::vector<uint32_t> lo_index; // nno: row in the lo array, or ~0u
	std::vector<int> parent;        // nno: tree parent, or -1
	// nno pairs {old, depth}: the parent's (i | j << 16) in the node's delta
	// dimension (0 when the parent is constant there) and the node's tree
	// depth (roots 1); the FP32C form builds weights along the tree from them
	std::vector<uint32_t> aux;
	int max_comps = 0, tree_depth = 0, tree_roots = 0, multi_delta = 0, ncoarse = 0;
	double coarse_threshold = 0.0;
};

// Builds the containment tree over the grid's node order and the records.
int build_layout(const HostGrid& g, DeviceLayout& L);

// ------------------------------------------------------- descent layout
//
// The FP32C walk descends the containment tree from the active nodes only.
// The tree children of a node are split into groups:
//   * a pair: two children that differ from the node in the same dimension d
//     only, with disjoint supports in d (the left and right halves of the
//     node's support at the next level) — at most one of them is active at a
//     point, and the point's coordinate picks which;
//   * a singleton: any other child.
// Group g (arrays of ngroups entries):
//   a[g] = {L, R (NONE for a singleton), d | kind << 16, parent's (i | j << 16)
//           in d (0 when the parent is constant there)}
//   b[g] = {L's (i | j << 16) in d, R's}
// kind: DESC_SIMPLE (L/R differ from the parent in d only), DESC_MULTI (L
// differs in several dimensions: all its components are checked),
// DESC_ALWAYS (L has the parent's components: active with the parent).
// Node n's groups are [first[n], first[n] + count[n]), ordered by their
// smallest child index; entry nno is a virtual parent of the tree roots.
constexpr uint32_t DESC_NONE = 0xffffffffu;
enum DescKind : uint32_t { DESC_SIMPLE = 0, DESC_MULTI = 1, DESC_ALWAYS = 2 };

struct DescentLayout
{
	std::vector<uint32_t> a;        // 4 per group
	std::vector<uint32_t> b;        // 2 per group
	std::vector<uint32_t> first;    // nno + 1
	std::vector<uint32_t> count;    // nno + 1
	std::vector<uint32_t> cmin, cmax; // smallest / largest child index per group
	int npairs = 0;
};

int build_descent(const HostGrid& g, const DeviceLayout& L, DescentLayout& D);

// Rows whose largest |surplus| is at least this keep an FP64 copy for the
// FP32C form's big terms (2^-16 of the grid's largest |surplus|, or
// SGI_COARSE_REL times it).
double coarse_threshold_for(const HostGrid& g);

} // namespace sgi

struct sgi_host_grid
{
	sgi::HostGrid g;
};

#endif
