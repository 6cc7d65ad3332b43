/* Kernel-level entry points with the reference's sparse (x86) signatures.
 *
 * The reference's tests and its parent call the per-variant kernel symbols
 * LinearBasis_<variant>_Generic_InterpolateArray[ManyMultistate] directly,
 * with the data its sparse loader builds (LinearBasis/tests/InterpolateArray/
 * test.cpp:285-313 for x86).  These two symbols take exactly those arguments
 * (the x86 loader's host containers, whose layouts are mirrored below) and
 * compute on the GPU, so a caller that holds the reference's DataSparse
 * containers switches by symbol name:
 *
 *   LinearBasis_b200_Generic_InterpolateArray               replaces
 *     LinearBasis_x86_Generic_InterpolateArray
 *     (LinearBasis/x86/src/InterpolateArray.cpp:9-54)
 *   LinearBasis_b200_Generic_InterpolateArrayManyMultistate replaces
 *     LinearBasis_x86_Generic_InterpolateArrayManyMultistate
 *     (LinearBasis/x86/src/InterpolateArrayManyMultistate.cpp:9-60)
 *
 * On the first call with a given grid the library rebuilds its own device
 * layout from the containers (node n's components from its chain of xps
 * entries, its surplus row from the matrix) and keeps it, keyed on the
 * containers' addresses and sizes and a sample of their contents; later
 * calls with the same containers reuse it.  A call then copies x in and the
 * values out (the FP64 form, summing in the containers' node order: within
 * 1e-12 of the reference kernels).  The device argument is not used.  Errors
 * print a message and abort, as the reference does.
 *
 * The reference's CUDA kernel symbols take its device containers
 * (XPS::Device, Chains::Device, Matrix<double>::Device,
 * LinearBasis/cuda/src/InterpolateArray.cu:239-244); objects that only its
 * own CUDA loader creates, so they have no counterpart here. */
#ifndef SGI_KERNELS_H
#define SGI_KERNELS_H

#include <cstdint>
#include <vector>

namespace sgi_x86 {

/* LinearBasis/x86/include/Data.h:213-217: one unique (level, index, dimension)
 * of the grid; entry 0 of an XPS vector is the empty one that ends chains. */
template <typename TIndex>
struct Index
{
	uint8_t i, j;
	TIndex index;
};

typedef std::vector<Index<uint16_t> > XPS;   /* Data.h:251 */
typedef std::vector<uint16_t> Chains;         /* Data.h:252: nfreqs entries per node, 0-terminated */

/* Data.h:127-130: rows of dimX values at a stride of dimX_aligned.  The
 * reference's vector uses a stateless aligned allocator, which leaves the
 * vector's layout that of std::vector. */
template <typename T>
class Matrix
{
public:
	std::vector<T> data;
	int dimY, dimX, dimX_aligned;
};

} // namespace sgi_x86

extern "C" {

void LinearBasis_b200_Generic_InterpolateArray(void* device, const int dim, const int DofPerNode,
	const double* x, const int nfreqs, const sgi_x86::XPS* xps, const sgi_x86::Chains* chains,
	const sgi_x86::Matrix<double>* surplus, double* value);

void LinearBasis_b200_Generic_InterpolateArrayManyMultistate(void* device, const int dim,
	const int DofPerNode, const int count, const double* const* x, const int* nfreqs,
	const sgi_x86::XPS* xps, const sgi_x86::Chains* chains, const sgi_x86::Matrix<double>* surplus,
	double** value);

}

#endif /* SGI_KERNELS_H */
