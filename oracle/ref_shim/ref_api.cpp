// Test infrastructure: a plain-C wrapper around the reference's own CPU
// interpolation code, compiled in place from the reference tree by
// oracle/Makefile into oracle/_ref/libref_<variant>.so.  It is the checker and
// the timed CPU baseline, never part of the product.
//
// One copy of this file is compiled per reference variant (NAMESPACE = gold,
// x86, avx2, avx512).  It provides what the missing parent project would provide:
//   * MPI_Process (declared at include/process.h:8-28) printing to stdio,
//   * Interpolator::getInstance/getParameters (include/interpolator.h:18-42)
//     with Parameters (LinearBasis/cpu/include/parameters.h) bound to globals,
//     so that DataDense::load (LinearBasis/gold/src/Data.cpp:322) can read
//     `nagents`,
//   * a `GoogleTest` class, which the reference's Data classes befriend
//     (LinearBasis/gold/include/Data.h:257, x86/include/Data.h:264), used here
//     to read the loaded index/xps/chains/surplus arrays.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <thread>
#include <string>
#include <vector>

#include "interpolator.h"
#include "Data.h"
#if defined(ORACLE_REF_AVX512)
#include "Device.h"
#endif

// ---------------------------------------------------------------- MPI_Process
MPI_Process* MPI_Process::GoogleTest(int, char**) { return nullptr; }
bool MPI_Process::isMaster() const { return true; }
int MPI_Process::getRoot() const { return 0; }
int MPI_Process::getRank() const { return 0; }
int MPI_Process::getSize() const { return 1; }
MPI_Comm MPI_Process::getComm() const { return 0; }
void MPI_Process::setComm(MPI_Comm) { }
void MPI_Process::abort() { fflush(stdout); fflush(stderr); ::abort(); }
void MPI_Process::cout(const char* format, ...)
{
	if (!getenv("ORACLE_REF_VERBOSE")) return;
	va_list args; va_start(args, format); vfprintf(stdout, format, args); va_end(args);
}
void MPI_Process::cerr(const char* format, ...)
{
	va_list args; va_start(args, format); vfprintf(stderr, format, args); va_end(args);
}
static MPI_Process the_process;
extern "C" int MPI_Process_get(MPI_Process** p) { *p = &the_process; return 0; }

// ------------------------------------------------------ Parameters/Interpolator
extern "C" {
static int g_priority = 0;
static int g_nagents = 0;
static double g_surplusCutoff = 0.0;
static bool g_surplusCutoffDefined = false;
}

namespace NAMESPACE {

Parameters::Parameters(const std::string&, const std::string&) :
	priority(g_priority), nagents(g_nagents),
	surplusCutoff(g_surplusCutoff), surplusCutoffDefined(g_surplusCutoffDefined) { }

const Parameters& Interpolator::getParameters() const { return params; }
Interpolator::Interpolator(const std::string& t, const std::string& c) : jit(false), params(t, c) { }
Interpolator::~Interpolator() { }
void Interpolator::interpolate(Device*, Data*, const int, const real*, const int, real*) { ::abort(); }
void Interpolator::interpolate(Device*, Data*, const real**, const int, real**) { ::abort(); }
Interpolator* Interpolator::getInstance()
{
	static Interpolator instance("oracle_ref");
	return &instance;
}

#if defined(ORACLE_REF_AVX512)
// Friend of Device (LinearBasis/avx512/include/Device.h): the avx512 kernel
// sizes its per-thread scratch by the device's thread count, which the
// parent's Devices sets; one thread here.
class Devices
{
public :
	static void serial(Device& d) { d.nthreads = 1; }
};
#else
class Device;
#endif

// Friend of DataDense/DataSparse: read-only accessors for the loaded state.
class GoogleTest
{
public :
	static int dim(DataDense& d) { return d.dim; }
	static int TotalDof(DataDense& d) { return d.TotalDof; }
	static Matrix<int>& index(DataDense& d, int s) { return d.index[s]; }
	static Matrix<double>& surplus(DataDense& d, int s) { return d.surplus[s]; }
#if !defined(ORACLE_REF_GOLD)
	static int nfreqs(DataSparse& d, int s) { return d.nfreqs[s]; }
	static XPS& xps(DataSparse& d, int s) { return d.xps[s]; }
	static Chains& chains(DataSparse& d, int s) { return d.chains[s]; }
#endif
};

} // namespace NAMESPACE

using namespace NAMESPACE;
typedef NAMESPACE::GoogleTest RefAccess;

#define CAT2(a, b, c) a##b##c
#define CAT(a, b, c) CAT2(a, b, c)
#define KERNEL_SINGLE CAT(LinearBasis_, NAMESPACE, _Generic_InterpolateArray)

#if defined(ORACLE_REF_GOLD)
typedef Data::Dense RefData;
extern "C" void KERNEL_SINGLE(Device* device, const int dim, const int DofPerNode, const double* x,
	const Matrix<int>* index, const Matrix<double>* surplus, double* value);
#else
typedef Data::Sparse RefData;
extern "C" void KERNEL_SINGLE(Device* device, const int dim, const int DofPerNode, const double* x,
	const int nfreqs, const XPS* xps, const Chains* chains, const Matrix<double>* surplus, double* value);
#endif

struct RefHandle
{
	RefData* data;
	int nstates;
};

extern "C" {

// Load `nstates` grid files (the reference loader; abort()s on malformed input,
// like the reference does).  `nagents` plays the role of the cfg's n_agents.
void* ref_load(const char* const* paths, int nstates, int nagents)
{
	g_nagents = nagents;
	RefHandle* h = new RefHandle;
	h->nstates = nstates;
	h->data = new RefData(nstates);
	for (int s = 0; s < nstates; s++)
		h->data->load(paths[s], s);
	return h;
}

void ref_free(void* hv)
{
	RefHandle* h = (RefHandle*)hv;
	delete h->data;
	delete h;
}

// info[0..5] = dim, nno, TotalDof, nfreqs, szxps, row stride (doubles) of surplus
void ref_info(void* hv, int istate, int* info)
{
	RefHandle* h = (RefHandle*)hv;
	RefData& d = *h->data;
	Matrix<double>& s = RefAccess::surplus(d, istate);
	info[0] = RefAccess::dim(d);
	info[1] = s.dimy();
	info[2] = RefAccess::TotalDof(d);
#if defined(ORACLE_REF_GOLD)
	info[3] = 0; info[4] = 0;
#else
	info[3] = RefAccess::nfreqs(d, istate);
	info[4] = (int)RefAccess::xps(d, istate).size();
#endif
	info[5] = s.dimy() > 1 ? (int)(&s(1, 0) - &s(0, 0)) : s.dimx();
}

// Surplus rows in the loader's row order (the x86 loader reorders them).
void ref_get_surplus(void* hv, int istate, double* out)
{
	RefHandle* h = (RefHandle*)hv;
	Matrix<double>& s = RefAccess::surplus(*h->data, istate);
	for (int i = 0; i < s.dimy(); i++)
		for (int j = 0; j < s.dimx(); j++)
			out[(size_t)i * s.dimx() + j] = s(i, j);
}

// Dense index matrix: out[n*2*dim + k] = i, out[n*2*dim + dim + k] = j.
void ref_get_index(void* hv, int istate, int* out)
{
	RefHandle* h = (RefHandle*)hv;
	RefData& d = *h->data;
	int dim = RefAccess::dim(d);
	int vdim = dim / AVX_VECTOR_SIZE + (dim % AVX_VECTOR_SIZE ? 1 : 0);
	vdim *= AVX_VECTOR_SIZE;
	Matrix<int>& m = RefAccess::index(d, istate);
	for (int n = 0; n < m.dimy(); n++)
		for (int k = 0; k < dim; k++)
		{
			out[(size_t)n * 2 * dim + k] = m(n, k);
			out[(size_t)n * 2 * dim + dim + k] = m(n, k + vdim);
		}
}

#if !defined(ORACLE_REF_GOLD) && !defined(ORACLE_REF_AVX)
// x86 xps: out[3*k + {0,1,2}] = {i, j, dim}
void ref_get_xps(void* hv, int istate, int* out)
{
	RefHandle* h = (RefHandle*)hv;
	XPS& x = RefAccess::xps(*h->data, istate);
	for (size_t k = 0; k < x.size(); k++)
	{
		out[3 * k + 0] = x[k].i;
		out[3 * k + 1] = x[k].j;
		out[3 * k + 2] = x[k].index;
	}
}

void ref_get_chains(void* hv, int istate, int* out)
{
	RefHandle* h = (RefHandle*)hv;
	Chains& c = RefAccess::chains(*h->data, istate);
	for (size_t k = 0; k < c.size(); k++)
		out[k] = c[k];
}

// Addresses of the loaded state's containers, as the reference's test hands
// them to a kernel symbol (LinearBasis/tests/InterpolateArray/test.cpp:312-313):
// out[0] XPS*, out[1] Chains*, out[2] Matrix<double>* (surplus); *nfreqs.
void ref_containers(void* hv, int istate, void** out, int* nfreqs)
{
	RefHandle* h = (RefHandle*)hv;
	out[0] = &RefAccess::xps(*h->data, istate);
	out[1] = &RefAccess::chains(*h->data, istate);
	out[2] = &RefAccess::surplus(*h->data, istate);
	*nfreqs = RefAccess::nfreqs(*h->data, istate);
}
#endif

// Interpolate npts points of state `istate`, one reference kernel call per
// point, points spread over `nthreads` host threads (the parent solver calls
// the plugin once per point from a thread pool).  X is npts x dim, out is
// npts x TotalDof (row-major, packed).
void ref_interpolate_batch(void* hv, int istate, long npts, const double* X, double* out, int nthreads)
{
	RefHandle* h = (RefHandle*)hv;
	RefData& d = *h->data;
	const int dim = RefAccess::dim(d);
	const int TD = RefAccess::TotalDof(d);
	const int TDpad = (TD + 15) / 16 * 16;
	if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
	if (nthreads < 1) nthreads = 1;
	std::atomic<long> next(0);
	auto worker = [&]()
	{
#if defined(ORACLE_REF_AVX512)
		Device dev;
		Devices::serial(dev);
		Device* device = &dev;
#else
		Device* device = nullptr;
#endif
		double* xbuf = (double*)aligned_alloc(64, sizeof(double) * ((dim + 15) / 16 * 16));
		double* vbuf = (double*)aligned_alloc(64, sizeof(double) * TDpad);
		memset(vbuf, 0, sizeof(double) * TDpad);
		for (;;)
		{
			long p0 = next.fetch_add(8);
			if (p0 >= npts) break;
			long p1 = p0 + 8 < npts ? p0 + 8 : npts;
			for (long p = p0; p < p1; p++)
			{
				memcpy(xbuf, X + (size_t)p * dim, sizeof(double) * dim);
#if defined(ORACLE_REF_AVX512)
				memset(vbuf, 0, sizeof(double) * TDpad);   // the kernel adds into value
#endif
#if defined(ORACLE_REF_GOLD)
				KERNEL_SINGLE(device, dim, TD, xbuf, &RefAccess::index(d, istate),
					&RefAccess::surplus(d, istate), vbuf);
#else
				KERNEL_SINGLE(device, dim, TD, xbuf, RefAccess::nfreqs(d, istate),
					&RefAccess::xps(d, istate), &RefAccess::chains(d, istate),
					&RefAccess::surplus(d, istate), vbuf);
#endif
				memcpy(out + (size_t)p * TD, vbuf, sizeof(double) * TD);
			}
		}
		free(xbuf);
		free(vbuf);
	};
	std::vector<std::thread> pool;
	for (int t = 1; t < nthreads; t++) pool.emplace_back(worker);
	worker();
	for (auto& t : pool) t.join();
}

} // extern "C"
