// The postprocessor plugin surface (include/sgi_plugin.h) over the C ABI.
//
// Error behaviour follows the reference plugin: a bad call prints the
// reference's message through the parent's MPI_Process (include/process.h),
// when the parent provides one, and aborts; without a parent it prints to
// stderr and calls abort().
#include <cuda_runtime_api.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "sgi.h"
#include "sgi_kernels.h"
#include "sgi_plugin.h"

// The parent's process facade (include/process.h:8-28), bound weakly.
class MPI_Process
{
public :
	void abort() __attribute__((weak));
	void cout(const char* format, ...) __attribute__((weak));
	void cerr(const char* format, ...) __attribute__((weak));
};
extern "C" int MPI_Process_get(MPI_Process**) __attribute__((weak));

namespace {

[[noreturn]] void die(const char* fmt, ...)
{
	char buf[2048];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	MPI_Process* process = nullptr;
	if (MPI_Process_get && MPI_Process_get(&process) == 0 && process)
	{
		process->cerr("%s", buf);
		process->abort();
	}
	fputs(buf, stderr);
	fflush(stderr);
	abort();
}

void say(const char* fmt, ...)
{
	if (!getenv("SGI_PLUGIN_VERBOSE")) return;
	va_list ap;
	va_start(ap, fmt);
	vfprintf(stdout, fmt, ap);
	va_end(ap);
}

// Globals behind Parameters' references (the reference keeps them global for
// Fortran, LinearBasis/cpu/include/parameters.c:1-17).
int g_priority = 0;
int g_nagents = 0;
double g_surplusCutoff = 0.0;
bool g_surplusCutoffDefined = false;

} // namespace

namespace SGI_PLUGIN_NAMESPACE {

class Device
{
public :
	int index = 0;
	int available = 1;
	int warpSize = 32;
	int cc = 0;
	int sms = 0;
};

size_t SIMDVector::getLength(size_t szelement) const
{
	if (szelement == 4 || szelement == 8) return (size_t)device->warpSize;
	die("Unsupported vector element size = %zu\n", szelement);
}

// Reads hddm-solver.cfg: "name value !comment" lines, the keys the CUDA
// variant reads (LinearBasis/cuda/src/parameters.cpp:96-150).
Parameters::Parameters(const std::string& targetSuffix, const std::string& configFile) :
	priority(g_priority), nagents(g_nagents), surplusCutoff(g_surplusCutoff),
	surplusCutoffDefined(g_surplusCutoffDefined)
{
	say("LOADING \"%s\" POSTPROCESSOR CONFIG (%s)\n", targetSuffix.c_str(), configFile.c_str());
	bool havePriority = false, haveNagents = false, haveCutoff = false;
	FILE* cfg = fopen(configFile.c_str(), "r");
	if (!cfg) die("Cannot open config file \"%s\"\n", configFile.c_str());
	char* line = nullptr;
	size_t szline = 0;
	while (getline(&line, &szline, cfg) != -1)
	{
		char* save = nullptr;
		char* name = strtok_r(line, " \t\n", &save);
		if (!name || name[0] == '!') continue;
		char* value = strtok_r(nullptr, " \t\n", &save);
		if (!value || value[0] == '!')
		{
			std::string n(name);
			fclose(cfg);
			free(line);
			die("Missing \"%s\" parameter value\n", n.c_str());
		}
		if (!strcmp(name, "priorityCUDA")) { priority = atoi(value); havePriority = true; }
		else if (!strcmp(name, "n_agents") || !strcmp(name, "nagents")) { nagents = atoi(value); haveNagents = true; }
		else if (!strcmp(name, "surplusCutoff")) { surplusCutoff = atof(value); haveCutoff = true; }
	}
	free(line);
	fclose(cfg);
	surplusCutoffDefined = haveCutoff;
	if (!havePriority) die("Required parameter \"%s\" is undefined\n", "priority");
	if (!haveNagents) die("Required parameter \"%s\" is undefined\n", "nagents");
}

// All states of one multistate set; each state a device grid.
class DataImpl : public Data
{
public :
	int nstates, dim = 0, TotalDof = 0;
	std::vector<sgi_grid_t> grids;
	std::vector<bool> loaded;

	explicit DataImpl(int n) : nstates(n), grids(n, nullptr), loaded(n, false) { }

	// LinearBasis/cuda/src/Data.cu:348-949 (via gold/src/Data.cpp:322-436 checks)
	void load(const char* filename, int istate) override
	{
		const Parameters& params = Interpolator::getInstance()->getParameters();
		if (istate < 0 || istate >= nstates) die("State %d index out of range 0 .. %d\n", istate, nstates - 1);
		if (loaded[istate]) die("State %d data is already loaded\n", istate);
		bool first = true;
		for (int s = 0; s < nstates; s++) if (loaded[s]) first = false;
		int dev = 0;
		cudaGetDevice(&dev);
		sgi_grid_t g = nullptr;
		int d = 0, td = 0;
		// SGI_LAYOUT_CACHE: unset or "0" reads the file as the reference does;
		// "1" keeps the built device layout in "<file>.sgi-layout"; any other
		// value is a directory for those caches
		const char* cache = getenv("SGI_LAYOUT_CACHE");
		if (cache && *cache && strcmp(cache, "0"))
		{
			std::string cpath;
			if (strcmp(cache, "1"))
			{
				const char* base = strrchr(filename, '/');
				cpath = std::string(cache) + "/" + (base ? base + 1 : filename) + ".sgi-layout";
			}
			int rc = sgi_grid_load(filename, params.nagents, dev, 0u, cpath.empty() ? nullptr : cpath.c_str(), &g, nullptr);
			if (rc) die("%s\n", sgi_last_error());
			sgi_grid_info info;
			sgi_grid_info_get(g, &info);
			d = info.dim; td = info.TotalDof;
		}
		else
		{
			sgi_host_grid_t hg = nullptr;
			int rc = sgi_host_grid_read_plt(filename, params.nagents, &hg);
			if (rc) die("%s\n", sgi_last_error());
			int nno = 0;
			sgi_host_grid_view(hg, &d, &nno, &td, nullptr, nullptr);
			if (!first && (d != dim || td != TotalDof)) sgi_host_grid_free(hg);
			else
			{
				rc = sgi_grid_create(hg, dev, 0u, &g);
				sgi_host_grid_free(hg);
				if (rc) die("%s\n", sgi_last_error());
			}
		}
		if (first) { dim = d; TotalDof = td; }
		else
		{
			if (d != dim) { if (g) sgi_grid_destroy(g); die("File \"%s\" # of dimensions (%d) mismatches another state (%d)\n", filename, d, dim); }
			if (td != TotalDof) { if (g) sgi_grid_destroy(g); die("File \"%s\" TotalDof (%d) mismatches another state (%d)\n", filename, td, TotalDof); }
		}
		grids[istate] = g;
		loaded[istate] = true;
	}

	void clear() override
	{
		for (int s = 0; s < nstates; s++)
		{
			if (grids[s]) sgi_grid_destroy(grids[s]);
			grids[s] = nullptr;
			loaded[s] = false;
		}
	}

	~DataImpl() override { clear(); }
};

namespace {
std::unique_ptr<Interpolator> interp;
std::mutex interp_mtx;
}

const Parameters& Interpolator::getParameters() const { return params; }

Interpolator::Interpolator(const std::string& targetSuffix, const std::string& configFile) :
	jit(false), params(targetSuffix, configFile) { }

Interpolator::~Interpolator() { }

Interpolator* Interpolator::getInstance()
{
	std::lock_guard<std::mutex> lk(interp_mtx);
	if (!interp) interp.reset(new Interpolator("b200"));
	return interp.get();
}

static void check_dof(const DataImpl* data, int DofPerNode)
{
	if (DofPerNode != data->TotalDof)
		die("Requested DofPerNode (%d) mismatches actual data TotalDof (%d)\n", DofPerNode, data->TotalDof);
}

void Interpolator::interpolate(Device* device, Data* data_, const int istate, const real* x,
	const int DofPerNode, real* value)
{
	(void)device;
	DataImpl* data = static_cast<DataImpl*>(data_);
	check_dof(data, DofPerNode);
	if (istate < 0 || istate >= data->nstates || !data->loaded[istate])
		die("State %d is not loaded\n", istate);
	const long long off[2] = { 0, 1 };
	int rc = sgi_interpolate_host(1, &data->grids[istate], off, x, value, SGI_FP64);
	if (rc) die("%s\n", sgi_last_error());
}

void Interpolator::interpolate(Device* device, Data* data_, const real** x, const int DofPerNode, real** value)
{
	(void)device;
	DataImpl* data = static_cast<DataImpl*>(data_);
	check_dof(data, DofPerNode);
	const int n = data->nstates;
	for (int s = 0; s < n; s++) if (!data->loaded[s]) die("State %d is not loaded\n", s);
	std::vector<long long> off(n + 1);
	for (int s = 0; s <= n; s++) off[s] = s;
	std::vector<double> xb((size_t)n * data->dim), vb((size_t)n * data->TotalDof);
	for (int s = 0; s < n; s++) memcpy(&xb[(size_t)s * data->dim], x[s], sizeof(double) * data->dim);
	int rc = sgi_interpolate_host(n, data->grids.data(), off.data(), xb.data(), vb.data(), SGI_FP64);
	if (rc) die("%s\n", sgi_last_error());
	for (int s = 0; s < n; s++) memcpy(value[s], &vb[(size_t)s * data->TotalDof], sizeof(double) * data->TotalDof);
}

} // namespace SGI_PLUGIN_NAMESPACE

using namespace SGI_PLUGIN_NAMESPACE;

namespace {

struct Devices
{
	std::vector<Device> devs;
	std::vector<std::unique_ptr<DeviceProperties>> props;
	std::vector<DeviceProperties*> props_raw;
	std::mutex mtx;
	Devices()
	{
		const int n = sgi_device_count();
		devs.resize(n);
		for (int i = 0; i < n; i++)
		{
			cudaDeviceProp p;
			if (cudaGetDeviceProperties(&p, i) == cudaSuccess)
			{
				devs[i].warpSize = p.warpSize;
				devs[i].cc = p.major * 10 + p.minor;
				devs[i].sms = p.multiProcessorCount;
			}
			devs[i].index = i;
		}
		for (int i = 0; i < n; i++)
		{
			props.emplace_back(new DeviceProperties(&devs[i]));
			props_raw.push_back(props.back().get());
		}
	}
};

Devices& devices()
{
	static Devices d;
	return d;
}

} // namespace

extern "C" Interpolator* getInterpolator() { return Interpolator::getInstance(); }

extern "C" Data* getData(int nstates) { return new DataImpl(nstates); }

extern "C" bool isSupported() { return sgi_device_count() > 0; }

extern "C" int getPriority() { return Interpolator::getInstance()->getParameters().priority; }

extern "C" void resetInterpolator()
{
	std::lock_guard<std::mutex> lk(interp_mtx);
	interp = nullptr;
}

extern "C" Device* tryAcquireDevice()
{
	Devices& d = devices();
	std::lock_guard<std::mutex> lk(d.mtx);
	for (auto& dev : d.devs)
		if (dev.available) { dev.available = 0; return &dev; }
	return nullptr;
}

extern "C" void releaseDevice(Device* device)
{
	if (!device) return;
	Devices& d = devices();
	std::lock_guard<std::mutex> lk(d.mtx);
	device->available++;
}

extern "C" void getDeviceProperties(DeviceProperties*** result, size_t* szresult)
{
	Devices& d = devices();
	*result = d.props_raw.empty() ? nullptr : d.props_raw.data();
	*szresult = d.props_raw.size();
}

extern "C" int sgi_plugin_data_load(Data* data, const char* filename, int istate)
{
	data->load(filename, istate);
	return 0;
}

extern "C" void sgi_plugin_interpolate(Device* device, Data* data, int istate, const double* x,
	int DofPerNode, double* value)
{
	getInterpolator()->interpolate(device, data, istate, x, DofPerNode, value);
}

extern "C" void sgi_plugin_interpolate_multistate(Device* device, Data* data, const double** x,
	int DofPerNode, double** value)
{
	getInterpolator()->interpolate(device, data, x, DofPerNode, value);
}

extern "C" void sgi_plugin_interpolate_batch(Device* device, Data* data_, int n, const int* istates,
	const double* x, int DofPerNode, double* value)
{
	(void)device;
	DataImpl* data = static_cast<DataImpl*>(data_);
	check_dof(data, DofPerNode);
	if (n < 0 || (n && (!istates || !x || !value))) die("Bad batch of %d points\n", n);
	if (!n) return;
	const int ns = data->nstates, dim = data->dim, TD = data->TotalDof;
	// group the pairs by state (counting sort, stable), one call over the set
	std::vector<long long> off(ns + 1, 0);
	for (int k = 0; k < n; k++)
	{
		const int s = istates[k];
		if (s < 0 || s >= ns || !data->loaded[s]) die("State %d is not loaded\n", s);
		off[s + 1]++;
	}
	for (int s = 0; s < ns; s++) off[s + 1] += off[s];
	std::vector<long long> pos(off.begin(), off.end() - 1);
	std::vector<int> row(n);
	std::vector<double> xb((size_t)n * dim), vb((size_t)n * TD);
	for (int k = 0; k < n; k++)
	{
		const long long r = pos[istates[k]]++;
		row[k] = (int)r;
		memcpy(&xb[(size_t)r * dim], x + (size_t)k * dim, sizeof(double) * dim);
	}
	int rc = sgi_interpolate_host(ns, data->grids.data(), off.data(), xb.data(), vb.data(), SGI_FP64);
	if (rc) die("%s\n", sgi_last_error());
	for (int k = 0; k < n; k++) memcpy(value + (size_t)k * TD, &vb[(size_t)row[k] * TD], sizeof(double) * TD);
}

extern "C" void sgi_plugin_data_free(Data* data) { delete data; }

extern "C" int sgi_plugin_device_index(const Device* device) { return device ? device->index : -1; }

// ------------------------------------------------ kernel-level entry points
//
// The reference's x86 kernel signatures over the x86 loader's containers
// (include/sgi_kernels.h).  The device layout of a container set is built
// once and kept, keyed on the containers' addresses and sizes and a hash of
// a sample of their contents.

namespace {

struct X86Key
{
	const void* xps;
	const void* chains;
	const void* surplus;
	size_t szxps, nchains;
	int dim, TD, nno, dimx, ld, nfreqs;
	uint64_t sample;

	bool operator==(const X86Key& o) const
	{
		return xps == o.xps && chains == o.chains && surplus == o.surplus && szxps == o.szxps &&
		       nchains == o.nchains && dim == o.dim && TD == o.TD && nno == o.nno && dimx == o.dimx &&
		       ld == o.ld && nfreqs == o.nfreqs && sample == o.sample;
	}
};

struct X86Grid
{
	X86Key key;
	int device;
	sgi_grid_t grid;
};

std::mutex x86_mtx;
std::vector<X86Grid> x86_grids;      // most recently built last
constexpr size_t X86_GRIDS_MAX = 64;

// FNV-1a over at most ~4,096 sampled entries of each container.
uint64_t x86_sample(const sgi_x86::XPS& xps, const sgi_x86::Chains& chains, const sgi_x86::Matrix<double>& s)
{
	uint64_t h = 1469598103934665603ull;
	auto mix = [&](const void* p, size_t n)
	{
		const unsigned char* b = static_cast<const unsigned char*>(p);
		for (size_t k = 0; k < n; k++) { h ^= b[k]; h *= 1099511628211ull; }
	};
	const size_t sx = std::max<size_t>(1, xps.size() / 4096);
	for (size_t k = 0; k < xps.size(); k += sx) mix(&xps[k], sizeof(xps[k]));
	const size_t sc = std::max<size_t>(1, chains.size() / 4096);
	for (size_t k = 0; k < chains.size(); k += sc) mix(&chains[k], sizeof(chains[k]));
	const size_t ss = std::max<size_t>(1, s.data.size() / 4096);
	for (size_t k = 0; k < s.data.size(); k += ss) mix(&s.data[k], sizeof(double));
	return h;
}

// The grid of one container set on the current device: node n's components
// from its chain (xps entries up to the first 0), its row of the matrix.
sgi_grid_t x86_grid(int dim, int DofPerNode, int nfreqs, const sgi_x86::XPS* xps_, const sgi_x86::Chains* chains_,
	const sgi_x86::Matrix<double>* surplus_)
{
	if (!xps_ || !chains_ || !surplus_) die("Null XPS, Chains or surplus\n");
	const sgi_x86::XPS& xps = *xps_;
	const sgi_x86::Chains& chains = *chains_;
	const sgi_x86::Matrix<double>& s = *surplus_;
	const int nno = s.dimY;
	if (dim <= 0 || nno < 0 || nfreqs < 0 || DofPerNode <= 0 || DofPerNode > s.dimX ||
	    s.dimX_aligned < s.dimX || s.data.size() < (size_t)nno * s.dimX_aligned ||
	    chains.size() < (size_t)nno * nfreqs)
		die("Inconsistent sparse data: dim %d, nno %d, nfreqs %d, DofPerNode %d, surplus %d x %d\n",
		    dim, nno, nfreqs, DofPerNode, s.dimY, s.dimX);
	int dev = 0;
	cudaGetDevice(&dev);
	const X86Key key{ xps.data(), chains.data(), s.data.data(), xps.size(), chains.size(), dim, DofPerNode, nno,
	                  s.dimX, s.dimX_aligned, nfreqs, x86_sample(xps, chains, s) };
	std::lock_guard<std::mutex> lk(x86_mtx);
	for (size_t k = 0; k < x86_grids.size(); k++)
		if (x86_grids[k].device == dev && x86_grids[k].key == key) return x86_grids[k].grid;
	std::vector<int> index((size_t)nno * 2 * dim, 0);
	std::vector<double> sur((size_t)nno * DofPerNode);
	for (int n = 0; n < nno; n++)
	{
		for (int f = 0; f < nfreqs; f++)
		{
			const uint16_t id = chains[(size_t)n * nfreqs + f];
			if (!id) break;
			if (id >= xps.size() || xps[id].index >= dim) die("Chain entry %d of node %d out of range\n", (int)id, n);
			index[(size_t)n * 2 * dim + xps[id].index] = xps[id].i;
			index[(size_t)n * 2 * dim + dim + xps[id].index] = xps[id].j;
		}
		memcpy(&sur[(size_t)n * DofPerNode], &s.data[(size_t)n * s.dimX_aligned], sizeof(double) * DofPerNode);
	}
	sgi_host_grid_t hg = nullptr;
	if (sgi_host_grid_from_dense(dim, nno, DofPerNode, index.data(), sur.data(), &hg)) die("%s\n", sgi_last_error());
	sgi_grid_t g = nullptr;
	const int rc = sgi_grid_create(hg, dev, 0u, &g);
	sgi_host_grid_free(hg);
	if (rc) die("%s\n", sgi_last_error());
	if (x86_grids.size() >= X86_GRIDS_MAX)
	{
		sgi_grid_destroy(x86_grids.front().grid);
		x86_grids.erase(x86_grids.begin());
	}
	x86_grids.push_back(X86Grid{ key, dev, g });
	return g;
}

} // namespace

// LinearBasis/x86/src/InterpolateArray.cpp:9-54
extern "C" void LinearBasis_b200_Generic_InterpolateArray(void* device, const int dim, const int DofPerNode,
	const double* x, const int nfreqs, const sgi_x86::XPS* xps, const sgi_x86::Chains* chains,
	const sgi_x86::Matrix<double>* surplus, double* value)
{
	(void)device;
	if (!x || !value) die("Null x or value\n");
	sgi_grid_t g = x86_grid(dim, DofPerNode, nfreqs, xps, chains, surplus);
	const long long off[2] = { 0, 1 };
	if (sgi_interpolate_host(1, &g, off, x, value, SGI_FP64)) die("%s\n", sgi_last_error());
}

// LinearBasis/x86/src/InterpolateArrayManyMultistate.cpp:9-60
extern "C" void LinearBasis_b200_Generic_InterpolateArrayManyMultistate(void* device, const int dim,
	const int DofPerNode, const int count, const double* const* x, const int* nfreqs, const sgi_x86::XPS* xps,
	const sgi_x86::Chains* chains, const sgi_x86::Matrix<double>* surplus, double** value)
{
	(void)device;
	if (count < 0 || (count && (!x || !nfreqs || !xps || !chains || !surplus || !value))) die("Bad multistate call\n");
	if (!count) return;
	std::vector<sgi_grid_t> grids(count);
	std::vector<long long> off(count + 1);
	std::vector<double> xb((size_t)count * dim), vb((size_t)count * DofPerNode);
	for (int k = 0; k < count; k++)
	{
		grids[k] = x86_grid(dim, DofPerNode, nfreqs[k], &xps[k], &chains[k], &surplus[k]);
		off[k] = k;
		if (!x[k] || !value[k]) die("Null x or value of state %d\n", k);
		memcpy(&xb[(size_t)k * dim], x[k], sizeof(double) * dim);
	}
	off[count] = count;
	if (sgi_interpolate_host(count, grids.data(), off.data(), xb.data(), vb.data(), SGI_FP64))
		die("%s\n", sgi_last_error());
	for (int k = 0; k < count; k++) memcpy(value[k], &vb[(size_t)k * DofPerNode], sizeof(double) * DofPerNode);
}
