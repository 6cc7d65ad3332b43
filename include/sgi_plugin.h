/*
 * sgi_plugin.h — the postprocessor plugin surface, as the parent HDDM solver
 * binds it (dlopen + dlsym of the extern "C" names, then virtual calls).
 *
 * The class declarations keep the reference's layout and virtual-function
 * order so that the vtables match:
 *   Interpolator  include/interpolator.h:18-42 (interpolate single, interpolate
 *                 multistate, destructor; members `bool jit; const Parameters`)
 *   Parameters    LinearBasis/cpu/include/parameters.h:9-18 with the fields of
 *                 parameters.c:1-17 held by reference
 *   Data          LinearBasis/cuda/include/Data.h:482-551 (virtual load, clear,
 *                 destructor)
 * `real` is double, as every reference kernel assumes.
 */
#ifndef SGI_PLUGIN_H
#define SGI_PLUGIN_H

#include <cstddef>
#include <string>

#ifndef SGI_PLUGIN_NAMESPACE
#define SGI_PLUGIN_NAMESPACE b200
#endif

namespace SGI_PLUGIN_NAMESPACE {

typedef double real;

class Device;

enum BasisType
{
	LinearBasisType,
	PolynomialBasisType
};

struct Parameters
{
	int& priority;              // priorityCUDA in hddm-solver.cfg
	int& nagents;               // n_agents / nagents: the grid dimension
	double& surplusCutoff;      // parsed, unused by the interpolation (as in the reference)
	bool& surplusCutoffDefined;

	Parameters(const std::string& targetSuffix, const std::string& configFile = "hddm-solver.cfg");
};

// A multistate set of grids (LinearBasis/cuda/include/Data.h:482-551: virtual
// load, virtual clear, virtual destructor, in that vtable order).  getData()
// returns the library's implementation.
class Data
{
public :
	// Reads one .plt grid (dimension checked against the config's n_agents,
	// all states sharing dim and TotalDof) and uploads it to the current CUDA
	// device.
	virtual void load(const char* filename, int istate) = 0;

	// Unloads all states.
	virtual void clear() = 0;

	virtual ~Data() { }
};

// Vector width hint of a device (LinearBasis/cuda/include/SIMDVector.h:10-38):
// a warp, for 4- and 8-byte elements.
class SIMDVector
{
	const Device* device;

public :
	explicit SIMDVector(const Device* d) : device(d) { }

	virtual size_t getLength(size_t szelement) const;

	virtual ~SIMDVector() { }
};

// LinearBasis/cuda/include/DeviceProperties.h:10-22
class DeviceProperties
{
	SIMDVector simdVector;

public :
	explicit DeviceProperties(const Device* device) : simdVector(device) { }

	virtual const SIMDVector* getSIMDVector() const { return &simdVector; }

	virtual ~DeviceProperties() { }
};

class Interpolator
{
	bool jit;

	const Parameters params;

public :
	const Parameters& getParameters() const;

	Interpolator(const std::string& targetSuffix, const std::string& configFile = "hddm-solver.cfg");

	static Interpolator* getInstance();

	// Interpolate one point of state istate.  Replaces
	// LinearBasis/cuda/src/Interpolator.cpp:41-73.
	virtual void interpolate(Device* device, Data* data,
		const int istate, const real* x, const int DofPerNode, real* value);

	// Interpolate one point per state, all states of `data`.  Replaces
	// LinearBasis/cuda/src/Interpolator.cpp:77-109.
	virtual void interpolate(Device* device, Data* data,
		const real** x, const int DofPerNode, real** value);

	virtual ~Interpolator();
};

} // namespace SGI_PLUGIN_NAMESPACE

extern "C" {

// LinearBasis/cuda/src/Interpolator.cpp:132-135
SGI_PLUGIN_NAMESPACE::Interpolator* getInterpolator();

// LinearBasis/cuda/src/Data.cu:1210-1213: a Data object for nstates states.
SGI_PLUGIN_NAMESPACE::Data* getData(int nstates);

// LinearBasis/cuda/src/supported.cpp:13-20: true if at least one GPU exists.
bool isSupported();

// LinearBasis/cuda/src/priority.cpp:5-10: priorityCUDA from the config.
int getPriority();

// LinearBasis/cuda/src/reset.cpp:14-17: drops the Interpolator singleton.
void resetInterpolator();

// LinearBasis/cuda/src/Devices.cu:115-123: exclusive per-thread GPU handles.
SGI_PLUGIN_NAMESPACE::Device* tryAcquireDevice();
void releaseDevice(SGI_PLUGIN_NAMESPACE::Device* device);

// LinearBasis/cuda/src/DeviceProperties.cpp:46-51
void getDeviceProperties(SGI_PLUGIN_NAMESPACE::DeviceProperties*** result, size_t* szresult);

// Plain-C helpers for hosts that cannot make C++ virtual calls (no reference
// counterpart): load a state, interpolate through the Interpolator singleton.
int sgi_plugin_data_load(SGI_PLUGIN_NAMESPACE::Data* data, const char* filename, int istate);
void sgi_plugin_interpolate(SGI_PLUGIN_NAMESPACE::Device* device, SGI_PLUGIN_NAMESPACE::Data* data,
	int istate, const double* x, int DofPerNode, double* value);
void sgi_plugin_interpolate_multistate(SGI_PLUGIN_NAMESPACE::Device* device, SGI_PLUGIN_NAMESPACE::Data* data,
	const double** x, int DofPerNode, double** value);
void sgi_plugin_data_free(SGI_PLUGIN_NAMESPACE::Data* data);

// Many (state, point) pairs in one call (no reference counterpart; the
// reference takes one point of one state, or one point per state, per call:
// include/interpolator.h:32-37).  Point k is x[k*dim .. k*dim + dim) of state
// istates[k] (states may repeat, in any order); its values go to
// value[k*DofPerNode ..].  The pairs are grouped by state and evaluated in
// one batched forward over the states' grids (FP64 form: the same bits as n
// single-state calls).  A solver's time step hands all its agents' points to
// one call instead of one call per point.  Errors abort with the reference's
// messages, as the Interpolator calls do.
void sgi_plugin_interpolate_batch(SGI_PLUGIN_NAMESPACE::Device* device, SGI_PLUGIN_NAMESPACE::Data* data,
	int n, const int* istates, const double* x, int DofPerNode, double* value);
int sgi_plugin_device_index(const SGI_PLUGIN_NAMESPACE::Device* device);

}

#endif /* SGI_PLUGIN_H */
