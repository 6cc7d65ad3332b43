// Test host for the plugin surface: binds the library the way the HDDM
// solver's postprocessor loader does (dlopen, dlsym of the extern "C" names,
// then virtual calls through the reference's class layouts declared in
// include/sgi_plugin.h), without linking against it.
//
//   plugin_host <library> <grid.plt> <nstates> <x_0> ... <x_{dim-1}>
//
// Loads the grid file into every state of one Data object, then prints
//   single <v_0> ... <v_{TotalDof-1}>           interpolate(device, data, 0, x, ...)
//   multi <s> <v_0> ... <v_{TotalDof-1}>        interpolate(device, data, xs, ...), per state
// with 17 significant digits.  hddm-solver.cfg must be in the working
// directory (n_agents = the grid's dimension).  Exit status 2 when the
// library or a symbol is missing or no GPU is supported.
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "sgi_plugin.h"

using namespace b200;

template <class F>
static F sym(void* so, const char* name)
{
	void* p = dlsym(so, name);
	if (!p) { fprintf(stderr, "missing symbol %s\n", name); exit(2); }
	return reinterpret_cast<F>(p);
}

int main(int argc, char** argv)
{
	if (argc < 4) { fprintf(stderr, "usage: %s <library> <grid.plt> <nstates> <x...>\n", argv[0]); return 2; }
	void* so = dlopen(argv[1], RTLD_NOW | RTLD_LOCAL);
	if (!so) { fprintf(stderr, "dlopen: %s\n", dlerror()); return 2; }
	auto isSupported = sym<bool (*)()>(so, "isSupported");
	auto getPriority = sym<int (*)()>(so, "getPriority");
	auto getInterp = sym<Interpolator* (*)()>(so, "getInterpolator");
	auto getDataFn = sym<Data* (*)(int)>(so, "getData");
	auto acquire = sym<Device* (*)()>(so, "tryAcquireDevice");
	auto release = sym<void (*)(Device*)>(so, "releaseDevice");
	if (!isSupported()) { fprintf(stderr, "no GPU\n"); return 2; }
	printf("priority %d\n", getPriority());

	const int nstates = atoi(argv[3]);
	std::vector<double> x;
	for (int k = 4; k < argc; k++) x.push_back(atof(argv[k]));

	Interpolator* I = getInterp();
	Data* data = getDataFn(nstates);
	for (int s = 0; s < nstates; s++) data->load(argv[2], s);   // virtual
	Device* dev = acquire();
	if (!dev) { fprintf(stderr, "no device acquired\n"); return 2; }

	// TotalDof is not part of the plugin surface: the caller knows it; here
	// the value array is sized generously and the known-answer length is
	// passed by the environment (default 118, the reference fixture's)
	const char* td_env = getenv("PLUGIN_HOST_TOTALDOF");
	const int TD = td_env ? atoi(td_env) : 118;
	std::vector<double> value(TD, 0.0);
	I->interpolate(dev, data, 0, x.data(), TD, value.data());   // virtual, single state
	printf("single");
	for (int o = 0; o < TD; o++) printf(" %.17g", value[o]);
	printf("\n");

	std::vector<std::vector<double>> vals(nstates, std::vector<double>(TD, 0.0));
	std::vector<const double*> xs(nstates, x.data());
	std::vector<double*> vs(nstates);
	for (int s = 0; s < nstates; s++) vs[s] = vals[s].data();
	I->interpolate(dev, data, xs.data(), TD, vs.data());          // virtual, one point per state
	for (int s = 0; s < nstates; s++)
	{
		printf("multi %d", s);
		for (int o = 0; o < TD; o++) printf(" %.17g", vals[s][o]);
		printf("\n");
	}
	release(dev);
	data->clear();
	delete data;
	dlclose(so);
	return 0;
}
