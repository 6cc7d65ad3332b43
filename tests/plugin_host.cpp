// Test host for the plugin surface: binds the library the way the HDDM
// solver's postprocessor loader does (dlopen, dlsym of the extern "C" names,
// then virtual calls through the reference's class layouts declared in
// include/sgi_plugin.h), without linking against it.
//
//   plugin_host <library> <grid.plt[,grid2.plt,...]> <nstates> <x_0> ... <x_{dim-1}>
//
// Loads the grid files into the states of one Data object (state s takes
// file s % nfiles), then prints
//   single <v_0> ... <v_{TotalDof-1}>           interpolate(device, data, 0, x, ...)
//   multi <s> <v_0> ... <v_{TotalDof-1}>        interpolate(device, data, xs, ...), per state
//   batch <k> <s> <v_0> ...                     sgi_plugin_interpolate_batch over 2 * nstates
//                                               (state, point) pairs: state (5k + 1) % nstates,
//                                               point x_d + 0.01 k (mod 1) in every dimension d
//   latency <n> <us per batch call> <us for n single calls>
// with 17 significant digits.  hddm-solver.cfg must be in the working
// directory (n_agents = the grid's dimension).  Exit status 2 when the
// library or a symbol is missing or no GPU is supported.
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
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

	auto batch = sym<void (*)(Device*, Data*, int, const int*, const double*, int, double*)>(
		so, "sgi_plugin_interpolate_batch");
	std::vector<std::string> files;
	for (std::string rest = argv[2];;)
	{
		const size_t c = rest.find(',');
		files.push_back(rest.substr(0, c));
		if (c == std::string::npos) break;
		rest = rest.substr(c + 1);
	}

	Interpolator* I = getInterp();
	Data* data = getDataFn(nstates);
	for (int s = 0; s < nstates; s++) data->load(files[s % files.size()].c_str(), s);   // virtual
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
	// many (state, point) pairs in one call
	const int dim = (int)x.size(), n = 2 * nstates;
	std::vector<int> st(n);
	std::vector<double> xb((size_t)n * dim), vb((size_t)n * TD, 0.0);
	for (int k = 0; k < n; k++)
	{
		st[k] = (3 * k + 1) % nstates;
		for (int d = 0; d < dim; d++) xb[(size_t)k * dim + d] = std::fmod(x[d] + 0.01 * k, 1.0);
	}
	batch(dev, data, n, st.data(), xb.data(), TD, vb.data());
	for (int k = 0; k < n; k++)
	{
		printf("batch %d %d", k, st[k]);
		for (int o = 0; o < TD; o++) printf(" %.17g", vb[(size_t)k * TD + o]);
		printf("\n");
	}
	// latency: one batch call against n single-state calls (best of 5)
	using clk = std::chrono::steady_clock;
	double tb = 1e30, ts = 1e30;
	for (int rep = 0; rep < 5; rep++)
	{
		auto t0 = clk::now();
		batch(dev, data, n, st.data(), xb.data(), TD, vb.data());
		auto t1 = clk::now();
		for (int k = 0; k < n; k++) I->interpolate(dev, data, st[k], &xb[(size_t)k * dim], TD, &vb[(size_t)k * TD]);
		auto t2 = clk::now();
		tb = std::min(tb, std::chrono::duration<double, std::micro>(t1 - t0).count());
		ts = std::min(ts, std::chrono::duration<double, std::micro>(t2 - t1).count());
	}
	printf("latency %d %.1f %.1f\n", n, tb, ts);
	release(dev);
	data->clear();
	delete data;
	dlclose(so);
	return 0;
}
