// Row-gather roof of one GPU: how fast random surplus-sized rows can be read
// from an L2-resident region, which is what the forward kernels do for every
// (point, active node) pair.  Not part of the library: it measures the peak
// that bench.py's gather roofline divides by.
//
//   make -C hddm-solver-postprocessors_b200 probe
//   hddm-solver-postprocessors_b200/lib/row_gather_probe
//
// Forms, each over 64M random row indices into a 48 MB region (all indices
// drawn below the region's row count, so every load is in bounds):
//   ldg    : a warp reads INFL rows per iteration with 16-byte loads, each
//            lane a contiguous piece of the row (rows of 256 B .. 2 KB);
//   noalloc: the same for 1 KB rows with ld.global.nc.L1::no_allocate;
//   ring   : a per-warp shared-memory ring of R 1 KB rows filled R - 1 rows
//            ahead with cp.async (16 bytes per lane per piece), read back from
//            shared memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
	printf("%s failed: %s\n", #x, cudaGetErrorString(e_)); return 1; } } while (0)

namespace {

template <int ROWB, int INFL, bool NOALLOC>
__global__ void __launch_bounds__(256) ldg_rows(const uint4* __restrict__ base, const uint32_t* __restrict__ idx,
	long long nidx, float* out)
{
	constexpr int PER = ROWB / 16;             // 16-byte pieces per row
	constexpr int LPR = PER < 32 ? PER : 32;   // lanes per row
	constexpr int RPW = 32 / LPR;              // rows per warp load
	constexpr int IT = PER / LPR;              // loads per lane per row
	const int lane = threadIdx.x & 31;
	const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = (gridDim.x * (long long)blockDim.x) >> 5;
	const int sub = lane / LPR, sl = lane % LPR;
	float acc = 0.f;
	for (long long r0 = warp * RPW * INFL; r0 + RPW * INFL <= nidx; r0 += nw * RPW * INFL)
	{
		uint4 v[INFL][IT];
#pragma unroll
		for (int f = 0; f < INFL; f++)
		{
			const uint4* p = base + (size_t)__ldg(idx + r0 + f * RPW + sub) * PER + sl;
#pragma unroll
			for (int t = 0; t < IT; t++)
			{
				if (NOALLOC)
					asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
						: "=r"(v[f][t].x), "=r"(v[f][t].y), "=r"(v[f][t].z), "=r"(v[f][t].w) : "l"(p + t * LPR));
				else v[f][t] = __ldg(p + t * LPR);
			}
		}
#pragma unroll
		for (int f = 0; f < INFL; f++)
#pragma unroll
			for (int t = 0; t < IT; t++)
				acc += __uint_as_float(v[f][t].x) + __uint_as_float(v[f][t].y) + __uint_as_float(v[f][t].z) +
				       __uint_as_float(v[f][t].w);
	}
	if (acc == 1.2345f) out[0] = acc;   // keeps the loads; never true for the zeroed region
}

__device__ __forceinline__ void cp_async16(void* smem, const void* g)
{
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(s), "l"(g));
}

template <int R>
__global__ void __launch_bounds__(256) ring_rows(const float4* __restrict__ base, const uint32_t* __restrict__ idx,
	long long nidx, float* out)
{
	extern __shared__ float4 sm[];
	const int lane = threadIdx.x & 31;
	float4* slots = sm + (size_t)(threadIdx.x >> 5) * R * 64;   // R rows of 64 float4
	const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = (gridDim.x * (long long)blockDim.x) >> 5;
	const long long mine = warp < nidx ? (nidx - 1 - warp) / nw + 1 : 0;   // rows warp + k * nw
	float acc = 0.f;
	for (int k = 0; k < R - 1; k++)
	{
		if (k < mine)
		{
			const float4* row = base + (size_t)__ldg(idx + warp + k * nw) * 64;
			cp_async16(slots + k * 64 + lane, row + lane);
			cp_async16(slots + k * 64 + 32 + lane, row + 32 + lane);
		}
		asm volatile("cp.async.commit_group;");
	}
	for (long long k = 0; k < mine; k++)
	{
		const long long kn = k + R - 1;
		if (kn < mine)
		{
			const int s = (int)(kn % R);
			const float4* row = base + (size_t)__ldg(idx + warp + kn * nw) * 64;
			cp_async16(slots + s * 64 + lane, row + lane);
			cp_async16(slots + s * 64 + 32 + lane, row + 32 + lane);
		}
		asm volatile("cp.async.commit_group;");
		asm volatile("cp.async.wait_group %0;" :: "n"(R - 1));
		__syncwarp();
		const int s = (int)(k % R);
		const float4 a = slots[s * 64 + lane], b = slots[s * 64 + 32 + lane];
		acc += a.x + a.w + b.x + b.w;
		__syncwarp();
	}
	asm volatile("cp.async.wait_group 0;");
	if (acc == 1.2345f) out[0] = acc;
}

} // namespace

int main()
{
	int sms = 0;
	CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
	const size_t region = 48ull << 20;
	const long long nidx = 64ll << 20;
	uint4* base = nullptr;
	uint32_t* didx = nullptr;
	float* out = nullptr;
	CK(cudaMalloc(&base, region));
	CK(cudaMemset(base, 0, region));
	CK(cudaMalloc(&didx, nidx * 4));
	CK(cudaMalloc(&out, 16));
	cudaEvent_t e0, e1;
	CK(cudaEventCreate(&e0));
	CK(cudaEventCreate(&e1));
	std::vector<uint32_t> h(nidx);
	std::mt19937_64 rng(1);
	auto timed = [&](const char* form, int rowb, int infl, int bps, auto launch) -> int
	{
		launch();
		CK(cudaGetLastError());
		CK(cudaEventRecord(e0));
		for (int r = 0; r < 3; r++) launch();
		CK(cudaEventRecord(e1));
		CK(cudaEventSynchronize(e1));
		float ms = 0.f;
		CK(cudaEventElapsedTime(&ms, e0, e1));
		const double rows = 3.0 * (double)nidx;
		printf("%-8s row %5d B  in flight %d  blocks/SM %d: %6.2f G rows/s  %6.2f TB/s\n", form, rowb, infl, bps,
		       rows / (ms * 1e-3) / 1e9, rows * rowb / (ms * 1e-3) / 1e12);
		return 0;
	};
	for (int rowb : { 256, 512, 1024, 2048 })
	{
		const uint32_t nrows = (uint32_t)(region / rowb);
		for (long long k = 0; k < nidx; k++) h[k] = (uint32_t)(rng() % nrows);
		CK(cudaMemcpy(didx, h.data(), nidx * 4, cudaMemcpyHostToDevice));
		for (int bps : { 4, 8 })
		{
			int rc = 0;
			if (rowb == 256)
			{
				rc |= timed("ldg", rowb, 2, bps, [&] { ldg_rows<256, 2, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
				rc |= timed("ldg", rowb, 4, bps, [&] { ldg_rows<256, 4, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
			}
			if (rowb == 512)
			{
				rc |= timed("ldg", rowb, 2, bps, [&] { ldg_rows<512, 2, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
				rc |= timed("ldg", rowb, 4, bps, [&] { ldg_rows<512, 4, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
			}
			if (rowb == 1024)
			{
				rc |= timed("ldg", rowb, 1, bps, [&] { ldg_rows<1024, 1, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
				rc |= timed("ldg", rowb, 2, bps, [&] { ldg_rows<1024, 2, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
				rc |= timed("noalloc", rowb, 2, bps, [&] { ldg_rows<1024, 2, true><<<sms * bps, 256>>>(base, didx, nidx, out); });
			}
			if (rowb == 2048)
			{
				rc |= timed("ldg", rowb, 1, bps, [&] { ldg_rows<2048, 1, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
				rc |= timed("ldg", rowb, 2, bps, [&] { ldg_rows<2048, 2, false><<<sms * bps, 256>>>(base, didx, nidx, out); });
			}
			if (rc) return 1;
		}
		if (rowb == 1024)
		{
			CK(cudaFuncSetAttribute(ring_rows<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * 4 * 1024));
			CK(cudaFuncSetAttribute(ring_rows<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * 8 * 1024));
			for (int bps : { 4, 6 })
				if (timed("ring", rowb, 4, bps, [&] {
					ring_rows<4><<<sms * bps, 256, 8 * 4 * 1024>>>(reinterpret_cast<const float4*>(base), didx, nidx, out); }))
					return 1;
			if (timed("ring", rowb, 8, 3, [&] {
				ring_rows<8><<<sms * 3, 256, 8 * 8 * 1024>>>(reinterpret_cast<const float4*>(base), didx, nidx, out); }))
				return 1;
		}
	}
	CK(cudaDeviceSynchronize());
	printf("ok\n");
	return 0;
}
