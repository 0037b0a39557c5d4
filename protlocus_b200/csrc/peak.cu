/*
 * peak.cu -- measured integer-pipe peak of the device (the roofline denominator
 * of the DP kernels, which are bound by integer ALU throughput, not by HBM or
 * tensor cores).
 *
 * Two streams of independent dependency chains, at full occupancy:
 *   int32  : r = max(r + d, e)                       2 lane-ops per step
 *   int16x2: r = __vmaxs2(__vadd2(r, d), e)          4 lane-ops per step
 * The reported peak is the larger lane-op rate.  Eight independent chains per
 * thread hide the ALU latency; the chain values are written out so nothing is
 * eliminated.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#define PEAK_CHAINS 8
#define PEAK_ITERS 4096

__global__ void __launch_bounds__(256) k_peak_i32(int *out, int seed)
{
	int r[PEAK_CHAINS], d[PEAK_CHAINS], e[PEAK_CHAINS];
#pragma unroll
	for (int k = 0; k < PEAK_CHAINS; ++k) r[k] = threadIdx.x + k, d[k] = seed + k - 3, e[k] = seed * (k + 1) - 40000;
	for (int it = 0; it < PEAK_ITERS; ++it) {
#pragma unroll
		for (int k = 0; k < PEAK_CHAINS; ++k) r[k] = max(r[k] + d[k], e[k]);
	}
	int acc = 0;
#pragma unroll
	for (int k = 0; k < PEAK_CHAINS; ++k) acc ^= r[k];
	out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void __launch_bounds__(256) k_peak_i16x2(unsigned *out, int seed)
{
	unsigned r[PEAK_CHAINS], d[PEAK_CHAINS], e[PEAK_CHAINS];
#pragma unroll
	for (int k = 0; k < PEAK_CHAINS; ++k)
		r[k] = threadIdx.x * 65537u + k, d[k] = (unsigned)(seed + k) * 0x00030001u, e[k] = 0x80108010u + k;
	for (int it = 0; it < PEAK_ITERS; ++it) {
#pragma unroll
		for (int k = 0; k < PEAK_CHAINS; ++k) r[k] = __vmaxs2(__vadd2(r[k], d[k]), e[k]);
	}
	unsigned acc = 0;
#pragma unroll
	for (int k = 0; k < PEAK_CHAINS; ++k) acc ^= r[k];
	out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

/* lane-ops per second of both streams; returns 1 on success */
extern "C" __attribute__((visibility("default")))
int pl_measure_int_peak(int32_t device, double *int32_lane_ops, double *int16x2_lane_ops)
{
	int n_sm = 0;
	void *buf = 0;
	cudaEvent_t a, b;
	float ms;
	double best32 = 0, best16 = 0;
	if (cudaSetDevice(device) != cudaSuccess) return 0;
	if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
	const int grid = n_sm * 8, block = 256;
	if (cudaMalloc(&buf, (size_t)grid * block * sizeof(int)) != cudaSuccess) return 0;
	cudaEventCreate(&a), cudaEventCreate(&b);
	const double steps = (double)grid * block * PEAK_ITERS * PEAK_CHAINS;
	for (int rep = 0; rep < 4; ++rep) {
		cudaEventRecord(a);
		k_peak_i32<<<grid, block>>>((int*)buf, 7 + rep);
		cudaEventRecord(b);
		cudaEventSynchronize(b);
		cudaEventElapsedTime(&ms, a, b);
		if (rep > 0 && steps * 2 / (ms * 1e-3) > best32) best32 = steps * 2 / (ms * 1e-3);
		cudaEventRecord(a);
		k_peak_i16x2<<<grid, block>>>((unsigned*)buf, 7 + rep);
		cudaEventRecord(b);
		cudaEventSynchronize(b);
		cudaEventElapsedTime(&ms, a, b);
		if (rep > 0 && steps * 4 / (ms * 1e-3) > best16) best16 = steps * 4 / (ms * 1e-3);
	}
	cudaEventDestroy(a), cudaEventDestroy(b);
	cudaFree(buf);
	if (cudaGetLastError() != cudaSuccess) return 0;
	*int32_lane_ops = best32, *int16x2_lane_ops = best16;
	return 1;
}
