// gf_probe.cu -- integer-pipe throughput probe: the denominator of the
// integer-pipe roofline of the squaring kernels (the device has no published
// INT32 modular-multiply peak).  Every thread runs 8 independent dependency
// chains so the measurement is throughput-bound, not latency-bound.
#include <cuda_runtime.h>

#include <cstdint>

#include "gf_arith.cuh"

namespace {

constexpr int CHAINS = 8;

template <int SET>
__global__ void __launch_bounds__(256) k_probe_mulmod(uint32_t *out, int iters, uint32_t seed)
{
	using Z = gfc::Zp<gfc::PrimeSet<SET>::p[0], gfc::PrimeSet<SET>::P31>;
	uint32_t x[CHAINS], w[CHAINS];
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
	for (int c = 0; c < CHAINS; ++c) { x[c] = (t * 2654435761u + c * 40503u + seed) % Z::p; w[c] = (x[c] ^ 0x9e3779b9u) % Z::p; }
	for (int i = 0; i < iters; ++i)
	{
#pragma unroll
		for (int c = 0; c < CHAINS; ++c) x[c] = Z::mul(x[c], w[c]);
	}
	uint32_t acc = 0;
#pragma unroll
	for (int c = 0; c < CHAINS; ++c) acc ^= x[c];
	if (acc == 0x12345678u) out[t] = acc;   // keeps the chains live
}

// Radix-2 butterfly throughput, with the root product the engine's transforms
// use for the prime set: a Montgomery product for the 32-bit primes, a Shoup
// product (root and quotient) for the 31-bit primes; then add + sub.
template <int SET>
__global__ void __launch_bounds__(256) k_probe_bfly(uint32_t *out, int iters, uint32_t seed)
{
	using Z = gfc::Zp<gfc::PrimeSet<SET>::p[0], gfc::PrimeSet<SET>::P31>;
	uint32_t a[CHAINS], b[CHAINS];
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	typename Z::root_t w;
	w.w = (seed * 747796405u + 2891336453u) % Z::p;
	if constexpr (gfc::PrimeSet<SET>::P31)
		w = gfc::RootS{ w.w, static_cast<uint32_t>((static_cast<uint64_t>(w.w) << 32) / Z::p) };
#pragma unroll
	for (int c = 0; c < CHAINS; ++c) { a[c] = (t * 2654435761u + c * 40503u) % Z::p; b[c] = (a[c] ^ 0x9e3779b9u) % Z::p; }
	for (int i = 0; i < iters; ++i)
	{
#pragma unroll
		for (int c = 0; c < CHAINS; ++c)
		{
			const uint32_t tt = Z::mulr(b[c], w);
			b[c] = Z::sub(a[c], tt);
			a[c] = Z::add(a[c], tt);
		}
	}
	uint32_t acc = 0;
#pragma unroll
	for (int c = 0; c < CHAINS; ++c) acc ^= a[c] ^ b[c];
	if (acc == 0x12345678u) out[t] = acc;
}

template <class K>
double time_kernel(K kernel, uint32_t *buf, int blocks, int iters)
{
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	kernel<<<blocks, 256>>>(buf, iters / 8, 1u);   // warm-up
	cudaEventRecord(e0);
	kernel<<<blocks, 256>>>(buf, iters, 2u);
	cudaEventRecord(e1);
	cudaEventSynchronize(e1);
	float ms = 0;
	cudaEventElapsedTime(&ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	return static_cast<double>(blocks) * 256.0 * CHAINS * iters / (ms * 1e-3);
}

}  // namespace

// Measures Montgomery products/s and radix-2 butterflies/s on `device` for
// the 32-bit (set 0) and 31-bit (set 1) primes: out[0..3] = mulmod32,
// mulmod31, butterfly32 (Montgomery root product), butterfly31 (Shoup root
// product) per second.  Returns 0 or -2.
extern "C" __attribute__((visibility("default"))) int gfc_probe_int_throughput(int device, double *out)
{
	if (cudaSetDevice(device) != cudaSuccess) return -2;
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	const int blocks = sms * 8;
	uint32_t *buf = nullptr;
	if (cudaMalloc(&buf, size_t(blocks) * 256 * sizeof(uint32_t)) != cudaSuccess) return -2;
	const int iters = 1 << 14;
	out[0] = time_kernel(k_probe_mulmod<0>, buf, blocks, iters);
	out[1] = time_kernel(k_probe_mulmod<1>, buf, blocks, iters);
	out[2] = time_kernel(k_probe_bfly<0>, buf, blocks, iters);
	out[3] = time_kernel(k_probe_bfly<1>, buf, blocks, iters);
	cudaFree(buf);
	return (cudaGetLastError() == cudaSuccess) ? 0 : -2;
}
