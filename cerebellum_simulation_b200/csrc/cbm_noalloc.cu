// PF->PC input sums with no device allocation.
//
// Some host programs cannot let a library allocate device memory when they
// call it: frameworks that own every device allocation through their own
// pool (a foreign cudaMalloc escapes their budget and fragments their
// arena), and real-time control loops that cannot absorb the latency of an
// allocation.
// For them this file computes the per-PC parallel-fibre input sums (the
// reference's updatePFPCOutGPU followed by sumInputsNew, in the same float
// order) from buffers the caller already holds, with its only scratch in a
// file-scope device array that exists for the life of the process.
//
// Limits and behaviour:
//   - numPC x bs <= kMaxPartials, where bs is the reduction width the
//     reference picks for a row of numGR/numPC fibres (512 for rows of 2048
//     or more); larger networks are rejected with CBM_ERR_ARG.
//   - The scratch array is shared by every call on a device and keeps the
//     last call's contents; each call overwrites every partial it reads, so
//     nothing needs clearing.  Calls whose kernels overlap on the GPU race on
//     the array; callers on several streams must order them.
//   - The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The address is kept for later calls; it
//     does not survive a reset of the device's context (cudaDeviceReset, or
//     a framework resetting the primary context), after which the module
//     may load elsewhere: each call checks that the kept address is still
//     device memory of the current device and looks it up again if not, but
//     after a reset the first call must again come before any capture.
//   - A CUDA error already pending in the calling thread (from the
//     caller's own earlier launches) is reported as such and left pending;
//     nothing is launched then.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/cbm_b200.h"

namespace {

constexpr uint32_t kMaxPartials = CBM_NOALLOC_MAX_PARTIALS;
constexpr int kMaxDevices = 64;

// Every device that loads the library holds this array until the process exits.
static __device__ __align__(256) float g_pfpcPartials[kMaxPartials];

std::mutex g_setupMutex;
float *g_partialsAddr[kMaxDevices] = {};


// callSumKernel's block size for a row (CBM_CORE_LIB_MGPU_DEV/src/cuda/kernels.cu:445-469)
uint32_t rowBlockSize(uint32_t rowLength)
{
	if (rowLength >= 2048) return 512;
	if (rowLength >= 512) return 128;
	if (rowLength >= 128) return 32;
	if (rowLength >= 32) return 8;
	return 2;
}

// Thread (pc, j): the running sum of the pairs x[i] + x[i+bs] for
// i = j, j+2bs, ... of the PC's row, x = w * (apBuf & mask != 0).
__global__ void partialsKernel(const uint32_t *apBuf, const uint32_t *mask, const float *w, uint32_t P,
		uint32_t bs, uint32_t numPC, float *partials)
{
	const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= numPC * bs) return;
	const uint32_t pc = id / bs, j = id % bs;
	const size_t row = (size_t)pc * P;
	float s = 0;
	for (uint32_t i = j; i < P; i += 2 * bs) {
		const size_t a = row + i, b = row + i + bs;
		const unsigned int pa = (apBuf[a] & mask[a]) > 0, pb = (apBuf[b] & mask[b]) > 0;
		s += w[a] * pa + w[b] * pb;
	}
	partials[id] = s;
}

// One block per PC: sumInputsNew's halving tree over the bs partials
// (strides bs/2 ... 1, kernels.cu:326-362).
__global__ void treeKernel(const float *partials, uint32_t bs, float *sums)
{
	__shared__ float s[512];
	const uint32_t pc = blockIdx.x;
	for (uint32_t t = threadIdx.x; t < bs; t += blockDim.x) s[t] = partials[(size_t)pc * bs + t];
	__syncthreads();
	for (uint32_t h = bs / 2; h >= 1; h /= 2) {
		float v = 0;
		const bool act = threadIdx.x < h;
		if (act) v = s[threadIdx.x] + s[threadIdx.x + h];
		__syncthreads();
		if (act) s[threadIdx.x] = v;
		__syncthreads();
	}
	if (threadIdx.x == 0) sums[pc] = s[0];
}

}  // namespace

// the C ABI's per-thread error message (cbm_capi.cu), read by cbm_last_error
extern thread_local std::string g_cbmLastError;

static int fail(int code, const std::string &msg)
{
	g_cbmLastError = msg;
	return code;
}

extern "C" int cbm_pfpc_sums_noalloc(const uint32_t *apBuf, const uint32_t *pfDelayMask, const float *weights,
		uint32_t numGR, uint32_t numPC, float *sums, void *stream)
{
	if (!apBuf || !pfDelayMask || !weights || !sums) return fail(CBM_ERR_ARG, "null buffer");
	if (numPC == 0 || numGR % numPC) return fail(CBM_ERR_ARG, "numGR must be a multiple of numPC");
	const uint32_t P = numGR / numPC;
	if (P < 4 || (P & (P - 1))) return fail(CBM_ERR_ARG, "fibres per PC must be a power of two >= 4");
	const uint32_t bs = rowBlockSize(P);
	if ((uint64_t)numPC * bs > kMaxPartials)
		return fail(CBM_ERR_ARG, "numPC x reduction width exceeds CBM_NOALLOC_MAX_PARTIALS (" +
				std::to_string(kMaxPartials) + ")");
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return fail(CBM_ERR_CUDA, cudaGetErrorString(e));
	if (dev < 0 || dev >= kMaxDevices) return fail(CBM_ERR_ARG, "device index out of range");
	e = cudaPeekAtLastError();
	if (e != cudaSuccess)
		return fail(CBM_ERR_CUDA, std::string("a CUDA error is already pending in this thread: ") + cudaGetErrorString(e));
	float *partials;
	{
		std::lock_guard<std::mutex> lock(g_setupMutex);
		if (g_partialsAddr[dev]) {
			// a kept address from before a context reset no longer resolves
			// to this device's memory: look it up again
			cudaPointerAttributes attr{};
			if (cudaPointerGetAttributes(&attr, g_partialsAddr[dev]) != cudaSuccess ||
					attr.type != cudaMemoryTypeDevice || attr.device != dev) {
				cudaGetLastError();  // the failed query's own error, not the caller's
				g_partialsAddr[dev] = nullptr;
			}
		}
		if (!g_partialsAddr[dev]) {
			void *p = nullptr;
			e = cudaGetSymbolAddress(&p, g_pfpcPartials);
			if (e != cudaSuccess) return fail(CBM_ERR_CUDA, std::string("scratch lookup: ") + cudaGetErrorString(e));
			g_partialsAddr[dev] = (float *)p;
		}
		partials = g_partialsAddr[dev];
	}
	cudaStream_t s = (cudaStream_t)stream;
	const uint32_t n = numPC * bs;
	partialsKernel<<<(n + 255) / 256, 256, 0, s>>>(apBuf, pfDelayMask, weights, P, bs, numPC, partials);
	e = cudaGetLastError();
	if (e != cudaSuccess) return fail(CBM_ERR_CUDA, std::string("partial sums launch: ") + cudaGetErrorString(e));
	treeKernel<<<numPC, bs < 256 ? bs : 256, 0, s>>>(partials, bs, sums);
	e = cudaGetLastError();
	if (e != cudaSuccess) return fail(CBM_ERR_CUDA, std::string("tree launch: ") + cudaGetErrorString(e));
	return CBM_OK;
}
