/* Test infrastructure (oracle build only): host-memory implementation of the
 * CUDA runtime subset declared in refshim/cuda_runtime.h. */
#include "cuda_runtime.h"
#include <cstdlib>
#include <cstring>

static int g_curDev = 0;

cudaError_t cudaMalloc(void **p, size_t n) { *p = calloc(n ? n : 1, 1); return *p ? cudaSuccess : cudaErrorMemoryAllocation; }
cudaError_t cudaMallocPitch(void **p, size_t *pitch, size_t width, size_t height)
{
	*pitch = width;
	return cudaMalloc(p, width * height);
}
cudaError_t cudaMallocHost(void **p, size_t n) { return cudaMalloc(p, n); }
cudaError_t cudaHostAlloc(void **p, size_t n, unsigned int) { return cudaMalloc(p, n); }
cudaError_t cudaFree(void *p) { free(p); return cudaSuccess; }
cudaError_t cudaFreeHost(void *p) { free(p); return cudaSuccess; }
cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind) { memmove(dst, src, n); return cudaSuccess; }
cudaError_t cudaMemcpyAsync(void *dst, const void *src, size_t n, cudaMemcpyKind k, cudaStream_t) { return cudaMemcpy(dst, src, n, k); }
cudaError_t cudaMemset(void *p, int v, size_t n) { memset(p, v, n); return cudaSuccess; }
cudaError_t cudaSetDevice(int d) { g_curDev = d; return cudaSuccess; }
cudaError_t cudaGetDevice(int *d) { *d = g_curDev; return cudaSuccess; }
cudaError_t cudaGetDeviceCount(int *n)
{
	const char *e = getenv("CBM_FAKE_NUM_GPUS");
	*n = e ? atoi(e) : 1;
	if (*n < 1) *n = 1;
	return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
cudaError_t cudaThreadSynchronize() { return cudaSuccess; }
cudaError_t cudaDeviceReset() { return cudaSuccess; }
cudaError_t cudaStreamCreate(cudaStream_t *s) { *s = new CUstream_st_shim(); (*s)->id = 0; return cudaSuccess; }
cudaError_t cudaStreamDestroy(cudaStream_t s) { delete s; return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGetLastError() { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "error"; }
