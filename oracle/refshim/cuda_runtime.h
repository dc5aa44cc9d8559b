/* Test infrastructure (oracle build only).
 *
 * A host-memory stand-in for the subset of the CUDA runtime API that the
 * reference's host orchestration calls (CBM_CORE_LIB_MGPU_DEV/src/interface/
 * cbmsimcore.cpp, src/innetmodules/innet.cpp, src/mzonemodules/mzone.cpp).
 * "Device" memory is ordinary heap memory, every copy completes before the
 * call returns and streams are empty handles.  Copies therefore finish before
 * the host reads them, which is the reference's NO_ASYNC ordering
 * (cbmsimcore.cpp:10).  cudaGetDeviceCount reports CBM_FAKE_NUM_GPUS
 * (default 1) so the reference's GR-sharded multi-GPU host path can run on a
 * CPU. */
#ifndef CBM_REFSHIM_CUDA_RUNTIME_H
#define CBM_REFSHIM_CUDA_RUNTIME_H
#include <cstddef>

enum cudaError_t { cudaSuccess = 0, cudaErrorInvalidValue = 1, cudaErrorMemoryAllocation = 2 };
typedef cudaError_t cudaError;
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1,
	cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3, cudaMemcpyDefault = 4 };
struct CUstream_st_shim { int id; };
typedef CUstream_st_shim *cudaStream_t;

#define cudaHostAllocDefault 0
#define cudaHostAllocPortable 1

cudaError_t cudaMalloc(void **p, size_t n);
template<class T> inline cudaError_t cudaMalloc(T **p, size_t n) { return cudaMalloc((void **)p, n); }
cudaError_t cudaMallocPitch(void **p, size_t *pitch, size_t width, size_t height);
template<class T> inline cudaError_t cudaMallocPitch(T **p, size_t *pitch, size_t w, size_t h)
{ return cudaMallocPitch((void **)p, pitch, w, h); }
cudaError_t cudaMallocHost(void **p, size_t n);
template<class T> inline cudaError_t cudaMallocHost(T **p, size_t n) { return cudaMallocHost((void **)p, n); }
cudaError_t cudaHostAlloc(void **p, size_t n, unsigned int flags);
cudaError_t cudaFree(void *p);
cudaError_t cudaFreeHost(void *p);
cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind k);
cudaError_t cudaMemcpyAsync(void *dst, const void *src, size_t n, cudaMemcpyKind k, cudaStream_t s = 0);
cudaError_t cudaMemset(void *p, int v, size_t n);
cudaError_t cudaSetDevice(int d);
cudaError_t cudaGetDevice(int *d);
cudaError_t cudaGetDeviceCount(int *n);
cudaError_t cudaDeviceSynchronize();
cudaError_t cudaThreadSynchronize();
cudaError_t cudaDeviceReset();
cudaError_t cudaStreamCreate(cudaStream_t *s);
cudaError_t cudaStreamDestroy(cudaStream_t s);
cudaError_t cudaStreamSynchronize(cudaStream_t s);
cudaError_t cudaGetLastError();
const char *cudaGetErrorString(cudaError_t e);
#endif
