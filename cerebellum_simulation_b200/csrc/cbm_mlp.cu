// The sweep surrogate: a small MLP (nIn -> h1 -> h2 -> nOut, ReLU) trained and
// run on the GPU with this file's own kernels.  Every matrix product is one
// kernel, gemmKernel, on the 5th-generation tensor cores: BF16 operands staged
// in shared memory in the canonical K-major layout, tcgen05.mma issued by one
// thread, the FP32 accumulator in tensor memory read back with tcgen05.ld for
// the epilogue (bias, ReLU, FP32 and/or BF16 store).  Weights are kept in
// FP32 (Adam) and rounded to BF16 for the products.
//
// No counterpart in the reference (its parameter sweeps simulate every
// candidate).
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/cbm_surrogate.h"
#include "cbm_tma.cuh"

extern thread_local std::string g_cbmLastError;

namespace cbm {
namespace mlp {

constexpr uint64_t kMmaWaitLimitNs = 2000000000ull;
constexpr int kKChunk = 64;  // K elements staged per round

__device__ __forceinline__ uint32_t smemU32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major, unswizzled operand: core
// matrices of 8 rows x 16 bytes, 8-row groups sbo bytes apart, the two
// 8-element K halves of an MMA lbo bytes apart.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = 0;
	d |= (uint64_t)((addr >> 4) & 0x3FFFu);
	d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
	d |= 1ull << 46;  // descriptor version of this architecture
	// base offset 0, absolute LBO mode 0, layout type 0 (no swizzle)
	return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t instrDesc(uint32_t n)
{
	return (1u << 4)            // D format F32
		| (1u << 7)             // A format BF16
		| (1u << 10)            // B format BF16
		| ((n >> 3) << 17)      // N / 8
		| ((128u >> 4) << 24);  // M / 16
}

// out[m][n] = act(sum_k A[m][k] * B[n][k] + bias[n]) for m < M, n < N.
// A is M x K, B is N x K, both BF16 row-major (K contiguous, lda = ldb = K);
// K is a multiple of 64; N <= NT.  One CTA of 128 threads per 128-row tile.
// outF (FP32, leading dimension ldo) and outH (BF16, ldo) may each be null.
template <int NT>
__global__ void __launch_bounds__(128) gemmKernel(const __nv_bfloat16 *__restrict__ A, const __nv_bfloat16 *__restrict__ B,
		int M, int N, int K, const float *__restrict__ bias, int relu, float *outF, __nv_bfloat16 *outH, int ldo,
		uint32_t *err)
{
	extern __shared__ uint8_t gemmSmemRaw[];
	uint8_t *sA = gemmSmemRaw + ((1024u - (smemU32(gemmSmemRaw) & 1023u)) & 1023u);
	uint8_t *sB = sA + 128 * kKChunk * 2;
	__shared__ __align__(8) uint64_t bar;
	__shared__ uint32_t tmemBase;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int m0 = blockIdx.x * 128;

	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemU32(&tmemBase)),
				"r"((uint32_t)NT) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	if (tid == 0) {
		tma::mbarInit(&bar, 1);
		tma::fenceBarrierInit();
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	const uint32_t tmem = tmemBase;

	// canonical layout of a staged chunk: row r, 16-byte K piece c at
	// (r / 8) * SBO + c * 128 + (r % 8) * 16, SBO = (kKChunk / 8) * 128
	constexpr uint32_t kLBO = 128, kSBO = (kKChunk / 8) * 128;
	constexpr uint32_t idesc = instrDesc(NT);
	bool ok = true;
	for (int k0 = 0; k0 < K; k0 += kKChunk) {
		// stage A rows [m0, m0+128) and B rows [0, NT) of columns [k0, k0+64)
		for (int q = tid; q < 128 * (kKChunk / 8); q += blockDim.x) {
			const int r = q / (kKChunk / 8), c = q % (kKChunk / 8);
			uint4 v = make_uint4(0, 0, 0, 0);
			if (m0 + r < M) v = *reinterpret_cast<const uint4 *>(A + (size_t)(m0 + r) * K + k0 + c * 8);
			*reinterpret_cast<uint4 *>(sA + (r / 8) * kSBO + c * kLBO + (r % 8) * 16) = v;
		}
		for (int q = tid; q < NT * (kKChunk / 8); q += blockDim.x) {
			const int r = q / (kKChunk / 8), c = q % (kKChunk / 8);
			uint4 v = make_uint4(0, 0, 0, 0);
			if (r < N) v = *reinterpret_cast<const uint4 *>(B + (size_t)r * K + k0 + c * 8);
			*reinterpret_cast<uint4 *>(sB + (r / 8) * kSBO + c * kLBO + (r % 8) * 16) = v;
		}
		// make the generic-proxy stores visible to the tensor cores
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		__syncthreads();
		if (tid == 0) {
			asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
			for (int ks = 0; ks < kKChunk; ks += 16) {
				const uint64_t da = smemDesc(smemU32(sA) + (ks / 8) * kLBO, kLBO, kSBO);
				const uint64_t db = smemDesc(smemU32(sB) + (ks / 8) * kLBO, kLBO, kSBO);
				const uint32_t accumulate = (k0 > 0 || ks > 0) ? 1u : 0u;
				asm volatile(
					"{\n\t.reg .pred p;\n\t"
					"setp.ne.b32 p, %4, 0;\n\t"
					"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
					::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
					: "memory");
			}
			asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
					::"r"(smemU32(&bar)) : "memory");
		}
		// the chunk's MMAs have read shared memory once the barrier flips
		const bool done = tma::waitBounded(&bar, (uint32_t)((k0 / kKChunk) & 1), kMmaWaitLimitNs);
		if (!__syncthreads_and(done)) {
			ok = false;
			break;
		}
		asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	}
	if (!ok) {
		if (tid == 0) atomicOr(err, 1u);
	} else {
		// epilogue: warp w owns TMEM lanes (rows) 32w..32w+31
		const int m = m0 + warp * 32 + lane;
		for (int c0 = 0; c0 < NT; c0 += 16) {
			uint32_t r[16];
			const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
			asm volatile(
				"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
				: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
				  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
				: "r"(taddr));
			asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
			if (m < M) {
#pragma unroll
				for (int j = 0; j < 16; j++) {
					const int n = c0 + j;
					if (n >= N) break;
					float v = __uint_as_float(r[j]);
					if (bias) v += bias[n];
					if (relu) v = v > 0.0f ? v : 0.0f;
					if (outF) outF[(size_t)m * ldo + n] = v;
					if (outH) outH[(size_t)m * ldo + n] = __float2bfloat16_rn(v);
				}
			}
		}
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	if (warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)NT) : "memory");
}

// ------------------------------------------------------------ elementwise
__global__ void toBf16Kernel(const float *in, __nv_bfloat16 *out, size_t n)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

// out[c][r] = in[r][c] for r < R, 0 for R <= r < Rp; in is R x C (ld C),
// out C x Rp (ld Rp).
__global__ void transposeKernel(const __nv_bfloat16 *in, int R, int C, int Rp, __nv_bfloat16 *out)
{
	__shared__ __nv_bfloat16 tile[32][33];
	const int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
	for (int j = threadIdx.y; j < 32; j += blockDim.y) {
		const int r = r0 + j;
		tile[j][threadIdx.x] = (r < R && c < C) ? in[(size_t)r * C + c] : __float2bfloat16_rn(0.0f);
	}
	__syncthreads();
	const int oc = r0 + threadIdx.x, or0 = blockIdx.x * 32;
	for (int j = threadIdx.y; j < 32; j += blockDim.y) {
		const int orow = or0 + j;
		if (orow < C && oc < Rp) out[(size_t)orow * Rp + oc] = tile[threadIdx.x][j];
	}
}

// Mean squared error over rows < rows and columns < cols of Y - T (both
// rows x ld); dY = 2 (Y - T) / (rows * cols) as BF16 (zero outside), the
// loss sum accumulated into *loss.
__global__ void mseGradKernel(const float *Y, const float *T, int rows, int cols, int ld, float *dYf,
		__nv_bfloat16 *dYh, float *loss)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	const size_t total = (size_t)rows * ld;
	float e2 = 0.0f;
	if (i < total) {
		const int c = (int)(i % ld);
		float g = 0.0f;
		if (c < cols) {
			const float d = Y[i] - T[i];
			e2 = d * d;
			g = 2.0f * d / ((float)rows * (float)cols);
		}
		dYf[i] = g;
		dYh[i] = __float2bfloat16_rn(g);
	}
	for (int o = 16; o > 0; o >>= 1) e2 += __shfl_down_sync(0xffffffffu, e2, o);
	if ((threadIdx.x & 31) == 0 && e2 != 0.0f) atomicAdd(loss, e2);
}

// g = g * (h > 0): the ReLU derivative applied to an upstream gradient; BF16 copy.
__global__ void reluBackKernel(float *g, const __nv_bfloat16 *h, size_t n, __nv_bfloat16 *gh)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) {
		const float v = __bfloat162float(h[i]) > 0.0f ? g[i] : 0.0f;
		g[i] = v;
		gh[i] = __float2bfloat16_rn(v);
	}
}

// db[c] = sum over rows of g[r][c] (rows x cols, ld cols).
__global__ void colSumKernel(const float *g, int rows, int cols, float *db)
{
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= cols) return;
	float s = 0.0f;
	for (int r = 0; r < rows; r++) s += g[(size_t)r * cols + c];
	db[c] = s;
}

// Adam (Kingma and Ba, 2015) on n parameters, bias-corrected step t.
__global__ void adamKernel(float *p, const float *g, float *m, float *v, size_t n, float lr, float b1, float b2,
		float eps, float c1, float c2)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float gi = g[i];
	const float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
	m[i] = mi;
	v[i] = vi;
	p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace mlp
}  // namespace cbm

using namespace cbm::mlp;

// ---------------------------------------------------------------- host side
struct cbm_mlp {
	int device = 0;
	uint32_t nIn = 0, h1 = 0, h2 = 0, nOut = 0;   // logical sizes
	uint32_t I = 0, H1 = 0, H2 = 0, O = 0;        // padded to multiples of 64
	uint32_t maxBatch = 0, Bp = 0;                // batch capacity, padded to 128
	cudaStream_t s = nullptr;
	// FP32 master parameters (flat: W1 [H1][I], b1, W2 [H2][H1], b2, W3 [O][H2], b3), grads, Adam moments
	float *P = nullptr, *G = nullptr, *Mo = nullptr, *Ve = nullptr;
	size_t nP = 0;
	size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
	// BF16 copies and activations
	__nv_bfloat16 *Wh = nullptr, *W2t = nullptr, *W3t = nullptr;
	__nv_bfloat16 *X = nullptr, *Xt = nullptr, *H1h = nullptr, *H1t = nullptr, *H2h = nullptr, *H2t = nullptr;
	__nv_bfloat16 *dYh = nullptr, *dYt = nullptr, *dH2h = nullptr, *dH2t = nullptr, *dH1h = nullptr, *dH1t = nullptr;
	float *Xf = nullptr, *Yf = nullptr, *Tf = nullptr, *dYf = nullptr, *dH2f = nullptr, *dH1f = nullptr;
	float *loss = nullptr;
	uint32_t *err = nullptr;
	uint64_t adamStep = 0;
	std::vector<void *> allocs;
};

static int mfail(int code, const std::string &m)
{
	g_cbmLastError = m;
	return code;
}

#define MCK(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return mfail(CBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); } while (0)

static uint32_t pad(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

template <typename T> static T *dalloc(cbm_mlp *n, size_t count)
{
	void *p = nullptr;
	if (cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess) return nullptr;
	cudaMemset(p, 0, std::max<size_t>(count * sizeof(T), 16));
	n->allocs.push_back(p);
	return (T *)p;
}

// C = act(A B^T + bias), A M x K, B N x K (BF16), N <= 256, K % 64 == 0.
template <int NT> static size_t gemmSmem() { return 1024 + (size_t)(128 + NT) * kKChunk * 2; }

static int gemm(cbm_mlp *n, const __nv_bfloat16 *A, const __nv_bfloat16 *B, int M, int N, int K, const float *bias,
		bool relu, float *outF, __nv_bfloat16 *outH, int ldo)
{
	const dim3 grid((M + 127) / 128);
	if (K % kKChunk) return mfail(CBM_ERR_ARG, "product depth must be a multiple of 64");
	if (N <= 64) gemmKernel<64><<<grid, 128, gemmSmem<64>(), n->s>>>(A, B, M, N, K, bias, relu, outF, outH, ldo, n->err);
	else if (N <= 256) gemmKernel<256><<<grid, 128, gemmSmem<256>(), n->s>>>(A, B, M, N, K, bias, relu, outF, outH, ldo, n->err);
	else return mfail(CBM_ERR_ARG, "layer wider than 256");
	MCK(cudaGetLastError(), "launching a tensor-core product");
	return CBM_OK;
}

static int transpose(cbm_mlp *n, const __nv_bfloat16 *in, int R, int C, int Rp, __nv_bfloat16 *out)
{
	transposeKernel<<<dim3((C + 31) / 32, (Rp + 31) / 32), dim3(32, 8), 0, n->s>>>(in, R, C, Rp, out);
	MCK(cudaGetLastError(), "transpose");
	return CBM_OK;
}

static int toBf16(cbm_mlp *n, const float *in, __nv_bfloat16 *out, size_t count)
{
	toBf16Kernel<<<(unsigned)((count + 255) / 256), 256, 0, n->s>>>(in, out, count);
	MCK(cudaGetLastError(), "cast");
	return CBM_OK;
}

static int checkErr(cbm_mlp *n)
{
	uint32_t e = 0;
	MCK(cudaMemcpyAsync(&e, n->err, 4, cudaMemcpyDeviceToHost, n->s), "reading the error word");
	MCK(cudaStreamSynchronize(n->s), "surrogate");
	if (e) return mfail(CBM_ERR_CUDA, "tensor-core product: a completion wait timed out on the device");
	return CBM_OK;
}

#define MTRY(x) do { int r_ = (x); if (r_ != CBM_OK) return r_; } while (0)

// Upload rows [0, b) of x (b x nIn, FP32) into the padded input, BF16 copy.
static int loadInput(cbm_mlp *n, const float *x, uint32_t b)
{
	std::vector<float> buf((size_t)n->Bp * n->I, 0.0f);
	for (uint32_t r = 0; r < b; r++) memcpy(&buf[(size_t)r * n->I], x + (size_t)r * n->nIn, 4ull * n->nIn);
	MCK(cudaMemcpyAsync(n->Xf, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice, n->s), "input");
	MTRY(toBf16(n, n->Xf, n->X, buf.size()));
	return CBM_OK;
}

static int forward(cbm_mlp *n, uint32_t b)
{
	const int Bp = (int)pad(b, 128);
	MTRY(toBf16(n, n->P, n->Wh, n->nP));
	const __nv_bfloat16 *W1 = n->Wh + n->oW1, *W2 = n->Wh + n->oW2, *W3 = n->Wh + n->oW3;
	MTRY(gemm(n, n->X, W1, Bp, n->H1, n->I, n->P + n->ob1, true, nullptr, n->H1h, n->H1));
	MTRY(gemm(n, n->H1h, W2, Bp, n->H2, n->H1, n->P + n->ob2, true, nullptr, n->H2h, n->H2));
	MTRY(gemm(n, n->H2h, W3, Bp, n->O, n->H2, n->P + n->ob3, false, n->Yf, nullptr, n->O));
	return CBM_OK;
}

// Gradients of the mean squared error over the b valid rows into G.
static int backward(cbm_mlp *n, uint32_t b)
{
	const int B = (int)b;
	const size_t yN = (size_t)b * n->O;
	MCK(cudaMemsetAsync(n->loss, 0, 4, n->s), "loss");
	mseGradKernel<<<(unsigned)((yN + 255) / 256), 256, 0, n->s>>>(n->Yf, n->Tf, B, n->nOut, n->O, n->dYf, n->dYh, n->loss);
	MCK(cudaGetLastError(), "loss");
	const __nv_bfloat16 *W2 = n->Wh + n->oW2, *W3 = n->Wh + n->oW3;
	// transposed operands of the weight-gradient products, whose depth is
	// the batch (zero-padded to a multiple of 64)
	const int Kb = (int)pad(b, 64);
	MTRY(transpose(n, n->dYh, B, n->O, Kb, n->dYt));      // O x Kb
	MTRY(transpose(n, n->H2h, B, n->H2, Kb, n->H2t));     // H2 x Kb
	MTRY(transpose(n, n->H1h, B, n->H1, Kb, n->H1t));     // H1 x Kb
	MTRY(transpose(n, n->X, B, n->I, Kb, n->Xt));         // I x Kb
	MTRY(transpose(n, W3, n->O, n->H2, n->O, n->W3t));    // H2 x O
	MTRY(transpose(n, W2, n->H2, n->H1, n->H2, n->W2t));  // H1 x H2
	// layer 3
	MTRY(gemm(n, n->dYt, n->H2t, n->O, n->H2, Kb, nullptr, false, n->G + n->oW3, nullptr, n->H2));
	colSumKernel<<<(n->O + 127) / 128, 128, 0, n->s>>>(n->dYf, B, n->O, n->G + n->ob3);
	MTRY(gemm(n, n->dYh, n->W3t, B, n->H2, n->O, nullptr, false, n->dH2f, nullptr, n->H2));
	reluBackKernel<<<(unsigned)(((size_t)B * n->H2 + 255) / 256), 256, 0, n->s>>>(n->dH2f, n->H2h, (size_t)B * n->H2, n->dH2h);
	// layer 2
	MTRY(transpose(n, n->dH2h, B, n->H2, Kb, n->dH2t));   // H2 x Kb
	MTRY(gemm(n, n->dH2t, n->H1t, n->H2, n->H1, Kb, nullptr, false, n->G + n->oW2, nullptr, n->H1));
	colSumKernel<<<(n->H2 + 127) / 128, 128, 0, n->s>>>(n->dH2f, B, n->H2, n->G + n->ob2);
	MTRY(gemm(n, n->dH2h, n->W2t, B, n->H1, n->H2, nullptr, false, n->dH1f, nullptr, n->H1));
	reluBackKernel<<<(unsigned)(((size_t)B * n->H1 + 255) / 256), 256, 0, n->s>>>(n->dH1f, n->H1h, (size_t)B * n->H1, n->dH1h);
	// layer 1
	MTRY(transpose(n, n->dH1h, B, n->H1, Kb, n->dH1t));   // H1 x Kb
	MTRY(gemm(n, n->dH1t, n->Xt, n->H1, n->I, Kb, nullptr, false, n->G + n->oW1, nullptr, n->I));
	colSumKernel<<<(n->H1 + 127) / 128, 128, 0, n->s>>>(n->dH1f, B, n->H1, n->G + n->ob1);
	MCK(cudaGetLastError(), "backward");
	return CBM_OK;
}

extern "C" {

int cbm_mlp_create(unsigned nIn, unsigned h1, unsigned h2, unsigned nOut, unsigned maxBatch, uint64_t seed, int device,
		cbm_mlp **out)
{
	if (!out) return mfail(CBM_ERR_ARG, "null argument: out");
	if (!nIn || !h1 || !h2 || !nOut || !maxBatch) return mfail(CBM_ERR_ARG, "sizes must be positive");
	if (pad(nIn, 64) > 256 || pad(h1, 64) > 256 || pad(h2, 64) > 256 || pad(nOut, 64) > 256)
		return mfail(CBM_ERR_ARG, "layers are at most 256 wide");
	cbm_mlp *n = new cbm_mlp();
	n->device = device;
	n->nIn = nIn; n->h1 = h1; n->h2 = h2; n->nOut = nOut;
	n->I = pad(nIn, 64); n->H1 = pad(h1, 64); n->H2 = pad(h2, 64); n->O = pad(nOut, 64);
	n->maxBatch = maxBatch;
	n->Bp = pad(maxBatch, 128);
	if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess) {
		delete n;
		return mfail(CBM_ERR_CUDA, "stream");
	}
	if (cudaFuncSetAttribute(gemmKernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemmSmem<64>()) != cudaSuccess ||
			cudaFuncSetAttribute(gemmKernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemmSmem<256>()) != cudaSuccess) {
		cudaStreamDestroy(n->s);
		delete n;
		return mfail(CBM_ERR_CUDA, "tensor-core product shared memory");
	}
	n->oW1 = 0; n->ob1 = n->oW1 + (size_t)n->H1 * n->I;
	n->oW2 = n->ob1 + n->H1; n->ob2 = n->oW2 + (size_t)n->H2 * n->H1;
	n->oW3 = n->ob2 + n->H2; n->ob3 = n->oW3 + (size_t)n->O * n->H2;
	n->nP = n->ob3 + n->O;
	const size_t B = n->Bp;
	n->P = dalloc<float>(n, n->nP); n->G = dalloc<float>(n, n->nP);
	n->Mo = dalloc<float>(n, n->nP); n->Ve = dalloc<float>(n, n->nP);
	n->Wh = dalloc<__nv_bfloat16>(n, n->nP);
	n->W2t = dalloc<__nv_bfloat16>(n, (size_t)n->H1 * n->H2);
	n->W3t = dalloc<__nv_bfloat16>(n, (size_t)n->H2 * n->O);
	n->X = dalloc<__nv_bfloat16>(n, B * n->I); n->Xt = dalloc<__nv_bfloat16>(n, B * n->I);
	n->Xf = dalloc<float>(n, B * n->I);
	n->H1h = dalloc<__nv_bfloat16>(n, B * n->H1); n->H1t = dalloc<__nv_bfloat16>(n, B * n->H1);
	n->H2h = dalloc<__nv_bfloat16>(n, B * n->H2); n->H2t = dalloc<__nv_bfloat16>(n, B * n->H2);
	n->Yf = dalloc<float>(n, B * n->O); n->Tf = dalloc<float>(n, B * n->O);
	n->dYf = dalloc<float>(n, B * n->O);
	n->dYh = dalloc<__nv_bfloat16>(n, B * n->O); n->dYt = dalloc<__nv_bfloat16>(n, B * n->O);
	n->dH2f = dalloc<float>(n, B * n->H2);
	n->dH2h = dalloc<__nv_bfloat16>(n, B * n->H2); n->dH2t = dalloc<__nv_bfloat16>(n, B * n->H2);
	n->dH1f = dalloc<float>(n, B * n->H1);
	n->dH1h = dalloc<__nv_bfloat16>(n, B * n->H1); n->dH1t = dalloc<__nv_bfloat16>(n, B * n->H1);
	n->loss = dalloc<float>(n, 1);
	n->err = dalloc<uint32_t>(n, 1);
	for (void *p : n->allocs) if (!p) { cbm_mlp_destroy(n); return mfail(CBM_ERR_CUDA, "device allocation failed"); }
	// He-uniform initial weights (logical part only), zero biases
	std::vector<float> p(n->nP, 0.0f);
	std::mt19937_64 rng(seed);
	auto init = [&](size_t off, uint32_t rows, uint32_t cols, uint32_t ld, uint32_t fanIn) {
		std::uniform_real_distribution<float> u(-1.0f, 1.0f);
		const float a = std::sqrt(6.0f / (float)fanIn);
		for (uint32_t r = 0; r < rows; r++)
			for (uint32_t c = 0; c < cols; c++) p[off + (size_t)r * ld + c] = a * u(rng);
	};
	init(n->oW1, h1, nIn, n->I, nIn);
	init(n->oW2, h2, h1, n->H1, h1);
	init(n->oW3, nOut, h2, n->H2, h2);
	if (cudaMemcpy(n->P, p.data(), p.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
		cbm_mlp_destroy(n);
		return mfail(CBM_ERR_CUDA, "uploading parameters");
	}
	*out = n;
	return CBM_OK;
}

void cbm_mlp_destroy(cbm_mlp *n)
{
	if (!n) return;
	for (void *p : n->allocs) cudaFree(p);
	if (n->s) cudaStreamDestroy(n->s);
	delete n;
}

uint64_t cbm_mlp_num_params(cbm_mlp *n) { return n ? n->nP : 0; }

int cbm_mlp_layout(cbm_mlp *n, unsigned *I, unsigned *H1, unsigned *H2, unsigned *O)
{
	if (!n || !I || !H1 || !H2 || !O) return mfail(CBM_ERR_ARG, "null argument");
	*I = n->I; *H1 = n->H1; *H2 = n->H2; *O = n->O;
	return CBM_OK;
}

int cbm_mlp_get_params(cbm_mlp *n, float *dst, uint64_t count)
{
	if (!n || !dst) return mfail(CBM_ERR_ARG, "null argument");
	if (count != n->nP) return mfail(CBM_ERR_ARG, "parameter count mismatch");
	cudaSetDevice(n->device);
	MCK(cudaMemcpy(dst, n->P, count * 4, cudaMemcpyDeviceToHost), "reading parameters");
	return CBM_OK;
}

int cbm_mlp_set_params(cbm_mlp *n, const float *src, uint64_t count)
{
	if (!n || !src) return mfail(CBM_ERR_ARG, "null argument");
	if (count != n->nP) return mfail(CBM_ERR_ARG, "parameter count mismatch");
	cudaSetDevice(n->device);
	MCK(cudaMemcpy(n->P, src, count * 4, cudaMemcpyHostToDevice), "writing parameters");
	MCK(cudaMemset(n->Mo, 0, count * 4), "resetting Adam");
	MCK(cudaMemset(n->Ve, 0, count * 4), "resetting Adam");
	n->adamStep = 0;
	return CBM_OK;
}

int cbm_mlp_forward(cbm_mlp *n, const float *x, unsigned batch, float *y)
{
	if (!n || !x || !y) return mfail(CBM_ERR_ARG, "null argument");
	cudaSetDevice(n->device);
	for (unsigned b0 = 0; b0 < batch; b0 += n->maxBatch) {
		const unsigned b = std::min(n->maxBatch, batch - b0);
		MTRY(loadInput(n, x + (size_t)b0 * n->nIn, b));
		MTRY(forward(n, b));
		std::vector<float> out((size_t)b * n->O);
		MCK(cudaMemcpyAsync(out.data(), n->Yf, out.size() * 4, cudaMemcpyDeviceToHost, n->s), "output");
		MTRY(checkErr(n));
		for (unsigned r = 0; r < b; r++) memcpy(y + (size_t)(b0 + r) * n->nOut, &out[(size_t)r * n->O], 4ull * n->nOut);
	}
	return CBM_OK;
}

static int loadTarget(cbm_mlp *n, const float *t, uint32_t b)
{
	std::vector<float> buf((size_t)b * n->O, 0.0f);
	for (uint32_t r = 0; r < b; r++) memcpy(&buf[(size_t)r * n->O], t + (size_t)r * n->nOut, 4ull * n->nOut);
	MCK(cudaMemcpyAsync(n->Tf, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice, n->s), "target");
	return CBM_OK;
}

int cbm_mlp_gradients(cbm_mlp *n, const float *x, const float *target, unsigned batch, float *grads, float *loss)
{
	if (!n || !x || !target || !grads) return mfail(CBM_ERR_ARG, "null argument");
	if (batch == 0 || batch > n->maxBatch) return mfail(CBM_ERR_ARG, "batch must be 1..maxBatch");
	cudaSetDevice(n->device);
	MTRY(loadInput(n, x, batch));
	MTRY(loadTarget(n, target, batch));
	MTRY(forward(n, batch));
	MTRY(backward(n, batch));
	MCK(cudaMemcpyAsync(grads, n->G, n->nP * 4, cudaMemcpyDeviceToHost, n->s), "gradients");
	float l = 0;
	MCK(cudaMemcpyAsync(&l, n->loss, 4, cudaMemcpyDeviceToHost, n->s), "loss");
	MTRY(checkErr(n));
	if (loss) *loss = l / ((float)batch * (float)n->nOut);
	return CBM_OK;
}

int cbm_mlp_train(cbm_mlp *n, const float *x, const float *target, unsigned count, unsigned batch, unsigned epochs,
		float lr, uint64_t seed, float *lastLoss)
{
	if (!n || !x || !target) return mfail(CBM_ERR_ARG, "null argument");
	if (batch == 0 || batch > n->maxBatch || count < batch) return mfail(CBM_ERR_ARG, "batch must be 1..maxBatch and <= count");
	cudaSetDevice(n->device);
	std::vector<uint32_t> order(count);
	for (uint32_t i = 0; i < count; i++) order[i] = i;
	std::mt19937_64 rng(seed);
	std::vector<float> xb((size_t)batch * n->nIn), tb((size_t)batch * n->nOut);
	float l = 0;
	double epochLoss = 0;
	for (unsigned e = 0; e < epochs; e++) {
		std::shuffle(order.begin(), order.end(), rng);
		epochLoss = 0;
		unsigned nb = 0;
		for (unsigned b0 = 0; b0 + batch <= count; b0 += batch, nb++) {
			for (unsigned r = 0; r < batch; r++) {
				memcpy(&xb[(size_t)r * n->nIn], x + (size_t)order[b0 + r] * n->nIn, 4ull * n->nIn);
				memcpy(&tb[(size_t)r * n->nOut], target + (size_t)order[b0 + r] * n->nOut, 4ull * n->nOut);
			}
			MTRY(loadInput(n, xb.data(), batch));
			MTRY(loadTarget(n, tb.data(), batch));
			MTRY(forward(n, batch));
			MTRY(backward(n, batch));
			n->adamStep++;
			const float b1 = 0.9f, b2 = 0.999f;
			const float c1 = 1.0f - (float)std::pow(b1, (double)n->adamStep), c2 = 1.0f - (float)std::pow(b2, (double)n->adamStep);
			adamKernel<<<(unsigned)((n->nP + 255) / 256), 256, 0, n->s>>>(n->P, n->G, n->Mo, n->Ve, n->nP, lr, b1, b2,
					1e-8f, c1, c2);
			MCK(cudaGetLastError(), "Adam");
			MCK(cudaMemcpyAsync(&l, n->loss, 4, cudaMemcpyDeviceToHost, n->s), "loss");
			MTRY(checkErr(n));
			epochLoss += l / ((double)batch * n->nOut);
		}
		epochLoss /= std::max(1u, nb);
	}
	if (lastLoss) *lastLoss = (float)epochLoss;
	return CBM_OK;
}

}  // extern "C"
