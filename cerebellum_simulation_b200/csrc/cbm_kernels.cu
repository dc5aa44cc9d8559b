// sm_100a kernels of the 1 ms cerebellar network step.
//
// One step t of the reference's CBMSimCore::calcActivity
// (CBM_CORE_LIB_MGPU_DEV/src/interface/cbmsimcore.cpp:139-310) is two kernels
// that run concurrently on two streams:
//
//  grPassKernel  one streaming pass over all granule cells: the GR membrane
//                update (kernels.cu:79-110), the MF->GR and GO->GR conductance
//                gathers (kernels.cu:169-199), PF->PC plasticity on plasticity
//                steps (kernels.cu:282-291), the GR history (kernels.cu:241-246),
//                the GR->GO, PF->BC and PF->SC spike counts (kernels.cu:112-167,
//                247-260) and the per-thread partial sums of the PF->PC
//                reduction in sumInputsNew's exact order (kernels.cu:262-376).
//  tailKernel    one CTA per network: every GO, SC, BC, PC, IO and NC update and
//                fan-out that the reference runs on the host
//                (innet.cpp:800-995, mzone.cpp:167-605).
//
// The reference moves its intermediate results through two host round trips
// per step; the same lags are kept here with device buffers indexed by step
// parity (GR->GO counts, GO spikes) or step mod 3 (PF->BC/SC/PC sums):
//   pass(t) reads GO spikes of t-1 and writes counts of step t;
//   tail(t) reads GR->GO counts of pass(t-1) and PF sums of pass(t-2).
// pass(t) and tail(t) therefore never touch the same buffer.
//
// Floating-point contract: this file is compiled with -fmad=false, so every
// float and double operation rounds once in source order, exactly as the
// oracle's -ffp-contract=off build.  Where the reference's C++ calls exp() on a
// float it gets glibc's expf; cbmExpf below evaluates the same published
// algorithm (ARM optimized-routines expf, as shipped in glibc 2.27+,
// with the fused multiply-adds of its x86-64 FMA build), so results match bit
// for bit.
#include <cstdint>
#include <cuda_runtime.h>

#include "cbm_device.cuh"
#include "cbm_kernels.cuh"
#include "cbm_rng.hpp"
#include "cbm_tma.cuh"

namespace cbm {

// 2^(i/32) as doubles with i/32 folded out of the exponent field:
// asuint64(2^(i/32)) - (i << 47).  Kernels copy it into shared memory:
// lanes index it with different i, which the constant cache would serialise.
__device__ uint64_t kExp2Tab[32] = {
	0x3ff0000000000000ull, 0x3fefd9b0d3158574ull, 0x3fefb5586cf9890full, 0x3fef9301d0125b51ull,
	0x3fef72b83c7d517bull, 0x3fef54873168b9aaull, 0x3fef387a6e756238ull, 0x3fef1e9df51fdee1ull,
	0x3fef06fe0a31b715ull, 0x3feef1a7373aa9cbull, 0x3feedea64c123422ull, 0x3feece086061892dull,
	0x3feebfdad5362a27ull, 0x3feeb42b569d4f82ull, 0x3feeab07dd485429ull, 0x3feea47eb03a5585ull,
	0x3feea09e667f3bcdull, 0x3fee9f75e8ec5f74ull, 0x3feea11473eb0187ull, 0x3feea589994cce13ull,
	0x3feeace5422aa0dbull, 0x3feeb737b0cdc5e5ull, 0x3feec49182a3f090ull, 0x3feed503b23e255dull,
	0x3feee89f995ad3adull, 0x3feeff76f2fb5e47ull, 0x3fef199bdd85529cull, 0x3fef3720dcef9069ull,
	0x3fef5818dcfba487ull, 0x3fef7c97337b9b5full, 0x3fefa4afa2a490daull, 0x3fefd0765b6e4540ull,
};

// exp of a float: x = (k + r) ln2/32, 2^(k/32) from the table (kExp2Tab or
// a shared-memory copy), 2^(r/32) from a cubic in r (coefficients of the
// published algorithm).
__device__ float cbmExpf(float x, const uint64_t *__restrict__ tab)
{
	const uint32_t ux = __float_as_uint(x);
	const uint32_t abstop = (ux >> 20) & 0x7ffu;
	if (abstop >= 0x42bu) {                       // |x| >= 88, inf or nan
		if (ux == 0xff800000u) return 0.0f;       // exp(-inf)
		if (abstop >= 0x7f8u) return x + x;       // inf or nan
		if (x > 0x1.62e42ep6f) return __int_as_float(0x7f800000);  // overflow
		if (x < -0x1.9fe368p6f) return 0.0f;                        // underflow
	}
	const double invLn2N = 0x1.71547652b82fep+0 * 32.0;
	const double shift = 0x1.8p+52;
	const double c0 = 0x1.c6af84b912394p-5 / 32.0 / 32.0 / 32.0;
	const double c1 = 0x1.ebfce50fac4f3p-3 / 32.0 / 32.0;
	const double c2 = 0x1.62e42ff0c52d6p-1 / 32.0;
	const double xd = (double)x;
	double kd = fma(invLn2N, xd, shift);
	const uint64_t ki = (uint64_t)__double_as_longlong(kd);
	kd = kd - shift;
	const double r = fma(invLn2N, xd, -kd);
	const uint64_t tb = tab[ki & 31u] + (ki << 47);
	const double s = __longlong_as_double((long long)tb);
	const double z = fma(c0, r, c1);
	const double r2 = r * r;
	double y = fma(c2, r, 1.0);
	y = fma(z, r2, y);
	y = y * s;
	return (float)y;
}

__global__ void expfProbeKernel(const float *in, float *out, uint32_t n)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = cbmExpf(in[i], kExp2Tab);
}

// exp of a double, where the reference calls the C library's double exp
// (the GO glutamate term, innet.cpp:850-858; the state-variable MF coding,
// Matthew_Sim_CBM/includes/statevariable.hpp:108-129).  The same published
// algorithm as glibc 2.28+ (ARM optimized-routines exp, N = 128) with the
// fused multiply-adds of its x86-64 FMA build: x = (k + r) ln2/128 with
// ln2/128 split in two parts, 2^(k/128) = H[k] (1 + T[k]) from the table,
// exp(r) - 1 from a quintic in r, and for |x| > 512 the rescaled paths that
// keep the scale finite.  kExpTab holds for each k the tail T[k] and
// asuint64(H[k]) - (k << 45), where H[k] is 2^(k/128) rounded to the nearest
// double and T[k] = (2^(k/128) - H[k]) / H[k] rounded likewise.
__device__ uint64_t kExpTab[256] = {
	0x0000000000000000ull, 0x3ff0000000000000ull, 0x3c9b3b4f1a88bf6eull, 0x3feff63da9fb3335ull,
	0xbc7160139cd8dc5dull, 0x3fefec9a3e778061ull, 0xbc905e7a108766d1ull, 0x3fefe315e86e7f85ull,
	0x3c8cd2523567f613ull, 0x3fefd9b0d3158574ull, 0xbc8bce8023f98efaull, 0x3fefd06b29ddf6deull,
	0x3c60f74e61e6c861ull, 0x3fefc74518759bc8ull, 0x3c90a3e45b33d399ull, 0x3fefbe3ecac6f383ull,
	0x3c979aa65d837b6dull, 0x3fefb5586cf9890full, 0x3c8eb51a92fdeffcull, 0x3fefac922b7247f7ull,
	0x3c3ebe3d702f9cd1ull, 0x3fefa3ec32d3d1a2ull, 0xbc6a033489906e0bull, 0x3fef9b66affed31bull,
	0xbc9556522a2fbd0eull, 0x3fef9301d0125b51ull, 0xbc5080ef8c4eea55ull, 0x3fef8abdc06c31ccull,
	0xbc91c923b9d5f416ull, 0x3fef829aaea92de0ull, 0x3c80d3e3e95c55afull, 0x3fef7a98c8a58e51ull,
	0xbc801b15eaa59348ull, 0x3fef72b83c7d517bull, 0xbc8f1ff055de323dull, 0x3fef6af9388c8deaull,
	0x3c8b898c3f1353bfull, 0x3fef635beb6fcb75ull, 0xbc96d99c7611eb26ull, 0x3fef5be084045cd4ull,
	0x3c9aecf73e3a2f60ull, 0x3fef54873168b9aaull, 0xbc8fe782cb86389dull, 0x3fef4d5022fcd91dull,
	0x3c8a6f4144a6c38dull, 0x3fef463b88628cd6ull, 0x3c807a05b0e4047dull, 0x3fef3f49917ddc96ull,
	0x3c968efde3a8a894ull, 0x3fef387a6e756238ull, 0x3c875e18f274487dull, 0x3fef31ce4fb2a63full,
	0x3c80472b981fe7f2ull, 0x3fef2b4565e27cddull, 0xbc96b87b3f71085eull, 0x3fef24dfe1f56381ull,
	0x3c82f7e16d09ab31ull, 0x3fef1e9df51fdee1ull, 0xbc3d219b1a6fbffaull, 0x3fef187fd0dad990ull,
	0x3c8b3782720c0ab4ull, 0x3fef1285a6e4030bull, 0x3c6e149289cecb8full, 0x3fef0cafa93e2f56ull,
	0x3c834d754db0abb6ull, 0x3fef06fe0a31b715ull, 0x3c864201e2ac744cull, 0x3fef0170fc4cd831ull,
	0x3c8fdd395dd3f84aull, 0x3feefc08b26416ffull, 0xbc86a3803b8e5b04ull, 0x3feef6c55f929ff1ull,
	0xbc924aedcc4b5068ull, 0x3feef1a7373aa9cbull, 0xbc9907f81b512d8eull, 0x3feeecae6d05d866ull,
	0xbc71d1e83e9436d2ull, 0x3feee7db34e59ff7ull, 0xbc991919b3ce1b15ull, 0x3feee32dc313a8e5ull,
	0x3c859f48a72a4c6dull, 0x3feedea64c123422ull, 0xbc9312607a28698aull, 0x3feeda4504ac801cull,
	0xbc58a78f4817895bull, 0x3feed60a21f72e2aull, 0xbc7c2c9b67499a1bull, 0x3feed1f5d950a897ull,
	0x3c4363ed60c2ac11ull, 0x3feece086061892dull, 0x3c9666093b0664efull, 0x3feeca41ed1d0057ull,
	0x3c6ecce1daa10379ull, 0x3feec6a2b5c13cd0ull, 0x3c93ff8e3f0f1230ull, 0x3feec32af0d7d3deull,
	0x3c7690cebb7aafb0ull, 0x3feebfdad5362a27ull, 0x3c931dbdeb54e077ull, 0x3feebcb299fddd0dull,
	0xbc8f94340071a38eull, 0x3feeb9b2769d2ca7ull, 0xbc87deccdc93a349ull, 0x3feeb6daa2cf6642ull,
	0xbc78dec6bd0f385full, 0x3feeb42b569d4f82ull, 0xbc861246ec7b5cf6ull, 0x3feeb1a4ca5d920full,
	0x3c93350518fdd78eull, 0x3feeaf4736b527daull, 0x3c7b98b72f8a9b05ull, 0x3feead12d497c7fdull,
	0x3c9063e1e21c5409ull, 0x3feeab07dd485429ull, 0x3c34c7855019c6eaull, 0x3feea9268a5946b7ull,
	0x3c9432e62b64c035ull, 0x3feea76f15ad2148ull, 0xbc8ce44a6199769full, 0x3feea5e1b976dc09ull,
	0xbc8c33c53bef4da8ull, 0x3feea47eb03a5585ull, 0xbc845378892be9aeull, 0x3feea34634ccc320ull,
	0xbc93cedd78565858ull, 0x3feea23882552225ull, 0x3c5710aa807e1964ull, 0x3feea155d44ca973ull,
	0xbc93b3efbf5e2228ull, 0x3feea09e667f3bcdull, 0xbc6a12ad8734b982ull, 0x3feea012750bdabfull,
	0xbc6367efb86da9eeull, 0x3fee9fb23c651a2full, 0xbc80dc3d54e08851ull, 0x3fee9f7df9519484ull,
	0xbc781f647e5a3ecfull, 0x3fee9f75e8ec5f74ull, 0xbc86ee4ac08b7db0ull, 0x3fee9f9a48a58174ull,
	0xbc8619321e55e68aull, 0x3fee9feb564267c9ull, 0x3c909ccb5e09d4d3ull, 0x3feea0694fde5d3full,
	0xbc7b32dcb94da51dull, 0x3feea11473eb0187ull, 0x3c94ecfd5467c06bull, 0x3feea1ed0130c132ull,
	0x3c65ebe1abd66c55ull, 0x3feea2f336cf4e62ull, 0xbc88a1c52fb3cf42ull, 0x3feea427543e1a12ull,
	0xbc9369b6f13b3734ull, 0x3feea589994cce13ull, 0xbc805e843a19ff1eull, 0x3feea71a4623c7adull,
	0xbc94d450d872576eull, 0x3feea8d99b4492edull, 0x3c90ad675b0e8a00ull, 0x3feeaac7d98a6699ull,
	0x3c8db72fc1f0eab4ull, 0x3feeace5422aa0dbull, 0xbc65b6609cc5e7ffull, 0x3feeaf3216b5448cull,
	0x3c7bf68359f35f44ull, 0x3feeb1ae99157736ull, 0xbc93091fa71e3d83ull, 0x3feeb45b0b91ffc6ull,
	0xbc5da9b88b6c1e29ull, 0x3feeb737b0cdc5e5ull, 0xbc6c23f97c90b959ull, 0x3feeba44cbc8520full,
	0xbc92434322f4f9aaull, 0x3feebd829fde4e50ull, 0xbc85ca6cd7668e4bull, 0x3feec0f170ca07baull,
	0x3c71affc2b91ce27ull, 0x3feec49182a3f090ull, 0x3c6dd235e10a73bbull, 0x3feec86319e32323ull,
	0xbc87c50422622263ull, 0x3feecc667b5de565ull, 0x3c8b1c86e3e231d5ull, 0x3feed09bec4a2d33ull,
	0xbc91bbd1d3bcbb15ull, 0x3feed503b23e255dull, 0x3c90cc319cee31d2ull, 0x3feed99e1330b358ull,
	0x3c8469846e735ab3ull, 0x3feede6b5579fdbfull, 0xbc82dfcd978e9db4ull, 0x3feee36bbfd3f37aull,
	0x3c8c1a7792cb3387ull, 0x3feee89f995ad3adull, 0xbc907b8f4ad1d9faull, 0x3feeee07298db666ull,
	0xbc55c3d956dcaebaull, 0x3feef3a2b84f15fbull, 0xbc90a40e3da6f640ull, 0x3feef9728de5593aull,
	0xbc68d6f438ad9334ull, 0x3feeff76f2fb5e47ull, 0xbc91eee26b588a35ull, 0x3fef05b030a1064aull,
	0x3c74ffd70a5fddcdull, 0x3fef0c1e904bc1d2ull, 0xbc91bdfbfa9298acull, 0x3fef12c25bd71e09ull,
	0x3c736eae30af0cb3ull, 0x3fef199bdd85529cull, 0x3c8ee3325c9ffd94ull, 0x3fef20ab5fffd07aull,
	0x3c84e08fd10959acull, 0x3fef27f12e57d14bull, 0x3c63cdaf384e1a67ull, 0x3fef2f6d9406e7b5ull,
	0x3c676b2c6c921968ull, 0x3fef3720dcef9069ull, 0xbc808a1883ccb5d2ull, 0x3fef3f0b555dc3faull,
	0xbc8fad5d3ffffa6full, 0x3fef472d4a07897cull, 0xbc900dae3875a949ull, 0x3fef4f87080d89f2ull,
	0x3c74a385a63d07a7ull, 0x3fef5818dcfba487ull, 0xbc82919e2040220full, 0x3fef60e316c98398ull,
	0x3c8e5a50d5c192acull, 0x3fef69e603db3285ull, 0x3c843a59ac016b4bull, 0x3fef7321f301b460ull,
	0xbc82d52107b43e1full, 0x3fef7c97337b9b5full, 0xbc892ab93b470dc9ull, 0x3fef864614f5a129ull,
	0x3c74b604603a88d3ull, 0x3fef902ee78b3ff6ull, 0x3c83c5ec519d7271ull, 0x3fef9a51fbc74c83ull,
	0xbc8ff7128fd391f0ull, 0x3fefa4afa2a490daull, 0xbc8dae98e223747dull, 0x3fefaf482d8e67f1ull,
	0x3c8ec3bc41aa2008ull, 0x3fefba1bee615a27ull, 0x3c842b94c3a9eb32ull, 0x3fefc52b376bba97ull,
	0x3c8a64a931d185eeull, 0x3fefd0765b6e4540ull, 0xbc8e37bae43be3edull, 0x3fefdbfdad9cbe14ull,
	0x3c77893b4d91cd9dull, 0x3fefe7c1819e90d8ull, 0x3c5305c14160cc89ull, 0x3feff3c22b8f71f1ull,
};

__device__ __forceinline__ double expSpecial(double tmp, uint64_t sbits, uint64_t ki)
{
	if ((ki & 0x80000000ull) == 0) {
		// k > 0: the scale's exponent may have overflowed; scale down by 2^1009
		const double scale = __longlong_as_double((long long)(sbits - (1009ull << 52)));
		return 0x1p1009 * fma(scale, tmp, scale);
	}
	// k < 0: the result may be subnormal; round once at the final precision
	const double scale = __longlong_as_double((long long)(sbits + (1022ull << 52)));
	double y = scale + scale * tmp;
	if (y < 1.0) {
		double lo = scale - y + scale * tmp;
		const double hi = 1.0 + y;
		lo = 1.0 - hi + y + lo;
		y = (hi + lo) - 1.0;
		if (y == 0.0) y = 0.0;
	}
	return 0x1p-1022 * y;
}

__device__ double cbmExp(double x, const uint64_t *__restrict__ tab)
{
	const uint64_t ux = (uint64_t)__double_as_longlong(x);
	uint32_t abstop = (uint32_t)(ux >> 52) & 0x7ffu;
	if (abstop - 0x3c9u >= 0x408u - 0x3c9u) {
		if (abstop - 0x3c9u >= 0x80000000u) return 1.0 + x;         // |x| < 2^-54
		if (abstop >= 0x409u) {                                      // |x| >= 1024
			if (ux == 0xfff0000000000000ull) return 0.0;             // exp(-inf)
			if (abstop >= 0x7ffu) return 1.0 + x;                    // inf or nan
			return (ux >> 63) ? 0.0 : __longlong_as_double(0x7ff0000000000000ll);
		}
		abstop = 0;  // 512 <= |x| < 1024: the rescaled paths
	}
	const double invLn2N = 0x1.71547652b82fep0 * 128.0, negLn2hiN = -0x1.62e42fefa0000p-8,
		negLn2loN = -0x1.cf79abc9e3b3ap-47, shift = 0x1.8p52;
	const double c2 = 0x1.ffffffffffdbdp-2, c3 = 0x1.555555555543cp-3, c4 = 0x1.55555cf172b91p-5,
		c5 = 0x1.1111167a4d017p-7;
	double kd = fma(invLn2N, x, shift);
	const uint64_t ki = (uint64_t)__double_as_longlong(kd);
	kd = kd - shift;
	const double r = fma(kd, negLn2loN, fma(kd, negLn2hiN, x));
	const uint32_t idx = 2u * (uint32_t)(ki & 127u);
	const double tail = __longlong_as_double((long long)tab[idx]);
	const uint64_t sbits = tab[idx + 1] + (ki << 45);
	const double r2 = r * r;
	const double tmp = fma(r2 * r2, fma(r, c5, c4), fma(r2, fma(r, c3, c2), tail + r));
	if (abstop == 0) return expSpecial(tmp, sbits, ki);
	const double scale = __longlong_as_double((long long)sbits);
	return fma(scale, tmp, scale);
}

__global__ void expProbeKernel(const double *in, double *out, uint32_t n)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = cbmExp(in[i], kExpTab);
}

__device__ __forceinline__ uint32_t spikeBit(const uint32_t *bits, uint32_t idx)
{
	return (bits[idx >> 5] >> (idx & 31u)) & 1u;
}

// Zone z's error drive at step t (setters, or the protocol for zone 0).
__device__ __forceinline__ float errDriveOf(const DevNet *N, uint64_t t, uint32_t z)
{
	if (z == 0 && N->protoSlots) return N->protoSlots[(t & 1) * 3 + 2];
	return N->ctl->errDrive[z];
}

// Report an error to the host: the error word lives in mapped pinned host
// memory, read after the host synchronises; a plain store (there is one
// error kind, so no read-modify-write is needed).
__device__ __forceinline__ void raiseError(const DevNet *N, uint32_t bit)
{
	*reinterpret_cast<volatile uint32_t *>(N->errFlag) = bit;
	__threadfence_system();
}

__device__ __forceinline__ const DevNet *locateNet(const DevNet *const *nets, const uint32_t *blockOffset,
		int numNets, uint32_t b, uint32_t &local)
{
	int lo = 0, hi = numNets - 1;
	while (lo < hi) {
		int mid = (lo + hi + 1) >> 1;
		if (blockOffset[mid] <= b) lo = mid; else hi = mid - 1;
	}
	local = b - blockOffset[lo];
	return nets[lo];
}

// ---------------------------------------------------------------- GR pass
// A block owns one PC row of the PF->PC reduction and a J-wide group of the
// reduction's thread index j: the cells pc*P + 2*bs*kk + h*bs + j for all
// kk < K, h in {0,1}, j in [j0, j0+J).  Every warp-row of J cells is
// contiguous, and each j's running sum over kk stays inside the block.
__global__ void __launch_bounds__(kPassThreads) grPassKernel(const DevNet *const *nets,
		const uint32_t *blockOffset, int numNets, uint32_t stepOffset)
{
	uint32_t local;
	const DevNet *__restrict__ N = locateNet(nets, blockOffset, numNets, blockIdx.x, local);
	const uint64_t t = stepsDone(N) + 1 + stepOffset;

	const uint32_t P = N->P, bs = N->bs, K = N->K, J = N->J, Z = N->numZones, numGR = N->numGR;
	const uint32_t pc = local / N->tilesPerPC;
	const uint32_t j0 = (local % N->tilesPerPC) * J;
	const uint32_t rows = 2 * K;

	extern __shared__ uint32_t smem[];
	uint32_t *sMF = smem;
	uint32_t *sGO = sMF + N->mfWords;
	uint32_t *sBC = sGO + N->goWords;
	uint32_t *sSC = sBC + N->bcLocal;
	float *sX = reinterpret_cast<float *>(sSC + N->scLocal);

	const uint32_t *mfSrc = N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords;
	const uint32_t *goSrc = N->goBits + (size_t)((t - 1) & 1) * N->goWords;
	for (uint32_t i = threadIdx.x; i < N->mfWords; i += blockDim.x) sMF[i] = mfSrc[i];
	for (uint32_t i = threadIdx.x; i < N->goWords; i += blockDim.x) sGO[i] = goSrc[i];
	for (uint32_t i = threadIdx.x; i < N->bcLocal + N->scLocal; i += blockDim.x) sBC[i] = 0;
	__syncthreads();

	const bool plastStep = stepMod(t, N->tsPerHistBinGR) == 0;
	float stepW[kMaxZones];
	for (uint32_t z = 0; z < Z; z++) {
		stepW[z] = 0.0f;
		if (plastStep) {
			const uint8_t sel = N->zones[z].plastSel[(t & 1) * N->numIO + N->zones[z].ioOfPC[pc]];
			stepW[z] = plasticityStep(N, t, z, sel);
		}
	}
	const float gLeak = N->gLeakGR, eLeak = N->eLeakGR, eGOIn = N->eGOGR;
	const float threshBase = N->threshRestGR, threshMax = N->threshMaxGR, threshDecay = N->threshDecGR;
	const float gDecMF = N->gDecMFtoGR, gIncMF = N->gIncMFtoGR, gDecGO = N->gDecGOtoGR, gIncGO = N->gIncGOtoGR;
	uint32_t *goCount = N->goCount + (size_t)(t & 1) * N->numGO;
	const uint32_t bcBase = (pc * P) >> N->bcShift, scBase = (pc * P) >> N->scShift;
	const bool bcWarpUniform = (1u << N->bcShift) >= J, scWarpUniform = (1u << N->scShift) >= J;

	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
	for (uint32_t r = warp; r < rows; r += nWarps) {
		const uint32_t base = pc * P + (r >> 1) * 2 * bs + (r & 1) * bs + j0;
		const bool active = lane < J;
		const uint32_t g = base + lane;
		uint32_t pf = 0;
		if (active) {
			float v = N->vGR[g];
			float gk = N->gKCaGR[g];
			float th = N->threshGR[g];
			const float gE = N->gESum[g];
			const float gI = N->gISum[g];
			const uint32_t ab = N->apBufGR[g];
			// calcActivityGRGPU (kernels.cu:79-110)
			float tempV = v + (gLeak + gk * gk * gk * gk) * (eLeak - v) - (gE) * v + (gI) * (eGOIn - v);
			float tempThresh = th + (threshBase - th) * threshDecay;
			const unsigned int tempAP = tempV > tempThresh;
			const float thN = tempAP * threshMax + (!tempAP) * tempThresh;
			const float gkd = gk * 0.9999f;
			const float gkN = tempAP * (gkd + 0.003f) + (!tempAP) * gkd;
			const uint32_t abN = (ab << 1) | tempAP;
			// updateGRInOPGPU for MF (this step's spikes) and GO (last step's)
			int cntMF = 0;
			for (uint32_t s = 0; s < N->nMFSlots; s++) cntMF += (int)spikeBit(sMF, N->mfIdx[(size_t)s * numGR + g]);
			int cntGO = 0;
			for (uint32_t s = 0; s < N->nGOSlots; s++) cntGO += (int)spikeBit(sGO, N->goIdx[(size_t)s * numGR + g]);
			const float gEN = gE * gDecMF + gIncMF * (cntMF);
			const float gIN = gI * gDecGO + gIncGO * (cntGO);
			N->vGR[g] = tempV;
			N->gKCaGR[g] = gkN;
			N->threshGR[g] = thN;
			N->gESum[g] = gEN;
			N->gISum[g] = gIN;
			N->apBufGR[g] = abN;
			// plasticity (phase 1) before this step's PF->PC output (phase 2)
			uint64_t h = 0;
			if (plastStep) h = N->historyGR[g];
			const uint32_t d = N->pfDelay[g];
			pf = d < 32u ? (abN >> d) & 1u : 0u;
			for (uint32_t z = 0; z < Z; z++) {
				float w = N->zones[z].w[g];
				if (plastStep) {
					w = w + ((h & 0x0000008000000000ull) > 0) * stepW[z];
					w = (w > 0) * w;
					w = (w > 1) + (w <= 1) * w;
					N->zones[z].w[g] = w;
				}
				sX[((size_t)z * rows + r) * J + lane] = w * pf;
			}
			if (plastStep) N->historyGR[g] = (h << 1) | ((abN & 0x0000001Fu) > 0);
			// GR->GO synapses whose delayed spike arrives now
			for (uint32_t s = 0; s < N->nOutSlots; s++) {
				const uint32_t c = N->outCon[(size_t)s * numGR + g];
				const uint32_t dl = c & 0xFFu;
				if (dl < 32u && ((abN >> dl) & 1u)) atomicAdd(&goCount[c >> 8], 1u);
			}
			if (!bcWarpUniform) atomicAdd(&sBC[(g >> N->bcShift) - bcBase], pf);
			if (!scWarpUniform) atomicAdd(&sSC[(g >> N->scShift) - scBase], pf);
		}
		const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, pf != 0));
		if (lane == 0 && cnt) {
			if (bcWarpUniform) atomicAdd(&sBC[(base >> N->bcShift) - bcBase], cnt);
			if (scWarpUniform) atomicAdd(&sSC[(base >> N->scShift) - scBase], cnt);
		}
	}
	__syncthreads();

	// sumInputsNew's per-thread running sums: tempSum += x[i] + x[i+bs]
	const uint32_t buf = (uint32_t)(t % 3);
	for (uint32_t task = threadIdx.x; task < Z * J; task += blockDim.x) {
		const uint32_t z = task / J, jj = task % J;
		const float *xs = sX + (size_t)z * rows * J + jj;
		float s = 0;
		for (uint32_t kk = 0; kk < K; kk++) s += xs[(2 * kk) * J] + xs[(2 * kk + 1) * J];
		N->zones[z].pcPartial[((size_t)buf * N->numPC + pc) * bs + j0 + jj] = s;
	}
	uint32_t *bcOut = N->bcCount + (size_t)buf * N->numBC;
	uint32_t *scOut = N->scCount + (size_t)buf * N->numSC;
	for (uint32_t i = threadIdx.x; i < N->bcLocal + N->scLocal; i += blockDim.x) {
		const uint32_t c = sBC[i];
		if (!c) continue;
		if (i < N->bcLocal) atomicAdd(&bcOut[bcBase + i], c);
		else atomicAdd(&scOut[scBase + i - N->bcLocal], c);
	}
}

// ------------------------------------------------------------ GR pass, TMA
// The same tile and per-cell work as grPassKernel for networks whose
// reduction width bs is at least 32 (tiles of 32-cell rows), with the tile's
// input rows streamed by TMA: one producer warp copies R = W*RW rows x 32
// cells of every GR array per stage into an S-deep ring of shared-memory
// stages; each of the W consumer warps updates RW rows of a stage, reading
// its inputs from shared memory and writing the new state straight to global
// memory.  Waits are bounded (kPassWaitLimitNs); a time-out sets
// kErrPassWait in the network's error word, which the host reports.
constexpr uint64_t kPassWaitLimitNs = 2000000000ull;

// Slot loops: MS > 0 compiles them for at most MS synapse slots per cell
// (predicated, fully unrolled); MS == 0 keeps runtime trip counts.
template <int MS>
__device__ __forceinline__ int countSpikes(const uint8_t *spikes, const uint16_t *idx, uint32_t n, uint32_t stride)
{
	int c = 0;
	if constexpr (MS > 0) {
#pragma unroll
		for (uint32_t s = 0; s < (uint32_t)MS; s++)
			if (s < n) c += spikes[idx[s * stride]];
	} else {
#pragma unroll 4
		for (uint32_t s = 0; s < n; s++) c += spikes[idx[s * stride]];
	}
	return c;
}

// Network shapes the TMA pass can be compiled for: slot counts, zones and
// whether every 32-cell row feeds a single BC and a single SC become
// compile-time constants (shared-memory offsets fold into immediates, slot
// loops lose their predicates).  Shape 0 reads them at run time.
template <int SH> struct PassShape {
	static constexpr uint32_t mf = 0, go = 0, out = 0, z = 0;
	static constexpr bool uniform = false, out16 = false;
};
// 4 MF and 3 GO dendrites, 4 GR->GO slots (streamed as the 16-bit table),
// one zone, BC and SC blocks of at least 32 cells (the eyelid networks)
template <> struct PassShape<1> {
	static constexpr uint32_t mf = 4, go = 3, out = 4, z = 1;
	static constexpr bool uniform = true, out16 = true;
};

template <int W, int RW, int S, int MINB, int MS, int SH>
__global__ void __launch_bounds__(32 * (W + 1), MINB) grPassTmaKernel(const DevNet *const *nets,
		const uint32_t *blockOffset, int numNets, uint32_t stepOffset, const DevNet *net0,
		const __grid_constant__ MFParam mfp, uint32_t *exitCount)
{
	// the next step's small-cell kernel may launch (it waits for this pass)
	pdlLaunchDependents();
	using Sh = PassShape<SH>;
	constexpr uint32_t R = W * RW;
	// one network: its descriptor comes as a parameter (a round trip fewer)
	uint32_t local = blockIdx.x;
	const DevNet *__restrict__ N = net0 ? net0 : locateNet(nets, blockOffset, numNets, blockIdx.x, local);
	const uint64_t t = stepsDone(N) + 1 + stepOffset;

	const uint32_t P = N->P, bs = N->bs, K = N->K, Z = Sh::z ? Sh::z : N->numZones;
	const uint32_t pc = local / N->tilesPerPC;
	const uint32_t j0 = (local % N->tilesPerPC) * 32u;
	const uint32_t rows = 2 * K, nStages = rows / R;
	const uint32_t nMFSlots = Sh::mf ? Sh::mf : N->nMFSlots, nGOSlots = Sh::go ? Sh::go : N->nGOSlots,
		nOutSlots = Sh::out ? Sh::out : N->nOutTma;
	const PassLayout L = passLayout(R, nMFSlots, nGOSlots, nOutSlots, Z, Sh::out16 ? 2u : 4u);

	extern __shared__ uint8_t passSmemRaw[];
	uint8_t *stages = passSmemRaw + ((128u - (tma::smemAddr(passSmemRaw) & 127u)) & 127u);
	uint64_t *full = reinterpret_cast<uint64_t *>(stages + (size_t)S * L.bytes);
	uint64_t *empty = full + S;
	// spikes of this step's MF and last step's GO as one byte per cell (the
	// sentinel index numMF / numGO reads 0)
	uint32_t *sBC = reinterpret_cast<uint32_t *>(empty + S);
	uint32_t *sSC = sBC + N->bcLocal;
	// 16-byte aligned: the spike tables after it take 16-byte stores
	float *sX = reinterpret_cast<float *>(sSC + ((N->bcLocal + N->scLocal + 3u) & ~3u) - N->bcLocal);
	uint8_t *sMF = reinterpret_cast<uint8_t *>(sX + (size_t)Z * rows * 32u);
	uint8_t *sGO = sMF + 32u * N->mfWords;

	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	if (threadIdx.x == 0) {
		for (int s = 0; s < S; s++) {
			tma::mbarInit(&full[s], 1);
			tma::mbarInit(&empty[s], W);
		}
		tma::fenceBarrierInit();
	}
	__syncthreads();

	const bool plastStep = stepMod(t, N->tsPerHistBinGR) == 0;
	const uint32_t rowBase = pc * rows;  // first row of the tile in the [numGR/bs][bs] view
	const uint32_t bcBase = (pc * P) >> N->bcShift, scBase = (pc * P) >> N->scShift;

	if (warp == W) {
		// ---- producer: lane 0 issues the copies; the whole warp takes the
		// running sums of the PF->PC reduction (sumInputsNew's per-thread
		// tempSum += x[i] + x[i+bs], kernels.cu:326-362, lane = j) stage by
		// stage in row order, as each stage is consumed
		const CUtensorMap *maps = N->passMaps;
		if (lane == 0)
			for (int m = 0; m < PM_W0 + (int)Z; m++) tma::prefetchMap(&maps[m]);
		const uint32_t tx = L.txBase + (plastStep ? L.txHist : 0u);
		uint32_t issued = 0, slot = 0, phase = 0;
		bool ok = true;
		float run[kMaxZones], even[kMaxZones];
#pragma unroll
		for (uint32_t z = 0; z < kMaxZones; z++) run[z] = even[z] = 0.0f;
		auto sumStage = [&](uint32_t sst) {
			for (uint32_t rr = 0; rr < R; rr++) {
				const uint32_t r = sst * R + rr;
#pragma unroll
				for (uint32_t z = 0; z < kMaxZones; z++) {
					if (z >= Z) break;
					const float x = sX[((size_t)z * rows + r) * 32u + lane];
					if (r & 1u) run[z] += even[z] + x;
					else even[z] = x;
				}
			}
		};
		{
			for (uint32_t st = 0; st < nStages; st++) {
				// refill number st/S of this slot waits until its previous
				// contents are consumed (and summed)
				if (st >= (uint32_t)S) {
					const bool done = tma::waitBounded(&empty[slot], phase ^ 1u, kPassWaitLimitNs);
					if (!__all_sync(0xffffffffu, done)) { ok = false; break; }
					sumStage(st - S);
				}
				issued = st + 1;
				if (lane != 0) { if (++slot == (uint32_t)S) { slot = 0; phase ^= 1u; } continue; }
				uint8_t *b = stages + (size_t)slot * L.bytes;
				uint64_t *bar = &full[slot];
				tma::arriveExpectTx(bar, tx);
				const int32_t x = (int32_t)j0, y = (int32_t)(rowBase + st * R);
#pragma unroll
				for (int m = PM_V; m <= PM_APBUF; m++) tma::load2d(b + (uint32_t)m * 128u * R, &maps[m], x, y, bar);
				tma::load3d(b + L.mfIdx, &maps[PM_MFIDX], x, y, 0, bar);
				tma::load3d(b + L.goIdx, &maps[PM_GOIDX], x, y, 0, bar);
				tma::load3d(b + L.outCon, &maps[Sh::out16 ? PM_OUTCON16 : PM_OUTCON], x, y, 0, bar);
				tma::load2d(b + L.pfDelay, &maps[PM_PFDELAY], x, y, bar);
				for (uint32_t z = 0; z < Z; z++) tma::load2d(b + L.w + z * 128u * R, &maps[PM_W0 + z], x, y, bar);
				if (plastStep) tma::load2d(b + L.hist, &maps[PM_HIST], x, y, bar);
				if (++slot == (uint32_t)S) { slot = 0; phase ^= 1u; }
			}
			__syncwarp();
			// the last stages, once consumed
			for (uint32_t st = issued > (uint32_t)S ? issued - S : 0; ok && st < issued; st++) {
				const bool done = tma::waitBounded(&empty[st % S], (st / S) & 1u, kPassWaitLimitNs);
				if (!__all_sync(0xffffffffu, done)) { ok = false; break; }
				sumStage(st);
			}
			if (ok) {
				const uint32_t buf = (uint32_t)(t % 3);
#pragma unroll
				for (uint32_t z = 0; z < kMaxZones; z++) {
					if (z >= Z) break;
					N->zones[z].pcPartial[((size_t)buf * N->numPC + pc) * bs + j0 + lane] = run[z];
				}
			} else if (lane == 0) {
				raiseError(N, kErrPassWait);
				// let the copies in flight land before the CTA's shared memory is released
				for (uint32_t st = issued > (uint32_t)S ? issued - S : 0; st < issued; st++)
					tma::waitBounded(&full[st % S], (st / S) & 1u, kPassWaitLimitNs);
			}
		}
	} else {
		// ---- consumers: warp w updates rows w, w+W, ..., w+(RW-1)W of every
		// stage.  They stage the spike tables while the first copies fly.
		const uint32_t *mfSrc = N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords;
		const uint32_t *goSrc = N->goBits + (size_t)((t - 1) & 1) * N->goWords;
		// one spike word per thread and round (the loads of a round in flight
		// together), spread to a byte per cell: (nibble * 0x204081) & 0x01010101
		// moves bit k of a nibble to bit 8k
		const uint32_t mfWords = N->mfWords, nWords = mfWords + N->goWords;
		for (uint32_t w0 = 0; w0 < nWords; w0 += 2u * 32u * W) {
			uint32_t v[2];
#pragma unroll
			for (int u = 0; u < 2; u++) {
				const uint32_t w = w0 + u * 32u * W + threadIdx.x;
				// MF words from the launch when it carries them (mfp.n > 0)
				v[u] = w >= nWords ? 0u : w >= mfWords ? __ldg(goSrc + (w - mfWords)) : mfp.n ? mfp.w[w] : __ldg(mfSrc + w);
			}
#pragma unroll
			for (int u = 0; u < 2; u++) {
				const uint32_t w = w0 + u * 32u * W + threadIdx.x;
				if (w < nWords) {
					uint4 *dst = reinterpret_cast<uint4 *>(w < mfWords ? sMF + 32u * w : sGO + 32u * (w - mfWords));
					uint32_t q[8];
#pragma unroll
					for (int k = 0; k < 8; k++) q[k] = (((v[u] >> (4 * k)) & 0xFu) * 0x00204081u) & 0x01010101u;
					dst[0] = make_uint4(q[0], q[1], q[2], q[3]);
					dst[1] = make_uint4(q[4], q[5], q[6], q[7]);
				}
			}
		}
		for (uint32_t i = threadIdx.x; i < N->bcLocal + N->scLocal; i += 32u * W) sBC[i] = 0;
		asm volatile("bar.sync 1, %0;" ::"r"(32u * W) : "memory");
		float stepW[kMaxZones];
#pragma unroll
		for (uint32_t z = 0; z < kMaxZones; z++) {
			stepW[z] = 0.0f;
			if (z < Z && plastStep) {
				const uint8_t sel = N->zones[z].plastSel[(t & 1) * N->numIO + N->zones[z].ioOfPC[pc]];
				stepW[z] = plasticityStep(N, t, z, sel);
			}
		}
		const float gLeak = N->gLeakGR, eLeak = N->eLeakGR, eGOIn = N->eGOGR;
		const float threshBase = N->threshRestGR, threshMax = N->threshMaxGR, threshDecay = N->threshDecGR;
		const float gDecMF = N->gDecMFtoGR, gIncMF = N->gIncMFtoGR, gDecGO = N->gDecGOtoGR, gIncGO = N->gIncGOtoGR;
		uint32_t *goCount = N->goCount + (size_t)(t & 1) * N->numGO;
		const bool bcWarpUniform = Sh::uniform || (1u << N->bcShift) >= 32u;
		const bool scWarpUniform = Sh::uniform || (1u << N->scShift) >= 32u;
		float *const vGR = N->vGR, *const gKCaGR = N->gKCaGR, *const threshGR = N->threshGR;
		float *const gESum = N->gESum, *const gISum = N->gISum;
		uint32_t *const apBufGR = N->apBufGR;
		uint64_t *const historyGR = N->historyGR;
		const uint32_t bcShift = N->bcShift, scShift = N->scShift;
		const uint32_t gTile = pc * P + j0 + lane;  // this lane's cell in row 0 of the tile
		uint32_t slot = 0, phase = 0;

		for (uint32_t st = 0; st < nStages; st++) {
			const bool ready = tma::waitBounded(&full[slot], phase, kPassWaitLimitNs);
			if (!__all_sync(0xffffffffu, ready)) {
				if (lane == 0) raiseError(N, kErrPassWait);
				break;
			}
			const uint8_t *b = stages + (size_t)slot * L.bytes;
			uint32_t pfs[RW];
#pragma unroll
			for (int q = 0; q < RW; q++) {
				const uint32_t rr = warp + q * W;          // row within the stage
				const uint32_t e = rr * 32u + lane;        // element within a region of R x 32
				const uint32_t r = st * R + rr;            // row within the tile
				const uint32_t g = gTile + r * bs;
				const float *sF = reinterpret_cast<const float *>(b);
				const float v = sF[0 * 32 * R + e];
				const float gk = sF[1 * 32 * R + e];
				const float th = sF[2 * 32 * R + e];
				const float gE = sF[3 * 32 * R + e];
				const float gI = sF[4 * 32 * R + e];
				const uint32_t ab = reinterpret_cast<const uint32_t *>(b)[5 * 32 * R + e];
				const uint16_t *mfI = reinterpret_cast<const uint16_t *>(b + L.mfIdx) + e;
				const uint16_t *goI = reinterpret_cast<const uint16_t *>(b + L.goIdx) + e;
				// the 32-bit slot table at element e (the 16-bit one is indexed from its base)
				const uint32_t *outC = reinterpret_cast<const uint32_t *>(b + L.outCon) + (Sh::out16 ? 0u : e);
				const uint32_t d = (b + L.pfDelay)[e];
				const uint64_t h = plastStep ? reinterpret_cast<const uint64_t *>(b + L.hist)[e] : 0ull;
				const int cntMF = countSpikes<MS>(sMF, mfI, nMFSlots, 32 * R);
				const int cntGO = countSpikes<MS>(sGO, goI, nGOSlots, 32 * R);

				// calcActivityGRGPU (kernels.cu:79-110)
				const float tempV = v + (gLeak + gk * gk * gk * gk) * (eLeak - v) - (gE) * v + (gI) * (eGOIn - v);
				const float tempThresh = th + (threshBase - th) * threshDecay;
				const unsigned int tempAP = tempV > tempThresh;
				const float thN = tempAP * threshMax + (!tempAP) * tempThresh;
				const float gkd = gk * 0.9999f;
				const float gkN = tempAP * (gkd + 0.003f) + (!tempAP) * gkd;
				const uint32_t abN = (ab << 1) | tempAP;
				// updateGRInOPGPU for MF (this step's spikes) and GO (last step's)
				const float gEN = gE * gDecMF + gIncMF * (cntMF);
				const float gIN = gI * gDecGO + gIncGO * (cntGO);
				vGR[g] = tempV;
				gKCaGR[g] = gkN;
				threshGR[g] = thN;
				gESum[g] = gEN;
				gISum[g] = gIN;
				apBufGR[g] = abN;
				// plasticity (phase 1) before this step's PF->PC output (phase 2)
				const uint32_t pf = d < 32u ? (abN >> d) & 1u : 0u;
#pragma unroll
				for (uint32_t z = 0; z < kMaxZones; z++) {
					if (z >= Z) break;
					float w = reinterpret_cast<const float *>(b + L.w)[z * 32 * R + e];
					if (plastStep) {
						w = w + ((h & 0x0000008000000000ull) > 0) * stepW[z];
						w = (w > 0) * w;
						w = (w > 1) + (w <= 1) * w;
						N->zones[z].w[g] = w;
					}
					sX[((size_t)z * rows + r) * 32u + lane] = w * pf;
				}
				if (plastStep) historyGR[g] = (h << 1) | ((abN & 0x0000001Fu) > 0);
				// GR->GO synapses whose delayed spike arrives now
				if (abN) {
					if constexpr (Sh::out16) {
						const uint16_t *outC16 = reinterpret_cast<const uint16_t *>(outC) + e;
#pragma unroll
						for (uint32_t s = 0; s < Sh::out; s++) {
							const uint32_t c = outC16[s * 32 * R];
							if (c != kOut16None && ((abN >> (c & 31u)) & 1u)) atomicAdd(&goCount[c >> 5], 1u);
						}
					} else if constexpr (MS > 0) {
#pragma unroll
						for (uint32_t s = 0; s < (uint32_t)MS; s++) {
							if (s >= nOutSlots) break;
							const uint32_t c = outC[s * 32 * R];
							const uint32_t dl = c & 0xFFu;
							if (dl < 32u && ((abN >> dl) & 1u)) atomicAdd(&goCount[c >> 8], 1u);
						}
					} else {
#pragma unroll 4
						for (uint32_t s = 0; s < nOutSlots; s++) {
							const uint32_t c = outC[s * 32 * R];
							const uint32_t dl = c & 0xFFu;
							if (dl < 32u && ((abN >> dl) & 1u)) atomicAdd(&goCount[c >> 8], 1u);
						}
					}
				}
				pfs[q] = pf;
			}
			__syncwarp();
			if (lane == 0) tma::arrive(&empty[slot]);
			if (++slot == (uint32_t)S) { slot = 0; phase ^= 1u; }
#pragma unroll
			for (int q = 0; q < RW; q++) {
				const uint32_t pf = pfs[q];
				const uint32_t g = gTile + (st * R + warp + q * W) * bs;
				if (!bcWarpUniform) atomicAdd(&sBC[(g >> bcShift) - bcBase], pf);
				if (!scWarpUniform) atomicAdd(&sSC[(g >> scShift) - scBase], pf);
				const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, pf != 0));
				if (lane == 0 && cnt) {
					const uint32_t base = g - lane;
					if (bcWarpUniform) atomicAdd(&sBC[(base >> bcShift) - bcBase], cnt);
					if (scWarpUniform) atomicAdd(&sSC[(base >> scShift) - scBase], cnt);
				}
			}
		}
	}
	__syncthreads();

	// GR->GO synapses past the streamed slot planes: their cells' new spike
	// buffers were written by this CTA before the barrier
	if (!Sh::out && N->ovStart) {
		const uint32_t e1 = N->ovStart[local + 1];
		uint32_t *goCountOv = N->goCount + (size_t)(t & 1) * N->numGO;
		for (uint32_t e = N->ovStart[local] + threadIdx.x; e < e1; e += blockDim.x) {
			const uint2 en = N->ovEntry[e];
			const uint32_t cl = en.x & 0xFFFFFFu, dl = en.x >> 24;
			const uint32_t g = pc * P + (cl >> 5) * bs + j0 + (cl & 31u);
			if ((N->apBufGR[g] >> dl) & 1u) atomicAdd(&goCountOv[en.y], 1u);
		}
	}

	// the BC and SC counts of the tile (the producer wrote the PF->PC partials)
	const uint32_t buf = (uint32_t)(t % 3);
	uint32_t *bcOut = N->bcCount + (size_t)buf * N->numBC;
	uint32_t *scOut = N->scCount + (size_t)buf * N->numSC;
	for (uint32_t i = threadIdx.x; i < N->bcLocal + N->scLocal; i += blockDim.x) {
		const uint32_t c = sBC[i];
		if (!c) continue;
		if (i < N->bcLocal) atomicAdd(&bcOut[bcBase + i], c);
		else atomicAdd(&scOut[scBase + i - N->bcLocal], c);
	}
	__syncthreads();
	passExitWait(exitCount);
}

// Geometries the host can pick: (consumer warps, rows per warp, stages,
// minimum resident CTAs per SM, slot bound MS); those with MS = 4 are also
// compiled for shape 1 (instantiated where passTmaKernelFor takes them).
#define CBM_PASS_TMA_CONFIGS(X) \
	X(8, 1, 3, 2, 4) X(8, 1, 3, 3, 4) X(8, 1, 4, 2, 4) X(8, 1, 2, 3, 4) X(4, 1, 4, 4, 4) X(4, 2, 3, 3, 4) X(4, 2, 4, 2, 4) \
	X(4, 2, 2, 4, 4) X(8, 1, 3, 2, 0) X(4, 1, 4, 1, 0) X(2, 1, 4, 1, 0) X(1, 1, 4, 1, 0)
#define CBM_PASS_TMA_INST(W, RW, S, B, M) \
	template __global__ void grPassTmaKernel<W, RW, S, B, M, 0>(const DevNet *const *, const uint32_t *, int, uint32_t, \
		const DevNet *, const __grid_constant__ MFParam, uint32_t *);
CBM_PASS_TMA_CONFIGS(CBM_PASS_TMA_INST)

int passTmaConfigCount()
{
	int n = 0;
#define CBM_PASS_TMA_COUNT(w, rw, s, b, m) n++;
	CBM_PASS_TMA_CONFIGS(CBM_PASS_TMA_COUNT)
#undef CBM_PASS_TMA_COUNT
	return n;
}

void passTmaConfig(int i, int *W, int *RW, int *S, int *B, int *M)
{
	int k = 0;
#define CBM_PASS_TMA_NTH(w, rw, s, b, m) if (k++ == i) { *W = w; *RW = rw; *S = s; *B = b; *M = m; return; }
	CBM_PASS_TMA_CONFIGS(CBM_PASS_TMA_NTH)
#undef CBM_PASS_TMA_NTH
}

const void *passTmaKernelFor(int W, int RW, int S, int B, int M, int shape)
{
#define CBM_PASS_TMA_PICK(w, rw, s, b, m) \
	if (W == w && RW == rw && S == s && B == b && M == m) { \
		if (shape == 0) return (const void *)&grPassTmaKernel<w, rw, s, b, m, 0>; \
		if (shape == 1 && m == 4) return (const void *)&grPassTmaKernel<w, rw, s, b, m, (m == 4 ? 1 : 0)>; \
		return nullptr; \
	}
	CBM_PASS_TMA_CONFIGS(CBM_PASS_TMA_PICK)
#undef CBM_PASS_TMA_PICK
	return nullptr;
}

int passShapeOf(const DevNet &h)
{
	using E = PassShape<1>;
	if (h.numZones == E::z && h.nMFSlots == E::mf && h.nGOSlots == E::go && h.nOutSlots == E::out &&
			(1u << h.bcShift) >= 32u && (1u << h.scShift) >= 32u && h.outCon16)
		return 1;
	return 0;
}

// ----------------------------------------------------- GR pass, persistent
// Single-network GR pass in persistent CTAs.  The work is cut into units of
// R = 2W rows x 32 cells of one tile, numbered tile-major; CTA c takes units
// c, c + gridDim, ... so that every SM gets the same number of units to
// within one.  A producer warp streams each unit's rows by TMA into an
// S-deep ring; consumer warp w updates rows 2w and 2w+1 of the unit, which
// are the two terms x[i], x[i+bs] of one step kk of sumInputsNew's per-thread
// running sum, and stores their sum (pairSum, one buffer per step parity).
// The running sums over kk (tempSum += x[i] + x[i+bs], kernels.cu:326-362)
// of step t-1 are taken in order at the start of step t's pass, when all of
// step t-1's pair sums are in memory, so the float order is the reference's
// and no CTA waits for another.  Spike counts go to global memory with
// integer reductions.
template <int MS>
__device__ __forceinline__ uint32_t outSpikes(const uint32_t *outC, uint32_t n, uint32_t stride, uint32_t abN,
		uint32_t *goCount)
{
	if (!abN) return 0;
	if constexpr (MS > 0) {
#pragma unroll
		for (uint32_t s = 0; s < (uint32_t)MS; s++) {
			if (s >= n) break;
			const uint32_t c = outC[s * stride];
			const uint32_t dl = c & 0xFFu;
			if (dl < 32u && ((abN >> dl) & 1u)) atomicAdd(&goCount[c >> 8], 1u);
		}
	} else {
#pragma unroll 4
		for (uint32_t s = 0; s < n; s++) {
			const uint32_t c = outC[s * stride];
			const uint32_t dl = c & 0xFFu;
			if (dl < 32u && ((abN >> dl) & 1u)) atomicAdd(&goCount[c >> 8], 1u);
		}
	}
	return 0;
}

template <int W, int S, int MINB, int MS>
__global__ void __launch_bounds__(32 * (W + 1), MINB) grPassPersistentKernel(const DevNet *const *nets,
		const uint32_t *blockOffset, int numNets, uint32_t stepOffset)
{
	(void)blockOffset; (void)numNets;
	constexpr uint32_t R = 2 * W;
	const DevNet *__restrict__ N = nets[0];
	const uint64_t t = stepsDone(N) + 1 + stepOffset;

	const uint32_t P = N->P, bs = N->bs, K = N->K, Z = N->numZones, numPC = N->numPC;
	const uint32_t rows = 2 * K, unitsPerTile = rows / R, tilesPerPC = N->tilesPerPC;
	const uint32_t numUnits = numPC * tilesPerPC * unitsPerTile;
	const uint32_t nMFSlots = N->nMFSlots, nGOSlots = N->nGOSlots, nOutSlots = N->nOutSlots;
	const PassLayout L = passLayout(R, nMFSlots, nGOSlots, nOutSlots, Z);

	extern __shared__ uint8_t passSmemRaw[];
	uint8_t *stages = passSmemRaw + ((128u - (tma::smemAddr(passSmemRaw) & 127u)) & 127u);
	uint64_t *full = reinterpret_cast<uint64_t *>(stages + (size_t)S * L.bytes);
	uint64_t *empty = full + S;
	float *sStepW = reinterpret_cast<float *>(empty + S);        // [numPC][Z] plasticity steps
	uint8_t *sMF = reinterpret_cast<uint8_t *>(sStepW + (size_t)numPC * Z);
	uint8_t *sGO = sMF + 32u * N->mfWords;

	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	if (threadIdx.x == 0) {
		for (int s = 0; s < S; s++) {
			tma::mbarInit(&full[s], 1);
			tma::mbarInit(&empty[s], W);
		}
		tma::fenceBarrierInit();
	}
	const bool plastStep = stepMod(t, N->tsPerHistBinGR) == 0;
	const uint32_t *mfSrc = N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords;
	const uint32_t *goSrc = N->goBits + (size_t)((t - 1) & 1) * N->goWords;
	for (uint32_t i = threadIdx.x; i < 32u * N->mfWords; i += blockDim.x) sMF[i] = (uint8_t)spikeBit(mfSrc, i);
	for (uint32_t i = threadIdx.x; i < 32u * N->goWords; i += blockDim.x) sGO[i] = (uint8_t)spikeBit(goSrc, i);
	if (plastStep) {
		for (uint32_t i = threadIdx.x; i < numPC * Z; i += blockDim.x) {
			const uint32_t pc = i / Z, z = i % Z;
			const uint8_t sel = N->zones[z].plastSel[(t & 1) * N->numIO + N->zones[z].ioOfPC[pc]];
			sStepW[i] = plasticityStep(N, t, z, sel);
		}
	}
	__syncthreads();

	if (warp == W) {
		// ---- producer
		if (lane == 0) {
			const CUtensorMap *maps = N->passMaps;
			for (int m = 0; m < PM_W0 + (int)Z; m++) tma::prefetchMap(&maps[m]);
			const uint32_t tx = L.txBase + (plastStep ? L.txHist : 0u);
			uint32_t issued = 0, slot = 0, phase = 0;
			bool ok = true;
			for (uint32_t u = blockIdx.x; u < numUnits; u += gridDim.x) {
				if (issued >= (uint32_t)S && !tma::waitBounded(&empty[slot], phase ^ 1u, kPassWaitLimitNs)) { ok = false; break; }
				const uint32_t tile = u / unitsPerTile, chunk = u % unitsPerTile;
				const uint32_t pc = tile / tilesPerPC, jt = tile % tilesPerPC;
				uint8_t *b = stages + (size_t)slot * L.bytes;
				uint64_t *bar = &full[slot];
				tma::arriveExpectTx(bar, tx);
				const int32_t x = (int32_t)(jt * 32u), y = (int32_t)(pc * rows + chunk * R);
#pragma unroll
				for (int m = PM_V; m <= PM_APBUF; m++) tma::load2d(b + (uint32_t)m * 128u * R, &maps[m], x, y, bar);
				tma::load3d(b + L.mfIdx, &maps[PM_MFIDX], x, y, 0, bar);
				tma::load3d(b + L.goIdx, &maps[PM_GOIDX], x, y, 0, bar);
				tma::load3d(b + L.outCon, &maps[PM_OUTCON], x, y, 0, bar);
				tma::load2d(b + L.pfDelay, &maps[PM_PFDELAY], x, y, bar);
				for (uint32_t z = 0; z < Z; z++) tma::load2d(b + L.w + z * 128u * R, &maps[PM_W0 + z], x, y, bar);
				if (plastStep) tma::load2d(b + L.hist, &maps[PM_HIST], x, y, bar);
				issued++;
				if (++slot == (uint32_t)S) { slot = 0; phase ^= 1u; }
			}
			if (!ok) {
				raiseError(N, kErrPassWait);
				for (uint32_t k = issued > (uint32_t)S ? issued - S : 0; k < issued; k++)
					tma::waitBounded(&full[k % S], (k / S) & 1u, kPassWaitLimitNs);
			}
		}
		return;
	}

	// ---- consumers
	const float gLeak = N->gLeakGR, eLeak = N->eLeakGR, eGOIn = N->eGOGR;
	const float threshBase = N->threshRestGR, threshMax = N->threshMaxGR, threshDecay = N->threshDecGR;
	const float gDecMF = N->gDecMFtoGR, gIncMF = N->gIncMFtoGR, gDecGO = N->gDecGOtoGR, gIncGO = N->gIncGOtoGR;
	uint32_t *goCount = N->goCount + (size_t)(t & 1) * N->numGO;
	const uint32_t buf = (uint32_t)(t % 3);
	uint32_t *bcOut = N->bcCount + (size_t)buf * N->numBC;
	uint32_t *scOut = N->scCount + (size_t)buf * N->numSC;
	const uint32_t bcShift = N->bcShift, scShift = N->scShift;
	const bool bcWarpUniform = (1u << bcShift) >= 32u, scWarpUniform = (1u << scShift) >= 32u;
	float *const vGR = N->vGR, *const gKCaGR = N->gKCaGR, *const threshGR = N->threshGR;
	float *const gESum = N->gESum, *const gISum = N->gISum;
	uint32_t *const apBufGR = N->apBufGR;
	uint64_t *const historyGR = N->historyGR;
	const uint32_t pairParity = (uint32_t)(t & 1), pairStride = numPC * K * bs;

	// running sums of step t-1 from its pair sums, in the reference's order
	{
		const uint32_t prevBuf = (uint32_t)((t - 1) % 3);
		const float *prevPairs = nullptr;
		for (uint32_t c = blockIdx.x * (W * 32u) + threadIdx.x; c < Z * numPC * bs; c += gridDim.x * (W * 32u)) {
			const uint32_t z = c / (numPC * bs), r = c % (numPC * bs), pc = r / bs, j = r % bs;
			prevPairs = N->zones[z].pairSum + (size_t)(pairParity ^ 1u) * pairStride + (size_t)pc * K * bs + j;
			float sum = 0;
#pragma unroll 8
			for (uint32_t k2 = 0; k2 < K; k2++) sum += prevPairs[(size_t)k2 * bs];
			N->zones[z].pcPartial[((size_t)prevBuf * numPC + pc) * bs + j] = sum;
		}
	}
	uint32_t slot = 0, phase = 0;

	for (uint32_t u = blockIdx.x; u < numUnits; u += gridDim.x) {
		const bool ready = tma::waitBounded(&full[slot], phase, kPassWaitLimitNs);
		if (!__all_sync(0xffffffffu, ready)) {
			if (lane == 0) raiseError(N, kErrPassWait);
			break;
		}
		const uint32_t tile = u / unitsPerTile, chunk = u % unitsPerTile;
		const uint32_t pc = tile / tilesPerPC, jt = tile % tilesPerPC;
		const uint32_t kk = (chunk * R) / 2 + warp;            // reduction step of this warp's row pair
		const uint32_t col = jt * 32u + lane;                  // reduction thread index j
		const uint8_t *b = stages + (size_t)slot * L.bytes;
		float x[2][kMaxZones];
		uint32_t pfs[2];
#pragma unroll
		for (int q = 0; q < 2; q++) {
			const uint32_t rr = 2 * warp + q;                  // row within the unit
			const uint32_t e = rr * 32u + lane;
			const uint32_t g = pc * P + (chunk * R + rr) * bs + col;
			const float *sF = reinterpret_cast<const float *>(b);
			const float v = sF[0 * 32 * R + e];
			const float gk = sF[1 * 32 * R + e];
			const float th = sF[2 * 32 * R + e];
			const float gE = sF[3 * 32 * R + e];
			const float gI = sF[4 * 32 * R + e];
			const uint32_t ab = reinterpret_cast<const uint32_t *>(b)[5 * 32 * R + e];
			const uint16_t *mfI = reinterpret_cast<const uint16_t *>(b + L.mfIdx) + e;
			const uint16_t *goI = reinterpret_cast<const uint16_t *>(b + L.goIdx) + e;
			const uint32_t *outC = reinterpret_cast<const uint32_t *>(b + L.outCon) + e;
			const uint32_t d = (b + L.pfDelay)[e];
			const uint64_t h = plastStep ? reinterpret_cast<const uint64_t *>(b + L.hist)[e] : 0ull;
			const int cntMF = countSpikes<MS>(sMF, mfI, nMFSlots, 32 * R);
			const int cntGO = countSpikes<MS>(sGO, goI, nGOSlots, 32 * R);

			// calcActivityGRGPU (kernels.cu:79-110)
			const float tempV = v + (gLeak + gk * gk * gk * gk) * (eLeak - v) - (gE) * v + (gI) * (eGOIn - v);
			const float tempThresh = th + (threshBase - th) * threshDecay;
			const unsigned int tempAP = tempV > tempThresh;
			const float thN = tempAP * threshMax + (!tempAP) * tempThresh;
			const float gkd = gk * 0.9999f;
			const float gkN = tempAP * (gkd + 0.003f) + (!tempAP) * gkd;
			const uint32_t abN = (ab << 1) | tempAP;
			// updateGRInOPGPU for MF (this step's spikes) and GO (last step's)
			const float gEN = gE * gDecMF + gIncMF * (cntMF);
			const float gIN = gI * gDecGO + gIncGO * (cntGO);
			vGR[g] = tempV;
			gKCaGR[g] = gkN;
			threshGR[g] = thN;
			gESum[g] = gEN;
			gISum[g] = gIN;
			apBufGR[g] = abN;
			// plasticity (phase 1) before this step's PF->PC output (phase 2)
			const uint32_t pf = d < 32u ? (abN >> d) & 1u : 0u;
#pragma unroll
			for (uint32_t z = 0; z < kMaxZones; z++) {
				x[q][z] = 0.0f;
				if (z >= Z) continue;
				float w = reinterpret_cast<const float *>(b + L.w)[z * 32 * R + e];
				if (plastStep) {
					w = w + ((h & 0x0000008000000000ull) > 0) * sStepW[pc * Z + z];
					w = (w > 0) * w;
					w = (w > 1) + (w <= 1) * w;
					N->zones[z].w[g] = w;
				}
				x[q][z] = w * pf;
			}
			if (plastStep) historyGR[g] = (h << 1) | ((abN & 0x0000001Fu) > 0);
			// GR->GO synapses whose delayed spike arrives now
			outSpikes<MS>(outC, nOutSlots, 32 * R, abN, goCount);
			pfs[q] = pf;
		}
		__syncwarp();
		if (lane == 0) tma::arrive(&empty[slot]);
		if (++slot == (uint32_t)S) { slot = 0; phase ^= 1u; }

		// x[i] + x[i+bs] of reduction step kk, per zone
#pragma unroll
		for (uint32_t z = 0; z < kMaxZones; z++) {
			if (z >= Z) break;
			N->zones[z].pairSum[(size_t)pairParity * pairStride + ((size_t)pc * K + kk) * bs + col] = x[0][z] + x[1][z];
		}
		// PF->BC and PF->SC counts
#pragma unroll
		for (int q = 0; q < 2; q++) {
			const uint32_t g = pc * P + (chunk * R + 2 * warp + q) * bs + col;
			const uint32_t pf = pfs[q];
			if (!bcWarpUniform && pf) atomicAdd(&bcOut[g >> bcShift], 1u);
			if (!scWarpUniform && pf) atomicAdd(&scOut[g >> scShift], 1u);
			const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, pf != 0));
			if (lane == 0 && cnt) {
				if (bcWarpUniform) atomicAdd(&bcOut[g >> bcShift], cnt);
				if (scWarpUniform) atomicAdd(&scOut[g >> scShift], cnt);
			}
		}
	}
}

#define CBM_PASS_PERSIST_CONFIGS(X) \
	X(4, 4, 2, 4) X(4, 3, 3, 4) X(2, 4, 4, 4) X(2, 6, 3, 4) X(8, 2, 2, 4) X(4, 4, 2, 0) X(2, 4, 2, 0) X(1, 4, 2, 0)
#define CBM_PASS_PERSIST_INST(W, S, B, M) \
	template __global__ void grPassPersistentKernel<W, S, B, M>(const DevNet *const *, const uint32_t *, int, uint32_t);
CBM_PASS_PERSIST_CONFIGS(CBM_PASS_PERSIST_INST)

const void *passPersistentKernelFor(int W, int S, int B, int M)
{
#define CBM_PASS_PERSIST_PICK(w, s, b, m) \
	if (W == w && S == s && B == b && M == m) return (const void *)&grPassPersistentKernel<w, s, b, m>;
	CBM_PASS_PERSIST_CONFIGS(CBM_PASS_PERSIST_PICK)
#undef CBM_PASS_PERSIST_PICK
	return nullptr;
}

// ------------------------------------------------------------------- tail
// Every small-cell update of step t for one network (one CTA per network).
// Statement forms follow the reference line by line so that each float and
// double operation is the same operation in the same order.
__device__ __forceinline__ float sumTree32(float v)
{
	// strides 16..1 of the halving tree, lane t accumulating t+h
	v = v + __shfl_down_sync(0xffffffffu, v, 16);
	v = v + __shfl_down_sync(0xffffffffu, v, 8);
	v = v + __shfl_down_sync(0xffffffffu, v, 4);
	v = v + __shfl_down_sync(0xffffffffu, v, 2);
	v = v + __shfl_down_sync(0xffffffffu, v, 1);
	return v;
}

// Reduction of one PC's bs partial sums with the halving tree of
// sumInputsNew (kernels.cu:326-362): strides bs/2, bs/4, ..., 1.
template <int PER> __device__ __forceinline__ float pcRowTreeWide(const float *part, uint32_t lane)
{
	// lane l holds partials l, l+32, ..., l+32(PER-1); strides >= 32 combine
	// registers of the same lane
	float v[PER];
#pragma unroll
	for (int m = 0; m < PER; m++) v[m] = part[lane + 32 * m];
#pragma unroll
	for (int h = PER / 2; h >= 1; h /= 2)
#pragma unroll
		for (int m = 0; m < h; m++) v[m] = v[m] + v[m + h];
	return sumTree32(v[0]);
}

__device__ float pcRowTree(const float *part, uint32_t bs, uint32_t lane)
{
	switch (bs) {
	case 512: return pcRowTreeWide<16>(part, lane);
	case 128: return pcRowTreeWide<4>(part, lane);
	case 32: return pcRowTreeWide<1>(part, lane);
	default: break;
	}
	float x = lane < bs ? part[lane] : 0.0f;
	for (uint32_t h = bs / 2; h >= 1; h /= 2) x = x + __shfl_down_sync(0xffffffffu, x, h);
	return x;
}

// Sequential left-to-right float sum of x[0..n) (the order of the
// reference's `sum = sum + x[j]` loops, from 0), eight loads in flight ahead
// of the adds.
__device__ __forceinline__ float orderedSum(const float *x, uint32_t n)
{
	float s = 0;
	uint32_t j = 0;
	for (; j + 8 <= n; j += 8) {
		float q[8];
#pragma unroll
		for (uint32_t u = 0; u < 8; u++) q[u] = x[j + u];
#pragma unroll
		for (uint32_t u = 0; u < 8; u++) s = s + q[u];
	}
	for (; j < n; j++) s = s + x[j];
	return s;
}

// Golgi role (one CTA per network): calcGOActivities, updateMFtoGOOut and
// updateGOtoGOOut (innet.cpp:816-980).  Reads GR->GO counts of pass(t-1),
// writes GO spikes of step t for pass(t+1).
// mfW: the step's MF spike words (its ring slot, or the launch's copy).
__device__ void golgiRole(const DevNet *__restrict__ N, uint64_t t, uint32_t *sm, const uint32_t *mfW)
{
	const uint32_t tid = threadIdx.x, nThr = blockDim.x, lane = tid & 31u;
	const uint32_t numGO = N->numGO;
	const uint32_t G = (uint32_t)((t - 1) & 1);
	uint64_t *sExp2 = reinterpret_cast<uint64_t *>(sm);
	uint32_t *sMF = sm + 64;
	uint32_t *sMFGO = sMF + N->mfWords;  // MF->GO input counts of this step
	float *sScale = reinterpret_cast<float *>(sMFGO + numGO);
	float *sV = sScale + numGO;
	float *sTh = sV + numGO;
	uint8_t *sAp = reinterpret_cast<uint8_t *>(sTh + numGO);
	for (uint32_t i = tid; i < N->mfWords; i += nThr) sMF[i] = mfW[i];
	for (uint32_t i = tid; i < numGO; i += nThr) sMFGO[i] = 0;
	if (tid < 32) sExp2[tid] = kExp2Tab[tid];
	__syncthreads();

	uint32_t *goIn = N->goCount + (size_t)G * numGO;
	uint32_t *goBitsOut = N->goBits + (size_t)(t & 1) * N->goWords;
	const float gIncGRtoGO = N->ctl->gIncGRtoGO;
	for (uint32_t base = 0; base < numGO; base += nThr) {
		const uint32_t i = base + tid;
		uint8_t ap = 0;
		if (i < numGO) {
			// every load of the update first, so that they are in flight
			// together (the compiler cannot reorder them past the stores)
			const unsigned int totalGRIn = goIn[i];
			const uint32_t inMF = N->inputMFGO[i];
			const float inDep = N->inputGOGABASynDepGO[i];
			const float gMF0 = N->gMFGO[i], gGR0 = N->gGRGO[i], gGO0 = N->gGOGO[i];
			const float glu0 = N->gluGO[i], mg0 = N->mGluRGO[i], mgi0 = N->gMGluRIncGO[i], gMGluR0 = N->gMGluRGO[i];
			const float thCur = N->threshCurGO[i], v0 = N->vGO[i], vCouple = N->vCoupleGO[i];
			const uint32_t apBuf = N->apBufGO[i];
			const float scale = N->goGABAOutSynScaleGOGO[i];

			goIn[i] = 0;
			N->sumGRInputGO[i] = totalGRIn;
			N->sumInputGOGABASynDepGO[i] = inDep;
			const float gMF = inMF * N->gIncMFtoGO + gMF0 * N->gDecMFtoGO;
			const float gGR = totalGRIn * gIncGRtoGO + gGR0 * N->gDecGRtoGO;
			const float gGO = inDep * N->gGABAIncGOtoGO + gGO0 * N->gGABADecGOtoGO;
			N->gMFGO[i] = gMF; N->gGRGO[i] = gGR; N->gGOGO[i] = gGO;
			float glu = glu0;
			glu = glu * N->gluDecayGO + totalGRIn * N->gluScaleGO * cbmExp(-1.5 * glu, kExpTab);
			float mg = mg0;
			mg = mg * N->mGluRDecayGO + glu * N->mGluRScaleGO * cbmExpf(-mg, sExp2);
			float mgi = mgi0;
			mgi = mgi * N->gMGluRIncDecayGO + mg * N->gMGluRIncScaleGO * cbmExpf(-mgi, sExp2);
			N->gluGO[i] = glu; N->mGluRGO[i] = mg; N->gMGluRIncGO[i] = mgi;
			N->gMGluRGO[i] = gMGluR0 * N->gMGluRDecGRtoGO + mgi * N->gMGluRScaleGRtoGO;
			float th = thCur + (N->threshRestGO - thCur) * N->threshDecGO;
			float v = v0;
			v = v + (N->gLeakGO * (N->eLeakGO - v)) + (gGO * (N->eGABAGO - v)) - (gMF + gGR) * v + vCouple;
			N->vGO[i] = v;
			ap = v > th;
			N->apGO[i] = ap;
			N->apBufGO[i] = (apBuf << 1) | (ap * 0x00000001u);
			th = ap * N->threshMaxGO + (!ap) * th;
			N->threshCurGO[i] = th;
			sScale[i] = scale;
			sV[i] = v; sTh[i] = th; sAp[i] = ap;
		}
		const uint32_t word = __ballot_sync(0xffffffffu, ap != 0);
		if (lane == 0 && i < numGO) goBitsOut[i >> 5] = word;
	}
	__syncthreads();
	// updateMFtoGOOut (innet.cpp:912-931): every spiking MF adds one to each
	// GO it targets (integer counts: the order of the additions is immaterial)
	for (uint32_t i = tid; i < N->numMF; i += nThr) {
		if (!spikeBit(sMF, i)) continue;
		const int n = N->numpMFfromMFtoGO[i];
		const uint32_t *dst = N->pMFfromMFtoGO + (size_t)i * N->maxnumpMFfromMFtoGO;
#pragma unroll 4
		for (int j = 0; j < n; j++) atomicAdd(&sMFGO[dst[j]], 1u);
	}
	// updateGOtoGOOut: GABA inputs in (source, slot) order, depression scale,
	// electrical coupling (innet.cpp:937-978)
	for (uint32_t d = tid; d < numGO; d += nThr) {
		uint32_t cnt = 0;
		float acc = 0;
		const uint32_t e0 = N->gogoStart[d], e1 = N->gogoStart[d + 1];
		const int nc = N->numpGOCoupInGOGO[d];
#pragma unroll 4
		for (uint32_t e = e0; e < e1; e++) {
			const uint32_t src = N->gogoSrc[e];
			if (sAp[src]) { cnt++; acc += sScale[src]; }
		}
		N->inputGOGO[d] = cnt;
		N->inputGOGABASynDepGO[d] = acc;
		const float s = sScale[d];
		const uint8_t ap = sAp[d];
		N->goGABAOutSynScaleGOGO[d] = s + (!ap) * (1 - s) * N->goGABAGOGOSynRec - ap * (s * (1 - N->goGABAGOGOSynDepF));
		float vc = 0;
		for (int j = 0; j < nc; j++) {
			const uint32_t n = N->pGOCoupInGOGO[(size_t)d * N->maxnumpGOCoupInGOGO + j];
			vc = vc + N->coupleRiRjRatioGO * (sV[n] - sV[d]);
		}
		N->vCoupleGO[d] = vc;
	}
	__syncthreads();
	for (uint32_t i = tid; i < numGO; i += nThr) N->inputMFGO[i] = sMFGO[i];
	// threshold coupling: the reference's serial sweep reads already-updated
	// thresholds of lower-indexed neighbours; the level schedule preserves it
	for (uint32_t L = 0; L < N->numCoupLevels; L++) {
		__syncthreads();
		for (uint32_t e = N->coupLevelStart[L] + tid; e < N->coupLevelStart[L + 1]; e += nThr) {
			const uint32_t i = N->coupLevelGO[e];
			const float own = sTh[i];
			float tc = 0;
			const int nc = N->numpGOCoupInGOGO[i];
			for (int j = 0; j < nc; j++) {
				const uint32_t n = N->pGOCoupInGOGO[(size_t)i * N->maxnumpGOCoupInGOGO + j];
				const float other = n < i ? N->threshCurGO[n] : sTh[n];
				tc = tc + N->coupleRiRjRatioGO * (other - own);
			}
			N->threshCurGO[i] = own + tc;
		}
	}
}

// Microzone role (one CTA per network): calcSCActivities (innet.cpp:892-911),
// the MF bookkeeping of updateMFInput (innet.cpp:800-815) and resetMFHist
// (:982-995), and every microzone update and fan-out (mzone.cpp:167-605).
// Reads the PF sums of pass(t-2).
// Barrier among the `count` threads of a warp group (barrier id >= 1).
__device__ __forceinline__ void barSync(uint32_t id, uint32_t count)
{
	asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Where the microzone role of step t finds the inputs that other kernels
// wrote: shared-memory copies when the network is staged, else global memory
// (mf, exp2 always in shared memory).  One copy per CTA, in shared memory.
struct ZoneIn {
	const uint32_t *mf;                 // MF spike bits of step t
	const uint32_t *bcSum, *scSum;      // PF->BC / PF->SC counts of pass(t-2)
	const float *pcPart[kMaxZones];     // [numPC][bs] PF->PC partial sums of pass(t-2) per zone
	const float *pcSum[kMaxZones];      // [numPC] PF->PC input sums of pass(t-2) per zone (pcSumMode), else null
	const uint64_t *exp2;               // cbmExpf table
	const float *err;                   // [numZones] error drives of step t, or null (read errDriveOf)
};

__device__ void protocolRecordWarp(const DevNet *__restrict__ N, uint64_t t, uint32_t lane);
__device__ void publishNC(const DevNet *N, uint64_t t, uint8_t *box);

// Warps of the microzone CTA's PC/BC/SC/MF group (the first ones); the rest
// form the NC/IO group.
__device__ __forceinline__ uint32_t zoneGroupAWarps(uint32_t nWarps) { return nWarps - nWarps / 3; }

// ncMailbox: mapped host memory that receives the step's NC spikes as soon
// as they are final (publishNC), or null.
__device__ void zoneRole(const DevNet *__restrict__ N, uint64_t t, uint32_t *sm, const ZoneIn &in,
		uint8_t *ncMailbox)
{
	const uint32_t tid = threadIdx.x, nThr = blockDim.x, lane = tid & 31u, warp = tid >> 5, nWarps = nThr >> 5;
	const uint32_t Z = N->numZones;
	const uint32_t numMF = N->numMF, numPC = N->numPC, numBC = N->numBC, numSC = N->numSC, numNC = N->numNC,
		numIO = N->numIO;
	const uint32_t R = (uint32_t)((t + 1) % 3);
	const uint8_t *mfRaw = N->hasMFRaw ? N->mfRaw + (size_t)stepMod(t - 1, N->mfRing) * numMF : nullptr;
	HostCtl *ctl = N->ctl;
	const uint32_t nMFNC = N->numpNCfromMFtoNC, nIONC = N->numpIOfromNCtoIO;
	// the step inputs (`in`) are ready for the PC/BC/SC/MF group when it
	// starts and for every thread after the two groups meet; the NC/IO group
	// needs none of them (its table is the global copy, its error drives
	// come from global memory), so that it may start before they arrive
	const uint32_t *sMF = nullptr;
	const uint64_t *exp2 = kExp2Tab;
	uint8_t *sApSC = reinterpret_cast<uint8_t *>(sm);
	float *ncScratch = reinterpret_cast<float *>(sApSC + ((numSC + 15) & ~15u));
	float *ioScratch = ncScratch + (size_t)Z * numNC * 2 * nMFNC;
	int *sFlags = reinterpret_cast<int *>(ioScratch + (size_t)Z * numIO * nIONC);

	// The PC/BC/SC/MF updates (warps [0, aW)) and the NC/IO updates (warps
	// [aW, all)) of a step do not read each other's results; the two warp
	// groups run them side by side and meet before the outputs.  The first
	// group (a warp per PC, then the element-parallel BC/SC/MF updates) gets
	// two thirds of the warps, the second (a warp per NC) the rest.
	const uint32_t aW = zoneGroupAWarps(nWarps), aThr = aW * 32u, bW = nWarps - aW, bThr = bW * 32u;
	const bool groupA = warp < aW;
	const uint32_t gTid = groupA ? tid : tid - aThr, gWarp = groupA ? warp : warp - aW;
	if (groupA) {
		sMF = in.mf;
		exp2 = in.exp2;
	}
	if (groupA) {
	// (tid, nThr, warp, nWarps) of the PC/BC/SC/MF warp group
	const uint32_t tid = gTid, nThr = aThr, warp = gWarp, nWarps = aW;
	// ---- phase 1 (cbmsimcore.cpp:192-200): PC and BC per zone, SC, and the
	// MF bookkeeping; the updates are independent.
	// calcPCActivities (mzone.cpp:187-226), one warp per PC; the SC
	// conductances update elementwise, their sum runs in the reference's order
	for (uint32_t task = warp; task < Z * numPC; task += nWarps) {
		const uint32_t z = Z == 1 ? 0u : task / numPC, i = Z == 1 ? task : task % numPC;
		const DevZone &Q = N->zones[z];
		const float inputSum = in.pcSum[z] ? in.pcSum[z][i] : pcRowTree(in.pcPart[z] + (size_t)i * N->bs, N->bs, lane);
		const uint32_t nSC = N->numpPCfromSCtoPC;
		for (uint32_t j = lane; j < nSC; j += 32) {
			const size_t k = (size_t)i * nSC + j;
			const float g0 = Q.gSCPC[k];
			const uint8_t inp = Q.inputSCPC[k];
			float g = g0;
			g = g + N->gIncSCtoPC * (1 - g) * inp;
			g = g * N->gDecSCtoPC;
			Q.gSCPC[k] = g;
		}
		__syncwarp();
		// lane 0: their sum in the reference's order, from the stored values
		const float gSCPCSum = lane == 0 ? orderedSum(Q.gSCPC + (size_t)i * nSC, nSC) : 0.0f;
		if (lane == 0) {
			const float gPF0 = Q.gPFPC[i], gBC0 = Q.gBCPC[i], vPC0 = Q.vPC[i], th0 = Q.threshPC[i];
			const uint32_t inBC = Q.inputBCPC[i], apBuf = Q.apBufPC[i];
			float gPF = gPF0 + inputSum * N->gIncGRtoPC;
			gPF = gPF * N->gDecGRtoPC;
			Q.gPFPC[i] = gPF;
			float gBC = gBC0 + inBC * N->gIncBCtoPC;
			gBC = gBC * N->gDecBCtoPC;
			Q.gBCPC[i] = gBC;
			float vPC = vPC0;
			vPC = vPC + (N->gLeakPC * (N->eLeakPC - vPC)) - (gPF * vPC) +
				(gBC * (N->eBCtoPC - vPC)) + (gSCPCSum * (N->eSCtoPC - vPC));
			Q.vPC[i] = vPC;
			float th = th0 + (N->threshDecPC * (N->threshRestPC - th0));
			const uint8_t ap = vPC > th;
			Q.apPC[i] = ap;
			Q.apBufPC[i] = (apBuf << 1) | (ap * 0x00000001u);
			Q.threshPC[i] = ap * N->threshMaxPC + (!ap) * th;
			if (ap) atomicAdd(&Q.scal[2], 1u);
		}
	}
	// calcBCActivities (mzone.cpp:228-256)
	for (uint32_t c = tid; c < Z * numBC; c += nThr) {
		const uint32_t bz = Z == 1 ? 0u : c / numBC, bi = Z == 1 ? c : c % numBC;
		const DevZone &Q = N->zones[bz];
		const uint32_t bInPF = in.bcSum[bi], bInPC = Q.inputPCBC[bi], bApBuf = Q.apBufBC[bi];
		const float bth0 = Q.threshBC[bi];
		float gPF = Q.gPFBC[bi] + (bInPF * N->gIncGRtoBC);
		gPF = gPF * N->gDecGRtoBC;
		Q.gPFBC[bi] = gPF;
		float gPC = Q.gPCBC[bi] + (bInPC * N->gIncPCtoBC);
		gPC = gPC * N->gDecPCtoBC;
		Q.gPCBC[bi] = gPC;
		float v = Q.vBC[bi];
		v = v + (N->gLeakBC * (N->eLeakBC - v)) - (gPF * v) + (gPC * (N->ePCtoBC - v));
		Q.vBC[bi] = v;
		float th = bth0 + N->threshDecBC * (N->threshRestBC - bth0);
		const uint8_t ap = v > th;
		Q.apBC[bi] = ap;
		Q.apBufBC[bi] = (bApBuf << 1) | (ap * 0x00000001u);
		Q.threshBC[bi] = ap * N->threshMaxBC + (!ap) * (th);
	}
	// calcSCActivities (innet.cpp:892-911)
	for (uint32_t c = tid; c < numSC; c += nThr) {
		const uint32_t sApBuf = N->apBufSC[c];
		const float sthOld = N->threshSC[c];
		float g = N->gPFSC[c] + (in.scSum[c] * N->gIncGRtoSC);
		g = g * N->gDecGRtoSC;
		N->gPFSC[c] = g;
		float v = N->vSC[c];
		v = v + (N->gLeakSC * (N->eLeakSC - v)) - g * v;
		N->vSC[c] = v;
		const uint8_t ap = v > sthOld;
		N->apSC[c] = ap;
		sApSC[c] = ap;
		N->apBufSC[c] = (sApBuf << 1) | (ap * 0x00000001u);
		float th = sthOld + N->threshDecSC * (N->threshRestSC - sthOld);
		N->threshSC[c] = ap * N->threshMaxSC + (!ap) * (th);
	}
	// updateMFInput's bookkeeping (innet.cpp:800-815)
	for (uint32_t c = tid; c < numMF; c += nThr) {
		const uint32_t m = spikeBit(sMF, c);
		N->histMF[c] = N->histMF[c] || (m > 0);
		N->apBufMF[c] = (N->apBufMF[c] << 1) | (m * 0x00000001u);
	}
	barSync(1, aThr);
	for (uint32_t i = tid; i < numBC; i += nThr) N->bcCount[(size_t)R * numBC + i] = 0;
	for (uint32_t i = tid; i < numSC; i += nThr) N->scCount[(size_t)R * numSC + i] = 0;
	}

	if (!groupA) {
	// (tid, nThr, warp, nWarps) of the NC/IO warp group
	const uint32_t tid = gTid, nThr = bThr, warp = gWarp, nWarps = bW;
	// this step's error drive of the IO a thread updates at the end, loaded
	// now so that the load overlaps the synapse and NC updates
	const float errOwn = tid < Z * numIO ? errDriveOf(N, t, Z == 1 ? 0u : tid / numIO) : 0.0f;
	// ---- phase 2: calcIOActivities (mzone.cpp:258-339) element-parallel,
	// calcNCActivities (mzone.cpp:341-407) one warp per NC.
	// NC->IO conductances: one thread per synapse, numbered from the group's
	// last thread down, so that they run on warps that take no NC (or the
	// last NCs).
	const uint32_t nIOSyn = Z * numIO * nIONC;
	for (uint32_t c = nThr - 1 - tid; c < nIOSyn; c += nThr) {
		const uint32_t iz = Z == 1 ? 0u : c / (numIO * nIONC), ik = Z == 1 ? c : c % (numIO * nIONC);
		const DevZone &Q = N->zones[iz];
		const float ig0 = Q.gNCIO[ik];
		const uint8_t iIn = Q.inputNCIO[ik];
		float g = ig0;
		g = g * cbmExpf(-N->msPerTimeStep / (-N->gDecTSofNCtoIO * cbmExpf(-g / N->gDecTTofNCtoIO, exp2) + N->gDecT0ofNCtoIO), exp2);
		g = g + iIn * N->gIncNCtoIO * cbmExpf(-g / N->gIncTauNCtoIO, exp2);
		Q.gNCIO[ik] = g;
		Q.inputNCIO[ik] = 0;
		ioScratch[c] = g;
	}
	// one warp per NC: its MF->NC synaptic conductances (lanes over the
	// synapses) into the warp's scratch, then the sums and the update, with
	// no barrier but the warp's own
	for (uint32_t task = warp; task < Z * numNC; task += nWarps) {
		const uint32_t z = Z == 1 ? 0u : task / numNC, i = Z == 1 ? task : task % numNC;
		const DevZone &Q = N->zones[z];
		float *const sNw = ncScratch + (size_t)task * 2 * nMFNC;
		for (uint32_t j = lane; j < nMFNC; j += 32) {
			const size_t nk = (size_t)i * nMFNC + j;
			const float nIn = Q.inputMFNC[nk], nWt = Q.mfSynWeightNC[nk];
			const float gmN0 = Q.gmaxNMDAofMFtoNC[nk], gN0 = Q.gMFNMDANC[nk];
			const float gmA0 = Q.gmaxAMPAofMFtoNC[nk], gA0 = Q.gMFAMPANC[nk];
			float gmN = gmN0;
			gmN = gmN * N->gmaxNMDADecMFtoNC + nIn * nWt * (1 - gmN);
			Q.gmaxNMDAofMFtoNC[nk] = gmN;
			float gN = gN0;
			gN = gN + N->gNMDAIncMFtoNC * (gmN - gN);
			Q.gMFNMDANC[nk] = gN;
			float gmA = gmA0;
			gmA = gmA * N->gmaxAMPADecMFtoNC + nIn * nWt * (1 - gmA);
			Q.gmaxAMPAofMFtoNC[nk] = gmA;
			float gA = gA0;
			gA = gA + N->gAMPAIncMFtoNC * (gmA - gA);
			Q.gMFAMPANC[nk] = gA;
			sNw[j] = gN;
			sNw[nMFNC + j] = gA;
		}
		__syncwarp();
		const float *sN = sNw;
		const float vNC0 = Q.vNC[i], thNC0 = Q.threshNC[i];
		const uint32_t apBufNC = Q.apBufNC[i];
		const uint32_t nPCNC = N->numpNCfromPCtoNC;
		for (uint32_t j = lane; j < nPCNC; j += 32) {
			const size_t k = (size_t)i * nPCNC + j;
			const float g0 = Q.gPCNC[k], scale = Q.gPCScaleNC[k];
			const uint8_t in = Q.inputPCNC[k];
			Q.gPCNC[k] = g0 * N->gDecPCtoNC + in * scale * (1 - g0);
		}
		__syncwarp();
		float gPCNCSum = lane == 0 ? orderedSum(Q.gPCNC + (size_t)i * nPCNC, nPCNC) : 0.0f;
		// lanes 0 and 1: the NMDA and AMPA sums over the NC's MF synapses in
		// the reference's order; eight loads in flight ahead of the adds
		const float partial = lane < 2 ? orderedSum(sN + lane * nMFNC, nMFNC) : 0.0f;
		const float ampaSum = __shfl_sync(0xffffffffu, partial, 1);
		if (lane == 0) {
			float gMFNMDASum = partial, gMFAMPASum = ampaSum;
			gMFNMDASum = gMFNMDASum * N->msPerTimeStep / ((float)nMFNC);
			gMFAMPASum = gMFAMPASum * N->msPerTimeStep / ((float)nMFNC);
			float vNC = vNC0;
			gMFNMDASum = gMFNMDASum * vNC / (-80.0f);
			gPCNCSum = gPCNCSum * N->msPerTimeStep / ((float)N->numpNCfromPCtoNC);
			vNC = vNC + N->gLeakNC * (N->eLeakNC - vNC) - (gMFNMDASum + gMFAMPASum) * vNC + gPCNCSum * (N->ePCtoNC - vNC);
			Q.vNC[i] = vNC;
			float th = thNC0 + N->threshDecNC * (N->threshRestNC - thNC0);
			const uint8_t ap = vNC > th;
			Q.apNC[i] = ap;
			Q.apBufNC[i] = (apBufNC << 1) | (ap * 0x00000001u);
			Q.threshNC[i] = ap * N->threshMaxNC + (!ap) * th;
		}
	}
	barSync(2, bThr);
	// every NC spike of the step is final: a host waiting on them gets them
	// now, from the group's last warp, which has no IO update (its system
	// fence overlaps the IO updates)
	if (ncMailbox && tid == nThr - 32u) publishNC(N, t, ncMailbox);
	for (uint32_t task = tid; task < Z * numIO; task += nThr) {
		const uint32_t z = Z == 1 ? 0u : task / numIO, i = Z == 1 ? task : task % numIO;
		const DevZone &Q = N->zones[z];
		const float v0 = Q.vIO[i], vCouple = Q.vCoupleIO[i], th0 = Q.threshIO[i];
		const float errDrive = task == tid ? errOwn : errDriveOf(N, t, z);
		const uint32_t apBuf = Q.apBufIO[i];
		float gNCSum = 0;
		for (uint32_t j = 0; j < nIONC; j++) gNCSum = gNCSum + ioScratch[(size_t)task * nIONC + j];
		gNCSum = gNCSum / 3.1;
		float v = v0;
		v = v + N->gLeakIO * (N->eLeakIO - v) + gNCSum * 1.5 * (N->eNCtoIO - v) + vCouple + errDrive;
		Q.vIO[i] = v;
		const uint8_t ap = v > th0;
		Q.apIO[i] = ap;
		Q.apBufIO[i] = (apBuf << 1) | (ap * 0x00000001u);
		Q.threshIO[i] = N->threshMaxIO * ap + (!ap) * (th0 + N->threshDecIO * (N->threshRestIO - th0));
	}
	}
	__syncthreads();
	sMF = in.mf;
	exp2 = in.exp2;

	// ---- microzone outputs (mzone.cpp:409-524) and the MF->NC population
	// bookkeeping (mzone.cpp:536-580): independent gathers, run as one flat
	// task space so that their loads are in flight together
	const bool popStep = stepMod(t, N->tsPerPopHistBinPC) == 0;
	// the device protocol's record of step t (its NC and PC spikes are final
	// now) on the last warp, beside the outputs: neither reads what the
	// other writes
	const bool recWarp = N->proto != nullptr && warp == nWarps - 1;
	const uint32_t oThr = N->proto != nullptr ? nThr - 32u : nThr;
	if (recWarp) protocolRecordWarp(N, t, lane);
	{
		const uint32_t nMFIn = Z * numNC * nMFNC, nBCPC = Z * numPC, nSCPC = Z * numPC * N->numpPCfromSCtoPC,
			nPCBC = Z * numBC, nPCNC = Z * numNC * N->numpNCfromPCtoNC, nIO = Z * numIO, nNC = Z * numNC;
		const uint32_t total = nMFIn + nBCPC + nSCPC + nPCBC + nPCNC + nIO + nNC + Z;
		for (uint32_t task = recWarp ? total : tid; task < total; task += oThr) {
			uint32_t r = task;
			if (r < nMFIn) {
				const uint32_t z = Z == 1 ? 0u : r / (numNC * nMFNC), k = Z == 1 ? r : r % (numNC * nMFNC);
				const uint32_t src = N->zones[z].pNCfromMFtoNC[k];
				N->zones[z].inputMFNC[k] = mfRaw ? mfRaw[src] : (uint8_t)spikeBit(sMF, src);
				continue;
			}
			r -= nMFIn;
			if (r < nBCPC) {
				const uint32_t z = Z == 1 ? 0u : r / numPC, i = Z == 1 ? r : r % numPC;
				const DevZone &Q = N->zones[z];
				uint32_t c = 0;
				const uint32_t e0 = Q.bcpcStart[i], e1 = Q.bcpcStart[i + 1];
#pragma unroll 4
				for (uint32_t e = e0; e < e1; e++) c += Q.apBC[Q.bcpcSrc[e]];
				Q.inputBCPC[i] = c;
				continue;
			}
			r -= nBCPC;
			if (r < nSCPC) {
				const uint32_t per = numPC * N->numpPCfromSCtoPC;
				const uint32_t z = Z == 1 ? 0u : r / per, k = Z == 1 ? r : r % per;
				N->zones[z].inputSCPC[k] = sApSC[N->zones[z].pPCfromSCtoPC[k]];
				continue;
			}
			r -= nSCPC;
			if (r < nPCBC) {
				const uint32_t z = Z == 1 ? 0u : r / numBC, i = Z == 1 ? r : r % numBC;
				const DevZone &Q = N->zones[z];
				uint32_t c = 0;
				const uint32_t e0 = Q.pcbcStart[i], e1 = Q.pcbcStart[i + 1];
#pragma unroll 4
				for (uint32_t e = e0; e < e1; e++) c += Q.apPC[Q.pcbcSrc[e]];
				Q.inputPCBC[i] = c;
				continue;
			}
			r -= nPCBC;
			if (r < nPCNC) {
				const uint32_t per = numNC * N->numpNCfromPCtoNC;
				const uint32_t z = Z == 1 ? 0u : r / per, k = Z == 1 ? r : r % per;
				N->zones[z].inputPCNC[k] = N->zones[z].apPC[N->zones[z].pNCfromPCtoNC[k]];
				continue;
			}
			r -= nPCNC;
			if (r < nIO) {
				const uint32_t z = Z == 1 ? 0u : r / numIO, i = Z == 1 ? r : r % numIO;
				const DevZone &Q = N->zones[z];
				const uint8_t ap = Q.apIO[i];
				const int32_t timer = Q.pfPCPlastTimerIO[i];
				const float vOwn = Q.vIO[i];
				float vc = 0;
				for (uint32_t j = 0; j < N->numpIOInIOIO; j++)
					vc = vc + N->coupleRiRjRatioIO * (Q.vIO[Q.pIOInIOIO[(size_t)i * N->numpIOInIOIO + j]] - vOwn);
				Q.pfPCPlastTimerIO[i] = (!ap) * (timer + 1) + ap * N->tsLTDStartAPIO;
				Q.vCoupleIO[i] = vc;
				continue;
			}
			r -= nIO;
			if (r < nNC) {
				const uint32_t z = Z == 1 ? 0u : r / numNC, i = Z == 1 ? r : r % numNC;
				const DevZone &Q = N->zones[z];
				const uint8_t apNC = Q.apNC[i];
				float p = Q.synIOPReleaseNC[i];
				p = p * cbmExpf(-N->msPerTimeStep / (N->relPDecTSofNCtoIO * cbmExpf(-p / N->relPDecTTofNCtoIO, exp2) + N->relPDecT0ofNCtoIO), exp2);
				p = p + apNC * N->relPIncNCtoIO * cbmExpf(-p / N->relPIncTauNCtoIO, exp2);
				Q.synIOPReleaseNC[i] = p;
				continue;
			}
			r -= nNC;
			{
				// updateMFNCSyn's population-activity bookkeeping for zone r
				const DevZone &Q = N->zones[r];
				int doLTD = 0, doLTP = 0;
				if (popStep) {
					uint32_t *s = Q.scal;
					const uint32_t sum = s[0], bin = s[1], popAct = s[2], noLTP = s[3], noLTD = s[4];
					const uint32_t old = Q.histPCPopAct[bin];
					const uint32_t newSum = sum - old + popAct;
					Q.histPCPopAct[bin] = popAct;
					s[0] = newSum;
					s[2] = 0;
					s[1] = (bin + 1) % N->numPopHistBinsPC;
					const float avgAllAPPC = ((float)newSum) / N->numPopHistBinsPC;
					if (avgAllAPPC >= N->synLTDPCPopActThreshMFtoNC && !noLTD) { doLTD = 1; s[4] = 1; }
					else if (avgAllAPPC < N->synLTDPCPopActThreshMFtoNC) s[4] = 0;
					if (avgAllAPPC <= N->synLTPPCPopActThreshMFtoNC && !noLTP) { doLTP = 1; s[3] = 1; }
					else if (avgAllAPPC > N->synLTPPCPopActThreshMFtoNC) s[3] = 0;
				}
				sFlags[2 * r] = doLTD;
				sFlags[2 * r + 1] = doLTP;
			}
		}
	}
	__syncthreads();

	// NC->IO release draws (mzone.cpp:505-511), MF->NC plasticity
	// (mzone.cpp:586-600), plasticity selector of the next step
	{
		const uint32_t nDraw = Z * numIO * nIONC, nW = popStep ? Z * numNC * nMFNC : 0, nSel = Z * numIO;
		const bool nextPlast = stepMod(t + 1, N->tsPerHistBinGR) == 0;
		for (uint32_t task = tid; task < nDraw + nW + nSel; task += nThr) {
			uint32_t r = task;
			if (r < nDraw) {
				const uint32_t per = numIO * nIONC;
				const uint32_t z = Z == 1 ? 0u : r / per, k = Z == 1 ? r : r % per;
				const uint32_t i = k / nIONC, j = k % nIONC;
				const DevZone &Q = N->zones[z];
				const double u = (double)rng::uniform24Keyed(Q.ncioKey, rng::ncioCounter(t, i, j, nIONC));
				Q.inputNCIO[k] = (u < Q.synIOPReleaseNC[Q.pIOfromNCtoIO[k]]);
				continue;
			}
			r -= nDraw;
			if (r < nW) {
				const uint32_t z = Z == 1 ? 0u : r / (numNC * nMFNC), k = Z == 1 ? r : r % (numNC * nMFNC);
				const DevZone &Q = N->zones[z];
				const int doLTD = sFlags[2 * z], doLTP = sFlags[2 * z + 1];
				const float wOld = Q.mfSynWeightNC[k];
				const float synWDelta = N->histMF[Q.pNCfromMFtoNC[k]] *
					(doLTD * N->synLTDStepSizeMFtoNC + doLTP * N->synLTPStepSizeMFtoNC);
				float w = wOld;
				w = w + synWDelta;
				w = (w > 0) * w;
				w = (w <= 1) * w + (w > 1);
				Q.mfSynWeightNC[k] = w;
				continue;
			}
			r -= nW;
			{
				const uint32_t z = Z == 1 ? 0u : r / numIO, i = Z == 1 ? r : r % numIO;
				const DevZone &Q = N->zones[z];
				uint8_t sel = 0;
				if (nextPlast) {
					const int32_t tm = Q.pfPCPlastTimerIO[i];
					sel = tm < N->tsLTDEndIO ? 1 : (tm > N->tsLTPStartAPIO ? 2 : 0);
				}
				Q.plastSel[((t + 1) & 1) * numIO + i] = sel;
			}
		}
	}
	__syncthreads();
	if (stepMod(t, N->numTSinMFHist) == 0)
		for (uint32_t i = tid; i < numMF; i += nThr) N->histMF[i] = 0;
	// the error drive is consumed once (mzone.cpp:334)
	if (tid < Z) ctl->errDrive[tid] = 0;
}

// Asynchronous global -> shared copies (no registers held while in flight).
__device__ __forceinline__ void cpAsync16(void *dst, const void *src)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smemAddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsync4(void *dst, const void *src)
{
	asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(tma::smemAddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncWaitAll()
{
	asm volatile("cp.async.wait_all;" ::: "memory");
}

// Copy a network's staging block (descriptor, step counter, staged arrays,
// segment table: one allocation laid out as its shared-memory copy) in one
// pass, every thread's copies in flight together; then point the copy's
// array pointers at shared memory.
__device__ void stageIn(const DevNet *N, uint8_t *base, uint32_t bytes)
{
	const uint32_t tid = threadIdx.x, nThr = blockDim.x;
	const uint8_t *src = reinterpret_cast<const uint8_t *>(N);
	for (uint32_t o = 16u * tid; o < bytes; o += 16u * nThr) cpAsync16(base + o, src + o);
	cpAsyncWaitAll();
	__syncthreads();
	DevNet *sNet = reinterpret_cast<DevNet *>(base);
	const StageSeg *segs = reinterpret_cast<const StageSeg *>(base + kStageArenaOff + sNet->zoneArenaBytes);
	for (uint32_t k = tid; k < sNet->numZoneSegs; k += nThr)
		*reinterpret_cast<uint8_t **>(reinterpret_cast<char *>(sNet) + segs[k].fieldOff) =
			base + kStageArenaOff + segs[k].smemOff;
}

// Copy the inputs of microzone step t that other kernels wrote
// (ZoneInputLayout) after the staging block and point `in` at them; the
// caller synchronises the CTA before use.  N is the staged descriptor, whose
// pointers to these inputs are global.
// mfParam: the launch's copy of the step's MF spike words, or null (the
// network's MF ring).
__device__ void stageInputs(const DevNet *N, uint64_t t, uint8_t *dyn, ZoneIn &in, const uint32_t *mfParam,
		uint32_t tid, uint32_t nThr)
{
	const uint32_t Z = N->numZones, numPC = N->numPC, bs = N->bs, R = (uint32_t)((t + 1) % 3);
	const ZoneInputLayout L = zoneInputLayout(N->mfWords, N->numBC, N->numSC, Z, numPC, N->bs);
	const uint32_t nPC = numPC * bs;
	const uint32_t *mfW = N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords;
	// small pieces as 4-byte words: table, MF bits, BC counts, SC counts
	const uint32_t e0 = 64, e1 = e0 + N->mfWords, e2 = e1 + N->numBC, e3 = e2 + N->numSC;
	for (uint32_t w = tid; w < e3; w += nThr) {
		const void *src;
		uint8_t *dst;
		if (w < e0) { src = reinterpret_cast<const uint32_t *>(kExp2Tab) + w; dst = dyn + L.exp2 + 4 * w; }
		else if (w < e1) {
			dst = dyn + L.mf + 4 * (w - e0);
			if (mfParam) {
				// the launch's copy: not global memory, so a plain store
				*reinterpret_cast<uint32_t *>(dst) = mfParam[w - e0];
				continue;
			}
			src = mfW + (w - e0);
		}
		else if (w < e2) { src = N->bcCount + (size_t)R * N->numBC + (w - e1); dst = dyn + L.bc + 4 * (w - e1); }
		else { src = N->scCount + (size_t)R * N->numSC + (w - e2); dst = dyn + L.sc + 4 * (w - e2); }
		cpAsync4(dst, src);
	}
	// the error drives: the protocol's slot for zone 0 under a device
	// protocol, else the setters' values (errDriveOf)
	if (tid < Z) {
		const float *src = tid == 0 && N->protoSlots ? N->protoSlots + (t & 1) * 3 + 2 : N->ctl->errDrive + tid;
		cpAsync4(dyn + L.err + 4 * tid, src);
	}
	// the PF->PC input sums of every zone when the GR pass made them, else
	// the partial sums: 16-byte pieces when the slot is 16-byte aligned
	// (numPC * bs a multiple of 4), else words
	for (uint32_t z = 0; z < Z; z++) {
		if (N->pcSumMode) {
			const float *src = N->zones[z].pcSum + (size_t)R * numPC;
			uint8_t *dst = dyn + L.pc + 4ull * z * numPC;
			for (uint32_t w = tid; w < numPC; w += nThr) cpAsync4(dst + 4 * w, src + w);
			continue;
		}
		const float *src = N->zones[z].pcPartial + (size_t)R * nPC;
		uint8_t *dst = dyn + L.pc + 4ull * z * nPC;
		if ((nPC & 3u) == 0)
			for (uint32_t w = 4 * tid; w < nPC; w += 4 * nThr) cpAsync16(dst + 4 * w, src + w);
		else
			for (uint32_t w = tid; w < nPC; w += nThr) cpAsync4(dst + 4 * w, src + w);
	}
	cpAsyncWaitAll();
	if (tid == 0) {
		in.mf = reinterpret_cast<const uint32_t *>(dyn + L.mf);
		in.bcSum = reinterpret_cast<const uint32_t *>(dyn + L.bc);
		in.scSum = reinterpret_cast<const uint32_t *>(dyn + L.sc);
		for (uint32_t z = 0; z < kMaxZones; z++) {
			in.pcPart[z] = reinterpret_cast<const float *>(dyn + L.pc) + (size_t)(z < Z ? z : 0) * nPC;
			in.pcSum[z] = N->pcSumMode ? reinterpret_cast<const float *>(dyn + L.pc) + (size_t)(z < Z ? z : 0) * numPC
				: nullptr;
		}
		in.exp2 = reinterpret_cast<const uint64_t *>(dyn + L.exp2);
		in.err = reinterpret_cast<const float *>(dyn + L.err);
	}
}

// Write the staged arrays that the step changes (the block's range from
// zoneWbOff to the end of the arena) back to global memory.
__device__ void stageOut(const DevNet *N, const uint8_t *base, const DevNet *sNet)
{
	const uint32_t from = kStageArenaOff + sNet->zoneWbOff, to = kStageArenaOff + sNet->zoneArenaBytes;
	uint4 *dst = reinterpret_cast<uint4 *>(const_cast<DevNet *>(N));
	const uint4 *src = reinterpret_cast<const uint4 *>(base);
	for (uint32_t i = from / 16u + threadIdx.x; i < to / 16u; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------- trial protocol
// Prepare step t+1 of a device protocol (in the Golgi CTA of step t, after
// its own work): the MF spikes of step t+1 into ring slot t % mfRing
// (PoissonRegenCells::calcActivity, poissonregencells.cpp:49-66, with the
// rate table ECManagementDelay::calcMFActivity picks, ecmanagementdelay.cpp:
// 175-194), and zone 0's error drive and PF->PC plasticity steps for step
// t+1 (ECManagementDelay::calcSimActivity, ecmanagementdelay.cpp:201-235).
// The draw of MF i for step t+1 is keyed by ((t+1) << 20) | i.
// Rate of fibre i under the state-variable coding at row `row` of the
// environment's values: gaussMFAct (statevariable.hpp:108-129) in its float
// and double steps.
__device__ __forceinline__ float stateVarRate(const DevProtocol *P, uint32_t i, uint64_t row)
{
	const uint32_t v = i / P->svPer;
	if (v >= P->svVars) return P->svRelaxed[i];
	float x = P->svValues[row * P->svVars + v];
	x = fmaxf(P->svLo, fminf(P->svHi, x));
	const float d = x - P->svMean[i];
	const float arg = (-(d * d)) / P->svDen;
	const float value = (float)(cbmExp((double)arg, kExpTab) / P->svNorm);
	const float a = value / P->svMaxPossible;
	return a * P->svExcited[i] + (1.0f - a) * P->svRelaxed[i];
}

__global__ void stateVarRatesKernel(const DevNet *N, uint64_t row, float *out)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < N->numMF) out[i] = stateVarRate(N->proto, i, stepMod(row, N->proto->svSteps));
}

__device__ void protocolPrepare(const DevNet *__restrict__ N, uint64_t t)
{
	DevProtocol *P = N->proto;
	const uint64_t k = t - P->startT;  // index of step t+1 within the protocol
	const int32_t time = (int32_t)stepMod(k, P->trialSteps);
	const uint32_t trial = (uint32_t)stepDiv(k, P->trialSteps);
	const bool csTrial = trial >= P->csStartTrial;
	const float *freq = P->freqBG;
	if (csTrial && time >= P->csOn && time < P->csOff) freq = time < P->csPOff ? P->freqCSPhasic : P->freqCSTonic;
	uint32_t *bits = const_cast<uint32_t *>(N->mfBits) + (size_t)stepMod(t, N->mfRing) * N->mfWords;
	const uint64_t ctr = (t + 1) << 20;
	const uint32_t numMF = N->numMF, words = N->mfWords;
	for (uint32_t base = 0; base < 32u * words; base += blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		uint32_t ap = 0;
		if (i < numMF) {
			float th = P->mfThresh[i];
			const float f = P->svValues ? stateVarRate(P, i, stepMod(k, P->svSteps)) : freq[i];
			th = th + (1 - th) * P->mfThreshDecay;
			const double u = (double)rng::uniform24Keyed(P->mfKey, ctr | i);
			ap = u < ((f * P->sPerTS) * th);
			th = (!ap) * th;
			P->mfThresh[i] = th;
		}
		const uint32_t word = __ballot_sync(0xffffffffu, ap != 0);
		if ((threadIdx.x & 31u) == 0 && i < 32u * words) bits[i >> 5] = word;
	}
	if (threadIdx.x == 0) {
		// every value loaded first, then the stores: one round trip
		int32_t *const ps = P->plastState;  // the eyelid driver's grPCPlastSet, grPCPlastReset
		float *const cur = P->curSteps;     // zone 0's LTD and LTP steps in force
		float *const slot = P->ctlSlots + ((t + 1) & 1) * 3;  // step t reads the other parity's slot
		const int32_t csOn = P->csOn, csOff = P->csOff, plastOn = P->plastOn, plastOff = P->plastOff;
		const float plastLTD = P->plastLTD, plastLTP = P->plastLTP, defaultLTD = P->defaultLTD,
			defaultLTP = P->defaultLTP, usErrDrive = P->usErrDrive;
		int32_t set = ps[0], reset = ps[1];
		float ltd = cur[0], ltp = cur[1];
		bool changed = false;
		if (time >= csOn + plastOn && !set && csTrial && time < csOff + plastOff) {
			set = 1; reset = 0;
			ltd = plastLTD; ltp = plastLTP;
			changed = true;
		}
		if (!reset && time >= csOff + plastOff && csTrial) {
			set = 0; reset = 1;
			ltd = defaultLTD; ltp = defaultLTP;
			changed = true;
		}
		if (changed) {
			ps[0] = set; ps[1] = reset;
			cur[0] = ltd; cur[1] = ltp;
		}
		slot[0] = ltd;
		slot[1] = ltp;
		slot[2] = (time == csOff - 1 && csTrial) ? usErrDrive : 0.0f;
	}
}

// Record step t of a device protocol (one warp of the microzone CTA of step
// t, once the step's NC and PC spikes are final; N may be its shared-memory
// copy): the eyelid integrator on
// zone 0's NC spikes every step (EyelidIntegrator::calcStep,
// eyelidintegrator.cpp:50-68) and, inside the recording window of a kept
// trial, NC and PC spike counts per bin and the integrator's output
// (ECTrialsData's PSH and eyelid trace, ecmanagementdelay.cpp:239-273).
__device__ void protocolRecordWarp(const DevNet *__restrict__ N, uint64_t t, uint32_t lane)
{
	const DevProtocol *P = N->proto;
	// every field is read before anything is written, so that the loads go
	// out together rather than one round trip after each store
	const uint64_t startT = P->startT;
	const uint32_t trialSteps = P->trialSteps, dataStart = P->dataStartTrial, numData = P->numDataTrials;
	const uint32_t recLen = P->recLen, binSteps = P->binSteps, nBins = P->nBins;
	const int32_t recFrom = P->recFrom;
	if (t < startT + 1) return;
	const uint64_t k = t - 1 - startT;
	const int32_t time = (int32_t)stepMod(k, trialSteps);
	const uint32_t trial = (uint32_t)stepDiv(k, trialSteps);
	const DevZone &Q = N->zones[0];
	const int32_t ct = time - recFrom;
	const bool rec = trial >= dataStart && trial < dataStart + numData && ct >= 0 && ct < (int32_t)recLen;
	const uint32_t dt = trial - dataStart;
	const uint32_t numNC = N->numNC, numPC = N->numPC;
	{
		// the integrator: lane i's conductance, then lane 0 sums them in
		// order i = 0, 1, ... as the reference's loop does
		const float decay = P->eyeGDecay, inc = P->eyeGInc, shift = P->eyeGShift, leak = P->eyeGLeak,
			maxAmp = P->eyeMaxAmp;
		float *const eyeG = P->eyeG, *const eyeVm = P->eyeVm, *const eyelid = P->eyelid;
		const float vm0 = lane == 0 ? *eyeVm : 0.0f;
		float gSum = 0;
		for (uint32_t i0 = 0; i0 < numNC; i0 += 32) {
			const uint32_t i = i0 + lane;
			float g = 0;
			if (i < numNC) {
				g = eyeG[i];
				g = g * decay;
				g = g + Q.apNC[i] * inc;
				eyeG[i] = g;
			}
			const uint32_t n = min(32u, numNC - i0);
			for (uint32_t q = 0; q < n; q++) gSum += __shfl_sync(0xffffffffu, g, q);
		}
		if (lane == 0) {
			gSum = gSum + shift;
			gSum = (gSum > 0) * gSum;
			float vm = vm0;
			vm = vm + (leak * (0 - vm)) + (gSum * (maxAmp - vm));
			*eyeVm = vm;
			if (rec) eyelid[(size_t)dt * recLen + ct] = vm;
		}
	}
	if (rec) {
		const uint32_t bin = (uint32_t)ct / binSteps;
		uint32_t *const ncPSH = P->ncPSH, *const pcPSH = P->pcPSH;
		for (uint32_t i = lane; i < numNC + numPC; i += 32) {
			if (i < numNC) ncPSH[((size_t)dt * nBins + bin) * numNC + i] += Q.apNC[i];
			else pcPSH[((size_t)dt * nBins + bin) * numPC + (i - numNC)] += Q.apPC[i - numNC];
		}
	}
}

// GR peri-stimulus histogram of step t (ECTrialsData::updatePSH("gr") of the
// eyelid driver, ecmanagementdelay.cpp:259-262; PeriStimHistFloat::update,
// peristimhistfloat.cpp): inside the recording window of a kept trial, the
// GR's spike of step t (bit 0 of its spike buffer, written by the step's GR
// pass) adds one to its count in the step's bin.  The kept trials add into
// one histogram, as the reference's does.  Counts stay below 65536 (the host
// checks binSteps x numDataTrials), so two u16 counts share a word safely.
__global__ void grPSHKernel(const DevNet *N, uint32_t stepOffset)
{
	const DevProtocol *P = N->proto;
	const uint64_t t = stepsDone(N) + 1 + stepOffset;
	if (!P || !P->grPSH || t < P->startT + 1) return;
	const uint64_t k = t - 1 - P->startT;
	const int32_t time = (int32_t)stepMod(k, P->trialSteps);
	const uint32_t trial = (uint32_t)stepDiv(k, P->trialSteps);
	const int32_t ct = time - P->recFrom;
	if (trial < P->dataStartTrial || trial >= P->dataStartTrial + P->numDataTrials || ct < 0 || ct >= P->recLen)
		return;
	const uint32_t i = 8u * (blockIdx.x * blockDim.x + threadIdx.x);
	if (i >= N->numGR) return;
	uint16_t *cnt = P->grPSH + (size_t)((uint32_t)ct / P->binSteps) * N->numGR + i;
	const uint4 a = *reinterpret_cast<const uint4 *>(N->apBufGR + i);
	const uint4 b = *reinterpret_cast<const uint4 *>(N->apBufGR + i + 4);
	uint4 c = *reinterpret_cast<const uint4 *>(cnt);
	c.x += (a.x & 1u) | ((a.y & 1u) << 16);
	c.y += (a.z & 1u) | ((a.w & 1u) << 16);
	c.z += (b.x & 1u) | ((b.y & 1u) << 16);
	c.w += (b.z & 1u) | ((b.w & 1u) << 16);
	*reinterpret_cast<uint4 *>(cnt) = c;
}

// The eyelid driver's trial data after step t (ecmanagementdelay.cpp:240-265,
// ECTrialsData): in the window of a kept trial, every histogram adds the
// step's value of each cell to the step's bin (PeriStimHistFloat::update,
// peristimhistfloat.cpp: spikes as 1 or 0, counts and floats as they are, in
// float, one add per step as the reference's), and at every 32nd window step
// after the first each raster takes the cells' apBuf words into its next row
// (SpikeRasterBitArray::updateRaster, spikerasterbitarray.cpp:62-80).  Rows
// are counted over all updates: (recLen - 1) / 32 updates a trial against
// recLen / 32 rows a raster trial.  One thread per cell; cells are GO, MF,
// SC, then zone 0's BC, PC, IO and NC.
// Cell c (GO, MF, SC, BC, PC, IO, NC in that order) of network N's
// ECTrialsData records at step stepsDone + 1 + stepOffset.
__device__ void trialDataCell(const DevNet *N, uint32_t stepOffset, uint32_t c)
{
	const DevProtocol *P = N->proto;
	const uint64_t t = stepsDone(N) + 1 + stepOffset;
	if (!P || !P->tdPSH || t < P->startT + 1) return;
	const uint64_t k = t - 1 - P->startT;
	const int32_t time = (int32_t)stepMod(k, P->trialSteps);
	const uint32_t trial = (uint32_t)stepDiv(k, P->trialSteps);
	const int32_t ct = time - P->recFrom;
	if (trial < P->dataStartTrial || trial >= P->dataStartTrial + P->numDataTrials || ct < 0 || ct >= P->recLen)
		return;
	const uint32_t nGO = N->numGO, nMF = N->numMF, nSC = N->numSC, nBC = N->numBC, nPC = N->numPC;
	const uint32_t nIO = N->numIO, nNC = N->numNC;
	if (c >= nGO + nMF + nSC + nBC + nPC + nIO + nNC) return;
	const DevZone &Z = N->zones[0];
	const size_t B = P->nBins, bin = (uint32_t)ct / P->binSteps;
	// histogram bases: go, grInputGO, goInputGO, goOutSynScale, mf, sc, bc, pc, io
	float *const hGO = P->tdPSH, *const hMF = hGO + 4 * B * nGO, *const hSC = hMF + B * nMF;
	float *const hBC = hSC + B * nSC, *const hPC = hBC + B * nBC, *const hIO = hPC + B * nPC;
	// raster row of this step: rt * rows + row within each raster, or none
	const uint32_t rows = (uint32_t)P->recLen / 32;
	uint64_t rrow = ~0ull;
	if (rows && ct > 0 && ct % 32 == 0) {
		const uint64_t u = (uint64_t)(trial - P->dataStartTrial) * (uint32_t)((P->recLen - 1) / 32) + (uint32_t)ct / 32 - 1;
		if (u < (uint64_t)P->numDataTrials * rows) rrow = u;
	}
	const size_t R = (size_t)P->numDataTrials * rows;
	uint32_t *const rGO = P->tdRaster, *const rSC = rGO + R * nGO, *const rBC = rSC + R * nSC;
	uint32_t *const rPC = rBC + R * nBC, *const rNC = rPC + R * nPC, *const rIO = rNC + R * nNC;
	uint32_t i = c;
	if (i < nGO) {
		float *h = hGO + bin * nGO + i;
		h[0] += (float)(N->apGO[i] > 0);
		h[B * nGO] += (float)N->sumGRInputGO[i];
		h[2 * B * nGO] += N->sumInputGOGABASynDepGO[i];
		h[3 * B * nGO] += N->goGABAOutSynScaleGOGO[i];
		if (rrow != ~0ull) rGO[rrow * nGO + i] = N->apBufGO[i];
		return;
	}
	i -= nGO;
	if (i < nMF) {
		hMF[bin * nMF + i] += (float)(N->apBufMF[i] & 1u);  // this step's MF spike
		return;
	}
	i -= nMF;
	if (i < nSC) {
		hSC[bin * nSC + i] += (float)(N->apSC[i] > 0);
		if (rrow != ~0ull) rSC[rrow * nSC + i] = N->apBufSC[i];
		return;
	}
	i -= nSC;
	if (i < nBC) {
		hBC[bin * nBC + i] += (float)(Z.apBC[i] > 0);
		if (rrow != ~0ull) rBC[rrow * nBC + i] = Z.apBufBC[i];
		return;
	}
	i -= nBC;
	if (i < nPC) {
		hPC[bin * nPC + i] += (float)(Z.apPC[i] > 0);
		if (rrow != ~0ull) rPC[rrow * nPC + i] = Z.apBufPC[i];
		return;
	}
	i -= nPC;
	if (i < nIO) {
		hIO[bin * nIO + i] += (float)(Z.apIO[i] > 0);
		if (rrow != ~0ull) rIO[rrow * nIO + i] = Z.apBufIO[i];
		return;
	}
	i -= nIO;
	if (rrow != ~0ull) rNC[rrow * nNC + i] = Z.apBufNC[i];
}

__global__ void trialDataKernel(const DevNet *N, uint32_t stepOffset)
{
	trialDataCell(N, stepOffset, blockIdx.x * blockDim.x + threadIdx.x);
}

// The batched form: thread c of the grid is cell c - cellOffset[n] of the
// network n with cellOffset[n] <= c < cellOffset[n + 1].
__global__ void trialDataBatchKernel(const DevNet *const *nets, const uint32_t *cellOffset, int numNets,
		uint32_t stepOffset)
{
	const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= cellOffset[numNets]) return;
	uint32_t local = 0;
	const DevNet *N = locateNet(nets, cellOffset, numNets, c, local);
	trialDataCell(N, stepOffset, local);
}

// Prepare the first step of a newly set protocol (the network's step tBase + 1).
__global__ void __launch_bounds__(kTailThreads) protocolPrimeKernel(const DevNet *N)
{
	protocolPrepare(N, stepsDone(N));
}

// Step t's NC spikes into mapped host memory for a host that waits on them
// (single steps through the reference API, cbm_sim_export's AP_NC): every
// zone's bytes from offset 8, a system-scope fence, then the step number as
// the 8-byte stamp at offset 0.  One thread of the microzone CTA, once the
// NC updates of the step are done.
__device__ void publishNC(const DevNet *N, uint64_t t, uint8_t *box)
{
	const uint32_t numNC = N->numNC;
	for (uint32_t z = 0; z < N->numZones; z++) {
		const uint8_t *ap = N->zones[z].apNC;
		for (uint32_t i = 0; i < numNC; i++) box[8 + z * numNC + i] = ap[i];
	}
	__threadfence_system();
	*reinterpret_cast<volatile uint64_t *>(box) = t;
}

// Small-cell update of step t: block 2n is network n's Golgi role, block
// 2n+1 its microzone role.  The two roles share no state.  The microzone
// role runs on shared-memory copies of its arrays and inputs when they fit
// (one bulk copy in and one out per step instead of a global round trip per
// phase).
__global__ void __launch_bounds__(kTailThreads, 1) tailKernel(const DevNet *const *nets, const uint32_t *stageBytes,
		uint32_t stepOffset, const DevNet *net0, uint32_t stage0, uint8_t *ncMailbox, const __grid_constant__ MFParam mfp)
{
	// the previous step first (its GR pass, and through that pass's exit
	// wait its small-cell kernel); then this step's GR pass may launch
	pdlWait();
	pdlLaunchDependents();
	const uint32_t net = blockIdx.x >> 1;
	// one network: descriptor and staging size come as parameters
	const DevNet *__restrict__ N = net0 ? net0 : nets[net];
	extern __shared__ __align__(16) uint32_t tailSmem[];
	__shared__ ZoneIn in;
	if (blockIdx.x & 1) {
		const uint32_t bytes = net0 ? stage0 : stageBytes[net];
		if (bytes) {
			uint8_t *base = reinterpret_cast<uint8_t *>(tailSmem);
			stageIn(N, base, bytes);
			const DevNet *sNet = reinterpret_cast<const DevNet *>(base);
			const uint64_t t = *reinterpret_cast<const uint64_t *>(base + kStageNetBytes) + 1 + stepOffset;
			uint8_t *dyn = base + bytes;
			// the PC/BC/SC/MF warp group copies the step inputs and waits for
			// them; the NC/IO group, which needs none, starts its updates
			const uint32_t aThr = 32u * zoneGroupAWarps(blockDim.x / 32u);
			if (threadIdx.x < aThr) {
				stageInputs(sNet, t, dyn, in, mfp.n ? mfp.w : nullptr, threadIdx.x, aThr);
				barSync(1, aThr);
			}
			const ZoneInputLayout L = zoneInputLayout(sNet->mfWords, sNet->numBC, sNet->numSC, sNet->numZones,
					sNet->numPC, sNet->bs);
			zoneRole(sNet, t, reinterpret_cast<uint32_t *>(dyn + L.bytes), in, ncMailbox);
			__syncthreads();
			stageOut(N, base, sNet);
		} else {
			// global-memory mode: the table and the MF bits in shared
			// memory, then the role's scratch
			const uint64_t t = stepsDone(N) + 1 + stepOffset;
			uint64_t *sExp2 = reinterpret_cast<uint64_t *>(tailSmem);
			uint32_t *sMF = tailSmem + 64;
			const uint32_t *mfW = mfp.n ? mfp.w : N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords;
			for (uint32_t i = threadIdx.x; i < N->mfWords; i += blockDim.x) sMF[i] = mfW[i];
			if (threadIdx.x < 32) sExp2[threadIdx.x] = kExp2Tab[threadIdx.x];
			const uint32_t R = (uint32_t)((t + 1) % 3);
			if (threadIdx.x == 0) {
				in.mf = sMF;
				in.bcSum = N->bcCount + (size_t)R * N->numBC;
				in.scSum = N->scCount + (size_t)R * N->numSC;
				for (uint32_t z = 0; z < kMaxZones; z++) {
					const DevZone &Q = N->zones[z < N->numZones ? z : 0];
					in.pcPart[z] = Q.pcPartial + (size_t)R * N->numPC * N->bs;
					in.pcSum[z] = N->pcSumMode ? Q.pcSum + (size_t)R * N->numPC : nullptr;
				}
				in.exp2 = sExp2;
				in.err = nullptr;
			}
			__syncthreads();
			zoneRole(N, t, sMF + ((N->mfWords + 3) & ~3u), in, ncMailbox);
		}
	} else {
		const uint64_t t = stepsDone(N) + 1 + stepOffset;
		uint32_t *ring = const_cast<uint32_t *>(N->mfBits) + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords;
		if (mfp.n) {
			// the launch's MF words into the ring, for the kernels after the
			// step (this step's kernels read the launch's copy)
			for (uint32_t i = threadIdx.x; i < mfp.n; i += blockDim.x) ring[i] = mfp.w[i];
		}
		golgiRole(N, t, tailSmem, mfp.n ? mfp.w : ring);
		if (N->proto) {
			__syncthreads();
			protocolPrepare(N, t);
		}
	}
}

__global__ void advanceStepKernel(uint64_t *const *tBases, int numNets, uint32_t steps)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < numNets) *tBases[i] += steps;
}

// exportAPGR (innet.cpp:687-701): the newest spike of every GR is bit 0 of
// its delay buffer.
__global__ void extractSpikesKernel(const uint32_t *apBuf, uint8_t *out, uint32_t n)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (uint8_t)(apBuf[i] & 1u);
}

// Second half of the measurement helpers' L2 flush: read back the buffer the
// flush has just written, so that the lines the next step finds in L2 are
// clean copies of it (the step is not charged for writing back the flush).
// The sink is written only if the buffer held a value the flush never
// writes, which keeps the loads live.
__global__ void flushReadKernel(const uint4 *buf, size_t n, uint32_t *sink)
{
	uint32_t acc = 0;
	for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
		const uint4 v = __ldcg(buf + i);
		acc |= (v.x ^ 0x5a5a5a5au) | (v.y ^ 0x5a5a5a5au) | (v.z ^ 0x5a5a5a5au) | (v.w ^ 0x5a5a5a5au);
	}
	if (acc) atomicOr(sink, acc);
}

}  // namespace cbm
