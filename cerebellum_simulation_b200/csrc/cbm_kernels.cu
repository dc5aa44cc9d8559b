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

namespace cbm {

// 2^(i/32) as doubles with i/32 folded out of the exponent field:
// asuint64(2^(i/32)) - (i << 47).
__constant__ uint64_t kExp2Tab[32] = {
	0x3ff0000000000000ull, 0x3fefd9b0d3158574ull, 0x3fefb5586cf9890full, 0x3fef9301d0125b51ull,
	0x3fef72b83c7d517bull, 0x3fef54873168b9aaull, 0x3fef387a6e756238ull, 0x3fef1e9df51fdee1ull,
	0x3fef06fe0a31b715ull, 0x3feef1a7373aa9cbull, 0x3feedea64c123422ull, 0x3feece086061892dull,
	0x3feebfdad5362a27ull, 0x3feeb42b569d4f82ull, 0x3feeab07dd485429ull, 0x3feea47eb03a5585ull,
	0x3feea09e667f3bcdull, 0x3fee9f75e8ec5f74ull, 0x3feea11473eb0187ull, 0x3feea589994cce13ull,
	0x3feeace5422aa0dbull, 0x3feeb737b0cdc5e5ull, 0x3feec49182a3f090ull, 0x3feed503b23e255dull,
	0x3feee89f995ad3adull, 0x3feeff76f2fb5e47ull, 0x3fef199bdd85529cull, 0x3fef3720dcef9069ull,
	0x3fef5818dcfba487ull, 0x3fef7c97337b9b5full, 0x3fefa4afa2a490daull, 0x3fefd0765b6e4540ull,
};

// exp of a float: x = (k + r) ln2/32, 2^(k/32) from the table, 2^(r/32) from
// a cubic in r (coefficients of the published algorithm).
__device__ float cbmExpf(float x)
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
	const uint64_t tb = kExp2Tab[ki & 31u] + (ki << 47);
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
	if (i < n) out[i] = cbmExpf(in[i]);
}

__device__ __forceinline__ uint32_t spikeBit(const uint32_t *bits, uint32_t idx)
{
	return (bits[idx >> 5] >> (idx & 31u)) & 1u;
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
	const uint64_t t = *N->tBase + 1 + stepOffset;

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

	const uint32_t *mfSrc = N->mfBits + (size_t)((t - 1) % N->mfRing) * N->mfWords;
	const uint32_t *goSrc = N->goBits + (size_t)((t - 1) & 1) * N->goWords;
	for (uint32_t i = threadIdx.x; i < N->mfWords; i += blockDim.x) sMF[i] = mfSrc[i];
	for (uint32_t i = threadIdx.x; i < N->goWords; i += blockDim.x) sGO[i] = goSrc[i];
	for (uint32_t i = threadIdx.x; i < N->bcLocal + N->scLocal; i += blockDim.x) sBC[i] = 0;
	__syncthreads();

	const bool plastStep = (t % N->tsPerHistBinGR) == 0;
	float stepW[kMaxZones];
	for (uint32_t z = 0; z < Z; z++) {
		stepW[z] = 0.0f;
		if (plastStep) {
			const uint8_t sel = N->zones[z].plastSel[(t & 1) * N->numIO + N->zones[z].ioOfPC[pc]];
			stepW[z] = sel == 1 ? N->ctl->ltdStep[z] : (sel == 2 ? N->ctl->ltpStep[z] : 0.0f);
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
__device__ float pcRowTree(const float *part, uint32_t bs, uint32_t lane)
{
	float v[16];
	const uint32_t per = bs >= 32 ? bs / 32 : 1;
	for (uint32_t m = 0; m < 16; m++) v[m] = 0.0f;
	for (uint32_t m = 0; m < per; m++) {
		const uint32_t idx = lane + 32 * m;
		v[m] = idx < bs ? part[idx] : 0.0f;
	}
	// strides >= 32 combine registers of the same lane
	for (uint32_t h = per / 2; h >= 1; h /= 2)
		for (uint32_t m = 0; m < h; m++) v[m] = v[m] + v[m + h];
	float x = v[0];
	if (bs >= 32) return sumTree32(x);
	for (uint32_t h = bs / 2; h >= 1; h /= 2) x = x + __shfl_down_sync(0xffffffffu, x, h);
	return x;
}

// Sequential left-to-right float sum of one value per lane (lanes 0..n-1),
// the order of the reference's `sum = sum + x[j]` loops; every lane gets it.
__device__ __forceinline__ float orderedLaneSum(float v, uint32_t n)
{
	float s = 0;
	for (uint32_t j = 0; j < n; j++) s = s + __shfl_sync(0xffffffffu, v, j);
	return s;
}

// Golgi role (one CTA per network): calcGOActivities, updateMFtoGOOut and
// updateGOtoGOOut (innet.cpp:816-980).  Reads GR->GO counts of pass(t-1),
// writes GO spikes of step t for pass(t+1).
__device__ void golgiRole(const DevNet *__restrict__ N, uint64_t t, uint32_t *sm)
{
	const uint32_t tid = threadIdx.x, nThr = blockDim.x, lane = tid & 31u;
	const uint32_t numGO = N->numGO;
	const uint32_t G = (uint32_t)((t - 1) & 1);
	const uint32_t *mfW = N->mfBits + (size_t)((t - 1) % N->mfRing) * N->mfWords;
	uint32_t *sMF = sm;
	float *sScale = reinterpret_cast<float *>(sMF + N->mfWords);
	float *sV = sScale + numGO;
	float *sTh = sV + numGO;
	uint8_t *sAp = reinterpret_cast<uint8_t *>(sTh + numGO);
	for (uint32_t i = tid; i < N->mfWords; i += nThr) sMF[i] = mfW[i];
	__syncthreads();

	uint32_t *goIn = N->goCount + (size_t)G * numGO;
	uint32_t *goBitsOut = N->goBits + (size_t)(t & 1) * N->goWords;
	const float gIncGRtoGO = N->ctl->gIncGRtoGO;
	for (uint32_t base = 0; base < numGO; base += nThr) {
		const uint32_t i = base + tid;
		uint8_t ap = 0;
		if (i < numGO) {
			const unsigned int totalGRIn = goIn[i];
			goIn[i] = 0;
			const uint32_t inMF = N->inputMFGO[i];
			const float inDep = N->inputGOGABASynDepGO[i];
			N->sumGRInputGO[i] = totalGRIn;
			N->sumInputGOGABASynDepGO[i] = inDep;
			const float gMF = inMF * N->gIncMFtoGO + N->gMFGO[i] * N->gDecMFtoGO;
			const float gGR = totalGRIn * gIncGRtoGO + N->gGRGO[i] * N->gDecGRtoGO;
			const float gGO = inDep * N->gGABAIncGOtoGO + N->gGOGO[i] * N->gGABADecGOtoGO;
			N->gMFGO[i] = gMF; N->gGRGO[i] = gGR; N->gGOGO[i] = gGO;
			float glu = N->gluGO[i];
			glu = glu * N->gluDecayGO + totalGRIn * N->gluScaleGO * exp(-1.5 * glu);
			float mg = N->mGluRGO[i];
			mg = mg * N->mGluRDecayGO + glu * N->mGluRScaleGO * cbmExpf(-mg);
			float mgi = N->gMGluRIncGO[i];
			mgi = mgi * N->gMGluRIncDecayGO + mg * N->gMGluRIncScaleGO * cbmExpf(-mgi);
			N->gluGO[i] = glu; N->mGluRGO[i] = mg; N->gMGluRIncGO[i] = mgi;
			N->gMGluRGO[i] = N->gMGluRGO[i] * N->gMGluRDecGRtoGO + mgi * N->gMGluRScaleGRtoGO;
			float th = N->threshCurGO[i] + (N->threshRestGO - N->threshCurGO[i]) * N->threshDecGO;
			float v = N->vGO[i];
			v = v + (N->gLeakGO * (N->eLeakGO - v)) + (gGO * (N->eGABAGO - v)) - (gMF + gGR) * v + N->vCoupleGO[i];
			N->vGO[i] = v;
			ap = v > th;
			N->apGO[i] = ap;
			N->apBufGO[i] = (N->apBufGO[i] << 1) | (ap * 0x00000001u);
			th = ap * N->threshMaxGO + (!ap) * th;
			N->threshCurGO[i] = th;
			sScale[i] = N->goGABAOutSynScaleGOGO[i];
			sV[i] = v; sTh[i] = th; sAp[i] = ap;
			// updateMFtoGOOut for this step's MF spikes, gathered per GO
			uint32_t cnt = 0;
			for (uint32_t e = N->mfgoStart[i]; e < N->mfgoStart[i + 1]; e++) cnt += spikeBit(sMF, N->mfgoSrc[e]);
			N->inputMFGO[i] = cnt;
		}
		const uint32_t word = __ballot_sync(0xffffffffu, ap != 0);
		if (lane == 0 && i < numGO) goBitsOut[i >> 5] = word;
	}
	__syncthreads();
	// updateGOtoGOOut: GABA inputs in (source, slot) order, depression scale,
	// electrical coupling (innet.cpp:937-978)
	for (uint32_t d = tid; d < numGO; d += nThr) {
		uint32_t cnt = 0;
		float acc = 0;
		for (uint32_t e = N->gogoStart[d]; e < N->gogoStart[d + 1]; e++) {
			const uint32_t src = N->gogoSrc[e];
			if (sAp[src]) { cnt++; acc += sScale[src]; }
		}
		N->inputGOGO[d] = cnt;
		N->inputGOGABASynDepGO[d] = acc;
		const float s = sScale[d];
		const uint8_t ap = sAp[d];
		N->goGABAOutSynScaleGOGO[d] = s + (!ap) * (1 - s) * N->goGABAGOGOSynRec - ap * (s * (1 - N->goGABAGOGOSynDepF));
		float vc = 0;
		const int nc = N->numpGOCoupInGOGO[d];
		for (int j = 0; j < nc; j++) {
			const uint32_t n = N->pGOCoupInGOGO[(size_t)d * N->maxnumpGOCoupInGOGO + j];
			vc = vc + N->coupleRiRjRatioGO * (sV[n] - sV[d]);
		}
		N->vCoupleGO[d] = vc;
	}
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
__device__ void zoneRole(const DevNet *__restrict__ N, uint64_t t, uint32_t *sm)
{
	const uint32_t tid = threadIdx.x, nThr = blockDim.x, lane = tid & 31u, warp = tid >> 5, nWarps = nThr >> 5;
	const uint32_t Z = N->numZones;
	const uint32_t numMF = N->numMF, numPC = N->numPC, numBC = N->numBC, numSC = N->numSC, numNC = N->numNC,
		numIO = N->numIO;
	const uint32_t R = (uint32_t)((t + 1) % 3);
	const uint32_t *mfW = N->mfBits + (size_t)((t - 1) % N->mfRing) * N->mfWords;
	const uint8_t *mfRaw = N->hasMFRaw ? N->mfRaw + (size_t)((t - 1) % N->mfRing) * numMF : nullptr;
	HostCtl *ctl = N->ctl;
	const uint32_t nMFNC = N->numpNCfromMFtoNC, nIONC = N->numpIOfromNCtoIO;
	uint32_t *sMF = sm;
	uint8_t *sApSC = reinterpret_cast<uint8_t *>(sMF + N->mfWords);
	float *ncScratch = reinterpret_cast<float *>(sApSC + ((numSC + 15) & ~15u));
	float *ioScratch = ncScratch + (size_t)Z * numNC * 2 * nMFNC;
	int *sFlags = reinterpret_cast<int *>(ioScratch + (size_t)Z * numIO * nIONC);
	for (uint32_t i = tid; i < N->mfWords; i += nThr) sMF[i] = mfW[i];
	__syncthreads();

	// ---- phase 1 (cbmsimcore.cpp:192-200): PC and BC per zone, SC
	for (uint32_t task = warp; task < Z * numPC; task += nWarps) {
		const uint32_t z = task / numPC, i = task % numPC;
		const DevZone &Q = N->zones[z];
		const float inputSum = pcRowTree(Q.pcPartial + ((size_t)R * numPC + i) * N->bs, N->bs, lane);
		// calcPCActivities (mzone.cpp:187-226); the SC conductances update
		// elementwise, their sum runs in the reference's order
		float gSCPCSum = 0;
		for (uint32_t j0 = 0; j0 < N->numpPCfromSCtoPC; j0 += 32) {
			const uint32_t j = j0 + lane;
			float g = 0;
			if (j < N->numpPCfromSCtoPC) {
				const size_t k = (size_t)i * N->numpPCfromSCtoPC + j;
				g = Q.gSCPC[k];
				g = g + N->gIncSCtoPC * (1 - g) * Q.inputSCPC[k];
				g = g * N->gDecSCtoPC;
				Q.gSCPC[k] = g;
			}
			const uint32_t n = min(32u, N->numpPCfromSCtoPC - j0);
			for (uint32_t q = 0; q < n; q++) gSCPCSum += __shfl_sync(0xffffffffu, g, q);
		}
		if (lane == 0) {
			float gPF = Q.gPFPC[i] + inputSum * N->gIncGRtoPC;
			gPF = gPF * N->gDecGRtoPC;
			Q.gPFPC[i] = gPF;
			float gBC = Q.gBCPC[i] + Q.inputBCPC[i] * N->gIncBCtoPC;
			gBC = gBC * N->gDecBCtoPC;
			Q.gBCPC[i] = gBC;
			float vPC = Q.vPC[i];
			vPC = vPC + (N->gLeakPC * (N->eLeakPC - vPC)) - (gPF * vPC) +
				(gBC * (N->eBCtoPC - vPC)) + (gSCPCSum * (N->eSCtoPC - vPC));
			Q.vPC[i] = vPC;
			float th = Q.threshPC[i] + (N->threshDecPC * (N->threshRestPC - Q.threshPC[i]));
			const uint8_t ap = vPC > th;
			Q.apPC[i] = ap;
			Q.apBufPC[i] = (Q.apBufPC[i] << 1) | (ap * 0x00000001u);
			Q.threshPC[i] = ap * N->threshMaxPC + (!ap) * th;
			if (ap) atomicAdd(&Q.scal[2], 1u);
		}
	}
	const uint32_t *bcSum = N->bcCount + (size_t)R * numBC;
	const uint32_t *scSum = N->scCount + (size_t)R * numSC;
	for (uint32_t task = tid; task < Z * numBC; task += nThr) {
		const uint32_t z = task / numBC, i = task % numBC;
		const DevZone &Q = N->zones[z];
		// calcBCActivities (mzone.cpp:228-256)
		float gPF = Q.gPFBC[i] + (bcSum[i] * N->gIncGRtoBC);
		gPF = gPF * N->gDecGRtoBC;
		Q.gPFBC[i] = gPF;
		float gPC = Q.gPCBC[i] + (Q.inputPCBC[i] * N->gIncPCtoBC);
		gPC = gPC * N->gDecPCtoBC;
		Q.gPCBC[i] = gPC;
		float v = Q.vBC[i];
		v = v + (N->gLeakBC * (N->eLeakBC - v)) - (gPF * v) + (gPC * (N->ePCtoBC - v));
		Q.vBC[i] = v;
		float th = Q.threshBC[i] + N->threshDecBC * (N->threshRestBC - Q.threshBC[i]);
		const uint8_t ap = v > th;
		Q.apBC[i] = ap;
		Q.apBufBC[i] = (Q.apBufBC[i] << 1) | (ap * 0x00000001u);
		Q.threshBC[i] = ap * N->threshMaxBC + (!ap) * (th);
	}
	for (uint32_t i = tid; i < numSC; i += nThr) {
		float g = N->gPFSC[i] + (scSum[i] * N->gIncGRtoSC);
		g = g * N->gDecGRtoSC;
		N->gPFSC[i] = g;
		float v = N->vSC[i];
		v = v + (N->gLeakSC * (N->eLeakSC - v)) - g * v;
		N->vSC[i] = v;
		const float thOld = N->threshSC[i];
		const uint8_t ap = v > thOld;
		N->apSC[i] = ap;
		sApSC[i] = ap;
		N->apBufSC[i] = (N->apBufSC[i] << 1) | (ap * 0x00000001u);
		float th = thOld + N->threshDecSC * (N->threshRestSC - thOld);
		N->threshSC[i] = ap * N->threshMaxSC + (!ap) * (th);
	}
	for (uint32_t i = tid; i < numMF; i += nThr) {
		const uint32_t m = spikeBit(sMF, i);
		N->histMF[i] = N->histMF[i] || (m > 0);
		N->apBufMF[i] = (N->apBufMF[i] << 1) | (m * 0x00000001u);
	}
	__syncthreads();
	for (uint32_t i = tid; i < numBC; i += nThr) N->bcCount[(size_t)R * numBC + i] = 0;
	for (uint32_t i = tid; i < numSC; i += nThr) N->scCount[(size_t)R * numSC + i] = 0;

	// ---- phase 2: calcIOActivities (mzone.cpp:258-339) element-parallel,
	// calcNCActivities (mzone.cpp:341-407) one warp per NC
	for (uint32_t task = tid; task < Z * numIO * nIONC; task += nThr) {
		const uint32_t z = task / (numIO * nIONC), k = task % (numIO * nIONC);
		const DevZone &Q = N->zones[z];
		float g = Q.gNCIO[k];
		g = g * cbmExpf(-N->msPerTimeStep / (-N->gDecTSofNCtoIO * cbmExpf(-g / N->gDecTTofNCtoIO) + N->gDecT0ofNCtoIO));
		g = g + Q.inputNCIO[k] * N->gIncNCtoIO * cbmExpf(-g / N->gIncTauNCtoIO);
		Q.gNCIO[k] = g;
		Q.inputNCIO[k] = 0;
		ioScratch[task] = g;
	}
	for (uint32_t task = warp; task < Z * numNC; task += nWarps) {
		const uint32_t z = task / numNC, i = task % numNC;
		const DevZone &Q = N->zones[z];
		float *sN = ncScratch + (size_t)task * 2 * nMFNC;
		for (uint32_t j = lane; j < nMFNC; j += 32) {
			const size_t k = (size_t)i * nMFNC + j;
			const float in = Q.inputMFNC[k], wt = Q.mfSynWeightNC[k];
			float gmN = Q.gmaxNMDAofMFtoNC[k];
			gmN = gmN * N->gmaxNMDADecMFtoNC + in * wt * (1 - gmN);
			Q.gmaxNMDAofMFtoNC[k] = gmN;
			float gN = Q.gMFNMDANC[k];
			gN = gN + N->gNMDAIncMFtoNC * (gmN - gN);
			Q.gMFNMDANC[k] = gN;
			float gmA = Q.gmaxAMPAofMFtoNC[k];
			gmA = gmA * N->gmaxAMPADecMFtoNC + in * wt * (1 - gmA);
			Q.gmaxAMPAofMFtoNC[k] = gmA;
			float gA = Q.gMFAMPANC[k];
			gA = gA + N->gAMPAIncMFtoNC * (gmA - gA);
			Q.gMFAMPANC[k] = gA;
			sN[j] = gN;
			sN[nMFNC + j] = gA;
		}
		float gPCNCSum = 0;
		for (uint32_t j0 = 0; j0 < N->numpNCfromPCtoNC; j0 += 32) {
			const uint32_t j = j0 + lane;
			float g = 0;
			if (j < N->numpNCfromPCtoNC) {
				const size_t k = (size_t)i * N->numpNCfromPCtoNC + j;
				g = Q.gPCNC[k] * N->gDecPCtoNC + Q.inputPCNC[k] * Q.gPCScaleNC[k] * (1 - Q.gPCNC[k]);
				Q.gPCNC[k] = g;
			}
			const uint32_t n = min(32u, N->numpNCfromPCtoNC - j0);
			for (uint32_t q = 0; q < n; q++) gPCNCSum = gPCNCSum + __shfl_sync(0xffffffffu, g, q);
		}
		__syncwarp();
		float partial = 0;
		if (lane < 2) {
			const float *src = sN + lane * nMFNC;
			for (uint32_t j = 0; j < nMFNC; j++) partial = partial + src[j];
		}
		const float ampaSum = __shfl_sync(0xffffffffu, partial, 1);
		if (lane == 0) {
			float gMFNMDASum = partial, gMFAMPASum = ampaSum;
			gMFNMDASum = gMFNMDASum * N->msPerTimeStep / ((float)nMFNC);
			gMFAMPASum = gMFAMPASum * N->msPerTimeStep / ((float)nMFNC);
			float vNC = Q.vNC[i];
			gMFNMDASum = gMFNMDASum * vNC / (-80.0f);
			gPCNCSum = gPCNCSum * N->msPerTimeStep / ((float)N->numpNCfromPCtoNC);
			vNC = vNC + N->gLeakNC * (N->eLeakNC - vNC) - (gMFNMDASum + gMFAMPASum) * vNC + gPCNCSum * (N->ePCtoNC - vNC);
			Q.vNC[i] = vNC;
			float th = Q.threshNC[i] + N->threshDecNC * (N->threshRestNC - Q.threshNC[i]);
			const uint8_t ap = vNC > th;
			Q.apNC[i] = ap;
			Q.apBufNC[i] = (Q.apBufNC[i] << 1) | (ap * 0x00000001u);
			Q.threshNC[i] = ap * N->threshMaxNC + (!ap) * th;
		}
	}
	__syncthreads();
	for (uint32_t task = tid; task < Z * numIO; task += nThr) {
		const uint32_t z = task / numIO, i = task % numIO;
		const DevZone &Q = N->zones[z];
		float gNCSum = 0;
		for (uint32_t j = 0; j < nIONC; j++) gNCSum = gNCSum + ioScratch[(size_t)task * nIONC + j];
		gNCSum = gNCSum / 3.1;
		float v = Q.vIO[i];
		v = v + N->gLeakIO * (N->eLeakIO - v) + gNCSum * 1.5 * (N->eNCtoIO - v) + Q.vCoupleIO[i] + ctl->errDrive[z];
		Q.vIO[i] = v;
		const uint8_t ap = v > Q.threshIO[i];
		Q.apIO[i] = ap;
		Q.apBufIO[i] = (Q.apBufIO[i] << 1) | (ap * 0x00000001u);
		Q.threshIO[i] = N->threshMaxIO * ap + (!ap) * (Q.threshIO[i] + N->threshDecIO * (N->threshRestIO - Q.threshIO[i]));
	}
	__syncthreads();

	// ---- microzone outputs (mzone.cpp:409-524)
	for (uint32_t task = tid; task < Z * numNC * nMFNC; task += nThr) {
		const uint32_t z = task / (numNC * nMFNC), k = task % (numNC * nMFNC);
		const uint32_t src = N->zones[z].pNCfromMFtoNC[k];
		N->zones[z].inputMFNC[k] = mfRaw ? mfRaw[src] : (uint8_t)spikeBit(sMF, src);
	}
	for (uint32_t task = tid; task < Z * numPC; task += nThr) {
		const uint32_t z = task / numPC, i = task % numPC;
		const DevZone &Q = N->zones[z];
		uint32_t c = 0;
		for (uint32_t e = Q.bcpcStart[i]; e < Q.bcpcStart[i + 1]; e++) c += Q.apBC[Q.bcpcSrc[e]];
		Q.inputBCPC[i] = c;
	}
	for (uint32_t task = tid; task < Z * numPC * N->numpPCfromSCtoPC; task += nThr) {
		const uint32_t per = numPC * N->numpPCfromSCtoPC;
		const uint32_t z = task / per, k = task % per;
		N->zones[z].inputSCPC[k] = sApSC[N->zones[z].pPCfromSCtoPC[k]];
	}
	for (uint32_t task = tid; task < Z * numBC; task += nThr) {
		const uint32_t z = task / numBC, i = task % numBC;
		const DevZone &Q = N->zones[z];
		uint32_t c = 0;
		for (uint32_t e = Q.pcbcStart[i]; e < Q.pcbcStart[i + 1]; e++) c += Q.apPC[Q.pcbcSrc[e]];
		Q.inputPCBC[i] = c;
	}
	for (uint32_t task = tid; task < Z * numNC * N->numpNCfromPCtoNC; task += nThr) {
		const uint32_t per = numNC * N->numpNCfromPCtoNC;
		const uint32_t z = task / per, k = task % per;
		N->zones[z].inputPCNC[k] = N->zones[z].apPC[N->zones[z].pNCfromPCtoNC[k]];
	}
	for (uint32_t task = tid; task < Z * numIO; task += nThr) {
		const uint32_t z = task / numIO, i = task % numIO;
		const DevZone &Q = N->zones[z];
		const uint8_t ap = Q.apIO[i];
		Q.pfPCPlastTimerIO[i] = (!ap) * (Q.pfPCPlastTimerIO[i] + 1) + ap * N->tsLTDStartAPIO;
		float vc = 0;
		for (uint32_t j = 0; j < N->numpIOInIOIO; j++)
			vc = vc + N->coupleRiRjRatioIO * (Q.vIO[Q.pIOInIOIO[(size_t)i * N->numpIOInIOIO + j]] - Q.vIO[i]);
		Q.vCoupleIO[i] = vc;
	}
	for (uint32_t task = tid; task < Z * numNC; task += nThr) {
		const uint32_t z = task / numNC, i = task % numNC;
		const DevZone &Q = N->zones[z];
		float p = Q.synIOPReleaseNC[i];
		p = p * cbmExpf(-N->msPerTimeStep / (N->relPDecTSofNCtoIO * cbmExpf(-p / N->relPDecTTofNCtoIO) + N->relPDecT0ofNCtoIO));
		p = p + Q.apNC[i] * N->relPIncNCtoIO * cbmExpf(-p / N->relPIncTauNCtoIO);
		Q.synIOPReleaseNC[i] = p;
	}
	const bool popStep = (t % N->tsPerPopHistBinPC) == 0;
	if (tid < Z) {
		const DevZone &Q = N->zones[tid];
		int doLTD = 0, doLTP = 0;
		if (popStep) {
			// updateMFNCSyn bookkeeping (mzone.cpp:536-580)
			uint32_t *s = Q.scal;
			s[0] = s[0] - Q.histPCPopAct[s[1]] + s[2];
			Q.histPCPopAct[s[1]] = s[2];
			s[2] = 0;
			s[1] = (s[1] + 1) % N->numPopHistBinsPC;
			const float avgAllAPPC = ((float)s[0]) / N->numPopHistBinsPC;
			if (avgAllAPPC >= N->synLTDPCPopActThreshMFtoNC && !s[4]) { doLTD = 1; s[4] = 1; }
			else if (avgAllAPPC < N->synLTDPCPopActThreshMFtoNC) s[4] = 0;
			if (avgAllAPPC <= N->synLTPPCPopActThreshMFtoNC && !s[3]) { doLTP = 1; s[3] = 1; }
			else if (avgAllAPPC > N->synLTPPCPopActThreshMFtoNC) s[3] = 0;
		}
		sFlags[2 * tid] = doLTD;
		sFlags[2 * tid + 1] = doLTP;
	}
	__syncthreads();

	// NC->IO release draws (mzone.cpp:505-511), MF->NC plasticity
	// (mzone.cpp:586-600), plasticity selector of the next step
	for (uint32_t task = tid; task < Z * numIO * nIONC; task += nThr) {
		const uint32_t per = numIO * nIONC;
		const uint32_t z = task / per, k = task % per;
		const uint32_t i = k / nIONC, j = k % nIONC;
		const DevZone &Q = N->zones[z];
		const double u = (double)rng::uniform24Keyed(Q.ncioKey, rng::ncioCounter(t, i, j, nIONC));
		Q.inputNCIO[k] = (u < Q.synIOPReleaseNC[Q.pIOfromNCtoIO[k]]);
	}
	if (popStep) {
		for (uint32_t task = tid; task < Z * numNC * nMFNC; task += nThr) {
			const uint32_t z = task / (numNC * nMFNC), k = task % (numNC * nMFNC);
			const DevZone &Q = N->zones[z];
			const int doLTD = sFlags[2 * z], doLTP = sFlags[2 * z + 1];
			const float synWDelta = N->histMF[Q.pNCfromMFtoNC[k]] *
				(doLTD * N->synLTDStepSizeMFtoNC + doLTP * N->synLTPStepSizeMFtoNC);
			float w = Q.mfSynWeightNC[k];
			w = w + synWDelta;
			w = (w > 0) * w;
			w = (w <= 1) * w + (w > 1);
			Q.mfSynWeightNC[k] = w;
		}
	}
	const bool nextPlast = ((t + 1) % N->tsPerHistBinGR) == 0;
	for (uint32_t task = tid; task < Z * numIO; task += nThr) {
		const uint32_t z = task / numIO, i = task % numIO;
		const DevZone &Q = N->zones[z];
		uint8_t sel = 0;
		if (nextPlast) {
			const int32_t tm = Q.pfPCPlastTimerIO[i];
			sel = tm < N->tsLTDEndIO ? 1 : (tm > N->tsLTPStartAPIO ? 2 : 0);
		}
		Q.plastSel[((t + 1) & 1) * numIO + i] = sel;
	}
	__syncthreads();
	if ((t % N->numTSinMFHist) == 0)
		for (uint32_t i = tid; i < numMF; i += nThr) N->histMF[i] = 0;
	if (tid < Z) ctl->errDrive[tid] = 0;
}

// Small-cell update of step t: block 2n is network n's Golgi role, block
// 2n+1 its microzone role.  The two roles share no state.
__global__ void __launch_bounds__(kTailThreads) tailKernel(const DevNet *const *nets, uint32_t stepOffset)
{
	const DevNet *__restrict__ N = nets[blockIdx.x >> 1];
	const uint64_t t = *N->tBase + 1 + stepOffset;
	extern __shared__ uint32_t tailSmem[];
	if (blockIdx.x & 1) zoneRole(N, t, tailSmem);
	else golgiRole(N, t, tailSmem);
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

}  // namespace cbm
