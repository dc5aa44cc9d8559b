// GR pass, vector form: the granule-cell step of one network with four
// consecutive cells per lane and dynamic work claiming.
//
// The per-cell arithmetic is the reference's (calcActivityGRGPU and
// updateGRInOPGPU, CBM_CORE_LIB_MGPU_DEV/src/cuda/kernels.cu:79-110 and
// 169-199; updateGRGOOutGPU / sumGRGOOutGPU :112-167; updatePFBCSCOutGPU
// :247-260; updatePFPCOutGPU :262-272; updateGRHistory :241-246;
// updatePFPCSynIO :282-291), in the same operation order as the per-tile TMA
// pass in cbm_kernels.cu.  What differs is how the work is cut:
//
//  * A unit is one pair of reduction rows (rows 2k and 2k+1 of a PC's
//    [2K][bs] block, the two terms x[i] and x[i+bs] of sumInputsNew's step k,
//    kernels.cu:326-362) times 64 consecutive values of the reduction index
//    j: 128 cells.  Lanes 0-15 take row 2k and lanes 16-31 row 2k+1, four
//    cells each, so every state array moves as one 16-byte load and one
//    16-byte store per lane, and each index plane as one 8-byte load.
//  * The CTAs are persistent (as many as fit on the GPU) and every warp
//    claims units from a counter, two at a time, so that every SM stays busy
//    to the end whatever the number of units, and CTAs that start late (the
//    small-cell kernel holds two SMs) simply claim fewer.
//  * The PF->PC reduction is split at its pair sums: a unit stores
//    x[i] + x[i+bs] for its 64 j (one value per pair, pairSum), and the
//    running sum over k (tempSum += x[i] + x[i+bs] in ascending k) of every
//    (PC, j) is taken in order at the start of the next step's pass, when all
//    pair sums of the step are in memory.  The float order is the
//    reference's, and no CTA waits for another.  The small-cell update reads
//    the sums two steps after the pass that made them (the reference's
//    lag), so taking them one pass later costs no latency.
//
// Scope: single networks whose shape is compiled in (4 MF and 3 GO
// dendrites, 4 GR->GO slots in the 16-bit table, one microzone), with a
// reduction width bs that is a multiple of 64 and BC / SC blocks of at least
// 64 cells (passVecCapable).  Other networks run the per-tile pass.
#include <cstdint>
#include <cuda_runtime.h>

#include "cbm_device.cuh"
#include "cbm_kernels.cuh"

namespace cbm {

namespace {

constexpr uint32_t kMF = 4, kGO = 3, kOut = 4;  // slot planes of the compiled shape

__device__ __forceinline__ uint32_t half16(uint2 w, uint32_t c)
{
	const uint32_t x = c < 2 ? w.x : w.y;
	return (c & 1u) ? (x >> 16) : (x & 0xFFFFu);
}

// sumInputsNew's halving tree (kernels.cu:326-362) over the bs values in
// sTree: strides bs/2 ... 1, thread i adding i + stride.  Strides of 32 and
// more are shared-memory levels of the block, the last five a warp's
// shuffles; thread 0 gets the sum.  Every thread of the block calls it.
__device__ float blockRowTree(float *sTree, uint32_t bs)
{
	__syncthreads();
	for (uint32_t h = bs / 2; h >= 32; h /= 2) {
		if (threadIdx.x < h) sTree[threadIdx.x] = sTree[threadIdx.x] + sTree[threadIdx.x + h];
		__syncthreads();
	}
	float v = 0.0f;
	if (threadIdx.x < 32) {
		v = sTree[threadIdx.x];
		v = v + __shfl_down_sync(0xffffffffu, v, 16);
		v = v + __shfl_down_sync(0xffffffffu, v, 8);
		v = v + __shfl_down_sync(0xffffffffu, v, 4);
		v = v + __shfl_down_sync(0xffffffffu, v, 2);
		v = v + __shfl_down_sync(0xffffffffu, v, 1);
	}
	return v;
}

// The network n with offset[n] <= g < offset[n + 1] (offset sorted), and g's
// index within it.
__device__ __forceinline__ int findNet(const uint32_t *offset, int numNets, uint32_t g, uint32_t &local)
{
	int lo = 0, hi = numNets - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (offset[mid] <= g) lo = mid; else hi = mid - 1;
	}
	local = g - offset[lo];
	return lo;
}

__device__ __forceinline__ float4 ldState(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void stState(float *p, float a, float b, float c, float d)
{
	*reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}

}  // namespace

// The per-network values a unit needs.
struct VecNet {
	float gLeak, eLeak, eGOIn, threshBase, threshMax, threshDecay, gDecMF, gIncMF, gDecGO, gIncGO;
	uint32_t numGR, P, bs, K, bcShift, scShift, jGroups;
	uint32_t *goCount;
	float *vGR, *gKCaGR, *threshGR, *gESum, *gISum, *wGR, *pairOut;
	uint32_t *apBufGR;
	uint64_t *historyGR;
	const uint16_t *mfIdx, *goIdx, *out16;
	const uint8_t *pfDelay;
};

__device__ __forceinline__ VecNet vecNet(const DevNet *N, uint64_t t)
{
	VecNet c;
	c.gLeak = N->gLeakGR; c.eLeak = N->eLeakGR; c.eGOIn = N->eGOGR;
	c.threshBase = N->threshRestGR; c.threshMax = N->threshMaxGR; c.threshDecay = N->threshDecGR;
	c.gDecMF = N->gDecMFtoGR; c.gIncMF = N->gIncMFtoGR; c.gDecGO = N->gDecGOtoGR; c.gIncGO = N->gIncGOtoGR;
	c.numGR = N->numGR; c.P = N->P; c.bs = N->bs; c.K = N->K;
	c.bcShift = N->bcShift; c.scShift = N->scShift; c.jGroups = N->bs / 64u;
	c.goCount = N->goCount + (size_t)(t & 1) * N->numGO;
	c.vGR = N->vGR; c.gKCaGR = N->gKCaGR; c.threshGR = N->threshGR; c.gESum = N->gESum; c.gISum = N->gISum;
	c.wGR = N->zones[0].w;
	c.pairOut = N->zones[0].pairSum + (size_t)(t & 1) * N->numPC * N->K * N->bs;
	c.apBufGR = N->apBufGR; c.historyGR = N->historyGR;
	c.mfIdx = N->mfIdx; c.goIdx = N->goIdx; c.out16 = N->outCon16; c.pfDelay = N->pfDelay;
	return c;
}

// Spike lookups from shared-memory byte tables (a single network).
struct SpikeBytes {
	const uint8_t *mfT, *goT;
	__device__ __forceinline__ int mf(uint32_t i) const { return mfT[i]; }
	__device__ __forceinline__ int go(uint32_t i) const { return goT[i]; }
};
// Spike lookups from the spike bit words in global memory (a batch: every
// network has its own, read through the L1 cache).
struct SpikeBits {
	const uint32_t *mfW, *goW;
	__device__ __forceinline__ int mf(uint32_t i) const { return (__ldg(mfW + (i >> 5)) >> (i & 31u)) & 1u; }
	__device__ __forceinline__ int go(uint32_t i) const { return (__ldg(goW + (i >> 5)) >> (i & 31u)) & 1u; }
};

// One unit u (128 cells) of a network at step t: every cell's update, its
// pair sums, its PF->BC/SC counts (into bcCnt / scCnt, indexed by the
// network's BC and SC numbers) and its GR->GO deliveries.
template <class Spikes, class StepOf>
__device__ __forceinline__ void vecUnit(const VecNet &n, bool plastStep, uint32_t u, uint32_t lane, const Spikes &sp,
		const StepOf &stepOf, uint32_t *bcCnt, uint32_t *scCnt)
{
	const float gLeak = n.gLeak, eLeak = n.eLeak, eGOIn = n.eGOIn;
	const float threshBase = n.threshBase, threshMax = n.threshMax, threshDecay = n.threshDecay;
	const float gDecMF = n.gDecMF, gIncMF = n.gIncMF, gDecGO = n.gDecGO, gIncGO = n.gIncGO;
	const uint32_t numGR = n.numGR, P = n.P, bs = n.bs, K = n.K, jGroups = n.jGroups;
	const uint32_t bcShift = n.bcShift, scShift = n.scShift;
	uint32_t *const goCount = n.goCount;
	float *const vGR = n.vGR, *const gKCaGR = n.gKCaGR, *const threshGR = n.threshGR;
	float *const gESum = n.gESum, *const gISum = n.gISum, *const wGR = n.wGR, *const pairOut = n.pairOut;
	uint32_t *const apBufGR = n.apBufGR;
	uint64_t *const historyGR = n.historyGR;
	const uint16_t *const mfIdx = n.mfIdx, *const goIdx = n.goIdx, *const out16 = n.out16;
	const uint8_t *const pfDelay = n.pfDelay;
	const uint32_t h = lane >> 4, l = lane & 15u;
	const uint32_t jg = u % jGroups, pk = u / jGroups, k = pk % K, pc = pk / K;
	const uint32_t rowStart = pc * P + (2u * k + h) * bs + jg * 64u;
	const uint32_t g = rowStart + 4u * l;  // this lane's first cell

	const float4 v4 = ldState(vGR + g), gk4 = ldState(gKCaGR + g), th4 = ldState(threshGR + g);
	const float4 gE4 = ldState(gESum + g), gI4 = ldState(gISum + g);
	const uint4 ab4 = *reinterpret_cast<const uint4 *>(apBufGR + g);
	uint2 mfw[kMF], gow[kGO];
#pragma unroll
	for (uint32_t s = 0; s < kMF; s++) mfw[s] = __ldg(reinterpret_cast<const uint2 *>(mfIdx + (size_t)s * numGR + g));
#pragma unroll
	for (uint32_t s = 0; s < kGO; s++) gow[s] = __ldg(reinterpret_cast<const uint2 *>(goIdx + (size_t)s * numGR + g));
	const uint32_t dly = __ldg(reinterpret_cast<const uint32_t *>(pfDelay + g));
	// the GR->GO slot words on their way to L2 with the rest (most warps
	// have a lane with a spike in its 32-step buffer and read them below)
#pragma unroll
	for (uint32_t s = 0; s < kOut; s++) asm volatile("prefetch.global.L2 [%0];" ::"l"(out16 + (size_t)s * numGR + g));
	const float4 w4 = ldState(wGR + g);
	ulonglong2 hA = make_ulonglong2(0, 0), hB = make_ulonglong2(0, 0);
	if (plastStep) {
		hA = *reinterpret_cast<const ulonglong2 *>(historyGR + g);
		hB = *reinterpret_cast<const ulonglong2 *>(historyGR + g + 2);
	}
	const float vIn[4] = {v4.x, v4.y, v4.z, v4.w}, gkIn[4] = {gk4.x, gk4.y, gk4.z, gk4.w};
	const float thIn[4] = {th4.x, th4.y, th4.z, th4.w}, gEIn[4] = {gE4.x, gE4.y, gE4.z, gE4.w};
	const float gIIn[4] = {gI4.x, gI4.y, gI4.z, gI4.w}, wIn[4] = {w4.x, w4.y, w4.z, w4.w};
	const uint32_t abIn[4] = {ab4.x, ab4.y, ab4.z, ab4.w};
	const uint64_t hIn[4] = {hA.x, hA.y, hB.x, hB.y};
	const float stepW = plastStep ? stepOf(pc) : 0.0f;

	float vO[4], gkO[4], thO[4], gEO[4], gIO[4], wO[4], x[4];
	uint32_t abO[4], pfCount = 0, anySpike = 0;
	uint64_t hO[4];
#pragma unroll
	for (uint32_t c = 0; c < 4; c++) {
		int cntMF = 0, cntGO = 0;
#pragma unroll
		for (uint32_t s = 0; s < kMF; s++) cntMF += sp.mf(half16(mfw[s], c));
#pragma unroll
		for (uint32_t s = 0; s < kGO; s++) cntGO += sp.go(half16(gow[s], c));
		const float v = vIn[c], gk = gkIn[c], th = thIn[c], gE = gEIn[c], gI = gIIn[c];
		// calcActivityGRGPU (kernels.cu:79-110)
		const float tempV = v + (gLeak + gk * gk * gk * gk) * (eLeak - v) - (gE) * v + (gI) * (eGOIn - v);
		const float tempThresh = th + (threshBase - th) * threshDecay;
		const unsigned int tempAP = tempV > tempThresh;
		thO[c] = tempAP * threshMax + (!tempAP) * tempThresh;
		const float gkd = gk * 0.9999f;
		gkO[c] = tempAP * (gkd + 0.003f) + (!tempAP) * gkd;
		const uint32_t abN = (abIn[c] << 1) | tempAP;
		abO[c] = abN;
		anySpike |= abN;
		vO[c] = tempV;
		// updateGRInOPGPU for MF (this step's spikes) and GO (last step's)
		gEO[c] = gE * gDecMF + gIncMF * (cntMF);
		gIO[c] = gI * gDecGO + gIncGO * (cntGO);
		// plasticity (phase 1) before this step's PF->PC output (phase 2)
		const uint32_t d = (dly >> (8u * c)) & 0xFFu;
		const uint32_t pf = d < 32u ? (abN >> d) & 1u : 0u;
		pfCount += pf;
		float w = wIn[c];
		if (plastStep) {
			w = w + ((hIn[c] & 0x0000008000000000ull) > 0) * stepW;
			w = (w > 0) * w;
			w = (w > 1) + (w <= 1) * w;
			hO[c] = (hIn[c] << 1) | ((abN & 0x0000001Fu) > 0);
		}
		wO[c] = w;
		x[c] = w * pf;
	}
	stState(vGR + g, vO[0], vO[1], vO[2], vO[3]);
	stState(gKCaGR + g, gkO[0], gkO[1], gkO[2], gkO[3]);
	stState(threshGR + g, thO[0], thO[1], thO[2], thO[3]);
	stState(gESum + g, gEO[0], gEO[1], gEO[2], gEO[3]);
	stState(gISum + g, gIO[0], gIO[1], gIO[2], gIO[3]);
	*reinterpret_cast<uint4 *>(apBufGR + g) = make_uint4(abO[0], abO[1], abO[2], abO[3]);
	if (plastStep) {
		stState(wGR + g, wO[0], wO[1], wO[2], wO[3]);
		*reinterpret_cast<ulonglong2 *>(historyGR + g) = make_ulonglong2(hO[0], hO[1]);
		*reinterpret_cast<ulonglong2 *>(historyGR + g + 2) = make_ulonglong2(hO[2], hO[3]);
	}
	// pair sums x[i] + x[i+bs]: row 2k's lane takes row 2k+1's values
	float q[4];
#pragma unroll
	for (uint32_t c = 0; c < 4; c++) q[c] = x[c] + __shfl_xor_sync(0xffffffffu, x[c], 16);
	if (h == 0) stState(pairOut + ((size_t)pc * K + k) * bs + jg * 64u + 4u * l, q[0], q[1], q[2], q[3]);
	// PF->BC and PF->SC counts of the 64 cells of each half (one BC and
	// one SC block each)
	pfCount += __shfl_xor_sync(0xffffffffu, pfCount, 8);
	pfCount += __shfl_xor_sync(0xffffffffu, pfCount, 4);
	pfCount += __shfl_xor_sync(0xffffffffu, pfCount, 2);
	pfCount += __shfl_xor_sync(0xffffffffu, pfCount, 1);
	if (l == 0 && pfCount) {
		atomicAdd(&bcCnt[rowStart >> bcShift], pfCount);
		atomicAdd(&scCnt[rowStart >> scShift], pfCount);
	}
	// GR->GO synapses whose delayed spike arrives now (lanes with a spike in
	// their buffers)
	if (anySpike) {
		uint2 ow[kOut];
#pragma unroll
		for (uint32_t s = 0; s < kOut; s++) ow[s] = __ldg(reinterpret_cast<const uint2 *>(out16 + (size_t)s * numGR + g));
#pragma unroll
		for (uint32_t c = 0; c < 4; c++) {
			if (!abO[c]) continue;
#pragma unroll
			for (uint32_t s = 0; s < kOut; s++) {
				const uint32_t o = half16(ow[s], c);
				if (o != kOut16None && ((abO[c] >> (o & 31u)) & 1u)) atomicAdd(&goCount[o >> 5], 1u);
			}
		}
	}
}

// Step t-1's PF->PC reduction, one (PC, 64-j chunk) task per warp: lanes
// take two consecutive j each, the running sums over k, in ascending k, of
// the stored pair sums (the reference's tempSum += x[i] + x[i+bs],
// kernels.cu:326-362), kept as the partial sums; the warp that completes a
// PC's last chunk (a counter per PC) then takes the halving tree over the
// PC's bs partial sums in registers (lane l holds partials l + 32 m, so every
// level of stride 32 or more pairs values of one lane) and stores the PC's
// input sum.
__device__ void reduceChunk(const DevNet *__restrict__ N, uint64_t t, uint32_t task, uint32_t lane)
{
	const uint32_t numPC = N->numPC, bs = N->bs, K = N->K;
	const uint32_t chunks = bs / 64u, pc = task / chunks, j = (task % chunks) * 64u + 2u * lane;
	const DevZone &Z0 = N->zones[0];
	const float *src = Z0.pairSum + (size_t)((t - 1) & 1) * numPC * K * bs + (size_t)pc * K * bs + j;
	float *part = Z0.pcPartial + (size_t)((t - 1) % 3) * numPC * bs + (size_t)pc * bs;
	float a0 = 0.0f, a1 = 0.0f;
	for (uint32_t k0 = 0; k0 < K; k0 += 16) {
		float2 q[16];
#pragma unroll
		for (uint32_t u = 0; u < 16; u++)
			q[u] = k0 + u < K ? __ldcg(reinterpret_cast<const float2 *>(src + (size_t)(k0 + u) * bs))
				: make_float2(0.0f, 0.0f);
#pragma unroll
		for (uint32_t u = 0; u < 16; u++)
			if (k0 + u < K) { a0 += q[u].x; a1 += q[u].y; }
	}
	*reinterpret_cast<float2 *>(part + j) = make_float2(a0, a1);
	__threadfence();
	uint32_t prev = 0;
	if (lane == 0) prev = atomicAdd(&N->pcDone[pc], 1u);
	prev = __shfl_sync(0xffffffffu, prev, 0);
	if (prev != chunks - 1) return;
	__threadfence();
	const uint32_t m = bs / 32u;  // partials per lane: 2, 4, 8 or 16
	float v[16];
#pragma unroll
	for (uint32_t i = 0; i < 16; i++) v[i] = i < m ? __ldcg(part + 32u * i + lane) : 0.0f;
#pragma unroll
	for (uint32_t hm = 8; hm >= 1; hm /= 2) {
		if (2u * hm <= m) {
#pragma unroll
			for (uint32_t i = 0; i < hm; i++) v[i] = v[i] + v[i + hm];
		}
	}
	float x = v[0];
	x = x + __shfl_down_sync(0xffffffffu, x, 16);
	x = x + __shfl_down_sync(0xffffffffu, x, 8);
	x = x + __shfl_down_sync(0xffffffffu, x, 4);
	x = x + __shfl_down_sync(0xffffffffu, x, 2);
	x = x + __shfl_down_sync(0xffffffffu, x, 1);
	if (lane == 0) {
		Z0.pcSum[(size_t)((t - 1) % 3) * numPC + pc] = x;
		N->pcDone[pc] = 0;  // for the next step's pass
	}
}

// CTAs of the vector pass that take step t-1's reduction (the first ones of
// the grid, one task per warp); the others take units.
__host__ __device__ __forceinline__ uint32_t vecReduceCTAs(uint32_t numPC, uint32_t bs)
{
	return (numPC * (bs / 64u) + kVecWarps - 1) / kVecWarps;
}

__global__ void __launch_bounds__(32 * kVecWarps, kVecMinBlocks) grPassVecKernel(const DevNet *__restrict__ N,
		uint32_t stepOffset, uint32_t claimSize)
{
	const uint64_t t = stepsDone(N) + 1 + stepOffset;
	const uint32_t numGR = N->numGR, numPC = N->numPC, bs = N->bs;
	const uint32_t lane = threadIdx.x & 31u;

	// the reduction CTAs: one task per warp, then done (their slots go to
	// the unit CTAs that did not fit at launch)
	const uint32_t redCTAs = vecReduceCTAs(numPC, bs);
	if (blockIdx.x < redCTAs) {
		const uint32_t task = blockIdx.x * kVecWarps + (threadIdx.x >> 5);
		if (task < numPC * (bs / 64u) && N->pairStep[(t - 1) & 1] == t - 1) reduceChunk(N, t, task, lane);
		return;
	}
	const uint32_t cta = blockIdx.x - redCTAs;

	extern __shared__ __align__(16) uint8_t vecSmem[];
	const uint32_t mfWords = N->mfWords, goWords = N->goWords;
	uint8_t *sMF = vecSmem;                       // this step's MF spikes, a byte per fibre
	uint8_t *sGO = sMF + 32u * mfWords;           // last step's GO spikes, a byte per cell
	float *sStep = reinterpret_cast<float *>(sGO + ((32u * goWords + 15u) & ~15u));  // PF->PC step per PC

	const bool plastStep = stepMod(t, N->tsPerHistBinGR) == 0;

	// ---- prologue: spike tables, plasticity steps, counters
	{
		const uint32_t *mfSrc = N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * mfWords;
		const uint32_t *goSrc = N->goBits + (size_t)((t - 1) & 1) * goWords;
		const uint32_t nWords = mfWords + goWords;
		for (uint32_t w = threadIdx.x; w < nWords; w += blockDim.x) {
			const uint32_t v = __ldg(w < mfWords ? mfSrc + w : goSrc + (w - mfWords));
			uint4 *dst = reinterpret_cast<uint4 *>(w < mfWords ? sMF + 32u * w : sGO + 32u * (w - mfWords));
			uint32_t q[8];
			// bit k of each nibble to bit 8k: (nibble * 0x204081) & 0x01010101
#pragma unroll
			for (int k = 0; k < 8; k++) q[k] = (((v >> (4 * k)) & 0xFu) * 0x00204081u) & 0x01010101u;
			dst[0] = make_uint4(q[0], q[1], q[2], q[3]);
			dst[1] = make_uint4(q[4], q[5], q[6], q[7]);
		}
		const DevZone &Z0 = N->zones[0];
		for (uint32_t pc = threadIdx.x; pc < numPC; pc += blockDim.x) {
			float s = 0.0f;
			if (plastStep) s = plasticityStep(N, t, 0, Z0.plastSel[(t & 1) * N->numIO + Z0.ioOfPC[pc]]);
			sStep[pc] = s;
		}
		if (cta == 0 && threadIdx.x == 0) {
			N->passClaim[(t + 1) % 3] = 0;  // the next step's counter (last used two steps ago)
			N->pairStep[t & 1] = t;         // read by the next step's pass, after this one ends
		}
	}
	__syncthreads();

	// ---- units
	const VecNet net = vecNet(N, t);
	const SpikeBytes sp{sMF, sGO};
	const auto stepOf = [&](uint32_t pc) { return sStep[pc]; };
	uint32_t *const bcOut = N->bcCount + (size_t)(t % 3) * N->numBC;
	uint32_t *const scOut = N->scCount + (size_t)(t % 3) * N->numSC;
	const uint32_t U = numGR / 128u;
	uint32_t *const claim = N->passClaim + t % 3;
	uint32_t base = 0;
	if (lane == 0) base = atomicAdd(claim, claimSize);
	base = __shfl_sync(0xffffffffu, base, 0);
	while (base < U) {
		// the next claim's round trip overlaps this one's units
		uint32_t next = 0;
		if (lane == 0) next = atomicAdd(claim, claimSize);
		const uint32_t end = min(U, base + claimSize);
		for (uint32_t u = base; u < end; u++) vecUnit(net, plastStep, u, lane, sp, stepOf, bcOut, scOut);
		base = __shfl_sync(0xffffffffu, next, 0);
	}
}

// Step t-1's PF->PC reduction of one PC of network N (one CTA): the running
// sums over k in ascending k, kept as the partial sums, and the halving tree
// over j, kept as the PC's input sum.
__device__ void reducePC(const DevNet *N, uint64_t t, uint32_t pc, float *sTree)
{
	const uint32_t numPC = N->numPC, bs = N->bs, K = N->K;
	const DevZone &Z0 = N->zones[0];
	const float *pairs = Z0.pairSum + (size_t)((t - 1) & 1) * numPC * K * bs + (size_t)pc * K * bs;
	float *part = Z0.pcPartial + (size_t)((t - 1) % 3) * numPC * bs + (size_t)pc * bs;
	for (uint32_t j = threadIdx.x; j < bs; j += blockDim.x) {
		float a = 0.0f;
		for (uint32_t k0 = 0; k0 < K; k0 += 8) {
			float q[8];
#pragma unroll
			for (uint32_t u = 0; u < 8; u++) q[u] = k0 + u < K ? pairs[(size_t)(k0 + u) * bs + j] : 0.0f;
#pragma unroll
			for (uint32_t u = 0; u < 8; u++)
				if (k0 + u < K) a += q[u];
		}
		part[j] = a;
		sTree[j] = a;
	}
	const float sum = blockRowTree(sTree, bs);
	if (threadIdx.x == 0) Z0.pcSum[(size_t)((t - 1) % 3) * numPC + pc] = sum;
	__syncthreads();
}

// The vector pass over a batch of networks of the compiled shape: one
// persistent launch whose warps claim kVecBatchClaim units at a time from a
// counter over the units of every network (unitOffset[n] is network n's
// first unit, unitOffset[numNets] the total; pcOffset likewise over their
// PCs).  Spikes are looked up in each network's spike bit words, PF->BC/SC
// counts go to global memory, and each network's previous-step PF->PC
// reduction is spread over the CTAs, one PC each.
__global__ void __launch_bounds__(32 * kVecWarps, kVecBatchMinBlocks) grPassVecBatchKernel(const DevNet *const *nets,
		const uint32_t *unitOffset, const uint32_t *pcOffset, int numNets, uint32_t stepOffset, uint32_t *claimBase)
{
	__shared__ float sTree[512];
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t t0 = stepsDone(nets[0]) + 1 + stepOffset;
	if (blockIdx.x == 0) {
		if (threadIdx.x == 0) claimBase[(t0 + 1) % 3] = 0;  // the next step's counter
		for (int n = threadIdx.x; n < numNets; n += blockDim.x) {
			const DevNet *N = nets[n];
			const uint64_t t = stepsDone(N) + 1 + stepOffset;
			N->pairStep[t & 1] = t;
		}
	}
	// previous-step PF->PC reductions, one (network, PC) per CTA in turn
	for (uint32_t q = blockIdx.x; q < pcOffset[numNets]; q += gridDim.x) {
		uint32_t pc = 0;
		const DevNet *N = nets[findNet(pcOffset, numNets, q, pc)];
		const uint64_t t = stepsDone(N) + 1 + stepOffset;
		if (N->pairStep[(t - 1) & 1] == t - 1) reducePC(N, t, pc, sTree);
	}

	const uint32_t U = unitOffset[numNets];
	uint32_t *const claim = claimBase + t0 % 3;
	uint32_t base = 0;
	if (lane == 0) base = atomicAdd(claim, kVecBatchClaim);
	base = __shfl_sync(0xffffffffu, base, 0);
	// the current network's values per warp in shared memory (read by the
	// unit as it needs them, not held in registers across units)
	__shared__ VecNet sNets[kVecWarps];
	VecNet &net = sNets[threadIdx.x >> 5];
	int cur = -1;
	const DevNet *N = nullptr;
	uint64_t t = 0;
	bool plastStep = false;
	SpikeBits sp{nullptr, nullptr};
	uint32_t *bcCnt = nullptr, *scCnt = nullptr;
	while (base < U) {
		uint32_t next = 0;
		if (lane == 0) next = atomicAdd(claim, kVecBatchClaim);
		const uint32_t end = min(U, base + kVecBatchClaim);
		for (uint32_t g = base; g < end; g++) {
			uint32_t u = 0;
			const int lo = findNet(unitOffset, numNets, g, u);
			if (lo != cur) {
				cur = lo;
				N = nets[lo];
				t = stepsDone(N) + 1 + stepOffset;
				__syncwarp();
				if (lane == 0) net = vecNet(N, t);
				__syncwarp();
				plastStep = stepMod(t, N->tsPerHistBinGR) == 0;
				sp = SpikeBits{N->mfBits + (size_t)stepMod(t - 1, N->mfRing) * N->mfWords,
						N->goBits + (size_t)((t - 1) & 1) * N->goWords};
				bcCnt = N->bcCount + (size_t)(t % 3) * N->numBC;
				scCnt = N->scCount + (size_t)(t % 3) * N->numSC;
			}
			const DevNet *Nc = N;
			const uint64_t tc = t;
			const auto stepOf = [&](uint32_t pc) {
				const DevZone &Z0 = Nc->zones[0];
				return plasticityStep(Nc, tc, 0, Z0.plastSel[(tc & 1) * Nc->numIO + Z0.ioOfPC[pc]]);
			};
			vecUnit(net, plastStep, u, lane, sp, stepOf, bcCnt, scCnt);
		}
		base = __shfl_sync(0xffffffffu, next, 0);
	}
}

// The running sums of step t's pair sums into its partial-sum buffer, for a
// switch from the vector pass to a pass that does not take them itself.
__global__ void pairReduceKernel(const DevNet *__restrict__ N, uint64_t t)
{
	const uint32_t numPC = N->numPC, bs = N->bs, K = N->K, nSeq = numPC * bs;
	const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= nSeq || N->pairStep[t & 1] != t) return;
	const float *src = N->zones[0].pairSum + (size_t)(t & 1) * numPC * K * bs + (size_t)(c / bs) * K * bs + c % bs;
	float sum = 0.0f;
	for (uint32_t k = 0; k < K; k++) sum += src[(size_t)k * bs];
	N->zones[0].pcPartial[(size_t)(t % 3) * nSeq + c] = sum;
}

// Step t's PF->PC input sums from its partial sums (blockIdx.x = PC).
__global__ void pcTreeKernel(const DevNet *__restrict__ N, uint64_t t)
{
	__shared__ float sTree[512];
	const uint32_t numPC = N->numPC, bs = N->bs, pc = blockIdx.x;
	const float *part = N->zones[0].pcPartial + (size_t)(t % 3) * numPC * bs + (size_t)pc * bs;
	for (uint32_t j = threadIdx.x; j < bs; j += blockDim.x) sTree[j] = part[j];
	const float sum = blockRowTree(sTree, bs);
	if (threadIdx.x == 0) N->zones[0].pcSum[(size_t)(t % 3) * numPC + pc] = sum;
}

const void *passVecBatchKernel() { return (const void *)&grPassVecBatchKernel; }

bool passVecCapable(const DevNet &h)
{
	return passShapeOf(h) == 1 && h.numZones == 1 && h.bs >= 64 && h.bs % 64 == 0 && h.numGR % 128 == 0 &&
		(1u << h.bcShift) >= 64u && (1u << h.scShift) >= 64u && !h.ovStart && h.outCon16 &&
		h.P % (2 * h.bs) == 0;
}

size_t passVecSmemBytes(const DevNet &h)
{
	return 32u * h.mfWords + ((32u * h.goWords + 15u) & ~15u) + 4ull * h.numPC;
}

uint32_t passVecReduceCTAs(const DevNet &h) { return vecReduceCTAs(h.numPC, h.bs); }

const void *passVecKernel() { return (const void *)&grPassVecKernel; }
const void *pairReduceKernelFn() { return (const void *)&pairReduceKernel; }
const void *pcTreeKernelFn() { return (const void *)&pcTreeKernel; }

}  // namespace cbm
