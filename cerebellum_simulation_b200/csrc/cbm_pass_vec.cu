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

__device__ __forceinline__ float4 ldState(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void stState(float *p, float a, float b, float c, float d)
{
	*reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}

}  // namespace

__global__ void __launch_bounds__(32 * kVecWarps, kVecMinBlocks) grPassVecKernel(const DevNet *__restrict__ N,
		uint32_t stepOffset)
{
	const uint64_t t = stepsDone(N) + 1 + stepOffset;
	const uint32_t numGR = N->numGR, P = N->P, bs = N->bs, K = N->K, numPC = N->numPC;
	const uint32_t numBC = N->numBC, numSC = N->numSC;
	const uint32_t lane = threadIdx.x & 31u;

	extern __shared__ __align__(16) uint8_t vecSmem[];
	const uint32_t mfWords = N->mfWords, goWords = N->goWords;
	uint8_t *sMF = vecSmem;                       // this step's MF spikes, a byte per fibre
	uint8_t *sGO = sMF + 32u * mfWords;           // last step's GO spikes, a byte per cell
	float *sStep = reinterpret_cast<float *>(sGO + ((32u * goWords + 15u) & ~15u));  // PF->PC step per PC
	uint32_t *sBC = reinterpret_cast<uint32_t *>(sStep + numPC);                      // PF->BC counts
	uint32_t *sSC = sBC + numBC;                                                      // PF->SC counts
	float *sTree = reinterpret_cast<float *>(sSC + numSC);                            // one PC's bs partial sums

	const bool plastStep = (t % N->tsPerHistBinGR) == 0;

	// ---- prologue: spike tables, plasticity steps, counters
	{
		const uint32_t *mfSrc = N->mfBits + (size_t)((t - 1) % N->mfRing) * mfWords;
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
		for (uint32_t i = threadIdx.x; i < numBC + numSC; i += blockDim.x) sBC[i] = 0;
		if (blockIdx.x == 0 && threadIdx.x == 0) {
			N->passClaim[(t + 1) % 3] = 0;  // the next step's counter (last used two steps ago)
			N->pairStep[t & 1] = t;         // read by the next step's pass, after this one ends
		}
	}
	// Step t-1's PF->PC reduction, one PC per CTA (CTAs 0 .. numPC-1): the
	// running sum over k of every j in ascending k (tempSum += x[i] +
	// x[i+bs]), kept as the partial sums, then the halving tree over j, kept
	// as the PC's input sum for the small-cell update.
	if (N->pairStep[(t - 1) & 1] == t - 1) {
		const DevZone &Z0 = N->zones[0];
		const float *pairs = Z0.pairSum + (size_t)((t - 1) & 1) * numPC * K * bs;
		float *part = Z0.pcPartial + (size_t)((t - 1) % 3) * numPC * bs;
		for (uint32_t pc = blockIdx.x; pc < numPC; pc += gridDim.x) {
			for (uint32_t j0 = 0; j0 < bs; j0 += 2u * blockDim.x) {
				const uint32_t ja = j0 + threadIdx.x, jb = ja + blockDim.x;
				const float *sa = pairs + (size_t)pc * K * bs + ja, *sb = pairs + (size_t)pc * K * bs + jb;
				float a = 0.0f, b = 0.0f;
				for (uint32_t k0 = 0; k0 < K; k0 += 8) {
					float qa[8], qb[8];
#pragma unroll
					for (uint32_t u = 0; u < 8; u++) {
						const bool in = k0 + u < K;
						qa[u] = in && ja < bs ? sa[(size_t)(k0 + u) * bs] : 0.0f;
						qb[u] = in && jb < bs ? sb[(size_t)(k0 + u) * bs] : 0.0f;
					}
#pragma unroll
					for (uint32_t u = 0; u < 8; u++) {
						if (k0 + u < K) { a += qa[u]; b += qb[u]; }
					}
				}
				if (ja < bs) { part[(size_t)pc * bs + ja] = a; sTree[ja] = a; }
				if (jb < bs) { part[(size_t)pc * bs + jb] = b; sTree[jb] = b; }
			}
			const float sum = blockRowTree(sTree, bs);
			if (threadIdx.x == 0) {
				Z0.pcSum[(size_t)((t - 1) % 3) * numPC + pc] = sum;
			}
			__syncthreads();
		}
	}
	__syncthreads();

	// ---- units
	const float gLeak = N->gLeakGR, eLeak = N->eLeakGR, eGOIn = N->eGOGR;
	const float threshBase = N->threshRestGR, threshMax = N->threshMaxGR, threshDecay = N->threshDecGR;
	const float gDecMF = N->gDecMFtoGR, gIncMF = N->gIncMFtoGR, gDecGO = N->gDecGOtoGR, gIncGO = N->gIncGOtoGR;
	uint32_t *const goCount = N->goCount + (size_t)(t & 1) * N->numGO;
	float *const vGR = N->vGR, *const gKCaGR = N->gKCaGR, *const threshGR = N->threshGR;
	float *const gESum = N->gESum, *const gISum = N->gISum;
	uint32_t *const apBufGR = N->apBufGR;
	uint64_t *const historyGR = N->historyGR;
	float *const wGR = N->zones[0].w;
	float *const pairOut = N->zones[0].pairSum + (size_t)(t & 1) * numPC * K * bs;
	const uint16_t *const mfIdx = N->mfIdx, *const goIdx = N->goIdx, *const out16 = N->outCon16;
	const uint8_t *const pfDelay = N->pfDelay;
	const uint32_t bcShift = N->bcShift, scShift = N->scShift;
	const uint32_t jGroups = bs / 64u, U = numGR / 128u;
	const uint32_t h = lane >> 4, l = lane & 15u;
	uint32_t *const claim = N->passClaim + t % 3;

	uint32_t base = 0;
	if (lane == 0) base = atomicAdd(claim, kVecClaim);
	base = __shfl_sync(0xffffffffu, base, 0);
	while (base < U) {
		// the next claim's round trip overlaps this one's units
		uint32_t next = 0;
		if (lane == 0) next = atomicAdd(claim, kVecClaim);
		const uint32_t end = min(U, base + kVecClaim);
		for (uint32_t u = base; u < end; u++) {
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
			const float stepW = sStep[pc];

			float vO[4], gkO[4], thO[4], gEO[4], gIO[4], wO[4], x[4];
			uint32_t abO[4], pfCount = 0, anySpike = 0;
			uint64_t hO[4];
#pragma unroll
			for (uint32_t c = 0; c < 4; c++) {
				int cntMF = 0, cntGO = 0;
#pragma unroll
				for (uint32_t s = 0; s < kMF; s++) cntMF += sMF[half16(mfw[s], c)];
#pragma unroll
				for (uint32_t s = 0; s < kGO; s++) cntGO += sGO[half16(gow[s], c)];
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
				atomicAdd(&sBC[rowStart >> bcShift], pfCount);
				atomicAdd(&sSC[rowStart >> scShift], pfCount);
			}
			// GR->GO synapses whose delayed spike arrives now; the slot table
			// is read only by lanes with a spike in their buffers
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
		base = __shfl_sync(0xffffffffu, next, 0);
	}
	__syncthreads();

	// ---- the CTA's BC and SC counts
	const uint32_t buf = (uint32_t)(t % 3);
	uint32_t *bcOut = N->bcCount + (size_t)buf * numBC;
	uint32_t *scOut = N->scCount + (size_t)buf * numSC;
	for (uint32_t i = threadIdx.x; i < numBC + numSC; i += blockDim.x) {
		const uint32_t c = sBC[i];
		if (!c) continue;
		if (i < numBC) atomicAdd(&bcOut[i], c);
		else atomicAdd(&scOut[i - numBC], c);
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

bool passVecCapable(const DevNet &h)
{
	return passShapeOf(h) == 1 && h.numZones == 1 && h.bs >= 64 && h.bs % 64 == 0 && h.numGR % 128 == 0 &&
		(1u << h.bcShift) >= 64u && (1u << h.scShift) >= 64u && !h.ovStart && h.outCon16 &&
		h.P % (2 * h.bs) == 0;
}

size_t passVecSmemBytes(const DevNet &h)
{
	return 32u * h.mfWords + ((32u * h.goWords + 15u) & ~15u) + 4ull * h.numPC + 4ull * (h.numBC + h.numSC) +
		4ull * h.bs;
}

const void *passVecKernel() { return (const void *)&grPassVecKernel; }
const void *pairReduceKernelFn() { return (const void *)&pairReduceKernel; }
const void *pcTreeKernelFn() { return (const void *)&pcTreeKernel; }

}  // namespace cbm
