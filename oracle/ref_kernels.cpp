/* Test infrastructure (oracle build only).
 *
 * CPU restatement of the kernel launchers that the reference's host code
 * calls (declared in CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/cuda/kernels.h:19-72,
 * kernels defined in CBM_CORE_LIB_MGPU_DEV/src/cuda/kernels.cu).  Each launcher
 * walks its grid serially and performs the same IEEE single-precision
 * operations in source order (built with -ffp-contract=off), so the reference's
 * unmodified host orchestration can run on a machine without a GPU.
 *
 * Order-sensitive detail reproduced exactly: sumInputsNew (kernels.cu:296-376)
 * gives each thread tid a running sum of the pairs (x[i] + x[i+bs]) for
 * i = tid, tid+2bs, ..., then reduces the bs partial sums with a halving tree
 * (strides bs/2 ... 1).  The last-warp part of that tree is written
 * warp-synchronously without __syncwarp; the intended lockstep semantics
 * (all loads of a statement before its stores) are what is restated here.
 *
 * The OpenMP pragmas only take effect in the all-core timing build
 * (oracle/_ref/ref_run_omp); every loop they split writes disjoint cells. */
#include <cstring>
#include <vector>
#include <CBMCoreInclude/cuda/kernels.h>

void callTestKernel(cudaStream_t &st, float *a, float *b, float *c)
{
	(void)st;
	for (int i = 0; i < 128; i++) c[i] = a[i] + b[i];
}

/* kernels.cu:79-110 */
void callGRActKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock,
		float *vm, float *gKCa, float *thresh,
		ct_uint32_t *apBuf, ct_uint8_t *apOutGR, ct_uint32_t *apGR,
		float *gESum, float *gISum,
		float gLeak, float eLeak, float eGOIn,
		float threshBase, float threshMax, float threshDecay)
{
	(void)st;
	long n = (long)numBlocks * numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (long i = 0; i < n; i++)
	{
		float tempV = vm[i];
		float tempGKCa = gKCa[i];
		tempV = tempV + (gLeak + tempGKCa * tempGKCa * tempGKCa * tempGKCa) * (eLeak - tempV)
			- (gESum[i]) * tempV + (gISum[i]) * (eGOIn - tempV);
		float tempThresh = thresh[i];
		tempThresh = tempThresh + (threshBase - tempThresh) * threshDecay;
		unsigned int tempAP = tempV > tempThresh;
		thresh[i] = tempAP * threshMax + (!tempAP) * tempThresh;
		tempGKCa = tempGKCa * 0.9999f;
		gKCa[i] = tempAP * (tempGKCa + 0.003f) + (!tempAP) * tempGKCa;
		apBuf[i] = (apBuf[i] << 1) | (tempAP);
		apOutGR[i] = tempAP;
		apGR[i] = tempAP;
		vm[i] = tempV;
	}
}

/* kernels.cu:296-376 for one (blockIdx.x, blockIdx.y) */
template<typename Type, bool inMultiPitch, bool outMultiPitch>
static void sumBlock(unsigned int blockSize, unsigned int bx, unsigned int by, unsigned int gridDimX,
		Type *input, size_t inputPitch, Type *output, size_t outputPitch, unsigned int rowLength)
{
	std::vector<Type> s(blockSize);
	Type *inputRow = inMultiPitch ? (Type *)((char *)input + by * inputPitch) : input + by;
	unsigned int gridSize = blockSize * 2 * gridDimX;
	for (unsigned int tid = 0; tid < blockSize; tid++)
	{
		unsigned int index = bx * (blockSize * 2) + tid;
		Type tempSum = 0;
		while (index < rowLength)
		{
			tempSum += inputRow[index] + inputRow[index + blockSize];
			index += gridSize;
		}
		s[tid] = tempSum;
	}
	for (unsigned int h = blockSize / 2; h >= 1; h /= 2)
	{
		for (unsigned int t = 0; t < h; t++) s[t] = s[t] + s[t + h];
	}
	Type *outputRow = outMultiPitch ? (Type *)((char *)output + by * outputPitch) : output + by;
	outputRow[bx] = s[0];
}

/* kernels.cu:435-470: block size picked from the elements per block. */
template<typename Type, bool inMultiP, bool outMultiP>
void callSumKernel(cudaStream_t &st, Type *inGPU, size_t inGPUP, Type *outSumGPU, size_t outSumGPUP,
		unsigned int nOutCells, unsigned int nOutCols, unsigned int rowLength)
{
	(void)st;
	unsigned int numElementsPerBlock = rowLength / nOutCols;
	unsigned int bs;
	if (numElementsPerBlock >= 2048) bs = 512;
	else if (numElementsPerBlock >= 512) bs = 128;
	else if (numElementsPerBlock >= 128) bs = 32;
	else if (numElementsPerBlock >= 32) bs = 8;
	else bs = 2;
#pragma omp parallel for schedule(static)
	for (int by = 0; by < (int)nOutCells; by++)
		for (unsigned int bx = 0; bx < nOutCols; bx++)
			sumBlock<Type, inMultiP, outMultiP>(bs, bx, by, nOutCols, inGPU, inGPUP, outSumGPU, outSumGPUP, rowLength);
}

template<typename Type>
void callBroadcastKernel(cudaStream_t &st, Type *broadcastVal, Type *outArray,
		unsigned int nBlocks, unsigned int rowLength)
{
	(void)st; (void)nBlocks;
	for (unsigned int i = 0; i < rowLength; i++) outArray[i] = *broadcastVal;
}

/* kernels.cu:112-150: one histogram row of numGO counters per block. */
void callUpdateGROutGOKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock, unsigned int numGO,
		ct_uint32_t *apBuf, ct_uint32_t *grInGOGPU, ct_uint32_t grInGOGPUPitch,
		ct_uint32_t *delayMasksGPU, ct_uint32_t delayMasksGPUPitch,
		ct_uint32_t *conGRtoGOGPU, size_t conGRtoGOGPUPitch,
		ct_int32_t *numGOPerGRGPU)
{
	(void)st;
	unsigned int nWrites = numGO / numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (int b = 0; b < (int)numBlocks; b++)
	{
		std::vector<ct_uint32_t> hist(numGO, 0u);
		for (unsigned int tid = 0; tid < numGRPerBlock; tid++)
		{
			unsigned long index = (unsigned long)b * numGRPerBlock + tid;
			int tempNS = numGOPerGRGPU[index];
			for (int i = 0; i < tempNS; i++)
			{
				ct_uint32_t *conRow = (ct_uint32_t *)((char *)conGRtoGOGPU + i * conGRtoGOGPUPitch);
				ct_uint32_t *delayRow = (ct_uint32_t *)((char *)delayMasksGPU + (size_t)i * delayMasksGPUPitch);
				if ((apBuf[index] & delayRow[index]) > 0) hist[conRow[index]] += 1;
			}
		}
		ct_uint32_t *goRow = (ct_uint32_t *)((char *)grInGOGPU + (size_t)b * grInGOGPUPitch);
		for (unsigned int k = 0; k < nWrites * numGRPerBlock; k++) goRow[k] = hist[k];
	}
}

/* kernels.cu:152-167 */
void callSumGRGOOutKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGOPerBlock,
		unsigned int numGROutRows, ct_uint32_t *grInGOGPU, size_t grInGOGPUPitch, ct_uint32_t *grInGOSGPU)
{
	(void)st;
	unsigned int n = numBlocks * numGOPerBlock;
	for (unsigned int index = 0; index < n; index++)
	{
		ct_uint32_t tempSum = 0;
		for (unsigned int r = 0; r < numGROutRows; r++)
			tempSum += ((ct_uint32_t *)((char *)grInGOGPU + r * grInGOGPUPitch))[index];
		grInGOSGPU[index] = tempSum;
	}
}

/* kernels.cu:169-199 */
void callUpdateInGROPKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock,
		unsigned int numInCells, ct_uint32_t *apInGPU, float *gGPU, size_t gGPUP,
		ct_uint32_t *conInGRGPU, size_t conInGRGPUP,
		ct_int32_t *numInPerGRGPU, float *gSumGPU, float gDecay, float gInc)
{
	(void)st; (void)gGPU; (void)gGPUP;
	unsigned int inNLoads = numInCells / numGRPerBlock;
	std::vector<ct_uint32_t> staged(inNLoads * numGRPerBlock);
	for (unsigned int k = 0; k < staged.size(); k++) staged[k] = apInGPU[k];
	long n = (long)numBlocks * numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (long index = 0; index < n; index++)
	{
		int tempNSyn = numInPerGRGPU[index];
		int tempApInSum = 0;
		for (int i = 0; i < tempNSyn; i++)
		{
			ct_uint32_t *conRow = (ct_uint32_t *)((char *)conInGRGPU + i * conInGRGPUP);
			tempApInSum += staged[conRow[index]];
		}
		gSumGPU[index] = gSumGPU[index] * gDecay + gInc * (tempApInSum);
	}
}

/* kernels.cu:247-260 */
void callUpdatePFBCSCOutKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock,
		ct_uint32_t *apBufGPU, ct_uint32_t *delayMaskGPU,
		ct_uint32_t *inPFBCGPU, size_t inPFBCGPUPitch, unsigned int numPFInPerBCP2,
		ct_uint32_t *inPFSCGPU, size_t inPFSCGPUPitch, unsigned int numPFInPerSCP2)
{
	(void)st;
	unsigned int numPFInPerBC = 1u << numPFInPerBCP2;
	unsigned int numPFInPerSC = 1u << numPFInPerSCP2;
	long n = (long)numBlocks * numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (long index = 0; index < n; index++)
	{
		ct_uint32_t *pfBCRow = (ct_uint32_t *)((char *)inPFBCGPU + (index >> numPFInPerBCP2) * inPFBCGPUPitch);
		ct_uint32_t *pfSCRow = (ct_uint32_t *)((char *)inPFSCGPU + (index >> numPFInPerSCP2) * inPFSCGPUPitch);
		ct_uint32_t tempOut = (apBufGPU[index] & delayMaskGPU[index]) > 0;
		pfBCRow[index & (numPFInPerBC - 1)] = tempOut;
		pfSCRow[index & (numPFInPerSC - 1)] = tempOut;
	}
}

/* kernels.cu:262-272 */
void callUpdatePFPCOutKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock,
		ct_uint32_t *apBufGPU, ct_uint32_t *delayMaskGPU,
		float *pfPCSynWGPU, float *inPFPCGPU, size_t inPFPCGPUPitch, unsigned int numPFInPerPCP2)
{
	(void)st;
	unsigned int numPFInPerPC = 1u << numPFInPerPCP2;
	long n = (long)numBlocks * numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (long index = 0; index < n; index++)
	{
		float *pfPCRow = (float *)((char *)inPFPCGPU + (index >> numPFInPerPCP2) * inPFPCGPUPitch);
		unsigned int tempOut = (apBufGPU[index] & delayMaskGPU[index]) > 0;
		pfPCRow[index & (numPFInPerPC - 1)] = pfPCSynWGPU[index] * tempOut;
	}
}

/* kernels.cu:241-246 (the bufTestMask argument is ignored there too) */
void callUpdateGRHistKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock,
		ct_uint32_t *apBufGPU, ct_uint64_t *historyGPU, ct_uint32_t apBufGRHistMask)
{
	(void)st; (void)apBufGRHistMask;
	long n = (long)numBlocks * numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (long i = 0; i < n; i++)
	{
		ct_uint64_t tempHist = historyGPU[i] << 1;
		historyGPU[i] = tempHist | ((apBufGPU[i] & 0x0000001F) > 0) * 0x00000001;
	}
}

/* kernels.cu:282-291 (bit 39 is hard-coded there; pastBinNToCheck is ignored) */
void callUpdatePFPCPlasticityIOKernel(cudaStream_t &st, unsigned int numBlocks, unsigned int numGRPerBlock,
		float *synWeightGPU, ct_uint64_t *historyGPU, unsigned int pastBinNToCheck,
		int offSet, float pfPCPlastStep)
{
	(void)st; (void)pastBinNToCheck;
	long n = (long)numBlocks * numGRPerBlock;
#pragma omp parallel for schedule(static)
	for (long k = 0; k < n; k++)
	{
		unsigned long i = (unsigned long)k + (unsigned long)offSet;
		synWeightGPU[i] = synWeightGPU[i] + ((historyGPU[i] & 0x0000008000000000ull) > 0) * pfPCPlastStep;
		synWeightGPU[i] = (synWeightGPU[i] > 0) * synWeightGPU[i];
		synWeightGPU[i] = (synWeightGPU[i] > 1) + (synWeightGPU[i] <= 1) * synWeightGPU[i];
	}
}

template void callSumKernel<float, true, false>
		(cudaStream_t &st, float *inPFGPU, size_t inPFGPUP, float *outPFSumGPU, size_t outPFSumGPUP,
		unsigned int nOutCells, unsigned int nOutCols, unsigned int rowLength);
template void callSumKernel<ct_uint32_t, true, false>
		(cudaStream_t &st, ct_uint32_t *inPFGPU, size_t inPFGPUP, ct_uint32_t *outPFSumGPU, size_t outPFSumGPUP,
		unsigned int nOutCells, unsigned int nOutCols, unsigned int rowLength);
template void callSumKernel<ct_uint32_t, false, false>
		(cudaStream_t &st, ct_uint32_t *inPFGPU, size_t inPFGPUP, ct_uint32_t *outPFSumGPU, size_t outPFSumGPUP,
		unsigned int nOutCells, unsigned int nOutCols, unsigned int rowLength);
template void callBroadcastKernel<ct_uint32_t>
		(cudaStream_t &st, ct_uint32_t *broadCastVal, ct_uint32_t *outArray, unsigned int nBlocks, unsigned int rowLength);
