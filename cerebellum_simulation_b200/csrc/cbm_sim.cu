// Host orchestration of the device-resident step; see cbm_sim.hpp.
#include "cbm_sim.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>

#include "cbm_kernels.cuh"
#include "cbm_rng.hpp"

namespace cbm {

std::string cudaErr(cudaError_t e, const char *what)
{
	if (e == cudaSuccess) return "";
	return std::string(what) + ": " + cudaGetErrorString(e);
}

#define CK(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return cudaErr(e_, what); } while (0)
#define CKS(expr) do { std::string s_ = (expr); if (!s_.empty()) return s_; } while (0)

// ------------------------------------------------------------------ Network
template <typename T> T *Network::alloc(size_t n)
{
	void *p = nullptr;
	// whole 16-byte units, so that arrays can be copied with 16-byte accesses
	size_t bytes = (std::max<size_t>(n * sizeof(T), 16) + 15) & ~(size_t)15;
	if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
	if (cudaMemset(p, 0, bytes) != cudaSuccess) { cudaFree(p); return nullptr; }
	allocs_.push_back(p);
	allocBytes_[p] = bytes;
	return (T *)p;
}

template <typename T> T *Network::upload(const T *src, size_t n)
{
	T *d = alloc<T>(n);
	if (d && n) cudaMemcpy(d, src, n * sizeof(T), cudaMemcpyHostToDevice);
	return d;
}

Network::~Network()
{
	for (void *p : allocs_) cudaFree(p);
	if (dNet_.ptr) cudaFree(dNet_.ptr);
	if (hPinnedBits_) cudaFreeHost(hPinnedBits_);
	if (hErr_) cudaFreeHost(hErr_);
	if (hMailbox_) cudaFreeHost(hMailbox_);
	if (hPinnedRaw_) cudaFreeHost(hPinnedRaw_);
	for (cudaEvent_t e : mfStageEv_) if (e) cudaEventDestroy(e);
}

// callSumKernel's block size for a row of rowLength elements
// (CBM_CORE_LIB_MGPU_DEV/src/cuda/kernels.cu:445-469)
static uint32_t reductionBlockSize(uint32_t rowLength)
{
	if (rowLength >= 2048) return 512;
	if (rowLength >= 512) return 128;
	if (rowLength >= 128) return 32;
	if (rowLength >= 32) return 8;
	return 2;
}

static bool singleBitOrZero(uint32_t m, uint32_t &bit)
{
	if (m == 0) { bit = kNoDelay; return true; }
	if (m & (m - 1)) return false;
	bit = (uint32_t)__builtin_ctz(m);
	return true;
}

size_t Network::passSmemBytes() const
{
	return sizeof(uint32_t) * ((size_t)h_.mfWords + h_.goWords + h_.bcLocal + h_.scLocal) +
		sizeof(float) * (size_t)h_.numZones * 2 * h_.K * h_.J;
}

size_t Network::passTmaSmemBytes(uint32_t R, uint32_t S, uint32_t outBytes) const
{
	const PassLayout L = passLayout(R, h_.nMFSlots, h_.nGOSlots, h_.nOutTma, h_.numZones, outBytes);
	return 128 + (size_t)S * L.bytes + 16ull * S + sizeof(uint32_t) * (((size_t)h_.bcLocal + h_.scLocal + 3) & ~(size_t)3) +
		sizeof(float) * (size_t)h_.numZones * 2 * h_.K * 32 + 32ull * (h_.mfWords + h_.goWords);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
		const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
		CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encodeTiledFn()
{
	static EncodeTiledFn fn = nullptr;
	if (!fn) {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
				q == cudaDriverEntryPointSuccess)
			fn = (EncodeTiledFn)p;
	}
	return fn;
}

std::string Network::buildPassMaps(uint32_t R)
{
	EncodeTiledFn enc = encodeTiledFn();
	if (!enc) return "cuTensorMapEncodeTiled is unavailable";
	const uint32_t N = h_.numGR, bs = h_.bs;
	if ((uint64_t)h_.numPC * h_.P != N || bs < 32 || N % bs || 2 * h_.K % R) return "GR pass tiling does not cover the cells";
	std::vector<CUtensorMap> maps(PM_COUNT);
	memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
	auto enc2 = [&](int m, const void *ptr, CUtensorMapDataType dt, uint32_t es) -> std::string {
		const cuuint64_t dims[2] = {bs, N / bs};
		const cuuint64_t strides[1] = {(cuuint64_t)bs * es};
		const cuuint32_t box[2] = {32, R};
		const cuuint32_t estr[2] = {1, 1};
		if (enc(&maps[m], dt, 2, const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
				CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
			return "encoding a TMA descriptor failed";
		return "";
	};
	auto enc3 = [&](int m, const void *ptr, CUtensorMapDataType dt, uint32_t es, uint32_t slots,
			uint32_t boxSlots) -> std::string {
		const cuuint64_t dims[3] = {bs, N / bs, slots};
		const cuuint64_t strides[2] = {(cuuint64_t)bs * es, (cuuint64_t)N * es};
		const cuuint32_t box[3] = {32, R, boxSlots};
		const cuuint32_t estr[3] = {1, 1, 1};
		if (enc(&maps[m], dt, 3, const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
				CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
			return "encoding a TMA descriptor failed";
		return "";
	};
	if (std::max({h_.nMFSlots, h_.nGOSlots, h_.nOutSlots}) > 256) return "more than 256 synapse slots per GR";
	CKS(enc2(PM_V, h_.vGR, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4));
	CKS(enc2(PM_GKCA, h_.gKCaGR, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4));
	CKS(enc2(PM_THRESH, h_.threshGR, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4));
	CKS(enc2(PM_GESUM, h_.gESum, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4));
	CKS(enc2(PM_GISUM, h_.gISum, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4));
	CKS(enc2(PM_APBUF, h_.apBufGR, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4));
	const uint32_t mfS = std::max(1u, h_.nMFSlots), goS = std::max(1u, h_.nGOSlots), outS = std::max(1u, h_.nOutSlots);
	const uint32_t outT = std::max(1u, h_.nOutTma);
	CKS(enc3(PM_MFIDX, h_.mfIdx, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, mfS, mfS));
	CKS(enc3(PM_GOIDX, h_.goIdx, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, goS, goS));
	CKS(enc3(PM_OUTCON, h_.outCon, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, outS, outT));
	if (h_.outCon16)
		CKS(enc3(PM_OUTCON16, h_.outCon16, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, outS, outT));
	CKS(enc2(PM_PFDELAY, h_.pfDelay, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1));
	CKS(enc2(PM_HIST, h_.historyGR, CU_TENSOR_MAP_DATA_TYPE_UINT64, 8));
	for (uint32_t z = 0; z < h_.numZones; z++) CKS(enc2(PM_W0 + z, h_.zones[z].w, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4));
	CUtensorMap *d = alloc<CUtensorMap>(PM_COUNT);
	if (!d) return "device allocation failed";
	CK(cudaMemcpy(d, maps.data(), PM_COUNT * sizeof(CUtensorMap), cudaMemcpyHostToDevice), "uploading TMA descriptors");
	h_.passMaps = d;
	return uploadDesc();
}

std::string Network::uploadDesc()
{
	CK(cudaMemcpy(dNet_.ptr, &h_, sizeof(DevNet), cudaMemcpyHostToDevice), "uploading the network descriptor");
	return "";
}

std::string Network::setPcSumMode(bool on, cudaStream_t s)
{
	if ((h_.pcSumMode != 0) == on) return "";
	const uint64_t T = hostT_;
	const DevNet *np = devPtr();
	if (on) {
		// the small-cell update of the next two steps reads the sums of steps
		// T-1 and T, which the pass before made as partial sums
		for (uint64_t st = T > 0 ? T - 1 : 0; T > 0 && st <= T; st++) {
			uint64_t a = st;
			void *args[] = {&np, &a};
			CK(cudaLaunchKernel(pcTreeKernelFn(), dim3(h_.numPC), dim3(256), args, 0, s), "PF->PC input sums");
		}
	} else if (T > 0) {
		// the vector pass left step T's reduction as pair sums
		uint64_t a = T;
		void *args[] = {&np, &a};
		const uint32_t seqs = h_.numPC * h_.bs;
		CK(cudaLaunchKernel(pairReduceKernelFn(), dim3((seqs + 255) / 256), dim3(256), args, 0, s), "PF->PC pair sums");
	}
	CK(cudaStreamSynchronize(s), "PF->PC sums");
	h_.pcSumMode = on ? 1u : 0u;
	return uploadDesc();
}

// Arrays the microzone CTA stages in shared memory for each step: its
// state (written back) and its connectivity (read only).  Arrays that the GR
// pass reads during the same step (weights, plasticity selectors, partial
// sums, counters) stay where they are.  When everything fits, the staged
// arrays move into one staging block behind the network descriptor and the
// step counter (stageBlockBytes), read-only arrays first, so that the CTA
// copies the block in one pass and writes back one contiguous range.
std::string Network::buildZoneStaging()
{
	std::vector<StageSeg> ro, wb;
	auto add = [&](size_t fieldOff, bool writeBack) -> std::string {
		void *ptr = *(void **)((char *)&h_ + fieldOff);
		auto it = allocBytes_.find(ptr);
		if (it == allocBytes_.end()) return "staging: unknown array";
		StageSeg sg;
		sg.fieldOff = (uint32_t)fieldOff;
		sg.bytes = (uint32_t)it->second;
		sg.smemOff = 0;
		sg.writeBack = writeBack ? 1u : 0u;
		(writeBack ? wb : ro).push_back(sg);
		return "";
	};
#define CBM_NET(f, wb) CKS(add(offsetof(DevNet, f), wb))
	CBM_NET(apSC, true); CBM_NET(apBufSC, true); CBM_NET(gPFSC, true); CBM_NET(threshSC, true); CBM_NET(vSC, true);
	CBM_NET(histMF, true); CBM_NET(apBufMF, true);
#undef CBM_NET
	for (uint32_t z = 0; z < h_.numZones; z++) {
		const size_t zb = offsetof(DevNet, zones) + z * sizeof(DevZone);
#define CBM_ZONE(f, wb) CKS(add(zb + offsetof(DevZone, f), wb))
		CBM_ZONE(pPCfromSCtoPC, false); CBM_ZONE(pNCfromPCtoNC, false); CBM_ZONE(pNCfromMFtoNC, false);
		CBM_ZONE(pIOfromNCtoIO, false); CBM_ZONE(pIOInIOIO, false); CBM_ZONE(bcpcStart, false);
		CBM_ZONE(bcpcSrc, false); CBM_ZONE(pcbcStart, false); CBM_ZONE(pcbcSrc, false); CBM_ZONE(gPCScaleNC, false);
		CBM_ZONE(apBC, true); CBM_ZONE(apBufBC, true); CBM_ZONE(inputPCBC, true); CBM_ZONE(gPFBC, true);
		CBM_ZONE(gPCBC, true); CBM_ZONE(threshBC, true); CBM_ZONE(vBC, true);
		CBM_ZONE(apPC, true); CBM_ZONE(apBufPC, true); CBM_ZONE(inputBCPC, true); CBM_ZONE(inputSCPC, true);
		CBM_ZONE(gPFPC, true); CBM_ZONE(gBCPC, true); CBM_ZONE(gSCPC, true); CBM_ZONE(vPC, true);
		CBM_ZONE(threshPC, true); CBM_ZONE(histPCPopAct, true); CBM_ZONE(scal, true);
		CBM_ZONE(apIO, true); CBM_ZONE(apBufIO, true); CBM_ZONE(inputNCIO, true); CBM_ZONE(gNCIO, true);
		CBM_ZONE(threshIO, true); CBM_ZONE(vIO, true); CBM_ZONE(vCoupleIO, true); CBM_ZONE(pfPCPlastTimerIO, true);
		CBM_ZONE(apNC, true); CBM_ZONE(apBufNC, true); CBM_ZONE(inputPCNC, true); CBM_ZONE(inputMFNC, true);
		CBM_ZONE(gPCNC, true); CBM_ZONE(mfSynWeightNC, true); CBM_ZONE(gmaxNMDAofMFtoNC, true);
		CBM_ZONE(gmaxAMPAofMFtoNC, true); CBM_ZONE(gMFNMDANC, true); CBM_ZONE(gMFAMPANC, true);
		CBM_ZONE(threshNC, true); CBM_ZONE(vNC, true); CBM_ZONE(synIOPReleaseNC, true);
#undef CBM_ZONE
	}
	std::vector<StageSeg> segs(ro);
	segs.insert(segs.end(), wb.begin(), wb.end());
	uint32_t arena = 0, wbOff = 0;
	for (size_t k = 0; k < segs.size(); k++) {
		if (k == ro.size()) wbOff = arena;
		segs[k].smemOff = arena;
		arena += segs[k].bytes;
	}
	if (wb.empty()) wbOff = arena;
	h_.numZoneSegs = 0;
	h_.zoneArenaBytes = 0;
	h_.zoneWbOff = 0;
	h_.zoneStageBytes = 0;
	h_.zoneSegs = nullptr;
	const uint32_t block = stageBlockBytes(arena, (uint32_t)segs.size());
	const ZoneInputLayout L = zoneInputLayout(h_.mfWords, h_.numBC, h_.numSC, h_.numZones, h_.numPC, h_.bs);
	if ((size_t)block + L.bytes + zoneScratchBytes() > kTailSmemBudget) return "";  // the CTA works on global memory
	if (const char *env = getenv("CBM_ZONE_STAGE"))  // "0": global-memory mode regardless of size (testing)
		if (!strcmp(env, "0")) return "";

	uint8_t *blk = nullptr;
	CK(cudaMalloc((void **)&blk, block), "allocating the staging block");
	zoneBlock_ = blk;
	dNet_.ptr = blk;  // the descriptor heads the block (freed with it)
	CK(cudaMemset(blk, 0, block), "clearing the staging block");
	for (const StageSeg &sg : segs) {
		void **field = (void **)((char *)&h_ + sg.fieldOff);
		uint8_t *dst = blk + kStageArenaOff + sg.smemOff;
		CK(cudaMemcpy(dst, *field, sg.bytes, cudaMemcpyDeviceToDevice), "filling the staging block");
		release(*field);
		*field = dst;
	}
	// the step counter lives in the block, so that the copy brings it along
	uint64_t *tb = (uint64_t *)(blk + kStageNetBytes);
	CK(cudaMemcpy(tb, h_.tBase, sizeof(uint64_t), cudaMemcpyDeviceToDevice), "moving the step counter");
	release(h_.tBase);
	h_.tBase = tb;
	StageSeg *dSegs = (StageSeg *)(blk + kStageArenaOff + arena);
	CK(cudaMemcpy(dSegs, segs.data(), segs.size() * sizeof(StageSeg), cudaMemcpyHostToDevice), "staging table");
	h_.zoneSegs = dSegs;
	h_.numZoneSegs = (uint32_t)segs.size();
	h_.zoneArenaBytes = arena;
	h_.zoneWbOff = wbOff;
	h_.zoneStageBytes = block;
	return "";
}

void Network::release(void *p)
{
	auto it = std::find(allocs_.begin(), allocs_.end(), p);
	if (it != allocs_.end()) allocs_.erase(it);
	allocBytes_.erase(p);
	cudaFree(p);
}

size_t Network::zoneScratchBytes() const
{
	// SC spikes, NC and IO scratch, plasticity flags
	return ((h_.numSC + 15) & ~15u) + 4ull * h_.numZones * h_.numNC * 2 * h_.numpNCfromMFtoNC +
		4ull * h_.numZones * h_.numIO * h_.numpIOfromNCtoIO + 8ull * kMaxZones;
}

size_t Network::tailSmemBytes() const
{
	// Golgi role: cbmExpf table, MF bits, MF->GO counts, GO scales,
	// potentials, thresholds, spikes
	const size_t golgi = 256 + 4ull * h_.mfWords + 16ull * h_.numGO + h_.numGO;
	// microzone role: staging block and inputs, or table and MF bits; then its scratch
	size_t zone = zoneScratchBytes();
	if (h_.numZoneSegs)
		zone += h_.zoneStageBytes +
			zoneInputLayout(h_.mfWords, h_.numBC, h_.numSC, h_.numZones, h_.numPC, h_.bs).bytes;
	else
		zone += 256 + 16ull * ((h_.mfWords + 3) / 4);
	return std::max(golgi, zone);
}

double Network::bytesPerStepAlgorithmic() const
{
	return (72.0 + 4.0 * avgMF_ + 4.0 * avgGO_ + 8.0 * avgOut_) * h_.numGR;
}

double Network::bytesPerStepLayout() const
{
	// GR state read and written (6 x 4 B each way), synapse slots (u16 MF and
	// GO indices, u32 GR->GO targets), the PF delay byte, the PF->PC weight
	// of every zone; history read + write and weight writes on plasticity steps
	const double perGR = 48.0 + 2.0 * h_.nMFSlots + 2.0 * h_.nGOSlots + (double)outBytes_ * outPlanes_ +
		12.0 * ovUsed_ / h_.numGR + 1.0 + 4.0 * h_.numZones +
		(16.0 + 4.0 * h_.numZones) / h_.tsPerHistBinGR;
	return perGR * h_.numGR;
}

std::string checkNetwork(const State &st)
{
	const ConParams &c = st.cp;
	const ActParams &a = st.ap;
	auto A = [&](const char *n, int z = -1) -> const NamedArray * { return const_cast<State &>(st).find(n, z); };
	if (st.numZones < 1 || st.numZones > (uint32_t)kMaxZones) return "zone count must be 1..4";
	if (!c.numMF || !c.numGO || !c.numSC || !c.numBC || !c.numPC || !c.numNC || !c.numIO)
		return "every cell count must be positive";
	if (c.numMF >= 65535 || c.numGO >= 65535) return "numMF and numGO must be below 65535";
	const uint32_t N = c.numGR, P = c.numpPCfromGRtoPC;
	if (P < 4 || (P & (P - 1)) || N % 32) return "GR per PC must be a power of two >= 4 and numGR a multiple of 32";
	if ((uint64_t)c.numPC * P != N) return "numGR must be numPC x GR per PC";
	if (c.numpBCfromGRtoBCP2 > 31 || c.numpSCfromGRtoSCP2 > 31 ||
			(1u << c.numpBCfromGRtoBCP2) != c.numpBCfromGRtoBC || (1u << c.numpSCfromGRtoSCP2) != c.numpSCfromGRtoSC)
		return "PF->BC/SC block sizes are not powers of two";
	if (a.tsPerHistBinGR == 0 || a.numTSinMFHist == 0 || a.tsPerPopHistBinPC == 0 || a.numPopHistBinsPC == 0)
		return "time-bin parameters must be positive";

	// GR synapse tables; the reference stores pGRfromMFtoGR with
	// maxnumpGRfromGOtoGR columns
	const int32_t *numMFin = A("numpGRfromMFtoGR")->as<int32_t>();
	const uint32_t *pMF = A("pGRfromMFtoGR")->as<uint32_t>();
	const int32_t *numGOin = A("numpGRfromGOtoGR")->as<int32_t>();
	const uint32_t *pGO = A("pGRfromGOtoGR")->as<uint32_t>();
	const int32_t *numOut = A("numpGRfromGRtoGO")->as<int32_t>();
	const uint32_t *pOut = A("pGRfromGRtoGO")->as<uint32_t>();
	const uint32_t *pOutMask = A("pGRDelayMaskfromGRtoGO")->as<uint32_t>();
	const uint32_t *pfMask = A("pGRDelayMaskfromGRtoBSP")->as<uint32_t>();
	const uint32_t strideGO = c.maxnumpGRfromGOtoGR, strideOut = c.maxnumpGRfromGRtoGO;
	uint32_t bit;
	for (uint32_t g = 0; g < N; g++) {
		if (numMFin[g] < 0 || (uint32_t)numMFin[g] > std::min(c.maxnumpGRfromMFtoGR, strideGO))
			return "MF->GR count out of range";
		if (numGOin[g] < 0 || (uint32_t)numGOin[g] > strideGO) return "GO->GR count out of range";
		if (numOut[g] < 0 || (uint32_t)numOut[g] > strideOut) return "GR->GO count out of range";
		for (int k = 0; k < numMFin[g]; k++)
			if (pMF[(size_t)g * strideGO + k] >= c.numMF) return "MF->GR index out of range";
		for (int k = 0; k < numGOin[g]; k++)
			if (pGO[(size_t)g * strideGO + k] >= c.numGO) return "GO->GR index out of range";
		for (int k = 0; k < numOut[g]; k++) {
			if (pOut[(size_t)g * strideOut + k] >= c.numGO) return "GR->GO index out of range";
			if (!singleBitOrZero(pOutMask[(size_t)g * strideOut + k], bit)) return "GR->GO delay masks must have one bit";
		}
		if (!singleBitOrZero(pfMask[g], bit)) return "PF delay masks must have one bit";
	}

	// MF->GO out-lists, GO->GO GABA out-lists and GO coupling in-lists
	auto lists = [&](const char *num, const char *idx, uint32_t rows, uint32_t stride, uint32_t lim) -> bool {
		const int32_t *n = A(num)->as<int32_t>();
		const uint32_t *p = A(idx)->as<uint32_t>();
		for (uint32_t i = 0; i < rows; i++) {
			if (n[i] < 0 || (uint32_t)n[i] > stride) return false;
			for (int j = 0; j < n[i]; j++) if (p[(size_t)i * stride + j] >= lim) return false;
		}
		return true;
	};
	if (!lists("numpMFfromMFtoGO", "pMFfromMFtoGO", c.numMF, c.maxnumpMFfromMFtoGO, c.numGO))
		return "MF->GO count or index out of range";
	if (!lists("numpGOGABAOutGOGO", "pGOGABAOutGOGO", c.numGO, c.maxnumpGOGABAOutGOGO, c.numGO))
		return "GO->GO count or index out of range";
	if (!lists("numpGOCoupInGOGO", "pGOCoupInGOGO", c.numGO, c.maxnumpGOCoupInGOGO, c.numGO))
		return "GO coupling count or index out of range";

	// microzone wiring: every entry of each table is an index
	for (uint32_t z = 0; z < st.numZones; z++) {
		auto all = [&](const char *n, uint32_t lim) -> bool {
			const NamedArray *x = A(n, (int)z);
			const uint32_t *p = x->as<uint32_t>();
			for (size_t k = 0; k < x->count; k++) if (p[k] >= lim) return false;
			return true;
		};
		if (!all("pPCfromSCtoPC", c.numSC) || !all("pNCfromPCtoNC", c.numPC) || !all("pNCfromMFtoNC", c.numMF) ||
				!all("pIOfromNCtoIO", c.numNC) || !all("pIOInIOIO", c.numIO) || !all("pBCfromBCtoPC", c.numPC) ||
				!all("pPCfromPCtoBC", c.numBC))
			return "microzone connectivity index out of range";
	}
	return "";
}

std::string Network::build(State *st, const std::vector<int> &seeds, uint32_t mfRing, uint32_t mfSeed)
{
	(void)mfSeed;
	st_ = st;
	const ConParams &c = st->cp;
	const ActParams &a = st->ap;
	// checkNetwork(*st) has passed: every count and index below is in range
	const uint32_t N = c.numGR, P = c.numpPCfromGRtoPC;

	DevNet &h = h_;
	h.numGR = N; h.numMF = c.numMF; h.numGO = c.numGO; h.numSC = c.numSC; h.numBC = c.numBC;
	h.numPC = c.numPC; h.numNC = c.numNC; h.numIO = c.numIO; h.numZones = st->numZones;
	h.P = P; h.bs = reductionBlockSize(P); h.K = P / (2 * h.bs); h.J = std::min<uint32_t>(32, h.bs);
	h.tilesPerPC = h.bs / h.J;
	h.bcShift = c.numpBCfromGRtoBCP2; h.scShift = c.numpSCfromGRtoSCP2;
	h.bcLocal = std::max<uint32_t>(1, P >> h.bcShift);
	h.scLocal = std::max<uint32_t>(1, P >> h.scShift);
	h.mfWords = c.numMF / 32 + 1; h.goWords = c.numGO / 32 + 1;
	h.maxnumpMFfromMFtoGO = c.maxnumpMFfromMFtoGO; h.maxnumpGOCoupInGOGO = c.maxnumpGOCoupInGOGO;
	h.numpPCfromSCtoPC = c.numpPCfromSCtoPC; h.numpNCfromPCtoNC = c.numpNCfromPCtoNC;
	h.numpNCfromMFtoNC = c.numpNCfromMFtoNC; h.numpIOfromNCtoIO = c.numpIOfromNCtoIO;
	h.numpIOInIOIO = c.numpIOInIOIO;
	h.numPopHistBinsPC = a.numPopHistBinsPC; h.tsPerPopHistBinPC = a.tsPerPopHistBinPC;
	h.tsPerHistBinGR = a.tsPerHistBinGR; h.numTSinMFHist = a.numTSinMFHist;
	h.mfRing = std::max<uint32_t>(1, mfRing);

	// parameters
	h.gLeakGR = a.gLeakGR; h.eLeakGR = a.eLeakGR; h.eGOGR = a.eGOGR; h.threshRestGR = a.threshRestGR;
	h.threshMaxGR = a.threshMaxGR; h.threshDecGR = a.threshDecGR;
	h.gDecMFtoGR = a.gDecMFtoGR; h.gIncMFtoGR = a.gIncMFtoGR; h.gDecGOtoGR = a.gDecGOtoGR; h.gIncGOtoGR = a.gIncGOtoGR;
	h.gIncMFtoGO = a.gIncMFtoGO; h.gDecMFtoGO = a.gDecMFtoGO; h.gDecGRtoGO = a.gDecGRtoGO;
	h.gGABAIncGOtoGO = a.gGABAIncGOtoGO; h.gGABADecGOtoGO = a.gGABADecGOtoGO; h.gluDecayGO = a.gluDecayGO;
	h.gluScaleGO = a.gluScaleGO; h.mGluRDecayGO = a.mGluRDecayGO; h.mGluRScaleGO = a.mGluRScaleGO;
	h.gMGluRIncDecayGO = a.gMGluRIncDecayGO; h.gMGluRIncScaleGO = a.gMGluRIncScaleGO;
	h.gMGluRDecGRtoGO = a.gMGluRDecGRtoGO; h.gMGluRScaleGRtoGO = a.gMGluRScaleGRtoGO;
	h.threshRestGO = a.threshRestGO; h.threshDecGO = a.threshDecGO; h.gLeakGO = a.gLeakGO;
	h.eLeakGO = a.eLeakGO; h.eGABAGO = a.eGABAGO; h.threshMaxGO = a.threshMaxGO;
	h.coupleRiRjRatioGO = a.coupleRiRjRatioGO; h.goGABAGOGOSynRec = a.goGABAGOGOSynRec;
	h.goGABAGOGOSynDepF = a.goGABAGOGOSynDepF;
	h.gIncGRtoSC = a.gIncGRtoSC; h.gDecGRtoSC = a.gDecGRtoSC; h.gLeakSC = a.gLeakSC; h.eLeakSC = a.eLeakSC;
	h.threshDecSC = a.threshDecSC; h.threshRestSC = a.threshRestSC; h.threshMaxSC = a.threshMaxSC;
	h.gIncGRtoBC = a.gIncGRtoBC; h.gDecGRtoBC = a.gDecGRtoBC; h.gIncPCtoBC = a.gIncPCtoBC;
	h.gDecPCtoBC = a.gDecPCtoBC; h.gLeakBC = a.gLeakBC; h.eLeakBC = a.eLeakBC; h.ePCtoBC = a.ePCtoBC;
	h.threshDecBC = a.threshDecBC; h.threshRestBC = a.threshRestBC; h.threshMaxBC = a.threshMaxBC;
	h.gIncGRtoPC = a.gIncGRtoPC; h.gDecGRtoPC = a.gDecGRtoPC; h.gIncBCtoPC = a.gIncBCtoPC;
	h.gDecBCtoPC = a.gDecBCtoPC; h.gIncSCtoPC = a.gIncSCtoPC; h.gDecSCtoPC = a.gDecSCtoPC;
	h.gLeakPC = a.gLeakPC; h.eLeakPC = a.eLeakPC; h.eBCtoPC = a.eBCtoPC; h.eSCtoPC = a.eSCtoPC;
	h.threshDecPC = a.threshDecPC; h.threshRestPC = a.threshRestPC; h.threshMaxPC = a.threshMaxPC;
	h.msPerTimeStep = a.msPerTimeStep; h.gDecTSofNCtoIO = a.gDecTSofNCtoIO; h.gDecTTofNCtoIO = a.gDecTTofNCtoIO;
	h.gDecT0ofNCtoIO = a.gDecT0ofNCtoIO; h.gIncNCtoIO = a.gIncNCtoIO; h.gIncTauNCtoIO = a.gIncTauNCtoIO;
	h.gLeakIO = a.gLeakIO; h.eLeakIO = a.eLeakIO; h.eNCtoIO = a.eNCtoIO; h.threshMaxIO = a.threshMaxIO;
	h.threshDecIO = a.threshDecIO; h.threshRestIO = a.threshRestIO; h.coupleRiRjRatioIO = a.coupleRiRjRatioIO;
	h.tsLTDStartAPIO = a.tsLTDStartAPIO; h.tsLTDEndIO = a.tsLTDStartAPIO + ((int)(a.tsLTDDurationIO));
	h.tsLTPStartAPIO = a.tsLTPStartAPIO;
	h.gmaxNMDADecMFtoNC = a.gmaxNMDADecMFtoNC; h.gNMDAIncMFtoNC = a.gNMDAIncMFtoNC;
	h.gmaxAMPADecMFtoNC = a.gmaxAMPADecMFtoNC; h.gAMPAIncMFtoNC = a.gAMPAIncMFtoNC;
	h.gDecPCtoNC = a.gDecPCtoNC; h.gLeakNC = a.gLeakNC; h.eLeakNC = a.eLeakNC; h.ePCtoNC = a.ePCtoNC;
	h.threshDecNC = a.threshDecNC; h.threshRestNC = a.threshRestNC; h.threshMaxNC = a.threshMaxNC;
	h.relPDecTSofNCtoIO = a.relPDecTSofNCtoIO; h.relPDecTTofNCtoIO = a.relPDecTTofNCtoIO;
	h.relPDecT0ofNCtoIO = a.relPDecT0ofNCtoIO; h.relPIncNCtoIO = a.relPIncNCtoIO;
	h.relPIncTauNCtoIO = a.relPIncTauNCtoIO;
	h.synLTDPCPopActThreshMFtoNC = a.synLTDPCPopActThreshMFtoNC;
	h.synLTPPCPopActThreshMFtoNC = a.synLTPPCPopActThreshMFtoNC;
	h.synLTDStepSizeMFtoNC = a.synLTDStepSizeMFtoNC; h.synLTPStepSizeMFtoNC = a.synLTPStepSizeMFtoNC;

	auto A = [&](const char *n, int z = -1) -> NamedArray * { return st->find(n, z); };

	// ---- GR synapse tables: [gr][slot] (reference) -> [slot][gr] with
	// sentinel padding; checkNetwork bounds every count and index once, so
	// the kernels need no bounds checks.
	const int32_t *numMFin = A("numpGRfromMFtoGR")->as<int32_t>();
	const uint32_t *pMF = A("pGRfromMFtoGR")->as<uint32_t>();
	const int32_t *numGOin = A("numpGRfromGOtoGR")->as<int32_t>();
	const uint32_t *pGO = A("pGRfromGOtoGR")->as<uint32_t>();
	const int32_t *numOut = A("numpGRfromGRtoGO")->as<int32_t>();
	const uint32_t *pOut = A("pGRfromGRtoGO")->as<uint32_t>();
	const uint32_t *pOutMask = A("pGRDelayMaskfromGRtoGO")->as<uint32_t>();
	const uint32_t *pfMask = A("pGRDelayMaskfromGRtoBSP")->as<uint32_t>();
	const uint32_t strideGO = c.maxnumpGRfromGOtoGR, strideOut = c.maxnumpGRfromGRtoGO;
	uint32_t nMF = 0, nGO = 0, nOut = 0;
	uint64_t sumMF = 0, sumGO = 0, sumOut = 0;
	for (uint32_t g = 0; g < N; g++) {
		nMF = std::max<uint32_t>(nMF, numMFin[g]); nGO = std::max<uint32_t>(nGO, numGOin[g]);
		nOut = std::max<uint32_t>(nOut, numOut[g]);
		sumMF += numMFin[g]; sumGO += numGOin[g]; sumOut += numOut[g];
	}
	avgMF_ = (double)sumMF / N; avgGO_ = (double)sumGO / N; avgOut_ = (double)sumOut / N;
	h.nMFSlots = nMF; h.nGOSlots = nGO; h.nOutSlots = nOut;
	std::vector<uint16_t> mfIdx((size_t)std::max(1u, nMF) * N, (uint16_t)c.numMF);
	std::vector<uint16_t> goIdx((size_t)std::max(1u, nGO) * N, (uint16_t)c.numGO);
	std::vector<uint32_t> outCon((size_t)std::max(1u, nOut) * N, kNoDelay);
	std::vector<uint8_t> pfDelay(N);
	for (uint32_t g = 0; g < N; g++) {
		for (int k = 0; k < numMFin[g]; k++) mfIdx[(size_t)k * N + g] = (uint16_t)pMF[(size_t)g * strideGO + k];
		for (int k = 0; k < numGOin[g]; k++) goIdx[(size_t)k * N + g] = (uint16_t)pGO[(size_t)g * strideGO + k];
		uint32_t bit = 0;
		for (int k = 0; k < numOut[g]; k++) {
			singleBitOrZero(pOutMask[(size_t)g * strideOut + k], bit);
			outCon[(size_t)k * N + g] = (pOut[(size_t)g * strideOut + k] << 8) | bit;
		}
		singleBitOrZero(pfMask[g], bit);
		pfDelay[g] = (uint8_t)bit;
	}
	h.mfIdx = upload(mfIdx.data(), mfIdx.size());
	h.goIdx = upload(goIdx.data(), goIdx.size());
	h.outCon = upload(outCon.data(), outCon.size());
	// Networks with more than 4 GR->GO synapses on some GR (a fan-out padded
	// to its maximum): the per-tile TMA pass streams the first 4 slot planes
	// and takes the rest from per-tile lists after its rows
	h.nOutTma = nOut;
	h.ovStart = nullptr;
	h.ovEntry = nullptr;
	if (nOut > kOutInline && h.J == 32) {
		const uint32_t tiles = c.numPC * h.tilesPerPC;
		std::vector<std::vector<uint2>> per(tiles);
		for (uint32_t g = 0; g < N; g++)
			for (int k = (int)kOutInline; k < numOut[g]; k++) {
				const uint32_t cv = outCon[(size_t)k * N + g];
				if ((cv & 0xFFu) >= 32u) continue;  // a synapse without a delay bit never fires
				const uint32_t off = g % P, r = off / h.bs, jf = off % h.bs;
				const uint32_t tile = (g / P) * h.tilesPerPC + jf / 32;
				per[tile].push_back(make_uint2((r * 32 + jf % 32) | ((cv & 0xFFu) << 24), cv >> 8));
			}
		std::vector<uint32_t> start(tiles + 1, 0);
		std::vector<uint2> ent;
		for (uint32_t b = 0; b < tiles; b++) {
			start[b] = (uint32_t)ent.size();
			ent.insert(ent.end(), per[b].begin(), per[b].end());
		}
		start[tiles] = (uint32_t)ent.size();
		if (ent.empty()) ent.push_back(make_uint2(0, 0));  // never read: every range is empty
		h.nOutTma = kOutInline;
		h.ovStart = upload(start.data(), start.size());
		h.ovEntry = upload(ent.data(), ent.size());
		ovEntries_ = start[tiles];
	}
	h.outCon16 = nullptr;
	if (c.numGO <= kOut16MaxGO) {
		// the 16-bit copy the shape-specialised GR pass streams
		std::vector<uint16_t> out16(outCon.size(), kOut16None);
		for (size_t i = 0; i < outCon.size(); i++)
			if ((outCon[i] & 0xFFu) < 32u) out16[i] = (uint16_t)(((outCon[i] >> 8) << 5) | (outCon[i] & 0x1Fu));
		h.outCon16 = upload(out16.data(), out16.size());
	}
	h.pfDelay = upload(pfDelay.data(), pfDelay.size());

	auto upF = [&](const char *n, int z = -1) { NamedArray *x = A(n, z); return upload(x->as<float>(), x->count); };
	auto upU = [&](const char *n, int z = -1) { NamedArray *x = A(n, z); return upload(x->as<uint32_t>(), x->count); };
	auto upB = [&](const char *n, int z = -1) { NamedArray *x = A(n, z); return upload(x->as<uint8_t>(), x->count); };
	auto upI = [&](const char *n, int z = -1) { NamedArray *x = A(n, z); return upload(x->as<int32_t>(), x->count); };

	h.vGR = upF("vGR"); h.gKCaGR = upF("gKCaGR"); h.threshGR = upF("threshGR");
	h.gESum = upF("gMFSumGR"); h.gISum = upF("gGOSumGR");
	h.apBufGR = upU("apBufGR");
	h.historyGR = upload(A("historyGR")->as<uint64_t>(), N);

	h.histMF = upB("histMF"); h.apBufMF = upU("apBufMF");
	h.apGO = upB("apGO"); h.apBufGO = upU("apBufGO"); h.vGO = upF("vGO"); h.vCoupleGO = upF("vCoupleGO");
	h.threshCurGO = upF("threshCurGO"); h.inputMFGO = upU("inputMFGO"); h.inputGOGO = upU("inputGOGO");
	h.inputGOGABASynDepGO = upF("inputGOGABASynDepGO"); h.goGABAOutSynScaleGOGO = upF("goGABAOutSynScaleGOGO");
	h.gMFGO = upF("gMFGO"); h.gGRGO = upF("gGRGO"); h.gGOGO = upF("gGOGO"); h.gMGluRGO = upF("gMGluRGO");
	h.gMGluRIncGO = upF("gMGluRIncGO"); h.mGluRGO = upF("mGluRGO"); h.gluGO = upF("gluGO");
	h.apSC = upB("apSC"); h.apBufSC = upU("apBufSC"); h.gPFSC = upF("gPFSC"); h.threshSC = upF("threshSC");
	h.vSC = upF("vSC");
	h.sumGRInputGO = alloc<uint32_t>(c.numGO); h.sumInputGOGABASynDepGO = alloc<float>(c.numGO);

	// MF->GO out-lists as stored; GO->GO in-lists per destination in the
	// reference's (source, slot) iteration order (innet.cpp:937-950)
	h.numpMFfromMFtoGO = upI("numpMFfromMFtoGO"); h.pMFfromMFtoGO = upU("pMFfromMFtoGO");
	{
		const int32_t *numOutGG = A("numpGOGABAOutGOGO")->as<int32_t>();
		const uint32_t *pOutGG = A("pGOGABAOutGOGO")->as<uint32_t>();
		std::vector<std::vector<uint32_t>> in(c.numGO);
		for (uint32_t i = 0; i < c.numGO; i++)
			for (int j = 0; j < numOutGG[i]; j++) in[pOutGG[(size_t)i * c.maxnumpGOGABAOutGOGO + j]].push_back(i);
		std::vector<uint32_t> start(c.numGO + 1, 0), src;
		for (uint32_t d = 0; d < c.numGO; d++) { start[d + 1] = start[d] + (uint32_t)in[d].size(); src.insert(src.end(), in[d].begin(), in[d].end()); }
		h.gogoStart = upload(start.data(), start.size());
		h.gogoSrc = upload(src.data(), src.size());
	}
	{
		const int32_t *numC = A("numpGOCoupInGOGO")->as<int32_t>();
		const uint32_t *pC = A("pGOCoupInGOGO")->as<uint32_t>();
		bool any = false;
		std::vector<uint32_t> level(c.numGO, 0);
		uint32_t maxLevel = 0;
		for (uint32_t i = 0; i < c.numGO; i++) {
			for (int j = 0; j < numC[i]; j++) {
				uint32_t n = pC[(size_t)i * c.maxnumpGOCoupInGOGO + j];
				any = true;
				if (n < i) level[i] = std::max(level[i], level[n] + 1);
			}
			maxLevel = std::max(maxLevel, level[i]);
		}
		h.numpGOCoupInGOGO = upI("numpGOCoupInGOGO"); h.pGOCoupInGOGO = upU("pGOCoupInGOGO");
		std::vector<uint32_t> lstart, lgo;
		if (any) {
			h.numCoupLevels = maxLevel + 1;
			lstart.assign(maxLevel + 2, 0);
			for (uint32_t i = 0; i < c.numGO; i++) lstart[level[i] + 1]++;
			for (uint32_t L = 0; L <= maxLevel; L++) lstart[L + 1] += lstart[L];
			lgo.assign(c.numGO, 0);
			std::vector<uint32_t> fillPos(lstart.begin(), lstart.end() - 1);
			for (uint32_t i = 0; i < c.numGO; i++) lgo[fillPos[level[i]]++] = i;
		} else {
			h.numCoupLevels = 0;
			lstart.assign(1, 0);
			lgo.assign(1, 0);
		}
		h.coupLevelStart = upload(lstart.data(), lstart.size());
		h.coupLevelGO = upload(lgo.data(), lgo.size());
	}

	// ---- microzones
	const uint32_t numGRPerIO = N / c.numIO;
	for (uint32_t z = 0; z < st->numZones; z++) {
		DevZone &Q = h.zones[z];
		Q.w = upF("pfSynWeightPC", z);
		Q.pcPartial = alloc<float>((size_t)3 * c.numPC * h.bs);
		Q.pairSum = alloc<float>((size_t)2 * c.numPC * h.K * h.bs);
		Q.pcSum = alloc<float>((size_t)3 * c.numPC);
		Q.plastSel = alloc<uint8_t>((size_t)2 * c.numIO);
		std::vector<uint32_t> ioOfPC(c.numPC);
		uint32_t cur = 0;
		for (uint32_t pc = 0; pc < c.numPC; pc++) {
			// runPFPCPlastCUDA's IO walk (mzone.cpp:682-705)
			if (pc * P >= (cur + 1) * numGRPerIO) cur++;
			ioOfPC[pc] = std::min<uint32_t>(cur, c.numIO - 1);
		}
		Q.ioOfPC = upload(ioOfPC.data(), ioOfPC.size());
		Q.pPCfromSCtoPC = upU("pPCfromSCtoPC", z); Q.pNCfromPCtoNC = upU("pNCfromPCtoNC", z);
		Q.pNCfromMFtoNC = upU("pNCfromMFtoNC", z); Q.pIOfromNCtoIO = upU("pIOfromNCtoIO", z);
		Q.pIOInIOIO = upU("pIOInIOIO", z);
		{
			const uint32_t *bcpc = A("pBCfromBCtoPC", z)->as<uint32_t>();
			std::vector<std::vector<uint32_t>> in(c.numPC);
			for (uint32_t bc = 0; bc < c.numBC; bc++)
				for (uint32_t j = 0; j < c.numpBCfromBCtoPC; j++) in[bcpc[(size_t)bc * c.numpBCfromBCtoPC + j]].push_back(bc);
			std::vector<uint32_t> start(c.numPC + 1, 0), src;
			for (uint32_t i = 0; i < c.numPC; i++) { start[i + 1] = start[i] + (uint32_t)in[i].size(); src.insert(src.end(), in[i].begin(), in[i].end()); }
			Q.bcpcStart = upload(start.data(), start.size()); Q.bcpcSrc = upload(src.data(), src.size());
		}
		{
			const uint32_t *pcbc = A("pPCfromPCtoBC", z)->as<uint32_t>();
			std::vector<std::vector<uint32_t>> in(c.numBC);
			for (uint32_t pc = 0; pc < c.numPC; pc++)
				for (uint32_t j = 0; j < c.numpPCfromPCtoBC; j++) in[pcbc[(size_t)pc * c.numpPCfromPCtoBC + j]].push_back(pc);
			std::vector<uint32_t> start(c.numBC + 1, 0), src;
			for (uint32_t i = 0; i < c.numBC; i++) { start[i + 1] = start[i] + (uint32_t)in[i].size(); src.insert(src.end(), in[i].begin(), in[i].end()); }
			Q.pcbcStart = upload(start.data(), start.size()); Q.pcbcSrc = upload(src.data(), src.size());
		}
		Q.apBC = upB("apBC", z); Q.apBufBC = upU("apBufBC", z); Q.inputPCBC = upU("inputPCBC", z);
		Q.gPFBC = upF("gPFBC", z); Q.gPCBC = upF("gPCBC", z); Q.threshBC = upF("threshBC", z); Q.vBC = upF("vBC", z);
		Q.apPC = upB("apPC", z); Q.apBufPC = upU("apBufPC", z); Q.inputBCPC = upU("inputBCPC", z);
		Q.inputSCPC = upB("inputSCPC", z); Q.gPFPC = upF("gPFPC", z); Q.gBCPC = upF("gBCPC", z);
		Q.gSCPC = upF("gSCPC", z); Q.vPC = upF("vPC", z); Q.threshPC = upF("threshPC", z);
		Q.histPCPopAct = upU("histPCPopAct", z);
		const ZoneScalars &zs = st->zoneScalars[z];
		uint32_t sc[5] = {zs.histPCPopActSum, zs.histPCPopActCurBinN, zs.pcPopAct, zs.noLTPMFNC, zs.noLTDMFNC};
		Q.scal = upload(sc, 5);
		Q.apIO = upB("apIO", z); Q.apBufIO = upU("apBufIO", z); Q.inputNCIO = upB("inputNCIO", z);
		Q.gNCIO = upF("gNCIO", z); Q.threshIO = upF("threshIO", z); Q.vIO = upF("vIO", z);
		Q.vCoupleIO = upF("vCoupleIO", z); Q.pfPCPlastTimerIO = upI("pfPCPlastTimerIO", z);
		Q.apNC = upB("apNC", z); Q.apBufNC = upU("apBufNC", z); Q.inputPCNC = upB("inputPCNC", z);
		Q.inputMFNC = upB("inputMFNC", z); Q.gPCNC = upF("gPCNC", z); Q.gPCScaleNC = upF("gPCScaleNC", z);
		Q.mfSynWeightNC = upF("mfSynWeightNC", z); Q.gmaxNMDAofMFtoNC = upF("gmaxNMDAofMFtoNC", z);
		Q.gmaxAMPAofMFtoNC = upF("gmaxAMPAofMFtoNC", z); Q.gMFNMDANC = upF("gMFNMDANC", z);
		Q.gMFAMPANC = upF("gMFAMPANC", z); Q.threshNC = upF("threshNC", z); Q.vNC = upF("vNC", z);
		Q.synIOPReleaseNC = upF("synIOPReleaseNC", z);
		int seed = z < seeds.size() ? seeds[z] : 1000 + (int)z;
		Q.ncioKey = rng::streamKey((uint32_t)seed, rng::kStreamNCIO);
		// plasticity selector for step 1 (the tail of step t sets it for t+1)
		std::vector<uint8_t> sel(2 * c.numIO, 0);
		if (1 % a.tsPerHistBinGR == 0) {
			const int32_t *tm = A("pfPCPlastTimerIO", z)->as<int32_t>();
			for (uint32_t i = 0; i < c.numIO; i++)
				sel[c.numIO + i] = tm[i] < h.tsLTDEndIO ? 1 : (tm[i] > h.tsLTPStartAPIO ? 2 : 0);
		}
		if (!Q.plastSel) return "device allocation failed";
		CK(cudaMemcpy(Q.plastSel, sel.data(), sel.size(), cudaMemcpyHostToDevice), "uploading the plasticity selector");
		ctl.ltdStep[z] = a.synLTDStepSizeGRtoPC;
		ctl.ltpStep[z] = a.synLTPStepSizeGRtoPC;
		ctl.errDrive[z] = zs.errDrive;
	}
	ctl.gIncGRtoGO = a.gIncGRtoGO;
	ctlDirty = true;

	// ---- pipeline and control
	h.pairStep = alloc<uint64_t>(2);
	h.passClaim = alloc<uint32_t>(4);
	h.pcDone = alloc<uint32_t>(c.numPC);
	h.goCount = alloc<uint32_t>((size_t)2 * c.numGO);
	h.bcCount = alloc<uint32_t>((size_t)3 * c.numBC);
	h.scCount = alloc<uint32_t>((size_t)3 * c.numSC);
	h.goBits = alloc<uint32_t>((size_t)2 * h.goWords);
	h.mfBits = alloc<uint32_t>((size_t)h.mfRing * h.mfWords);
	h.mfRaw = alloc<uint8_t>((size_t)h.mfRing * c.numMF);
	h.hasMFRaw = 0;
	h.tBase = alloc<uint64_t>(1);
	h.ctl = alloc<HostCtl>(1);
	if (!h.pairStep || !h.passClaim || !h.pcDone || !h.goCount || !h.bcCount || !h.scCount || !h.goBits ||
			!h.mfBits || !h.mfRaw || !h.tBase || !h.ctl)
		return "device allocation failed";
	// the error word in mapped pinned host memory: the host reads it after a
	// synchronisation without a copy
	if (cudaHostAlloc((void **)&hErr_, sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess)
		return "pinned allocation failed";
	*hErr_ = 0;
	CK(cudaHostGetDevicePointer((void **)&h.errFlag, hErr_, 0), "mapping the error word");
	for (void *p : allocs_) if (!p) return "device allocation failed";
	CKS(buildZoneStaging());
	if (cudaMallocHost((void **)&hPinnedBits_, (size_t)kMFStage * h.mfWords * 4) != cudaSuccess ||
			cudaMallocHost((void **)&hPinnedRaw_, (size_t)kMFStage * c.numMF) != cudaSuccess)
		return "pinned allocation failed";
	for (cudaEvent_t &e : mfStageEv_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
	const size_t boxBytes = (8 + (size_t)h.numZones * c.numNC + 63) & ~(size_t)63;
	if (cudaHostAlloc((void **)&hMailbox_, boxBytes, cudaHostAllocMapped) != cudaSuccess)
		return "pinned allocation failed";
	memset(hMailbox_, 0, boxBytes);
	CK(cudaHostGetDevicePointer((void **)&dMailbox_, hMailbox_, 0), "mapping the NC mailbox");
	// a staged network's descriptor heads its staging block; otherwise the
	// descriptor and the step counter get an allocation of their own
	if (zoneBlock_) {
		dNet_.ptr = zoneBlock_;
	} else {
		CK(cudaMalloc(&dNet_.ptr, kStageArenaOff), "allocating the network descriptor");
		CK(cudaMemset(dNet_.ptr, 0, kStageArenaOff), "clearing the network descriptor");
		uint64_t *tb = (uint64_t *)((char *)dNet_.ptr + kStageNetBytes);
		CK(cudaMemcpy(tb, h.tBase, sizeof(uint64_t), cudaMemcpyDeviceToDevice), "moving the step counter");
		release(h.tBase);
		h.tBase = tb;
	}
	dNet_.bytes = sizeof(DevNet);
	CK(cudaMemcpy(dNet_.ptr, &h, sizeof(DevNet), cudaMemcpyHostToDevice), "uploading the network descriptor");
	CK(cudaDeviceSynchronize(), "network build");
	hostT_ = 0;
	return "";
}

void Network::setPlastSteps(uint32_t z, float ltd, float ltp) { ctl.ltdStep[z] = ltd; ctl.ltpStep[z] = ltp; ctlDirty = true; }
void Network::resetPlastSteps(uint32_t z)
{
	ctl.ltdStep[z] = st_->ap.synLTDStepSizeGRtoPC;
	ctl.ltpStep[z] = st_->ap.synLTPStepSizeGRtoPC;
	ctlDirty = true;
}
void Network::setErrDrive(uint32_t z, float rel) { ctl.errDrive[z] = rel * st_->ap.maxExtIncVIO; ctlDirty = true; }
void Network::setGIncGRtoGO(float v) { ctl.gIncGRtoGO = v; ctlDirty = true; }
void Network::resetGIncGRtoGO() { ctl.gIncGRtoGO = st_->ap.gIncGRtoGO; ctlDirty = true; }

std::string Network::setStateVarInput(const cbm_statevar_input &in, cudaStream_t s)
{
	const ConParams &c = st_->cp;
	if (!in.mean || !in.relaxed || !in.excited || !in.values) return "state-variable input: a table is missing";
	if (in.numVars == 0 || in.fibresPerVar == 0 || in.numSteps == 0) return "state-variable input: empty coding";
	if (!(in.den > 0) || !(in.norm > 0) || !(in.lo <= in.hi)) return "state-variable input: bad width or range";
	// an eyelid protocol with no CS trial, no US and no kept trial: the MF
	// generator alone, fed by the coding
	cbm_eyelid_protocol p{};
	p.trialSteps = 1u << 30;
	p.csOn = p.csOff = p.csPhasicOff = 0;
	p.csStartTrial = 0xFFFFFFFFu;
	p.mfSeed = in.mfSeed;
	p.mfThreshDecayTau = in.mfThreshDecayTau;
	p.mfFreqBG = p.mfFreqCSTonic = p.mfFreqCSPhasic = in.relaxed;
	p.numDataTrials = 0;
	p.postCS = 1;
	p.binSteps = 1;
	p.eyeGDecayTau = 10.5f; p.eyeGInc = 0.012f; p.eyeGShift = -0.13f; p.eyeGLeakRaw = 0.13f; p.eyeMaxAmp = 100.0f;
	DevProtocol sv{};
	sv.svMean = upload(in.mean, c.numMF);
	sv.svRelaxed = upload(in.relaxed, c.numMF);
	sv.svExcited = upload(in.excited, c.numMF);
	sv.svValues = upload(in.values, (size_t)in.numSteps * in.numVars);
	if (!sv.svMean || !sv.svRelaxed || !sv.svExcited || !sv.svValues) return "device allocation failed";
	sv.svSteps = in.numSteps;
	sv.svVars = in.numVars; sv.svPer = in.fibresPerVar;
	sv.svLo = in.lo; sv.svHi = in.hi; sv.svDen = in.den; sv.svMaxPossible = in.maxPossible;
	sv.svNorm = in.norm;
	return setProtocol(p, s, &sv);
}

std::string Network::stateVarRates(uint64_t row, float *out, cudaStream_t s)
{
	if (!h_.proto || !hProto_.svValues) return "no state-variable input is running";
	float *d = nullptr;
	CK(cudaMalloc(&d, 4ull * h_.numMF), "rates buffer");
	stateVarRatesKernel<<<(h_.numMF + 255) / 256, 256, 0, s>>>(devPtr(), row, d);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, 4ull * h_.numMF, cudaMemcpyDeviceToHost, s);
	if (e == cudaSuccess) e = cudaStreamSynchronize(s);
	cudaFree(d);
	CK(e, "state-variable rates");
	return "";
}

std::string Network::setProtocol(const cbm_eyelid_protocol &p, cudaStream_t s, const DevProtocol *sv)
{
	const ConParams &c = st_->cp;
	const ActParams &a = st_->ap;
	if (!p.mfFreqBG || !p.mfFreqCSTonic || !p.mfFreqCSPhasic) return "protocol: MF rate tables missing";
	if (p.trialSteps == 0 || p.binSteps == 0) return "protocol: trialSteps and binSteps must be positive";
	if (p.csOn < 0 || p.csOff < p.csOn || p.csOff > (int32_t)p.trialSteps || p.csPhasicOff < p.csOn ||
			p.csPhasicOff > p.csOff)
		return "protocol: need 0 <= csOn <= csPhasicOff <= csOff <= trialSteps";
	if (p.preCS < 0 || p.postCS < 0 || p.mfThreshDecayTau <= 0 || p.eyeGDecayTau <= 0)
		return "protocol: negative window or time constant";
	const int32_t recFrom = p.csOn - p.preCS, recLen = p.csOff + p.postCS - recFrom;
	if (recLen <= 0) return "protocol: empty recording window";
	// the MF spikes of step t+1 are written while step t reads its own slot
	if (h_.mfRing < 2) {
		uint32_t *bits = alloc<uint32_t>(2ull * h_.mfWords);
		uint8_t *raw = alloc<uint8_t>(2ull * c.numMF);
		if (!bits || !raw) return "device allocation failed";
		h_.mfBits = bits;
		h_.mfRaw = raw;
		h_.mfRing = 2;
	}
	h_.hasMFRaw = 0;
	DevProtocol d{};
	d.startT = hostT_;
	d.trialSteps = p.trialSteps;
	d.csStartTrial = p.csStartTrial;
	d.csOn = p.csOn; d.csOff = p.csOff; d.csPOff = p.csPhasicOff;
	d.plastOn = p.plastOnDelay; d.plastOff = p.plastOffDelay;
	d.plastLTD = p.plastLTD; d.plastLTP = p.plastLTP;
	d.usErrDrive = p.usErrDrive * a.maxExtIncVIO;  // MZone::setErrDrive (mzone.cpp:167-173)
	d.defaultLTD = a.synLTDStepSizeGRtoPC; d.defaultLTP = a.synLTPStepSizeGRtoPC;
	d.freqBG = upload(p.mfFreqBG, c.numMF);
	d.freqCSTonic = upload(p.mfFreqCSTonic, c.numMF);
	d.freqCSPhasic = upload(p.mfFreqCSPhasic, c.numMF);
	std::vector<float> ones(c.numMF, 1.0f);  // PoissonRegenCells starts every threshold at 1
	d.mfThresh = upload(ones.data(), ones.size());
	// The driver builds its generator with 1 ms steps (ecmanagementdelay.cpp:96),
	// and seeds it with a draw of a generator seeded by mfSeed
	// (poissonregencells.cpp:12-19): the first draw of the seed's stream.
	const float msPerTS = 1.0f;
	d.sPerTS = msPerTS / 1000;
	// 1 - exp(...) of poissonregencells.cpp:20: the argument is a float, so
	// C++ picks the float overload (the C library's expf) and the subtraction
	// is in float too
	d.mfThreshDecay = 1.0f - expf(-msPerTS / p.mfThreshDecayTau);
	const double u0 = (double)rng::uniform24((uint32_t)p.mfSeed, rng::kStreamNCIO, 0);
	const int derived = (int)(u0 * 2147483648.0);
	d.mfKey = rng::streamKey((uint32_t)derived, rng::kStreamNCIO);
	int32_t ps[2] = {0, 1};  // grPCPlastSet = false, grPCPlastReset = true (ecmanagementdelay.cpp:168-169)
	d.plastState = upload(ps, 2);
	// the steps in force when the protocol starts: the setters' current values
	float cur[2] = {ctl.ltdStep[0], ctl.ltpStep[0]};
	d.curSteps = upload(cur, 2);
	d.ctlSlots = alloc<float>(6);
	d.dataStartTrial = p.dataStartTrial; d.numDataTrials = p.numDataTrials;
	d.binSteps = p.binSteps;
	d.recFrom = recFrom; d.recLen = recLen;
	d.nBins = ((uint32_t)recLen + p.binSteps - 1) / p.binSteps;
	const size_t nd = std::max<uint32_t>(1, p.numDataTrials);
	d.ncPSH = alloc<uint32_t>(nd * d.nBins * c.numNC);
	d.pcPSH = alloc<uint32_t>(nd * d.nBins * c.numPC);
	d.eyelid = alloc<float>(nd * (size_t)recLen);
	d.eyeG = alloc<float>(c.numNC);
	d.eyeVm = alloc<float>(1);
	// EyelidIntegrator(numNC, msPerTimeStep, 10.5, 0.012, -0.13, 0.13, 100)
	// (ecmanagementdelay.cpp:108, eyelidintegrator.cpp:13-28)
	const int eyeMS = (int)(unsigned)a.msPerTimeStep;
	d.eyeGDecay = expf(-eyeMS / p.eyeGDecayTau);
	d.eyeGInc = p.eyeGInc;
	d.eyeGShift = p.eyeGShift;
	d.eyeGLeak = p.eyeGLeakRaw / (6 - eyeMS);
	d.eyeMaxAmp = p.eyeMaxAmp;
	if (sv) {
		d.svMean = sv->svMean; d.svRelaxed = sv->svRelaxed; d.svExcited = sv->svExcited; d.svValues = sv->svValues;
		d.svSteps = sv->svSteps; d.svVars = sv->svVars; d.svPer = sv->svPer;
		d.svLo = sv->svLo; d.svHi = sv->svHi; d.svDen = sv->svDen; d.svMaxPossible = sv->svMaxPossible;
		d.svNorm = sv->svNorm;
	}
	for (void *q : {(void *)d.freqBG, (void *)d.freqCSTonic, (void *)d.freqCSPhasic, (void *)d.mfThresh,
			(void *)d.plastState, (void *)d.curSteps, (void *)d.ctlSlots, (void *)d.ncPSH, (void *)d.pcPSH, (void *)d.eyelid, (void *)d.eyeG, (void *)d.eyeVm})
		if (!q) return "device allocation failed";
	DevProtocol *dp = upload(&d, 1);
	if (!dp) return "device allocation failed";
	hProto_ = d;
	h_.proto = dp;
	h_.protoSlots = d.ctlSlots;
	CK(cudaMemcpyAsync(dNet_.ptr, &h_, sizeof(DevNet), cudaMemcpyHostToDevice, s), "uploading the network descriptor");
	protocolPrimeKernel<<<1, kTailThreads, 0, s>>>(devPtr());
	CK(cudaGetLastError(), "starting the protocol");
	CK(cudaStreamSynchronize(s), "starting the protocol");
	return "";
}

size_t Network::recordBytes(int kind) const
{
	if (!h_.proto) return 0;
	const size_t nd = std::max<uint32_t>(1, hProto_.numDataTrials);
	switch (kind) {
	case CBM_REC_NC_PSH: return 4 * nd * hProto_.nBins * h_.numNC;
	case CBM_REC_PC_PSH: return 4 * nd * hProto_.nBins * h_.numPC;
	case CBM_REC_EYELID: return 4 * nd * (size_t)hProto_.recLen;
	case CBM_REC_GR_PSH: return hProto_.grPSH ? 2ull * hProto_.nBins * h_.numGR : 0;
	default: break;
	}
	size_t off, n;
	return trialDataRecord(kind, &off, &n) ? 4 * n : 0;
}

// Where a trial-data record sits in its buffer (elements), or false for
// another kind or while the trial data is not recorded.
bool Network::trialDataRecord(int kind, size_t *offset, size_t *count) const
{
	if (!hProto_.tdPSH) return false;
	const size_t B = hProto_.nBins, R = (size_t)hProto_.numDataTrials * ((uint32_t)hProto_.recLen / 32);
	const uint32_t psh[9] = {h_.numGO, h_.numGO, h_.numGO, h_.numGO, h_.numMF, h_.numSC, h_.numBC, h_.numPC, h_.numIO};
	const uint32_t raster[6] = {h_.numGO, h_.numSC, h_.numBC, h_.numPC, h_.numNC, h_.numIO};
	size_t off = 0;
	if (kind >= CBM_REC_PSH_GO && kind <= CBM_REC_PSH_IO) {
		for (int k = 0; k < kind - CBM_REC_PSH_GO; k++) off += B * psh[k];
		*offset = off;
		*count = B * psh[kind - CBM_REC_PSH_GO];
		return true;
	}
	if (kind >= CBM_REC_RASTER_GO && kind <= CBM_REC_RASTER_IO) {
		for (int k = 0; k < kind - CBM_REC_RASTER_GO; k++) off += R * raster[k];
		*offset = off;
		*count = R * raster[kind - CBM_REC_RASTER_GO];
		return true;
	}
	return false;
}

std::string Network::recordTrialData(cudaStream_t s)
{
	if (!h_.proto) return "the trial data records a running protocol: set one first";
	if (hProto_.tdPSH) return "";
	if (hProto_.recLen < 32) return "the recording window must be at least 32 steps for the trial-data rasters";
	const size_t B = hProto_.nBins, R = (size_t)hProto_.numDataTrials * ((uint32_t)hProto_.recLen / 32);
	const size_t nPSH = B * (4ull * h_.numGO + h_.numMF + h_.numSC + h_.numBC + h_.numPC + h_.numIO);
	const size_t nRaster = R * ((size_t)h_.numGO + h_.numSC + h_.numBC + h_.numPC + h_.numNC + h_.numIO);
	float *psh = alloc<float>(nPSH);  // zeroed
	uint32_t *raster = alloc<uint32_t>(std::max<size_t>(1, nRaster));
	if (!psh || !raster) return "device allocation failed";
	hProto_.tdPSH = psh;
	hProto_.tdRaster = raster;
	CK(cudaMemcpyAsync(h_.proto, &hProto_, sizeof(DevProtocol), cudaMemcpyHostToDevice, s), "uploading the protocol");
	CK(cudaStreamSynchronize(s), "uploading the protocol");
	return "";
}

std::string Network::recordGR(cudaStream_t s)
{
	if (!h_.proto) return "the GR histogram records a running protocol: set one first";
	if (hProto_.grPSH) return "";
	if ((uint64_t)hProto_.binSteps * std::max<uint32_t>(1, hProto_.numDataTrials) > 65535)
		return "GR histogram counts are 16-bit: binSteps x numDataTrials must be at most 65535";
	uint16_t *c = alloc<uint16_t>((size_t)hProto_.nBins * h_.numGR);  // zeroed
	if (!c) return "device allocation failed";
	hProto_.grPSH = c;
	CK(cudaMemcpyAsync(h_.proto, &hProto_, sizeof(DevProtocol), cudaMemcpyHostToDevice, s), "uploading the protocol");
	CK(cudaStreamSynchronize(s), "uploading the protocol");
	return "";
}

std::string Network::readRecord(int kind, void *dst, size_t bytes, cudaStream_t s)
{
	if (!h_.proto) return "no protocol is running";
	const size_t need = recordBytes(kind);
	if (!need) return "unknown record kind";
	if (bytes != need) return "record size mismatch";
	size_t off = 0, n = 0;
	const void *src = kind == CBM_REC_NC_PSH ? (const void *)hProto_.ncPSH
		: kind == CBM_REC_PC_PSH ? (const void *)hProto_.pcPSH
		: kind == CBM_REC_GR_PSH ? (const void *)hProto_.grPSH
		: kind == CBM_REC_EYELID ? (const void *)hProto_.eyelid
		: !trialDataRecord(kind, &off, &n) ? nullptr
		: kind <= CBM_REC_PSH_IO ? (const void *)(hProto_.tdPSH + off) : (const void *)(hProto_.tdRaster + off);
	if (!src) return "unknown record kind";
	CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "reading a record");
	CK(cudaStreamSynchronize(s), "reading a record");
	return "";
}

std::string Network::uploadMFBits(const uint32_t *bits, uint64_t firstSlot, uint64_t n, cudaStream_t s)
{
	if (firstSlot + n > h_.mfRing) return "MF ring too small";
	CK(cudaMemcpyAsync((void *)(h_.mfBits + firstSlot * h_.mfWords), bits, n * h_.mfWords * 4,
			cudaMemcpyHostToDevice, s), "uploading MF spikes");
	return "";
}

size_t Network::fieldBytes(Field f) const
{
	const DevNet &h = h_;
	switch (f) {
	case F_AP_GR: return h.numGR;
	case F_VM_GR: case F_GESUM_GR: case F_GISUM_GR: case F_APBUF_GR: case F_THRESH_GR: case F_GKCA_GR: return 4ull * h.numGR;
	case F_HIST_GR: return 8ull * h.numGR;
	case F_AP_GO: return h.numGO;
	case F_VM_GO: case F_APBUF_GO: case F_SUM_GR_INPUT_GO: case F_SUM_GO_INPUT_GO: case F_GO_OUT_SCALE_GOGO: return 4ull * h.numGO;
	case F_AP_SC: return h.numSC;
	case F_VM_SC: case F_APBUF_SC: return 4ull * h.numSC;
	case F_HIST_MF: return h.numMF;
	case F_APBUF_MF: return 4ull * h.numMF;
	case F_AP_BC: return h.numBC;
	case F_VM_BC: case F_APBUF_BC: return 4ull * h.numBC;
	case F_AP_PC: return h.numPC;
	case F_VM_PC: case F_APBUF_PC: return 4ull * h.numPC;
	case F_AP_IO: return h.numIO;
	case F_VM_IO: case F_APBUF_IO: return 4ull * h.numIO;
	case F_AP_NC: return h.numNC;
	case F_VM_NC: case F_APBUF_NC: return 4ull * h.numNC;
	case F_PFPC_WEIGHT: return 4ull * h.numGR;
	case F_MFNC_WEIGHT: return 4ull * h.numNC * h.numpNCfromMFtoNC;
	default: return 0;
	}
}

std::string Network::exportField(Field f, uint32_t zone, void *dst, size_t bytes, cudaStream_t s)
{
	if (bytes != fieldBytes(f) || bytes == 0) return "export buffer size mismatch";
	if (zone >= h_.numZones) return "zone out of range";
	const DevNet &h = h_;
	const DevZone &Q = h.zones[zone];
	const void *src = nullptr;
	switch (f) {
	case F_AP_GR: {
		uint8_t *tmp = nullptr;
		CK(cudaMallocAsync((void **)&tmp, h.numGR, s), "export scratch");
		extractSpikesKernel<<<(h.numGR + 255) / 256, 256, 0, s>>>(h.apBufGR, tmp, h.numGR);
		CK(cudaMemcpyAsync(dst, tmp, h.numGR, cudaMemcpyDeviceToHost, s), "export");
		CK(cudaFreeAsync(tmp, s), "export scratch");
		return "";
	}
	case F_VM_GR: src = h.vGR; break;
	case F_GESUM_GR: src = h.gESum; break;
	case F_GISUM_GR: src = h.gISum; break;
	case F_APBUF_GR: src = h.apBufGR; break;
	case F_HIST_GR: src = h.historyGR; break;
	case F_THRESH_GR: src = h.threshGR; break;
	case F_GKCA_GR: src = h.gKCaGR; break;
	case F_AP_GO: src = h.apGO; break;
	case F_VM_GO: src = h.vGO; break;
	case F_APBUF_GO: src = h.apBufGO; break;
	case F_SUM_GR_INPUT_GO: src = h.sumGRInputGO; break;
	case F_SUM_GO_INPUT_GO: src = h.sumInputGOGABASynDepGO; break;
	case F_GO_OUT_SCALE_GOGO: src = h.goGABAOutSynScaleGOGO; break;
	case F_AP_SC: src = h.apSC; break;
	case F_VM_SC: src = h.vSC; break;
	case F_APBUF_SC: src = h.apBufSC; break;
	case F_HIST_MF: src = h.histMF; break;
	case F_APBUF_MF: src = h.apBufMF; break;
	case F_AP_BC: src = Q.apBC; break;
	case F_VM_BC: src = Q.vBC; break;
	case F_APBUF_BC: src = Q.apBufBC; break;
	case F_AP_PC: src = Q.apPC; break;
	case F_VM_PC: src = Q.vPC; break;
	case F_APBUF_PC: src = Q.apBufPC; break;
	case F_AP_IO: src = Q.apIO; break;
	case F_VM_IO: src = Q.vIO; break;
	case F_APBUF_IO: src = Q.apBufIO; break;
	case F_AP_NC: src = Q.apNC; break;
	case F_VM_NC: src = Q.vNC; break;
	case F_APBUF_NC: src = Q.apBufNC; break;
	case F_PFPC_WEIGHT: src = Q.w; break;
	case F_MFNC_WEIGHT: src = Q.mfSynWeightNC; break;
	default: return "unknown field";
	}
	CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "export");
	return "";
}

// sumInputsNew's halving tree over one PC row's partial sums
static float hostRowTree(std::vector<float> v)
{
	for (size_t h = v.size() / 2; h >= 1; h /= 2)
		for (size_t t = 0; t < h; t++) v[t] = v[t] + v[t + h];
	return v[0];
}

std::string Network::writeToState(cudaStream_t s)
{
	CK(cudaStreamSynchronize(s), "sync before writeToState");
	const DevNet &h = h_;
	auto D = [&](const char *n, int z, const void *src) -> std::string {
		NamedArray *x = st_->find(n, z);
		CK(cudaMemcpy(x->bytes.data(), src, x->bytes.size(), cudaMemcpyDeviceToHost), n);
		return "";
	};
	// InNet::writeToState (innet.cpp:608-667)
	{
		std::vector<uint32_t> ab(h.numGR);
		CK(cudaMemcpy(ab.data(), h.apBufGR, 4ull * h.numGR, cudaMemcpyDeviceToHost), "apBufGR");
		uint8_t *apGR = st_->find("apGR")->as<uint8_t>();
		// outputGRGPU holds zeros until the first step (innet.cpp:477)
		for (uint32_t i = 0; i < h.numGR; i++) apGR[i] = hostT_ ? (uint8_t)(ab[i] & 1u) : 0;
		memcpy(st_->find("apBufGR")->bytes.data(), ab.data(), 4ull * h.numGR);
	}
	CKS(D("gMFSumGR", -1, h.gESum)); CKS(D("gGOSumGR", -1, h.gISum)); CKS(D("threshGR", -1, h.threshGR));
	CKS(D("vGR", -1, h.vGR)); CKS(D("gKCaGR", -1, h.gKCaGR)); CKS(D("historyGR", -1, h.historyGR));
	{
		const uint32_t buf = (uint32_t)((hostT_ + 2) % 3);
		CKS(D("inputSumPFSC", -1, h.scCount + (size_t)buf * h.numSC));
	}
	// state the reference keeps on the host, here on the device
	CKS(D("histMF", -1, h.histMF)); CKS(D("apBufMF", -1, h.apBufMF));
	CKS(D("apGO", -1, h.apGO)); CKS(D("apBufGO", -1, h.apBufGO)); CKS(D("vGO", -1, h.vGO));
	CKS(D("vCoupleGO", -1, h.vCoupleGO)); CKS(D("threshCurGO", -1, h.threshCurGO));
	CKS(D("inputMFGO", -1, h.inputMFGO)); CKS(D("inputGOGO", -1, h.inputGOGO));
	CKS(D("inputGOGABASynDepGO", -1, h.inputGOGABASynDepGO)); CKS(D("goGABAOutSynScaleGOGO", -1, h.goGABAOutSynScaleGOGO));
	CKS(D("gMFGO", -1, h.gMFGO)); CKS(D("gGRGO", -1, h.gGRGO)); CKS(D("gGOGO", -1, h.gGOGO));
	CKS(D("gMGluRGO", -1, h.gMGluRGO)); CKS(D("gMGluRIncGO", -1, h.gMGluRIncGO)); CKS(D("mGluRGO", -1, h.mGluRGO));
	CKS(D("gluGO", -1, h.gluGO));
	CKS(D("apSC", -1, h.apSC)); CKS(D("apBufSC", -1, h.apBufSC)); CKS(D("gPFSC", -1, h.gPFSC));
	CKS(D("threshSC", -1, h.threshSC)); CKS(D("vSC", -1, h.vSC));
	for (uint32_t z = 0; z < h.numZones; z++) {
		const DevZone &Q = h.zones[z];
		int zi = (int)z;
		// MZone::writeToState (mzone.cpp:139-147)
		CKS(D("pfSynWeightPC", zi, Q.w));
		{
			const uint32_t buf = (uint32_t)((hostT_ + 2) % 3);
			std::vector<float> part((size_t)h.numPC * h.bs);
			CK(cudaMemcpy(part.data(), Q.pcPartial + (size_t)buf * h.numPC * h.bs, part.size() * 4, cudaMemcpyDeviceToHost), "pcPartial");
			float *dst = st_->find("inputSumPFPC", zi)->as<float>();
			for (uint32_t pc = 0; pc < h.numPC; pc++)
				dst[pc] = hostRowTree(std::vector<float>(part.begin() + (size_t)pc * h.bs, part.begin() + (size_t)(pc + 1) * h.bs));
		}
		CKS(D("apBC", zi, Q.apBC)); CKS(D("apBufBC", zi, Q.apBufBC)); CKS(D("inputPCBC", zi, Q.inputPCBC));
		CKS(D("gPFBC", zi, Q.gPFBC)); CKS(D("gPCBC", zi, Q.gPCBC)); CKS(D("threshBC", zi, Q.threshBC));
		CKS(D("vBC", zi, Q.vBC));
		CKS(D("apPC", zi, Q.apPC)); CKS(D("apBufPC", zi, Q.apBufPC)); CKS(D("inputBCPC", zi, Q.inputBCPC));
		CKS(D("inputSCPC", zi, Q.inputSCPC)); CKS(D("gPFPC", zi, Q.gPFPC)); CKS(D("gBCPC", zi, Q.gBCPC));
		CKS(D("gSCPC", zi, Q.gSCPC)); CKS(D("vPC", zi, Q.vPC)); CKS(D("threshPC", zi, Q.threshPC));
		CKS(D("histPCPopAct", zi, Q.histPCPopAct));
		CKS(D("apIO", zi, Q.apIO)); CKS(D("apBufIO", zi, Q.apBufIO)); CKS(D("inputNCIO", zi, Q.inputNCIO));
		CKS(D("gNCIO", zi, Q.gNCIO)); CKS(D("threshIO", zi, Q.threshIO)); CKS(D("vIO", zi, Q.vIO));
		CKS(D("vCoupleIO", zi, Q.vCoupleIO)); CKS(D("pfPCPlastTimerIO", zi, Q.pfPCPlastTimerIO));
		CKS(D("apNC", zi, Q.apNC)); CKS(D("apBufNC", zi, Q.apBufNC)); CKS(D("inputPCNC", zi, Q.inputPCNC));
		CKS(D("inputMFNC", zi, Q.inputMFNC)); CKS(D("gPCNC", zi, Q.gPCNC)); CKS(D("gPCScaleNC", zi, Q.gPCScaleNC));
		CKS(D("mfSynWeightNC", zi, Q.mfSynWeightNC)); CKS(D("gmaxNMDAofMFtoNC", zi, Q.gmaxNMDAofMFtoNC));
		CKS(D("gmaxAMPAofMFtoNC", zi, Q.gmaxAMPAofMFtoNC)); CKS(D("gMFNMDANC", zi, Q.gMFNMDANC));
		CKS(D("gMFAMPANC", zi, Q.gMFAMPANC)); CKS(D("threshNC", zi, Q.threshNC)); CKS(D("vNC", zi, Q.vNC));
		CKS(D("synIOPReleaseNC", zi, Q.synIOPReleaseNC));
		uint32_t sc[5];
		CK(cudaMemcpy(sc, Q.scal, sizeof(sc), cudaMemcpyDeviceToHost), "zone scalars");
		ZoneScalars &zs = st_->zoneScalars[z];
		zs.histPCPopActSum = sc[0]; zs.histPCPopActCurBinN = sc[1]; zs.pcPopAct = sc[2];
		zs.noLTPMFNC = (uint8_t)sc[3]; zs.noLTDMFNC = (uint8_t)sc[4];
		zs.errDrive = ctl.errDrive[z];
	}
	return "";
}

std::string Network::resetGOGODepression(cudaStream_t s)
{
	std::vector<float> ones(h_.numGO, 1.0f);
	CK(cudaMemcpyAsync(h_.inputGOGABASynDepGO, ones.data(), 4ull * h_.numGO, cudaMemcpyHostToDevice, s), "reset");
	CK(cudaMemsetAsync(h_.goGABAOutSynScaleGOGO, 0, 4ull * h_.numGO, s), "reset");
	CK(cudaStreamSynchronize(s), "reset");
	float *a = st_->find("inputGOGABASynDepGO")->as<float>();
	float *b = st_->find("goGABAOutSynScaleGOGO")->as<float>();
	for (uint32_t i = 0; i < h_.numGO; i++) { a[i] = 1.0f; b[i] = 0.0f; }
	return "";
}

// --------------------------------------------------------------- Simulator
Simulator::~Simulator()
{
	dropGraphs();
	if (flushBuf_.ptr) cudaFree(flushBuf_.ptr);
	if (hExport_) cudaFreeHost(hExport_);
	for (cudaEvent_t e : stepEv_) if (e) cudaEventDestroy(e);
	for (Network *n : nets_) delete n;
	for (DeviceBuf *b : {&dNetPtrs_, &dBlockOffset_, &dTBasePtrs_, &dStageBytes_, &dCellOffset_, &dVecUnitOffset_,
			&dVecPcOffset_, &dVecClaim_, &dExitCount_})
		if (b->ptr) cudaFree(b->ptr);
	if (s0_) cudaStreamDestroy(s0_);
	if (s1_) cudaStreamDestroy(s1_);
	for (cudaEvent_t e : {fork_, join_, ev0_, ev1_, tev0_, tev1_}) if (e) cudaEventDestroy(e);
	for (cudaEvent_t e : passEv_) cudaEventDestroy(e);
	for (cudaEvent_t e : tailEv_) cudaEventDestroy(e);
}

std::string Simulator::create(const std::vector<State *> &states, const std::vector<std::vector<int>> &seeds,
		int device, uint32_t mfRing, const std::vector<uint32_t> *mfSeeds)
{
	device_ = device;
	// host-side validation first, so a malformed network is rejected
	// before any device work
	for (const State *st : states) CKS(checkNetwork(*st));
	CK(cudaSetDevice(device), "selecting the device");
	// The small-cell CTAs (one SM's register file each) go on the
	// high-priority stream so that they are dispatched before the GR pass
	// fills every SM; graphs keep the per-node priority.
	int leastPrio = 0, greatestPrio = 0;
	CK(cudaDeviceGetStreamPriorityRange(&leastPrio, &greatestPrio), "stream priorities");
	CK(cudaStreamCreateWithPriority(&s0_, cudaStreamNonBlocking, leastPrio), "stream");
	CK(cudaStreamCreateWithPriority(&s1_, cudaStreamNonBlocking, greatestPrio), "stream");
	CK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "event");
	CK(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "event");
	CK(cudaEventCreate(&ev0_), "event");
	CK(cudaEventCreate(&ev1_), "event");
	CK(cudaEventCreate(&tev0_), "event");
	CK(cudaEventCreate(&tev1_), "event");
	std::vector<DevNet *> ptrs;
	std::vector<uint64_t *> tb;
	std::vector<uint32_t> offs, stage;
	for (size_t i = 0; i < states.size(); i++) {
		Network *n = new Network();
		nets_.push_back(n);
		std::vector<int> sd = i < seeds.size() ? seeds[i] : std::vector<int>();
		CKS(n->build(states[i], sd, mfRing, mfSeeds && i < mfSeeds->size() ? (*mfSeeds)[i] : 0));
		offs.push_back(passBlocks_);
		passBlocks_ += n->passBlocks();
		ptrs.push_back(n->devPtr());
		tb.push_back(n->dev().tBase);
		stage.push_back(n->stageBytes());
		passSmem_ = std::max(passSmem_, n->passSmemBytes());
		tailSmem_ = std::max(tailSmem_, n->tailSmemBytes());
	}
	auto up = [&](DeviceBuf &b, const void *src, size_t bytes) -> std::string {
		CK(cudaMalloc(&b.ptr, bytes), "allocating launch tables");
		b.bytes = bytes;
		CK(cudaMemcpy(b.ptr, src, bytes, cudaMemcpyHostToDevice), "uploading launch tables");
		return "";
	};
	CKS(up(dNetPtrs_, ptrs.data(), ptrs.size() * sizeof(DevNet *)));
	CKS(up(dBlockOffset_, offs.data(), offs.size() * sizeof(uint32_t)));
	CKS(up(dTBasePtrs_, tb.data(), tb.size() * sizeof(uint64_t *)));
	CKS(up(dStageBytes_, stage.data(), stage.size() * sizeof(uint32_t)));
	const uint32_t zero = 0;
	CKS(up(dExitCount_, &zero, sizeof(zero)));
	if (passSmem_ > 48 * 1024)
		CK(cudaFuncSetAttribute(grPassKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)passSmem_), "pass smem");
	if (tailSmem_ > 48 * 1024)
		CK(cudaFuncSetAttribute(tailKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tailSmem_), "tail smem");

	// GR-pass kernel: the per-tile TMA pass with a default geometry where
	// every network has 32-cell tile rows, else the plain pass.
	// CBM_PASS_TMA="W,RW,S,B,M" / CBM_PASS_PERSIST="W,S,B,M" pick another
	// compiled geometry (tuning), CBM_PASS_TMA=0 the plain pass kernel.
	PassGeometry g;
	if (const char *env = getenv("CBM_PASS_PERSIST")) {
		if (strcmp(env, "0") != 0) {
			g.kind = 2;
			if (sscanf(env, "%d,%d,%d,%d", &g.W, &g.S, &g.B, &g.M) != 4) return "CBM_PASS_PERSIST must be W,S,B,M";
			return usePassGeometry(g);
		}
	}
	if (const char *env = getenv("CBM_PASS_TMA")) {
		if (!strcmp(env, "0")) { g.kind = 0; return usePassGeometry(g); }
		g.kind = 1;
		if (sscanf(env, "%d,%d,%d,%d,%d", &g.W, &g.RW, &g.S, &g.B, &g.M) != 5) return "CBM_PASS_TMA must be W,RW,S,B,M";
		return usePassGeometry(g);
	}
	const std::vector<PassGeometry> cands = passCandidates();
	return usePassGeometry(cands.front());
}

std::vector<PassGeometry> Simulator::passCandidates() const
{
	// the default first: 4 consumer warps of 1 row, 4 stages, 4 CTAs/SM,
	// slot loops for at most 4 slots (8,1,3,2 with open slot loops past 4)
	std::vector<PassGeometry> out;
	// the vector pass where it applies (networks of the compiled shape),
	// after the per-tile default: on the 1M eyelid network it measured
	// 31 us flushed against 24 us for the per-tile pass, its units being two
	// dependent round trips each where the per-tile pass keeps four stages
	// of loads in flight.  CBM_PASS_VEC=0 leaves it out, CBM_PASS_VEC=1 puts
	// it first.
	const char *vecEnv = getenv("CBM_PASS_VEC");
	bool vec = !nets_.empty() && !(vecEnv && !strcmp(vecEnv, "0"));
	for (Network *n : nets_) vec = vec && passVecCapable(n->dev());
	PassGeometry v;
	v.kind = 3;
	const bool vecFirst = vec && vecEnv && !strcmp(vecEnv, "1");
	if (vecFirst) out.push_back(v);
	bool tma = !nets_.empty();
	uint32_t minRows = UINT32_MAX, maxSlots = 0;
	for (Network *n : nets_) {
		tma = tma && n->passTmaCapable();
		minRows = std::min(minRows, n->passRows());
		maxSlots = std::max({maxSlots, n->dev().nMFSlots, n->dev().nGOSlots, n->dev().nOutTma});
	}
	if (tma) {
		PassGeometry d;
		d.kind = 1;
		if (maxSlots <= 4) { d.W = 4; d.RW = 1; d.S = 4; d.B = 4; d.M = 4; }
		else { d.W = 8; d.RW = 1; d.S = 3; d.B = 2; d.M = 0; }
		// Networks whose per-step working set stays in L2 (GR state read and
		// written, synapse slots, delays, weights: about 75 B a GR) are bound
		// by issue and latency: two rows per consumer warp.  On the 1M-GR
		// network 4,2,2,4 ran 9.6 % faster back to back than 4,1,4,4 (1.9 %
		// slower after an L2 flush); where the state streams from HBM (the
		// dense 4M network) single rows and a deeper ring are faster.
		int l2 = 0;
		cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device_);
		double set = 0;
		for (Network *n : nets_) {
			const DevNet &h = n->dev();
			set += (48.0 + 2.0 * (h.nMFSlots + h.nGOSlots + h.nOutTma) + 1.0 + 4.0 * h.numZones) * h.numGR;
		}
		if (maxSlots <= 4 && set <= 0.75 * l2 && 8u <= minRows) {
			PassGeometry r = d;
			r.RW = 2;
			r.S = 2;
			out.push_back(r);
		}
		if ((uint32_t)(d.W * d.RW) <= minRows) out.push_back(d);
		if (vec && !vecFirst) out.push_back(v);
		for (int i = 0; i < passTmaConfigCount(); i++) {
			PassGeometry c;
			c.kind = 1;
			passTmaConfig(i, &c.W, &c.RW, &c.S, &c.B, &c.M);
			if ((uint32_t)(c.W * c.RW) > minRows || (c.M > 0 && maxSlots > (uint32_t)c.M)) continue;
			bool listed = false;
			for (const PassGeometry &o : out)
				listed = listed || (o.kind == 1 && c.W == o.W && c.RW == o.RW && c.S == o.S && c.B == o.B && c.M == o.M);
			if (listed) continue;
			out.push_back(c);
		}
	}
	if (vec && !vecFirst && !tma) out.push_back(v);
	PassGeometry plain;
	plain.kind = 0;
	out.push_back(plain);
	return out;
}

std::string Simulator::usePassGeometry(const PassGeometry &g)
{
	CK(cudaSetDevice(device_), "selecting the device");
	uint32_t minRows = UINT32_MAX, maxSlots = 0;
	bool capable = !nets_.empty();
	uint32_t maxSlotsTile = 0;  // the per-tile pass streams nOutTma GR->GO planes
	for (Network *n : nets_) {
		capable = capable && n->passTmaCapable();
		minRows = std::min(minRows, n->passRows());
		maxSlots = std::max({maxSlots, n->dev().nMFSlots, n->dev().nGOSlots, n->dev().nOutSlots});
		maxSlotsTile = std::max({maxSlotsTile, n->dev().nMFSlots, n->dev().nGOSlots, n->dev().nOutTma});
	}
	for (Network *n : nets_) { n->outBytes_ = 4; n->outPlanes_ = n->dev().nOutSlots; n->ovUsed_ = 0; }
	// leaving the vector pass: the last step's PF->PC reduction is still pair
	// sums, and the small-cell update goes back to partial sums
	if (passVec_ && g.kind != 3)
		for (Network *n : nets_) CKS(n->setPcSumMode(false, s0_));
	if (g.kind == 3 && nets_.size() > 1) {
		for (Network *n : nets_)
			if (!passVecCapable(n->dev())) return "the vector GR pass runs networks of its compiled shape";
		const void *fn = passVecBatchKernel();
		if (!dVecUnitOffset_.ptr) {
			std::vector<uint32_t> units(1, 0), pcs(1, 0);
			for (Network *n : nets_) {
				units.push_back(units.back() + n->dev().numGR / 128u);
				pcs.push_back(pcs.back() + n->dev().numPC);
			}
			auto up = [&](DeviceBuf &b, const std::vector<uint32_t> &v) -> std::string {
				CK(cudaMalloc(&b.ptr, v.size() * sizeof(uint32_t)), "allocating vector-pass tables");
				b.bytes = v.size() * sizeof(uint32_t);
				CK(cudaMemcpy(b.ptr, v.data(), b.bytes, cudaMemcpyHostToDevice), "uploading vector-pass tables");
				return "";
			};
			CKS(up(dVecUnitOffset_, units));
			CKS(up(dVecPcOffset_, pcs));
			CKS(up(dVecClaim_, std::vector<uint32_t>(4, 0)));
		}
		int perSM = 0, numSMs = 0;
		CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, 32 * kVecWarps, 0), "pass occupancy");
		CK(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device_), "SM count");
		uint32_t units = 0;
		for (Network *n : nets_) units += n->dev().numGR / 128u;
		const uint32_t claims = (units + kVecBatchClaim - 1) / kVecBatchClaim;
		passGrid_ = std::max<uint32_t>(1, std::min<uint32_t>((claims + kVecWarps - 1) / kVecWarps,
				(uint32_t)std::max(1, perSM) * (uint32_t)numSMs));
		CK(cudaMemset(dVecClaim_.ptr, 0, dVecClaim_.bytes), "pass claim counters");
		for (Network *n : nets_) CKS(n->setPcSumMode(true, s0_));
		passTmaFn_ = fn;
		passVec_ = true;
		passPersistent_ = false;
		passTmaW_ = kVecWarps - 1;
		passTmaR_ = passTmaS_ = 0;
		passTmaSmem_ = 0;
		passGeom_ = g;
		dropGraphs();
		return "";
	}
	if (g.kind == 3) {
		if (nets_.size() != 1 || !passVecCapable(nets_[0]->dev()))
			return "the vector GR pass runs networks of its compiled shape";
		Network &n = *nets_[0];
		const size_t smem = passVecSmemBytes(n.dev());
		const void *fn = passVecKernel();
		CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "pass smem");
		int perSM = 0, numSMs = 0;
		CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, 32 * kVecWarps, smem), "pass occupancy");
		CK(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device_), "SM count");
		// units claimed at a time (CBM_VEC_CLAIM, tuning; default kVecClaim)
		vecClaim_ = kVecClaim;
		if (const char *env = getenv("CBM_VEC_CLAIM")) {
			const int c = atoi(env);
			if (c < 1 || c > 64) return "CBM_VEC_CLAIM must be 1..64";
			vecClaim_ = (uint32_t)c;
		}
		// every CTA resident from the start: the small-cell kernel's two
		// CTAs hold an SM each while the pass runs
		const uint32_t claims = (n.dev().numGR / 128u + vecClaim_ - 1) / vecClaim_;
		const uint32_t sms = (uint32_t)std::max(1, numSMs - 2);
		passGrid_ = std::max<uint32_t>(1, std::min<uint32_t>((claims + kVecWarps - 1) / kVecWarps,
				(uint32_t)std::max(1, perSM) * sms)) + passVecReduceCTAs(n.dev());
		// claim counters from zero (another pass kind may have run meanwhile)
		CK(cudaMemset(n.dev().passClaim, 0, 4 * sizeof(uint32_t)), "pass claim counters");
		CKS(n.setPcSumMode(true, s0_));
		passTmaFn_ = fn;
		passVec_ = true;
		passPersistent_ = false;
		passTmaW_ = kVecWarps - 1;  // launchPass's block is 32 * (W + 1) threads
		passTmaR_ = passTmaS_ = 0;
		passTmaSmem_ = smem;
		passGeom_ = g;
		dropGraphs();
		return "";
	}
	passVec_ = false;
	if (g.kind == 0) {
		passTmaFn_ = nullptr;
		passPersistent_ = false;
		passTmaW_ = passTmaR_ = passTmaS_ = 0;
		passGeom_ = g;
		dropGraphs();
		return "";
	}
	if (!capable) return "the TMA GR pass needs tiles of 32-cell rows in every network";
	if (g.M > 0 && (g.kind == 1 ? maxSlotsTile : maxSlots) > (uint32_t)g.M)
		return "a network has more synapse slots than the geometry's slot bound";
	const void *fn = nullptr;
	uint32_t R = 0, threads = 0, grid = passBlocks_;
	size_t smem = 0;
	if (g.kind == 1) {
		// the shape-specialised instance when every network has that shape
		// (CBM_PASS_SHAPE=0 keeps the run-time-shape kernel: testing)
		int shape = g.M == 4 ? 1 : 0;
		for (Network *n : nets_) if (passShapeOf(n->dev()) != 1) shape = 0;
		if (const char *env = getenv("CBM_PASS_SHAPE"))
			if (!strcmp(env, "0")) shape = 0;
		fn = passTmaKernelFor(g.W, g.RW, g.S, g.B, g.M, shape);
		if (!fn) return "per-tile GR-pass geometry not compiled in";
		R = (uint32_t)(g.W * g.RW);
		if (R > minRows) return "more rows per stage than a tile has";
		for (Network *n : nets_) smem = std::max(smem, n->passTmaSmemBytes(R, (uint32_t)g.S, shape == 1 ? 2u : 4u));
		for (Network *n : nets_) {
			n->outBytes_ = shape == 1 ? 2u : 4u;
			n->outPlanes_ = n->dev().nOutTma;
			n->ovUsed_ = n->ovEntries_;
		}
		threads = 32u * (g.W + 1);
	} else {
		if (nets_.size() != 1) return "the persistent GR pass runs one network";
		if (nets_[0]->dev().ovStart) return "the persistent GR pass streams every GR->GO slot; this network has per-tile lists";
		fn = passPersistentKernelFor(g.W, g.S, g.B, g.M);
		if (!fn) return "persistent GR-pass geometry not compiled in";
		R = (uint32_t)(2 * g.W);
		if (R > minRows) return "more rows per unit than a tile has";
		Network &n = *nets_[0];
		const PassLayout L = passLayout(R, n.dev().nMFSlots, n.dev().nGOSlots, n.dev().nOutSlots, n.dev().numZones);
		smem = 128 + (size_t)g.S * L.bytes + 16ull * g.S + 4ull * n.dev().numPC * n.dev().numZones +
			32ull * (n.dev().mfWords + n.dev().goWords);
		threads = 32u * (g.W + 1);
	}
	if (smem > 227 * 1024) return "GR-pass geometry needs more shared memory than a CTA has";
	for (Network *n : nets_) CKS(n->buildPassMaps(R));
	CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "pass smem");
	if (g.kind == 2) {
		int perSM = 0, numSMs = 0;
		CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, (int)threads, smem), "pass occupancy");
		CK(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device_), "SM count");
		Network &n = *nets_[0];
		const uint32_t units = n.dev().numPC * n.dev().tilesPerPC * (n.passRows() / R);
		grid = std::min<uint32_t>(units, (uint32_t)std::max(1, perSM) * (uint32_t)numSMs);
	}
	passTmaFn_ = fn;
	passPersistent_ = g.kind == 2;
	passTmaW_ = (uint32_t)g.W;
	passTmaR_ = R;
	passTmaS_ = (uint32_t)g.S;
	passTmaSmem_ = smem;
	passGrid_ = grid;
	passGeom_ = g;
	// captured graphs hold the old kernel
	dropGraphs();
	return "";
}

std::string Simulator::uploadCtl()
{
	for (Network *n : nets_) {
		if (!n->ctlDirty) continue;
		CK(cudaMemcpyAsync(n->h_.ctl, &n->ctl, sizeof(HostCtl), cudaMemcpyHostToDevice, s0_), "uploading setters");
		// the next step consumes the error drive on the device (mzone.cpp:334)
		for (int z = 0; z < kMaxZones; z++) n->ctl.errDrive[z] = 0;
		CK(cudaStreamSynchronize(s0_), "uploading setters");
		n->ctlDirty = false;
	}
	return "";
}

std::string Simulator::enqueueStep(uint32_t k, bool instrument, bool chained)
{
	const DevNet *const *netsArg = (const DevNet *const *)dNetPtrs_.ptr;
	const uint32_t *stageArg = (const uint32_t *)dStageBytes_.ptr;
	const uint32_t *offsArg = (const uint32_t *)dBlockOffset_.ptr;
	int numNetsArg = (int)nets_.size();
	uint32_t stepArg = k;
	const DevNet *net0Arg = nets_.size() == 1 ? nets_[0]->devPtr() : nullptr;
	const uint32_t stage0Arg = nets_.size() == 1 ? nets_[0]->stageBytes() : 0u;
	uint32_t vecClaimArg = vecClaim_;
	auto launchPass = [&](cudaStream_t st, bool dependent) -> std::string {
		if (passTmaFn_) {
			// the per-tile pass takes the single network's descriptor too; the
			// vector pass takes it alone
			// chained single steps: the pass's last CTA waits for the step's
			// small-cell kernel (passExitWait) on this simulator's counter
			uint32_t *exitArg = chained ? (uint32_t *)dExitCount_.ptr : nullptr;
			void *argsTma[] = {&netsArg, &offsArg, &numNetsArg, &stepArg, &net0Arg, &stepMF_, &exitArg};
			void *argsVec[] = {&net0Arg, &stepArg, &vecClaimArg};
			const uint32_t *unitOffArg = (const uint32_t *)dVecUnitOffset_.ptr;
			const uint32_t *pcOffArg = (const uint32_t *)dVecPcOffset_.ptr;
			uint32_t *claimArg = (uint32_t *)dVecClaim_.ptr;
			void *argsVecBatch[] = {&netsArg, &unitOffArg, &pcOffArg, &numNetsArg, &stepArg, &claimArg};
			void **args = !passVec_ ? argsTma : nets_.size() == 1 ? argsVec : argsVecBatch;
			cudaLaunchConfig_t cfg = {};
			cfg.gridDim = dim3(passGrid_);
			cfg.blockDim = dim3(32 * (passTmaW_ + 1));
			cfg.dynamicSmemBytes = passTmaSmem_;
			cfg.stream = st;
			cudaLaunchAttribute attr;
			attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
			attr.val.programmaticStreamSerializationAllowed = 1;
			cfg.attrs = &attr;
			cfg.numAttrs = dependent ? 1 : 0;
			CK(cudaLaunchKernelExC(&cfg, passTmaFn_, args), "launching the GR pass");
		} else {
			cudaLaunchConfig_t cfg = {};
			cfg.gridDim = dim3(passBlocks_);
			cfg.blockDim = dim3(kPassThreads);
			cfg.dynamicSmemBytes = passSmem_;
			cfg.stream = st;
			cudaLaunchAttribute attr;
			attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
			attr.val.programmaticStreamSerializationAllowed = 1;
			cfg.attrs = &attr;
			cfg.numAttrs = dependent ? 1 : 0;
			CK(cudaLaunchKernelEx(&cfg, grPassKernel, netsArg, offsArg, numNetsArg, stepArg), "launching the GR pass");
		}
		return "";
	};
	if (instrument) {
		// fork/join on two streams with external events around each kernel
		CK(cudaEventRecord(fork_, s0_), "fork");
		CK(cudaStreamWaitEvent(s1_, fork_, 0), "fork");
		CK(cudaEventRecordWithFlags(passEv_[2 * k], s0_, cudaEventRecordExternal), "pass timing");
		CKS(launchPass(s0_, false));
		CK(cudaEventRecordWithFlags(passEv_[2 * k + 1], s0_, cudaEventRecordExternal), "pass timing");
		CK(cudaEventRecordWithFlags(tailEv_[2 * k], s1_, cudaEventRecordExternal), "tail timing");
		tailKernel<<<2 * (unsigned)nets_.size(), kTailThreads, tailSmem_, s1_>>>(netsArg, stageArg, k, net0Arg, stage0Arg,
				mailboxArg_, stepMF_);
		CK(cudaGetLastError(), "launching the small-cell update");
		CK(cudaEventRecordWithFlags(tailEv_[2 * k + 1], s1_, cudaEventRecordExternal), "tail timing");
		CK(cudaEventRecord(join_, s1_), "join");
		CK(cudaStreamWaitEvent(s0_, join_, 0), "join");
		return recordStep(k);
	}
	if (chained) {
		// steps launched one at a time: the small-cell kernel is the
		// programmatic dependent of the previous step's GR pass and waits for
		// it on the device (pdlWait, cbm_kernels.cuh), so that it is resident
		// when that pass ends; the GR pass follows as before, and its exit
		// wait makes a finished pass a finished step, so no join is needed
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = dim3(2 * (unsigned)nets_.size());
		cfg.blockDim = dim3(kTailThreads);
		cfg.dynamicSmemBytes = tailSmem_;
		cfg.stream = s0_;
		cudaLaunchAttribute attr;
		attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
		attr.val.programmaticStreamSerializationAllowed = 1;
		cfg.attrs = &attr;
		cfg.numAttrs = 1;
		CK(cudaLaunchKernelEx(&cfg, tailKernel, netsArg, stageArg, k, net0Arg, stage0Arg, mailboxArg_, stepMF_),
				"launching the small-cell update");
		CKS(launchPass(s0_, true));
		return recordStep(k);
	}
	// One stream: the small-cell CTAs launch first and let the GR pass start
	// as soon as they are resident (programmatic dependent launch; the two
	// kernels of a step share no buffer), so the pass cannot take the SMs the
	// small-cell CTAs need.  The next step waits for both.
	tailKernel<<<2 * (unsigned)nets_.size(), kTailThreads, tailSmem_, s0_>>>(netsArg, stageArg, k, net0Arg, stage0Arg,
			mailboxArg_, stepMF_);
	CK(cudaGetLastError(), "launching the small-cell update");
	CK(cudaEventRecord(join_, s0_), "join");
	CKS(launchPass(s0_, true));
	CK(cudaStreamWaitEvent(s0_, join_, 0), "join");
	return recordStep(k);
}

std::string Simulator::recordStep(uint32_t k)
{
	// after both kernels of the step: its GR spikes into the histogram, and
	// its small-cell state into the trial data
	if (nets_.size() != 1) {
		if (!dCellOffset_.ptr) return "";  // no instance records its trial data
		trialDataBatchKernel<<<(cellTotal_ + 255) / 256, 256, 0, s0_>>>((const DevNet *const *)dNetPtrs_.ptr,
				(const uint32_t *)dCellOffset_.ptr, (int)nets_.size(), k);
		CK(cudaGetLastError(), "launching the trial-data record");
		return "";
	}
	const DevNet &h = nets_[0]->dev();
	if (nets_[0]->recordsGR()) {
		const uint32_t threads = (h.numGR + 7) / 8;
		grPSHKernel<<<(threads + 255) / 256, 256, 0, s0_>>>(nets_[0]->devPtr(), k);
		CK(cudaGetLastError(), "launching the GR histogram");
	}
	if (nets_[0]->recordsTrialData()) {
		const uint32_t cells = h.numGO + h.numMF + h.numSC + h.numBC + h.numPC + h.numIO + h.numNC;
		trialDataKernel<<<(cells + 255) / 256, 256, 0, s0_>>>(nets_[0]->devPtr(), k);
		CK(cudaGetLastError(), "launching the trial-data record");
	}
	return "";
}

std::string Simulator::launchSteps(uint32_t nsteps)
{
	CK(cudaSetDevice(device_), "selecting the device");
	CKS(uploadCtl());
	// Every step is launched on the stream directly, its two kernels each
	// the programmatic dependent of the kernel before (enqueueStep, chained),
	// so that each is resident before its predecessor ends.  A single-step
	// graph launch queued behind a running one started about seven
	// microseconds after it ended on B200, a plain kernel launch about five.
	// The device step counter is not advanced per step: step k since the
	// last settleSteps() runs with step offset k.  Deferred MF input travels
	// in the launches (mfByParam) or is copied in from its pinned slot first.
	for (uint32_t k = 0; k < nsteps; k++) {
		if (directPending_ >= (1u << 30)) CKS(settleSteps());
		if (pendingMF_ >= 0) {
			Network &n = *nets_[0];
			const int slot = pendingMF_;
			const uint32_t *bits = n.hPinnedBits_ + (size_t)slot * n.h_.mfWords;
			if (mfByParam()) {
				// the launches carry the words: the slot is free once they are issued
				stepMF_.n = n.h_.mfWords;
				memcpy(stepMF_.w, bits, 4ull * n.h_.mfWords);
				n.mfStageUsed_[slot] = false;
			} else {
				CK(cudaMemcpyAsync((void *)n.h_.mfBits, bits, 4ull * n.h_.mfWords, cudaMemcpyHostToDevice, s0_),
						"MF upload");
				CK(cudaEventRecord(n.mfStageEv_[slot], s0_), "MF staging");
			}
			pendingMF_ = -1;
		}
		// one network: its small-cell kernel publishes the step's NC spikes
		mailboxArg_ = nets_.size() == 1 ? nets_[0]->dMailbox_ : nullptr;
		// the chain needs the per-tile pass's exit wait; other pass kinds
		// are launched in plain stream order
		std::string e = enqueueStep(directPending_, false, passTmaFn_ && !passVec_ && !passPersistent_);
		mailboxArg_ = nullptr;
		stepMF_.n = 0;
		if (!e.empty()) return e;
		directPending_++;
		for (Network *n : nets_) n->hostT_ += 1;
	}
	lastStepPublishes_ = nsteps > 0 && nets_.size() == 1;
	directCopySinceStep_ = false;
	return "";
}

bool Simulator::mfByParam() const
{
	// the per-tile GR pass and the small-cell kernel take the words from
	// their launch; the other pass kinds read the MF ring
	return nets_.size() == 1 && nets_[0]->dev().mfWords <= kMFParamWords && passTmaFn_ && !passVec_ &&
		!passPersistent_;
}

std::string Simulator::settleSteps()
{
	if (!directPending_) return "";
	CK(cudaSetDevice(device_), "selecting the device");
	advanceStepKernel<<<1, 64, 0, s0_>>>((uint64_t *const *)dTBasePtrs_.ptr, (int)nets_.size(), directPending_);
	CK(cudaGetLastError(), "advancing the step counter");
	directPending_ = 0;
	return "";
}

std::string Simulator::flushPendingMF()
{
	if (pendingMF_ < 0) return "";
	Network &n = *nets_[0];
	const int k = pendingMF_;
	pendingMF_ = -1;
	directCopySinceStep_ = true;
	CK(cudaMemcpyAsync((void *)n.h_.mfBits, n.hPinnedBits_ + (size_t)k * n.h_.mfWords, 4ull * n.h_.mfWords,
			cudaMemcpyHostToDevice, s0_), "MF upload");
	CK(cudaEventRecord(n.mfStageEv_[k], s0_), "MF staging");
	return "";
}

void Simulator::dropGraphs()
{
	if (graphExec_) { cudaGraphExecDestroy(graphExec_); graphExec_ = nullptr; }
	if (flushKernGraph_) { cudaGraphExecDestroy(flushKernGraph_); flushKernGraph_ = nullptr; }
}

std::string Simulator::setProtocol(size_t i, const cbm_eyelid_protocol &p)
{
	CK(cudaSetDevice(device_), "selecting the device");
	lastStepPublishes_ = false;
	pendingMF_ = -1;  // the protocol drives the MF input from now on
	CKS(settleSteps());
	CKS(uploadCtl());
	CK(cudaStreamSynchronize(s0_), "sync");
	return nets_[i]->setProtocol(p, s0_);
}

std::string Simulator::setStateVarInput(size_t i, const cbm_statevar_input &in)
{
	CK(cudaSetDevice(device_), "selecting the device");
	lastStepPublishes_ = false;
	pendingMF_ = -1;  // the coding drives the MF input from now on
	CKS(settleSteps());
	CKS(uploadCtl());
	CK(cudaStreamSynchronize(s0_), "sync");
	return nets_[i]->setStateVarInput(in, s0_);
}

std::string Simulator::recordGR()
{
	CK(cudaSetDevice(device_), "selecting the device");
	if (nets_.size() != 1) return "the GR histogram is recorded for single-network simulators";
	CK(cudaStreamSynchronize(s0_), "sync");
	const bool was = nets_[0]->recordsGR();
	CKS(nets_[0]->recordGR(s0_));
	if (!was) dropGraphs();  // the step graphs gain the histogram kernel
	return "";
}

std::string Simulator::recordTrialData(size_t i)
{
	CK(cudaSetDevice(device_), "selecting the device");
	if (i >= nets_.size()) return "instance out of range";
	CK(cudaStreamSynchronize(s0_), "sync");
	const bool was = nets_[i]->recordsTrialData();
	CKS(nets_[i]->recordTrialData(s0_));
	if (nets_.size() > 1 && !dCellOffset_.ptr) {
		// the batched record kernel's map from grid threads to instances
		std::vector<uint32_t> off(1, 0);
		for (Network *n : nets_) {
			const DevNet &h = n->dev();
			off.push_back(off.back() + h.numGO + h.numMF + h.numSC + h.numBC + h.numPC + h.numIO + h.numNC);
		}
		CK(cudaMalloc(&dCellOffset_.ptr, off.size() * sizeof(uint32_t)), "cell offsets");
		dCellOffset_.bytes = off.size() * sizeof(uint32_t);
		CK(cudaMemcpy(dCellOffset_.ptr, off.data(), dCellOffset_.bytes, cudaMemcpyHostToDevice), "cell offsets");
		cellTotal_ = off.back();
	}
	if (!was) dropGraphs();  // the step graphs gain the trial-data kernel
	return "";
}

std::string Simulator::stageMF(size_t i, const uint8_t *mf)
{
	Network &n = *nets_[i];
	if (n.hasProtocol()) return "a device protocol drives the MF input of this network";
	const uint32_t W = n.h_.mfWords, M = n.h_.numMF;
	const uint32_t k = n.mfStageNext_++ % kMFStage;
	if (n.mfStageUsed_[k]) {
		// usually long done: a query is cheaper than a synchronisation
		const cudaError_t q = cudaEventQuery(n.mfStageEv_[k]);
		if (q == cudaErrorNotReady) CK(cudaEventSynchronize(n.mfStageEv_[k]), "MF staging");
		else CK(q, "MF staging");
	}
	uint32_t *bits = n.hPinnedBits_ + (size_t)k * W;
	memset(bits, 0, 4ull * W);
	bool raw = false;
	// eight input bytes at a time: the bytes' low bits gathered by one
	// multiply; any byte above 1 marks raw (graded) input
	uint64_t hi = 0;
	uint32_t c = 0;
	for (; c + 8 <= M; c += 8) {
		uint64_t x;
		memcpy(&x, mf + c, 8);
		hi |= x & 0xFEFEFEFEFEFEFEFEull;
		const uint64_t lo = (x | (x >> 1) | (x >> 2) | (x >> 3) | (x >> 4) | (x >> 5) | (x >> 6) | (x >> 7)) &
			0x0101010101010101ull;
		bits[c >> 5] |= (uint32_t)((lo * 0x0102040810204080ull) >> 56) << (c & 31);
	}
	for (; c < M; c++) {
		if (mf[c]) bits[c >> 5] |= 1u << (c & 31);
		if (mf[c] > 1) raw = true;
	}
	if (hi) raw = true;
	if (nets_.size() == 1 && n.h_.mfRing == 1 && !raw && !n.h_.hasMFRaw) {
		// the next single step's graph copies slot k (and records its event)
		pendingMF_ = (int)k;
		n.mfStageUsed_[k] = true;
		return "";
	}
	pendingMF_ = -1;  // this input supersedes a deferred one
	directCopySinceStep_ = true;
	const uint64_t slot = n.hostT_ % n.h_.mfRing;
	CK(cudaMemcpyAsync((void *)(n.h_.mfBits + slot * W), bits, 4ull * W, cudaMemcpyHostToDevice, s0_), "MF upload");
	if (raw || n.h_.hasMFRaw) {
		uint8_t *rb = n.hPinnedRaw_ + (size_t)k * M;
		memcpy(rb, mf, M);
		CK(cudaMemcpyAsync((void *)(n.h_.mfRaw + slot * M), rb, M, cudaMemcpyHostToDevice, s0_), "MF upload");
		if (!n.h_.hasMFRaw) {
			// from now on NC inputs take the raw bytes (mzone.cpp:521)
			n.h_.hasMFRaw = 1;
			CK(cudaMemcpyAsync((char *)n.dNet_.ptr + offsetof(DevNet, hasMFRaw), &n.h_.hasMFRaw, 4,
					cudaMemcpyHostToDevice, s0_), "MF mode");
			CK(cudaStreamSynchronize(s0_), "MF mode");
		}
	}
	CK(cudaEventRecord(n.mfStageEv_[k], s0_), "MF staging");
	n.mfStageUsed_[k] = true;
	return "";
}

std::string Simulator::exportField(size_t i, Field f, uint32_t zone, void *dst, size_t bytes)
{
	CK(cudaSetDevice(device_), "selecting the device");
	if (bytes > hExportBytes_) {
		if (hExport_) cudaFreeHost(hExport_);
		hExport_ = nullptr;
		hExportBytes_ = 0;
		CK(cudaMallocHost((void **)&hExport_, bytes), "pinned allocation");
		hExportBytes_ = bytes;
	}
	if (lastStepPublishes_ && f == F_AP_NC) {
		// after a single step of one network: the small-cell kernel
		// writes the NC spikes and then the step number into mapped host
		// memory; wait for the stamp (bounded), without a copy or a stream
		// synchronisation, while the step's GR pass may still run
		Network &n = *nets_[i];
		const uint64_t want = n.hostT_;
		const volatile uint64_t *stamp = reinterpret_cast<const volatile uint64_t *>(n.hMailbox_);
		bool seen = *stamp == want;
		if (!seen) {
			const auto t0 = std::chrono::steady_clock::now();
			for (uint32_t spin = 0; !seen; spin++) {
				seen = *stamp == want;
				if ((spin & 1023u) == 1023u &&
						std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10))
					break;
			}
		}
		if (seen) {
			std::atomic_thread_fence(std::memory_order_acquire);
			if (!directCopySinceStep_) markInputSlotsFree();
			CKS(checkDeviceErrors());
			memcpy(dst, n.hMailbox_ + 8 + (size_t)zone * n.dev().numNC, bytes);
			return "";
		}
		// no stamp: the synchronising path below reports what happened
	}
	// on the step stream, after every kernel launched so far
	CKS(nets_[i]->exportField(f, zone, hExport_, bytes, s0_));
	CK(cudaStreamSynchronize(s0_), "export");
	markInputSlotsFree();
	CKS(checkDeviceErrors());
	memcpy(dst, hExport_, bytes);
	return "";
}

std::string Simulator::runGraph(uint64_t nsteps, uint32_t chunk, bool instrument)
{
	CK(cudaSetDevice(device_), "selecting the device");
	lastStepPublishes_ = false;
	CKS(settleSteps());
	CKS(flushPendingMF());
	CKS(uploadCtl());
	if (chunk == 0) chunk = 1;
	if (!graphExec_ || graphChunk_ != chunk || graphInstrumented_ != instrument) {
		if (graphExec_) { cudaGraphExecDestroy(graphExec_); graphExec_ = nullptr; }
		while (instrument && passEv_.size() < 2 * (size_t)chunk) {
			cudaEvent_t e, f;
			CK(cudaEventCreate(&e), "event");
			CK(cudaEventCreate(&f), "event");
			passEv_.push_back(e);
			tailEv_.push_back(f);
		}
		cudaGraph_t g;
		CK(cudaStreamBeginCapture(s0_, cudaStreamCaptureModeThreadLocal), "graph capture");
		for (uint32_t k = 0; k < chunk; k++) {
			std::string e = enqueueStep(k, instrument);
			if (!e.empty()) { cudaStreamEndCapture(s0_, &g); return e; }
		}
		advanceStepKernel<<<1, 64, 0, s0_>>>((uint64_t *const *)dTBasePtrs_.ptr, (int)nets_.size(), chunk);
		CK(cudaStreamEndCapture(s0_, &g), "graph capture");
		CK(cudaGraphInstantiate(&graphExec_, g, cudaGraphInstantiateFlagUseNodePriority), "graph instantiate");
		cudaGraphDestroy(g);
		graphChunk_ = chunk;
		graphInstrumented_ = instrument;
	}
	const uint64_t reps = nsteps / chunk, rem = nsteps % chunk;
	CK(cudaEventRecord(ev0_, s0_), "timing");
	for (uint64_t r = 0; r < reps; r++) CK(cudaGraphLaunch(graphExec_, s0_), "graph launch");
	for (Network *n : nets_) n->hostT_ += reps * chunk;
	if (rem) CKS(launchSteps((uint32_t)rem));
	CK(cudaEventRecord(ev1_, s0_), "timing");
	CK(cudaEventSynchronize(ev1_), "graph run");
	CKS(checkDeviceErrors());
	CK(cudaEventElapsedTime(&lastGraphMs_, ev0_, ev1_), "timing");
	lastPassMs_ = 0;
	if (instrument && reps) {
		// pass durations of the last chunk replayed
		float total = 0;
		for (uint32_t k = 0; k < chunk; k++) {
			float ms = 0;
			CK(cudaEventElapsedTime(&ms, passEv_[2 * k], passEv_[2 * k + 1]), "pass timing");
			total += ms;
		}
		lastPassMs_ = total / chunk;
		total = 0;
		for (uint32_t k = 0; k < chunk; k++) {
			float ms = 0;
			CK(cudaEventElapsedTime(&ms, tailEv_[2 * k], tailEv_[2 * k + 1]), "tail timing");
			total += ms;
		}
		lastTailMs_ = total / chunk;
	}
	return "";
}

// The L2 flush before a timed step: 2 x L2 bytes written, then read back,
// so that every line the step finds in L2 is a clean line of the flush
// buffer and none of the step's inputs (CBM_FLUSH_READ=0: written only, the
// step then also pays for writing the flush's dirty lines back).
void Simulator::enqueueFlush()
{
	if (!flushBuf_.ptr) return;
	cudaMemsetAsync(flushBuf_.ptr, 0x5a, flushBuf_.bytes, s0_);
	const char *env = getenv("CBM_FLUSH_READ");
	if (env && !strcmp(env, "0")) return;
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
	flushReadKernel<<<4 * sms, 512, 0, s0_>>>((const uint4 *)flushBuf_.ptr, flushBuf_.bytes / 16,
			(uint32_t *)flushBuf_.ptr);
}

std::string Simulator::runFlushed(uint64_t nsteps, size_t flushBytes, float *stepMs)
{
	CK(cudaSetDevice(device_), "selecting the device");
	lastStepPublishes_ = false;
	CKS(settleSteps());
	CKS(flushPendingMF());
	CKS(uploadCtl());
	if (flushBytes && flushBytes != flushBuf_.bytes) {
		// the kernel-timing flush graph writes the old buffer
		if (flushKernGraph_) { cudaGraphExecDestroy(flushKernGraph_); flushKernGraph_ = nullptr; }
		if (flushBuf_.ptr) cudaFree(flushBuf_.ptr);
		flushBuf_.ptr = nullptr;
		CK(cudaMalloc(&flushBuf_.ptr, flushBytes), "allocating the L2 flush buffer");
		flushBuf_.bytes = flushBytes;
	}
	// each step launched as launchSteps launches it, after the flush and
	// between a pair of events on the step stream; batches of kBatch steps
	// between synchronisations, the step counter advanced once per batch
	constexpr uint32_t kBatch = 256;
	while (stepEv_.size() < 2 * kBatch) {
		cudaEvent_t e;
		CK(cudaEventCreate(&e), "event");
		stepEv_.push_back(e);
	}
	double total = 0;
	for (uint64_t done = 0; done < nsteps;) {
		const uint32_t b = (uint32_t)std::min<uint64_t>(kBatch, nsteps - done);
		for (uint32_t k = 0; k < b; k++) {
			enqueueFlush();
			CK(cudaEventRecord(stepEv_[2 * k], s0_), "step timing");
			CKS(enqueueStep(k, false));
			CK(cudaEventRecord(stepEv_[2 * k + 1], s0_), "step timing");
		}
		advanceStepKernel<<<1, 64, 0, s0_>>>((uint64_t *const *)dTBasePtrs_.ptr, (int)nets_.size(), b);
		CK(cudaGetLastError(), "advancing the step counter");
		CK(cudaStreamSynchronize(s0_), "steps");
		for (uint32_t k = 0; k < b; k++) {
			float ms = 0;
			CK(cudaEventElapsedTime(&ms, stepEv_[2 * k], stepEv_[2 * k + 1]), "step timing");
			total += ms;
		}
		for (Network *n : nets_) n->hostT_ += b;
		done += b;
	}
	CKS(checkDeviceErrors());
	*stepMs = (float)total;
	return "";
}

std::string Simulator::runFlushedKernels(uint64_t nsteps, size_t flushBytes, float *passMs, float *tailMs)
{
	CK(cudaSetDevice(device_), "selecting the device");
	lastStepPublishes_ = false;
	CKS(settleSteps());
	CKS(flushPendingMF());
	CKS(uploadCtl());
	if (flushBytes && flushBytes != flushBuf_.bytes) {
		if (flushBuf_.ptr) cudaFree(flushBuf_.ptr);
		flushBuf_.ptr = nullptr;
		if (flushKernGraph_) { cudaGraphExecDestroy(flushKernGraph_); flushKernGraph_ = nullptr; }
		CK(cudaMalloc(&flushBuf_.ptr, flushBytes), "allocating the L2 flush buffer");
		flushBuf_.bytes = flushBytes;
	}
	while (passEv_.size() < 2) {
		cudaEvent_t e, f;
		CK(cudaEventCreate(&e), "event");
		CK(cudaEventCreate(&f), "event");
		passEv_.push_back(e);
		tailEv_.push_back(f);
	}
	if (!flushKernGraph_) {
		// one step in the two-stream form, events around each kernel, after
		// a write of the flush buffer
		cudaGraph_t g;
		CK(cudaStreamBeginCapture(s0_, cudaStreamCaptureModeThreadLocal), "graph capture");
		enqueueFlush();
		std::string e = enqueueStep(0, true);
		advanceStepKernel<<<1, 64, 0, s0_>>>((uint64_t *const *)dTBasePtrs_.ptr, (int)nets_.size(), 1);
		cudaError_t ce = cudaStreamEndCapture(s0_, &g);
		if (!e.empty()) return e;
		CK(ce, "graph capture");
		CK(cudaGraphInstantiate(&flushKernGraph_, g, cudaGraphInstantiateFlagUseNodePriority), "graph instantiate");
		cudaGraphDestroy(g);
	}
	double pass = 0, tail = 0;
	for (uint64_t k = 0; k < nsteps; k++) {
		CK(cudaGraphLaunch(flushKernGraph_, s0_), "graph launch");
		CK(cudaStreamSynchronize(s0_), "step");
		float a = 0, b = 0;
		CK(cudaEventElapsedTime(&a, passEv_[0], passEv_[1]), "pass timing");
		CK(cudaEventElapsedTime(&b, tailEv_[0], tailEv_[1]), "tail timing");
		pass += a;
		tail += b;
		for (Network *n : nets_) n->hostT_ += 1;
	}
	CKS(checkDeviceErrors());
	*passMs = nsteps ? (float)(pass / nsteps) : 0.0f;
	*tailMs = nsteps ? (float)(tail / nsteps) : 0.0f;
	return "";
}

std::string Simulator::timerStart()
{
	CK(cudaEventRecord(tev0_, s0_), "timer");
	return "";
}

std::string Simulator::timerStop(float *ms)
{
	CK(cudaEventRecord(tev1_, s0_), "timer");
	CK(cudaEventSynchronize(tev1_), "timer");
	CK(cudaEventElapsedTime(ms, tev0_, tev1_), "timer");
	return "";
}

void Simulator::markInputSlotsFree()
{
	// every copy enqueued so far has run: no staging slot needs a query
	for (Network *n : nets_)
		for (bool &u : n->mfStageUsed_) u = false;
}

std::string Simulator::sync()
{
	CKS(settleSteps());
	CK(cudaStreamSynchronize(s0_), "sync");
	CK(cudaStreamSynchronize(s1_), "sync");
	markInputSlotsFree();
	CK(cudaGetLastError(), "sync");
	return checkDeviceErrors();
}

std::string Simulator::checkDeviceErrors()
{
	// after a synchronisation with the kernels that may have written them
	for (Network *n : nets_) {
		const uint32_t flag = *reinterpret_cast<volatile uint32_t *>(n->hErr_);
		if (flag & kErrPassWait) return "GR pass: a pipeline wait timed out on the device";
		if (flag) return "device error word set";
	}
	return "";
}

}  // namespace cbm
