// Device-resident layout of one network instance.
//
// Granule cells (GR) are stored structure-of-arrays, one element per cell,
// in the reference's GR order.  Connectivity arrives in the reference's
// cell-major form ([gr][synapse], innetconnectivitystate.h:130-143) and is
// re-laid out synapse-major ([synapse][gr]) with 16-bit indices, padded with
// a sentinel index whose spike bit is always zero so the gathers need no
// per-cell counts.  GR->GO synapses carry their axonal delay as a bit number
// packed with the target.  Small-cell state (GO, SC, BC, PC, IO, NC) keeps the
// reference's array names and layouts (innetactivitystate.h,
// mzoneactivitystate.h).
#pragma once
#include <cstdint>
#include <cuda.h>

#if defined(__CUDACC__)
#define CBM_LAYOUT_FN __host__ __device__ inline
#else
#define CBM_LAYOUT_FN inline
#endif

namespace cbm {

constexpr int kMaxZones = 4;
constexpr uint32_t kNoDelay = 0xFFu;

// Bits of DevNet::errFlag.
constexpr uint32_t kErrPassWait = 1u;  // a GR-pass pipeline wait timed out

// TMA descriptors of the GR arrays the GR pass streams, each viewed as rows
// of bs cells ([numGR/bs][bs], slot tables as [slot][numGR/bs][bs]) and
// copied in boxes of 32 cells x R rows (x all slots).
enum PassMap : int {
	PM_V = 0, PM_GKCA, PM_THRESH, PM_GESUM, PM_GISUM, PM_APBUF,  // 4-byte state, read and rewritten
	PM_MFIDX, PM_GOIDX, PM_OUTCON, PM_PFDELAY, PM_HIST, PM_OUTCON16, PM_W0,
	PM_COUNT = PM_W0 + kMaxZones
};

// 16-bit GR->GO synapse: (GO << 5) | delay bit, for networks of at most
// 2047 GO; kOut16None marks an empty slot.
constexpr uint16_t kOut16None = 0xFFFFu;
constexpr uint32_t kOut16MaxGO = 2047u;
// GR->GO slot planes the per-tile pass streams when some GR has more synapses
// (the rest go to per-tile lists).
constexpr uint32_t kOutInline = 4u;

// A step's MF spike words passed by value to the step's kernels (one
// network launched a step at a time: the host packs the caller's input and
// the launch carries it, with no copy ahead of the kernels).  n = 0: the
// kernels read the network's MF ring.  Networks of up to 32 x kMFParamWords
// - 1 fibres.
constexpr uint32_t kMFParamWords = 64;
struct MFParam {
	uint32_t n;
	uint32_t w[kMFParamWords];
};

// A device array that a small-cell CTA copies into shared memory for the
// step (and back when it changes): the CTA then runs on a shared-memory copy
// of the network descriptor whose pointer at fieldOff points into the copy.
struct StageSeg {
	uint32_t fieldOff;   // byte offset of the array's pointer within DevNet
	uint32_t bytes;      // array size, a multiple of 16
	uint32_t smemOff;    // offset in the staging arena (16-byte aligned)
	uint32_t writeBack;  // copied back to global memory after the step
};

// Shared-memory layout of one pipeline stage of the GR pass (R rows of 32
// cells); every region starts on a 128-byte boundary.
struct PassLayout {
	uint32_t mfIdx, goIdx, outCon, pfDelay, w, hist;  // region offsets (the six state arrays start at 0)
	uint32_t bytes;    // stage size
	uint32_t txBase;   // bytes the stage's copies deliver, history excluded
	uint32_t txHist;   // bytes of the history box (plasticity steps only)
};

CBM_LAYOUT_FN uint32_t align128(uint32_t x) { return (x + 127u) & ~127u; }

// outBytes: 4 for the 32-bit GR->GO slot table, 2 for the 16-bit one.
CBM_LAYOUT_FN PassLayout passLayout(uint32_t R, uint32_t nMF, uint32_t nGO, uint32_t nOut, uint32_t Z,
		uint32_t outBytes = 4)
{
	const uint32_t mfS = nMF ? nMF : 1, goS = nGO ? nGO : 1, outS = nOut ? nOut : 1;
	const uint32_t row4 = 128u * R;  // one 4-byte array: R rows x 32 cells
	PassLayout L;
	uint32_t o = 6 * row4;
	L.mfIdx = o; o = align128(o + 64u * R * mfS);
	L.goIdx = o; o = align128(o + 64u * R * goS);
	L.outCon = o; o = align128(o + 32u * outBytes * R * outS);
	L.pfDelay = o; o = align128(o + 32u * R);
	L.w = o; o = align128(o + row4 * Z);
	L.hist = o; o = align128(o + 256u * R);
	L.bytes = o;
	L.txBase = 6 * row4 + 64u * R * mfS + 64u * R * goS + 32u * outBytes * R * outS + 32u * R + row4 * Z;
	L.txHist = 256u * R;
	return L;
}

// Values the host may change between steps (setter calls of the reference's
// API): read by the kernels of the next step.
struct HostCtl {
	float ltdStep[kMaxZones];   // MZone::tempGRPCLTDStep (mzone.cpp:726-736)
	float ltpStep[kMaxZones];   // MZone::tempGRPCLTPStep
	float errDrive[kMaxZones];  // MZoneActivityState::errDrive (mzone.cpp:167-173), consumed by the IO update
	float gIncGRtoGO;           // InNet::tempGIncGRtoGO (innet.cpp:669-677)
	uint32_t pad[3];
};

// The eyelid-conditioning trial driven on the device (the reference's
// ECManagementDelay, Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp):
// MF input from a Poisson regenerating population (PoissonRegenCells,
// CBM_TOOLS_LIB_DEV/src/poissonregencells.cpp:49-66) with background / CS
// tonic / CS phasic rates, the US error drive and the PF->PC plasticity
// window, and the recording of the trials it keeps (NC and PC spike counts
// per bin, the eyelid integrator's output, eyelidintegrator.cpp:50-68).
// Steps of the protocol are numbered from startT: step t has in-trial time
// (t - 1 - startT) % trialSteps and trial (t - 1 - startT) / trialSteps.
struct DevProtocol {
	uint64_t startT;
	uint32_t trialSteps, csStartTrial;
	int32_t csOn, csOff, csPOff, plastOn, plastOff;  // plastOn/Off: steps after csOn / csOff
	float plastLTD, plastLTP, usErrDrive;           // usErrDrive already times maxExtIncVIO
	float defaultLTD, defaultLTP;                   // resetGRPCPlastSteps values
	// MF generator
	const float *freqBG, *freqCSTonic, *freqCSPhasic;  // Hz, numMF each
	float *mfThresh;       // regeneration state per MF
	uint64_t mfKey;        // stream key of the MF draws
	float sPerTS, mfThreshDecay;
	int32_t *plastState;   // [2]: the eyelid driver's grPCPlastSet, grPCPlastReset
	float *curSteps;       // [2]: zone 0's LTD and LTP steps in force
	float *ctlSlots;       // [2][3]: zone 0's LTD step, LTP step and error drive per step parity
	// recording
	uint32_t dataStartTrial, numDataTrials, binSteps, nBins;
	int32_t recFrom, recLen;   // in-trial window [recFrom, recFrom + recLen)
	uint32_t *ncPSH;       // [numDataTrials][nBins][numNC]
	uint32_t *pcPSH;       // [numDataTrials][nBins][numPC]
	float *eyelid;         // [numDataTrials][recLen] integrator output per step
	float *eyeG;           // [numNC] integrator conductances
	float *eyeVm;          // [1]
	uint16_t *grPSH;       // [nBins][numGR] GR spike counts of the kept trials, or null
	// the eyelid driver's trial data, or null: histograms go, grInputGO,
	// goInputGO, goOutSynScale, mf, sc, bc, pc, io, each f32 [nBins][cells];
	// rasters go, sc, bc, pc, nc, io, each u32 [numDataTrials][recLen / 32][cells]
	float *tdPSH;
	uint32_t *tdRaster;
	float eyeGDecay, eyeGInc, eyeGShift, eyeGLeak, eyeMaxAmp;
	// state-variable MF coding (cbm_statevar_input), or svValues null: the
	// rate tables above
	const float *svMean, *svRelaxed, *svExcited, *svValues;
	uint64_t svSteps;
	uint32_t svVars, svPer;
	float svLo, svHi, svDen, svMaxPossible;
	double svNorm;
};

struct DevZone {
	float *w;           // pfSynWeightPC, PC-major (mzone.cpp:97-103)
	float *pcPartial;   // [3][numPC][bs] per-thread partial sums of the PF->PC reduction
	float *pairSum;     // [2][numPC][K][bs] x[i] + x[i+bs] of the reduction per step parity (persistent and vector GR passes)
	float *pcSum;       // [3][numPC] PF->PC input sums (the whole reduction), made by the vector GR pass
	uint8_t *plastSel;  // [2][numIO]: 0 none, 1 LTD, 2 LTP for the next plasticity step
	const uint32_t *ioOfPC;  // IO whose timer drives each PC block's plasticity (mzone.cpp:682-705)

	// microzone connectivity (mzoneconnectivitystate.h), reference layouts
	const uint32_t *pPCfromSCtoPC, *pNCfromPCtoNC, *pNCfromMFtoNC, *pIOfromNCtoIO, *pIOInIOIO;
	// destination-side lists built from pBCfromBCtoPC / pPCfromPCtoBC
	const uint32_t *bcpcStart, *bcpcSrc;  // per PC: BCs that target it (with repeats)
	const uint32_t *pcbcStart, *pcbcSrc;  // per BC: PCs that target it (with repeats)

	// activity (mzoneactivitystate.h)
	uint8_t *apBC; uint32_t *apBufBC, *inputPCBC; float *gPFBC, *gPCBC, *threshBC, *vBC;
	uint8_t *apPC; uint32_t *apBufPC, *inputBCPC; uint8_t *inputSCPC;
	float *gPFPC, *gBCPC, *gSCPC, *vPC, *threshPC; uint32_t *histPCPopAct;
	uint32_t *scal;  // histPCPopActSum, histPCPopActCurBinN, pcPopAct, noLTPMFNC, noLTDMFNC
	uint8_t *apIO; uint32_t *apBufIO; uint8_t *inputNCIO;
	float *gNCIO, *threshIO, *vIO, *vCoupleIO; int32_t *pfPCPlastTimerIO;
	uint8_t *apNC; uint32_t *apBufNC; uint8_t *inputPCNC, *inputMFNC;
	float *gPCNC, *gPCScaleNC, *mfSynWeightNC, *gmaxNMDAofMFtoNC, *gmaxAMPAofMFtoNC,
		*gMFNMDANC, *gMFAMPANC, *threshNC, *vNC, *synIOPReleaseNC;
	uint64_t ncioKey;   // stream key of this zone's release draws
};

struct DevNet {
	// ---- sizes
	uint32_t numGR, numMF, numGO, numSC, numBC, numPC, numNC, numIO, numZones;
	uint32_t P, bs, K, J, tilesPerPC;     // PF->PC reduction geometry (kernels.cu:435-470)
	uint32_t bcShift, scShift, bcLocal, scLocal;
	uint32_t nMFSlots, nGOSlots, nOutSlots;
	uint32_t nOutTma;                     // GR->GO slot planes the per-tile TMA pass streams (the rest: ovStart)
	uint32_t mfWords, goWords;            // spike-bit vectors incl. the always-zero sentinel
	uint32_t maxnumpMFfromMFtoGO, maxnumpGOCoupInGOGO;
	uint32_t numpPCfromSCtoPC, numpNCfromPCtoNC, numpNCfromMFtoNC, numpIOfromNCtoIO, numpIOInIOIO;
	uint32_t numPopHistBinsPC, tsPerPopHistBinPC, tsPerHistBinGR, numTSinMFHist;
	uint32_t numCoupLevels;
	uint32_t mfRing;                      // slots in the MF input ring
	uint32_t hasMFRaw;
	uint32_t pcSumMode;                   // 1: the small-cell update reads pcSum, else it reduces pcPartial

	// ---- parameters (activityparams.h)
	float gLeakGR, eLeakGR, eGOGR, threshRestGR, threshMaxGR, threshDecGR;
	float gDecMFtoGR, gIncMFtoGR, gDecGOtoGR, gIncGOtoGR;
	float gIncMFtoGO, gDecMFtoGO, gDecGRtoGO, gGABAIncGOtoGO, gGABADecGOtoGO, gluDecayGO,
		gluScaleGO, mGluRDecayGO, mGluRScaleGO, gMGluRIncDecayGO, gMGluRIncScaleGO,
		gMGluRDecGRtoGO, gMGluRScaleGRtoGO, threshRestGO, threshDecGO, gLeakGO, eLeakGO,
		eGABAGO, threshMaxGO, coupleRiRjRatioGO, goGABAGOGOSynRec, goGABAGOGOSynDepF;
	float gIncGRtoSC, gDecGRtoSC, gLeakSC, eLeakSC, threshDecSC, threshRestSC, threshMaxSC;
	float gIncGRtoBC, gDecGRtoBC, gIncPCtoBC, gDecPCtoBC, gLeakBC, eLeakBC, ePCtoBC,
		threshDecBC, threshRestBC, threshMaxBC;
	float gIncGRtoPC, gDecGRtoPC, gIncBCtoPC, gDecBCtoPC, gIncSCtoPC, gDecSCtoPC, gLeakPC,
		eLeakPC, eBCtoPC, eSCtoPC, threshDecPC, threshRestPC, threshMaxPC;
	float msPerTimeStep, gDecTSofNCtoIO, gDecTTofNCtoIO, gDecT0ofNCtoIO, gIncNCtoIO,
		gIncTauNCtoIO, gLeakIO, eLeakIO, eNCtoIO, threshMaxIO, threshDecIO, threshRestIO,
		coupleRiRjRatioIO;
	int32_t tsLTDStartAPIO, tsLTDEndIO, tsLTPStartAPIO;
	float gmaxNMDADecMFtoNC, gNMDAIncMFtoNC, gmaxAMPADecMFtoNC, gAMPAIncMFtoNC, gDecPCtoNC,
		gLeakNC, eLeakNC, ePCtoNC, threshDecNC, threshRestNC, threshMaxNC;
	float relPDecTSofNCtoIO, relPDecTTofNCtoIO, relPDecT0ofNCtoIO, relPIncNCtoIO, relPIncTauNCtoIO;
	float synLTDPCPopActThreshMFtoNC, synLTPPCPopActThreshMFtoNC, synLTDStepSizeMFtoNC,
		synLTPStepSizeMFtoNC;

	// ---- GR state and connectivity
	float *vGR, *gKCaGR, *threshGR, *gESum, *gISum;
	uint32_t *apBufGR;
	uint64_t *historyGR;
	const uint16_t *mfIdx;    // [nMFSlots][numGR], sentinel numMF
	const uint16_t *goIdx;    // [nGOSlots][numGR], sentinel numGO
	const uint32_t *outCon;   // [nOutSlots][numGR]: (GO << 8) | delay bit, kNoDelay when empty
	const uint16_t *outCon16; // the same as 16-bit entries (kOut16None when empty), or null (> 2047 GO)
	// GR->GO synapses in slots >= nOutTma, per TMA-pass tile (null when none):
	// tile b's are ovEntry[ovStart[b] .. ovStart[b+1]), x = tile-local cell
	// (row * 32 + lane) | delay bit << 24, y = GO
	const uint32_t *ovStart;
	const uint2 *ovEntry;
	const uint8_t *pfDelay;   // delay bit of the PF->BC/SC/PC output, kNoDelay when none

	// ---- GO / MF / SC state (innetactivitystate.h)
	uint8_t *histMF; uint32_t *apBufMF;
	uint8_t *apGO; uint32_t *apBufGO; float *vGO, *vCoupleGO, *threshCurGO;
	uint32_t *inputMFGO, *inputGOGO; float *inputGOGABASynDepGO, *goGABAOutSynScaleGOGO;
	float *gMFGO, *gGRGO, *gGOGO, *gMGluRGO, *gMGluRIncGO, *mGluRGO, *gluGO;
	uint8_t *apSC; uint32_t *apBufSC; float *gPFSC, *threshSC, *vSC;
	uint32_t *sumGRInputGO; float *sumInputGOGABASynDepGO;

	// ---- input-net connectivity used by the small-cell updates
	const int32_t *numpMFfromMFtoGO; const uint32_t *pMFfromMFtoGO;
	const uint32_t *gogoStart, *gogoSrc;  // per GO: sources of GO->GO synapses in (source, slot) order
	const int32_t *numpGOCoupInGOGO; const uint32_t *pGOCoupInGOGO;
	const uint32_t *coupLevelStart, *coupLevelGO;  // coupling sweep schedule

	// ---- step pipeline
	uint64_t *pairStep;  // [2] the step whose PF->PC pair sums each pairSum slot holds (vector GR pass)
	uint32_t *passClaim; // [3] work counters of the vector GR pass, per step mod 3
	uint32_t *pcDone;    // [numPC] reduction chunks of the previous step done per PC (vector GR pass)
	uint32_t *goCount;   // [2][numGO] GR->GO input counts per step parity
	uint32_t *bcCount;   // [3][numBC] PF->BC counts
	uint32_t *scCount;   // [3][numSC] PF->SC counts
	uint32_t *goBits;    // [2][goWords] GO spikes per step parity
	const uint32_t *mfBits;  // [mfRing][mfWords] MF spikes per step
	const uint8_t *mfRaw;    // [mfRing][numMF] raw MF input bytes (NC inputs), or null
	uint64_t *tBase;     // steps completed
	HostCtl *ctl;
	uint32_t *errFlag;   // error word (kErr* bits), in mapped pinned host memory
	const CUtensorMap *passMaps;  // [PM_COUNT] descriptors of the TMA GR pass, or null
	DevProtocol *proto;           // device-driven trial protocol, or null
	float *protoSlots;            // its ctlSlots (read without going through proto), or null
	const StageSeg *zoneSegs;     // arrays the microzone CTA stages in shared memory
	uint32_t numZoneSegs;         // 0: the microzone CTA works on global memory
	uint32_t zoneArenaBytes;      // staged arrays: read-only ones, then from zoneWbOff on the written ones
	uint32_t zoneWbOff;
	uint32_t zoneStageBytes;      // the whole staging block (stageBlockBytes)

	DevZone zones[kMaxZones];
};

// Staging block of a network whose microzone arrays fit in shared memory: one
// allocation that the microzone CTA copies as it is, laid out as its shared
// memory copy: the descriptor, the step counter (tBase points here), the
// staged arrays, then the StageSeg table.  Networks that are not staged
// allocate the descriptor and the step counter alone (kStageArenaOff bytes).
constexpr uint32_t kStageNetBytes = (uint32_t)((sizeof(DevNet) + 15) & ~(size_t)15);
constexpr uint32_t kStageArenaOff = kStageNetBytes + 16;
#if defined(__CUDACC__)
// t mod d and t / d for a step count t: 32-bit arithmetic while both fit in
// 32 bits (a 64-bit division is a long out-of-line routine that measured
// microseconds on the small-cell update's critical path), the 64-bit form
// beyond.
__device__ __forceinline__ uint32_t stepMod(uint64_t t, uint32_t d)
{
	return (t >> 32) == 0 ? (uint32_t)t % d : (uint32_t)(t % d);
}
__device__ __forceinline__ uint64_t stepMod(uint64_t t, uint64_t d)
{
	return ((t | d) >> 32) == 0 ? (uint64_t)((uint32_t)t % (uint32_t)d) : t % d;
}
__device__ __forceinline__ uint64_t stepDiv(uint64_t t, uint32_t d)
{
	return (t >> 32) == 0 ? (uint64_t)((uint32_t)t / d) : t / d;
}

// Steps the network has completed: every descriptor allocation holds the
// step counter at kStageNetBytes (DevNet::tBase points there), so kernels
// read it together with the descriptor instead of after it.
__device__ __forceinline__ uint64_t stepsDone(const DevNet *N)
{
	return *reinterpret_cast<const uint64_t *>(reinterpret_cast<const char *>(N) + kStageNetBytes);
}

// Zone z's PF->PC step for plasticity selector sel (1 LTD, 2 LTP) at step t:
// the host setters' value, or for zone 0 under a device protocol the value
// the protocol set for step t.
__device__ __forceinline__ float plasticityStep(const DevNet *N, uint64_t t, uint32_t z, uint8_t sel)
{
	if (sel == 0) return 0.0f;
	if (z == 0 && N->protoSlots) return N->protoSlots[(t & 1) * 3 + (sel == 1 ? 0 : 1)];
	return sel == 1 ? N->ctl->ltdStep[z] : N->ctl->ltpStep[z];
}
#endif

CBM_LAYOUT_FN uint32_t stageBlockBytes(uint32_t arenaBytes, uint32_t numSegs)
{
	return kStageArenaOff + arenaBytes + ((numSegs * (uint32_t)sizeof(StageSeg) + 15u) & ~15u);
}

// Inputs of a microzone step that other kernels write, copied into shared
// memory after the staging block: the cbmExpf table, the MF spike bits of
// step t, the PF->BC and PF->SC counts, every zone's error drive of step t
// and the PF->PC partial sums of pass(t-2) for every zone (byte offsets,
// 16-byte aligned).
struct ZoneInputLayout {
	uint32_t exp2, mf, bc, sc, err, pc, bytes;
};
CBM_LAYOUT_FN ZoneInputLayout zoneInputLayout(uint32_t mfWords, uint32_t numBC, uint32_t numSC, uint32_t Z,
		uint32_t numPC, uint32_t bs)
{
	ZoneInputLayout L;
	uint32_t o = 0;
	L.exp2 = o; o += 256;
	L.mf = o; o += (4 * mfWords + 15) & ~15u;
	L.bc = o; o += (4 * numBC + 15) & ~15u;
	L.sc = o; o += (4 * numSC + 15) & ~15u;
	L.err = o; o += (4 * Z + 15) & ~15u;  // every zone's error drive of step t
	L.pc = o; o += (4 * Z * numPC * bs + 15) & ~15u;
	L.bytes = o;
	return L;
}

}  // namespace cbm
