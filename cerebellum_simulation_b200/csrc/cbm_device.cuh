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

namespace cbm {

constexpr int kMaxZones = 4;
constexpr uint32_t kNoDelay = 0xFFu;

// Values the host may change between steps (setter calls of the reference's
// API): read by the kernels of the next step.
struct HostCtl {
	float ltdStep[kMaxZones];   // MZone::tempGRPCLTDStep (mzone.cpp:726-736)
	float ltpStep[kMaxZones];   // MZone::tempGRPCLTPStep
	float errDrive[kMaxZones];  // MZoneActivityState::errDrive (mzone.cpp:167-173), consumed by the IO update
	float gIncGRtoGO;           // InNet::tempGIncGRtoGO (innet.cpp:669-677)
	uint32_t pad[3];
};

struct DevZone {
	float *w;           // pfSynWeightPC, PC-major (mzone.cpp:97-103)
	float *pcPartial;   // [3][numPC][bs] per-thread partial sums of the PF->PC reduction
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
	uint32_t mfWords, goWords;            // spike-bit vectors incl. the always-zero sentinel
	uint32_t maxnumpMFfromMFtoGO, maxnumpGOCoupInGOGO;
	uint32_t numpPCfromSCtoPC, numpNCfromPCtoNC, numpNCfromMFtoNC, numpIOfromNCtoIO, numpIOInIOIO;
	uint32_t numPopHistBinsPC, tsPerPopHistBinPC, tsPerHistBinGR, numTSinMFHist;
	uint32_t numCoupLevels;
	uint32_t mfRing;                      // slots in the MF input ring
	uint32_t hasMFRaw;

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
	const uint32_t *mfgoStart, *mfgoSrc;  // per GO: MF sources (with repeats) of updateMFtoGOOut
	const int32_t *numpGOCoupInGOGO; const uint32_t *pGOCoupInGOGO;
	const uint32_t *coupLevelStart, *coupLevelGO;  // coupling sweep schedule

	// ---- step pipeline
	uint32_t *goCount;   // [2][numGO] GR->GO input counts per step parity
	uint32_t *bcCount;   // [3][numBC] PF->BC counts
	uint32_t *scCount;   // [3][numSC] PF->SC counts
	uint32_t *goBits;    // [2][goWords] GO spikes per step parity
	const uint32_t *mfBits;  // [mfRing][mfWords] MF spikes per step
	const uint8_t *mfRaw;    // [mfRing][numMF] raw MF input bytes (NC inputs), or null
	uint64_t *tBase;     // steps completed
	HostCtl *ctl;
	uint32_t *errFlag;   // device error word (bounds violations found by checks)

	DevZone zones[kMaxZones];
};

}  // namespace cbm
