// Host-side network state: the reference's CBMState with its parameter
// objects and the four state containers, held as named arrays.
//
// File format and parameter derivation follow
//   CBM_STATE_LIB_DEV/src/interfaces/cbmstate.cpp:12-33, 86-103 (file layout)
//   CBM_STATE_LIB_DEV/src/params/connectivityparams.cpp:12-218
//   CBM_STATE_LIB_DEV/src/params/activityparams.cpp:12-42, 243-253, 418-636
//   CBM_STATE_LIB_DEV/src/state/*.cpp stateRW / initializeVals
// so that files written by either implementation load in the other.
#pragma once
#include <cstdint>
#include <map>
#include <ostream>
#include <string>
#include <vector>

namespace cbm {

enum DType : int { U8 = 0, I32 = 1, U32 = 2, F32 = 3, U64 = 4 };
size_t dtypeSize(DType t);

struct NamedArray {
	std::string name;
	DType dtype;
	size_t count = 0;
	std::vector<uint8_t> bytes;
	template <typename T> T *as() { return reinterpret_cast<T *>(bytes.data()); }
	template <typename T> const T *as() const { return reinterpret_cast<const T *>(bytes.data()); }
};

// ConnectivityParams (connectivityparams.h:116-144): the raw key map plus
// every derived size.
struct ConParams {
	std::map<std::string, uint32_t> raw;
	uint32_t maxnumpGOGABAInGOGO = 0, maxnumpGOGABAOutGOGO = 0;
	std::vector<float> gogoGABALocalCon;  // rows of 3
	uint32_t maxnumpGOCoupInGOGO = 1, maxnumpGOCoupOutGOGO = 1;
	std::vector<float> gogoCoupLocalCon{1, 1, 0};
	bool hasGABAMatrix = false;

	uint32_t glX, glY, numGL, maxnumpGLfromGLtoGR, lownumpGLfromGLtoGR, maxnumpGLfromGLtoGO,
		maxnumpGLfromGOtoGL, numMF, numpMFfromMFtoGL, maxnumpMFfromMFtoGO, maxnumpMFfromMFtoGR,
		numpMFfromMFtoNC, goX, goY, numGO, maxnumpGOfromGRtoGO, maxnumpGOfromGLtoGO,
		maxnumpGOfromMFtoGO, maxnumpGOfromGOtoGL, maxnumpGOfromGOtoGR, grX, grY, numGR, numGRP2,
		grPFVelInGRXPerTStep, grAFDelayInTStep, maxnumpGRfromGRtoGO, maxnumpGRfromGLtoGR,
		maxnumpGRfromGOtoGR, maxnumpGRfromMFtoGR, numSC, numpSCfromGRtoSC, numpSCfromGRtoSCP2,
		numpSCfromSCtoPC, numPC, numpPCfromGRtoPC, numpPCfromGRtoPCP2, numpPCfromBCtoPC,
		numpPCfromPCtoBC, numpPCfromSCtoPC, numpPCfromPCtoNC, numBC, numpBCfromGRtoBC,
		numpBCfromGRtoBCP2, numpBCfromBCtoPC, numpBCfromPCtoBC, numNC, numpNCfromPCtoNC,
		numpNCfromNCtoIO, numpNCfromMFtoNC, numIO, numpIOfromIOtoPC, numpIOfromNCtoIO,
		numpIOInIOIO, numpIOOutIOIO;

	void derive();
};

// ActivityParams (activityparams.h:40-204): raw float map plus derived values.
struct ActParams {
	std::map<std::string, float> raw;

	float msPerTimeStep, msPerHistBinMF; uint32_t numTSinMFHist;
	float eLeakGO, eMGluRGO, eGABAGO, threshMaxGO, threshRestGO, gIncMFtoGO, gIncGRtoGO,
		gGABAIncGOtoGO, coupleRiRjRatioGO, gMGluRScaleGRtoGO, gMGluRIncScaleGO, mGluRScaleGO,
		gluScaleGO, gLeakGO, goGABAGOGOSynRecTau, goGABAGOGOSynRec, goGABAGOGOSynDepF,
		gDecTauMFtoGO, gDecMFtoGO, gDecTauGRtoGO, gDecGRtoGO, gGABADecTauGOtoGO, gGABADecGOtoGO,
		mGluRDecayGO, gMGluRIncDecayGO, gMGluRDecGRtoGO, gluDecayGO, threshDecTauGO, threshDecGO;
	float eLeakGR, eGOGR, eMFGR, threshMaxGR, threshRestGR, gIncMFtoGR, gIncGOtoGR, gDecTauMFtoGR,
		gDecMFtoGR, gDecTauGOtoGR, gDecGOtoGR, threshDecTauGR, threshDecGR, gLeakGR, msPerHistBinGR;
	uint32_t tsPerHistBinGR;
	float eLeakSC, gLeakSC, gDecTauGRtoSC, gDecGRtoSC, threshMaxSC, threshRestSC, threshDecTauSC,
		threshDecSC, gIncGRtoSC;
	float eLeakBC, ePCtoBC, gLeakBC, gDecTauGRtoBC, gDecGRtoBC, gDecTauPCtoBC, gDecPCtoBC,
		threshDecTauBC, threshDecBC, threshRestBC, threshMaxBC, gIncGRtoBC, gIncPCtoBC;
	float initSynWofGRtoPC, eLeakPC, eBCtoPC, eSCtoPC, threshMaxPC, threshRestPC, threshDecTauPC,
		threshDecPC, gLeakPC, gDecTauGRtoPC, gDecGRtoPC, gDecTauBCtoPC, gDecBCtoPC, gDecTauSCtoPC,
		gDecSCtoPC, gIncSCtoPC, gIncGRtoPC, gIncBCtoPC;
	uint32_t tsPopHistPC, tsPerPopHistBinPC, numPopHistBinsPC;
	float synLTPStepSizeGRtoPC, synLTDStepSizeGRtoPC;
	float coupleRiRjRatioIO, eLeakIO, eNCtoIO, gLeakIO, gDecTSofNCtoIO, gDecTTofNCtoIO,
		gDecT0ofNCtoIO, gIncNCtoIO, gIncTauNCtoIO, threshRestIO, threshMaxIO, threshDecTauIO,
		threshDecIO;
	uint32_t tsLTDDurationIO; int32_t tsLTDStartAPIO, tsLTPStartAPIO; uint32_t grPCHistCheckBinIO;
	float maxExtIncVIO;
	float eLeakNC, ePCtoNC, gmaxNMDADecTauMFtoNC, gmaxNMDADecMFtoNC, gmaxAMPADecTauMFtoNC,
		gmaxAMPADecMFtoNC, gNMDAIncMFtoNC, gAMPAIncMFtoNC, gIncAvgPCtoNC, gDecTauPCtoNC,
		gDecPCtoNC, gLeakNC, threshDecTauNC, threshDecNC, threshMaxNC, threshRestNC,
		relPDecTSofNCtoIO, relPDecTTofNCtoIO, relPDecT0ofNCtoIO, relPIncNCtoIO, relPIncTauNCtoIO,
		initSynWofMFtoNC, synLTDPCPopActThreshMFtoNC, synLTPPCPopActThreshMFtoNC,
		synLTDStepSizeMFtoNC, synLTPStepSizeMFtoNC;

	void derive();
	// ActivityParams::setParam (activityparams.cpp:423-434): only known keys.
	bool set(const std::string &key, float value);
};

// Per-zone values the reference keeps in MZoneActivityState but never writes
// to the file (mzoneactivitystate.h:69-85).
struct ZoneScalars {
	uint32_t histPCPopActSum = 0, histPCPopActCurBinN = 0, pcPopAct = 0;
	float errDrive = 0;
	uint8_t noLTPMFNC = 0, noLTDMFNC = 0;
};

class State {
public:
	uint32_t numZones = 0;
	ConParams cp;
	ActParams ap;
	std::vector<NamedArray> innetCon, innetAct;
	std::vector<std::vector<NamedArray>> zoneCon, zoneAct;
	std::vector<ZoneScalars> zoneScalars;

	// CBMState(fstream&) (cbmstate.cpp:12-33).  Returns "" or an error.
	std::string load(const std::string &path);
	// The same from bytes in memory (a stream's content from its current
	// position): *consumed receives the bytes the state occupies, so that
	// whatever follows it (the eyelid driver's trial data) can be read next.
	std::string loadBytes(const std::string &data, size_t *consumed);
	// CBMState::writeState (cbmstate.cpp:86-103).
	std::string save(const std::string &path) const;
	// The same into a stream at its current position.
	std::string writeTo(std::ostream &out) const;
	// Bytes writeTo emits.
	size_t fileBytes() const;
	// A new network of the given parameter texts with every array at the
	// reference's initial values (initializeVals of the four containers) and
	// the microzone wiring of MZoneConnectivityState (mzoneconnectivitystate.cpp:
	// 213-417).  Input-net connectivity arrays are left at the reference's
	// "unconnected" values (counts 0, indices UINT_MAX) for the caller to fill.
	std::string create(const std::string &conText, const std::string &actText, uint32_t nZones,
			const std::vector<int> &pcncSeeds);
	// CBMState(actPF, conPF, nZones, innetCRSeed, mzoneCRSeed, mzoneARSeed)
	// (cbmstate.cpp:60-64, 176-204): create() plus the reference's own
	// generator for the input net and the PC->NC wiring, drawing from its
	// random generator seeded as the reference seeds it (cbm_netgen.cpp).
	// The microzone activity seeds are not used by the reference.
	std::string generate(const std::string &conText, const std::string &actText, uint32_t nZones, int innetSeed,
			const std::vector<int> &mzoneConSeeds);

	NamedArray *find(const std::string &name, int zone = -1);
	const NamedArray *find(const std::string &name, int zone = -1) const;

private:
	std::string parseHeader(const std::string &text, size_t &pos, bool withZones);
	void allocate();
	void fixLoaded();
};

// The seeds CBMState(actPF, conPF, nZones) draws from the wall clock:
// innet, then connectivity and activity per zone.
std::vector<int> clockSeeds(uint32_t nZones);

// Byte-exact text of the parameter header as CBMState::writeState emits it.
std::string formatHeader(const State &s);

}  // namespace cbm
