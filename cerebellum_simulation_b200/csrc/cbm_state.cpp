// Host-side network state; see cbm_state.hpp.
#include "cbm_state.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>

#include "cbm_rng.hpp"

namespace cbm {

size_t dtypeSize(DType t)
{
	switch (t) {
	case U8: return 1;
	case I32: case U32: case F32: return 4;
	case U64: return 8;
	}
	return 0;
}

// ------------------------------------------------------------- parameters
void ConParams::derive()
{
	// connectivityparams.cpp:90-183; raw[] inserts missing keys as 0 like
	// the reference's std::map::operator[].
	glX = 1u << raw["glXP2"]; glY = 1u << raw["glYP2"]; numGL = glX * glY;
	maxnumpGLfromGLtoGR = raw["maxnumpGLfromGLtoGR"];
	lownumpGLfromGLtoGR = raw["lownumpGLfromGLtoGR"];
	maxnumpGLfromGLtoGO = raw["maxnumpGLfromGLtoGO"];
	maxnumpGLfromGOtoGL = raw["maxnumpGLfromGOtoGL"];
	numMF = 1u << raw["numMFP2"];
	numpMFfromMFtoGL = numGL / numMF;
	maxnumpMFfromMFtoGO = numpMFfromMFtoGL * maxnumpGLfromGLtoGO;
	maxnumpMFfromMFtoGR = numpMFfromMFtoGL * maxnumpGLfromGLtoGR;
	numpMFfromMFtoNC = 1;
	goX = 1u << raw["goXP2"]; goY = 1u << raw["goYP2"]; numGO = goX * goY;
	maxnumpGOfromGRtoGO = raw["maxnumpGOfromGRtoGO"];
	maxnumpGOfromGLtoGO = raw["maxnumpGOfromGLtoGO"];
	maxnumpGOfromMFtoGO = maxnumpGOfromGLtoGO;
	maxnumpGOfromGOtoGL = raw["maxnumpGOfromGOtoGL"];
	maxnumpGOfromGOtoGR = maxnumpGOfromGOtoGL * maxnumpGLfromGLtoGR;
	(void)raw["spanGODecDenOnGLX"]; (void)raw["spanGODecDenOnGLY"];
	(void)raw["spanGOAscDenOnGRX"]; (void)raw["spanGOAscDenOnGRY"];
	(void)raw["spanGOAxonOnGLX"]; (void)raw["spanGOAxonOnGLY"];
	grX = 1u << raw["grXP2"]; grY = 1u << raw["grYP2"]; numGR = grX * grY;
	numGRP2 = raw["grXP2"] + raw["grYP2"];
	grPFVelInGRXPerTStep = raw["grPFVelInGRXPerTStep"];
	grAFDelayInTStep = raw["grAFDelayInTStep"];
	maxnumpGRfromGRtoGO = raw["maxnumpGRfromGRtoGO"];
	maxnumpGRfromGLtoGR = raw["maxnumpGRfromGLtoGR"];
	maxnumpGRfromGOtoGR = raw["maxnumpGRfromGOtoGR"];
	maxnumpGRfromMFtoGR = raw["maxnumpGRfromMFtoGR"];
	(void)raw["spanGRDenOnGLX"]; (void)raw["spanGRDenOnGLY"];
	numSC = 1u << raw["numSCP2"];
	numpSCfromGRtoSC = numGR / numSC;
	numpSCfromGRtoSCP2 = numGRP2 - raw["numSCP2"];
	numpSCfromSCtoPC = 1;
	numPC = 1u << raw["numPCP2"];
	numpPCfromGRtoPC = numGR / numPC;
	numpPCfromGRtoPCP2 = numGRP2 - raw["numPCP2"];
	numpPCfromBCtoPC = 16;
	numpPCfromPCtoBC = 16;
	numpPCfromSCtoPC = numSC / numPC;
	numpPCfromPCtoNC = raw["numpPCfromPCtoNC"];
	numBC = numPC * 4;
	numpBCfromGRtoBC = numGR / numBC;
	numpBCfromGRtoBCP2 = numGRP2 - (raw["numPCP2"] + 2);
	numpBCfromBCtoPC = 4;
	numpBCfromPCtoBC = 4;
	numNC = 1u << raw["numNCP2"];
	numpNCfromPCtoNC = numPC / numNC * numpPCfromPCtoNC;
	numpNCfromNCtoIO = 1u << raw["numIOP2"];
	numpNCfromMFtoNC = numMF / numNC;
	numIO = 1u << raw["numIOP2"];
	numpIOfromIOtoPC = numPC / numIO;
	numpIOfromNCtoIO = numNC;
	numpIOInIOIO = numIO - 1;
	numpIOOutIOIO = numIO - 1;
}

void ActParams::derive()
{
	// activityparams.cpp:436-636.  The reference calls exp() on float
	// arguments, which C++ resolves to the float overload: std::exp(float).
	float ms = msPerTimeStep = raw["msPerTimeStep"];
	msPerHistBinMF = raw["msPerHistBinMF"];
	numTSinMFHist = (uint32_t)(msPerHistBinMF / ms);
	if (raw.find("coupleRiRjRatioGO") == raw.end()) raw["coupleRiRjRatioGO"] = 0;
	if (raw.find("goGABAGOGOSynRecTau") == raw.end()) raw["goGABAGOGOSynRecTau"] = 1;
	if (raw.find("goGABAGOGOSynDepF") == raw.end()) raw["goGABAGOGOSynDepF"] = 1;
	auto ex = [](float v) { return std::exp(v); };
	eLeakGO = raw["eLeakGO"]; eMGluRGO = raw["eMGluRGO"]; eGABAGO = raw["eGABAGO"];
	threshMaxGO = raw["threshMaxGO"]; threshRestGO = raw["threshBaseGO"];
	gIncMFtoGO = raw["gMFIncGO"]; gIncGRtoGO = raw["gGRIncGO"]; gGABAIncGOtoGO = raw["gGOIncGO"];
	coupleRiRjRatioGO = raw["coupleRiRjRatioGO"];
	gMGluRScaleGRtoGO = raw["gMGluRScaleGO"]; gMGluRIncScaleGO = raw["gMGluRIncScaleGO"];
	mGluRScaleGO = raw["mGluRScaleGO"]; gluScaleGO = raw["gluScaleGO"];
	gLeakGO = raw["rawGLeakGO"] / (6 - ms);
	gDecTauMFtoGO = raw["gMFDecayTGO"]; gDecMFtoGO = ex(-ms / gDecTauMFtoGO);
	gDecTauGRtoGO = raw["gGRDecayTGO"]; gDecGRtoGO = ex(-ms / gDecTauGRtoGO);
	gGABADecTauGOtoGO = raw["gGODecayTGO"]; gGABADecGOtoGO = ex(-ms / gGABADecTauGOtoGO);
	goGABAGOGOSynRecTau = raw["goGABAGOGOSynRecTau"];
	goGABAGOGOSynRec = 1 - ex(-ms / goGABAGOGOSynRecTau);
	goGABAGOGOSynDepF = raw["goGABAGOGOSynDepF"];
	mGluRDecayGO = raw["mGluRDecayGO"]; gMGluRIncDecayGO = raw["gMGluRIncDecayGO"];
	gMGluRDecGRtoGO = raw["gMGluRDecayGO"]; gluDecayGO = raw["gluDecayGO"];
	threshDecTauGO = raw["threshDecayTGO"]; threshDecGO = 1 - ex(-ms / threshDecTauGO);

	eLeakGR = raw["eLeakGR"]; eGOGR = raw["eGOGR"]; eMFGR = raw["eMFGR"];
	threshMaxGR = raw["threshMaxGR"]; threshRestGR = raw["threshBaseGR"];
	gIncMFtoGR = raw["gMFIncGR"]; gIncGOtoGR = raw["gGOIncGR"];
	gDecTauMFtoGR = raw["gMFDecayTGR"]; gDecMFtoGR = ex(-ms / gDecTauMFtoGR);
	gDecTauGOtoGR = raw["gGODecayTGR"]; gDecGOtoGR = ex(-ms / gDecTauGOtoGR);
	threshDecTauGR = raw["threshDecayTGR"]; threshDecGR = 1 - ex(-ms / threshDecTauGR);
	gLeakGR = raw["rawGLeakGR"] / (6 - ms);
	msPerHistBinGR = raw["msPerHistBinGR"]; tsPerHistBinGR = (uint32_t)(msPerHistBinGR / ms);

	eLeakSC = raw["eLeakSC"]; gLeakSC = raw["rawGLeakSC"] / (6 - ms);
	gDecTauGRtoSC = raw["gPFDecayTSC"]; gDecGRtoSC = ex(-ms / gDecTauGRtoSC);
	threshMaxSC = raw["threshMaxSC"]; threshRestSC = raw["threshBaseSC"];
	threshDecTauSC = raw["threshDecayTSC"]; threshDecSC = 1 - ex(-ms / threshDecTauSC);
	gIncGRtoSC = raw["pfIncSC"];

	eLeakBC = raw["eLeakBC"]; ePCtoBC = raw["ePCBC"]; gLeakBC = raw["rawGLeakBC"] / (6 - ms);
	gDecTauGRtoBC = raw["gPFDecayTBC"]; gDecGRtoBC = ex(-ms / gDecTauGRtoBC);
	gDecTauPCtoBC = raw["gPCDecayTBC"]; gDecPCtoBC = ex(-ms / gDecTauPCtoBC);
	threshDecTauBC = raw["threshDecayTBC"]; threshDecBC = 1 - ex(-ms / threshDecTauBC);
	threshRestBC = raw["threshBaseBC"]; threshMaxBC = raw["threshMaxBC"];
	gIncGRtoBC = raw["pfIncConstBC"]; gIncPCtoBC = raw["pcIncConstBC"];

	initSynWofGRtoPC = raw["pfSynWInitPC"]; eLeakPC = raw["eLeakPC"];
	eBCtoPC = raw["eBCPC"]; eSCtoPC = raw["eSCPC"];
	threshMaxPC = raw["threshMaxPC"]; threshRestPC = raw["threshBasePC"];
	threshDecTauPC = raw["threshDecayTPC"]; threshDecPC = 1 - ex(-ms / threshDecTauPC);
	gLeakPC = raw["rawGLeakPC"] / (6 - ms);
	gDecTauGRtoPC = raw["gPFDecayTPC"]; gDecGRtoPC = ex(-ms / gDecTauGRtoPC);
	gDecTauBCtoPC = raw["gBCDecayTPC"]; gDecBCtoPC = ex(-ms / gDecTauBCtoPC);
	gDecTauSCtoPC = raw["gSCDecayTPC"]; gDecSCtoPC = ex(-ms / gDecTauSCtoPC);
	gIncSCtoPC = raw["gSCIncConstPC"]; gIncGRtoPC = raw["gPFScaleConstPC"];
	gIncBCtoPC = raw["gBCScaleConstPC"];
	tsPopHistPC = (uint32_t)(40 / ms);
	tsPerPopHistBinPC = (uint32_t)(5 / ms);
	numPopHistBinsPC = tsPerPopHistBinPC ? tsPopHistPC / tsPerPopHistBinPC : 0;

	coupleRiRjRatioIO = raw["coupleScaleIO"]; eLeakIO = raw["eLeakIO"]; eNCtoIO = raw["eNCIO"];
	gLeakIO = raw["rawGLeakIO"] / (6 - ms);
	gDecTSofNCtoIO = raw["gNCDecTSIO"]; gDecTTofNCtoIO = raw["gNCDecTTIO"];
	gDecT0ofNCtoIO = raw["gNCDecT0IO"]; gIncNCtoIO = raw["gNCIncScaleIO"];
	gIncTauNCtoIO = raw["gNCIncTIO"]; threshRestIO = raw["threshBaseIO"];
	threshMaxIO = raw["threshMaxIO"];
	threshDecTauIO = raw["threshDecayTIO"]; threshDecIO = 1 - ex(-ms / threshDecTauIO);
	tsLTDDurationIO = (uint32_t)(raw["msLTDDurationIO"] / ms);
	tsLTDStartAPIO = (int32_t)(raw["msLTDStartAPIO"] / ms);
	tsLTPStartAPIO = (int32_t)(raw["msLTPStartAPIO"] / ms);
	synLTPStepSizeGRtoPC = raw["grPCLTPIncIO"]; synLTDStepSizeGRtoPC = raw["grPCLTDDecIO"];
	grPCHistCheckBinIO = tsPerHistBinGR ? (uint32_t)std::abs(tsLTDStartAPIO / ((int)tsPerHistBinGR)) : 0;
	maxExtIncVIO = raw["maxErrDriveIO"];

	eLeakNC = raw["eLeakNC"]; ePCtoNC = raw["ePCNC"];
	gmaxNMDADecTauMFtoNC = raw["mfNMDADecayTNC"]; gmaxNMDADecMFtoNC = ex(-ms / gmaxNMDADecTauMFtoNC);
	gmaxAMPADecTauMFtoNC = raw["mfAMPADecayTNC"]; gmaxAMPADecMFtoNC = ex(-ms / gmaxAMPADecTauMFtoNC);
	gNMDAIncMFtoNC = 1 - ex(-ms / raw["rawGMFNMDAIncNC"]);
	gAMPAIncMFtoNC = 1 - ex(-ms / raw["rawGMFAMPAIncNC"]);
	gIncAvgPCtoNC = raw["gPCScaleAvgNC"];
	gDecTauPCtoNC = raw["gPCDecayTNC"]; gDecPCtoNC = ex(-ms / gDecTauPCtoNC);
	gLeakNC = raw["rawGLeakNC"] / (6 - ms);
	threshDecTauNC = raw["threshDecayTNC"]; threshDecNC = 1 - ex(-ms / threshDecTauNC);
	threshMaxNC = raw["threshMaxNC"]; threshRestNC = raw["threshBaseNC"];
	relPDecTSofNCtoIO = raw["outIORelPDecTSNC"]; relPDecTTofNCtoIO = raw["outIORelPDecTTNC"];
	relPDecT0ofNCtoIO = raw["outIORelPDecT0NC"]; relPIncNCtoIO = raw["outIORelPIncScaleNC"];
	relPIncTauNCtoIO = raw["outIORelPIncTNC"]; initSynWofMFtoNC = raw["mfSynWInitNC"];
	synLTDPCPopActThreshMFtoNC = raw["mfNCLTDThreshNC"];
	synLTPPCPopActThreshMFtoNC = raw["mfNCLTPThreshNC"];
	synLTDStepSizeMFtoNC = raw["mfNCLTDDecNC"]; synLTPStepSizeMFtoNC = raw["mfNCLTPIncNC"];
}

bool ActParams::set(const std::string &key, float value)
{
	auto it = raw.find(key);
	if (it == raw.end()) return false;
	it->second = value;
	derive();
	return true;
}

// ----------------------------------------------------------------- layout
namespace {
struct Spec { const char *name; DType t; size_t count; };

// Arrays in stateRW order; innetconnectivitystate.cpp:530-606.  The GR-side
// MF index table is allocated and stored with maxnumpGRfromGOtoGR columns
// there (innetconnectivitystate.cpp:527, 605) and is kept that way.
std::vector<Spec> innetConSpecs(const ConParams &c)
{
	size_t GL = c.numGL, MF = c.numMF, GO = c.numGO, GR = c.numGR;
	return {
		{"haspGLfromMFtoGL", U8, GL}, {"pGLfromMFtoGL", U32, GL},
		{"numpGLfromGLtoGO", I32, GL}, {"pGLfromGLtoGO", U32, GL * c.maxnumpGLfromGLtoGO},
		{"numpGLfromGOtoGL", I32, GL}, {"pGLfromGOtoGL", U32, GL * c.maxnumpGLfromGOtoGL},
		{"numpGLfromGLtoGR", I32, GL}, {"pGLfromGLtoGR", U32, GL * c.maxnumpGLfromGLtoGR},
		{"numpMFfromMFtoGL", I32, MF}, {"pMFfromMFtoGL", U32, MF * c.numpMFfromMFtoGL},
		{"numpMFfromMFtoGR", I32, MF}, {"pMFfromMFtoGR", U32, MF * c.maxnumpMFfromMFtoGR},
		{"numpMFfromMFtoGO", I32, MF}, {"pMFfromMFtoGO", U32, MF * c.maxnumpMFfromMFtoGO},
		{"numpGOfromGLtoGO", I32, GO}, {"pGOfromGLtoGO", U32, GO * c.maxnumpGOfromGLtoGO},
		{"numpGOfromGOtoGL", I32, GO}, {"pGOfromGOtoGL", U32, GO * c.maxnumpGOfromGOtoGL},
		{"numpGOfromMFtoGO", I32, GO}, {"pGOfromMFtoGO", U32, GO * c.maxnumpGOfromMFtoGO},
		{"numpGOfromGOtoGR", I32, GO}, {"pGOfromGOtoGR", U32, GO * c.maxnumpGOfromGOtoGR},
		{"numpGOfromGRtoGO", I32, GO}, {"pGOfromGRtoGO", U32, GO * c.maxnumpGOfromGRtoGO},
		{"numpGOGABAInGOGO", I32, GO}, {"pGOGABAInGOGO", U32, GO * c.maxnumpGOGABAInGOGO},
		{"numpGOGABAOutGOGO", I32, GO}, {"pGOGABAOutGOGO", U32, GO * c.maxnumpGOGABAOutGOGO},
		{"numpGOCoupInGOGO", I32, GO}, {"pGOCoupInGOGO", U32, GO * c.maxnumpGOCoupInGOGO},
		{"numpGOCoupOutGOGO", I32, GO}, {"pGOCoupOutGOGO", U32, GO * c.maxnumpGOCoupOutGOGO},
		{"pGRDelayMaskfromGRtoBSP", U32, GR},
		{"numpGRfromGLtoGR", I32, GR}, {"pGRfromGLtoGR", U32, GR * c.maxnumpGRfromGOtoGR},
		{"numpGRfromGRtoGO", I32, GR}, {"pGRfromGRtoGO", U32, GR * c.maxnumpGRfromGRtoGO},
		{"pGRDelayMaskfromGRtoGO", U32, GR * c.maxnumpGRfromGRtoGO},
		{"numpGRfromGOtoGR", I32, GR}, {"pGRfromGOtoGR", U32, GR * c.maxnumpGRfromGOtoGR},
		{"numpGRfromMFtoGR", I32, GR}, {"pGRfromMFtoGR", U32, GR * c.maxnumpGRfromGOtoGR},
	};
}

// mzoneconnectivitystate.cpp:142-163.  The fifth stored block is a second
// copy of pBCfromPCtoBC (the reference writes and reads it where
// pPCfromPCtoBC belongs); pPCfromPCtoBC itself is rebuilt after loading.
const char *kDupBlock = "pBCfromPCtoBC#2";
std::vector<Spec> zoneConSpecs(const ConParams &c)
{
	return {
		{"pBCfromBCtoPC", U32, (size_t)c.numBC * c.numpBCfromBCtoPC},
		{"pBCfromPCtoBC", U32, (size_t)c.numBC * c.numpBCfromPCtoBC},
		{"pSCfromSCtoPC", U32, (size_t)c.numSC * c.numpSCfromSCtoPC},
		{"pPCfromBCtoPC", U32, (size_t)c.numPC * c.numpPCfromBCtoPC},
		{kDupBlock, U32, (size_t)c.numPC * c.numpPCfromPCtoBC},
		{"pPCfromSCtoPC", U32, (size_t)c.numPC * c.numpPCfromSCtoPC},
		{"pPCfromPCtoNC", U32, (size_t)c.numPC * c.numpPCfromPCtoNC},
		{"pPCfromIOtoPC", U32, (size_t)c.numPC},
		{"pNCfromPCtoNC", U32, (size_t)c.numNC * c.numpNCfromPCtoNC},
		{"pNCfromNCtoIO", U32, (size_t)c.numNC * c.numpNCfromNCtoIO},
		{"pNCfromMFtoNC", U32, (size_t)c.numNC * c.numpNCfromMFtoNC},
		{"pIOfromIOtoPC", U32, (size_t)c.numIO * c.numpIOfromIOtoPC},
		{"pIOfromNCtoIO", U32, (size_t)c.numIO * c.numpIOfromNCtoIO},
		{"pIOInIOIO", U32, (size_t)c.numIO * c.numpIOInIOIO},
		{"pIOOutIOIO", U32, (size_t)c.numIO * c.numpIOOutIOIO},
	};
}

// innetactivitystate.cpp:233-275
std::vector<Spec> innetActSpecs(const ConParams &c)
{
	size_t MF = c.numMF, GO = c.numGO, GR = c.numGR, SC = c.numSC;
	return {
		{"histMF", U8, MF}, {"apBufMF", U32, MF},
		{"apGO", U8, GO}, {"apBufGO", U32, GO}, {"vGO", F32, GO}, {"vCoupleGO", F32, GO},
		{"threshCurGO", F32, GO}, {"inputMFGO", U32, GO}, {"inputGOGO", U32, GO},
		{"gMFGO", F32, GO}, {"gGRGO", F32, GO}, {"gGOGO", F32, GO}, {"gMGluRGO", F32, GO},
		{"gMGluRIncGO", F32, GO}, {"mGluRGO", F32, GO}, {"gluGO", F32, GO},
		{"apGR", U8, GR}, {"apBufGR", U32, GR},
		{"gMFGR", F32, GR * c.maxnumpGRfromMFtoGR}, {"gMFSumGR", F32, GR},
		{"gGOGR", F32, GR * c.maxnumpGRfromGOtoGR}, {"gGOSumGR", F32, GR},
		{"threshGR", F32, GR}, {"vGR", F32, GR}, {"gKCaGR", F32, GR}, {"historyGR", U64, GR},
		{"apSC", U8, SC}, {"apBufSC", U32, SC}, {"gPFSC", F32, SC}, {"threshSC", F32, SC},
		{"vSC", F32, SC}, {"inputSumPFSC", U32, SC},
	};
}

// mzoneactivitystate.cpp:299-355
std::vector<Spec> zoneActSpecs(const ConParams &c, const ActParams &a)
{
	size_t BC = c.numBC, PC = c.numPC, IO = c.numIO, NC = c.numNC;
	return {
		{"apBC", U8, BC}, {"apBufBC", U32, BC}, {"inputPCBC", U32, BC}, {"gPFBC", F32, BC},
		{"gPCBC", F32, BC}, {"threshBC", F32, BC}, {"vBC", F32, BC},
		{"apPC", U8, PC}, {"apBufPC", U32, PC}, {"inputBCPC", U32, PC},
		{"inputSCPC", U8, PC * c.numpPCfromSCtoPC}, {"pfSynWeightPC", F32, PC * c.numpPCfromGRtoPC},
		{"inputSumPFPC", F32, PC}, {"gPFPC", F32, PC}, {"gBCPC", F32, PC},
		{"gSCPC", F32, PC * c.numpPCfromSCtoPC}, {"vPC", F32, PC}, {"threshPC", F32, PC},
		{"histPCPopAct", U32, a.numPopHistBinsPC},
		{"apIO", U8, IO}, {"apBufIO", U32, IO}, {"inputNCIO", U8, IO * c.numpIOfromNCtoIO},
		{"gNCIO", F32, IO * c.numpIOfromNCtoIO}, {"threshIO", F32, IO}, {"vIO", F32, IO},
		{"vCoupleIO", F32, IO}, {"pfPCPlastTimerIO", I32, IO},
		{"apNC", U8, NC}, {"apBufNC", U32, NC}, {"inputPCNC", U8, NC * c.numpNCfromPCtoNC},
		{"inputMFNC", U8, NC * c.numpNCfromMFtoNC}, {"gPCNC", F32, NC * c.numpNCfromPCtoNC},
		{"gPCScaleNC", F32, NC * c.numpNCfromPCtoNC}, {"mfSynWeightNC", F32, NC * c.numpNCfromMFtoNC},
		{"gmaxNMDAofMFtoNC", F32, NC * c.numpNCfromMFtoNC}, {"gmaxAMPAofMFtoNC", F32, NC * c.numpNCfromMFtoNC},
		{"gMFNMDANC", F32, NC * c.numpNCfromMFtoNC}, {"gMFAMPANC", F32, NC * c.numpNCfromMFtoNC},
		{"threshNC", F32, NC}, {"vNC", F32, NC}, {"synIOPReleaseNC", F32, NC},
	};
}

std::vector<NamedArray> makeArrays(const std::vector<Spec> &specs)
{
	std::vector<NamedArray> out;
	for (const Spec &s : specs) {
		if (!strcmp(s.name, kDupBlock)) continue;
		NamedArray a;
		a.name = s.name; a.dtype = s.t; a.count = s.count;
		a.bytes.assign(s.count * dtypeSize(s.t), 0);
		out.push_back(std::move(a));
	}
	return out;
}

NamedArray *findIn(std::vector<NamedArray> &v, const std::string &n)
{
	for (auto &a : v) if (a.name == n) return &a;
	return nullptr;
}

template <typename T> void fill(NamedArray *a, T v)
{
	T *p = a->as<T>();
	for (size_t i = 0; i < a->count; i++) p[i] = v;
}

struct Tok {
	const std::string &s;
	size_t &pos;
	bool next(std::string &out)
	{
		while (pos < s.size() && isspace((unsigned char)s[pos])) pos++;
		size_t b = pos;
		while (pos < s.size() && !isspace((unsigned char)s[pos])) pos++;
		out = s.substr(b, pos - b);
		return !out.empty();
	}
};
}  // namespace

// ---------------------------------------------------------------- parsing
std::string State::parseHeader(const std::string &text, size_t &pos, bool withZones)
{
	Tok tk{text, pos};
	std::string key, val;
	if (withZones) {
		if (!tk.next(key)) return "missing zone count";
		numZones = (uint32_t)strtoul(key.c_str(), nullptr, 10);
	}
	// ConnectivityParams(fstream&) (connectivityparams.cpp:12-88)
	for (;;) {
		if (!tk.next(key)) return "connectivity parameters not terminated";
		if (key == "connectivityParamEnd") { tk.next(val); break; }
		if (key == "GOGOLocalMatrix" || key == "GOGOCoupLocalMatrix") {
			bool coup = key == "GOGOCoupLocalMatrix";
			std::string k2, v2;
			if (!tk.next(k2) || !tk.next(v2)) return "bad GO-GO matrix";
			uint32_t nin = (uint32_t)strtoul(v2.c_str(), nullptr, 10);
			if (!tk.next(k2) || !tk.next(v2)) return "bad GO-GO matrix";
			uint32_t nout = (uint32_t)strtoul(v2.c_str(), nullptr, 10);
			std::vector<float> m(3 * (size_t)nout);
			for (auto &f : m) { if (!tk.next(v2)) return "bad GO-GO matrix"; f = strtof(v2.c_str(), nullptr); }
			if (coup) { cp.maxnumpGOCoupInGOGO = nin; cp.maxnumpGOCoupOutGOGO = nout; cp.gogoCoupLocalCon = m; }
			else { cp.maxnumpGOGABAInGOGO = nin; cp.maxnumpGOGABAOutGOGO = nout; cp.gogoGABALocalCon = m; cp.hasGABAMatrix = true; }
			continue;
		}
		if (!tk.next(val)) return "connectivity parameter without value";
		cp.raw[key] = (uint32_t)strtoul(val.c_str(), nullptr, 10);
	}
	if (!cp.hasGABAMatrix) return "connectivity parameters lack a GOGOLocalMatrix block";
	// ActivityParams(fstream&) (activityparams.cpp:12-42)
	for (;;) {
		if (!tk.next(key) || !tk.next(val)) return "activity parameters not terminated";
		if (key == "activityParamEnd") break;
		ap.raw[key] = strtof(val.c_str(), nullptr);
	}
	cp.derive();
	ap.derive();
	return "";
}

void State::allocate()
{
	innetCon = makeArrays(innetConSpecs(cp));
	innetAct = makeArrays(innetActSpecs(cp));
	for (const char *n : {"inputGOGABASynDepGO", "goGABAOutSynScaleGOGO"}) {
		NamedArray a; a.name = n; a.dtype = F32; a.count = cp.numGO; a.bytes.assign(4 * (size_t)cp.numGO, 0);
		innetAct.push_back(std::move(a));
	}
	zoneCon.assign(numZones, {});
	zoneAct.assign(numZones, {});
	zoneScalars.assign(numZones, ZoneScalars());
	for (uint32_t z = 0; z < numZones; z++) {
		zoneCon[z] = makeArrays(zoneConSpecs(cp));
		NamedArray a; a.name = "pPCfromPCtoBC"; a.dtype = U32;
		a.count = (size_t)cp.numPC * cp.numpPCfromPCtoBC; a.bytes.assign(4 * a.count, 0);
		zoneCon[z].push_back(std::move(a));
		zoneAct[z] = makeArrays(zoneActSpecs(cp, ap));
	}
}

NamedArray *State::find(const std::string &name, int zone)
{
	if (zone < 0) {
		if (auto *a = findIn(innetCon, name)) return a;
		return findIn(innetAct, name);
	}
	if ((uint32_t)zone >= numZones) return nullptr;
	if (auto *a = findIn(zoneCon[zone], name)) return a;
	return findIn(zoneAct[zone], name);
}

const NamedArray *State::find(const std::string &name, int zone) const
{
	return const_cast<State *>(this)->find(name, zone);
}

// Values the reference's loader leaves undefined are set here:
//  - pPCfromPCtoBC: rebuilt with connectPCtoBC's formula
//    (mzoneconnectivitystate.cpp:242-257), because the file holds a second
//    copy of pBCfromPCtoBC in its place (mzoneconnectivitystate.cpp:150);
//  - the unsaved per-zone scalars: histogram sum recomputed from the stored
//    bins, everything else zero (their values in initializeVals).
// The two GO->GO depression arrays get the values the reference's stateRW
// assigns on every read (innetactivitystate.cpp:247-248).
void State::fixLoaded()
{
	fill<float>(find("inputGOGABASynDepGO"), 1.0f);
	fill<float>(find("goGABAOutSynScaleGOGO"), 0.0f);
	for (uint32_t z = 0; z < numZones; z++) {
		uint32_t *p = find("pPCfromPCtoBC", (int)z)->as<uint32_t>();
		int bcToPCRatio = (int)(cp.numBC / cp.numPC);
		for (int i = 0; i < (int)cp.numPC; i++)
			for (int j = 0; j < (int)cp.numpPCfromPCtoBC; j++) {
				int bcInd = i * bcToPCRatio - 6 + j;
				p[(size_t)i * cp.numpPCfromPCtoBC + j] = (uint32_t)((bcInd % (int)cp.numBC + (int)cp.numBC) % (int)cp.numBC);
			}
		const uint32_t *h = find("histPCPopAct", (int)z)->as<uint32_t>();
		ZoneScalars zs;
		for (uint32_t k = 0; k < ap.numPopHistBinsPC; k++) zs.histPCPopActSum += h[k];
		zoneScalars[z] = zs;
	}
}

std::string State::load(const std::string &path)
{
	std::ifstream f(path, std::ios::binary);
	if (!f) return "cannot open " + path;
	std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	size_t used = 0;
	return loadBytes(data, &used);
}

std::string State::loadBytes(const std::string &data, size_t *consumed)
{
	size_t pos = 0;
	cp = ConParams(); ap = ActParams();
	std::string err = parseHeader(data, pos, true);
	if (!err.empty()) return err;
	if (cp.numGR == 0 || cp.numMF == 0 || cp.numGO == 0 || cp.numPC == 0 || cp.numNC == 0 ||
			cp.numIO == 0 || cp.numSC == 0 || cp.numSC < cp.numPC || cp.numMF < cp.numNC ||
			cp.numPC < cp.numNC || ap.numPopHistBinsPC == 0 || ap.tsPerHistBinGR == 0 ||
			ap.numTSinMFHist == 0 || ap.tsPerPopHistBinPC == 0)
		return "network sizes or time-bin parameters out of the supported range";
	pos += 1;  // cbmstate.cpp:19
	allocate();
	auto readSec = [&](const std::vector<Spec> &specs, std::vector<NamedArray> &arrs) -> bool {
		for (const Spec &s : specs) {
			size_t nb = s.count * dtypeSize(s.t);
			if (pos + nb > data.size()) return false;
			NamedArray *a = findIn(arrs, !strcmp(s.name, kDupBlock) ? "pBCfromPCtoBC" : s.name);
			memcpy(a->bytes.data(), data.data() + pos, nb);
			pos += nb;
		}
		return true;
	};
	if (!readSec(innetConSpecs(cp), innetCon)) return "state file truncated";
	for (uint32_t z = 0; z < numZones; z++) if (!readSec(zoneConSpecs(cp), zoneCon[z])) return "state file truncated";
	if (!readSec(innetActSpecs(cp), innetAct)) return "state file truncated";
	for (uint32_t z = 0; z < numZones; z++) if (!readSec(zoneActSpecs(cp, ap), zoneAct[z])) return "state file truncated";
	fixLoaded();
	*consumed = pos;
	return "";
}

static std::string fmtFloat(float v)
{
	std::ostringstream os;
	os << v;  // ostream's default float format, as writeParams uses
	return os.str();
}

std::string formatHeader(const State &s)
{
	std::ostringstream os;
	os << s.numZones << "\n";
	for (const auto &kv : s.cp.raw) os << kv.first << " " << kv.second << "\n";
	os << "GOGOLocalMatrix\n";
	os << "maxnumpGOInGOtoGO " << s.cp.maxnumpGOGABAInGOGO << "\n";
	os << "maxnumpGOOutGOtoGO " << s.cp.maxnumpGOGABAOutGOGO << "\n";
	for (uint32_t i = 0; i < s.cp.maxnumpGOGABAOutGOGO; i++)
		os << fmtFloat(s.cp.gogoGABALocalCon[3 * i]) << " " << fmtFloat(s.cp.gogoGABALocalCon[3 * i + 1]) << " "
		   << fmtFloat(s.cp.gogoGABALocalCon[3 * i + 2]) << "\n";
	os << "GOGOCoupLocalMatrix\n";
	os << "maxnumpGOCoupInGOtoGO " << s.cp.maxnumpGOCoupInGOGO << "\n";
	os << "maxnumpGOCoupOutGOtoGO " << s.cp.maxnumpGOCoupOutGOGO << "\n";
	for (uint32_t i = 0; i < s.cp.maxnumpGOCoupOutGOGO; i++)
		os << fmtFloat(s.cp.gogoCoupLocalCon[3 * i]) << " " << fmtFloat(s.cp.gogoCoupLocalCon[3 * i + 1]) << " "
		   << fmtFloat(s.cp.gogoCoupLocalCon[3 * i + 2]) << "\n";
	os << "connectivityParamEnd 1\n";
	for (const auto &kv : s.ap.raw) os << kv.first << " " << fmtFloat(kv.second) << "\n";
	os << "activityParamEnd 1\n";
	return os.str();
}

std::string State::save(const std::string &path) const
{
	std::ofstream f(path, std::ios::binary | std::ios::trunc);
	if (!f) return "cannot open " + path + " for writing";
	return writeTo(f);
}

size_t State::fileBytes() const
{
	size_t n = formatHeader(*this).size();
	auto secBytes = [&](const std::vector<Spec> &specs) {
		for (const Spec &s : specs) n += s.count * dtypeSize(s.t);
	};
	secBytes(innetConSpecs(cp));
	for (uint32_t z = 0; z < numZones; z++) secBytes(zoneConSpecs(cp));
	secBytes(innetActSpecs(cp));
	for (uint32_t z = 0; z < numZones; z++) secBytes(zoneActSpecs(cp, ap));
	return n;
}

std::string State::writeTo(std::ostream &f) const
{
	std::string h = formatHeader(*this);
	f.write(h.data(), (std::streamsize)h.size());
	auto writeSec = [&](const std::vector<Spec> &specs, const std::vector<NamedArray> &arrs) {
		for (const Spec &s : specs) {
			const char *n = !strcmp(s.name, kDupBlock) ? "pBCfromPCtoBC" : s.name;
			for (const auto &a : arrs)
				if (a.name == n) { f.write((const char *)a.bytes.data(), (std::streamsize)(s.count * dtypeSize(s.t))); break; }
		}
	};
	writeSec(innetConSpecs(cp), innetCon);
	for (uint32_t z = 0; z < numZones; z++) writeSec(zoneConSpecs(cp), zoneCon[z]);
	writeSec(innetActSpecs(cp), innetAct);
	for (uint32_t z = 0; z < numZones; z++) writeSec(zoneActSpecs(cp, ap), zoneAct[z]);
	return f.good() ? "" : "write error";
}

// ------------------------------------------------------------- new state
// connectPCtoNC (mzoneconnectivitystate.cpp:268-345): each NC takes a
// regular block of PCs, every NC but the last adds random PCs (drawPC)
// that are not full and not yet connected to it, and the last NC takes the
// PCs with free output slots.
void wirePCtoNC(State &s, uint32_t z, const std::function<uint32_t()> &drawPC)
{
	const ConParams &cp = s.cp;
	uint32_t *ncpc = s.find("pNCfromPCtoNC", (int)z)->as<uint32_t>();
	uint32_t *pcnc = s.find("pPCfromPCtoNC", (int)z)->as<uint32_t>();
	std::fill(ncpc, ncpc + (size_t)cp.numNC * cp.numpNCfromPCtoNC, 0xFFFFFFFFu);
	std::fill(pcnc, pcnc + (size_t)cp.numPC * cp.numpPCfromPCtoNC, 0xFFFFFFFFu);
	std::vector<int> pcNum(cp.numPC, 1);
	const uint32_t perNC = cp.numPC / cp.numNC;
	for (uint32_t i = 0; i < cp.numNC; i++)
		for (uint32_t j = 0; j < perNC; j++) {
			uint32_t pc = i * perNC + j;
			ncpc[(size_t)i * cp.numpNCfromPCtoNC + j] = pc;
			pcnc[(size_t)pc * cp.numpPCfromPCtoNC + 0] = i;
		}
	for (uint32_t i = 0; i + 1 < cp.numNC; i++)
		for (uint32_t j = cp.numpNCfromPCtoNC / 3; j < cp.numpNCfromPCtoNC; j++) {
			uint32_t pc = 0;
			for (int tries = 0; tries < 1000000; tries++) {
				pc = drawPC();
				if ((uint32_t)pcNum[pc] >= cp.numpPCfromPCtoNC) continue;
				bool ok = true;
				for (int k = 0; k < pcNum[pc]; k++) if (pcnc[(size_t)pc * cp.numpPCfromPCtoNC + k] == i) { ok = false; break; }
				if (ok) break;
			}
			ncpc[(size_t)i * cp.numpNCfromPCtoNC + j] = pc;
			pcnc[(size_t)pc * cp.numpPCfromPCtoNC + pcNum[pc]] = i;
			pcNum[pc]++;
		}
	uint32_t numSyn = perNC;
	for (uint32_t h = 1; h < cp.numpPCfromPCtoNC; h++)
		for (uint32_t i = 0; i < cp.numPC; i++)
			if ((uint32_t)pcNum[i] < cp.numpPCfromPCtoNC && numSyn < cp.numpNCfromPCtoNC) {
				ncpc[(size_t)(cp.numNC - 1) * cp.numpNCfromPCtoNC + numSyn] = i;
				pcnc[(size_t)i * cp.numpPCfromPCtoNC + pcNum[i]] = cp.numNC - 1;
				pcNum[i]++;
				numSyn++;
			}
}

std::string State::create(const std::string &conText, const std::string &actText, uint32_t nZones,
		const std::vector<int> &pcncSeeds)
{
	cp = ConParams(); ap = ActParams();
	numZones = nZones;
	std::string text = conText + "\n" + actText;
	size_t pos = 0;
	std::string err = parseHeader(text, pos, false);
	if (!err.empty()) return err;
	if (cp.numGR == 0 || cp.numSC < cp.numPC || cp.numPC < cp.numNC || cp.numMF < cp.numNC ||
			ap.numPopHistBinsPC == 0 || ap.tsPerHistBinGR == 0 || ap.numTSinMFHist == 0)
		return "network sizes or time-bin parameters out of the supported range";
	allocate();
	// InNetConnectivityState::initializeVals (innetconnectivitystate.cpp:650-713)
	for (auto &a : innetCon) {
		if (a.name.compare(0, 4, "nump") == 0 || a.name == "haspGLfromMFtoGL" || a.name == "pGRDelayMaskfromGRtoBSP")
			memset(a.bytes.data(), 0, a.bytes.size());
		else fill<uint32_t>(&a, 0xFFFFFFFFu);
	}
	// InNetActivityState::initializeVals (innetactivitystate.cpp:277-337)
	fill<float>(find("vGO"), ap.eLeakGO);
	fill<float>(find("threshCurGO"), ap.threshRestGO);
	fill<float>(find("goGABAOutSynScaleGOGO"), 1.0f);
	fill<float>(find("threshGR"), ap.threshRestGR);
	fill<float>(find("vGR"), ap.eLeakGR);
	fill<float>(find("threshSC"), ap.threshRestSC);
	fill<float>(find("vSC"), ap.eLeakSC);
	for (uint32_t z = 0; z < numZones; z++) {
		// MZoneActivityState::initializeVals (mzoneactivitystate.cpp:357-445)
		fill<float>(find("threshBC", z), ap.threshRestBC);
		fill<float>(find("vBC", z), ap.eLeakBC);
		fill<float>(find("vPC", z), ap.eLeakPC);
		fill<float>(find("threshPC", z), ap.threshRestPC);
		fill<float>(find("pfSynWeightPC", z), ap.initSynWofGRtoPC);
		fill<float>(find("threshIO", z), ap.threshRestIO);
		fill<float>(find("vIO", z), ap.eLeakIO);
		fill<float>(find("threshNC", z), ap.threshRestNC);
		fill<float>(find("vNC", z), ap.eLeakNC);
		fill<float>(find("gPCScaleNC", z), ap.gIncAvgPCtoNC);
		fill<float>(find("mfSynWeightNC", z), ap.initSynWofMFtoNC);
		// MZoneConnectivityState wiring (mzoneconnectivitystate.cpp:190-417)
		for (auto &a : zoneCon[z]) fill<uint32_t>(&a, 0xFFFFFFFFu);
		int nPC = (int)cp.numPC, nBC = (int)cp.numBC, ratio = nBC / nPC;
		auto wrap = [](int v, int n) { return (uint32_t)((v % n + n) % n); };
		uint32_t *bcpc = find("pBCfromBCtoPC", z)->as<uint32_t>();
		const int offs[4][4] = {{1, -1, 2, -2}, {1, -1, 3, -3}, {3, -3, 6, -6}, {4, -4, 9, -9}};
		for (int i = 0; i < nPC; i++)
			for (int r = 0; r < 4 && r < ratio; r++)
				for (int j = 0; j < 4; j++) bcpc[(size_t)(i * ratio + r) * 4 + j] = wrap(i + offs[r][j], nPC);
		uint32_t *pcbc = find("pPCfromPCtoBC", z)->as<uint32_t>();
		for (int i = 0; i < nPC; i++)
			for (int j = 0; j < (int)cp.numpPCfromPCtoBC; j++) pcbc[(size_t)i * cp.numpPCfromPCtoBC + j] = wrap(i * ratio - 6 + j, nBC);
		// connectSCtoPC
		uint32_t *scpc = find("pSCfromSCtoPC", z)->as<uint32_t>();
		uint32_t *pcsc = find("pPCfromSCtoPC", z)->as<uint32_t>();
		for (uint32_t i = 0; i < cp.numSC; i++) {
			uint32_t pc = i / cp.numpPCfromSCtoPC;
			scpc[i] = pc;
			pcsc[(size_t)pc * cp.numpPCfromSCtoPC + i % cp.numpPCfromSCtoPC] = i;
		}
		// connectPCtoNC: the reference draws the random extra synapses with
		// SFMT IRandomX from the zone's seed; this library's own networks draw
		// them from its counter-based stream keyed by the zone's seed
		// (State::generate uses the reference's generator)
		{
			uint64_t ctr = 0;
			const uint32_t seed = (uint32_t)(z < pcncSeeds.size() ? pcncSeeds[z] : (int)(7919 + z));
			const uint32_t nPC = cp.numPC;
			wirePCtoNC(*this, z, [&]() { return (uint32_t)(rng::uniform24(seed, rng::kStreamWiring, ctr++) * nPC); });
		}
		// connectNCtoIO, connectMFtoNC, connectIOtoPC, connectIOtoIO
		uint32_t *ionc = find("pIOfromNCtoIO", z)->as<uint32_t>();
		uint32_t *ncio = find("pNCfromNCtoIO", z)->as<uint32_t>();
		for (uint32_t i = 0; i < cp.numIO; i++)
			for (uint32_t j = 0; j < cp.numpIOfromNCtoIO; j++) {
				ionc[(size_t)i * cp.numpIOfromNCtoIO + j] = j;
				ncio[(size_t)j * cp.numpNCfromNCtoIO + i] = i;
			}
		uint32_t *ncmf = find("pNCfromMFtoNC", z)->as<uint32_t>();
		for (uint32_t i = 0; i < cp.numMF; i++) ncmf[(size_t)(i / cp.numpNCfromMFtoNC) * cp.numpNCfromMFtoNC + i % cp.numpNCfromMFtoNC] = i;
		uint32_t *iopc = find("pIOfromIOtoPC", z)->as<uint32_t>();
		uint32_t *pcio = find("pPCfromIOtoPC", z)->as<uint32_t>();
		for (uint32_t i = 0; i < cp.numIO; i++)
			for (uint32_t j = 0; j < cp.numpIOfromIOtoPC; j++) {
				uint32_t pc = i * cp.numpIOfromIOtoPC + j;
				iopc[(size_t)i * cp.numpIOfromIOtoPC + j] = pc;
				pcio[pc] = i;
			}
		uint32_t *ioio = find("pIOInIOIO", z)->as<uint32_t>();
		for (uint32_t i = 0; i < cp.numIO; i++) {
			uint32_t in = 0;
			for (uint32_t j = 0; j < cp.numpIOInIOIO; j++) {
				if (in == i) in++;
				ioio[(size_t)i * cp.numpIOInIOIO + j] = in;
				in++;
			}
		}
		zoneScalars[z] = ZoneScalars();
	}
	return "";
}

}  // namespace cbm
