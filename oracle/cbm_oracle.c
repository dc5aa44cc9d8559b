/* Test infrastructure: CPU oracle for the 1 ms cerebellar network step.
 * See cbm_oracle.h.  Compiled with -O2 -ffp-contract=off (oracle/Makefile):
 * every float and double operation is performed once, in the reference's
 * source order, with no fused multiply-add.
 *
 * Type rules of the reference that matter for bit-exact results:
 *  - the reference is C++; exp() of a float argument resolves to the float
 *    overload (expf), exp() of a double argument to the double version.  The
 *    calls below use expf/exp accordingly, per call site.
 *  - literals such as 1.5 and 3.1 are double, so those expressions are
 *    evaluated in double and rounded to float on assignment.
 *  - bool/uint8 flags multiply floats as 0/1 integers. */
#include "cbm_oracle.h"
#include "cbm_stream.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ maps */
/* std::map<std::string, T> with operator[] semantics: keys kept sorted
 * byte-wise; a lookup of a missing key inserts it with value 0
 * (connectivityparams.cpp:12-184 and activityparams.cpp:436-636 rely on
 * this, and writeParams then writes the inserted keys). */
typedef struct { char key[96]; float f; uint32_t u; } kv_t;
typedef struct { kv_t *e; int n, cap; } kvmap_t;

static kv_t *map_at(kvmap_t *m, const char *k)
{
	int lo = 0, hi = m->n;
	while (lo < hi)
	{
		int mid = (lo + hi) / 2;
		int c = strcmp(m->e[mid].key, k);
		if (c == 0) return &m->e[mid];
		if (c < 0) lo = mid + 1; else hi = mid;
	}
	if (m->n == m->cap)
	{
		m->cap = m->cap ? 2 * m->cap : 64;
		m->e = (kv_t *)realloc(m->e, sizeof(kv_t) * m->cap);
	}
	memmove(&m->e[lo + 1], &m->e[lo], sizeof(kv_t) * (m->n - lo));
	memset(&m->e[lo], 0, sizeof(kv_t));
	snprintf(m->e[lo].key, sizeof(m->e[lo].key), "%s", k);
	m->n++;
	return &m->e[lo];
}
static int map_has(const kvmap_t *m, const char *k)
{
	for (int i = 0; i < m->n; i++) if (!strcmp(m->e[i].key, k)) return 1;
	return 0;
}
#define CU(k) (map_at(&o->conMap, k)->u)
#define AF(k) (map_at(&o->actMap, k)->f)

/* ----------------------------------------------------------- the network */
typedef struct {
	/* connectivity (mzoneconnectivitystate.h) */
	uint32_t *pBCfromBCtoPC, *pBCfromPCtoBC, *pSCfromSCtoPC, *pPCfromBCtoPC, *pPCfromPCtoBC,
		*pPCfromSCtoPC, *pPCfromPCtoNC, *pPCfromIOtoPC, *pNCfromPCtoNC, *pNCfromNCtoIO,
		*pNCfromMFtoNC, *pIOfromIOtoPC, *pIOfromNCtoIO, *pIOInIOIO, *pIOOutIOIO;
	/* activity (mzoneactivitystate.h) */
	uint8_t *apBC; uint32_t *apBufBC, *inputPCBC; float *gPFBC, *gPCBC, *threshBC, *vBC;
	uint8_t *apPC; uint32_t *apBufPC, *inputBCPC; uint8_t *inputSCPC; float *pfSynWeightPC,
		*inputSumPFPC, *gPFPC, *gBCPC, *gSCPC, *vPC, *threshPC; uint32_t *histPCPopAct;
	uint32_t histPCPopActSum, histPCPopActCurBinN, pcPopAct;
	uint8_t *apIO; uint32_t *apBufIO; uint8_t *inputNCIO; float errDrive; float *gNCIO, *threshIO,
		*vIO, *vCoupleIO; int32_t *pfPCPlastTimerIO;
	uint8_t noLTPMFNC, noLTDMFNC;
	uint8_t *apNC; uint32_t *apBufNC; uint8_t *inputPCNC, *inputMFNC; float *gPCNC, *gPCScaleNC,
		*mfSynWeightNC, *gmaxNMDAofMFtoNC, *gmaxAMPAofMFtoNC, *gMFNMDANC, *gMFAMPANC,
		*threshNC, *vNC, *synIOPReleaseNC;
	/* MZone object state (mzone.cpp) */
	float tempGRPCLTDStep, tempGRPCLTPStep;
	float *rowsPFPC;          /* inputPFPCGPU: numPC x numpPCfromGRtoPC */
	float *sumPFPCdev;        /* inputSumPFPCMZGPU */
	float *inputSumPFPCMZH;   /* host copy */
	float *pfPCPlastStepIO;
	int seed;
} zone_t;

struct cbm_oracle {
	kvmap_t conMap, actMap;
	uint32_t numZones;
	/* GOGO local matrices (connectivityparams.cpp:41-87) */
	uint32_t maxnumpGOGABAInGOGO, maxnumpGOGABAOutGOGO, maxnumpGOCoupInGOGO, maxnumpGOCoupOutGOGO;
	float *gogoGABALocalCon, *gogoCoupLocalCon;
	int hasGOGOCouple;
	/* derived connectivity (connectivityparams.cpp:90-183) */
	uint32_t glX, glY, numGL, maxnumpGLfromGLtoGR, lownumpGLfromGLtoGR, maxnumpGLfromGLtoGO,
		maxnumpGLfromGOtoGL, numMF, cp_numpMFfromMFtoGL, maxnumpMFfromMFtoGO, maxnumpMFfromMFtoGR,
		numpMFfromMFtoNC, goX, goY, numGO, maxnumpGOfromGRtoGO, maxnumpGOfromGLtoGO,
		maxnumpGOfromMFtoGO, maxnumpGOfromGOtoGL, maxnumpGOfromGOtoGR, grX, grY, numGR, numGRP2,
		grPFVelInGRXPerTStep, grAFDelayInTStep, maxnumpGRfromGRtoGO, maxnumpGRfromGLtoGR,
		maxnumpGRfromGOtoGR, maxnumpGRfromMFtoGR, numSC, numpSCfromGRtoSC, numpSCfromGRtoSCP2,
		numpSCfromSCtoPC, numPC, numpPCfromGRtoPC, numpPCfromGRtoPCP2, numpPCfromBCtoPC,
		numpPCfromPCtoBC, numpPCfromSCtoPC, numpPCfromPCtoNC, numBC, numpBCfromGRtoBC,
		numpBCfromGRtoBCP2, numpBCfromBCtoPC, numpBCfromPCtoBC, numNC, numpNCfromPCtoNC,
		numpNCfromNCtoIO, numpNCfromMFtoNC, numIO, numpIOfromIOtoPC, numpIOfromNCtoIO,
		numpIOInIOIO, numpIOOutIOIO;
	/* derived activity parameters (activityparams.h) */
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

	/* input-net connectivity (innetconnectivitystate.h), file order */
	uint8_t *haspGLfromMFtoGL; uint32_t *pGLfromMFtoGL; int32_t *numpGLfromGLtoGO; uint32_t *pGLfromGLtoGO;
	int32_t *numpGLfromGOtoGL; uint32_t *pGLfromGOtoGL; int32_t *numpGLfromGLtoGR; uint32_t *pGLfromGLtoGR;
	int32_t *numpMFfromMFtoGL; uint32_t *pMFfromMFtoGL; int32_t *numpMFfromMFtoGR; uint32_t *pMFfromMFtoGR;
	int32_t *numpMFfromMFtoGO; uint32_t *pMFfromMFtoGO;
	int32_t *numpGOfromGLtoGO; uint32_t *pGOfromGLtoGO; int32_t *numpGOfromGOtoGL; uint32_t *pGOfromGOtoGL;
	int32_t *numpGOfromMFtoGO; uint32_t *pGOfromMFtoGO; int32_t *numpGOfromGOtoGR; uint32_t *pGOfromGOtoGR;
	int32_t *numpGOfromGRtoGO; uint32_t *pGOfromGRtoGO; int32_t *numpGOGABAInGOGO; uint32_t *pGOGABAInGOGO;
	int32_t *numpGOGABAOutGOGO; uint32_t *pGOGABAOutGOGO; int32_t *numpGOCoupInGOGO; uint32_t *pGOCoupInGOGO;
	int32_t *numpGOCoupOutGOGO; uint32_t *pGOCoupOutGOGO;
	uint32_t *pGRDelayMaskfromGRtoBSP; int32_t *numpGRfromGLtoGR; uint32_t *pGRfromGLtoGR;
	int32_t *numpGRfromGRtoGO; uint32_t *pGRfromGRtoGO; uint32_t *pGRDelayMaskfromGRtoGO;
	int32_t *numpGRfromGOtoGR; uint32_t *pGRfromGOtoGR; int32_t *numpGRfromMFtoGR; uint32_t *pGRfromMFtoGR;

	/* input-net activity (innetactivitystate.h), file order */
	uint8_t *histMF; uint32_t *apBufMF;
	uint8_t *apGO; uint32_t *apBufGO; float *vGO, *vCoupleGO, *threshCurGO; uint32_t *inputMFGO, *inputGOGO;
	float *inputGOGABASynDepGO, *goGABAOutSynScaleGOGO;
	float *gMFGO, *gGRGO, *gGOGO, *gMGluRGO, *gMGluRIncGO, *mGluRGO, *gluGO;
	uint8_t *apGR; uint32_t *apBufGR; float *gMFGR, *gMFSumGR, *gGOGR, *gGOSumGR, *threshGR, *vGR, *gKCaGR;
	uint64_t *historyGR;
	uint8_t *apSC; uint32_t *apBufSC; float *gPFSC, *threshSC, *vSC; uint32_t *inputSumPFSC;

	zone_t *zones;

	/* InNet object state (innet.cpp) */
	float tempGIncGRtoGO;
	uint8_t *outputGR;        /* outputGRGPU */
	uint32_t *apMFH, *apMFdev, *apGOH, *apGOdev;
	uint32_t *pendBC, *sumBCdev, *inputSumPFBCH;   /* PF->BC counts */
	uint32_t *pendSC, *sumSCdev, *inputSumPFSCH;   /* PF->SC counts */
	uint32_t *pendGO, *sumGOdev, *grInputGOSumH;   /* GR->GO counts */
	uint32_t *sumGRInputGO; float *sumInputGOGABASynDepGO;
	const uint8_t *mfIn;      /* MZone::apMFInput */
	uint64_t curTime;
};

/* ----------------------------------------------------------- parameters */
static void derive_con(cbm_oracle *o)
{
	/* connectivityparams.cpp:90-183 */
	o->glX = 1u << CU("glXP2"); o->glY = 1u << CU("glYP2"); o->numGL = o->glX * o->glY;
	o->maxnumpGLfromGLtoGR = CU("maxnumpGLfromGLtoGR");
	o->lownumpGLfromGLtoGR = CU("lownumpGLfromGLtoGR");
	o->maxnumpGLfromGLtoGO = CU("maxnumpGLfromGLtoGO");
	o->maxnumpGLfromGOtoGL = CU("maxnumpGLfromGOtoGL");
	o->numMF = 1u << CU("numMFP2");
	o->cp_numpMFfromMFtoGL = o->numGL / o->numMF;
	o->maxnumpMFfromMFtoGO = o->cp_numpMFfromMFtoGL * o->maxnumpGLfromGLtoGO;
	o->maxnumpMFfromMFtoGR = o->cp_numpMFfromMFtoGL * o->maxnumpGLfromGLtoGR;
	o->numpMFfromMFtoNC = 1;
	o->goX = 1u << CU("goXP2"); o->goY = 1u << CU("goYP2"); o->numGO = o->goX * o->goY;
	o->maxnumpGOfromGRtoGO = CU("maxnumpGOfromGRtoGO");
	o->maxnumpGOfromGLtoGO = CU("maxnumpGOfromGLtoGO");
	o->maxnumpGOfromMFtoGO = o->maxnumpGOfromGLtoGO;
	o->maxnumpGOfromGOtoGL = CU("maxnumpGOfromGOtoGL");
	o->maxnumpGOfromGOtoGR = o->maxnumpGOfromGOtoGL * o->maxnumpGLfromGLtoGR;
	(void)CU("spanGODecDenOnGLX"); (void)CU("spanGODecDenOnGLY");
	(void)CU("spanGOAscDenOnGRX"); (void)CU("spanGOAscDenOnGRY");
	(void)CU("spanGOAxonOnGLX"); (void)CU("spanGOAxonOnGLY");
	o->grX = 1u << CU("grXP2"); o->grY = 1u << CU("grYP2"); o->numGR = o->grX * o->grY;
	o->numGRP2 = CU("grXP2") + CU("grYP2");
	o->grPFVelInGRXPerTStep = CU("grPFVelInGRXPerTStep");
	o->grAFDelayInTStep = CU("grAFDelayInTStep");
	o->maxnumpGRfromGRtoGO = CU("maxnumpGRfromGRtoGO");
	o->maxnumpGRfromGLtoGR = CU("maxnumpGRfromGLtoGR");
	o->maxnumpGRfromGOtoGR = CU("maxnumpGRfromGOtoGR");
	o->maxnumpGRfromMFtoGR = CU("maxnumpGRfromMFtoGR");
	(void)CU("spanGRDenOnGLX"); (void)CU("spanGRDenOnGLY");
	o->numSC = 1u << CU("numSCP2");
	o->numpSCfromGRtoSC = o->numGR / o->numSC;
	o->numpSCfromGRtoSCP2 = o->numGRP2 - CU("numSCP2");
	o->numpSCfromSCtoPC = 1;
	o->numPC = 1u << CU("numPCP2");
	o->numpPCfromGRtoPC = o->numGR / o->numPC;
	o->numpPCfromGRtoPCP2 = o->numGRP2 - CU("numPCP2");
	o->numpPCfromBCtoPC = 16;
	o->numpPCfromPCtoBC = 16;
	o->numpPCfromSCtoPC = o->numSC / o->numPC;
	o->numpPCfromPCtoNC = CU("numpPCfromPCtoNC");
	o->numBC = o->numPC * 4;
	o->numpBCfromGRtoBC = o->numGR / o->numBC;
	o->numpBCfromGRtoBCP2 = o->numGRP2 - (CU("numPCP2") + 2);
	o->numpBCfromBCtoPC = 4;
	o->numpBCfromPCtoBC = 4;
	o->numNC = 1u << CU("numNCP2");
	o->numpNCfromPCtoNC = o->numPC / o->numNC * o->numpPCfromPCtoNC;
	o->numpNCfromNCtoIO = 1u << CU("numIOP2");
	o->numpNCfromMFtoNC = o->numMF / o->numNC;
	o->numIO = 1u << CU("numIOP2");
	o->numpIOfromIOtoPC = o->numPC / o->numIO;
	o->numpIOfromNCtoIO = o->numNC;
	o->numpIOInIOIO = o->numIO - 1;
	o->numpIOOutIOIO = o->numIO - 1;
}

static void derive_act(cbm_oracle *o)
{
	/* activityparams.cpp:436-636; exp() of a float argument is expf */
	float ms;
	o->msPerTimeStep = ms = AF("msPerTimeStep");
	o->msPerHistBinMF = AF("msPerHistBinMF");
	o->numTSinMFHist = (uint32_t)(o->msPerHistBinMF / ms);
	if (!map_has(&o->actMap, "coupleRiRjRatioGO")) map_at(&o->actMap, "coupleRiRjRatioGO")->f = 0;
	if (!map_has(&o->actMap, "goGABAGOGOSynRecTau")) map_at(&o->actMap, "goGABAGOGOSynRecTau")->f = 1;
	if (!map_has(&o->actMap, "goGABAGOGOSynDepF")) map_at(&o->actMap, "goGABAGOGOSynDepF")->f = 1;
	o->eLeakGO = AF("eLeakGO"); o->eMGluRGO = AF("eMGluRGO"); o->eGABAGO = AF("eGABAGO");
	o->threshMaxGO = AF("threshMaxGO"); o->threshRestGO = AF("threshBaseGO");
	o->gIncMFtoGO = AF("gMFIncGO"); o->gIncGRtoGO = AF("gGRIncGO"); o->gGABAIncGOtoGO = AF("gGOIncGO");
	o->coupleRiRjRatioGO = AF("coupleRiRjRatioGO");
	o->gMGluRScaleGRtoGO = AF("gMGluRScaleGO"); o->gMGluRIncScaleGO = AF("gMGluRIncScaleGO");
	o->mGluRScaleGO = AF("mGluRScaleGO"); o->gluScaleGO = AF("gluScaleGO");
	o->gLeakGO = AF("rawGLeakGO") / (6 - ms);
	o->gDecTauMFtoGO = AF("gMFDecayTGO"); o->gDecMFtoGO = expf(-ms / o->gDecTauMFtoGO);
	o->gDecTauGRtoGO = AF("gGRDecayTGO"); o->gDecGRtoGO = expf(-ms / o->gDecTauGRtoGO);
	o->gGABADecTauGOtoGO = AF("gGODecayTGO"); o->gGABADecGOtoGO = expf(-ms / o->gGABADecTauGOtoGO);
	o->goGABAGOGOSynRecTau = AF("goGABAGOGOSynRecTau");
	o->goGABAGOGOSynRec = 1 - expf(-ms / o->goGABAGOGOSynRecTau);
	o->goGABAGOGOSynDepF = AF("goGABAGOGOSynDepF");
	o->mGluRDecayGO = AF("mGluRDecayGO"); o->gMGluRIncDecayGO = AF("gMGluRIncDecayGO");
	o->gMGluRDecGRtoGO = AF("gMGluRDecayGO"); o->gluDecayGO = AF("gluDecayGO");
	o->threshDecTauGO = AF("threshDecayTGO"); o->threshDecGO = 1 - expf(-ms / o->threshDecTauGO);

	o->eLeakGR = AF("eLeakGR"); o->eGOGR = AF("eGOGR"); o->eMFGR = AF("eMFGR");
	o->threshMaxGR = AF("threshMaxGR"); o->threshRestGR = AF("threshBaseGR");
	o->gIncMFtoGR = AF("gMFIncGR"); o->gIncGOtoGR = AF("gGOIncGR");
	o->gDecTauMFtoGR = AF("gMFDecayTGR"); o->gDecMFtoGR = expf(-ms / o->gDecTauMFtoGR);
	o->gDecTauGOtoGR = AF("gGODecayTGR"); o->gDecGOtoGR = expf(-ms / o->gDecTauGOtoGR);
	o->threshDecTauGR = AF("threshDecayTGR"); o->threshDecGR = 1 - expf(-ms / o->threshDecTauGR);
	o->gLeakGR = AF("rawGLeakGR") / (6 - ms);
	o->msPerHistBinGR = AF("msPerHistBinGR"); o->tsPerHistBinGR = (uint32_t)(o->msPerHistBinGR / ms);

	o->eLeakSC = AF("eLeakSC"); o->gLeakSC = AF("rawGLeakSC") / (6 - ms);
	o->gDecTauGRtoSC = AF("gPFDecayTSC"); o->gDecGRtoSC = expf(-ms / o->gDecTauGRtoSC);
	o->threshMaxSC = AF("threshMaxSC"); o->threshRestSC = AF("threshBaseSC");
	o->threshDecTauSC = AF("threshDecayTSC"); o->threshDecSC = 1 - expf(-ms / o->threshDecTauSC);
	o->gIncGRtoSC = AF("pfIncSC");

	o->eLeakBC = AF("eLeakBC"); o->ePCtoBC = AF("ePCBC"); o->gLeakBC = AF("rawGLeakBC") / (6 - ms);
	o->gDecTauGRtoBC = AF("gPFDecayTBC"); o->gDecGRtoBC = expf(-ms / o->gDecTauGRtoBC);
	o->gDecTauPCtoBC = AF("gPCDecayTBC"); o->gDecPCtoBC = expf(-ms / o->gDecTauPCtoBC);
	o->threshDecTauBC = AF("threshDecayTBC"); o->threshDecBC = 1 - expf(-ms / o->threshDecTauBC);
	o->threshRestBC = AF("threshBaseBC"); o->threshMaxBC = AF("threshMaxBC");
	o->gIncGRtoBC = AF("pfIncConstBC"); o->gIncPCtoBC = AF("pcIncConstBC");

	o->initSynWofGRtoPC = AF("pfSynWInitPC"); o->eLeakPC = AF("eLeakPC");
	o->eBCtoPC = AF("eBCPC"); o->eSCtoPC = AF("eSCPC");
	o->threshMaxPC = AF("threshMaxPC"); o->threshRestPC = AF("threshBasePC");
	o->threshDecTauPC = AF("threshDecayTPC"); o->threshDecPC = 1 - expf(-ms / o->threshDecTauPC);
	o->gLeakPC = AF("rawGLeakPC") / (6 - ms);
	o->gDecTauGRtoPC = AF("gPFDecayTPC"); o->gDecGRtoPC = expf(-ms / o->gDecTauGRtoPC);
	o->gDecTauBCtoPC = AF("gBCDecayTPC"); o->gDecBCtoPC = expf(-ms / o->gDecTauBCtoPC);
	o->gDecTauSCtoPC = AF("gSCDecayTPC"); o->gDecSCtoPC = expf(-ms / o->gDecTauSCtoPC);
	o->gIncSCtoPC = AF("gSCIncConstPC"); o->gIncGRtoPC = AF("gPFScaleConstPC");
	o->gIncBCtoPC = AF("gBCScaleConstPC");
	o->tsPopHistPC = (uint32_t)(40 / ms);
	o->tsPerPopHistBinPC = (uint32_t)(5 / ms);
	o->numPopHistBinsPC = o->tsPopHistPC / o->tsPerPopHistBinPC;

	o->coupleRiRjRatioIO = AF("coupleScaleIO"); o->eLeakIO = AF("eLeakIO"); o->eNCtoIO = AF("eNCIO");
	o->gLeakIO = AF("rawGLeakIO") / (6 - ms);
	o->gDecTSofNCtoIO = AF("gNCDecTSIO"); o->gDecTTofNCtoIO = AF("gNCDecTTIO");
	o->gDecT0ofNCtoIO = AF("gNCDecT0IO"); o->gIncNCtoIO = AF("gNCIncScaleIO");
	o->gIncTauNCtoIO = AF("gNCIncTIO"); o->threshRestIO = AF("threshBaseIO");
	o->threshMaxIO = AF("threshMaxIO");
	o->threshDecTauIO = AF("threshDecayTIO"); o->threshDecIO = 1 - expf(-ms / o->threshDecTauIO);
	o->tsLTDDurationIO = (uint32_t)(AF("msLTDDurationIO") / ms);
	o->tsLTDStartAPIO = (int32_t)(AF("msLTDStartAPIO") / ms);
	o->tsLTPStartAPIO = (int32_t)(AF("msLTPStartAPIO") / ms);
	o->synLTPStepSizeGRtoPC = AF("grPCLTPIncIO"); o->synLTDStepSizeGRtoPC = AF("grPCLTDDecIO");
	o->grPCHistCheckBinIO = (uint32_t)abs(o->tsLTDStartAPIO / ((int)o->tsPerHistBinGR));
	o->maxExtIncVIO = AF("maxErrDriveIO");

	o->eLeakNC = AF("eLeakNC"); o->ePCtoNC = AF("ePCNC");
	o->gmaxNMDADecTauMFtoNC = AF("mfNMDADecayTNC"); o->gmaxNMDADecMFtoNC = expf(-ms / o->gmaxNMDADecTauMFtoNC);
	o->gmaxAMPADecTauMFtoNC = AF("mfAMPADecayTNC"); o->gmaxAMPADecMFtoNC = expf(-ms / o->gmaxAMPADecTauMFtoNC);
	o->gNMDAIncMFtoNC = 1 - expf(-ms / AF("rawGMFNMDAIncNC"));
	o->gAMPAIncMFtoNC = 1 - expf(-ms / AF("rawGMFAMPAIncNC"));
	o->gIncAvgPCtoNC = AF("gPCScaleAvgNC");
	o->gDecTauPCtoNC = AF("gPCDecayTNC"); o->gDecPCtoNC = expf(-ms / o->gDecTauPCtoNC);
	o->gLeakNC = AF("rawGLeakNC") / (6 - ms);
	o->threshDecTauNC = AF("threshDecayTNC"); o->threshDecNC = 1 - expf(-ms / o->threshDecTauNC);
	o->threshMaxNC = AF("threshMaxNC"); o->threshRestNC = AF("threshBaseNC");
	o->relPDecTSofNCtoIO = AF("outIORelPDecTSNC"); o->relPDecTTofNCtoIO = AF("outIORelPDecTTNC");
	o->relPDecT0ofNCtoIO = AF("outIORelPDecT0NC"); o->relPIncNCtoIO = AF("outIORelPIncScaleNC");
	o->relPIncTauNCtoIO = AF("outIORelPIncTNC"); o->initSynWofMFtoNC = AF("mfSynWInitNC");
	o->synLTDPCPopActThreshMFtoNC = AF("mfNCLTDThreshNC");
	o->synLTPPCPopActThreshMFtoNC = AF("mfNCLTPThreshNC");
	o->synLTDStepSizeMFtoNC = AF("mfNCLTDDecNC"); o->synLTPStepSizeMFtoNC = AF("mfNCLTPIncNC");
}

/* ---------------------------------------------------------- file format */
typedef struct { const char *buf; size_t len, pos; } rd_t;

static int next_tok(rd_t *r, char *out, size_t outlen)
{
	while (r->pos < r->len && (r->buf[r->pos] == ' ' || r->buf[r->pos] == '\n' ||
			r->buf[r->pos] == '\t' || r->buf[r->pos] == '\r')) r->pos++;
	size_t s = r->pos;
	while (r->pos < r->len && !(r->buf[r->pos] == ' ' || r->buf[r->pos] == '\n' ||
			r->buf[r->pos] == '\t' || r->buf[r->pos] == '\r')) r->pos++;
	size_t n = r->pos - s;
	if (n == 0 || n >= outlen) return -1;
	memcpy(out, r->buf + s, n);
	out[n] = 0;
	return 0;
}

/* reading: 1 = from r, 0 = to w, 2 = allocate only (a new state),
 * 3 = find the array named want (found, foundBytes) */
typedef struct { int reading; rd_t *r; FILE *w; int err; const char *want; void *found; size_t foundBytes; } io_t;

static void *blk(io_t *io, void *p, size_t bytes)
{
	if (io->err || io->reading == 2) return p;
	if (io->reading)
	{
		if (io->r->pos + bytes > io->r->len) { io->err = 1; return p; }
		memcpy(p, io->r->buf + io->r->pos, bytes);
		io->r->pos += bytes;
	}
	else if (bytes && fwrite(p, 1, bytes, io->w) != bytes) io->err = 1;
	return p;
}

/* an array's block, or in find mode its address when its field name
 * (the text after "->") is the one wanted */
static void blk_named(io_t *io, const char *field, void *p, size_t bytes)
{
	if (io->reading != 3) { blk(io, p, bytes); return; }
	const char *arrow = strstr(field, "->");
	if (arrow && !io->found && !strcmp(arrow + 2, io->want)) { io->found = p; io->foundBytes = bytes; }
}

#define ALLOC(ptr, n) do { size_t cnt_ = (size_t)(n); if (!(ptr)) (ptr) = calloc(cnt_ ? cnt_ : 1, sizeof(*(ptr))); } while (0)
#define RW(ptr, n) do { ALLOC(ptr, n); blk_named(io, #ptr, (ptr), (size_t)(n) * sizeof(*(ptr))); } while (0)

/* innetconnectivitystate.cpp:530-606 */
static void rw_innet_con(cbm_oracle *o, io_t *io)
{
	RW(o->haspGLfromMFtoGL, o->numGL); RW(o->pGLfromMFtoGL, o->numGL);
	RW(o->numpGLfromGLtoGO, o->numGL); RW(o->pGLfromGLtoGO, (size_t)o->numGL * o->maxnumpGLfromGLtoGO);
	RW(o->numpGLfromGOtoGL, o->numGL); RW(o->pGLfromGOtoGL, (size_t)o->numGL * o->maxnumpGLfromGOtoGL);
	RW(o->numpGLfromGLtoGR, o->numGL); RW(o->pGLfromGLtoGR, (size_t)o->numGL * o->maxnumpGLfromGLtoGR);
	RW(o->numpMFfromMFtoGL, o->numMF); RW(o->pMFfromMFtoGL, (size_t)o->numMF * o->cp_numpMFfromMFtoGL);
	RW(o->numpMFfromMFtoGR, o->numMF); RW(o->pMFfromMFtoGR, (size_t)o->numMF * o->maxnumpMFfromMFtoGR);
	RW(o->numpMFfromMFtoGO, o->numMF); RW(o->pMFfromMFtoGO, (size_t)o->numMF * o->maxnumpMFfromMFtoGO);
	RW(o->numpGOfromGLtoGO, o->numGO); RW(o->pGOfromGLtoGO, (size_t)o->numGO * o->maxnumpGOfromGLtoGO);
	RW(o->numpGOfromGOtoGL, o->numGO); RW(o->pGOfromGOtoGL, (size_t)o->numGO * o->maxnumpGOfromGOtoGL);
	RW(o->numpGOfromMFtoGO, o->numGO); RW(o->pGOfromMFtoGO, (size_t)o->numGO * o->maxnumpGOfromMFtoGO);
	RW(o->numpGOfromGOtoGR, o->numGO); RW(o->pGOfromGOtoGR, (size_t)o->numGO * o->maxnumpGOfromGOtoGR);
	RW(o->numpGOfromGRtoGO, o->numGO); RW(o->pGOfromGRtoGO, (size_t)o->numGO * o->maxnumpGOfromGRtoGO);
	RW(o->numpGOGABAInGOGO, o->numGO); RW(o->pGOGABAInGOGO, (size_t)o->numGO * o->maxnumpGOGABAInGOGO);
	RW(o->numpGOGABAOutGOGO, o->numGO); RW(o->pGOGABAOutGOGO, (size_t)o->numGO * o->maxnumpGOGABAOutGOGO);
	RW(o->numpGOCoupInGOGO, o->numGO); RW(o->pGOCoupInGOGO, (size_t)o->numGO * o->maxnumpGOCoupInGOGO);
	RW(o->numpGOCoupOutGOGO, o->numGO); RW(o->pGOCoupOutGOGO, (size_t)o->numGO * o->maxnumpGOCoupOutGOGO);
	RW(o->pGRDelayMaskfromGRtoBSP, o->numGR);
	RW(o->numpGRfromGLtoGR, o->numGR); RW(o->pGRfromGLtoGR, (size_t)o->numGR * o->maxnumpGRfromGOtoGR);
	RW(o->numpGRfromGRtoGO, o->numGR); RW(o->pGRfromGRtoGO, (size_t)o->maxnumpGRfromGRtoGO * o->numGR);
	RW(o->pGRDelayMaskfromGRtoGO, (size_t)o->maxnumpGRfromGRtoGO * o->numGR);
	RW(o->numpGRfromGOtoGR, o->numGR); RW(o->pGRfromGOtoGR, (size_t)o->maxnumpGRfromGOtoGR * o->numGR);
	/* pGRfromMFtoGR is allocated and stored with maxnumpGRfromGOtoGR columns
	 * (innetconnectivitystate.cpp:527, 605) */
	RW(o->numpGRfromMFtoGR, o->numGR); RW(o->pGRfromMFtoGR, (size_t)o->maxnumpGRfromGOtoGR * o->numGR);
}

/* mzoneconnectivitystate.cpp:142-163; the fifth block holds pBCfromPCtoBC
 * again (the reference writes and reads it where pPCfromPCtoBC belongs). */
static void rw_mzone_con(cbm_oracle *o, zone_t *z, io_t *io)
{
	RW(z->pBCfromBCtoPC, (size_t)o->numBC * o->numpBCfromBCtoPC);
	RW(z->pBCfromPCtoBC, (size_t)o->numBC * o->numpBCfromPCtoBC);
	RW(z->pSCfromSCtoPC, (size_t)o->numSC * o->numpSCfromSCtoPC);
	RW(z->pPCfromBCtoPC, (size_t)o->numPC * o->numpPCfromBCtoPC);
	blk(io, z->pBCfromPCtoBC, (size_t)o->numPC * o->numpPCfromPCtoBC * sizeof(uint32_t));
	ALLOC(z->pPCfromPCtoBC, (size_t)o->numPC * o->numpPCfromPCtoBC);
	RW(z->pPCfromSCtoPC, (size_t)o->numPC * o->numpPCfromSCtoPC);
	RW(z->pPCfromPCtoNC, (size_t)o->numPC * o->numpPCfromPCtoNC);
	RW(z->pPCfromIOtoPC, o->numPC);
	RW(z->pNCfromPCtoNC, (size_t)o->numNC * o->numpNCfromPCtoNC);
	RW(z->pNCfromNCtoIO, (size_t)o->numNC * o->numpNCfromNCtoIO);
	RW(z->pNCfromMFtoNC, (size_t)o->numNC * o->numpNCfromMFtoNC);
	RW(z->pIOfromIOtoPC, (size_t)o->numIO * o->numpIOfromIOtoPC);
	RW(z->pIOfromNCtoIO, (size_t)o->numIO * o->numpIOfromNCtoIO);
	RW(z->pIOInIOIO, (size_t)o->numIO * o->numpIOInIOIO);
	RW(z->pIOOutIOIO, (size_t)o->numIO * o->numpIOOutIOIO);
}

/* innetactivitystate.cpp:233-275 (the two GO->GO depression arrays are not
 * stored; they are reset to 1 and 0 on every read and write) */
static void rw_innet_act(cbm_oracle *o, io_t *io)
{
	RW(o->histMF, o->numMF); RW(o->apBufMF, o->numMF);
	RW(o->apGO, o->numGO); RW(o->apBufGO, o->numGO); RW(o->vGO, o->numGO); RW(o->vCoupleGO, o->numGO);
	RW(o->threshCurGO, o->numGO); RW(o->inputMFGO, o->numGO); RW(o->inputGOGO, o->numGO);
	ALLOC(o->inputGOGABASynDepGO, o->numGO); ALLOC(o->goGABAOutSynScaleGOGO, o->numGO);
	for (uint32_t i = 0; i < o->numGO; i++) { o->inputGOGABASynDepGO[i] = 1; o->goGABAOutSynScaleGOGO[i] = 0; }
	RW(o->gMFGO, o->numGO); RW(o->gGRGO, o->numGO); RW(o->gGOGO, o->numGO); RW(o->gMGluRGO, o->numGO);
	RW(o->gMGluRIncGO, o->numGO); RW(o->mGluRGO, o->numGO); RW(o->gluGO, o->numGO);
	RW(o->apGR, o->numGR); RW(o->apBufGR, o->numGR);
	RW(o->gMFGR, (size_t)o->numGR * o->maxnumpGRfromMFtoGR); RW(o->gMFSumGR, o->numGR);
	RW(o->gGOGR, (size_t)o->numGR * o->maxnumpGRfromGOtoGR); RW(o->gGOSumGR, o->numGR);
	RW(o->threshGR, o->numGR); RW(o->vGR, o->numGR); RW(o->gKCaGR, o->numGR); RW(o->historyGR, o->numGR);
	RW(o->apSC, o->numSC); RW(o->apBufSC, o->numSC); RW(o->gPFSC, o->numSC); RW(o->threshSC, o->numSC);
	RW(o->vSC, o->numSC); RW(o->inputSumPFSC, o->numSC);
}

/* mzoneactivitystate.cpp:299-355 */
static void rw_mzone_act(cbm_oracle *o, zone_t *z, io_t *io)
{
	RW(z->apBC, o->numBC); RW(z->apBufBC, o->numBC); RW(z->inputPCBC, o->numBC); RW(z->gPFBC, o->numBC);
	RW(z->gPCBC, o->numBC); RW(z->threshBC, o->numBC); RW(z->vBC, o->numBC);
	RW(z->apPC, o->numPC); RW(z->apBufPC, o->numPC); RW(z->inputBCPC, o->numPC);
	RW(z->inputSCPC, (size_t)o->numPC * o->numpPCfromSCtoPC);
	RW(z->pfSynWeightPC, (size_t)o->numPC * o->numpPCfromGRtoPC);
	RW(z->inputSumPFPC, o->numPC); RW(z->gPFPC, o->numPC); RW(z->gBCPC, o->numPC);
	RW(z->gSCPC, (size_t)o->numPC * o->numpPCfromSCtoPC); RW(z->vPC, o->numPC); RW(z->threshPC, o->numPC);
	RW(z->histPCPopAct, o->numPopHistBinsPC);
	RW(z->apIO, o->numIO); RW(z->apBufIO, o->numIO);
	RW(z->inputNCIO, (size_t)o->numIO * o->numpIOfromNCtoIO); RW(z->gNCIO, (size_t)o->numIO * o->numpIOfromNCtoIO);
	RW(z->threshIO, o->numIO); RW(z->vIO, o->numIO); RW(z->vCoupleIO, o->numIO); RW(z->pfPCPlastTimerIO, o->numIO);
	RW(z->apNC, o->numNC); RW(z->apBufNC, o->numNC);
	RW(z->inputPCNC, (size_t)o->numNC * o->numpNCfromPCtoNC); RW(z->inputMFNC, (size_t)o->numNC * o->numpNCfromMFtoNC);
	RW(z->gPCNC, (size_t)o->numNC * o->numpNCfromPCtoNC); RW(z->gPCScaleNC, (size_t)o->numNC * o->numpNCfromPCtoNC);
	RW(z->mfSynWeightNC, (size_t)o->numNC * o->numpNCfromMFtoNC);
	RW(z->gmaxNMDAofMFtoNC, (size_t)o->numNC * o->numpNCfromMFtoNC);
	RW(z->gmaxAMPAofMFtoNC, (size_t)o->numNC * o->numpNCfromMFtoNC);
	RW(z->gMFNMDANC, (size_t)o->numNC * o->numpNCfromMFtoNC); RW(z->gMFAMPANC, (size_t)o->numNC * o->numpNCfromMFtoNC);
	RW(z->threshNC, o->numNC); RW(z->vNC, o->numNC); RW(z->synIOPReleaseNC, o->numNC);
}

static void setup_runtime(cbm_oracle *o)
{
	/* InNet::InNet / initCUDA and MZone::MZone / initCUDA (innet.cpp:11-606,
	 * mzone.cpp:12-137): device copies start from the state, pipeline
	 * buffers and host mirrors start at zero. */
	o->tempGIncGRtoGO = o->gIncGRtoGO;
	o->outputGR = calloc(o->numGR, 1);
	o->apMFH = calloc(o->numMF, 4); o->apMFdev = calloc(o->numMF, 4);
	o->apGOH = calloc(o->numGO, 4); o->apGOdev = calloc(o->numGO, 4);
	o->pendBC = calloc(o->numBC, 4); o->sumBCdev = calloc(o->numBC, 4); o->inputSumPFBCH = calloc(o->numBC, 4);
	o->pendSC = calloc(o->numSC, 4); o->sumSCdev = calloc(o->numSC, 4); o->inputSumPFSCH = calloc(o->numSC, 4);
	o->pendGO = calloc(o->numGO, 4); o->sumGOdev = calloc(o->numGO, 4); o->grInputGOSumH = calloc(o->numGO, 4);
	o->sumGRInputGO = calloc(o->numGO, 4); o->sumInputGOGABASynDepGO = calloc(o->numGO, 4);
	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		zone_t *z = &o->zones[zi];
		z->tempGRPCLTDStep = o->synLTDStepSizeGRtoPC;
		z->tempGRPCLTPStep = o->synLTPStepSizeGRtoPC;
		z->rowsPFPC = calloc(o->numGR, 4);
		z->sumPFPCdev = calloc(o->numPC, 4);
		z->inputSumPFPCMZH = calloc(o->numPC, 4);
		z->pfPCPlastStepIO = calloc(o->numIO, 4);
		z->seed = 1000 + (int)zi;
		/* values the reference's loader does not restore; set as the B200 loader does */
		int bcToPCRatio = (int)(o->numBC / o->numPC);
		for (int i = 0; i < (int)o->numPC; i++)
			for (int j = 0; j < (int)o->numpPCfromPCtoBC; j++)
			{
				int bcInd = i * bcToPCRatio - 6 + j;
				z->pPCfromPCtoBC[(size_t)i * o->numpPCfromPCtoBC + j] =
					(uint32_t)((bcInd % (int)o->numBC + (int)o->numBC) % (int)o->numBC);
			}
		uint32_t s = 0;
		for (uint32_t k = 0; k < o->numPopHistBinsPC; k++) s += z->histPCPopAct[k];
		z->histPCPopActSum = s; z->histPCPopActCurBinN = 0; z->pcPopAct = 0; z->errDrive = 0;
		z->noLTPMFNC = 0; z->noLTDMFNC = 0;
	}
	o->curTime = 0;
}

static int parse_header(cbm_oracle *o, rd_t *rp);

cbm_oracle *cbm_oracle_load(const char *path, char *err, size_t errlen)
{
	FILE *f = fopen(path, "rb");
	if (!f) { snprintf(err, errlen, "cannot open %s", path); return NULL; }
	fseek(f, 0, SEEK_END);
	long len = ftell(f);
	fseek(f, 0, SEEK_SET);
	char *buf = malloc((size_t)len + 1);
	if (fread(buf, 1, (size_t)len, f) != (size_t)len) { fclose(f); free(buf); snprintf(err, errlen, "read error"); return NULL; }
	fclose(f);
	rd_t r = { buf, (size_t)len, 0 };
	cbm_oracle *o = calloc(1, sizeof(cbm_oracle));
	if (parse_header(o, &r)) goto bad;
	o->zones = calloc(o->numZones ? o->numZones : 1, sizeof(zone_t));
	io_t io = { 1, &r, NULL, 0 };
	rw_innet_con(o, &io);
	for (uint32_t z = 0; z < o->numZones; z++) rw_mzone_con(o, &o->zones[z], &io);
	rw_innet_act(o, &io);
	for (uint32_t z = 0; z < o->numZones; z++) rw_mzone_act(o, &o->zones[z], &io);
	if (io.err) { snprintf(err, errlen, "state file truncated"); free(buf); cbm_oracle_free(o); return NULL; }
	free(buf);
	setup_runtime(o);
	return o;
bad:
	snprintf(err, errlen, "malformed parameter header");
	free(buf);
	cbm_oracle_free(o);
	return NULL;
}

/* The state file's text header (cbmstate.cpp:12-19): numZones, the
 * connectivity parameters (ConnectivityParams(fstream&),
 * connectivityparams.cpp:12-88), the activity parameters
 * (ActivityParams(fstream&), activityparams.cpp:12-30), then one separator
 * byte.  Derives both parameter sets.  Returns 0, or -1 when malformed. */
static int parse_header(cbm_oracle *o, rd_t *rp)
{
	rd_t r = *rp;
	char tok[128];
	/* cbmstate.cpp:14: numZones, then ConnectivityParams(fstream&) */
	if (next_tok(&r, tok, sizeof tok)) goto bad;
	o->numZones = (uint32_t)strtoul(tok, NULL, 10);
	for (;;)
	{
		if (next_tok(&r, tok, sizeof tok)) goto bad;
		if (!strcmp(tok, "connectivityParamEnd")) { if (next_tok(&r, tok, sizeof tok)) goto bad; break; }
		if (!strcmp(tok, "GOGOLocalMatrix") || !strcmp(tok, "GOGOCoupLocalMatrix"))
		{
			int coup = !strcmp(tok, "GOGOCoupLocalMatrix");
			uint32_t vin, vout;
			if (next_tok(&r, tok, sizeof tok) || next_tok(&r, tok, sizeof tok)) goto bad;
			vin = (uint32_t)strtoul(tok, NULL, 10);
			if (next_tok(&r, tok, sizeof tok) || next_tok(&r, tok, sizeof tok)) goto bad;
			vout = (uint32_t)strtoul(tok, NULL, 10);
			float *m = calloc((size_t)vout * 3 + 1, sizeof(float));
			for (uint32_t i = 0; i < vout * 3; i++) { if (next_tok(&r, tok, sizeof tok)) goto bad; m[i] = strtof(tok, NULL); }
			if (coup) { o->hasGOGOCouple = 1; o->maxnumpGOCoupInGOGO = vin; o->maxnumpGOCoupOutGOGO = vout; o->gogoCoupLocalCon = m; }
			else { o->maxnumpGOGABAInGOGO = vin; o->maxnumpGOGABAOutGOGO = vout; o->gogoGABALocalCon = m; }
			continue;
		}
		char val[128];
		if (next_tok(&r, val, sizeof val)) goto bad;
		map_at(&o->conMap, tok)->u = (uint32_t)strtoul(val, NULL, 10);
	}
	if (!o->hasGOGOCouple)
	{
		o->maxnumpGOCoupInGOGO = 1; o->maxnumpGOCoupOutGOGO = 1;
		o->gogoCoupLocalCon = calloc(3, sizeof(float));
		o->gogoCoupLocalCon[0] = 1; o->gogoCoupLocalCon[1] = 1; o->gogoCoupLocalCon[2] = 0;
	}
	for (;;)
	{
		char val[128];
		if (next_tok(&r, tok, sizeof tok) || next_tok(&r, val, sizeof val)) goto bad;
		if (!strcmp(tok, "activityParamEnd")) break;
		map_at(&o->actMap, tok)->f = strtof(val, NULL);
	}
	r.pos += 1; /* cbmstate.cpp:19 */
	derive_con(o);
	derive_act(o);
	*rp = r;
	return 0;
bad:
	return -1;
}

static void write_params(cbm_oracle *o, FILE *f)
{
	/* connectivityparams.cpp:192-218 and activityparams.cpp:243-253 */
	fprintf(f, "%u\n", o->numZones);
	for (int i = 0; i < o->conMap.n; i++) fprintf(f, "%s %u\n", o->conMap.e[i].key, o->conMap.e[i].u);
	fprintf(f, "GOGOLocalMatrix\n");
	fprintf(f, "maxnumpGOInGOtoGO %u\n", o->maxnumpGOGABAInGOGO);
	fprintf(f, "maxnumpGOOutGOtoGO %u\n", o->maxnumpGOGABAOutGOGO);
	for (uint32_t i = 0; i < o->maxnumpGOGABAOutGOGO; i++)
		fprintf(f, "%g %g %g\n", o->gogoGABALocalCon[3 * i], o->gogoGABALocalCon[3 * i + 1], o->gogoGABALocalCon[3 * i + 2]);
	fprintf(f, "GOGOCoupLocalMatrix\n");
	fprintf(f, "maxnumpGOCoupInGOtoGO %u\n", o->maxnumpGOCoupInGOGO);
	fprintf(f, "maxnumpGOCoupOutGOtoGO %u\n", o->maxnumpGOCoupOutGOGO);
	for (uint32_t i = 0; i < o->maxnumpGOCoupOutGOGO; i++)
		fprintf(f, "%g %g %g\n", o->gogoCoupLocalCon[3 * i], o->gogoCoupLocalCon[3 * i + 1], o->gogoCoupLocalCon[3 * i + 2]);
	fprintf(f, "connectivityParamEnd 1\n");
	for (int i = 0; i < o->actMap.n; i++) fprintf(f, "%s %g\n", o->actMap.e[i].key, (double)o->actMap.e[i].f);
	fprintf(f, "activityParamEnd 1\n");
}

int cbm_oracle_save(cbm_oracle *o, const char *path)
{
	/* CBMSimCore::writeToState (cbmsimcore.cpp:65-80): device GR arrays back
	 * into the state (innet.cpp:608-667), the PC weights and PC input sums
	 * (mzone.cpp:139-147), then CBMState::writeState. */
	memcpy(o->apGR, o->outputGR, o->numGR);
	for (uint32_t i = 0; i < o->numSC; i++) o->inputSumPFSC[i] = o->inputSumPFSCH[i];
	for (uint32_t zi = 0; zi < o->numZones; zi++)
		for (uint32_t i = 0; i < o->numPC; i++) o->zones[zi].inputSumPFPC[i] = o->zones[zi].inputSumPFPCMZH[i];
	FILE *f = fopen(path, "wb");
	if (!f) return -1;
	write_params(o, f);
	io_t io = { 0, NULL, f, 0 };
	rw_innet_con(o, &io);
	for (uint32_t z = 0; z < o->numZones; z++) rw_mzone_con(o, &o->zones[z], &io);
	rw_innet_act(o, &io);
	for (uint32_t z = 0; z < o->numZones; z++) rw_mzone_act(o, &o->zones[z], &io);
	fclose(f);
	return io.err ? -1 : 0;
}

/* ------------------------------------------------------------ new state */
#define FILL(ptr, n, v) do { for (size_t i_ = 0; i_ < (size_t)(n); i_++) (ptr)[i_] = (v); } while (0)

cbm_oracle *cbm_oracle_new(const char *conText, const char *actText, uint32_t nZones, const int *pcncSeeds,
		char *err, size_t errlen)
{
	/* CBMState(actPF, conPF, nZones, ...) (CBM_STATE_LIB_DEV/src/interfaces/
	 * cbmstate.cpp:60-64, 176-204) without the spatial input-net generator:
	 * the parameters, every array allocated, the initial values of
	 * InNetConnectivityState::initializeVals (innetconnectivitystate.cpp:
	 * 650-713), InNetActivityState::initializeVals (innetactivitystate.cpp:
	 * 277-337), MZoneActivityState::initializeVals (mzoneactivitystate.cpp:
	 * 357-445) and the microzone wiring of MZoneConnectivityState
	 * (mzoneconnectivitystate.cpp:12-40, 187-417).  The input-net tables are
	 * left at their initial values for the caller to fill.  The random
	 * PC->NC synapses (connectPCtoNC's IRandomX draws from SFMT seeded with
	 * the zone's seed) are drawn from the counter-based stream keyed by
	 * pcncSeeds[z], index = (int)(draw * numPC), retried while the PC is full
	 * or already connected to that NC. */
	size_t lc = strlen(conText), la = strlen(actText);
	char *buf = malloc(lc + la + 32);
	int n0 = snprintf(buf, 32, "%u\n", nZones);
	memcpy(buf + n0, conText, lc);
	buf[n0 + lc] = '\n';
	memcpy(buf + n0 + lc + 1, actText, la);
	size_t len = (size_t)n0 + lc + 1 + la;
	buf[len] = '\n';
	rd_t r = { buf, len + 1, 0 };
	cbm_oracle *o = calloc(1, sizeof(cbm_oracle));
	if (parse_header(o, &r))
	{
		snprintf(err, errlen, "malformed parameter text");
		free(buf);
		cbm_oracle_free(o);
		return NULL;
	}
	free(buf);
	o->zones = calloc(o->numZones ? o->numZones : 1, sizeof(zone_t));
	io_t io = { 2, NULL, NULL, 0, NULL, NULL, 0 };
	rw_innet_con(o, &io);
	for (uint32_t z = 0; z < o->numZones; z++) rw_mzone_con(o, &o->zones[z], &io);
	rw_innet_act(o, &io);
	for (uint32_t z = 0; z < o->numZones; z++) rw_mzone_act(o, &o->zones[z], &io);

	/* input-net connectivity: counts and has-flags 0, indices UINT_MAX,
	 * the BSP delay masks 0 */
	FILL(o->pGLfromMFtoGL, o->numGL, UINT32_MAX);
	FILL(o->pGLfromGLtoGO, (size_t)o->numGL * o->maxnumpGLfromGLtoGO, UINT32_MAX);
	FILL(o->pGLfromGOtoGL, (size_t)o->numGL * o->maxnumpGLfromGOtoGL, UINT32_MAX);
	FILL(o->pGLfromGLtoGR, (size_t)o->numGL * o->maxnumpGLfromGLtoGR, UINT32_MAX);
	FILL(o->pMFfromMFtoGL, (size_t)o->numMF * o->cp_numpMFfromMFtoGL, UINT32_MAX);
	FILL(o->pMFfromMFtoGR, (size_t)o->numMF * o->maxnumpMFfromMFtoGR, UINT32_MAX);
	FILL(o->pMFfromMFtoGO, (size_t)o->numMF * o->maxnumpMFfromMFtoGO, UINT32_MAX);
	FILL(o->pGOfromGLtoGO, (size_t)o->numGO * o->maxnumpGOfromGLtoGO, UINT32_MAX);
	FILL(o->pGOfromGOtoGL, (size_t)o->numGO * o->maxnumpGOfromGOtoGL, UINT32_MAX);
	FILL(o->pGOfromMFtoGO, (size_t)o->numGO * o->maxnumpGOfromMFtoGO, UINT32_MAX);
	FILL(o->pGOfromGOtoGR, (size_t)o->numGO * o->maxnumpGOfromGOtoGR, UINT32_MAX);
	FILL(o->pGOfromGRtoGO, (size_t)o->numGO * o->maxnumpGOfromGRtoGO, UINT32_MAX);
	FILL(o->pGOGABAInGOGO, (size_t)o->numGO * o->maxnumpGOGABAInGOGO, UINT32_MAX);
	FILL(o->pGOGABAOutGOGO, (size_t)o->numGO * o->maxnumpGOGABAOutGOGO, UINT32_MAX);
	FILL(o->pGOCoupInGOGO, (size_t)o->numGO * o->maxnumpGOCoupInGOGO, UINT32_MAX);
	FILL(o->pGOCoupOutGOGO, (size_t)o->numGO * o->maxnumpGOCoupOutGOGO, UINT32_MAX);
	/* the GR tables, over the whole allocation (pGRfromGLtoGR and
	 * pGRfromMFtoGR are stored with maxnumpGRfromGOtoGR columns) */
	FILL(o->pGRfromGLtoGR, (size_t)o->numGR * o->maxnumpGRfromGOtoGR, UINT32_MAX);
	FILL(o->pGRfromGRtoGO, (size_t)o->numGR * o->maxnumpGRfromGRtoGO, UINT32_MAX);
	FILL(o->pGRDelayMaskfromGRtoGO, (size_t)o->numGR * o->maxnumpGRfromGRtoGO, UINT32_MAX);
	FILL(o->pGRfromGOtoGR, (size_t)o->numGR * o->maxnumpGRfromGOtoGR, UINT32_MAX);
	FILL(o->pGRfromMFtoGR, (size_t)o->numGR * o->maxnumpGRfromGOtoGR, UINT32_MAX);

	/* input-net activity (everything else starts at 0) */
	FILL(o->vGO, o->numGO, o->eLeakGO);
	FILL(o->threshCurGO, o->numGO, o->threshRestGO);
	FILL(o->threshGR, o->numGR, o->threshRestGR);
	FILL(o->vGR, o->numGR, o->eLeakGR);
	FILL(o->threshSC, o->numSC, o->threshRestSC);
	FILL(o->vSC, o->numSC, o->eLeakSC);

	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		zone_t *z = &o->zones[zi];
		/* MZoneActivityState::initializeVals */
		FILL(z->threshBC, o->numBC, o->threshRestBC);
		FILL(z->vBC, o->numBC, o->eLeakBC);
		FILL(z->vPC, o->numPC, o->eLeakPC);
		FILL(z->threshPC, o->numPC, o->threshRestPC);
		FILL(z->pfSynWeightPC, (size_t)o->numPC * o->numpPCfromGRtoPC, o->initSynWofGRtoPC);
		FILL(z->threshIO, o->numIO, o->threshRestIO);
		FILL(z->vIO, o->numIO, o->eLeakIO);
		FILL(z->threshNC, o->numNC, o->threshRestNC);
		FILL(z->vNC, o->numNC, o->eLeakNC);
		FILL(z->gPCScaleNC, (size_t)o->numNC * o->numpNCfromPCtoNC, o->gIncAvgPCtoNC);
		FILL(z->mfSynWeightNC, (size_t)o->numNC * o->numpNCfromMFtoNC, o->initSynWofMFtoNC);
		/* MZoneConnectivityState::initalizeVars */
		FILL(z->pBCfromBCtoPC, (size_t)o->numBC * o->numpBCfromBCtoPC, UINT32_MAX);
		FILL(z->pBCfromPCtoBC, (size_t)o->numBC * o->numpBCfromPCtoBC, UINT32_MAX);
		FILL(z->pSCfromSCtoPC, (size_t)o->numSC * o->numpSCfromSCtoPC, UINT32_MAX);
		FILL(z->pPCfromBCtoPC, (size_t)o->numPC * o->numpPCfromBCtoPC, UINT32_MAX);
		FILL(z->pPCfromPCtoBC, (size_t)o->numPC * o->numpPCfromPCtoBC, UINT32_MAX);
		FILL(z->pPCfromSCtoPC, (size_t)o->numPC * o->numpPCfromSCtoPC, UINT32_MAX);
		FILL(z->pPCfromPCtoNC, (size_t)o->numPC * o->numpPCfromPCtoNC, UINT32_MAX);
		FILL(z->pPCfromIOtoPC, o->numPC, UINT32_MAX);
		FILL(z->pNCfromPCtoNC, (size_t)o->numNC * o->numpNCfromPCtoNC, UINT32_MAX);
		FILL(z->pNCfromNCtoIO, (size_t)o->numNC * o->numpNCfromNCtoIO, UINT32_MAX);
		FILL(z->pNCfromMFtoNC, (size_t)o->numNC * o->numpNCfromMFtoNC, UINT32_MAX);
		FILL(z->pIOfromIOtoPC, (size_t)o->numIO * o->numpIOfromIOtoPC, UINT32_MAX);
		FILL(z->pIOfromNCtoIO, (size_t)o->numIO * o->numpIOfromNCtoIO, UINT32_MAX);
		FILL(z->pIOInIOIO, (size_t)o->numIO * o->numpIOInIOIO, UINT32_MAX);
		FILL(z->pIOOutIOIO, (size_t)o->numIO * o->numpIOOutIOIO, UINT32_MAX);
		const int nPC = (int)o->numPC, nBC = (int)o->numBC, ratio = nBC / nPC;
		/* connectBCtoPC: BC r of each PC's block projects to PCs at the
		 * offsets of its row */
		static const int offs[4][4] = { {1, -1, 2, -2}, {1, -1, 3, -3}, {3, -3, 6, -6}, {4, -4, 9, -9} };
		for (int i = 0; i < nPC; i++)
			for (int rr = 0; rr < 4; rr++)
				for (int j = 0; j < 4; j++)
					z->pBCfromBCtoPC[(size_t)(i * ratio + rr) * o->numpBCfromBCtoPC + j] =
						(uint32_t)(((i + offs[rr][j]) % nPC + nPC) % nPC);
		/* connectPCtoBC */
		for (int i = 0; i < nPC; i++)
			for (int j = 0; j < (int)o->numpPCfromPCtoBC; j++)
			{
				int bcInd = i * ratio - 6 + j;
				z->pPCfromPCtoBC[(size_t)i * o->numpPCfromPCtoBC + j] = (uint32_t)((bcInd % nBC + nBC) % nBC);
			}
		/* connectSCtoPC */
		for (uint32_t i = 0; i < o->numSC; i++)
			for (uint32_t j = 0; j < o->numpSCfromSCtoPC; j++)
			{
				uint32_t pcInd = i / o->numpPCfromSCtoPC;
				z->pSCfromSCtoPC[(size_t)i * o->numpSCfromSCtoPC + j] = pcInd;
				z->pPCfromSCtoPC[(size_t)pcInd * o->numpPCfromSCtoPC + i % o->numpPCfromSCtoPC] = i;
			}
		/* connectPCtoNC */
		int *pcNum = malloc(sizeof(int) * o->numPC);
		for (uint32_t i = 0; i < o->numPC; i++) pcNum[i] = 1;
		const uint32_t perNC = o->numPC / o->numNC;
		for (uint32_t i = 0; i < o->numNC; i++)
			for (uint32_t j = 0; j < perNC; j++)
			{
				uint32_t pcInd = i * perNC + j;
				z->pNCfromPCtoNC[(size_t)i * o->numpNCfromPCtoNC + j] = pcInd;
				z->pPCfromPCtoNC[(size_t)pcInd * o->numpPCfromPCtoNC + 0] = i;
			}
		const uint32_t seed = (uint32_t)(pcncSeeds ? pcncSeeds[zi] : (int)(7919 + zi));
		uint64_t ctr = 0;
		for (uint32_t i = 0; i + 1 < o->numNC; i++)
			for (uint32_t j = o->numpNCfromPCtoNC / 3; j < o->numpNCfromPCtoNC; j++)
			{
				uint32_t pcInd = 0;
				for (long tries = 0; tries < 1000000; tries++)
				{
					pcInd = (uint32_t)(cbm_oracle_uniform24(seed, CBM_STREAM_WIRING, ctr++) * o->numPC);
					if ((uint32_t)pcNum[pcInd] >= o->numpPCfromPCtoNC) continue;
					int connect = 1;
					for (int k = 0; k < pcNum[pcInd]; k++)
						if (z->pPCfromPCtoNC[(size_t)pcInd * o->numpPCfromPCtoNC + k] == i) { connect = 0; break; }
					if (connect) break;
				}
				z->pNCfromPCtoNC[(size_t)i * o->numpNCfromPCtoNC + j] = pcInd;
				z->pPCfromPCtoNC[(size_t)pcInd * o->numpPCfromPCtoNC + pcNum[pcInd]] = i;
				pcNum[pcInd]++;
			}
		{
			uint32_t numSyn = perNC;
			for (uint32_t h = 1; h < o->numpPCfromPCtoNC; h++)
				for (uint32_t i = 0; i < o->numPC; i++)
					if ((uint32_t)pcNum[i] < o->numpPCfromPCtoNC)
					{
						z->pNCfromPCtoNC[(size_t)(o->numNC - 1) * o->numpNCfromPCtoNC + numSyn] = i;
						z->pPCfromPCtoNC[(size_t)i * o->numpPCfromPCtoNC + pcNum[i]] = o->numNC - 1;
						pcNum[i]++;
						numSyn++;
					}
		}
		free(pcNum);
		/* connectNCtoIO */
		for (uint32_t i = 0; i < o->numIO; i++)
			for (uint32_t j = 0; j < o->numpIOfromNCtoIO; j++)
			{
				z->pIOfromNCtoIO[(size_t)i * o->numpIOfromNCtoIO + j] = j;
				z->pNCfromNCtoIO[(size_t)j * o->numpNCfromNCtoIO + i] = i;
			}
		/* connectMFtoNC */
		for (uint32_t i = 0; i < o->numMF; i++)
			z->pNCfromMFtoNC[(size_t)(i / o->numpNCfromMFtoNC) * o->numpNCfromMFtoNC + i % o->numpNCfromMFtoNC] = i;
		/* connectIOtoPC */
		for (uint32_t i = 0; i < o->numIO; i++)
			for (uint32_t j = 0; j < o->numpIOfromIOtoPC; j++)
			{
				uint32_t pcInd = i * o->numpIOfromIOtoPC + j;
				z->pIOfromIOtoPC[(size_t)i * o->numpIOfromIOtoPC + j] = pcInd;
				z->pPCfromIOtoPC[pcInd] = i;
			}
		/* connectIOtoIO */
		for (uint32_t i = 0; i < o->numIO; i++)
		{
			uint32_t inInd = 0;
			for (uint32_t j = 0; j < o->numpIOInIOIO; j++)
			{
				if (inInd == i) inInd++;
				z->pIOInIOIO[(size_t)i * o->numpIOInIOIO + j] = inInd;
				inInd++;
			}
		}
	}
	setup_runtime(o);
	return o;
}

void *cbm_oracle_array(cbm_oracle *o, const char *name, int zone, uint64_t *bytes)
{
	io_t io = { 3, NULL, NULL, 0, name, NULL, 0 };
	if (zone < 0)
	{
		rw_innet_con(o, &io);
		if (!io.found) rw_innet_act(o, &io);
	}
	else if ((uint32_t)zone < o->numZones)
	{
		rw_mzone_con(o, &o->zones[zone], &io);
		if (!io.found) rw_mzone_act(o, &o->zones[zone], &io);
	}
	if (bytes) *bytes = io.foundBytes;
	return io.found;
}

int cbm_oracle_con(const cbm_oracle *o, const char *key, uint32_t *value)
{
	/* derived connectivity parameters (connectivityparams.cpp:90-183) by name */
#define CON_KEY(f) if (!strcmp(key, #f)) { *value = o->f; return 0; }
	CON_KEY(numGL) CON_KEY(numMF) CON_KEY(numGO) CON_KEY(numGR) CON_KEY(numSC) CON_KEY(numPC) CON_KEY(numBC)
	CON_KEY(numNC) CON_KEY(numIO) CON_KEY(maxnumpGLfromGLtoGR) CON_KEY(maxnumpGLfromGLtoGO)
	CON_KEY(maxnumpGLfromGOtoGL) CON_KEY(maxnumpMFfromMFtoGO) CON_KEY(maxnumpMFfromMFtoGR)
	CON_KEY(maxnumpGOfromGRtoGO) CON_KEY(maxnumpGOfromGLtoGO) CON_KEY(maxnumpGOfromMFtoGO)
	CON_KEY(maxnumpGOfromGOtoGL) CON_KEY(maxnumpGOfromGOtoGR) CON_KEY(maxnumpGRfromGRtoGO)
	CON_KEY(maxnumpGRfromGLtoGR) CON_KEY(maxnumpGRfromGOtoGR) CON_KEY(maxnumpGRfromMFtoGR)
	CON_KEY(maxnumpGOGABAInGOGO) CON_KEY(maxnumpGOGABAOutGOGO) CON_KEY(maxnumpGOCoupInGOGO)
	CON_KEY(maxnumpGOCoupOutGOGO) CON_KEY(numpPCfromGRtoPC) CON_KEY(numpBCfromGRtoBC) CON_KEY(numpSCfromGRtoSC)
#undef CON_KEY
	return -1;
}

void cbm_oracle_free(cbm_oracle *o)
{
	/* the process-lifetime allocations of a test oracle are released with
	 * the process; only the top-level objects are freed here */
	if (!o) return;
	free(o->conMap.e);
	free(o->actMap.e);
	free(o->zones);
	free(o);
}

void cbm_oracle_set_seeds(cbm_oracle *o, const int *s)
{
	for (uint32_t z = 0; z < o->numZones; z++) o->zones[z].seed = s[z];
}
void cbm_oracle_update_err_drive(cbm_oracle *o, unsigned zone, float rel)
{
	/* mzone.cpp:167-173 */
	o->zones[zone].errDrive = rel * o->maxExtIncVIO;
}
void cbm_oracle_set_plast_steps(cbm_oracle *o, unsigned zone, float ltd, float ltp)
{
	o->zones[zone].tempGRPCLTDStep = ltd;
	o->zones[zone].tempGRPCLTPStep = ltp;
}
void cbm_oracle_reset_plast_steps(cbm_oracle *o, unsigned zone)
{
	o->zones[zone].tempGRPCLTDStep = o->synLTDStepSizeGRtoPC;
	o->zones[zone].tempGRPCLTPStep = o->synLTPStepSizeGRtoPC;
}
void cbm_oracle_set_ginc_grgo(cbm_oracle *o, float inc) { o->tempGIncGRtoGO = inc; }
void cbm_oracle_reset_ginc_grgo(cbm_oracle *o) { o->tempGIncGRtoGO = o->gIncGRtoGO; }

/* --------------------------------------------------------- the GR kernels */
/* sumInputsNew order (kernels.cu:296-376) for one row of rowLength values */
static float sum_row_ordered(const float *row, uint32_t rowLength)
{
	uint32_t bs;
	if (rowLength >= 2048) bs = 512;
	else if (rowLength >= 512) bs = 128;
	else if (rowLength >= 128) bs = 32;
	else if (rowLength >= 32) bs = 8;
	else bs = 2;
	float s[512];
	for (uint32_t tid = 0; tid < bs; tid++)
	{
		float acc = 0;
		for (uint32_t i = tid; i < rowLength; i += 2 * bs) acc += row[i] + row[i + bs];
		s[tid] = acc;
	}
	for (uint32_t h = bs / 2; h >= 1; h /= 2)
		for (uint32_t t = 0; t < h; t++) s[t] = s[t] + s[t + h];
	return s[0];
}

static void gr_activity(cbm_oracle *o)
{
	/* kernels.cu:79-110 */
	const float gLeak = o->gLeakGR, eLeak = o->eLeakGR, eGOIn = o->eGOGR;
	const float threshBase = o->threshRestGR, threshMax = o->threshMaxGR, threshDecay = o->threshDecGR;
	#pragma omp parallel for schedule(static)
	for (uint32_t i = 0; i < o->numGR; i++)
	{
		float tempV = o->vGR[i];
		float tempGKCa = o->gKCaGR[i];
		tempV = tempV + (gLeak + tempGKCa * tempGKCa * tempGKCa * tempGKCa) * (eLeak - tempV)
			- (o->gMFSumGR[i]) * tempV + (o->gGOSumGR[i]) * (eGOIn - tempV);
		float tempThresh = o->threshGR[i];
		tempThresh = tempThresh + (threshBase - tempThresh) * threshDecay;
		unsigned int tempAP = tempV > tempThresh;
		o->threshGR[i] = tempAP * threshMax + (!tempAP) * tempThresh;
		tempGKCa = tempGKCa * 0.9999f;
		o->gKCaGR[i] = tempAP * (tempGKCa + 0.003f) + (!tempAP) * tempGKCa;
		o->apBufGR[i] = (o->apBufGR[i] << 1) | tempAP;
		o->outputGR[i] = (uint8_t)tempAP;
		o->vGR[i] = tempV;
	}
}

static void gr_inputs(cbm_oracle *o, float *gSum, const uint32_t *ap, const int32_t *num,
		const uint32_t *con, uint32_t stride, float gDecay, float gInc)
{
	/* kernels.cu:169-199 (con is [gr][stride], as in the state) */
	#pragma omp parallel for schedule(static)
	for (uint32_t i = 0; i < o->numGR; i++)
	{
		int n = num[i];
		int tempApInSum = 0;
		for (int k = 0; k < n; k++) tempApInSum += (int)ap[con[(size_t)i * stride + k]];
		gSum[i] = gSum[i] * gDecay + gInc * (tempApInSum);
	}
}

/* ------------------------------------------------------- small cells */
static void calc_pc(cbm_oracle *o, zone_t *z)
{
	/* mzone.cpp:187-226 */
	for (uint32_t i = 0; i < o->numPC; i++)
	{
		float gSCPCSum;
		z->gPFPC[i] = z->gPFPC[i] + z->inputSumPFPCMZH[i] * o->gIncGRtoPC;
		z->gPFPC[i] = z->gPFPC[i] * o->gDecGRtoPC;
		z->gBCPC[i] = z->gBCPC[i] + z->inputBCPC[i] * o->gIncBCtoPC;
		z->gBCPC[i] = z->gBCPC[i] * o->gDecBCtoPC;
		gSCPCSum = 0;
		for (uint32_t j = 0; j < o->numpPCfromSCtoPC; j++)
		{
			float *g = &z->gSCPC[(size_t)i * o->numpPCfromSCtoPC + j];
			*g = *g + o->gIncSCtoPC * (1 - *g) * z->inputSCPC[(size_t)i * o->numpPCfromSCtoPC + j];
			*g = *g * o->gDecSCtoPC;
			gSCPCSum += *g;
		}
		z->vPC[i] = z->vPC[i] +
			(o->gLeakPC * (o->eLeakPC - z->vPC[i])) -
			(z->gPFPC[i] * z->vPC[i]) +
			(z->gBCPC[i] * (o->eBCtoPC - z->vPC[i])) +
			(gSCPCSum * (o->eSCtoPC - z->vPC[i]));
		z->threshPC[i] = z->threshPC[i] + (o->threshDecPC * (o->threshRestPC - z->threshPC[i]));
		z->apPC[i] = z->vPC[i] > z->threshPC[i];
		z->apBufPC[i] = (z->apBufPC[i] << 1) | (z->apPC[i] * 0x00000001);
		z->threshPC[i] = z->apPC[i] * o->threshMaxPC + (!z->apPC[i]) * z->threshPC[i];
		z->pcPopAct = z->pcPopAct + z->apPC[i];
	}
}

static void calc_bc(cbm_oracle *o, zone_t *z)
{
	/* mzone.cpp:228-256; the PF->BC sums are the input net's (cbmsimcore.cpp:195) */
	for (uint32_t i = 0; i < o->numBC; i++)
	{
		z->gPFBC[i] = z->gPFBC[i] + (o->inputSumPFBCH[i] * o->gIncGRtoBC);
		z->gPFBC[i] = z->gPFBC[i] * o->gDecGRtoBC;
		z->gPCBC[i] = z->gPCBC[i] + (z->inputPCBC[i] * o->gIncPCtoBC);
		z->gPCBC[i] = z->gPCBC[i] * o->gDecPCtoBC;
		z->vBC[i] = z->vBC[i] +
			(o->gLeakBC * (o->eLeakBC - z->vBC[i])) -
			(z->gPFBC[i] * z->vBC[i]) +
			(z->gPCBC[i] * (o->ePCtoBC - z->vBC[i]));
		z->threshBC[i] = z->threshBC[i] + o->threshDecBC * (o->threshRestBC - z->threshBC[i]);
		z->apBC[i] = z->vBC[i] > z->threshBC[i];
		z->apBufBC[i] = (z->apBufBC[i] << 1) | (z->apBC[i] * 0x00000001);
		z->threshBC[i] = z->apBC[i] * o->threshMaxBC + (!z->apBC[i]) * (z->threshBC[i]);
	}
}

static void calc_sc(cbm_oracle *o)
{
	/* innet.cpp:892-911 */
	for (uint32_t i = 0; i < o->numSC; i++)
	{
		o->gPFSC[i] = o->gPFSC[i] + (o->inputSumPFSCH[i] * o->gIncGRtoSC);
		o->gPFSC[i] = o->gPFSC[i] * o->gDecGRtoSC;
		o->vSC[i] = o->vSC[i] + (o->gLeakSC * (o->eLeakSC - o->vSC[i])) - o->gPFSC[i] * o->vSC[i];
		o->apSC[i] = o->vSC[i] > o->threshSC[i];
		o->apBufSC[i] = (o->apBufSC[i] << 1) | (o->apSC[i] * 0x00000001);
		o->threshSC[i] = o->threshSC[i] + o->threshDecSC * (o->threshRestSC - o->threshSC[i]);
		o->threshSC[i] = o->apSC[i] * o->threshMaxSC + (!o->apSC[i]) * (o->threshSC[i]);
	}
}

static void calc_go(cbm_oracle *o)
{
	/* innet.cpp:816-891 (one GPU: totalGRIn is the single device's sum) */
	for (uint32_t i = 0; i < o->numGO; i++)
	{
		unsigned int totalGRIn = o->grInputGOSumH[i];
		o->sumGRInputGO[i] = totalGRIn;
		o->sumInputGOGABASynDepGO[i] = o->inputGOGABASynDepGO[i];
		o->gMFGO[i] = o->inputMFGO[i] * o->gIncMFtoGO + o->gMFGO[i] * o->gDecMFtoGO;
		o->gGRGO[i] = totalGRIn * o->tempGIncGRtoGO + o->gGRGO[i] * o->gDecGRtoGO;
		o->gGOGO[i] = o->inputGOGABASynDepGO[i] * o->gGABAIncGOtoGO + o->gGOGO[i] * o->gGABADecGOtoGO;
		o->gluGO[i] = o->gluGO[i] * o->gluDecayGO + totalGRIn * o->gluScaleGO * exp(-1.5 * o->gluGO[i]);
		o->mGluRGO[i] = o->mGluRGO[i] * o->mGluRDecayGO + o->gluGO[i] * o->mGluRScaleGO * expf(-o->mGluRGO[i]);
		o->gMGluRIncGO[i] = o->gMGluRIncGO[i] * o->gMGluRIncDecayGO + o->mGluRGO[i] * o->gMGluRIncScaleGO * expf(-o->gMGluRIncGO[i]);
		o->gMGluRGO[i] = o->gMGluRGO[i] * o->gMGluRDecGRtoGO + o->gMGluRIncGO[i] * o->gMGluRScaleGRtoGO;
		o->threshCurGO[i] = o->threshCurGO[i] + (o->threshRestGO - o->threshCurGO[i]) * o->threshDecGO;
		o->vGO[i] = o->vGO[i] + (o->gLeakGO * (o->eLeakGO - o->vGO[i]))
			+ (o->gGOGO[i] * (o->eGABAGO - o->vGO[i]))
			- (o->gMFGO[i] + o->gGRGO[i]) * o->vGO[i]
			+ o->vCoupleGO[i];
		o->apGO[i] = o->vGO[i] > o->threshCurGO[i];
		o->apGOH[i] = o->apGO[i];
		o->apBufGO[i] = (o->apBufGO[i] << 1) | (o->apGO[i] * 0x00000001);
		o->threshCurGO[i] = o->apGO[i] * o->threshMaxGO + (!o->apGO[i]) * o->threshCurGO[i];
		o->inputMFGO[i] = 0;
		o->inputGOGO[i] = 0;
		o->inputGOGABASynDepGO[i] = 0;
	}
}

static void mf_to_go_out(cbm_oracle *o)
{
	/* innet.cpp:912-931 */
	for (uint32_t i = 0; i < o->numMF; i++)
		if (o->apMFH[i])
			for (int j = 0; j < o->numpMFfromMFtoGO[i]; j++)
				o->inputMFGO[o->pMFfromMFtoGO[(size_t)i * o->maxnumpMFfromMFtoGO + j]]++;
}

static void go_to_go_out(cbm_oracle *o)
{
	/* innet.cpp:932-980, serial loop order */
	for (uint32_t i = 0; i < o->numGO; i++)
	{
		if (o->apGO[i])
			for (int j = 0; j < o->numpGOGABAOutGOGO[i]; j++)
			{
				uint32_t d = o->pGOGABAOutGOGO[(size_t)i * o->maxnumpGOGABAOutGOGO + j];
				o->inputGOGO[d]++;
				o->inputGOGABASynDepGO[d] += o->goGABAOutSynScaleGOGO[i];
			}
		o->goGABAOutSynScaleGOGO[i] = o->goGABAOutSynScaleGOGO[i] +
			(!o->apGO[i]) * (1 - o->goGABAOutSynScaleGOGO[i]) * o->goGABAGOGOSynRec -
			o->apGO[i] * (o->goGABAOutSynScaleGOGO[i] * (1 - o->goGABAGOGOSynDepF));
	}
	for (uint32_t i = 0; i < o->numGO; i++)
	{
		float threshCoupleGO;
		o->vCoupleGO[i] = 0;
		threshCoupleGO = 0;
		for (int j = 0; j < o->numpGOCoupInGOGO[i]; j++)
		{
			uint32_t n = o->pGOCoupInGOGO[(size_t)i * o->maxnumpGOCoupInGOGO + j];
			o->vCoupleGO[i] = o->vCoupleGO[i] + o->coupleRiRjRatioGO * (o->vGO[n] - o->vGO[i]);
			threshCoupleGO = threshCoupleGO + o->coupleRiRjRatioGO * (o->threshCurGO[n] - o->threshCurGO[i]);
		}
		o->threshCurGO[i] = o->threshCurGO[i] + threshCoupleGO;
	}
}

static void calc_io(cbm_oracle *o, zone_t *z)
{
	/* mzone.cpp:258-339 */
	for (uint32_t i = 0; i < o->numIO; i++)
	{
		float gNCSum = 0;
		for (uint32_t j = 0; j < o->numpIOfromNCtoIO; j++)
		{
			float *g = &z->gNCIO[(size_t)i * o->numpIOfromNCtoIO + j];
			uint8_t *in = &z->inputNCIO[(size_t)i * o->numpIOfromNCtoIO + j];
			*g = *g * expf(-o->msPerTimeStep / (-o->gDecTSofNCtoIO * expf(-*g / o->gDecTTofNCtoIO) + o->gDecT0ofNCtoIO));
			*g = *g + *in * o->gIncNCtoIO * expf(-*g / o->gIncTauNCtoIO);
			gNCSum = gNCSum + *g;
			*in = 0;
		}
		gNCSum = gNCSum / 3.1;
		z->vIO[i] = z->vIO[i] +
			o->gLeakIO * (o->eLeakIO - z->vIO[i]) +
			gNCSum * 1.5 * (o->eNCtoIO - z->vIO[i]) +
			z->vCoupleIO[i] +
			z->errDrive;
		z->apIO[i] = z->vIO[i] > z->threshIO[i];
		z->apBufIO[i] = (z->apBufIO[i] << 1) | (z->apIO[i] * 0x00000001);
		z->threshIO[i] = o->threshMaxIO * z->apIO[i] +
			(!z->apIO[i]) * (z->threshIO[i] + o->threshDecIO * (o->threshRestIO - z->threshIO[i]));
	}
	z->errDrive = 0;
}

static void calc_nc(cbm_oracle *o, zone_t *z)
{
	/* mzone.cpp:341-407 */
	for (uint32_t i = 0; i < o->numNC; i++)
	{
		float gMFNMDASum = 0, gMFAMPASum = 0, gPCNCSum = 0;
		for (uint32_t j = 0; j < o->numpNCfromMFtoNC; j++)
		{
			size_t k = (size_t)i * o->numpNCfromMFtoNC + j;
			z->gmaxNMDAofMFtoNC[k] = z->gmaxNMDAofMFtoNC[k] * o->gmaxNMDADecMFtoNC +
				z->inputMFNC[k] * z->mfSynWeightNC[k] * (1 - z->gmaxNMDAofMFtoNC[k]);
			z->gMFNMDANC[k] = z->gMFNMDANC[k] + o->gNMDAIncMFtoNC * (z->gmaxNMDAofMFtoNC[k] - z->gMFNMDANC[k]);
			gMFNMDASum = gMFNMDASum + z->gMFNMDANC[k];
			z->gmaxAMPAofMFtoNC[k] = z->gmaxAMPAofMFtoNC[k] * o->gmaxAMPADecMFtoNC +
				z->inputMFNC[k] * z->mfSynWeightNC[k] * (1 - z->gmaxAMPAofMFtoNC[k]);
			z->gMFAMPANC[k] = z->gMFAMPANC[k] + o->gAMPAIncMFtoNC * (z->gmaxAMPAofMFtoNC[k] - z->gMFAMPANC[k]);
			gMFAMPASum = gMFAMPASum + z->gMFAMPANC[k];
		}
		gMFNMDASum = gMFNMDASum * o->msPerTimeStep / ((float)o->numpNCfromMFtoNC);
		gMFAMPASum = gMFAMPASum * o->msPerTimeStep / ((float)o->numpNCfromMFtoNC);
		gMFNMDASum = gMFNMDASum * z->vNC[i] / (-80.0f);
		for (uint32_t j = 0; j < o->numpNCfromPCtoNC; j++)
		{
			size_t k = (size_t)i * o->numpNCfromPCtoNC + j;
			z->gPCNC[k] = z->gPCNC[k] * o->gDecPCtoNC + z->inputPCNC[k] * z->gPCScaleNC[k] * (1 - z->gPCNC[k]);
			gPCNCSum = gPCNCSum + z->gPCNC[k];
		}
		gPCNCSum = gPCNCSum * o->msPerTimeStep / ((float)o->numpNCfromPCtoNC);
		z->vNC[i] = z->vNC[i] + o->gLeakNC * (o->eLeakNC - z->vNC[i]) -
			(gMFNMDASum + gMFAMPASum) * z->vNC[i] + gPCNCSum * (o->ePCtoNC - z->vNC[i]);
		z->threshNC[i] = z->threshNC[i] + o->threshDecNC * (o->threshRestNC - z->threshNC[i]);
		z->apNC[i] = z->vNC[i] > z->threshNC[i];
		z->apBufNC[i] = (z->apBufNC[i] << 1) | (z->apNC[i] * 0x00000001);
		z->threshNC[i] = z->apNC[i] * o->threshMaxNC + (!z->apNC[i]) * z->threshNC[i];
	}
}

static void zone_outputs(cbm_oracle *o, zone_t *z)
{
	/* updateMFNCOut mzone.cpp:514-524 (raw input bytes) */
	for (uint32_t i = 0; i < o->numNC; i++)
		for (uint32_t j = 0; j < o->numpNCfromMFtoNC; j++)
			z->inputMFNC[(size_t)i * o->numpNCfromMFtoNC + j] = o->mfIn[z->pNCfromMFtoNC[(size_t)i * o->numpNCfromMFtoNC + j]];
	/* updateBCPCOut mzone.cpp:449-465 */
	for (uint32_t i = 0; i < o->numPC; i++) z->inputBCPC[i] = 0;
	for (uint32_t i = 0; i < o->numBC; i++)
		if (z->apBC[i])
			for (uint32_t j = 0; j < o->numpBCfromBCtoPC; j++)
				z->inputBCPC[z->pBCfromBCtoPC[(size_t)i * o->numpBCfromBCtoPC + j]]++;
	/* updateSCPCOut mzone.cpp:467-477 */
	for (uint32_t i = 0; i < o->numPC; i++)
		for (uint32_t j = 0; j < o->numpPCfromSCtoPC; j++)
			z->inputSCPC[(size_t)i * o->numpPCfromSCtoPC + j] = o->apSC[z->pPCfromSCtoPC[(size_t)i * o->numpPCfromSCtoPC + j]];
	/* updatePCOut mzone.cpp:409-447 */
	for (uint32_t i = 0; i < o->numBC; i++) z->inputPCBC[i] = 0;
	for (uint32_t i = 0; i < o->numPC; i++)
		for (uint32_t j = 0; j < o->numpPCfromPCtoBC; j++)
			z->inputPCBC[z->pPCfromPCtoBC[(size_t)i * o->numpPCfromPCtoBC + j]] += z->apPC[i];
	for (uint32_t i = 0; i < o->numNC; i++)
		for (uint32_t j = 0; j < o->numpNCfromPCtoNC; j++)
			z->inputPCNC[(size_t)i * o->numpNCfromPCtoNC + j] = z->apPC[z->pNCfromPCtoNC[(size_t)i * o->numpNCfromPCtoNC + j]];
	/* updateIOOut mzone.cpp:479-493 */
	for (uint32_t i = 0; i < o->numIO; i++)
	{
		z->pfPCPlastTimerIO[i] = (!z->apIO[i]) * (z->pfPCPlastTimerIO[i] + 1) + z->apIO[i] * o->tsLTDStartAPIO;
		z->vCoupleIO[i] = 0;
		for (uint32_t j = 0; j < o->numpIOInIOIO; j++)
			z->vCoupleIO[i] = z->vCoupleIO[i] + o->coupleRiRjRatioIO *
				(z->vIO[z->pIOInIOIO[(size_t)i * o->numpIOInIOIO + j]] - z->vIO[i]);
	}
	/* updateNCOut mzone.cpp:495-512 with the counter-based release draws */
	for (uint32_t i = 0; i < o->numNC; i++)
	{
		z->synIOPReleaseNC[i] = z->synIOPReleaseNC[i] *
			expf(-o->msPerTimeStep / (o->relPDecTSofNCtoIO * expf(-z->synIOPReleaseNC[i] / o->relPDecTTofNCtoIO) + o->relPDecT0ofNCtoIO));
		z->synIOPReleaseNC[i] = z->synIOPReleaseNC[i] + z->apNC[i] * o->relPIncNCtoIO *
			expf(-z->synIOPReleaseNC[i] / o->relPIncTauNCtoIO);
	}
	for (uint32_t i = 0; i < o->numIO; i++)
		for (uint32_t j = 0; j < o->numpIOfromNCtoIO; j++)
		{
			double u = (double)cbm_oracle_uniform24((uint32_t)z->seed, CBM_STREAM_NCIO,
					cbm_oracle_ncio_counter(o->curTime, i, j, o->numpIOfromNCtoIO));
			z->inputNCIO[(size_t)i * o->numpIOfromNCtoIO + j] =
				(u < z->synIOPReleaseNC[z->pIOfromNCtoIO[(size_t)i * o->numpIOfromNCtoIO + j]]);
		}
}

static void mfnc_syn(cbm_oracle *o, zone_t *z, uint64_t t)
{
	/* mzone.cpp:526-605 */
	if (t % o->tsPerPopHistBinPC != 0) return;
	z->histPCPopActSum = z->histPCPopActSum - z->histPCPopAct[z->histPCPopActCurBinN] + z->pcPopAct;
	z->histPCPopAct[z->histPCPopActCurBinN] = z->pcPopAct;
	z->pcPopAct = 0;
	z->histPCPopActCurBinN++;
	z->histPCPopActCurBinN = z->histPCPopActCurBinN % o->numPopHistBinsPC;
	float avgAllAPPC = ((float)z->histPCPopActSum) / o->numPopHistBinsPC;
	int doLTD = 0, doLTP = 0;
	if (avgAllAPPC >= o->synLTDPCPopActThreshMFtoNC && !z->noLTDMFNC) { doLTD = 1; z->noLTDMFNC = 1; }
	else if (avgAllAPPC < o->synLTDPCPopActThreshMFtoNC) z->noLTDMFNC = 0;
	if (avgAllAPPC <= o->synLTPPCPopActThreshMFtoNC && !z->noLTPMFNC) { doLTP = 1; z->noLTPMFNC = 1; }
	else if (avgAllAPPC > o->synLTPPCPopActThreshMFtoNC) z->noLTPMFNC = 0;
	for (uint32_t i = 0; i < o->numNC; i++)
		for (uint32_t j = 0; j < o->numpNCfromMFtoNC; j++)
		{
			size_t k = (size_t)i * o->numpNCfromMFtoNC + j;
			float synWDelta = o->histMF[z->pNCfromMFtoNC[k]] *
				(doLTD * o->synLTDStepSizeMFtoNC + doLTP * o->synLTPStepSizeMFtoNC);
			z->mfSynWeightNC[k] = z->mfSynWeightNC[k] + synWDelta;
			z->mfSynWeightNC[k] = (z->mfSynWeightNC[k] > 0) * z->mfSynWeightNC[k];
			z->mfSynWeightNC[k] = (z->mfSynWeightNC[k] <= 1) * z->mfSynWeightNC[k] + (z->mfSynWeightNC[k] > 1);
		}
}

static void pfpc_plasticity(cbm_oracle *o, zone_t *z, uint64_t t)
{
	/* mzone.cpp:643-724 with kernels.cu:282-291 */
	if (t % o->tsPerHistBinGR != 0) return;
	for (uint32_t i = 0; i < o->numIO; i++)
	{
		if (z->pfPCPlastTimerIO[i] < (o->tsLTDStartAPIO + ((int)(o->tsLTDDurationIO)))) z->pfPCPlastStepIO[i] = z->tempGRPCLTDStep;
		else if (z->pfPCPlastTimerIO[i] > o->tsLTPStartAPIO) z->pfPCPlastStepIO[i] = z->tempGRPCLTPStep;
		else z->pfPCPlastStepIO[i] = 0;
	}
	uint32_t numGRPerIO = o->numGR / o->numIO;
	uint32_t curIOInd = 0;
	for (uint32_t i = 0; i < o->numGR; i += o->numpPCfromGRtoPC)
	{
		if (i >= (curIOInd + 1) * numGRPerIO) curIOInd++;
		float step = z->pfPCPlastStepIO[curIOInd];
		#pragma omp parallel for schedule(static)
		for (uint32_t k = i; k < i + o->numpPCfromGRtoPC; k++)
		{
			float *w = &z->pfSynWeightPC[k];
			*w = *w + ((o->historyGR[k] & 0x0000008000000000ull) > 0) * step;
			*w = (*w > 0) * *w;
			*w = (*w > 1) + (*w <= 1) * *w;
		}
	}
}

void cbm_oracle_step(cbm_oracle *o, const uint8_t *mf)
{
	/* updateMFInput (cbmsimcore.cpp:312-320, innet.cpp:800-815) */
	for (uint32_t i = 0; i < o->numMF; i++)
	{
		o->histMF[i] = o->histMF[i] || (mf[i] > 0);
		o->apMFH[i] = (mf[i] > 0);
		o->apBufMF[i] = (o->apBufMF[i] << 1) | ((mf[i] > 0) * 0x00000001);
	}
	o->mfIn = mf;

	/* calcActivity, phase 1 (cbmsimcore.cpp:142-201) */
	o->curTime++;
	uint64_t t = o->curTime;
	gr_activity(o);
	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		zone_t *z = &o->zones[zi];
		#pragma omp parallel for schedule(static)
		for (uint32_t pc = 0; pc < o->numPC; pc++)
			z->sumPFPCdev[pc] = sum_row_ordered(&z->rowsPFPC[(size_t)pc * o->numpPCfromGRtoPC], o->numpPCfromGRtoPC);
	}
	memcpy(o->sumBCdev, o->pendBC, o->numBC * 4);
	memcpy(o->sumSCdev, o->pendSC, o->numSC * 4);
	memcpy(o->sumGOdev, o->pendGO, o->numGO * 4);
	for (uint32_t zi = 0; zi < o->numZones; zi++) pfpc_plasticity(o, &o->zones[zi], t);
	memcpy(o->apMFdev, o->apMFH, o->numMF * 4);
	memcpy(o->apGOdev, o->apGOH, o->numGO * 4);
	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		calc_pc(o, &o->zones[zi]);
		calc_bc(o, &o->zones[zi]);
	}
	calc_sc(o);

	/* phase 2 (cbmsimcore.cpp:203-309) */
	gr_inputs(o, o->gMFSumGR, o->apMFdev, o->numpGRfromMFtoGR, o->pGRfromMFtoGR, o->maxnumpGRfromGOtoGR,
			o->gDecMFtoGR, o->gIncMFtoGR);
	gr_inputs(o, o->gGOSumGR, o->apGOdev, o->numpGRfromGOtoGR, o->pGRfromGOtoGR, o->maxnumpGRfromGOtoGR,
			o->gDecGOtoGR, o->gIncGOtoGR);
	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		zone_t *z = &o->zones[zi];
		#pragma omp parallel for schedule(static)
		for (uint32_t i = 0; i < o->numGR; i++)
		{
			unsigned int pf = (o->apBufGR[i] & o->pGRDelayMaskfromGRtoBSP[i]) > 0;
			z->rowsPFPC[i] = z->pfSynWeightPC[i] * pf;
		}
		memcpy(z->inputSumPFPCMZH, z->sumPFPCdev, o->numPC * 4);
	}
	memset(o->pendBC, 0, o->numBC * 4);
	memset(o->pendSC, 0, o->numSC * 4);
	memset(o->pendGO, 0, o->numGO * 4);
	{
		/* integer counts: any summation order gives the same values */
		uint32_t *pendBC = o->pendBC, *pendSC = o->pendSC, *pendGO = o->pendGO;
		const uint32_t nBC = o->numBC, nSC = o->numSC, nGO = o->numGO;
		#pragma omp parallel for schedule(static) reduction(+: pendBC[:nBC], pendSC[:nSC], pendGO[:nGO])
		for (uint32_t i = 0; i < o->numGR; i++)
		{
			unsigned int pf = (o->apBufGR[i] & o->pGRDelayMaskfromGRtoBSP[i]) > 0;
			pendBC[i >> o->numpBCfromGRtoBCP2] += pf;
			pendSC[i >> o->numpSCfromGRtoSCP2] += pf;
			for (int k = 0; k < o->numpGRfromGRtoGO[i]; k++)
			{
				size_t s = (size_t)i * o->maxnumpGRfromGRtoGO + k;
				if ((o->apBufGR[i] & o->pGRDelayMaskfromGRtoGO[s]) > 0) pendGO[o->pGRfromGRtoGO[s]] += 1;
			}
		}
	}
	memcpy(o->inputSumPFBCH, o->sumBCdev, o->numBC * 4);
	memcpy(o->inputSumPFSCH, o->sumSCdev, o->numSC * 4);
	memcpy(o->grInputGOSumH, o->sumGOdev, o->numGO * 4);
	if (t % o->tsPerHistBinGR == 0)
		#pragma omp parallel for schedule(static)
		for (uint32_t i = 0; i < o->numGR; i++)
			o->historyGR[i] = (o->historyGR[i] << 1) | ((o->apBufGR[i] & 0x0000001F) > 0);

	calc_go(o);
	mf_to_go_out(o);
	go_to_go_out(o);
	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		zone_t *z = &o->zones[zi];
		calc_io(o, z);
		calc_nc(o, z);
		zone_outputs(o, z);
		mfnc_syn(o, z, t);
	}
	/* resetMFHist innet.cpp:982-995 */
	if (t % o->numTSinMFHist == 0)
		for (uint32_t i = 0; i < o->numMF; i++) o->histMF[i] = 0;
}

size_t cbm_oracle_trace_record_bytes(const cbm_oracle *o)
{
	return (o->numGR + 7) / 8 + (size_t)o->numGO * 9 + (size_t)o->numSC * 5 +
		(size_t)o->numZones * ((size_t)o->numBC * 5 + (size_t)o->numPC * 5 + (size_t)o->numIO * 5 + (size_t)o->numNC * 5);
}

static uint8_t *put(uint8_t *p, const void *src, size_t n) { memcpy(p, src, n); return p + n; }

static void trace_record(cbm_oracle *o, uint8_t *p)
{
	size_t nb = (o->numGR + 7) / 8;
	memset(p, 0, nb);
	for (uint32_t i = 0; i < o->numGR; i++) if (o->outputGR[i]) p[i >> 3] |= (uint8_t)(1u << (i & 7));
	p += nb;
	p = put(p, o->apGO, o->numGO);
	p = put(p, o->vGO, (size_t)o->numGO * 4);
	p = put(p, o->sumGRInputGO, (size_t)o->numGO * 4);
	p = put(p, o->apSC, o->numSC);
	p = put(p, o->vSC, (size_t)o->numSC * 4);
	for (uint32_t zi = 0; zi < o->numZones; zi++)
	{
		zone_t *z = &o->zones[zi];
		p = put(p, z->apBC, o->numBC); p = put(p, z->vBC, (size_t)o->numBC * 4);
		p = put(p, z->apPC, o->numPC); p = put(p, z->vPC, (size_t)o->numPC * 4);
		p = put(p, z->apIO, o->numIO); p = put(p, z->vIO, (size_t)o->numIO * 4);
		p = put(p, z->apNC, o->numNC); p = put(p, z->vNC, (size_t)o->numNC * 4);
	}
}

void cbm_oracle_run(cbm_oracle *o, const uint8_t *mf, uint64_t nsteps, uint8_t *trace)
{
	size_t rb = cbm_oracle_trace_record_bytes(o);
	for (uint64_t s = 0; s < nsteps; s++)
	{
		cbm_oracle_step(o, mf + s * o->numMF);
		if (trace) trace_record(o, trace + s * rb);
	}
}

static void protocol_window(const cbm_oracle_protocol *p, int32_t *from, int32_t *len, uint32_t *bins)
{
	*from = p->csOn - p->preCS;
	*len = p->csOff + p->postCS - *from;
	*bins = ((uint32_t)*len + p->binSteps - 1) / p->binSteps;
}

void cbm_oracle_protocol_sizes(const cbm_oracle *o, const cbm_oracle_protocol *p, uint64_t *ncPSH,
		uint64_t *pcPSH, uint64_t *eyelid)
{
	int32_t from, len; uint32_t bins;
	protocol_window(p, &from, &len, &bins);
	uint64_t nd = p->numDataTrials ? p->numDataTrials : 1;
	*ncPSH = nd * bins * o->numNC;
	*pcPSH = nd * bins * o->numPC;
	*eyelid = nd * (uint64_t)len;
}

/* cells of each trial-data record, in record order */
static void trial_data_cells(const cbm_oracle *o, uint32_t psh[9], uint32_t raster[6])
{
	const uint32_t p9[9] = {o->numGO, o->numGO, o->numGO, o->numGO, o->numMF, o->numSC, o->numBC, o->numPC, o->numIO};
	const uint32_t r6[6] = {o->numGO, o->numSC, o->numBC, o->numPC, o->numNC, o->numIO};
	memcpy(psh, p9, sizeof(p9));
	memcpy(raster, r6, sizeof(r6));
}

void cbm_oracle_trial_data_sizes(const cbm_oracle *o, const cbm_oracle_protocol *p, uint64_t *psh,
		uint64_t *raster)
{
	int32_t from, len; uint32_t bins, pc[9], rc[6];
	protocol_window(p, &from, &len, &bins);
	trial_data_cells(o, pc, rc);
	*psh = 0; *raster = 0;
	for (int k = 0; k < 9; k++) *psh += (uint64_t)bins * pc[k];
	for (int k = 0; k < 6; k++) *raster += (uint64_t)p->numDataTrials * (uint32_t)(len / 32) * rc[k];
}

/* One step of ECTrialsData recording at window step ct of kept trial dt
 * (ecmanagementdelay.cpp:240-265): every histogram adds the step's value to
 * its bin (PeriStimHistFloat::update, peristimhistfloat.cpp: u8 spikes as
 * (ap > 0), u32 counts and floats as they are, in float); every 32nd window
 * step after the first, each raster takes the cells' apBuf words into its
 * next row (SpikeRasterBitArray::updateRaster, spikerasterbitarray.cpp:62-80),
 * rows counted over all updates, recLen / 32 rows to a raster trial. */
static void trial_data_step(const cbm_oracle *o, const cbm_oracle_protocol *p, const uint8_t *apMF, uint32_t dt,
		int32_t ct, float *psh, uint32_t *raster)
{
	int32_t from, len; uint32_t bins, pc[9], rc[6];
	protocol_window(p, &from, &len, &bins);
	trial_data_cells(o, pc, rc);
	const zone_t *z = &o->zones[0];
	const uint32_t bin = (uint32_t)ct / p->binSteps;
	if (psh)
	{
		float *h[9];
		h[0] = psh;
		for (int k = 1; k < 9; k++) h[k] = h[k - 1] + (size_t)bins * pc[k - 1];
		for (int k = 0; k < 9; k++) h[k] += (size_t)bin * pc[k];
		for (uint32_t i = 0; i < o->numGO; i++)
		{
			h[0][i] += (float)(o->apGO[i] > 0);
			h[1][i] += o->sumGRInputGO[i];
			h[2][i] += o->sumInputGOGABASynDepGO[i];
			h[3][i] += o->goGABAOutSynScaleGOGO[i];
		}
		for (uint32_t i = 0; i < o->numMF; i++) h[4][i] += (float)(apMF[i] > 0);
		for (uint32_t i = 0; i < o->numSC; i++) h[5][i] += (float)(o->apSC[i] > 0);
		for (uint32_t i = 0; i < o->numBC; i++) h[6][i] += (float)(z->apBC[i] > 0);
		for (uint32_t i = 0; i < o->numPC; i++) h[7][i] += (float)(z->apPC[i] > 0);
		for (uint32_t i = 0; i < o->numIO; i++) h[8][i] += (float)(z->apIO[i] > 0);
	}
	const uint32_t rows = (uint32_t)len / 32;
	if (!raster || !rows || ct % 32 != 0 || ct == 0) return;
	const uint64_t u = (uint64_t)dt * (uint32_t)((len - 1) / 32) + (uint32_t)ct / 32 - 1;
	const uint64_t rt = u / rows, row = u % rows;
	if (rt >= p->numDataTrials) return;
	const uint32_t *src[6] = {o->apBufGO, o->apBufSC, z->apBufBC, z->apBufPC, z->apBufNC, z->apBufIO};
	uint32_t *r = raster;
	for (int k = 0; k < 6; k++)
	{
		memcpy(r + ((size_t)rt * rows + row) * rc[k], src[k], rc[k] * sizeof(uint32_t));
		r += (size_t)p->numDataTrials * rows * rc[k];
	}
}

static void run_protocol(cbm_oracle *o, const cbm_oracle_protocol *p, const float *rates, const float *stepRates,
		uint64_t rateRows, uint64_t nsteps, uint8_t *trace, uint32_t *ncPSH, uint32_t *pcPSH, float *eyelid,
		float *psh, uint32_t *raster);

void cbm_oracle_run_protocol(cbm_oracle *o, const cbm_oracle_protocol *p, const float *rates, uint64_t nsteps,
		uint8_t *trace, uint32_t *ncPSH, uint32_t *pcPSH, float *eyelid, float *psh, uint32_t *raster)
{
	run_protocol(o, p, rates, NULL, 0, nsteps, trace, ncPSH, pcPSH, eyelid, psh, raster);
}

void cbm_oracle_run_protocol_step_rates(cbm_oracle *o, const cbm_oracle_protocol *p, const float *stepRates,
		uint64_t rateRows, uint64_t nsteps, uint8_t *trace, uint32_t *ncPSH, uint32_t *pcPSH, float *eyelid)
{
	run_protocol(o, p, stepRates, stepRates, rateRows, nsteps, trace, ncPSH, pcPSH, eyelid, NULL, NULL);
}

static void run_protocol(cbm_oracle *o, const cbm_oracle_protocol *p, const float *rates, const float *stepRates,
		uint64_t rateRows, uint64_t nsteps, uint8_t *trace, uint32_t *ncPSH, uint32_t *pcPSH, float *eyelid,
		float *psh, uint32_t *raster)
{
	const uint32_t numMF = o->numMF, numNC = o->numNC, numPC = o->numPC;
	const float *freqBG = rates, *freqCST = rates + numMF, *freqCSP = rates + 2 * (size_t)numMF;
	int32_t recFrom, recLen; uint32_t nBins;
	protocol_window(p, &recFrom, &recLen, &nBins);
	uint64_t nNC, nPC, nEye;
	cbm_oracle_protocol_sizes(o, p, &nNC, &nPC, &nEye);
	memset(ncPSH, 0, nNC * 4); memset(pcPSH, 0, nPC * 4); memset(eyelid, 0, nEye * 4);
	uint64_t nPSH, nRaster;
	cbm_oracle_trial_data_sizes(o, p, &nPSH, &nRaster);
	if (psh) memset(psh, 0, nPSH * 4);
	if (raster) memset(raster, 0, nRaster * 4);
	/* PoissonRegenCells(numMF, mfSeed, tau, 1) (ecmanagementdelay.cpp:96,
	 * poissonregencells.cpp:10-35): its generator's seed is the first draw of
	 * a generator seeded with mfSeed, scaled to [0, 2^31) */
	const float msPerTS = 1.0f, sPerTS = msPerTS / 1000;
	/* 1 - exp(...) as poissonregencells.cpp:20 computes it: exp of a float
	 * argument is the float overload in C++ (expf), the subtraction float */
	const float threshDecay = 1.0f - expf(-msPerTS / p->mfThreshDecayTau);
	const double u0 = (double)cbm_oracle_uniform24((uint32_t)p->mfSeed, CBM_STREAM_NCIO, 0);
	const uint32_t mfGenSeed = (uint32_t)(int)(u0 * 2147483648.0);
	float *thresh = malloc(numMF * sizeof(float));
	uint8_t *apMF = malloc(numMF);
	for (uint32_t i = 0; i < numMF; i++) thresh[i] = 1;
	/* EyelidIntegrator(numNC, msPerTimeStep, ...) (eyelidintegrator.cpp:13-28) */
	const int eyeMS = (int)(unsigned)o->msPerTimeStep;
	const float eyeGDecay = expf(-eyeMS / p->eyeGDecayTau), eyeGLeak = p->eyeGLeakRaw / (6 - eyeMS);
	float *gIn = calloc(numNC, sizeof(float));
	float vm = 0;
	int plastSet = 0, plastReset = 1;
	size_t rb = cbm_oracle_trace_record_bytes(o);
	zone_t *z0 = &o->zones[0];
	for (uint64_t s = 0; s < nsteps; s++)
	{
		const uint64_t t = o->curTime + 1;
		const int32_t time = (int32_t)(s % p->trialSteps);
		const uint32_t trial = (uint32_t)(s / p->trialSteps);
		const int csTrial = trial >= p->csStartTrial;
		/* calcMFActivity (ecmanagementdelay.cpp:175-194) */
		const float *freq = freqBG;
		if (csTrial && time >= p->csOn && time < p->csOff) freq = time < p->csPhasicOff ? freqCSP : freqCST;
		if (stepRates) freq = stepRates + (s % rateRows) * numMF;
		for (uint32_t i = 0; i < numMF; i++)
		{
			thresh[i] = thresh[i] + (1 - thresh[i]) * threshDecay;
			apMF[i] = (double)cbm_oracle_uniform24(mfGenSeed, CBM_STREAM_NCIO, (t << 20) | i) <
				((freq[i] * sPerTS) * thresh[i]);
			thresh[i] = (!apMF[i]) * thresh[i];
		}
		/* calcSimActivity (ecmanagementdelay.cpp:196-235) */
		if (time == p->csOff - 1 && csTrial) cbm_oracle_update_err_drive(o, 0, p->usErrDrive);
		if (time >= p->csOn + p->plastOnDelay && !plastSet && csTrial && time < p->csOff + p->plastOffDelay)
		{
			plastSet = 1; plastReset = 0;
			cbm_oracle_set_plast_steps(o, 0, p->plastLTD, p->plastLTP);
		}
		if (!plastReset && time >= p->csOff + p->plastOffDelay && csTrial)
		{
			plastSet = 0; plastReset = 1;
			cbm_oracle_reset_plast_steps(o, 0);
		}
		cbm_oracle_step(o, apMF);
		if (trace) trace_record(o, trace + s * rb);
		/* EyelidIntegrator::calcStep (eyelidintegrator.cpp:50-68) */
		float gSum = 0;
		for (uint32_t i = 0; i < numNC; i++)
		{
			gIn[i] = gIn[i] * eyeGDecay;
			gIn[i] = gIn[i] + z0->apNC[i] * p->eyeGInc;
			gSum += gIn[i];
		}
		gSum = gSum + p->eyeGShift;
		gSum = (gSum > 0) * gSum;
		vm = vm + (eyeGLeak * (0 - vm)) + (gSum * (p->eyeMaxAmp - vm));
		const int32_t ct = time - recFrom;
		if (trial >= p->dataStartTrial && trial < p->dataStartTrial + p->numDataTrials && ct >= 0 && ct < recLen)
		{
			const size_t dt = trial - p->dataStartTrial, bin = (size_t)ct / p->binSteps;
			for (uint32_t i = 0; i < numNC; i++) ncPSH[(dt * nBins + bin) * numNC + i] += z0->apNC[i];
			for (uint32_t i = 0; i < numPC; i++) pcPSH[(dt * nBins + bin) * numPC + i] += z0->apPC[i];
			eyelid[dt * recLen + ct] = vm;
			trial_data_step(o, p, apMF, (uint32_t)dt, ct, psh, raster);
		}
	}
	free(thresh); free(apMF); free(gIn);
}

void cbm_oracle_expf_array(const float *in, float *out, uint64_t n)
{
	/* the host C library's expf, which the reference's exp(float) calls use */
	for (uint64_t i = 0; i < n; i++) out[i] = expf(in[i]);
}

void cbm_oracle_exp_array(const double *in, double *out, uint64_t n)
{
	/* the host C library's exp, which the reference's exp(double) calls use */
	for (uint64_t i = 0; i < n; i++) out[i] = exp(in[i]);
}

uint32_t cbm_oracle_num(const cbm_oracle *o, const char *w)
{
	if (!strcmp(w, "GR")) return o->numGR;
	if (!strcmp(w, "GO")) return o->numGO;
	if (!strcmp(w, "MF")) return o->numMF;
	if (!strcmp(w, "SC")) return o->numSC;
	if (!strcmp(w, "BC")) return o->numBC;
	if (!strcmp(w, "PC")) return o->numPC;
	if (!strcmp(w, "NC")) return o->numNC;
	if (!strcmp(w, "IO")) return o->numIO;
	if (!strcmp(w, "zones")) return o->numZones;
	if (!strcmp(w, "step")) return (uint32_t)o->curTime;
	return 0;
}
