/* Test infrastructure (oracle build only).
 *
 * Harness around the reference's own, unmodified host code (compiled from the
 * reference tree by oracle/Makefile against the shims in oracle/refshim).
 *
 *   ref_gen  ACT CON NZONES INNETSEED MZCSEED MZASEED OUT
 *       builds a new network with the reference's generator
 *       (CBMState(fstream&, fstream&, nZones, seeds), CBM_STATE_LIB_DEV/src/
 *       interfaces/cbmstate.cpp:60-64) and writes it with CBMState::writeState
 *       (cbmstate.cpp:86-103).  Linked against the reference's vendored SFMT.
 *
 *   ref_run STATE MFBYTES STEPS TRACE FINALSTATE [SEED...] [-e EVENTS] [-g NGPUP2] [-t]
 *       loads STATE with CBMState(fstream&) (cbmstate.cpp:12-33), runs STEPS
 *       calls of updateMFInput + calcActivity (CBM_CORE_LIB_MGPU_DEV/src/
 *       interface/cbmsimcore.cpp:139-320) and writes one trace record per step
 *       plus the final state (CBMSimCore::writeToState, cbmsimcore.cpp:75-80).
 *       -t times the steps and writes no trace.
 *       -p PROTOCOL -r RECORDS: the MF input comes from the reference's
 *       PoissonRegenCells (CBM_TOOLS_LIB_DEV/src/poissonregencells.cpp) and the
 *       eyelid-conditioning driver's per-step calls are made in the order of
 *       ECManagementDelay::calcMFActivity / calcSimActivity
 *       (Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp:175-273,
 *       restated below); the reference's EyelidIntegrator
 *       (CBM_TOOLS_LIB_DEV/src/eyelidintegrator.cpp) runs on zone 0's NC
 *       spikes; RECORDS receives NC and PC spike counts per bin and the
 *       integrator's output over the recording window of the kept trials,
 *       then the reference's GR peri-stimulus histogram (PeriStimHistFloat,
 *       CBM_DATA_LIB_DEV/src/peristimhist/peristimhistfloat.cpp, updated with
 *       exportAPGR as the eyelid driver does,
 *       Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp:262) as
 *       f32 [bins][numGR], then the reference's ECTrialsData
 *       (CBM_DATA_LIB_DEV/src/interfaces/ectrialsdata.cpp) built and filled
 *       as the eyelid driver does (ecmanagementdelay.cpp:107-156, 240-265):
 *       its histograms go, grInputGO, goInputGO, goOutSynScale, mf, sc, bc,
 *       pc, io, gr (numGR / 10 cells) as f32 [bins][cells], and its rasters
 *       go, sc, bc, pc, nc, io as u32 [numDataTrials][window / 32][cells],
 *       and its smoothed eyelid trace (EyelidOut) as f32
 *       [numDataTrials][window] (MFBYTES is then ignored).  -m MFPOP then writes the
 *       reference's ECMFPopulation estimated from that ECTrialsData
 *       (CBM_TOOLS_LIB_DEV/src/ecmfpopulation.cpp:11-65) with writeToFile, and
 *       -d DATA the ECTrialsData itself with its writeData, and -s SESSION
 *       the state followed by the ECTrialsData, as the driver's
 *       writeDataToFile writes them.  PROTOCOL is "key value" text: trialSteps,
 *       csOn, csOff, csPhasicOff, csStartTrial, plastOnDelay, plastOffDelay,
 *       plastLTD, plastLTP, usErrDrive, mfSeed, mfThreshDecayTau, rates (a file
 *       of 3 x numMF f32: background, CS tonic, CS phasic), dataStartTrial,
 *       numDataTrials, preCS, postCS, binSteps, eyeGDecayTau, eyeGInc,
 *       eyeGShift, eyeGLeakRaw, eyeMaxAmp.
 *
 * After loading, two fields the reference's loader leaves undefined are set
 * the way the B200 loader sets them:
 *   - pPCfromPCtoBC: MZoneConnectivityState::stateRW reads pBCfromPCtoBC a
 *     second time in its place (mzoneconnectivitystate.cpp:150); it is
 *     rebuilt from connectPCtoBC's formula (mzoneconnectivitystate.cpp:242-257).
 *   - histPCPopActSum / histPCPopActCurBinN / pcPopAct / errDrive /
 *     noLTPMFNC / noLTDMFNC: not in the file (mzoneactivitystate.cpp:299-355);
 *     set to the histogram's sum and zeros.
 *
 * Trace record per step (all little-endian, no padding):
 *   apGR bits  ceil(numGR/8) bytes, GR i at byte i/8 bit i%8
 *   apGO u8[numGO], vGO f32[numGO], sumGRInputGO u32[numGO]
 *   apSC u8[numSC], vSC f32[numSC]
 *   per zone: apBC u8[numBC] vBC f32[numBC] apPC u8[numPC] vPC f32[numPC]
 *             apIO u8[numIO] vIO f32[numIO] apNC u8[numNC] vNC f32[numNC]
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <fstream>
#include <iostream>
#include <chrono>

#include <CBMStateInclude/interfaces/cbmstate.h>

#ifndef CBM_REF_GEN_ONLY
#include <map>
#include <CBMCoreInclude/interface/cbmsimcore.h>
#include <CBMToolsInclude/poissonregencells.h>
#include <CBMToolsInclude/eyelidintegrator.h>
#include <CBMDataInclude/peristimhist/peristimhistfloat.h>
#include <CBMDataInclude/interfaces/ectrialsdata.h>
#include <CBMToolsInclude/ecmfpopulation.h>
uint64_t cbm_refshim_step = 0;
void cbm_refshim_set_step(uint64_t t) { cbm_refshim_step = t; }
#endif

static void fixLoadedState(CBMState *st)
{
	ConnectivityParams *cp = st->getConParamsInternal();
	ActivityParams *ap = st->getActParamsInternal();
	for (unsigned int z = 0; z < st->getNumZones(); z++)
	{
		MZoneConnectivityState *cs = st->getMZoneConStateInternal(z);
		int bcToPCRatio = cp->numBC / cp->numPC;
		for (int i = 0; i < (int)cp->numPC; i++)
			for (int j = 0; j < (int)cp->numpPCfromPCtoBC; j++)
			{
				int bcInd = i * bcToPCRatio - 6 + j;
				cs->pPCfromPCtoBC[i][j] = (bcInd % (int)cp->numBC + (int)cp->numBC) % (int)cp->numBC;
			}
		MZoneActivityState *as = st->getMZoneActStateInternal(z);
		ct_uint32_t sum = 0;
		for (unsigned int k = 0; k < ap->numPopHistBinsPC; k++) sum += as->histPCPopAct[k];
		as->histPCPopActSum = sum;
		as->histPCPopActCurBinN = 0;
		as->pcPopAct = 0;
		as->errDrive = 0;
		as->noLTPMFNC = 0;
		as->noLTDMFNC = 0;
	}
}

#ifdef CBM_REF_GEN_ONLY
int main(int argc, char **argv)
{
	if (argc != 8)
	{
		fprintf(stderr, "usage: ref_gen ACT CON NZONES INNETSEED MZCSEED MZASEED OUT\n");
		return 2;
	}
	std::fstream act(argv[1], std::ios::in), con(argv[2], std::ios::in);
	if (!act.good() || !con.good()) { fprintf(stderr, "cannot open params\n"); return 1; }
	unsigned int nZones = (unsigned int)atoi(argv[3]);
	int innetSeed = atoi(argv[4]);
	std::vector<int> cseeds(nZones), aseeds(nZones);
	for (unsigned int z = 0; z < nZones; z++) { cseeds[z] = atoi(argv[5]) + (int)z; aseeds[z] = atoi(argv[6]) + (int)z; }
	CBMState st(act, con, nZones, innetSeed, cseeds.data(), aseeds.data());
	std::fstream out(argv[7], std::ios::out | std::ios::binary | std::ios::trunc);
	st.writeState(out);
	out.close();
	return 0;
}
#else

struct Event { unsigned long t; std::string kind; int zone; float a, b; };

static std::vector<Event> readEvents(const char *path)
{
	std::vector<Event> ev;
	std::ifstream f(path);
	std::string kind;
	unsigned long t;
	while (f >> t >> kind)
	{
		Event e; e.t = t; e.kind = kind; e.zone = 0; e.a = 0; e.b = 0;
		if (kind == "errdrive") f >> e.zone >> e.a;
		else if (kind == "plast") f >> e.zone >> e.a >> e.b;
		else if (kind == "plastreset") f >> e.zone;
		else if (kind == "grgoinc") f >> e.a;
		else if (kind == "grgoincreset") {}
		else { fprintf(stderr, "bad event %s\n", kind.c_str()); exit(2); }
		ev.push_back(e);
	}
	return ev;
}

template<typename T> static void put(FILE *f, const T *p, size_t n) { if (n) fwrite(p, sizeof(T), n, f); }

// Trial protocol of the eyelid driver (see the file comment).
struct Protocol
{
	std::map<std::string, std::string> kv;
	bool load(const char *path)
	{
		std::ifstream f(path);
		if (!f.good()) return false;
		std::string k, v;
		while (f >> k >> v) kv[k] = v;
		return true;
	}
	double num(const char *k) const { auto it = kv.find(k); return it == kv.end() ? 0.0 : atof(it->second.c_str()); }
	std::string str(const char *k) const { auto it = kv.find(k); return it == kv.end() ? "" : it->second; }
};

int main(int argc, char **argv)
{
	if (argc < 6)
	{
		fprintf(stderr, "usage: ref_run STATE MFBYTES STEPS TRACE FINALSTATE [SEED...] [-e EVENTS] [-g NGPUP2] [-t] [-w WARMUP]\n");
		return 2;
	}
	const char *statePath = argv[1], *mfPath = argv[2], *tracePath = argv[4], *finalPath = argv[5];
	unsigned long steps = strtoul(argv[3], NULL, 10);
	std::vector<int> seeds;
	const char *eventsPath = NULL, *protocolPath = NULL, *recordsPath = NULL, *mfPopPath = NULL, *dataPath = NULL, *sessionPath = NULL;
	int numGPUP2 = 0;
	bool timeOnly = false;
	unsigned long warm = 0;  // leading steps run before the clock starts
	for (int i = 6; i < argc; i++)
	{
		if (!strcmp(argv[i], "-e") && i + 1 < argc) eventsPath = argv[++i];
		else if (!strcmp(argv[i], "-p") && i + 1 < argc) protocolPath = argv[++i];
		else if (!strcmp(argv[i], "-r") && i + 1 < argc) recordsPath = argv[++i];
		else if (!strcmp(argv[i], "-m") && i + 1 < argc) mfPopPath = argv[++i];
		else if (!strcmp(argv[i], "-d") && i + 1 < argc) dataPath = argv[++i];
		else if (!strcmp(argv[i], "-s") && i + 1 < argc) sessionPath = argv[++i];
		else if (!strcmp(argv[i], "-g") && i + 1 < argc) numGPUP2 = atoi(argv[++i]);
		else if (!strcmp(argv[i], "-t")) timeOnly = true;
		else if (!strcmp(argv[i], "-w") && i + 1 < argc) warm = strtoul(argv[++i], NULL, 10);
		else seeds.push_back(atoi(argv[i]));
	}

	std::fstream in(statePath, std::ios::in | std::ios::binary);
	if (!in.good()) { fprintf(stderr, "cannot open state\n"); return 1; }
	CBMState *st = new CBMState(in);
	in.close();
	fixLoadedState(st);
	ConnectivityParams *cp = st->getConParamsInternal();
	unsigned int nZones = st->getNumZones();
	while (seeds.size() < nZones) seeds.push_back(1000 + (int)seeds.size());

	std::vector<ct_uint8_t> mf;
	Protocol proto;
	const bool useProtocol = protocolPath != NULL;
	if (useProtocol && (!proto.load(protocolPath) || !recordsPath)) { fprintf(stderr, "bad protocol\n"); return 1; }
	if (!useProtocol)
	{
		FILE *f = fopen(mfPath, "rb");
		if (!f) { fprintf(stderr, "cannot open mf\n"); return 1; }
		mf.resize((size_t)steps * cp->numMF);
		size_t got = fread(mf.data(), 1, mf.size(), f);
		fclose(f);
		if (got != mf.size()) { fprintf(stderr, "mf file too short (%zu of %zu)\n", got, mf.size()); return 1; }
	}
	std::vector<Event> events;
	if (eventsPath) events = readEvents(eventsPath);

	cbm_refshim_set_step(0);
	CBMSimCore *sim = new CBMSimCore(st, seeds.data(), 0, numGPUP2);
	InNetInterface *inet = sim->getInputNet();
	MZoneInterface **zones = sim->getMZoneList();

	FILE *tr = NULL;
	if (!timeOnly)
	{
		tr = fopen(tracePath, "wb");
		if (!tr) { fprintf(stderr, "cannot open trace\n"); return 1; }
	}
	std::vector<ct_uint8_t> bits((cp->numGR + 7) / 8);
	size_t evi = 0;

	// eyelid driver state (ecmanagementdelay.cpp:90-170)
	const unsigned int trialSteps = (unsigned int)proto.num("trialSteps");
	const int csOn = (int)proto.num("csOn"), csOff = (int)proto.num("csOff"), csPOff = (int)proto.num("csPhasicOff");
	const unsigned int csStartTN = (unsigned int)proto.num("csStartTrial");
	const int plastOn = (int)proto.num("plastOnDelay"), plastOff = (int)proto.num("plastOffDelay");
	const float plastLTD = (float)proto.num("plastLTD"), plastLTP = (float)proto.num("plastLTP");
	const float usErr = (float)proto.num("usErrDrive");
	const unsigned int dataStartTN = (unsigned int)proto.num("dataStartTrial"), numDataT = (unsigned int)proto.num("numDataTrials");
	const int recFrom = csOn - (int)proto.num("preCS"), recLen = csOff + (int)proto.num("postCS") - recFrom;
	const unsigned int binSteps = useProtocol ? (unsigned int)proto.num("binSteps") : 1;
	const unsigned int nBins = useProtocol ? ((unsigned int)recLen + binSteps - 1) / binSteps : 0;
	std::vector<float> freqBG, freqCST, freqCSP;
	PoissonRegenCells *mfs = NULL;
	EyelidIntegrator *eyelid = NULL;
	std::vector<ct_uint32_t> ncPSH, pcPSH;
	PeriStimHistFloat *grPSH = NULL;
	ECTrialsData *data = NULL;
	// the driver's histograms and rasters, in the order RECORDS holds them
	const char *pshNames[] = {"go", "grInputGO", "goInputGO", "goOutSynScale", "mf", "sc", "bc", "pc", "io", "gr"};
	const char *rasterNames[] = {"go", "sc", "bc", "pc", "nc", "io"};
	std::vector<float> eyeTrace;
	bool grPCPlastSet = false, grPCPlastReset = true;
	if (useProtocol)
	{
		freqBG.resize(cp->numMF); freqCST.resize(cp->numMF); freqCSP.resize(cp->numMF);
		FILE *f = fopen(proto.str("rates").c_str(), "rb");
		if (!f) { fprintf(stderr, "cannot open rates\n"); return 1; }
		size_t got = fread(freqBG.data(), 4, cp->numMF, f) + fread(freqCST.data(), 4, cp->numMF, f) +
			fread(freqCSP.data(), 4, cp->numMF, f);
		fclose(f);
		if (got != 3 * (size_t)cp->numMF) { fprintf(stderr, "rates file too short\n"); return 1; }
		cbm_refshim_set_step(0);
		mfs = new PoissonRegenCells(cp->numMF, (int)proto.num("mfSeed"), (float)proto.num("mfThreshDecayTau"), 1);
		eyelid = new EyelidIntegrator(cp->numNC, (unsigned int)st->getActParamsInternal()->msPerTimeStep,
				(float)proto.num("eyeGDecayTau"), (float)proto.num("eyeGInc"), (float)proto.num("eyeGShift"),
				(float)proto.num("eyeGLeakRaw"), (float)proto.num("eyeMaxAmp"));
		const size_t nd = numDataT ? numDataT : 1;
		ncPSH.assign(nd * nBins * cp->numNC, 0);
		pcPSH.assign(nd * nBins * cp->numPC, 0);
		eyeTrace.assign(nd * (size_t)recLen, 0.0f);
		grPSH = new PeriStimHistFloat(recLen, (int)binSteps, (int)cp->numGR);
		// ECTrialsData as the eyelid driver builds it (ecmanagementdelay.cpp:107-156),
		// with this protocol's window and bin width
		std::map<std::string, PSHParams> pshParams;
		std::map<std::string, RasterParams> rasterParams;
		std::map<std::string, RawUIntParams> uintParams;
		const unsigned int pshCells[] = {cp->numGO, cp->numGO, cp->numGO, cp->numGO, cp->numMF, cp->numSC,
			cp->numBC, cp->numPC, cp->numIO, cp->numGR / 10};
		const unsigned int rasterCells[] = {cp->numGO, cp->numSC, cp->numBC, cp->numPC, cp->numNC, cp->numIO};
		for (int k = 0; k < 10; k++) { PSHParams pp; pp.numTimeStepsPerBin = binSteps; pp.numCells = pshCells[k]; pshParams[pshNames[k]] = pp; }
		for (int k = 0; k < 6; k++) { RasterParams rp; rp.numCells = rasterCells[k]; rasterParams[rasterNames[k]] = rp; }
		EyelidOutParams eyelidParams;
		eyelidParams.numTimeStepSmooth = 4;
		data = new ECTrialsData((unsigned int)proto.num("preCS"), (unsigned int)(csOff - csOn),
				(unsigned int)proto.num("postCS"), (unsigned int)st->getActParamsInternal()->msPerTimeStep,
				numDataT, pshParams, rasterParams, uintParams, eyelidParams);
	}

	auto t0 = std::chrono::steady_clock::now();
	for (unsigned long t = 1; t <= steps; t++)
	{
		if (t == warm + 1) t0 = std::chrono::steady_clock::now();
		if (useProtocol)
		{
			const int time = (int)((t - 1) % trialSteps);
			const unsigned int trial = (unsigned int)((t - 1) / trialSteps);
			const bool csTrial = trial >= csStartTN;
			// calcMFActivity (ecmanagementdelay.cpp:175-194); the MF draws of step t
			cbm_refshim_set_step(t);
			const float *freq = freqBG.data();
			if (csTrial && time >= csOn && time < csOff) freq = time < csPOff ? freqCSP.data() : freqCST.data();
			const ct_uint8_t *apMF = mfs->calcActivity(freq);
			// calcSimActivity (ecmanagementdelay.cpp:196-235)
			if (time == csOff - 1 && csTrial) sim->updateErrDrive(0, usErr);
			if (time >= csOn + plastOn && !grPCPlastSet && csTrial && time < csOff + plastOff)
			{
				grPCPlastSet = true;
				grPCPlastReset = false;
				zones[0]->setGRPCPlastSteps(plastLTD, plastLTP);
			}
			if (!grPCPlastReset && time >= csOff + plastOff && csTrial)
			{
				grPCPlastSet = false;
				grPCPlastReset = true;
				zones[0]->resetGRPCPlastSteps();
			}
			sim->updateMFInput(apMF);
			sim->calcActivity();
			const ct_uint8_t *apNC = zones[0]->exportAPNC();
			const float vm = eyelid->calcStep(apNC);
			const int ct = time - recFrom;
			if (trial >= dataStartTN && trial < dataStartTN + numDataT && ct >= 0 && ct < recLen)
			{
				const size_t dt = trial - dataStartTN, bin = (size_t)ct / binSteps;
				const ct_uint8_t *apPC = zones[0]->exportAPPC();
				for (unsigned int i = 0; i < cp->numNC; i++) ncPSH[(dt * nBins + bin) * cp->numNC + i] += apNC[i];
				for (unsigned int i = 0; i < cp->numPC; i++) pcPSH[(dt * nBins + bin) * cp->numPC + i] += apPC[i];
				eyeTrace[dt * recLen + ct] = vm;
				grPSH->update(inet->exportAPGR());
				// ecmanagementdelay.cpp:244-265
				if (data->getTSPerRasterUpdate() > 0 && ct % data->getTSPerRasterUpdate() == 0 && ct > 0)
				{
					data->updateRaster("go", inet->exportAPBufGO());
					data->updateRaster("sc", inet->exportAPBufSC());
					data->updateRaster("bc", zones[0]->exportAPBufBC());
					data->updateRaster("pc", zones[0]->exportAPBufPC());
					data->updateRaster("nc", zones[0]->exportAPBufNC());
					data->updateRaster("io", zones[0]->exportAPBufIO());
				}
				data->updatePSH("go", inet->exportAPGO());
				data->updatePSH("grInputGO", inet->exportSumGRInputGO());
				data->updatePSH("goInputGO", inet->exportSumGOInputGO());
				data->updatePSH("goOutSynScale", inet->exportGOOutSynScaleGOGO());
				data->updatePSH("mf", apMF);
				data->updatePSH("gr", inet->exportAPGR());
				data->updatePSH("sc", inet->exportAPSC());
				data->updatePSH("bc", zones[0]->exportAPBC());
				data->updatePSH("pc", zones[0]->exportAPPC());
				data->updatePSH("io", zones[0]->exportAPIO());
				data->updateEyelid(vm);
			}
		}
		while (!useProtocol && evi < events.size() && events[evi].t == t)
		{
			const Event &e = events[evi++];
			if (e.kind == "errdrive") sim->updateErrDrive((unsigned)e.zone, e.a);
			else if (e.kind == "plast") zones[e.zone]->setGRPCPlastSteps(e.a, e.b);
			else if (e.kind == "plastreset") zones[e.zone]->resetGRPCPlastSteps();
			else if (e.kind == "grgoinc") inet->setGIncGRtoGO(e.a);
			else if (e.kind == "grgoincreset") inet->resetGIncGRtoGO();
		}
		if (!useProtocol)
		{
			sim->updateMFInput(&mf[(size_t)(t - 1) * cp->numMF]);
			cbm_refshim_set_step(t);
			sim->calcActivity();
		}
		if (timeOnly) continue;

		const ct_uint8_t *apGR = inet->exportAPGR();
		std::fill(bits.begin(), bits.end(), 0);
		for (unsigned int i = 0; i < cp->numGR; i++) if (apGR[i]) bits[i >> 3] |= (ct_uint8_t)(1u << (i & 7));
		put(tr, bits.data(), bits.size());
		put(tr, inet->exportAPGO(), cp->numGO);
		put(tr, inet->exportVmGO(), cp->numGO);
		put(tr, inet->exportSumGRInputGO(), cp->numGO);
		put(tr, inet->exportAPSC(), cp->numSC);
		put(tr, inet->exportVmSC(), cp->numSC);
		for (unsigned int z = 0; z < nZones; z++)
		{
			put(tr, zones[z]->exportAPBC(), cp->numBC);
			put(tr, zones[z]->exportVmBC(), cp->numBC);
			put(tr, zones[z]->exportAPPC(), cp->numPC);
			put(tr, zones[z]->exportVmPC(), cp->numPC);
			put(tr, zones[z]->exportAPIO(), cp->numIO);
			put(tr, zones[z]->exportVmIO(), cp->numIO);
			put(tr, zones[z]->exportAPNC(), cp->numNC);
			put(tr, zones[z]->exportVmNC(), cp->numNC);
		}
	}
	auto t1 = std::chrono::steady_clock::now();
	double sec = std::chrono::duration<double>(t1 - t0).count();
	if (tr) fclose(tr);
	printf("{\"steps\": %lu, \"seconds\": %.6f, \"steps_per_s\": %.3f, \"num_gr\": %u}\n",
			steps - (warm < steps ? warm : steps), sec, sec > 0 ? (steps - (warm < steps ? warm : steps)) / sec : 0.0, cp->numGR);
	fflush(stdout);

	if (useProtocol)
	{
		FILE *f = fopen(recordsPath, "wb");
		if (!f) { fprintf(stderr, "cannot open records\n"); return 1; }
		put(f, ncPSH.data(), ncPSH.size());
		put(f, pcPSH.data(), pcPSH.size());
		put(f, eyeTrace.data(), eyeTrace.size());
		const std::vector<std::vector<float> > cells = grPSH->getPopPSHs();  // [cell][bin]
		std::vector<float> byBin((size_t)grPSH->getNumBins() * cp->numGR);
		for (unsigned int i = 0; i < cp->numGR; i++)
			for (unsigned int b = 0; b < grPSH->getNumBins(); b++) byBin[(size_t)b * cp->numGR + i] = cells[i][b];
		put(f, byBin.data(), byBin.size());
		// the driver's histograms [bin][cell], then its rasters [trial][row][cell]
		// as 32-step words (bit 31 the earliest step, SpikeRasterBitArray's order
		// of getPopSpikesAtTS; rows the raster did not reach are whatever its
		// allocation held)
		for (int k = 0; k < 10; k++)
		{
			PeriStimHistFloat *h = data->getPSH(pshNames[k]);
			const std::vector<std::vector<float> > c = h->getPopPSHs();
			std::vector<float> v((size_t)h->getNumBins() * h->getNumCells());
			for (unsigned int i = 0; i < h->getNumCells(); i++)
				for (unsigned int b = 0; b < h->getNumBins(); b++) v[(size_t)b * h->getNumCells() + i] = c[i][b];
			put(f, v.data(), v.size());
		}
		const unsigned int rows = (unsigned int)recLen / 32;
		for (int k = 0; k < 6; k++)
		{
			ISpikeRaster *r = data->getRaster(rasterNames[k]);
			const unsigned int n = r->getNumCells();
			std::vector<ct_uint32_t> w((size_t)numDataT * rows * n, 0);
			for (unsigned int tr2 = 0; tr2 < numDataT; tr2++)
				for (unsigned int ts = 0; ts < rows * 32; ts++)
				{
					const std::vector<bool> aps = r->getPopSpikesAtTS(ts, tr2);
					for (unsigned int i = 0; i < n; i++)
						if (aps[i]) w[((size_t)tr2 * rows + ts / 32) * n + i] |= 0x80000000u >> (ts % 32);
				}
			put(f, w.data(), w.size());
		}
		// the driver's smoothed eyelid trace (EyelidOut, eyelidout.cpp), [numDataTrials][window]
		for (unsigned int tr2 = 0; tr2 < numDataT; tr2++)
		{
			const std::vector<float> e = data->getEyelidData()->getEyelidData(tr2);
			put(f, e.data(), e.size());
		}
		fclose(f);
		if (dataPath)
		{
			// the driver's data file (ECTrialsData::writeData, ectrialsdata.cpp)
			std::fstream df(dataPath, std::ios::out | std::ios::binary | std::ios::trunc);
			data->writeData(df);
		}
		if (sessionPath)
		{
			// ECManagementDelay::writeDataToFile (ecmanagementdelay.cpp:275-290):
			// the state, then the trial data, in one file
			std::fstream sf(sessionPath, std::ios::out | std::ios::binary | std::ios::trunc);
			sim->writeToState(sf);
			data->writeData(sf);
		}
		if (mfPopPath)
		{
			// the MF rates the reference estimates from the run's MF histogram
			// (ECMFPopulation(ECTrialsData *), ecmfpopulation.cpp:11-65), in its file format
			ECMFPopulation pop(data);
			std::fstream pf(mfPopPath, std::ios::out | std::ios::binary | std::ios::trunc);
			pop.writeToFile(pf);
		}
		delete data;
		delete grPSH;
		delete mfs;
		delete eyelid;
	}
	if (strcmp(finalPath, "-") != 0)
	{
		std::fstream out(finalPath, std::ios::out | std::ios::binary | std::ios::trunc);
		sim->writeToState(out);
		out.close();
	}
	delete sim;
	delete st;
	return 0;
}
#endif
