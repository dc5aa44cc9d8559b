// C ABI (include/cbm_b200.h) over the state and simulator classes.
#include "../../include/cbm_b200.h"

#include <cstdio>
#include <algorithm>
#include <cstring>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "cbm_kernels.cuh"
#include "cbm_sim.hpp"
#include "cbm_state.hpp"

using namespace cbm;

struct cbm_state { State st; };
struct cbm_sim { Simulator sim; cbm_state *owner = nullptr; };

// last error message of the calling thread (cbm_last_error)
thread_local std::string g_cbmLastError;

static int fail(int code, const std::string &msg)
{
	g_cbmLastError = msg;
	return code;
}

static int classify(const std::string &msg)
{
	if (msg.find("out of range") != std::string::npos) return CBM_ERR_RANGE;
	if (msg.find("must") != std::string::npos || msg.find("supported") != std::string::npos ||
			msg.find("one bit") != std::string::npos || msg.find("powers of two") != std::string::npos)
		return CBM_ERR_UNSUPPORTED;
	if (msg.find("cannot open") != std::string::npos || msg.find("write error") != std::string::npos) return CBM_ERR_IO;
	if (msg.find("truncated") != std::string::npos || msg.find("parameter") != std::string::npos ||
			msg.find("matrix") != std::string::npos || msg.find("zone count") != std::string::npos)
		return CBM_ERR_FORMAT;
	return CBM_ERR_CUDA;
}

#define TRY(expr) do { std::string e_ = (expr); if (!e_.empty()) return fail(classify(e_), e_); } while (0)
#define NEED(p) do { if (!(p)) return fail(CBM_ERR_ARG, "null argument: " #p); } while (0)

extern "C" {

const char *cbm_last_error(void) { return g_cbmLastError.c_str(); }

int cbm_state_load(const char *path, cbm_state **out)
{
	NEED(path); NEED(out);
	cbm_state *s = new (std::nothrow) cbm_state();
	if (!s) return fail(CBM_ERR_ARG, "out of host memory");
	std::string e = s->st.load(path);
	if (!e.empty()) { delete s; return fail(classify(e), e); }
	*out = s;
	return CBM_OK;
}

int cbm_state_new(const char *conText, const char *actText, unsigned nZones, const int *seeds, cbm_state **out)
{
	NEED(conText); NEED(actText); NEED(out);
	if (nZones < 1 || nZones > (unsigned)kMaxZones) return fail(CBM_ERR_ARG, "zone count must be 1..4");
	cbm_state *s = new (std::nothrow) cbm_state();
	if (!s) return fail(CBM_ERR_ARG, "out of host memory");
	std::vector<int> sd;
	if (seeds) sd.assign(seeds, seeds + nZones);
	std::string e = s->st.create(conText, actText, nZones, sd);
	if (!e.empty()) { delete s; return fail(classify(e), e); }
	*out = s;
	return CBM_OK;
}

int cbm_state_generate(const char *conText, const char *actText, unsigned nZones, const int *seeds, cbm_state **out)
{
	NEED(conText); NEED(actText); NEED(out);
	if (nZones < 1 || nZones > (unsigned)kMaxZones) return fail(CBM_ERR_ARG, "zone count must be 1..4");
	std::vector<int> sd = seeds ? std::vector<int>(seeds, seeds + 1 + 2 * nZones) : clockSeeds(nZones);
	std::vector<int> conSeeds;
	for (unsigned z = 0; z < nZones; z++) conSeeds.push_back(sd[1 + z]);
	cbm_state *s = new (std::nothrow) cbm_state();
	if (!s) return fail(CBM_ERR_ARG, "out of host memory");
	std::string e = s->st.generate(conText, actText, nZones, sd[0], conSeeds);
	if (!e.empty()) { delete s; return fail(classify(e), e); }
	*out = s;
	return CBM_OK;
}

int cbm_state_save(cbm_state *s, const char *path)
{
	NEED(s); NEED(path);
	TRY(s->st.save(path));
	// innetactivitystate.cpp:247-248 run on write as well
	NamedArray *a = s->st.find("inputGOGABASynDepGO"), *b = s->st.find("goGABAOutSynScaleGOGO");
	if (a) for (size_t i = 0; i < a->count; i++) a->as<float>()[i] = 1.0f;
	if (b) for (size_t i = 0; i < b->count; i++) b->as<float>()[i] = 0.0f;
	return CBM_OK;
}

int cbm_state_load_mem(const void *data, uint64_t len, uint64_t *consumed, cbm_state **out)
{
	NEED(data); NEED(out);
	cbm_state *s = new (std::nothrow) cbm_state();
	if (!s) return fail(CBM_ERR_ARG, "out of host memory");
	size_t used = 0;
	std::string e = s->st.loadBytes(std::string((const char *)data, (size_t)len), &used);
	if (!e.empty()) { delete s; return fail(classify(e), e); }
	if (consumed) *consumed = used;
	*out = s;
	return CBM_OK;
}

// Serialises st into dst (cap bytes) through a memory stream; *size gets the
// bytes the state occupies.  dst == NULL only asks for the size.
static int saveToMemory(const State &st, void *dst, uint64_t cap, uint64_t *size)
{
	const size_t n = st.fileBytes();
	*size = n;
	if (!dst) return CBM_OK;
	if (cap < n) return fail(CBM_ERR_ARG, "buffer smaller than the state (" + std::to_string(n) + " bytes)");
	std::ostringstream os(std::ios::binary);
	std::string e = st.writeTo(os);
	if (!e.empty()) return fail(CBM_ERR_IO, e);
	const std::string &b = os.str();
	if (b.size() != n) return fail(CBM_ERR_IO, "state serialisation size mismatch");
	memcpy(dst, b.data(), n);
	return CBM_OK;
}

int cbm_state_save_mem(cbm_state *s, void *dst, uint64_t cap, uint64_t *size)
{
	NEED(s); NEED(size);
	int rc = saveToMemory(s->st, dst, cap, size);
	if (rc != CBM_OK || !dst) return rc;
	// innetactivitystate.cpp:247-248 run on write as well
	NamedArray *a = s->st.find("inputGOGABASynDepGO"), *b = s->st.find("goGABAOutSynScaleGOGO");
	if (a) for (size_t i = 0; i < a->count; i++) a->as<float>()[i] = 1.0f;
	if (b) for (size_t i = 0; i < b->count; i++) b->as<float>()[i] = 0.0f;
	return CBM_OK;
}

void cbm_state_free(cbm_state *s) { delete s; }

int cbm_state_num_zones(const cbm_state *s, unsigned *out)
{
	NEED(s); NEED(out);
	*out = s->st.numZones;
	return CBM_OK;
}

int cbm_state_array(cbm_state *s, const char *name, int zone, void **data, uint64_t *count, int *dtype)
{
	NEED(s); NEED(name); NEED(data); NEED(count); NEED(dtype);
	NamedArray *a = s->st.find(name, zone);
	if (!a) return fail(CBM_ERR_ARG, std::string("no array ") + name);
	*data = a->bytes.data();
	*count = a->count;
	*dtype = (int)a->dtype;
	return CBM_OK;
}

#define CP_FIELDS(X) X(glX) X(glY) X(numGL) X(maxnumpGLfromGLtoGR) X(lownumpGLfromGLtoGR) X(maxnumpGLfromGLtoGO) \
	X(maxnumpGLfromGOtoGL) X(numMF) X(numpMFfromMFtoGL) X(maxnumpMFfromMFtoGO) X(maxnumpMFfromMFtoGR) \
	X(numpMFfromMFtoNC) X(goX) X(goY) X(numGO) X(maxnumpGOfromGRtoGO) X(maxnumpGOfromGLtoGO) \
	X(maxnumpGOfromMFtoGO) X(maxnumpGOfromGOtoGL) X(maxnumpGOfromGOtoGR) X(grX) X(grY) X(numGR) X(numGRP2) \
	X(grPFVelInGRXPerTStep) X(grAFDelayInTStep) X(maxnumpGRfromGRtoGO) X(maxnumpGRfromGLtoGR) \
	X(maxnumpGRfromGOtoGR) X(maxnumpGRfromMFtoGR) X(numSC) X(numpSCfromGRtoSC) X(numpSCfromGRtoSCP2) \
	X(numpSCfromSCtoPC) X(numPC) X(numpPCfromGRtoPC) X(numpPCfromGRtoPCP2) X(numpPCfromBCtoPC) \
	X(numpPCfromPCtoBC) X(numpPCfromSCtoPC) X(numpPCfromPCtoNC) X(numBC) X(numpBCfromGRtoBC) \
	X(numpBCfromGRtoBCP2) X(numpBCfromBCtoPC) X(numpBCfromPCtoBC) X(numNC) X(numpNCfromPCtoNC) \
	X(numpNCfromNCtoIO) X(numpNCfromMFtoNC) X(numIO) X(numpIOfromIOtoPC) X(numpIOfromNCtoIO) \
	X(numpIOInIOIO) X(numpIOOutIOIO) X(maxnumpGOGABAInGOGO) X(maxnumpGOGABAOutGOGO) \
	X(maxnumpGOCoupInGOGO) X(maxnumpGOCoupOutGOGO)

int cbm_state_con_param(const cbm_state *s, const char *name, uint32_t *value)
{
	NEED(s); NEED(name); NEED(value);
	const ConParams &c = s->st.cp;
#define X(f) if (!strcmp(name, #f)) { *value = c.f; return CBM_OK; }
	CP_FIELDS(X)
#undef X
	auto it = c.raw.find(name);
	if (it != c.raw.end()) { *value = it->second; return CBM_OK; }
	return fail(CBM_ERR_ARG, std::string("no connectivity parameter ") + name);
}

#define AP_FIELDS(X) X(msPerTimeStep) X(msPerHistBinMF) X(numTSinMFHist) X(eLeakGO) X(eMGluRGO) X(eGABAGO) \
	X(threshMaxGO) X(threshRestGO) X(gIncMFtoGO) X(gIncGRtoGO) X(gGABAIncGOtoGO) X(coupleRiRjRatioGO) \
	X(gMGluRScaleGRtoGO) X(gMGluRIncScaleGO) X(mGluRScaleGO) X(gluScaleGO) X(gLeakGO) X(goGABAGOGOSynRecTau) \
	X(goGABAGOGOSynRec) X(goGABAGOGOSynDepF) X(gDecTauMFtoGO) X(gDecMFtoGO) X(gDecTauGRtoGO) X(gDecGRtoGO) \
	X(gGABADecTauGOtoGO) X(gGABADecGOtoGO) X(mGluRDecayGO) X(gMGluRIncDecayGO) X(gMGluRDecGRtoGO) \
	X(gluDecayGO) X(threshDecTauGO) X(threshDecGO) X(eLeakGR) X(eGOGR) X(eMFGR) X(threshMaxGR) \
	X(threshRestGR) X(gIncMFtoGR) X(gIncGOtoGR) X(gDecTauMFtoGR) X(gDecMFtoGR) X(gDecTauGOtoGR) X(gDecGOtoGR) \
	X(threshDecTauGR) X(threshDecGR) X(gLeakGR) X(msPerHistBinGR) X(tsPerHistBinGR) X(eLeakSC) X(gLeakSC) \
	X(gDecTauGRtoSC) X(gDecGRtoSC) X(threshMaxSC) X(threshRestSC) X(threshDecTauSC) X(threshDecSC) \
	X(gIncGRtoSC) X(eLeakBC) X(ePCtoBC) X(gLeakBC) X(gDecTauGRtoBC) X(gDecGRtoBC) X(gDecTauPCtoBC) \
	X(gDecPCtoBC) X(threshDecTauBC) X(threshDecBC) X(threshRestBC) X(threshMaxBC) X(gIncGRtoBC) X(gIncPCtoBC) \
	X(initSynWofGRtoPC) X(eLeakPC) X(eBCtoPC) X(eSCtoPC) X(threshMaxPC) X(threshRestPC) X(threshDecTauPC) \
	X(threshDecPC) X(gLeakPC) X(gDecTauGRtoPC) X(gDecGRtoPC) X(gDecTauBCtoPC) X(gDecBCtoPC) X(gDecTauSCtoPC) \
	X(gDecSCtoPC) X(gIncSCtoPC) X(gIncGRtoPC) X(gIncBCtoPC) X(tsPopHistPC) X(tsPerPopHistBinPC) \
	X(numPopHistBinsPC) X(synLTPStepSizeGRtoPC) X(synLTDStepSizeGRtoPC) X(coupleRiRjRatioIO) X(eLeakIO) \
	X(eNCtoIO) X(gLeakIO) X(gDecTSofNCtoIO) X(gDecTTofNCtoIO) X(gDecT0ofNCtoIO) X(gIncNCtoIO) X(gIncTauNCtoIO) \
	X(threshRestIO) X(threshMaxIO) X(threshDecTauIO) X(threshDecIO) X(tsLTDDurationIO) X(tsLTDStartAPIO) \
	X(tsLTPStartAPIO) X(grPCHistCheckBinIO) X(maxExtIncVIO) X(eLeakNC) X(ePCtoNC) X(gmaxNMDADecTauMFtoNC) \
	X(gmaxNMDADecMFtoNC) X(gmaxAMPADecTauMFtoNC) X(gmaxAMPADecMFtoNC) X(gNMDAIncMFtoNC) X(gAMPAIncMFtoNC) \
	X(gIncAvgPCtoNC) X(gDecTauPCtoNC) X(gDecPCtoNC) X(gLeakNC) X(threshDecTauNC) X(threshDecNC) X(threshMaxNC) \
	X(threshRestNC) X(relPDecTSofNCtoIO) X(relPDecTTofNCtoIO) X(relPDecT0ofNCtoIO) X(relPIncNCtoIO) \
	X(relPIncTauNCtoIO) X(initSynWofMFtoNC) X(synLTDPCPopActThreshMFtoNC) X(synLTPPCPopActThreshMFtoNC) \
	X(synLTDStepSizeMFtoNC) X(synLTPStepSizeMFtoNC)

int cbm_state_act_param(const cbm_state *s, const char *name, double *value)
{
	NEED(s); NEED(name); NEED(value);
	const ActParams &a = s->st.ap;
#define X(f) if (!strcmp(name, #f)) { *value = (double)a.f; return CBM_OK; }
	AP_FIELDS(X)
#undef X
	auto it = a.raw.find(name);
	if (it != a.raw.end()) { *value = it->second; return CBM_OK; }
	return fail(CBM_ERR_ARG, std::string("no activity parameter ") + name);
}

int cbm_state_set_act_param(cbm_state *s, const char *key, float value)
{
	NEED(s); NEED(key);
	if (!s->st.ap.set(key, value)) return fail(CBM_ERR_ARG, std::string("unknown activity parameter ") + key);
	return CBM_OK;
}

int cbm_state_param_names(const cbm_state *s, int which, char *buf, uint64_t size, uint64_t *needed)
{
	NEED(s); NEED(needed);
	if (which != 0 && which != 1) return fail(CBM_ERR_ARG, "which must be 0 (connectivity) or 1 (activity)");
	std::string list;
	if (which == 0) for (const auto &kv : s->st.cp.raw) list += kv.first + "\n";
	else for (const auto &kv : s->st.ap.raw) list += kv.first + "\n";
	*needed = list.size() + 1;
	if (!buf || size < list.size() + 1) return fail(CBM_ERR_ARG, "name buffer too small");
	memcpy(buf, list.c_str(), list.size() + 1);
	return CBM_OK;
}

int cbm_state_raw_param(const cbm_state *s, int which, const char *name, double *value)
{
	NEED(s); NEED(name); NEED(value);
	if (which == 0) {
		auto it = s->st.cp.raw.find(name);
		if (it == s->st.cp.raw.end()) return fail(CBM_ERR_ARG, std::string("no connectivity parameter ") + name);
		*value = it->second;
		return CBM_OK;
	}
	if (which == 1) {
		auto it = s->st.ap.raw.find(name);
		if (it == s->st.ap.raw.end()) return fail(CBM_ERR_ARG, std::string("no activity parameter ") + name);
		*value = it->second;
		return CBM_OK;
	}
	return fail(CBM_ERR_ARG, "which must be 0 (connectivity) or 1 (activity)");
}

static int simCreate(cbm_state *s, const int *seeds, int device, uint32_t ring, cbm_sim **out)
{
	NEED(s); NEED(out);
	cbm_sim *sim = new (std::nothrow) cbm_sim();
	if (!sim) return fail(CBM_ERR_ARG, "out of host memory");
	std::vector<std::vector<int>> sd(1);
	if (seeds) sd[0].assign(seeds, seeds + s->st.numZones);
	std::string e = sim->sim.create({&s->st}, sd, device, ring);
	if (!e.empty()) { delete sim; return fail(classify(e), e); }
	sim->owner = s;
	*out = sim;
	return CBM_OK;
}

int cbm_sim_create(cbm_state *s, const int *seeds, int device, cbm_sim **out)
{
	return simCreate(s, seeds, device, 4, out);
}

int cbm_sim_create_resident(cbm_state *s, const int *seeds, int device, uint64_t mfSteps, cbm_sim **out)
{
	if (mfSteps == 0 || mfSteps > 0xFFFFFFFFull) return fail(CBM_ERR_ARG, "mfSteps must be 1..2^32-1");
	return simCreate(s, seeds, device, (uint32_t)mfSteps, out);
}

#define NET(sim) (sim)->sim.net(0)
#define ZONE_OK(sim, z) do { if ((z) >= NET(sim).dev().numZones) return fail(CBM_ERR_ARG, "zone out of range"); } while (0)

int cbm_sim_update_mf(cbm_sim *sim, const uint8_t *mf)
{
	NEED(sim); NEED(mf);
	TRY(sim->sim.stageMF(0, mf));
	return CBM_OK;
}

int cbm_sim_calc_activity(cbm_sim *sim)
{
	NEED(sim);
	TRY(sim->sim.launchSteps(1));
	return CBM_OK;
}

int cbm_sim_update_err_drive(cbm_sim *sim, unsigned zone, float rel)
{
	NEED(sim); ZONE_OK(sim, zone);
	NET(sim).setErrDrive(zone, rel);
	return CBM_OK;
}

int cbm_sim_set_plast_steps(cbm_sim *sim, unsigned zone, float ltd, float ltp)
{
	NEED(sim); ZONE_OK(sim, zone);
	NET(sim).setPlastSteps(zone, ltd, ltp);
	return CBM_OK;
}

int cbm_sim_reset_plast_steps(cbm_sim *sim, unsigned zone)
{
	NEED(sim); ZONE_OK(sim, zone);
	NET(sim).resetPlastSteps(zone);
	return CBM_OK;
}

int cbm_sim_set_ginc_grgo(cbm_sim *sim, float inc)
{
	NEED(sim);
	NET(sim).setGIncGRtoGO(inc);
	return CBM_OK;
}

int cbm_sim_reset_ginc_grgo(cbm_sim *sim)
{
	NEED(sim);
	NET(sim).resetGIncGRtoGO();
	return CBM_OK;
}

int cbm_sim_export(cbm_sim *sim, int field, unsigned zone, void *dst, uint64_t bytes)
{
	NEED(sim); NEED(dst);
	if (field < 0 || field >= CBM_FIELD_COUNT) return fail(CBM_ERR_ARG, "unknown field");
	TRY(sim->sim.exportField(0, (Field)field, zone, dst, bytes));
	return CBM_OK;
}

uint64_t cbm_sim_field_bytes(cbm_sim *sim, int field)
{
	if (!sim || field < 0 || field >= CBM_FIELD_COUNT) return 0;
	return NET(sim).fieldBytes((Field)field);
}

int cbm_sim_write_to_state(cbm_sim *sim)
{
	NEED(sim);
	TRY(sim->sim.sync());
	TRY(NET(sim).writeToState(sim->sim.stream()));
	return CBM_OK;
}

int cbm_sim_save(cbm_sim *sim, const char *path)
{
	NEED(sim); NEED(path);
	TRY(sim->sim.sync());
	TRY(NET(sim).writeToState(sim->sim.stream()));
	TRY(NET(sim).state()->save(path));
	TRY(NET(sim).resetGOGODepression(sim->sim.stream()));
	return CBM_OK;
}

int cbm_sim_save_mem(cbm_sim *sim, void *dst, uint64_t cap, uint64_t *size)
{
	NEED(sim); NEED(size);
	if (!dst) return saveToMemory(*NET(sim).state(), nullptr, 0, size);
	TRY(sim->sim.sync());
	TRY(NET(sim).writeToState(sim->sim.stream()));
	int rc = saveToMemory(*NET(sim).state(), dst, cap, size);
	if (rc != CBM_OK) return rc;
	TRY(NET(sim).resetGOGODepression(sim->sim.stream()));
	return CBM_OK;
}

int cbm_sim_steps_done(cbm_sim *sim, uint64_t *steps)
{
	NEED(sim); NEED(steps);
	*steps = NET(sim).stepsDone();
	return CBM_OK;
}

int cbm_sim_mf_words(cbm_sim *sim, uint32_t *words)
{
	NEED(sim); NEED(words);
	*words = NET(sim).mfWords();
	return CBM_OK;
}

int cbm_sim_load_mf_stream(cbm_sim *sim, const uint32_t *bits, uint64_t nsteps)
{
	NEED(sim); NEED(bits);
	Network &n = NET(sim);
	if (n.hasProtocol()) return fail(CBM_ERR_ARG, "a device protocol drives the MF input of this network");
	if (nsteps > n.mfRing()) return fail(CBM_ERR_ARG, "more MF steps than the resident ring holds");
	// rows land in the slots of the next nsteps steps
	const uint64_t first = n.stepsDone() % n.mfRing();
	const uint32_t W = n.mfWords();
	const uint64_t tail = std::min<uint64_t>(nsteps, n.mfRing() - first);
	TRY(n.uploadMFBits(bits, first, tail, sim->sim.stream()));
	if (nsteps > tail) TRY(n.uploadMFBits(bits + tail * W, 0, nsteps - tail, sim->sim.stream()));
	TRY(sim->sim.sync());
	return CBM_OK;
}

int cbm_sim_run(cbm_sim *sim, uint64_t nsteps, uint32_t chunk, float *gpuMs, float *passMs)
{
	NEED(sim);
	TRY(sim->sim.runGraph(nsteps, chunk, passMs != nullptr));
	if (gpuMs) *gpuMs = sim->sim.lastGraphMs();
	if (passMs) *passMs = sim->sim.lastPassMs();
	return CBM_OK;
}

int cbm_sim_run_flushed(cbm_sim *sim, uint64_t nsteps, uint64_t flushBytes, float *stepMs)
{
	NEED(sim); NEED(stepMs);
	TRY(sim->sim.runFlushed(nsteps, (size_t)flushBytes, stepMs));
	return CBM_OK;
}

int cbm_sim_run_flushed_kernels(cbm_sim *sim, uint64_t nsteps, uint64_t flushBytes, float *passMs, float *tailMs)
{
	NEED(sim); NEED(passMs); NEED(tailMs);
	TRY(sim->sim.runFlushedKernels(nsteps, (size_t)flushBytes, passMs, tailMs));
	return CBM_OK;
}

int cbm_sim_set_eyelid_protocol(cbm_sim *sim, const cbm_eyelid_protocol *protocol)
{
	NEED(sim); NEED(protocol);
	TRY(sim->sim.setProtocol(0, *protocol));
	return CBM_OK;
}

int cbm_sim_set_statevar_input(cbm_sim *sim, const cbm_statevar_input *input)
{
	NEED(sim); NEED(input);
	TRY(sim->sim.setStateVarInput(0, *input));
	return CBM_OK;
}

int cbm_sim_statevar_rates(cbm_sim *sim, uint64_t step, float *out)
{
	NEED(sim); NEED(out);
	TRY(sim->sim.sync());
	TRY(NET(sim).stateVarRates(step, out, sim->sim.stream()));
	return CBM_OK;
}

uint64_t cbm_sim_trial_record_bytes(cbm_sim *sim, int kind)
{
	return sim ? NET(sim).recordBytes(kind) : 0;
}

int cbm_sim_trial_record(cbm_sim *sim, int kind, void *dst, uint64_t bytes)
{
	NEED(sim); NEED(dst);
	TRY(NET(sim).readRecord(kind, dst, (size_t)bytes, sim->sim.stream()));
	return CBM_OK;
}

int cbm_sim_record_gr(cbm_sim *sim)
{
	NEED(sim);
	TRY(sim->sim.recordGR());
	return CBM_OK;
}

int cbm_sim_record_trial_data(cbm_sim *sim)
{
	NEED(sim);
	TRY(sim->sim.recordTrialData());
	return CBM_OK;
}

// ---------------------------------------------------------------- batches
struct cbm_batch {
	Simulator sim;
	std::vector<cbm_state *> states;
	std::vector<std::vector<int>> seeds;
	int device = 0;
	// protocols as set, with copies of their rate tables (for the autotuner's scratch copy)
	std::vector<int> hasProto;
	std::vector<cbm_eyelid_protocol> protos;
	std::vector<std::vector<float>> rates;
};

static int batchBuild(Simulator &sim, const std::vector<cbm_state *> &states, const std::vector<std::vector<int>> &seeds,
		int device)
{
	std::vector<State *> st;
	for (cbm_state *s : states) st.push_back(&s->st);
	std::string e = sim.create(st, seeds, device, 2);
	if (!e.empty()) return fail(classify(e), e);
	return CBM_OK;
}

int cbm_batch_create(cbm_state *const *states, unsigned n, const int *mzoneSeeds, int device, cbm_batch **out)
{
	NEED(states); NEED(out);
	if (n == 0) return fail(CBM_ERR_ARG, "empty batch");
	cbm_batch *b = new (std::nothrow) cbm_batch();
	if (!b) return fail(CBM_ERR_ARG, "out of host memory");
	size_t k = 0;
	for (unsigned i = 0; i < n; i++) {
		if (!states[i]) { delete b; return fail(CBM_ERR_ARG, "null state"); }
		b->states.push_back(states[i]);
		std::vector<int> sd;
		if (mzoneSeeds) sd.assign(mzoneSeeds + k, mzoneSeeds + k + states[i]->st.numZones);
		k += states[i]->st.numZones;
		b->seeds.push_back(sd);
	}
	b->device = device;
	b->hasProto.assign(n, 0);
	b->protos.resize(n);
	b->rates.resize(n);
	int rc = batchBuild(b->sim, b->states, b->seeds, device);
	if (rc != CBM_OK) { delete b; return rc; }
	*out = b;
	return CBM_OK;
}

void cbm_batch_destroy(cbm_batch *b) { delete b; }

#define BATCH_OK(b, i) do { NEED(b); if ((i) >= (b)->states.size()) return fail(CBM_ERR_ARG, "instance out of range"); } while (0)

int cbm_batch_set_eyelid_protocol(cbm_batch *b, unsigned i, const cbm_eyelid_protocol *p)
{
	BATCH_OK(b, i); NEED(p);
	TRY(b->sim.setProtocol(i, *p));
	const uint32_t M = b->states[i]->st.cp.numMF;
	std::vector<float> &r = b->rates[i];
	r.resize(3ull * M);
	memcpy(r.data(), p->mfFreqBG, 4ull * M);
	memcpy(r.data() + M, p->mfFreqCSTonic, 4ull * M);
	memcpy(r.data() + 2 * M, p->mfFreqCSPhasic, 4ull * M);
	b->protos[i] = *p;
	b->hasProto[i] = 1;
	return CBM_OK;
}

int cbm_batch_run(cbm_batch *b, uint64_t nsteps, uint32_t chunk, float *gpuMs)
{
	NEED(b);
	TRY(b->sim.runGraph(nsteps, chunk, false));
	if (gpuMs) *gpuMs = b->sim.lastGraphMs();
	return CBM_OK;
}

int cbm_batch_autotune(cbm_batch *b, uint32_t nsteps, char *choice, size_t choiceLen, float *ms)
{
	NEED(b);
	if (nsteps == 0) return fail(CBM_ERR_ARG, "nsteps must be positive");
	const uint32_t chunk = std::min<uint32_t>(nsteps, 25);
	PassGeometry best;
	float bestMs = -1;
	{
		Simulator scratch;
		int rc = batchBuild(scratch, b->states, b->seeds, b->device);
		if (rc != CBM_OK) return rc;
		for (size_t i = 0; i < b->states.size(); i++) {
			if (!b->hasProto[i]) continue;
			cbm_eyelid_protocol p = b->protos[i];
			const uint32_t M = b->states[i]->st.cp.numMF;
			p.mfFreqBG = b->rates[i].data();
			p.mfFreqCSTonic = b->rates[i].data() + M;
			p.mfFreqCSPhasic = b->rates[i].data() + 2 * M;
			TRY(scratch.setProtocol(i, p));
		}
		for (const PassGeometry &g : scratch.passCandidates()) {
			if (!scratch.usePassGeometry(g).empty()) continue;
			TRY(scratch.runGraph(2 * chunk, chunk, false));  // warm-up and capture
			TRY(scratch.runGraph(nsteps - nsteps % chunk ? nsteps - nsteps % chunk : chunk, chunk, false));
			const float t = scratch.lastGraphMs();
			if (bestMs < 0 || t < bestMs) { bestMs = t; best = g; }
		}
	}
	if (bestMs < 0) return fail(CBM_ERR_UNSUPPORTED, "no GR-pass geometry runs this batch");
	TRY(b->sim.usePassGeometry(best));
	if (choice && choiceLen) snprintf(choice, choiceLen, "%d,%d,%d,%d,%d,%d", best.kind, best.W, best.RW, best.S, best.B, best.M);
	if (ms) *ms = bestMs;
	return CBM_OK;
}

int cbm_batch_pass_geometry(cbm_batch *b, unsigned *kind, unsigned *consumerWarps, unsigned *rowsPerStage,
		unsigned *stages)
{
	NEED(b); NEED(kind); NEED(consumerWarps); NEED(rowsPerStage); NEED(stages);
	b->sim.passGeometry(kind, consumerWarps, rowsPerStage, stages);
	return CBM_OK;
}

uint64_t cbm_batch_trial_record_bytes(cbm_batch *b, unsigned i, int kind)
{
	if (!b || i >= b->states.size()) return 0;
	return b->sim.net(i).recordBytes(kind);
}

int cbm_batch_trial_record(cbm_batch *b, unsigned i, int kind, void *dst, uint64_t bytes)
{
	BATCH_OK(b, i); NEED(dst);
	TRY(b->sim.sync());
	TRY(b->sim.net(i).readRecord(kind, dst, (size_t)bytes, b->sim.stream()));
	return CBM_OK;
}

int cbm_batch_record_trial_data(cbm_batch *b, unsigned i)
{
	BATCH_OK(b, i);
	TRY(b->sim.recordTrialData(i));
	return CBM_OK;
}

int cbm_batch_write_to_state(cbm_batch *b, unsigned i)
{
	BATCH_OK(b, i);
	TRY(b->sim.sync());
	TRY(b->sim.net(i).writeToState(b->sim.stream()));
	return CBM_OK;
}

uint64_t cbm_batch_num_gr(cbm_batch *b)
{
	if (!b) return 0;
	uint64_t n = 0;
	for (cbm_state *s : b->states) n += s->st.cp.numGR;
	return n;
}

int cbm_sim_last_tail_ms(cbm_sim *sim, float *ms)
{
	NEED(sim); NEED(ms);
	*ms = sim->sim.lastTailMs();
	return CBM_OK;
}

int cbm_sim_timer_start(cbm_sim *sim)
{
	NEED(sim);
	TRY(sim->sim.timerStart());
	return CBM_OK;
}

int cbm_sim_timer_stop(cbm_sim *sim, float *ms)
{
	NEED(sim); NEED(ms);
	TRY(sim->sim.timerStop(ms));
	return CBM_OK;
}

double cbm_sim_algorithmic_bytes_per_step(cbm_sim *sim)
{
	return sim ? NET(sim).bytesPerStepAlgorithmic() : 0.0;
}

double cbm_sim_layout_bytes_per_step(cbm_sim *sim)
{
	return sim ? NET(sim).bytesPerStepLayout() : 0.0;
}

int cbm_sim_pass_geometry(cbm_sim *sim, unsigned *kind, unsigned *consumerWarps, unsigned *rowsPerStage,
		unsigned *stages)
{
	NEED(sim); NEED(kind); NEED(consumerWarps); NEED(rowsPerStage); NEED(stages);
	sim->sim.passGeometry(kind, consumerWarps, rowsPerStage, stages);
	return CBM_OK;
}

void cbm_sim_destroy(cbm_sim *sim) { delete sim; }

int cbm_device_expf(int device, const float *in, float *out, uint64_t n)
{
	NEED(in); NEED(out);
	if (cudaSetDevice(device) != cudaSuccess) return fail(CBM_ERR_CUDA, "cannot select device");
	float *d = nullptr;
	if (cudaMalloc(&d, 2 * n * sizeof(float)) != cudaSuccess) return fail(CBM_ERR_CUDA, "device allocation failed");
	cudaMemcpy(d, in, n * sizeof(float), cudaMemcpyHostToDevice);
	expfProbeKernel<<<(unsigned)((n + 255) / 256), 256>>>(d, d + n, (uint32_t)n);
	cudaError_t e = cudaMemcpy(out, d + n, n * sizeof(float), cudaMemcpyDeviceToHost);
	cudaFree(d);
	if (e != cudaSuccess) return fail(CBM_ERR_CUDA, cudaGetErrorString(e));
	return CBM_OK;
}

int cbm_device_exp(int device, const double *in, double *out, uint64_t n)
{
	NEED(in); NEED(out);
	if (n > 0xFFFFFFFFull) return fail(CBM_ERR_ARG, "at most 2^32-1 values per call");
	if (cudaSetDevice(device) != cudaSuccess) return fail(CBM_ERR_CUDA, "cannot select device");
	double *d = nullptr;
	if (cudaMalloc(&d, 2 * n * sizeof(double)) != cudaSuccess) return fail(CBM_ERR_CUDA, "device allocation failed");
	cudaMemcpy(d, in, n * sizeof(double), cudaMemcpyHostToDevice);
	expProbeKernel<<<(unsigned)((n + 255) / 256), 256>>>(d, d + n, (uint32_t)n);
	cudaError_t e = cudaMemcpy(out, d + n, n * sizeof(double), cudaMemcpyDeviceToHost);
	cudaFree(d);
	if (e != cudaSuccess) return fail(CBM_ERR_CUDA, cudaGetErrorString(e));
	return CBM_OK;
}

}  // extern "C"
