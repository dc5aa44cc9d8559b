/* C ABI of the B200 cerebellar network step.
 *
 * This is the boundary a host program binds to in place of the reference's
 * CBM_CORE_LIB (CBMSimCore / InNetInterface / MZoneInterface) and
 * CBM_STATE_LIB (CBMState).  Every call returns a status code (CBM_OK on
 * success); cbm_last_error() describes the last failure of the calling
 * thread.  Objects are not thread-safe: one thread per simulator, like the
 * reference (its GUI serialises access through a mutex,
 * Eyelid_Sim_CBM_Dev/src/gui/simthread.cpp:196).
 *
 * Reference interfaces replaced (paths within the reference project):
 *   CBMState         CBM_STATE_LIB_DEV/CBMStateInclude/interfaces/cbmstate.h:37-62
 *   CBMSimCore       CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/cbmsimcore.h:35-49
 *   InNetInterface   CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/innetinterface.h:18-41
 *   MZoneInterface   CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/mzoneinterface.h:18-34
 */
#ifndef CBM_B200_H
#define CBM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CBM_OK 0
#define CBM_ERR_ARG 1          /* bad argument (null pointer, zone or size out of range) */
#define CBM_ERR_CUDA 2         /* CUDA runtime error */
#define CBM_ERR_IO 3           /* file could not be read or written */
#define CBM_ERR_FORMAT 4       /* malformed or truncated state file / parameter text */
#define CBM_ERR_RANGE 5        /* connectivity index or count out of range */
#define CBM_ERR_UNSUPPORTED 6  /* network shape outside what the kernels implement */

/* array element types reported by cbm_state_array */
#define CBM_U8 0
#define CBM_I32 1
#define CBM_U32 2
#define CBM_F32 3
#define CBM_U64 4

/* fields readable with cbm_sim_export; the *_GR, *_GO, *_SC and *_MF fields
 * are the input net's, the rest are per microzone */
enum cbm_field {
	CBM_AP_GR = 0,            /* u8[numGR]   InNetInterface::exportAPGR   (innet.cpp:687) */
	CBM_VM_GR,                /* f32[numGR]  exportVmGR                   (innet.cpp:715) */
	CBM_GESUM_GR,             /* f32[numGR]  exportGESumGR                (innet.cpp:730) */
	CBM_GISUM_GR,             /* f32[numGR]  exportGISumGR                (innet.cpp:735) */
	CBM_APBUF_GR,             /* u32[numGR]  exportAPBufGR                (innet.cpp:768) */
	CBM_HIST_GR,              /* u64[numGR]  GR spike history (innetactivitystate.h:79) */
	CBM_THRESH_GR,            /* f32[numGR] */
	CBM_GKCA_GR,              /* f32[numGR] */
	CBM_AP_GO,                /* u8[numGO]   exportAPGO                   (innet.cpp:683) */
	CBM_VM_GO,                /* f32[numGO]  exportVmGO                   (innet.cpp:721) */
	CBM_APBUF_GO,             /* u32[numGO]  exportAPBufGO                (innet.cpp:764) */
	CBM_SUM_GR_INPUT_GO,      /* u32[numGO]  exportSumGRInputGO           (innet.cpp:741) */
	CBM_SUM_GO_INPUT_GO,      /* f32[numGO]  exportSumGOInputGO           (innet.cpp:746) */
	CBM_GO_OUT_SCALE_GOGO,    /* f32[numGO]  exportGOOutSynScaleGOGO      (innet.cpp:751) */
	CBM_AP_SC,                /* u8[numSC]   exportAPSC                   (innet.cpp:679) */
	CBM_VM_SC,                /* f32[numSC]  exportVmSC                   (innet.cpp:725) */
	CBM_APBUF_SC,             /* u32[numSC]  exportAPBufSC                (innet.cpp:773) */
	CBM_HIST_MF,              /* u8[numMF]   exportHistMF                 (innet.cpp:756) */
	CBM_APBUF_MF,             /* u32[numMF]  exportAPBufMF                (innet.cpp:760) */
	CBM_AP_BC,                /* u8[numBC]   MZoneInterface::exportAPBC   (mzone.cpp:743) */
	CBM_VM_BC,                /* f32[numBC]  exportVmBC                   (mzone.cpp:756) */
	CBM_APBUF_BC,             /* u32[numBC]  exportAPBufBC                (mzone.cpp:773) */
	CBM_AP_PC,                /* u8[numPC]   exportAPPC                   (mzone.cpp:747) */
	CBM_VM_PC,                /* f32[numPC]  exportVmPC                   (mzone.cpp:760) */
	CBM_APBUF_PC,             /* u32[numPC]  exportAPBufPC                (mzone.cpp:777) */
	CBM_AP_IO,                /* u8[numIO]   exportAPIO                   (mzone.cpp:751) */
	CBM_VM_IO,                /* f32[numIO]  exportVmIO                   (mzone.cpp:768) */
	CBM_APBUF_IO,             /* u32[numIO]  exportAPBufIO                (mzone.cpp:781) */
	CBM_AP_NC,                /* u8[numNC]   exportAPNC                   (mzone.cpp:739) */
	CBM_VM_NC,                /* f32[numNC]  exportVmNC                   (mzone.cpp:764) */
	CBM_APBUF_NC,             /* u32[numNC]  exportAPBufNC                (mzone.cpp:785) */
	CBM_PFPC_WEIGHT,          /* f32[numGR]  PF->PC weights, PC-major (mzone.cpp:97-103) */
	CBM_MFNC_WEIGHT,          /* f32[numNC*numMF/numNC] MF->NC weights (mzoneactivitystate.h:93) */
	CBM_FIELD_COUNT
};

typedef struct cbm_state cbm_state;
typedef struct cbm_sim cbm_sim;

/* Message of the last failed call on this thread ("" if none). */
const char *cbm_last_error(void);

/* ------------------------------------------------------------- CBMState */
/* CBMState(fstream&): read a state file in the reference's format
 * (cbmstate.cpp:12-33).  Fields the reference's loader leaves undefined are
 * defined here: pPCfromPCtoBC is rebuilt with connectPCtoBC's formula
 * (mzoneconnectivitystate.cpp:242-257, the file holds pBCfromPCtoBC twice,
 * :150) and the unsaved microzone scalars start from the stored histogram
 * (histPCPopActSum) and zero. */
int cbm_state_load(const char *path, cbm_state **out);

/* CBMState(fstream&) on a stream positioned mid-file: reads one state from
 * the len bytes at data (the stream's content from its position on) and sets
 * *consumed (if not NULL) to the bytes the state took, so that a caller can
 * position the stream after it, where the eyelid driver's session file keeps
 * its trial data (ECManagementDelay(fstream&), Eyelid_Sim_CBM_Dev/src/
 * ectrial/ecmanagementdelay.cpp:26-50).  Same interface as cbm_state_load
 * otherwise (cbmstate.cpp:12-33). */
int cbm_state_load_mem(const void *data, uint64_t len, uint64_t *consumed, cbm_state **out);

/* A new network from the texts of a connectivity-parameter file and an
 * activity-parameter file (the two fstreams of CBMState(actPF, conPF,
 * nZones, ...), cbmstate.cpp:60-64 / 176-204).  Activity state takes the
 * reference's initial values and the microzone wiring its formulas
 * (mzoneconnectivitystate.cpp:213-417); wiringSeeds (one per zone, may be
 * NULL) seed the random part of the PC->NC wiring.  Input-net connectivity is
 * left "unconnected" for the caller to fill through cbm_state_array. */
int cbm_state_new(const char *conParamsText, const char *actParamsText, unsigned nZones,
		const int *wiringSeeds, cbm_state **out);

/* CBMState(actPF, conPF, nZones, innetCRSeed, mzoneCRSeed, mzoneARSeed)
 * (cbmstate.cpp:60-64, 176-204) from the parameter texts: the network with
 * the reference's own generator, i.e. the spatial glomerulus-mediated
 * input-net wiring and GR delays (innetconnectivitystate.cpp:12-44,
 * 716-1123), the microzone wiring with its random PC->NC synapses
 * (mzoneconnectivitystate.cpp:12-40, 187-417) and the initial activity, all
 * drawn from the reference's random generator (SFMT, as CRandomSFMT0) seeded
 * as the reference seeds it.  seeds: 1 + 2 nZones values (innetCRSeed, then
 * mzoneCRSeed[nZones], then mzoneARSeed[nZones], which the reference does
 * not use), or NULL to draw them from the wall clock as CBMState(actPF,
 * conPF, nZones) does (cbmstate.cpp:35-57).  The state file equals the
 * reference's for the same parameters and seeds. */
int cbm_state_generate(const char *conParamsText, const char *actParamsText, unsigned nZones, const int *seeds,
		cbm_state **out);

/* CBMState::writeState (cbmstate.cpp:86-103), byte-compatible with the
 * reference.  Like the reference it resets the two GO->GO depression arrays
 * of the state it writes (innetactivitystate.cpp:247-248). */
int cbm_state_save(cbm_state *s, const char *path);

/* CBMState::writeState(fstream&) into memory, for a caller that writes the
 * state into an open stream followed by other data (ECManagementDelay::
 * writeDataToFile, ecmanagementdelay.cpp:275-290): *size receives the bytes
 * the state occupies; with dst == NULL nothing else happens, otherwise the
 * state is written to dst (cap bytes, at least *size, or CBM_ERR_ARG) and the
 * GO->GO depression arrays are reset as cbm_state_save does. */
int cbm_state_save_mem(cbm_state *s, void *dst, uint64_t cap, uint64_t *size);
void cbm_state_free(cbm_state *s);
int cbm_state_num_zones(const cbm_state *s, unsigned *out);

/* Named array of the state (the reference's member names, e.g. "vGR",
 * "pGRfromMFtoGR", "pfSynWeightPC"); zone -1 for input-net arrays.  The
 * pointer stays valid until the state is freed. */
int cbm_state_array(cbm_state *s, const char *name, int zone, void **data, uint64_t *count, int *dtype);

/* Connectivity / activity parameter by the reference's member name
 * (e.g. "numGR", "numpPCfromGRtoPC", "gDecMFtoGR", "tsPerHistBinGR"). */
int cbm_state_con_param(const cbm_state *s, const char *name, uint32_t *value);
int cbm_state_act_param(const cbm_state *s, const char *name, double *value);
/* ActivityParams::setParam (activityparams.cpp:423-434): raw key, re-derive. */
int cbm_state_set_act_param(cbm_state *s, const char *rawKey, float value);
/* The keys of the parameter file as read (which: 0 connectivity, 1 activity),
 * in the order of the reference's paramMap (a std::map, so sorted), each
 * followed by '\n', NUL-terminated.  *needed gets the bytes the list takes
 * with its NUL; a buffer too small fails with CBM_ERR_ARG.  Backs
 * getParamCopy (connectivityparams.cpp / activityparams.cpp:404-416). */
int cbm_state_param_names(const cbm_state *s, int which, char *buf, uint64_t size, uint64_t *needed);
/* A key of the parameter file as read, before derivation: ActivityParams::
 * getParam (activityparams.cpp:418-421) and the connectivity paramMap. */
int cbm_state_raw_param(const cbm_state *s, int which, const char *name, double *value);

/* ----------------------------------------------------------- CBMSimCore */
/* CBMSimCore(CBMState*, int *mzoneRSeed, gpuIndStart, numGPUP2)
 * (cbmsimcore.cpp:14-17, 337-392).  The whole network lives on `device`.
 * mzoneSeeds (one per zone, may be NULL) key each microzone's NC->IO release
 * draws.  The state is borrowed and must outlive the simulator, as in the
 * reference (ecmanagementbase.cpp destroys the core first). */
int cbm_sim_create(cbm_state *s, const int *mzoneSeeds, int device, cbm_sim **out);

/* As cbm_sim_create with room for mfSteps steps of resident MF input
 * (cbm_sim_load_mf_stream / cbm_sim_run). */
int cbm_sim_create_resident(cbm_state *s, const int *mzoneSeeds, int device, uint64_t mfSteps, cbm_sim **out);

/* CBMSimCore::updateMFInput (cbmsimcore.cpp:312-320): numMF bytes, nonzero
 * = spike; the raw byte value feeds the NC inputs as in mzone.cpp:521.
 * Takes effect for the next cbm_sim_calc_activity. */
int cbm_sim_update_mf(cbm_sim *sim, const uint8_t *mf);

/* CBMSimCore::calcActivity (cbmsimcore.cpp:139-310): one 1 ms step.  Returns
 * once the step is queued on the device; calls without an export in between
 * queue steps back to back.  An AP_NC export after a step of one network
 * returns as soon as that step's NC spikes are final. */
int cbm_sim_calc_activity(cbm_sim *sim);

/* CBMSimCore::updateErrDrive (cbmsimcore.cpp:322-325). */
int cbm_sim_update_err_drive(cbm_sim *sim, unsigned zone, float errDriveRelative);

/* MZoneInterface::setGRPCPlastSteps / resetGRPCPlastSteps (mzone.cpp:726-736) */
int cbm_sim_set_plast_steps(cbm_sim *sim, unsigned zone, float ltdStep, float ltpStep);
int cbm_sim_reset_plast_steps(cbm_sim *sim, unsigned zone);

/* InNetInterface::setGIncGRtoGO / resetGIncGRtoGO (innet.cpp:669-677) */
int cbm_sim_set_ginc_grgo(cbm_sim *sim, float inc);
int cbm_sim_reset_ginc_grgo(cbm_sim *sim);

/* Copy one field (enum cbm_field) into dst; bytes must equal
 * cbm_sim_field_bytes(sim, field).  zone selects the microzone for
 * per-zone fields and is ignored otherwise (pass 0). */
int cbm_sim_export(cbm_sim *sim, int field, unsigned zone, void *dst, uint64_t bytes);
uint64_t cbm_sim_field_bytes(cbm_sim *sim, int field);

/* CBMSimCore::writeToState() (cbmsimcore.cpp:65-73): device state back
 * into the borrowed CBMState. */
int cbm_sim_write_to_state(cbm_sim *sim);

/* CBMSimCore::writeToState(fstream&) (cbmsimcore.cpp:75-80): write back and
 * save; like the reference, the save also resets the live GO->GO depression
 * arrays. */
int cbm_sim_save(cbm_sim *sim, const char *path);

/* CBMSimCore::writeToState(fstream&) (cbmsimcore.cpp:75-80) into memory:
 * *size receives the bytes of the state; with dst == NULL nothing else
 * happens, otherwise the device state is written back and serialised into
 * dst (cap bytes, at least *size, or CBM_ERR_ARG), as cbm_sim_save does. */
int cbm_sim_save_mem(cbm_sim *sim, void *dst, uint64_t cap, uint64_t *size);

int cbm_sim_steps_done(cbm_sim *sim, uint64_t *steps);
/* Words per MF bit row: bit k of word k/32 is MF k (numMF/32 + 1 words). */
int cbm_sim_mf_words(cbm_sim *sim, uint32_t *words);

/* Resident input path: nsteps bit rows, step s's row at bits + s*words,
 * copied into HBM as the input of the next nsteps steps. */
int cbm_sim_load_mf_stream(cbm_sim *sim, const uint32_t *bits, uint64_t nsteps);

/* Run nsteps steps from the resident input as CUDA-graph chunks of
 * graphChunk steps.  On return *gpuMs (if not NULL) holds the device time of
 * the run and *passMs (if not NULL) the mean duration of the GR pass kernel
 * over the last chunk. */
int cbm_sim_run(cbm_sim *sim, uint64_t nsteps, uint32_t graphChunk, float *gpuMs, float *passMs);

/* Device-timeline timer on the simulator's launch stream: events recorded
 * at start and stop; *ms receives the time between them (host gaps
 * included). */
int cbm_sim_timer_start(cbm_sim *sim);
int cbm_sim_timer_stop(cbm_sim *sim, float *ms);

/* ---- Trials driven on the device.
 *
 * The eyelid-conditioning driver of the reference (ECManagementDelay,
 * Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp:175-273) as a device
 * protocol, so that whole trials run without a host call per step:
 *   - MF input from the reference's Poisson regenerating population
 *     (PoissonRegenCells, CBM_TOOLS_LIB_DEV/src/poissonregencells.cpp:49-66)
 *     with background rates, and in CS trials phasic rates in
 *     [csOn, csPhasicOff) and tonic rates in [csPhasicOff, csOff);
 *   - the US as updateErrDrive(0, usErrDrive) at step csOff - 1 of CS trials;
 *   - PF->PC steps (plastLTD, plastLTP) set on zone 0 from csOn + plastOnDelay
 *     and reset at csOff + plastOffDelay of CS trials;
 *   - recording of trials [dataStartTrial, dataStartTrial + numDataTrials):
 *     NC and PC spike counts of zone 0 per bin of binSteps steps over the
 *     window [csOn - preCS, csOff + postCS), and the eyelid integrator
 *     (EyelidIntegrator, CBM_TOOLS_LIB_DEV/src/eyelidintegrator.cpp:50-68)
 *     on zone 0's NC spikes, one value per step of the window.
 * Trial steps are counted from the call: the next step is step 0 of trial 0.
 * The MF draw of fibre i at simulator step t is the counter-based stream of
 * the NC->IO draws keyed by a seed derived from mfSeed, counter (t << 20) | i.
 * While a protocol runs, cbm_sim_update_mf and cbm_sim_load_mf_stream fail. */
typedef struct cbm_eyelid_protocol {
	uint32_t trialSteps;          /* steps per trial (5000) */
	int32_t csOn, csOff;          /* in-trial steps of CS onset and offset (2000, 2500) */
	int32_t csPhasicOff;          /* end of the phasic CS rates (csOn: tonic rates only) */
	uint32_t csStartTrial;        /* first trial with CS and US */
	int32_t plastOnDelay, plastOffDelay;  /* 200, 200 */
	float plastLTD, plastLTP;     /* -0.0005 x LTD/LTP ratio, 0.0005 */
	float usErrDrive;             /* relative error drive of the US (1.0) */
	int32_t mfSeed;               /* seed of the MF generator */
	float mfThreshDecayTau;       /* ms (4) */
	const float *mfFreqBG;        /* Hz, numMF values each, host memory */
	const float *mfFreqCSTonic;
	const float *mfFreqCSPhasic;
	uint32_t dataStartTrial, numDataTrials;
	int32_t preCS, postCS;        /* 500, 500 */
	uint32_t binSteps;            /* 10 */
	float eyeGDecayTau, eyeGInc, eyeGShift, eyeGLeakRaw, eyeMaxAmp;  /* 10.5, 0.012, -0.13, 0.13, 100 */
} cbm_eyelid_protocol;

/* Record kinds of cbm_sim_trial_record. */
enum {
	CBM_REC_NC_PSH = 0,  /* u32 [numDataTrials][bins][numNC] */
	CBM_REC_PC_PSH = 1,  /* u32 [numDataTrials][bins][numPC] */
	CBM_REC_EYELID = 2,  /* f32 [numDataTrials][window steps] */
	CBM_REC_GR_PSH = 3,  /* u16 [bins][numGR], summed over the kept trials (cbm_sim_record_gr) */
	/* The eyelid driver's ECTrialsData records (cbm_sim_record_trial_data).
	 * Histograms: f32 [bins][cells] summed over the kept trials, as
	 * PeriStimHistFloat holds them. */
	CBM_REC_PSH_GO = 4,             /* GO spikes */
	CBM_REC_PSH_GR_INPUT_GO = 5,    /* GR->GO input counts (exportSumGRInputGO) */
	CBM_REC_PSH_GO_INPUT_GO = 6,    /* GO->GO input (exportSumGOInputGO) */
	CBM_REC_PSH_GO_OUT_SCALE = 7,   /* GO->GO output scale (exportGOOutSynScaleGOGO) */
	CBM_REC_PSH_MF = 8,             /* MF spikes */
	CBM_REC_PSH_SC = 9,
	CBM_REC_PSH_BC = 10,            /* zone 0 */
	CBM_REC_PSH_PC = 11,            /* zone 0 */
	CBM_REC_PSH_IO = 12,            /* zone 0 */
	/* Rasters: u32 [numDataTrials][window steps / 32][cells], the cells' apBuf
	 * words at every 32nd window step after the first, as SpikeRasterBitArray
	 * holds them: rows are counted over all updates, so when the window is a
	 * multiple of 32 steps its rows drift across trials as the reference's
	 * do; rows no update reached stay zero. */
	CBM_REC_RASTER_GO = 13,
	CBM_REC_RASTER_SC = 14,
	CBM_REC_RASTER_BC = 15,         /* zone 0 */
	CBM_REC_RASTER_PC = 16,         /* zone 0 */
	CBM_REC_RASTER_NC = 17,         /* zone 0 */
	CBM_REC_RASTER_IO = 18          /* zone 0 */
};

/* Start a device protocol on network 0 of the simulator (no counterpart in
 * the reference's core library: it replaces the eyelid driver's per-step calls). */
int cbm_sim_set_eyelid_protocol(cbm_sim *sim, const cbm_eyelid_protocol *protocol);
/* State-variable MF input on the device: the mossy fibres of network 0 code
 * the state of an environment (the cart-pole driver's MF input,
 * Matthew_Sim_CBM/includes/statevariable.hpp:108-129 with the fibre
 * assignment of :35-43 and the rates of environment.cpp:19-39) and fire as
 * the reference's regenerating Poisson cells (poissonregencells.cpp:49-66),
 * all generated on the device from the next step on.  Fibre i codes
 * variable v = i / fibresPerVar (fibres past numVars * fibresPerVar stay at
 * their relaxed rate) at
 *   x = clamp(value of v, lo, hi), d = x - mean[i] (float),
 *   a = (float)(exp((double)(-(d*d) / den)) / norm) / maxPossible,
 *   rate = a * excited[i] + (1 - a) * relaxed[i]    (float),
 * gaussMFAct's arithmetic, with the C library's double exp.  The values of
 * the environment's state come from `values`, one row of numVars floats per
 * step, used cyclically; the fibres' draws are keyed as the eyelid
 * protocol's (mfSeed).  No CS, US, plasticity window or trial records: the
 * setters keep their values.  No counterpart in the reference's core
 * library (it replaces the driver's per-step MF update). */
typedef struct cbm_statevar_input {
	uint32_t numVars, fibresPerVar;
	float lo, hi;                 /* range of every variable */
	float den;                    /* 2 width^2, width = gaussWidth x the fibres' spacing */
	double norm;                  /* sqrt(2 pi width^2) */
	float maxPossible;            /* (float)(1 / norm) */
	const float *mean;            /* numMF preferred values, host memory */
	const float *relaxed, *excited;  /* numMF Hz each, host memory */
	const float *values;          /* [numSteps][numVars], host memory */
	uint64_t numSteps;
	int32_t mfSeed;
	float mfThreshDecayTau;       /* ms (4) */
} cbm_statevar_input;
int cbm_sim_set_statevar_input(cbm_sim *sim, const cbm_statevar_input *input);
/* The MF rates (Hz, numMF floats into out) the running state-variable
 * input gives for row `step` of its values, computed on the device by the
 * same function the generator uses.  No counterpart in the reference. */
int cbm_sim_statevar_rates(cbm_sim *sim, uint64_t step, float *out);

/* Size in bytes of a record of the running protocol (0 without one). */
uint64_t cbm_sim_trial_record_bytes(cbm_sim *sim, int kind);
/* Copy a record of the running protocol to host memory. */
int cbm_sim_trial_record(cbm_sim *sim, int kind, void *dst, uint64_t bytes);
/* Record the running protocol's GR peri-stimulus histogram on the device from
 * the next step on: in the recording window of every kept trial, each GR's
 * spike adds to its count in the step's bin, all kept trials into one
 * histogram.  Replaces the eyelid driver's per-step exportAPGR into
 * ECTrialsData::updatePSH("gr") (Eyelid_Sim_CBM_Dev/src/ectrial/
 * ecmanagementdelay.cpp:259-262, CBM_DATA_LIB_DEV/src/peristimhist/
 * peristimhistfloat.cpp update), whose float counts these u16 counts equal.
 * Needs a protocol, and binSteps x numDataTrials of at most 65535; the
 * counts start at zero. */
int cbm_sim_record_gr(cbm_sim *sim);
/* Record the running protocol's ECTrialsData histograms and rasters
 * (CBM_REC_PSH_* and CBM_REC_RASTER_*) on the device from the next step on,
 * as the eyelid driver fills them after each step of the window of a kept
 * trial (Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp:240-265,
 * CBM_DATA_LIB_DEV/src/interfaces/ectrialsdata.cpp): one small kernel after
 * each step instead of the per-step exports and host loops.  Needs a
 * protocol whose window is at least 32 steps; the records start at zero. */
int cbm_sim_record_trial_data(cbm_sim *sim);

/* ---- Batched instances (no counterpart in the reference, which runs one
 * network per CBMSimCore).  n independent networks of any sizes, seeds and
 * parameters advance together: every step is one GR-pass launch over all of
 * them and one small-cell launch with two CTAs per network, replayed as CUDA
 * graphs.  Each instance is driven by a device protocol
 * (cbm_batch_set_eyelid_protocol); the states must outlive the batch. */
typedef struct cbm_batch cbm_batch;

/* mzoneSeeds: n x (that state's zone count) seeds, or NULL (1000 + zone). */
int cbm_batch_create(cbm_state *const *states, unsigned n, const int *mzoneSeeds, int device, cbm_batch **out);
void cbm_batch_destroy(cbm_batch *b);
int cbm_batch_set_eyelid_protocol(cbm_batch *b, unsigned instance, const cbm_eyelid_protocol *protocol);
/* Advance every instance nsteps steps (graphs of graphChunk steps); *gpuMs
 * receives the device time (events on the launch stream), may be NULL. */
int cbm_batch_run(cbm_batch *b, uint64_t nsteps, uint32_t graphChunk, float *gpuMs);
/* Time every compiled GR-pass geometry that fits all instances on a scratch
 * copy of the batch (the same states and protocols; the batch itself does not
 * advance) over nsteps steps each, and keep the fastest.  *choice receives
 * "kind,W,RW,S,B,M" and *ms its time; either may be NULL. */
int cbm_batch_autotune(cbm_batch *b, uint32_t nsteps, char *choice, size_t choiceLen, float *ms);
/* cbm_sim_pass_geometry for a batch's one GR-pass launch.  No counterpart in
 * the reference. */
int cbm_batch_pass_geometry(cbm_batch *b, unsigned *kind, unsigned *consumerWarps, unsigned *rowsPerStage,
		unsigned *stages);
uint64_t cbm_batch_trial_record_bytes(cbm_batch *b, unsigned instance, int kind);
int cbm_batch_trial_record(cbm_batch *b, unsigned instance, int kind, void *dst, uint64_t bytes);
/* Record instance i's ECTrialsData (as cbm_sim_record_trial_data, from the
 * next step on; its protocol must be set).  One kernel after each step
 * records every instance that does; read with cbm_batch_trial_record
 * (CBM_REC_PSH_* / CBM_REC_RASTER_*). */
int cbm_batch_record_trial_data(cbm_batch *b, unsigned instance);
/* Write instance i's device state into its cbm_state (writeToState). */
int cbm_batch_write_to_state(cbm_batch *b, unsigned instance);
/* Total GR of the instances (GR updates per batch step). */
uint64_t cbm_batch_num_gr(cbm_batch *b);

/* Measurement helper, no counterpart in the reference: nsteps steps with
 * resident MF input, each launched alone after a write of a flushBytes
 * device buffer (an L2 flush when larger than the L2 cache); *stepMs is the
 * summed device time of the steps alone (events on the launch stream around
 * each step). */
int cbm_sim_run_flushed(cbm_sim *sim, uint64_t nsteps, uint64_t flushBytes, float *stepMs);
/* Measurement helper: nsteps flushed steps as cbm_sim_run_flushed, with the
 * two step kernels on separate streams and events around each; *passMs and
 * *tailMs are the mean GR-pass and small-cell kernel durations. */
int cbm_sim_run_flushed_kernels(cbm_sim *sim, uint64_t nsteps, uint64_t flushBytes, float *passMs, float *tailMs);

/* Mean duration of the small-cell update kernel over the last chunk of the
 * last cbm_sim_run that timed the GR pass (0 before). */
int cbm_sim_last_tail_ms(cbm_sim *sim, float *ms);

/* Algorithmic HBM bytes of one step: (72 + 4 n_mf + 4 n_go + 8 n_out) per GR
 * with the network's mean synapse counts. */
double cbm_sim_algorithmic_bytes_per_step(cbm_sim *sim);

/* Bytes the GR pass moves per step with this library's layout (16-bit
 * synapse indices, 8-bit delays, packed GR->GO targets): reads and writes of
 * the GR state, indices, delays and weights, history and weight writes every
 * tsPerHistBinGR steps averaged.  No counterpart in the reference. */
double cbm_sim_layout_bytes_per_step(cbm_sim *sim);

/* Which GR-pass kernel runs: *kind 0 = plain (one warp-row per load), 1 =
 * TMA-pipelined per tile, 2 = TMA-pipelined persistent, 3 = vector pass
 * (four cells per lane, claimed 128-cell units); *consumerWarps,
 * *rowsPerStage, *stages describe the TMA pipeline (0 for the plain kernel).
 * No counterpart in the reference. */
int cbm_sim_pass_geometry(cbm_sim *sim, unsigned *kind, unsigned *consumerWarps, unsigned *rowsPerStage,
		unsigned *stages);

void cbm_sim_destroy(cbm_sim *sim);

/* PF->PC input sums without device allocation.  No counterpart in the
 * reference; it is for callers that cannot let a library allocate device
 * memory while they call it (a framework that owns every allocation through
 * its own pool, a real-time loop that cannot absorb allocation latency).
 * From buffers on the current device it computes, for each of
 * numPC rows of numGR/numPC parallel fibres, the sum of
 * weights[i] * ((apBuf[i] & pfDelayMask[i]) != 0) in the reference's
 * order (updatePFPCOutGPU then sumInputsNew) into sums[numPC], on `stream`
 * (a cudaStream_t, NULL for the default stream).
 * Scratch is one file-scope device array of CBM_NOALLOC_MAX_PARTIALS floats
 * that every device loading the library keeps until exit: numPC times the
 * reduction width (512 for rows of 2048 fibres or more) must fit in it, or
 * the call fails with CBM_ERR_ARG.  All calls on a device share the array;
 * each call rewrites the part it reads, so no clearing is needed, but calls
 * that overlap on the GPU race.  The first call on a device looks up the
 * array's address; make it before any stream capture.  The address is kept;
 * after a reset of the device's context it is looked up again, and the
 * first call after the reset must again precede any capture.  A CUDA error
 * already pending in the calling thread fails the call (CBM_ERR_CUDA) and is
 * left pending. */
#define CBM_NOALLOC_MAX_PARTIALS 65536
int cbm_pfpc_sums_noalloc(const uint32_t *apBuf, const uint32_t *pfDelayMask, const float *weights,
		uint32_t numGR, uint32_t numPC, float *sums, void *stream);

/* Device evaluation of the float exponential the small-cell updates use
 * (the published expf algorithm glibc ships), for checking it against the
 * host's expf: out[i] = exp(in[i]) for n values in host memory. */
int cbm_device_expf(int device, const float *in, float *out, uint64_t n);

/* Device evaluation of the double exponential the GO glutamate update and
 * the state-variable MF coding use (the published exp algorithm glibc
 * ships), for checking it against the host's exp: out[i] = exp(in[i]) for
 * n values in host memory. */
int cbm_device_exp(int device, const double *in, double *out, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif
