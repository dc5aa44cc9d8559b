/* Test infrastructure: the CPU oracle for the 1 ms cerebellar network step.
 *
 * This library is the checker that the B200 implementation is compared
 * against.  Only tests, the smoke check and the CPU-baseline leg of the
 * benchmark load it; the product never does.
 *
 * It restates, in plain C and in the reference's operation order, the
 * reference's CBMSimCore::calcActivity (CBM_CORE_LIB_MGPU_DEV/src/interface/
 * cbmsimcore.cpp:139-310) for one GPU with NO_ASYNC ordering, together with
 * the reference's state-file reader/writer (CBM_STATE_LIB_DEV/src/interfaces/
 * cbmstate.cpp:12-33, 86-103) and parameter derivation (CBM_STATE_LIB_DEV/src/
 * params/activityparams.cpp:436-636, connectivityparams.cpp:12-184).
 *
 * It is pinned against the reference's own host code run through
 * oracle/_ref/ref_run on the same inputs (tests/test_oracle_pin.py). */
#ifndef CBM_ORACLE_H
#define CBM_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct cbm_oracle cbm_oracle;

/* Loads a reference-format state file.  Returns NULL on error and writes a
 * message to err (errlen bytes). */
cbm_oracle *cbm_oracle_load(const char *path, char *err, size_t errlen);
void cbm_oracle_free(cbm_oracle *o);

/* CBMState(actPF, conPF, nZones, ...) from parameter text, with the
 * microzone wiring and every initial value but the input-net tables, which
 * stay at their initial values (counts 0, indices UINT_MAX) for the caller
 * to fill through cbm_oracle_array.  pcncSeeds (nZones entries, or NULL)
 * key each zone's random PC->NC synapses.  NULL on error (message in err). */
cbm_oracle *cbm_oracle_new(const char *conText, const char *actText, uint32_t nZones, const int *pcncSeeds,
		char *err, size_t errlen);
/* Address and size of a state array by its reference name (zone < 0: the
 * input net; else that microzone); NULL when there is none. */
void *cbm_oracle_array(cbm_oracle *o, const char *name, int zone, uint64_t *bytes);
/* A derived connectivity parameter by name; 0, or -1 for an unknown name. */
int cbm_oracle_con(const cbm_oracle *o, const char *key, uint32_t *value);

/* Mirror of the reference's CBMSimCore(state, mzoneRSeed, ...) seeds and of
 * its host setters (cbmsimcore.cpp:322, mzone.cpp:726-736, innet.cpp:669-677). */
void cbm_oracle_set_seeds(cbm_oracle *o, const int *mzoneSeeds);
void cbm_oracle_update_err_drive(cbm_oracle *o, unsigned zone, float rel);
void cbm_oracle_set_plast_steps(cbm_oracle *o, unsigned zone, float ltd, float ltp);
void cbm_oracle_reset_plast_steps(cbm_oracle *o, unsigned zone);
void cbm_oracle_set_ginc_grgo(cbm_oracle *o, float inc);
void cbm_oracle_reset_ginc_grgo(cbm_oracle *o);

/* One step: updateMFInput(mf) then calcActivity().  mf has numMF bytes. */
void cbm_oracle_step(cbm_oracle *o, const uint8_t *mf);

/* Runs nsteps steps with mf = nsteps*numMF bytes.  When trace is not NULL it
 * receives one trace record per step (layout as oracle/ref_driver.cpp). */
void cbm_oracle_run(cbm_oracle *o, const uint8_t *mf, uint64_t nsteps, uint8_t *trace);

size_t cbm_oracle_trace_record_bytes(const cbm_oracle *o);
/* writeToState(fstream&) of the reference: returns 0 on success. */
int cbm_oracle_save(cbm_oracle *o, const char *path);

/* out[i] = the host C library's expf(in[i]) (the reference's exp(float)). */
void cbm_oracle_expf_array(const float *in, float *out, uint64_t n);
/* out[i] = the host C library's exp(in[i]) (the reference's exp(double)). */
void cbm_oracle_exp_array(const double *in, double *out, uint64_t n);

/* The eyelid-conditioning driver (ECManagementDelay::calcMFActivity and
 * calcSimActivity, Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp:
 * 175-273) around nsteps steps, starting at trial 0, step 0: MF input from a
 * Poisson regenerating population (PoissonRegenCells, CBM_TOOLS_LIB_DEV/src/
 * poissonregencells.cpp:49-66) whose draw of fibre i at step t is keyed by
 * ((t << 20) | i) under a seed derived from mfSeed, the US error drive, the
 * PF->PC step window, the eyelid integrator (eyelidintegrator.cpp:13-68) and
 * the records of the kept trials (NC / PC counts per bin, integrator output
 * per step of the window).  rates: 3 x numMF floats (background, CS tonic,
 * CS phasic).  Field meanings as cbm_eyelid_protocol in include/cbm_b200.h. */
typedef struct {
	uint32_t trialSteps; int32_t csOn, csOff, csPhasicOff; uint32_t csStartTrial;
	int32_t plastOnDelay, plastOffDelay; float plastLTD, plastLTP, usErrDrive;
	int32_t mfSeed; float mfThreshDecayTau;
	uint32_t dataStartTrial, numDataTrials; int32_t preCS, postCS; uint32_t binSteps;
	float eyeGDecayTau, eyeGInc, eyeGShift, eyeGLeakRaw, eyeMaxAmp;
} cbm_oracle_protocol;

/* Record sizes in elements: *ncPSH, *pcPSH (u32) and *eyelid (f32). */
void cbm_oracle_protocol_sizes(const cbm_oracle *o, const cbm_oracle_protocol *p, uint64_t *ncPSH,
		uint64_t *pcPSH, uint64_t *eyelid);
/* Sizes in elements of the trial-data records (the eyelid driver's
 * ECTrialsData, ecmanagementdelay.cpp:107-156, 236-265): *psh f32 and
 * *raster u32.  psh: the peri-stimulus histograms go, grInputGO, goInputGO,
 * goOutSynScale, mf, sc, bc, pc, io, each f32 [bins][cells] summed over the
 * kept trials; raster: the apBuf words of go, sc, bc, pc, nc, io, each u32
 * [numDataTrials][recLen / 32][cells] (zone 0 for the microzone cells). */
void cbm_oracle_trial_data_sizes(const cbm_oracle *o, const cbm_oracle_protocol *p, uint64_t *psh,
		uint64_t *raster);
/* psh and raster (either may be NULL) receive the trial-data records. */
void cbm_oracle_run_protocol(cbm_oracle *o, const cbm_oracle_protocol *p, const float *rates, uint64_t nsteps,
		uint8_t *trace, uint32_t *ncPSH, uint32_t *pcPSH, float *eyelid, float *psh, uint32_t *raster);

/* The same driver with the MF rates of step s (0-based within the run)
 * taken from row s % rateRows of stepRates ([rateRows][numMF] Hz) instead
 * of the protocol's three tables: the state-variable MF input, whose rates
 * the caller computes from the environment's values (gaussMFAct,
 * Matthew_Sim_CBM/includes/statevariable.hpp:108-129). */
void cbm_oracle_run_protocol_step_rates(cbm_oracle *o, const cbm_oracle_protocol *p, const float *stepRates,
		uint64_t rateRows, uint64_t nsteps, uint8_t *trace, uint32_t *ncPSH, uint32_t *pcPSH, float *eyelid);

/* Sizes, for callers sizing buffers. */
uint32_t cbm_oracle_num(const cbm_oracle *o, const char *what);

#ifdef __cplusplus
}
#endif
#endif
