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

/* Sizes, for callers sizing buffers. */
uint32_t cbm_oracle_num(const cbm_oracle *o, const char *what);

#ifdef __cplusplus
}
#endif
#endif
