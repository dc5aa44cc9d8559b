/* Test infrastructure (oracle "run" build only).
 *
 * Replaces the reference's SFMT generator classes (Agner Fog's CRandomSFMT,
 * vendored at CBM_Cart_On_Cart/includes/sfmt.h:213-251) with a counter-based
 * stream so that the reference's stochastic NC->IO release draws
 * (CBM_CORE_LIB_MGPU_DEV/src/mzonemodules/mzone.cpp:509) are the same numbers
 * the B200 implementation draws.  The draw of one object at a step is keyed by
 * (object seed, step, index within the step); the harness sets the step before
 * every calcActivity through cbm_refshim_set_step.  Connectivity generation,
 * which needs the real SFMT sequence, is done by the separate "gen" build. */
#ifndef CBM_REFSHIM_SFMT_H
#define CBM_REFSHIM_SFMT_H
#include <stdint.h>
#include "../../../cbm_stream.h"

extern uint64_t cbm_refshim_step;
void cbm_refshim_set_step(uint64_t t);

class CRandomSFMT {
public:
	CRandomSFMT(int seed, int IncludeMother = 1) : seed_((uint32_t)seed), step_(~0ull), n_(0) { (void)IncludeMother; }
	void RandomInit(int seed) { seed_ = (uint32_t)seed; step_ = ~0ull; n_ = 0; }
	double Random()
	{
		if (step_ != cbm_refshim_step) { step_ = cbm_refshim_step; n_ = 0; }
		uint64_t c = (step_ << 20) | n_;
		n_++;
		return (double)cbm_oracle_uniform24(seed_, CBM_STREAM_NCIO, c);
	}
	uint32_t BRandom() { return (uint32_t)(Random() * 4294967296.0); }
	// interval max - min + 1 in 64 bits (SFMT's IRandom takes it as an unsigned 32-bit count)
	int IRandom(int min, int max) { return min + (int)(Random() * (double)((int64_t)max - min + 1)); }
	int IRandomX(int min, int max) { return IRandom(min, max); }
private:
	uint32_t seed_;
	uint64_t step_;
	uint64_t n_;
};

class CRandomSFMT0 : public CRandomSFMT {
public:
	CRandomSFMT0(int seed) : CRandomSFMT(seed, 0) {}
};

class CRandomSFMT1 : public CRandomSFMT {
public:
	CRandomSFMT1(int seed) : CRandomSFMT(seed, 1) {}
};
#endif
