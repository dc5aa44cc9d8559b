/* Test infrastructure: CPU copy of the counter-based random stream that both
 * the oracle and the reference harness consume, so that the reference's
 * stochastic NC->IO release (CBM_CORE_LIB_MGPU_DEV/src/mzonemodules/mzone.cpp:509,
 * `randGen->Random() < synIOPReleaseNC`) draws the same numbers on every
 * side.
 *
 * Mixer: SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom
 * number generators", OOPSLA 2014; finaliser constants as published by
 * Vigna).  A draw is keyed by (seed, stream id, counter); its top 24 bits
 * give a float in [0,1) that converts to double exactly. */
#ifndef CBM_ORACLE_STREAM_H
#define CBM_ORACLE_STREAM_H
#include <stdint.h>

#define CBM_STREAM_NCIO 0x4E43494Fu /* "NCIO": NC->IO release draws */
#define CBM_STREAM_MF   0x4D46494Eu /* "MFIN": mossy-fibre Poisson draws */
#define CBM_STREAM_WIRING 0x57495245u /* "WIRE": network construction draws */

static inline uint64_t cbm_oracle_splitmix64(uint64_t x)
{
	uint64_t z = x + 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

/* Uniform float in [0,1) with 24 random bits. */
static inline float cbm_oracle_uniform24(uint32_t seed, uint32_t stream, uint64_t counter)
{
	uint64_t key = cbm_oracle_splitmix64(((uint64_t)seed << 32) | stream);
	uint64_t h = cbm_oracle_splitmix64(key ^ counter);
	return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f);
}

/* Counter of the j-th NC->IO draw of IO cell i at 1-based step t: draws of a
 * step are numbered in the reference's loop order (mzone.cpp:505-511). */
static inline uint64_t cbm_oracle_ncio_counter(uint64_t t, uint32_t i, uint32_t j, uint32_t numNCPerIO)
{
	return (t << 20) | (uint64_t)(i * numNCPerIO + j);
}
#endif
