// Counter-based random stream shared by host and device code.
//
// The reference draws its stochastic NC->IO transmitter release from an SFMT
// generator owned by each microzone (CBM_CORE_LIB_MGPU_DEV/src/mzonemodules/
// mzone.cpp:18, 509).  A sequential generator cannot be evaluated inside a
// data-parallel step, so every random number here is a pure function of
// (seed, stream id, counter): SplitMix64 (Steele, Lea and Flood, OOPSLA 2014,
// finaliser constants as published by Vigna) applied twice, top 24 bits
// scaled into [0,1).  A 24-bit float converts to double exactly, so the
// reference's `double < float` comparison gives the same answer on every side.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CBM_HD __host__ __device__ __forceinline__
#else
#define CBM_HD inline
#endif

namespace cbm {
namespace rng {

constexpr uint32_t kStreamNCIO = 0x4E43494Fu;    // NC->IO release draws
constexpr uint32_t kStreamMF = 0x4D46494Eu;      // mossy-fibre spike draws
constexpr uint32_t kStreamWiring = 0x57495245u;  // network construction

CBM_HD uint64_t splitmix64(uint64_t x)
{
	uint64_t z = x + 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

CBM_HD uint64_t streamKey(uint32_t seed, uint32_t stream)
{
	return splitmix64(((uint64_t)seed << 32) | stream);
}

CBM_HD float uniform24Keyed(uint64_t key, uint64_t counter)
{
	uint64_t h = splitmix64(key ^ counter);
	return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f);
}

CBM_HD float uniform24(uint32_t seed, uint32_t stream, uint64_t counter)
{
	return uniform24Keyed(streamKey(seed, stream), counter);
}

// Counter of the j-th release draw of IO cell i at 1-based step t, numbered
// in the reference's loop order (mzone.cpp:505-511).
CBM_HD uint64_t ncioCounter(uint64_t t, uint32_t i, uint32_t j, uint32_t numNCPerIO)
{
	return (t << 20) | (uint64_t)(i * numNCPerIO + j);
}

}  // namespace rng
}  // namespace cbm
