// Network generation of the reference's state library: CBMState(actPF,
// conPF, nZones, innetCRSeed, mzoneCRSeed, mzoneARSeed)
// (CBM_STATE_LIB_DEV/src/interfaces/cbmstate.cpp:60-64, 176-204), whose
// input net comes from InNetConnectivityState's spatial generator
// (CBM_STATE_LIB_DEV/src/state/innetconnectivitystate.cpp:12-44, 716-1123)
// and whose PC->NC wiring draws from the microzone's seed
// (mzoneconnectivitystate.cpp:268-345), both with the random generator the
// reference uses, CRandomSFMT0.
//
// That generator is the SIMD-oriented Fast Mersenne Twister of Saito and
// Matsumoto (2006), here with the MEXP 11213 parameter set the reference's
// copy is compiled with, and the integer and float conversions of Agner
// Fog's randomc wrapper (BRandom, IRandom, IRandomX, Random; no
// Mother-of-All combination).  It is written out here in plain integer
// arithmetic: a 128-bit word is two 64-bit halves.
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <functional>
#include <utility>

#include "cbm_state.hpp"

namespace cbm {

namespace {

class Sfmt {
public:
	explicit Sfmt(int seed)
	{
		uint32_t y = (uint32_t)seed;
		w_[0] = y;
		for (uint32_t i = 1; i < 4 * kN; i++) {
			y = 1812433253u * (y ^ (y >> 30)) + i;
			w_[i] = y;
		}
		certifyPeriod();
		generate();
	}

	uint32_t bits()
	{
		if (ix_ >= 4 * kN) generate();
		return w_[ix_++];
	}

	// integer in [min, max] from the top bits of bits() * interval
	int irandom(int min, int max)
	{
		if (max <= min) return max == min ? min : (int)0x80000000;
		const uint32_t interval = (uint32_t)(max - min + 1);
		return (int32_t)(uint32_t)(((uint64_t)bits() * interval) >> 32) + min;
	}

	// the same with rejection of the incomplete last interval
	int irandomx(int min, int max)
	{
		if (max <= min) return max == min ? min : (int)0x80000000;
		const uint32_t interval = (uint32_t)(max - min + 1);
		if (interval != lastInterval_) {
			rLimit_ = (uint32_t)((1ull << 32) / interval) * interval - 1;
			lastInterval_ = interval;
		}
		uint64_t v;
		do v = (uint64_t)bits() * interval;
		while ((uint32_t)v > rLimit_);
		return (int32_t)(uint32_t)(v >> 32) + min;
	}

	// double in [0, 1) from 52 bits of two consecutive words
	double random()
	{
		if (ix_ >= 4 * kN - 1) generate();
		const uint64_t r = (uint64_t)w_[ix_] | ((uint64_t)w_[ix_ + 1] << 32);
		ix_ += 2;
		return (double)(int64_t)(r >> 12) * (1.0 / (67108864.0 * 67108864.0));
	}

private:
	// MEXP 11213: 88 128-bit words, feedback at 68, shifts and masks of the
	// published parameter set
	static constexpr uint32_t kN = 88, kM = 68, kSL1 = 14, kSL2 = 3, kSR1 = 7, kSR2 = 3;
	static constexpr uint32_t kMask[4] = {0xeffff7fbu, 0xffffffefu, 0xdfdfbfffu, 0x7fffdbfdu};
	static constexpr uint32_t kParity[4] = {0x00000001u, 0x00000000u, 0xe8148000u, 0xd0c7afa3u};

	uint32_t w_[4 * kN];
	uint32_t ix_ = 0, lastInterval_ = 0, rLimit_ = 0;

	void certifyPeriod()
	{
		uint32_t t = 0;
		for (int i = 0; i < 4; i++) t ^= kParity[i] & w_[i];
		for (int s = 16; s > 0; s >>= 1) t ^= t >> s;
		if (t & 1) return;
		// flip the lowest set bit of the first non-zero parity word
		for (int i = 0; i < 4; i++)
			if (kParity[i]) {
				w_[i] ^= kParity[i] & (~kParity[i] + 1);
				return;
			}
	}

	struct W128 { uint64_t lo, hi; };
	W128 get(uint32_t i) const
	{
		return {(uint64_t)w_[4 * i] | ((uint64_t)w_[4 * i + 1] << 32), (uint64_t)w_[4 * i + 2] | ((uint64_t)w_[4 * i + 3] << 32)};
	}
	void put(uint32_t i, W128 v)
	{
		w_[4 * i] = (uint32_t)v.lo; w_[4 * i + 1] = (uint32_t)(v.lo >> 32);
		w_[4 * i + 2] = (uint32_t)v.hi; w_[4 * i + 3] = (uint32_t)(v.hi >> 32);
	}
	// one step of the recursion: a ^ (a << 8 SL2 bits) ^ ((b >> SR1 per
	// 32-bit lane) & mask) ^ (c >> 8 SR2 bits) ^ (d << SL1 per lane)
	static W128 recursion(W128 a, W128 b, W128 c, W128 d)
	{
		const uint32_t sa = 8 * kSL2, sc = 8 * kSR2;
		W128 a1 = {a.lo << sa, (a.hi << sa) | (a.lo >> (64 - sa))};
		W128 c1 = {(c.lo >> sc) | (c.hi << (64 - sc)), c.hi >> sc};
		auto lanes = [](uint64_t x, int sh, bool left, uint32_t m0, uint32_t m1) {
			uint32_t l = (uint32_t)x, h = (uint32_t)(x >> 32);
			l = left ? l << sh : l >> sh;
			h = left ? h << sh : h >> sh;
			return (uint64_t)(l & m0) | ((uint64_t)(h & m1) << 32);
		};
		W128 b1 = {lanes(b.lo, kSR1, false, kMask[0], kMask[1]), lanes(b.hi, kSR1, false, kMask[2], kMask[3])};
		W128 d1 = {lanes(d.lo, kSL1, true, ~0u, ~0u), lanes(d.hi, kSL1, true, ~0u, ~0u)};
		return {a.lo ^ a1.lo ^ c1.lo ^ b1.lo ^ d1.lo, a.hi ^ a1.hi ^ c1.hi ^ b1.hi ^ d1.hi};
	}
	void generate()
	{
		W128 r1 = get(kN - 2), r2 = get(kN - 1);
		for (uint32_t i = 0; i < kN; i++) {
			const W128 r = recursion(get(i), get(i < kN - kM ? i + kM : i + kM - kN), r1, r2);
			put(i, r);
			r1 = r2;
			r2 = r;
		}
		ix_ = 0;
	}
};
constexpr uint32_t Sfmt::kMask[4];
constexpr uint32_t Sfmt::kParity[4];

// A 2-D table of the state: row r of `cols` entries.
struct Table {
	uint32_t *p;
	size_t cols;
	uint32_t *operator[](size_t r) { return p + r * cols; }
};

Table table(State &s, const char *name, size_t rows)
{
	NamedArray *a = s.find(name);
	return {a->as<uint32_t>(), a->count / rows};
}
int32_t *counts(State &s, const char *name) { return s.find(name)->as<int32_t>(); }

// connectCommon (innetconnectivitystate.cpp:964-1083): for each of the
// source's srcMaxNumCon slots, every source cell in random order connects to
// a destination cell near its scaled grid position (spread by the span),
// within the destination's normal connection count for the first
// normAttempts tries and its maximum after that.
void connectCommon(Table src, int32_t *srcNum, Table dst, int32_t *dstNum, uint32_t srcMaxNumCon,
		uint32_t numSrcCells, uint32_t dstMaxNumCon, uint32_t dstNormNumCon, uint32_t srcGridX, uint32_t srcGridY,
		uint32_t dstGridX, uint32_t dstGridY, uint32_t spanX, uint32_t spanY, uint32_t normAttempts,
		uint32_t maxAttempts, bool needUnique, Sfmt &rng)
{
	const float scaleX = (float)srcGridX / (float)dstGridX;
	(void)srcGridY;
	std::vector<uint8_t> done(numSrcCells);
	for (uint32_t i = 0; i < srcMaxNumCon; i++) {
		std::fill(done.begin(), done.end(), 0);
		uint32_t nDone = 0;
		while (nDone < numSrcCells) {
			const int srcInd = rng.irandom(0, (int)numSrcCells - 1);
			if (done[srcInd]) continue;
			done[srcInd] = 1;
			nDone++;
			const int srcPosX = (int)((uint32_t)srcInd % srcGridX), srcPosY = (int)((uint32_t)srcInd / srcGridX);
			int lim = (int)dstNormNumCon;
			for (uint32_t att = 0; att < maxAttempts; att++) {
				if (att == normAttempts) lim = (int)dstMaxNumCon;
				// both coordinates are scaled by the x ratio, as in the reference
				int x = (int)std::round((float)srcPosX / scaleX);
				int y = (int)std::round((float)srcPosY / scaleX);
				x = (int)(x + std::round((rng.random() - 0.5) * spanX));
				y = (int)(y + std::round((rng.random() - 0.5) * spanY));
				x = (int)(((uint32_t)x % dstGridX + dstGridX) % dstGridX);
				y = (int)(((uint32_t)y % dstGridY + dstGridY) % dstGridY);
				const uint32_t d = (uint32_t)y * dstGridX + (uint32_t)x;
				if (needUnique) {
					bool unique = true;
					for (uint32_t j = 0; j < i; j++)
						if (d == src[srcInd][j]) { unique = false; break; }
					if (!unique) continue;
				}
				if (dstNum[d] < lim) {
					dst[d][dstNum[d]] = (uint32_t)srcInd;
					dstNum[d]++;
					src[srcInd][i] = d;
					srcNum[srcInd]++;
					break;
				}
			}
		}
	}
}

// translateCommon (innetconnectivitystate.cpp:1085-1123): connections
// through the glomeruli, pre -> GL -> post, listed on both sides.
void translateCommon(Table preGL, const int32_t *preGLNum, Table glPost, const int32_t *glPostNum, Table pre,
		int32_t *preNum, Table post, int32_t *postNum, uint32_t numPre)
{
	for (uint32_t i = 0; i < numPre; i++) {
		preNum[i] = 0;
		for (int j = 0; j < preGLNum[i]; j++) {
			const uint32_t gl = preGL[i][j];
			for (int k = 0; k < glPostNum[gl]; k++) {
				const uint32_t p = glPost[gl][k];
				pre[i][preNum[i]] = p;
				preNum[i]++;
				post[p][postNum[p]] = i;
				postNum[p]++;
			}
		}
	}
}

}  // namespace

void wirePCtoNC(State &s, uint32_t z, const std::function<uint32_t()> &drawPC);

std::string State::generate(const std::string &conText, const std::string &actText, uint32_t nZones, int innetSeed,
		const std::vector<int> &mzoneConSeeds)
{
	std::string err = create(conText, actText, nZones, mzoneConSeeds);
	if (!err.empty()) return err;
	if (mzoneConSeeds.size() < nZones) return "one connectivity seed per microzone is needed";
	// the microzones' PC->NC wiring with IRandomX draws of the zone's seed
	for (uint32_t z = 0; z < nZones; z++) {
		Sfmt rng(mzoneConSeeds[z]);
		const int numPC = (int)cp.numPC;
		wirePCtoNC(*this, z, [&]() { return (uint32_t)rng.irandomx(0, numPC - 1); });
	}
	// the reference's initializeVals sets three tables to "unconnected" over
	// a count that is not their allocated size (innetconnectivitystate.cpp:
	// 661, 703, 712): pGLfromGLtoGR over numGL x maxnumpGLfromGOtoGL entries,
	// pGRfromGLtoGR over numGR x maxnumpGRfromGLtoGR and pGRfromMFtoGR over
	// numGR x maxnumpGRfromMFtoGR; entries past that keep the zeros of a
	// fresh allocation
	for (auto tb : {std::make_pair("pGLfromGLtoGR", (size_t)cp.numGL * cp.maxnumpGLfromGOtoGL),
			std::make_pair("pGRfromGLtoGR", (size_t)cp.numGR * cp.maxnumpGRfromGLtoGR),
			std::make_pair("pGRfromMFtoGR", (size_t)cp.numGR * cp.maxnumpGRfromMFtoGR)}) {
		NamedArray *a = find(tb.first);
		uint32_t *p = a->as<uint32_t>();
		for (size_t i = tb.second; i < a->count; i++) p[i] = 0;
	}
	auto rawU = [&](const char *k) { return cp.raw.count(k) ? cp.raw.at(k) : 0u; };
	Sfmt rng(innetSeed);
	const uint32_t GL = cp.numGL, GR = cp.numGR, GO = cp.numGO, MF = cp.numMF;
	// connectGRGL
	connectCommon(table(*this, "pGRfromGLtoGR", GR), counts(*this, "numpGRfromGLtoGR"), table(*this, "pGLfromGLtoGR", GL),
			counts(*this, "numpGLfromGLtoGR"), cp.maxnumpGRfromGLtoGR, GR, cp.maxnumpGLfromGLtoGR,
			cp.lownumpGLfromGLtoGR, cp.grX, cp.grY, cp.glX, cp.glY, rawU("spanGRDenOnGLX"), rawU("spanGRDenOnGLY"),
			20000, 50000, true, rng);
	// connectGOGL: GO dendrites, then GO axons
	connectCommon(table(*this, "pGOfromGLtoGO", GO), counts(*this, "numpGOfromGLtoGO"), table(*this, "pGLfromGLtoGO", GL),
			counts(*this, "numpGLfromGLtoGO"), cp.maxnumpGOfromGLtoGO, GO, cp.maxnumpGLfromGLtoGO,
			cp.maxnumpGLfromGLtoGO, cp.goX, cp.goY, cp.glX, cp.glY, rawU("spanGODecDenOnGLX"),
			rawU("spanGODecDenOnGLY"), 20000, 50000, false, rng);
	connectCommon(table(*this, "pGOfromGOtoGL", GO), counts(*this, "numpGOfromGOtoGL"), table(*this, "pGLfromGOtoGL", GL),
			counts(*this, "numpGLfromGOtoGL"), cp.maxnumpGOfromGOtoGL, GO, cp.maxnumpGLfromGOtoGL,
			cp.maxnumpGLfromGOtoGL, cp.goX, cp.goY, cp.glX, cp.glY, rawU("spanGOAxonOnGLX"),
			rawU("spanGOAxonOnGLY"), 20000, 50000, false, rng);
	// connectMFGL (innetconnectivitystate.cpp:755-796): every fibre but the
	// last takes numpMFfromMFtoGL free glomeruli at random, the last fibre
	// the glomeruli left over
	{
		uint8_t *has = find("haspGLfromMFtoGL")->as<uint8_t>();
		uint32_t *glMF = find("pGLfromMFtoGL")->as<uint32_t>();
		Table mfGL = table(*this, "pMFfromMFtoGL", MF);
		int32_t *mfGLNum = counts(*this, "numpMFfromMFtoGL");
		for (uint32_t i = 0; i + 1 < MF; i++)
			for (uint32_t j = 0; j < cp.numpMFfromMFtoGL; j++)
				for (;;) {
					const int g = rng.irandom(0, (int)GL - 1);
					if (!has[g]) {
						glMF[g] = i;
						has[g] = 1;
						mfGL[i][j] = (uint32_t)g;
						mfGLNum[i]++;
						break;
					}
				}
		uint32_t last = 0;
		for (uint32_t g = 0; g < GL; g++)
			if (!has[g]) {
				has[g] = 1;
				glMF[g] = MF - 1;
				mfGL[MF - 1][last++] = g;
			}
	}
	// translateMFGL, translateGOGL
	translateCommon(table(*this, "pMFfromMFtoGL", MF), counts(*this, "numpMFfromMFtoGL"), table(*this, "pGLfromGLtoGR", GL),
			counts(*this, "numpGLfromGLtoGR"), table(*this, "pMFfromMFtoGR", MF), counts(*this, "numpMFfromMFtoGR"),
			table(*this, "pGRfromMFtoGR", GR), counts(*this, "numpGRfromMFtoGR"), MF);
	translateCommon(table(*this, "pMFfromMFtoGL", MF), counts(*this, "numpMFfromMFtoGL"), table(*this, "pGLfromGLtoGO", GL),
			counts(*this, "numpGLfromGLtoGO"), table(*this, "pMFfromMFtoGO", MF), counts(*this, "numpMFfromMFtoGO"),
			table(*this, "pGOfromMFtoGO", GO), counts(*this, "numpGOfromMFtoGO"), MF);
	translateCommon(table(*this, "pGOfromGOtoGL", GO), counts(*this, "numpGOfromGOtoGL"), table(*this, "pGLfromGLtoGR", GL),
			counts(*this, "numpGLfromGLtoGR"), table(*this, "pGOfromGOtoGR", GO), counts(*this, "numpGOfromGOtoGR"),
			table(*this, "pGRfromGOtoGR", GR), counts(*this, "numpGRfromGOtoGR"), GO);
	// connectGRGO
	connectCommon(table(*this, "pGOfromGRtoGO", GO), counts(*this, "numpGOfromGRtoGO"), table(*this, "pGRfromGRtoGO", GR),
			counts(*this, "numpGRfromGRtoGO"), cp.maxnumpGOfromGRtoGO, GO, cp.maxnumpGRfromGRtoGO,
			cp.maxnumpGRfromGRtoGO, cp.goX, cp.goY, cp.grX, cp.grY, rawU("spanGOAscDenOnGRX"),
			rawU("spanGOAscDenOnGRY"), 20000, 50000, false, rng);
	// connectGOGO (innetconnectivitystate.cpp:852-918): each GO's local
	// matrix entries (dx, dy, probability), GABA then coupling
	{
		auto gogo = [&](const std::vector<float> &m, uint32_t nOut, const char *outN, const char *outC,
				const char *inN, const char *inC, uint32_t i) {
			Table out = table(*this, outN, GO), in = table(*this, inN, GO);
			int32_t *outNum = counts(*this, outC), *inNum = counts(*this, inC);
			const int cx = (int)(i % cp.goX), cy = (int)(i / cp.goX);
			for (uint32_t j = 0; j < nOut; j++) {
				if (rng.random() >= (1 - m[3 * j + 2])) {
					int x = (int)(cx + m[3 * j]);
					x = (int)(((uint32_t)x % cp.goX + cp.goX) % cp.goX);
					int y = (int)(cy + m[3 * j + 1]);
					y = (int)(((uint32_t)y % cp.goY + cp.goY) % cp.goY);
					const uint32_t d = cp.goX * (uint32_t)y + (uint32_t)x;
					out[i][outNum[i]] = d;
					outNum[i]++;
					in[d][inNum[d]] = i;
					inNum[d]++;
				}
			}
		};
		for (uint32_t i = 0; i < GO; i++) {
			gogo(cp.gogoGABALocalCon, cp.maxnumpGOGABAOutGOGO, "pGOGABAOutGOGO", "numpGOGABAOutGOGO",
					"pGOGABAInGOGO", "numpGOGABAInGOGO", i);
			gogo(cp.gogoCoupLocalCon, cp.maxnumpGOCoupOutGOGO, "pGOCoupOutGOGO", "numpGOCoupOutGOGO",
					"pGOCoupInGOGO", "numpGOCoupInGOGO", i);
		}
	}
	// assignGRDelays (innetconnectivitystate.cpp:920-962), with the
	// activity parameters' time step as an integer
	{
		const uint32_t msPerStep = (uint32_t)ap.msPerTimeStep;
		uint32_t *bsp = find("pGRDelayMaskfromGRtoBSP")->as<uint32_t>();
		Table out = table(*this, "pGRfromGRtoGO", GR), mask = table(*this, "pGRDelayMaskfromGRtoGO", GR);
		const int32_t *outNum = counts(*this, "numpGRfromGRtoGO");
		for (uint32_t i = 0; i < GR; i++) {
			const int x = (int)(i % cp.grX);
			const int dBSP = std::abs((int)(cp.grX / 2 - (uint32_t)x));
			bsp[i] = 0x1u << (int)(((uint32_t)dBSP / cp.grPFVelInGRXPerTStep + cp.grAFDelayInTStep) / msPerStep);
			for (int j = 0; j < outNum[i]; j++) {
				const int goX = (int)((float)(out[i][j] % cp.goX) * ((float)cp.grX / cp.goX));
				int d = std::abs(goX - x);
				if (d > (int)(cp.grX / 2)) d = goX < x ? goX + (int)cp.grX - x : x + (int)cp.grX - goX;
				mask[i][j] = 0x1u << (int)(((uint32_t)d / cp.grPFVelInGRXPerTStep + cp.grAFDelayInTStep) / msPerStep);
			}
		}
	}
	return "";
}

std::vector<int> clockSeeds(uint32_t nZones)
{
	// CBMState(actPF, conPF, nZones) (cbmstate.cpp:35-57): the seeds drawn
	// from a generator seeded with the wall clock
	Sfmt rng((int)time(nullptr));
	std::vector<int> out;
	out.push_back(rng.irandom(0, INT_MAX));
	for (uint32_t z = 0; z < nZones; z++) {
		out.push_back(rng.irandom(0, INT_MAX));
		out.push_back(rng.irandom(0, INT_MAX));
	}
	return out;
}

}  // namespace cbm
