/* Test infrastructure: the reference's state-variable MF rate coding
 * (StateVariable, Matthew_Sim_CBM/includes/statevariable.hpp, compiled from
 * the reference tree), set up as Environment::setupStateVariables does
 * (Matthew_Sim_CBM/src/environments/environment.cpp:42-58: ordered fibre
 * assignment from an unassigned list built from the last fibre down) with
 * Gaussian updates (initializeGaussian, gaussMFAct).
 *
 * usage: ref_statevar NUMMF NVARS MIN MAX GAUSSWIDTH RELAXED EXCITED VALUES NSTEPS OUT
 *   RELAXED, EXCITED: NUMMF f32 each; VALUES: NSTEPS x NVARS f32 state values;
 *   OUT receives NSTEPS x NUMMF f32 rates (fibres outside every variable's
 *   share keep their relaxed rate). */
#include <cassert>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <sys/types.h>
#include <vector>

#include "statevariable.hpp"

uint64_t cbm_refshim_step = 0;
void cbm_refshim_set_step(uint64_t t) { cbm_refshim_step = t; }

struct ValueSource {
	float value = 0;
	float get() { return value; }
};

static bool readAll(const char *path, std::vector<float> &v)
{
	FILE *f = fopen(path, "rb");
	if (!f) return false;
	const size_t got = fread(v.data(), sizeof(float), v.size(), f);
	fclose(f);
	return got == v.size();
}

int main(int argc, char **argv)
{
	if (argc != 11) { fprintf(stderr, "usage: see the file header\n"); return 2; }
	const int numMF = atoi(argv[1]), nVars = atoi(argv[2]);
	const float lo = (float)atof(argv[3]), hi = (float)atof(argv[4]), width = (float)atof(argv[5]);
	const long nSteps = atol(argv[9]);
	std::vector<float> relaxed(numMF), excited(numMF), values((size_t)nSteps * nVars);
	if (!readAll(argv[6], relaxed) || !readAll(argv[7], excited) || !readAll(argv[8], values)) {
		fprintf(stderr, "cannot read inputs\n");
		return 1;
	}
	std::vector<float> freq(relaxed);
	std::vector<ValueSource> sources(nVars);
	std::vector<StateVariable<ValueSource> *> svs;
	for (int v = 0; v < nVars; v++) {
		svs.push_back(new StateVariable<ValueSource>("sv" + std::to_string(v), GAUSSIAN, 1.0f / nVars));
		svs.back()->initialize(numMF, &freq, &relaxed, &excited);
	}
	std::vector<int> unassigned;
	for (int i = numMF - 1; i >= 0; i--) unassigned.push_back(i);
	for (int v = 0; v < nVars; v++) {
		svs[v]->assignOrderedMFInds(unassigned);
		svs[v]->initializeGaussian(lo, hi, &sources[v], &ValueSource::get, width);
	}
	FILE *out = fopen(argv[10], "wb");
	if (!out) return 1;
	for (long s = 0; s < nSteps; s++) {
		for (int v = 0; v < nVars; v++) {
			sources[v].value = values[(size_t)s * nVars + v];
			svs[v]->update();
		}
		fwrite(freq.data(), sizeof(float), freq.size(), out);
	}
	fclose(out);
	for (auto *sv : svs) delete sv;
	return 0;
}
