// A driver written against the reference's CBMState / CBMSimCore classes,
// compiled against include/cbm_core.hpp.  With one argument it only loads a
// state; with two it also steps the network on GPU 0 and reads NC spikes.
#include <cbm_core.hpp>

#include <cstdio>
#include <vector>

int main(int argc, char **argv)
{
	if (argc < 2) return 2;
	CBMState st(argv[1]);
	std::printf("zones %u\n", st.getNumZones());
	if (argc > 2) {
		int seeds[1] = {7};
		CBMSimCore sim(&st, seeds, 0, -1);
		std::vector<ct_uint8_t> mf(1024, 0);
		for (int t = 0; t < 50; t++) {
			for (size_t i = 0; i < mf.size(); i++) mf[i] = ((i * 2654435761u + t * 40503u) % 97) < 3;
			sim.updateMFInput(mf.data());
			sim.calcActivity();
		}
		const ct_uint8_t *nc = sim.getMZoneList()[0]->exportAPNC();
		const float *vpc = sim.getMZoneList()[0]->exportVmPC();
		std::printf("steps 50 nc0 %d vpc0 %.6f\n", nc[0], vpc[0]);
		sim.writeToState(argv[2]);
	}
	return 0;
}
