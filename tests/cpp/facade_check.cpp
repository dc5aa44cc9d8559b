// A driver written against the reference's CBMState / CBMSimCore classes,
// compiled against include/cbm_core.hpp.  With one argument it loads a state
// and goes through the state library's accessors; with two it steps the
// network on GPU 0 and reads NC spikes.  "--stream OUT" (after the state)
// writes the state and then other data into one fstream and reads both
// back, as the eyelid driver's session file does (ECManagementDelay::
// writeDataToFile and its resume constructor, Eyelid_Sim_CBM_Dev/src/
// ectrial/ecmanagementdelay.cpp:26-50, 275-290); after the stepping run's
// two arguments it does the same with CBMSimCore::writeToState(fstream&).
#include <cbm_core.hpp>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

// The state, then a trailer, in one stream; then both read back from one
// stream: the state through CBMState(fstream&), the trailer after it.
template <typename W> static void streamRoundTrip(const char *path, W writeState)
{
	{
		std::fstream out(path, std::ios::out | std::ios::binary | std::ios::trunc);
		writeState(out);
		out << "trailer 4242\n";
	}
	std::fstream in(path, std::ios::in | std::ios::binary);
	CBMState back(in);
	std::string word;
	int value = 0;
	in >> word >> value;
	std::printf("stream zones %u trailer %s %d\n", back.getNumZones(), word.c_str(), value);
	std::string again = std::string(path) + ".again";
	back.writeState(again);
}

int main(int argc, char **argv)
{
	if (argc < 2) return 2;
	// "--generate ACT CON OUT": CBMState(actPF, conPF, 1, 11, {22}, {33}) and
	// writeState, as the reference's driver builds a new network
	if (!std::strcmp(argv[1], "--generate") && argc == 5) {
		std::fstream act(argv[2], std::ios::in), con(argv[3], std::ios::in);
		int cs[1] = {22}, as[1] = {33};
		CBMState st(act, con, 1, 11, cs, as);
		st.writeState(std::string(argv[4]));
		std::printf("generated zones %u\n", st.getNumZones());
		return 0;
	}
	const char *streamOut = nullptr;
	for (int i = 1; i + 1 < argc; i++)
		if (!std::strcmp(argv[i], "--stream")) { streamOut = argv[i + 1]; argc = i; break; }
	CBMState st(argv[1]);
	if (streamOut && argc == 2)
		streamRoundTrip(streamOut, [&](std::fstream &f) { st.writeState(f); });
	std::printf("zones %u\n", st.getNumZones());
	// the state library's accessors, as the eyelid driver reaches them
	// (ecmanagementdelay.cpp:106-150); they edit the state, so only without
	// the stepping run
	if (argc == 2) {
	IConnectivityParams *cp = st.getConnectivityParams();
	IActivityParams *ap = st.getActivityParams();
	std::printf("cells %u %u %u %u %u %u %u %u ms %u\n", cp->getNumGR(), cp->getNumGO(), cp->getNumMF(),
			cp->getNumSC(), cp->getNumBC(), cp->getNumPC(), cp->getNumNC(), cp->getNumIO(), ap->getMSPerTimeStep());
	const float ltd = ap->getParam("grPCLTDDecIO");
	const bool set = ap->setParam("grPCLTDDecIO", 2 * ltd), bad = ap->setParam("noSuchParam", 1);
	std::printf("params %zu %zu ltd %g set %d %g bad %d\n", cp->getParamCopy().size(), ap->getParamCopy().size(),
			ltd, (int)set, ap->getParam("grPCLTDDecIO"), (int)bad);
	IInNetConState *con = st.getInnetConState();
	std::printf("gr0 mf %zu go %zu go0 gr %zu incomplete %zu\n", con->getpGRfromMFtoGR(0).size(),
			con->getpGRfromGOtoGR(0).size(), con->getpGOfromGRtoGOCon(0).size(),
			con->getGRIncompIndfromGRtoGO().size());
	// a GO->GO pair added to and removed from both lists of GO 0 and GO 1
	const size_t out0 = con->getpGOOutGOGOCon(0).size(), in0 = con->getpGOInGOGOCon(1).size();
	const bool add = con->addGOGOConPair(0, 1);
	const size_t out1 = con->getpGOOutGOGOCon(0).size(), in1 = con->getpGOInGOGOCon(1).size();
	const ct_uint32_t last = out1 ? con->getpGOOutGOGOCon(0).back() : 0;
	const bool del = con->deleteGOGOConPair(0, 1), again = con->deleteGOGOConPair(0, 1);
	std::printf("gogo %zu %zu add %d %zu %zu last %u del %d again %d %zu %zu\n", out0, in0, (int)add, out1, in1,
			last, (int)del, (int)again, con->getpGOOutGOGOCon(0).size(), con->getpGOInGOGOCon(1).size());
	st.array<float>("pfSynWeightPC", 0)[0] = 0.25f;
	std::vector<float> w = st.getMZoneActState(0)->getGRPCSynWeightLinear();
	st.getMZoneActState(0)->resetGRPCSynWeight();
	std::printf("weights %zu %g reset %g equivalent %d\n", w.size(), w[0],
			st.getMZoneActState(0)->getGRPCSynWeightLinear()[0], (int)st.equivalent(st));
	}
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
		if (streamOut) streamRoundTrip(streamOut, [&](std::fstream &f) { sim.writeToState(f); });
	}
	return 0;
}
