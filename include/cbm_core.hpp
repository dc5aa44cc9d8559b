// C++ facade with the reference's CBM_CORE_LIB / CBM_STATE_LIB class names
// and signatures, implemented inline over the C ABI of cbm_b200.h, so that a
// driver written against the reference compiles against this header and links
// libcbm_b200.so instead of the reference's libraries.
//
// Mirrors (paths within the reference project):
//   CBMState        CBM_STATE_LIB_DEV/CBMStateInclude/interfaces/cbmstate.h:37-62
//   IConnectivityParams, IActivityParams, IInNetConState, IMZoneActState
//                   CBM_STATE_LIB_DEV/CBMStateInclude/interfaces/i*.h
//   CBMSimCore      CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/cbmsimcore.h:35-49
//   InNetInterface  CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/innetinterface.h:18-41
//   MZoneInterface  CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/mzoneinterface.h:18-34
//
// Error convention: the reference's calls return void and print CUDA errors;
// here a failed call throws cbm::Error carrying the C ABI's status and
// message (cbm_last_error).  Export pointers stay valid until the next
// export of the same field or the object's destruction, like the
// reference's host mirrors (innet.cpp:687-772).
#ifndef CBM_CORE_HPP
#define CBM_CORE_HPP

#include <algorithm>
#include <climits>
#include <deque>
#include <cstdint>
#include <fstream>
#include <iterator>
#include <map>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cbm_b200.h"

typedef uint8_t ct_uint8_t;
typedef uint32_t ct_uint32_t;
typedef int32_t ct_int32_t;
typedef uint64_t ct_uint64_t;

namespace cbm {

struct Error : std::runtime_error {
	int code;
	Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc)
{
	if (rc != CBM_OK) throw Error(rc, cbm_last_error());
}

// Keys of a state's parameter file (0 connectivity, 1 activity), in the
// reference's paramMap order.
inline std::vector<std::string> paramNames(const cbm_state *s, int which)
{
	uint64_t need = 0;
	cbm_state_param_names(s, which, nullptr, 0, &need);
	std::string buf(need, '\0');
	check(cbm_state_param_names(s, which, &buf[0], need, &need));
	std::vector<std::string> names;
	std::istringstream in(buf.c_str());
	for (std::string line; std::getline(in, line);) names.push_back(line);
	return names;
}

inline double rawParam(const cbm_state *s, int which, const std::string &name)
{
	double v = 0;
	check(cbm_state_raw_param(s, which, name.c_str(), &v));
	return v;
}

}  // namespace cbm

// IConnectivityParams (iconnectivityparams.h): cell counts and the
// parameter file's values.  showParams prints the file's keys and values.
class IConnectivityParams {
public:
	explicit IConnectivityParams(cbm_state *const *s) : s_(s) {}
	virtual ~IConnectivityParams() {}
	virtual void showParams(std::ostream &outSt)
	{
		for (const auto &kv : getParamCopy()) outSt << kv.first << " " << kv.second << std::endl;
	}
	virtual ct_uint32_t getGOX() { return con("goX"); }
	virtual ct_uint32_t getGOY() { return con("goY"); }
	virtual ct_uint32_t getGRX() { return con("grX"); }
	virtual ct_uint32_t getGRY() { return con("grY"); }
	virtual ct_uint32_t getGLX() { return con("glX"); }
	virtual ct_uint32_t getGLY() { return con("glY"); }
	virtual ct_uint32_t getNumMF() { return con("numMF"); }
	virtual ct_uint32_t getNumGO() { return con("numGO"); }
	virtual ct_uint32_t getNumGR() { return con("numGR"); }
	virtual ct_uint32_t getNumGL() { return con("numGL"); }
	virtual ct_uint32_t getNumSC() { return con("numSC"); }
	virtual ct_uint32_t getNumBC() { return con("numBC"); }
	virtual ct_uint32_t getNumPC() { return con("numPC"); }
	virtual ct_uint32_t getNumNC() { return con("numNC"); }
	virtual ct_uint32_t getNumIO() { return con("numIO"); }
	virtual std::map<std::string, ct_uint32_t> getParamCopy()
	{
		std::map<std::string, ct_uint32_t> m;
		for (const std::string &n : cbm::paramNames(*s_, 0)) m[n] = (ct_uint32_t)cbm::rawParam(*s_, 0, n);
		return m;
	}

private:
	ct_uint32_t con(const char *name)
	{
		uint32_t v = 0;
		cbm::check(cbm_state_con_param(*s_, name, &v));
		return v;
	}
	cbm_state *const *s_;
};

// IActivityParams (iactivityparams.h): getParam / setParam work on the
// parameter file's keys, and setParam re-derives the values the step uses
// (activityparams.cpp:418-434).
class IActivityParams {
public:
	explicit IActivityParams(cbm_state *const *s) : s_(s) {}
	virtual ~IActivityParams() {}
	virtual unsigned int getMSPerTimeStep()
	{
		double v = 0;
		cbm::check(cbm_state_act_param(*s_, "msPerTimeStep", &v));
		return (unsigned int)v;
	}
	virtual void showParams(std::ostream &outSt)
	{
		for (const auto &kv : getParamCopy()) outSt << kv.first << " " << kv.second << std::endl;
	}
	virtual std::map<std::string, float> getParamCopy()
	{
		std::map<std::string, float> m;
		for (const std::string &n : cbm::paramNames(*s_, 1)) m[n] = (float)cbm::rawParam(*s_, 1, n);
		return m;
	}
	// an unknown key reads 0, as the reference's paramMap[key] does
	virtual float getParam(std::string paramName)
	{
		double v = 0;
		return cbm_state_raw_param(*s_, 1, paramName.c_str(), &v) == CBM_OK ? (float)v : 0.0f;
	}
	virtual bool setParam(std::string paramName, float value)
	{
		return cbm_state_set_act_param(*s_, paramName.c_str(), value) == CBM_OK;
	}

private:
	cbm_state *const *s_;
};

class CBMState;

// IInNetConState (iinnetconstate.h): per-cell connection lists of the input
// network, read from (and, for the GO->GO pairs, edited in) the state arrays
// before a simulator is built on them (innetconnectivitystate.cpp:245-470).
class IInNetConState {
public:
	explicit IInNetConState(CBMState *st) : st_(st) {}
	virtual ~IInNetConState() {}
	virtual std::vector<ct_uint32_t> getpGOfromGOtoGLCon(int goN) { return con("numpGOfromGOtoGL", "pGOfromGOtoGL", goN); }
	virtual std::vector<ct_uint32_t> getpGOfromGLtoGOCon(int goN) { return con("numpGOfromGLtoGO", "pGOfromGLtoGO", goN); }
	virtual std::vector<ct_uint32_t> getpMFfromMFtoGLCon(int mfN) { return con("numpMFfromMFtoGL", "pMFfromMFtoGL", mfN); }
	virtual std::vector<ct_uint32_t> getpGLfromGLtoGRCon(int glN) { return con("numpGLfromGLtoGR", "pGLfromGLtoGR", glN); }
	virtual std::vector<ct_uint32_t> getpGRfromMFtoGR(int grN) { return con("numpGRfromMFtoGR", "pGRfromMFtoGR", grN); }
	virtual std::vector<std::vector<ct_uint32_t> > getpGRPopfromMFtoGR() { return all("numpGRfromMFtoGR", "pGRfromMFtoGR"); }
	virtual std::vector<ct_uint32_t> getpGRfromGOtoGR(int grN) { return con("numpGRfromGOtoGR", "pGRfromGOtoGR", grN); }
	virtual std::vector<std::vector<ct_uint32_t> > getpGRPopfromGOtoGR() { return all("numpGRfromGOtoGR", "pGRfromGOtoGR"); }
	virtual std::vector<ct_uint32_t> getpGOfromGRtoGOCon(int goN) { return con("numpGOfromGRtoGO", "pGOfromGRtoGO", goN); }
	virtual std::vector<ct_uint32_t> getpGOfromGOtoGRCon(int goN) { return con("numpGOfromGOtoGR", "pGOfromGOtoGR", goN); }
	virtual std::vector<ct_uint32_t> getpMFfromMFtoGRCon(int mfN) { return con("numpMFfromMFtoGR", "pMFfromMFtoGR", mfN); }
	virtual std::vector<ct_uint32_t> getpMFfromMFtoGOCon(int mfN) { return con("numpMFfromMFtoGO", "pMFfromMFtoGO", mfN); }
	virtual std::vector<ct_uint32_t> getpGOfromMFtoGOCon(int goN) { return con("numpGOfromMFtoGO", "pGOfromMFtoGO", goN); }
	virtual std::vector<std::vector<ct_uint32_t> > getpGOPopfromMFtoGOCon() { return all("numpGOfromMFtoGO", "pGOfromMFtoGO"); }
	virtual std::vector<ct_uint32_t> getpGOOutGOGOCon(int goN) { return con("numpGOGABAOutGOGO", "pGOGABAOutGOGO", goN); }
	virtual std::vector<ct_uint32_t> getpGOInGOGOCon(int goN) { return con("numpGOGABAInGOGO", "pGOGABAInGOGO", goN); }
	// cells whose GR->GO lists are below their maximum (innetconnectivitystate.cpp:371-396)
	virtual std::vector<ct_uint32_t> getGOIncompIndfromGRtoGO() { return incomplete("numpGOfromGRtoGO", "maxnumpGOfromGRtoGO"); }
	virtual std::vector<ct_uint32_t> getGRIncompIndfromGRtoGO() { return incomplete("numpGRfromGRtoGO", "maxnumpGRfromGRtoGO"); }
	// remove / add one GO->GO GABA pair in both directions' lists
	// (innetconnectivitystate.cpp:398-452)
	virtual bool deleteGOGOConPair(int srcGON, int destGON);
	virtual bool addGOGOConPair(int srcGON, int destGON);

private:
	struct Table { int32_t *num; ct_uint32_t *p; uint64_t rows, stride; };
	Table table(const char *num, const char *list);
	std::vector<ct_uint32_t> con(const char *num, const char *list, int n)
	{
		Table t = table(num, list);
		if (n < 0 || (uint64_t)n >= t.rows) throw cbm::Error(CBM_ERR_ARG, "cell index out of range");
		const ct_uint32_t *row = t.p + (uint64_t)n * t.stride;
		return std::vector<ct_uint32_t>(row, row + t.num[n]);
	}
	std::vector<std::vector<ct_uint32_t> > all(const char *num, const char *list)
	{
		Table t = table(num, list);
		std::vector<std::vector<ct_uint32_t> > v(t.rows);
		for (uint64_t i = 0; i < t.rows; i++) v[i].assign(t.p + i * t.stride, t.p + i * t.stride + t.num[i]);
		return v;
	}
	std::vector<ct_uint32_t> incomplete(const char *num, const char *maxName);
	CBMState *st_;
};

// IMZoneActState (imzoneactstate.h): zone z's PF->PC weights, PC-major
// (mzoneactivitystate.cpp:202-228).
class IMZoneActState {
public:
	IMZoneActState(CBMState *st, unsigned int zone) : st_(st), zone_(zone) {}
	virtual ~IMZoneActState() {}
	virtual std::vector<float> getGRPCSynWeightLinear();
	virtual void resetGRPCSynWeight();

private:
	CBMState *st_;
	unsigned int zone_;
};

namespace cbm {
// The rest of a stream from its get position (the C ABI parses memory).
inline std::string restOf(std::istream &in, std::streampos &start)
{
	start = in.tellg();
	std::string data((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
	return data;
}
// Writes one of the C ABI's two-call serialisations into a stream.
template <typename F> void writeSerialised(std::ostream &out, F save)
{
	uint64_t n = 0;
	check(save(nullptr, 0, &n));
	std::vector<char> buf((size_t)n);
	check(save(buf.data(), n, &n));
	out.write(buf.data(), (std::streamsize)n);
	if (!out) throw Error(CBM_ERR_IO, "stream write failed");
}
}  // namespace cbm

class CBMState {
public:
	// CBMState(fstream&) (cbmstate.h:37): reads one state from the stream's
	// position and leaves the stream just after it, where the eyelid driver's
	// session file continues with its trial data.
	explicit CBMState(std::fstream &infile)
	{
		std::streampos start;
		std::string data = cbm::restOf(infile, start);
		uint64_t used = 0;
		cbm::check(cbm_state_load_mem(data.data(), data.size(), &used, &s_));
		infile.clear();
		infile.seekg(start + (std::streamoff)used);
	}
	// The same from a file name.
	explicit CBMState(const std::string &statePath) { cbm::check(cbm_state_load(statePath.c_str(), &s_)); }
	// CBMState(actPF, conPF, nZones) and CBMState(actPF, conPF, nZones,
	// innetCRSeed, mzoneCRSeed, mzoneARSeed) (cbmstate.h:38-40): a new
	// network from the parameter files with the reference's own generator and
	// random sequence; without seeds they come from the wall clock.
	CBMState(std::fstream &actPFile, std::fstream &conPFile, unsigned int nZones)
	{
		generate(actPFile, conPFile, nZones, nullptr);
	}
	CBMState(std::fstream &actPFile, std::fstream &conPFile, unsigned int nZones, int innetCRSeed, int *mzoneCRSeed,
			int *mzoneARSeed)
	{
		std::vector<int> seeds(1, innetCRSeed);
		for (unsigned int z = 0; z < nZones; z++) seeds.push_back(mzoneCRSeed[z]);
		for (unsigned int z = 0; z < nZones; z++) seeds.push_back(mzoneARSeed[z]);
		generate(actPFile, conPFile, nZones, seeds.data());
	}
	// CBMState(actPF, conPF, nZones, innetCRSeed, mzoneCRSeed, mzoneARSeed) from the
	// parameter texts; the input-net wiring is left for the caller (see cbm_state_new).
	CBMState(const std::string &actParamsText, const std::string &conParamsText, unsigned int nZones,
			const int *mzoneCRSeed = nullptr)
	{
		cbm::check(cbm_state_new(conParamsText.c_str(), actParamsText.c_str(), nZones, mzoneCRSeed, &s_));
	}
	CBMState(const CBMState &) = delete;
	CBMState &operator=(const CBMState &) = delete;
	virtual ~CBMState() { cbm_state_free(s_); }

	// writeState(fstream&) (cbmstate.h:43): the state at the stream's position.
	void writeState(std::fstream &outfile)
	{
		cbm::writeSerialised(outfile, [this](void *d, uint64_t c, uint64_t *n) { return cbm_state_save_mem(s_, d, c, n); });
	}
	void writeState(const std::string &path) { cbm::check(cbm_state_save(s_, path.c_str())); }
	ct_uint32_t getNumZones()
	{
		unsigned n = 0;
		cbm::check(cbm_state_num_zones(s_, &n));
		return n;
	}
	template <typename T> T *array(const char *name, int zone = -1, uint64_t *count = nullptr)
	{
		void *p = nullptr;
		uint64_t n = 0;
		int dt = 0;
		cbm::check(cbm_state_array(s_, name, zone, &p, &n, &dt));
		if (count) *count = n;
		return static_cast<T *>(p);
	}
	cbm_state *handle() { return s_; }

private:
	void generate(std::fstream &actPFile, std::fstream &conPFile, unsigned int nZones, const int *seeds)
	{
		std::streampos a0, c0;
		const std::string act = cbm::restOf(actPFile, a0), con = cbm::restOf(conPFile, c0);
		cbm::check(cbm_state_generate(con.c_str(), act.c_str(), nZones, seeds, &s_));
	}

public:

	// the reference's accessors; the objects live as long as the state
	IConnectivityParams *getConnectivityParams() { return &conParams_; }
	IActivityParams *getActivityParams() { return &actParams_; }
	IInNetConState *getInnetConState() { return &innetCon_; }
	IMZoneActState *getMZoneActState(unsigned int zoneN)
	{
		if (zoneN >= getNumZones()) throw cbm::Error(CBM_ERR_ARG, "zone out of range");
		while (zoneAct_.size() <= zoneN) zoneAct_.emplace_back(this, (unsigned int)zoneAct_.size());
		return &zoneAct_[zoneN];
	}
	// CBMState::equivalent (cbmstate.cpp:105-121, innetconnectivitystate.cpp:
	// 228-243): the same zone count, MF->GL glomeruli, GO->GR and GR<-GO counts
	bool equivalent(CBMState &compState)
	{
		if (getNumZones() != compState.getNumZones()) return false;
		for (const char *n : {"haspGLfromMFtoGL", "numpGOfromGOtoGR", "numpGRfromGOtoGR"}) {
			uint64_t a = 0, b = 0;
			const uint8_t *x = array<uint8_t>(n, -1, &a), *y = compState.array<uint8_t>(n, -1, &b);
			const uint64_t bytes = std::string(n) == "haspGLfromMFtoGL" ? a : 4 * a;
			if (a != b || !std::equal(x, x + bytes, y)) return false;
		}
		return true;
	}

private:
	cbm_state *s_ = nullptr;
	IConnectivityParams conParams_{&s_};
	IActivityParams actParams_{&s_};
	IInNetConState innetCon_{this};
	std::deque<IMZoneActState> zoneAct_;  // stable addresses as zones are added
};

inline IInNetConState::Table IInNetConState::table(const char *num, const char *list)
{
	Table t;
	uint64_t cnt = 0;
	t.num = st_->array<int32_t>(num, -1, &t.rows);
	t.p = st_->array<ct_uint32_t>(list, -1, &cnt);
	t.stride = t.rows ? cnt / t.rows : 0;
	return t;
}

inline std::vector<ct_uint32_t> IInNetConState::incomplete(const char *num, const char *maxName)
{
	uint64_t rows = 0;
	const int32_t *k = st_->array<int32_t>(num, -1, &rows);
	uint32_t limit = 0;
	cbm::check(cbm_state_con_param(st_->handle(), maxName, &limit));
	std::vector<ct_uint32_t> v;
	for (uint64_t i = 0; i < rows; i++) if ((uint32_t)k[i] < limit) v.push_back((ct_uint32_t)i);
	return v;
}

inline bool IInNetConState::deleteGOGOConPair(int srcGON, int destGON)
{
	Table out = table("numpGOGABAOutGOGO", "pGOGABAOutGOGO"), in = table("numpGOGABAInGOGO", "pGOGABAInGOGO");
	ct_uint32_t *o = out.p + (uint64_t)srcGON * out.stride;
	int at = -1;
	for (int i = 0; i < out.num[srcGON]; i++) if (o[i] == (ct_uint32_t)destGON) { at = i; break; }
	if (at < 0) return false;
	for (int i = at; i < out.num[srcGON] - 1; i++) o[i] = o[i + 1];
	out.num[srcGON]--;
	// the reference removes the last matching entry of the in-list (with
	// in- and out-lists that mirror each other, as every state has them)
	ct_uint32_t *q = in.p + (uint64_t)destGON * in.stride;
	int last = -1;
	for (int i = 0; i < in.num[destGON]; i++) if (q[i] == (ct_uint32_t)srcGON) last = i;
	if (last >= 0) {
		for (int i = last; i < in.num[destGON] - 1; i++) q[i] = q[i + 1];
		in.num[destGON]--;
	}
	return true;
}

inline bool IInNetConState::addGOGOConPair(int srcGON, int destGON)
{
	Table out = table("numpGOGABAOutGOGO", "pGOGABAOutGOGO"), in = table("numpGOGABAInGOGO", "pGOGABAInGOGO");
	if ((uint64_t)out.num[srcGON] >= out.stride || (uint64_t)in.num[destGON] >= in.stride) return false;
	out.p[(uint64_t)srcGON * out.stride + out.num[srcGON]++] = (ct_uint32_t)destGON;
	in.p[(uint64_t)destGON * in.stride + in.num[destGON]++] = (ct_uint32_t)srcGON;
	return true;
}

inline std::vector<float> IMZoneActState::getGRPCSynWeightLinear()
{
	uint64_t n = 0;
	const float *w = st_->array<float>("pfSynWeightPC", (int)zone_, &n);
	return std::vector<float>(w, w + n);
}

inline void IMZoneActState::resetGRPCSynWeight()
{
	double w0 = 0;
	cbm::check(cbm_state_act_param(st_->handle(), "initSynWofGRtoPC", &w0));
	uint64_t n = 0;
	float *w = st_->array<float>("pfSynWeightPC", (int)zone_, &n);
	for (uint64_t i = 0; i < n; i++) w[i] = (float)w0;
}

class InNetInterface {
public:
	explicit InNetInterface(cbm_sim *sim) : sim_(sim) {}
	virtual ~InNetInterface() {}

	virtual void setGIncGRtoGO(float inc) { cbm::check(cbm_sim_set_ginc_grgo(sim_, inc)); }
	virtual void resetGIncGRtoGO() { cbm::check(cbm_sim_reset_ginc_grgo(sim_)); }

	virtual const ct_uint8_t *exportAPSC() { return field<ct_uint8_t>(CBM_AP_SC); }
	virtual const ct_uint8_t *exportAPGO() { return field<ct_uint8_t>(CBM_AP_GO); }
	virtual const ct_uint8_t *exportAPGR() { return field<ct_uint8_t>(CBM_AP_GR); }
	virtual const ct_uint8_t *exportHistMF() { return field<ct_uint8_t>(CBM_HIST_MF); }
	virtual const ct_uint32_t *exportAPBufMF() { return field<ct_uint32_t>(CBM_APBUF_MF); }
	virtual const ct_uint32_t *exportAPBufGR() { return field<ct_uint32_t>(CBM_APBUF_GR); }
	virtual const ct_uint32_t *exportAPBufGO() { return field<ct_uint32_t>(CBM_APBUF_GO); }
	virtual const ct_uint32_t *exportAPBufSC() { return field<ct_uint32_t>(CBM_APBUF_SC); }
	virtual const float *exportVmGR() { return field<float>(CBM_VM_GR); }
	virtual const float *exportVmGO() { return field<float>(CBM_VM_GO); }
	virtual const float *exportVmSC() { return field<float>(CBM_VM_SC); }
	virtual const float *exportGESumGR() { return field<float>(CBM_GESUM_GR); }
	virtual const float *exportGISumGR() { return field<float>(CBM_GISUM_GR); }
	virtual const ct_uint32_t *exportSumGRInputGO() { return field<ct_uint32_t>(CBM_SUM_GR_INPUT_GO); }
	virtual const float *exportSumGOInputGO() { return field<float>(CBM_SUM_GO_INPUT_GO); }
	virtual const float *exportGOOutSynScaleGOGO() { return field<float>(CBM_GO_OUT_SCALE_GOGO); }

protected:
	template <typename T> const T *field(int f)
	{
		std::vector<uint8_t> &buf = mirror_[f];
		buf.resize(cbm_sim_field_bytes(sim_, f));
		cbm::check(cbm_sim_export(sim_, f, zone_, buf.data(), buf.size()));
		return reinterpret_cast<const T *>(buf.data());
	}
	cbm_sim *sim_;
	unsigned zone_ = 0;
	std::vector<uint8_t> mirror_[CBM_FIELD_COUNT];
};

class MZoneInterface : protected InNetInterface {
public:
	MZoneInterface(cbm_sim *sim, unsigned zone) : InNetInterface(sim) { zone_ = zone; }
	virtual ~MZoneInterface() {}

	virtual void setGRPCPlastSteps(float ltdStep, float ltpStep) { cbm::check(cbm_sim_set_plast_steps(sim_, zone_, ltdStep, ltpStep)); }
	virtual void resetGRPCPlastSteps() { cbm::check(cbm_sim_reset_plast_steps(sim_, zone_)); }

	virtual const ct_uint8_t *exportAPBC() { return field<ct_uint8_t>(CBM_AP_BC); }
	virtual const ct_uint8_t *exportAPPC() { return field<ct_uint8_t>(CBM_AP_PC); }
	virtual const ct_uint8_t *exportAPIO() { return field<ct_uint8_t>(CBM_AP_IO); }
	virtual const ct_uint8_t *exportAPNC() { return field<ct_uint8_t>(CBM_AP_NC); }
	virtual const ct_uint32_t *exportAPBufBC() { return field<ct_uint32_t>(CBM_APBUF_BC); }
	virtual const ct_uint32_t *exportAPBufPC() { return field<ct_uint32_t>(CBM_APBUF_PC); }
	virtual const ct_uint32_t *exportAPBufIO() { return field<ct_uint32_t>(CBM_APBUF_IO); }
	virtual const ct_uint32_t *exportAPBufNC() { return field<ct_uint32_t>(CBM_APBUF_NC); }
	virtual const float *exportVmBC() { return field<float>(CBM_VM_BC); }
	virtual const float *exportVmPC() { return field<float>(CBM_VM_PC); }
	virtual const float *exportVmNC() { return field<float>(CBM_VM_NC); }
	virtual const float *exportVmIO() { return field<float>(CBM_VM_IO); }
};

class CBMSimCore {
public:
	// CBMSimCore(CBMState*, int gpuIndStart=-1, int numGPUP2=-1): the whole
	// network runs on device max(gpuIndStart, 0); zone seeds default to 1000+z.
	CBMSimCore(CBMState *state, int gpuIndStart = -1, int numGPUP2 = -1) { construct(state, nullptr, gpuIndStart, numGPUP2); }
	CBMSimCore(CBMState *state, int *mzoneRSeed, int gpuIndStart = -1, int numGPUP2 = -1)
	{
		construct(state, mzoneRSeed, gpuIndStart, numGPUP2);
	}
	CBMSimCore(const CBMSimCore &) = delete;
	CBMSimCore &operator=(const CBMSimCore &) = delete;
	~CBMSimCore()
	{
		for (MZoneInterface *z : zones_) delete z;
		delete innet_;
		cbm_sim_destroy(sim_);
	}

	void calcActivity() { cbm::check(cbm_sim_calc_activity(sim_)); }
	void updateMFInput(const ct_uint8_t *mfIn) { cbm::check(cbm_sim_update_mf(sim_, mfIn)); }
	void updateErrDrive(unsigned int zoneN, float errDriveRelative) { cbm::check(cbm_sim_update_err_drive(sim_, zoneN, errDriveRelative)); }
	void writeToState() { cbm::check(cbm_sim_write_to_state(sim_)); }
	// writeToState(fstream&) (cbmsimcore.h:46): the device state written back,
	// then the state at the stream's position.
	void writeToState(std::fstream &outfile)
	{
		cbm::writeSerialised(outfile, [this](void *d, uint64_t c, uint64_t *n) { return cbm_sim_save_mem(sim_, d, c, n); });
	}
	void writeToState(const std::string &path) { cbm::check(cbm_sim_save(sim_, path.c_str())); }
	InNetInterface *getInputNet() { return innet_; }
	MZoneInterface **getMZoneList() { return zones_.data(); }
	cbm_sim *handle() { return sim_; }

private:
	void construct(CBMState *state, int *mzoneRSeed, int gpuIndStart, int numGPUP2)
	{
		(void)numGPUP2;
		cbm::check(cbm_sim_create(state->handle(), mzoneRSeed, gpuIndStart < 0 ? 0 : gpuIndStart, &sim_));
		innet_ = new InNetInterface(sim_);
		for (unsigned z = 0; z < state->getNumZones(); z++) zones_.push_back(new MZoneInterface(sim_, z));
	}
	cbm_sim *sim_ = nullptr;
	InNetInterface *innet_ = nullptr;
	std::vector<MZoneInterface *> zones_;
};

#endif
