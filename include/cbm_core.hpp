// C++ facade with the reference's CBM_CORE_LIB / CBM_STATE_LIB class names
// and signatures, implemented inline over the C ABI of cbm_b200.h, so that a
// driver written against the reference compiles against this header and links
// libcbm_b200.so instead of the reference's libraries.
//
// Mirrors (paths within the reference project):
//   CBMState        CBM_STATE_LIB_DEV/CBMStateInclude/interfaces/cbmstate.h:37-62
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

#include <climits>
#include <cstdint>
#include <fstream>
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

// Path of an fstream the reference's API passes around: the facade reopens
// the named file because the C ABI works on paths.
struct StreamPath {
	std::string path;
};

}  // namespace cbm

class CBMState {
public:
	// CBMState(fstream&) reads a state file; this facade takes its path.
	explicit CBMState(const std::string &statePath) { cbm::check(cbm_state_load(statePath.c_str(), &s_)); }
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
	cbm_state *s_ = nullptr;
};

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
