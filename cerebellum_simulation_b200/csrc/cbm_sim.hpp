// Host object driving one or more device-resident networks: the B200
// counterpart of the reference's CBMSimCore + InNet + MZone objects
// (CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/cbmsimcore.h:32-75,
// innetmodules/innet.h, mzonemodules/mzone.h).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/cbm_b200.h"
#include "cbm_device.cuh"
#include "cbm_state.hpp"

namespace cbm {

// Fields a caller can read back (the reference's export* calls and the
// state arrays behind them).
enum Field : int {
	F_AP_GR = 0, F_VM_GR, F_GESUM_GR, F_GISUM_GR, F_APBUF_GR, F_HIST_GR, F_THRESH_GR, F_GKCA_GR,
	F_AP_GO, F_VM_GO, F_APBUF_GO, F_SUM_GR_INPUT_GO, F_SUM_GO_INPUT_GO, F_GO_OUT_SCALE_GOGO,
	F_AP_SC, F_VM_SC, F_APBUF_SC, F_HIST_MF, F_APBUF_MF,
	F_AP_BC, F_VM_BC, F_APBUF_BC, F_AP_PC, F_VM_PC, F_APBUF_PC, F_AP_IO, F_VM_IO, F_APBUF_IO,
	F_AP_NC, F_VM_NC, F_APBUF_NC, F_PFPC_WEIGHT, F_MFNC_WEIGHT,
	F_COUNT
};

struct DeviceBuf {
	void *ptr = nullptr;
	size_t bytes = 0;
};

class Network;

// Host-side validation of a network before it goes to a device: the
// structural limits of the kernels and every connectivity count and index.
// Returns an empty string or the reason; Simulator::create calls it first.
std::string checkNetwork(const State &st);

// Pinned staging slots for host MF input per network (updateMFInput).
constexpr uint32_t kMFStage = 8;

// A GR-pass kernel choice: kind 0 plain, 1 per-tile TMA (W consumer warps of
// RW rows, S stages, B CTAs/SM, slot bound M), 2 persistent TMA (W, S, B, M),
// 3 vector (cbm_pass_vec.cu; no parameters).
struct PassGeometry {
	int kind = 0, W = 0, RW = 1, S = 0, B = 0, M = 0;
};

// A set of networks that advance together: one network for the drop-in
// CBMSimCore path, many for the batched sweep.
class Simulator {
public:
	~Simulator();
	std::string create(const std::vector<State *> &states, const std::vector<std::vector<int>> &seeds,
			int device, uint32_t mfRing, const std::vector<uint32_t> *mfSeeds = nullptr);
	size_t numNets() const { return nets_.size(); }
	Network &net(size_t i) { return *nets_[i]; }

	// One step of every network with MF input already in each network's ring.
	std::string launchSteps(uint32_t nsteps);
	// Add the steps launched one at a time since the last call to the device
	// step counter (one kernel on the step stream); every other operation
	// that launches work reading the counter calls it first.
	std::string settleSteps();
	// Host MF input for the next step of network i (updateMFInput).
	std::string stageMF(size_t i, const uint8_t *mf);
	// Start a device-driven trial protocol on network i from the next step.
	std::string setProtocol(size_t i, const cbm_eyelid_protocol &p);
	// Start the state-variable MF input (cbm_statevar_input) on network i.
	std::string setStateVarInput(size_t i, const cbm_statevar_input &in);
	// Record network 0's GR peri-stimulus histogram (single-network simulators).
	std::string recordGR();
	std::string recordTrialData(size_t i = 0);
	// Run nsteps as CUDA-graph chunks of chunk steps (inputs resident in HBM).
	// With instrument, external events around every GR pass of the chunk
	// give lastPassMs(): the pass's mean duration over the last replay.
	std::string runGraph(uint64_t nsteps, uint32_t chunk, bool instrument = false);
	// Measurement helper: nsteps single-step graph launches, each after a
	// write and read-back of a flushBytes device buffer (an L2 flush when
	// larger than L2, leaving only clean lines of the buffer in L2), with
	// events on the launch stream around every step only; *stepMs is the
	// summed step time.
	void enqueueFlush();
	std::string runFlushed(uint64_t nsteps, size_t flushBytes, float *stepMs);
	// The same steps in the two-stream form with events around each kernel:
	// mean GR-pass and small-cell kernel durations of a step after a flush.
	std::string runFlushedKernels(uint64_t nsteps, size_t flushBytes, float *passMs, float *tailMs);
	std::string sync();
	// A field of network i into host memory: the copy and a read of every
	// network's device error word share one synchronisation.
	std::string exportField(size_t i, Field f, uint32_t zone, void *dst, size_t bytes);
	cudaStream_t stream() const { return s0_; }
	int device() const { return device_; }
	// Time of the last runGraph call measured with events on the launch stream.
	float lastGraphMs() const { return lastGraphMs_; }
	float lastPassMs() const { return lastPassMs_; }
	float lastTailMs() const { return lastTailMs_; }
	// rows per stage and stages of the TMA GR pass (0, 0 when the plain pass runs)
	uint32_t passStageRows() const { return passTmaR_; }
	uint32_t passStages() const { return passTmaS_; }
	// GR-pass kernels that fit every network (the default first), the one in
	// use, and switching to another (graphs are re-captured).
	std::vector<PassGeometry> passCandidates() const;
	const PassGeometry &passGeometryInUse() const { return passGeom_; }
	std::string usePassGeometry(const PassGeometry &g);
	// Device error word of every network (kErr* bits): non-empty on error.
	std::string checkDeviceErrors();
	void passGeometry(unsigned *kind, unsigned *warps, unsigned *rows, unsigned *stages) const
	{
		*kind = passVec_ ? 3u : passTmaFn_ ? (passPersistent_ ? 2u : 1u) : 0u;
		*warps = passTmaW_;
		*rows = passTmaR_;
		*stages = passTmaS_;
	}
	std::string timerStart();
	std::string timerStop(float *ms);

private:
	friend class Network;
	std::string uploadCtl();
	// chained: launched one at a time, the small-cell kernel as the
	// programmatic dependent of the previous step (see launchSteps)
	std::string enqueueStep(uint32_t stepOffset, bool instrument, bool chained = false);
	std::string recordStep(uint32_t stepOffset);
	void dropGraphs();
	void markInputSlotsFree();  // after a full synchronisation
	// Issue the copy of MF input that a single-step graph would have carried.
	std::string flushPendingMF();
	// One network, one-slot MF ring, spike-bit input: updateMFInput only
	// packs the bits into pinned slot k, and the next step launched by
	// launchSteps copies them in before its kernels.
	int pendingMF_ = -1;
	bool directCopySinceStep_ = false;  // an MF copy issued outside launchSteps since its last step
	// Steps launched one at a time (launchSteps) since the device step
	// counter was last advanced: step k of them ran with step offset k.
	uint32_t directPending_ = 0;
	// The MF words the next enqueued step's kernels take from their launch
	// (n = 0: they read the MF ring); see mfByParam().
	MFParam stepMF_{};
	bool mfByParam() const;
	uint8_t *hExport_ = nullptr;           // pinned export staging
	size_t hExportBytes_ = 0;
	std::vector<Network *> nets_;
	int device_ = 0;
	cudaStream_t s0_ = nullptr, s1_ = nullptr;
	cudaEvent_t fork_ = nullptr, join_ = nullptr, ev0_ = nullptr, ev1_ = nullptr, tev0_ = nullptr, tev1_ = nullptr;
	DeviceBuf dNetPtrs_, dBlockOffset_, dTBasePtrs_, dStageBytes_;
	DeviceBuf dExitCount_;    // the per-tile pass's CTAs that finished a chained single step (passExitWait)
	DeviceBuf dCellOffset_;   // trialDataBatchKernel's instance map (batches recording trial data)
	// the batched vector pass: first 128-cell unit and first PC of each
	// network (numNets + 1 prefix sums each), and its three claim counters
	DeviceBuf dVecUnitOffset_, dVecPcOffset_, dVecClaim_;
	uint32_t cellTotal_ = 0;
	uint32_t passBlocks_ = 0;
	size_t passSmem_ = 0, tailSmem_ = 0;
	// TMA GR pass geometry (passTmaFn_ null: the plain pass kernel runs)
	const void *passTmaFn_ = nullptr;
	uint32_t passTmaW_ = 0, passTmaR_ = 0, passTmaS_ = 0, passGrid_ = 0;
	bool passPersistent_ = false;
	bool passVec_ = false;  // the vector pass (kind 3) runs
	// the small-cell kernel argument of the step being enqueued: the NC
	// mailbox for steps launched one at a time (one network), else null
	uint8_t *mailboxArg_ = nullptr;
	bool lastStepPublishes_ = false;  // the last launch was a single step that writes the mailbox
	uint32_t vecClaim_ = 2;  // its units claimed at a time (single network)
	PassGeometry passGeom_;
	size_t passTmaSmem_ = 0;
	cudaGraphExec_t graphExec_ = nullptr;
	uint32_t graphChunk_ = 0;
	bool graphInstrumented_ = false;
	std::vector<cudaEvent_t> passEv_, tailEv_;
	cudaGraphExec_t flushKernGraph_ = nullptr;
	DeviceBuf flushBuf_;
	std::vector<cudaEvent_t> stepEv_;  // runFlushed: a pair around each step of a batch
	float lastGraphMs_ = 0, lastPassMs_ = 0, lastTailMs_ = 0;
};

class Network {
public:
	~Network();
	std::string build(State *st, const std::vector<int> &seeds, uint32_t mfRing, uint32_t mfSeed);
	// host setters of the reference's API
	void setPlastSteps(uint32_t zone, float ltd, float ltp);
	void resetPlastSteps(uint32_t zone);
	void setErrDrive(uint32_t zone, float rel);
	void setGIncGRtoGO(float v);
	void resetGIncGRtoGO();
	// Enqueue a copy of one field into host memory on stream s (bytes must
	// equal fieldBytes); the caller synchronises before reading dst.
	std::string exportField(Field f, uint32_t zone, void *dst, size_t bytes, cudaStream_t s);
	size_t fieldBytes(Field f) const;
	// CBMSimCore::writeToState(): device values back into the state.
	std::string writeToState(cudaStream_t s);
	// The reference's writeState resets the GO->GO depression arrays of the
	// live state (innetactivitystate.cpp:247-248); mirrored on the device.
	std::string resetGOGODepression(cudaStream_t s);
	// Device-driven trial protocol (cbm_eyelid_protocol) from the next step on.
	// sv: the state-variable coding's fields of the protocol descriptor, or null
	std::string setProtocol(const cbm_eyelid_protocol &p, cudaStream_t s, const DevProtocol *sv = nullptr);
	std::string setStateVarInput(const cbm_statevar_input &in, cudaStream_t s);
	std::string stateVarRates(uint64_t row, float *out, cudaStream_t s);
	// Allocate and start the protocol's GR peri-stimulus histogram.
	std::string recordGR(cudaStream_t s);
	bool recordsGR() const { return hProto_.grPSH != nullptr; }
	std::string recordTrialData(cudaStream_t s);
	bool recordsTrialData() const { return hProto_.tdPSH != nullptr; }
	bool trialDataRecord(int kind, size_t *offset, size_t *count) const;
	bool hasProtocol() const { return h_.proto != nullptr; }
	size_t recordBytes(int kind) const;
	std::string readRecord(int kind, void *dst, size_t bytes, cudaStream_t s);
	// MF spikes for steps [t0, t0+n) as bit rows, into the ring.
	std::string uploadMFBits(const uint32_t *bits, uint64_t firstSlot, uint64_t n, cudaStream_t s);
	uint64_t stepsDone() const { return hostT_; }
	const DevNet &dev() const { return h_; }
	DevNet *devPtr() const { return (DevNet *)dNet_.ptr; }
	State *state() { return st_; }
	uint32_t passBlocks() const { return h_.numPC * h_.tilesPerPC; }
	size_t passSmemBytes() const;
	size_t tailSmemBytes() const;
	// bytes of the staging block the microzone CTA copies, 0 when not staged
	uint32_t stageBytes() const { return h_.numZoneSegs ? h_.zoneStageBytes : 0; }
	// TMA GR pass: possible when every row of the reduction tile is 32 cells
	// Re-upload the host copy of the descriptor (h_) to the device.
	std::string uploadDesc();
	// Switch the small-cell update between pass-made PF->PC input sums (the
	// vector pass) and partial sums, converting the last steps' buffers.
	std::string setPcSumMode(bool on, cudaStream_t s);
	bool passTmaCapable() const { return h_.J == 32; }
	uint32_t passRows() const { return 2 * h_.K; }
	// Encode the TMA descriptors for boxes of R rows and upload them.
	std::string buildPassMaps(uint32_t R);
	size_t passTmaSmemBytes(uint32_t R, uint32_t S, uint32_t outBytes = 4) const;
	size_t zoneScratchBytes() const;
	// shared memory a small-cell CTA may use (the staged arrays included)
	static constexpr size_t kTailSmemBudget = 200 * 1024;
	uint32_t mfWords() const { return h_.mfWords; }
	uint32_t mfRing() const { return h_.mfRing; }
	double bytesPerStepAlgorithmic() const;  // 72 + 4 n_mf + 4 n_go + 8 n_out per GR
	double bytesPerStepLayout() const;       // what this layout moves (see cbm_sim_layout_bytes_per_step)

	HostCtl ctl{};
	bool ctlDirty = true;
	uint64_t hostT_ = 0;
	std::vector<uint32_t> stagedBits;
	std::vector<uint8_t> stagedRaw;

private:
	friend class Simulator;
	template <typename T> T *alloc(size_t n);
	template <typename T> T *upload(const T *src, size_t n);
	State *st_ = nullptr;
	DevNet h_{};
	DeviceBuf dNet_;
	std::string buildZoneStaging();
	void release(void *p);   // free one of allocs_
	void *zoneBlock_ = nullptr;  // staging block (owned through dNet_), or null
	DevProtocol hProto_{};  // host copy of the protocol descriptor
	std::vector<void *> allocs_;
	std::map<const void *, size_t> allocBytes_;
	double avgMF_ = 0, avgGO_ = 0, avgOut_ = 0;
	uint32_t outBytes_ = 4;  // bytes per GR->GO slot the GR pass in use streams
	uint32_t outPlanes_ = 0; // GR->GO slot planes it streams
	size_t ovEntries_ = 0;   // GR->GO synapses in the per-tile lists
	size_t ovUsed_ = 0;      // those the GR pass in use reads (0 unless the per-tile pass)
	// pinned staging of host MF input: kMFStage slots, each reused once the
	// copy that last read it has run (mfStageEv_)
	uint32_t *hErr_ = nullptr;  // the error word (mapped pinned host memory; h_.errFlag maps it)
	// NC mailbox (mapped pinned host memory): step stamp, then every zone's
	// NC spikes, written by the small-cell kernel of single-step launches
	uint8_t *hMailbox_ = nullptr, *dMailbox_ = nullptr;
	uint32_t *hPinnedBits_ = nullptr;
	uint8_t *hPinnedRaw_ = nullptr;
	cudaEvent_t mfStageEv_[kMFStage] = {};
	bool mfStageUsed_[kMFStage] = {};
	uint32_t mfStageNext_ = 0;
};

std::string cudaErr(cudaError_t e, const char *what);

}  // namespace cbm
