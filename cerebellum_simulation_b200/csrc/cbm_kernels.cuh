// Kernel entry points of the step (definitions in cbm_kernels.cu).
#pragma once
#include <cstdint>
#include "cbm_device.cuh"

namespace cbm {

constexpr int kPassThreads = 256;
// 24 warps: at 80 registers a thread the small-cell update keeps every value
// in registers (at 1024 threads, 64 registers, it spilled, and the spill
// reloads went to L2 between its phases)
constexpr int kTailThreads = 768;

// Programmatic dependent launch between the two kernels of consecutive
// steps.  Steps launched one at a time run as small-cell(t) -> pass(t) ->
// small-cell(t+1) -> ..., each launched as the programmatic dependent of the
// kernel before it, so that the next kernel is resident before its
// predecessor ends.  Two rules keep that equal to full stream order:
//  - the small-cell kernel waits for its predecessor (the previous step's
//    GR pass) before it reads anything, and only then lets its own
//    dependent (this step's GR pass) launch;
//  - the last CTA of such a GR pass to finish waits for its predecessor
//    (this step's small-cell kernel) before it exits, so that a finished
//    GR pass means a finished step (passExitWait).
// A pass lets the next small-cell kernel launch from its start.  Launched
// without the attribute (CUDA graphs), each wait returns at once.
__device__ __forceinline__ void pdlWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdlLaunchDependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
// At the end of a GR-pass CTA, after a barrier of the whole CTA: with a
// counter (chained single steps), the launch's last CTA to get here resets
// it and waits for the step's small-cell kernel; the others exit, so that
// the slots of early CTAs go to later waves.
__device__ __forceinline__ void passExitWait(uint32_t *exitCount)
{
	if (exitCount && threadIdx.x == 0 && atomicAdd(exitCount, 1u) == gridDim.x - 1u) {
		*exitCount = 0;
		pdlWait();
	}
}

__global__ void grPassKernel(const DevNet *const *nets, const uint32_t *blockOffset, int numNets,
		uint32_t stepOffset);
// TMA GR pass with W consumer warps of RW rows each per stage, S stages
// deep, at least B resident CTAs per SM, synapse-slot loops bounded by M
// (0: any count), compiled for network shape `shape` (0: any network; see
// passShapeOf); launched with 32 * (W + 1) threads, the grPassKernel
// arguments and the descriptor of a single network (null for a batch).
// Returns null for a geometry that is not compiled in.
const void *passTmaKernelFor(int W, int RW, int S, int B, int M, int shape);
// The most specific pass shape a network matches (0 when none).
int passShapeOf(const DevNet &h);
// The compiled per-tile geometries, in table order.
int passTmaConfigCount();
void passTmaConfig(int i, int *W, int *RW, int *S, int *B, int *M);
// Persistent single-network TMA GR pass: W consumer warps (2W rows per
// unit), S stages, B resident CTAs per SM, slot bound M; grid of any size,
// 32 * (W + 1) threads, the grPassKernel arguments with one network.
const void *passPersistentKernelFor(int W, int S, int B, int M);
// Vector GR pass (cbm_pass_vec.cu): single network of the compiled shape,
// kVecWarps warps per CTA, arguments (descriptor, stepOffset, units per
// claim), passVecSmemBytes of dynamic shared memory.  The first
// passVecReduceCTAs CTAs take the previous step's PF->PC reduction; the
// others are persistent and claim units of 128 cells from DevNet::passClaim.
constexpr int kVecWarps = 8;
constexpr int kVecMinBlocks = 3;
constexpr uint32_t kVecClaim = 2;
constexpr uint32_t kVecBatchClaim = 8;
constexpr int kVecBatchMinBlocks = 2;
// The batched form (several networks of the shape; arguments nets,
// unitOffset, pcOffset, numNets, stepOffset, claim counters [3]).
const void *passVecBatchKernel();
bool passVecCapable(const DevNet &h);
size_t passVecSmemBytes(const DevNet &h);
uint32_t passVecReduceCTAs(const DevNet &h);
const void *passVecKernel();
// pairReduceKernel(N, t): step t's PF->PC running sums from its pair sums
// (numPC * bs threads), for a switch away from the vector pass.
const void *pairReduceKernelFn();
// pcTreeKernel(N, t): step t's PF->PC input sums (pcSum) from its partial
// sums, one block of 256 threads per PC, for a switch to the vector pass.
const void *pcTreeKernelFn();
// Small-cell update; stageBytes[n] is network n's staging block size (0:
// its microzone CTA works on global memory).  With one network, net0 and
// stage0 give its descriptor and staging size directly (else null, 0).
// ncMailbox (one network, or null): mapped host memory that receives the
// step's NC spikes and then the step number (publishNC).  mfp.n > 0 (one
// network): the step's MF spike words, which the Golgi CTA also writes into
// the MF ring for the kernels after the step.
__global__ void tailKernel(const DevNet *const *nets, const uint32_t *stageBytes, uint32_t stepOffset,
		const DevNet *net0, uint32_t stage0, uint8_t *ncMailbox, const __grid_constant__ MFParam mfp);
__global__ void protocolPrimeKernel(const DevNet *N);
// GR peri-stimulus histogram of step t = stepsDone(N) + 1 + stepOffset, after
// the GR pass of that step: 8 GR per thread.
__global__ void grPSHKernel(const DevNet *N, uint32_t stepOffset);
__global__ void trialDataKernel(const DevNet *N, uint32_t stepOffset);
// All networks of a batch: cellOffset[n] is the first grid thread of network
// n's small cells (cellOffset[numNets] the total).
__global__ void trialDataBatchKernel(const DevNet *const *nets, const uint32_t *cellOffset, int numNets,
		uint32_t stepOffset);
__global__ void advanceStepKernel(uint64_t *const *tBases, int numNets, uint32_t steps);
__global__ void extractSpikesKernel(const uint32_t *apBuf, uint8_t *out, uint32_t n);
__global__ void flushReadKernel(const uint4 *buf, size_t n, uint32_t *sink);
__global__ void expfProbeKernel(const float *in, float *out, uint32_t n);
__global__ void expProbeKernel(const double *in, double *out, uint32_t n);
// The state-variable input's MF rates for row `row` of its values.
__global__ void stateVarRatesKernel(const DevNet *N, uint64_t row, float *out);

}  // namespace cbm
