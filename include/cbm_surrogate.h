/* The sweep surrogate: a small ReLU MLP (nIn -> h1 -> h2 -> nOut) that
 * predicts a trial's response (for example the NC rate trace of an eyelid
 * trial) from a parameter vector, trained and evaluated on the GPU by this
 * library's own BF16 tensor-core kernels (tcgen05, FP32 accumulation in
 * tensor memory).  No counterpart in the reference, which simulates every
 * candidate of a parameter sweep.  Layers are at most 256 wide; every call
 * takes host arrays, row-major, one sample per row.  Status codes and
 * cbm_last_error() as in cbm_b200.h. */
#ifndef CBM_SURROGATE_H
#define CBM_SURROGATE_H
#include <stdint.h>
#include "cbm_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct cbm_mlp cbm_mlp;

/* He-uniform initial weights from seed, zero biases; maxBatch samples per
 * device pass. */
int cbm_mlp_create(unsigned nIn, unsigned h1, unsigned h2, unsigned nOut, unsigned maxBatch, uint64_t seed, int device,
		cbm_mlp **out);
void cbm_mlp_destroy(cbm_mlp *mlp);

/* Parameters as one FP32 vector: W1 [H1][I], b1 [H1], W2 [H2][H1], b2 [H2],
 * W3 [O][H2], b3 [O] with every size padded to a multiple of 64 (padding
 * entries are zero and stay zero); cbm_mlp_layout gives the padded sizes. */
uint64_t cbm_mlp_num_params(cbm_mlp *mlp);
int cbm_mlp_layout(cbm_mlp *mlp, unsigned *I, unsigned *H1, unsigned *H2, unsigned *O);
int cbm_mlp_get_params(cbm_mlp *mlp, float *params, uint64_t count);
/* Also resets the optimiser state. */
int cbm_mlp_set_params(cbm_mlp *mlp, const float *params, uint64_t count);

/* y[batch][nOut] = MLP(x[batch][nIn]). */
int cbm_mlp_forward(cbm_mlp *mlp, const float *x, unsigned batch, float *y);
/* Gradients (same layout as the parameters) of the mean squared error
 * between MLP(x) and target over batch <= maxBatch samples; *loss (may be
 * NULL) receives the loss. */
int cbm_mlp_gradients(cbm_mlp *mlp, const float *x, const float *target, unsigned batch, float *grads, float *loss);
/* epochs of Adam (lr, beta 0.9 / 0.999) over count samples in shuffled
 * minibatches of batch (<= maxBatch); *lastLoss: mean loss of the last epoch. */
int cbm_mlp_train(cbm_mlp *mlp, const float *x, const float *target, unsigned count, unsigned batch, unsigned epochs,
		float lr, uint64_t seed, float *lastLoss);

#ifdef __cplusplus
}
#endif
#endif
