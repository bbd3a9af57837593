/* qb_mlp.h -- the lambda-placement network on the tensor cores.
 *
 * No counterpart in the reference: QligFEP places lambda windows with a fixed
 * schedule (get_lambdas, src/QligFEP/qligfep.py:414-445).  This network
 * predicts, from a coarse pilot run of a perturbation, where a given number of
 * windows should go.  It is a 12 -> 64 -> 64 -> 11 perceptron with SiLU
 * activations, run and trained by hand-written tcgen05 kernels: BF16
 * operands, FP32 accumulation in tensor memory, FP32 master weights and Adam.
 *
 * Parameters are one float vector: W1[64][12], b1[64], W2[64][64], b2[64],
 * W3[11][64], b3[11] (row = output unit).  All buffers are host memory; every
 * call copies in, runs one kernel launch on `device` and copies out.
 */
#ifndef QB_MLP_H
#define QB_MLP_H

#ifdef __cplusplus
extern "C" {
#endif

#define QB_MLP_IN 12
#define QB_MLP_HIDDEN 64
#define QB_MLP_OUT 11
#define QB_MLP_NPARAM 5707          /* 64*12 + 64 + 64*64 + 64 + 11*64 + 11 */
#define QB_MLP_MAX_SAMPLES 4096

typedef struct qb_mlp_adam {
  float lr, beta1, beta2, eps;
  float weight_decay;   /* decoupled (AdamW): every step also subtracts lr*weight_decay*w from each weight */
} qb_mlp_adam;

/* y[n][11] = network(x[n][12]). */
int qb_mlp_forward(const float *params, const float *x, int n, float *y, int device);

/* Mean squared error over the n x 11 outputs against t, and its gradient
 * with respect to every parameter (same layout as params). */
int qb_mlp_loss_grad(const float *params, const float *x, const float *t, int n, float *loss, float *grad,
                     int device);

/* iters full-batch Adam steps on the mean squared error, all inside one launch;
 * params is updated in place and loss_history[iters] receives the loss of
 * every step (before that step's update). */
int qb_mlp_train(float *params, const float *x, const float *t, int n, int iters, const qb_mlp_adam *adam,
                 float *loss_history, int device);

/* Polls each tensor-core completion wait of the network kernel makes before it
 * gives up (process-wide; the default, 2^26, is seconds).  A wait that gives up
 * makes the call return QB_ERR_TIMEOUT after the kernel has drained its
 * in-flight tensor-core work and released its tensor memory, so the context
 * stays usable.  0 makes every wait give up at once, which is how the time-out
 * path is tested; pass 67108864 to restore the default. */
#define QB_MLP_DEFAULT_WAIT_LIMIT 67108864LL
int qb_mlp_set_wait_limit(long long polls);

#ifdef __cplusplus
}
#endif
#endif
