/*
 * les_mlp.h -- C ABI of the learned sub-grid closure: a per-point multilayer
 * perceptron evaluated and trained on the sm_100a tensor cores.
 *
 * The closure has no counterpart in the reference: it replaces the eddy
 * viscosity of complen.f90:1-28 and the stresses of compsgs1.f90:1-53
 * (tau_ij = -2 nu_t S_ij) with tau_ij predicted from the local resolved
 * velocity gradients.  The solver uses it when its configuration has
 * imodel = LES_SGS_LEARNED (les_gpu.h) and a network is attached with
 * les_gpu_set_mlp; stages whose mean dissipation -<tau_ij S_ij> comes out
 * negative, or (les_gpu_set_learned_guard) outside a factor of the
 * Smagorinsky-Lilly estimate, fall back to the Deardorff stresses.
 *
 * Network: 11 -> 64 -> 64 -> 64 -> 6, GELU (tanh form) after the hidden
 * layers, bf16 weights and activations, f32 accumulation.  The closure is
 * dimensionless, so that one network serves every grid and filter width
 * Delta = (dx dy dz)^(1/3):
 *   inputs  x = (ux, vx, wx, uy, vy, wy, uz, vz, wz) / |G|  (|G| the
 *           Frobenius norm of the nine resolved gradients at the cell
 *           centre), min(z_w / Delta, 16), z_w / h  (z_w the distance to the
 *           nearest wall, h = zl / 2), normalised as
 *           x_j' = (x_j - in_shift_j) * in_scale_j
 *   outputs y -> c = y * out_scale + out_shift and
 *           tau_ij = (Delta |G|)^2 c_ij for
 *           (tau11, tau22, tau33, tau12, tau13, tau23)
 * Parameters (LES_MLP_NPARAM floats, this order):
 *   W1[64][11], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[6][64], b4[6]
 * Normalisation (LES_MLP_NNORM floats):
 *   in_shift[11], in_scale[11], out_scale[6], out_shift[6]
 *
 * Operator entry points take device pointers and a CUDA stream (NULL = the
 * legacy default stream); they return 0 or an LES_E* code of les_gpu.h.
 */
#ifndef LES_MLP_H
#define LES_MLP_H

#include "les_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LES_MLP_NIN    11
#define LES_MLP_NHID   64
#define LES_MLP_NOUT   6
#define LES_MLP_NPARAM 9478
#define LES_MLP_NNORM  34
/* Sample layouts on the device: features bf16 [n][16] (normalised inputs in
 * columns 0..10; the network ignores 11..15), outputs and targets f32 [n][8]
 * (columns 6, 7 unused). */
#define LES_MLP_FEAT_STRIDE 16
#define LES_MLP_OUT_STRIDE  8

typedef struct les_mlp les_mlp;

int les_mlp_create(int device, les_mlp** out);
void les_mlp_destroy(les_mlp* m);
const char* les_mlp_last_error(const les_mlp* m);

/* Host arrays: params[LES_MLP_NPARAM], norm[LES_MLP_NNORM].  Setting the
 * parameters also resets the optimiser state. */
int les_mlp_set_params(les_mlp* m, const float* params, const float* norm);
int les_mlp_get_params(les_mlp* m, float* params, float* norm);

/* Limit of each wait for a tensor-core MMA in this network's kernels
 * (inference in les_mlp_forward and in the solver's learned stage,
 * training in les_mlp_loss_grad / les_mlp_adam_step); default 1 s, range
 * [0, 60] s.  A wait that runs out makes the kernel give up its tiles,
 * drain the outstanding MMA (bounded by a fixed 1 s), release its tensor
 * memory and return; the host then sees LES_ETIMEOUT (les_mlp_loss_grad,
 * les_mlp_adam_step, or les_gpu_sync of a handle using the network) and the
 * CUDA context stays usable.  0 gives up at the first poll that finds an
 * MMA unfinished, which tests use to exercise that path.  Synchronises the
 * device. */
int les_mlp_set_wait_limit(les_mlp* m, double seconds);

/* y[n][8] = network(feat[n][16]) in normalised units (asynchronous). */
int les_mlp_forward(les_mlp* m, const void* feat, long long n, float* y, void* stream);

/* Mean-squared error over the n samples and 6 outputs, and its gradient
 * grad[LES_MLP_NPARAM] (device, flat parameter order).  Synchronous. */
int les_mlp_loss_grad(les_mlp* m, const void* feat, const float* target, long long n, float* grad, double* loss,
                      void* stream);

/* One Adam step (Kingma & Ba 2015; beta1 0.9, beta2 0.999, eps 1e-8, bias
 * corrected) on f32 master parameters from the gradient of the batch; the
 * bf16 copies used by the kernels are refreshed.  *loss (optional) receives
 * the batch loss before the step, which makes the call synchronous. */
int les_mlp_adam_step(les_mlp* m, const void* feat, const float* target, long long n, float lr, double* loss,
                      void* stream);

/* Attach (or with m == NULL detach) a network to a solver handle whose
 * configuration has imodel = LES_SGS_LEARNED.  re_tau (> 0) is the run's
 * friction Reynolds number, recorded with the network; the features do not
 * depend on it.  Resets the stage counters of les_gpu_learned_counts.  The
 * handle keeps a reference to m: destroy the handle first. */
int les_gpu_set_mlp(les_handle* h, les_mlp* m, double re_tau);

/* After a synchronising call: 1 if the last stage used the network (0 if
 * it fell back to the Deardorff stresses) and that stage's mean
 * dissipation -<tau'_ij S_ij> of the applied (projected) stresses. */
int les_gpu_learned_status(les_handle* h, int* used, double* dissipation);

/* The stress the solver applies is the network's with its local
 * backscatter removed: where tau_ij S_ij > 0 (energy flowing from the
 * sub-filter to the resolved scales) the component along S is subtracted,
 * tau' = tau - (tau:S / S:S) S, so the applied stress never injects energy
 * at a point.
 *
 * The fallback test of each stage: the network is used when the mean
 * dissipation -<tau_ij S_ij> of its raw prediction is >= 0 (the spec'd
 * test) and, with ratio > 0, the applied mean -<tau'_ij S_ij> lies within a
 * factor ratio of the reference <(C_s Delta)^2 |S|^3>, the Smagorinsky
 * estimate with Lilly's constant C_s = 0.17, |S| = (2 S_ij S_ij)^(1/2), on
 * the same state.  The second test keeps a network out of states whose
 * sub-filter dissipation it would misjudge by more than that factor.
 * Default ratio 4; ratio <= 0 disables it.  Drops the handle's captured
 * step graphs. */
int les_gpu_set_learned_guard(les_handle* h, double ratio);
/* After a synchronising call: the reference (Smagorinsky) mean dissipation
 * of the last learned stage. */
int les_gpu_learned_reference(les_handle* h, double* dissipation);
/* Stages evaluated with the network attached since les_gpu_set_mlp, and
 * how many of them used it (synchronising). */
int les_gpu_learned_counts(les_handle* h, long long* stages, long long* used);

/* Training data (synchronous; out pointers are device memory).
 *
 * les_gpu_learn_filter: explicit filter of the handle's current state onto
 * the grid (nnx/fxy, nny/fxy, nnz/fz), fz = 1 or 2: box average over the
 * fine cells in z, box-filter transfer sin(k D/2)/(k D/2) with D the coarse
 * cell size and truncation to the coarse modes in x and y.  out: 9 planes
 * of (nnz/fz, nny/fxy, nnx/fxy) doubles, in order u, v (cell centres),
 * w (coarse w-levels), tau11, tau22, tau33, tau12, tau13, tau23 with
 * tau_ij = filt(u_i u_j) - filt(u_i) filt(u_j) (w averaged to the centres);
 * with_model != 0 adds the filtered Deardorff stress of the fine run,
 * -2 nu_t S_ij with nu_t = 0.1 dsl sqrt(e) at the fine cell centres, so
 * tau_ij is the total sub-filter stress the coarse grid misses.  fz is 1 or
 * even; w at the coarse faces is the z box of fz fine cells centred on the
 * face (trapezoid weights).
 *
 * les_gpu_learned_features: the network's raw inputs at every cell centre
 * of the current state, f32 [nnx*nny*nnz][16]: columns 0..10 the inputs x
 * above, unnormalised; column 11 Delta |G|; 12..15 zero.  Computed by the
 * kernels the learned stage uses. */
int les_gpu_learn_filter(les_handle* h, int fxy, int fz, int with_model, double* out);
int les_gpu_learned_features(les_handle* h, float* feat);

#ifdef __cplusplus
}
#endif

#endif /* LES_MLP_H */
