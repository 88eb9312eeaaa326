/* ym_learned.h -- the learned SU(3) Metropolis proposal: network shape,
 * parameter layout, feature and objective definitions, C ABI.
 *
 * No reference counterpart: the reference samples SU(3) with a fixed
 * proposal (su3_ensemble.rs:342-391) and judges samplers by the
 * integrated-autocorrelation ESS of a measured series
 * (su2_ensemble.rs:375-463, sampling_efficiency.rs:57-135).  This proposal is
 * judged the same way, against plain Metropolis.
 *
 * Proposal.  For a link visit with staple sum A (the matrix whose product
 * with the link gives the local plaquette sum, ReTr(U A)), a small network
 * maps sixteen gauge-invariant features of A alone to eight generator
 * logits and one angle-scale output.  Each of the visit's eight hits draws
 * a generator a with probability p_a = F/8 + (1 - F) softmax(logits)_a
 * (F = YM_LP_GENERATOR_FLOOR keeps every direction in play, so the chain
 * stays ergodic however the logits train) from bits 52..62 of its angle
 * word, an angle theta on the reference's paired grid with half width
 * s = SCALE_MIN + (SCALE_MAX - SCALE_MIN) * sigmoid(y8), proposes
 * exp(i theta T^a) U and accepts iff u < exp(-max(dS, 0)) with dS in
 * binary64.  A is fixed during the visit and the features do not depend on
 * U, so q(U'|U) = q(U|U') for every hit: the proposal is symmetric and the
 * exact accept/reject keeps detailed balance without a Hastings ratio.
 *
 * Features of A (Ah = A/6, B = Ah Ah^dagger, d = det Ah, all invariant under
 * A -> g A h^dagger for g, h in SU(3)):
 *   t1 = ReTr B / 3, t2 = Tr(B B) / 3, t3 = ReTr(B B B) / 3, k = beta sqrt(t1)
 *   f = [t1, t2, t3, sqrt(t1), Re d, Im d, |d|^2, t2 - t1^2, beta/6, k/6,
 *        (k/6)^2, 1/(1+k), (beta/6) Re d, (beta/6) t2, (beta/6)|d|^2,
 *        (beta/6)(t2 - t1^2)]
 *
 * Network.  x = bf16(f); h1 = bf16(relu(W1 x + b1)); h2 = bf16(relu(W2 h1 +
 * b2)); y = W3 h2 + b3; BF16 weights and activations, FP32 accumulation.
 * Outputs 0..7 are the generator logits, output 8 the scale, outputs 9..15
 * are padding kept at zero.
 *
 * Objective (training).  The expected squared change of the local action
 * in one hit (the plaquette is the action, so this is the per-hit motion of
 * the observable the sampler is judged on) plus an entropy term that keeps
 * the generator logits near uniform unless a consistent gain moves them
 * (E is linear in the probabilities, so without it gradient noise alone
 * drifts the softmax onto one generator),
 *   O = E + YM_LP_ENTROPY_WEIGHT * H(q),  H(q) = -sum_a q_a log q_a,
 *   q = softmax(logits),
 *   E = sum_a p_a * (1/2K) sum_{k, +-} alpha(dS_a(theta)) dS_a(theta)^2,
 *   theta = +-s (k + 1/2)/K, K = YM_LP_QUADRATURE,
 *   alpha = min(1, exp(-dS)),  dS_a(theta) = (beta/3)(ReTr M - ReTr(R_a(theta) M)),
 * M = U A, R_a(theta) = exp(i theta T^a); training maximises the mean of O
 * over the links of one checkerboard sub-sweep per configuration with Adam.
 */
#ifndef YM_LEARNED_H
#define YM_LEARNED_H

#include <stdint.h>

#include "ym_status.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    YM_LP_FEATURES = 16,
    YM_LP_HIDDEN = 64,
    YM_LP_OUTPUTS = 16,      /* 9 used: 8 generator logits + scale */
    YM_LP_USED_OUTPUTS = 9,
    YM_LP_QUADRATURE = 4,
    /* fp32 parameter vector: W1[64][16] b1[64] W2[64][64] b2[64] W3[16][64] b3[16],
     * weights row-major [out][in] */
    YM_LP_OFF_W1 = 0,
    YM_LP_OFF_B1 = 1024,
    YM_LP_OFF_W2 = 1088,
    YM_LP_OFF_B2 = 5184,
    YM_LP_OFF_W3 = 5248,
    YM_LP_OFF_B3 = 6272,
    YM_LP_PARAMS = 6288
};

#define YM_LP_SCALE_MIN 0.05
#define YM_LP_SCALE_MAX 2.5
#define YM_LP_GENERATOR_FLOOR 0.5
#define YM_LP_ENTROPY_WEIGHT 0.02

typedef struct ym_ensemble ym_ensemble;
typedef struct ym_proposal_model ym_proposal_model;

/* A model on a device: fp32 master parameters, Adam moments, the BF16
 * weight image the kernels stage into shared memory, and training buffers.
 * Parameters start from a seeded He-uniform draw with the last layer scaled
 * by 1/8, zero generator logits and the scale bias set so that s equals
 * initial_scale. */
int32_t ym_model_create(int32_t device, uint64_t seed, double initial_scale,
                        ym_proposal_model **out);
int32_t ym_model_destroy(ym_proposal_model *model);
int32_t ym_model_get_params(ym_proposal_model *model, float *params /* YM_LP_PARAMS */);
/* Replaces the parameters (padding outputs 9..15 are zeroed) and resets Adam. */
int32_t ym_model_set_params(ym_proposal_model *model, const float *params);

/* Network outputs y[n][16] for host features x[n][16] (tensor-core forward). */
int32_t ym_model_forward(ym_proposal_model *model, const float *features, int64_t n,
                         float *outputs);
/* Objective and gradient over host records, without an update:
 * features[n][16], m[n][18] (U A, row-major re/im), beta[n];
 * objective = mean O, grad[YM_LP_PARAMS] = d(-mean O)/d params. */
int32_t ym_model_gradient(ym_proposal_model *model, const float *features, const float *m,
                          const double *beta, int64_t n, double *objective, float *grad);

/* Training records of one checkerboard sub-sweep (parity, mu) of every chain
 * of an SU(3) two-row ensemble, in chain order then storage order within the
 * parity: features[n][16], m[n][18] and the chain's beta; n_out receives the
 * record count (sum of V/2).  Pass NULL buffers to query n_out only. */
int32_t ym_learned_records(ym_ensemble *ens, int32_t parity, int32_t mu, float *features,
                           float *m, double *beta, int64_t *n_out);

/* On-device training: n_steps times {sweeps_per_step plain sweeps of ens
 * (uniform generators, half width plain_angle), records of sub-sweep
 * (step mod 8), objective and gradient, one Adam step with learning rate lr
 * (beta1 0.9, beta2 0.999, eps 1e-8)}.  objective_history[n_steps] receives
 * the objective of each step before its update (may be NULL). */
int32_t ym_model_train(ym_proposal_model *model, ym_ensemble *ens, int64_t n_steps,
                       int64_t sweeps_per_step, double plain_angle, double lr,
                       double *objective_history);

/* n_sweeps learned-proposal checkerboard sweeps of an SU(3) two-row
 * ensemble (same stream keys, sub-sweep order, accounting and per-sweep
 * reunitarisation as ym_su3_metropolis_sweeps). */
int32_t ym_su3_learned_sweeps(ym_ensemble *ens, ym_proposal_model *model, int64_t n_sweeps);
/* The measured cadence of ym_su3_measured_sweeps with learned sweeps. */
int32_t ym_su3_learned_measured_sweeps(ym_ensemble *ens, ym_proposal_model *model,
                                       int64_t n_measurements, int64_t sweeps_per_measurement,
                                       double *series);

/* Failure detection of the tensor-core kernels: every wait for an MMA group
 * gives up after a time limit, sets an error bit and returns, and the host
 * reports YM_ERR_DEVICE_WAIT_TIMEOUT.  This runs that wait on a barrier that
 * nothing completes, with limit_ns in [1e3, 1e9]; it returns
 * YM_ERR_DEVICE_WAIT_TIMEOUT when the wait gave up as designed (and leaves
 * the device usable), YM_OK would mean the wait did not run. */
int32_t ym_device_wait_selftest(int32_t device, int64_t limit_ns);

#ifdef __cplusplus
}
#endif

#endif /* YM_LEARNED_H */
