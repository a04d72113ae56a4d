/*
 * C ABI of the B200 multislice mixed-probe ptychography path.
 *
 * Every entry point takes raw device pointers, sizes and a cudaStream_t passed
 * as void* (NULL = legacy default stream), launches asynchronously on that
 * stream and returns a status code (PTYCHO_OK = 0).  On failure a message is
 * kept per host thread and returned by ptycho_get_last_error().  Nothing here
 * allocates device memory: callers (the Python host layer uses the PyTorch
 * caching allocator) pass every buffer, including scratch.  Complex arrays are
 * interleaved float32 pairs (complex64), C-contiguous.
 *
 * Reference interfaces replaced (quantem 0.1.8, src/quantem/diffractive_imaging):
 *   ptycho_forward_loss      probe_models.py:718-720 (ProbePixelated.forward),
 *                            object_models.py:678-680 (ObjectPixelated.forward),
 *                            ptychography_base.py:892-906 (forward_operator),
 *                            detector_models.py:22-30 (DetectorPixelated.forward),
 *                            ptychography_base.py:908-932 (error_estimate)
 *   ptycho_forward_adjoint   the above plus loss.backward() of ptychography.py:326-328
 *   ptycho_obj_constrain     object_models.py:289-300 (apply_hard_constraints, complex)
 *   ptycho_obj_constrain_vjp autograd of the same constraint
 *   ptycho_obj_transmission, object_models.py:289-339 for complex, pure-phase and
 *   ptycho_obj_transmission_vjp potential objects (+ exp(i V), object_models.py:252-256)
 *                            and their autograd
 *   ptycho_fft2              torch.fft.fft2/ifft2 of the probe stack
 *                            (ptycho_utils.py:133-135) and of the probe gradient
 *   ptycho_probe_orthogonalize,
 *   ptycho_probe_orthogonalize_vjp
 *                            probe_models.py:484-525 (_probe_orthogonalization_constraint)
 *                            and its autograd
 *   ptycho_probe_center,
 *   ptycho_probe_center_vjp  probe_models.py:467-482 (_probe_center_of_mass_constraint)
 *                            and its autograd
 *   ptycho_probe_tv          probe_models.py:460-466 (_probe_tv_constraint) and its gradient
 *   ptycho_reduce_partials,
 *   ptycho_reduce_loss       deterministic reductions of per-CTA partials
 *   ptycho_adam_step,
 *   ptycho_sgd_step          torch.optim.Adam/AdamW/SGD step (optimizer_mixin.py:117-123,
 *                            ptychography_opt.py:336-344)
 */
#ifndef PTYCHO_B200_H
#define PTYCHO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PTYCHO_OK = 0,
  PTYCHO_ERR_INVALID = 1,     /* bad pointer, size, alignment or option */
  PTYCHO_ERR_UNSUPPORTED = 2, /* probe size / configuration not built */
  PTYCHO_ERR_CUDA = 3,        /* CUDA launch or runtime error */
  PTYCHO_ERR_NONFINITE = 4    /* reserved: non-finite values detected */
};

enum {
  PTYCHO_LOSS_L2_AMPLITUDE = 0,
  PTYCHO_LOSS_L1_AMPLITUDE = 1,
  PTYCHO_LOSS_L2_INTENSITY = 2,
  PTYCHO_LOSS_L1_INTENSITY = 3,
  PTYCHO_LOSS_POISSON = 4
};

/* Arguments of one position batch.  Shapes: S slices, P probe modes, N x N probe
 * window (N = 64 or 128), object Ho x Wo, npos scan positions, B positions in
 * this batch, grid CTAs. */
typedef struct ptycho_batch_args {
  const void* obj;           /* complex64 (S, Ho, Wo): hard-constrained object */
  const void* probe_hat;     /* complex64 (P, N, N): fft2 of the probe modes */
  const void* prop;          /* complex64 (S-1, N, N): Fresnel propagators (may be NULL if S == 1
                                or if prop_r/prop_c are given) */
  const float* positions;    /* float32 (npos, 2): scan positions [px] (row, col) */
  const int64_t* batch_idx;  /* int64 (B,): positions / targets rows of this batch */
  const float* targets;      /* float32 (npos, N, N): measured amplitudes/intensities, detector layout */
  const float* mask;         /* float32 (N, N): detector mask, detector layout */
  void* grad_obj;            /* complex64 (S, Ho, Wo): object gradient, accumulated (adjoint only) */
  void* probe_grad_part;     /* complex64 (grid, P, N, N): per-CTA partials (adjoint only) */
  void* scratch;             /* complex64 (grid, P*S + P + 1, N, N) serial / (grid, S, N, N) cluster
                                (adjoint only); size it with ptycho_batch_plan */
  double* loss_part;         /* float64 (grid,): per-CTA loss partials */
  float* out_intensity;      /* optional float32 (B, N, N): predicted intensities, detector layout */
  void* out_exit;            /* optional complex64 (P, B, N, N): exit waves */
  void* out_waves;           /* optional complex64 (S, P, B, N, N): wave entering each slice */
  int* status;               /* optional int32 status word: bits 0-19 count non-finite predicted
                                intensities, bits 20-30 count batch indices outside [0, npos)
                                (those positions are skipped); each field saturates at its
                                maximum instead of carrying into the next */
  const void* prop_r;        /* optional complex64 (S-1, N): separable propagator factors, */
  const void* prop_c;        /*   K_s[kr][kc] = prop_r[s][kr] * prop_c[s][kc] (kept in shared memory) */
  int n, S, P, B, Ho, Wo, npos, grid;
  int loss_type;             /* PTYCHO_LOSS_* */
  float loss_scale;          /* npos_total / (B * mean_intensity) */
  float inv_mean_intensity;  /* 1 / mean_intensity */
  int variant;               /* PTYCHO_VARIANT_*: how probe modes map onto CTAs */
  int analytic;              /* adjoint launch: 0 = autograd gradients, 1 = analytic update directions
                                (serial variant; needs an_norm and the partials in real space) */
  float* an_norm;            /* analytic: float32 (S, P, Ho, Wo) zero-initialised accumulator of
                                sum_patches(|psi|^2) */
  int recompute_every;       /* n = 256 adjoint: 0 keeps every slice's incident wave; k > 0 keeps the
                                wave entering every k-th slice and recomputes the others in the
                                reverse sweep (smaller scratch, S - S/k extra propagations per mode) */
  float* grad_positions;     /* optional float32 (B, 2), adjoint launch: dL/d(scan position) (row, column)
                                of every batch entry, summed over the modes (serial variant, n < 256,
                                autograd adjoint).  Positions enter through the fractional probe shift
                                only (dataset_models.py:1487-1490, ptycho_utils.py:128-176); entries
                                whose index is invalid are left untouched.  ABI version 2. */
  const float* descan;       /* optional float32 (npos, 2): descan shifts [px] (row, column).  The exit
                                wave is multiplied by exp(-2 pi i (fftfreq(r) d_r + fftfreq(c) d_c)) on
                                the real-space grid before the detector (ptychography_base.py:903-905,
                                ptycho_utils.py:156-176).  Serial variant, n < 256.  ABI version 3. */
  float* grad_descan;        /* optional float32 (B, 2), adjoint launch with descan: dL/d(descan shift)
                                of every batch entry, summed over the modes (autograd adjoint).
                                ABI version 3. */
  float* grad_prop;          /* optional float32 (S-1, 2), zero-filled by the caller, S <= 17; adjoint
                                launch: accumulates, over the batch and the modes, sum_k fftfreq_index(k)
                                Im(conj(dL/dZ_s(k)) Z_s(k)) along rows / columns for the propagated
                                wave Z_s = K_s fft2(chi_s) of every slice.  A per-axis phase ramp
                                exp(-2 pi i a_s fftfreq_index) of K_s changes the loss at the rate
                                2 pi times this sum (the probe tilt, probe_models.py:418-425).  The
                                adjoint then needs the larger scratch that ptycho_batch_plan reports
                                for these arguments.  ABI version 3. */
} ptycho_batch_args;

enum {
  PTYCHO_VARIANT_AUTO = 0,    /* the faster of the two on B200 (currently serial) */
  PTYCHO_VARIANT_SERIAL = 1,  /* one CTA per position, modes in sequence */
  PTYCHO_VARIANT_CLUSTER = 2  /* one thread-block cluster of P CTAs per position */
};

/* Copy the last error message of this host thread into buf (NUL-terminated). */
int ptycho_get_last_error(char* buf, size_t len);

/* Library ABI version (increments on incompatible changes). */
int ptycho_abi_version(void);

/* Number of SMs of the current device. */
int ptycho_sm_count(int* out);

/* Number of complex64 elements of scratch / partial buffers for a batch launch
 * without grad_prop (ptycho_batch_plan sizes every launch). */
int ptycho_workspace_elems(int n, int S, int P, int grid, int64_t* scratch_elems,
                           int64_t* partial_elems);

/* Launch plan of a batch: resolved variant, grid (CTAs) and the complex64
 * element counts of the scratch and probe-gradient partial buffers the adjoint
 * launch needs.  Reads n, S, P, B and variant from *a. */
int ptycho_batch_plan(const ptycho_batch_args* a, int adjoint, int* variant, int* grid, int64_t* scratch_elems,
                      int64_t* partial_elems, int* partial_parts);

/* ---- optional object constraints (object_models.py:273-480) and the FOV mask
 * (ptychography_base.py:191-216).  Objects are (S, Ho, Wo) complex64 or float32,
 * hw = Ho * Wo, count = S * hw; masks are float32 (Ho, Wo).  work: float64 scratch of
 * ptycho_obj_constraint_work_elems() elements.  Every reduction is fixed-order. ---- */

/* float64 elements of the work buffer the functions below need. */
int ptycho_obj_constraint_work_elems(void);

/* out (Ho, Wo) = sum over positions of intensity (n, n) placed at each position's
 * wrapped patch window (rounded half to even), as the reference's probe overlap with
 * |probe mode 0|^2 (ptychography_base.py:201-216). */
int ptycho_probe_overlap(const float* intensity, int n, const float* positions, int npos, int Ho, int Wo, float* out,
                         void* stream);

/* Hard constraint of complex (pure = 0) or pure-phase (pure = 1) objects with the FOV
 * mask m: amp m exp(i (angle - mean angle) m) m (object_models.py:292-300, 322-323; the
 * amplitude carries the mask twice, as in the reference), and its VJP w.r.t. the raw
 * object (grad_raw must not alias obj or grad_c). */
int ptycho_obj_constrain_fov(const void* obj, const float* mask, int64_t hw, void* out, int64_t count, int pure,
                             double* work, int nwork, void* stream);
int ptycho_obj_constrain_fov_vjp(const void* obj, const float* mask, int64_t hw, const void* grad_c, void* grad_raw,
                                 int64_t count, int pure, double* work, int nwork, void* stream);

/* Potential hard constraint (object_models.py:301-323): out = (V - offset), clamped at 0
 * with positivity, times apply_mask (may be NULL).  With fix_baseline the offset is
 * factor * the mean of V over the background pixels of baseline_mask (mask < 0.5 max), or
 * factor * min V when baseline_mask is NULL or has no background.  The VJP treats the
 * offset as a constant (detached, as in the reference). */
int ptycho_obj_potential_base(const float* v, const float* baseline_mask, const float* apply_mask, int64_t hw,
                              float* out, int64_t count, int positivity, int fix_baseline, float factor,
                              double* work, int nwork, void* stream);
int ptycho_obj_potential_base_vjp(const float* v, const float* baseline_mask, const float* apply_mask, int64_t hw,
                                  const float* grad_out, float* grad_v, int64_t count, int positivity,
                                  int fix_baseline, float factor, double* work, int nwork, void* stream);

/* Transmission exp(i V) of a real potential (object_models.py:252-256) and its VJP
 * dL/dV = Re(conj(G) i t). */
int ptycho_phase_exp(const float* v, void* out, int64_t count, void* stream);
int ptycho_phase_exp_vjp(const float* v, const void* grad_t, float* grad_v, int64_t count, void* stream);

/* Gaussian blur of every slice (object_models.py:437-479): zero-padded 'same'
 * correlation with the odd tap vector (<= 255 taps) along the rows, then the columns;
 * complex objects blur their real and imaginary parts.  Self-adjoint, so it is its own
 * VJP.  tmp: a buffer of the object's size, aliasing neither in nor out. */
int ptycho_obj_blur(const void* in, void* out, void* tmp, int S, int Ho, int Wo, int is_complex, const float* taps,
                    int ntaps, void* stream);

/* Butterworth filter (object_models.py:481-520): per slice, mean removed, ifft2(fft2(x)
 * env), mean added back (the real part for a real potential, is_real = 1); env: float32
 * (Ho, Wo) envelope on the fftfreq grid.  The 2-D transform is a direct DFT along each
 * axis (object sides <= 6144).  tmp: complex64 2 * S * Ho * Wo; means: complex64 2 * S.
 * The filter is self-adjoint: the VJP is P g - mean(P g) + mean(g) per slice. */
int ptycho_obj_butterworth(const void* in, void* out, int S, int Ho, int Wo, int is_real, const float* env, void* tmp,
                           void* means, void* stream);
int ptycho_obj_butterworth_vjp(const void* grad_out, void* grad_in, int S, int Ho, int Wo, int is_real,
                               const float* env, void* tmp, void* means, void* stream);

/* identical_slices (object_models.py:330-333): every slice replaced by the mean over the
 * slices (the reference averages in place under no_grad: its VJP is the identity). */
int ptycho_obj_slice_mean(const void* in, void* out, int S, int64_t hw, int is_complex, void* stream);

/* Soft constraints of the hard-constrained object (object_models.py:341-435): kind 0
 * complex (TV and surface terms of phase and amplitude), 1 pure phase (phase terms), 2
 * real potential.  Writes the loss (device float) and its gradient w.r.t. obj (torch
 * convention; zero at zero-magnitude pixels). */
int ptycho_obj_soft_loss(const void* obj, int S, int Ho, int Wo, int kind, float tv_weight_z, float tv_weight_xy,
                         float surface_zero_weight, double* work, int nwork, float* loss, void* grad, void* stream);

/* Forward model + loss of one batch (no gradients). */
int ptycho_forward_loss(const ptycho_batch_args* a, void* stream);

/* Forward model + loss + adjoint of one batch in a single persistent launch. */
int ptycho_forward_adjoint(const ptycho_batch_args* a, void* stream);

/* Largest number of datasets of one ptycho_forward_adjoint_multi launch. */
#define PTYCHO_MAX_DATASETS 16

/* Forward + loss + adjoint of several independent datasets (same n; any S, P,
 * object size, scan size, loss, analytic flag) in one persistent launch of the
 * serial kernel: CTAs are partitioned between datasets by their sets[d].grid
 * (each dataset's buffers sized for its grid with ptycho_batch_plan semantics).
 * Replaces a loop of Ptychography.reconstruct calls over datasets. */
int ptycho_forward_adjoint_multi(const ptycho_batch_args* sets, int nsets, void* stream);

/* count 2-D FFTs of n x n complex64 arrays, out = scale * (i)fft2(in), unnormalised
 * transform; in and out may alias. */
int ptycho_fft2(const void* in, void* out, int count, int n, int inverse, float scale, void* stream);

/* out[i] = sum_g parts[g * count + i] (complex64), fixed summation order. */
int ptycho_reduce_partials(const void* parts, void* out, int nparts, int64_t count, void* stream);

/* out[0] = (float) sum_g parts[g], fixed summation order. */
int ptycho_reduce_loss(const double* parts, int nparts, float* out, void* stream);

/* Complex object hard constraint: out = clamp(|o|,0,1) exp(i(angle(o) - mean angle)).
 * work: float64 scratch of nwork >= 2 * ptycho_reduce_blocks() elements. */
int ptycho_obj_constrain(const void* obj, void* out, int64_t count, double* work, int nwork, void* stream);

/* Gradient of ptycho_obj_constrain: grad_raw = scale[0] * J^H grad_c (torch convention).
 * `work` must be the buffer used by the matching ptycho_obj_constrain call;
 * `scale` is a device float (e.g. autograd's incoming gradient), NULL means 1. */
int ptycho_obj_constrain_vjp(const void* obj, const void* grad_c, void* grad_raw, int64_t count,
                             double* work, int nwork, const float* scale, void* stream);

/* Object types of ptycho_obj_transmission (object_models.py:123-136). */
#define PTYCHO_OBJ_COMPLEX 0    /* complex64 object, amplitude clamped to [0, 1] */
#define PTYCHO_OBJ_PURE_PHASE 1 /* complex64 object, amplitude dropped */
#define PTYCHO_OBJ_POTENTIAL 2  /* float32 potential V, transmission exp(i V) */

/* Transmission the batch kernels multiply by, from the raw object of any type:
 * apply_hard_constraints (object_models.py:289-339) followed by the exp(i V) of
 * _get_obj_patches for potentials (object_models.py:252-256).
 *   complex:    out = clamp(|o|,0,1) exp(i(angle(o) - mean angle))   (= ptycho_obj_constrain)
 *   pure phase: out = exp(i(angle(o) - mean angle))
 *   potential:  V' = V - offset, clamped at 0 when `positivity`; out = exp(i V'); offset =
 *               baseline_factor * min(V) when `fix_baseline`, else 0.
 * obj: complex64 (complex, pure phase) or float32 (potential), `count` elements; out:
 * complex64.  work: float64 scratch of nwork >= 2 * ptycho_reduce_blocks() elements,
 * reused by the matching _vjp call. */
int ptycho_obj_transmission(const void* obj, void* out, int64_t count, int obj_type, int positivity,
                            int fix_baseline, float baseline_factor, double* work, int nwork, void* stream);

/* Gradient of ptycho_obj_transmission w.r.t. the raw object (torch convention; float32
 * for potentials, the offset is detached as in the reference), scaled by the device
 * float scale[0] (NULL means 1).  Same arguments and `work` as the forward call. */
int ptycho_obj_transmission_vjp(const void* obj, const void* grad_t, void* grad_raw, int64_t count, int obj_type,
                                int positivity, int fix_baseline, float baseline_factor, double* work, int nwork,
                                const float* scale, void* stream);

/* Blocks used by the reductions (size of `work` is 2x this). */
int ptycho_reduce_blocks(void);

/* torch.optim.Adam / AdamW step on float32 data viewed as reals.  bc1 = 1 - beta1^t,
 * bc2_sqrt = sqrt(1 - beta2^t); decoupled != 0 selects AdamW weight decay.  lr_dev,
 * if not NULL, is a device float that overrides lr (graph-replay friendly). */
int ptycho_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t count,
                     float lr, const float* lr_dev, float beta1, float beta2, float eps,
                     float weight_decay, int decoupled, float bc1, float bc2_sqrt, void* stream);

/* Adam with the step count held on the device (*step_dev, advanced with
 * ptycho_add_scalar before the update) so that a captured iteration replays
 * with the right bias corrections; lr from *lr_dev. */
int ptycho_adam_step_dev(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t count,
                         const float* lr_dev, const float* step_dev, float beta1, float beta2, float eps,
                         float weight_decay, int decoupled, void* stream);

/* x[0] += v on the device (step counters of captured iterations). */
int ptycho_add_scalar(float* x, float v, void* stream);

/* torch.optim.SGD step without momentum: param -= lr * (grad + wd * param). */
int ptycho_sgd_step(float* param, const float* grad, int64_t count, float lr, const float* lr_dev,
                    float weight_decay, void* stream);

/* torch.optim.Adam / AdamW step with amsgrad=True (optimizer_mixin.py:117-123): as
 * ptycho_adam_step, with max_exp_avg_sq = max(max_exp_avg_sq, exp_avg_sq) in the denominator. */
int ptycho_adam_amsgrad_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                             float* max_exp_avg_sq, int64_t count, float lr, const float* lr_dev, float beta1,
                             float beta2, float eps, float weight_decay, int decoupled, float bc1, float bc2_sqrt,
                             void* stream);

/* torch.optim.SGD step with momentum: g = grad + wd * param; buf = g on the first step
 * (first_step != 0), else momentum * buf + (1 - dampening) * g; param -= lr * (g + momentum *
 * buf) with nesterov, lr * buf otherwise. */
int ptycho_sgd_momentum_step(float* param, const float* grad, float* momentum_buffer, int64_t count, float lr,
                             const float* lr_dev, float weight_decay, float momentum, float dampening, int nesterov,
                             int first_step, void* stream);

/* Analytic (autograd=False) update, finalisation steps after an analytic adjoint launch
 * (a->analytic = 1; object_models.py:686-725, probe_models.py:774-783):
 *   ptycho_patch_energy_max        out[0] = max over slices and batch positions of sum |o_patch|^2
 *                                  (the probe update's obj_normalization);
 *   ptycho_analytic_obj_finalize   out[s] = -upd[s] / sum_p max(norm[s, p]) with maxes (S*P floats) as work;
 *   ptycho_analytic_probe_finalize probe_grad *= -1 / (obj_norm[0] * ortho_norm). */
int ptycho_patch_energy_max(const void* obj, const float* positions, const int64_t* batch_idx, int S, int Ho,
                            int Wo, int n, int B, int npos, float* out, void* stream);
int ptycho_analytic_obj_finalize(const void* upd, const float* norm, float* maxes, int S, int P, int64_t plane,
                                 void* out, void* stream);
int ptycho_analytic_probe_finalize(void* probe_grad, int64_t count, const float* obj_norm, float ortho_norm,
                                   void* stream);

/* Measurement utility (no reference counterpart): FP32 FMA throughput probe used to
 * state the FP32-pipe roofline.  `out` holds blocks * 512 floats; each thread runs
 * 16 independent FMA chains of `iters` steps (32 * iters flops per thread). */
int ptycho_fp32_fma_probe(float* out, int iters, int blocks, void* stream);

/* Largest launch grid accepted by ptycho_forward_loss_noalloc. */
#define PTYCHO_NOALLOC_MAX_GRID 1024

/* No counterpart in the reference.  Same as ptycho_forward_loss followed by
 * ptycho_reduce_loss, for callers that cannot allocate device memory (their
 * memory belongs to another framework's allocator, or allocation and the device
 * synchronisation it can cause are not allowed where they run).  The per-CTA
 * loss partials live in a static device array owned by the library
 * (PTYCHO_NOALLOC_MAX_GRID doubles, held on every GPU that loads the library
 * until exit); a->loss_part is ignored and the summed loss is written to the
 * device float *out_loss.  Nothing is allocated or freed.  a->grid above
 * PTYCHO_NOALLOC_MAX_GRID is rejected with PTYCHO_ERR_INVALID.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  That address is cached for
 * the life of the process, so a device reset (cudaDeviceReset, or a new primary
 * context) between calls is not supported.  All calls on a device share the
 * array: calls that overlap on the GPU race. */
int ptycho_forward_loss_noalloc(const ptycho_batch_args* a, float* out_loss, void* stream);


/* ------------------------------------------------------------------------
 * Learned initialiser: CNN training and inference kernels.
 *
 * They replace the torch.nn layers of the reference's UNet-like CNN2d
 * (src/quantem/core/ml/cnn.py:17-212): Conv2dBlock = Conv2d 3x3 with circular
 * padding, activation, BatchNorm2d (core/ml/blocks.py:53-140); the 2x2 MaxPool2d
 * between levels (cnn.py:86, 184-191); Upsample2dBlock = ConvTranspose2d 3x3
 * stride 2 + 1x1 Conv2d + BatchNorm2d (blocks.py:143-205); channel
 * concatenation of the skips (cnn.py:194-198).
 *
 * Activations are channels-last matrices: R = B*H*W rows (r = (b*H + y)*W + x)
 * with a leading dimension ld >= C, so a channel slice of a wider buffer is a
 * column offset plus the wider ld.  BF16 tensors are passed as void*.
 * ------------------------------------------------------------------------ */

/* GEMM epilogue flags. */
#define PTYCHO_GEMM_BF16 1   /* store BF16 instead of FP32 */
#define PTYCHO_GEMM_RELU 2   /* max(x, 0) after the bias */
#define PTYCHO_GEMM_ATOMIC 4 /* add into FP32 C atomically, C not cleared (splits > 1 without it clears C) */
/* Activation applied after the bias, in flag bits 8-11: PTYCHO_GEMM_ACT(a) with a one of
 * PTYCHO_ACT_* (core/ml/activation_functions.py:166-181, torch's default parameters);
 * PTYCHO_GEMM_RELU is PTYCHO_GEMM_ACT(PTYCHO_ACT_RELU).  Not with atomic / split-K output. */
#define PTYCHO_GEMM_ACT(a) ((a) << 8)
enum {
  PTYCHO_ACT_NONE = 0,
  PTYCHO_ACT_RELU = 1,
  PTYCHO_ACT_LEAKY_RELU = 2, /* slope 0.01 */
  PTYCHO_ACT_ELU = 3,        /* alpha 1 */
  PTYCHO_ACT_TANH = 4,
  PTYCHO_ACT_SIGMOID = 5,
  PTYCHO_ACT_SOFTPLUS = 6    /* beta 1, threshold 20 */
};

/* C[M][ldc] (op)= A[M][lda] * B[N][ldb]^T (+ bias[N]): BF16 operands, K-major
 * (K contiguous), FP32 accumulation on the tcgen05 tensor cores (TMA-fed
 * 128 x {32,64,128} tiles, accumulator in tensor memory).  Replaces the matrix
 * products inside nn.Conv2d / nn.ConvTranspose2d forward and backward.  A and B
 * 16-byte aligned, lda and ldb multiples of 8.  splits > 1 splits K across CTAs.
 * `status` (optional device int) gets bit 0 set if a bounded wait expired. */
int ptycho_gemm_bf16(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
                     const float* bias, int flags, int splits, int* status, void* stream);

/* col[r][(ky*3+kx)*C + c] = x[b, (y+ky-1) mod H, (x+kx-1) mod W, c] (BF16): the
 * circular-padded 3x3 patches of nn.Conv2d(padding=1, padding_mode="circular"). */
int ptycho_cnn_im2col3x3(const void* x, int B, int H, int W, int C, int ldx, void* col, int ldcol, void* stream);

/* Adjoint of ptycho_cnn_im2col3x3 on FP32: dx (+)= fold(dcol). */
int ptycho_cnn_col2im3x3(const float* dcol, int ldcol, int B, int H, int W, int C, float* dx, int ldx, int accumulate,
                         void* stream);

/* nn.ConvTranspose2d(k=3, stride=2, padding=1, output_padding=1) output assembly:
 * out (B, 2H, 2W, Co) BF16 = bias + sum of the per-input-pixel products
 * colT[(b,iy,ix)][(ky*3+kx)*Co + co] landing on (2iy-1+ky, 2ix-1+kx). */
int ptycho_cnn_convT_gather(const float* colT, int ldcol, int B, int H, int W, int Co, const float* bias, void* out,
                            int ldo, void* stream);

/* Adjoint of the assembly: dcol[(b,iy,ix)][(ky*3+kx)*Co + co] = dout[b, 2iy-1+ky, 2ix-1+kx, co] (BF16, 0 outside). */
int ptycho_cnn_convT_im2col(const float* dout, int ldo, int B, int H, int W, int Co, void* dcol, int ldcol,
                            void* stream);

/* out[z][c][r] = in[z][r][c]; dtypes 0 = FP32, 1 = BF16 (layout changes between
 * NCHW and channels-last, and operand transposes for the weight gradients). */
int ptycho_cnn_transpose(const void* in, int in_dtype, int R, int C, int ldi, int64_t batch_stride_in, void* out,
                         int out_dtype, int ldo, int64_t batch_stride_out, int batch, void* stream);

/* nn.BatchNorm2d forward (torch.nn.functional.batch_norm): training = batch
 * statistics (biased variance for normalisation, running statistics updated with
 * the unbiased one and `momentum`), else running statistics.  gamma == NULL skips
 * the normalisation (plain BF16 conversion).  Writes the used mean / rstd.
 * `work` holds >= 2 * C doubles (more gives more parallel partial sums). */
int ptycho_cnn_bn_forward(const float* x, int ldx, int R, int C, const float* gamma, const float* beta,
                          float* run_mean, float* run_var, float momentum, float eps, int training, float* mean,
                          float* rstd, double* work, int64_t work_elems, void* out, int ldo, void* stream);

/* Backward of batch norm (gamma != NULL) followed by the derivative of the activation that
 * produced its input x (act = PTYCHO_ACT_*, taken from the activation's output x; 1 = the
 * ReLU mask [x > 0], 0 = none): dz = act'(x) * dBN(dy).  Writes dgamma / dbeta and dz as
 * FP32 and/or BF16 (either may be NULL). */
int ptycho_cnn_bn_backward(const float* dy, int lddy, const float* x, int ldx, int R, int C, const float* gamma,
                           const float* mean, const float* rstd, int training, int act, float* dgamma, float* dbeta,
                           double* work, int64_t work_elems, float* dz32, void* dz16, int ldz, void* stream);

/* Dropout in place (nn.Dropout, core/ml/blocks.py:134-135): x[r][c] *= keep / (1 - p) with
 * keep = u >= p for a uniform u drawn from a counter-based hash of (seed, r * C + c); the same
 * seed regenerates the mask for the backward.  dtype 0 = FP32, 1 = BF16; 0 <= p <= 1. */
int ptycho_cnn_dropout(void* x, int dtype, int R, int C, int ld, float p, uint64_t seed, void* stream);

/* out[c] (+)= sum_r a[r][c] (bias gradients), deterministic order. */
int ptycho_cnn_colsum(const float* a, int lda, int R, int C, float* out, int accumulate, double* work,
                      int64_t work_elems, void* stream);

/* nn.MaxPool2d(2, 2) on BF16 with the argmax code (2*dy + dx) per output. */
int ptycho_cnn_maxpool2(const void* in, int ldi, int B, int H, int W, int C, void* out, int ldo, void* argmax,
                        void* stream);

/* Its adjoint: din (+)= dout routed to the argmax positions (FP32). */
int ptycho_cnn_maxpool2_backward(const float* dout, int lddo, const void* argmax, int B, int H, int W, int C,
                                 float* din, int lddi, int accumulate, void* stream);

/* out (BF16) = in (FP32), n values: BF16 weight copies of the FP32 master weights. */
int ptycho_cnn_cast_bf16(const float* in, void* out, int64_t n, void* stream);

/* Learned-initialiser input features: for each of npos patterns (n x n, FP32,
 * intensities or amplitudes when `amplitudes` != 0) and each bin x bin block
 * (u, v): out[p][u*(n/bin) + v] = (sqrt(norm * block intensity sum) - mean[u*(n/bin)+v]) * scale
 * as BF16 (mean may be NULL; norm = 1 / mean pattern total makes the features
 * dose-independent).  One row per scan position = the channels-last input
 * matrix of the CNN on the scan grid. */
int ptycho_cnn_bin_features(const float* patterns, int npos, int n, int bin, int amplitudes, float norm,
                            const float* mean, float scale, void* out, int ldo, void* stream);

/* loss = mean((pred - target)^2) (device float); dpred = 2 (pred - target) / n as
 * FP32 and/or BF16 (either may be NULL).  work >= 296 doubles. */
int ptycho_cnn_mse(const float* pred, const float* target, int64_t n, float* loss, float* dpred32, void* dpred16,
                   double* work, int64_t work_elems, void* stream);

/* ------------------------------------------------------------------------
 * Dataset preprocessing on the GPU (PtychographyDatasetRaster.preprocess,
 * dataset_models.py:946-1025).
 * ------------------------------------------------------------------------ */

/* Centre of mass of npos patterns (nr x nc, FP32), optionally times a detector
 * mask: com[p] = sum(I r)/sum(I), com[npos + p] = sum(I c)/sum(I) in pixels
 * (replaces _set_intensities_com, dataset_models.py:1058-1073).  FP64 sums. */
int ptycho_pattern_com(const float* intensities, const float* mask, int npos, int nr, int nc, double* com,
                       void* stream);

/* I = max(I, 0), a = sqrt(I) for `count` values: writes the clipped intensities
 * and amplitudes (either may be NULL), a complex64 copy of a for the Fourier
 * shift, and sums[0] = sum I, sums[1] = sum a (FP64, fixed order through `work`,
 * >= 1184 doubles).  First half of the per-position loop of
 * _normalize_diffraction_intensities (dataset_models.py:1419-1427). */
int ptycho_pattern_prepare(const float* intensities, int64_t count, float* intensities_out, float* amplitudes_out,
                           void* amplitudes_c, double* work, int64_t work_elems, double* sums, void* stream);

/* spectra (npos, n, n) complex64 *= exp(-2 pi i (cs_p qc + rs_p qr)), rs = shifts[p],
 * cs = shifts[npos + p], q = fftfreq(n): the Fourier-shift ramp of shift_array
 * (ptycho_utils.py:264-271) between ptycho_fft2 forward and inverse. */
int ptycho_pattern_shift_ramp(void* spectra, const double* shifts, int npos, int n, void* stream);

/* centred amplitudes = fftshift(max(Re(shifted) * scale, 0)) (n even) and their
 * squares (dataset_models.py:1429-1435). */
int ptycho_pattern_center(const void* shifted, int npos, int n, float scale, float* centered_amplitudes,
                          float* centered_intensities, void* stream);

/* The bilinear form of the same centring (`preprocess(bilinear=True)`, shift_array with
 * bilinear=True, ptycho_utils.py:273-284): amplitudes (npos, n, n) float32 rolled by
 * floor(shift) and blended with the next pixel by the fractional parts, periodic, in float64,
 * then centred amplitudes = fftshift(max(., 0)) and (nullable) their squares; shifts (2, npos)
 * = (rs, cs) as for ptycho_pattern_shift_ramp, n even.  Outputs must not alias the input. */
int ptycho_pattern_bilinear(const float* amplitudes, const double* shifts, int npos, int n,
                            float* centered_amplitudes, float* centered_intensities, void* stream);

/* ---- probe-mode orthogonalisation (ProbePixelated._probe_orthogonalization_constraint,
 * probe_models.py:484-525): modified Gram-Schmidt with the running vector, every mode
 * rescaled to its original norm, modes sorted by descending intensity; one CTA. ---- */

/* complex64 elements of the work buffer for P modes of nn elements (1 <= P <= 16). */
int64_t ptycho_probe_ortho_work_elems(int P, int64_t nn);

/* out (P, nn) = sorted orthogonalised modes of probe (P, nn), complex64; `work` keeps
 * what the gradient needs.  out must not alias probe. */
int ptycho_probe_orthogonalize(const void* probe, void* out, int P, int64_t nn, void* work, int64_t work_elems,
                               void* stream);

/* grad_probe = gradient w.r.t. probe of a real loss whose gradient w.r.t. the sorted
 * output is grad_sorted (torch convention); `work` from the matching forward call.
 * grad_probe must not alias probe, grad_sorted or work (PTYCHO_ERR_INVALID). */
int ptycho_probe_orthogonalize_vjp(const void* probe, const void* grad_sorted, void* grad_probe, int P, int64_t nn,
                                   void* work, int64_t work_elems, void* stream);

/* ---- optional probe constraints (replace ProbeConstraints, probe_models.py:430-482) ---- */

/* Complex elements of the `work` buffer of ptycho_probe_center / _vjp for P modes of n x n. */
int64_t ptycho_probe_center_work_elems(int P, int n);

/* The centre-of-mass constraint (`center_probe`, probe_models.py:467-482, with
 * fourier_shift_expand, ptycho_utils.py:128-139): for every mode the centre of mass of
 * |probe|^2 on the fftshifted grid minus n / 2 is computed (float64) and the mode is
 * Fourier-shifted by minus it: out = ifft2(fft2(probe) exp(2 pi i (k_r c_r + k_c c_c))),
 * k = fftfreq(n).  probe, out: (P, n, n) complex64, 1 <= P <= 16, n in {64, 96, 128, 256}.
 * `work` (ptycho_probe_center_work_elems complex elements) keeps the shifted spectrum and the
 * centres of mass for ptycho_probe_center_vjp.  out must not alias probe or work. */
int ptycho_probe_center(const void* probe, void* out, int P, int n, void* work, int64_t work_elems, void* stream);

/* grad_probe = gradient w.r.t. probe (torch convention) of a real loss whose gradient w.r.t.
 * the centred probe is grad_out: the adjoint of the shift plus the path through the centre
 * of mass.  `work` from the matching ptycho_probe_center call, unchanged since.  grad_probe
 * must not alias probe or work (PTYCHO_ERR_INVALID); it may alias grad_out. */
int ptycho_probe_center_vjp(const void* probe, const void* grad_out, void* grad_probe, int P, int n, void* work,
                            int64_t work_elems, void* stream);

/* float64 elements of the `work` buffer of ptycho_probe_tv. */
int ptycho_probe_tv_work_elems(void);

/* The probe TV soft loss (`tv_weight`, probe_models.py:460-466): loss[0] = weight x
 * (mean |probe[..., c + 1] - probe[..., c]| + mean |probe[..., r + 1, :] - probe[..., r, :]|)
 * over all P modes of n x n (n >= 2); with grad (nullable) its gradient, weight / (P n (n - 1))
 * x the sum of d / |d| over the differences touching each element with the sign of its
 * position in d (0 where d = 0).  grad must not alias probe.  Deterministic. */
int ptycho_probe_tv(const void* probe, int P, int n, float weight, float* loss, void* grad, double* work, int nwork,
                    void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PTYCHO_B200_H */
