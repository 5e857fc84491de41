/*
 * hsflow.h -- C ABI of libhsflow.so, the B200 (sm_100a) implementation of the
 * Horn-Schunck stencil path of chick/hindemith.
 *
 * Conventions for every entry point:
 *   - Images are dense FP32 planes, row-major, x (width) fastest: element (x, y) is
 *     at p[x + y * ld]  (the reference's index x + y*W, Types/Array2D.cpp:302).
 *     H, W >= 1; ld >= W, ld % 4 == 0; every plane pointer is 16-byte aligned.
 *   - Pointers named in/out/u/v/I0/... are DEVICE pointers owned by the caller.
 *     Stencil taps (weights/offx/offy) are HOST arrays, copied into the launch.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Nothing blocks
 *     the host; errors found by argument checks are returned before any launch,
 *     launch errors are returned from the launching call.
 *   - Every call returns an hs_status; hs_last_error() gives a one-line detail
 *     for the calling thread.  No C++ exception crosses this boundary.
 *   - Scratch memory is the caller's: functions that need it take
 *     (workspace, workspace_bytes) and say how much through *_workspace_bytes().
 *
 * Each function cites the reference interface it replaces (paths inside
 * chick/hindemith).
 */
#ifndef HSFLOW_H
#define HSFLOW_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HS_API __attribute__((visibility("default")))
#else
#define HS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hs_status {
    HS_OK = 0,
    HS_ERR_INVALID_ARG = 1,   /* null pointer, non-positive size, bad op code, ... */
    HS_ERR_ALIGNMENT = 2,     /* ld % 4 != 0 or a plane not 16-byte aligned */
    HS_ERR_WORKSPACE = 3,     /* workspace missing or smaller than required */
    HS_ERR_CUDA = 4,          /* a CUDA runtime call or launch failed */
    HS_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
    HS_ERR_UNSUPPORTED = 6,   /* valid request this build does not implement */
    HS_ERR_NO_DEVICE = 7      /* no usable sm_100 device */
} hs_status;

/* Binary operator codes, the reference's op names (Array2DOp.cpp:36-51). */
typedef enum hs_binop { HS_OP_ADD = 0, HS_OP_SUB = 1, HS_OP_MUL = 2, HS_OP_DIV = 3 } hs_binop;

#define HS_MAX_TAPS 64
#define HS_MAX_SWEEPS_PER_PASS 8

/* Tuning of the sweep kernels.  Zero-initialise for the defaults. */
typedef struct hs_config {
    int sweeps_per_pass;  /* temporal-blocking depth T (1..8) = sweeps per HBM pass; 0 = default:
                           * for hs_forward / hs_sweeps / hs_forward_noalloc a measured table by
                           * image size and form (within 6 % of the autotuned best on B200 from
                           * 240x320 to 4096^2, 16 % at 512^2 in the fast form), 4 for the
                           * other calls */
    int rows_per_segment; /* rows each warp streams per work item; 0 = default */
    int fast_math;        /* 0 (default): the reference program's operation order, one
                             rounding per operation -- bit-identical to the reference's
                             FP32 semantics for any T;  1: factored stencil, fused
                             multiply-adds and a per-pixel reciprocal, within 1e-4 */
    float avg_edge;       /* weight of the 4 edge taps of the 3x3 average; 0 = 1/6 */
    float avg_corner;     /* weight of the 4 corner taps; 0 = 1/12 (both 0 = the HS stencil) */
    int layout;           /* columns per lane of the sweep kernels: 0 = chosen by image size
                             (4 from 250 kpx for one pair, from 2 Mpx of average pair size in
                             the training calls; the batched launch keeps 2), 1 = 2 (64-column
                             strips), 2 = 4 (128-column strips; fast_math only).  Results do not
                             depend on it. */
    int reserved[2];      /* must be zero */
} hs_config;

/* ---- library ---------------------------------------------------------------- */
HS_API const char *hs_status_string(hs_status status);
HS_API const char *hs_last_error(void);
HS_API int hs_version(void);

/* ---- structured-grid operations (the reference's operator plugins) ------------ */

/* out = S * in: out(x,y) = sum_d w[d] * in(clamp(x+offx[d]), clamp(y+offy[d])), summed
 * from 0 in tap order, one rounding per operation.  1 <= ntaps <= HS_MAX_TAPS.
 * Replaces Stencil2DMVMSetupLaunch + Stencil2DMVMElementLevel::compile
 * (Operations/StructuredGrid/Stencil2DMVM.cpp:62, :34-59).  in != out. */
HS_API hs_status hs_stencil2d(const float *weights, const int *offx, const int *offy, int ntaps,
                       const float *in, float *out, int H, int W, int ld, void *stream);

/* a = b op c (Operations/DenseLinearAlgebra/Array2DOp.cpp:27-118). */
HS_API hs_status hs_array2d_op(int op, const float *b, const float *c, float *a, int H, int W, int ld,
                        void *stream);
/* a = b op s (Array2DScalarOp.cpp:29-118). */
HS_API hs_status hs_array2d_scalar_op(int op, const float *b, float s, float *a, int H, int W, int ld,
                               void *stream);
/* a = s op b (ScalarArray2DOp.cpp:29-119). */
HS_API hs_status hs_scalar_array2d_op(int op, float s, const float *b, float *a, int H, int W, int ld,
                               void *stream);
/* a = b (Array2DCopy.cpp:23-93). */
HS_API hs_status hs_array2d_copy(const float *b, float *a, int H, int W, int ld, void *stream);

/* ---- Horn-Schunck ----------------------------------------------------------- */

/* 2x2x2 derivatives in one pass: Ix = Dx*I0 + Dx*I1, Iy = Dy*I0 + Dy*I1,
 * It = Dt*I1 - Dt*I0 with Dx, Dy, Dt the 4-tap stencils over {0,1}^2 (weights -1/4,
 * +1/4 for Dx/Dy, 1/4 for Dt) and clamp-to-edge taps.  Bit-identical to the
 * reference program's FP32 result.  Replaces the fused derivative strand the
 * reference builds from Stencil2DMVM + Array2DOp (Stencil2DMVM.cpp:34-59,
 * Array2DOp.cpp:27-53, fused by fusion.cpp:113-303). */
HS_API hs_status hs_derivs(const float *I0, const float *I1, int H, int W, int ld, float *Ix,
                    float *Iy, float *It, void *stream);

/* Scratch needed by hs_sweeps: two planes (the ping-pong copy of u, v). */
HS_API size_t hs_sweeps_workspace_bytes(int H, int W, int ld);

/* `iters` Jacobi sweeps in place on (u, v), from their current contents:
 *   ubar = A*u; vbar = A*v          (A: 3x3 clamp-to-edge average, 1/6 edges, 1/12 corners)
 *   t = (Ix*ubar + Iy*vbar + It) / (alpha2 + Ix*Ix + Iy*Iy)
 *   u = ubar - Ix*t; v = vbar - Iy*t
 * T sweeps run per pass over HBM (cfg->sweeps_per_pass).  iters >= 0.
 * Replaces the Iterator's host loop (execute.cpp:35-45) over the two fused sweep
 * kernels (Stencil2DMVM.cpp:34-59 + Array2DOp/Array2DScalarOp/Array2DCopy chains). */
HS_API hs_status hs_sweeps(const float *Ix, const float *Iy, const float *It, int H, int W, int ld,
                    float alpha2, int iters, float *u, float *v, void *workspace,
                    size_t workspace_bytes, const hs_config *cfg, void *stream);

/* Scratch needed by hs_forward: five planes (Ix, Iy, It and the ping-pong copy). */
HS_API size_t hs_forward_workspace_bytes(int H, int W, int ld);

/* The plain per-pair drop-in: derivatives, u = v = 0, `iters` sweeps with
 * alpha2 = alpha * alpha (FP32).  Replaces backend.run for a compiled Horn-Schunck
 * program (backend.cpp:320-638) end to end on the device. */
HS_API hs_status hs_forward(const float *I0, const float *I1, int H, int W, int ld, float alpha,
                     int iters, float *u, float *v, void *workspace, size_t workspace_bytes,
                     const hs_config *cfg, void *stream);

/* ---- batched Horn-Schunck ---------------------------------------------------- */

#define HS_MAX_BATCH 128

/* One image pair of a batch.  Device pointers; each pair has its own size, alpha and
 * sweep count. */
typedef struct hs_pair_desc {
    const float *I0, *I1;  /* inputs, H x ld planes */
    float *u, *v;          /* outputs, H x ld planes */
    int H, W, ld;
    float alpha;           /* alpha2 = alpha * alpha */
    int iters;             /* Jacobi sweeps, >= 0 */
    int reserved;          /* must be zero */
} hs_pair_desc;

/* Workspace hs_forward_batched needs for these pairs and config (0 if they are invalid):
 * five planes per pair plus one counter per work tile and a 256-byte header. */
HS_API size_t hs_forward_batched_workspace_bytes(const hs_pair_desc *pairs, int n,
                                                 const hs_config *cfg);

/* hs_forward for n (1..HS_MAX_BATCH) pairs of uneven size in one persistent launch:
 * every (pass, pair, tile) is a work item taken from a device queue; a tile waits only
 * for its neighbours' previous pass (bounded waits).  Results equal hs_forward per pair.
 * Stream-ordered and free of host synchronisation, allocation and pageable copies, so it
 * can be captured in a CUDA graph (make one call before capturing: the first call sets
 * kernel attributes).  `device_status` (device int, may be NULL) receives HS_OK or
 * HS_ERR_TIMEOUT when the stream reaches the end of the call.  The workspace must be
 * 256-byte aligned.  Replaces looping backend.run over the pairs (backend.cpp:320). */
HS_API hs_status hs_forward_batched(const hs_pair_desc *pairs, int n, void *workspace,
                                    size_t workspace_bytes, const hs_config *cfg,
                                    int *device_status, void *stream);

/* ---- differentiable Horn-Schunck --------------------------------------------- */

/* Bytes of the derivative planes (Ix, Iy, It; three planes, each rounded up to 256
 * bytes) and of the checkpoints ceil(iters/ckpt_every) x (u, v) kept by the forward. */
HS_API size_t hs_derivs_bytes(int H, int W, int ld);
HS_API size_t hs_checkpoint_bytes(int H, int W, int ld, int iters, int ckpt_every);
HS_API size_t hs_forward_train_workspace_bytes(int H, int W, int ld);

/* hs_forward that also keeps what the backward needs: `derivs` receives Ix, Iy, It and
 * `ckpt` the state (u, v) before sweeps 0, c, 2c, ... (c = ckpt_every) and after the last
 * sweep (hs_checkpoint_bytes: ceil(iters / c) + 1 plane pairs).  `alpha` is a DEVICE
 * pointer to one float (a learnable alpha never needs a host round trip).  It runs the
 * batched training passes with one pair (hs_forward_train_batched); the workspace
 * (hs_forward_train_workspace_bytes) holds the passes' ping-pong planes.  Results equal
 * hs_forward's.  No counterpart in the reference, which has no gradients. */
HS_API hs_status hs_forward_train(const float *I0, const float *I1, int H, int W, int ld,
                                  const float *alpha, int iters, int ckpt_every, float *u,
                                  float *v, float *derivs, float *ckpt, void *workspace,
                                  size_t workspace_bytes, const hs_config *cfg, void *stream);

HS_API size_t hs_backward_workspace_bytes(int H, int W, int ld, int ckpt_every);

/* Gradients of a loss L(u, v) through the whole forward: given dL/du, dL/dv it writes
 * dL/dI0, dL/dI1 (planes) and dL/dalpha (one device float).  Each checkpoint interval's
 * states are recomputed from its checkpoint, then its sweeps are reversed with the
 * adjoint kernel (transposed clamp-to-edge average, adjoint of the pointwise update);
 * the derivative stencils are transposed last.  The same passes as hs_backward_batched
 * with one pair; needs alpha != 0.  Deterministic. */
HS_API hs_status hs_backward(const float *derivs, int H, int W, int ld, const float *alpha,
                             int iters, int ckpt_every, const float *ckpt, const float *dLdu,
                             const float *dLdv, float *dI0, float *dI1, float *dalpha,
                             void *workspace, size_t workspace_bytes, const hs_config *cfg,
                             void *stream);

/* n pairs (1..32) of one differentiable batch; all device pointers.  The forward reads
 * I0, I1, alpha and writes u, v; the backward reads dLdu, dLdv, alpha and writes dI0,
 * dI1 and dalpha (one float). */
typedef struct hs_train_pair {
    const float *I0, *I1;
    float *u, *v;
    const float *alpha;
    const float *dLdu, *dLdv;
    float *dI0, *dI1;
    float *dalpha;
    int H, W, ld;
    int reserved; /* must be zero */
} hs_train_pair;

/* Workspace shared by hs_forward_train_batched and the matching hs_backward_batched
 * (derivatives, checkpoints, one interval's states, adjoint buffers per pair). */
HS_API size_t hs_train_workspace_bytes(const hs_train_pair *pairs, int n, int iters, int ckpt_every);

/* Forward of n pairs with checkpoints every ckpt_every sweeps kept in the workspace; each
 * pass is one launch over all pairs.  Results equal hs_forward per pair. */
HS_API hs_status hs_forward_train_batched(const hs_train_pair *pairs, int n, int iters,
                                          int ckpt_every, void *workspace, size_t workspace_bytes,
                                          const hs_config *cfg, void *stream);

/* Backward of the preceding hs_forward_train_batched (same pairs, iters, ckpt_every and
 * workspace): each checkpoint interval's states are recomputed by dump passes (each stage
 * of a T-sweep pass writes its state), on a library-owned side stream up to two intervals
 * ahead, and the adjoint runs temporally blocked on the caller's stream, min(4,
 * sweeps_per_pass) adjoint sweeps per HBM pass in passes of balanced depth that may span
 * two intervals.  The side stream joins a capture of the caller's stream through events and
 * is joined back before the call returns.  Needs alpha != 0.  Deterministic. */
HS_API hs_status hs_backward_batched(const hs_train_pair *pairs, int n, int iters, int ckpt_every,
                                     void *workspace, size_t workspace_bytes,
                                     const hs_config *cfg, void *stream);

/* ---- coarse-to-fine pieces ---------------------------------------------------- */

/* out = every second pixel of the 5x5 binomial blur ([1 4 6 4 1]/16 per axis, clamp-to-edge
 * taps) of in: out is ceil(H/2) x ceil(W/2) with row stride ldo.  The reference builds
 * pyramids from Stencil2DMVM (Stencil2DMVM.cpp:34-59); this fuses the blur and the
 * decimation.  The adjoint overwrites din (H x W, stride ld) with the transpose applied
 * to dout. */
HS_API hs_status hs_blur_down(const float *in, int H, int W, int ld, float *out, int ldo, void *stream);
HS_API hs_status hs_blur_down_adjoint(const float *dout, int H, int W, int ld, int ldo, float *din,
                                      void *stream);

/* fine (H x W) = scale * 2x bilinear upsampling of coarse (ceil(H/2) x ceil(W/2), stride
 * ldc), half-pixel centres, clamped coarse indices (scale = 2 for a flow field).  No
 * counterpart in the reference.  The adjoint overwrites dcoarse. */
HS_API hs_status hs_upsample2(const float *coarse, int ldc, float *fine, int H, int W, int ld,
                              float scale, void *stream);
HS_API hs_status hs_upsample2_adjoint(const float *dfine, int H, int W, int ld, float *dcoarse,
                                      int ldc, float scale, void *stream);

/* dst = src backward-warped by the offsets (u, v) with WarpImg2D's semantics
 * (Operations/OpticalFlow/WarpImg2D.cpp:33-75): bilinear when the 2x2 footprint at
 * (x + u, y + v) lies inside the image, else the source pixel; bit-identical to the
 * template's float/double arithmetic.  The adjoint overwrites dsrc with dL/dsrc and du, dv
 * with dL/du, dL/dv (piecewise derivative).  dL/dsrc is a scatter along the flow, summed
 * as 64-bit fixed-point integers with one power-of-two scale per call (chosen from
 * max |ddst| and max(|u|, |v|) so that no sum can overflow), hence deterministic: the same
 * inputs give the same bits on every run.  Non-finite ddst or offsets give NaN in dsrc.
 * The workspace (hs_warp_adjoint_workspace_bytes, 256-byte aligned) holds the sums. */
HS_API hs_status hs_warp(const float *src, const float *u, const float *v, int H, int W, int ld,
                         float *dst, void *stream);
HS_API size_t hs_warp_adjoint_workspace_bytes(int H, int W, int ld);
HS_API hs_status hs_warp_adjoint(const float *src, const float *u, const float *v,
                                 const float *ddst, int H, int W, int ld, float *dsrc, float *du,
                                 float *dv, void *workspace, size_t workspace_bytes,
                                 void *stream);

/* ---- Horn-Schunck as a linear system (CG family) ------------------------------ */

/* Krylov powers of the HS normal-equations operator, HSMatrixPowers.cpp:72-106 (setup
 * :129-226): V[0] = (r0, r1) and V[s] = M V[s-1] for s = 1 .. steps-1, where
 *   M(u, v) = (Ix g, Iy g) + lam (deg u - sum of the 4-neighbours of u, same for v),
 *   g = Ix u + Iy v, neighbours outside the image absent,
 * in the template's operation order (bit-identical to its FP32 semantics).  V0, V1 hold
 * `steps` planes each, power s at V + s * power_stride floats (power_stride >= H*ld, a
 * multiple of 4).  cfg->sweeps_per_pass (1..4, 0 = 4) powers are computed per pass over
 * HBM, streaming the image in column strips with the powers as a register pipeline, each warp
 * over cfg->rows_per_segment rows (0 = about one wave of warps over the image). */
HS_API hs_status hs_matrix_powers(float lam, const float *Ix, const float *Iy, const float *r0,
                                  const float *r1, int H, int W, int ld, int steps, float *V0,
                                  float *V1, size_t power_stride, const hs_config *cfg,
                                  void *stream);

/* The 2x2 block-Jacobi preconditioner of the HS system, ApplyHSPreconditioner.cpp:46-97:
 *   a = diag0 + n s2, d = diag1 + n s2 (n = neighbours present), b = c = offdiag,
 *   det = a d - b c; |det| > 1e-15: y0 = (x0 d - b x1)/det, y1 = (-c x0 + a x1)/det;
 *   else y = x.
 * s2 is the stencil's third weight (the template's getData("2")). */
HS_API hs_status hs_apply_hs_preconditioner(float s2, const float *diag0, const float *diag1,
                                            const float *offdiag, const float *x0,
                                            const float *x1, int H, int W, int ld, float *y0,
                                            float *y1, void *stream);

/* Self-test of the failure path of the batched launch's bounded waits (no counterpart in
 * the reference, whose runtime has no device-side waits): one thread waits with the same
 * bounded wait on a flag that nothing sets, gives up after max_polls polls
 * (1 .. 2^22, with a nanosleep back-off of at most 256 ns each) and writes HS_ERR_TIMEOUT to
 * *device_status (a device int the caller zeroed).  The kernel then returns normally. */
HS_API hs_status hs_selftest_bounded_wait(int *device_status, int max_polls, void *stream);

/* ---- Lucas-Kanade and Brox on the same grid substrate -------------------------- */

/* LKLeastSquares.cpp:44-79: for pixels at least `radius` from the left/top border and
 * radius+1 from the right/bottom one, the 2x2 least-squares flow over the window
 * dx, dy in [-radius, radius) (sums from 0, dx outer), solved by Cramer's rule; du = dv = 0
 * elsewhere and where the determinant is 0.  radius 1..16. */
HS_API hs_status hs_lk_least_squares(const float *err, const float *Ix, const float *Iy, int H,
                                     int W, int ld, int radius, float *du, float *dv,
                                     void *stream);

/* SetBroxMatrix.cpp:38-80 (redblack = 0) and SetBroxRedblackMatrix.cpp:38-80 (redblack = 1).
 * `data` holds the diagonals as planes diag_stride floats apart: top, left, mid, right,
 * bottom (5) -- or top, left, right, bottom (4) with the middle term in `adiag`.  A
 * diagonal is indexed by the column of its entry (the neighbour); entries no pixel writes
 * keep their values. */
HS_API hs_status hs_set_brox_matrix(const float *psi, int H, int W, int ld, float alpha,
                                    float *data, size_t diag_stride, int redblack, float *adiag,
                                    void *stream);

/* SpmvDIA2D.cpp:36-45: y = sum over the diagonals d (<= 16, offsets by value) whose
 * neighbour (x + offx[d], y + offy[d]) is inside the grid of data[d] * x at that neighbour. */
HS_API hs_status hs_spmv_dia2d(const float *data, size_t diag_stride, const int *offx,
                               const int *offy, int ndiags, const float *x, int H, int W, int ld,
                               float *y, void *stream);

/* ApplyBroxPreconditioner.cpp:46-62: a = diag0 + mid, d = diag1 + mid, b = c = offdiag;
 * |a d - b c| > 1e-4: the 2x2 solve; else y = x.  `mid` is the matrix's middle diagonal. */
HS_API hs_status hs_apply_brox_preconditioner(const float *mid, const float *diag0,
                                              const float *diag1, const float *offdiag,
                                              const float *x0, const float *x1, int H, int W,
                                              int ld, float *y0, float *y1, void *stream);

/* ---- fused kernels for arbitrary Stencil / Array2D programs --------------------- */

#define HS_FUSED_MAX_IN 16
#define HS_FUSED_MAX_OUT 8
#define HS_FUSED_MAX_SCALARS 64
#define HS_FUSED_MAX_SUMS 8

/* Arguments of one fused group of statements: planes share H, W and ld. */
typedef struct hs_fused_args {
    const float *in[HS_FUSED_MAX_IN];
    float *out[HS_FUSED_MAX_OUT];
    float s[HS_FUSED_MAX_SCALARS];
    int H, W, ld;
    int nsums;      /* sum2d reductions in the body (0..HS_FUSED_MAX_SUMS) */
    double *sums;   /* device: nsums doubles, written */
    int reserved[4]; /* must be zero */
} hs_fused_args;

/* Workspace (per-block partial sums) for a fused group with nsums reductions. */
HS_API size_t hs_fused_workspace_bytes(int H, int W, int nsums);

/* Runs one fused group: `body` is the CUDA C of one pixel, written with IN(k),
 * LD(k, dx, dy) (clamp-to-edge neighbour), OUT(k) = ..., S(k), SUM(k, v) and the
 * coordinates X, Y.  The library wraps it in its kernel skeleton, compiles it once with
 * NVRTC for sm_100a (-fmad=false unless fast_math, so each operation rounds once, as
 * the reference's statements do) and caches it by source.  Replaces the reference's
 * generated-kernel path (fusion.cpp:113-303, lm.cpp:467-755, oclgen.cpp:156-185) and
 * Array2DSum (Array2DSum.cpp:25-119).  The first call for a body compiles and loads a
 * module: make it outside stream capture.  HS_ERR_UNSUPPORTED if NVRTC is missing. */
HS_API hs_status hs_fused_launch(const char *body, int fast_math, const hs_fused_args *args,
                                 void *workspace, size_t workspace_bytes, void *stream);

/* ---- loss ------------------------------------------------------------------- */

/* One flow field and its target for the mean end-point-error loss; du, dv receive the
 * gradient (backward only). */
typedef struct hs_epe_pair {
    const float *u, *v, *ut, *vt;
    float *du, *dv;
    int H, W, ld;
    int reserved; /* must be zero */
} hs_epe_pair;

/* *loss (device float) = (1/n) sum_i mean_px sqrt((u-ut)^2 + (v-vt)^2 + eps) over n <= 32
 * pairs, summed deterministically (double partials in a fixed order).  The reference's
 * Array2DSum (Operations/DenseLinearAlgebra/Array2DSum.cpp:25-119) is its reduction
 * building block; this fuses the pointwise error into the reduction.  The backward writes
 * du, dv = dloss * (u-ut, v-vt) / (n H W sqrt(...)) with dloss a device float. */
HS_API size_t hs_epe_workspace_bytes(int n);
HS_API hs_status hs_epe_loss_batched(const hs_epe_pair *pairs, int n, float eps, float *loss,
                                     void *workspace, size_t workspace_bytes, void *stream);
HS_API hs_status hs_epe_loss_backward_batched(const hs_epe_pair *pairs, int n, float eps,
                                              const float *dloss, void *stream);

/* ---- allocation-free forward ------------------------------------------------- */

/* Size of the library-owned scratch that hs_forward_noalloc uses: 48 MiB, enough for
 * planes of up to H * ld * 4 = 10,066,176 bytes (e.g. 1920x1080 with ld = 1920). */
#define HS_NOALLOC_SCRATCH_BYTES (48u << 20)

/* hs_forward without a caller-supplied workspace.  No counterpart in the reference: it
 * serves callers that cannot allocate device memory -- a frame loop that must not call
 * cudaMalloc/cudaFree (they can synchronise the device mid-stream), or a host binding
 * that has no way to own and release a device buffer.  The caller still passes the
 * inputs I0, I1 and the outputs u, v; the scratch is a static __device__ array of
 * HS_NOALLOC_SCRATCH_BYTES inside this library, held by every GPU that loads the
 * library until the process exits.  Nothing here allocates or frees memory.
 *   - Sizes whose five scratch planes exceed HS_NOALLOC_SCRATCH_BYTES are rejected with
 *     HS_ERR_WORKSPACE before any device work.
 *   - The first call on a device looks up the scratch's device address (with that
 *     device current); make that first call before any stream capture.  The address
 *     is kept for the life of the process: after cudaDeviceReset, or after the device's
 *     primary context is released and created again, the module may load elsewhere, so
 *     such a caller must not use this entry point on that device any more.
 *   - All calls on a device share the one scratch array and it keeps the last call's
 *     contents (each call initialises what it reads).  Calls that overlap on the GPU --
 *     concurrent streams, or several host threads -- race on it; serialise them.
 * Results are identical to hs_forward with the same arguments and config. */
HS_API hs_status hs_forward_noalloc(const float *I0, const float *I1, int H, int W, int ld,
                                    float alpha, int iters, float *u, float *v,
                                    const hs_config *cfg, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HSFLOW_H */
