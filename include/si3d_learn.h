/* Learned initial guess for the zeta solve: a small BF16 convolutional network that predicts the
 * increment zeta(n+1) - zeta(n) from quantities the solver already holds, used as the CG starting
 * point (x0 = sp + prediction).  CG still iterates to the unchanged tolerance, so the prediction only
 * changes the iteration count, never the accepted solution's accuracy.
 *
 * The reference has no counterpart: SolverSparse always starts NSPCG from sp
 * (si3d_procedures.f90:1970).  These entry points are the project's own.
 *
 * Network (fixed shape): input image of 4 channels per horizontal cell (i, j):
 *   c0 = (qq - A sp) / sigma      residual of the right-hand side at the default guess
 *   c1 = (sp - spp) / sigma       last increment of the surface
 *   c2 = hhs / 30 m               depth
 *   c3 = 1 on wet cells, 0 on land
 * with sigma = rms over wet cells of (qq - A sp).  stem: 3x3 conv 4 -> 32 + ReLU; 4 residual blocks
 * x <- x + ReLU(3x3 conv 32 -> 32 (x) + b); head: 3x3 conv 32 -> 1.  Activations and weights are BF16,
 * every accumulation FP32, the output FP32; prediction = sigma * output on wet cells.
 *
 * Parameter vector (FP32, SI3D_NET_NPARAM values), conv weights indexed [tap][cin][cout] with
 * tap = (di + 1) * 3 + (dj + 1) for the neighbour (i + di, j + dj):
 *   stem W [9][4][32], stem b [32], block k = 0..3: W [9][32][32], b [32], head W [9][32], head b [1].
 * Images are channels-last, [B][H][W][C], pixel (i, j) of image b at (b * H + i) * W + j; outside the
 * image every input reads as zero. */
#ifndef SI3D_LEARN_H
#define SI3D_LEARN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SI3D_NET_IN 4
#define SI3D_NET_C 32
#define SI3D_NET_BLOCKS 4
#define SI3D_NET_NPARAM (9 * 4 * 32 + 32 + 4 * (9 * 32 * 32 + 32) + 9 * 32 + 1)

/* ---------------------------------------------------------------- use inside the time step */
/* Load network parameters (host FP32, SI3D_NET_NPARAM values) into a solver handle.  With
 * x0_mode = SI3D_X0_LEARNED the leapfrog solve of every step then starts from sp + prediction (the
 * solve the network is trained on, where sp is the current zeta) and the trapezoidal solves after it
 * from the latest solution.  NULL unloads. */
int si3d_learn_set_params(int handle, const float* params_host);

/* Record training examples: while `dev_buf` is non-NULL, every zeta solve writes one image
 * [im1][jm1][5] FP32 (channels c0..c3 above, then the target (zeta_solution - sp) / sigma) into slot
 * (solve counter mod nslots) of dev_buf (device memory, nslots * im1 * jm1 * 5 floats, owned by the
 * caller).  Returns the handle's image height/width through h/w. */
int si3d_learn_record(int handle, float* dev_buf, int nslots, int* h, int* w);
/* Number of solves recorded since recording was (re)enabled. */
int si3d_learn_recorded(int handle);

/* ---------------------------------------------------------------- training kernels (device pointers) */
/* Workspace bytes that si3d_net_forward/backward need for B images of H x W. */
size_t si3d_net_workspace_bytes(int B, int H, int W);
/* out[B][H][W] = network(feat[B][H][W][4]); keeps the activations in ws for the backward pass. */
int si3d_net_forward(const float* params, const float* feat, int B, int H, int W, float* out, void* ws,
                     size_t ws_bytes);
/* Masked mean-square loss over pixels with mask > 0: loss_dev[0] = sum mask (out - t)^2 / sum mask,
 * loss_dev[1] = sum mask, gout = d loss / d out.  n = B * H * W.  loss_dev is device memory of
 * 2 + 2 * 148 floats (the tail holds block partial sums). */
int si3d_net_loss(const float* out, const float* target, const float* mask, int n, float* gout, float* loss_dev);
/* grad[SI3D_NET_NPARAM] = d loss / d params, from gout and the activations of the last forward. */
int si3d_net_backward(const float* params, const float* feat, const float* gout, int B, int H, int W, float* grad,
                      void* ws, size_t ws_bytes);
/* One Adam step (bias-corrected, step number t >= 1) on n parameters. */
int si3d_net_adam(float* params, const float* grad, float* m, float* v, int n, float lr, float beta1, float beta2,
                  float eps, int t);
/* Synchronise the device (the training kernels run on the default stream). */
int si3d_net_sync(void);

#ifdef __cplusplus
}
#endif

#endif
