// pb_mlp.cuh — the small MLP of the learned preconditioner correction: forward, backward
// and Adam update as hand-written FP32 kernels.
#pragma once
#include "pb_common.cuh"

#define PB_MLP_IN  12        // features per current cell
#define PB_MLP_H   128       // hidden width (two hidden layers)
#define PB_MLP_OUT 2         // Re, Im of the normalised diagonal correction
// parameter layout: W1[H][IN], b1[H], W2[H][H], b2[H], W3[OUT][H], b3[OUT]
#define PB_MLP_OFF_W1 0
#define PB_MLP_OFF_B1 (PB_MLP_OFF_W1 + PB_MLP_H * PB_MLP_IN)
#define PB_MLP_OFF_W2 (PB_MLP_OFF_B1 + PB_MLP_H)
#define PB_MLP_OFF_B2 (PB_MLP_OFF_W2 + PB_MLP_H * PB_MLP_H)
#define PB_MLP_OFF_W3 (PB_MLP_OFF_B2 + PB_MLP_H)
#define PB_MLP_OFF_B3 (PB_MLP_OFF_W3 + PB_MLP_OUT * PB_MLP_H)
#define PB_MLP_NPARAM (PB_MLP_OFF_B3 + PB_MLP_OUT)

// y[n][OUT] = MLP(x[n][IN]) on the device (weights d_w).
int pb_mlp_forward_dev(const float *d_w, int n, const float *d_x, float *d_y, cudaStream_t s);
