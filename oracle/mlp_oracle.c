/*
 * Cost-model oracle -- TEST INFRASTRUCTURE, not product code.
 *
 * A plain scalar C restatement, in double precision, of the learned
 * dispatch's FP32 MLP (the GPU kernels in fastfib_b200/csrc/ffg_mlp.cu):
 *   x (8) -> tanh(W1 x + b1) (32) -> tanh(W2 h1 + b2) (32) -> W3 h2 + b3 (4)
 * with parameters packed W1[32][8] b1[32] W2[32][32] b2[32] W3[4][32] b3[4],
 * the loss 1/2 mean over rows of (output[method] - y)^2, and its gradient by
 * backpropagation.  The reference has no learned part (it dispatches by fixed
 * thresholds, src/mul_basic.c:30-38); this file is the CPU side of the
 * gradient check of the GPU training and inference kernels.
 */
#include "fastfib_oracle.h"

#include <math.h>
#include <string.h>

#define D 8
#define H 32
#define K 4
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + H * D)
#define OFF_W2 (OFF_B1 + H)
#define OFF_B2 (OFF_W2 + H * H)
#define OFF_W3 (OFF_B2 + H)
#define OFF_B3 (OFF_W3 + K * H)
#define NPARAM (OFF_B3 + K)

size_t fo_mlp_nparam(void) { return NPARAM; }

static void forward(const float *P, const float *x, double *h1, double *h2, double *out) {
    for (int j = 0; j < H; j++) {
        double z = P[OFF_B1 + j];
        for (int i = 0; i < D; i++) z += (double)P[OFF_W1 + j * D + i] * x[i];
        h1[j] = tanh(z);
    }
    for (int k = 0; k < H; k++) {
        double z = P[OFF_B2 + k];
        for (int j = 0; j < H; j++) z += (double)P[OFF_W2 + k * H + j] * h1[j];
        h2[k] = tanh(z);
    }
    for (int m = 0; m < K; m++) {
        double o = P[OFF_B3 + m];
        for (int k = 0; k < H; k++) o += (double)P[OFF_W3 + m * H + k] * h2[k];
        out[m] = o;
    }
}

void fo_mlp_predict(const float *params, const float *X, size_t n, double *out) {
    double h1[H], h2[H];
    for (size_t r = 0; r < n; r++) forward(params, X + r * D, h1, h2, out + r * K);
}

double fo_mlp_grad(const float *params, const float *X, const int32_t *method, const float *y, size_t n,
                   double *grad) {
    memset(grad, 0, NPARAM * sizeof(double));
    double loss = 0;
    for (size_t r = 0; r < n; r++) {
        const float *x = X + r * D;
        const int m = method[r];
        double h1[H], h2[H], out[K], dz2[H];
        forward(params, x, h1, h2, out);
        const double err = out[m] - y[r], dout = err / (double)n;
        loss += 0.5 * err * err;
        grad[OFF_B3 + m] += dout;
        for (int k = 0; k < H; k++) {
            grad[OFF_W3 + m * H + k] += dout * h2[k];
            dz2[k] = dout * params[OFF_W3 + m * H + k] * (1 - h2[k] * h2[k]);
            grad[OFF_B2 + k] += dz2[k];
            for (int j = 0; j < H; j++) grad[OFF_W2 + k * H + j] += dz2[k] * h1[j];
        }
        for (int j = 0; j < H; j++) {
            double dh = 0;
            for (int k = 0; k < H; k++) dh += params[OFF_W2 + k * H + j] * dz2[k];
            const double dz1 = dh * (1 - h1[j] * h1[j]);
            grad[OFF_B1 + j] += dz1;
            for (int i = 0; i < D; i++) grad[OFF_W1 + j * D + i] += dz1 * x[i];
        }
    }
    return loss / (double)n;
}
