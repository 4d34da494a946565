// The learned cost model of the multiply dispatch: a small FP32 MLP
//   x (FFG_MLP_D features) -> tanh(W1 x + b1) (H) -> tanh(W2 h1 + b2) (H)
//     -> W3 h2 + b3 (FFG_MLP_K outputs: predicted log2 microseconds per
//        product of each method)
// trained on the autotuner's own timings.  A training row is (features,
// method, measured log2 us); the loss is 1/2 the mean squared error of the
// row's method output only.
//
// k_mlp_train runs whole training in one CTA of 256 threads: parameters,
// gradients and Adam moments live in shared memory; per epoch every warp
// takes 32 rows at a time (one per lane), runs forward and backward in
// registers, sums each gradient over the warp with shuffles and adds it to
// shared memory, then the CTA applies one Adam step.  k_mlp_grad is one
// full-batch gradient (for the check against the CPU restatement);
// k_mlp_infer evaluates every output for a list of feature rows, one thread
// a row.
#include "ffg.h"
#include "ffg_internal.h"

namespace ffg {

constexpr int D = FFG_MLP_D, H = FFG_MLP_H, K = FFG_MLP_K;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * D, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + K * H, NPARAM = OFF_B3 + K;
static_assert(NPARAM == FFG_MLP_NPARAM, "parameter layout");
constexpr int MLP_THREADS = 256; // 255 registers a thread: a row's activations stay in registers

FFG_DEV_INLINE float warp_sum(float v) {
#pragma unroll
    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

// Forward of one row: hidden activations and the output of `method`.
FFG_DEV_INLINE float mlp_forward(const float *P, const float *x, int method, float (&h1)[H], float (&h2)[H]) {
#pragma unroll
    for (int j = 0; j < H; j++) {
        float z = P[OFF_B1 + j];
#pragma unroll
        for (int i = 0; i < D; i++) z += P[OFF_W1 + j * D + i] * x[i];
        h1[j] = tanhf(z);
    }
#pragma unroll
    for (int k = 0; k < H; k++) {
        float z = P[OFF_B2 + k];
#pragma unroll
        for (int j = 0; j < H; j++) z += P[OFF_W2 + k * H + j] * h1[j];
        h2[k] = tanhf(z);
    }
    float o = P[OFF_B3 + method];
#pragma unroll
    for (int k = 0; k < H; k++) o += P[OFF_W3 + method * H + k] * h2[k];
    return o;
}

// Adds this warp's gradient of rows (one per lane, `active` lanes valid,
// scale dscale) into G.  Lanes hold their row; every parameter's
// contribution is summed over the warp, then added once.
FFG_DEV_INLINE float mlp_backward_add(const float *P, float *G, const float *x, int method, float y, bool active,
                                      float dscale) {
    const int lane = threadIdx.x & 31;
    float h1[H], h2[H];
    float o = active ? mlp_forward(P, x, method, h1, h2) : 0.f;
    if (!active) {
#pragma unroll
        for (int j = 0; j < H; j++) h1[j] = h2[j] = 0.f;
    }
    const float err = active ? o - y : 0.f;
    const float dout = err * dscale;
    // output layer: only `method`'s row; lanes may differ, so loop over methods
#pragma unroll
    for (int m = 0; m < K; m++) {
        const float dm = method == m ? dout : 0.f;
        const float sb = warp_sum(dm);
        if (lane == 0) atomicAdd(&G[OFF_B3 + m], sb);
#pragma unroll
        for (int k = 0; k < H; k++) {
            const float s = warp_sum(dm * h2[k]);
            if (lane == 0) atomicAdd(&G[OFF_W3 + m * H + k], s);
        }
    }
    float dz2[H];
#pragma unroll
    for (int k = 0; k < H; k++) dz2[k] = dout * P[OFF_W3 + method * H + k] * (1.f - h2[k] * h2[k]);
#pragma unroll
    for (int k = 0; k < H; k++) {
        const float sb = warp_sum(dz2[k]);
        if (lane == 0) atomicAdd(&G[OFF_B2 + k], sb);
    }
#pragma unroll
    for (int k = 0; k < H; k++)
#pragma unroll
        for (int j = 0; j < H; j++) {
            const float s = warp_sum(dz2[k] * h1[j]);
            if (lane == (j & 31)) atomicAdd(&G[OFF_W2 + k * H + j], s);
        }
#pragma unroll
    for (int j = 0; j < H; j++) {
        float dh = 0.f;
#pragma unroll
        for (int k = 0; k < H; k++) dh += P[OFF_W2 + k * H + j] * dz2[k];
        const float dz1 = dh * (1.f - h1[j] * h1[j]);
        const float sb = warp_sum(dz1);
        if (lane == 0) atomicAdd(&G[OFF_B1 + j], sb);
#pragma unroll
        for (int i = 0; i < D; i++) {
            const float s = warp_sum(dz1 * x[i]);
            if (lane == i) atomicAdd(&G[OFF_W1 + j * D + i], s);
        }
    }
    return 0.5f * err * err;
}

// One pass over all rows: gradient of the mean loss into G (zeroed by the
// caller), the summed loss returned to thread 0 (via red).
FFG_DEV_INLINE void mlp_epoch_grad(const float *P, float *G, const float *__restrict__ X, const int32_t *__restrict__ M,
                                   const float *__restrict__ Y, uint32_t n, float *red) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const float dscale = 1.f / (float)n;
    float lsum = 0.f;
    for (uint32_t base = warp * 32; base < n; base += nw * 32) {
        const uint32_t r = base + lane;
        const bool active = r < n;
        float x[D];
#pragma unroll
        for (int i = 0; i < D; i++) x[i] = active ? X[(size_t)r * D + i] : 0.f;
        const int m = active ? M[r] : 0;
        const float y = active ? Y[r] : 0.f;
        lsum += mlp_backward_add(P, G, x, m, y, active, dscale);
    }
    lsum = warp_sum(lsum);
    if (lane == 0) atomicAdd(red, lsum);
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_train(float *params, const float *__restrict__ X,
                                                           const int32_t *__restrict__ M, const float *__restrict__ Y,
                                                           uint32_t n, uint32_t epochs, float lr, float *loss_hist) {
    __shared__ float P[NPARAM], G[NPARAM], Am[NPARAM], Av[NPARAM];
    __shared__ float red;
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) {
        P[i] = params[i];
        Am[i] = Av[i] = 0.f;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float b1t = 1.f, b2t = 1.f;
    for (uint32_t e = 0; e < epochs; e++) {
        for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) G[i] = 0.f;
        if (threadIdx.x == 0) red = 0.f;
        __syncthreads();
        mlp_epoch_grad(P, G, X, M, Y, n, &red);
        __syncthreads();
        b1t *= b1;
        b2t *= b2;
        for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) {
            const float g = G[i];
            Am[i] = b1 * Am[i] + (1.f - b1) * g;
            Av[i] = b2 * Av[i] + (1.f - b2) * g * g;
            const float mh = Am[i] / (1.f - b1t), vh = Av[i] / (1.f - b2t);
            P[i] -= lr * mh / (sqrtf(vh) + eps);
        }
        if (threadIdx.x == 0 && loss_hist) loss_hist[e] = red / (float)n;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) params[i] = P[i];
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_grad(const float *params, const float *__restrict__ X,
                                                          const int32_t *__restrict__ M, const float *__restrict__ Y,
                                                          uint32_t n, float *grad, float *loss) {
    __shared__ float P[NPARAM], G[NPARAM];
    __shared__ float red;
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) {
        P[i] = params[i];
        G[i] = 0.f;
    }
    if (threadIdx.x == 0) red = 0.f;
    __syncthreads();
    mlp_epoch_grad(P, G, X, M, Y, n, &red);
    __syncthreads();
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) grad[i] = G[i];
    if (threadIdx.x == 0) *loss = red / (float)n;
}

__global__ void __launch_bounds__(256) k_mlp_infer(const float *params, const float *__restrict__ X, uint32_t n,
                                                   float *out) {
    __shared__ float P[NPARAM];
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float x[D], h1[H], h2[H];
#pragma unroll
    for (int i = 0; i < D; i++) x[i] = X[(size_t)r * D + i];
    mlp_forward(P, x, 0, h1, h2);
#pragma unroll
    for (int m = 0; m < K; m++) {
        float o = P[OFF_B3 + m];
#pragma unroll
        for (int k = 0; k < H; k++) o += P[OFF_W3 + m * H + k] * h2[k];
        out[(size_t)r * K + m] = o;
    }
}

cudaError_t launch_mlp_train(float *d_params, const float *d_X, const int32_t *d_M, const float *d_Y, uint32_t n,
                             uint32_t epochs, float lr, float *d_loss_hist, cudaStream_t st) {
    k_mlp_train<<<1, MLP_THREADS, 0, st>>>(d_params, d_X, d_M, d_Y, n, epochs, lr, d_loss_hist);
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float *d_params, const float *d_X, const int32_t *d_M, const float *d_Y, uint32_t n,
                            float *d_grad, float *d_loss, cudaStream_t st) {
    k_mlp_grad<<<1, MLP_THREADS, 0, st>>>(d_params, d_X, d_M, d_Y, n, d_grad, d_loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const float *d_params, const float *d_X, uint32_t n, float *d_out, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_mlp_infer<<<(n + 255) / 256, 256, 0, st>>>(d_params, d_X, n, d_out);
    return cudaGetLastError();
}

} // namespace ffg
