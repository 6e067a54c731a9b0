// k_mlp.cu -- the learned r predictor: a 12 -> 64 -> 64 -> 1 MLP with GELU,
// trained and evaluated by these kernels (no framework).
//
// It predicts y = log(d_m / d_{m-1}), the growth of the top-1 squared
// discord distance from one length to the next, from features of the
// previous lengths (see paddi_r_features).  Training minimises the pinball
// (quantile) loss at quantile tau, so the prediction is a low quantile of
// the growth: r^2 = d_{m-1} * exp(y_hat) then usually lies just below the
// true top-1 distance.  A guess above it only costs a retry: PALMAD lowers r
// the way MERLIN does and the discords do not depend on r.
//
// Parameter vector (FP32, MLP_NPARAM values):
//   W1[64][12]  b1[64]  W2[64][64]  b2[64]  W3[64]  b3
// Inference uses a BF16 copy of the weights with FP32 accumulation.
//
// One warp evaluates one sample; lane l owns hidden units l and l + 32.
// Training: each CTA (one warp) accumulates the gradient of its samples in
// shared memory (rows padded to avoid bank conflicts) and adds it to the
// global gradient once; an Adam kernel applies the step.
#include <cuda_bf16.h>

#include "paddi_internal.cuh"

namespace {

constexpr int F = MLP_NFEAT, H = MLP_HIDDEN;
constexpr int OW1 = 0, OB1 = OW1 + H * F, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H,
              OB3 = OW3 + H;
static_assert(OB3 + 1 == MLP_NPARAM, "parameter layout");

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678f)); }
__device__ __forceinline__ float gelu_d(float z)
{
    // d/dz [z Phi(z)] = Phi(z) + z phi(z)
    return 0.5f * (1.f + erff(z * 0.70710678f)) + z * 0.39894228f * expf(-0.5f * z * z);
}

template <typename W>
__device__ __forceinline__ float ld(const W *p, int i);
template <>
__device__ __forceinline__ float ld<float>(const float *p, int i) { return p[i]; }
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16 *p, int i)
{
    return __bfloat162float(p[i]);
}

// View of the parameters; W2 rows may be padded (shared-memory copies use a
// stride of 65 so that a warp reading one column hits 32 different banks).
template <typename W>
struct MlpView {
    const W *w1, *b1, *w2, *b2, *w3, *b3;
    int w2s;
};

template <typename W>
__device__ __forceinline__ MlpView<W> packed_view(const W *P)
{
    return MlpView<W>{P + OW1, P + OB1, P + OW2, P + OB2, P + OW3, P + OB3, H};
}

// Forward pass of one sample by one warp; returns y_hat on every lane and the
// pre-activations / activations of the lane's two units per layer.
template <typename W>
__device__ float mlp_forward(const MlpView<W> &P, const float *x, int lane, float (&z1)[2],
                             float (&h1)[2], float (&z2)[2], float (&h2)[2])
{
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int u = lane + 32 * q;
        float a = ld(P.b1, u);
#pragma unroll
        for (int k = 0; k < F; ++k) a = fmaf(ld(P.w1, u * F + k), x[k], a);
        z1[q] = a;
        h1[q] = gelu(a);
    }
    float a0 = ld(P.b2, lane), a1 = ld(P.b2, lane + 32);
#pragma unroll 4
    for (int v = 0; v < H; ++v) {
        const float hv = __shfl_sync(0xffffffffu, v < 32 ? h1[0] : h1[1], v & 31);
        a0 = fmaf(ld(P.w2, lane * P.w2s + v), hv, a0);
        a1 = fmaf(ld(P.w2, (lane + 32) * P.w2s + v), hv, a1);
    }
    z2[0] = a0;
    z2[1] = a1;
    h2[0] = gelu(a0);
    h2[1] = gelu(a1);
    float y = ld(P.w3, lane) * h2[0] + ld(P.w3, lane + 32) * h2[1];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
    return y + ld(P.b3, 0);
}

template <typename W>
__global__ void k_mlp_forward(const float *__restrict__ X, int n, const W *__restrict__ Pg,
                              float *Y)
{
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const MlpView<W> P = packed_view(Pg);
    for (int s = wid; s < n; s += nw) {
        float x[F];
#pragma unroll
        for (int k = 0; k < F; ++k) x[k] = X[(size_t)s * F + k];
        float z1[2], h1[2], z2[2], h2[2];
        const float y = mlp_forward(P, x, lane, z1, h1, z2, h2);
        if (lane == 0) Y[s] = y;
    }
}

// Gradient of the mean pinball loss over samples [0, n) (added into G; the
// mean loss into *loss).  Shared memory: the parameters (W2 rows padded) and
// this CTA's gradient.
constexpr int WS = H + 1; // padded row stride of W2 and dW2 in shared memory

__global__ void __launch_bounds__(32)
k_mlp_grad(const float *__restrict__ X, const float *__restrict__ Yt, int n, float tau,
           const float *__restrict__ Pg, float *G, float *loss)
{
    __shared__ float sW1[H * F], sB1[H], sW2[H * WS], sB2[H], sW3[H], sB3;
    __shared__ float gW1[H * F], gB1[H], gW2[H * WS], gB2[H], gW3[H];
    __shared__ float gB3, lsum;
    const int lane = threadIdx.x;
    for (int i = lane; i < H * F; i += 32) {
        sW1[i] = Pg[OW1 + i];
        gW1[i] = 0.f;
    }
    for (int i = lane; i < H * H; i += 32) sW2[(i / H) * WS + i % H] = Pg[OW2 + i];
    for (int i = lane; i < H * WS; i += 32) gW2[i] = 0.f;
    for (int i = lane; i < H; i += 32) {
        sB1[i] = Pg[OB1 + i];
        sB2[i] = Pg[OB2 + i];
        sW3[i] = Pg[OW3 + i];
        gB1[i] = 0.f;
        gB2[i] = 0.f;
        gW3[i] = 0.f;
    }
    if (lane == 0) {
        sB3 = Pg[OB3];
        gB3 = 0.f;
        lsum = 0.f;
    }
    __syncwarp();
    const MlpView<float> P{sW1, sB1, sW2, sB2, sW3, &sB3, WS};
    const float inv_n = 1.f / (float)n;
    for (int s = blockIdx.x; s < n; s += gridDim.x) {
        float x[F];
#pragma unroll
        for (int k = 0; k < F; ++k) x[k] = X[(size_t)s * F + k];
        float z1[2], h1[2], z2[2], h2[2];
        const float yh = mlp_forward(P, x, lane, z1, h1, z2, h2);
        const float e = Yt[s] - yh;
        const float l = e > 0.f ? tau * e : (tau - 1.f) * e;
        const float dy = (e > 0.f ? -tau : 1.f - tau) * inv_n;
        if (lane == 0) {
            lsum += l;
            gB3 += dy;
        }
        float dz2[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int u = lane + 32 * q;
            gW3[u] += dy * h2[q];
            dz2[q] = dy * sW3[u] * gelu_d(z2[q]);
            gB2[u] += dz2[q];
        }
        // dW2[u][v] += dz2[u] h1[v]; each lane owns rows u = lane, lane + 32
#pragma unroll 4
        for (int v = 0; v < H; ++v) {
            const float hv = __shfl_sync(0xffffffffu, v < 32 ? h1[0] : h1[1], v & 31);
            gW2[lane * WS + v] += dz2[0] * hv;
            gW2[(lane + 32) * WS + v] += dz2[1] * hv;
        }
        // dh1[v] = sum_u W2[u][v] dz2[u]; each lane owns columns v = lane, lane + 32
        float dh1a = 0.f, dh1b = 0.f;
#pragma unroll 4
        for (int u = 0; u < H; ++u) {
            const float du = __shfl_sync(0xffffffffu, u < 32 ? dz2[0] : dz2[1], u & 31);
            dh1a = fmaf(sW2[u * WS + lane], du, dh1a);
            dh1b = fmaf(sW2[u * WS + lane + 32], du, dh1b);
        }
        const float dz1[2] = {dh1a * gelu_d(z1[0]), dh1b * gelu_d(z1[1])};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int v = lane + 32 * q;
            gB1[v] += dz1[q];
#pragma unroll
            for (int k = 0; k < F; ++k) gW1[v * F + k] += dz1[q] * x[k];
        }
        __syncwarp();
    }
    __syncwarp();
    for (int i = lane; i < H * F; i += 32) atomicAdd(G + OW1 + i, gW1[i]);
    for (int i = lane; i < H; i += 32) {
        atomicAdd(G + OB1 + i, gB1[i]);
        atomicAdd(G + OB2 + i, gB2[i]);
        atomicAdd(G + OW3 + i, gW3[i]);
    }
    for (int i = lane; i < H * H; i += 32) atomicAdd(G + OW2 + i, gW2[(i / H) * WS + i % H]);
    if (lane == 0) {
        atomicAdd(G + OB3, gB3);
        atomicAdd(loss, lsum * inv_n);
    }
}

// Adam step with bias correction; clears the gradient for the next batch.
__global__ void k_mlp_adam(float *P, float *G, float *M, float *V, int np, float lr, float b1,
                           float b2, float eps, float bc1, float bc2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    G[i] = 0.f;
}

__global__ void k_to_bf16(const float *P, __nv_bfloat16 *Q, int np)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < np) Q[i] = __float2bfloat16_rn(P[i]);
}

} // namespace

cudaError_t paddi_launch_mlp_forward(const float *X, int n, const void *P, bool bf16, float *Y,
                                     cudaStream_t st)
{
    const int warps = n < 4096 ? n : 4096;
    const int threads = 128;
    const int grid = (warps * 32 + threads - 1) / threads;
    if (bf16)
        k_mlp_forward<__nv_bfloat16><<<grid > 0 ? grid : 1, threads, 0, st>>>(
            X, n, static_cast<const __nv_bfloat16 *>(P), Y);
    else
        k_mlp_forward<float><<<grid > 0 ? grid : 1, threads, 0, st>>>(
            X, n, static_cast<const float *>(P), Y);
    return cudaGetLastError();
}

cudaError_t paddi_launch_mlp_grad(const float *X, const float *Y, int n, float tau,
                                  const float *P, float *G, float *loss, int num_sms,
                                  cudaStream_t st)
{
    int grid = num_sms * 16;
    if (grid > n) grid = n > 0 ? n : 1;
    k_mlp_grad<<<grid, 32, 0, st>>>(X, Y, n, tau, P, G, loss);
    return cudaGetLastError();
}

cudaError_t paddi_launch_mlp_adam(float *P, float *G, float *M, float *V, float lr, int step,
                                  cudaStream_t st)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(P, G, M, V, MLP_NPARAM, lr, b1, b2, eps,
                                                         bc1, bc2);
    return cudaGetLastError();
}

cudaError_t paddi_launch_mlp_to_bf16(const float *P, void *Q, cudaStream_t st)
{
    k_to_bf16<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(P, static_cast<__nv_bfloat16 *>(Q),
                                                        MLP_NPARAM);
    return cudaGetLastError();
}
