// The kernels of the learned start block's network (a multilayer perceptron in FP32: dense layers, ReLU, mean squared
// error, Adam): its inference and its training run on the GPU by these kernels alone. No counterpart in the reference.
//
// denseProduct is a shared-memory tiled FP32 product C = op(A) op(B) with the layers' epilogues; the network is small
// (a few hundred units, a few hundred designs), so one 32 x 32 tile per block of 256 threads (each thread a 2 x 2
// patch) keeps every launch a single wave.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

namespace
{

constexpr int DENSE_TILE = 32;
constexpr int DENSE_DEPTH = 16;

} // namespace

// C (m x n, row-major, leading dimension n) = op(A) op(B) (+ bias[j]) then the epilogue: 0 none, 1 ReLU, 2 multiply
// by the mask (mask[i * n + j] > 0) (ReLU's derivative at the layer's output). op(A) is m x k: A row-major m x k, or
// (transposeA) A row-major k x m read transposed; op(B) is k x n: B row-major k x n, or (transposeB) n x k
// transposed. Every term of an element is summed in k order.
__global__ void __launch_bounds__(256) denseProduct(const float* a, const float* b, float* c, int m, int n, int k,
                                                    int transposeA, int transposeB, const float* bias, int epilogue,
                                                    const float* mask)
{
    __shared__ float sa[DENSE_DEPTH][DENSE_TILE + 1];
    __shared__ float sb[DENSE_DEPTH][DENSE_TILE + 1];
    const int row0 = blockIdx.y * DENSE_TILE;
    const int col0 = blockIdx.x * DENSE_TILE;
    const int tx = threadIdx.x & 15; // columns tx and tx + 16
    const int ty = threadIdx.x >> 4; // rows ty and ty + 16
    float acc[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
    for (int p0 = 0; p0 < k; p0 += DENSE_DEPTH)
    {
        for (int e = threadIdx.x; e < DENSE_DEPTH * DENSE_TILE; e += blockDim.x)
        {
            const int p = e / DENSE_TILE;
            const int t = e - p * DENSE_TILE;
            const int kk = p0 + p;
            const int i = row0 + t;
            const int j = col0 + t;
            float va = 0.0f;
            float vb = 0.0f;
            if (kk < k && i < m)
                va = transposeA ? a[static_cast<std::int64_t>(kk) * m + i] : a[static_cast<std::int64_t>(i) * k + kk];
            if (kk < k && j < n)
                vb = transposeB ? b[static_cast<std::int64_t>(j) * k + kk] : b[static_cast<std::int64_t>(kk) * n + j];
            sa[p][t] = va;
            sb[p][t] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int p = 0; p < DENSE_DEPTH; ++p)
        {
            const float a0 = sa[p][ty];
            const float a1 = sa[p][ty + 16];
            const float b0 = sb[p][tx];
            const float b1 = sb[p][tx + 16];
            acc[0][0] = fmaf(a0, b0, acc[0][0]);
            acc[0][1] = fmaf(a0, b1, acc[0][1]);
            acc[1][0] = fmaf(a1, b0, acc[1][0]);
            acc[1][1] = fmaf(a1, b1, acc[1][1]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v)
        {
            const int i = row0 + ty + 16 * u;
            const int j = col0 + tx + 16 * v;
            if (i >= m || j >= n)
                continue;
            float value = acc[u][v];
            if (bias != nullptr)
                value += bias[j];
            if (epilogue == 1)
                value = fmaxf(value, 0.0f);
            else if (epilogue == 2)
                value = mask[static_cast<std::int64_t>(i) * n + j] > 0.0f ? value : 0.0f;
            c[static_cast<std::int64_t>(i) * n + j] = value;
        }
}

// grad = 2 (y - t) / count, and the squared errors' partial sums per block (partials[blockIdx.x]).
__global__ void squaredError(const float* y, const float* t, float* grad, std::int64_t count, float* partials)
{
    __shared__ float sums[256];
    float sum = 0.0f;
    for (std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < count;
         e += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
    {
        const float d = y[e] - t[e];
        grad[e] = 2.0f * d / static_cast<float>(count);
        sum = fmaf(d, d, sum);
    }
    sums[threadIdx.x] = sum;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1)
    {
        if (static_cast<int>(threadIdx.x) < stride)
            sums[threadIdx.x] += sums[threadIdx.x + stride];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        partials[blockIdx.x] = sums[0];
}

// bias gradient: out[j] = sum over the rows i of g[i * n + j], rows in order.
__global__ void columnSums(const float* g, int rows, int n, float* out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    float sum = 0.0f;
    for (int i = 0; i < rows; ++i)
        sum += g[static_cast<std::int64_t>(i) * n + j];
    out[j] = sum;
}

// Adam (Kingma and Ba, 2015) on `count` parameters: step t >= 1.
__global__ void adamStep(float* w, const float* g, float* m, float* v, std::int64_t count, float rate, float beta1,
                         float beta2, float epsilon, int t)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= count)
        return;
    const float gi = g[e];
    const float mi = beta1 * m[e] + (1.0f - beta1) * gi;
    const float vi = beta2 * v[e] + (1.0f - beta2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    const float mh = mi / (1.0f - powf(beta1, static_cast<float>(t)));
    const float vh = vi / (1.0f - powf(beta2, static_cast<float>(t)));
    w[e] -= rate * mh / (sqrtf(vh) + epsilon);
}

} // namespace oosgpu::device
