// The learned start block's network on the GPU: a multilayer perceptron inputs -> hidden -> hidden -> outputs (ReLU
// after each hidden layer) in FP32, trained by full-batch Adam on the mean squared error, all of it by the kernels of
// mlp_kernels.cu. Parameters in one flat array: W1 (inputs x hidden, row-major), b1, W2 (hidden x hidden), b2,
// W3 (hidden x outputs), b3; He initialisation from splitmix64 and Box-Muller. No counterpart in the reference.

#include "factor_internal.hpp"
#include "host_api.hpp"
#include "oos_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace oosgpu::device
{
__global__ void denseProduct(const float* a, const float* b, float* c, int m, int n, int k, int transposeA,
                             int transposeB, const float* bias, int epilogue, const float* mask);
__global__ void squaredError(const float* y, const float* t, float* grad, std::int64_t count, float* partials);
__global__ void columnSums(const float* g, int rows, int n, float* out);
__global__ void adamStep(float* w, const float* g, float* m, float* v, std::int64_t count, float rate, float beta1,
                         float beta2, float epsilon, int t);
} // namespace oosgpu::device

namespace
{

constexpr int ERROR_BLOCKS = 64;

void check(cudaError_t status, const char* what)
{
    if (status != cudaSuccess)
        throw oosgpu::Error(oosgpu::STATUS_CUDA, std::string(what) + ": " + cudaGetErrorString(status));
}

template <typename T> struct DeviceBuffer
{
    T* data = nullptr;
    std::size_t count = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer()
    {
        if (data != nullptr)
            cudaFree(data);
    }
    void ensure(std::size_t n, const char* what)
    {
        if (n <= count && data != nullptr)
            return;
        if (data != nullptr)
            cudaFree(data);
        data = nullptr;
        count = 0;
        check(cudaMalloc(reinterpret_cast<void**>(&data), std::max<std::size_t>(n, 1) * sizeof(T)), what);
        count = n;
    }
};

std::uint64_t splitmix(std::uint64_t& state)
{
    std::uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double uniform(std::uint64_t& state)
{
    return static_cast<double>(splitmix(state) >> 11) * (1.0 / 9007199254740992.0);
}

unsigned blocks(std::int64_t items, int threads)
{
    return static_cast<unsigned>((items + threads - 1) / threads);
}

} // namespace

struct oosgpu_mlp
{
    int inputs = 0;
    int hidden = 0;
    int outputs = 0;
    int step = 0;
    std::int64_t offsets[7] = {};
    DeviceBuffer<float> parameters, gradients, moment1, moment2;
    DeviceBuffer<float> x, target, h1, h2, y, dy, dh1, dh2, partials;
    cudaStream_t stream = nullptr;

    [[nodiscard]] std::int64_t parameterCount() const { return offsets[6]; }
    float* w(int layer) { return parameters.data + offsets[2 * layer]; }
    float* b(int layer) { return parameters.data + offsets[2 * layer + 1]; }
    float* gw(int layer) { return gradients.data + offsets[2 * layer]; }
    float* gb(int layer) { return gradients.data + offsets[2 * layer + 1]; }

    void dense(const float* a, const float* bm, float* c, int m, int n, int k, bool ta, bool tb, const float* bias,
               int epilogue, const float* mask)
    {
        const dim3 grid(blocks(n, 32), blocks(m, 32));
        oosgpu::device::denseProduct<<<grid, 256, 0, stream>>>(a, bm, c, m, n, k, ta ? 1 : 0, tb ? 1 : 0, bias,
                                                               epilogue, mask);
        check(cudaGetLastError(), "network: dense product");
    }

    void prepare(int batch)
    {
        x.ensure(static_cast<std::size_t>(batch) * inputs, "network: inputs");
        target.ensure(static_cast<std::size_t>(batch) * outputs, "network: targets");
        h1.ensure(static_cast<std::size_t>(batch) * hidden, "network: activations");
        h2.ensure(static_cast<std::size_t>(batch) * hidden, "network: activations");
        y.ensure(static_cast<std::size_t>(batch) * outputs, "network: outputs");
        dy.ensure(static_cast<std::size_t>(batch) * outputs, "network: gradients");
        dh1.ensure(static_cast<std::size_t>(batch) * hidden, "network: gradients");
        dh2.ensure(static_cast<std::size_t>(batch) * hidden, "network: gradients");
        partials.ensure(ERROR_BLOCKS, "network: loss");
    }

    void forward(int batch)
    {
        dense(x.data, w(0), h1.data, batch, hidden, inputs, false, false, b(0), 1, nullptr);
        dense(h1.data, w(1), h2.data, batch, hidden, hidden, false, false, b(1), 1, nullptr);
        dense(h2.data, w(2), y.data, batch, outputs, hidden, false, false, b(2), 0, nullptr);
    }

    // The gradients of the mean squared error over the batch into `gradients`; returns the loss.
    float backward(int batch)
    {
        const std::int64_t count = static_cast<std::int64_t>(batch) * outputs;
        oosgpu::device::squaredError<<<ERROR_BLOCKS, 256, 0, stream>>>(y.data, target.data, dy.data, count,
                                                                       partials.data);
        check(cudaGetLastError(), "network: loss");
        // layer 3: dW3 = h2^T dy, db3 = column sums of dy, dh2 = (dy W3^T) . [h2 > 0]
        dense(h2.data, dy.data, gw(2), hidden, outputs, batch, true, false, nullptr, 0, nullptr);
        oosgpu::device::columnSums<<<blocks(outputs, 128), 128, 0, stream>>>(dy.data, batch, outputs, gb(2));
        dense(dy.data, w(2), dh2.data, batch, hidden, outputs, false, true, nullptr, 2, h2.data);
        // layer 2
        dense(h1.data, dh2.data, gw(1), hidden, hidden, batch, true, false, nullptr, 0, nullptr);
        oosgpu::device::columnSums<<<blocks(hidden, 128), 128, 0, stream>>>(dh2.data, batch, hidden, gb(1));
        dense(dh2.data, w(1), dh1.data, batch, hidden, hidden, false, true, nullptr, 2, h1.data);
        // layer 1
        dense(x.data, dh1.data, gw(0), inputs, hidden, batch, true, false, nullptr, 0, nullptr);
        oosgpu::device::columnSums<<<blocks(hidden, 128), 128, 0, stream>>>(dh1.data, batch, hidden, gb(0));
        check(cudaGetLastError(), "network: bias gradients");
        std::vector<float> sums(ERROR_BLOCKS);
        check(cudaMemcpyAsync(sums.data(), partials.data, ERROR_BLOCKS * sizeof(float), cudaMemcpyDeviceToHost,
                                      stream),
                      "network: loss");
        check(cudaStreamSynchronize(stream), "network: loss");
        double total = 0.0;
        for (const float v : sums)
            total += v;
        return static_cast<float>(total / static_cast<double>(count));
    }

    void upload(float* dst, const float* src, std::size_t n, const char* what)
    {
        check(cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyHostToDevice, stream), what);
    }
};

namespace
{

void requireShape(const oosgpu_mlp* mlp, int batch)
{
    if (mlp == nullptr)
        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "network: null handle");
    if (batch < 1)
        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "network: the batch must hold at least one sample");
}

void requireData(const void* p, const char* what)
{
    if (p == nullptr)
        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, std::string("network: null ") + what);
}

} // namespace

extern "C" int oosgpu_mlp_create(int32_t inputs, int32_t hidden, int32_t outputs, uint64_t seed, int device,
                                 oosgpu_mlp** out)
{
    return oosgpu::runGuarded(
        [&]
        {
            requireData(out, "output handle");
            if (inputs < 1 || hidden < 1 || outputs < 1)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "network: the layer widths must be positive");
            check(cudaSetDevice(device), "cudaSetDevice");
            auto mlp = std::make_unique<oosgpu_mlp>();
            mlp->inputs = inputs;
            mlp->hidden = hidden;
            mlp->outputs = outputs;
            const std::int64_t sizes[6] = {static_cast<std::int64_t>(inputs) * hidden, hidden,
                                           static_cast<std::int64_t>(hidden) * hidden, hidden,
                                           static_cast<std::int64_t>(hidden) * outputs, outputs};
            for (int i = 0; i < 6; ++i)
                mlp->offsets[i + 1] = mlp->offsets[i] + sizes[i];
            const auto count = static_cast<std::size_t>(mlp->parameterCount());
            check(cudaStreamCreateWithFlags(&mlp->stream, cudaStreamNonBlocking), "network: stream");
            mlp->parameters.ensure(count, "network: parameters");
            mlp->gradients.ensure(count, "network: gradients");
            mlp->moment1.ensure(count, "network: Adam moments");
            mlp->moment2.ensure(count, "network: Adam moments");
            // He initialisation: N(0, 2 / fan_in) weights, zero biases.
            std::vector<float> host(count, 0.0f);
            std::uint64_t state = seed;
            const int fanIn[3] = {inputs, hidden, hidden};
            for (int layer = 0; layer < 3; ++layer)
            {
                const double sigma = std::sqrt(2.0 / fanIn[layer]);
                for (std::int64_t e = mlp->offsets[2 * layer]; e < mlp->offsets[2 * layer + 1]; ++e)
                {
                    const double u1 = 1.0 - uniform(state);
                    const double u2 = uniform(state);
                    host[static_cast<std::size_t>(e)] = static_cast<float>(
                        sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
                }
            }
            mlp->upload(mlp->parameters.data, host.data(), count, "network: parameters");
            check(cudaMemsetAsync(mlp->moment1.data, 0, count * sizeof(float), mlp->stream), "memset");
            check(cudaMemsetAsync(mlp->moment2.data, 0, count * sizeof(float), mlp->stream), "memset");
            check(cudaStreamSynchronize(mlp->stream), "network: set-up");
            *out = mlp.release();
        });
}

extern "C" void oosgpu_mlp_destroy(oosgpu_mlp* mlp)
{
    if (mlp == nullptr)
        return;
    if (mlp->stream != nullptr)
    {
        cudaStreamSynchronize(mlp->stream);
        cudaStreamDestroy(mlp->stream);
    }
    delete mlp;
}

extern "C" int64_t oosgpu_mlp_parameter_count(const oosgpu_mlp* mlp)
{
    return mlp == nullptr ? 0 : mlp->parameterCount();
}

extern "C" int oosgpu_mlp_get_parameters(oosgpu_mlp* mlp, float* parameters)
{
    return oosgpu::runGuarded(
        [&]
        {
            requireShape(mlp, 1);
            requireData(parameters, "parameters");
            check(cudaMemcpyAsync(parameters, mlp->parameters.data, mlp->parameterCount() * sizeof(float),
                                          cudaMemcpyDeviceToHost, mlp->stream),
                          "network: parameters");
            check(cudaStreamSynchronize(mlp->stream), "network: parameters");
        });
}

extern "C" int oosgpu_mlp_set_parameters(oosgpu_mlp* mlp, const float* parameters)
{
    return oosgpu::runGuarded(
        [&]
        {
            requireShape(mlp, 1);
            requireData(parameters, "parameters");
            mlp->upload(mlp->parameters.data, parameters, static_cast<std::size_t>(mlp->parameterCount()),
                        "network: parameters");
            check(cudaStreamSynchronize(mlp->stream), "network: parameters");
        });
}

extern "C" int oosgpu_mlp_predict(oosgpu_mlp* mlp, const float* inputs, int32_t batch, float* outputs)
{
    return oosgpu::runGuarded(
        [&]
        {
            requireShape(mlp, batch);
            requireData(inputs, "inputs");
            requireData(outputs, "outputs");
            mlp->prepare(batch);
            mlp->upload(mlp->x.data, inputs, static_cast<std::size_t>(batch) * mlp->inputs, "network: inputs");
            mlp->forward(batch);
            check(cudaMemcpyAsync(outputs, mlp->y.data, static_cast<std::size_t>(batch) * mlp->outputs * sizeof(float),
                                          cudaMemcpyDeviceToHost, mlp->stream),
                          "network: outputs");
            check(cudaStreamSynchronize(mlp->stream), "network: predict");
        });
}

extern "C" int oosgpu_mlp_gradients(oosgpu_mlp* mlp, const float* inputs, const float* targets, int32_t batch,
                                    float* gradients, float* loss)
{
    return oosgpu::runGuarded(
        [&]
        {
            requireShape(mlp, batch);
            requireData(inputs, "inputs");
            requireData(targets, "targets");
            mlp->prepare(batch);
            mlp->upload(mlp->x.data, inputs, static_cast<std::size_t>(batch) * mlp->inputs, "network: inputs");
            mlp->upload(mlp->target.data, targets, static_cast<std::size_t>(batch) * mlp->outputs, "network: targets");
            mlp->forward(batch);
            const float value = mlp->backward(batch);
            if (loss != nullptr)
                *loss = value;
            if (gradients != nullptr)
            {
                check(cudaMemcpyAsync(gradients, mlp->gradients.data, mlp->parameterCount() * sizeof(float),
                                              cudaMemcpyDeviceToHost, mlp->stream),
                              "network: gradients");
                check(cudaStreamSynchronize(mlp->stream), "network: gradients");
            }
        });
}

extern "C" int oosgpu_mlp_train(oosgpu_mlp* mlp, const float* inputs, const float* targets, int32_t batch,
                                int32_t epochs, float rate, float* losses)
{
    return oosgpu::runGuarded(
        [&]
        {
            requireShape(mlp, batch);
            requireData(inputs, "inputs");
            requireData(targets, "targets");
            if (epochs < 0 || !(rate > 0.0f))
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT,
                                    "network: expected epochs >= 0 and a positive learning rate");
            mlp->prepare(batch);
            mlp->upload(mlp->x.data, inputs, static_cast<std::size_t>(batch) * mlp->inputs, "network: inputs");
            mlp->upload(mlp->target.data, targets, static_cast<std::size_t>(batch) * mlp->outputs, "network: targets");
            const std::int64_t count = mlp->parameterCount();
            for (int epoch = 0; epoch < epochs; ++epoch)
            {
                mlp->forward(batch);
                const float value = mlp->backward(batch);
                if (losses != nullptr)
                    losses[epoch] = value;
                ++mlp->step;
                oosgpu::device::adamStep<<<blocks(count, 256), 256, 0, mlp->stream>>>(
                    mlp->parameters.data, mlp->gradients.data, mlp->moment1.data, mlp->moment2.data, count, rate,
                    0.9f, 0.999f, 1.0e-8f, mlp->step);
                check(cudaGetLastError(), "network: Adam step");
            }
            check(cudaStreamSynchronize(mlp->stream), "network: training");
        });
}
