// Device evaluation of the hdcx/fpmath.h functions compared bit for bit with
// the host evaluation compiled from the same header. Prints the number of
// mismatches per function; exit status 0 when there are none.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "hdcx/fpmath.h"

namespace {

constexpr int kFunctions = 8;
const char* kNames[kFunctions] = {"sin", "cos", "exp", "log", "pow", "pow5", "acos", "atan2"};

__host__ __device__ float evaluate(int f, float x, float y)
{
    switch (f) {
    case 0: return hdcx_fp_sin(x);
    case 1: return hdcx_fp_cos(x);
    case 2: return hdcx_fp_exp(x);
    case 3: return hdcx_fp_log(x);
    case 4: return hdcx_fp_pow(x, y);
    case 5: return hdcx_fp_pow5(x);
    case 6: return hdcx_fp_acos(x);
    default: return hdcx_fp_atan2(y, x);
    }
}

__global__ void evaluateKernel(const float* x, const float* y, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int f = 0; f < kFunctions; ++f) out[static_cast<size_t>(f) * n + i] = evaluate(f, x[i], y[i]);
}

uint32_t nextRandom(uint64_t& state)
{
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return static_cast<uint32_t>(state >> 32);
}

float bitsToFloat(uint32_t u)
{
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace

int main(int argc, char** argv)
{
    const int n = argc > 1 ? std::atoi(argv[1]) : (1 << 22);
    std::vector<float> x(n), y(n);
    uint64_t state = 0x9e3779b97f4a7c15ull;
    const float specials[] = {0.0f, -0.0f, 1.0f, -1.0f, 0.5f, 2.0f, INFINITY, -INFINITY, NAN,
                              1e-45f, 1e-40f, 1.17549435e-38f, 3.4e38f, 88.72f, -103.9f, 1.41421356f};
    const int nSpecial = static_cast<int>(sizeof specials / sizeof specials[0]);
    for (int i = 0; i < n; ++i) {
        const uint32_t r = nextRandom(state);
        if (i < nSpecial * nSpecial) {
            x[i] = specials[i % nSpecial];
            y[i] = specials[i / nSpecial];
        } else if (r & 1u) {
            // Uniform in [-64, 64] and [-300, 300]: the ordinary argument ranges.
            x[i] = -64.0f + 128.0f * static_cast<float>(nextRandom(state) >> 8) * 0x1p-24f;
            y[i] = -300.0f + 600.0f * static_cast<float>(nextRandom(state) >> 8) * 0x1p-24f;
        } else {
            // Arbitrary bit patterns (every exponent, NaNs and infinities included).
            x[i] = bitsToFloat(nextRandom(state));
            y[i] = bitsToFloat(nextRandom(state));
        }
    }
    float *dx = nullptr, *dy = nullptr, *dout = nullptr;
    const size_t bytes = sizeof(float) * static_cast<size_t>(n);
    if (cudaMalloc(&dx, bytes) != cudaSuccess || cudaMalloc(&dy, bytes) != cudaSuccess ||
        cudaMalloc(&dout, bytes * kFunctions) != cudaSuccess) {
        std::printf("cuda allocation failed\n");
        return 2;
    }
    cudaMemcpy(dx, x.data(), bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dy, y.data(), bytes, cudaMemcpyHostToDevice);
    evaluateKernel<<<(n + 255) / 256, 256>>>(dx, dy, dout, n);
    std::vector<float> out(static_cast<size_t>(n) * kFunctions);
    const cudaError_t status = cudaMemcpy(out.data(), dout, bytes * kFunctions, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dout);
    if (status != cudaSuccess) {
        std::printf("cuda error: %s\n", cudaGetErrorString(status));
        return 2;
    }
    int bad = 0;
    for (int f = 0; f < kFunctions; ++f) {
        long mismatches = 0;
        for (int i = 0; i < n; ++i) {
            const float host = evaluate(f, x[i], y[i]);
            const float dev = out[static_cast<size_t>(f) * n + i];
            uint32_t hb, db;
            std::memcpy(&hb, &host, 4);
            std::memcpy(&db, &dev, 4);
            // Any NaN matches any NaN; everything else must match bit for bit.
            const bool same = (std::isnan(host) && std::isnan(dev)) || hb == db;
            if (!same) {
                if (mismatches < 3)
                    std::printf("  %s(%a, %a): host %a device %a\n", kNames[f], x[i], y[i], host, dev);
                ++mismatches;
            }
        }
        std::printf("%s %d %ld\n", kNames[f], n, mismatches);
        if (mismatches) bad = 1;
    }
    return bad;
}
