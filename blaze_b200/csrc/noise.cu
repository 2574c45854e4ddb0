// noise.cu — blz_noise: the reference's noise library (noise.cuh) evaluated
// over arrays of positions.  One thread per position in a grid-stride loop;
// the function is uniform across the launch, so its switch does not diverge.
#include <cstdio>

#include "kernels.cuh"
#include "noise.cuh"

namespace blz {

__global__ void __launch_bounds__(256) k_noise(blz_noise_args a, const float *__restrict__ pos3, long long n,
                                               float *__restrict__ out) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride)
        out[t] = noise::eval(a, pos3[3 * t], pos3[3 * t + 1], pos3[3 * t + 2]);
}

static int noise_blocks(long long n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (n + 255) / 256, cap = 8LL * sms;
    return (int)(want < cap ? want : cap);
}

static int noise_fail(int code, const char *fmt, const char *detail) {
    char buf[256];
    std::snprintf(buf, sizeof buf, fmt, detail);
    set_thread_error(buf);
    return code;
}

static bool noise_args_ok(const blz_noise_args *a) {
    const bool basis_ok = a->basis >= 0 && a->basis <= BLZ_NOISE_SPOTS && a->basis_out >= 0 &&
                          a->basis_out <= BLZ_NOISE_SPOTS;
    return a->func >= 0 && a->func < BLZ_NOISE_COUNT && basis_ok && a->octaves >= 0 && a->octaves <= 64 &&
           a->min_num <= a->max_num && a->shape >= BLZ_SHAPE_STEP && a->shape <= BLZ_SHAPE_QUADRATIC &&
           (long long)a->max_num - a->min_num < 0x7fffffffLL;
}

} // namespace blz

using namespace blz;

extern "C" int blz_noise(const blz_noise_args *a, const float *pos3, long long n, float *out, int on_device,
                         void *stream) {
    if (!a || n < 0 || (n > 0 && (!pos3 || !out)))
        return noise_fail(BLZ_ERR_ARG, "blz_noise: %s", "null argument or negative count");
    if (!noise_args_ok(a))
        return noise_fail(BLZ_ERR_ARG, "blz_noise: %s",
                          "bad function, basis, shape, octaves (0..64) or feature-point range");
    if (n == 0) return BLZ_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (on_device) {
        k_noise<<<noise_blocks(n), 256, 0, st>>>(*a, pos3, n, out);
        e = cudaGetLastError();
        return e == cudaSuccess ? BLZ_OK : noise_fail(BLZ_ERR_CUDA, "blz_noise: %s", cudaGetErrorString(e));
    }
    float *d = nullptr;
    e = cudaMalloc(&d, sizeof(float) * 4 * (size_t)n);
    if (e != cudaSuccess) return noise_fail(BLZ_ERR_CUDA, "blz_noise: %s", cudaGetErrorString(e));
    e = cudaMemcpyAsync(d, pos3, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_noise<<<noise_blocks(n), 256, 0, st>>>(*a, d, n, d + 3 * (size_t)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d + 3 * (size_t)n, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    return e == cudaSuccess ? BLZ_OK : noise_fail(BLZ_ERR_CUDA, "blz_noise: %s", cudaGetErrorString(e));
}
