// unet.cu — the learned warm start of the pressure solve: a 4-level 3-D
// U-Net (channels 16/32/64/128, two 3x3x3 convolutions + ReLU per level,
// 2x2x2 average pooling, 2x2x2 stride-2 transposed convolutions, skip
// concatenation, a 1x1x1 head).  No counterpart in the reference, which has
// no learned components; its solve (src/FluidSolver.cu:517-599) is what the
// network warm-starts.
//
// Inputs per cell (channels-last BF16, 16 channels, 4 used):
//   0  b / rms(b)                b = rho dx^2/dt * rhs, the system's right side
//   1  Neumann ghost indicator   1 in halo voxels beyond a wall (or any open
//                                face when the solve has no Dirichlet ghost)
//   2  p_prev / rms(p_prev)
//   3  r / rms(r)                r = b - A p_prev, A the solver's 7-point operator
// Output: delta = head(features) and the correction d = kappa*rms(r)*delta.
// The solver may sweep p and d alike k times first (d with a zero right-hand
// side; Gauss-Seidel is affine, so S^k(p + alpha d) = S^k(p) + alpha M^k d
// for every alpha; blz_unet_set_smoothing, default k = 0) and adds
// alpha M^k d.  By default alpha minimises the error's energy norm,
// alpha = <d, r> / <d, A d> (A symmetric positive definite), which weighs
// the smooth error Gauss-Seidel removes slowest as the sweep count does, and
// can never raise ||p* - p||_A.  The other choice (blz_unet_set_step)
// minimises the residual norm ||b - A (S^k(p) + alpha M^k d)||, the
// combination chosen on what the stopping rule measures.  A useless d gets
// alpha ~ 0.  rms() and the inner products run over the whole grid in FP64;
// kappa is a constant of the trained weights (the training set's mean
// rms(p* - p_prev) / rms(r)).
//
// The 3x3x3 and the transposed convolutions (forward, data and weight
// gradients) run on the tcgen05 tensor cores (unet_conv.cu).  Pooling, bias
// gradients, the loss and Adam are SIMT kernels: together they are a small
// share of the FLOPs.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "kernels.cuh"

using bf16 = __nv_bfloat16;

namespace blz {
namespace {

constexpr int kSlack = BLZ_CONV_SLACK;
constexpr int kInCh = 16;

struct LDims { int W, H, D; };

__host__ __device__ __forceinline__ long long pvox(const LDims &d, int x, int y, int z) {
    return ((long long)(z + 1) * (d.H + 2) + (y + 1)) * (long long)(d.W + 2) + (x + 1);
}

size_t tensor_voxels(const LDims &d) {
    return 2 * (size_t)kSlack + (size_t)(d.W + 2) * (size_t)(d.H + 2) * (size_t)(d.D + 2);
}

// A full-grid scalar field, natural layout (x fastest) when b == nullptr,
// colour packed (red r, black b) otherwise.
struct CellArr {
    const float *r, *b;
    __device__ __forceinline__ float at(int i, int j, int k, int W, int H) const {
        if (!b) return __ldg(r + lin(i, j, k, W, H));
        return __ldg((((i + j + k) & 1) ? b : r) + pidx(i, j, k, W >> 1, H));
    }
};

struct GridInfo {
    int W, H, D;
    OpenFaces open;
    int dirichlet;
    float scale;                          // rho dx^2 / dt
};

// b, p and r = b - A p of one cell (A p = sum over the in-domain neighbours
// of p - p_nb, plus p for each p = 0 ghost of a Dirichlet open face), the
// operator the Gauss-Seidel sweeps solve.
__device__ __forceinline__ void cell_brp(const GridInfo &g, const CellArr &rhs, const CellArr &p, int i, int j,
                                         int k, float &b, float &pc, float &r) {
    pc = p.at(i, j, k, g.W, g.H);
    b = g.scale * rhs.at(i, j, k, g.W, g.H);
    float ap = 0.0f;
    const bool d = g.dirichlet;
    if (i > 0) ap += pc - p.at(i - 1, j, k, g.W, g.H); else if (d && g.open.xlo) ap += pc;
    if (i < g.W - 1) ap += pc - p.at(i + 1, j, k, g.W, g.H); else if (d && g.open.xhi) ap += pc;
    if (j > 0) ap += pc - p.at(i, j - 1, k, g.W, g.H); else if (d && g.open.ylo) ap += pc;
    if (j < g.H - 1) ap += pc - p.at(i, j + 1, k, g.W, g.H); else if (d && g.open.yhi) ap += pc;
    if (k > 0) ap += pc - p.at(i, j, k - 1, g.W, g.H); else if (d && g.open.zlo) ap += pc;
    if (k < g.D - 1) ap += pc - p.at(i, j, k + 1, g.W, g.H); else if (d && g.open.zhi) ap += pc;
    r = b - ap;
}

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// x, y, z of index v of a W x H x D box in 32-bit arithmetic (every index
// here is below 2^32: blz_unet_create caps the grid at 2^28 cells).
__device__ __forceinline__ void split3(long long v, int W, int H, int &x, int &y, int &z) {
    const unsigned u = (unsigned)v, q = u / (unsigned)W, zq = q / (unsigned)H;
    x = (int)(u - q * (unsigned)W);
    y = (int)(q - zq * (unsigned)H);
    z = (int)zq;
}

constexpr int kNormThreads = 256;
constexpr int kNormBlocks = 1024;                  // partials capacity (blocks of the reductions)

// Grid of a grid-stride reduction kernel: one wave of as many blocks as are
// resident on the device's SMs (at most kNormBlocks), so no block waits for a
// second wave.
template <typename K>
static int one_wave(K kernel) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kNormThreads, 0);
    return std::max(1, std::min(kNormBlocks, sms * std::max(1, per)));
}

// Sums of b^2, p^2, r^2 over the grid (FP64), one triple per block.
__global__ void __launch_bounds__(kNormThreads)
k_unet_norms(GridInfo g, CellArr rhs, CellArr p, double *partials) {
    const long long n = (long long)g.W * g.H * g.D;
    double sb = 0.0, sp = 0.0, sr = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        split3(t, g.W, g.H, i, j, k);
        float b, pc, r;
        cell_brp(g, rhs, p, i, j, k, b, pc, r);
        sb += (double)b * b;
        sp += (double)pc * pc;
        sr += (double)r * r;
    }
    __shared__ double s[3][kNormThreads / 32];
    sb = warp_sum_d(sb); sp = warp_sum_d(sp); sr = warp_sum_d(sr);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { s[0][w] = sb; s[1][w] = sp; s[2][w] = sr; }
    __syncthreads();
    if (w == 0) {
        sb = lane < kNormThreads / 32 ? s[0][lane] : 0.0;
        sp = lane < kNormThreads / 32 ? s[1][lane] : 0.0;
        sr = lane < kNormThreads / 32 ? s[2][lane] : 0.0;
        sb = warp_sum_d(sb); sp = warp_sum_d(sp); sr = warp_sum_d(sr);
        if (lane == 0) {
            partials[3 * blockIdx.x] = sb;
            partials[3 * blockIdx.x + 1] = sp;
            partials[3 * blockIdx.x + 2] = sr;
        }
    }
}

// scales = {1/rms(b), 1/rms(p), 1/rms(r), kappa*rms(r)} (0 where an rms is 0).
__global__ void k_unet_scales(const double *partials, int nblk, double ncells, float kappa, float *scales) {
    __shared__ double s[3][32];
    double a[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        for (int q = 0; q < 3; ++q) a[q] += partials[3 * b + q];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < 3; ++q) {
        a[q] = warp_sum_d(a[q]);
        if (lane == 0) s[q][w] = a[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double rms[3];
        for (int q = 0; q < 3; ++q) {
            double t = 0.0;
            for (int i = 0; i < (int)(blockDim.x + 31) / 32; ++i) t += s[q][i];
            rms[q] = sqrt(t / ncells);
        }
        scales[0] = rms[0] > 0.0 ? (float)(1.0 / rms[0]) : 0.0f;
        scales[1] = rms[1] > 0.0 ? (float)(1.0 / rms[1]) : 0.0f;
        scales[2] = rms[2] > 0.0 ? (float)(1.0 / rms[2]) : 0.0f;
        scales[3] = (float)(kappa * rms[2]);
    }
}

// Input tensor of the crop [o, o + dims) of the grid, halo included: a halo
// voxel inside the grid carries the grid's values, one outside carries the
// Neumann-ghost indicator.
__global__ void k_unet_input(GridInfo g, CellArr rhs, CellArr p, int ox, int oy, int oz, LDims d,
                             const float *__restrict__ scales, bf16 *__restrict__ x0) {
    const long long Wp = d.W + 2, Hp = d.H + 2;
    const long long n = Wp * Hp * (d.D + 2);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    int xp, yp, zp;
    split3(t, (int)Wp, (int)Hp, xp, yp, zp);
    const int i = ox + xp - 1, j = oy + yp - 1, k = oz + zp - 1;
    float v[kInCh];
#pragma unroll
    for (int c = 0; c < kInCh; ++c) v[c] = 0.0f;
    if (i >= 0 && i < g.W && j >= 0 && j < g.H && k >= 0 && k < g.D) {
        float b, pc, r;
        cell_brp(g, rhs, p, i, j, k, b, pc, r);
        v[0] = b * scales[0];
        v[2] = pc * scales[1];
        v[3] = r * scales[2];
    } else {
        // Open in the solve's sense only when it is a p = 0 ghost.
        const bool d_ = g.dirichlet;
        bool neumann = false;
        if (i < 0) neumann |= !(d_ && g.open.xlo);
        if (i >= g.W) neumann |= !(d_ && g.open.xhi);
        if (j < 0) neumann |= !(d_ && g.open.ylo);
        if (j >= g.H) neumann |= !(d_ && g.open.yhi);
        if (k < 0) neumann |= !(d_ && g.open.zlo);
        if (k >= g.D) neumann |= !(d_ && g.open.zhi);
        v[1] = neumann ? 1.0f : 0.0f;
    }
    __nv_bfloat162 h[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    uint4 *dst = reinterpret_cast<uint4 *>(x0 + t * kInCh);
    dst[0] = *reinterpret_cast<uint4 *>(&h[0]);
    dst[1] = *reinterpret_cast<uint4 *>(&h[4]);
}

__device__ __forceinline__ void unpack8(const uint4 &q, float f[8]) {
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float f[8]) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    return *reinterpret_cast<uint4 *>(h);
}
__device__ __forceinline__ uint4 ld8(const bf16 *p) { return __ldg(reinterpret_cast<const uint4 *>(p)); }
__device__ __forceinline__ void st8(bf16 *p, const float f[8]) { *reinterpret_cast<uint4 *>(p) = pack8(f); }

// 2x2x2 average pooling: x (fine dims df, channel stride xs, first channel
// xoff) -> y (coarse, C channels).  One thread per coarse voxel and 8 channels.
__global__ void k_pool2(const bf16 *__restrict__ x, int xs, int xoff, LDims df, int C, bf16 *__restrict__ y) {
    const LDims dc{df.W >> 1, df.H >> 1, df.D >> 1};
    const int g8 = C >> 3;
    const long long n = (long long)dc.W * dc.H * dc.D * g8;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int c = (int)((unsigned)t % (unsigned)g8) * 8;
    const long long v = (unsigned)t / (unsigned)g8;
    int cx, cy, cz;
    split3(v, dc.W, dc.H, cx, cy, cz);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        float f[8];
        unpack8(ld8(x + pvox(df, 2 * cx + (q & 1), 2 * cy + ((q >> 1) & 1), 2 * cz + (q >> 2)) * xs + xoff + c), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[e] += f[e];
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] *= 0.125f;
    st8(y + pvox(dc, cx, cy, cz) * C + c, acc);
}

// Gradient of the skip tensor s (stored in channels [C, 2C) of the concat
// tensor cat at fine dims df): (dcat[C:2C] + pool backward of dpool) masked
// by s > 0.  Output: C channels.
__global__ void k_skip_grad(const bf16 *__restrict__ dcat, const bf16 *__restrict__ cat,
                            const bf16 *__restrict__ dpool, LDims df, int C, bf16 *__restrict__ out) {
    const LDims dc{df.W >> 1, df.H >> 1, df.D >> 1};
    const int g8 = C >> 3;
    const long long n = (long long)df.W * df.H * df.D * g8;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int c = (int)((unsigned)t % (unsigned)g8) * 8;
    const long long v = (unsigned)t / (unsigned)g8;
    int x, y, z;
    split3(v, df.W, df.H, x, y, z);
    const long long f = pvox(df, x, y, z);
    float a[8], s[8], p[8], o[8];
    unpack8(ld8(dcat + f * 2 * C + C + c), a);
    unpack8(ld8(cat + f * 2 * C + C + c), s);
    unpack8(ld8(dpool + pvox(dc, x >> 1, y >> 1, z >> 1) * C + c), p);
#pragma unroll
    for (int e = 0; e < 8; ++e) o[e] = s[e] > 0.0f ? a[e] + 0.125f * p[e] : 0.0f;
    st8(out + f * C + c, o);
}

// Bias gradient: db[c] += sum over the voxels of g[P][goff + c] (C channels,
// channel stride gs), the whole padded tensor (its halo is zero).  Thread t
// sums 8 channels (group t % (C / 8)) over a strided set of voxels; the
// block reduces them in shared memory and adds one FP32 atomic per channel.
template <int C>
__global__ void __launch_bounds__(256) k_bias_grad(const bf16 *__restrict__ g, int gs, int goff, long long nvox,
                                                   float *__restrict__ db) {
    constexpr int NG = C / 8, VPB = 256 / NG;
    __shared__ float red[256][9];
    const int tid = threadIdx.x, grp = tid % NG;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (long long v = (long long)blockIdx.x * VPB + tid / NG; v < nvox; v += (long long)gridDim.x * VPB) {
        float f[8];
        unpack8(ld8(g + v * gs + goff + grp * 8), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[e] += f[e];
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) red[tid][e] = acc[e];
    __syncthreads();
    if (tid < C) {
        float t = 0.0f;
        for (int r = tid / 8; r < 256; r += NG) t += red[r][tid % 8];
        atomicAdd(db + tid, t);
    }
}

// Head: out = b + w . d0b[v] (16 channels).
__device__ __forceinline__ float head_out(const bf16 *d0b, long long P, const float *head, float f[16]) {
    unpack8(ld8(d0b + P * 16), f);
    unpack8(ld8(d0b + P * 16 + 8), f + 8);
    float o = __ldg(head + 16);
#pragma unroll
    for (int c = 0; c < 16; ++c) o = fmaf(__ldg(head + c), f[c], o);
    return o;
}

// Warm start, step 1: the correction d = kappa rms(r) * out over the grid
// (colour packed, FP32).
__global__ void k_unet_delta(const bf16 *__restrict__ d0b, LDims d, const float *__restrict__ head,
                             const float *__restrict__ scales, float *__restrict__ dr, float *__restrict__ db) {
    const long long n = (long long)d.W * d.H * d.D;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i, j, k;
    split3(t, d.W, d.H, i, j, k);
    float f[16];
    (((i + j + k) & 1) ? db : dr)[pidx(i, j, k, d.W >> 1, d.H)] = __ldg(scales + 3) * head_out(d0b, pvox(d, i, j, k), head, f);
}

// Step 3: <r, q>, <q, q>, <d, r> and <d, q> (FP64) with r = b - A p and
// q = A d, one quadruple per block.
__global__ void __launch_bounds__(kNormThreads)
k_unet_project(GridInfo g, CellArr rhs, CellArr p, CellArr dl, double *partials) {
    const long long n = (long long)g.W * g.H * g.D;
    const GridInfo g0{g.W, g.H, g.D, g.open, g.dirichlet, 0.0f};
    double rq = 0.0, qq = 0.0, dr = 0.0, dq = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        split3(t, g.W, g.H, i, j, k);
        float b, pc, r, zb, dc, mq;
        cell_brp(g, rhs, p, i, j, k, b, pc, r);
        cell_brp(g0, rhs, dl, i, j, k, zb, dc, mq);      // with b = 0: mq = -(A d)
        rq -= (double)r * (double)mq;
        qq += (double)mq * (double)mq;
        dr += (double)dc * (double)r;
        dq -= (double)dc * (double)mq;
    }
    __shared__ double s[4][kNormThreads / 32];
    double a[4] = {rq, qq, dr, dq};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < 4; ++q) {
        a[q] = warp_sum_d(a[q]);
        if (lane == 0) s[q][w] = a[q];
    }
    __syncthreads();
    if (w == 0)
        for (int q = 0; q < 4; ++q) {
            double v = lane < kNormThreads / 32 ? s[q][lane] : 0.0;
            v = warp_sum_d(v);
            if (lane == 0) partials[4 * blockIdx.x + q] = v;
        }
}

// The step along d:
//   BLZ_WARM_STEP_RESIDUAL  alpha = <r, A d> / <A d, A d>, minimising the
//                           residual norm ||b - A (p + alpha d)||;
//   BLZ_WARM_STEP_ENERGY    alpha = <d, r> / <d, A d>, minimising the error's
//                           energy norm ||e - alpha d||_A (A symmetric
//                           positive definite: a Dirichlet face or more).
// Either is 0 when its denominator is 0.
__global__ void k_unet_alpha(const double *partials, int nblk, int mode, float *alpha) {
    __shared__ double s[4][32];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        for (int q = 0; q < 4; ++q) a[q] += partials[4 * b + q];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < 4; ++q) {
        a[q] = warp_sum_d(a[q]);
        if (lane == 0) s[q][w] = a[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = 0; i < (int)(blockDim.x + 31) / 32; ++i)
            for (int q = 0; q < 4; ++q) t[q] += s[q][i];
        if (mode == BLZ_WARM_STEP_ENERGY) *alpha = t[3] > 0.0 ? (float)(t[2] / t[3]) : 0.0f;
        else *alpha = t[1] > 0.0 ? (float)(t[0] / t[1]) : 0.0f;
    }
}

// Step 4: p += alpha d (both colour packed, n/2 values each).
__global__ void k_unet_update(long long half, const float *__restrict__ dr, const float *__restrict__ db,
                              const float *__restrict__ alpha, float *__restrict__ pr, float *__restrict__ pb) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= half) return;
    const float a = __ldg(alpha);
    pr[t] = fmaf(a, __ldg(dr + t), pr[t]);
    pb[t] = fmaf(a, __ldg(db + t), pb[t]);
}

// Raw network output over the crop, natural layout.
__global__ void k_unet_out(const bf16 *__restrict__ d0b, LDims d, const float *__restrict__ head,
                           float *__restrict__ out) {
    const long long n = (long long)d.W * d.H * d.D;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i, j, k;
    split3(t, d.W, d.H, i, j, k);
    float f[16];
    out[t] = head_out(d0b, pvox(d, i, j, k), head, f);
}

// Loss L = mean over the crop of (out - target)^2, target = (p* - p_prev)/scales[3].
// Writes dL/d(pre-activation of the last convolution) and accumulates the
// head's gradient (17 values) and {sum diff^2, sum target^2} with atomics.
constexpr int kLossThreads = 256;
__global__ void __launch_bounds__(kLossThreads)
k_unet_loss(const bf16 *__restrict__ d0b, LDims d, int ox, int oy, int oz, GridInfo g, CellArr p, CellArr pt,
            const float *__restrict__ head, const float *__restrict__ scales, float inv_n,
            bf16 *__restrict__ gd0b, float *__restrict__ ghead, double *__restrict__ sums) {
    const long long n = (long long)d.W * d.H * d.D;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float gw[17];
#pragma unroll
    for (int c = 0; c < 17; ++c) gw[c] = 0.0f;
    double l2 = 0.0, t2 = 0.0;
    if (t < n) {
        int x, y, z;
        split3(t, d.W, d.H, x, y, z);
        const long long P = pvox(d, x, y, z);
        float f[16];
        const float o = head_out(d0b, P, head, f);
        const int i = ox + x, j = oy + y, k = oz + z;
        const float so = __ldg(scales + 3);
        const float dp = pt.at(i, j, k, g.W, g.H) - p.at(i, j, k, g.W, g.H);
        const float tgt = so > 0.0f ? dp / so : 0.0f;
        const float diff = o - tgt;
        l2 = (double)diff * diff;
        t2 = (double)tgt * tgt;
        const float go = 2.0f * diff * inv_n;
        float gf[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            gw[c] = go * f[c];
            gf[c] = f[c] > 0.0f ? go * __ldg(head + c) : 0.0f;
        }
        gw[16] = go;
        st8(gd0b + P * 16, gf);
        st8(gd0b + P * 16 + 8, gf + 8);
    }
    __shared__ float sg[17][kLossThreads / 32];
    __shared__ double sl[2][kLossThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 17; ++c) {
        const float s = warp_sum_f(gw[c]);
        if (lane == 0) sg[c][w] = s;
    }
    l2 = warp_sum_d(l2);
    t2 = warp_sum_d(t2);
    if (lane == 0) { sl[0][w] = l2; sl[1][w] = t2; }
    __syncthreads();
    if (threadIdx.x < 17) {
        float s = 0.0f;
        for (int q = 0; q < kLossThreads / 32; ++q) s += sg[threadIdx.x][q];
        atomicAdd(ghead + threadIdx.x, s);
    } else if (threadIdx.x < 19) {
        const int c = threadIdx.x - 17;
        double s = 0.0;
        for (int q = 0; q < kLossThreads / 32; ++q) s += sl[c][q];
        atomicAdd(sums + c, s);
    }
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float bc1,
                       float bc2) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.0f - b1) * gt;
    const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    p[t] -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
}

// BF16 copies of one 3x3x3 layer: wf[t][co][ci] = W[t][co][ci] (forward) and
// wd[t][ci][co] = W[26 - t][co][ci] (data gradient: flipped taps, transposed).
__global__ void k_export_conv(const float *__restrict__ w, int co, int ci, bf16 *__restrict__ wf,
                              bf16 *__restrict__ wd) {
    const long long n = 27LL * co * ci;
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int t = (int)(e / ((long long)co * ci)), o = (int)((e / ci) % co), i = (int)(e % ci);
    const bf16 h = __float2bfloat16_rn(w[e]);
    wf[e] = h;
    wd[((size_t)(26 - t) * ci + i) * co + o] = h;
}

// BF16 copy of a transposed convolution's weights, same [8][cout][cin] order.
__global__ void k_export_up(const float *__restrict__ w, long long n, bf16 *__restrict__ wf) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e < n) wf[e] = __float2bfloat16_rn(w[e]);
}

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// ---------------------------------------------------------------------------
// Network definition
// ---------------------------------------------------------------------------
enum LayerKind { kConv3 = 0, kUp = 1, kHead = 2 };
struct LayerDef { int kind, cin, cout, level; };
enum LayerId { E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, D0A, D0B, U2, U1, U0, HEAD, NLAYERS };
constexpr LayerDef kLayers[NLAYERS] = {
    {kConv3, 16, 16, 0},   {kConv3, 16, 16, 0},  {kConv3, 16, 32, 1}, {kConv3, 32, 32, 1},
    {kConv3, 32, 64, 2},   {kConv3, 64, 64, 2},  {kConv3, 64, 128, 3}, {kConv3, 128, 128, 3},
    {kConv3, 128, 64, 2},  {kConv3, 64, 64, 2},  {kConv3, 64, 32, 1}, {kConv3, 32, 32, 1},
    {kConv3, 32, 16, 0},   {kConv3, 16, 16, 0},
    {kUp, 128, 64, 2},     {kUp, 64, 32, 1},     {kUp, 32, 16, 0},
    {kHead, 16, 1, 0}};
constexpr int taps_of(int kind) { return kind == kConv3 ? 27 : kind == kUp ? 8 : 1; }

struct Ten {
    bf16 *buf = nullptr;
    int C = 0, level = 0;
    bf16 *base() const { return buf + (size_t)kSlack * C; }
};

} // namespace
} // namespace blz

using namespace blz;

struct blz_unet {
    LDims L[4]{};
    int device = 0;
    size_t w_off[NLAYERS]{}, b_off[NLAYERS]{}, bf_off[NLAYERS]{};
    size_t n_params = 0, n_bf = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    bf16 *wf = nullptr, *wd = nullptr;
    bool bf_dirty = true;
    int adam_t = 0;
    float kappa = 1.0f;
    int nb_norms = kNormBlocks, nb_project = kNormBlocks;   // one-wave grids of the reductions
    // forward activations
    Ten X0, e0a, cat0, d0a, d0b, p1, e1a, cat1, d1a, d1b, p2, e2a, cat2, d2a, d2b, p3, e3a, e3b;
    // gradients (allocated by the first training call)
    bool have_grads = false;
    Ten g_d0b, g_d0a, g_cat0, g_e0b, g_e0a, g_p1, g_d1b, g_d1a, g_cat1, g_e1b, g_e1a, g_p2, g_d2b, g_d2a, g_cat2,
        g_e2b, g_e2a, g_p3, g_e3b, g_e3a;
    double *partials = nullptr, *sums = nullptr, *h_sums = nullptr;
    float *scales = nullptr;
    float *dpk = nullptr, *alpha = nullptr;     // warm start: packed correction + zero rhs; its step
    int smooth = 0;                             // sweeps of p and d before the step is chosen
    int step_mode = BLZ_WARM_STEP_ENERGY;       // how the step along d is chosen
    int *err = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    std::vector<bf16 *> allocs;
};

namespace {

int ufail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_thread_error(buf);
    return code;
}

#define UCK(x)                                                                            \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess) return ufail(BLZ_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_)); \
    } while (0)
#define UCKL()                                                                            \
    do {                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess)                                                            \
            return ufail(BLZ_ERR_CUDA, "kernel launch failed (%s:%d): %s", __FILE__, __LINE__, \
                         cudaGetErrorString(e_));                                         \
    } while (0)

int alloc_ten(blz_unet *u, Ten &t, int C, int level) {
    t.C = C;
    t.level = level;
    const size_t bytes = tensor_voxels(u->L[level]) * C * sizeof(bf16);
    UCK(cudaMalloc(&t.buf, bytes));
    u->allocs.push_back(t.buf);
    UCK(cudaMemset(t.buf, 0, bytes));
    return BLZ_OK;
}

void release(blz_unet *u) {
    for (bf16 *p : u->allocs) cudaFree(p);
    cudaFree(u->params); cudaFree(u->grads); cudaFree(u->adam_m); cudaFree(u->adam_v);
    cudaFree(u->wf); cudaFree(u->wd);
    cudaFree(u->partials); cudaFree(u->sums); cudaFree(u->scales); cudaFree(u->err);
    cudaFree(u->dpk); cudaFree(u->alpha);
    if (u->h_sums) cudaFreeHost(u->h_sums);
    if (u->ev0) cudaEventDestroy(u->ev0);
    if (u->ev1) cudaEventDestroy(u->ev1);
}

GridInfo grid_info(const blz_params &P) {
    const SolveParams sp = solve_params_of(P);
    return {P.width, P.height, P.depth, sp.open, sp.dirichlet, sp.scale};
}

int refresh_bf16(blz_unet *u, cudaStream_t st) {
    if (!u->bf_dirty) return BLZ_OK;
    for (int l = 0; l < NLAYERS; ++l) {
        if (kLayers[l].kind == kUp) {
            const long long n = 8LL * kLayers[l].cout * kLayers[l].cin;
            k_export_up<<<nblk(n, 256), 256, 0, st>>>(u->params + u->w_off[l], n, u->wf + u->bf_off[l]);
            ++u->launches;
        }
        if (kLayers[l].kind != kConv3) continue;
        const long long n = 27LL * kLayers[l].cout * kLayers[l].cin;
        k_export_conv<<<nblk(n, 256), 256, 0, st>>>(u->params + u->w_off[l], kLayers[l].cout, kLayers[l].cin,
                                                    u->wf + u->bf_off[l], u->wd + u->bf_off[l]);
        ++u->launches;
    }
    UCKL();
    u->bf_dirty = false;
    return BLZ_OK;
}

int conv_fwd(blz_unet *u, int l, const Ten &x, const Ten &y, int y_off, cudaStream_t st) {
    const LayerDef &L = kLayers[l];
    const LDims &d = u->L[L.level];
    const ConvDesc cd{d.W, d.H, d.D, L.cin, L.cout, 1, 0, y.C, y_off};
    cudaError_t e = launch_conv3d(cd, x.base(), u->wf + u->bf_off[l], u->params + u->b_off[l], y.base(), u->err, st);
    if (e != cudaSuccess) return ufail(BLZ_ERR_CUDA, "conv layer %d: %s", l, cudaGetErrorString(e));
    ++u->launches;
    return BLZ_OK;
}

// Data gradient of layer l: gx = conv(gy, flipped W^T), masked by aux > 0 when aux is given.
int conv_dgrad(blz_unet *u, int l, const Ten &gy, const Ten &gx, const Ten *aux, cudaStream_t st) {
    const LayerDef &L = kLayers[l];
    const LDims &d = u->L[L.level];
    const ConvDesc cd{d.W, d.H, d.D, L.cout, L.cin, 0, 0, gx.C, 0};
    cudaError_t e = launch_conv3d(cd, gy.base(), u->wd + u->bf_off[l], nullptr, gx.base(), u->err, st,
                                  aux ? aux->base() : nullptr);
    if (e != cudaSuccess) return ufail(BLZ_ERR_CUDA, "conv dgrad layer %d: %s", l, cudaGetErrorString(e));
    ++u->launches;
    return BLZ_OK;
}

void launch_bias_grad(const bf16 *g, int gs, int goff, int C, const LDims &d, float *db, cudaStream_t st) {
    const long long nvox = (long long)(d.W + 2) * (d.H + 2) * (d.D + 2);
    const int vpb = 256 / (C / 8);
    const unsigned blocks = (unsigned)std::min<long long>(8 * 148, (nvox + vpb - 1) / vpb);
    switch (C) {
    case 16: k_bias_grad<16><<<blocks, 256, 0, st>>>(g, gs, goff, nvox, db); break;
    case 32: k_bias_grad<32><<<blocks, 256, 0, st>>>(g, gs, goff, nvox, db); break;
    case 64: k_bias_grad<64><<<blocks, 256, 0, st>>>(g, gs, goff, nvox, db); break;
    default: k_bias_grad<128><<<blocks, 256, 0, st>>>(g, gs, goff, nvox, db); break;
    }
}

int conv_wgrad(blz_unet *u, int l, const Ten &gy, const Ten &x, cudaStream_t st) {
    const LayerDef &L = kLayers[l];
    const LDims &d = u->L[L.level];
    const cudaError_t e = launch_wgrad_tc(0, d.W, d.H, d.D, L.cin, L.cout, x.base(), x.C, gy.base(), gy.C, 0,
                                          u->grads + u->w_off[l], u->err, st);
    if (e != cudaSuccess)
        return ufail(BLZ_ERR_CUDA, "conv weight gradient layer %d (%d -> %d): %s", l, L.cin, L.cout,
                     cudaGetErrorString(e));
    launch_bias_grad(gy.base(), gy.C, 0, L.cout, d, u->grads + u->b_off[l], st);
    u->launches += 2;
    UCKL();
    return BLZ_OK;
}

int up_fwd(blz_unet *u, int l, const Ten &x, const Ten &y, cudaStream_t st) {
    const LayerDef &L = kLayers[l];
    const LDims &dc = u->L[L.level + 1];
    const cudaError_t e = launch_upconv_tc(dc.W, dc.H, dc.D, L.cin, L.cout, x.base(), u->wf + u->bf_off[l],
                                           u->params + u->b_off[l], y.base(), y.C, u->err, st);
    if (e != cudaSuccess)
        return ufail(BLZ_ERR_CUDA, "transposed convolution %d (%d -> %d): %s", l, L.cin, L.cout, cudaGetErrorString(e));
    ++u->launches;
    UCKL();
    return BLZ_OK;
}

// Backward of transposed conv l: weight/bias gradients and the coarse input's
// gradient (masked by the coarse activation x > 0).  gy: fine concat gradient
// (channels [0, cout)).
int up_bwd(blz_unet *u, int l, const Ten &gy, const Ten &x, const Ten &gx, cudaStream_t st) {
    const LayerDef &L = kLayers[l];
    const LDims &dc = u->L[L.level + 1];
    if (x.C != L.cin || gx.C != L.cin)
        return ufail(BLZ_ERR_ARG, "transposed convolution %d: coarse tensors need %d channels", l, L.cin);
    const cudaError_t e = launch_wgrad_tc(1, dc.W, dc.H, dc.D, L.cin, L.cout, x.base(), x.C, gy.base(), gy.C, 0,
                                          u->grads + u->w_off[l], u->err, st);
    if (e != cudaSuccess)
        return ufail(BLZ_ERR_CUDA, "transposed convolution %d weight gradient (%d -> %d): %s", l, L.cin, L.cout,
                     cudaGetErrorString(e));
    launch_bias_grad(gy.base(), gy.C, 0, L.cout, u->L[L.level], u->grads + u->b_off[l], st);
    const cudaError_t e2 = launch_upconv_dgrad_tc(dc.W, dc.H, dc.D, L.cin, L.cout, gy.base(), gy.C,
                                                  u->wf + u->bf_off[l], x.base(), gx.base(), u->err, st);
    if (e2 != cudaSuccess)
        return ufail(BLZ_ERR_CUDA, "transposed convolution %d data gradient (%d -> %d): %s", l, L.cin, L.cout,
                     cudaGetErrorString(e2));
    u->launches += 3;
    UCKL();
    return BLZ_OK;
}

int pool(blz_unet *u, const Ten &x, int xoff, int C, const Ten &y, cudaStream_t st) {
    const LDims &df = u->L[y.level - 1];
    const long long n = (long long)(df.W / 2) * (df.H / 2) * (df.D / 2) * (C / 8);
    k_pool2<<<nblk(n, 256), 256, 0, st>>>(x.base(), x.C, xoff, df, C, y.base());
    ++u->launches;
    UCKL();
    return BLZ_OK;
}

int skip_grad(blz_unet *u, const Ten &gcat, const Ten &cat, const Ten &gpool, const Ten &out, cudaStream_t st) {
    const LDims &df = u->L[out.level];
    const long long n = (long long)df.W * df.H * df.D * (out.C / 8);
    k_skip_grad<<<nblk(n, 256), 256, 0, st>>>(gcat.base(), cat.base(), gpool.base(), df, out.C, out.base());
    ++u->launches;
    UCKL();
    return BLZ_OK;
}

int prepare_input(blz_unet *u, const GridInfo &g, const CellArr &rhs, const CellArr &p, const int org[3],
                  cudaStream_t st) {
    k_unet_norms<<<u->nb_norms, kNormThreads, 0, st>>>(g, rhs, p, u->partials);
    k_unet_scales<<<1, 256, 0, st>>>(u->partials, u->nb_norms, (double)g.W * g.H * g.D, u->kappa, u->scales);
    const LDims &d = u->L[0];
    const long long n = (long long)(d.W + 2) * (d.H + 2) * (d.D + 2);
    k_unet_input<<<nblk(n, 256), 256, 0, st>>>(g, rhs, p, org[0], org[1], org[2], d, u->scales, u->X0.base());
    u->launches += 3;
    UCKL();
    return BLZ_OK;
}

int forward_core(blz_unet *u, cudaStream_t st) {
    int rc;
    if ((rc = refresh_bf16(u, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E0A, u->X0, u->e0a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E0B, u->e0a, u->cat0, 16, st)) != BLZ_OK) return rc;
    if ((rc = pool(u, u->cat0, 16, 16, u->p1, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E1A, u->p1, u->e1a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E1B, u->e1a, u->cat1, 32, st)) != BLZ_OK) return rc;
    if ((rc = pool(u, u->cat1, 32, 32, u->p2, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E2A, u->p2, u->e2a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E2B, u->e2a, u->cat2, 64, st)) != BLZ_OK) return rc;
    if ((rc = pool(u, u->cat2, 64, 64, u->p3, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E3A, u->p3, u->e3a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, E3B, u->e3a, u->e3b, 0, st)) != BLZ_OK) return rc;
    if ((rc = up_fwd(u, U2, u->e3b, u->cat2, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, D2A, u->cat2, u->d2a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, D2B, u->d2a, u->d2b, 0, st)) != BLZ_OK) return rc;
    if ((rc = up_fwd(u, U1, u->d2b, u->cat1, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, D1A, u->cat1, u->d1a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, D1B, u->d1a, u->d1b, 0, st)) != BLZ_OK) return rc;
    if ((rc = up_fwd(u, U0, u->d1b, u->cat0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, D0A, u->cat0, u->d0a, 0, st)) != BLZ_OK) return rc;
    if ((rc = conv_fwd(u, D0B, u->d0a, u->d0b, 0, st)) != BLZ_OK) return rc;
    UCKL();
    return BLZ_OK;
}

int alloc_grads(blz_unet *u) {
    if (u->have_grads) return BLZ_OK;
    int rc;
    struct { Ten *t; int C, level; } g[] = {
        {&u->g_d0b, 16, 0}, {&u->g_d0a, 16, 0}, {&u->g_cat0, 32, 0}, {&u->g_e0b, 16, 0}, {&u->g_e0a, 16, 0},
        {&u->g_p1, 16, 1}, {&u->g_d1b, 32, 1}, {&u->g_d1a, 32, 1}, {&u->g_cat1, 64, 1}, {&u->g_e1b, 32, 1},
        {&u->g_e1a, 32, 1}, {&u->g_p2, 32, 2}, {&u->g_d2b, 64, 2}, {&u->g_d2a, 64, 2}, {&u->g_cat2, 128, 2},
        {&u->g_e2b, 64, 2}, {&u->g_e2a, 64, 2}, {&u->g_p3, 64, 3}, {&u->g_e3b, 128, 3}, {&u->g_e3a, 128, 3}};
    for (auto &e : g)
        if ((rc = alloc_ten(u, *e.t, e.C, e.level)) != BLZ_OK) return rc;
    UCK(cudaMalloc(&u->grads, u->n_params * sizeof(float)));
    UCK(cudaMalloc(&u->adam_m, u->n_params * sizeof(float)));
    UCK(cudaMalloc(&u->adam_v, u->n_params * sizeof(float)));
    UCK(cudaMemset(u->grads, 0, u->n_params * sizeof(float)));
    UCK(cudaMemset(u->adam_m, 0, u->n_params * sizeof(float)));
    UCK(cudaMemset(u->adam_v, 0, u->n_params * sizeof(float)));
    u->have_grads = true;
    return BLZ_OK;
}

// Backward pass from the head's gradient (in g_d0b) to every parameter.
int backward_core(blz_unet *u, cudaStream_t st) {
    int rc;
#define STEP(x) if ((rc = (x)) != BLZ_OK) return rc
    // level 0 decoder
    STEP(conv_wgrad(u, D0B, u->g_d0b, u->d0a, st));
    STEP(conv_dgrad(u, D0B, u->g_d0b, u->g_d0a, &u->d0a, st));
    STEP(conv_wgrad(u, D0A, u->g_d0a, u->cat0, st));
    STEP(conv_dgrad(u, D0A, u->g_d0a, u->g_cat0, nullptr, st));
    STEP(up_bwd(u, U0, u->g_cat0, u->d1b, u->g_d1b, st));
    // level 1 decoder
    STEP(conv_wgrad(u, D1B, u->g_d1b, u->d1a, st));
    STEP(conv_dgrad(u, D1B, u->g_d1b, u->g_d1a, &u->d1a, st));
    STEP(conv_wgrad(u, D1A, u->g_d1a, u->cat1, st));
    STEP(conv_dgrad(u, D1A, u->g_d1a, u->g_cat1, nullptr, st));
    STEP(up_bwd(u, U1, u->g_cat1, u->d2b, u->g_d2b, st));
    // level 2 decoder
    STEP(conv_wgrad(u, D2B, u->g_d2b, u->d2a, st));
    STEP(conv_dgrad(u, D2B, u->g_d2b, u->g_d2a, &u->d2a, st));
    STEP(conv_wgrad(u, D2A, u->g_d2a, u->cat2, st));
    STEP(conv_dgrad(u, D2A, u->g_d2a, u->g_cat2, nullptr, st));
    STEP(up_bwd(u, U2, u->g_cat2, u->e3b, u->g_e3b, st));
    // bottleneck
    STEP(conv_wgrad(u, E3B, u->g_e3b, u->e3a, st));
    STEP(conv_dgrad(u, E3B, u->g_e3b, u->g_e3a, &u->e3a, st));
    STEP(conv_wgrad(u, E3A, u->g_e3a, u->p3, st));
    STEP(conv_dgrad(u, E3A, u->g_e3a, u->g_p3, nullptr, st));
    // level 2 encoder
    STEP(skip_grad(u, u->g_cat2, u->cat2, u->g_p3, u->g_e2b, st));
    STEP(conv_wgrad(u, E2B, u->g_e2b, u->e2a, st));
    STEP(conv_dgrad(u, E2B, u->g_e2b, u->g_e2a, &u->e2a, st));
    STEP(conv_wgrad(u, E2A, u->g_e2a, u->p2, st));
    STEP(conv_dgrad(u, E2A, u->g_e2a, u->g_p2, nullptr, st));
    // level 1 encoder
    STEP(skip_grad(u, u->g_cat1, u->cat1, u->g_p2, u->g_e1b, st));
    STEP(conv_wgrad(u, E1B, u->g_e1b, u->e1a, st));
    STEP(conv_dgrad(u, E1B, u->g_e1b, u->g_e1a, &u->e1a, st));
    STEP(conv_wgrad(u, E1A, u->g_e1a, u->p1, st));
    STEP(conv_dgrad(u, E1A, u->g_e1a, u->g_p1, nullptr, st));
    // level 0 encoder
    STEP(skip_grad(u, u->g_cat0, u->cat0, u->g_p1, u->g_e0b, st));
    STEP(conv_wgrad(u, E0B, u->g_e0b, u->e0a, st));
    STEP(conv_dgrad(u, E0B, u->g_e0b, u->g_e0a, &u->e0a, st));
    STEP(conv_wgrad(u, E0A, u->g_e0a, u->X0, st));
#undef STEP
    return BLZ_OK;
}

int check_grid(const blz_unet *u, const blz_params *P, const int org[3]) {
    if (!P) return ufail(BLZ_ERR_ARG, "null grid parameters");
    if (P->width < 1 || P->height < 1 || P->depth < 1) return ufail(BLZ_ERR_ARG, "bad grid dims");
    const int o[3] = {org ? org[0] : 0, org ? org[1] : 0, org ? org[2] : 0};
    const int dims[3] = {P->width, P->height, P->depth}, cd[3] = {u->L[0].W, u->L[0].H, u->L[0].D};
    for (int a = 0; a < 3; ++a)
        if (o[a] < 0 || o[a] + cd[a] > dims[a])
            return ufail(BLZ_ERR_ARG, "crop [%d, %d) on axis %d exceeds the grid (%d)", o[a], o[a] + cd[a], a, dims[a]);
    return BLZ_OK;
}

int sync_conv_flag(blz_unet *u, cudaStream_t st) {
    int flag = 0;
    UCK(cudaMemcpyAsync(&flag, u->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    UCK(cudaStreamSynchronize(st));
    if (flag) return ufail(BLZ_ERR_TIMEOUT, "tensor-core completion wait timed out");
    return BLZ_OK;
}

} // namespace

namespace blz {
// Learned warm start, in the order blz_solve runs it:
// unet_correction computes d (colour packed) from rhs and the current p; the
// solver then smooths p and d alike (unet_smoothing(u) sweeps each, d with a
// zero right-hand side: Gauss-Seidel is affine, so this is exactly smoothing
// p + alpha d for every alpha at once); unet_combine picks alpha minimising the
// residual norm of p + alpha d and adds alpha d.
// Allocates the correction buffers once (at attachment, so that a warm start
// captured into a graph allocates nothing).
int unet_prepare(blz_unet *u, const blz_params &P) {
    (void)P;
    if (u->dpk) return BLZ_OK;
    const LDims &d = u->L[0];
    const long long n = (long long)d.W * d.H * d.D;
    UCK(cudaMalloc(&u->dpk, sizeof(float) * 2 * n));         // d (n) then a zero right-hand side (n)
    UCK(cudaMemset(u->dpk, 0, sizeof(float) * 2 * n));
    return BLZ_OK;
}

int unet_correction(blz_unet *u, const blz_params &P, const float *rhs_r, const float *rhs_b, const float *p_r,
                    const float *p_b, cudaStream_t st, long long *launches, float **d_r, float **d_b,
                    const float **z_r, const float **z_b) {
    if (u->L[0].W != P.width || u->L[0].H != P.height || u->L[0].D != P.depth)
        return ufail(BLZ_ERR_ARG, "warm-start network built for %dx%dx%d, grid is %dx%dx%d", u->L[0].W, u->L[0].H,
                     u->L[0].D, P.width, P.height, P.depth);
    const long long l0 = u->launches;
    const GridInfo g = grid_info(P);
    const int org[3] = {0, 0, 0};
    int rc;
    UCK(cudaMemsetAsync(u->err, 0, sizeof(int), st));
    if ((rc = prepare_input(u, g, CellArr{rhs_r, rhs_b}, CellArr{p_r, p_b}, org, st)) != BLZ_OK) return rc;
    if ((rc = forward_core(u, st)) != BLZ_OK) return rc;
    const LDims &d = u->L[0];
    const long long n = (long long)d.W * d.H * d.D;
    if ((rc = unet_prepare(u, P)) != BLZ_OK) return rc;
    float *dr = u->dpk, *db = u->dpk + n / 2;
    k_unet_delta<<<nblk(n, 256), 256, 0, st>>>(u->d0b.base(), d, u->params + u->w_off[HEAD], u->scales, dr, db);
    ++u->launches;
    UCKL();
    *d_r = dr;
    *d_b = db;
    *z_r = u->dpk + n;
    *z_b = u->dpk + n + n / 2;
    if (launches) *launches += u->launches - l0;
    return BLZ_OK;
}

int unet_combine(blz_unet *u, const blz_params &P, const float *rhs_r, const float *rhs_b, float *p_r, float *p_b,
                 cudaStream_t st, long long *launches) {
    const GridInfo g = grid_info(P);
    const LDims &d = u->L[0];
    const long long n = (long long)d.W * d.H * d.D;
    const float *dr = u->dpk, *db = u->dpk + n / 2;
    k_unet_project<<<u->nb_project, kNormThreads, 0, st>>>(g, CellArr{rhs_r, rhs_b}, CellArr{p_r, p_b},
                                                         CellArr{dr, db}, u->partials);
    k_unet_alpha<<<1, 256, 0, st>>>(u->partials, u->nb_project, u->step_mode, u->alpha);
    k_unet_update<<<nblk(n / 2, 256), 256, 0, st>>>(n / 2, dr, db, u->alpha, p_r, p_b);
    u->launches += 3;
    if (launches) *launches += 3;
    UCKL();
    return BLZ_OK;
}

int unet_smoothing(const blz_unet *u) { return u->smooth; }
int unet_timeout_flag(blz_unet *u, cudaStream_t st) { return sync_conv_flag(u, st); }
} // namespace blz

extern "C" {

int blz_unet_layer_info(int layer, long long info[6]) {
    if (layer < 0 || layer >= NLAYERS || !info) return ufail(BLZ_ERR_ARG, "no layer %d", layer);
    size_t off = 0;
    for (int l = 0; l <= layer; ++l) {
        const LayerDef &L = kLayers[l];
        const size_t wn = (size_t)taps_of(L.kind) * L.cout * L.cin;
        if (l == layer) {
            info[0] = L.kind; info[1] = L.cin; info[2] = L.cout; info[3] = taps_of(L.kind);
            info[4] = (long long)off; info[5] = (long long)(off + wn);
        }
        off += wn + L.cout;
    }
    return BLZ_OK;
}

int blz_unet_create(int width, int height, int depth, blz_unet **out) {
    if (!out) return ufail(BLZ_ERR_ARG, "null output");
    *out = nullptr;
    if (width < 8 || height < 8 || depth < 8 || width % 8 || height % 8 || depth % 8)
        return ufail(BLZ_ERR_ARG, "network dims must be positive multiples of 8 (got %d x %d x %d)", width, height,
                     depth);
    if ((long long)width * height * depth > (1LL << 28))
        return ufail(BLZ_ERR_ARG, "network grid above 2^28 cells (%d x %d x %d)", width, height, depth);
    blz_unet *u = new blz_unet();
    for (int l = 0; l < 4; ++l) u->L[l] = {width >> l, height >> l, depth >> l};
    cudaGetDevice(&u->device);
    u->nb_norms = one_wave(k_unet_norms);
    u->nb_project = one_wave(k_unet_project);
    size_t off = 0, bf = 0;
    for (int l = 0; l < NLAYERS; ++l) {
        const LayerDef &L = kLayers[l];
        const size_t wn = (size_t)taps_of(L.kind) * L.cout * L.cin;
        u->w_off[l] = off;
        u->b_off[l] = off + wn;
        off += wn + L.cout;
        if (L.kind == kConv3 || L.kind == kUp) { u->bf_off[l] = bf; bf += wn; }
    }
    u->n_params = off;
    u->n_bf = bf;
    int rc = BLZ_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == BLZ_OK) rc = ufail(BLZ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    };
    ck(cudaMalloc(&u->params, off * sizeof(float)), "cudaMalloc params");
    if (rc == BLZ_OK) ck(cudaMemset(u->params, 0, off * sizeof(float)), "cudaMemset params");
    ck(cudaMalloc(&u->wf, bf * sizeof(bf16)), "cudaMalloc wf");
    ck(cudaMalloc(&u->wd, bf * sizeof(bf16)), "cudaMalloc wd");
    ck(cudaMalloc(&u->partials, 4 * kNormBlocks * sizeof(double)), "cudaMalloc partials");
    ck(cudaMalloc(&u->sums, 2 * sizeof(double)), "cudaMalloc sums");
    ck(cudaMallocHost(&u->h_sums, 2 * sizeof(double)), "cudaMallocHost");
    ck(cudaMalloc(&u->scales, 4 * sizeof(float)), "cudaMalloc scales");
    ck(cudaMalloc(&u->alpha, sizeof(float)), "cudaMalloc alpha");
    if (rc == BLZ_OK) ck(cudaMemset(u->alpha, 0, sizeof(float)), "cudaMemset alpha");
    ck(cudaMalloc(&u->err, sizeof(int)), "cudaMalloc err");
    if (rc == BLZ_OK) ck(cudaMemset(u->err, 0, sizeof(int)), "cudaMemset err");
    if (rc == BLZ_OK) ck(cudaMemset(u->scales, 0, 4 * sizeof(float)), "cudaMemset scales");
    ck(cudaEventCreate(&u->ev0), "cudaEventCreate");
    ck(cudaEventCreate(&u->ev1), "cudaEventCreate");
    struct { Ten *t; int C, level; } act[] = {
        {&u->X0, 16, 0}, {&u->e0a, 16, 0}, {&u->cat0, 32, 0}, {&u->d0a, 16, 0}, {&u->d0b, 16, 0},
        {&u->p1, 16, 1}, {&u->e1a, 32, 1}, {&u->cat1, 64, 1}, {&u->d1a, 32, 1}, {&u->d1b, 32, 1},
        {&u->p2, 32, 2}, {&u->e2a, 64, 2}, {&u->cat2, 128, 2}, {&u->d2a, 64, 2}, {&u->d2b, 64, 2},
        {&u->p3, 64, 3}, {&u->e3a, 128, 3}, {&u->e3b, 128, 3}};
    for (auto &e : act)
        if (rc == BLZ_OK) rc = alloc_ten(u, *e.t, e.C, e.level);
    if (rc != BLZ_OK) {
        release(u);
        delete u;
        return rc;
    }
    *out = u;
    return BLZ_OK;
}

int blz_unet_destroy(blz_unet *u) {
    if (!u) return BLZ_OK;
    cudaDeviceSynchronize();
    release(u);
    delete u;
    return BLZ_OK;
}

long long blz_unet_num_params(const blz_unet *u) { return u ? (long long)u->n_params : 0; }

long long blz_unet_kernel_launches(const blz_unet *u) { return u ? u->launches : 0; }

int blz_unet_set_smoothing(blz_unet *u, int sweeps) {
    if (!u || sweeps < 0) return ufail(BLZ_ERR_ARG, "bad smoothing sweep count");
    u->smooth = sweeps;
    return BLZ_OK;
}

int blz_unet_set_step(blz_unet *u, int mode) {
    if (!u || (mode != BLZ_WARM_STEP_RESIDUAL && mode != BLZ_WARM_STEP_ENERGY))
        return ufail(BLZ_ERR_ARG, "bad warm-start step mode");
    u->step_mode = mode;
    return BLZ_OK;
}

float blz_unet_last_alpha(const blz_unet *u) {
    float a = 0.0f;
    if (u && u->alpha) cudaMemcpy(&a, u->alpha, sizeof(float), cudaMemcpyDeviceToHost);
    return a;
}

int blz_unet_set_params(blz_unet *u, const float *params, int on_device) {
    if (!u || !params) return ufail(BLZ_ERR_ARG, "null argument");
    UCK(cudaMemcpy(u->params, params, u->n_params * sizeof(float),
                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    u->bf_dirty = true;
    u->adam_t = 0;
    if (u->have_grads) {
        UCK(cudaMemset(u->adam_m, 0, u->n_params * sizeof(float)));
        UCK(cudaMemset(u->adam_v, 0, u->n_params * sizeof(float)));
    }
    return BLZ_OK;
}

int blz_unet_get_params(const blz_unet *u, float *params, int on_device) {
    if (!u || !params) return ufail(BLZ_ERR_ARG, "null argument");
    UCK(cudaMemcpy(params, u->params, u->n_params * sizeof(float),
                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
    return BLZ_OK;
}

int blz_unet_get_grads(const blz_unet *u, float *grads, int on_device) {
    if (!u || !grads) return ufail(BLZ_ERR_ARG, "null argument");
    if (!u->have_grads) return ufail(BLZ_ERR_STATE, "no gradients: call blz_unet_loss_grad first");
    UCK(cudaMemcpy(grads, u->grads, u->n_params * sizeof(float),
                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
    return BLZ_OK;
}

int blz_unet_set_kappa(blz_unet *u, float kappa) {
    if (!u || !(kappa >= 0.0f)) return ufail(BLZ_ERR_ARG, "bad kappa");
    u->kappa = kappa;
    return BLZ_OK;
}

int blz_unet_forward(blz_unet *u, const blz_params *grid, const int origin[3], const float *rhs, const float *p,
                     float *out, void *stream) {
    if (!u || !rhs || !p || !out) return ufail(BLZ_ERR_ARG, "null argument");
    int rc = check_grid(u, grid, origin);
    if (rc != BLZ_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int org[3] = {origin ? origin[0] : 0, origin ? origin[1] : 0, origin ? origin[2] : 0};
    UCK(cudaMemsetAsync(u->err, 0, sizeof(int), st));
    if ((rc = prepare_input(u, grid_info(*grid), CellArr{rhs, nullptr}, CellArr{p, nullptr}, org, st)) != BLZ_OK)
        return rc;
    if ((rc = forward_core(u, st)) != BLZ_OK) return rc;
    const LDims &d = u->L[0];
    k_unet_out<<<nblk((long long)d.W * d.H * d.D, 256), 256, 0, st>>>(u->d0b.base(), d, u->params + u->w_off[HEAD],
                                                                      out);
    ++u->launches;
    UCKL();
    return sync_conv_flag(u, st);
}

int blz_unet_loss_grad(blz_unet *u, const blz_params *grid, const int origin[3], const float *rhs, const float *p,
                       const float *p_target, double *loss, void *stream) {
    if (!u || !rhs || !p || !p_target) return ufail(BLZ_ERR_ARG, "null argument");
    int rc = check_grid(u, grid, origin);
    if (rc != BLZ_OK) return rc;
    if ((rc = alloc_grads(u)) != BLZ_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int org[3] = {origin ? origin[0] : 0, origin ? origin[1] : 0, origin ? origin[2] : 0};
    const GridInfo g = grid_info(*grid);
    UCK(cudaMemsetAsync(u->err, 0, sizeof(int), st));
    UCK(cudaMemsetAsync(u->grads, 0, u->n_params * sizeof(float), st));
    UCK(cudaMemsetAsync(u->sums, 0, 2 * sizeof(double), st));
    if ((rc = prepare_input(u, g, CellArr{rhs, nullptr}, CellArr{p, nullptr}, org, st)) != BLZ_OK) return rc;
    if ((rc = forward_core(u, st)) != BLZ_OK) return rc;
    const LDims &d = u->L[0];
    const long long n = (long long)d.W * d.H * d.D;
    k_unet_loss<<<nblk(n, kLossThreads), kLossThreads, 0, st>>>(
        u->d0b.base(), d, org[0], org[1], org[2], g, CellArr{p, nullptr}, CellArr{p_target, nullptr},
        u->params + u->w_off[HEAD], u->scales, (float)(1.0 / (double)n), u->g_d0b.base(), u->grads + u->w_off[HEAD],
        u->sums);
    ++u->launches;
    UCKL();
    if ((rc = backward_core(u, st)) != BLZ_OK) return rc;
    UCK(cudaMemcpyAsync(u->h_sums, u->sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if ((rc = sync_conv_flag(u, st)) != BLZ_OK) return rc;
    if (loss) {
        loss[0] = u->h_sums[0] / (double)n;
        loss[1] = u->h_sums[1] / (double)n;
    }
    return BLZ_OK;
}

static const Ten *tensor_by_id(const blz_unet *u, int id) {
    const Ten *t[] = {&u->X0,    &u->e0a,   &u->cat0,  &u->d0a,   &u->d0b,   &u->p1,    &u->e1a,   &u->cat1,
                      &u->d1a,   &u->d1b,   &u->p2,    &u->e2a,   &u->cat2,  &u->d2a,   &u->d2b,   &u->p3,
                      &u->e3a,   &u->e3b,   &u->g_d0b, &u->g_d0a, &u->g_cat0, &u->g_e0b, &u->g_e0a, &u->g_p1,
                      &u->g_d1b, &u->g_d1a, &u->g_cat1, &u->g_e1b, &u->g_e1a, &u->g_p2, &u->g_d2b, &u->g_d2a,
                      &u->g_cat2, &u->g_e2b, &u->g_e2a, &u->g_p3, &u->g_e3b, &u->g_e3a};
    if (id < 0 || id >= (int)(sizeof t / sizeof t[0])) return nullptr;
    return t[id];
}

// Padded shape (D+2, H+2, W+2, C) of tensor `id`: the 18 activations in
// forward order (X0 e0a cat0 d0a d0b p1 e1a cat1 d1a d1b p2 e2a cat2 d2a d2b
// p3 e3a e3b), then the 20 activation gradients (g_d0b g_d0a g_cat0 g_e0b
// g_e0a g_p1 g_d1b g_d1a g_cat1 g_e1b g_e1a g_p2 g_d2b g_d2a g_cat2 g_e2b
// g_e2a g_p3 g_e3b g_e3a), which exist after the first training call.
int blz_unet_tensor_shape(const blz_unet *u, int id, int shape[4]) {
    const Ten *t = u ? tensor_by_id(u, id) : nullptr;
    if (!t || !shape) return ufail(BLZ_ERR_ARG, "no tensor %d", id);
    if (!t->buf) return ufail(BLZ_ERR_STATE, "tensor %d not allocated (gradients need a training call)", id);
    const LDims &d = u->L[t->level];
    shape[0] = d.D + 2; shape[1] = d.H + 2; shape[2] = d.W + 2; shape[3] = t->C;
    return BLZ_OK;
}

int blz_unet_get_tensor(const blz_unet *u, int id, float *out, long long capacity) {
    const Ten *t = u ? tensor_by_id(u, id) : nullptr;
    if (!t || !out) return ufail(BLZ_ERR_ARG, "no tensor %d", id);
    if (!t->buf) return ufail(BLZ_ERR_STATE, "tensor %d not allocated (gradients need a training call)", id);
    const LDims &d = u->L[t->level];
    const size_t n = (size_t)(d.W + 2) * (d.H + 2) * (d.D + 2) * t->C;
    if ((long long)n > capacity) return ufail(BLZ_ERR_ARG, "capacity %lld < %zu", capacity, n);
    std::vector<uint16_t> h(n);
    UCK(cudaDeviceSynchronize());
    UCK(cudaMemcpy(h.data(), t->base(), n * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) {
        const uint32_t bits = (uint32_t)h[i] << 16;
        std::memcpy(out + i, &bits, sizeof bits);
    }
    return BLZ_OK;
}

int blz_unet_adam(blz_unet *u, float lr, float beta1, float beta2, float eps, void *stream) {
    if (!u) return ufail(BLZ_ERR_ARG, "null network");
    if (!u->have_grads) return ufail(BLZ_ERR_STATE, "no gradients: call blz_unet_loss_grad first");
    cudaStream_t st = (cudaStream_t)stream;
    ++u->adam_t;
    const float bc1 = 1.0f - powf(beta1, (float)u->adam_t), bc2 = 1.0f - powf(beta2, (float)u->adam_t);
    k_adam<<<nblk((long long)u->n_params, 256), 256, 0, st>>>(u->params, u->grads, u->adam_m, u->adam_v,
                                                              (long long)u->n_params, lr, beta1, beta2, eps, bc1, bc2);
    ++u->launches;
    UCKL();
    u->bf_dirty = true;
    return BLZ_OK;
}

} // extern "C"
