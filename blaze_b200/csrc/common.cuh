// common.cuh — device-side geometry, samplers and noise shared by the kernels.
//
// Fields are plain FP32 arrays in the reference layout (x fastest,
// index = i + j*w + k*w*h, src/Grid.h:256-268).  Kernels receive raw
// pointers and the geometry by value: no device objects, no pointer chasing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/blaze_b200.h"

namespace blz {

// Kernel-side copy of the scene geometry and the physical parameters.
struct Geom {
    int W, H, D;             // T dims
    float dx, dt, inv_dx;
    float dmin[3], dsize[3]; // world-space domain min and size (y flipped)
};

// One staggered field: pointer, dims and sample offsets (FluidSolver.cu:36-43).
struct FieldRef {
    const float *__restrict__ a;
    int w, h, d;
    float ox, oy, oz;
};

__device__ __forceinline__ size_t lin(int i, int j, int k, int w, int h) {
    return (size_t)i + (size_t)w * ((size_t)j + (size_t)h * (size_t)k);
}

__device__ __forceinline__ FieldRef fT(const float *a, const Geom &g) { return {a, g.W, g.H, g.D, 0.5f, 0.5f, 0.5f}; }
__device__ __forceinline__ FieldRef fU(const float *a, const Geom &g) { return {a, g.W + 1, g.H, g.D, 0.0f, 0.5f, 0.5f}; }
__device__ __forceinline__ FieldRef fV(const float *a, const Geom &g) { return {a, g.W, g.H + 1, g.D, 0.5f, 0.0f, 0.5f}; }
__device__ __forceinline__ FieldRef fW(const float *a, const Geom &g) { return {a, g.W, g.H, g.D + 1, 0.5f, 0.5f, 0.0f}; }

// Sample coordinate clamp [0, n - 1.001] (src/Grid.h:96-98).
__device__ __forceinline__ float clamp_coord(float g, int n) {
    return fmaxf(fminf(g, (float)n - 1.001f), 0.0f);
}

__device__ __forceinline__ float ldg(const float *p) { return __ldg(p); }

// Clamped trilinear sample at an object-space position (src/Grid.h:94-108).
// Offsets within a field are 32-bit: the solver refuses grids whose
// (W + 1)(H + 1)(D + 1) reaches 2^31.
__device__ __forceinline__ float trilinear(const FieldRef &f, float inv_dx, float px, float py, float pz) {
    const float gX = clamp_coord(px * inv_dx - f.ox, f.w);
    const float gY = clamp_coord(py * inv_dx - f.oy, f.h);
    const float gZ = clamp_coord(pz * inv_dx - f.oz, f.d);
    const int x0 = (int)gX, y0 = (int)gY, z0 = (int)gZ;
    const float fx = gX - (float)x0, fy = gY - (float)y0, fz = gZ - (float)z0;
    const int sy = f.w, sz = f.w * f.h;
    const float *p = f.a + (x0 + sy * y0 + sz * z0);
    const float a000 = ldg(p), a100 = ldg(p + 1);
    const float a010 = ldg(p + sy), a110 = ldg(p + sy + 1);
    const float a001 = ldg(p + sz), a101 = ldg(p + sz + 1);
    const float a011 = ldg(p + sy + sz), a111 = ldg(p + sy + sz + 1);
    return (1.0f - fz) * ((1.0f - fy) * (a000 * (1.0f - fx) + a100 * fx) + fy * (a010 * (1.0f - fx) + a110 * fx))
         + fz * ((1.0f - fy) * (a001 * (1.0f - fx) + a101 * fx) + fy * (a011 * (1.0f - fx) + a111 * fx));
}

// Lagrange cubic on nodes -1, 0, 1, 2 (src/Grid.h:148-163).
__device__ __forceinline__ float cerp(float q0, float q1, float q2, float q3, float s) {
    const float s2 = s * s, s3 = s2 * s;
    return (-1.0f / 3.0f * s + 0.5f * s2 - 1.0f / 6.0f * s3) * q0
         + (1.0f - s2 + 0.5f * (s3 - s)) * q1
         + (s + 0.5f * (s2 - s3)) * q2
         + (1.0f / 6.0f * (s3 - s)) * q3;
}

// Separable tricubic (x, then y, then z) with edge-clamped stencil indices;
// CLAMP zeroes negatives after every 1-D stage (src/Grid.h:165-222).
template <bool CLAMP>
__device__ __forceinline__ float tricubic(const FieldRef &f, float inv_dx, float px, float py, float pz) {
    const float gX = clamp_coord(px * inv_dx - f.ox, f.w);
    const float gY = clamp_coord(py * inv_dx - f.oy, f.h);
    const float gZ = clamp_coord(pz * inv_dx - f.oz, f.d);
    const int i1 = (int)gX, j1 = (int)gY, k1 = (int)gZ;
    const int i0 = max(i1 - 1, 0), i2 = i1 + 1, i3 = min(i1 + 2, f.w - 1);
    const float sx = gX - (float)i1, sy = gY - (float)j1, sz = gZ - (float)k1;
    const int rs = f.w, ps = f.w * f.h;             // 32-bit offsets, as in trilinear
    float zs[4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const int kz = kk == 0 ? max(k1 - 1, 0) : kk == 3 ? min(k1 + 2, f.d - 1) : k1 + kk - 1;
        float ys[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int jy = jj == 0 ? max(j1 - 1, 0) : jj == 3 ? min(j1 + 2, f.h - 1) : j1 + jj - 1;
            const float *row = f.a + (rs * jy + ps * kz);
            float v = cerp(ldg(row + i0), ldg(row + i1), ldg(row + i2), ldg(row + i3), sx);
            ys[jj] = CLAMP ? fmaxf(v, 0.0f) : v;
        }
        const float v = cerp(ys[0], ys[1], ys[2], ys[3], sy);
        zs[kk] = CLAMP ? fmaxf(v, 0.0f) : v;
    }
    const float v = cerp(zs[0], zs[1], zs[2], zs[3], sz);
    return CLAMP ? fmaxf(v, 0.0f) : v;
}

__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

// ---------------------------------------------------------------------------
// Gradient noise: cudaNoise's perlinNoise (reference thirdparty/cuda-noise/
// cuda_noise.cuh:570-615) evaluated with explicitly rounded operations, so the
// result is independent of this build's FMA contraction and equals the
// oracle's FP32 value bit for bit.  Where the library's source has a multiply
// feeding an add in one expression, the reference build fuses the two (the
// left product when both operands are products), and so does this code; the
// result then equals the reference build's bit for bit.  The lattice hash
// (46-57) takes a float sum of the corner coordinates (120-124) truncated to
// unsigned (cvt.rzi.u32 saturates).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lattice_hash(uint32_t s) {
    s = (s + 0x7ed55d16u) + (s << 12);
    s = (s ^ 0xc761c23cu) ^ (s >> 19);
    s = (s + 0x165667b1u) + (s << 5);
    s = (s + 0xd3a2646cu) ^ (s << 9);
    s = (s + 0xfd7046c5u) + (s << 3);
    s = (s ^ 0xb55a4f09u) ^ (s >> 16);
    return s;
}

// The reference build forms the lattice sum as fma(z, 149812, fma(x, 1723,
// y*93241)) + 3824 + seed; past 2^24 the fused roundings pick different
// lattice gradients, so the same sequence is written out explicitly here.
__device__ __forceinline__ uint32_t lattice_seed(float x, float y, float z, float seed) {
    float acc = __fmaf_rn(x, 1723.0f, __fmul_rn(y, 93241.0f));
    acc = __fmaf_rn(z, 149812.0f, acc);
    acc = __fadd_rn(acc, 3824.0f);
    acc = __fadd_rn(acc, seed);
    return lattice_hash(__float2uint_rz(acc));
}

__device__ __forceinline__ float lattice_grad(int h, float x, float y, float z) {
    switch (h & 0xF) {
    case 0x0: return __fadd_rn(x, y);   case 0x1: return __fadd_rn(-x, y);
    case 0x2: return __fsub_rn(x, y);   case 0x3: return __fsub_rn(-x, y);
    case 0x4: return __fadd_rn(x, z);   case 0x5: return __fadd_rn(-x, z);
    case 0x6: return __fsub_rn(x, z);   case 0x7: return __fsub_rn(-x, z);
    case 0x8: return __fadd_rn(y, z);   case 0x9: return __fadd_rn(-y, z);
    case 0xA: return __fsub_rn(y, z);   case 0xB: return __fsub_rn(-y, z);
    case 0xC: return __fadd_rn(y, x);   case 0xD: return __fadd_rn(-y, z);
    case 0xE: return __fsub_rn(y, x);   default:  return __fsub_rn(-y, z);
    }
}

// fade (204-207): t^3 (t (6t - 15) + 10), the inner polynomial fused.
__device__ __forceinline__ float fade5(float t) {
    const float a = __fmul_rn(__fmul_rn(t, t), t);
    const float b = __fmaf_rn(t, __fmaf_rn(t, 6.0f, -15.0f), 10.0f);
    return __fmul_rn(a, b);
}

// lerp (167-170): a (1 - r) + b r with the left product fused.
__device__ __forceinline__ float lerp_rn(float a, float b, float r) {
    return __fmaf_rn(a, __fsub_rn(1.0f, r), __fmul_rn(b, r));
}

__device__ __forceinline__ float perlin(float px, float py, float pz, float scale, int seed) {
    const float fs = (float)seed;
    px = __fmul_rn(px, scale); py = __fmul_rn(py, scale); pz = __fmul_rn(pz, scale);
    const float ix = floorf(px), iy = floorf(py), iz = floorf(pz);
    px = __fsub_rn(px, ix); py = __fsub_rn(py, iy); pz = __fsub_rn(pz, iz);
    const float u = fade5(px), v = fade5(py), w = fade5(pz);
    const float ix1 = __fadd_rn(ix, 1.0f), iy1 = __fadd_rn(iy, 1.0f), iz1 = __fadd_rn(iz, 1.0f);
    const float px1 = __fsub_rn(px, 1.0f), py1 = __fsub_rn(py, 1.0f), pz1 = __fsub_rn(pz, 1.0f);
    const float i000 = lattice_grad((int)lattice_seed(ix, iy, iz, fs), px, py, pz);
    const float i100 = lattice_grad((int)lattice_seed(ix1, iy, iz, fs), px1, py, pz);
    const float i010 = lattice_grad((int)lattice_seed(ix, iy1, iz, fs), px, py1, pz);
    const float i110 = lattice_grad((int)lattice_seed(ix1, iy1, iz, fs), px1, py1, pz);
    const float i001 = lattice_grad((int)lattice_seed(ix, iy, iz1, fs), px, py, pz1);
    const float i101 = lattice_grad((int)lattice_seed(ix1, iy, iz1, fs), px1, py, pz1);
    const float i011 = lattice_grad((int)lattice_seed(ix, iy1, iz1, fs), px, py1, pz1);
    const float i111 = lattice_grad((int)lattice_seed(ix1, iy1, iz1, fs), px1, py1, pz1);
    const float x00 = lerp_rn(i000, i100, u), x10 = lerp_rn(i010, i110, u);
    const float x01 = lerp_rn(i001, i101, u), x11 = lerp_rn(i011, i111, u);
    const float y0 = lerp_rn(x00, x10, v), y1 = lerp_rn(x01, x11, v);
    return lerp_rn(y0, y1, w);
}

// Colour-packed pressure/rhs addressing.  Cell (i,j,k) has colour
// c = (i+j+k)&1 (0 = red) and packed index (i>>1) + (W/2)*(j + H*k) in the
// array of its colour; each colour's rows are contiguous, so a half sweep
// streams its own colour and the other colour's rows.
struct Packed {
    float *red, *black;
    int Wh;                  // W / 2 (W even)
};

__device__ __forceinline__ size_t pidx(int i, int j, int k, int Wh, int H) {
    return (size_t)(i >> 1) + (size_t)Wh * ((size_t)j + (size_t)H * (size_t)k);
}

// Which domain faces are open (closed_bounds == 0).  j == 0 is the world top
// (yMax, closed_bounds[3]) because object space flips y.
struct OpenFaces { bool xlo, xhi, ylo, yhi, zlo, zhi; };

} // namespace blz
