// noise.cuh — the reference's noise library (thirdparty/cuda-noise/
// cuda_noise.cuh, from github.com/covexp/cuda-noise) as device functions.
//
// Every rounding is explicit (__fmaf_rn, __fmul_rn, __fadd_rn, ...), so this
// build's own FMA contraction cannot change a bit.  The fused multiply-adds
// sit where the reference's CUDA build (-O3 --use_fast_math) fuses the
// library's source when a function is compiled at its own call site: a
// multiply feeding an add in one expression is fused, the left product when
// both operands are products, a product by 2 having become an add first; a
// product used only by adds is fused into each of them across statements.
// Conversions are the GPU's (truncating, saturating).  A division by a
// loop-invariant value is a multiply by its correctly rounded reciprocal,
// formed once (spots' profiles, whose 1 - d r then fuses; fractalSimplex).
#pragma once

#include "common.cuh"
#include "../../include/blaze_b200.h"

namespace blz {
namespace noise {

// Integer sums wrap, as the reference's do on the GPU (cell indices come from
// saturating conversions and may sit at INT_MAX).
__device__ __forceinline__ int wadd(int a, int b) { return (int)((uint32_t)a + (uint32_t)b); }

__device__ __forceinline__ float unit_rand(uint32_t s) {            // randomFloat, 68-74
    return __fmul_rn(__uint2float_rn(lattice_hash(s)), 2.3283064365386963e-10f);
}

__device__ __forceinline__ int int_range(int lo, int hi, int seed) {  // randomIntRange, 59-65
    const int base = (int)lattice_hash((uint32_t)seed);
    return base % (1 + hi - lo) + lo;
}

__device__ __forceinline__ float to_signed(float x) { return __fmaf_rn(x, 2.0f, -1.0f); }   // 88-92

// randomGrid (114-118): the unit random of the hashed float lattice sum.
__device__ __forceinline__ float grid_rand(int x, int y, int z, int seed) {
    float a = __fmaf_rn(__int2float_rn(x), 1723.0f, __fmul_rn(__int2float_rn(y), 93241.0f));
    a = __fmaf_rn(__int2float_rn(z), 149812.0f, a);
    a = __fadd_rn(__fadd_rn(a, 3824.0f), __int2float_rn(seed));
    return to_signed(unit_rand(__float2uint_rz(a)));
}

// cubic (173-176): Catmull-Rom through four samples.
__device__ __forceinline__ float cubic(float p0, float p1, float p2, float p3, float x) {
    const float c3 = __fsub_rn(__fmaf_rn(3.0f, __fsub_rn(p1, p2), p3), p0);
    float c2 = __fmaf_rn(-5.0f, p1, __fadd_rn(p0, p0));
    c2 = __fmaf_rn(4.0f, p2, c2);
    c2 = __fmaf_rn(x, c3, __fsub_rn(c2, p3));
    const float c1 = __fmaf_rn(x, c2, __fsub_rn(p2, p0));
    return __fmaf_rn(__fmul_rn(0.5f, x), c1, p1);
}

__device__ __forceinline__ float fade(float t) { return fade5(t); }             // 204-207
__device__ __forceinline__ float lerp(float a, float b, float r) { return lerp_rn(a, b, r); }

// One simplex corner: (0.6 - r^2)^4 times the dot product of r with edge
// direction g of the library's twelve (160-162): rows 0-3 (+-1, +-1, 0),
// 4-7 (+-1, 0, +-1), 8-11 (0, +-1, +-1), the first sign from bit 0 of g, the
// second from bit 1.
__device__ __forceinline__ float simplex_corner(int g, float x, float y, float z) {
    float t = __fmaf_rn(-z, z, __fmaf_rn(-y, y, __fmaf_rn(-x, x, 0.6f)));
    if (t < 0.0f) return 0.0f;
    t = __fmul_rn(t, t);
    const int a = g >> 2;
    const float s1 = (g & 1) ? -1.0f : 1.0f, s2 = (g & 2) ? -1.0f : 1.0f;
    const float g0 = a == 2 ? 0.0f : s1, g1 = a == 0 ? s2 : (a == 2 ? s1 : 0.0f), g2 = a == 0 ? 0.0f : s2;
    const float d = __fmaf_rn(g2, z, __fmaf_rn(g0, x, __fmul_rn(g1, y)));
    return __fmul_rn(__fmul_rn(t, t), d);
}

// simplexNoise (230-321).
__device__ inline float simplex(float px, float py, float pz, float scale, int seed) {
    const float xin = __fmul_rn(px, scale), yin = __fmul_rn(py, scale), zin = __fmul_rn(pz, scale);
    const float F3 = 1.0f / 3.0f, G3 = 1.0f / 6.0f;
    const float sum = __fadd_rn(__fadd_rn(xin, yin), zin);
    const int i = __float2int_rz(floorf(__fmaf_rn(sum, F3, xin)));
    const int j = __float2int_rz(floorf(__fmaf_rn(sum, F3, yin)));
    const int k = __float2int_rz(floorf(__fmaf_rn(sum, F3, zin)));
    const float ijk = __int2float_rn((int)((uint32_t)i + (uint32_t)j + (uint32_t)k));
    const float x0 = __fsub_rn(xin, __fmaf_rn(-ijk, G3, __int2float_rn(i)));
    const float y0 = __fsub_rn(yin, __fmaf_rn(-ijk, G3, __int2float_rn(j)));
    const float z0 = __fsub_rn(zin, __fmaf_rn(-ijk, G3, __int2float_rn(k)));
    int i1, j1, k1, i2, j2, k2;
    if (x0 >= y0) {
        if (y0 >= z0) { i1 = 1; j1 = 0; k1 = 0; i2 = 1; j2 = 1; k2 = 0; }
        else if (x0 >= z0) { i1 = 1; j1 = 0; k1 = 0; i2 = 1; j2 = 0; k2 = 1; }
        else { i1 = 0; j1 = 0; k1 = 1; i2 = 1; j2 = 0; k2 = 1; }
    } else {
        if (y0 < z0) { i1 = 0; j1 = 0; k1 = 1; i2 = 0; j2 = 1; k2 = 1; }
        else if (x0 < z0) { i1 = 0; j1 = 1; k1 = 0; i2 = 0; j2 = 1; k2 = 1; }
        else { i1 = 0; j1 = 1; k1 = 0; i2 = 1; j2 = 1; k2 = 0; }
    }
    const float G2 = 2.0f * G3, G3x3 = 3.0f * G3;
    // corner hash (calcPerm12, 222-226) of the lattice sum in wrapping int arithmetic
    auto edge = [&](int di, int dj, int dk) {
        const uint32_t h = (uint32_t)seed + (uint32_t)(i + di) * 607495u + (uint32_t)(j + dj) * 359609u +
                           (uint32_t)(k + dk) * 654846u;
        return (int)(lattice_hash(h) % 12u);
    };
    const float n0 = simplex_corner(edge(0, 0, 0), x0, y0, z0);
    const float n1 = simplex_corner(edge(i1, j1, k1), __fadd_rn(__fsub_rn(x0, (float)i1), G3),
                                    __fadd_rn(__fsub_rn(y0, (float)j1), G3), __fadd_rn(__fsub_rn(z0, (float)k1), G3));
    const float n2 = simplex_corner(edge(i2, j2, k2), __fadd_rn(__fsub_rn(x0, (float)i2), G2),
                                    __fadd_rn(__fsub_rn(y0, (float)j2), G2), __fadd_rn(__fsub_rn(z0, (float)k2), G2));
    const float n3 = simplex_corner(edge(1, 1, 1), __fadd_rn(__fsub_rn(x0, 1.0f), G3x3),
                                    __fadd_rn(__fsub_rn(y0, 1.0f), G3x3), __fadd_rn(__fsub_rn(z0, 1.0f), G3x3));
    return __fmul_rn(32.0f, __fadd_rn(__fadd_rn(__fadd_rn(n0, n1), n2), n3));
}

__device__ __forceinline__ float checker(float px, float py, float pz, float scale) {     // 324-335
    const int s = wadd(wadd(__float2int_rz(__fmul_rn(px, scale)), __float2int_rz(__fmul_rn(py, scale))),
                       __float2int_rz(__fmul_rn(pz, scale)));
    return s % 2 == 0 ? 1.0f : -1.0f;
}

// Offset of feature point i of cell (a, b, c) along one axis (spots 358-360,
// worleyNoise 412-414): a jittered unit random; i scales the z term.
__device__ __forceinline__ float feature_offset(int seed, int a, int b, int c, int i, float ka, float kb, float kc,
                                                float k0, float jitter) {
    float s = __fmaf_rn(__int2float_rn(a), ka, __int2float_rn(seed));
    s = __fmaf_rn(__int2float_rn(b), kb, s);
    s = __fmaf_rn(__fmul_rn(__int2float_rn(c), kc), __int2float_rn(i), s);
    s = __fadd_rn(s, k0);
    return __fmaf_rn(unit_rand(__float2uint_rz(s)), jitter, -__fmul_rn(jitter, 0.5f));
}

// Squared distance (and, for spots, the per-axis offsets) to feature point i.
struct FeatureDist { float du, dv, dw, d2; };

__device__ __forceinline__ FeatureDist feature_dist(int seed, int a, int b, int c, int i, float u, float v, float w,
                                                    float jitter) {
    FeatureDist f;
    f.du = __fsub_rn(u, feature_offset(seed, a, b, c, i, 23784.0f, 9183.0f, 23874.0f, 27432.0f, jitter));
    f.dv = __fsub_rn(v, feature_offset(seed, a, b, c, i, 12743.0f, 45191.0f, 144421.0f, 76671.0f, jitter));
    f.dw = __fsub_rn(w, feature_offset(seed, a, b, c, i, 82734.0f, 900213.0f, 443241.0f, 199823.0f, jitter));
    f.d2 = __fmaf_rn(f.dw, f.dw, __fmaf_rn(f.du, f.du, __fmul_rn(f.dv, f.dv)));
    return f;
}

// Feature points per cell (randomIntRange of the hashed cell sum).
__device__ __forceinline__ int feature_count(int seed, int a, int b, int c, float kc, float k0, int lo, int hi) {
    float s = __fmaf_rn(__int2float_rn(a), 823746.0f, __int2float_rn(seed));
    s = __fmaf_rn(__int2float_rn(b), 12306.0f, s);
    s = __fmaf_rn(__int2float_rn(c), kc, s);
    if (k0 != 0.0f) s = __fadd_rn(s, k0);
    return int_range(lo, hi, __float2int_rz(s));
}

// spots (337-393): the best profile value over the feature points of the
// 27 cells around the position.
__device__ inline float spots(float px, float py, float pz, float scale, int seed, float size, int lo, int hi,
                              float jitter, int shape) {
    if (size < 0.000000001f) return 0.0f;
    const int ix = __float2int_rz(__fmul_rn(px, scale)), iy = __float2int_rz(__fmul_rn(py, scale));
    const int iz = __float2int_rz(__fmul_rn(pz, scale));
    const float u = __fsub_rn(px, __int2float_rn(ix)), v = __fsub_rn(py, __int2float_rn(iy));
    const float w = __fsub_rn(pz, __int2float_rn(iz));
    const float rsize = __frcp_rn(size);
    float val = -1.0f;
    for (int x = -1; x < 2; ++x)
        for (int y = -1; y < 2; ++y)
            for (int z = -1; z < 2; ++z) {
                const int a = wadd(ix, x), b = wadd(iy, y), c = wadd(iz, z);
                const int count = feature_count(seed, a, b, c, 823452.0f, 3234874.0f, lo, hi);
                const float uu = __fsub_rn(u, (float)x), vv = __fsub_rn(v, (float)y), ww = __fsub_rn(w, (float)z);
                for (int i = 0; i < count; ++i) {
                    const FeatureDist f = feature_dist(seed, a, b, c, i, uu, vv, ww, jitter);
                    if (shape == BLZ_SHAPE_STEP) {
                        val = fmaxf(val, f.d2 < size ? 1.0f : -1.0f);
                    } else if (shape == BLZ_SHAPE_LINEAR) {
                        const float d1 = __fadd_rn(__fadd_rn(fabsf(f.du), fabsf(f.dv)), fabsf(f.dw));
                        val = fmaxf(val, __fmaf_rn(-__saturatef(d1), rsize, 1.0f));
                    } else if (shape == BLZ_SHAPE_QUADRATIC) {
                        val = fmaxf(val, __fmaf_rn(-__saturatef(f.d2), rsize, 1.0f));
                    }
                }
            }
    return val;
}

// worleyNoise (395-436): the squared distance to the nearest feature point,
// clamped and mapped to [-1, 1].
__device__ inline float worley(float px, float py, float pz, float scale, int seed, float size, int lo, int hi,
                               float jitter) {
    if (size < 0.000000001f) return 0.0f;
    const int ix = __float2int_rz(__fmul_rn(px, scale)), iy = __float2int_rz(__fmul_rn(py, scale));
    const int iz = __float2int_rz(__fmul_rn(pz, scale));
    const float u = __fsub_rn(px, __int2float_rn(ix)), v = __fsub_rn(py, __int2float_rn(iy));
    const float w = __fsub_rn(pz, __int2float_rn(iz));
    float best = 1000000.0f;
    for (int x = -1; x < 2; ++x)
        for (int y = -1; y < 2; ++y)
            for (int z = -1; z < 2; ++z) {
                const int a = wadd(ix, x), b = wadd(iy, y), c = wadd(iz, z);
                const int count = feature_count(seed, a, b, c, 67262.0f, 0.0f, lo, hi);
                const float uu = __fsub_rn(u, (float)x), vv = __fsub_rn(v, (float)y), ww = __fsub_rn(w, (float)z);
                for (int i = 0; i < count; ++i) best = fminf(best, feature_dist(seed, a, b, c, i, uu, vv, ww, jitter).d2);
            }
    return to_signed(__saturatef(best));
}

// tricubic (438-469) of the seed-0 value lattice: x first, then y, then z.
__device__ inline float tricubic(int x, int y, int z, float u, float v, float w) {
    float ys[4];
#pragma unroll 1
    for (int dz = 0; dz < 4; ++dz) {
        float xs[4];
#pragma unroll
        for (int dy = 0; dy < 4; ++dy) {
            const int yy = wadd(y, dy - 1), zz = wadd(z, dz - 1);
            xs[dy] = cubic(grid_rand(wadd(x, -1), yy, zz, 0), grid_rand(x, yy, zz, 0), grid_rand(wadd(x, 1), yy, zz, 0),
                           grid_rand(wadd(x, 2), yy, zz, 0), u);
        }
        ys[dz] = cubic(xs[0], xs[1], xs[2], xs[3], v);
    }
    return cubic(ys[0], ys[1], ys[2], ys[3], w);
}

__device__ __forceinline__ float discrete(float px, float py, float pz, float scale, int seed) {   // 472-480
    return grid_rand(__float2int_rz(__fmul_rn(px, scale)), __float2int_rz(__fmul_rn(py, scale)),
                     __float2int_rz(__fmul_rn(pz, scale)), seed);
}

// Trilinear blend of the eight lattice values of cell (ix, iy, iz).
__device__ __forceinline__ float value_lerp(int ix, int iy, int iz, int seed, float u, float v, float w) {
    const int jx = wadd(ix, 1), jy = wadd(iy, 1), jz = wadd(iz, 1);
    const float x00 = lerp(grid_rand(ix, iy, iz, seed), grid_rand(jx, iy, iz, seed), u);
    const float x10 = lerp(grid_rand(ix, jy, iz, seed), grid_rand(jx, jy, iz, seed), u);
    const float x01 = lerp(grid_rand(ix, iy, jz, seed), grid_rand(jx, iy, jz, seed), u);
    const float x11 = lerp(grid_rand(ix, jy, jz, seed), grid_rand(jx, jy, jz, seed), u);
    return lerp(lerp(x00, x10, v), lerp(x01, x11, v), w);
}

// linearValue (482-515): the library ignores scale here.
__device__ __forceinline__ float linear_value(float px, float py, float pz, float, int seed) {
    const int s = __float2int_rz(__int2float_rn(seed));
    const int ix = __float2int_rz(px), iy = __float2int_rz(py), iz = __float2int_rz(pz);
    return value_lerp(ix, iy, iz, s, __fsub_rn(px, __int2float_rn(ix)), __fsub_rn(py, __int2float_rn(iy)),
                      __fsub_rn(pz, __int2float_rn(iz)));
}

// fadedValue (517-550): the cell comes from the scaled position, the
// fraction from the unscaled one, as in the library.
__device__ __forceinline__ float faded_value(float px, float py, float pz, float scale, int seed) {
    const int s = __float2int_rz(__int2float_rn(seed));
    const int ix = __float2int_rz(__fmul_rn(px, scale)), iy = __float2int_rz(__fmul_rn(py, scale));
    const int iz = __float2int_rz(__fmul_rn(pz, scale));
    const float u = fade(__fsub_rn(px, __int2float_rn(ix))), v = fade(__fsub_rn(py, __int2float_rn(iy)));
    const float w = fade(__fsub_rn(pz, __int2float_rn(iz)));
    return __fmul_rn(value_lerp(ix, iy, iz, s, u, v, w), 0.5f);
}

// cubicValue (552-568): the library ignores seed here.
__device__ __forceinline__ float cubic_value(float px, float py, float pz, float scale, int) {
    px = __fmul_rn(px, scale); py = __fmul_rn(py, scale); pz = __fmul_rn(pz, scale);
    const int ix = __float2int_rz(px), iy = __float2int_rz(py), iz = __float2int_rz(pz);
    return tricubic(ix, iy, iz, __fsub_rn(px, __int2float_rn(ix)), __fsub_rn(py, __int2float_rn(iy)),
                    __fsub_rn(pz, __int2float_rn(iz)));
}

// One basis of the generic repeater (734-779) at the library's fixed offset
// for that basis, scale 1.
__device__ inline float basis_at(int basis, float px, float py, float pz, float scale, int seed) {
    switch (basis) {
    case BLZ_NOISE_CHECKER:
        return checker(__fmaf_rn(px, scale, 53872.1923f), __fmaf_rn(py, scale, 58334.4081f),
                       __fmaf_rn(pz, scale, 9358.34667f), 1.0f);
    case BLZ_NOISE_DISCRETE:
        return discrete(__fmaf_rn(px, scale, 7852.53114f), __fmaf_rn(py, scale, 319739.059f),
                        __fmaf_rn(pz, scale, 451336.504f), 1.0f, seed);
    case BLZ_NOISE_LINEARVALUE:
        return linear_value(__fmaf_rn(px, scale, 940.748139f), __fmaf_rn(py, scale, 10196.4500f),
                            __fmaf_rn(pz, scale, 25650.9789f), 1.0f, seed);
    case BLZ_NOISE_FADEDVALUE:
        return faded_value(__fmaf_rn(px, scale, 7683.26428f), __fmaf_rn(py, scale, 2417.78195f),
                           __fmaf_rn(pz, scale, 93889.4897f), 1.0f, seed);
    case BLZ_NOISE_CUBICVALUE:
        return cubic_value(__fmaf_rn(px, scale, 6546.80178f), __fmaf_rn(py, scale, 14459.4682f),
                           __fmaf_rn(pz, scale, 11616.5811f), 1.0f, seed);
    case BLZ_NOISE_PERLIN:
        return perlin(__fmaf_rn(px, scale, 1764.66931f), __fmaf_rn(py, scale, 2593.55017f),
                      __fmaf_rn(pz, scale, 4813.24412f), 1.0f, seed);
    case BLZ_NOISE_SIMPLEX:
        return simplex(__fmaf_rn(px, scale, 7442.93020f), __fmaf_rn(py, scale, 8341.06698f),
                       __fmaf_rn(pz, scale, 66848.7870f), 1.0f, seed);
    case BLZ_NOISE_WORLEY:
        return worley(__fmaf_rn(px, scale, 7619.01285f), __fmaf_rn(py, scale, 57209.0681f),
                      __fmaf_rn(pz, scale, 1167.91397f), 1.0f, seed, 0.1f, 4, 4, 1.0f);
    case BLZ_NOISE_SPOTS:
        return spots(__fmaf_rn(px, scale, 33836.4116f), __fmaf_rn(py, scale, 2242.51045f),
                     __fmaf_rn(pz, scale, 6720.07486f), 1.0f, seed, 0.1f, 0, 4, 1.0f, BLZ_SHAPE_LINEAR);
    default:
        return 0.0f;
    }
}

__device__ inline float repeater(float px, float py, float pz, float scale, int seed, int n, float lac, float decay,
                                 int basis) {
    float acc = 0.0f, amp = 1.0f;
    for (int i = 0; i < n; ++i) {
        acc = __fmaf_rn(basis_at(basis, px, py, pz, scale, seed), amp, acc);
        scale = __fmul_rn(scale, lac);
        amp = __fmul_rn(amp, decay);
    }
    return acc;
}

// A basis as turbulence evaluates it (804-865): the library's own scale and
// arguments, no offset.  Discrete and spots give nothing there.
__device__ inline float turb_basis(int basis, float px, float py, float pz, float scale, int seed) {
    switch (basis) {
    case BLZ_NOISE_CHECKER: return checker(px, py, pz, scale);
    case BLZ_NOISE_LINEARVALUE: return linear_value(px, py, pz, scale, seed);
    case BLZ_NOISE_FADEDVALUE: return faded_value(px, py, pz, scale, seed);
    case BLZ_NOISE_CUBICVALUE: return cubic_value(px, py, pz, scale, seed);
    case BLZ_NOISE_PERLIN: return perlin(px, py, pz, scale, seed);
    case BLZ_NOISE_SIMPLEX: return simplex(px, py, pz, scale, seed);
    case BLZ_NOISE_WORLEY: return worley(px, py, pz, scale, seed, 1.0f, 4, 4, 1.0f);
    default: return 0.0f;
    }
}

// The seed salts of turbulence's first pass, per basis and axis (806-848).
__device__ __forceinline__ int turb_salt(int basis, int axis) {
    switch (basis) {
    case BLZ_NOISE_CHECKER: return axis == 0 ? 0x34ff8885 : axis == 1 ? 0x2d03cba3 : 0x5a76fb1b;
    case BLZ_NOISE_LINEARVALUE: return axis == 0 ? 0x5527fdb8 : axis == 1 ? 0x42af1a2e : 0x1482ee8c;
    case BLZ_NOISE_FADEDVALUE: return axis == 0 ? 0x295590fc : axis == 1 ? 0x30731854 : 0x73d2ca4c;
    case BLZ_NOISE_CUBICVALUE: return axis == 0 ? 0x663a1f09 : axis == 1 ? 0x429bf56b : 0x37fa6fe9;
    case BLZ_NOISE_PERLIN: return axis == 0 ? 0x74827384 : axis == 1 ? 0x10938478 : 0x62723883;
    case BLZ_NOISE_SIMPLEX: return axis == 0 ? 0x47829472 : axis == 1 ? 0x58273829 : 0x10294647;
    case BLZ_NOISE_WORLEY: return axis == 0 ? 0x1d96f515 : axis == 1 ? 0x4df308f0 : 0x2b79442a;
    default: return 0;
    }
}

__device__ inline float turbulence(float px, float py, float pz, float sin_, float sout, int seed, float strength,
                                   int bin, int bout) {
    if (bin != BLZ_NOISE_DISCRETE && bin != BLZ_NOISE_SPOTS) {
        // each axis is offset at the position already offset along the axes before it
        px = __fmaf_rn(turb_basis(bin, px, py, pz, sin_, seed ^ turb_salt(bin, 0)), strength, px);
        py = __fmaf_rn(turb_basis(bin, px, py, pz, sin_, seed ^ turb_salt(bin, 1)), strength, py);
        pz = __fmaf_rn(turb_basis(bin, px, py, pz, sin_, seed ^ turb_salt(bin, 2)), strength, pz);
    }
    // the library's second pass uses scaleIn for simplex and worley
    const float so = (bout == BLZ_NOISE_SIMPLEX || bout == BLZ_NOISE_WORLEY) ? sin_ : sout;
    return turb_basis(bout, px, py, pz, so, seed);
}

// The selected function at one position.
__device__ inline float eval(const blz_noise_args &a, float px, float py, float pz) {
    const int n = a.octaves;
    float scale = a.scale, amp = 1.0f, acc;
    switch (a.func) {
    case BLZ_NOISE_CHECKER: return checker(px, py, pz, a.scale);
    case BLZ_NOISE_DISCRETE: return discrete(px, py, pz, a.scale, a.seed);
    case BLZ_NOISE_LINEARVALUE: return linear_value(px, py, pz, a.scale, a.seed);
    case BLZ_NOISE_FADEDVALUE: return faded_value(px, py, pz, a.scale, a.seed);
    case BLZ_NOISE_CUBICVALUE: return cubic_value(px, py, pz, a.scale, a.seed);
    case BLZ_NOISE_PERLIN: return perlin(px, py, pz, a.scale, a.seed);
    case BLZ_NOISE_SIMPLEX: return simplex(px, py, pz, a.scale, a.seed);
    case BLZ_NOISE_WORLEY: return worley(px, py, pz, a.scale, a.seed, a.size, a.min_num, a.max_num, a.jitter);
    case BLZ_NOISE_SPOTS:
        return spots(px, py, pz, a.scale, a.seed, a.size, a.min_num, a.max_num, a.jitter, a.shape);
    case BLZ_NOISE_REPEATER_PERLIN:                               // 620-633: the octave seeds ignore seed
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            const float p = perlin(__fmul_rn(px, scale), __fmul_rn(py, scale), __fmul_rn(pz, scale), 1.0f,
                                   (int)((uint32_t)(i + 38) * 27389482u));
            acc = __fmaf_rn(p, amp, acc);
            scale = __fmul_rn(scale, a.lacunarity);
            amp = __fmul_rn(amp, a.decay);
        }
        return acc;
    case BLZ_NOISE_REPEATER_PERLIN_BOUNDED:                       // 636-656
        acc = 1.0f;
        for (int i = 0; i < n; ++i) {
            const float p = perlin(__fmul_rn(px, scale), __fmul_rn(py, scale), __fmul_rn(pz, scale), 1.0f,
                                   a.seed ^ (int)((uint32_t)(i + 38) * 27389482u));
            acc = __fmul_rn(acc, __fmaf_rn(-__saturatef(__fmaf_rn(0.5f, p, 0.5f)), amp, 1.0f));
            if (acc < a.threshold) return 0.0f;
            scale = __fmul_rn(scale, a.lacunarity);
            amp = __fmul_rn(amp, a.decay);
        }
        return acc;
    case BLZ_NOISE_REPEATER_PERLIN_ABS:                           // 659-673
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            const float p = perlin(__fmul_rn(px, scale), __fmul_rn(py, scale), __fmul_rn(pz, scale), 1.0f, a.seed);
            acc = __fmaf_rn(fabsf(p), amp, acc);
            scale = __fmul_rn(scale, a.lacunarity);
            amp = __fmul_rn(amp, a.decay);
        }
        return to_signed(acc);
    case BLZ_NOISE_REPEATER_SIMPLEX:                              // 676-690
    case BLZ_NOISE_REPEATER_SIMPLEX_ABS: {                        // 693-707
        const bool absval = a.func == BLZ_NOISE_REPEATER_SIMPLEX_ABS;
        int seed = a.seed;
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            const float s = simplex(px, py, pz, scale, seed);
            acc = __fmaf_rn(__fmul_rn(absval ? fabsf(s) : s, amp), 0.35f, acc);
            scale = __fmul_rn(scale, a.lacunarity);
            amp = __fmul_rn(amp, a.decay);
            seed ^= (int)(absval ? (uint32_t)(i + 198273) * 928374u : (uint32_t)(i + 672381) * 200394u);
        }
        return absval ? to_signed(acc) : acc;
    }
    case BLZ_NOISE_REPEATER_SIMPLEX_BOUNDED:                      // 710-731
        acc = 1.0f;
        for (int i = 0; i < n; ++i) {
            const float s = simplex(__fmaf_rn(px, scale, 32240.7922f), __fmaf_rn(py, scale, 835622.882f),
                                    __fmaf_rn(pz, scale, 824.371968f), 1.0f, a.seed);
            acc = __fsub_rn(acc, __fmul_rn(__saturatef(__fmaf_rn(s, 0.3f, 0.5f)), amp));
            if (acc < a.threshold) return 0.0f;
            scale = __fmul_rn(scale, a.lacunarity);
            amp = __fmul_rn(amp, a.decay);
        }
        return acc;
    case BLZ_NOISE_REPEATER:
        return repeater(px, py, pz, a.scale, a.seed, n, a.lacunarity, a.decay, a.basis);
    case BLZ_NOISE_FRACTAL_SIMPLEX: {                             // 782-801
        const float rdu = __frcp_rn(a.du);
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            const float s = simplex(__fmaf_rn(px, scale, 617.437379f), __fmaf_rn(py, scale, 196410.219f),
                                    __fmaf_rn(pz, scale, 321280.627f), 1.0f, (int)((uint32_t)a.seed * (uint32_t)(i + 1)));
            acc = __fmaf_rn(s, amp, acc);
            scale = __fmul_rn(scale, a.lacunarity);
            amp = __fmul_rn(amp, a.decay);
            if (scale > rdu) break;
        }
        return acc;
    }
    case BLZ_NOISE_TURBULENCE:
        return turbulence(px, py, pz, a.scale, a.scale_out, a.seed, a.strength, a.basis, a.basis_out);
    case BLZ_NOISE_REPEATER_TURBULENCE: {                         // 867-874
        px = __fmaf_rn(repeater(px, py, pz, a.scale, a.seed ^ 0x41728394, n, 2.0f, 0.5f, a.basis), a.strength, px);
        py = __fmaf_rn(repeater(px, py, pz, a.scale, a.seed ^ 0x72837263, n, 2.0f, 0.5f, a.basis), a.strength, py);
        pz = __fmaf_rn(repeater(px, py, pz, a.scale, a.seed ^ 0x26837363, n, 2.0f, 0.5f, a.basis), a.strength, pz);
        return repeater(px, py, pz, a.scale_out, a.seed ^ 0x3f821dab, n, 2.0f, 0.5f, a.basis_out);
    }
    default:
        return 0.0f;
    }
}

}  // namespace noise
}  // namespace blz
