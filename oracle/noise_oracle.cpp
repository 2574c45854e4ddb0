// noise_oracle.cpp — CPU restatement of the reference's noise library
// (thirdparty/cuda-noise/cuda_noise.cuh, vendored by Blaze from
// github.com/covexp/cuda-noise, no pinned version).
//
// TEST INFRASTRUCTURE ONLY: the checker for blz_noise.  Pinned against the
// reference's own CUDA build (tests/golden/noise.npz).
//
// Arithmetic is FP32, one IEEE operation at a time (the library is built with
// -ffp-contract=off), so every rounding is written out; fm() marks a fused
// multiply-add.  They sit where the reference's CUDA build (its documented
// flags: -O3 --use_fast_math) fuses the library's source, found by comparing
// candidate forms with that build's output (tests/golden/noise.npz):
//   - a multiply feeding an add or subtract is fused; when both operands are
//     products, the left one (cubic's 2 p0 - 5 p1 fuses 5 p1: a product by 2
//     has become an add first);
//   - a product whose only users are adds is fused into each of them, across
//     statements (simplexNoise's skew s and unskew t); a product that also
//     feeds anything else (a floor, a conversion) stays rounded.
// These are the forms at a function's own call site.  Where the reference
// build inlines several evaluations into one function and shares their
// lattice products (the cubic-value repeater, turbulence over value noise),
// its heuristic fuses the other product of some lattice-hash sums instead
// (x*1723 + y*93241: the y product); the test hook
// orc_noise_set_lattice_patterns reproduces such patterns.
// Conversions follow the GPU's: float -> int and float -> unsigned truncate
// toward zero and saturate (NaN -> 0); int arithmetic wraps.  A division by a
// loop-invariant value is a multiply by its reciprocal, formed once (spots'
// profiles 1 - d / size, which then fuse; fractalSimplex's 1 / du).
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../include/blaze_b200.h"

namespace nz {

static inline float fm(float a, float b, float c) { return std::fma(a, b, c); }

static inline uint32_t mix(uint32_t s) {                     // hash, cuda_noise.cuh:46-57
    s = (s + 0x7ed55d16u) + (s << 12);
    s = (s ^ 0xc761c23cu) ^ (s >> 19);
    s = (s + 0x165667b1u) + (s << 5);
    s = (s + 0xd3a2646cu) ^ (s << 9);
    s = (s + 0xfd7046c5u) + (s << 3);
    s = (s ^ 0xb55a4f09u) ^ (s >> 16);
    return s;
}

static inline uint32_t f2u(float x) {                        // cvt.rzi.u32.f32
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}

static inline int32_t f2i(float x) {                         // cvt.rzi.s32.f32
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

static inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

// randomFloat (68-74): the hash over 2^32 (the divisor rounds to 2^32).
static inline float unit_rand(uint32_t s) { return (float)mix(s) * 2.3283064365386963e-10f; }

// randomIntRange (59-65), signed remainder as in C.
static inline int int_range(int lo, int hi, int32_t seed) {
    const int32_t base = (int32_t)mix((uint32_t)seed);
    return base % (1 + hi - lo) + lo;
}

static inline float to_signed(float x) { return fm(x, 2.0f, -1.0f); }     // mapToSigned (88-92)
static inline float sat(float x) { return x != x ? 0.0f : std::fmin(std::fmax(x, 0.0f), 1.0f); }

// randomGrid (114-118): hash of the float lattice sum, as signed unit value.
static inline float grid_rand(int x, int y, int z, int seed) {
    float a = fm((float)x, 1723.0f, (float)y * 93241.0f);
    a = fm((float)z, 149812.0f, a);
    a = a + 3824.0f;
    a = a + (float)seed;
    return to_signed(unit_rand(f2u(a)));
}

// randomIntGrid (120-124).
static inline uint32_t grid_hash(float x, float y, float z, float seed) {
    float a = fm(x, 1723.0f, y * 93241.0f);
    a = fm(z, 149812.0f, a);
    a = a + 3824.0f;
    a = a + seed;
    return mix(f2u(a));
}

static inline float lerp(float a, float b, float r) { return fm(a, 1.0f - r, b * r); }   // 167-170

// Test hook (orc_noise_set_lattice_patterns): the k-th value-noise
// evaluation at a position (a trilinear or tricubic lattice blend) takes
// pattern k of the list, the last one repeating; a set bit fuses the y
// product of that lattice point's hash sum instead of the x product.  Bit
// dx + 2 dy + 4 dz for the trilinear corners, dx + 4 dy + 16 dz (offsets
// 0..3 from x-1, y-1, z-1) for the tricubic points.  No patterns (the
// default) is the form of a standalone call.
static uint64_t g_patterns[16];
static int g_npatterns = 0;
static thread_local int t_blend = 0;

static inline uint64_t next_pattern() {
    if (g_npatterns == 0) return 0;
    const int k = t_blend++;
    return g_patterns[k < g_npatterns ? k : g_npatterns - 1];
}

static inline float grid_rand_p(int x, int y, int z, int seed, bool yfirst) {
    if (!yfirst) return grid_rand(x, y, z, seed);
    float a = fm((float)y, 93241.0f, (float)x * 1723.0f);
    a = fm((float)z, 149812.0f, a);
    a = a + 3824.0f;
    a = a + (float)seed;
    return to_signed(unit_rand(f2u(a)));
}

// cubic (173-176): Catmull-Rom through four samples.
static inline float cubic(float p0, float p1, float p2, float p3, float x) {
    const float c3 = fm(3.0f, p1 - p2, p3) - p0;
    float c2 = fm(-5.0f, p1, 2.0f * p0);
    c2 = fm(4.0f, p2, c2);
    c2 = c2 - p3;
    c2 = fm(x, c3, c2);
    const float c1 = fm(x, c2, p2 - p0);
    return fm(0.5f * x, c1, p1);
}

static inline float grad(uint32_t h, float x, float y, float z) {    // 179-201
    switch (h & 0xF) {
    case 0x0: return x + y;   case 0x1: return -x + y;
    case 0x2: return x - y;   case 0x3: return -x - y;
    case 0x4: return x + z;   case 0x5: return -x + z;
    case 0x6: return x - z;   case 0x7: return -x - z;
    case 0x8: return y + z;   case 0x9: return -y + z;
    case 0xA: return y - z;   case 0xB: return -y - z;
    case 0xC: return y + x;   case 0xD: return -y + z;
    case 0xE: return y - x;   default:  return -y - z;
    }
}

static inline float fade(float t) {                          // 204-207
    const float inner = fm(t, fm(t, 6.0f, -15.0f), 10.0f);
    return t * t * t * inner;
}

// The twelve edge directions of simplexNoise's gradient table (160-162).
static const float kEdges[12][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
                                    {1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};

static inline float dot3(const float g[3], float x, float y, float z) { return fm(g[2], z, fm(g[0], x, g[1] * y)); }

static inline int edge12(int32_t p) { return (int)(uint8_t)(mix((uint32_t)p) % 12u); }   // calcPerm12 (222-226)

// simplexNoise (230-321).
float simplex(float px, float py, float pz, float scale, int seed) {
    const float xin = px * scale, yin = py * scale, zin = pz * scale;
    const float F3 = 1.0f / 3.0f, G3 = 1.0f / 6.0f;
    const float sum = (xin + yin) + zin;                 // skew: s = sum F3, fused into xin + s
    const int i = f2i(std::floor(fm(sum, F3, xin))), j = f2i(std::floor(fm(sum, F3, yin)));
    const int k = f2i(std::floor(fm(sum, F3, zin)));
    const float ijk = (float)wadd(wadd(i, j), k);         // unskew: t = ijk G3, fused into i - t
    const float x0 = xin - fm(-ijk, G3, (float)i), y0 = yin - fm(-ijk, G3, (float)j), z0 = zin - fm(-ijk, G3, (float)k);
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
    const float x1 = (x0 - (float)i1) + G3, y1 = (y0 - (float)j1) + G3, z1 = (z0 - (float)k1) + G3;
    const float x2 = (x0 - (float)i2) + G2, y2 = (y0 - (float)j2) + G2, z2 = (z0 - (float)k2) + G2;
    const float x3 = (x0 - 1.0f) + G3x3, y3 = (y0 - 1.0f) + G3x3, z3 = (z0 - 1.0f) + G3x3;
    auto corner = [&](int di, int dj, int dk) {
        return edge12(wadd(wadd(wadd(seed, wmul(wadd(i, di), 607495)), wmul(wadd(j, dj), 359609)),
                           wmul(wadd(k, dk), 654846)));
    };
    const int g0 = corner(0, 0, 0), g1 = corner(i1, j1, k1), g2 = corner(i2, j2, k2), g3 = corner(1, 1, 1);
    auto contrib = [&](int g, float x, float y, float z) {
        float tt = fm(-z, z, fm(-y, y, fm(-x, x, 0.6f)));
        if (tt < 0.0f) return 0.0f;
        tt = tt * tt;
        return tt * tt * dot3(kEdges[g], x, y, z);
    };
    const float n0 = contrib(g0, x0, y0, z0), n1 = contrib(g1, x1, y1, z1);
    const float n2 = contrib(g2, x2, y2, z2), n3 = contrib(g3, x3, y3, z3);
    return 32.0f * (((n0 + n1) + n2) + n3);
}

float checker(float px, float py, float pz, float scale) {                  // 324-335
    const int s = wadd(wadd(f2i(px * scale), f2i(py * scale)), f2i(pz * scale));
    return s % 2 == 0 ? 1.0f : -1.0f;
}

// The feature-point offset of spots and worleyNoise (358-360, 412-414): a
// jittered unit random per axis, the cell's point number i scaling the z term.
static inline float jit(int32_t seed, int a, int b, int c, int i, float ka, float kb, float kc, float k0,
                        float jitter) {
    float s = fm((float)a, ka, (float)seed);
    s = fm((float)b, kb, s);
    s = fm((float)c * kc, (float)i, s);
    s = s + k0;
    return fm(unit_rand(f2u(s)), jitter, -(jitter / 2.0f));
}

float spots(float px, float py, float pz, float scale, int seed, float size, int lo, int hi, float jitter,
            int shape) {                                                     // 337-393
    if (size < 0.000000001f) return 0.0f;
    const int ix = f2i(px * scale), iy = f2i(py * scale), iz = f2i(pz * scale);
    const float u = px - (float)ix, v = py - (float)iy, w = pz - (float)iz;
    const float rsize = 1.0f / size;
    float val = -1.0f;
    for (int x = -1; x < 2; ++x)
        for (int y = -1; y < 2; ++y)
            for (int z = -1; z < 2; ++z) {
                const int a = wadd(ix, x), b = wadd(iy, y), c = wadd(iz, z);
                float sd = fm((float)a, 823746.0f, (float)seed);
                sd = fm((float)b, 12306.0f, sd);
                sd = fm((float)c, 823452.0f, sd);
                sd = sd + 3234874.0f;
                const int count = int_range(lo, hi, f2i(sd));
                for (int i = 0; i < count; ++i) {
                    const float dU = (u - (float)x) - jit(seed, a, b, c, i, 23784.0f, 9183.0f, 23874.0f, 27432.0f, jitter);
                    const float dV = (v - (float)y) - jit(seed, a, b, c, i, 12743.0f, 45191.0f, 144421.0f, 76671.0f, jitter);
                    const float dW = (w - (float)z) - jit(seed, a, b, c, i, 82734.0f, 900213.0f, 443241.0f, 199823.0f, jitter);
                    const float d2 = fm(dW, dW, fm(dU, dU, dV * dV));
                    if (shape == BLZ_SHAPE_STEP) {
                        val = std::fmax(val, d2 < size ? 1.0f : -1.0f);
                    } else if (shape == BLZ_SHAPE_LINEAR) {
                        const float d1 = (std::fabs(dU) + std::fabs(dV)) + std::fabs(dW);
                        val = std::fmax(val, fm(-sat(d1), rsize, 1.0f));  // clamp (76-85) clamps to [0, 1]
                    } else if (shape == BLZ_SHAPE_QUADRATIC) {
                        val = std::fmax(val, fm(-sat(d2), rsize, 1.0f));
                    }
                }
            }
    return val;
}

float worley(float px, float py, float pz, float scale, int seed, float size, int lo, int hi, float jitter) {
    if (size < 0.000000001f) return 0.0f;                                   // 395-436
    const int ix = f2i(px * scale), iy = f2i(py * scale), iz = f2i(pz * scale);
    const float u = px - (float)ix, v = py - (float)iy, w = pz - (float)iz;
    float best = 1000000.0f;
    for (int x = -1; x < 2; ++x)
        for (int y = -1; y < 2; ++y)
            for (int z = -1; z < 2; ++z) {
                const int a = wadd(ix, x), b = wadd(iy, y), c = wadd(iz, z);
                float sd = fm((float)a, 823746.0f, (float)seed);
                sd = fm((float)b, 12306.0f, sd);
                sd = fm((float)c, 67262.0f, sd);
                const int count = int_range(lo, hi, f2i(sd));
                for (int i = 0; i < count; ++i) {
                    const float dU = (u - (float)x) - jit(seed, a, b, c, i, 23784.0f, 9183.0f, 23874.0f, 27432.0f, jitter);
                    const float dV = (v - (float)y) - jit(seed, a, b, c, i, 12743.0f, 45191.0f, 144421.0f, 76671.0f, jitter);
                    const float dW = (w - (float)z) - jit(seed, a, b, c, i, 82734.0f, 900213.0f, 443241.0f, 199823.0f, jitter);
                    const float d2 = fm(dW, dW, fm(dU, dU, dV * dV));
                    if (d2 < best) best = d2;
                }
            }
    return fm(sat(best), 2.0f, -1.0f);
}

// tricubic (438-469) of the seed-0 value lattice: x first, then y, then z.
static float tricubic(int x, int y, int z, float u, float v, float w) {
    const uint64_t pat = next_pattern();
    float ys[4];
    for (int dz = 0; dz < 4; ++dz) {
        float xs[4];
        for (int dy = 0; dy < 4; ++dy) {
            float p[4];
            for (int dx = 0; dx < 4; ++dx) {
                const int xx = wadd(x, dx - 1), yy = wadd(y, dy - 1), zz = wadd(z, dz - 1);
                p[dx] = grid_rand_p(xx, yy, zz, 0, (pat >> (dx + 4 * dy + 16 * dz)) & 1u);
            }
            xs[dy] = cubic(p[0], p[1], p[2], p[3], u);
        }
        ys[dz] = cubic(xs[0], xs[1], xs[2], xs[3], v);
    }
    return cubic(ys[0], ys[1], ys[2], ys[3], w);
}

float discrete(float px, float py, float pz, float scale, int seed) {       // 472-480
    return grid_rand(f2i(px * scale), f2i(py * scale), f2i(pz * scale), seed);
}

// Trilinear blend of the eight lattice values around cell (ix, iy, iz).
static inline float value_lerp(int ix, int iy, int iz, int seed, float u, float v, float w) {
    const uint64_t p = next_pattern();
    auto g = [&](int dx, int dy, int dz) {
        return grid_rand_p(wadd(ix, dx), wadd(iy, dy), wadd(iz, dz), seed, (p >> (dx + 2 * dy + 4 * dz)) & 1u);
    };
    const float x00 = lerp(g(0, 0, 0), g(1, 0, 0), u);
    const float x10 = lerp(g(0, 1, 0), g(1, 1, 0), u);
    const float x01 = lerp(g(0, 0, 1), g(1, 0, 1), u);
    const float x11 = lerp(g(0, 1, 1), g(1, 1, 1), u);
    return lerp(lerp(x00, x10, v), lerp(x01, x11, v), w);
}

float linear_value(float px, float py, float pz, float /*scale: unused by the library*/, int seed) {   // 482-515
    const int s = f2i((float)seed);
    const int ix = f2i(px), iy = f2i(py), iz = f2i(pz);
    return value_lerp(ix, iy, iz, s, px - (float)ix, py - (float)iy, pz - (float)iz);
}

float faded_value(float px, float py, float pz, float scale, int seed) {     // 517-550
    const int s = f2i((float)seed);
    const int ix = f2i(px * scale), iy = f2i(py * scale), iz = f2i(pz * scale);
    const float u = fade(px - (float)ix), v = fade(py - (float)iy), w = fade(pz - (float)iz);
    return value_lerp(ix, iy, iz, s, u, v, w) * 0.5f;
}

float cubic_value(float px, float py, float pz, float scale, int /*seed: unused by the library*/) {  // 552-568
    px = px * scale; py = py * scale; pz = pz * scale;
    const int ix = f2i(px), iy = f2i(py), iz = f2i(pz);
    return tricubic(ix, iy, iz, px - (float)ix, py - (float)iy, pz - (float)iz);
}

float perlin(float px, float py, float pz, float scale, int seed) {          // 570-615
    const float fs = (float)seed;
    px = px * scale; py = py * scale; pz = pz * scale;
    const float ix = std::floor(px), iy = std::floor(py), iz = std::floor(pz);
    px = px - ix; py = py - iy; pz = pz - iz;
    const float u = fade(px), v = fade(py), w = fade(pz);
    const float ix1 = ix + 1.0f, iy1 = iy + 1.0f, iz1 = iz + 1.0f;
    const float qx = px - 1.0f, qy = py - 1.0f, qz = pz - 1.0f;
    const float i000 = grad(grid_hash(ix, iy, iz, fs), px, py, pz);
    const float i100 = grad(grid_hash(ix1, iy, iz, fs), qx, py, pz);
    const float i010 = grad(grid_hash(ix, iy1, iz, fs), px, qy, pz);
    const float i110 = grad(grid_hash(ix1, iy1, iz, fs), qx, qy, pz);
    const float i001 = grad(grid_hash(ix, iy, iz1, fs), px, py, qz);
    const float i101 = grad(grid_hash(ix1, iy, iz1, fs), qx, py, qz);
    const float i011 = grad(grid_hash(ix, iy1, iz1, fs), px, qy, qz);
    const float i111 = grad(grid_hash(ix1, iy1, iz1, fs), qx, qy, qz);
    const float y0 = lerp(lerp(i000, i100, u), lerp(i010, i110, u), v);
    const float y1 = lerp(lerp(i001, i101, u), lerp(i011, i111, u), v);
    return lerp(y0, y1, w);
}

// One basis of the generic repeater (734-779), at the library's fixed offset
// of that basis and scale 1.
static float basis_at(int basis, float px, float py, float pz, float scale, int seed) {
    switch (basis) {
    case BLZ_NOISE_CHECKER:
        return checker(fm(px, scale, 53872.1923f), fm(py, scale, 58334.4081f), fm(pz, scale, 9358.34667f), 1.0f);
    case BLZ_NOISE_DISCRETE:
        return discrete(fm(px, scale, 7852.53114f), fm(py, scale, 319739.059f), fm(pz, scale, 451336.504f), 1.0f,
                        seed);
    case BLZ_NOISE_LINEARVALUE:
        return linear_value(fm(px, scale, 940.748139f), fm(py, scale, 10196.4500f), fm(pz, scale, 25650.9789f), 1.0f,
                            seed);
    case BLZ_NOISE_FADEDVALUE:
        return faded_value(fm(px, scale, 7683.26428f), fm(py, scale, 2417.78195f), fm(pz, scale, 93889.4897f), 1.0f,
                           seed);
    case BLZ_NOISE_CUBICVALUE:
        return cubic_value(fm(px, scale, 6546.80178f), fm(py, scale, 14459.4682f), fm(pz, scale, 11616.5811f), 1.0f,
                           seed);
    case BLZ_NOISE_PERLIN:
        return perlin(fm(px, scale, 1764.66931f), fm(py, scale, 2593.55017f), fm(pz, scale, 4813.24412f), 1.0f, seed);
    case BLZ_NOISE_SIMPLEX:
        return simplex(fm(px, scale, 7442.93020f), fm(py, scale, 8341.06698f), fm(pz, scale, 66848.7870f), 1.0f, seed);
    case BLZ_NOISE_WORLEY:
        return worley(fm(px, scale, 7619.01285f), fm(py, scale, 57209.0681f), fm(pz, scale, 1167.91397f), 1.0f, seed,
                      0.1f, 4, 4, 1.0f);
    case BLZ_NOISE_SPOTS:
        return spots(fm(px, scale, 33836.4116f), fm(py, scale, 2242.51045f), fm(pz, scale, 6720.07486f), 1.0f, seed,
                     0.1f, 0, 4, 1.0f, BLZ_SHAPE_LINEAR);
    default:
        return 0.0f;
    }
}

static float repeater(float px, float py, float pz, float scale, int seed, int n, float lac, float decay, int basis) {
    float acc = 0.0f, amp = 1.0f;
    for (int i = 0; i < n; ++i) {
        acc = fm(basis_at(basis, px, py, pz, scale, seed), amp, acc);
        scale = scale * lac;
        amp = amp * decay;
    }
    return acc;
}

// The first pass of turbulence (804-848): one noise offset per axis, each
// evaluated at the position already offset along the axes before it.
static void turb_offset(int basis, float &px, float &py, float &pz, float scale, int seed, float strength) {
    auto f = [&](int salt) -> float {
        switch (basis) {
        case BLZ_NOISE_CHECKER: return checker(px, py, pz, scale);
        case BLZ_NOISE_LINEARVALUE: return linear_value(px, py, pz, scale, seed ^ salt);
        case BLZ_NOISE_FADEDVALUE: return faded_value(px, py, pz, scale, seed ^ salt);
        case BLZ_NOISE_CUBICVALUE: return cubic_value(px, py, pz, scale, seed ^ salt);
        case BLZ_NOISE_PERLIN: return perlin(px, py, pz, scale, seed ^ salt);
        case BLZ_NOISE_SIMPLEX: return simplex(px, py, pz, scale, seed ^ salt);
        case BLZ_NOISE_WORLEY: return worley(px, py, pz, scale, seed ^ salt, 1.0f, 4, 4, 1.0f);
        default: return 0.0f;
        }
    };
    static const int kSalt[9][3] = {
        {0x34ff8885, 0x2d03cba3, 0x5a76fb1b}, {0, 0, 0},
        {0x5527fdb8, 0x42af1a2e, 0x1482ee8c}, {0x295590fc, 0x30731854, 0x73d2ca4c},
        {0x663a1f09, 0x429bf56b, 0x37fa6fe9}, {0x74827384, 0x10938478, 0x62723883},
        {0x47829472, 0x58273829, 0x10294647}, {0x1d96f515, 0x4df308f0, 0x2b79442a}, {0, 0, 0}};
    if (basis == BLZ_NOISE_DISCRETE || basis == BLZ_NOISE_SPOTS || basis < 0 || basis > 8) return;
    px = fm(f(kSalt[basis][0]), strength, px);
    py = fm(f(kSalt[basis][1]), strength, py);
    pz = fm(f(kSalt[basis][2]), strength, pz);
}

float turbulence(float px, float py, float pz, float scale_in, float scale_out, int seed, float strength, int bin,
                 int bout) {
    turb_offset(bin, px, py, pz, scale_in, seed, strength);
    switch (bout) {                                                          // 850-864
    case BLZ_NOISE_CHECKER: return checker(px, py, pz, scale_out);
    case BLZ_NOISE_LINEARVALUE: return linear_value(px, py, pz, scale_out, seed);
    case BLZ_NOISE_FADEDVALUE: return faded_value(px, py, pz, scale_out, seed);
    case BLZ_NOISE_CUBICVALUE: return cubic_value(px, py, pz, scale_out, seed);
    case BLZ_NOISE_PERLIN: return perlin(px, py, pz, scale_out, seed);
    case BLZ_NOISE_SIMPLEX: return simplex(px, py, pz, scale_in, seed);      // the library uses scaleIn here
    case BLZ_NOISE_WORLEY: return worley(px, py, pz, scale_in, seed, 1.0f, 4, 4, 1.0f);
    default: return 0.0f;
    }
}

float eval(const blz_noise_args &a, float px, float py, float pz) {
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
    case BLZ_NOISE_REPEATER_PERLIN:                                          // 620-633: octave seeds fixed
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            acc = fm(perlin(px * scale, py * scale, pz * scale, 1.0f, wmul(i + 38, 27389482)), amp, acc);
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
        }
        return acc;
    case BLZ_NOISE_REPEATER_PERLIN_BOUNDED:                                  // 636-656
        acc = 1.0f;
        for (int i = 0; i < n; ++i) {
            const float p = perlin(px * scale, py * scale, pz * scale, 1.0f, a.seed ^ wmul(i + 38, 27389482));
            acc = acc * fm(-sat(fm(0.5f, p, 0.5f)), amp, 1.0f);
            if (acc < a.threshold) return 0.0f;
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
        }
        return acc;
    case BLZ_NOISE_REPEATER_PERLIN_ABS:                                      // 659-673
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            acc = fm(std::fabs(perlin(px * scale, py * scale, pz * scale, 1.0f, a.seed)), amp, acc);
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
        }
        return to_signed(acc);
    case BLZ_NOISE_REPEATER_SIMPLEX: {                                       // 676-690
        int seed = a.seed;
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            acc = fm(simplex(px, py, pz, scale, seed) * amp, 0.35f, acc);
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
            seed = seed ^ wmul(i + 672381, 200394);
        }
        return acc;
    }
    case BLZ_NOISE_REPEATER_SIMPLEX_ABS: {                                   // 693-707
        int seed = a.seed;
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            acc = fm(std::fabs(simplex(px, py, pz, scale, seed)) * amp, 0.35f, acc);
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
            seed = seed ^ wmul(i + 198273, 928374);
        }
        return to_signed(acc);
    }
    case BLZ_NOISE_REPEATER_SIMPLEX_BOUNDED:                                 // 710-731
        acc = 1.0f;
        for (int i = 0; i < n; ++i) {
            const float sn = simplex(fm(px, scale, 32240.7922f), fm(py, scale, 835622.882f), fm(pz, scale, 824.371968f),
                                     1.0f, a.seed);
            acc = acc - sat(fm(sn, 0.3f, 0.5f)) * amp;
            if (acc < a.threshold) return 0.0f;
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
        }
        return acc;
    case BLZ_NOISE_REPEATER:
        return repeater(px, py, pz, a.scale, a.seed, n, a.lacunarity, a.decay, a.basis);
    case BLZ_NOISE_FRACTAL_SIMPLEX: {                                        // 782-801
        const float rdu = 1.0f / a.du;
        acc = 0.0f;
        for (int i = 0; i < n; ++i) {
            const float sn = simplex(fm(px, scale, 617.437379f), fm(py, scale, 196410.219f), fm(pz, scale, 321280.627f),
                                     1.0f, wmul(a.seed, i + 1));
            acc = fm(sn, amp, acc);
            scale = scale * a.lacunarity;
            amp = amp * a.decay;
            if (scale > rdu) break;
        }
        return acc;
    }
    case BLZ_NOISE_TURBULENCE:
        return turbulence(px, py, pz, a.scale, a.scale_out, a.seed, a.strength, a.basis, a.basis_out);
    case BLZ_NOISE_REPEATER_TURBULENCE: {                                    // 867-874
        float qx = px, qy = py, qz = pz;
        qx = fm(repeater(qx, qy, qz, a.scale, a.seed ^ 0x41728394, n, 2.0f, 0.5f, a.basis), a.strength, qx);
        qy = fm(repeater(qx, qy, qz, a.scale, a.seed ^ 0x72837263, n, 2.0f, 0.5f, a.basis), a.strength, qy);
        qz = fm(repeater(qx, qy, qz, a.scale, a.seed ^ 0x26837363, n, 2.0f, 0.5f, a.basis), a.strength, qz);
        return repeater(qx, qy, qz, a.scale_out, a.seed ^ 0x3f821dab, n, 2.0f, 0.5f, a.basis_out);
    }
    default:
        return 0.0f;
    }
}

} // namespace nz

extern "C" {

// Test hook: see next_pattern (at most 16 patterns; count 0 restores the
// standalone form).
int orc_noise_set_lattice_patterns(const unsigned long long *patterns, int count) {
    if (count < 0 || count > 16 || (count > 0 && !patterns)) return -2;
    for (int i = 0; i < count; ++i) nz::g_patterns[i] = patterns[i];
    nz::g_npatterns = count;
    return 0;
}

// blz_noise restated: a->func at n positions (host arrays).
int orc_noise(const blz_noise_args *a, const float *pos3, long long n, float *out) {
    if (!a || (n > 0 && (!pos3 || !out))) return -2;
#pragma omp parallel for schedule(dynamic, 64)
    for (long long t = 0; t < n; ++t) {
        nz::t_blend = 0;
        out[t] = nz::eval(*a, pos3[3 * t], pos3[3 * t + 1], pos3[3 * t + 2]);
    }
    return 0;
}

} // extern "C"
