// blaze_oracle.cpp — CPU oracle of Blaze's per-frame fluid step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by the
// tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, never
// by the product path (libblaze_b200.so has no CPU fallback).
//
// It restates, stage by stage, the algorithm of the Blaze reference
// (asiroisvigneux/Blaze; paths below are inside that project) in plain C++,
// templated on the arithmetic type: the FP64 instantiation is the yardstick for the
// FP32 CUDA kernels, the FP32 one mirrors the reference's own arithmetic for
// comparisons against the reference's CUDA build.  Float constants of the
// reference (1.001f, 1e-20f, 1e-5) keep their float values in both.
//
// Gradient noise is always evaluated in FP32 with the reference's exact
// operation order (cuda_noise.cuh:120-124): its lattice hash takes the bits of
// a rounded float, so a wider type would decorrelate the noise entirely.
//
// Parity pins: tests/golden/ holds outputs of the reference's own CUDA build
// (compiled from its sources by oracle/Makefile's `ref` target, run on a
// B200) on seeded inputs; tests/test_oracle_golden.py checks this file
// against them.  The reference itself ships no tests or fixtures.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/blaze_b200.h"

namespace orc {

// ---------------------------------------------------------------------------
// Gradient noise (third-party cudaNoise by H. Lehtinen, vendored in the
// reference as thirdparty/cuda-noise/cuda_noise.cuh, no version recorded).
// ---------------------------------------------------------------------------

// Integer hash, cuda_noise.cuh:46-57 (the published 6-step 32-bit mix).
static inline uint32_t lattice_hash(uint32_t s) {
    s = (s + 0x7ed55d16u) + (s << 12);
    s = (s ^ 0xc761c23cu) ^ (s >> 19);
    s = (s + 0x165667b1u) + (s << 5);
    s = (s + 0xd3a2646cu) ^ (s << 9);
    s = (s + 0xfd7046c5u) + (s << 3);
    s = (s ^ 0xb55a4f09u) ^ (s >> 16);
    return s;
}

// float -> unsigned with the GPU's cvt.rzi.u32.f32 behaviour: truncate toward
// zero, saturate to [0, 2^32-1], NaN -> 0.
static inline uint32_t f2u_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}

// Lattice seed, cuda_noise.cuh:120-124: x*1723 + y*93241 + z*149812 + 3824 +
// seed in float.  The reference's CUDA build contracts the sum into
// fma(z, 149812, fma(x, 1723, y*93241)), then adds 3824 and seed; once a
// product exceeds 2^24 the contraction changes the rounded value and with it
// the hashed lattice gradient, so the oracle forms it the same way.  Pinned
// bit for bit against the reference build's own noise (tests/golden/perlin.npz,
// tests/golden/noise.npz).
static inline uint32_t lattice_seed(float x, float y, float z, float seed) {
    float acc = std::fma(x, 1723.0f, y * 93241.0f);
    acc = std::fma(z, 149812.0f, acc);
    acc = acc + 3824.0f;
    acc = acc + seed;
    return lattice_hash(f2u_sat(acc));
}

// Gradient selection, cuda_noise.cuh:179-201.
static inline float lattice_grad(int h, float x, float y, float z) {
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

// fade and lerp (cuda_noise.cuh:204-207, 167-170) as the reference's CUDA
// build evaluates them: a multiply feeding an add in the same expression is
// one fused multiply-add (the left product when both operands are products).
static inline float fade5(float t) {
    return t * t * t * std::fma(t, std::fma(t, 6.0f, -15.0f), 10.0f);
}
static inline float lerpf(float a, float b, float r) {
    return std::fma(a, 1.0f - r, b * r);
}

// perlinNoise, cuda_noise.cuh:570-615.
float perlin(float px, float py, float pz, float scale, int seed) {
    const float fs = (float)seed;
    px *= scale; py *= scale; pz *= scale;
    const float ix = std::floor(px), iy = std::floor(py), iz = std::floor(pz);
    px -= ix; py -= iy; pz -= iz;
    const float u = fade5(px), v = fade5(py), w = fade5(pz);
    const float i000 = lattice_grad((int)lattice_seed(ix, iy, iz, fs), px, py, pz);
    const float i100 = lattice_grad((int)lattice_seed(ix + 1.0f, iy, iz, fs), px - 1.0f, py, pz);
    const float i010 = lattice_grad((int)lattice_seed(ix, iy + 1.0f, iz, fs), px, py - 1.0f, pz);
    const float i110 = lattice_grad((int)lattice_seed(ix + 1.0f, iy + 1.0f, iz, fs), px - 1.0f, py - 1.0f, pz);
    const float i001 = lattice_grad((int)lattice_seed(ix, iy, iz + 1.0f, fs), px, py, pz - 1.0f);
    const float i101 = lattice_grad((int)lattice_seed(ix + 1.0f, iy, iz + 1.0f, fs), px - 1.0f, py, pz - 1.0f);
    const float i011 = lattice_grad((int)lattice_seed(ix, iy + 1.0f, iz + 1.0f, fs), px, py - 1.0f, pz - 1.0f);
    const float i111 = lattice_grad((int)lattice_seed(ix + 1.0f, iy + 1.0f, iz + 1.0f, fs), px - 1.0f, py - 1.0f, pz - 1.0f);
    const float x00 = lerpf(i000, i100, u), x10 = lerpf(i010, i110, u);
    const float x01 = lerpf(i001, i101, u), x11 = lerpf(i011, i111, u);
    const float y0 = lerpf(x00, x10, v), y1 = lerpf(x01, x11, v);
    return lerpf(y0, y1, w);
}

// ---------------------------------------------------------------------------
// MAC grid geometry (Grid.h:40-337; field setup FluidSolver.cu:36-43).
// ---------------------------------------------------------------------------
template <class R> struct Field {
    R *a;
    int w, h, d;
    R ox, oy, oz;
    bool flip;                                  // V: y is flipped (Q1)
    R &at(int i, int j, int k) const {
        return a[(size_t)i + (size_t)w * ((size_t)j + (size_t)h * (size_t)k)];
    }
    size_t size() const { return (size_t)w * h * d; }
};

template <class R> struct Geo {
    int W, H, D;
    R dx, dt;
    R dmin[3], dsize[3];
    const blz_params *P;
    explicit Geo(const blz_params *p) : W(p->width), H(p->height), D(p->depth),
        dx((R)p->dx), dt((R)p->dt), P(p) {
        for (int c = 0; c < 3; ++c) {
            dmin[c] = (R)p->domain_min[c];
            // mDomSize = domainMax - domainMin, formed in float (Grid.h:240)
            dsize[c] = (R)(p->domain_max[c] - p->domain_min[c]);
        }
    }
    Field<R> T(R *a) const { return {a, W, H, D, R(0.5), R(0.5), R(0.5), false}; }
    Field<R> U(R *a) const { return {a, W + 1, H, D, R(0), R(0.5), R(0.5), false}; }
    Field<R> V(R *a) const { return {a, W, H + 1, D, R(0.5), R(0), R(0.5), true}; }
    Field<R> Wf(R *a) const { return {a, W, H, D + 1, R(0.5), R(0.5), R(0), false}; }
    size_t nT() const { return (size_t)W * H * D; }
    size_t nU() const { return (size_t)(W + 1) * H * D; }
    size_t nV() const { return (size_t)W * (H + 1) * D; }
    size_t nW() const { return (size_t)W * H * (D + 1); }
};

// Upper clamp of a sample coordinate: n - 1.001f evaluated in float (Grid.h:96-98).
template <class R> static inline R clamp_hi(int n) { return (R)((float)n - 1.001f); }

template <class R> static inline R clampc(R g, int n) {
    return std::fmax(std::fmin(g, clamp_hi<R>(n)), R(0));
}

// Trilinear sample at an object-space position (Grid.h:94-108).
template <class R>
static R trilinear(const Field<R> &f, R dx, R px, R py, R pz) {
    const R gX = clampc(px / dx - f.ox, f.w);
    const R gY = clampc(py / dx - f.oy, f.h);
    const R gZ = clampc(pz / dx - f.oz, f.d);
    const int x0 = (int)gX, y0 = (int)gY, z0 = (int)gZ;
    const R fx = gX - x0, fy = gY - y0, fz = gZ - z0;
    return (R(1) - fz) * ((R(1) - fy) * (f.at(x0, y0, z0) * (R(1) - fx) + f.at(x0 + 1, y0, z0) * fx)
                          + fy * (f.at(x0, y0 + 1, z0) * (R(1) - fx) + f.at(x0 + 1, y0 + 1, z0) * fx))
         + fz * ((R(1) - fy) * (f.at(x0, y0, z0 + 1) * (R(1) - fx) + f.at(x0 + 1, y0, z0 + 1) * fx)
                 + fy * (f.at(x0, y0 + 1, z0 + 1) * (R(1) - fx) + f.at(x0 + 1, y0 + 1, z0 + 1) * fx));
}

// Four-point Lagrange cubic on nodes -1, 0, 1, 2 (Grid.h:148-163).
template <class R> static inline R cerp(R q0, R q1, R q2, R q3, R s) {
    return (-R(1) / R(3) * s + R(0.5) * s * s - R(1) / R(6) * s * s * s) * q0
         + (R(1) - s * s + R(0.5) * (s * s * s - s)) * q1
         + (s + R(0.5) * (s * s - s * s * s)) * q2
         + (R(1) / R(6) * (s * s * s - s)) * q3;
}

// Separable tricubic, x then y then z; clamp == true clamps every 1-D stage
// at zero (cerpc).  Stencil indices clamp at the field edges (Grid.h:165-222).
template <class R>
static R tricubic(const Field<R> &f, R dx, R px, R py, R pz, bool clamp) {
    const R gX = clampc(px / dx - f.ox, f.w);
    const R gY = clampc(py / dx - f.oy, f.h);
    const R gZ = clampc(pz / dx - f.oz, f.d);
    const int i1 = (int)gX, j1 = (int)gY, k1 = (int)gZ;
    const int is[4] = {std::max(i1 - 1, 0), i1, i1 + 1, std::min(i1 + 2, f.w - 1)};
    const int js[4] = {std::max(j1 - 1, 0), j1, j1 + 1, std::min(j1 + 2, f.h - 1)};
    const int ks[4] = {std::max(k1 - 1, 0), k1, k1 + 1, std::min(k1 + 2, f.d - 1)};
    const R sx = gX - i1, sy = gY - j1, sz = gZ - k1;
    auto c = [clamp](R a, R b, R cc, R d, R s) {
        R v = cerp(a, b, cc, d, s);
        return clamp ? std::fmax(v, R(0)) : v;
    };
    R zs[4];
    for (int kk = 0; kk < 4; ++kk) {
        R ys[4];
        for (int jj = 0; jj < 4; ++jj)
            ys[jj] = c(f.at(is[0], js[jj], ks[kk]), f.at(is[1], js[jj], ks[kk]),
                       f.at(is[2], js[jj], ks[kk]), f.at(is[3], js[jj], ks[kk]), sx);
        zs[kk] = c(ys[0], ys[1], ys[2], ys[3], sy);
    }
    return c(zs[0], zs[1], zs[2], zs[3], sz);
}

template <class R> struct V3 { R x, y, z; };
template <class R> static inline R len3(R x, R y, R z) { return std::sqrt(x * x + y * y + z * z); }

template <class R>
static inline V3<R> vel_at(const Geo<R> &g, const Field<R> &U, const Field<R> &V,
                           const Field<R> &W, R px, R py, R pz) {
    return {trilinear(U, g.dx, px, py, pz), trilinear(V, g.dx, px, py, pz),
            trilinear(W, g.dx, px, py, pz)};
}

// ---------------------------------------------------------------------------
// Sourcing (FluidSolver.cu:57-116, Grid.h:309-335).
// ---------------------------------------------------------------------------
template <class R> static inline R cubic_pulse(R x, R w) {   // Grid.h:309-313
    if (x > w) return R(0);
    x /= w;
    return R(1) - x * x * (R(3) - R(2) * x);
}

static inline int trunc_int(double v) {   // C cast with a guard against overflow
    v = std::fmin(std::fmax(v, -1073741824.0), 1073741824.0);
    return (int)v;
}

template <class R>
static void sphere_to_grid(const Geo<R> &g, const Field<R> &f, R px, R py, R pz, R pscale, R value) {
    const R radius = pscale / R(2);
    const R dx = g.dx;
    auto xw = [&](R x) { return x - g.dmin[0]; };
    auto yw = [&](R y) { return g.dsize[1] - (y - g.dmin[1]); };
    auto zw = [&](R z) { return z - g.dmin[2]; };
    const int imin = std::max(trunc_int(xw(px - radius) / dx - f.ox), 0);
    const int imax = std::min(trunc_int(xw(px + radius) / dx - f.ox) + 1, f.w);
    const int jmin = std::max(trunc_int(yw(py + radius) / dx - f.oy), 0);
    const int jmax = std::min(trunc_int(yw(py - radius) / dx - f.oy) + 1, f.h);
    const int kmin = std::max(trunc_int(zw(pz - radius) / dx - f.oz), 0);
    const int kmax = std::min(trunc_int(zw(pz + radius) / dx - f.oz) + 1, f.d);
    const R ox = xw(px), oy = yw(py), oz = zw(pz);
    for (int i = imin; i < imax; ++i)
        for (int j = jmin; j < jmax; ++j)
            for (int k = kmin; k < kmax; ++k) {
                const R ddx = ox - (R(i) + f.ox) * dx;
                const R ddy = oy - (R(j) + f.oy) * dx;
                const R ddz = oz - (R(k) + f.oz) * dx;
                const R mask = cubic_pulse(len3(ddx, ddy, ddz), radius);
                if (mask > R(0)) f.at(i, j, k) += f.flip ? -value * mask : value * mask;
            }
}

// Dn (may be null): the density scalar of target mode (no counterpart in the
// reference), on the T grid, splatted like T with each particle's density
// dens[p] (null: 1 per particle) under the same |value| > 1e-5 rules.
template <class R>
void add_source(const blz_params *P, const float *rec, int n, R *T, R *U, R *V, R *W, const float *dens = nullptr,
                R *Dn = nullptr) {
    Geo<R> g(P);
    std::vector<R> bT(g.nT(), R(0)), bU(g.nU(), R(0)), bV(g.nV(), R(0)), bW(g.nW(), R(0));
    std::vector<R> bD(Dn ? g.nT() : 0, R(0));
    Field<R> fT = g.T(bT.data()), fU = g.U(bU.data()), fV = g.V(bV.data()), fW = g.Wf(bW.data());
    Field<R> fD = g.T(Dn ? bD.data() : bT.data());
    const R half_dx = (R)(P->dx / 2.0f);
    for (int p = 0; p < n; ++p) {
        const float *r = rec + 8 * (size_t)p;
        const R px = r[0], py = r[1], pz = r[2], ps = r[6];
        if (!(ps > half_dx)) continue;
        if (std::fabs(r[7]) > 1e-5) sphere_to_grid(g, fT, px, py, pz, ps, (R)r[7]);
        if (std::fabs(r[3]) > 1e-5) sphere_to_grid(g, fU, px, py, pz, ps, (R)r[3]);
        if (std::fabs(r[4]) > 1e-5) sphere_to_grid(g, fV, px, py, pz, ps, (R)r[4]);
        if (std::fabs(r[5]) > 1e-5) sphere_to_grid(g, fW, px, py, pz, ps, (R)r[5]);
        if (Dn) {
            const float d = dens ? dens[p] : 1.0f;
            if (std::fabs(d) > 1e-5) sphere_to_grid(g, fD, px, py, pz, ps, (R)d);
        }
    }
    auto apply = [](R *front, const std::vector<R> &back) {
        for (size_t i = 0; i < back.size(); ++i)
            if (std::fabs(back[i]) > R(1e-5)) front[i] = back[i];
    };
    apply(T, bT); apply(U, bU); apply(V, bV); apply(W, bW);
    if (Dn) apply(Dn, bD);
}

// ---------------------------------------------------------------------------
// Forces (FluidSolver.cu:118-390), applied in step() order (858-936).
// ---------------------------------------------------------------------------
template <class R> static void scale_all(R *a, size_t n, R s) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) a[i] *= s;
}

// computeVorticity, FluidSolver.cu:174-201: centred differences of trilinear
// samples taken at the six neighbouring cell centres.
template <class R>
static V3<R> vorticity_at(const Geo<R> &g, const Field<R> &U, const Field<R> &V,
                          const Field<R> &W, int i, int j, int k) {
    const R dx = g.dx;
    auto c = [dx](int n) { return (R(n) + R(0.5)) * dx; };
    const R x0 = c(i - 1), x1 = c(i), x2 = c(i + 1);
    const R y0 = c(j - 1), y1 = c(j), y2 = c(j + 1);
    const R z0 = c(k - 1), z1 = c(k), z2 = c(k + 1);
    const R w_121 = trilinear(W, dx, x1, y2, z1), w_101 = trilinear(W, dx, x1, y0, z1);
    const R v_112 = trilinear(V, dx, x1, y1, z2), v_110 = trilinear(V, dx, x1, y1, z0);
    const R u_112 = trilinear(U, dx, x1, y1, z2), u_110 = trilinear(U, dx, x1, y1, z0);
    const R w_211 = trilinear(W, dx, x2, y1, z1), w_011 = trilinear(W, dx, x0, y1, z1);
    const R v_211 = trilinear(V, dx, x2, y1, z1), v_011 = trilinear(V, dx, x0, y1, z1);
    const R u_121 = trilinear(U, dx, x1, y2, z1), u_101 = trilinear(U, dx, x1, y0, z1);
    const R s = R(2) * dx;
    return {(w_121 - w_101 - (v_112 - v_110)) / s,
            (u_112 - u_110 - (w_211 - w_011)) / s,
            (v_211 - v_011 - (u_121 - u_101)) / s};
}

// vorticity_confinement_kernel, FluidSolver.cu:203-248.  Force per cell for
// 2 <= i <= W-3 (same for j, k), split half to each adjacent face.  The
// normalised N of the reference (line 226) is never used; the force takes the
// unnormalised gradient of |omega| (line 240).  Gather form: each face adds
// the contributions of its lower then its upper cell.
template <class R>
static void vorticity(const Geo<R> &g, R *U, R *V, R *W, R conf) {
    const int Wd = g.W, Hd = g.H, Dd = g.D;
    Field<R> fU = g.U(U), fV = g.V(V), fW = g.Wf(W);
    const R dx = g.dx, dt = g.dt;
    const R tiny = (R)(1e-20f * (1.0f / ((float)g.P->dx * (float)g.P->dt)));
    std::vector<R> fx(g.nT(), R(0)), fy(g.nT(), R(0)), fz(g.nT(), R(0));
    std::vector<char> act(g.nT(), 0);
    auto id = [&](int i, int j, int k) { return (size_t)i + (size_t)Wd * ((size_t)j + (size_t)Hd * k); };
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= Dd - 3; ++k)
        for (int j = 2; j <= Hd - 3; ++j)
            for (int i = 2; i <= Wd - 3; ++i) {
                V3<R> om = vorticity_at(g, fU, fV, fW, i, j, k);
                V3<R> o211 = vorticity_at(g, fU, fV, fW, i + 1, j, k);
                V3<R> o011 = vorticity_at(g, fU, fV, fW, i - 1, j, k);
                V3<R> o121 = vorticity_at(g, fU, fV, fW, i, j + 1, k);
                V3<R> o101 = vorticity_at(g, fU, fV, fW, i, j - 1, k);
                V3<R> o112 = vorticity_at(g, fU, fV, fW, i, j, k + 1);
                V3<R> o110 = vorticity_at(g, fU, fV, fW, i, j, k - 1);
                const R s = R(2) * dx;
                const R gx = (len3(o211.x, o211.y, o211.z) - len3(o011.x, o011.y, o011.z)) / s;
                const R gy = (len3(o121.x, o121.y, o121.z) - len3(o101.x, o101.y, o101.z)) / s;
                const R gz = (len3(o112.x, o112.y, o112.z) - len3(o110.x, o110.y, o110.z)) / s;
                const R px = (R(i) + R(0.5)) * dx, py = (R(j) + R(0.5)) * dx, pz = (R(k) + R(0.5)) * dx;
                V3<R> vel = vel_at(g, fU, fV, fW, px, py, pz);
                const R speed = len3(vel.x, vel.y, vel.z);
                const R onorm = len3(om.x, om.y, om.z) + tiny;
                if (onorm > speed) { om.x = speed * om.x / onorm; om.y = speed * om.y / onorm; om.z = speed * om.z / onorm; }
                const R cx = gy * om.z - gz * om.y;
                const R cy = gz * om.x - gx * om.z;
                const R cz = gx * om.y - gy * om.x;
                const R sc = conf * dx;
                const size_t c = id(i, j, k);
                fx[c] = R(0.5) * dt * (sc * cx);
                fy[c] = R(0.5) * dt * (sc * cy);
                fz[c] = R(0.5) * dt * (sc * cz);
                act[c] = 1;
            }
    // U faces (i, j, k): lower cell i-1, upper cell i.
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i <= Wd; ++i) {
                R &u = fU.at(i, j, k);
                if (i - 1 >= 0 && act[id(i - 1, j, k)]) u += fx[id(i - 1, j, k)];
                if (i < Wd && act[id(i, j, k)]) u += fx[id(i, j, k)];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j <= Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                R &v = fV.at(i, j, k);
                if (j - 1 >= 0 && act[id(i, j - 1, k)]) v += fy[id(i, j - 1, k)];
                if (j < Hd && act[id(i, j, k)]) v += fy[id(i, j, k)];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                R &w = fW.at(i, j, k);
                if (k - 1 >= 0 && act[id(i, j, k - 1)]) w += fz[id(i, j, k - 1)];
                if (k < Dd && act[id(i, j, k)]) w += fz[id(i, j, k)];
            }
}

// add_buoyancy_kernel, FluidSolver.cu:142-156: V += dt*beta*T_lin*g at V faces.
// With the density scalar of target mode (Dn, no reference counterpart):
// V += dt*(beta*T_lin - alpha*rho_lin)*g, the smoke's weight pulling down.
template <class R>
static void buoyancy(const Geo<R> &g, const R *T, R *V, R beta, R grav, const R *Dn = nullptr, R alpha = R(0)) {
    Field<R> fT = g.T(const_cast<R *>(T)), fV = g.V(V);
    Field<R> fD = g.T(const_cast<R *>(Dn ? Dn : T));
    const R dx = g.dx, dt = g.dt;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g.D; ++k)
        for (int j = 0; j <= g.H; ++j)
            for (int i = 0; i < g.W; ++i) {
                const R px = (R(i) + R(0.5)) * dx, py = R(j) * dx, pz = (R(k) + R(0.5)) * dx;
                const R temp = trilinear(fT, dx, px, py, pz);
                if (Dn) {
                    const R rho = trilinear(fD, dx, px, py, pz);
                    fV.at(i, j, k) += dt * ((beta * temp - alpha * rho) * grav);
                } else {
                    fV.at(i, j, k) += dt * (beta * temp * grav);
                }
            }
}

// add_wind_kernel, FluidSolver.cu:337-390: relax U, V, W toward the wind in
// two-voxel slabs at both ends of the wind axis; noise from three seeds.
template <class R>
static void wind(const Geo<R> &g, R *U, R *V, R *W, float time) {
    const blz_params *P = g.P;
    Field<R> fU = g.U(U), fV = g.V(V), fW = g.Wf(W);
    const int Wd = g.W, Hd = g.H, Dd = g.D;
    const float dxf = P->dx;
    const float freq = 1.0f / P->wind_turb_scale;
    const float dsx = P->domain_max[0] - P->domain_min[0];
    const float dsy = P->domain_max[1] - P->domain_min[1];
    const float dsz = P->domain_max[2] - P->domain_min[2];
    const float avg_dom = (dsx + dsy + dsz) / 3.0f;
    const float offset = std::fmod(time * avg_dom * P->wind_speed, 25000.0f);
    const R dt = g.dt, amp = (R)P->wind_amp;
    const bool alongX = P->wind_dir <= 1;
    const R dir = (P->wind_dir == 0 || P->wind_dir == 2) ? R(1) : R(-1);
    const int pad = 2;
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= Dd; ++k)
        for (int j = 0; j <= Hd; ++j)
            for (int i = 0; i <= Wd; ++i) {
                if (alongX) { if (i >= pad && i < (Wd + 1) - pad) continue; }
                else        { if (k >= pad && k < (Dd + 1) - pad) continue; }
                const float x = (float)i * dxf, y = (float)j * dxf, z = (float)k * dxf + offset;
                const R nU = (R)(P->wind_turb_amp * perlin(x, y, z, freq, 123));
                const R nV = (R)(P->wind_turb_amp * perlin(x, y, z, freq, 456));
                const R nW = (R)(P->wind_turb_amp * perlin(x, y, z, freq, 789));
                const R one_m = R(1) - dt;
                if (j < Hd && k < Dd) {
                    R &u = fU.at(i, j, k);
                    u = u * one_m + (amp * ((alongX ? dir : R(0)) + nU)) * dt;
                }
                if (i < Wd && k < Dd) {
                    R &v = fV.at(i, j, k);
                    v = v * one_m + (amp * nV) * dt;
                }
                if (i < Wd && j < Hd) {
                    R &w = fW.at(i, j, k);
                    w = w * one_m + (amp * ((alongX ? R(0) : dir) + nW)) * dt;
                }
            }
}

template <class R> static inline R fit01(R v, R a, R b, R lo, R hi) {   // FluidSolver.cu:250-252
    return std::fmax(std::fmin((v - a) / (b - a), R(1)), R(0)) * (hi - lo) + lo;
}

// compute_turbulence_kernel + add_curl_noise_kernel, FluidSolver.cu:271-335.
// The noise field is masked Perlin noise on cell indices; the "curl" uses the
// reference's differences verbatim, including V in dudx and dwdz (276, 278).
template <class R>
static void turbulence(const Geo<R> &g, const R *T, R *U, R *V, R *W, float time) {
    const blz_params *P = g.P;
    const int Wd = g.W, Hd = g.H, Dd = g.D;
    Field<R> fT = g.T(const_cast<R *>(T)), fU = g.U(U), fV = g.V(V), fW = g.Wf(W);
    std::vector<R> nU(g.nU()), nV(g.nV()), nW(g.nW());
    Field<R> gU = g.U(nU.data()), gV = g.V(nV.data()), gW = g.Wf(nW.data());
    const float freq = 1.0f / P->turbulence_scale;
    const float avg_grid = (float)(Wd + Hd + Dd) / 3.0f;
    const float offset = std::fmod(time * avg_grid, 25000.0f);
    const R amp = (R)P->turbulence_amp, dx = g.dx;
    const R tr0 = P->turb_mask_temp_ramp[0], tr1 = P->turb_mask_temp_ramp[1];
    const R vr0 = P->turb_mask_vel_ramp[0], vr1 = P->turb_mask_vel_ramp[1];
    auto mask = [&](R px, R py, R pz) {
        const R tm = fit01(trilinear(fT, dx, px, py, pz), tr0, tr1, R(1), R(0));
        V3<R> v = vel_at(g, fU, fV, fW, px, py, pz);
        const R vm = fit01(len3(v.x, v.y, v.z), vr0, vr1, R(0), R(1));
        return tm * vm;
    };
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= Dd; ++k)
        for (int j = 0; j <= Hd; ++j)
            for (int i = 0; i <= Wd; ++i) {
                if (j < Hd && k < Dd) {
                    const R m = mask(R(i) * dx, (R(j) + R(0.5)) * dx, (R(k) + R(0.5)) * dx);
                    gU.at(i, j, k) = m * amp * (R)perlin((float)i + offset, (float)j, (float)k, freq, 123);
                }
                if (i < Wd && k < Dd) {
                    const R m = mask((R(i) + R(0.5)) * dx, R(j) * dx, (R(k) + R(0.5)) * dx);
                    gV.at(i, j, k) = m * amp * (R)perlin((float)i, (float)j + offset, (float)k, freq, 123);
                }
                if (i < Wd && j < Hd) {
                    const R m = mask((R(i) + R(0.5)) * dx, (R(j) + R(0.5)) * dx, R(k) * dx);
                    gW.at(i, j, k) = m * amp * (R)perlin((float)i, (float)j, (float)k + offset, freq, 123);
                }
            }
    const R dt = g.dt;
    const R tiny = (R)(1e-20f * (1.0f / ((float)P->dx * (float)P->dt)));
    std::vector<R> cx(g.nT()), cy(g.nT()), cz(g.nT());
    auto id = [&](int i, int j, int k) { return (size_t)i + (size_t)Wd * ((size_t)j + (size_t)Hd * k); };
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                const R nv = gV.at(i, j, k);
                const R dudx = (gU.at(i + 1, j, k) - nv) / dx;
                const R dvdy = (gV.at(i, j + 1, k) - nv) / dx;
                const R dwdz = (gW.at(i, j, k + 1) - nv) / dx;
                R c0 = dvdy - dwdz, c1 = dwdz - dudx, c2 = dudx - dvdy;
                const R ax = (gU.at(i, j, k) + gU.at(i + 1, j, k)) / R(2);
                const R ay = (gV.at(i, j, k) + gV.at(i, j + 1, k)) / R(2);
                const R az = (gW.at(i, j, k) + gW.at(i, j, k + 1)) / R(2);
                const R avg_speed = len3(ax, ay, az);
                const R den = len3(c0, c1, c2) + tiny;
                c0 = avg_speed * c0 / den; c1 = avg_speed * c1 / den; c2 = avg_speed * c2 / den;
                const size_t c = id(i, j, k);
                cx[c] = R(0.5) * dt * c0; cy[c] = R(0.5) * dt * c1; cz[c] = R(0.5) * dt * c2;
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i <= Wd; ++i) {
                R &u = fU.at(i, j, k);
                if (i - 1 >= 0) u += cx[id(i - 1, j, k)];
                if (i < Wd) u += cx[id(i, j, k)];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j <= Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                R &v = fV.at(i, j, k);
                if (j - 1 >= 0) v += cy[id(i, j - 1, k)];
                if (j < Hd) v += cy[id(i, j, k)];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                R &w = fW.at(i, j, k);
                if (k - 1 >= 0) w += cz[id(i, j, k - 1)];
                if (k < Dd) w += cz[id(i, j, k)];
            }
}

template <class R>
void forces(const blz_params *P, float time, R *T, R *U, R *V, R *W, const R *Dn = nullptr) {
    Geo<R> g(P);
    if (std::fabs(P->cooling_rate) > 0.0f) scale_all(T, g.nT(), R(1) - g.dt * (R)P->cooling_rate);
    if (P->drag > 0.0f) {
        const R s = R(1) - g.dt * (R)P->drag;
        scale_all(U, g.nU(), s); scale_all(V, g.nV(), s); scale_all(W, g.nW(), s);
    }
    if (std::fabs(P->vorticity_conf) > 0.0f) vorticity(g, U, V, W, (R)P->vorticity_conf);
    if (Dn && (std::fabs(P->buoyancy) > 0.0f || std::fabs(P->buoyancy_alpha) > 0.0f))
        buoyancy(g, T, V, (R)P->buoyancy, (R)P->gravity, Dn, (R)P->buoyancy_alpha);
    else if (std::fabs(P->buoyancy) > 0.0f)
        buoyancy(g, T, V, (R)P->buoyancy, (R)P->gravity);
    if (P->wind_amp > 0.0f) wind(g, U, V, W, time);
    if (P->turbulence_amp > 0.0f) turbulence(g, T, U, V, W, time);
}

// ---------------------------------------------------------------------------
// Projection (FluidSolver.cu:475-669, 823-856).
// ---------------------------------------------------------------------------
// Which domain faces are open.  j == 0 is yMax because y is flipped (Q1).
struct Open { bool xlo, xhi, ylo, yhi, zlo, zhi; };
static inline Open open_faces(const blz_params *P) {
    return {!P->closed_bounds[0], !P->closed_bounds[1], !P->closed_bounds[3],
            !P->closed_bounds[2], !P->closed_bounds[4], !P->closed_bounds[5]};
}

// compute_divergence_kernel, FluidSolver.cu:475-515.
template <class R>
void divergence(const blz_params *P, const R *U, const R *V, const R *W, R *rhs) {
    Geo<R> g(P);
    Field<R> fU = g.U(const_cast<R *>(U)), fV = g.V(const_cast<R *>(V)), fW = g.Wf(const_cast<R *>(W));
    const R s = R(1) / g.dx;
    const Open o = open_faces(P);
    const int Wd = g.W, Hd = g.H, Dd = g.D;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                R r = -s * (fU.at(i + 1, j, k) - fU.at(i, j, k) + fV.at(i, j + 1, k) - fV.at(i, j, k)
                            + fW.at(i, j, k + 1) - fW.at(i, j, k));
                if (i == 0) { if (!o.xlo) r -= s * fU.at(i, j, k); }
                else if (i == Wd - 1) { if (!o.xhi) r += s * fU.at(i + 1, j, k); }
                if (j == 0) { if (!o.ylo) r -= s * fV.at(i, j, k); }
                else if (j == Hd - 1) { if (!o.yhi) r += s * fV.at(i, j + 1, k); }
                if (k == 0) { if (!o.zlo) r -= s * fW.at(i, j, k); }
                else if (k == Dd - 1) { if (!o.zhi) r += s * fW.at(i, j, k + 1); }
                rhs[(size_t)i + (size_t)Wd * ((size_t)j + (size_t)Hd * k)] = r;
            }
}

// One Gauss-Seidel update of cell (i,j,k): p = (scale*rhs + sum p_nb) / n_nb
// (FluidSolver.cu:532-561).  REF_COMPAT counts in-domain neighbours only;
// FREE_SURFACE also counts a p = 0 ghost across each open face.
template <class R>
static inline R gs_cell(const Geo<R> &g, const Open &o, bool dirichlet, const R *rhs, const R *p,
                        R scale, int i, int j, int k) {
    const size_t sx = 1, sy = (size_t)g.W, sz = (size_t)g.W * g.H;
    const size_t c = (size_t)i + sy * j + sz * k;
    R num = scale * rhs[c];
    R den = R(0);
    if (i > 0) { num += p[c - sx]; den += R(1); } else if (dirichlet && o.xlo) den += R(1);
    if (i < g.W - 1) { num += p[c + sx]; den += R(1); } else if (dirichlet && o.xhi) den += R(1);
    if (j > 0) { num += p[c - sy]; den += R(1); } else if (dirichlet && o.ylo) den += R(1);
    if (j < g.H - 1) { num += p[c + sy]; den += R(1); } else if (dirichlet && o.yhi) den += R(1);
    if (k > 0) { num += p[c - sz]; den += R(1); } else if (dirichlet && o.zlo) den += R(1);
    if (k < g.D - 1) { num += p[c + sz]; den += R(1); } else if (dirichlet && o.zhi) den += R(1);
    return num / den;
}

template <class R>
static void gs_sweeps(const Geo<R> &g, const blz_params *P, const R *rhs, R *p, int n) {
    const Open o = open_faces(P);
    const bool dir = P->bc_mode == BLZ_BC_FREE_SURFACE;
    const R scale = (R)P->density * g.dx * g.dx / g.dt;
    const int Wd = g.W, Hd = g.H, Dd = g.D;
    for (int it = 0; it < n; ++it) {
        if (P->gs_order == BLZ_GS_PLANE) {
            // Race-free form of gs_solve_kernel (FluidSolver.cu:526-597):
            // plane k updates its (i+j)-even cells, then its odd cells.
            for (int k = 0; k < Dd; ++k)
                for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
                    for (int j = 0; j < Hd; ++j)
                        for (int i = (j + colour) & 1; i < Wd; i += 2)
                            p[(size_t)i + (size_t)Wd * ((size_t)j + (size_t)Hd * k)] =
                                gs_cell(g, o, dir, rhs, p, scale, i, j, k);
                }
        } else {
            for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
                for (int k = 0; k < Dd; ++k)
                    for (int j = 0; j < Hd; ++j)
                        for (int i = (j + k + colour) & 1; i < Wd; i += 2)
                            p[(size_t)i + (size_t)Wd * ((size_t)j + (size_t)Hd * k)] =
                                gs_cell(g, o, dir, rhs, p, scale, i, j, k);
            }
        }
    }
}

// FP64 ||b - A p|| and ||b|| with b = (rho dx^2/dt) rhs and A the GS stencil.
// Partial sums per plane, added in plane order: the result does not depend on
// the thread count.
template <class R>
void residual(const blz_params *P, const R *rhs, const R *p, double *res, double *bn) {
    Geo<R> g(P);
    const Open o = open_faces(P);
    const bool dir = P->bc_mode == BLZ_BC_FREE_SURFACE;
    const double scale = (double)P->density * (double)P->dx * (double)P->dx / (double)P->dt;
    const int Wd = g.W, Hd = g.H, Dd = g.D;
    std::vector<double> rr(Dd, 0.0), bb(Dd, 0.0);
    const size_t sy = (size_t)Wd, sz = (size_t)Wd * Hd;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k) {
        double r2 = 0.0, b2 = 0.0;
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                const size_t c = (size_t)i + sy * j + sz * k;
                const double b = scale * (double)rhs[c];
                double nb = 0.0, n = 0.0;
                if (i > 0) { nb += p[c - 1]; n += 1; } else if (dir && o.xlo) n += 1;
                if (i < Wd - 1) { nb += p[c + 1]; n += 1; } else if (dir && o.xhi) n += 1;
                if (j > 0) { nb += p[c - sy]; n += 1; } else if (dir && o.ylo) n += 1;
                if (j < Hd - 1) { nb += p[c + sy]; n += 1; } else if (dir && o.yhi) n += 1;
                if (k > 0) { nb += p[c - sz]; n += 1; } else if (dir && o.zlo) n += 1;
                if (k < Dd - 1) { nb += p[c + sz]; n += 1; } else if (dir && o.zhi) n += 1;
                const double r = b - (n * (double)p[c] - nb);
                r2 += r * r; b2 += b * b;
            }
        rr[k] = r2; bb[k] = b2;
    }
    double r2 = 0.0, b2 = 0.0;
    for (int k = 0; k < Dd; ++k) { r2 += rr[k]; b2 += bb[k]; }
    *res = std::sqrt(r2); *bn = std::sqrt(b2);
}

// Sweeps in chunks of check_every until ||r||/||b|| <= tol or max_iter sweeps
// (tol <= 0: exactly max_iter sweeps, the reference's fixed maxIterSolve).
template <class R>
void solve(const blz_params *P, const R *rhs, R *p, int *iters, double *res, double *bn) {
    Geo<R> g(P);
    if (P->reset_pressure) std::fill(p, p + g.nT(), R(0));
    int done = 0;
    if (P->tol <= 0.0) {
        gs_sweeps(g, P, rhs, p, P->max_iter);
        done = P->max_iter;
    } else {
        const int chunk = std::max(1, P->check_every);
        double r, b;
        residual(P, rhs, p, &r, &b);
        while (done < P->max_iter && !(b == 0.0 || r / b <= P->tol)) {
            const int n = std::min(chunk, P->max_iter - done);
            gs_sweeps(g, P, rhs, p, n);
            done += n;
            residual(P, rhs, p, &r, &b);
        }
    }
    *iters = done;
    residual(P, rhs, p, res, bn);
}

// pressure_gradient_update_kernel, FluidSolver.cu:601-669, in two phases:
// interior faces first, then the domain faces (set to 0 at walls).  Open faces
// copy the inner neighbour after its update in REF_COMPAT (the reference's
// racy copy, read as post-update), or take the Dirichlet ghost gradient in
// FREE_SURFACE.
template <class R>
void gradient(const blz_params *P, const R *p, R *U, R *V, R *W) {
    Geo<R> g(P);
    Field<R> fU = g.U(U), fV = g.V(V), fW = g.Wf(W);
    const R s = g.dt / ((R)P->density * g.dx);
    const int Wd = g.W, Hd = g.H, Dd = g.D;
    const Open o = open_faces(P);
    const bool dir = P->bc_mode == BLZ_BC_FREE_SURFACE;
    auto P_ = [&](int i, int j, int k) { return p[(size_t)i + (size_t)Wd * ((size_t)j + (size_t)Hd * k)]; };
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j < Hd; ++j)
            for (int i = 0; i < Wd; ++i) {
                if (i > 0) fU.at(i, j, k) -= s * (P_(i, j, k) - P_(i - 1, j, k));
                if (j > 0) fV.at(i, j, k) -= s * (P_(i, j, k) - P_(i, j - 1, k));
                if (k > 0) fW.at(i, j, k) -= s * (P_(i, j, k) - P_(i, j, k - 1));
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int j = 0; j < Hd; ++j) {
            R &a = fU.at(0, j, k), &b = fU.at(Wd, j, k);
            a = !o.xlo ? R(0) : dir ? a - s * P_(0, j, k) : fU.at(1, j, k);
            b = !o.xhi ? R(0) : dir ? b + s * P_(Wd - 1, j, k) : fU.at(Wd - 1, j, k);
        }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Dd; ++k)
        for (int i = 0; i < Wd; ++i) {
            R &a = fV.at(i, 0, k), &b = fV.at(i, Hd, k);
            a = !o.ylo ? R(0) : dir ? a - s * P_(i, 0, k) : fV.at(i, 1, k);
            b = !o.yhi ? R(0) : dir ? b + s * P_(i, Hd - 1, k) : fV.at(i, Hd - 1, k);
        }
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Hd; ++j)
        for (int i = 0; i < Wd; ++i) {
            R &a = fW.at(i, j, 0), &b = fW.at(i, j, Dd);
            a = !o.zlo ? R(0) : dir ? a - s * P_(i, j, 0) : fW.at(i, j, 1);
            b = !o.zhi ? R(0) : dir ? b + s * P_(i, j, Dd - 1) : fW.at(i, j, Dd - 1);
        }
}

// ---------------------------------------------------------------------------
// Advection (advect_RK3_kernel, FluidSolver.cu:431-456; order 942-951).
// ---------------------------------------------------------------------------
template <class R>
static void advect_field(const Geo<R> &g, const Field<R> &U, const Field<R> &V, const Field<R> &W,
                         const Field<R> &src, R *dst, bool clamp) {
    const R dx = g.dx, dt = g.dt;
    const R a = R(2) / R(9), b = R(3) / R(9), c = R(4) / R(9);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < src.d; ++k)
        for (int j = 0; j < src.h; ++j)
            for (int i = 0; i < src.w; ++i) {
                const R px = (R(i) + src.ox) * dx, py = (R(j) + src.oy) * dx, pz = (R(k) + src.oz) * dx;
                const V3<R> k1 = vel_at(g, U, V, W, px, py, pz);
                const R h1 = R(0.5) * dt, h2 = R(0.75) * dt;
                R qx, qy, qz;
                if (g.P->advect_scheme == BLZ_ADVECT_EULER) {       // FluidSolver.cu:392-407
                    qx = px - dt * k1.x; qy = py - dt * k1.y; qz = pz - dt * k1.z;
                } else if (g.P->advect_scheme == BLZ_ADVECT_RK2) {  // FluidSolver.cu:409-429
                    const V3<R> m = vel_at(g, U, V, W, px - h1 * k1.x, py - h1 * k1.y, pz - h1 * k1.z);
                    qx = px - dt * m.x; qy = py - dt * m.y; qz = pz - dt * m.z;
                } else {                                            // FluidSolver.cu:431-456
                    const V3<R> k2 = vel_at(g, U, V, W, px - h1 * k1.x, py - h1 * k1.y, pz - h1 * k1.z);
                    const V3<R> k3 = vel_at(g, U, V, W, px - h2 * k2.x, py - h2 * k2.y, pz - h2 * k2.z);
                    qx = px - dt * (a * k1.x + b * k2.x + c * k3.x);
                    qy = py - dt * (a * k1.y + b * k2.y + c * k3.y);
                    qz = pz - dt * (a * k1.z + b * k2.z + c * k3.z);
                }
                dst[(size_t)i + (size_t)src.w * ((size_t)j + (size_t)src.h * k)] =
                    tricubic(src, dx, qx, qy, qz, clamp);
            }
}

template <class R>
void advect(const blz_params *P, R *T, R *U, R *V, R *W, R *Dn = nullptr) {
    Geo<R> g(P);
    std::vector<R> nT(g.nT()), nU(g.nU()), nV(g.nV()), nW(g.nW());
    Field<R> fT = g.T(T), fU = g.U(U), fV = g.V(V), fW = g.Wf(W);
    if (Dn) {                                     // the density scalar, clamped like T
        std::vector<R> nD(g.nT());
        advect_field(g, fU, fV, fW, g.T(Dn), nD.data(), true);
        std::copy(nD.begin(), nD.end(), Dn);
    }
    advect_field(g, fU, fV, fW, fT, nT.data(), true);
    advect_field(g, fU, fV, fW, fU, nU.data(), false);
    advect_field(g, fU, fV, fW, fV, nV.data(), false);
    advect_field(g, fU, fV, fW, fW, nW.data(), false);
    std::copy(nT.begin(), nT.end(), T); std::copy(nU.begin(), nU.end(), U);
    std::copy(nV.begin(), nV.end(), V); std::copy(nW.begin(), nW.end(), W);
}

// FluidSolver::step, FluidSolver.cu:858-955.
template <class R>
void step(const blz_params *P, float time, R *T, R *U, R *V, R *W, R *p, R *rhs,
          int *iters, double *res, double *bn, R *Dn = nullptr) {
    forces(P, time, T, U, V, W, Dn);
    divergence(P, U, V, W, rhs);
    solve(P, rhs, p, iters, res, bn);
    gradient(P, p, U, V, W);
    advect(P, T, U, V, W, Dn);
}

} // namespace orc

// ---------------------------------------------------------------------------
// C ABI for ctypes (tests, smoke check, bench CPU baseline).
// ---------------------------------------------------------------------------
extern "C" {

float orc_perlin(float x, float y, float z, float scale, int seed) {
    return orc::perlin(x, y, z, scale, seed);
}

#define ORC_EXPORT_ALL(SUF, R)                                                              \
    void orc_add_source_##SUF(const blz_params *P, const float *rec, int n, R *T, R *U,       \
                              R *V, R *W, const float *dens, R *Dn) {                        \
        orc::add_source<R>(P, rec, n, T, U, V, W, dens, Dn); }                               \
    void orc_forces_##SUF(const blz_params *P, float time, R *T, R *U, R *V, R *W,           \
                          const R *Dn) { orc::forces<R>(P, time, T, U, V, W, Dn); }          \
    void orc_divergence_##SUF(const blz_params *P, const R *U, const R *V, const R *W,       \
                              R *rhs) { orc::divergence<R>(P, U, V, W, rhs); }               \
    void orc_gs_sweeps_##SUF(const blz_params *P, const R *rhs, R *p, int n) {               \
        orc::Geo<R> g(P); orc::gs_sweeps<R>(g, P, rhs, p, n); }                              \
    void orc_solve_##SUF(const blz_params *P, const R *rhs, R *p, int *it, double *res,      \
                         double *bn) { orc::solve<R>(P, rhs, p, it, res, bn); }              \
    void orc_residual_##SUF(const blz_params *P, const R *rhs, const R *p, double *res,      \
                            double *bn) { orc::residual<R>(P, rhs, p, res, bn); }            \
    void orc_gradient_##SUF(const blz_params *P, const R *p, R *U, R *V, R *W) {             \
        orc::gradient<R>(P, p, U, V, W); }                                                   \
    void orc_advect_##SUF(const blz_params *P, R *T, R *U, R *V, R *W, R *Dn) {              \
        orc::advect<R>(P, T, U, V, W, Dn); }                                                 \
    void orc_step_##SUF(const blz_params *P, float time, R *T, R *U, R *V, R *W, R *p,       \
                        R *rhs, int *it, double *res, double *bn, R *Dn) {                   \
        orc::step<R>(P, time, T, U, V, W, p, rhs, it, res, bn, Dn); }

ORC_EXPORT_ALL(f64, double)
ORC_EXPORT_ALL(f32, float)

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Threads of the oracle's later parallel loops (the single-core baseline).
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

} // extern "C"
