// k_project.cu — divergence, red-black Gauss-Seidel, FP64 residual and the
// pressure-gradient subtract (reference src/FluidSolver.cu:475-669, 823-856).
//
// Pressure and rhs live colour packed in HBM: cell (i,j,k) of colour
// c = (i+j+k)&1 sits at (i>>1) + (W/2)*(j + H*k) of its colour's array.  A half
// sweep of colour c writes only c's array and reads only the other colour's,
// all rows contiguous; red cells of a row are even or odd i according to the
// row parity (j+k)&1.
#include <algorithm>
#include <type_traits>

#include <cuda.h>   // CUtensorMap and its enums; the encoder comes from cudaGetDriverEntryPoint

#include "kernels.cuh"

namespace blz {

__device__ __forceinline__ float pval(const float *__restrict__ pr, const float *__restrict__ pb,
                                      int i, int j, int k, int Wh, int H) {
    const float *a = ((i + j + k) & 1) ? pb : pr;
    return __ldg(a + pidx(i, j, k, Wh, H));
}

// compute_divergence_kernel (FluidSolver.cu:475-515): rhs = -div/dx, with the
// flux of a solid wall face removed.  One thread per packed pair (2m, 2m+1).
__global__ void k_divergence(Geom g, const float *__restrict__ U, const float *__restrict__ V,
                             const float *__restrict__ W, OpenFaces o, float *__restrict__ rr,
                             float *__restrict__ rb) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    const int Wh = g.W >> 1;
    if (m >= Wh || j >= g.H || k >= g.D) return;
    const float s = 1.0f / g.dx;
    float out[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int i = 2 * m + t;
        const float u0 = __ldg(U + lin(i, j, k, g.W + 1, g.H)), u1 = __ldg(U + lin(i + 1, j, k, g.W + 1, g.H));
        const float v0 = __ldg(V + lin(i, j, k, g.W, g.H + 1)), v1 = __ldg(V + lin(i, j + 1, k, g.W, g.H + 1));
        const float w0 = __ldg(W + lin(i, j, k, g.W, g.H)), w1 = __ldg(W + lin(i, j, k + 1, g.W, g.H));
        float r = -s * (u1 - u0 + v1 - v0 + w1 - w0);
        if (i == 0) { if (!o.xlo) r -= s * u0; }
        else if (i == g.W - 1) { if (!o.xhi) r += s * u1; }
        if (j == 0) { if (!o.ylo) r -= s * v0; }
        else if (j == g.H - 1) { if (!o.yhi) r += s * v1; }
        if (k == 0) { if (!o.zlo) r -= s * w0; }
        else if (k == g.D - 1) { if (!o.zhi) r += s * w1; }
        out[t] = r;
    }
    const size_t q = pidx(2 * m, j, k, Wh, g.H);
    const bool even_red = ((j + k) & 1) == 0;         // cell 2m is red
    rr[q] = even_red ? out[0] : out[1];
    rb[q] = even_red ? out[1] : out[0];
}

void launch_divergence(const Geom &g, const float *U, const float *V, const float *W,
                       const OpenFaces &o, float *rhs_r, float *rhs_b, cudaStream_t st) {
    const dim3 b(32, 8, 1);
    const dim3 gr(((g.W >> 1) + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, g.D);
    k_divergence<<<gr, b, 0, st>>>(g, U, V, W, o, rhs_r, rhs_b);
}

// Quotient num/den for the neighbour count den in {1..6} as
// RN(num * hi + RN(num * lo)), hi = RN(1/den) and lo = RN(1/den - hi): two
// instructions on the FMA pipe instead of an IEEE division (a reciprocal and
// an int-to-float conversion per cell on the XU pipe) or a remainder-
// corrected product (three).  The result is within about half an ulp of the
// quotient and, unlike num * RN(1/den) alone, carries no bias: RN(1/3),
// RN(1/5) and RN(1/6) are all slightly large, and a sweep that scaled every
// update by 1 + 3e-8 would converge to the solution of A - 1.8e-7 I, whose
// smooth modes differ from A's by parts in 10^4 at 256^3.
__device__ __forceinline__ float inv_count(float den) {
    return den == 6.0f ? 1.0f / 6.0f : den == 5.0f ? 0.2f : den == 4.0f ? 0.25f
         : den == 3.0f ? 1.0f / 3.0f : den == 2.0f ? 0.5f : 1.0f;
}
__device__ __forceinline__ float inv_count_lo(float den) {
    return den == 6.0f ? -4.967053879312289e-09f : den == 5.0f ? -2.9802322831784522e-09f
         : den == 3.0f ? -9.934107758624577e-09f : 0.0f;
}
__device__ __forceinline__ float div_hl(float num, float hi, float lo) {
    return __fmaf_rn(num, hi, __fmul_rn(num, lo));
}
__device__ __forceinline__ float div_count(float num, float den) {
    return div_hl(num, inv_count(den), inv_count_lo(den));
}

// One Gauss-Seidel update p = (scale*rhs + sum p_nb)/n_nb (FluidSolver.cu:
// 532-561), summed in the reference's neighbour order.  n_nb counts the
// in-domain neighbours, plus a p = 0 ghost per open face when dirichlet.
__device__ __forceinline__ float gs_update(const Geom &g, const SolveParams &sp, float rhs,
                                           const float *__restrict__ po, size_t q, int i, int j,
                                           int k, int s, int Wh) {
    // The same rounded operations as gs_quad (a missing neighbour adds +0):
    // num = RN(scale * rhs + x-), then RN adds of x+, y-, y+, z-, z+.
    float den = 0.0f;
    const bool dir = sp.dirichlet;
    float xm = 0.0f, xp = 0.0f, ym = 0.0f, yp = 0.0f, zm = 0.0f, zp = 0.0f;
    if (i > 0) { xm = __ldg(po + q - (s ? 0 : 1)); den += 1.0f; } else if (dir && sp.open.xlo) den += 1.0f;
    if (i < g.W - 1) { xp = __ldg(po + q + (s ? 1 : 0)); den += 1.0f; } else if (dir && sp.open.xhi) den += 1.0f;
    if (j > 0) { ym = __ldg(po + q - Wh); den += 1.0f; } else if (dir && sp.open.ylo) den += 1.0f;
    if (j < g.H - 1) { yp = __ldg(po + q + Wh); den += 1.0f; } else if (dir && sp.open.yhi) den += 1.0f;
    const size_t pl = (size_t)Wh * g.H;
    if (k > 0) { zm = __ldg(po + q - pl); den += 1.0f; } else if (dir && sp.open.zlo) den += 1.0f;
    if (k < g.D - 1) { zp = __ldg(po + q + pl); den += 1.0f; } else if (dir && sp.open.zhi) den += 1.0f;
    float num = __fmaf_rn(sp.scale, rhs, xm);
    num = __fadd_rn(num, xp);
    num = __fadd_rn(num, ym);
    num = __fadd_rn(num, yp);
    num = __fadd_rn(num, zm);
    num = __fadd_rn(num, zp);
    return div_count(num, den);
}

// Half sweep of colour `colour` over the whole grid (3-D red-black order).
__global__ void k_rbgs_half(Geom g, SolveParams sp, const float *__restrict__ rhs_c,
                            const float *__restrict__ p_o, float *__restrict__ p_c, int colour) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    const int Wh = g.W >> 1;
    if (m >= Wh || j >= g.H || k >= g.D) return;
    const int s = (j + k + colour) & 1;               // i = 2m + s
    const int i = 2 * m + s;
    const size_t q = pidx(i, j, k, Wh, g.H);
    p_c[q] = gs_update(g, sp, __ldg(rhs_c + q), p_o, q, i, j, k, s, Wh);
}

// Half sweep with four consecutive packed cells per thread (W % 8 == 0):
// 128-bit loads of the rhs row segment, of the other colour's segments in
// rows j-1, j, j+1 and planes k-1, k+1, plus one scalar for the x neighbour
// that falls outside the segment; 128-bit store.
__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }

// Neighbour counts' reciprocals (hi, lo of div_hl) of a quad: the count is
// the same for every cell of the quad except the one at a row end (cell 0
// when the row's cells sit at even i and the quad starts the row, cell 3
// when odd and it ends the row), so they are formed three times per quad.
struct QuadDen {
    float l0, i0, lb, ib, l3, i3;
};

__device__ __forceinline__ QuadDen quad_den(const SolveParams &sp, int s, bool first, bool last, bool has_ym,
                                            bool has_yp, bool has_zm, bool has_zp) {
    const bool dir = sp.dirichlet;
    QuadDen q;
    const float db = 2.0f + (has_ym ? 1.0f : (dir && sp.open.ylo ? 1.0f : 0.0f)) +
                     (has_yp ? 1.0f : (dir && sp.open.yhi ? 1.0f : 0.0f)) +
                     (has_zm ? 1.0f : (dir && sp.open.zlo ? 1.0f : 0.0f)) +
                     (has_zp ? 1.0f : (dir && sp.open.zhi ? 1.0f : 0.0f));
    const float d0 = (s == 0 && first) ? db - 1.0f + (dir && sp.open.xlo ? 1.0f : 0.0f) : db;
    const float d3 = (s == 1 && last) ? db - 1.0f + (dir && sp.open.xhi ? 1.0f : 0.0f) : db;
    q.ib = inv_count(db);
    q.i0 = inv_count(d0);
    q.i3 = inv_count(d3);
    q.lb = inv_count_lo(db);
    q.l0 = inv_count_lo(d0);
    q.l3 = inv_count_lo(d3);
    return q;
}

// Updates four consecutive packed cells m0..m0+3 of one row given their
// neighbour counts: o is the other colour at the same packed indices, xe its
// value just outside the segment (m0-1 when the row's cells sit at even i,
// m0+4 when odd), ym/yp/zm/zp the other colour in rows j-1, j+1 and planes
// k-1, k+1.  A missing neighbour arrives as 0 (the caller passes zero4 and
// xe = 0), so the sum is branch free and in the reference's order.
__device__ __forceinline__ float4 gs_quad(float scale, int s, float4 r, float4 o, float xe, float4 ym, float4 yp,
                                          float4 zm, float4 zp, const QuadDen &q) {
    float xl[4], xr[4];
    if (s == 0) {
        xl[0] = xe; xl[1] = o.x; xl[2] = o.y; xl[3] = o.z;
        xr[0] = o.x; xr[1] = o.y; xr[2] = o.z; xr[3] = o.w;
    } else {
        xl[0] = o.x; xl[1] = o.y; xl[2] = o.z; xl[3] = o.w;
        xr[0] = o.y; xr[1] = o.z; xr[2] = o.w; xr[3] = xe;
    }
    const float ra[4] = {r.x, r.y, r.z, r.w};
    const float yma[4] = {ym.x, ym.y, ym.z, ym.w}, ypa[4] = {yp.x, yp.y, yp.z, yp.w};
    const float zma[4] = {zm.x, zm.y, zm.z, zm.w}, zpa[4] = {zp.x, zp.y, zp.z, zp.w};
    float out[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        // every rounding explicit, so the packed form (gs_quad_pk) has the
        // same bits
        float num = __fmaf_rn(scale, ra[t], xl[t]);
        num = __fadd_rn(num, xr[t]);
        num = __fadd_rn(num, yma[t]);
        num = __fadd_rn(num, ypa[t]);
        num = __fadd_rn(num, zma[t]);
        num = __fadd_rn(num, zpa[t]);
        const float hi = t == 0 ? q.i0 : t == 3 ? q.i3 : q.ib;
        const float lo = t == 0 ? q.l0 : t == 3 ? q.l3 : q.lb;
        out[t] = div_hl(num, hi, lo);
    }
    return make_float4(out[0], out[1], out[2], out[3]);
}

// gs_quad on Blackwell's paired FP32 instructions: cells (0,1) and (2,3) of
// the quad go through one fma/add/mul.rn.f32x2 each, every lane rounded as
// IEEE FP32, in gs_quad's order, so the bits equal gs_quad's.
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2(float lo, float hi) {
    f2_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_split(f2_t v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
    f2_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
    f2_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
    f2_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

__device__ __forceinline__ f2_t gs_pair(f2_t scale2, f2_t r, f2_t xl, f2_t xr, f2_t ym, f2_t yp, f2_t zm, f2_t zp,
                                        f2_t hi, f2_t lo) {
    f2_t num = f2_fma(scale2, r, xl);
    num = f2_add(num, xr);
    num = f2_add(num, ym);
    num = f2_add(num, yp);
    num = f2_add(num, zm);
    num = f2_add(num, zp);
    return f2_fma(num, hi, f2_mul(num, lo));
}

__device__ __forceinline__ float4 gs_quad_pk(float scale, int s, float4 r, float4 o, float xe, float4 ym, float4 yp,
                                             float4 zm, float4 zp, const QuadDen &q) {
    const f2_t sc = f2(scale, scale);
    const f2_t xl01 = s == 0 ? f2(xe, o.x) : f2(o.x, o.y), xl23 = s == 0 ? f2(o.y, o.z) : f2(o.z, o.w);
    const f2_t xr01 = s == 0 ? f2(o.x, o.y) : f2(o.y, o.z), xr23 = s == 0 ? f2(o.z, o.w) : f2(o.w, xe);
    const f2_t a = gs_pair(sc, f2(r.x, r.y), xl01, xr01, f2(ym.x, ym.y), f2(yp.x, yp.y), f2(zm.x, zm.y),
                           f2(zp.x, zp.y), f2(q.i0, q.ib), f2(q.l0, q.lb));
    const f2_t b = gs_pair(sc, f2(r.z, r.w), xl23, xr23, f2(ym.z, ym.w), f2(yp.z, yp.w), f2(zm.z, zm.w),
                           f2(zp.z, zp.w), f2(q.ib, q.i3), f2(q.lb, q.l3));
    float4 out;
    f2_split(a, out.x, out.y);
    f2_split(b, out.z, out.w);
    return out;
}

__device__ __forceinline__ float4 gs_segment(const SolveParams &sp, int s, bool first, bool last, float4 r,
                                             float4 o, float xe, float4 ym, float4 yp, float4 zm, float4 zp,
                                             bool has_ym, bool has_yp, bool has_zm, bool has_zp) {
    return gs_quad(sp.scale, s, r, o, xe, ym, yp, zm, zp,
                   quad_den(sp, s, first, last, has_ym, has_yp, has_zm, has_zp));
}

// Half sweep, four packed cells per thread along x (W % 8 == 0), KZ
// consecutive planes per thread: the thread marches in z carrying the other
// colour's segments of planes k-1 and k in registers, so each plane adds one
// 128-bit load of plane k+1 instead of two.  Every variant performs the same
// operations per cell, so all give bitwise identical results.
template <int KZ>
__device__ __forceinline__ void seg_sweep(const Geom &g, const SolveParams &sp, const float *__restrict__ rhs_c,
                                          const float *__restrict__ p_o, float *__restrict__ p_c, int colour,
                                          int mq, int j, int k0) {
    const int Wh = g.W >> 1;
    const int m0 = mq * 4;
    const size_t pl = (size_t)Wh * g.H;
    const size_t row = (size_t)m0 + (size_t)Wh * (size_t)j;
    const bool has_ym = j > 0, has_yp = j < g.H - 1;
    const bool first = m0 == 0, last = m0 + 4 == Wh;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 zm = k0 > 0 ? ld4(p_o + row + (size_t)(k0 - 1) * pl) : zero4;
    float4 cur = ld4(p_o + row + (size_t)k0 * pl);
#pragma unroll
    for (int kk = 0; kk < KZ; ++kk) {
        const int k = k0 + kk;
        if (k >= g.D) break;
        const size_t q = row + (size_t)k * pl;
        const bool has_zm = k > 0, has_zp = k < g.D - 1;
        const float4 zp = has_zp ? ld4(p_o + q + pl) : zero4;
        const float4 r = ld4(rhs_c + q);
        const float4 ym = has_ym ? ld4(p_o + q - Wh) : zero4;
        const float4 yp = has_yp ? ld4(p_o + q + Wh) : zero4;
        const int s = (j + k + colour) & 1;
        const float xe = s == 0 ? (first ? 0.0f : __ldg(p_o + q - 1)) : (last ? 0.0f : __ldg(p_o + q + 4));
        *reinterpret_cast<float4 *>(p_c + q) =
            gs_segment(sp, s, first, last, r, cur, xe, ym, yp, zm, zp, has_ym, has_yp, has_zm, has_zp);
        zm = cur;
        cur = zp;
    }
}

template <int KZ>
__global__ void __launch_bounds__(256)
k_rbgs_seg(Geom g, SolveParams sp, const float *__restrict__ rhs_c, const float *__restrict__ p_o,
           float *__restrict__ p_c, int colour) {
    const int Wq = g.W >> 3;
    const int mq = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * KZ;
    if (mq >= Wq || j >= g.H || k0 >= g.D) return;
    seg_sweep<KZ>(g, sp, rhs_c, p_o, p_c, colour, mq, j, k0);
}

// ---------------------------------------------------------------------------
// Temporal blocking: two red-black sweeps per pass over HBM, out of place
// (reads rhs and the black half of p_in, writes both halves of p_out; a
// red update never reads the old red values, so p_in's red half is not
// needed).  A CTA owns TY full-width rows and ZC planes of the output and
// carries a 4-row / 4-plane halo; it marches a wavefront along z: at step t
// level 0 updates red on plane t, level 1 black on t-1, level 2 red on t-2,
// level 3 black on t-3, each level over a region one row and one plane
// narrower than the one before, so every update reads exactly the values
// the in-place sweeps would.  Per cell the arithmetic is gs_quad's, so a
// pass equals two sweeps of the segment kernel bit for bit.  HBM traffic
// per pass is about 10 B/cell instead of 24 B/cell for two unblocked sweeps;
// the price is recomputing the halo.
//
// A thread owns one quad in each of two adjacent rows (A = 2y, B = 2y + 1)
// and carries both rows' plane windows in registers: the z neighbours, and
// the y neighbour inside the pair, come from registers; the y neighbour
// outside the pair and the rhs come from shared memory; the x neighbour
// beyond the quad comes from a warp shuffle when a warp spans exactly one
// row (W = 256), else from shared memory.
//
// One barrier per step suffices: in step t every level reads only planes
// written in step t-1 (level 0 the black input staged then, level 1 red
// t-1 from level 0, level 2 black t-2 from level 1, level 3 red t-3 from
// level 2), and the slots written in step t (red t and t-2, black t+1 and
// t-1) are, modulo the four-slot rings, none of the slots read in it (red
// t-1 and t-3, black t and t-2); every slot's previous contents were last
// read in step t-1.
//
// Missing neighbours read zeros instead of being selected away: the p
// slots start zero-filled and rows outside the domain are never written
// (their register windows stay zero); the row pads hold the x neighbour
// beyond either row end; and a plane outside the domain is zero in the
// register windows (the staged input reads zero there and level 0 sets zero
// past the last plane).  Adding +0 is what the segment kernel does for a
// missing neighbour, so the sums are the same bits; only the neighbour
// counts of the two end planes differ from the interior ones.
// ---------------------------------------------------------------------------
constexpr int kTbThreads = 384;
constexpr int kTbSlots = 18;
// Dynamic shared memory of one pass at most: the 227 KB a block may opt into,
// less room for the static shared memory (the TMA variant's mbarriers).
constexpr int kTbSmemMax = 227 * 1024 - 1024;

// Rows of output per CTA: as many as the thread budget (one thread per quad
// of a row pair; TY + 8 rows with the halo, rounded up to a whole pair) and
// the shared memory (18 plane slots of rows of Wq + 1 float4, the last a
// zero pad) allow.
__host__ __device__ inline int tb_rows_tile(int Wq, int H) {
    const int by_threads = 2 * (kTbThreads / Wq);
    const int by_smem = kTbSmemMax / (kTbSlots * (Wq + 1) * 16);
    const int ty = ((by_threads < by_smem ? by_threads : by_smem) & ~1) - 8;
    return ty < H ? ty : H;
}
__host__ __device__ inline int tb_rows_alloc(int TY) { return (TY + 8 + 1) & ~1; }

// TMA staging: the rhs and input planes arrive as bulk tensor copies (one
// box of Wh floats x the CTA's rows x 1 plane per copy) into dense ring
// slots, completing on one mbarrier per slot.  Rows and planes outside the
// grid arrive as zeros (the copies' out-of-bounds fill).  Every wait is
// bounded in time (kTbWaitNs on the device's global timer).  When a wait of
// any thread gives up, the whole CTA stops the pass: it counts the failure in
// g_tb_timeouts, waits once more (bounded) for the copies it issued last so
// that none lands in shared memory after the CTA has exited, and returns
// without computing on unfilled slots.  The pass's output is then incomplete
// and the solver reports BLZ_ERR_TIMEOUT.
constexpr int kTbDenseSlots = 10;                 // 4 red rhs, 4 black rhs, 2 input
constexpr unsigned long long kTbWaitNs = 10ull * 1000ull * 1000ull;   // 10 ms; a normal wait takes microseconds
__device__ unsigned int g_tb_timeouts;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long tb_now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of the mbarrier at `bar`; false after kTbWaitNs.
__device__ __forceinline__ bool tb_wait(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = tb_now_ns();
    for (;;) {
        for (int it = 0; it < 64; ++it) {
            uint32_t done;
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                         " selp.u32 %0, 1, 0, p;\n}\n"
                         : "=r"(done) : "r"(bar), "r"(parity) : "memory");
            if (done) return true;
        }
        if (tb_now_ns() - t0 > kTbWaitNs) return false;
    }
}

__host__ __device__ inline int tb_dense_slot_bytes(int Wq, int rows_alloc) {
    return (rows_alloc * Wq * 16 + 127) & ~127;
}

// One tile of a temporal-blocking pass: output rows [j0, j0 + TY) and planes
// [z0, z1) of one grid, by a CTA of nrp row pairs x Wq quads (thread (mq, rp)
// owns quad mq of rows 2 rp and 2 rp + 1; `live` is false for threads of the
// CTA beyond that shape, which only meet the barriers).  `leader` is one
// thread of the CTA (TMA issue).  The tensor maps are used with TMA only.
template <bool WARPROW, bool TMA, bool PK>
__device__ __forceinline__ void tb2_tile(const Geom &g, const SolveParams &sp, const float *__restrict__ rhs_r,
                                         const float *__restrict__ rhs_b, const float *__restrict__ pin_b,
                                         float *__restrict__ pout_r, float *__restrict__ pout_b, int TY, int j0,
                                         int z0, int z1, int mq, int rp, int nrp, bool live, bool leader,
                                         const CUtensorMap *map_r, const CUtensorMap *map_b,
                                         const CUtensorMap *map_in) {
    // Shared memory, in units of one plane slot (2*nrp rows of
    // Wq + 1 float4; the last float4 of each row is a zero pad), addressed
    // by 32-bit byte offsets:
    //   [0, 8)   p, colour c and plane k at slot c*4 + (k & 3)
    //   [8, 12)  red rhs, plane k at 8 + (k & 3)
    //   [12, 16) black rhs, plane k at 12 + (k & 3)
    //   [16, 18) black p input staging, plane k at 16 + (k & 1)
    // rhs and staged input are prefetched one step ahead with cp.async and
    // only ever read back by the thread that loaded them.
    //
    // With TMA the rhs and input slots are dense rows of Wq float4 (only
    // their owner reads them) in a region of kTbDenseSlots 128-byte-aligned
    // slots ahead of the p slots: red rhs k at (k & 3), black rhs k at
    // 4 + (k & 3), input k at 8 + (k & 1).
    extern __shared__ __align__(128) float4 sm4[];
    __shared__ __align__(8) uint64_t tbar[kTbDenseSlots];
    const int Wh = g.W >> 1, Wq = Wh >> 2, D = g.D;
    const int rows_alloc = 2 * nrp;
    const int dslot = TMA ? tb_dense_slot_bytes(Wq, rows_alloc) : 0;
    char *const raw = reinterpret_cast<char *>(sm4);
    char *const dbase = TMA ? raw + ((128u - (smem_addr(raw) & 127u)) & 127u) : raw;
    char *const smc = dbase + (TMA ? kTbDenseSlots * dslot : 0);
    const uint32_t sm_base = static_cast<uint32_t>(__cvta_generic_to_shared(smc));
    const int rows = TY + 8;
    const int rA = 2 * rp, rB = rA + 1;
    const int jA = j0 - 4 + rA, jB = jA + 1;
    const bool okA = live && jA >= 0 && jA < g.H, okB = live && rB < rows && jB >= 0 && jB < g.H;
    const int m0 = 4 * mq;
    const long long pl = (long long)Wh * g.H;
    const long long offA = (long long)m0 + (long long)Wh * (okA ? jA : 0);
    const long long offB = (long long)m0 + (long long)Wh * (okB ? jB : 0);
    const bool first = m0 == 0, last = m0 + 4 == Wh;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const int rowb = (Wq + 1) * 16, slotb = rows_alloc * rowb;
    const int ownA = rA * rowb + mq * 16, ownB = ownA + rowb;
    const int denA = (rA * Wq + mq) * 16, denB = denA + Wq * 16;       // dense-slot offsets (TMA)
    auto slot = [&](int c, int k) { return (c * 4 + (k & 3)) * slotb; };
    auto lds4 = [&](int off) { return *reinterpret_cast<const float4 *>(smc + off); };
    auto lds1 = [&](int off) { return *reinterpret_cast<const float *>(smc + off); };
    auto sts4 = [&](int off, float4 v) { *reinterpret_cast<float4 *>(smc + off) = v; };
    auto cp16 = [&](int off, const float *src) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sm_base + (uint32_t)off), "l"(src)
                     : "memory");
    };
    if (live) {
#pragma unroll
        for (int sl = 0; sl < 8; ++sl) {
            sts4(sl * slotb + ownA, zero4);
            sts4(sl * slotb + ownB, zero4);
            if (last) {                               // the rows' pads
                sts4(sl * slotb + ownA + 16, zero4);
                sts4(sl * slotb + ownB + 16, zero4);
            }
        }
    }
    // Rows on which level h updates: bit h (the halo shrinks by one row per
    // level; level 3's rows are the CTA's output rows).
    auto rowmask = [&](int r, bool ok) {
        return ok ? ((r >= 1 && r < rows - 1 ? 1u : 0u) | (r >= 2 && r < rows - 2 ? 2u : 0u) |
                     (r >= 3 && r < rows - 3 ? 4u : 0u) | (r >= 4 && r < rows - 4 ? 8u : 0u))
                  : 0u;
    };
    const unsigned mA = rowmask(rA, okA), mB = rowmask(rB, okB);
    auto kact = [&](int h, int k) { return k >= z0 - 3 + h && k < z1 + 3 - h && k >= 0 && k < D; };
    auto kin = [&](int k) { return k >= 0 && k < D; };
    // Neighbour counts of each row's quad on planes with both z neighbours,
    // for row parity s = 0 and 1.
    const bool hymA = jA > 0, hypA = jA < g.H - 1, hymB = jB > 0, hypB = jB < g.H - 1;
    const QuadDen qA0 = quad_den(sp, 0, first, last, hymA, hypA, true, true);
    const QuadDen qA1 = quad_den(sp, 1, first, last, hymA, hypA, true, true);
    const QuadDen qB0 = quad_den(sp, 0, first, last, hymB, hypB, true, true);
    const QuadDen qB1 = quad_den(sp, 1, first, last, hymB, hypB, true, true);
    const int RR = 8 * slotb, RB = 12 * slotb, STG = 16 * slotb;
    const uint32_t dbase_u = smem_addr(dbase);
    // TMA: one bulk tensor copy of plane k into dense slot ds.
    auto tma_fill = [&](const CUtensorMap *m, int ds, int k) {
        const uint32_t bar = smem_addr(&tbar[ds]);
        const uint32_t bytes = (uint32_t)(rows_alloc * Wh * 4);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3, %4}], [%5];"
                     ::"r"(dbase_u + (uint32_t)(ds * dslot)), "l"(reinterpret_cast<uint64_t>(m)), "r"(0),
                       "r"(j0 - 4), "r"(k), "r"(bar)
                     : "memory");
    };
    // Fill order: red planes z0-3.. in slots k & 3, black planes z0-2.. in
    // 4 + (k & 3), input planes z0-2.. in 8 + (k & 1); the n-th fill of a
    // slot completes its mbarrier's phase n.
    auto wait_red = [&](int k) { return tb_wait(smem_addr(&tbar[k & 3]), ((k - (z0 - 3)) >> 2) & 1); };
    auto wait_black = [&](int k) { return tb_wait(smem_addr(&tbar[4 + (k & 3)]), ((k - (z0 - 2)) >> 2) & 1); };
    auto wait_in = [&](int k) { return tb_wait(smem_addr(&tbar[8 + (k & 1)]), ((k - (z0 - 2)) >> 1) & 1); };
    // ALL: every plane asked for is known to be in range (steady steps).
    auto prefetch = [&](int k_red, int k_black, int k_in, auto all_c) __attribute__((always_inline)) {
        constexpr bool ALL = decltype(all_c)::value;
        if constexpr (TMA) {
            if (!leader) return;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (ALL || (k_red >= z0 - 3 && k_red < z1 + 3)) tma_fill(map_r, k_red & 3, k_red);
            if (ALL || (k_black >= z0 - 2 && k_black < z1 + 2)) tma_fill(map_b, 4 + (k_black & 3), k_black);
            if (ALL || (k_in >= z0 - 2 && k_in < z1 + 4)) tma_fill(map_in, 8 + (k_in & 1), k_in);
            return;
        }
        // red rhs: levels 0 and 2 cover planes [z0-3, z1+3); black rhs: levels 1 and 3 cover [z0-2, z1+2)
        if (ALL || (kin(k_red) && k_red >= z0 - 3 && k_red < z1 + 3)) {
            const int o = RR + (k_red & 3) * slotb;
            if (okA) cp16(o + ownA, rhs_r + offA + k_red * pl);
            if (okB) cp16(o + ownB, rhs_r + offB + k_red * pl);
        }
        if (ALL || (kin(k_black) && k_black >= z0 - 2 && k_black < z1 + 2)) {
            const int o = RB + (k_black & 3) * slotb;
            if (okA) cp16(o + ownA, rhs_b + offA + k_black * pl);
            if (okB) cp16(o + ownB, rhs_b + offB + k_black * pl);
        }
        if (ALL || (kin(k_in) && k_in < z1 + 4)) {
            const int o = STG + (k_in & 1) * slotb;
            if (okA) cp16(o + ownA, pin_b + offA + k_in * pl);
            if (okB) cp16(o + ownB, pin_b + offB + k_in * pl);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // rhs of colour c, plane k, for the row whose element offsets are
    // (own, den): from its padded slot (cp.async) or its dense slot (TMA).
    auto rhs_ld = [&](int c, int k, int own, int den) -> float4 {
        if constexpr (TMA) return lds4((int)(dbase - smc) + ((c ? 4 : 0) + (k & 3)) * dslot + den);
        return lds4((c ? RB : RR) + (k & 3) * slotb + own);
    };
    if constexpr (TMA) {
        if (leader) {
            for (int i = 0; i < kTbDenseSlots; ++i)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&tbar[i])) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    // register windows of each row: black planes t-3..t+1, red planes t-4..t
    float4 bm3A = zero4, bm2A = zero4, bp1A, rm4A = zero4, rm3A = zero4, rm2A = zero4, rm1A = zero4, r0A = zero4;
    float4 bm3B = zero4, bm2B = zero4, bp1B, rm4B = zero4, rm3B = zero4, rm2B = zero4, rm1B = zero4, r0B = zero4;
    float4 bm1A = okA && kin(z0 - 4) ? ld4(pin_b + offA + (z0 - 4) * pl) : zero4;
    float4 b0A = okA && kin(z0 - 3) ? ld4(pin_b + offA + (z0 - 3) * pl) : zero4;
    float4 bm1B = okB && kin(z0 - 4) ? ld4(pin_b + offB + (z0 - 4) * pl) : zero4;
    float4 b0B = okB && kin(z0 - 3) ? ld4(pin_b + offB + (z0 - 3) * pl) : zero4;
    if (live) {
        sts4(slot(1, z0 - 4) + ownA, bm1A);
        sts4(slot(1, z0 - 3) + ownA, b0A);
        sts4(slot(1, z0 - 4) + ownB, bm1B);
        sts4(slot(1, z0 - 3) + ownB, b0B);
    }
    prefetch(z0 - 3, z0 - 4, z0 - 2, std::false_type{});   // what the first step reads
    // One quad update of row parity S: colour c on plane k, `own` the row's
    // element offset, o the other colour's own quad, ym/yp/zm/zp its
    // neighbours.  INNER: plane k is known to have both z neighbours.
    auto update = [&](auto s_c, auto inner_c, int c, int k, int own, int den, float4 o, float4 ym, float4 yp,
                      float4 zm, float4 zp, const QuadDen &qi, bool hym, bool hyp) __attribute__((always_inline))
        -> float4 {
        constexpr int S = decltype(s_c)::value;
        constexpr bool INNER = decltype(inner_c)::value;
        float xe;
        if constexpr (WARPROW) {
            const float v = S == 0 ? __shfl_up_sync(0xffffffffu, o.w, 1) : __shfl_down_sync(0xffffffffu, o.x, 1);
            xe = (S == 0 ? first : last) ? 0.0f : v;
        } else {
            const int b = slot(c ^ 1, k) + own;
            xe = S == 0 ? lds1(b - 4) : lds1(b + 16);
        }
        const float4 rv = rhs_ld(c, k, own, den);
        if constexpr (PK) {
            if (INNER || (k > 0 && k < D - 1)) return gs_quad_pk(sp.scale, S, rv, o, xe, ym, yp, zm, zp, qi);
            return gs_quad_pk(sp.scale, S, rv, o, xe, ym, yp, zm, zp,
                              quad_den(sp, S, first, last, hym, hyp, k > 0, k < D - 1));
        }
        if (INNER || (k > 0 && k < D - 1)) return gs_quad(sp.scale, S, rv, o, xe, ym, yp, zm, zp, qi);
        return gs_quad(sp.scale, S, rv, o, xe, ym, yp, zm, zp, quad_den(sp, S, first, last, hym, hyp, k > 0, k < D - 1));
    };
    // The four levels of step t.  Every level of a step has, in row A, row
    // parity (jA + t) & 1 (level h: plane t - h, colour h & 1), row B the
    // other one.  MODE 0 checks everything; in steady steps (every level
    // active, every level's plane interior, t + 1 < D) MODE 1 checks only
    // the row masks, and MODE 2 (both rows update on every level) nothing.
    // The arithmetic is the same in every mode.
    auto levels = [&](int t, auto sa_c, auto mode_c) __attribute__((always_inline)) {
        constexpr int SA = decltype(sa_c)::value, SB = 1 - SA;
        constexpr int MODE = decltype(mode_c)::value;
        constexpr bool STEADY = MODE > 0, ROWS = MODE == 2;
        const std::integral_constant<int, SA> sA{};
        const std::integral_constant<int, SB> sB{};
        const std::integral_constant<bool, STEADY> in{};
        const QuadDen &qa = SA ? qA1 : qA0;
        const QuadDen &qb = SB ? qB1 : qB0;
        if (STEADY || kact(0, t)) {
            const int b = slot(1, t);
            if (ROWS || (mA & 1u)) {
                r0A = update(sA, in, 0, t, ownA, denA, b0A, lds4(b + ownA - rowb), b0B, bm1A, bp1A, qa, hymA, hypA);
                sts4(slot(0, t) + ownA, r0A);
            }
            if (ROWS || (mB & 1u)) {
                r0B = update(sB, in, 0, t, ownB, denB, b0B, b0A, lds4(b + ownB + rowb), bm1B, bp1B, qb, hymB, hypB);
                sts4(slot(0, t) + ownB, r0B);
            }
        }
        if (!STEADY && t >= D) { r0A = zero4; r0B = zero4; }
        if (STEADY || kact(1, t - 1)) {
            const int b = slot(0, t - 1), w = slot(1, t - 1);
            if (ROWS || (mA & 2u)) {
                bm1A = update(sA, in, 1, t - 1, ownA, denA, rm1A, lds4(b + ownA - rowb), rm1B, rm2A, r0A, qa, hymA,
                              hypA);
                sts4(w + ownA, bm1A);
            }
            if (ROWS || (mB & 2u)) {
                bm1B = update(sB, in, 1, t - 1, ownB, denB, rm1B, rm1A, lds4(b + ownB + rowb), rm2B, r0B, qb, hymB,
                              hypB);
                sts4(w + ownB, bm1B);
            }
        }
        if (STEADY || kact(2, t - 2)) {
            const int b = slot(1, t - 2), w = slot(0, t - 2);
            if (ROWS || (mA & 4u)) {
                rm2A = update(sA, in, 0, t - 2, ownA, denA, bm2A, lds4(b + ownA - rowb), bm2B, bm3A, bm1A, qa, hymA,
                              hypA);
                sts4(w + ownA, rm2A);
            }
            if (ROWS || (mB & 4u)) {
                rm2B = update(sB, in, 0, t - 2, ownB, denB, bm2B, bm2A, lds4(b + ownB + rowb), bm3B, bm1B, qb, hymB,
                              hypB);
                sts4(w + ownB, rm2B);
            }
        }
        const int k3 = t - 3;
        if (STEADY || kact(3, k3)) {
            const int b = slot(0, k3);
            const bool outp = STEADY || k3 >= z0;
            if (ROWS || (mA & 8u)) {
                bm3A = update(sA, in, 1, k3, ownA, denA, rm3A, lds4(b + ownA - rowb), rm3B, rm4A, rm2A, qa, hymA,
                              hypA);
                if (outp) {
                    *reinterpret_cast<float4 *>(pout_r + offA + k3 * pl) = rm3A;
                    *reinterpret_cast<float4 *>(pout_b + offA + k3 * pl) = bm3A;
                }
            }
            if (ROWS || (mB & 8u)) {
                bm3B = update(sB, in, 1, k3, ownB, denB, rm3B, rm3A, lds4(b + ownB + rowb), rm4B, rm2B, qb, hymB,
                              hypB);
                if (outp) {
                    *reinterpret_cast<float4 *>(pout_r + offB + k3 * pl) = rm3B;
                    *reinterpret_cast<float4 *>(pout_b + offB + k3 * pl) = bm3B;
                }
            }
        }
    };
    // Both rows of this thread update on every level of a steady step.
    const bool rows_full = mA == 15u && mB == 15u;
    // One step of the wavefront; STEADY is CTA-uniform, so every thread
    // meets the same barriers.
    auto step = [&](int t, auto steady_c) __attribute__((always_inline)) -> bool {
        constexpr bool STEADY = decltype(steady_c)::value;
        const bool in1 = STEADY || kin(t + 1);
        if constexpr (TMA) {
            // this step's copies were issued in the previous one; slots are
            // overwritten only after the barrier (their last readers were in
            // the previous step)
            bool ok = wait_red(t);
            if (STEADY || t - 1 >= z0 - 2) ok = wait_black(t - 1) && ok;
            ok = wait_in(t + 1) && ok;
            if (__syncthreads_or(!ok)) {
                // CTA-uniform: stop the pass.  The copies issued in the
                // previous step are the only ones that can still be in
                // flight; wait for them once more before exiting.
                if (leader) atomicAdd(&g_tb_timeouts, 1u);
                wait_red(t);
                if (STEADY || t - 1 >= z0 - 2) wait_black(t - 1);
                wait_in(t + 1);
                return false;
            }
            const int st = (int)(dbase - smc) + (8 + ((t + 1) & 1)) * dslot;
            bp1A = okA && in1 ? lds4(st + denA) : zero4;
            bp1B = okB && in1 ? lds4(st + denB) : zero4;
            __syncthreads();
            prefetch(t + 1, t, t + 2, steady_c);
        } else {
            prefetch(t + 1, t, t + 2, steady_c);      // what the next step reads
            asm volatile("cp.async.wait_group 1;" ::: "memory");
            const int st = STG + ((t + 1) & 1) * slotb;
            bp1A = okA && in1 ? lds4(st + ownA) : zero4;
            bp1B = okB && in1 ? lds4(st + ownB) : zero4;
            __syncthreads();
        }
        if (live) {
            sts4(slot(1, t + 1) + ownA, bp1A);
            sts4(slot(1, t + 1) + ownB, bp1B);
        }
        const bool odd = (jA + t) & 1;
        if constexpr (STEADY) {
            if (rows_full) {
                if (odd) levels(t, std::integral_constant<int, 1>{}, std::integral_constant<int, 2>{});
                else levels(t, std::integral_constant<int, 0>{}, std::integral_constant<int, 2>{});
            } else {
                if (odd) levels(t, std::integral_constant<int, 1>{}, std::integral_constant<int, 1>{});
                else levels(t, std::integral_constant<int, 0>{}, std::integral_constant<int, 1>{});
            }
        } else {
            if (odd) levels(t, std::integral_constant<int, 1>{}, std::integral_constant<int, 0>{});
            else levels(t, std::integral_constant<int, 0>{}, std::integral_constant<int, 0>{});
        }
        rm4A = rm3A; rm3A = rm2A; rm2A = rm1A; rm1A = r0A;
        bm3A = bm2A; bm2A = bm1A; bm1A = b0A; b0A = bp1A;
        rm4B = rm3B; rm3B = rm2B; rm2B = rm1B; rm1B = r0B;
        bm3B = bm2B; bm2B = bm1B; bm1B = b0B; b0B = bp1B;
        return true;
    };
    // Steady steps: t in [ts, te).  From z0 + 3 every level is active; from
    // 4 level 3's plane t - 3 has a z- neighbour; below z1 + 2 every level is
    // active and every prefetch is in range; below D - 2 planes t + 1 and t + 2
    // exist and level 0's plane t has a z+ neighbour.
    const int ts = max(z0 + 3, 4), te = min(z1 + 2, D - 2);
    for (int t = z0 - 3; t < z1 + 3; ++t) {
        const bool ok = t >= ts && t < te ? step(t, std::true_type{}) : step(t, std::false_type{});
        if (!ok) return;
    }
    if constexpr (!TMA) asm volatile("cp.async.wait_group 0;" ::: "memory");
}

template <bool WARPROW, bool TMA, bool PK = false>
__global__ void __launch_bounds__(kTbThreads, 1)
k_rbgs_tb2(Geom g, SolveParams sp, const float *__restrict__ rhs_r, const float *__restrict__ rhs_b,
           const float *__restrict__ pin_b, float *__restrict__ pout_r, float *__restrict__ pout_b, int TY, int ZC,
           const __grid_constant__ CUtensorMap map_r, const __grid_constant__ CUtensorMap map_b,
           const __grid_constant__ CUtensorMap map_in) {
    const int z0 = blockIdx.y * ZC, z1 = z0 + ZC < g.D ? z0 + ZC : g.D;
    tb2_tile<WARPROW, TMA, PK>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, blockIdx.x * TY, z0, z1, threadIdx.x,
                               threadIdx.y, blockDim.y, true, threadIdx.x == 0 && threadIdx.y == 0, &map_r, &map_b,
                               &map_in);
}

static bool tb_supported(const Geom &g) {
    if ((g.W & 7) != 0) return false;
    const int Wq = g.W >> 3;
    return Wq <= 48 && tb_rows_tile(Wq, g.H) >= 1;
}

static size_t tb_smem(const Geom &g, int TY) {
    return sizeof(float4) * kTbSlots * (size_t)tb_rows_alloc(TY) * ((g.W >> 3) + 1);
}

// TMA layout: alignment slack, the dense slots, the 8 padded p slots (never
// more than tb_smem for the 9 or more rows a tile has).
static size_t tb_smem_tma(const Geom &g, int TY) {
    const int Wq = g.W >> 3, ra = tb_rows_alloc(TY);
    return 128 + (size_t)kTbDenseSlots * tb_dense_slot_bytes(Wq, ra) + sizeof(float4) * 8 * (size_t)ra * (Wq + 1);
}

TensorMapEncodeFn tensor_map_encoder() {
    static TensorMapEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TensorMapEncodeFn>(p);
    }
    return fn;
}

// Tensor map of one colour-packed plane stack (Wh x H x D floats) with a box
// of Wh x rows x 1: whole rows from x = 0, so every copy starts 16-byte
// aligned; out-of-range rows and planes read as zeros.
static bool tb_tensor_map(CUtensorMap *m, const float *base, const Geom &g, int rows) {
    TensorMapEncodeFn enc = tensor_map_encoder();
    if (!enc) return false;
    const int Wh = g.W >> 1;
    const cuuint64_t dims[3] = {(cuuint64_t)Wh, (cuuint64_t)g.H, (cuuint64_t)g.D};
    const cuuint64_t strides[2] = {(cuuint64_t)Wh * 4, (cuuint64_t)Wh * g.H * 4};
    const cuuint32_t box[3] = {(cuuint32_t)Wh, (cuuint32_t)rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || Wh > 256 || rows > 256) return false;
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Timeouts counted by the TMA waits since the last call (then reset).
unsigned int tb_take_timeouts() {
    unsigned int n = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&n, g_tb_timeouts, sizeof n) != cudaSuccess) return 0;
    if (n) cudaMemcpyToSymbol(g_tb_timeouts, &zero, sizeof zero);
    return n;
}

static int device_sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cache[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 1;
    }
    return cache[dev];
}

// One pass = two sweeps from (p_in) into (p_out).  ZC <= 0: planes per CTA
// chosen so that the row bands times the z chunks fill the SMs in one wave
// (one CTA per SM: its shared memory is most of the SM's), at least 8
// planes.
static void launch_tb_pass(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                           const float *pin_b, float *pout_r, float *pout_b, int ZC, bool tma, bool pk,
                           cudaStream_t st) {
    const int Wq = g.W >> 3, TY = tb_rows_tile(Wq, g.H);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_rbgs_tb2<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2<false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        attr_set = true;
    }
    CUtensorMap mr{}, mb{}, mi{};
    const int ra = tb_rows_alloc(TY);
    if (tma) tma = tb_tensor_map(&mr, rhs_r, g, ra) && tb_tensor_map(&mb, rhs_b, g, ra) && tb_tensor_map(&mi, pin_b, g, ra);
    const size_t smem = tma ? tb_smem_tma(g, TY) : tb_smem(g, TY);
    if (ZC <= 0) {
        const int bands = (g.H + TY - 1) / TY;
        const int chunks = std::max(1, device_sm_count() / bands);
        ZC = std::max(8, (g.D + chunks - 1) / chunks);
    }
    const dim3 b(Wq, ra / 2, 1);
    const dim3 gr((g.H + TY - 1) / TY, (g.D + ZC - 1) / ZC, 1);
    if (tma) {
        if (Wq == 32)
            k_rbgs_tb2<true, true><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC, mr, mb, mi);
        else
            k_rbgs_tb2<false, true><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC, mr, mb, mi);
    } else if (pk) {
        if (Wq == 32)
            k_rbgs_tb2<true, false, true><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC, mr,
                                                               mb, mi);
        else
            k_rbgs_tb2<false, false, true><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC, mr,
                                                                mb, mi);
    } else {
        if (Wq == 32)
            k_rbgs_tb2<true, false><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC, mr, mb, mi);
        else
            k_rbgs_tb2<false, false><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC, mr, mb,
                                                         mi);
    }
}

// A pass restricted to planes [zlo, zhi) of the grid (one z slab of a grid
// decomposed over ranks): chunk blockIdx.y covers ZC planes from zlo.  A tile
// reads the black input on planes [z0 - 4, z1 + 4) and writes planes
// [z0, z1) only, so on the slab the result is bitwise that of a whole-grid
// pass given the same input on [zlo - 4, zhi + 4).  Loads by cp.async (no
// TMA).
template <bool WARPROW, bool PK>
__global__ void __launch_bounds__(kTbThreads, 1)
k_rbgs_tb2_slab(Geom g, SolveParams sp, const float *__restrict__ rhs_r, const float *__restrict__ rhs_b,
                const float *__restrict__ pin_b, float *__restrict__ pout_r, float *__restrict__ pout_b, int TY,
                int ZC, int zlo, int zhi) {
    const int z0 = zlo + blockIdx.y * ZC, z1 = z0 + ZC < zhi ? z0 + ZC : zhi;
    tb2_tile<WARPROW, false, PK>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, blockIdx.x * TY, z0, z1,
                                 threadIdx.x, threadIdx.y, blockDim.y, true, threadIdx.x == 0 && threadIdx.y == 0,
                                 nullptr, nullptr, nullptr);
}

bool slab_pass_supported(const Geom &g) { return tb_supported(g); }

void launch_tb_pass_slab(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                         const float *pin_b, float *pout_r, float *pout_b, int zlo, int zhi, bool pk,
                         cudaStream_t st) {
    const int Wq = g.W >> 3, TY = tb_rows_tile(Wq, g.H);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_rbgs_tb2_slab<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2_slab<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2_slab<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_rbgs_tb2_slab<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        attr_set = true;
    }
    const int ra = tb_rows_alloc(TY);
    const size_t smem = tb_smem(g, TY);
    // z chunks so that the row bands times the chunks fill the SMs, at least 8 planes
    const int bands = (g.H + TY - 1) / TY, depth = zhi - zlo;
    const int chunks = std::max(1, device_sm_count() / bands);
    const int ZC = std::max(8, (depth + chunks - 1) / chunks);
    const dim3 b(Wq, ra / 2, 1);
    const dim3 gr(bands, (depth + ZC - 1) / ZC, 1);
    if (pk) {
        if (Wq == 32)
            k_rbgs_tb2_slab<true, true><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC,
                                                             zlo, zhi);
        else
            k_rbgs_tb2_slab<false, true><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC,
                                                              zlo, zhi);
    } else {
        if (Wq == 32)
            k_rbgs_tb2_slab<true, false><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC,
                                                              zlo, zhi);
        else
            k_rbgs_tb2_slab<false, false><<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC,
                                                               zlo, zhi);
    }
}

// (planes per thread, rows per block) of each segment-kernel variant; the
// variants after them are the temporal-blocking pass with ZC planes per CTA
// (0: sized to fill the SMs): 9 with its rhs and input planes staged by TMA,
// 10 with the stencil on paired FP32 instructions (gs_quad_pk).
static const int kVariantKZ[kSegVariants] = {1, 2, 4, 8, 2, 4};
static const int kVariantBY[kSegVariants] = {8, 8, 4, 4, 4, 8};
static const int kVariantZC[kSweepVariants - kSegVariants] = {16, 32, 0, 0, 0};
static const bool kVariantTMA[kSweepVariants - kSegVariants] = {false, false, false, true, false};
static const bool kVariantPK[kSweepVariants - kSegVariants] = {false, false, false, false, true};

bool sweep_variant_uses_tma(int v) { return v >= kSegVariants && v < kSweepVariants && kVariantTMA[v - kSegVariants]; }

int sweep_variant_count(const Geom &g) {
    if ((g.W & 7) != 0) return 0;
    return tb_supported(g) ? kSweepVariants : kSegVariants;
}

void launch_rbgs_sweeps(const Geom &g, const SolveParams &sp, const float *rhs_r,
                        const float *rhs_b, float *p_r, float *p_b, int sweeps, cudaStream_t st,
                        long long *launches, int variant, float *q_r, float *q_b) {
    if (variant >= kSegVariants && variant < kSweepVariants && q_r && q_b && tb_supported(g)) {
        // Passes alternate p -> q -> p, an even number of them, so the
        // result lands in p; the remaining sweeps run unblocked.
        const int passes = (sweeps / 4) * 2;
        const int zc = kVariantZC[variant - kSegVariants];
        const bool tma = kVariantTMA[variant - kSegVariants], pk = kVariantPK[variant - kSegVariants];
        for (int i = 0; i < passes; ++i) {
            if ((i & 1) == 0) launch_tb_pass(g, sp, rhs_r, rhs_b, p_b, q_r, q_b, zc, tma, pk, st);
            else launch_tb_pass(g, sp, rhs_r, rhs_b, q_b, p_r, p_b, zc, tma, pk, st);
        }
        *launches += passes;
        sweeps -= 2 * passes;
        variant = 2;
    }
    if (sweeps <= 0) return;
    if ((g.W & 7) == 0) {
        const int v = (variant >= 0 && variant < kSegVariants) ? variant : 0;
        const int Wq = g.W >> 3, kz = kVariantKZ[v], by = kVariantBY[v];
        const int bx = std::min(32, Wq);
        const dim3 b(bx, std::max(1, std::min(by * (32 / bx), 256 / bx)), 1);
        const dim3 gr((Wq + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, (g.D + kz - 1) / kz);
        for (int it = 0; it < sweeps; ++it) {
            for (int c = 0; c < 2; ++c) {
                const float *rc = c ? rhs_b : rhs_r;
                const float *po = c ? p_r : p_b;
                float *pc = c ? p_b : p_r;
                switch (kz) {
                case 1: k_rbgs_seg<1><<<gr, b, 0, st>>>(g, sp, rc, po, pc, c); break;
                case 2: k_rbgs_seg<2><<<gr, b, 0, st>>>(g, sp, rc, po, pc, c); break;
                case 4: k_rbgs_seg<4><<<gr, b, 0, st>>>(g, sp, rc, po, pc, c); break;
                default: k_rbgs_seg<8><<<gr, b, 0, st>>>(g, sp, rc, po, pc, c); break;
                }
            }
        }
    } else {
        const dim3 b(32, 8, 1);
        const dim3 gr(((g.W >> 1) + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, g.D);
        for (int it = 0; it < sweeps; ++it) {
            k_rbgs_half<<<gr, b, 0, st>>>(g, sp, rhs_r, p_b, p_r, 0);
            k_rbgs_half<<<gr, b, 0, st>>>(g, sp, rhs_b, p_r, p_b, 1);
        }
    }
    *launches += 2LL * sweeps;
}

// The reference's schedule made race free (FluidSolver.cu:517-599): plane by
// plane, cells with (i+j) even first, then (i+j) odd.  In plane k the 2-D
// colour (i+j)&1 equals the 3-D colour xor (k&1), so a 2-D half plane is one
// packed colour array restricted to plane k.
__global__ void k_plane_half(Geom g, SolveParams sp, const float *__restrict__ rhs_c,
                             const float *__restrict__ p_o, float *__restrict__ p_c, int colour,
                             int k) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int Wh = g.W >> 1;
    if (m >= Wh || j >= g.H) return;
    const int s = (j + k + colour) & 1;
    const int i = 2 * m + s;
    const size_t q = pidx(i, j, k, Wh, g.H);
    p_c[q] = gs_update(g, sp, __ldg(rhs_c + q), p_o, q, i, j, k, s, Wh);
}

void launch_plane_sweeps(const Geom &g, const SolveParams &sp, const float *rhs_r,
                         const float *rhs_b, float *p_r, float *p_b, int sweeps, cudaStream_t st,
                         long long *launches) {
    const dim3 b(32, 8, 1);
    const dim3 gr(((g.W >> 1) + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, 1);
    for (int it = 0; it < sweeps; ++it)
        for (int k = 0; k < g.D; ++k) {
            // 2-D colour 0 ((i+j) even) is 3-D colour (k & 1).
            const int c0 = k & 1, c1 = c0 ^ 1;
            k_plane_half<<<gr, b, 0, st>>>(g, sp, c0 ? rhs_b : rhs_r, c0 ? p_r : p_b, c0 ? p_b : p_r, c0, k);
            k_plane_half<<<gr, b, 0, st>>>(g, sp, c1 ? rhs_b : rhs_r, c1 ? p_r : p_b, c1 ? p_b : p_r, c1, k);
        }
    *launches += 2LL * sweeps * g.D;
}

// ---------------------------------------------------------------------------
// FP64 residual ||b - A p||_2 and ||b||_2, b = scale*rhs.  Grid-stride over
// row segments with a fixed launch shape, warp-shuffle then shared-memory
// reduction per block, then one block sums the per-block partials in order:
// the result is bit-reproducible.  Per cell, A p is formed in deviation form
// sum_nb (p_c - p_nb) (+ p_c per Dirichlet ghost): differences of a smooth
// pressure are exact in FP32, so the stencil loses nothing to the magnitude
// of p; b and r are then FP64 and the squares accumulate in FP64.
// ---------------------------------------------------------------------------
constexpr int kResThreads = 256;

// Tiles of the z-marching residual (W % 8 == 0 and W <= 2048): a block of
// kResThreads threads covers kResThreads / Wq rows of quads and kResKZ planes.
// 16 planes and at most 64 registers (four blocks per SM): at 256^3 the 512
// tiles are one wave, with 32 warps per SM waiting on DRAM.
constexpr int kResKZ = 16;
constexpr int kResBlocksPerSM = 4;

__host__ __device__ inline bool residual_tiled(const Geom &g) { return (g.W & 7) == 0 && (g.W >> 3) <= kResThreads; }
__host__ __device__ inline int residual_tile_rows(const Geom &g) { return kResThreads / (g.W >> 3); }
__host__ __device__ inline int residual_tiles_y(const Geom &g) {
    const int R = residual_tile_rows(g);
    return (g.H + R - 1) / R;
}

__host__ __device__ inline int residual_tiles(const Geom &g) {
    return residual_tiles_y(g) * ((g.D + kResKZ - 1) / kResKZ);
}

// Partial sums one residual of g produces: one per tile, else one per block.
int residual_blocks(const Geom &g) {
    if (residual_tiled(g)) return residual_tiles(g);
    const long long items = (long long)(g.W >> 1) * g.H * g.D / ((g.W & 7) == 0 ? 4 : 1);
    return (int)std::min<long long>((items + kResThreads - 1) / kResThreads, 148 * 8);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float ghost_terms(const SolveParams &sp, bool has_xm, bool has_xp, bool has_ym,
                                             bool has_yp, bool has_zm, bool has_zp) {
    if (!sp.dirichlet) return 0.0f;
    const OpenFaces &o = sp.open;
    return (float)((!has_xm && o.xlo) + (!has_xp && o.xhi) + (!has_ym && o.ylo) + (!has_yp && o.yhi) +
                   (!has_zm && o.zlo) + (!has_zp && o.zhi));
}

// Residual contributions of four packed cells of one colour (layout as in
// gs_segment; own = this colour's values).
__device__ __forceinline__ void residual_segment(const SolveParams &sp, double scale, int s, bool first,
                                                 bool last, float4 rhs, float4 own, float4 o, float xe,
                                                 float4 ym, float4 yp, float4 zm, float4 zp, bool has_ym,
                                                 bool has_yp, bool has_zm, bool has_zp, double &r2,
                                                 double &b2) {
    float xl[4], xr[4];
    if (s == 0) {
        xl[0] = xe; xl[1] = o.x; xl[2] = o.y; xl[3] = o.z;
        xr[0] = o.x; xr[1] = o.y; xr[2] = o.z; xr[3] = o.w;
    } else {
        xl[0] = o.x; xl[1] = o.y; xl[2] = o.z; xl[3] = o.w;
        xr[0] = o.y; xr[1] = o.z; xr[2] = o.w; xr[3] = xe;
    }
    const float ra[4] = {rhs.x, rhs.y, rhs.z, rhs.w}, pa[4] = {own.x, own.y, own.z, own.w};
    const float yma[4] = {ym.x, ym.y, ym.z, ym.w}, ypa[4] = {yp.x, yp.y, yp.z, yp.w};
    const float zma[4] = {zm.x, zm.y, zm.z, zm.w}, zpa[4] = {zp.x, zp.y, zp.z, zp.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const bool has_xm = !(s == 0 && first && t == 0);
        const bool has_xp = !(s == 1 && last && t == 3);
        const float pc = pa[t];
        float d = ghost_terms(sp, has_xm, has_xp, has_ym, has_yp, has_zm, has_zp) * pc;
        if (has_xm) d += pc - xl[t];
        if (has_xp) d += pc - xr[t];
        if (has_ym) d += pc - yma[t];
        if (has_yp) d += pc - ypa[t];
        if (has_zm) d += pc - zma[t];
        if (has_zp) d += pc - zpa[t];
        const double b = scale * (double)ra[t];
        const double r = b - (double)d;
        r2 += r * r;
        b2 += b * b;
    }
}

// Block `blk` of `nblk` of the segment residual: grid-stride over the row
// segments, then the block's FP64 sums go to partials[2*blk], [2*blk + 1].
__device__ __forceinline__ void residual_seg_block(const Geom &g, const SolveParams &sp, double scale,
                                                   const float *__restrict__ rr, const float *__restrict__ rb,
                                                   const float *__restrict__ pr, const float *__restrict__ pb,
                                                   int blk, int nblk, double *__restrict__ partials) {
    const int Wh = g.W >> 1, Wq = Wh >> 2;
    const int items = Wq * g.H * g.D;
    const int pl = Wh * g.H;
    double r2 = 0.0, b2 = 0.0;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int t = blk * kResThreads + threadIdx.x; t < items; t += nblk * kResThreads) {
        const int mq = t % Wq, jk = t / Wq;
        const int j = jk % g.H, k = jk / g.H;
        const int m0 = 4 * mq;
        const int q = m0 + Wh * j + pl * k;
        const bool has_ym = j > 0, has_yp = j < g.H - 1, has_zm = k > 0, has_zp = k < g.D - 1;
        const bool first = m0 == 0, last = m0 + 4 == Wh;
        const float4 pr4 = ld4(pr + q), pb4 = ld4(pb + q);
        const int sr = (j + k) & 1, sb = sr ^ 1;        // red / black row offsets
        // red cells: the other colour is black
        residual_segment(sp, scale, sr, first, last, ld4(rr + q), pr4, pb4,
                         sr == 0 ? (first ? 0.f : __ldg(pb + q - 1)) : (last ? 0.f : __ldg(pb + q + 4)),
                         has_ym ? ld4(pb + q - Wh) : zero4, has_yp ? ld4(pb + q + Wh) : zero4,
                         has_zm ? ld4(pb + q - pl) : zero4, has_zp ? ld4(pb + q + pl) : zero4,
                         has_ym, has_yp, has_zm, has_zp, r2, b2);
        residual_segment(sp, scale, sb, first, last, ld4(rb + q), pb4, pr4,
                         sb == 0 ? (first ? 0.f : __ldg(pr + q - 1)) : (last ? 0.f : __ldg(pr + q + 4)),
                         has_ym ? ld4(pr + q - Wh) : zero4, has_yp ? ld4(pr + q + Wh) : zero4,
                         has_zm ? ld4(pr + q - pl) : zero4, has_zp ? ld4(pr + q + pl) : zero4,
                         has_ym, has_yp, has_zm, has_zp, r2, b2);
    }
    __shared__ double s_r[kResThreads / 32], s_b[kResThreads / 32];
    r2 = warp_sum(r2);
    b2 = warp_sum(b2);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_r[wid] = r2; s_b[wid] = b2; }
    __syncthreads();
    if (wid == 0) {
        r2 = lane < kResThreads / 32 ? s_r[lane] : 0.0;
        b2 = lane < kResThreads / 32 ? s_b[lane] : 0.0;
        r2 = warp_sum(r2);
        b2 = warp_sum(b2);
        if (lane == 0) { partials[2 * blk] = r2; partials[2 * blk + 1] = b2; }
    }
}

__device__ __forceinline__ void block_pair_sum(double r2, double b2, double *__restrict__ out) {
    __shared__ double s_r[kResThreads / 32], s_b[kResThreads / 32];
    r2 = warp_sum(r2);
    b2 = warp_sum(b2);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_r[wid] = r2; s_b[wid] = b2; }
    __syncthreads();
    if (wid == 0) {
        r2 = lane < kResThreads / 32 ? s_r[lane] : 0.0;
        b2 = lane < kResThreads / 32 ? s_b[lane] : 0.0;
        r2 = warp_sum(r2);
        b2 = warp_sum(b2);
        if (lane == 0) { out[0] = r2; out[1] = b2; }
    }
    __syncthreads();                                  // s_r / s_b are reused by the block's next tile
}

// Tile `blk` of the z-marching residual: each thread takes one quad of a row
// through kResKZ planes, carrying both colours' quads of planes k-1, k, k+1
// in registers (one new plane of each per step), red cells then black cells
// per plane; the block's FP64 sums go to partials[2*blk], [2*blk + 1].
__device__ __forceinline__ void residual_tile_block(const Geom &g, const SolveParams &sp, double scale,
                                                    const float *__restrict__ rr, const float *__restrict__ rb,
                                                    const float *__restrict__ pr, const float *__restrict__ pb,
                                                    int blk, double *__restrict__ partials) {
    const int Wh = g.W >> 1, Wq = Wh >> 2;
    const int R = residual_tile_rows(g), ty = residual_tiles_y(g);
    const int t = threadIdx.x;
    const int mq = t % Wq, jr = t / Wq;
    const int j = (blk % ty) * R + jr, k0 = (blk / ty) * kResKZ;
    double r2 = 0.0, b2 = 0.0;
    if (jr < R && j < g.H) {
        const size_t pl = (size_t)Wh * g.H;
        const size_t row = (size_t)4 * mq + (size_t)Wh * j;
        const bool has_ym = j > 0, has_yp = j < g.H - 1;
        const bool first = mq == 0, last = 4 * mq + 4 == Wh;
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 rm = k0 > 0 ? ld4(pr + row + (k0 - 1) * pl) : zero4, bm = k0 > 0 ? ld4(pb + row + (k0 - 1) * pl) : zero4;
        float4 rc = ld4(pr + row + k0 * pl), bc = ld4(pb + row + k0 * pl);
        const int k1 = k0 + kResKZ < g.D ? k0 + kResKZ : g.D;
        for (int k = k0; k < k1; ++k) {
            const size_t q = row + (size_t)k * pl;
            const bool has_zm = k > 0, has_zp = k < g.D - 1;
            const float4 rp = has_zp ? ld4(pr + q + pl) : zero4, bp = has_zp ? ld4(pb + q + pl) : zero4;
            const int sr = (j + k) & 1, sb = sr ^ 1;
            residual_segment(sp, scale, sr, first, last, ld4(rr + q), rc, bc,
                             sr == 0 ? (first ? 0.f : __ldg(pb + q - 1)) : (last ? 0.f : __ldg(pb + q + 4)),
                             has_ym ? ld4(pb + q - Wh) : zero4, has_yp ? ld4(pb + q + Wh) : zero4, bm, bp,
                             has_ym, has_yp, has_zm, has_zp, r2, b2);
            residual_segment(sp, scale, sb, first, last, ld4(rb + q), bc, rc,
                             sb == 0 ? (first ? 0.f : __ldg(pr + q - 1)) : (last ? 0.f : __ldg(pr + q + 4)),
                             has_ym ? ld4(pr + q - Wh) : zero4, has_yp ? ld4(pr + q + Wh) : zero4, rm, rp,
                             has_ym, has_yp, has_zm, has_zp, r2, b2);
            rm = rc; rc = rp; bm = bc; bc = bp;
        }
    }
    block_pair_sum(r2, b2, partials + 2 * (size_t)blk);
}

// The residual blocks of one grid (residual_blocks(g) of them): tiles when
// residual_tiled(g), else the grid-stride segments.
__device__ __forceinline__ void residual_block(const Geom &g, const SolveParams &sp, double scale,
                                               const float *__restrict__ rr, const float *__restrict__ rb,
                                               const float *__restrict__ pr, const float *__restrict__ pb, int blk,
                                               int nblk, double *__restrict__ partials) {
    if (residual_tiled(g)) residual_tile_block(g, sp, scale, rr, rb, pr, pb, blk, partials);
    else residual_seg_block(g, sp, scale, rr, rb, pr, pb, blk, nblk, partials);
}

// One block per tile when residual_tiled(g), else grid-stride segments.
__global__ void __launch_bounds__(kResThreads, kResBlocksPerSM)
k_residual_seg(Geom g, SolveParams sp, double scale, const float *__restrict__ rr,
               const float *__restrict__ rb, const float *__restrict__ pr, const float *__restrict__ pb,
               double *__restrict__ partials) {
    residual_block(g, sp, scale, rr, rb, pr, pb, blockIdx.x, gridDim.x, partials);
}

// One packed pair per item (any even W).
__global__ void __launch_bounds__(kResThreads)
k_residual(Geom g, SolveParams sp, double scale, const float *__restrict__ rr,
           const float *__restrict__ rb, const float *__restrict__ pr, const float *__restrict__ pb,
           double *__restrict__ partials) {
    const int Wh = g.W >> 1;
    const int items = Wh * g.H * g.D;
    double r2 = 0.0, b2 = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < items; t += gridDim.x * blockDim.x) {
        const int m = t % Wh, jk = t / Wh;
        const int j = jk % g.H, k = jk / g.H;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * m + h;
            const bool black = (i + j + k) & 1;
            const double b = scale * (double)__ldg((black ? rb : rr) + t);
            const float pc = __ldg((black ? pb : pr) + t);
            const bool has_xm = i > 0, has_xp = i < g.W - 1, has_ym = j > 0, has_yp = j < g.H - 1;
            const bool has_zm = k > 0, has_zp = k < g.D - 1;
            float d = ghost_terms(sp, has_xm, has_xp, has_ym, has_yp, has_zm, has_zp) * pc;
            if (has_xm) d += pc - pval(pr, pb, i - 1, j, k, Wh, g.H);
            if (has_xp) d += pc - pval(pr, pb, i + 1, j, k, Wh, g.H);
            if (has_ym) d += pc - pval(pr, pb, i, j - 1, k, Wh, g.H);
            if (has_yp) d += pc - pval(pr, pb, i, j + 1, k, Wh, g.H);
            if (has_zm) d += pc - pval(pr, pb, i, j, k - 1, Wh, g.H);
            if (has_zp) d += pc - pval(pr, pb, i, j, k + 1, Wh, g.H);
            const double r = b - (double)d;
            r2 += r * r;
            b2 += b * b;
        }
    }
    __shared__ double s_r[kResThreads / 32], s_b[kResThreads / 32];
    r2 = warp_sum(r2);
    b2 = warp_sum(b2);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_r[wid] = r2; s_b[wid] = b2; }
    __syncthreads();
    if (wid == 0) {
        r2 = lane < kResThreads / 32 ? s_r[lane] : 0.0;
        b2 = lane < kResThreads / 32 ? s_b[lane] : 0.0;
        r2 = warp_sum(r2);
        b2 = warp_sum(b2);
        if (lane == 0) { partials[2 * blockIdx.x] = r2; partials[2 * blockIdx.x + 1] = b2; }
    }
}

// Sums n {r2, b2} pairs in a fixed order with one 1024-thread block; lane 0
// of warp 0 writes the totals to out2 (global or shared memory).
__device__ __forceinline__ void reduce_pairs_block(const double *__restrict__ partials, int n, double *out2) {
    __shared__ double s_r[32], s_b[32];
    double r2 = 0.0, b2 = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) { r2 += partials[2 * t]; b2 += partials[2 * t + 1]; }
    r2 = warp_sum(r2);
    b2 = warp_sum(b2);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_r[wid] = r2; s_b[wid] = b2; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x / 32;
        r2 = lane < nw ? s_r[lane] : 0.0;
        b2 = lane < nw ? s_b[lane] : 0.0;
        r2 = warp_sum(r2);
        b2 = warp_sum(b2);
        if (lane == 0) { out2[0] = r2; out2[1] = b2; }
    }
}

__global__ void __launch_bounds__(1024) k_reduce_pairs(const double *__restrict__ partials, int n,
                                                       double *__restrict__ out2) {
    reduce_pairs_block(partials, n, out2);
}

int launch_residual(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                    const float *p_r, const float *p_b, double *partials, int max_partials,
                    double *out2, cudaStream_t st) {
    // max_partials is residual_blocks(g) (the partials buffer of the solver)
    const int parts = std::min(residual_blocks(g), max_partials);
    const double scale = (double)sp.scale_d;
    if ((g.W & 7) == 0) {
        k_residual_seg<<<parts, kResThreads, 0, st>>>(g, sp, scale, rhs_r, rhs_b, p_r, p_b, partials);
    } else {
        k_residual<<<parts, kResThreads, 0, st>>>(g, sp, scale, rhs_r, rhs_b, p_r, p_b, partials);
    }
    k_reduce_pairs<<<1, 1024, 0, st>>>(partials, parts, out2);
    return 2;
}

// The residual tiles blk0 .. blk0 + gridDim.x - 1 of a tiled grid (the
// tiles of a z slab), partial sums at their whole-grid indices.
__global__ void __launch_bounds__(kResThreads, kResBlocksPerSM)
k_residual_tiles(Geom g, SolveParams sp, double scale, const float *__restrict__ rr,
                 const float *__restrict__ rb, const float *__restrict__ pr, const float *__restrict__ pb, int blk0,
                 double *__restrict__ partials) {
    residual_tile_block(g, sp, scale, rr, rb, pr, pb, blk0 + (int)blockIdx.x, partials);
}

int residual_slab_tiles(const Geom &g, int z0, int z1, int *first, int *count) {
    if (!residual_tiled(g) || z0 < 0 || z1 > g.D || z0 >= z1 || z0 % kResKZ != 0 || (z1 % kResKZ != 0 && z1 != g.D))
        return -1;
    const int ty = residual_tiles_y(g);
    *first = (z0 / kResKZ) * ty;
    *count = ((z1 + kResKZ - 1) / kResKZ - z0 / kResKZ) * ty;
    return 0;
}

int launch_residual_slab(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                         const float *p_r, const float *p_b, int z0, int z1, double *partials, cudaStream_t st) {
    int first = 0, count = 0;
    if (residual_slab_tiles(g, z0, z1, &first, &count) != 0) return -1;
    k_residual_tiles<<<count, kResThreads, 0, st>>>(g, sp, (double)sp.scale_d, rhs_r, rhs_b, p_r, p_b, first,
                                                     partials);
    return 1;
}

void launch_reduce_pairs(const double *partials, int n, double *out2, cudaStream_t st) {
    k_reduce_pairs<<<1, 1024, 0, st>>>(partials, n, out2);
}

// pressure_gradient_update_kernel (FluidSolver.cu:601-669).  Interior faces
// subtract dt/(rho dx) * grad p.  Domain faces: 0 at a wall; at an open face
// REF_COMPAT copies the inner neighbour's updated value (the reference's copy,
// read after the update; the thread of the inner face writes both, so no
// thread reads a face another thread writes), FREE_SURFACE applies the
// gradient against the p = 0 ghost.
// DEFECT: the pressure is p0 + delta (the defect-correction solve, p0 in
// pr/pb and delta in dr/db); each difference is formed as
// (p0_a - p0_b) + (delta_a - delta_b), so the gradient keeps the correction's
// digits that p0 + delta rounded to FP32 would lose.
template <bool DEFECT>
__global__ void k_gradient(Geom g, SolveParams sp, float s, const float *__restrict__ pr,
                           const float *__restrict__ pb, float *__restrict__ U,
                           float *__restrict__ V, float *__restrict__ W, const float *__restrict__ dr,
                           const float *__restrict__ db) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.W || j > g.H || k > g.D) return;
    const int Wh = g.W >> 1, H = g.H;
    const OpenFaces &o = sp.open;
    const bool dir = sp.dirichlet;
    auto P = [&](int a, int b, int c) { return pval(pr, pb, a, b, c, Wh, H); };
    // p(a) - p(b), and p(a) alone (the difference to a Dirichlet ghost)
    auto dP = [&](int a1, int b1, int c1, int a2, int b2, int c2) -> float {
        if (DEFECT)
            return (P(a1, b1, c1) - P(a2, b2, c2)) + (pval(dr, db, a1, b1, c1, Wh, H) - pval(dr, db, a2, b2, c2, Wh, H));
        return P(a1, b1, c1) - P(a2, b2, c2);
    };
    auto P1 = [&](int a, int b, int c) -> float {
        if (DEFECT) return (P(a, b, c) - 0.0f) + (pval(dr, db, a, b, c, Wh, H) - 0.0f);
        return P(a, b, c) - 0.0f;
    };
    auto P1n = [&](int a, int b, int c) -> float {       // 0 - p(a)
        if (DEFECT) return (0.0f - P(a, b, c)) + (0.0f - pval(dr, db, a, b, c, Wh, H));
        return 0.0f - P(a, b, c);
    };
    if (j < g.H && k < g.D) {
        const size_t q = lin(i, j, k, g.W + 1, g.H);
        if (i > 0 && i < g.W) {
            const float u = U[q] - s * dP(i, j, k, i - 1, j, k);
            U[q] = u;
            if (!dir && i == 1 && o.xlo) U[q - 1] = u;
            if (!dir && i == g.W - 1 && o.xhi) U[q + 1] = u;
        } else if (i == 0) {
            if (!o.xlo) U[q] = 0.0f;
            else if (dir) U[q] -= s * P1(0, j, k);
        } else {
            if (!o.xhi) U[q] = 0.0f;
            else if (dir) U[q] -= s * P1n(g.W - 1, j, k);
        }
    }
    if (i < g.W && k < g.D) {
        const size_t q = lin(i, j, k, g.W, g.H + 1);
        const size_t row = (size_t)g.W;
        if (j > 0 && j < g.H) {
            const float v = V[q] - s * dP(i, j, k, i, j - 1, k);
            V[q] = v;
            if (!dir && j == 1 && o.ylo) V[q - row] = v;
            if (!dir && j == g.H - 1 && o.yhi) V[q + row] = v;
        } else if (j == 0) {
            if (!o.ylo) V[q] = 0.0f;
            else if (dir) V[q] -= s * P1(i, 0, k);
        } else {
            if (!o.yhi) V[q] = 0.0f;
            else if (dir) V[q] -= s * P1n(i, g.H - 1, k);
        }
    }
    if (i < g.W && j < g.H) {
        const size_t q = lin(i, j, k, g.W, g.H);
        const size_t plane = (size_t)g.W * g.H;
        if (k > 0 && k < g.D) {
            const float w = W[q] - s * dP(i, j, k, i, j, k - 1);
            W[q] = w;
            if (!dir && k == 1 && o.zlo) W[q - plane] = w;
            if (!dir && k == g.D - 1 && o.zhi) W[q + plane] = w;
        } else if (k == 0) {
            if (!o.zlo) W[q] = 0.0f;
            else if (dir) W[q] -= s * P1(i, j, 0);
        } else {
            if (!o.zhi) W[q] = 0.0f;
            else if (dir) W[q] -= s * P1n(i, j, g.D - 1);
        }
    }
}

void launch_gradient(const Geom &g, const SolveParams &sp, float s, const float *p_r,
                     const float *p_b, float *U, float *V, float *W, cudaStream_t st, const float *d_r,
                     const float *d_b) {
    if (d_r && d_b)
        k_gradient<true><<<face_grid(g), face_block(), 0, st>>>(g, sp, s, p_r, p_b, U, V, W, d_r, d_b);
    else
        k_gradient<false><<<face_grid(g), face_block(), 0, st>>>(g, sp, s, p_r, p_b, U, V, W, nullptr, nullptr);
}

// The defect of the current pressure for the defect-correction solve, in
// FP64 from the FP32 arrays: with b = scale * rhs, the sweeps' right-hand side
// rhs' = (b - A p) / scale (stored FP32; the sweeps solve A delta = b - A p
// for the correction delta) and the residual of the pressure p + delta,
// r = b - A p - A delta (both stencils in deviation form, exact in FP64).
// Per-block partial sums of r^2 and b^2 go to part[2 * block] and
// part[2 * block + 1]; k_defect_total sums them in block order into
// out2 = {||r||^2, ||b||^2}.
constexpr int kDefectThreads = 256;
constexpr int kDefectBlocks = 1184;

__device__ __forceinline__ double stencil64(const float *__restrict__ pr, const float *__restrict__ pb, int i, int j,
                                            int k, int W, int H, int D, int Wh, const OpenFaces &o, bool dir) {
    const double pc = (double)pval(pr, pb, i, j, k, Wh, H);
    double d = 0.0;
    if (i > 0) d += pc - (double)pval(pr, pb, i - 1, j, k, Wh, H); else if (dir && o.xlo) d += pc;
    if (i < W - 1) d += pc - (double)pval(pr, pb, i + 1, j, k, Wh, H); else if (dir && o.xhi) d += pc;
    if (j > 0) d += pc - (double)pval(pr, pb, i, j - 1, k, Wh, H); else if (dir && o.ylo) d += pc;
    if (j < H - 1) d += pc - (double)pval(pr, pb, i, j + 1, k, Wh, H); else if (dir && o.yhi) d += pc;
    if (k > 0) d += pc - (double)pval(pr, pb, i, j, k - 1, Wh, H); else if (dir && o.zlo) d += pc;
    if (k < D - 1) d += pc - (double)pval(pr, pb, i, j, k + 1, Wh, H); else if (dir && o.zhi) d += pc;
    return d;
}

__global__ void __launch_bounds__(kDefectThreads)
k_defect(Geom g, SolveParams sp, const float *__restrict__ rhs_r, const float *__restrict__ rhs_b,
         const float *__restrict__ pr, const float *__restrict__ pb, const float *__restrict__ dr,
         const float *__restrict__ db, float *__restrict__ def_r, float *__restrict__ def_b,
         double *__restrict__ part) {
    const int Wh = g.W >> 1, H = g.H;
    const long long n = (long long)g.W * g.H * g.D;
    double r2 = 0.0, b2 = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.W), j = (int)((c / g.W) % g.H), k = (int)(c / ((long long)g.W * g.H));
        const size_t q = pidx(i, j, k, Wh, H);
        const bool black = (i + j + k) & 1;
        const double b = sp.scale_d * (double)(black ? rhs_b : rhs_r)[q];
        const double bp = b - stencil64(pr, pb, i, j, k, g.W, g.H, g.D, Wh, sp.open, sp.dirichlet);
        (black ? def_b : def_r)[q] = (float)(bp / sp.scale_d);
        const double r = bp - stencil64(dr, db, i, j, k, g.W, g.H, g.D, Wh, sp.open, sp.dirichlet);
        r2 += r * r;
        b2 += b * b;
    }
    __shared__ double sr[kDefectThreads], sb[kDefectThreads];
    sr[threadIdx.x] = r2;
    sb[threadIdx.x] = b2;
    __syncthreads();
    for (int t = kDefectThreads / 2; t > 0; t >>= 1) {
        if (threadIdx.x < t) { sr[threadIdx.x] += sr[threadIdx.x + t]; sb[threadIdx.x] += sb[threadIdx.x + t]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = sr[0]; part[2 * blockIdx.x + 1] = sb[0]; }
}

__global__ void k_defect_total(const double *__restrict__ part, int nb, double *__restrict__ out2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double r2 = 0.0, b2 = 0.0;
    for (int t = 0; t < nb; ++t) { r2 += part[2 * t]; b2 += part[2 * t + 1]; }
    out2[0] = r2;
    out2[1] = b2;
}

// p = RN(p + delta) and delta = (p + delta) - RN(p + delta), exactly (Knuth's
// TwoSum: the rounding error of a float sum is itself a float), over both
// colours: the folded pressure after a defect solve, with nothing lost.
__device__ __forceinline__ void two_sum(float &a, float &b) {
    const float s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    const float ap = __fsub_rn(s, bp);
    b = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
    a = s;
}
__global__ void k_fold(long long n, float *__restrict__ pr, float *__restrict__ pb, float *__restrict__ dr,
                       float *__restrict__ db) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        float a = pr[t], b = dr[t];
        two_sum(a, b);
        pr[t] = a;
        dr[t] = b;
        a = pb[t];
        b = db[t];
        two_sum(a, b);
        pb[t] = a;
        db[t] = b;
    }
}

int launch_defect(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b, const float *p_r,
                  const float *p_b, const float *d_r, const float *d_b, float *def_r, float *def_b, double *partials,
                  int max_partials, double *out2, cudaStream_t st) {
    const int nb = std::min(kDefectBlocks, max_partials);
    k_defect<<<nb, kDefectThreads, 0, st>>>(g, sp, rhs_r, rhs_b, p_r, p_b, d_r, d_b, def_r, def_b, partials);
    k_defect_total<<<1, 32, 0, st>>>(partials, nb, out2);
    return 2;
}

void launch_fold(const Geom &g, float *p_r, float *p_b, float *d_r, float *d_b, cudaStream_t st) {
    const long long n = (long long)g.W * g.H * g.D / 2;
    k_fold<<<(int)std::min<long long>((n + 255) / 256, 4736), 256, 0, st>>>(n, p_r, p_b, d_r, d_b);
}

__global__ void k_pack(Geom g, const float *__restrict__ nat, float *__restrict__ red,
                       float *__restrict__ black) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int Wh = g.W >> 1;
    if (m >= Wh || j >= g.H) return;
    const float a = nat[lin(2 * m, j, k, g.W, g.H)], b = nat[lin(2 * m + 1, j, k, g.W, g.H)];
    const size_t q = pidx(2 * m, j, k, Wh, g.H);
    const bool even_red = ((j + k) & 1) == 0;
    red[q] = even_red ? a : b;
    black[q] = even_red ? b : a;
}

__global__ void k_unpack(Geom g, const float *__restrict__ red, const float *__restrict__ black,
                         float *__restrict__ nat) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int Wh = g.W >> 1;
    if (m >= Wh || j >= g.H) return;
    const size_t q = pidx(2 * m, j, k, Wh, g.H);
    const bool even_red = ((j + k) & 1) == 0;
    nat[lin(2 * m, j, k, g.W, g.H)] = even_red ? red[q] : black[q];
    nat[lin(2 * m + 1, j, k, g.W, g.H)] = even_red ? black[q] : red[q];
}

void launch_pack(const Geom &g, const float *nat, float *red, float *black, cudaStream_t st) {
    const dim3 b(32, 8, 1);
    const dim3 gr(((g.W >> 1) + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, g.D);
    k_pack<<<gr, b, 0, st>>>(g, nat, red, black);
}

void launch_unpack(const Geom &g, const float *red, const float *black, float *nat,
                   cudaStream_t st) {
    const dim3 b(32, 8, 1);
    const dim3 gr(((g.W >> 1) + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, g.D);
    k_unpack<<<gr, b, 0, st>>>(g, red, black, nat);
}

// ---------------------------------------------------------------------------
// Batched solve over many independent grids (the graph is built in batch.cu).
// Work items are the single-grid segment kernel's threads of every grid, in
// grid order; a persistent grid-stride launch covers them all, so each half
// sweep of the whole batch is one launch.  Items of a grid whose solve has
// finished are skipped.  Per grid, every item does exactly what the
// single-grid kernel's thread does, and the residual blocks and their
// reduction are the single-grid residual's, so a grid's sweeps, residuals
// and stopping point equal those of its own solve bit for bit.
// ---------------------------------------------------------------------------
long long batch_sweep_items(const Geom &g, int kz) {
    return (long long)(g.W >> 3) * g.H * ((g.D + kz - 1) / kz);
}

// Items of the grids still running: act->n grids, grid act->sim[i] owning
// items [act->item0[i], act->item0[i+1]) (rebuilt after every check).
template <int KZ>
__global__ void __launch_bounds__(256)
k_batch_sweep(const BatchSim *__restrict__ sims, const BatchActive *__restrict__ act, int colour) {
    extern __shared__ long long s_item0[];
    const int na = act->n;
    int *s_sim = reinterpret_cast<int *>(s_item0 + na + 1);
    for (int i = threadIdx.x; i <= na; i += blockDim.x) {
        s_item0[i] = act->item0[i];
        if (i < na) s_sim[i] = act->sim[i];
    }
    __syncthreads();
    const long long total = s_item0[na];
    for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < total;
         it += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = na - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_item0[mid] <= it) lo = mid; else hi = mid - 1;
        }
        const BatchSim &S = sims[s_sim[lo]];
        const long long local = it - s_item0[lo];
        const int Wq = S.g.W >> 3;
        const int mq = (int)(local % Wq);
        const long long rest = local / Wq;
        const int j = (int)(rest % S.g.H), k0 = (int)(rest / S.g.H) * KZ;
        seg_sweep<KZ>(S.g, S.sp, colour ? S.rhs_b : S.rhs_r, colour ? S.p_r : S.p_b, colour ? S.p_b : S.p_r,
                      colour, mq, j, k0);
    }
}

int batch_sweep_grid(int kz, int block) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    switch (kz) {
    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_sweep<1>, block, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_sweep<2>, block, 0); break;
    case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_sweep<4>, block, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_sweep<8>, block, 0); break;
    }
    return sms * std::max(1, per);
}

void launch_batch_sweeps(const BatchSim *sims, const BatchActive *act, int nsims, int sweeps, int kz, int grid,
                         int block, cudaStream_t st) {
    const size_t smem = sizeof(long long) * (size_t)(nsims + 1) + sizeof(int) * (size_t)nsims;
    for (int it = 0; it < sweeps; ++it)
        for (int c = 0; c < 2; ++c) {
            switch (kz) {
            case 1: k_batch_sweep<1><<<grid, block, smem, st>>>(sims, act, c); break;
            case 2: k_batch_sweep<2><<<grid, block, smem, st>>>(sims, act, c); break;
            case 4: k_batch_sweep<4><<<grid, block, smem, st>>>(sims, act, c); break;
            default: k_batch_sweep<8><<<grid, block, smem, st>>>(sims, act, c); break;
            }
        }
}

// Temporal blocking over a batch: one CTA per tile (grid, row band, z chunk)
// of every grid, each tile exactly a tile of that grid's own pass, so a
// grid's pressure equals two of its own sweeps bit for bit.  The CTA's 384
// threads map onto the tile's Wq x nrp shape; threads beyond it only meet
// the barriers.  Tiles of a grid whose solve has finished return at once.
// Phase 0 reads p (black) and writes the grid's scratch q; phase 1 reads q
// and writes p, so an even number of passes leaves the result in p.  PK: the
// stencil on paired FP32 instructions (the same bits).
template <bool PK>
__global__ void __launch_bounds__(kTbThreads, 1)
k_batch_tb2(const BatchSim *__restrict__ sims, const BatchTile *__restrict__ tiles,
            const BatchCtl *__restrict__ ctl, int phase) {
    const BatchTile T = tiles[blockIdx.x];
    if (!ctl[T.sim].active) return;
    const BatchSim &S = sims[T.sim];
    const Geom g = S.g;
    const SolveParams sp = S.sp;
    const int Wq = g.W >> 3, nrp = (T.ty + 9) >> 1;
    const int mq = (int)threadIdx.x % Wq, rp = (int)threadIdx.x / Wq;
    const float *pin_b = phase ? S.q_b : S.p_b;
    float *out_r = phase ? S.p_r : S.q_r;
    float *out_b = phase ? S.p_b : S.q_b;
    tb2_tile<false, false, PK>(g, sp, S.rhs_r, S.rhs_b, pin_b, out_r, out_b, T.ty, T.j0, T.z0, T.z1, mq, rp, nrp,
                               rp < nrp, threadIdx.x == 0, nullptr, nullptr, nullptr);
}

bool batch_tb_supported(const Geom &g) { return tb_supported(g); }

int batch_tb_rows(const Geom &g) { return tb_rows_tile(g.W >> 3, g.H); }

size_t batch_tb_smem(const Geom &g) { return tb_smem(g, batch_tb_rows(g)); }

void launch_batch_tb(const BatchSim *sims, const BatchTile *tiles, int ntiles, const BatchCtl *ctl, int sweeps,
                     size_t smem, bool pk, cudaStream_t st) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_batch_tb2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        cudaFuncSetAttribute(k_batch_tb2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmemMax);
        attr_set = true;
    }
    for (int pass = 0; pass < sweeps / 2; ++pass) {
        if (pk) k_batch_tb2<true><<<ntiles, kTbThreads, smem, st>>>(sims, tiles, ctl, pass & 1);
        else k_batch_tb2<false><<<ntiles, kTbThreads, smem, st>>>(sims, tiles, ctl, pass & 1);
    }
}

__device__ __forceinline__ int find_sim(const int *__restrict__ start, int nsims, int b) {
    int lo = 0, hi = nsims - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(start + mid) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Residual blocks of every active grid: grid s owns blocks [blk0[s], blk0[s+1]),
// as many as its own residual launch has.
__global__ void __launch_bounds__(kResThreads)
k_batch_residual(const BatchSim *__restrict__ sims, const int *__restrict__ blk0, int nsims,
                 const BatchCtl *__restrict__ ctl, double *__restrict__ partials) {
    const int s = find_sim(blk0, nsims, blockIdx.x);
    if (!ctl[s].active) return;
    const BatchSim &S = sims[s];
    const int b0 = __ldg(blk0 + s);
    residual_block(S.g, S.sp, S.sp.scale_d, S.rhs_r, S.rhs_b, S.p_r, S.p_b, blockIdx.x - b0,
                   __ldg(blk0 + s + 1) - b0, partials + 2 * (size_t)b0);
}

// One block per grid: its residual totals and the single-grid loop's decision.
__global__ void __launch_bounds__(1024)
k_batch_check(const BatchSim *__restrict__ sims, const int *__restrict__ blk0, const double *__restrict__ partials,
              BatchCtl *__restrict__ ctl, int after_sweeps, int chunk) {
    const int s = blockIdx.x;
    if (!ctl[s].active) return;
    __shared__ double out2[2];
    const int b0 = blk0[s];
    reduce_pairs_block(partials + 2 * (size_t)b0, blk0[s + 1] - b0, out2);
    __syncthreads();
    if (threadIdx.x == 0) {
        BatchCtl c = ctl[s];
        if (after_sweeps) c.iters += chunk;
        c.checks += 1;
        c.r2 = out2[0];
        c.b2 = out2[1];
        const bool conv = c.b2 == 0.0 || sqrt(c.r2) / sqrt(c.b2) <= sims[s].tol;
        c.converged = conv;
        c.active = (!conv && c.iters < sims[s].max_iter) ? 1 : 0;
        ctl[s] = c;
    }
}

void launch_batch_check(const BatchSim *sims, const int *blk0, int nsims, int total_blocks, BatchCtl *ctl,
                        double *partials, int after_sweeps, int chunk, cudaStream_t st) {
    k_batch_residual<<<total_blocks, kResThreads, 0, st>>>(sims, blk0, nsims, ctl, partials);
    k_batch_check<<<nsims, 1024, 0, st>>>(sims, blk0, partials, ctl, after_sweeps, chunk);
}

} // namespace blz
