// k_project.cu — divergence, red-black Gauss-Seidel, FP64 residual and the
// pressure-gradient subtract (reference src/FluidSolver.cu:475-669, 823-856).
//
// Pressure and rhs live colour packed in HBM: cell (i,j,k) of colour
// c = (i+j+k)&1 sits at (i>>1) + (W/2)*(j + H*k) of its colour's array.  A half
// sweep of colour c writes only c's array and reads only the other colour's,
// all rows contiguous; red cells of a row are even or odd i according to the
// row parity (j+k)&1.
#include <algorithm>

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

// Quotient num/den for the neighbour count den in {1..6} on the FMA pipe:
// q0 = num*RN(1/den), then one remainder correction e = num - q0*den (exact
// with an FMA) and q = q0 + e*RN(1/den) (Markstein's correction step).  An
// IEEE division would put a reciprocal and an int-to-float conversion per
// cell on the XU pipe, which bounds the sweep well below HBM speed.
__device__ __forceinline__ float inv_count(float den) {
    return den == 6.0f ? 1.0f / 6.0f : den == 5.0f ? 0.2f : den == 4.0f ? 0.25f
         : den == 3.0f ? 1.0f / 3.0f : den == 2.0f ? 0.5f : 1.0f;
}
__device__ __forceinline__ float div_count(float num, float den) {
    const float inv = inv_count(den);
    const float q0 = num * inv;
    const float e = fmaf(-q0, den, num);
    return fmaf(e, inv, q0);
}

// One Gauss-Seidel update p = (scale*rhs + sum p_nb)/n_nb (FluidSolver.cu:
// 532-561), summed in the reference's neighbour order.  n_nb counts the
// in-domain neighbours, plus a p = 0 ghost per open face when dirichlet.
__device__ __forceinline__ float gs_update(const Geom &g, const SolveParams &sp, float rhs,
                                           const float *__restrict__ po, size_t q, int i, int j,
                                           int k, int s, int Wh) {
    float num = sp.scale * rhs;
    float den = 0.0f;
    const bool dir = sp.dirichlet;
    if (i > 0) { num += __ldg(po + q - (s ? 0 : 1)); den += 1.0f; } else if (dir && sp.open.xlo) den += 1.0f;
    if (i < g.W - 1) { num += __ldg(po + q + (s ? 1 : 0)); den += 1.0f; } else if (dir && sp.open.xhi) den += 1.0f;
    if (j > 0) { num += __ldg(po + q - Wh); den += 1.0f; } else if (dir && sp.open.ylo) den += 1.0f;
    if (j < g.H - 1) { num += __ldg(po + q + Wh); den += 1.0f; } else if (dir && sp.open.yhi) den += 1.0f;
    const size_t pl = (size_t)Wh * g.H;
    if (k > 0) { num += __ldg(po + q - pl); den += 1.0f; } else if (dir && sp.open.zlo) den += 1.0f;
    if (k < g.D - 1) { num += __ldg(po + q + pl); den += 1.0f; } else if (dir && sp.open.zhi) den += 1.0f;
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

// Updates four consecutive packed cells m0..m0+3 of one row: o is the other
// colour at the same packed indices, xe its value just outside the segment
// (m0-1 when the row's cells sit at even i, m0+4 when odd), ym/yp/zm/zp the
// other colour in rows j-1, j+1 and planes k-1, k+1.
__device__ __forceinline__ float4 gs_segment(const SolveParams &sp, int s, bool first, bool last, float4 r,
                                             float4 o, float xe, float4 ym, float4 yp, float4 zm, float4 zp,
                                             bool has_ym, bool has_yp, bool has_zm, bool has_zp) {
    float xl[4], xr[4];
    if (s == 0) {
        xl[0] = xe; xl[1] = o.x; xl[2] = o.y; xl[3] = o.z;
        xr[0] = o.x; xr[1] = o.y; xr[2] = o.z; xr[3] = o.w;
    } else {
        xl[0] = o.x; xl[1] = o.y; xl[2] = o.z; xl[3] = o.w;
        xr[0] = o.y; xr[1] = o.z; xr[2] = o.w; xr[3] = xe;
    }
    // A missing neighbour arrives as 0 (the caller passes zero4 and xe = 0),
    // so the sum is branch free and in the reference's order; only the
    // neighbour count differs, and it is the same for every cell of the quad
    // except the one at a row end, so the count and its reciprocal are formed
    // three times per quad rather than per cell.
    const bool dir = sp.dirichlet;
    const float den_b = 2.0f + (has_ym ? 1.0f : (dir && sp.open.ylo ? 1.0f : 0.0f)) +
                        (has_yp ? 1.0f : (dir && sp.open.yhi ? 1.0f : 0.0f)) +
                        (has_zm ? 1.0f : (dir && sp.open.zlo ? 1.0f : 0.0f)) +
                        (has_zp ? 1.0f : (dir && sp.open.zhi ? 1.0f : 0.0f));
    const float den0 = (s == 0 && first) ? den_b - 1.0f + (dir && sp.open.xlo ? 1.0f : 0.0f) : den_b;
    const float den3 = (s == 1 && last) ? den_b - 1.0f + (dir && sp.open.xhi ? 1.0f : 0.0f) : den_b;
    const float inv_b = inv_count(den_b), inv0 = inv_count(den0), inv3 = inv_count(den3);
    const float ra[4] = {r.x, r.y, r.z, r.w};
    const float yma[4] = {ym.x, ym.y, ym.z, ym.w}, ypa[4] = {yp.x, yp.y, yp.z, yp.w};
    const float zma[4] = {zm.x, zm.y, zm.z, zm.w}, zpa[4] = {zp.x, zp.y, zp.z, zp.w};
    float out[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        float num = sp.scale * ra[t];
        num += xl[t];
        num += xr[t];
        num += yma[t];
        num += ypa[t];
        num += zma[t];
        num += zpa[t];
        const float den = t == 0 ? den0 : t == 3 ? den3 : den_b;
        const float inv = t == 0 ? inv0 : t == 3 ? inv3 : inv_b;
        const float q0 = num * inv;
        out[t] = fmaf(fmaf(-q0, den, num), inv, q0);
    }
    return make_float4(out[0], out[1], out[2], out[3]);
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
// the in-place sweeps would (the z neighbours from the thread's own
// registers, the in-plane neighbours from shared memory, four plane slots
// per colour).  Per cell the arithmetic is gs_segment's, so a pass equals
// two sweeps of the segment kernel bit for bit.  HBM traffic per pass is
// about 10 B/cell instead of 24 B/cell for two unblocked sweeps; the price is
// recomputing the halo.
// ---------------------------------------------------------------------------
constexpr int kTbThreads = 768;

__host__ __device__ inline int tb_rows_tile(int Wq, int H) {
    const int ty = kTbThreads / Wq - 8;
    return ty < H ? ty : H;
}

__device__ __forceinline__ void cp_async16_tb(float4 *dst, const float *src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

__global__ void __launch_bounds__(kTbThreads, 1)
k_rbgs_tb2(Geom g, SolveParams sp, const float *__restrict__ rhs_r, const float *__restrict__ rhs_b,
           const float *__restrict__ pin_b, float *__restrict__ pout_r, float *__restrict__ pout_b, int TY, int ZC) {
    // Shared memory, in units of one plane slot (rows x Wq float4):
    //   [0, 8)   p, colour c and plane k at slot c*4 + (k & 3)
    //   [8, 12)  red rhs, plane k at 8 + (k & 3)
    //   [12, 16) black rhs, plane k at 12 + (k & 3)
    //   [16, 18) black p input staging, plane k at 16 + (k & 1)
    // rhs and staged input are prefetched one step ahead with cp.async and
    // only ever read back by the thread that loaded them.
    extern __shared__ float4 sm4[];
    const int Wh = g.W >> 1, Wq = Wh >> 2;
    const int rows = TY + 8;
    const int mq = threadIdx.x, r = threadIdx.y;
    const int j0 = blockIdx.x * TY, z0 = blockIdx.y * ZC;
    const int z1 = z0 + ZC < g.D ? z0 + ZC : g.D;
    const int j = j0 - 4 + r;
    const bool row_ok = j >= 0 && j < g.H;
    const int m0 = 4 * mq;
    const size_t pl = (size_t)Wh * g.H;
    const size_t rowoff = (size_t)m0 + (size_t)Wh * (size_t)(row_ok ? j : 0);
    const bool first = m0 == 0, last = m0 + 4 == Wh;
    const bool has_ym = j > 0, has_yp = j < g.H - 1;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const size_t slot = (size_t)rows * Wq;
    auto S = [&](int colour, int plane, int row) -> float4 * {
        return sm4 + (size_t)(colour * 4 + (plane & 3)) * slot + (size_t)row * Wq;
    };
    float4 *own = sm4 + (size_t)r * Wq + mq;                 // this thread's element of slot 0
    auto RR = [&](int plane) { return own + (size_t)(8 + (plane & 3)) * slot; };
    auto RB = [&](int plane) { return own + (size_t)(12 + (plane & 3)) * slot; };
    auto ST = [&](int plane) { return own + (size_t)(16 + (plane & 1)) * slot; };
    auto valid = [&](int k) { return row_ok && k >= 0 && k < g.D; };
    auto prefetch = [&](int k_red, int k_black, int k_in) {
        // red rhs: levels 0 and 2 cover planes [z0-3, z1+3); black rhs: levels 1 and 3 cover [z0-2, z1+2)
        if (valid(k_red) && k_red >= z0 - 3 && k_red < z1 + 3) cp_async16_tb(RR(k_red), rhs_r + rowoff + (size_t)k_red * pl);
        if (valid(k_black) && k_black >= z0 - 2 && k_black < z1 + 2) cp_async16_tb(RB(k_black), rhs_b + rowoff + (size_t)k_black * pl);
        if (valid(k_in) && k_in < z1 + 4) cp_async16_tb(ST(k_in), pin_b + rowoff + (size_t)k_in * pl);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // One level: the colour `c` cells of this thread's quad on plane k.
    auto update = [&](int c, int k, float4 o, float4 zm, float4 zp) -> float4 {
        const int oc = c ^ 1;
        const float4 *so = S(oc, k, r);
        const float4 ym = has_ym ? S(oc, k, r - 1)[mq] : zero4;
        const float4 yp = has_yp ? S(oc, k, r + 1)[mq] : zero4;
        const int s = (j + k + c) & 1;
        const float *sf = reinterpret_cast<const float *>(so);
        const float xe = s == 0 ? (first ? 0.0f : sf[m0 - 1]) : (last ? 0.0f : sf[m0 + 4]);
        const bool has_zm = k > 0, has_zp = k < g.D - 1;
        const float4 rv = c ? *RB(k) : *RR(k);
        return gs_segment(sp, s, first, last, rv, o, xe, ym, yp, has_zm ? zm : zero4, has_zp ? zp : zero4,
                          has_ym, has_yp, has_zm, has_zp);
    };
    auto active = [&](int h, int k) {
        return row_ok && r >= 1 + h && r < rows - 1 - h && k >= z0 - 3 + h && k < z1 + 3 - h && k >= 0 &&
               k < g.D;
    };
    // register windows: black planes t-3..t+1, red planes t-4..t
    float4 bm3 = zero4, bm2 = zero4, bp1;
    float4 bm1 = valid(z0 - 4) ? ld4(pin_b + rowoff + (size_t)(z0 - 4) * pl) : zero4;
    float4 b0 = valid(z0 - 3) ? ld4(pin_b + rowoff + (size_t)(z0 - 3) * pl) : zero4;
    float4 rm4 = zero4, rm3 = zero4, rm2 = zero4, rm1 = zero4, r0 = zero4;
    S(1, z0 - 4, r)[mq] = bm1;
    S(1, z0 - 3, r)[mq] = b0;
    prefetch(z0 - 3, z0 - 4, z0 - 2);                 // what the first step reads
    for (int t = z0 - 3; t < z1 + 3; ++t) {
        prefetch(t + 1, t, t + 2);                    // what the next step reads
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        bp1 = valid(t + 1) ? *ST(t + 1) : zero4;
        S(1, t + 1, r)[mq] = bp1;
        __syncthreads();
        if (active(0, t)) { r0 = update(0, t, b0, bm1, bp1); S(0, t, r)[mq] = r0; }
        __syncthreads();
        if (active(1, t - 1)) { bm1 = update(1, t - 1, rm1, rm2, r0); S(1, t - 1, r)[mq] = bm1; }
        __syncthreads();
        if (active(2, t - 2)) { rm2 = update(0, t - 2, bm2, bm3, bm1); S(0, t - 2, r)[mq] = rm2; }
        __syncthreads();
        const int k3 = t - 3;
        if (active(3, k3)) {
            bm3 = update(1, k3, rm3, rm4, rm2);
            if (k3 >= z0 && r >= 4 && r < 4 + TY) {
                *reinterpret_cast<float4 *>(pout_r + rowoff + (size_t)k3 * pl) = rm3;
                *reinterpret_cast<float4 *>(pout_b + rowoff + (size_t)k3 * pl) = bm3;
            }
        }
        rm4 = rm3; rm3 = rm2; rm2 = rm1; rm1 = r0;
        bm3 = bm2; bm2 = bm1; bm1 = b0; b0 = bp1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

static bool tb_supported(const Geom &g) {
    if ((g.W & 7) != 0) return false;
    const int Wq = g.W >> 3;
    return Wq <= 48 && tb_rows_tile(Wq, g.H) >= 1;
}

static size_t tb_smem(const Geom &g, int TY) { return sizeof(float4) * 18 * (size_t)(TY + 8) * (g.W >> 3); }

// One pass = two sweeps from (p_in) into (p_out).
static void launch_tb_pass(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                           const float *pin_b, float *pout_r, float *pout_b, int ZC, cudaStream_t st) {
    const int Wq = g.W >> 3, TY = tb_rows_tile(Wq, g.H);
    const size_t smem = tb_smem(g, TY);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_rbgs_tb2, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_set = true;
    }
    const dim3 b(Wq, TY + 8, 1);
    const dim3 gr((g.H + TY - 1) / TY, (g.D + ZC - 1) / ZC, 1);
    k_rbgs_tb2<<<gr, b, smem, st>>>(g, sp, rhs_r, rhs_b, pin_b, pout_r, pout_b, TY, ZC);
}

// (planes per thread, rows per block) of each segment-kernel variant; the
// variants after them are the temporal-blocking pass with ZC planes per CTA.
static const int kVariantKZ[kSegVariants] = {1, 2, 4, 8, 2, 4};
static const int kVariantBY[kSegVariants] = {8, 8, 4, 4, 4, 8};
static const int kVariantZC[kSweepVariants - kSegVariants] = {16, 32};

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
        for (int i = 0; i < passes; ++i) {
            if ((i & 1) == 0) launch_tb_pass(g, sp, rhs_r, rhs_b, p_b, q_r, q_b, zc, st);
            else launch_tb_pass(g, sp, rhs_r, rhs_b, q_b, p_r, p_b, zc, st);
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

int residual_blocks(const Geom &g) {
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

__global__ void __launch_bounds__(kResThreads)
k_residual_seg(Geom g, SolveParams sp, double scale, const float *__restrict__ rr,
               const float *__restrict__ rb, const float *__restrict__ pr, const float *__restrict__ pb,
               double *__restrict__ partials) {
    residual_seg_block(g, sp, scale, rr, rb, pr, pb, blockIdx.x, gridDim.x, partials);
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
    const int blocks = std::min(residual_blocks(g), max_partials);
    const double scale = (double)sp.scale_d;
    if ((g.W & 7) == 0)
        k_residual_seg<<<blocks, kResThreads, 0, st>>>(g, sp, scale, rhs_r, rhs_b, p_r, p_b, partials);
    else
        k_residual<<<blocks, kResThreads, 0, st>>>(g, sp, scale, rhs_r, rhs_b, p_r, p_b, partials);
    k_reduce_pairs<<<1, 1024, 0, st>>>(partials, blocks, out2);
    return 2;
}

// pressure_gradient_update_kernel (FluidSolver.cu:601-669).  Interior faces
// subtract dt/(rho dx) * grad p.  Domain faces: 0 at a wall; at an open face
// REF_COMPAT copies the inner neighbour's updated value (the reference's copy,
// read after the update; the thread of the inner face writes both, so no
// thread reads a face another thread writes), FREE_SURFACE applies the
// gradient against the p = 0 ghost.
__global__ void k_gradient(Geom g, SolveParams sp, float s, const float *__restrict__ pr,
                           const float *__restrict__ pb, float *__restrict__ U,
                           float *__restrict__ V, float *__restrict__ W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.W || j > g.H || k > g.D) return;
    const int Wh = g.W >> 1, H = g.H;
    const OpenFaces &o = sp.open;
    const bool dir = sp.dirichlet;
    auto P = [&](int a, int b, int c) { return pval(pr, pb, a, b, c, Wh, H); };
    if (j < g.H && k < g.D) {
        const size_t q = lin(i, j, k, g.W + 1, g.H);
        if (i > 0 && i < g.W) {
            const float u = U[q] - s * (P(i, j, k) - P(i - 1, j, k));
            U[q] = u;
            if (!dir && i == 1 && o.xlo) U[q - 1] = u;
            if (!dir && i == g.W - 1 && o.xhi) U[q + 1] = u;
        } else if (i == 0) {
            if (!o.xlo) U[q] = 0.0f;
            else if (dir) U[q] -= s * (P(0, j, k) - 0.0f);
        } else {
            if (!o.xhi) U[q] = 0.0f;
            else if (dir) U[q] -= s * (0.0f - P(g.W - 1, j, k));
        }
    }
    if (i < g.W && k < g.D) {
        const size_t q = lin(i, j, k, g.W, g.H + 1);
        const size_t row = (size_t)g.W;
        if (j > 0 && j < g.H) {
            const float v = V[q] - s * (P(i, j, k) - P(i, j - 1, k));
            V[q] = v;
            if (!dir && j == 1 && o.ylo) V[q - row] = v;
            if (!dir && j == g.H - 1 && o.yhi) V[q + row] = v;
        } else if (j == 0) {
            if (!o.ylo) V[q] = 0.0f;
            else if (dir) V[q] -= s * (P(i, 0, k) - 0.0f);
        } else {
            if (!o.yhi) V[q] = 0.0f;
            else if (dir) V[q] -= s * (0.0f - P(i, g.H - 1, k));
        }
    }
    if (i < g.W && j < g.H) {
        const size_t q = lin(i, j, k, g.W, g.H);
        const size_t plane = (size_t)g.W * g.H;
        if (k > 0 && k < g.D) {
            const float w = W[q] - s * (P(i, j, k) - P(i, j, k - 1));
            W[q] = w;
            if (!dir && k == 1 && o.zlo) W[q - plane] = w;
            if (!dir && k == g.D - 1 && o.zhi) W[q + plane] = w;
        } else if (k == 0) {
            if (!o.zlo) W[q] = 0.0f;
            else if (dir) W[q] -= s * (P(i, j, 0) - 0.0f);
        } else {
            if (!o.zhi) W[q] = 0.0f;
            else if (dir) W[q] -= s * (0.0f - P(i, j, g.D - 1));
        }
    }
}

void launch_gradient(const Geom &g, const SolveParams &sp, float s, const float *p_r,
                     const float *p_b, float *U, float *V, float *W, cudaStream_t st) {
    k_gradient<<<face_grid(g), face_block(), 0, st>>>(g, sp, s, p_r, p_b, U, V, W);
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
    residual_seg_block(S.g, S.sp, S.sp.scale_d, S.rhs_r, S.rhs_b, S.p_r, S.p_b, blockIdx.x - b0,
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
