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

// One Gauss-Seidel update p = (scale*rhs + sum p_nb)/n_nb (FluidSolver.cu:
// 532-561), summed in the reference's neighbour order.  n_nb counts the
// in-domain neighbours, plus a p = 0 ghost per open face when dirichlet.
__device__ __forceinline__ float gs_update(const Geom &g, const SolveParams &sp, float rhs,
                                           const float *__restrict__ po, size_t q, int i, int j,
                                           int k, int s, int Wh) {
    float num = sp.scale * rhs;
    int den = 0;
    const bool dir = sp.dirichlet;
    if (i > 0) { num += __ldg(po + q - (s ? 0 : 1)); ++den; } else if (dir && sp.open.xlo) ++den;
    if (i < g.W - 1) { num += __ldg(po + q + (s ? 1 : 0)); ++den; } else if (dir && sp.open.xhi) ++den;
    if (j > 0) { num += __ldg(po + q - Wh); ++den; } else if (dir && sp.open.ylo) ++den;
    if (j < g.H - 1) { num += __ldg(po + q + Wh); ++den; } else if (dir && sp.open.yhi) ++den;
    const size_t pl = (size_t)Wh * g.H;
    if (k > 0) { num += __ldg(po + q - pl); ++den; } else if (dir && sp.open.zlo) ++den;
    if (k < g.D - 1) { num += __ldg(po + q + pl); ++den; } else if (dir && sp.open.zhi) ++den;
    return num / (float)den;
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

void launch_rbgs_sweeps(const Geom &g, const SolveParams &sp, const float *rhs_r,
                        const float *rhs_b, float *p_r, float *p_b, int sweeps, cudaStream_t st,
                        long long *launches) {
    const dim3 b(32, 8, 1);
    const dim3 gr(((g.W >> 1) + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, g.D);
    for (int it = 0; it < sweeps; ++it) {
        k_rbgs_half<<<gr, b, 0, st>>>(g, sp, rhs_r, p_b, p_r, 0);
        k_rbgs_half<<<gr, b, 0, st>>>(g, sp, rhs_b, p_r, p_b, 1);
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
// packed pairs with a fixed launch shape, warp-shuffle then shared-memory
// reduction per block, then one block sums the per-block partials in order:
// the result is bit-reproducible.
// ---------------------------------------------------------------------------
constexpr int kResThreads = 256;

int residual_blocks(const Geom &g) {
    const long long items = (long long)(g.W >> 1) * g.H * g.D;
    return (int)std::min<long long>((items + kResThreads - 1) / kResThreads, 148 * 8);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kResThreads)
k_residual(Geom g, SolveParams sp, double scale, const float *__restrict__ rr,
           const float *__restrict__ rb, const float *__restrict__ pr, const float *__restrict__ pb,
           double *__restrict__ partials) {
    const int Wh = g.W >> 1;
    const long long items = (long long)Wh * g.H * g.D;
    double r2 = 0.0, b2 = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < items;
         t += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(t % Wh);
        const long long jk = t / Wh;
        const int j = (int)(jk % g.H), k = (int)(jk / g.H);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * m + h;
            const bool black = (i + j + k) & 1;
            const size_t q = (size_t)t;
            const double b = scale * (double)__ldg((black ? rb : rr) + q);
            double nb = 0.0, n = 0.0;
            const OpenFaces &o = sp.open;
            const bool dir = sp.dirichlet;
            if (i > 0) { nb += pval(pr, pb, i - 1, j, k, Wh, g.H); n += 1.0; } else if (dir && o.xlo) n += 1.0;
            if (i < g.W - 1) { nb += pval(pr, pb, i + 1, j, k, Wh, g.H); n += 1.0; } else if (dir && o.xhi) n += 1.0;
            if (j > 0) { nb += pval(pr, pb, i, j - 1, k, Wh, g.H); n += 1.0; } else if (dir && o.ylo) n += 1.0;
            if (j < g.H - 1) { nb += pval(pr, pb, i, j + 1, k, Wh, g.H); n += 1.0; } else if (dir && o.yhi) n += 1.0;
            if (k > 0) { nb += pval(pr, pb, i, j, k - 1, Wh, g.H); n += 1.0; } else if (dir && o.zlo) n += 1.0;
            if (k < g.D - 1) { nb += pval(pr, pb, i, j, k + 1, Wh, g.H); n += 1.0; } else if (dir && o.zhi) n += 1.0;
            const double p = (double)__ldg((black ? pb : pr) + q);
            const double r = b - (n * p - nb);
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

__global__ void __launch_bounds__(1024) k_reduce_pairs(const double *__restrict__ partials, int n,
                                                       double *__restrict__ out2) {
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

int launch_residual(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                    const float *p_r, const float *p_b, double *partials, int max_partials,
                    double *out2, cudaStream_t st) {
    const int blocks = std::min(residual_blocks(g), max_partials);
    const double scale = (double)sp.scale_d;
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

} // namespace blz
