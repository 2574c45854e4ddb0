// k_source.cu — particle sourcing (reference src/FluidSolver.cu:57-116 and
// Grid::sphereToGrid / cubicPulse, src/Grid.h:309-335), as a gather.
//
// The reference clears four back buffers over the whole grid, splats every
// particle with float atomics and copies |back| > 1e-5 into the front
// buffers (three full-grid passes, order-dependent sums).  Here the host bins
// the particles by 8^3 blocks of cells (the records come from host memory
// anyway) and each bin is one CTA: every cell sums the cubic pulses of the
// particles overlapping its bin in particle order and writes the front buffer
// once where |sum| > 1e-5.  No atomics, no accumulator buffers, no clear
// pass, and the sums are bitwise reproducible.
#include "kernels.cuh"

namespace blz {

__device__ __forceinline__ float cubic_pulse(float x, float w) {   // Grid.h:309-313
    if (x > w) return 0.0f;
    x /= w;
    return 1.0f - x * x * (3.0f - 2.0f * x);
}

constexpr int kSplatChunk = 64;

__global__ void __launch_bounds__(512)
k_splat_gather(Geom g, const float *__restrict__ rec8, const int *__restrict__ boxes,
               const int *__restrict__ bin_start, const int *__restrict__ bin_list,
               const int *__restrict__ active, int nbx, int nby, float *__restrict__ T,
               float *__restrict__ U, float *__restrict__ V, float *__restrict__ W,
               const float *__restrict__ dens, float *__restrict__ Dn) {
    __shared__ float s_rec[kSplatChunk * 9];
    __shared__ int s_box[kSplatChunk * kSplatBoxInts];
    const int b = active[blockIdx.x];
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    const int i = bx * kSplatBin + threadIdx.x, j = by * kSplatBin + threadIdx.y, k = bz * kSplatBin + threadIdx.z;
    const int tid = threadIdx.x + kSplatBin * (threadIdx.y + kSplatBin * threadIdx.z);
    const float ox[4] = {0.5f, 0.0f, 0.5f, 0.5f}, oy[4] = {0.5f, 0.5f, 0.0f, 0.5f}, oz[4] = {0.5f, 0.5f, 0.5f, 0.0f};
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f}, acc_d = 0.0f;
    const int p0 = bin_start[b], p1 = bin_start[b + 1];
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    for (int base = p0; base < p1; base += kSplatChunk) {
        const int n = min(kSplatChunk, p1 - base);
        for (int t = tid; t < n * 8; t += nthr)
            s_rec[9 * (t / 8) + t % 8] = rec8[(size_t)bin_list[base + t / 8] * 8 + t % 8];
        if (Dn)
            for (int t = tid; t < n; t += nthr) s_rec[9 * t + 8] = dens[bin_list[base + t]];
        for (int t = tid; t < n * kSplatBoxInts; t += nthr)
            s_box[t] = boxes[(size_t)bin_list[base + t / kSplatBoxInts] * kSplatBoxInts + t % kSplatBoxInts];
        __syncthreads();
        for (int q = 0; q < n; ++q) {
            const float *r = s_rec + 9 * q;
            const float radius = r[6] / 2.0f;
            const float px = r[0] - g.dmin[0], py = g.dsize[1] - (r[1] - g.dmin[1]), pz = r[2] - g.dmin[2];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const int *bb = s_box + kSplatBoxInts * q + 6 * f;   // imin, imax, jmin, jmax, kmin, kmax (empty if skipped)
                if (i < bb[0] || i >= bb[1] || j < bb[2] || j >= bb[3] || k < bb[4] || k >= bb[5]) continue;
                const float value = f == 0 ? r[7] : r[2 + f];
                const float ddx = px - ((float)i + ox[f]) * g.dx;
                const float ddy = py - ((float)j + oy[f]) * g.dx;
                const float ddz = pz - ((float)k + oz[f]) * g.dx;
                const float mask = cubic_pulse(len3(ddx, ddy, ddz), radius);
                if (mask > 0.0f) acc[f] += f == 2 ? -value * mask : value * mask;   // V flips (Grid.h:331)
            }
            if (Dn) {                                     // density: T's geometry, its own box and value
                const int *bb = s_box + kSplatBoxInts * q + 24;
                if (i >= bb[0] && i < bb[1] && j >= bb[2] && j < bb[3] && k >= bb[4] && k < bb[5]) {
                    const float ddx = px - ((float)i + 0.5f) * g.dx;
                    const float ddy = py - ((float)j + 0.5f) * g.dx;
                    const float ddz = pz - ((float)k + 0.5f) * g.dx;
                    const float mask = cubic_pulse(len3(ddx, ddy, ddz), radius);
                    if (mask > 0.0f) acc_d += r[8] * mask;
                }
            }
        }
        __syncthreads();
    }
    // set_source_from_back_to_front_kernel (FluidSolver.cu:99-116)
    if (i < g.W && j < g.H && k < g.D && fabsf(acc[0]) > 1e-5f) T[lin(i, j, k, g.W, g.H)] = acc[0];
    if (i <= g.W && j < g.H && k < g.D && fabsf(acc[1]) > 1e-5f) U[lin(i, j, k, g.W + 1, g.H)] = acc[1];
    if (i < g.W && j <= g.H && k < g.D && fabsf(acc[2]) > 1e-5f) V[lin(i, j, k, g.W, g.H + 1)] = acc[2];
    if (i < g.W && j < g.H && k <= g.D && fabsf(acc[3]) > 1e-5f) W[lin(i, j, k, g.W, g.H)] = acc[3];
    if (Dn && i < g.W && j < g.H && k < g.D && fabsf(acc_d) > 1e-5f) Dn[lin(i, j, k, g.W, g.H)] = acc_d;
}

void launch_splat_gather(const Geom &g, const float *rec8, const int *boxes, const int *bin_start,
                         const int *bin_list, const int *active, int n_active, int nbx, int nby,
                         float *T, float *U, float *V, float *W, cudaStream_t st, const float *dens, float *Dn) {
    if (n_active <= 0) return;
    const dim3 b(kSplatBin, kSplatBin, kSplatBin);
    k_splat_gather<<<n_active, b, 0, st>>>(g, rec8, boxes, bin_start, bin_list, active, nbx, nby, T, U, V, W, dens,
                                           Dn);
}

} // namespace blz
