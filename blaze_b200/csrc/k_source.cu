// k_source.cu — particle sourcing (reference src/FluidSolver.cu:57-116 and
// Grid::sphereToGrid / cubicPulse, src/Grid.h:309-335).
//
// The splat accumulates into dedicated, always-zero accumulators instead of
// clearing the four back buffers over the whole grid; the apply pass then
// visits only the box the particles can reach, copies |acc| > 1e-5 into the
// front buffer (set_source_from_back_to_front_kernel) and re-zeroes acc.
#include "kernels.cuh"

namespace blz {

struct SplatField { float ox, oy, oz; int w, h, d; bool flip; };

__device__ __forceinline__ SplatField splat_field(const Geom &g, int f) {
    switch (f) {
    case BLZ_FIELD_T: return {0.5f, 0.5f, 0.5f, g.W, g.H, g.D, false};
    case BLZ_FIELD_U: return {0.0f, 0.5f, 0.5f, g.W + 1, g.H, g.D, false};
    case BLZ_FIELD_V: return {0.5f, 0.0f, 0.5f, g.W, g.H + 1, g.D, true};
    default:          return {0.5f, 0.5f, 0.0f, g.W, g.H, g.D + 1, false};
    }
}

__device__ __forceinline__ int trunc_i(float v) {   // C cast, guarded against overflow
    return (int)fminf(fmaxf(v, -1.0e9f), 1.0e9f);
}

__device__ __forceinline__ float cubic_pulse(float x, float w) {   // Grid.h:309-313
    if (x > w) return 0.0f;
    x /= w;
    return 1.0f - x * x * (3.0f - 2.0f * x);
}

// One block per particle, one warp per field (T, U, V, W); the warp's lanes
// stride over the particle's bounding box of that field.
__global__ void __launch_bounds__(128)
k_splat(Geom g, const float *__restrict__ rec8, int n, float *__restrict__ accT,
        float *__restrict__ accU, float *__restrict__ accV, float *__restrict__ accW) {
    const int p = blockIdx.x;
    if (p >= n) return;
    const int f = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float *r = rec8 + 8 * (size_t)p;
    const float px = r[0], py = r[1], pz = r[2], ps = r[6];
    if (!(ps > g.dx / 2.0f)) return;                    // FluidSolver.cu:83
    const float value = f == 0 ? r[7] : r[2 + f];       // temp, vel.x, vel.y, vel.z
    if (!(fabsf(value) > 1e-5f)) return;                // FluidSolver.cu:84-95
    float *acc = f == 0 ? accT : f == 1 ? accU : f == 2 ? accV : accW;
    const SplatField sf = splat_field(g, f);
    const float radius = ps / 2.0f, dx = g.dx;
    const int imin = max(trunc_i(((px - radius) - g.dmin[0]) / dx - sf.ox), 0);
    const int imax = min(trunc_i(((px + radius) - g.dmin[0]) / dx - sf.ox) + 1, sf.w);
    const int jmin = max(trunc_i((g.dsize[1] - ((py + radius) - g.dmin[1])) / dx - sf.oy), 0);
    const int jmax = min(trunc_i((g.dsize[1] - ((py - radius) - g.dmin[1])) / dx - sf.oy) + 1, sf.h);
    const int kmin = max(trunc_i(((pz - radius) - g.dmin[2]) / dx - sf.oz), 0);
    const int kmax = min(trunc_i(((pz + radius) - g.dmin[2]) / dx - sf.oz) + 1, sf.d);
    const int nx = imax - imin, ny = jmax - jmin, nz = kmax - kmin;
    if (nx <= 0 || ny <= 0 || nz <= 0) return;
    const float ox = px - g.dmin[0], oy = g.dsize[1] - (py - g.dmin[1]), oz = pz - g.dmin[2];
    const float sv = sf.flip ? -value : value;
    const int cells = nx * ny * nz;
    for (int c = lane; c < cells; c += 32) {
        const int i = imin + c % nx, j = jmin + (c / nx) % ny, k = kmin + c / (nx * ny);
        const float ddx = ox - ((float)i + sf.ox) * dx;
        const float ddy = oy - ((float)j + sf.oy) * dx;
        const float ddz = oz - ((float)k + sf.oz) * dx;
        const float mask = cubic_pulse(len3(ddx, ddy, ddz), radius);
        if (mask > 0.0f) atomicAdd(acc + lin(i, j, k, sf.w, sf.h), sv * mask);
    }
}

void launch_splat(const Geom &g, const float *rec8, int n, float *accT, float *accU, float *accV,
                  float *accW, cudaStream_t st) {
    if (n <= 0) return;
    k_splat<<<n, 128, 0, st>>>(g, rec8, n, accT, accU, accV, accW);
}

__global__ void k_source_apply(int w, int h, int i0, int j0, int k0, int nx, int ny, int nz,
                               float *__restrict__ front, float *__restrict__ acc) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z * blockDim.z + threadIdx.z;
    if (a >= nx || b >= ny || c >= nz) return;
    const size_t q = lin(i0 + a, j0 + b, k0 + c, w, h);
    const float v = acc[q];
    if (fabsf(v) > 1e-5f) front[q] = v;                // FluidSolver.cu:104-115
    if (v != 0.0f) acc[q] = 0.0f;
}

void launch_source_apply(const Geom &g, const int box[3][2], float *front, float *acc, int field,
                         cudaStream_t st) {
    const int nx = box[0][1] - box[0][0], ny = box[1][1] - box[1][0], nz = box[2][1] - box[2][0];
    if (nx <= 0 || ny <= 0 || nz <= 0) return;
    const int w = field == BLZ_FIELD_U ? g.W + 1 : g.W;
    const int h = field == BLZ_FIELD_V ? g.H + 1 : g.H;
    const dim3 b(32, 4, 2);
    const dim3 gr((nx + 31) / 32, (ny + 3) / 4, (nz + 1) / 2);
    k_source_apply<<<gr, b, 0, st>>>(w, h, box[0][0], box[1][0], box[2][0], nx, ny, nz, front, acc);
}

} // namespace blz
