// noalloc.cu — the FP64 pressure residual without any device allocation.
//
// blz_residual() works on a solver's own buffers and its reduction scratch is
// allocated when the solver is created.  Some callers cannot allocate: a host
// application (a renderer's frame loop, a plugin inside a content-creation
// tool) that owns every byte of device memory through its own pool and does
// not let plugins call cudaMalloc, or code that must not stall the device,
// which cudaMalloc and cudaFree can do by synchronising.  This entry point
// takes the caller's rhs and pressure and writes the two norms to the
// caller's memory; its only scratch is the fixed array below, one FP64 pair
// per z-plane, which every GPU that loads the library holds until exit.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "kernels.cuh"

namespace blz {

// Largest depth (z-planes) the scratch holds: 2 doubles per plane, 64 KiB.
constexpr int kNoAllocMaxPlanes = 4096;
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_plane_partials[2 * kNoAllocMaxPlanes];

__device__ __forceinline__ double nb_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// One block per z-plane: sum of r^2 and b^2 over the plane (natural layout),
// written to the plane's slot.  Every slot is written before it is read, so
// nothing needs clearing between calls.
__global__ void __launch_bounds__(kNoAllocThreads)
k_residual_planes(Geom g, SolveParams sp, double scale, const float *__restrict__ rhs,
                  const float *__restrict__ p, double *__restrict__ partials) {
    const int k = blockIdx.x;
    const int n = g.W * g.H;
    const size_t sy = (size_t)g.W, sz = (size_t)g.W * g.H;
    double r2 = 0.0, b2 = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int i = t % g.W, j = t / g.W;
        const size_t c = (size_t)t + sz * (size_t)k;
        // Same arithmetic as the solver's residual kernels: A p in deviation
        // form sum_nb (p_c - p_nb) (+ p_c per Dirichlet ghost) in FP32, then
        // b, r and the squares in FP64.
        const double b = scale * (double)rhs[c];
        const float pc = p[c];
        const OpenFaces &o = sp.open;
        const bool dir = sp.dirichlet;
        float d = 0.0f;
        if (dir) {
            d = (float)((i == 0 && o.xlo) + (i == g.W - 1 && o.xhi) + (j == 0 && o.ylo) + (j == g.H - 1 && o.yhi) +
                        (k == 0 && o.zlo) + (k == g.D - 1 && o.zhi)) * pc;
        }
        if (i > 0) d += pc - p[c - 1];
        if (i < g.W - 1) d += pc - p[c + 1];
        if (j > 0) d += pc - p[c - sy];
        if (j < g.H - 1) d += pc - p[c + sy];
        if (k > 0) d += pc - p[c - sz];
        if (k < g.D - 1) d += pc - p[c + sz];
        const double r = b - (double)d;
        r2 += r * r;
        b2 += b * b;
    }
    __shared__ double s_r[kNoAllocThreads / 32], s_b[kNoAllocThreads / 32];
    r2 = nb_warp_sum(r2);
    b2 = nb_warp_sum(b2);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_r[wid] = r2; s_b[wid] = b2; }
    __syncthreads();
    if (wid == 0) {
        r2 = lane < kNoAllocThreads / 32 ? s_r[lane] : 0.0;
        b2 = lane < kNoAllocThreads / 32 ? s_b[lane] : 0.0;
        r2 = nb_warp_sum(r2);
        b2 = nb_warp_sum(b2);
        if (lane == 0) { partials[2 * k] = r2; partials[2 * k + 1] = b2; }
    }
}

// Sums the plane pairs in plane order and writes {||r||, ||b||}.
__global__ void __launch_bounds__(1024)
k_residual_planes_total(const double *__restrict__ partials, int planes, double *__restrict__ out2) {
    __shared__ double s_r[32], s_b[32];
    double r2 = 0.0, b2 = 0.0;
    for (int t = threadIdx.x; t < planes; t += blockDim.x) { r2 += partials[2 * t]; b2 += partials[2 * t + 1]; }
    r2 = nb_warp_sum(r2);
    b2 = nb_warp_sum(b2);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_r[wid] = r2; s_b[wid] = b2; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x / 32;
        r2 = lane < nw ? s_r[lane] : 0.0;
        b2 = lane < nw ? s_b[lane] : 0.0;
        r2 = nb_warp_sum(r2);
        b2 = nb_warp_sum(b2);
        if (lane == 0) { out2[0] = sqrt(r2); out2[1] = sqrt(b2); }
    }
}

} // namespace blz

using namespace blz;

namespace {
// Device address of g_plane_partials per device.  In host code the array's
// name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, looked up once per device with that device current.
std::mutex g_scratch_mu;
double *g_scratch_addr[kNoAllocMaxDevices] = {};
// Failures are reported through blz_last_error(NULL), like every other call
// made without a solver.
int noalloc_fail(int code, const char *msg, cudaError_t e = cudaSuccess) {
    char buf[256];
    if (e != cudaSuccess) std::snprintf(buf, sizeof buf, "blz_residual_noalloc: %s: %s", msg, cudaGetErrorString(e));
    else std::snprintf(buf, sizeof buf, "blz_residual_noalloc: %s", msg);
    blz::set_thread_error(buf);
    return code;
}
} // namespace

extern "C" {

int blz_residual_noalloc(const blz_params *prm, const float *rhs_dev, const float *p_dev, double *out2_dev,
                         void *cuda_stream) {
    if (!prm || !rhs_dev || !p_dev || !out2_dev) return noalloc_fail(BLZ_ERR_ARG, "null argument");
    if (prm->width < 4 || prm->height < 4 || prm->depth < 4)
        return noalloc_fail(BLZ_ERR_ARG, "grid dims must be >= 4");
    if (prm->depth > kNoAllocMaxPlanes)
        return noalloc_fail(BLZ_ERR_ARG, "depth exceeds the 4096 z-planes the static residual scratch holds");
    if ((long long)prm->width * prm->height > (1LL << 30) || (long long)prm->width * prm->height * prm->depth > (1LL << 31))
        return noalloc_fail(BLZ_ERR_ARG, "grid too large for 32-bit plane indexing");
    if (!(prm->dt > 0.0f) || !(prm->density > 0.0f) || !(prm->dx > 0.0f))
        return noalloc_fail(BLZ_ERR_ARG, "dx, dt and density must be positive");
    // The same check as blz_create: an unknown boundary mode is an error, not
    // a silent Neumann solve.
    if (prm->bc_mode != BLZ_BC_REF_COMPAT && prm->bc_mode != BLZ_BC_FREE_SURFACE)
        return noalloc_fail(BLZ_ERR_ARG, "bad bc_mode");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(BLZ_ERR_CUDA, "cudaGetDevice", e);
    if (dev < 0 || dev >= kNoAllocMaxDevices) return noalloc_fail(BLZ_ERR_ARG, "device ordinal beyond 63");
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            void *addr = nullptr;
            e = cudaGetSymbolAddress(&addr, g_plane_partials);
            if (e != cudaSuccess) return noalloc_fail(BLZ_ERR_CUDA, "cudaGetSymbolAddress(g_plane_partials)", e);
            g_scratch_addr[dev] = static_cast<double *>(addr);
        }
        scratch = g_scratch_addr[dev];
    }
    Geom g{};
    g.W = prm->width; g.H = prm->height; g.D = prm->depth;
    g.dx = prm->dx; g.dt = prm->dt; g.inv_dx = 1.0f / prm->dx;
    SolveParams sp{};
    sp.scale = (prm->density * prm->dx * prm->dx) / prm->dt;
    sp.scale_d = (double)prm->density * (double)prm->dx * (double)prm->dx / (double)prm->dt;
    sp.open = {!prm->closed_bounds[0], !prm->closed_bounds[1], !prm->closed_bounds[3],
               !prm->closed_bounds[2], !prm->closed_bounds[4], !prm->closed_bounds[5]};
    sp.dirichlet = prm->bc_mode == BLZ_BC_FREE_SURFACE;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    k_residual_planes<<<g.D, kNoAllocThreads, 0, st>>>(g, sp, sp.scale_d, rhs_dev, p_dev, scratch);
    k_residual_planes_total<<<1, 1024, 0, st>>>(scratch, g.D, out2_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(BLZ_ERR_CUDA, "residual kernel launch", e);
    return BLZ_OK;
}

} // extern "C"
