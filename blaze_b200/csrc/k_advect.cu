// k_advect.cu — RK3 semi-Lagrangian advection with tricubic interpolation
// (reference src/FluidSolver.cu:431-456, launched for T, U, V, W at 942-945).
//
// One kernel advances all four fields: the thread at (i,j,k) of the union
// face range produces T(i,j,k), U(i,j,k), V(i,j,k) and W(i,j,k) where those
// exist, so the velocity neighbourhood each backtrace samples is shared in L1
// by the four traces of a thread and its warp neighbours.
#include "kernels.cuh"

namespace blz {

__device__ __forceinline__ void vel_at(const FieldRef &u, const FieldRef &v, const FieldRef &w,
                                       float r, float px, float py, float pz, float &vx, float &vy,
                                       float &vz) {
    vx = trilinear(u, r, px, py, pz);
    vy = trilinear(v, r, px, py, pz);
    vz = trilinear(w, r, px, py, pz);
}

// Backtrace from the sample point of src at (i,j,k) with trilinear velocity:
// RK3 (stages at 0.5 dt and 0.75 dt, weights 2/9, 3/9, 4/9;
// FluidSolver.cu:431-456), forward Euler (392-407) or midpoint RK2
// (409-429); then the tricubic sample at the departure point.
template <int SCHEME>
__device__ __forceinline__ void departure(const Geom &g, const FieldRef &src, const FieldRef &u, const FieldRef &v,
                                          const FieldRef &w, int i, int j, int k, float &qx, float &qy, float &qz) {
    const float r = g.inv_dx, dt = g.dt;
    const float px = ((float)i + src.ox) * g.dx, py = ((float)j + src.oy) * g.dx, pz = ((float)k + src.oz) * g.dx;
    float k1x, k1y, k1z;
    vel_at(u, v, w, r, px, py, pz, k1x, k1y, k1z);
    if (SCHEME == BLZ_ADVECT_EULER) {
        qx = px - dt * k1x; qy = py - dt * k1y; qz = pz - dt * k1z;
    } else if (SCHEME == BLZ_ADVECT_RK2) {
        const float h1 = 0.5f * dt;
        float mx, my, mz;
        vel_at(u, v, w, r, px - h1 * k1x, py - h1 * k1y, pz - h1 * k1z, mx, my, mz);
        qx = px - dt * mx; qy = py - dt * my; qz = pz - dt * mz;
    } else {
        float k2x, k2y, k2z, k3x, k3y, k3z;
        const float h1 = 0.5f * dt, h2 = 0.75f * dt;
        vel_at(u, v, w, r, px - h1 * k1x, py - h1 * k1y, pz - h1 * k1z, k2x, k2y, k2z);
        vel_at(u, v, w, r, px - h2 * k2x, py - h2 * k2y, pz - h2 * k2z, k3x, k3y, k3z);
        const float a = 2.0f / 9.0f, b = 3.0f / 9.0f, c = 4.0f / 9.0f;
        qx = px - dt * (a * k1x + b * k2x + c * k3x);
        qy = py - dt * (a * k1y + b * k2y + c * k3y);
        qz = pz - dt * (a * k1z + b * k2z + c * k3z);
    }
}

template <bool CLAMP, int SCHEME>
__device__ __forceinline__ float advect_one(const Geom &g, const FieldRef &src, const FieldRef &u,
                                            const FieldRef &v, const FieldRef &w, int i, int j,
                                            int k) {
    float qx, qy, qz;
    departure<SCHEME>(g, src, u, v, w, i, j, k, qx, qy, qz);
    return tricubic<CLAMP>(src, g.inv_dx, qx, qy, qz);
}

template <int SCHEME, bool DENS>
__global__ void __launch_bounds__(256)
k_advect(Geom g, const float *__restrict__ T, const float *__restrict__ U,
         const float *__restrict__ V, const float *__restrict__ W, float *__restrict__ Tn,
         float *__restrict__ Un, float *__restrict__ Vn, float *__restrict__ Wn,
         const float *__restrict__ D, float *__restrict__ Dn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.W || j > g.H || k > g.D) return;
    const FieldRef u = fU(U, g), v = fV(V, g), w = fW(W, g);
    if (i < g.W && j < g.H && k < g.D) {
        if (DENS) {                               // T and the density scalar share one backtrace
            float qx, qy, qz;
            departure<SCHEME>(g, fT(T, g), u, v, w, i, j, k, qx, qy, qz);
            Tn[lin(i, j, k, g.W, g.H)] = tricubic<true>(fT(T, g), g.inv_dx, qx, qy, qz);
            Dn[lin(i, j, k, g.W, g.H)] = tricubic<true>(fT(D, g), g.inv_dx, qx, qy, qz);
        } else {
            Tn[lin(i, j, k, g.W, g.H)] = advect_one<true, SCHEME>(g, fT(T, g), u, v, w, i, j, k);
        }
    }
    if (j < g.H && k < g.D)
        Un[lin(i, j, k, g.W + 1, g.H)] = advect_one<false, SCHEME>(g, u, u, v, w, i, j, k);
    if (i < g.W && k < g.D)
        Vn[lin(i, j, k, g.W, g.H + 1)] = advect_one<false, SCHEME>(g, v, u, v, w, i, j, k);
    if (i < g.W && j < g.H)
        Wn[lin(i, j, k, g.W, g.H)] = advect_one<false, SCHEME>(g, w, u, v, w, i, j, k);
}

template <int SCHEME>
static void launch_scheme(const Geom &g, const float *T, const float *U, const float *V, const float *W, float *Tn,
                          float *Un, float *Vn, float *Wn, cudaStream_t st, const float *D, float *Dn) {
    if (D && Dn)
        k_advect<SCHEME, true><<<face_grid(g), face_block(), 0, st>>>(g, T, U, V, W, Tn, Un, Vn, Wn, D, Dn);
    else
        k_advect<SCHEME, false><<<face_grid(g), face_block(), 0, st>>>(g, T, U, V, W, Tn, Un, Vn, Wn, D, Dn);
}

void launch_advect(const Geom &g, const float *T, const float *U, const float *V, const float *W,
                   float *Tn, float *Un, float *Vn, float *Wn, cudaStream_t st, int scheme, const float *D,
                   float *Dn) {
    if (scheme == BLZ_ADVECT_EULER) launch_scheme<BLZ_ADVECT_EULER>(g, T, U, V, W, Tn, Un, Vn, Wn, st, D, Dn);
    else if (scheme == BLZ_ADVECT_RK2) launch_scheme<BLZ_ADVECT_RK2>(g, T, U, V, W, Tn, Un, Vn, Wn, st, D, Dn);
    else launch_scheme<BLZ_ADVECT_RK3>(g, T, U, V, W, Tn, Un, Vn, Wn, st, D, Dn);
}

} // namespace blz
