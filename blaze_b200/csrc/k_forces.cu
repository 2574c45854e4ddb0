// k_forces.cu — cooldown, drag, vorticity confinement, buoyancy, wind and
// turbulence (reference src/FluidSolver.cu:118-390), in gather form.
//
// The reference scatters confinement and pseudo-curl forces with float
// atomics (FluidSolver.cu:242-247, 287-292).  Here every face gathers the
// contributions of its two adjacent cells, which makes the pass deterministic
// and free of atomics.  Vorticity, buoyancy and wind only touch a face's own
// value, so they are fused into one in-place face pass.
#include <algorithm>

#include "kernels.cuh"

namespace blz {

dim3 face_block() { return dim3(32, 4, 2); }
dim3 face_grid(const Geom &g) {
    const dim3 b = face_block();
    return dim3((g.W + 1 + b.x - 1) / b.x, (g.H + 1 + b.y - 1) / b.y, (g.D + 1 + b.z - 1) / b.z);
}
static dim3 cell_grid(const Geom &g, dim3 b) {
    return dim3((g.W + b.x - 1) / b.x, (g.H + b.y - 1) / b.y, (g.D + b.z - 1) / b.z);
}

// temperature_cooldown_kernel / apply_drag_kernel (FluidSolver.cu:118-140).
__global__ void k_scale(float *__restrict__ a, size_t n, float s) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a[i] *= s;
}

void launch_scale(float *a, size_t n, float s, cudaStream_t st) {
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 16);
    k_scale<<<blocks, threads, 0, st>>>(a, n, s);
}

// computeVorticity (FluidSolver.cu:174-201) for cells 1..n-2 in each axis:
// centred differences of trilinear samples at the neighbouring cell centres.
__global__ void k_vort_omega(Geom g, const float *__restrict__ U, const float *__restrict__ V,
                             const float *__restrict__ W, float *__restrict__ ox,
                             float *__restrict__ oy, float *__restrict__ oz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i < 1 || j < 1 || k < 1 || i > g.W - 2 || j > g.H - 2 || k > g.D - 2) return;
    const FieldRef u = fU(U, g), v = fV(V, g), w = fW(W, g);
    const float dx = g.dx, r = g.inv_dx;
    const float x0 = ((float)(i - 1) + 0.5f) * dx, x1 = ((float)i + 0.5f) * dx, x2 = ((float)(i + 1) + 0.5f) * dx;
    const float y0 = ((float)(j - 1) + 0.5f) * dx, y1 = ((float)j + 0.5f) * dx, y2 = ((float)(j + 1) + 0.5f) * dx;
    const float z0 = ((float)(k - 1) + 0.5f) * dx, z1 = ((float)k + 0.5f) * dx, z2 = ((float)(k + 1) + 0.5f) * dx;
    const float w_121 = trilinear(w, r, x1, y2, z1), w_101 = trilinear(w, r, x1, y0, z1);
    const float v_112 = trilinear(v, r, x1, y1, z2), v_110 = trilinear(v, r, x1, y1, z0);
    const float u_112 = trilinear(u, r, x1, y1, z2), u_110 = trilinear(u, r, x1, y1, z0);
    const float w_211 = trilinear(w, r, x2, y1, z1), w_011 = trilinear(w, r, x0, y1, z1);
    const float v_211 = trilinear(v, r, x2, y1, z1), v_011 = trilinear(v, r, x0, y1, z1);
    const float u_121 = trilinear(u, r, x1, y2, z1), u_101 = trilinear(u, r, x1, y0, z1);
    const float s = 2.0f * dx;
    const size_t c = lin(i, j, k, g.W, g.H);
    ox[c] = (w_121 - w_101 - (v_112 - v_110)) / s;
    oy[c] = (u_112 - u_110 - (w_211 - w_011)) / s;
    oz[c] = (v_211 - v_011 - (u_121 - u_101)) / s;
}

void launch_vort_omega(const Geom &g, const float *U, const float *V, const float *W, float *ox,
                       float *oy, float *oz, cudaStream_t st) {
    const dim3 b(32, 4, 2);
    k_vort_omega<<<cell_grid(g, b), b, 0, st>>>(g, U, V, W, ox, oy, oz);
}

// vorticity_confinement_kernel (FluidSolver.cu:203-248) for 2 <= i <= W-3
// (same for j, k): force = eps*dx*(grad|omega| x omega) with omega clamped to
// the local speed.  Stores the per-face half increment 0.5*dt*force.
__global__ void k_vort_force(Geom g, const float *__restrict__ U, const float *__restrict__ V,
                             const float *__restrict__ W, const float *__restrict__ ox,
                             const float *__restrict__ oy, const float *__restrict__ oz,
                             ForceParams fp, float *__restrict__ fx, float *__restrict__ fy,
                             float *__restrict__ fz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i < 2 || j < 2 || k < 2 || i > g.W - 3 || j > g.H - 3 || k > g.D - 3) return;
    const size_t sy = (size_t)g.W, sz = (size_t)g.W * g.H;
    const size_t c = lin(i, j, k, g.W, g.H);
    auto mag = [&](size_t q) { return len3(__ldg(ox + q), __ldg(oy + q), __ldg(oz + q)); };
    const float s = 2.0f * g.dx;
    const float gx = (mag(c + 1) - mag(c - 1)) / s;
    const float gy = (mag(c + sy) - mag(c - sy)) / s;
    const float gz = (mag(c + sz) - mag(c - sz)) / s;
    float wx = __ldg(ox + c), wy = __ldg(oy + c), wz = __ldg(oz + c);
    const float px = ((float)i + 0.5f) * g.dx, py = ((float)j + 0.5f) * g.dx, pz = ((float)k + 0.5f) * g.dx;
    const float vx = trilinear(fU(U, g), g.inv_dx, px, py, pz);
    const float vy = trilinear(fV(V, g), g.inv_dx, px, py, pz);
    const float vz = trilinear(fW(W, g), g.inv_dx, px, py, pz);
    const float speed = len3(vx, vy, vz);
    const float onorm = len3(wx, wy, wz) + fp.tiny;
    if (onorm > speed) { wx = speed * wx / onorm; wy = speed * wy / onorm; wz = speed * wz / onorm; }
    const float sc = fp.conf * g.dx, h = 0.5f * g.dt;
    fx[c] = h * (sc * (gy * wz - gz * wy));
    fy[c] = h * (sc * (gz * wx - gx * wz));
    fz[c] = h * (sc * (gx * wy - gy * wx));
}

void launch_vort_force(const Geom &g, const float *U, const float *V, const float *W,
                       const float *ox, const float *oy, const float *oz, const ForceParams &fp,
                       float *fx, float *fy, float *fz, cudaStream_t st) {
    const dim3 b(32, 4, 2);
    k_vort_force<<<cell_grid(g, b), b, 0, st>>>(g, U, V, W, ox, oy, oz, fp, fx, fy, fz);
}

__device__ __forceinline__ bool vort_active(const Geom &g, int i, int j, int k) {
    return i >= 2 && j >= 2 && k >= 2 && i <= g.W - 3 && j <= g.H - 3 && k <= g.D - 3;
}

// One in-place pass over every face: confinement gather, then buoyancy
// (add_buoyancy_kernel, FluidSolver.cu:142-156), then the wind relaxation in
// the two-voxel slabs at both ends of the wind axis (add_wind_kernel,
// FluidSolver.cu:337-390) — the reference's order.
__global__ void k_face_forces(Geom g, float *__restrict__ U, float *__restrict__ V,
                              float *__restrict__ W, const float *__restrict__ T,
                              const float *__restrict__ fx, const float *__restrict__ fy,
                              const float *__restrict__ fz, ForceParams fp, const float *__restrict__ Dn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.W || j > g.H || k > g.D) return;
    bool in_slab = false;
    float nU = 0.0f, nV = 0.0f, nW = 0.0f;
    if (fp.wind_on) {
        in_slab = fp.wind_along_x ? (i < 2 || i >= g.W - 1) : (k < 2 || k >= g.D - 1);
        if (in_slab) {
            const float x = (float)i * g.dx, y = (float)j * g.dx, z = (float)k * g.dx + fp.wind_offset;
            nU = fp.wind_turb_amp * perlin(x, y, z, fp.wind_freq, 123);
            nV = fp.wind_turb_amp * perlin(x, y, z, fp.wind_freq, 456);
            nW = fp.wind_turb_amp * perlin(x, y, z, fp.wind_freq, 789);
        }
    }
    const float one_m = 1.0f - g.dt;
    if (j < g.H && k < g.D) {                     // U face
        const size_t q = lin(i, j, k, g.W + 1, g.H);
        float u = U[q];
        if (fp.vort_on) {
            if (vort_active(g, i - 1, j, k)) u += __ldg(fx + lin(i - 1, j, k, g.W, g.H));
            if (vort_active(g, i, j, k)) u += __ldg(fx + lin(i, j, k, g.W, g.H));
        }
        if (in_slab) u = u * one_m + (fp.wind_amp * ((fp.wind_along_x ? fp.wind_dir_sign : 0.0f) + nU)) * g.dt;
        U[q] = u;
    }
    if (i < g.W && k < g.D) {                     // V face
        const size_t q = lin(i, j, k, g.W, g.H + 1);
        float v = V[q];
        if (fp.vort_on) {
            if (vort_active(g, i, j - 1, k)) v += __ldg(fy + lin(i, j - 1, k, g.W, g.H));
            if (vort_active(g, i, j, k)) v += __ldg(fy + lin(i, j, k, g.W, g.H));
        }
        if (fp.buoy_on) {
            const float px = ((float)i + 0.5f) * g.dx, py = (float)j * g.dx, pz = ((float)k + 0.5f) * g.dx;
            const float temp = trilinear(fT(T, g), g.inv_dx, px, py, pz);
            if (fp.dens_on) {                         // target mode: the density's weight pulls down
                const float rho = trilinear(fT(Dn, g), g.inv_dx, px, py, pz);
                v += g.dt * ((fp.beta * temp - fp.alpha * rho) * fp.grav);
            } else {
                v += g.dt * (fp.beta * temp * fp.grav);
            }
        }
        if (in_slab) v = v * one_m + (fp.wind_amp * nV) * g.dt;
        V[q] = v;
    }
    if (i < g.W && j < g.H) {                     // W face
        const size_t q = lin(i, j, k, g.W, g.H);
        float w = W[q];
        if (fp.vort_on) {
            if (vort_active(g, i, j, k - 1)) w += __ldg(fz + lin(i, j, k - 1, g.W, g.H));
            if (vort_active(g, i, j, k)) w += __ldg(fz + lin(i, j, k, g.W, g.H));
        }
        if (in_slab) w = w * one_m + (fp.wind_amp * ((fp.wind_along_x ? 0.0f : fp.wind_dir_sign) + nW)) * g.dt;
        W[q] = w;
    }
}

void launch_face_forces(const Geom &g, float *U, float *V, float *W, const float *T,
                        const float *fx, const float *fy, const float *fz, const ForceParams &fp,
                        cudaStream_t st, const float *Dn) {
    k_face_forces<<<face_grid(g), face_block(), 0, st>>>(g, U, V, W, T, fx, fy, fz, fp, Dn);
}

__device__ __forceinline__ float fit01(float v, float a, float b, float lo, float hi) {
    return fmaxf(fminf((v - a) / (b - a), 1.0f), 0.0f) * (hi - lo) + lo;   // FluidSolver.cu:250-252
}

// compute_turbulence_kernel (FluidSolver.cu:295-335): masked Perlin noise per
// face; the noise lattice position is the face index plus a time offset.
__global__ void k_turb_noise(Geom g, const float *__restrict__ T, const float *__restrict__ U,
                             const float *__restrict__ V, const float *__restrict__ W,
                             float *__restrict__ nU, float *__restrict__ nV, float *__restrict__ nW,
                             ForceParams fp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.W || j > g.H || k > g.D) return;
    const FieldRef t = fT(T, g), u = fU(U, g), v = fV(V, g), w = fW(W, g);
    const float r = g.inv_dx;
    auto mask = [&](float px, float py, float pz) {
        const float tm = fit01(trilinear(t, r, px, py, pz), fp.tr0, fp.tr1, 1.0f, 0.0f);
        const float sp = len3(trilinear(u, r, px, py, pz), trilinear(v, r, px, py, pz),
                              trilinear(w, r, px, py, pz));
        return tm * fit01(sp, fp.vr0, fp.vr1, 0.0f, 1.0f);
    };
    const float fi = (float)i, fj = (float)j, fk = (float)k, dx = g.dx;
    if (j < g.H && k < g.D) {
        const float m = mask(fi * dx, (fj + 0.5f) * dx, (fk + 0.5f) * dx);
        nU[lin(i, j, k, g.W + 1, g.H)] =
            m == 0.0f ? 0.0f : m * fp.turb_amp * perlin(fi + fp.turb_offset, fj, fk, fp.turb_freq, 123);
    }
    if (i < g.W && k < g.D) {
        const float m = mask((fi + 0.5f) * dx, fj * dx, (fk + 0.5f) * dx);
        nV[lin(i, j, k, g.W, g.H + 1)] =
            m == 0.0f ? 0.0f : m * fp.turb_amp * perlin(fi, fj + fp.turb_offset, fk, fp.turb_freq, 123);
    }
    if (i < g.W && j < g.H) {
        const float m = mask((fi + 0.5f) * dx, (fj + 0.5f) * dx, fk * dx);
        nW[lin(i, j, k, g.W, g.H)] =
            m == 0.0f ? 0.0f : m * fp.turb_amp * perlin(fi, fj, fk + fp.turb_offset, fp.turb_freq, 123);
    }
}

void launch_turb_noise(const Geom &g, const float *T, const float *U, const float *V,
                       const float *W, float *nU, float *nV, float *nW, const ForceParams &fp,
                       cudaStream_t st) {
    k_turb_noise<<<face_grid(g), face_block(), 0, st>>>(g, T, U, V, W, nU, nV, nW, fp);
}

// Pseudo-curl of the noise field at cell (i,j,k) (add_curl_noise_kernel,
// FluidSolver.cu:271-293), rescaled to the cell's mean noise speed and
// multiplied by 0.5*dt.  dudx and dwdz subtract the V noise, as the
// reference does (lines 276, 278).
__device__ __forceinline__ float3 pseudo_curl(const Geom &g, const float *__restrict__ nU,
                                              const float *__restrict__ nV,
                                              const float *__restrict__ nW, float tiny, int i,
                                              int j, int k) {
    const float u0 = __ldg(nU + lin(i, j, k, g.W + 1, g.H)), u1 = __ldg(nU + lin(i + 1, j, k, g.W + 1, g.H));
    const float v0 = __ldg(nV + lin(i, j, k, g.W, g.H + 1)), v1 = __ldg(nV + lin(i, j + 1, k, g.W, g.H + 1));
    const float w0 = __ldg(nW + lin(i, j, k, g.W, g.H)), w1 = __ldg(nW + lin(i, j, k + 1, g.W, g.H));
    // Explicit roundings: where the differences are equal (e.g. masked-out
    // noise on three faces) the curl must be exactly zero.  A contracted
    // fma(a, s, -b*s) leaves a rounding residue instead, which the
    // normalisation below inflates to the full noise speed in an arbitrary
    // direction.
    const float dudx = __fmul_rn(__fsub_rn(u1, v0), g.inv_dx);
    const float dvdy = __fmul_rn(__fsub_rn(v1, v0), g.inv_dx);
    const float dwdz = __fmul_rn(__fsub_rn(w1, v0), g.inv_dx);
    float cx = __fsub_rn(dvdy, dwdz), cy = __fsub_rn(dwdz, dudx), cz = __fsub_rn(dudx, dvdy);
    const float avg = len3((u0 + u1) / 2.0f, (v0 + v1) / 2.0f, (w0 + w1) / 2.0f);
    const float den = len3(cx, cy, cz) + tiny;
    const float h = 0.5f * g.dt;
    return make_float3(h * (avg * cx / den), h * (avg * cy / den), h * (avg * cz / den));
}

__global__ void k_turb_apply(Geom g, float *__restrict__ U, float *__restrict__ V,
                             float *__restrict__ W, const float *__restrict__ nU,
                             const float *__restrict__ nV, const float *__restrict__ nW,
                             ForceParams fp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.W || j > g.H || k > g.D) return;
    const bool self = i < g.W && j < g.H && k < g.D;
    float3 c = make_float3(0.f, 0.f, 0.f);
    if (self) c = pseudo_curl(g, nU, nV, nW, fp.tiny, i, j, k);
    if (j < g.H && k < g.D) {
        const size_t q = lin(i, j, k, g.W + 1, g.H);
        float u = U[q];
        if (i >= 1) u += pseudo_curl(g, nU, nV, nW, fp.tiny, i - 1, j, k).x;
        if (self) u += c.x;
        U[q] = u;
    }
    if (i < g.W && k < g.D) {
        const size_t q = lin(i, j, k, g.W, g.H + 1);
        float v = V[q];
        if (j >= 1) v += pseudo_curl(g, nU, nV, nW, fp.tiny, i, j - 1, k).y;
        if (self) v += c.y;
        V[q] = v;
    }
    if (i < g.W && j < g.H) {
        const size_t q = lin(i, j, k, g.W, g.H);
        float w = W[q];
        if (k >= 1) w += pseudo_curl(g, nU, nV, nW, fp.tiny, i, j, k - 1).z;
        if (self) w += c.z;
        W[q] = w;
    }
}

void launch_turb_apply(const Geom &g, float *U, float *V, float *W, const float *nU,
                       const float *nV, const float *nW, const ForceParams &fp, cudaStream_t st) {
    k_turb_apply<<<face_grid(g), face_block(), 0, st>>>(g, U, V, W, nU, nV, nW, fp);
}

__global__ void k_perlin(const float *__restrict__ pos3, int n, float scale, int seed,
                         float *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = perlin(pos3[3 * t], pos3[3 * t + 1], pos3[3 * t + 2], scale, seed);
}

void launch_perlin(const float *pos3, int n, float scale, int seed, float *out, cudaStream_t st) {
    if (n > 0) k_perlin<<<(n + 255) / 256, 256, 0, st>>>(pos3, n, scale, seed, out);
}

} // namespace blz
