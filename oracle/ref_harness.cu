// ref_harness.cu — drives the Blaze reference's own CUDA build.
//
// TEST INFRASTRUCTURE ONLY.  Built by `make -C oracle ref` into
// oracle/_ref/libblaze_ref.so, which compiles the reference's
// src/FluidSolver.cu and src/RenderEngine.cu where they lie (unmodified;
// included below; lodepng.cpp, which the renderer's PNG writer calls, is
// compiled from the reference's thirdparty/ tree) with the
// reference's documented flags.  It serves as (a) a parity pin: the tests run
// the reference's kernels on seeded inputs and compare the oracle with them,
// and (b) the reference timing arm of bench.py.  Nothing in the product links
// it.
//
// The harness reaches FluidSolver's private device buffers by compiling the
// reference with `private` defined as `public` (standard and third-party
// headers are included first, so only the reference's own classes see it).
#include <cassert>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <streambuf>
#include <string>
#include <vector>
#include <strings.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../thirdparty/rapidjson/document.h"
#include "../thirdparty/rapidjson/writer.h"
#include "../thirdparty/rapidjson/stringbuffer.h"

#include "../include/blaze_b200.h"

// Standard headers the reference's renderer and its image libraries
// (lodepng, tinyexr) use, included before `private` is redefined.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <limits>
#include <map>
#include <set>
#include <utility>

// Ray.h calls uint_as_float, a device function older CUDA releases declared
// and CUDA 12.9 no longer does; this maps it to the current intrinsic.
__device__ __forceinline__ float uint_as_float(unsigned int u) { return __uint_as_float(u); }

#define private public
#include "FluidSolver.cu"
#include "RenderEngine.cu"
#undef private

namespace {

struct RefSim {
    SceneSettings scn;
    Timer tmr;
    FluidSolver *fs = nullptr;
    std::string dir;
    int max_particles = 0;
};

__global__ void front_ptr_kernel(Grid **g, float **out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *out = (*g)->mFrontBuffer;
}

__global__ void ref_perlin_kernel(const float *pos, int n, float scale, int seed, float *out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = cudaNoise::perlinNoise(make_float3(pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]), scale, seed);
}

float *front_of(RefSim *r, int f) {
    Grid **g = f == 0 ? r->fs->d_mT : f == 1 ? r->fs->d_mU : f == 2 ? r->fs->d_mV : r->fs->d_mW;
    float **slot = nullptr;
    cudaMalloc(&slot, sizeof(float *));
    front_ptr_kernel<<<1, 1>>>(g, slot);
    float *p = nullptr;
    cudaMemcpy(&p, slot, sizeof p, cudaMemcpyDeviceToHost);
    cudaFree(slot);
    return p;
}

size_t n_of(const RefSim *r, int f) {
    const size_t W = r->scn.gridRes.x, H = r->scn.gridRes.y, D = r->scn.gridRes.z;
    switch (f) {
    case 0: case 4: case 5: return W * H * D;
    case 1: return (W + 1) * H * D;
    case 2: return W * (H + 1) * D;
    case 3: return W * H * (D + 1);
    }
    return 0;
}

} // namespace

extern "C" {

void *ref_create(const blz_params *p) {
    RefSim *r = new RefSim();
    std::memset(&r->scn, 0, sizeof r->scn);
    SceneSettings &s = r->scn;
    char tmpl[] = "/tmp/blaze_ref_XXXXXX";
    if (!mkdtemp(tmpl)) { delete r; return nullptr; }
    r->dir = tmpl;
    std::snprintf(s.sceneDir, sizeof s.sceneDir, "%s", tmpl);
    std::snprintf(s.sceneName, sizeof s.sceneName, "harness");
    std::snprintf(s.particleFile, sizeof s.particleFile, "src_0000.part");
    s.sourceAnimated = true;                       // re-read the file every frame
    s.sourceRange = make_int2(-1000000000, 1000000000);
    s.sourceMaxParticleCount = r->max_particles = p->max_particles > 0 ? p->max_particles : 1;
    s.domainBboxMin = make_float3(p->domain_min[0], p->domain_min[1], p->domain_min[2]);
    s.domainBboxMax = make_float3(p->domain_max[0], p->domain_max[1], p->domain_max[2]);
    for (int i = 0; i < 6; ++i) s.closedBounds[i] = p->closed_bounds[i] != 0;
    s.maxIterSolve = p->max_iter;
    s.dx = p->dx;
    s.dt = p->dt;
    s.gridRes = make_int3(p->width, p->height, p->depth);
    s.density = p->density;
    s.gravity = p->gravity;
    s.buoyancy = p->buoyancy;
    s.coolingRate = p->cooling_rate;
    s.vorticityConf = p->vorticity_conf;
    s.drag = p->drag;
    s.windDir = p->wind_dir;
    s.windAmp = p->wind_amp;
    s.windSpeed = p->wind_speed;
    s.windTurbAmp = p->wind_turb_amp;
    s.windTurbScale = p->wind_turb_scale;
    s.turbulence_amp = p->turbulence_amp;
    s.turbulence_scale = p->turbulence_scale;
    s.turbMaskTempRamp = make_float2(p->turb_mask_temp_ramp[0], p->turb_mask_temp_ramp[1]);
    s.turbMaskVelRamp = make_float2(p->turb_mask_vel_ramp[0], p->turb_mask_vel_ramp[1]);
    r->tmr.iter = 0;
    r->tmr.time = 0.0f;
    r->fs = new FluidSolver(&r->tmr, &r->scn);
    return r;
}

void ref_destroy(void *h) {
    RefSim *r = (RefSim *)h;
    if (!r) return;
    delete r->fs;
    char path[512];
    std::snprintf(path, sizeof path, "rm -rf '%s'", r->dir.c_str());
    if (system(path) != 0) { /* best effort cleanup */ }
    delete r;
}

// The sweep count of the next solves (FluidSolver::mMaxIter, set from
// SceneSettings::maxIterSolve by the constructor, FluidSolver.cu:676 and
// read by project(), 841).
void ref_set_max_iter(void *h, int n) { ((RefSim *)h)->fs->mMaxIter = n; }

void ref_set_time(void *h, int iter, float time) {
    RefSim *r = (RefSim *)h;
    r->tmr.iter = iter;
    r->tmr.time = time;
}

// Writes the particles as the .part file the reference parses for the
// current frame (Parser.h:181-188).
int ref_set_particles(void *h, const float *rec8, int n) {
    RefSim *r = (RefSim *)h;
    if (n < 0 || n > r->max_particles) return -2;
    char path[600];
    std::snprintf(path, sizeof path, "%s/src_%04d.part", r->scn.sceneDir, r->tmr.iter);
    FILE *f = std::fopen(path, "wb");
    if (!f) return -1;
    const size_t w = std::fwrite(rec8, sizeof(float) * 8, (size_t)n, f);
    std::fclose(f);
    return w == (size_t)n ? 0 : -1;
}

int ref_add_source(void *h) { ((RefSim *)h)->fs->addSource(); return cudaGetLastError() == cudaSuccess ? 0 : -1; }
int ref_step(void *h) { ((RefSim *)h)->fs->step(); return cudaGetLastError() == cudaSuccess ? 0 : -1; }
int ref_project(void *h) { ((RefSim *)h)->fs->project(); return cudaGetLastError() == cudaSuccess ? 0 : -1; }

// Individual stages with the launch shapes of FluidSolver::step
// (FluidSolver.cu:858-955) and FluidSolver::project (823-856).
int ref_stage(void *h, int stage) {
    RefSim *r = (RefSim *)h;
    FluidSolver *fs = r->fs;
    const int W = fs->mWidth, H = fs->mHeight, D = fs->mDepth;
    const dim3 block(8, 8, 8);
    const dim3 gridT(W / block.x, H / block.y, D / block.z);
    const dim3 gridU((W + 1) / block.x + 1, H / block.y, D / block.z);
    const dim3 gridV(W / block.x, (H + 1) / block.y + 1, D / block.z);
    const dim3 gridW(W / block.x, H / block.y, (D + 1) / block.z + 1);
    const dim3 gridUVW(W + 1 / block.x + 1, (H + 1) / block.y + 1, (D + 1) / block.z + 1);
    const dim3 gridP((W + 1) / block.x + 1, (H + 1) / block.y + 1, (D + 1) / block.z + 1);
    switch (stage) {
    case 0: temperature_cooldown_kernel<<<gridT, block>>>(fs->d_mT, fs->mCoolingRate, fs->mDt); break;
    case 1: apply_drag_kernel<<<gridUVW, block>>>(fs->d_mU, fs->d_mV, fs->d_mW, fs->mDrag, fs->mDt); break;
    case 2:
        copy_velocity_to_back_buffer_kernel<<<gridUVW, block>>>(fs->d_mU, fs->d_mV, fs->d_mW);
        vorticity_confinement_kernel<<<gridT, block>>>(fs->d_mT, fs->d_mU, fs->d_mV, fs->d_mW, fs->mVorticeConf, fs->mDx, fs->mDt);
        swap_vel_grids_kernel<<<1, 1>>>(fs->d_mU, fs->d_mV, fs->d_mW);
        break;
    case 3: add_buoyancy_kernel<<<gridV, block>>>(fs->d_mT, fs->d_mV, fs->mBuoyancy, fs->mGravity, fs->mDt); break;
    case 4:
        add_wind_kernel<<<gridUVW, block>>>(fs->d_mU, fs->d_mV, fs->d_mW, r->scn.windDir, r->scn.windAmp, r->scn.windSpeed,
                                           r->scn.windTurbAmp, r->scn.windTurbScale, fs->mDt, r->tmr.time);
        break;
    case 5:
        compute_turbulence_kernel<<<gridUVW, block>>>(fs->d_mT, fs->d_mU, fs->d_mV, fs->d_mW, fs->mTurbulenceAmp,
                                                     fs->mTurbulenceScale, fs->mTurbMaskTempRamp, fs->mTurbMaskVelRamp,
                                                     fs->mDt, r->tmr.time);
        add_curl_noise_kernel<<<gridT, block>>>(fs->d_mU, fs->d_mV, fs->d_mW, fs->mDx, fs->mDt);
        break;
    case 6:
        compute_divergence_kernel<<<gridT, block>>>(fs->d_mRhs, fs->d_mU, fs->d_mV, fs->d_mW, W, H, D, fs->mDensity, fs->mDx);
        break;
    case 7:
        gs_solve_kernel<<<dim3(W / 16, H / 16, 1), dim3(16, 16, 1)>>>(fs->d_mRhs, fs->d_mP, fs->mDensity, fs->mDx, fs->mDt,
                                                                      W, H, D, fs->mMaxIter);
        break;
    case 8:
        pressure_gradient_update_kernel<<<gridP, block>>>(fs->d_mP, fs->d_mU, fs->d_mV, fs->d_mW, W, H, D, fs->mDensity,
                                                          fs->mDx, fs->mDt);
        break;
    case 9:
        advect_RK3_kernel<<<gridT, block>>>(fs->d_mT, fs->d_mU, fs->d_mV, fs->d_mW, fs->mDt, true);
        advect_RK3_kernel<<<gridU, block>>>(fs->d_mU, fs->d_mU, fs->d_mV, fs->d_mW, fs->mDt, false);
        advect_RK3_kernel<<<gridV, block>>>(fs->d_mV, fs->d_mU, fs->d_mV, fs->d_mW, fs->mDt, false);
        advect_RK3_kernel<<<gridW, block>>>(fs->d_mW, fs->d_mU, fs->d_mV, fs->d_mW, fs->mDt, false);
        swap_grids_kernel<<<1, 1>>>(fs->d_mT, fs->d_mU, fs->d_mV, fs->d_mW);
        break;
    default: return -2;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ref_get_field(void *h, int f, float *dst) {
    RefSim *r = (RefSim *)h;
    const size_t n = n_of(r, f);
    if (!n) return -2;
    const float *src = f == 4 ? r->fs->d_mP : f == 5 ? r->fs->d_mRhs : front_of(r, f);
    return cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

int ref_set_field(void *h, int f, const float *src) {
    RefSim *r = (RefSim *)h;
    const size_t n = n_of(r, f);
    if (!n) return -2;
    float *dst = f == 4 ? r->fs->d_mP : f == 5 ? r->fs->d_mRhs : front_of(r, f);
    return cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}

// The reference's RenderEngine (RenderEngine.cu:250-365) on the harness
// solver's temperature field: the renderer fields of blz_render_params are
// copied into the simulation's SceneSettings, which RenderEngine reads.
void *ref_render_create(void *h, const blz_render_params *rp) {
    RefSim *r = (RefSim *)h;
    SceneSettings &s = r->scn;
    s.renderRes = make_int2(rp->width, rp->height);
    s.camFocal = rp->cam_focal;
    s.camAperture = rp->cam_aperture;
    s.camU = make_float3(rp->cam_u[0], rp->cam_u[1], rp->cam_u[2]);
    s.camV = make_float3(rp->cam_v[0], rp->cam_v[1], rp->cam_v[2]);
    s.camW = make_float3(rp->cam_w[0], rp->cam_w[1], rp->cam_w[2]);
    s.camTrans = make_float3(rp->cam_trans[0], rp->cam_trans[1], rp->cam_trans[2]);
    s.rndrPStep = rp->p_step;
    s.rndrSStep = rp->s_step;
    s.rndrCutoff = rp->cutoff;
    s.shaderDensityScale = rp->density_scale;
    s.shaderShadowDensityScale = rp->shadow_density_scale;
    s.shaderAbsorption = rp->absorption;
    s.shaderScattering = make_float3(rp->scattering[0], rp->scattering[1], rp->scattering[2]);
    s.shaderVolumeColor = make_float3(rp->volume_color[0], rp->volume_color[1], rp->volume_color[2]);
    s.shaderGain = rp->gain;
    s.shaderEmissionScale = rp->emission_scale;
    s.shaderTempRampSize = rp->ramp_size;
    s.shaderTempRange = make_float2(rp->temp_range[0], rp->temp_range[1]);
    for (int i = 0; i < rp->ramp_size; ++i) {
        s.shaderColorRampKeys[i] = rp->ramp_keys[i];
        s.shaderColorRampColors[i] = make_float3(rp->ramp_colors[i][0], rp->ramp_colors[i][1], rp->ramp_colors[i][2]);
    }
    s.multiScatterScale = rp->multi_scatter_scale;
    s.multiScatterDensityMask = make_float2(rp->multi_scatter_density_mask[0], rp->multi_scatter_density_mask[1]);
    s.multiScatterColor = make_float3(rp->multi_scatter_color[0], rp->multi_scatter_color[1], rp->multi_scatter_color[2]);
    s.multiScatterBlurIter = rp->multi_scatter_blur_iter;
    s.lightCount = rp->light_count;
    for (int i = 0; i < rp->light_count; ++i) {
        s.lightExposure[i] = rp->light_exposure[i];
        s.lightIntensity[i] = rp->light_intensity[i];
        s.lightSamples[i] = 1;
        s.lightDir[i] = make_float3(rp->light_dir[i][0], rp->light_dir[i][1], rp->light_dir[i][2]);
        s.lightColor[i] = make_float3(rp->light_color[i][0], rp->light_color[i][1], rp->light_color[i][2]);
    }
    std::snprintf(s.renderFile, sizeof s.renderFile, "render_####.exr");
    RenderEngine *e = new RenderEngine(&r->tmr, s);
    return cudaDeviceSynchronize() == cudaSuccess ? e : nullptr;
}

// One render of the solver's current T; device milliseconds in *ms.
int ref_render(void *h, void *eng, float *ms) {
    RefSim *r = (RefSim *)h;
    RenderEngine *e = (RenderEngine *)eng;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    e->render(r->fs->getTempGrid());
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.0f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms) *ms = t;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// The frame buffer (mRdrWidth * mRdrHeight float3, row 0 at the top).
int ref_render_get(void *eng, float *rgb) {
    RenderEngine *e = (RenderEngine *)eng;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1;
    std::memcpy(rgb, e->mFrameBuffer, sizeof(float) * 3 * (size_t)e->mRdrWidth * e->mRdrHeight);
    return 0;
}

void ref_render_destroy(void *eng) {
    delete (RenderEngine *)eng;
    cudaDeviceSynchronize();
}

int ref_perlin(const float *pos3, int n, float scale, int seed, float *out) {
    if (n <= 0) return 0;
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * 4 * (size_t)n) != cudaSuccess) return -1;
    cudaMemcpy(d, pos3, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    ref_perlin_kernel<<<(n + 255) / 256, 256>>>(d, n, scale, seed, d + 3 * (size_t)n);
    const cudaError_t e = cudaMemcpy(out, d + 3 * (size_t)n, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

} // extern "C"

// ---------------------------------------------------------------------------
// The reference's noise library (thirdparty/cuda-noise/cuda_noise.cuh, which
// FluidSolver.cu includes) at n positions: one function, selected by
// a.func, per launch.  Used to generate tests/golden/noise.npz.
// ---------------------------------------------------------------------------
namespace {
__global__ void ref_noise_kernel(blz_noise_args a, const float *pos, int n, float *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    using namespace cudaNoise;
    const float3 p = make_float3(pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]);
    const basisFunction bi = (basisFunction)a.basis, bo = (basisFunction)a.basis_out;
    float v = 0.0f;
    switch (a.func) {
    case BLZ_NOISE_CHECKER: v = checker(p, a.scale, a.seed); break;
    case BLZ_NOISE_DISCRETE: v = discreteNoise(p, a.scale, a.seed); break;
    case BLZ_NOISE_LINEARVALUE: v = linearValue(p, a.scale, a.seed); break;
    case BLZ_NOISE_FADEDVALUE: v = fadedValue(p, a.scale, a.seed); break;
    case BLZ_NOISE_CUBICVALUE: v = cubicValue(p, a.scale, a.seed); break;
    case BLZ_NOISE_PERLIN: v = perlinNoise(p, a.scale, a.seed); break;
    case BLZ_NOISE_SIMPLEX: v = simplexNoise(p, a.scale, a.seed); break;
    case BLZ_NOISE_WORLEY: v = worleyNoise(p, a.scale, a.seed, a.size, a.min_num, a.max_num, a.jitter); break;
    case BLZ_NOISE_SPOTS:
        v = spots(p, a.scale, a.seed, a.size, a.min_num, a.max_num, a.jitter, (profileShape)a.shape);
        break;
    case BLZ_NOISE_REPEATER_PERLIN: v = repeaterPerlin(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay); break;
    case BLZ_NOISE_REPEATER_PERLIN_BOUNDED:
        v = repeaterPerlinBounded(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay, a.threshold);
        break;
    case BLZ_NOISE_REPEATER_PERLIN_ABS: v = repeaterPerlinAbs(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay); break;
    case BLZ_NOISE_REPEATER_SIMPLEX: v = repeaterSimplex(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay); break;
    case BLZ_NOISE_REPEATER_SIMPLEX_ABS:
        v = repeaterSimplexAbs(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay);
        break;
    case BLZ_NOISE_REPEATER_SIMPLEX_BOUNDED:
        v = repeaterSimplexBounded(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay, a.threshold);
        break;
    case BLZ_NOISE_REPEATER: v = repeater(p, a.scale, a.seed, a.octaves, a.lacunarity, a.decay, bi); break;
    case BLZ_NOISE_FRACTAL_SIMPLEX:
        v = fractalSimplex(p, a.scale, a.seed, a.du, a.octaves, a.lacunarity, a.decay);
        break;
    case BLZ_NOISE_TURBULENCE: v = turbulence(p, a.scale, a.scale_out, a.seed, a.strength, bi, bo); break;
    case BLZ_NOISE_REPEATER_TURBULENCE:
        v = repeaterTurbulence(p, a.scale, a.scale_out, a.seed, a.strength, a.octaves, bi, bo);
        break;
    default: break;
    }
    out[t] = v;
}
} // namespace

extern "C" int ref_noise(const blz_noise_args *a, const float *pos3, int n, float *out) {
    if (n <= 0) return 0;
    if (!a || a->func < 0 || a->func >= BLZ_NOISE_COUNT || a->basis < 0 || a->basis > 8 || a->basis_out < 0 ||
        a->basis_out > 8 || a->min_num > a->max_num || a->octaves < 0 || a->octaves > 64)
        return -2;
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * 4 * (size_t)n) != cudaSuccess) return -1;
    cudaMemcpy(d, pos3, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    ref_noise_kernel<<<(n + 127) / 128, 128>>>(*a, d, n, d + 3 * (size_t)n);
    const cudaError_t e = cudaMemcpy(out, d + 3 * (size_t)n, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}
