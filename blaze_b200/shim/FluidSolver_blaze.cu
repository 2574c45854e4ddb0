// FluidSolver_blaze.cu — drop-in implementation of the reference's
// class FluidSolver (src/FluidSolver.h:38-110, unchanged) over the C ABI of
// libblaze_b200.so.
//
// A maintainer replaces src/FluidSolver.cu with this file and links
// libblaze_b200.so; main.cu and the renderer compile as before:
//   - FluidSolver(Timer*, SceneSettings*) / ~FluidSolver  -> blz_create / blz_destroy
//   - addSource(): the reference's Parser::sourceParticleParse and animated-
//     source rules (FluidSolver.cu:770-821), then blz_set_particles +
//     blz_add_source
//   - step(): blz_step with Timer::time; per-stage device times go into the
//     Timer fields so Timer::getStats() still reports them
//   - getTempGrid() (inline in the header) returns d_mT: a device Grid object
//     whose front buffer is re-pointed at the library's current T after
//     every step, so RenderEngine::render reads it through Grid::at.
// The class's other device buffers are not allocated (the library owns the
// fields); errors print the library's message and exit, as checkCudaErrors
// does in the reference.
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "FluidSolver.h"
#include "blaze_b200.h"

namespace {

std::mutex g_mu;
std::unordered_map<const FluidSolver *, blz_solver *> g_handle;

blz_solver *handle_of(const FluidSolver *fs) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_handle.find(fs);
    return it == g_handle.end() ? nullptr : it->second;
}

void die(blz_solver *s, int rc, const char *what) {
    std::fprintf(stderr, "blaze_b200 %s failed (%d): %s\n", what, rc, blz_last_error(s));
    std::exit(EXIT_FAILURE);
}

#define BLZ_CHECK(s, call)                 \
    do {                                   \
        int rc_ = (call);                  \
        if (rc_ != BLZ_OK) die(s, rc_, #call); \
    } while (0)

__global__ void shim_grid_new(Grid **slot, float *front, int w, int h, int d, float dx, SceneSettings scn) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        *slot = new Grid(front, front, w, h, d, 0.5f, 0.5f, 0.5f, dx, scn.domainBboxMin, scn.domainBboxMax,
                         false, scn);
}

// Re-points the T grid object at the library's current front buffer.
__global__ void shim_grid_repoint(Grid **slot, float *front, int w, int h, int d, float dx, SceneSettings scn) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        **slot = Grid(front, front, w, h, d, 0.5f, 0.5f, 0.5f, dx, scn.domainBboxMin, scn.domainBboxMax, false, scn);
}

__global__ void shim_grid_delete(Grid **slot) {
    if (threadIdx.x == 0 && blockIdx.x == 0) delete *slot;
}

blz_params params_from(const SceneSettings &s) {
    blz_params p;
    blz_default_params(&p);
    p.width = s.gridRes.x; p.height = s.gridRes.y; p.depth = s.gridRes.z;
    p.dx = s.dx; p.dt = s.dt;
    p.domain_min[0] = s.domainBboxMin.x; p.domain_min[1] = s.domainBboxMin.y; p.domain_min[2] = s.domainBboxMin.z;
    p.domain_max[0] = s.domainBboxMax.x; p.domain_max[1] = s.domainBboxMax.y; p.domain_max[2] = s.domainBboxMax.z;
    for (int i = 0; i < 6; ++i) p.closed_bounds[i] = s.closedBounds[i] ? 1 : 0;
    p.density = s.density; p.gravity = s.gravity; p.buoyancy = s.buoyancy;
    p.cooling_rate = s.coolingRate; p.vorticity_conf = s.vorticityConf; p.drag = s.drag;
    p.wind_dir = s.windDir; p.wind_amp = s.windAmp; p.wind_speed = s.windSpeed;
    p.wind_turb_amp = s.windTurbAmp; p.wind_turb_scale = s.windTurbScale;
    p.turbulence_amp = s.turbulence_amp; p.turbulence_scale = s.turbulence_scale;
    p.turb_mask_temp_ramp[0] = s.turbMaskTempRamp.x; p.turb_mask_temp_ramp[1] = s.turbMaskTempRamp.y;
    p.turb_mask_vel_ramp[0] = s.turbMaskVelRamp.x; p.turb_mask_vel_ramp[1] = s.turbMaskVelRamp.y;
    // The reference's solve: maxIterSolve sweeps, warm-started, Neumann at every face.
    p.max_iter = s.maxIterSolve;
    p.tol = 0.0;
    p.bc_mode = BLZ_BC_REF_COMPAT;
    p.gs_order = BLZ_GS_RB3D;
    p.reset_pressure = 0;
    p.max_particles = s.sourceMaxParticleCount > 0 ? s.sourceMaxParticleCount : 1;
    return p;
}

clock_t ms_to_clock(float ms) { return (clock_t)((double)ms * 1e-3 * CLOCKS_PER_SEC); }

} // namespace

FluidSolver::FluidSolver(Timer *tmr, SceneSettings *scn)
    : mScn(scn), mTmr(tmr), d_mT(nullptr), d_mU(nullptr), d_mV(nullptr), d_mW(nullptr),
      mByteSize(0), mByteSizeU(0), mByteSizeV(0), mByteSizeW(0),
      d_mTFront(nullptr), d_mTBack(nullptr), d_mUFront(nullptr), d_mUBack(nullptr),
      d_mVFront(nullptr), d_mVBack(nullptr), d_mWFront(nullptr), d_mWBack(nullptr),
      d_mRhs(nullptr), d_mP(nullptr),
      mSingleFrameSourceInit(false), mParticleCount(0),
      mWidth(scn->gridRes.x), mHeight(scn->gridRes.y), mDepth(scn->gridRes.z),
      mDensity(scn->density), mBuoyancy(scn->buoyancy), mCoolingRate(scn->coolingRate),
      mGravity(scn->gravity), mVorticeConf(scn->vorticityConf), mDrag(scn->drag),
      mTurbulenceAmp(scn->turbulence_amp), mTurbulenceScale(scn->turbulence_scale),
      mTurbMaskTempRamp(scn->turbMaskTempRamp), mTurbMaskVelRamp(scn->turbMaskVelRamp),
      mDx(scn->dx), mDt(scn->dt), mMaxIter(scn->maxIterSolve) {
    blz_params p = params_from(*scn);
    blz_solver *s = nullptr;
    BLZ_CHECK(nullptr, blz_create(&p, &s));
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_handle[this] = s;
    }
    const size_t n = (size_t)scn->sourceMaxParticleCount;
    h_mPartPos = (float3 *)std::malloc(n * sizeof(float3));
    h_mPartVel = (float3 *)std::malloc(n * sizeof(float3));
    h_mPartPscale = (float *)std::malloc(n * sizeof(float));
    h_mPartTemp = (float *)std::malloc(n * sizeof(float));
    d_mPartPos = nullptr; d_mPartVel = nullptr; d_mPartPscale = nullptr; d_mPartTemp = nullptr;
    checkCudaErrors(cudaMalloc((void **)&d_mT, sizeof(Grid *)));
    shim_grid_new<<<1, 1>>>(d_mT, (float *)blz_field_ptr(s, BLZ_FIELD_T), mWidth, mHeight, mDepth, mDx, *scn);
    checkCudaErrors(cudaGetLastError());
    checkCudaErrors(cudaDeviceSynchronize());
}

FluidSolver::~FluidSolver() {
    blz_solver *s = handle_of(this);
    shim_grid_delete<<<1, 1>>>(d_mT);
    cudaDeviceSynchronize();
    cudaFree(d_mT);
    blz_destroy(s);
    std::free(h_mPartPos); std::free(h_mPartVel); std::free(h_mPartPscale); std::free(h_mPartTemp);
    std::lock_guard<std::mutex> lk(g_mu);
    g_handle.erase(this);
}

void FluidSolver::addSource() {
    blz_solver *s = handle_of(this);
    mTmr->source_in = clock();
    if (!mScn->sourceAnimated ||
        (mScn->sourceAnimated && mTmr->iter >= mScn->sourceRange.x && mTmr->iter <= mScn->sourceRange.y)) {
        if (!mSingleFrameSourceInit || mScn->sourceAnimated) {
            Parser::sourceParticleParse(mScn, h_mPartPos, h_mPartVel, h_mPartPscale, h_mPartTemp, mParticleCount,
                                        mTmr->iter);
            std::vector<float> rec((size_t)mParticleCount * 8);
            for (int i = 0; i < mParticleCount; ++i) {
                float *r = &rec[(size_t)i * 8];
                r[0] = h_mPartPos[i].x; r[1] = h_mPartPos[i].y; r[2] = h_mPartPos[i].z;
                r[3] = h_mPartVel[i].x; r[4] = h_mPartVel[i].y; r[5] = h_mPartVel[i].z;
                r[6] = h_mPartPscale[i]; r[7] = h_mPartTemp[i];
            }
            BLZ_CHECK(s, blz_set_particles(s, rec.data(), mParticleCount));
            mSingleFrameSourceInit = true;
        }
        if (mParticleCount > 0) BLZ_CHECK(s, blz_add_source(s));
    }
    checkCudaErrors(cudaDeviceSynchronize());
    mTmr->source_out = clock();
}

void FluidSolver::project() {
    blz_solver *s = handle_of(this);
    blz_step_stats st;
    BLZ_CHECK(s, blz_project(s, &st));
}

void FluidSolver::step() {
    blz_solver *s = handle_of(this);
    blz_step_stats st;
    BLZ_CHECK(s, blz_step(s, mTmr->time, &st));
    shim_grid_repoint<<<1, 1>>>(d_mT, (float *)blz_field_ptr(s, BLZ_FIELD_T), mWidth, mHeight, mDepth, mDx, *mScn);
    checkCudaErrors(cudaGetLastError());
    checkCudaErrors(cudaDeviceSynchronize());
    // Device stage times in the reference's Timer brackets (FluidSolver.cu:866-949).
    mTmr->cooldown_in = mTmr->drag_in = mTmr->vorticity_in = mTmr->buoyancy_in = mTmr->wind_in = 0;
    mTmr->cooldown_out = mTmr->drag_out = mTmr->vorticity_out = mTmr->buoyancy_out = mTmr->wind_out = 0;
    mTmr->turbulence_in = 0; mTmr->turbulence_out = ms_to_clock(st.ms_forces);
    mTmr->computeDivergence_in = 0; mTmr->computeDivergence_out = ms_to_clock(st.ms_divergence);
    mTmr->gsSolve_in = 0; mTmr->gsSolve_out = ms_to_clock(st.ms_solve);
    mTmr->pressureGradientUpdate_in = 0; mTmr->pressureGradientUpdate_out = ms_to_clock(st.ms_gradient);
    mTmr->advect_in = 0; mTmr->advect_out = ms_to_clock(st.ms_advect);
}

// ---------------------------------------------------------------------------
// Test hooks: drive the drop-in class exactly as main.cu does, and read T
// through getTempGrid() the way RenderEngine's kernels do ((*grid)->at).
// ---------------------------------------------------------------------------
namespace {
struct ShimSim { SceneSettings scn; Timer tmr; FluidSolver *fs; };

__global__ void shim_read_T(Grid **grid, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i < (*grid)->mWidth) out[i + (size_t)(*grid)->mWidth * (j + (size_t)(*grid)->mHeight * k)] = (*grid)->at(i, j, k);
}
} // namespace

extern "C" {

void *blz_shim_create(const blz_params *p, const char *scene_dir, const char *particle_file, int animated) {
    ShimSim *r = new ShimSim();
    std::memset(&r->scn, 0, sizeof r->scn);
    SceneSettings &s = r->scn;
    std::snprintf(s.sceneDir, sizeof s.sceneDir, "%s", scene_dir);
    std::snprintf(s.particleFile, sizeof s.particleFile, "%s", particle_file);
    s.sourceAnimated = animated != 0;
    s.sourceRange = make_int2(-1000000000, 1000000000);
    s.sourceMaxParticleCount = p->max_particles;
    s.domainBboxMin = make_float3(p->domain_min[0], p->domain_min[1], p->domain_min[2]);
    s.domainBboxMax = make_float3(p->domain_max[0], p->domain_max[1], p->domain_max[2]);
    for (int i = 0; i < 6; ++i) s.closedBounds[i] = p->closed_bounds[i] != 0;
    s.maxIterSolve = p->max_iter; s.dx = p->dx; s.dt = p->dt;
    s.gridRes = make_int3(p->width, p->height, p->depth);
    s.density = p->density; s.gravity = p->gravity; s.buoyancy = p->buoyancy;
    s.coolingRate = p->cooling_rate; s.vorticityConf = p->vorticity_conf; s.drag = p->drag;
    s.windDir = p->wind_dir; s.windAmp = p->wind_amp; s.windSpeed = p->wind_speed;
    s.windTurbAmp = p->wind_turb_amp; s.windTurbScale = p->wind_turb_scale;
    s.turbulence_amp = p->turbulence_amp; s.turbulence_scale = p->turbulence_scale;
    s.turbMaskTempRamp = make_float2(p->turb_mask_temp_ramp[0], p->turb_mask_temp_ramp[1]);
    s.turbMaskVelRamp = make_float2(p->turb_mask_vel_ramp[0], p->turb_mask_vel_ramp[1]);
    r->tmr.iter = 0;
    r->tmr.time = 0.0f;
    r->fs = new FluidSolver(&r->tmr, &r->scn);
    return r;
}

void blz_shim_frame(void *h) {
    ShimSim *r = (ShimSim *)h;
    r->fs->addSource();
    r->fs->step();
    r->tmr.iter++;
    r->tmr.time += r->scn.dt;
}

int blz_shim_read_temp(void *h, float *host_out) {
    ShimSim *r = (ShimSim *)h;
    const int W = r->scn.gridRes.x, H = r->scn.gridRes.y, D = r->scn.gridRes.z;
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * (size_t)W * H * D) != cudaSuccess) return -1;
    shim_read_T<<<dim3((W + 127) / 128, H, D), 128>>>(r->fs->getTempGrid(), d);
    cudaError_t e = cudaMemcpy(host_out, d, sizeof(float) * (size_t)W * H * D, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

void blz_shim_destroy(void *h) {
    ShimSim *r = (ShimSim *)h;
    delete r->fs;
    delete r;
}

} // extern "C"
