// solver.cu — the C ABI of libblaze_b200.so: solver object, step
// orchestration and field access (reference src/FluidSolver.cu:671-955).
//
// Ownership follows the reference's FluidSolver: the solver owns every device
// buffer; parameters are copied at creation.  All work is ordered on one
// stream (library owned unless the caller sets one).  Errors are returned as
// BLZ_ERR_* codes with a message; nothing here exits the process.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <sys/stat.h>

#include "kernels.cuh"

using namespace blz;

struct blz_solver {
    blz_params P{};
    Geom g{};
    cudaStream_t st = nullptr;
    bool own_stream = false;
    int device = 0;
    float *T[2]{}, *U[2]{}, *V[2]{}, *W[2]{};
    float *Dn[2]{};                             // density scalar (density_field only)
    int cur = 0;                                // front = [cur]
    float *p_r = nullptr, *p_b = nullptr, *rhs_r = nullptr, *rhs_b = nullptr;
    // Defect-correction solve (params.defect_correction): the sweeps solve
    // A delta = b - A p for the correction delta (dl) with the defect as
    // right-hand side (df); afterwards p = RN(p + delta) and delta keeps the
    // exact rounding remainder, so p + delta carries the solution past the
    // FP32 floor.  sr/sx: the right-hand side and unknown the sweeps work on
    // (df/dl, or rhs/p without defect correction).
    float *df_r = nullptr, *df_b = nullptr, *dl_r = nullptr, *dl_b = nullptr;
    const float *sr_r = nullptr, *sr_b = nullptr;
    float *sx_r = nullptr, *sx_b = nullptr;
    bool defect_valid = false;                  // dl holds the remainder of the last solve
    float *scratch = nullptr;                   // 6 T-sized arrays (vorticity)
    // sourcing: compacted particle records, per-field index boxes and the
    // 8^3-cell bins (CSR) built on the host by blz_set_particles
    float *parts = nullptr;
    float *pdens = nullptr;                     // per-particle density (density_field only)
    int *boxes = nullptr, *bin_start = nullptr, *bin_list = nullptr, *active = nullptr;
    int n_parts = 0, cap_parts = 0, cap_list = 0, n_active = 0;
    int nbx = 0, nby = 0, nbz = 0;
    double *partials = nullptr;
    int n_partials = 0;
    double *d_norm2 = nullptr, *h_norm2 = nullptr;
    cudaEvent_t ev[10]{};
    long long launches = 0;
    blz_unet *warm = nullptr;                   // learned warm start (caller owned)
    int variant = -2;                           // sweep launch shape (-2: not chosen yet)
    // device-loop solve: instantiated graphs (one per check interval used)
    // and their control block
    struct SolveGraph {
        int chunk = 0;
        cudaGraphExec_t exec = nullptr;
        int body = 0, prologue = 0;
    };
    SolveGraph graphs[8];
    SolveCtl *ctl = nullptr, *h_ctl = nullptr;
    // automatic check interval (check_every < 0): the last solve's sweeps and
    // its measured cost of one residual check in sweeps
    int last_iters = 0;
    double check_ratio = 0.0;
    std::string err;
};

static thread_local std::string g_thread_err;

static int fail(blz_solver *s, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    g_thread_err = buf;
    return code;
}

namespace blz {
void set_thread_error(const char *msg) { g_thread_err = msg; }
} // namespace blz

#define CK(s, x)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess)                                                              \
            return fail((s), BLZ_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_));    \
    } while (0)

#define CKL(s)                                                                              \
    do {                                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                \
        if (e_ != cudaSuccess)                                                              \
            return fail((s), BLZ_ERR_CUDA, "kernel launch failed (%s:%d): %s", __FILE__,   \
                        __LINE__, cudaGetErrorString(e_));                                  \
    } while (0)

static size_t n_of(const blz_params &P, int f) {
    const size_t W = P.width, H = P.height, D = P.depth;
    switch (f) {
    case BLZ_FIELD_T: case BLZ_FIELD_P: case BLZ_FIELD_RHS: return W * H * D;
    case BLZ_FIELD_DENSITY: return P.density_field ? W * H * D : 0;
    case BLZ_FIELD_U: return (W + 1) * H * D;
    case BLZ_FIELD_V: return W * (H + 1) * D;
    case BLZ_FIELD_W: return W * H * (D + 1);
    default: return 0;
    }
}

static OpenFaces open_faces(const blz_params &P) {
    return {!P.closed_bounds[0], !P.closed_bounds[1], !P.closed_bounds[3],
            !P.closed_bounds[2], !P.closed_bounds[4], !P.closed_bounds[5]};
}

static SolveParams solve_params(const blz_params &P) {
    SolveParams sp{};
    sp.scale = (P.density * P.dx * P.dx) / P.dt;          // FluidSolver.cu:530
    sp.scale_d = (double)P.density * (double)P.dx * (double)P.dx / (double)P.dt;
    sp.open = open_faces(P);
    sp.dirichlet = P.bc_mode == BLZ_BC_FREE_SURFACE;
    return sp;
}

namespace blz {
SolveParams solve_params_of(const blz_params &P) { return solve_params(P); }
} // namespace blz

extern "C" {

int blz_default_params(blz_params *p) {
    if (!p) return fail(nullptr, BLZ_ERR_ARG, "null params");
    std::memset(p, 0, sizeof *p);
    p->width = p->height = p->depth = 64;
    p->dx = 1.0f / 64.0f;
    p->dt = 1.0f / 24.0f;
    p->domain_max[0] = p->domain_max[1] = p->domain_max[2] = 1.0f;
    for (int i = 0; i < 6; ++i) p->closed_bounds[i] = 1;
    p->density = 0.1f;
    p->gravity = -9.8f;
    p->wind_turb_scale = 1.0f;
    p->turbulence_scale = 1.0f;
    p->turb_mask_temp_ramp[0] = 1e30f; p->turb_mask_temp_ramp[1] = 2e30f;
    p->turb_mask_vel_ramp[0] = -1.0f; p->turb_mask_vel_ramp[1] = 0.0f;
    p->max_iter = 200;
    p->tol = 0.0;
    p->check_every = 10;
    p->bc_mode = BLZ_BC_REF_COMPAT;
    p->gs_order = BLZ_GS_RB3D;
    p->reset_pressure = 0;
    p->max_particles = 1 << 16;
    p->device_loop = 1;
    p->sweep_variant = -1;
    return BLZ_OK;
}

const char *blz_last_error(const blz_solver *s) { return s ? s->err.c_str() : g_thread_err.c_str(); }

long long blz_kernel_launches(const blz_solver *s) { return s ? s->launches : 0; }

size_t blz_field_size(const blz_solver *s, int field) { return s ? n_of(s->P, field) : 0; }

static void release(blz_solver *s) {
    if (!s) return;
    for (int b = 0; b < 2; ++b) {
        cudaFree(s->T[b]); cudaFree(s->U[b]); cudaFree(s->V[b]); cudaFree(s->W[b]); cudaFree(s->Dn[b]);
    }
    cudaFree(s->pdens);
    cudaFree(s->p_r); cudaFree(s->p_b); cudaFree(s->rhs_r); cudaFree(s->rhs_b);
    cudaFree(s->df_r); cudaFree(s->df_b); cudaFree(s->dl_r); cudaFree(s->dl_b);
    cudaFree(s->scratch);
    cudaFree(s->parts); cudaFree(s->boxes); cudaFree(s->bin_start); cudaFree(s->bin_list); cudaFree(s->active);
    cudaFree(s->partials); cudaFree(s->d_norm2);
    if (s->h_norm2) cudaFreeHost(s->h_norm2);
    for (auto &gr : s->graphs)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    cudaFree(s->ctl);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    for (auto &e : s->ev) if (e) cudaEventDestroy(e);
    if (s->own_stream && s->st) cudaStreamDestroy(s->st);
}

int blz_create(const blz_params *p, blz_solver **out) {
    if (!p || !out) return fail(nullptr, BLZ_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->width < 4 || p->height < 4 || p->depth < 4)
        return fail(nullptr, BLZ_ERR_ARG, "grid dims must be >= 4 (got %d x %d x %d)", p->width, p->height, p->depth);
    if (p->width & 1)
        return fail(nullptr, BLZ_ERR_ARG, "width must be even for the colour-packed solve (got %d)", p->width);
    if ((long long)(p->width + 1) * (p->height + 1) * (p->depth + 1) >= (1LL << 31))
        return fail(nullptr, BLZ_ERR_ARG, "grid too large for 32-bit field offsets");
    if (!(p->dx > 0.0f) || !(p->dt > 0.0f) || !(p->density > 0.0f))
        return fail(nullptr, BLZ_ERR_ARG, "dx, dt and density must be positive");
    if (p->max_iter < 0 || p->max_particles < 0)
        return fail(nullptr, BLZ_ERR_ARG, "negative max_iter or max_particles");
    if (p->bc_mode != BLZ_BC_REF_COMPAT && p->bc_mode != BLZ_BC_FREE_SURFACE)
        return fail(nullptr, BLZ_ERR_ARG, "bad bc_mode %d", p->bc_mode);
    if (p->gs_order != BLZ_GS_RB3D && p->gs_order != BLZ_GS_PLANE)
        return fail(nullptr, BLZ_ERR_ARG, "bad gs_order %d", p->gs_order);
    if (p->advect_scheme < BLZ_ADVECT_RK3 || p->advect_scheme > BLZ_ADVECT_RK2)
        return fail(nullptr, BLZ_ERR_ARG, "bad advect_scheme %d", p->advect_scheme);
    if (p->density_field != 0 && p->density_field != 1)
        return fail(nullptr, BLZ_ERR_ARG, "density_field must be 0 or 1 (got %d)", p->density_field);
    if (p->defect_correction != 0 && p->defect_correction != 1)
        return fail(nullptr, BLZ_ERR_ARG, "defect_correction must be 0 or 1 (got %d)", p->defect_correction);

    blz_solver *s = new blz_solver();
    s->P = *p;
    Geom &g = s->g;
    g.W = p->width; g.H = p->height; g.D = p->depth;
    g.dx = p->dx; g.dt = p->dt; g.inv_dx = 1.0f / p->dx;
    for (int c = 0; c < 3; ++c) {
        g.dmin[c] = p->domain_min[c];
        g.dsize[c] = p->domain_max[c] - p->domain_min[c];
    }
    auto bail = [&](int code) { release(s); delete s; return code; };
    cudaError_t e = cudaGetDevice(&s->device);
    if (e != cudaSuccess) { int r = fail(s, BLZ_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e)); return bail(r); }
    auto alloc = [&](float **ptr, size_t n) -> bool {
        if (cudaMalloc(ptr, n * sizeof(float)) != cudaSuccess) return false;
        return cudaMemset(*ptr, 0, n * sizeof(float)) == cudaSuccess;
    };
    const size_t nT = n_of(*p, 0), nU = n_of(*p, 1), nV = n_of(*p, 2), nW = n_of(*p, 3);
    bool ok = true;
    for (int b = 0; b < 2 && ok; ++b)
        ok = alloc(&s->T[b], nT) && alloc(&s->U[b], nU) && alloc(&s->V[b], nV) && alloc(&s->W[b], nW);
    ok = ok && alloc(&s->p_r, nT / 2) && alloc(&s->p_b, nT / 2) && alloc(&s->rhs_r, nT / 2) && alloc(&s->rhs_b, nT / 2);
    if (p->defect_correction) {
        ok = ok && alloc(&s->df_r, nT / 2) && alloc(&s->df_b, nT / 2) && alloc(&s->dl_r, nT / 2) && alloc(&s->dl_b, nT / 2);
        s->sr_r = s->df_r; s->sr_b = s->df_b; s->sx_r = s->dl_r; s->sx_b = s->dl_b;
    } else {
        s->sr_r = s->rhs_r; s->sr_b = s->rhs_b; s->sx_r = s->p_r; s->sx_b = s->p_b;
    }
    ok = ok && alloc(&s->scratch, 6 * nT);
    if (p->density_field) ok = ok && alloc(&s->Dn[0], nT) && alloc(&s->Dn[1], nT);
    (void)nU; (void)nV; (void)nW;
    s->cap_parts = std::max(p->max_particles, 1);
    s->nbx = (g.W + kSplatBin) / kSplatBin;          // covers face index W
    s->nby = (g.H + kSplatBin) / kSplatBin;
    s->nbz = (g.D + kSplatBin) / kSplatBin;
    const size_t nbins = (size_t)s->nbx * s->nby * s->nbz;
    ok = ok && alloc(&s->parts, 8 * (size_t)s->cap_parts);
    if (p->density_field) ok = ok && alloc(&s->pdens, (size_t)s->cap_parts);
    ok = ok && cudaMalloc(&s->boxes, sizeof(int) * kSplatBoxInts * (size_t)s->cap_parts) == cudaSuccess;
    ok = ok && cudaMalloc(&s->bin_start, sizeof(int) * (nbins + 1)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->active, sizeof(int) * nbins) == cudaSuccess;
    s->n_partials = residual_blocks(g);
    ok = ok && cudaMalloc(&s->partials, 2 * sizeof(double) * s->n_partials) == cudaSuccess;
    ok = ok && cudaMalloc(&s->d_norm2, 2 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMallocHost(&s->h_norm2, 2 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->ctl, sizeof(SolveCtl)) == cudaSuccess;
    ok = ok && cudaMallocHost(&s->h_ctl, sizeof(SolveCtl)) == cudaSuccess;
    if (!ok) { cudaGetLastError(); int r = fail(s, BLZ_ERR_ALLOC, "device allocation failed for %dx%dx%d", g.W, g.H, g.D); return bail(r); }
    for (auto &ev : s->ev)
        if (cudaEventCreate(&ev) != cudaSuccess) { int r = fail(s, BLZ_ERR_CUDA, "cudaEventCreate failed"); return bail(r); }
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
        int r = fail(s, BLZ_ERR_CUDA, "cudaStreamCreate failed");
        return bail(r);
    }
    s->own_stream = true;
    if (cudaDeviceSynchronize() != cudaSuccess) { int r = fail(s, BLZ_ERR_CUDA, "initial synchronize failed"); return bail(r); }
    *out = s;
    return BLZ_OK;
}

int blz_destroy(blz_solver *s) {
    if (!s) return BLZ_OK;
    if (s->st) cudaStreamSynchronize(s->st);
    release(s);
    delete s;
    return BLZ_OK;
}

int blz_set_stream(blz_solver *s, void *stream) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    CK(s, cudaStreamSynchronize(s->st));
    if (s->own_stream) cudaStreamDestroy(s->st);
    if (stream) { s->st = (cudaStream_t)stream; s->own_stream = false; }
    else {
        CK(s, cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    return BLZ_OK;
}

// The cells of one field a particle's splat visits: the reference's box
// (Grid.h:319-324) in the same float operations, so host and device agree.
static inline int trunc_box(float v) { return (int)std::fmin(std::fmax(v, -1.0e9f), 1.0e9f); }

// Boxes 0-3: T, U, V, W; box 4: the density scalar (T grid, empty unless
// the solver carries it), tested with the particle's density `dens`.
static void particle_boxes(const blz_params &P, const float *r, float dens, int out[kSplatBoxInts]) {
    const float ox[5] = {0.5f, 0.0f, 0.5f, 0.5f, 0.5f}, oy[5] = {0.5f, 0.5f, 0.0f, 0.5f, 0.5f};
    const float oz[5] = {0.5f, 0.5f, 0.5f, 0.0f, 0.5f};
    const float dsy = P.domain_max[1] - P.domain_min[1];
    const float radius = r[6] / 2.0f, dx = P.dx;
    for (int f = 0; f < 5; ++f) {
        int *b = out + 6 * f;
        if (f == 4 && !P.density_field) { for (int a = 0; a < 6; ++a) b[a] = 0; continue; }
        const float value = f == 0 ? r[7] : f == 4 ? dens : r[2 + f];
        if (!(std::fabs(value) > 1e-5f)) { for (int a = 0; a < 6; ++a) b[a] = 0; continue; }
        const int w = P.width + (f == 1), h = P.height + (f == 2), d = P.depth + (f == 3);
        b[0] = std::max(trunc_box(((r[0] - radius) - P.domain_min[0]) / dx - ox[f]), 0);
        b[1] = std::min(trunc_box(((r[0] + radius) - P.domain_min[0]) / dx - ox[f]) + 1, w);
        b[2] = std::max(trunc_box((dsy - ((r[1] + radius) - P.domain_min[1])) / dx - oy[f]), 0);
        b[3] = std::min(trunc_box((dsy - ((r[1] - radius) - P.domain_min[1])) / dx - oy[f]) + 1, h);
        b[4] = std::max(trunc_box(((r[2] - radius) - P.domain_min[2]) / dx - oz[f]), 0);
        b[5] = std::min(trunc_box(((r[2] + radius) - P.domain_min[2]) / dx - oz[f]) + 1, d);
        if (b[1] <= b[0] || b[3] <= b[2] || b[5] <= b[4]) for (int a = 0; a < 6; ++a) b[a] = 0;
    }
}

static int set_particles(blz_solver *s, const float *rec8, const float *dens, int n) {
    if (n < 0 || (n > 0 && !rec8)) return fail(s, BLZ_ERR_ARG, "bad particle array (n=%d)", n);
    if (n > s->cap_parts) return fail(s, BLZ_ERR_ARG, "%d particles exceed max_particles=%d", n, s->cap_parts);
    const float half_dx = s->P.dx / 2.0f;
    // Keep the particles whose pscale passes the reference's cut
    // (FluidSolver.cu:83), in order, with their per-field boxes.
    std::vector<float> keep, keep_dens;
    std::vector<int> boxes;
    keep.reserve(8 * (size_t)n);
    boxes.reserve(kSplatBoxInts * (size_t)n);
    for (int p = 0; p < n; ++p) {
        const float *r = rec8 + 8 * (size_t)p;
        for (int c = 0; c < 8; ++c)
            if (!std::isfinite(r[c])) return fail(s, BLZ_ERR_NAN, "particle %d has a non-finite value", p);
        const float d = dens ? dens[p] : 1.0f;
        if (!std::isfinite(d)) return fail(s, BLZ_ERR_NAN, "particle %d has a non-finite density", p);
        if (!(r[6] > half_dx)) continue;
        int b[kSplatBoxInts];
        particle_boxes(s->P, r, d, b);
        keep.insert(keep.end(), r, r + 8);
        if (s->P.density_field) keep_dens.push_back(d);
        boxes.insert(boxes.end(), b, b + kSplatBoxInts);
    }
    const int m = (int)(keep.size() / 8);
    // Bin every kept particle into each 8^3 block its boxes overlap (CSR,
    // particle order inside each bin).
    const int nbx = s->nbx, nby = s->nby, nbz = s->nbz;
    const size_t nbins = (size_t)nbx * nby * nbz;
    std::vector<int> count(nbins + 1, 0);
    auto bin_range = [&](const int *b, int lo[3], int hi[3]) {
        lo[0] = lo[1] = lo[2] = 1 << 30; hi[0] = hi[1] = hi[2] = -1;
        bool any = false;
        for (int f = 0; f < 5; ++f) {
            const int *bb = b + 6 * f;
            if (bb[1] <= bb[0]) continue;
            any = true;
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], bb[2 * a] / kSplatBin);
                hi[a] = std::max(hi[a], (bb[2 * a + 1] - 1) / kSplatBin);
            }
        }
        return any;
    };
    for (int p = 0; p < m; ++p) {
        int lo[3], hi[3];
        if (!bin_range(&boxes[kSplatBoxInts * (size_t)p], lo, hi)) continue;
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) count[(size_t)x + nbx * ((size_t)y + (size_t)nby * z) + 1]++;
    }
    for (size_t b = 0; b < nbins; ++b) count[b + 1] += count[b];
    const int total = count[nbins];
    std::vector<int> list(std::max(total, 1)), fillpos(count.begin(), count.end() - 1), active;
    for (int p = 0; p < m; ++p) {
        int lo[3], hi[3];
        if (!bin_range(&boxes[kSplatBoxInts * (size_t)p], lo, hi)) continue;
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) list[fillpos[(size_t)x + nbx * ((size_t)y + (size_t)nby * z)]++] = p;
    }
    for (size_t b = 0; b < nbins; ++b)
        if (count[b + 1] > count[b]) active.push_back((int)b);
    if (total > s->cap_list) {
        cudaFree(s->bin_list);
        s->bin_list = nullptr;
        s->cap_list = 0;
        if (cudaMalloc(&s->bin_list, sizeof(int) * (size_t)total) != cudaSuccess) {
            cudaGetLastError();
            return fail(s, BLZ_ERR_ALLOC, "bin list allocation failed (%d entries)", total);
        }
        s->cap_list = total;
    }
    if (m > 0) {
        CK(s, cudaMemcpyAsync(s->parts, keep.data(), sizeof(float) * keep.size(), cudaMemcpyHostToDevice, s->st));
        CK(s, cudaMemcpyAsync(s->boxes, boxes.data(), sizeof(int) * boxes.size(), cudaMemcpyHostToDevice, s->st));
        if (s->P.density_field)
            CK(s, cudaMemcpyAsync(s->pdens, keep_dens.data(), sizeof(float) * keep_dens.size(),
                                  cudaMemcpyHostToDevice, s->st));
    }
    CK(s, cudaMemcpyAsync(s->bin_start, count.data(), sizeof(int) * (nbins + 1), cudaMemcpyHostToDevice, s->st));
    if (total > 0) CK(s, cudaMemcpyAsync(s->bin_list, list.data(), sizeof(int) * (size_t)total, cudaMemcpyHostToDevice, s->st));
    if (!active.empty())
        CK(s, cudaMemcpyAsync(s->active, active.data(), sizeof(int) * active.size(), cudaMemcpyHostToDevice, s->st));
    CK(s, cudaStreamSynchronize(s->st));
    s->n_parts = m;
    s->n_active = (int)active.size();
    return BLZ_OK;
}

int blz_set_particles(blz_solver *s, const float *rec8, int n) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    return set_particles(s, rec8, nullptr, n);
}

int blz_set_particles_ex(blz_solver *s, const float *rec8, const float *density, int n) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    if (!s->P.density_field) return fail(s, BLZ_ERR_STATE, "particle densities need density_field = 1");
    return set_particles(s, rec8, density, n);
}

int blz_add_source(blz_solver *s) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    if (s->n_active <= 0) return BLZ_OK;
    const int c = s->cur;
    launch_splat_gather(s->g, s->parts, s->boxes, s->bin_start, s->bin_list, s->active, s->n_active, s->nbx,
                        s->nby, s->T[c], s->U[c], s->V[c], s->W[c], s->st, s->pdens, s->Dn[c]);
    CKL(s);
    s->launches += 1;
    return BLZ_OK;
}

static ForceParams force_params(const blz_solver *s, float time) {
    const blz_params &P = s->P;
    ForceParams fp{};
    fp.vort_on = std::fabs(P.vorticity_conf) > 0.0f;
    fp.dens_on = P.density_field != 0;
    fp.alpha = P.buoyancy_alpha;
    fp.buoy_on = std::fabs(P.buoyancy) > 0.0f || (fp.dens_on && std::fabs(P.buoyancy_alpha) > 0.0f);
    fp.wind_on = P.wind_amp > 0.0f;
    fp.conf = P.vorticity_conf;
    fp.tiny = 1e-20f * (1.0f / (P.dx * P.dt));
    fp.beta = P.buoyancy;
    fp.grav = P.gravity;
    fp.wind_along_x = P.wind_dir <= 1;
    fp.wind_dir_sign = (P.wind_dir == 0 || P.wind_dir == 2) ? 1.0f : -1.0f;
    fp.wind_amp = P.wind_amp;
    fp.wind_turb_amp = P.wind_turb_amp;
    fp.wind_freq = 1.0f / P.wind_turb_scale;
    const float avg_dom = ((P.domain_max[0] - P.domain_min[0]) + (P.domain_max[1] - P.domain_min[1]) +
                           (P.domain_max[2] - P.domain_min[2])) / 3.0f;
    fp.wind_offset = std::fmod(time * avg_dom * P.wind_speed, 25000.0f);       // FluidSolver.cu:353-354
    fp.turb_amp = P.turbulence_amp;
    fp.turb_freq = 1.0f / P.turbulence_scale;
    const float avg_grid = (float)(P.width + P.height + P.depth) / 3.0f;
    fp.turb_offset = std::fmod(time * avg_grid, 25000.0f);                      // FluidSolver.cu:305-306
    fp.tr0 = P.turb_mask_temp_ramp[0]; fp.tr1 = P.turb_mask_temp_ramp[1];
    fp.vr0 = P.turb_mask_vel_ramp[0]; fp.vr1 = P.turb_mask_vel_ramp[1];
    return fp;
}

int blz_forces(blz_solver *s, float time) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    const blz_params &P = s->P;
    const Geom &g = s->g;
    const int c = s->cur, b = c ^ 1;
    float *T = s->T[c], *U = s->U[c], *V = s->V[c], *W = s->W[c];
    const size_t nT = n_of(P, 0);
    if (std::fabs(P.cooling_rate) > 0.0f) {                                     // FluidSolver.cu:868-872
        launch_scale(T, nT, 1.0f - P.dt * P.cooling_rate, s->st); CKL(s); s->launches++;
    }
    if (P.drag > 0.0f) {                                                        // FluidSolver.cu:878-882
        const float k = 1.0f - P.dt * P.drag;
        launch_scale(U, n_of(P, 1), k, s->st); CKL(s);
        launch_scale(V, n_of(P, 2), k, s->st); CKL(s);
        launch_scale(W, n_of(P, 3), k, s->st); CKL(s);
        s->launches += 3;
    }
    const ForceParams fp = force_params(s, time);
    float *om = s->scratch, *vf = s->scratch + 3 * nT;
    if (fp.vort_on) {
        launch_vort_omega(g, U, V, W, om, om + nT, om + 2 * nT, s->st); CKL(s);
        launch_vort_force(g, U, V, W, om, om + nT, om + 2 * nT, fp, vf, vf + nT, vf + 2 * nT, s->st); CKL(s);
        s->launches += 2;
    }
    if (fp.vort_on || fp.buoy_on || fp.wind_on) {
        launch_face_forces(g, U, V, W, T, vf, vf + nT, vf + 2 * nT, fp, s->st, s->Dn[c]); CKL(s);
        s->launches++;
    }
    if (P.turbulence_amp > 0.0f) {                                              // FluidSolver.cu:925-934
        launch_turb_noise(g, T, U, V, W, s->U[b], s->V[b], s->W[b], fp, s->st); CKL(s);
        launch_turb_apply(g, U, V, W, s->U[b], s->V[b], s->W[b], fp, s->st); CKL(s);
        s->launches += 2;
    }
    return BLZ_OK;
}

int blz_divergence(blz_solver *s) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    const int c = s->cur;
    launch_divergence(s->g, s->U[c], s->V[c], s->W[c], open_faces(s->P), s->rhs_r, s->rhs_b, s->st);
    CKL(s);
    s->launches++;
    return BLZ_OK;
}

// FP64 residual norms of (rr/rb, pr/pb), synchronised to the host.
static int residual_on(blz_solver *s, const float *rr, const float *rb, const float *pr, const float *pb, double *r,
                       double *b) {
    const SolveParams sp = solve_params(s->P);
    s->launches += launch_residual(s->g, sp, rr, rb, pr, pb, s->partials, s->n_partials, s->d_norm2, s->st);
    CKL(s);
    CK(s, cudaMemcpyAsync(s->h_norm2, s->d_norm2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(s, cudaStreamSynchronize(s->st));
    *r = std::sqrt(s->h_norm2[0]);
    *b = std::sqrt(s->h_norm2[1]);
    return BLZ_OK;
}

// ||b - A p|| and ||b|| of the current rhs and p.
static int residual_sync(blz_solver *s, double *r, double *b) {
    return residual_on(s, s->rhs_r, s->rhs_b, s->p_r, s->p_b, r, b);
}

static DefectArrays defect_arrays(blz_solver *s) {
    return DefectArrays{s->rhs_r, s->rhs_b, s->p_r, s->p_b, s->dl_r, s->dl_b, s->df_r, s->df_b};
}

// The defect of p (+ delta) into df with the norms of b - A (p + delta)
// in d_norm2 (defect-correction solves).
static int launch_defect_of(blz_solver *s) {
    const DefectArrays a = defect_arrays(s);
    s->launches += launch_defect(s->g, solve_params(s->P), a.rhs_r, a.rhs_b, a.p_r, a.p_b, a.d_r, a.d_b, a.df_r,
                                 a.df_b, s->partials, s->n_partials, s->d_norm2, s->st);
    CKL(s);
    return BLZ_OK;
}

// The residual the solve's stopping rule reads, synchronised to the host.  A
// defect-correction solve (after sweeps) first folds delta into p, then forms
// a fresh FP64 defect, whose norms are those of the pressure p + delta.
static int solve_residual(blz_solver *s, double *r, double *b, bool after_sweeps) {
    if (!s->P.defect_correction) return residual_on(s, s->sr_r, s->sr_b, s->sx_r, s->sx_b, r, b);
    if (after_sweeps) {
        launch_fold(s->g, s->p_r, s->p_b, s->dl_r, s->dl_b, s->st);
        CKL(s);
        s->launches++;
    }
    int rc = launch_defect_of(s);
    if (rc != BLZ_OK) return rc;
    CK(s, cudaMemcpyAsync(s->h_norm2, s->d_norm2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(s, cudaStreamSynchronize(s->st));
    *r = std::sqrt(s->h_norm2[0]);
    *b = std::sqrt(s->h_norm2[1]);
    return BLZ_OK;
}

// Sweep launch-shape autotuner: each variant (segment-kernel shapes and the
// temporal-blocking passes) runs sweeps on scratch copies of p (the solver's
// state is untouched; rhs is only read), timed with CUDA events around a
// graph launch; the fastest is kept per (device, grid dims) for the life of
// the process.  BLZ_SWEEP_VARIANT or params.sweep_variant forces a choice.
// Scratch pressure of the temporal-blocking sweeps (slot 4 of the six
// T-sized scratch arrays; the autotuner's copy of p uses slots 0-1).
static float *q_r(blz_solver *s) { return s->scratch + 4 * n_of(s->P, 0); }
static float *q_b(blz_solver *s) { return s->scratch + 4 * n_of(s->P, 0) + n_of(s->P, 0) / 2; }

static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int>, int> g_tune_cache;

// The tuner's choices persist across processes in a small text file, one
// line "<device name>|<W>|<H>|<D>|<variants offered>|<variant count> <choice>"
// per grid: BLZ_TUNE_CACHE names the file ("off" or empty: none), default
// $XDG_CACHE_HOME/blaze_b200/sweep_variants.txt or ~/.cache/... .
static std::string tune_cache_path() {
    if (const char *p = std::getenv("BLZ_TUNE_CACHE")) {
        if (!*p || std::strcmp(p, "off") == 0) return std::string();
        return p;
    }
    std::string base;
    if (const char *x = std::getenv("XDG_CACHE_HOME")) base = x;
    else if (const char *h = std::getenv("HOME")) base = std::string(h) + "/.cache";
    else return std::string();
    return base + "/blaze_b200/sweep_variants.txt";
}

static std::string tune_key(int device, const Geom &g, int offered) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return std::string();
    char buf[400];
    std::snprintf(buf, sizeof buf, "%s|%d|%d|%d|%d|%d", prop.name, g.W, g.H, g.D, offered, kSweepVariants);
    for (char *c = buf; *c; ++c)
        if (*c == ' ') *c = '_';
    return buf;
}

static int tune_file_lookup(const std::string &key) {
    const std::string path = tune_cache_path();
    if (path.empty() || key.empty()) return -1;
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return -1;
    char line[512];
    int found = -1;
    while (std::fgets(line, sizeof line, f)) {
        char k[450];
        int v = -1;
        if (std::sscanf(line, "%449s %d", k, &v) == 2 && key == k) found = v;   // the last entry wins
    }
    std::fclose(f);
    return found;
}

static void tune_file_store(const std::string &key, int v) {
    const std::string path = tune_cache_path();
    if (path.empty() || key.empty()) return;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && slash > 0) {
        // create the directory chain (best effort)
        for (size_t i = 1; i <= slash; ++i)
            if (path[i] == '/' || i == slash) mkdir(path.substr(0, i == slash ? slash : i).c_str(), 0755);
    }
    if (FILE *f = std::fopen(path.c_str(), "a")) {
        std::fprintf(f, "%s %d\n", key.c_str(), v);
        std::fclose(f);
    }
}

static int choose_variant(blz_solver *s) {
    if (s->variant != -2) return BLZ_OK;
    const int nv = s->P.temporal_block == 1 ? std::min(sweep_variant_count(s->g), kSegVariants)
                                            : sweep_variant_count(s->g);
    if (nv == 0) { s->variant = -1; return BLZ_OK; }
    if (s->P.sweep_variant >= 0) { s->variant = std::min(s->P.sweep_variant, nv - 1); return BLZ_OK; }
    if (const char *env = std::getenv("BLZ_SWEEP_VARIANT")) {
        s->variant = std::max(0, std::min(std::atoi(env), nv - 1));
        return BLZ_OK;
    }
    const auto key = std::make_tuple(s->device, s->g.W, s->g.H, s->g.D * 2 + (nv > kSegVariants ? 1 : 0));
    const std::string fkey = tune_key(s->device, s->g, nv);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) { s->variant = it->second; return BLZ_OK; }
        const int v = tune_file_lookup(fkey);
        if (v >= 0 && v < nv) {
            g_tune_cache[key] = v;
            s->variant = v;
            return BLZ_OK;
        }
    }
    const size_t half = n_of(s->P, 0) / 2;
    float *tr = s->scratch, *tb = s->scratch + half;
    CK(s, cudaMemcpyAsync(tr, s->p_r, half * sizeof(float), cudaMemcpyDeviceToDevice, s->st));
    CK(s, cudaMemcpyAsync(tb, s->p_b, half * sizeof(float), cudaMemcpyDeviceToDevice, s->st));
    const SolveParams sp = solve_params(s->P);
    long long dummy = 0;
    // Direct launches first: they set the kernels' attributes outside any
    // capture and warm the SM clock.
    for (int v = 0; v < nv; ++v)
        launch_rbgs_sweeps(s->g, sp, s->rhs_r, s->rhs_b, tr, tb, 4, s->st, &dummy, v, q_r(s), q_b(s));
    CKL(s);
    CK(s, cudaStreamSynchronize(s->st));
    // Each variant is timed as the solve runs it: kTuneSweeps sweeps (one
    // residual-check interval at the default) captured in a CUDA graph, so
    // the launch count of a variant does not count against it.  An untimed
    // round, then two timed rounds in opposite orders (the SM clock ramps up
    // under load); each variant keeps its faster time.
    constexpr int kTuneSweeps = 20;
    cudaStream_t ts = nullptr;
    CK(s, cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking));
    std::vector<cudaGraphExec_t> ex(nv, nullptr);
    std::vector<long long> per_graph(nv, 0);
    std::vector<float> t_min(nv, 1e30f);
    cudaError_t err = cudaSuccess;
    for (int v = 0; v < nv && err == cudaSuccess; ++v) {
        cudaGraph_t gph = nullptr;
        err = cudaStreamBeginCapture(ts, cudaStreamCaptureModeThreadLocal);
        if (err != cudaSuccess) break;
        launch_rbgs_sweeps(s->g, sp, s->rhs_r, s->rhs_b, tr, tb, kTuneSweeps, ts, &per_graph[v], v, q_r(s),
                           q_b(s));
        err = cudaStreamEndCapture(ts, &gph);
        if (err == cudaSuccess) err = cudaGraphInstantiate(&ex[v], gph, 0);
        if (gph) cudaGraphDestroy(gph);
    }
    for (int v = 0; v < nv && err == cudaSuccess; ++v) {
        err = cudaGraphLaunch(ex[v], ts);
        if (err == cudaSuccess) dummy += per_graph[v];
    }
    for (int round = 0; round < 2 && err == cudaSuccess; ++round)
        for (int i = 0; i < nv && err == cudaSuccess; ++i) {
            const int v = round == 0 ? i : nv - 1 - i;
            float ms = 0.0f;
            err = cudaEventRecord(s->ev[6], ts);
            if (err == cudaSuccess) err = cudaGraphLaunch(ex[v], ts);
            if (err == cudaSuccess) dummy += per_graph[v];
            if (err == cudaSuccess) err = cudaEventRecord(s->ev[7], ts);
            if (err == cudaSuccess) err = cudaEventSynchronize(s->ev[7]);
            if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, s->ev[6], s->ev[7]);
            if (err == cudaSuccess) t_min[v] = std::min(t_min[v], ms);
        }
    cudaStreamSynchronize(ts);
    for (auto e : ex)
        if (e) cudaGraphExecDestroy(e);
    cudaStreamDestroy(ts);
    if (err != cudaSuccess) return fail(s, BLZ_ERR_CUDA, "sweep autotuner: %s", cudaGetErrorString(err));
    const int best = (int)(std::min_element(t_min.begin(), t_min.end()) - t_min.begin());
    if (std::getenv("BLZ_TUNE_VERBOSE")) {
        std::fprintf(stderr, "sweep autotuner %dx%dx%d, us per sweep:", s->g.W, s->g.H, s->g.D);
        for (int v = 0; v < nv; ++v) std::fprintf(stderr, " v%d=%.2f", v, 1e3f * t_min[v] / kTuneSweeps);
        std::fprintf(stderr, " -> v%d\n", best);
    }
    s->launches += dummy;
    s->variant = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
    tune_file_store(fkey, best);
    return BLZ_OK;
}

static int sweeps_on(blz_solver *s, int n, const float *rr, const float *rb, float *pr, float *pb) {
    const SolveParams sp = solve_params(s->P);
    if (s->P.gs_order == BLZ_GS_PLANE) {
        launch_plane_sweeps(s->g, sp, rr, rb, pr, pb, n, s->st, &s->launches);
    } else {
        int rc = choose_variant(s);
        if (rc != BLZ_OK) return rc;
        launch_rbgs_sweeps(s->g, sp, rr, rb, pr, pb, n, s->st, &s->launches, s->variant, q_r(s), q_b(s));
    }
    CKL(s);
    return BLZ_OK;
}

// Sweeps of the system the solve works on (sr, sx).
static int sweeps(blz_solver *s, int n) { return sweeps_on(s, n, s->sr_r, s->sr_b, s->sx_r, s->sx_b); }

// The residual-controlled solve as one graph launch (graph_solve.cu).
// Residual checks are a stopping test: every `chunk` sweeps the FP64
// residual decides whether the solve goes on.  With check_every < 0 the
// interval is chosen per solve from 20, 40, ..., 320 (those dividing
// max_iter) to minimise the expected cost of the checks plus the sweeps
// past convergence, (N / c) * r + c / 2 in sweeps, with N the previous
// solve's sweep count and r the measured cost of one check in sweeps (1.5
// before any measurement).  The stopping rule itself is unchanged.
static int check_chunk(const blz_solver *s) {
    const blz_params &P = s->P;
    if (P.check_every >= 1) return P.check_every;
    if (P.check_every == 0) return 1;
    constexpr int kBase = 20;
    if (s->last_iters <= 0) return kBase;
    const double r = s->check_ratio > 0.0 ? s->check_ratio : 1.5;
    int best = kBase;
    double best_cost = 1e300;
    for (int c = kBase; c <= 16 * kBase; c *= 2) {
        if (P.max_iter % c != 0) continue;
        const double cost = s->last_iters / (double)c * r + 0.5 * c;
        if (cost < best_cost) { best_cost = cost; best = c; }
    }
    return best;
}

static int solve_device_loop(blz_solver *s, blz_step_stats *st, int chunk) {
    const blz_params &P = s->P;
    int rc = choose_variant(s);
    if (rc != BLZ_OK) return rc;
    blz_solver::SolveGraph *gr = nullptr;
    for (auto &x : s->graphs)
        if (x.exec && x.chunk == chunk) gr = &x;
    const DefectArrays dfa = defect_arrays(s);
    if (!gr) {
        for (auto &x : s->graphs)
            if (!x.exec) { gr = &x; break; }
        if (!gr) return fail(s, BLZ_ERR_STATE, "too many check intervals");
        cudaError_t e = build_solve_graph(s->g, solve_params(P), s->sr_r, s->sr_b, s->sx_r, s->sx_b, s->partials,
                                          s->n_partials, s->d_norm2, s->ctl, chunk, P.max_iter, P.tol, s->variant,
                                          s->st, &gr->exec, &gr->body, &gr->prologue, q_r(s), q_b(s),
                                          P.defect_correction ? &dfa : nullptr);
        if (e != cudaSuccess) return fail(s, BLZ_ERR_CUDA, "building the solve graph failed: %s", cudaGetErrorString(e));
        gr->chunk = chunk;
    }
    CK(s, cudaGraphLaunch(gr->exec, s->st));
    CK(s, cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s->st));
    CK(s, cudaStreamSynchronize(s->st));
    const SolveCtl &c = *s->h_ctl;
    s->launches += gr->prologue + (long long)(c.checks - 1) * gr->body;
    s->last_iters = c.iters;
    if (c.iters > 0 && c.checks > 0 && c.sweep_ns > 0)
        s->check_ratio = ((double)c.check_ns / c.checks) / ((double)c.sweep_ns / c.iters);
    if (st) {
        const double r = std::sqrt(c.r2), b = std::sqrt(c.b2);
        st->iterations = c.iters;
        st->residual = r;
        st->rhs_norm = b;
        st->rel_residual = b > 0.0 ? r / b : 0.0;
        st->converged = c.converged;
        st->ms_sweeps = (float)(c.sweep_ns * 1e-6);
        st->ms_checks = (float)(c.check_ns * 1e-6);
        st->residual_checks = c.checks;
        st->sweep_variant = s->variant;
        st->device_loop = 1;
        st->check_interval = chunk;
        if (!std::isfinite(r)) return fail(s, BLZ_ERR_NAN, "non-finite residual after %d sweeps", c.iters);
    }
    return BLZ_OK;
}

static int solve_body(blz_solver *s, blz_step_stats *st);

// The TMA-staged pass counts bounded waits that gave up; after work that may
// have used it, a nonzero count is reported (that pass's result is wrong).
static int check_tb_timeouts(blz_solver *s) {
    if (!sweep_variant_uses_tma(s->variant)) return BLZ_OK;
    CK(s, cudaStreamSynchronize(s->st));
    if (tb_take_timeouts()) return fail(s, BLZ_ERR_TIMEOUT, "temporal-blocking pass: a bounded TMA wait gave up");
    return BLZ_OK;
}

// The learned warm start of the attached network, ordered on s->st with no
// host synchronisation (so a batch can capture it in a graph): the network's
// correction d, `pre` smoothing sweeps of p and of d (sweep variant
// `variant`, or the solver's autotuned one when < 0), then p += alpha d.
static int warm_start(blz_solver *s, int variant, int *pre) {
    const blz_params &P = s->P;
    float *d_r = nullptr, *d_b = nullptr;
    const float *z_r = nullptr, *z_b = nullptr;
    int rc = unet_correction(s->warm, P, s->rhs_r, s->rhs_b, s->p_r, s->p_b, s->st, &s->launches, &d_r, &d_b,
                             &z_r, &z_b);
    if (rc != BLZ_OK) return fail(s, rc, "warm start: %s", g_thread_err.c_str());
    *pre = unet_smoothing(s->warm);
    if (*pre > 0 && P.gs_order == BLZ_GS_RB3D) {
        if (variant < 0) {
            if ((rc = sweeps(s, *pre)) != BLZ_OK) return rc;
            variant = s->variant;
        } else {
            launch_rbgs_sweeps(s->g, solve_params(P), s->sr_r, s->sr_b, s->sx_r, s->sx_b, *pre, s->st,
                               &s->launches, variant, q_r(s), q_b(s));
        }
        launch_rbgs_sweeps(s->g, solve_params(P), z_r, z_b, d_r, d_b, *pre, s->st, &s->launches, variant, q_r(s),
                           q_b(s));
        CKL(s);
    } else {
        *pre = 0;
    }
    rc = unet_combine(s->warm, P, s->sr_r, s->sr_b, s->sx_r, s->sx_b, s->st, &s->launches);
    if (rc != BLZ_OK) return fail(s, rc, "warm start: %s", g_thread_err.c_str());
    return BLZ_OK;
}

int blz_solve(blz_solver *s, blz_step_stats *st) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    const blz_params &P = s->P;
    const size_t half = n_of(P, 0) / 2;
    if (P.reset_pressure) {
        CK(s, cudaMemsetAsync(s->p_r, 0, half * sizeof(float), s->st));
        CK(s, cudaMemsetAsync(s->p_b, 0, half * sizeof(float), s->st));
    }
    if (P.defect_correction) {
        // The correction starts at the previous solve's rounding remainder
        // (zero when p was set or swept since); the defect b - A p is formed
        // in FP64 and kept as the sweeps' right-hand side.
        if (!s->defect_valid || P.reset_pressure) {
            CK(s, cudaMemsetAsync(s->dl_r, 0, half * sizeof(float), s->st));
            CK(s, cudaMemsetAsync(s->dl_b, 0, half * sizeof(float), s->st));
        }
        const int rc0 = launch_defect_of(s);
        if (rc0 != BLZ_OK) return rc0;
        s->defect_valid = false;
    }
    int pre = 0;                                 // sweeps of p before the solve proper
    if (s->warm) {
        CK(s, cudaEventRecord(s->ev[8], s->st));
        const int rc = warm_start(s, -1, &pre);
        if (rc != BLZ_OK) return rc;
        CK(s, cudaEventRecord(s->ev[9], s->st));
    }
    int rc = solve_body(s, st);
    if (rc != BLZ_OK) return rc;
    if ((rc = check_tb_timeouts(s)) != BLZ_OK) return rc;
    if (P.defect_correction) {                 // p = RN(p + delta), delta = the exact remainder
        launch_fold(s->g, s->p_r, s->p_b, s->dl_r, s->dl_b, s->st);
        CKL(s);
        s->launches++;
        s->defect_valid = true;
    }
    if (s->warm) {
        if ((rc = unet_timeout_flag(s->warm, s->st)) != BLZ_OK) return fail(s, rc, "warm start: %s", g_thread_err.c_str());
        if (st) {
            float t = 0.0f;
            CK(s, cudaEventElapsedTime(&t, s->ev[8], s->ev[9]));
            st->ms_warm_start = t;
            st->warm_started = 1;
            st->iterations += pre;
        }
    } else if (st) {
        st->ms_warm_start = 0.0f;
        st->warm_started = 0;
    }
    return BLZ_OK;
}

int blz_set_warm_start(blz_solver *s, blz_unet *u) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    if (u) {
        if (blz_unet_num_params(u) <= 0) return fail(s, BLZ_ERR_ARG, "bad network");
        if (s->P.width % 8 || s->P.height % 8 || s->P.depth % 8)
            return fail(s, BLZ_ERR_ARG, "the warm start needs grid dims that are multiples of 8");
        const int rc = unet_prepare(u, s->P);
        if (rc != BLZ_OK) return fail(s, rc, "warm start: %s", g_thread_err.c_str());
    }
    s->warm = u;
    return BLZ_OK;
}

static int solve_body(blz_solver *s, blz_step_stats *st) {
    const blz_params &P = s->P;
    const int chunk = check_chunk(s);
    if (P.device_loop && P.tol > 0.0 && P.gs_order == BLZ_GS_RB3D && P.max_iter % chunk == 0)
        return solve_device_loop(s, st, chunk);
    int done = 0, rc, checks = 0;
    double r = 0.0, b = 0.0;
    bool have = false;
    float ms_sweeps = 0.0f;
    // Sweep batches are bracketed by events; their elapsed time is read after
    // the residual check's synchronisation, so timing adds no stall.
    auto timed_sweeps = [&](int n) -> int {
        CK(s, cudaEventRecord(s->ev[6], s->st));
        int e = sweeps(s, n);
        if (e != BLZ_OK) return e;
        CK(s, cudaEventRecord(s->ev[7], s->st));
        return BLZ_OK;
    };
    auto add_elapsed = [&]() {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, s->ev[6], s->ev[7]) == cudaSuccess) ms_sweeps += t;
    };
    if (P.tol <= 0.0) {
        if ((rc = timed_sweeps(P.max_iter)) != BLZ_OK) return rc;
        done = P.max_iter;
    } else {
        if ((rc = solve_residual(s, &r, &b, false)) != BLZ_OK) return rc;
        ++checks;
        while (done < P.max_iter && !(b == 0.0 || r / b <= P.tol)) {
            const int n = std::min(chunk, P.max_iter - done);
            if ((rc = timed_sweeps(n)) != BLZ_OK) return rc;
            done += n;
            if ((rc = solve_residual(s, &r, &b, true)) != BLZ_OK) return rc;
            ++checks;
            add_elapsed();
        }
        have = true;
    }
    s->last_iters = done;
    if (st) {
        if (!have) {
            if ((rc = solve_residual(s, &r, &b, done > 0)) != BLZ_OK) return rc;
            ++checks;
            if (done > 0) add_elapsed();
        }
        st->iterations = done;
        st->residual = r;
        st->rhs_norm = b;
        st->rel_residual = b > 0.0 ? r / b : 0.0;
        st->converged = P.tol <= 0.0 || b == 0.0 || r / b <= P.tol;
        st->ms_sweeps = ms_sweeps;
        st->residual_checks = checks;
        st->sweep_variant = s->variant;
        st->device_loop = 0;
        st->check_interval = chunk;
        st->ms_checks = 0.0f;
        if (!std::isfinite(r)) return fail(s, BLZ_ERR_NAN, "non-finite residual after %d sweeps", done);
    }
    return BLZ_OK;
}

int blz_sweeps(blz_solver *s, int n) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    if (n < 0) return fail(s, BLZ_ERR_ARG, "negative sweep count %d", n);
    s->defect_valid = false;                    // p changes on its own: drop the remainder
    const int rc = n > 0 ? sweeps_on(s, n, s->rhs_r, s->rhs_b, s->p_r, s->p_b) : BLZ_OK;
    return rc != BLZ_OK ? rc : check_tb_timeouts(s);
}

int blz_tight_solve(blz_solver *s, double tol, int max_sweeps, double omega, int *sweeps_out, double *rel_out) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    if (!(tol > 0.0) || max_sweeps < 0 || !(omega > 0.0 && omega < 2.0))
        return fail(s, BLZ_ERR_ARG, "tight solve needs tol > 0, max_sweeps >= 0 and omega in (0, 2)");
    int sw = 0;
    double rel = 0.0;
    s->defect_valid = false;
    const int e = tight_solve(s->g, solve_params(s->P), s->rhs_r, s->rhs_b, s->p_r, s->p_b, tol, max_sweeps, omega,
                              50, s->st, &sw, &rel, &s->launches);
    if (e != 0) {
        cudaGetLastError();
        return fail(s, BLZ_ERR_CUDA, "tight solve: %s", cudaGetErrorString((cudaError_t)e));
    }
    if (sweeps_out) *sweeps_out = sw;
    if (rel_out) *rel_out = rel;
    return BLZ_OK;
}

int blz_gradient(blz_solver *s) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    const int c = s->cur;
    const float sc = s->P.dt / (s->P.density * s->P.dx);                       // FluidSolver.cu:612
    const bool dl = s->P.defect_correction && s->defect_valid;   // the pressure is p + delta
    launch_gradient(s->g, solve_params(s->P), sc, s->p_r, s->p_b, s->U[c], s->V[c], s->W[c], s->st,
                    dl ? s->dl_r : nullptr, dl ? s->dl_b : nullptr);
    CKL(s);
    s->launches++;
    return BLZ_OK;
}

int blz_project(blz_solver *s, blz_step_stats *st) {
    int rc;
    if ((rc = blz_divergence(s)) != BLZ_OK) return rc;
    if ((rc = blz_solve(s, st)) != BLZ_OK) return rc;
    return blz_gradient(s);
}

int blz_advect(blz_solver *s) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    const int c = s->cur, b = c ^ 1;
    launch_advect(s->g, s->T[c], s->U[c], s->V[c], s->W[c], s->T[b], s->U[b], s->V[b], s->W[b], s->st,
                  s->P.advect_scheme, s->Dn[c], s->Dn[b]);
    CKL(s);
    s->launches++;
    s->cur = b;                                                                 // swap_grids_kernel
    return BLZ_OK;
}

int blz_step(blz_solver *s, float time, blz_step_stats *st) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    int rc;
    CK(s, cudaEventRecord(s->ev[0], s->st));
    if ((rc = blz_forces(s, time)) != BLZ_OK) return rc;
    CK(s, cudaEventRecord(s->ev[1], s->st));
    if ((rc = blz_divergence(s)) != BLZ_OK) return rc;
    CK(s, cudaEventRecord(s->ev[2], s->st));
    if ((rc = blz_solve(s, st)) != BLZ_OK) return rc;
    CK(s, cudaEventRecord(s->ev[3], s->st));
    if ((rc = blz_gradient(s)) != BLZ_OK) return rc;
    CK(s, cudaEventRecord(s->ev[4], s->st));
    if ((rc = blz_advect(s)) != BLZ_OK) return rc;
    CK(s, cudaEventRecord(s->ev[5], s->st));
    if (st) {
        CK(s, cudaEventSynchronize(s->ev[5]));
        auto ms = [&](int a, int b) { float t = 0.f; cudaEventElapsedTime(&t, s->ev[a], s->ev[b]); return t; };
        st->ms_source = 0.0f;
        st->ms_forces = ms(0, 1);
        st->ms_divergence = ms(1, 2);
        st->ms_solve = ms(2, 3);
        st->ms_gradient = ms(3, 4);
        st->ms_advect = ms(4, 5);
        st->ms_total = ms(0, 5);
    }
    return BLZ_OK;
}

int blz_residual(blz_solver *s, double *res, double *bn) {
    if (!s || !res || !bn) return fail(s, BLZ_ERR_ARG, "null argument");
    return residual_sync(s, res, bn);
}

int blz_perlin(const float *pos3, int n, float scale, int seed, float *out) {
    if (n < 0 || (n > 0 && (!pos3 || !out))) return fail(nullptr, BLZ_ERR_ARG, "bad perlin arguments");
    if (n == 0) return BLZ_OK;
    float *d = nullptr;
    CK(nullptr, cudaMalloc(&d, sizeof(float) * 4 * (size_t)n));
    cudaError_t e = cudaMemcpy(d, pos3, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        launch_perlin(d, n, scale, seed, d + 3 * (size_t)n, nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 3 * (size_t)n, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(nullptr, BLZ_ERR_CUDA, "blz_perlin: %s", cudaGetErrorString(e));
    return BLZ_OK;
}

static float *front_of(blz_solver *s, int f) {
    const int c = s->cur;
    switch (f) {
    case BLZ_FIELD_T: return s->T[c];
    case BLZ_FIELD_U: return s->U[c];
    case BLZ_FIELD_V: return s->V[c];
    case BLZ_FIELD_W: return s->W[c];
    case BLZ_FIELD_DENSITY: return s->Dn[c];
    default: return nullptr;
    }
}

void *blz_field_ptr(blz_solver *s, int field) { return s ? (void *)front_of(s, field) : nullptr; }

int blz_get_field(blz_solver *s, int f, float *dst, int on_device) {
    if (!s || !dst) return fail(s, BLZ_ERR_ARG, "null argument");
    const size_t n = n_of(s->P, f);
    if (!n) return fail(s, BLZ_ERR_ARG, "bad field %d", f);
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const float *src = front_of(s, f);
    if (f == BLZ_FIELD_P || f == BLZ_FIELD_RHS) {
        float *tmp = s->scratch;
        launch_unpack(s->g, f == BLZ_FIELD_P ? s->p_r : s->rhs_r, f == BLZ_FIELD_P ? s->p_b : s->rhs_b, tmp, s->st);
        CKL(s);
        s->launches++;
        src = tmp;
    }
    CK(s, cudaMemcpyAsync(dst, src, n * sizeof(float), kind, s->st));
    CK(s, cudaStreamSynchronize(s->st));
    return BLZ_OK;
}

int blz_set_field(blz_solver *s, int f, const float *src, int on_device) {
    if (!s || !src) return fail(s, BLZ_ERR_ARG, "null argument");
    const size_t n = n_of(s->P, f);
    if (!n) return fail(s, BLZ_ERR_ARG, "bad field %d", f);
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (f == BLZ_FIELD_P) s->defect_valid = false;
    if (f == BLZ_FIELD_P || f == BLZ_FIELD_RHS) {
        float *tmp = s->scratch;
        CK(s, cudaMemcpyAsync(tmp, src, n * sizeof(float), kind, s->st));
        launch_pack(s->g, tmp, f == BLZ_FIELD_P ? s->p_r : s->rhs_r, f == BLZ_FIELD_P ? s->p_b : s->rhs_b, s->st);
        CKL(s);
        s->launches++;
    } else {
        CK(s, cudaMemcpyAsync(front_of(s, f), src, n * sizeof(float), kind, s->st));
    }
    CK(s, cudaStreamSynchronize(s->st));
    return BLZ_OK;
}

// ---- z-slab decomposition of the solve ------------------------------------
// Every rank holds the whole grid and updates only its slab of planes; the
// caller moves halo planes between ranks (blaze_b200/slab.py).

int blz_slab_info(blz_solver *s, int *supported, int *n_partials, long long *plane_floats) {
    if (!s || !supported || !n_partials || !plane_floats) return fail(s, BLZ_ERR_ARG, "null argument");
    int first = 0, count = 0;
    *supported = slab_pass_supported(s->g) && residual_slab_tiles(s->g, 0, s->g.D, &first, &count) == 0 &&
                 s->P.gs_order == BLZ_GS_RB3D && !s->P.defect_correction;
    *n_partials = residual_blocks(s->g);
    *plane_floats = (long long)(s->g.W / 2) * s->g.H;
    return BLZ_OK;
}

// The colour-packed array of (buffer, colour): p or the pass scratch q.
static float *slab_array(blz_solver *s, int buf, int colour) {
    if (buf == 0) return colour ? s->p_b : s->p_r;
    return colour ? q_b(s) : q_r(s);
}

static int slab_planes_arg(blz_solver *s, int buf, int colour, int z0, int z1, const void *dev) {
    if (!dev) return fail(s, BLZ_ERR_ARG, "null device buffer");
    if ((buf != 0 && buf != 1) || (colour != 0 && colour != 1) || z0 < 0 || z1 > s->g.D || z0 > z1)
        return fail(s, BLZ_ERR_ARG, "slab planes: buffer %d colour %d planes [%d, %d) of %d", buf, colour, z0, z1,
                    s->g.D);
    return BLZ_OK;
}

int blz_slab_get_planes(blz_solver *s, int buf, int colour, int z0, int z1, void *dst) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    int rc = slab_planes_arg(s, buf, colour, z0, z1, dst);
    if (rc != BLZ_OK) return rc;
    const size_t pl = (size_t)(s->g.W / 2) * s->g.H;
    if (z1 > z0)
        CK(s, cudaMemcpyAsync(dst, slab_array(s, buf, colour) + pl * z0, pl * (z1 - z0) * sizeof(float),
                              cudaMemcpyDeviceToDevice, s->st));
    return BLZ_OK;
}

int blz_slab_set_planes(blz_solver *s, int buf, int colour, int z0, int z1, const void *src) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    int rc = slab_planes_arg(s, buf, colour, z0, z1, src);
    if (rc != BLZ_OK) return rc;
    const size_t pl = (size_t)(s->g.W / 2) * s->g.H;
    s->defect_valid = false;
    if (z1 > z0)
        CK(s, cudaMemcpyAsync(slab_array(s, buf, colour) + pl * z0, src, pl * (z1 - z0) * sizeof(float),
                              cudaMemcpyDeviceToDevice, s->st));
    return BLZ_OK;
}

int blz_slab_pass(blz_solver *s, int z0, int z1, int from_q) {
    if (!s) return fail(nullptr, BLZ_ERR_ARG, "null solver");
    int ok = 0, np = 0;
    long long pf = 0;
    blz_slab_info(s, &ok, &np, &pf);
    if (!ok) return fail(s, BLZ_ERR_STATE, "slab pass: needs W %% 8 == 0, the temporal-blocking pass, "
                                           "RB3D order and no defect correction");
    if (z0 < 0 || z1 > s->g.D || z0 >= z1 || (from_q != 0 && from_q != 1))
        return fail(s, BLZ_ERR_ARG, "slab pass: planes [%d, %d) of %d, from_q %d", z0, z1, s->g.D, from_q);
    s->defect_valid = false;
    const SolveParams sp = solve_params(s->P);
    if (from_q) launch_tb_pass_slab(s->g, sp, s->rhs_r, s->rhs_b, q_b(s), s->p_r, s->p_b, z0, z1, true, s->st);
    else launch_tb_pass_slab(s->g, sp, s->rhs_r, s->rhs_b, s->p_b, q_r(s), q_b(s), z0, z1, true, s->st);
    CKL(s);
    s->launches++;
    return BLZ_OK;
}

int blz_slab_residual(blz_solver *s, int z0, int z1, double *partials, int *first, int *count) {
    if (!s || !partials || !first || !count) return fail(s, BLZ_ERR_ARG, "null argument");
    if (residual_slab_tiles(s->g, z0, z1, first, count) != 0)
        return fail(s, BLZ_ERR_ARG, "slab residual: planes [%d, %d) of %d must be whole residual tiles of %d planes",
                    z0, z1, s->g.D, BLZ_SLAB_ALIGN);
    launch_residual_slab(s->g, solve_params(s->P), s->rhs_r, s->rhs_b, s->p_r, s->p_b, z0, z1, partials, s->st);
    CKL(s);
    s->launches++;
    return BLZ_OK;
}

int blz_reduce_partials(blz_solver *s, const double *partials, double *res, double *bn) {
    if (!s || !partials || !res || !bn) return fail(s, BLZ_ERR_ARG, "null argument");
    launch_reduce_pairs(partials, residual_blocks(s->g), s->d_norm2, s->st);
    CKL(s);
    s->launches++;
    CK(s, cudaMemcpyAsync(s->h_norm2, s->d_norm2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(s, cudaStreamSynchronize(s->st));
    *res = std::sqrt(s->h_norm2[0]);
    *bn = std::sqrt(s->h_norm2[1]);
    return BLZ_OK;
}

} // extern "C"

namespace blz {
blz_unet *solver_warm(blz_solver *s) { return s->warm; }
int solver_warm_start(blz_solver *s, int variant, int *pre) { return warm_start(s, variant, pre); }
// What the batch (batch.cu) needs of a solver: its solve arrays and
// parameters, and the front/back flip a replayed frame graph implies.
void solver_batch_view(blz_solver *s, BatchSim *out, const blz_params **P) {
    out->g = s->g;
    out->sp = solve_params(s->P);
    out->rhs_r = s->rhs_r;
    out->rhs_b = s->rhs_b;
    out->p_r = s->p_r;
    out->p_b = s->p_b;
    out->q_r = q_r(s);
    out->q_b = q_b(s);
    out->max_iter = s->P.max_iter;
    out->tol = s->P.tol;
    if (P) *P = &s->P;
}
void solver_flip_front(blz_solver *s) { s->cur ^= 1; }
void solver_add_launches(blz_solver *s, long long n) { s->launches += n; }
cudaStream_t solver_stream(blz_solver *s) { return s->st; }
const blz_params *solver_params(blz_solver *s) { return &s->P; }
} // namespace blz
