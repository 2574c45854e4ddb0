// batch.cu — many independent simulations of uneven grid sizes stepped
// together.  No counterpart in the reference, which runs one FluidSolver.
//
// The pressure solve is the frame's dominant cost and, for grids of 48^3..128^3
// cells, a single grid's half sweep is a few microseconds of HBM traffic, less
// than a kernel launch.  The batch therefore runs every grid's solve in the
// same launches: each half sweep is one persistent grid-stride launch over the
// segment work items of the grids still running (k_batch_sweep; the list is
// rebuilt after every check, so a grid that finished costs nothing), the FP64 residual is one
// launch over every grid's residual blocks plus one block per grid deciding
// continue/stop, and a CUDA graph with a conditional WHILE node repeats
// {check_every sweeps, residual, decision} until no grid is left running.
// Each grid stops exactly where its own device-loop solve stops, with the
// same pressure bit for bit.  The launch shape (planes per thread and block
// size) is autotuned per batch on scratch copies of the pressures.
//
// When no grid's forces depend on time (no curl noise, no moving wind
// noise), a whole frame — every grid's forces and divergence, the batched
// solve, every grid's gradient and advection — is one graph launch (one graph
// per front/back parity of the grids' fields).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "kernels.cuh"

using namespace blz;

namespace {

__global__ void k_batch_begin(BatchCtl *ctl, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) ctl[s] = BatchCtl{0, 0, 0, 1, 0.0, 0.0};
}

// Lists the grids still running with their item offsets (for the next
// sweeps) and, inside the solve graph, sets whether the loop goes on.
__global__ void k_batch_active(const BatchCtl *__restrict__ ctl, int n, const long long *__restrict__ item0,
                               BatchActive *act, int *act_sim, long long *act_item0, int set_cond,
                               cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    int na = 0;
    long long acc = 0;
    for (int s = 0; s < n; ++s) {
        if (!ctl[s].active) continue;
        act_sim[na] = s;
        act_item0[na] = acc;
        acc += item0[s + 1] - item0[s];
        ++na;
    }
    act_item0[na] = acc;
    act->n = na;
    act->sim = act_sim;
    act->item0 = act_item0;
    if (set_cond) cudaGraphSetConditional(h, na > 0 ? 1u : 0u);
}

constexpr int kKZ[4] = {1, 2, 4, 8};
constexpr int kBlocks[2] = {128, 256};
constexpr int kTbZC[3] = {8, 16, 32};         // planes per temporal-blocking tile

} // namespace

struct blz_batch {
    std::vector<blz_solver *> sims;
    std::vector<const blz_params *> params;
    int n = 0, chunk = 1;
    cudaStream_t st = nullptr;
    BatchSim *d_sims = nullptr;
    BatchCtl *d_ctl = nullptr, *h_ctl = nullptr;
    long long *d_item0 = nullptr;             // 4 tables (kz = 1, 2, 4, 8) of n + 1 offsets
    BatchActive *d_act = nullptr;             // grids still running, rebuilt after each check
    int *d_act_sim = nullptr;
    long long *d_act_item0 = nullptr;
    int *d_blk0 = nullptr;
    int total_blocks = 0;
    double *partials = nullptr;
    int kz = -1, block = 256, grid = 0;       // chosen launch shape (kz < 0: not tuned yet)
    // temporal blocking (two sweeps per pass over HBM): planes per tile, 0
    // when the segment kernel was chosen (or the batch does not allow it)
    int tb_zc = 0;
    bool tb_pk = false;                       // paired-FP32 stencil in the tiles
    int force_zc = -1;                        // blz_batch_set_sweep: -1 autotune, 0 segment, > 0 tiles of that many planes
    bool force_pk = false;                    // ... with the paired-FP32 stencil
    bool tb_ok = false;                       // every grid's shape allows it and check_every % 4 == 0
    BatchTile *d_tiles = nullptr;             // tiles of the current tb_zc, heaviest first
    int ntiles = 0, tiles_cap = 0;
    size_t tb_smem = 0;                       // largest dynamic shared memory of a tile
    bool time_free = false;                   // frame graphs allowed
    cudaGraphExec_t solve_exec = nullptr;
    cudaGraphExec_t frame_exec[2] = {nullptr, nullptr};
    long long frame_stage_launches[2] = {0, 0};
    int parity = 0;                           // front/back parity of the grids (all equal)
    long long launches = 0;
    int prologue = 0, body = 0;               // kernels per graph part
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.0f;
    // learned warm starts (solvers with an attached network): smoothing
    // sweeps each ran before the batched loop, and the launches one solve
    // graph replays for them
    std::vector<int> pre;
    long long warm_launches = 0;
};

// Sweep variant of the warm starts' smoothing sweeps inside a batch graph
// (a segment-kernel shape: every variant gives the same bits, and the
// solver's own autotuner cannot run inside a capture).
constexpr int kBatchWarmVariant = 2;

static thread_local std::string g_batch_err;

static int bfail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_thread_error(buf);
    return code;
}

#define BCK(x)                                                                                  \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) return bfail(BLZ_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

static const long long *item0_of(const blz_batch *b, int kz) {
    const int t = kz == 1 ? 0 : kz == 2 ? 1 : kz == 4 ? 2 : 3;
    return b->d_item0 + (size_t)t * (b->n + 1);
}

static void active_list(blz_batch *b, int kz, int set_cond, cudaGraphConditionalHandle h) {
    k_batch_active<<<1, 32, 0, b->st>>>(b->d_ctl, b->n, item0_of(b, kz), b->d_act, b->d_act_sim, b->d_act_item0,
                                        set_cond, h);
}

// Tiles of every grid for zc planes per tile (rows per tile as the grid's own
// pass), ordered heaviest first so the block scheduler ends with the small
// ones; uploaded to b->d_tiles.
static int build_tiles(blz_batch *b, const std::vector<BatchSim> &h, int zc) {
    struct Item { BatchTile t; long long cost; };
    std::vector<Item> items;
    for (int i = 0; i < b->n; ++i) {
        const Geom &g = h[i].g;
        const int ty = batch_tb_rows(g), wq = g.W >> 3;
        for (int j0 = 0; j0 < g.H; j0 += ty)
            for (int z0 = 0; z0 < g.D; z0 += zc) {
                const int z1 = std::min(z0 + zc, g.D);
                items.push_back({BatchTile{i, j0, z0, z1, ty}, (long long)(ty + 8) * wq * (z1 - z0 + 6)});
            }
    }
    std::stable_sort(items.begin(), items.end(), [](const Item &x, const Item &y) { return x.cost > y.cost; });
    std::vector<BatchTile> t(items.size());
    for (size_t i = 0; i < items.size(); ++i) t[i] = items[i].t;
    if ((int)t.size() > b->tiles_cap) {
        cudaFree(b->d_tiles);
        b->d_tiles = nullptr;
        b->tiles_cap = 0;
        BCK(cudaMalloc(&b->d_tiles, sizeof(BatchTile) * t.size()));
        b->tiles_cap = (int)t.size();
    }
    BCK(cudaMemcpyAsync(b->d_tiles, t.data(), sizeof(BatchTile) * t.size(), cudaMemcpyHostToDevice, b->st));
    BCK(cudaStreamSynchronize(b->st));
    b->ntiles = (int)t.size();
    return BLZ_OK;
}

// Body of the batched solve, appended to the capture in progress on b->st:
// check_every sweeps over the grids still running, their residual and decision.
static void capture_body(blz_batch *b, cudaGraphConditionalHandle h) {
    if (b->tb_zc > 0)
        launch_batch_tb(b->d_sims, b->d_tiles, b->ntiles, b->d_ctl, b->chunk, b->tb_smem, b->tb_pk, b->st);
    else launch_batch_sweeps(b->d_sims, b->d_act, b->n, b->chunk, b->kz, b->grid, b->block, b->st);
    launch_batch_check(b->d_sims, b->d_blk0, b->n, b->total_blocks, b->d_ctl, b->partials, 1, b->chunk, b->st);
    active_list(b, b->kz, 1, h);
}

// Builds [stages before the solve] + solve loop + [stages after] as one graph.
// with_stages: every grid's forces + divergence before and gradient + advect
// after the loop (their launches are counted into *stage_launches).
static int build_graph(blz_batch *b, bool with_stages, cudaGraphExec_t *out, long long *stage_launches) {
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphConditionalHandle h;
    cudaGraphNode_t cond;
    int rc = BLZ_OK;
    long long l0 = 0, l1 = 0;
    auto launches_now = [&]() {
        long long t = 0;
        for (auto *s : b->sims) t += blz_kernel_launches(s);
        return t;
    };
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, graph, 0, 0);
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(b->st, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) goto done;
    l0 = launches_now();
    if (with_stages)
        for (auto *s : b->sims) {
            if ((rc = blz_forces(s, 0.0f)) != BLZ_OK || (rc = blz_divergence(s)) != BLZ_OK) break;
        }
    if (rc == BLZ_OK) {
        // Learned warm starts of the solvers that have a network, one after
        // another on the batch stream (networks of equal dims may be shared).
        long long w0 = launches_now();
        for (int i = 0; i < b->n && rc == BLZ_OK; ++i)
            if (solver_warm(b->sims[i])) rc = solver_warm_start(b->sims[i], kBatchWarmVariant, &b->pre[i]);
            else b->pre[i] = 0;
        b->warm_launches = launches_now() - w0;
    }
    if (rc == BLZ_OK) {
        k_batch_begin<<<(b->n + 255) / 256, 256, 0, b->st>>>(b->d_ctl, b->n);
        launch_batch_check(b->d_sims, b->d_blk0, b->n, b->total_blocks, b->d_ctl, b->partials, 0, b->chunk, b->st);
        active_list(b, b->kz, 1, h);
        cudaStreamCaptureStatus status;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        e = cudaStreamGetCaptureInfo(b->st, &status, nullptr, nullptr, &deps, &ndeps);
        if (e == cudaSuccess) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&cond, graph, deps, ndeps, &cp);
            if (e == cudaSuccess) {
                body = cp.conditional.phGraph_out[0];
                e = cudaStreamUpdateCaptureDependencies(b->st, &cond, 1, cudaStreamSetCaptureDependencies);
            }
        }
    }
    {
        cudaGraph_t g2 = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(b->st, &g2);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess || rc != BLZ_OK) goto done;
    e = cudaStreamBeginCaptureToGraph(b->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) goto done;
    capture_body(b, h);
    {
        cudaGraph_t g2 = nullptr;
        e = cudaStreamEndCapture(b->st, &g2);
    }
    if (e != cudaSuccess) goto done;
    if (with_stages) {
        e = cudaStreamBeginCaptureToGraph(b->st, graph, &cond, nullptr, 1, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) goto done;
        for (auto *s : b->sims) {
            if ((rc = blz_gradient(s)) != BLZ_OK || (rc = blz_advect(s)) != BLZ_OK) break;
        }
        cudaGraph_t g2 = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(b->st, &g2);
        if (e == cudaSuccess) e = e2;
        if (e != cudaSuccess || rc != BLZ_OK) goto done;
    }
    l1 = launches_now();
    if (stage_launches) *stage_launches = l1 - l0;
    e = cudaGraphInstantiate(out, graph, 0);
done:
    if (e != cudaSuccess) {
        cudaStreamCaptureStatus status;
        if (cudaStreamIsCapturing(b->st, &status) == cudaSuccess && status != cudaStreamCaptureStatusNone) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(b->st, &junk);
        }
        cudaGetLastError();
        if (rc == BLZ_OK) rc = bfail(BLZ_ERR_CUDA, "building the batch graph failed: %s", cudaGetErrorString(e));
    }
    if (graph) cudaGraphDestroy(graph);
    return rc;
}

// Autotuner: the segment kernel's planes per thread x block size (two sweeps
// of the whole batch timed) against temporal blocking with 8, 16 or 32
// planes per tile, scalar or paired-FP32 stencil (four sweeps timed), per
// sweep, on scratch copies of every pressure (all shapes give identical
// results).
static int tune(blz_batch *b) {
    if (b->kz >= 0) return BLZ_OK;
    std::vector<BatchSim> h(b->n), hs(b->n);
    BCK(cudaMemcpy(h.data(), b->d_sims, sizeof(BatchSim) * b->n, cudaMemcpyDeviceToHost));
    size_t total = 0;
    for (auto &s : h) total += (size_t)s.g.W * s.g.H * s.g.D;
    float *scratch = nullptr;
    BatchSim *d_scr = nullptr;
    BCK(cudaMalloc(&scratch, total * sizeof(float)));
    cudaError_t e = cudaMalloc(&d_scr, sizeof(BatchSim) * b->n);
    size_t off = 0;
    for (int i = 0; i < b->n && e == cudaSuccess; ++i) {
        const size_t half = (size_t)h[i].g.W * h[i].g.H * h[i].g.D / 2;
        hs[i] = h[i];
        hs[i].p_r = scratch + off;
        hs[i].p_b = scratch + off + half;
        e = cudaMemcpyAsync(hs[i].p_r, h[i].p_r, half * sizeof(float), cudaMemcpyDeviceToDevice, b->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hs[i].p_b, h[i].p_b, half * sizeof(float), cudaMemcpyDeviceToDevice, b->st);
        off += 2 * half;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_scr, hs.data(), sizeof(BatchSim) * b->n, cudaMemcpyHostToDevice, b->st);
    if (e == cudaSuccess) {
        k_batch_begin<<<(b->n + 255) / 256, 256, 0, b->st>>>(b->d_ctl, b->n);
        e = cudaGetLastError();
    }
    float best = 1e30f;
    for (int ki = 0; ki < 4 && e == cudaSuccess; ++ki)
        for (int bi = 0; bi < 2 && e == cudaSuccess; ++bi) {
            const int kz = kKZ[ki], blk = kBlocks[bi], grid = batch_sweep_grid(kz, blk);
            active_list(b, kz, 0, 0);
            launch_batch_sweeps(d_scr, b->d_act, b->n, 1, kz, grid, blk, b->st);
            e = cudaEventRecord(b->ev0, b->st);
            launch_batch_sweeps(d_scr, b->d_act, b->n, 2, kz, grid, blk, b->st);
            if (e == cudaSuccess) e = cudaEventRecord(b->ev1, b->st);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventSynchronize(b->ev1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            b->launches += 7;
            if (e == cudaSuccess && ms / 2.0f < best) { best = ms / 2.0f; b->kz = kz; b->block = blk; b->grid = grid; }
        }
    b->tb_zc = 0;
    b->tb_pk = false;
    int tb_best = b->force_zc > 0 ? b->force_zc : 0;
    bool pk_best = b->force_zc > 0 && b->force_pk;
    for (int zi = 0; zi < 3 && b->tb_ok && b->force_zc < 0 && e == cudaSuccess; ++zi) {
        const int zc = kTbZC[zi];
        const int rc = build_tiles(b, h, zc);
        if (rc != BLZ_OK) { e = cudaErrorUnknown; break; }
        for (int pk = 0; pk < 2 && e == cudaSuccess; ++pk) {
            launch_batch_tb(d_scr, b->d_tiles, b->ntiles, b->d_ctl, 4, b->tb_smem, pk != 0, b->st);
            e = cudaEventRecord(b->ev0, b->st);
            launch_batch_tb(d_scr, b->d_tiles, b->ntiles, b->d_ctl, 4, b->tb_smem, pk != 0, b->st);
            if (e == cudaSuccess) e = cudaEventRecord(b->ev1, b->st);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventSynchronize(b->ev1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            b->launches += 4;
            if (e == cudaSuccess && ms / 4.0f < best) { best = ms / 4.0f; tb_best = zc; pk_best = pk != 0; }
        }
    }
    if (e == cudaSuccess && tb_best > 0) {
        b->tb_zc = tb_best;
        b->tb_pk = pk_best;
        if (build_tiles(b, h, tb_best) != BLZ_OK) e = cudaErrorUnknown;
        // no sweeps: only the kernels' shared-memory limit, set outside the capture
        launch_batch_tb(d_scr, b->d_tiles, b->ntiles, b->d_ctl, 0, b->tb_smem, false, b->st);
    }
    cudaStreamSynchronize(b->st);
    cudaFree(scratch);
    cudaFree(d_scr);
    if (e != cudaSuccess) {
        b->kz = -1;
        return bfail(BLZ_ERR_CUDA, "batch autotune failed: %s", cudaGetErrorString(e));
    }
    return BLZ_OK;
}

static void release(blz_batch *b) {
    if (b->solve_exec) cudaGraphExecDestroy(b->solve_exec);
    for (auto &x : b->frame_exec) if (x) cudaGraphExecDestroy(x);
    cudaFree(b->d_sims); cudaFree(b->d_ctl); cudaFree(b->d_item0); cudaFree(b->d_blk0); cudaFree(b->partials);
    cudaFree(b->d_act); cudaFree(b->d_act_sim); cudaFree(b->d_act_item0); cudaFree(b->d_tiles);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
}

static int read_stats(blz_batch *b, blz_step_stats *stats, int loop_ran) {
    BCK(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(BatchCtl) * b->n, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    for (int i = 0; i < b->n; ++i)
        if (blz_unet *u = solver_warm(b->sims[i])) {
            const int rc = unet_timeout_flag(u, b->st);
            if (rc != BLZ_OK) return bfail(rc, "simulation %d: a warm-start completion wait gave up", i);
        }
    int max_checks = 0;
    for (int i = 0; i < b->n; ++i) max_checks = std::max(max_checks, b->h_ctl[i].checks);
    if (loop_ran) b->launches += b->prologue + (long long)std::max(0, max_checks - 1) * b->body;
    BCK(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
    for (int i = 0; i < b->n; ++i) {
        const BatchCtl &c = b->h_ctl[i];
        const double r = std::sqrt(c.r2), bn = std::sqrt(c.b2);
        if (!std::isfinite(r)) return bfail(BLZ_ERR_NAN, "simulation %d: non-finite residual after %d sweeps", i, c.iters);
        if (!stats) continue;
        blz_step_stats &st = stats[i];
        st = blz_step_stats{};
        st.iterations = c.iters;
        st.converged = c.converged;
        st.residual = r;
        st.rhs_norm = bn;
        st.rel_residual = bn > 0.0 ? r / bn : 0.0;
        st.residual_checks = c.checks;
        st.sweep_variant = b->tb_zc > 0 ? (b->tb_pk ? 200 : 100) + b->tb_zc : b->kz;
        st.device_loop = 1;
        if (solver_warm(b->sims[i])) {
            st.warm_started = 1;
            st.iterations += b->pre[i];
        }
    }
    return BLZ_OK;
}

// The solve-only graph.  Capturing it counts the warm starts' launches into
// their solvers once; they are counted per replay instead (warm_launches).
static int build_solve_graph_of(blz_batch *b) {
    std::vector<long long> before(b->n);
    for (int i = 0; i < b->n; ++i) before[i] = blz_kernel_launches(b->sims[i]);
    const int rc = build_graph(b, false, &b->solve_exec, nullptr);
    for (int i = 0; i < b->n; ++i) solver_add_launches(b->sims[i], before[i] - blz_kernel_launches(b->sims[i]));
    return rc;
}

extern "C" {

int blz_batch_create(blz_solver *const *sims, int n, blz_batch **out) {
    if (!out || !sims || n < 1) return bfail(BLZ_ERR_ARG, "need at least one solver");
    *out = nullptr;
    blz_batch *b = new blz_batch();
    b->n = n;
    b->pre.assign(n, 0);
    std::vector<BatchSim> h(n);
    std::vector<long long> item0(4 * (size_t)(n + 1));
    std::vector<int> blk0(n + 1);
    for (int i = 0; i < n; ++i) {
        if (!sims[i]) { delete b; return bfail(BLZ_ERR_ARG, "solver %d is null", i); }
        const blz_params *P = nullptr;
        solver_batch_view(sims[i], &h[i], &P);
        if (P->width % 8 || P->gs_order != BLZ_GS_RB3D || !(P->tol > 0.0) || P->check_every < 1 ||
            P->max_iter % P->check_every) {
            delete b;
            return bfail(BLZ_ERR_ARG, "solver %d: the batch needs width %% 8 == 0, 3-D red-black order, tol > 0 "
                                      "and max_iter a multiple of check_every >= 1", i);
        }
        if (P->defect_correction) {
            delete b;
            return bfail(BLZ_ERR_ARG, "solver %d: the batch solves p directly (defect_correction must be 0)", i);
        }
        if (i > 0 && P->check_every != b->params[0]->check_every) {
            delete b;
            return bfail(BLZ_ERR_ARG, "solver %d: all solvers of a batch need the same check_every", i);
        }
        b->sims.push_back(sims[i]);
        b->params.push_back(P);
    }
    b->chunk = b->params[0]->check_every;
    b->tb_ok = b->chunk % 4 == 0;
    for (int i = 0; i < n; ++i) {
        if (!batch_tb_supported(h[i].g)) b->tb_ok = false;
        else b->tb_smem = std::max(b->tb_smem, batch_tb_smem(h[i].g));
    }
    b->time_free = true;
    for (const blz_params *P : b->params)
        if (std::fabs(P->turbulence_amp) > 0.0f || (P->wind_amp > 0.0f && P->wind_speed != 0.0f && P->wind_turb_amp != 0.0f))
            b->time_free = false;
    for (int t = 0; t < 4; ++t) {
        long long acc = 0;
        for (int i = 0; i < n; ++i) {
            item0[(size_t)t * (n + 1) + i] = acc;
            acc += batch_sweep_items(h[i].g, kKZ[t]);
        }
        item0[(size_t)t * (n + 1) + n] = acc;
    }
    int acc = 0;
    for (int i = 0; i < n; ++i) { blk0[i] = acc; acc += residual_blocks(h[i].g); }
    blk0[n] = acc;
    b->total_blocks = acc;
    int rc = BLZ_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == BLZ_OK) rc = bfail(BLZ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    };
    ck(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaMalloc(&b->d_sims, sizeof(BatchSim) * n), "cudaMalloc");
    ck(cudaMalloc(&b->d_ctl, sizeof(BatchCtl) * n), "cudaMalloc");
    ck(cudaMallocHost(&b->h_ctl, sizeof(BatchCtl) * n), "cudaMallocHost");
    ck(cudaMalloc(&b->d_item0, sizeof(long long) * item0.size()), "cudaMalloc");
    ck(cudaMalloc(&b->d_blk0, sizeof(int) * (n + 1)), "cudaMalloc");
    ck(cudaMalloc(&b->d_act, sizeof(BatchActive)), "cudaMalloc");
    ck(cudaMalloc(&b->d_act_sim, sizeof(int) * n), "cudaMalloc");
    ck(cudaMalloc(&b->d_act_item0, sizeof(long long) * (n + 1)), "cudaMalloc");
    ck(cudaMalloc(&b->partials, sizeof(double) * 2 * (size_t)acc), "cudaMalloc");
    ck(cudaEventCreate(&b->ev0), "cudaEventCreate");
    ck(cudaEventCreate(&b->ev1), "cudaEventCreate");
    if (rc == BLZ_OK) ck(cudaMemcpy(b->d_sims, h.data(), sizeof(BatchSim) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
    if (rc == BLZ_OK) ck(cudaMemcpy(b->d_item0, item0.data(), sizeof(long long) * item0.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    if (rc == BLZ_OK) ck(cudaMemcpy(b->d_blk0, blk0.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice), "cudaMemcpy");
    for (int i = 0; i < n && rc == BLZ_OK; ++i) rc = blz_set_stream(sims[i], b->st);
    b->prologue = 1 + 2 + 1;                 // begin, residual + decision, active list
    if (rc != BLZ_OK) {
        release(b);
        delete b;
        return rc;
    }
    *out = b;
    return BLZ_OK;
}

int blz_batch_destroy(blz_batch *b) {
    if (!b) return BLZ_OK;
    cudaStreamSynchronize(b->st);
    // The solvers fall back to their own streams.
    for (auto *s : b->sims) blz_set_stream(s, nullptr);
    release(b);
    delete b;
    return BLZ_OK;
}

void *blz_batch_stream(blz_batch *b) { return b ? (void *)b->st : nullptr; }

int blz_batch_set_sweep(blz_batch *b, int planes, int paired) {
    if (!b) return bfail(BLZ_ERR_ARG, "null batch");
    if (planes < -1) return bfail(BLZ_ERR_ARG, "planes must be -1 (autotune), 0 (segment kernel) or > 0");
    if (planes > 0 && !b->tb_ok)
        return bfail(BLZ_ERR_ARG, "temporal blocking needs check_every %% 4 == 0 and every grid with width %% 8 == 0, "
                                  "width <= 384");
    BCK(cudaStreamSynchronize(b->st));
    b->force_zc = planes;
    b->force_pk = paired != 0;
    b->kz = -1;                               // tune again at the next solve
    if (b->solve_exec) { cudaGraphExecDestroy(b->solve_exec); b->solve_exec = nullptr; }
    for (auto &x : b->frame_exec)
        if (x) { cudaGraphExecDestroy(x); x = nullptr; }
    return BLZ_OK;
}

long long blz_batch_kernel_launches(const blz_batch *b) { return b ? b->launches : 0; }

float blz_batch_last_ms(const blz_batch *b) { return b ? b->last_ms : 0.0f; }

int blz_batch_add_source(blz_batch *b) {
    if (!b) return bfail(BLZ_ERR_ARG, "null batch");
    for (auto *s : b->sims) {
        const long long l0 = blz_kernel_launches(s);
        const int rc = blz_add_source(s);
        if (rc != BLZ_OK) return rc;
        b->launches += blz_kernel_launches(s) - l0;
    }
    return BLZ_OK;
}

// The batched solve alone (after every solver's divergence).
int blz_batch_solve(blz_batch *b, blz_step_stats *stats) {
    if (!b) return bfail(BLZ_ERR_ARG, "null batch");
    int rc = tune(b);
    if (rc != BLZ_OK) return rc;
    b->body = (b->tb_zc > 0 ? b->chunk / 2 : 2 * b->chunk) + 2 + 1;
    if (!b->solve_exec && (rc = build_solve_graph_of(b)) != BLZ_OK) return rc;
    BCK(cudaEventRecord(b->ev0, b->st));
    BCK(cudaGraphLaunch(b->solve_exec, b->st));
    BCK(cudaEventRecord(b->ev1, b->st));
    b->launches += b->warm_launches;
    return read_stats(b, stats, 1);
}

// One frame of every simulation: forces (at times[i]), divergence, the
// batched solve, gradient and advection (sourcing is blz_batch_add_source).
int blz_batch_step(blz_batch *b, const float *times, blz_step_stats *stats) {
    if (!b) return bfail(BLZ_ERR_ARG, "null batch");
    int rc = tune(b);
    if (rc != BLZ_OK) return rc;
    b->body = (b->tb_zc > 0 ? b->chunk / 2 : 2 * b->chunk) + 2 + 1;
    if (b->time_free) {
        const int par = b->parity;
        if (!b->frame_exec[par]) {
            // Capturing runs no kernel but flips every solver's front index
            // (blz_advect) and counts launches that did not happen: undo both.
            std::vector<long long> before(b->n);
            for (int i = 0; i < b->n; ++i) before[i] = blz_kernel_launches(b->sims[i]);
            rc = build_graph(b, true, &b->frame_exec[par], &b->frame_stage_launches[par]);
            for (int i = 0; i < b->n; ++i) {
                solver_flip_front(b->sims[i]);
                solver_add_launches(b->sims[i], before[i] - blz_kernel_launches(b->sims[i]));
            }
            if (rc != BLZ_OK) return rc;
        }
        BCK(cudaEventRecord(b->ev0, b->st));
        BCK(cudaGraphLaunch(b->frame_exec[par], b->st));
        BCK(cudaEventRecord(b->ev1, b->st));
        for (auto *s : b->sims) solver_flip_front(s);
        b->parity ^= 1;
        b->launches += b->frame_stage_launches[par];
        return read_stats(b, stats, 1);
    }
    if (!b->solve_exec && (rc = build_solve_graph_of(b)) != BLZ_OK) return rc;
    BCK(cudaEventRecord(b->ev0, b->st));
    b->launches += b->warm_launches;
    long long l0 = 0, l1 = 0;
    for (auto *s : b->sims) l0 += blz_kernel_launches(s);
    for (int i = 0; i < b->n; ++i) {
        if ((rc = blz_forces(b->sims[i], times ? times[i] : 0.0f)) != BLZ_OK) return rc;
        if ((rc = blz_divergence(b->sims[i])) != BLZ_OK) return rc;
    }
    BCK(cudaGraphLaunch(b->solve_exec, b->st));
    for (auto *s : b->sims) {
        if ((rc = blz_gradient(s)) != BLZ_OK) return rc;
        if ((rc = blz_advect(s)) != BLZ_OK) return rc;
    }
    BCK(cudaEventRecord(b->ev1, b->st));
    for (auto *s : b->sims) l1 += blz_kernel_launches(s);
    b->launches += l1 - l0;
    b->parity ^= 1;
    return read_stats(b, stats, 1);
}

} // extern "C"
