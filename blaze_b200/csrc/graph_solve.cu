// graph_solve.cu — the residual-controlled pressure solve as one CUDA graph.
//
// The host loop of blz_solve synchronises after every residual check to
// decide whether to continue (one device->host round trip per check_every
// sweeps).  Here the decision stays on the device: a conditional WHILE node
// runs {check_every sweeps, FP64 residual, control kernel} until the control
// kernel clears the condition (converged, or max_iter sweeps done).  The
// schedule is the host loop's exactly: one check before any sweep, then one
// after every check_every sweeps, capped at max_iter (a multiple of
// check_every on this path).
#include <cmath>

#include "kernels.cuh"

namespace blz {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void k_ctl_begin(SolveCtl *c) {
    c->iters = 0;
    c->checks = 0;
    c->converged = 0;
    c->sweep_ns = 0;
    c->check_ns = 0;
}

// Ends the sweep interval (stop != 0) and starts the check interval, or
// starts a sweep interval.
__global__ void k_ctl_mark(SolveCtl *c, int stop) {
    const unsigned long long t = global_ns();
    if (stop) { c->sweep_ns += t - c->t0; c->t1 = t; }
    else c->t0 = t;
}

// Reads {||r||^2, ||b||^2}, records them, and sets whether the loop goes on.
__global__ void k_ctl_check(SolveCtl *c, const double *__restrict__ norm2, cudaGraphConditionalHandle h,
                            int after_sweeps, int chunk, int max_iter, double tol) {
    if (after_sweeps) {
        c->iters += chunk;
        c->check_ns += global_ns() - c->t1;
    }
    c->checks += 1;
    const double r2 = norm2[0], b2 = norm2[1];
    c->r2 = r2;
    c->b2 = b2;
    const bool conv = b2 == 0.0 || sqrt(r2) / sqrt(b2) <= tol;
    c->converged = conv;
    cudaGraphSetConditional(h, (!conv && c->iters < max_iter) ? 1u : 0u);
}

#define CKG(x)                                      \
    do {                                            \
        cudaError_t e_ = (x);                       \
        if (e_ != cudaSuccess) { err = e_; goto done; } \
    } while (0)

cudaError_t build_solve_graph(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                              float *p_r, float *p_b, double *partials, int n_partials, double *norm2,
                              SolveCtl *ctl, int chunk, int max_iter, double tol, int variant, cudaStream_t st,
                              cudaGraphExec_t *exec_out, int *body_kernels, int *prologue_kernels, float *q_r,
                              float *q_b, const DefectArrays *dfa) {
    cudaError_t err = cudaSuccess;
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphConditionalHandle handle;
    cudaGraphNode_t cond_node;
    long long dummy = 0;
    *exec_out = nullptr;
    // The stopping test: the FP64 residual of (rhs, p); for a defect-
    // correction solve (after sweeps) d folded into p and a fresh defect,
    // whose norms are those of the pressure p + d.  Returns its launches.
    auto check = [&](bool after) -> int {
        if (!dfa) return launch_residual(g, sp, rhs_r, rhs_b, p_r, p_b, partials, n_partials, norm2, st);
        int n = 0;
        if (after) { launch_fold(g, dfa->p_r, dfa->p_b, dfa->d_r, dfa->d_b, st); ++n; }
        return n + launch_defect(g, sp, dfa->rhs_r, dfa->rhs_b, dfa->p_r, dfa->p_b, dfa->d_r, dfa->d_b, dfa->df_r,
                                 dfa->df_b, partials, n_partials, norm2, st);
    };
    CKG(cudaGraphCreate(&graph, 0));
    CKG(cudaGraphConditionalHandleCreate(&handle, graph, 0, 0));
    // Prologue: reset the control block, check once before any sweep.
    CKG(cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    k_ctl_begin<<<1, 1, 0, st>>>(ctl);
    *prologue_kernels = 1 + check(false) + 1;
    k_ctl_check<<<1, 1, 0, st>>>(ctl, norm2, handle, 0, chunk, max_iter, tol);
    {
        cudaStreamCaptureStatus status;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        CKG(cudaStreamGetCaptureInfo(st, &status, nullptr, nullptr, &deps, &ndeps));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        CKG(cudaGraphAddNode(&cond_node, graph, deps, ndeps, &cp));
        body = cp.conditional.phGraph_out[0];
        CKG(cudaStreamUpdateCaptureDependencies(st, &cond_node, 1, cudaStreamSetCaptureDependencies));
    }
    CKG(cudaStreamEndCapture(st, &graph));
    // Body: chunk sweeps (timed with the global timer), residual, decision.
    CKG(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    k_ctl_mark<<<1, 1, 0, st>>>(ctl, 0);
    launch_rbgs_sweeps(g, sp, rhs_r, rhs_b, p_r, p_b, chunk, st, &dummy, variant, q_r, q_b);
    k_ctl_mark<<<1, 1, 0, st>>>(ctl, 1);
    *body_kernels = 2 + (int)dummy + check(true) + 1;
    k_ctl_check<<<1, 1, 0, st>>>(ctl, norm2, handle, 1, chunk, max_iter, tol);
    CKG(cudaStreamEndCapture(st, &body));
    CKG(cudaGraphInstantiate(exec_out, graph, 0));
done:
    if (err != cudaSuccess) {
        cudaStreamCaptureStatus status;
        if (cudaStreamIsCapturing(st, &status) == cudaSuccess && status != cudaStreamCaptureStatusNone) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(st, &junk);
            if (junk) cudaGraphDestroy(junk);
        }
        cudaGetLastError();
    }
    if (graph) cudaGraphDestroy(graph);
    return err;
}

} // namespace blz
