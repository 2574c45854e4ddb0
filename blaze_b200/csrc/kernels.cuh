// kernels.cuh — host-side launchers of the fluid-step kernels.
#pragma once
#include <cuda.h>   // CUtensorMap and its enums (the encoder comes from cudaGetDriverEntryPoint)
#include <cuda_runtime.h>

#include "common.cuh"

namespace blz {

// Parameters of the force stages, resolved on the host once per step.
struct ForceParams {
    int   vort_on, buoy_on, wind_on;
    float conf, tiny;                 // tiny = 1e-20f * (1/(dx*dt)), FluidSolver.cu:226
    float beta, grav;
    int   wind_along_x;               // wind_dir <= 1
    float wind_dir_sign;              // +1 for dirs 0 and 2, else -1
    float wind_amp, wind_turb_amp, wind_freq, wind_offset;
    float turb_amp, turb_freq, turb_offset;
    float tr0, tr1, vr0, vr1;
    int   dens_on;                    // density scalar carried (target mode)
    float alpha;                      // its buoyancy weight
};

struct SolveParams {
    float scale;                      // rho dx^2 / dt (FluidSolver.cu:530)
    double scale_d;                   // the same in FP64 (residual only)
    OpenFaces open;
    int dirichlet;                    // BLZ_BC_FREE_SURFACE
};

// Launch shape for kernels over the union of the face ranges
// [0,W] x [0,H] x [0,D].
dim3 face_block();
dim3 face_grid(const Geom &g);

// -- sourcing ---------------------------------------------------------------
// Cells per bin edge of the sourcing gather (one CTA of kSplatBin^3 threads).
constexpr int kSplatBin = 8;
// Ints per particle of the per-field index boxes: T, U, V, W and the density
// scalar, 6 each.
constexpr int kSplatBoxInts = 30;
// dens (per kept particle) and Dn: the density scalar, both null when the
// solver does not carry it.
void launch_splat_gather(const Geom &g, const float *rec8, const int *boxes, const int *bin_start,
                         const int *bin_list, const int *active, int n_active, int nbx, int nby,
                         float *T, float *U, float *V, float *W, cudaStream_t st, const float *dens = nullptr,
                         float *Dn = nullptr);

// -- forces -------------------------------------------------------------------
void launch_scale(float *a, size_t n, float s, cudaStream_t st);
void launch_vort_omega(const Geom &g, const float *U, const float *V, const float *W, float *ox,
                       float *oy, float *oz, cudaStream_t st);
void launch_vort_force(const Geom &g, const float *U, const float *V, const float *W,
                       const float *ox, const float *oy, const float *oz, const ForceParams &fp,
                       float *fx, float *fy, float *fz, cudaStream_t st);
void launch_face_forces(const Geom &g, float *U, float *V, float *W, const float *T,
                        const float *fx, const float *fy, const float *fz, const ForceParams &fp,
                        cudaStream_t st, const float *Dn = nullptr);
void launch_turb_noise(const Geom &g, const float *T, const float *U, const float *V,
                       const float *W, float *nU, float *nV, float *nW, const ForceParams &fp,
                       cudaStream_t st);
void launch_turb_apply(const Geom &g, float *U, float *V, float *W, const float *nU,
                       const float *nV, const float *nW, const ForceParams &fp, cudaStream_t st);

// cuTensorMapEncodeTiled, looked up once through the runtime's driver entry
// point (nullptr when the driver has none).
typedef CUresult (*TensorMapEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TensorMapEncodeFn tensor_map_encoder();

// -- projection ---------------------------------------------------------------
void launch_divergence(const Geom &g, const float *U, const float *V, const float *W,
                       const OpenFaces &o, float *rhs_r, float *rhs_b, cudaStream_t st);
// Red-black sweeps.  For W % 8 == 0, `variant` picks one of
// kSegVariants launch shapes of the segment kernel (planes per thread and
// rows per block), or (variants kSegVariants.. kSweepVariants-1, with a
// scratch pressure q of the grid's size) the temporal-blocking kernel, two
// sweeps per pass; all give identical results.  Other W use the one-cell
// kernel.  sweep_variant_count: variants available for this grid (0: W % 8).
constexpr int kSegVariants = 6;
constexpr int kSweepVariants = 11;
int  sweep_variant_count(const Geom &g);
// The temporal-blocking variant whose loads are TMA bulk copies (bounded
// waits that may give up: tb_take_timeouts).
bool sweep_variant_uses_tma(int v);
// Bounded TMA waits of the temporal-blocking pass that gave up since the last
// call (then reset); nonzero means a pass produced a wrong result.
unsigned int tb_take_timeouts();
void launch_rbgs_sweeps(const Geom &g, const SolveParams &sp, const float *rhs_r,
                        const float *rhs_b, float *p_r, float *p_b, int sweeps, cudaStream_t st,
                        long long *launches, int variant = 0, float *q_r = nullptr, float *q_b = nullptr);
// The pressure system solved in FP64 (SOR, natural layout) to relative
// residual tol, the result rounded into p (tight.cu).  Returns 0 or a
// cudaError_t.
int tight_solve(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b, float *p_r,
                float *p_b, double tol, int max_sweeps, double omega, int check_every, cudaStream_t st, int *sweeps,
                double *rel, long long *launches);
void launch_plane_sweeps(const Geom &g, const SolveParams &sp, const float *rhs_r,
                         const float *rhs_b, float *p_r, float *p_b, int sweeps, cudaStream_t st,
                         long long *launches);
// Writes partial sums to `partials` (2 doubles per block) and the totals
// {||r||^2, ||b||^2} to out2.  Returns the number of launches (2).
int  launch_residual(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                     const float *p_r, const float *p_b, double *partials, int max_partials,
                     double *out2, cudaStream_t st);
int  residual_blocks(const Geom &g);
// z-slab decomposition of a solve.  slab_pass_supported: the temporal-blocking
// pass applies to g.  launch_tb_pass_slab: one pass (two sweeps) over planes
// [zlo, zhi), black input pin_b (read on [zlo - 4, zhi + 4)), both colours out.
// residual_slab_tiles: the residual partials (whole-grid indices [first,
// first + count)) of planes [z0, z1), z0 and z1 multiples of the tiles'
// depth (z1 may be D); -1 when g's residual is not tiled or the range is
// not aligned.  launch_residual_slab writes them (reads p planes z0 - 1 and
// z1); launch_reduce_pairs sums n pairs in the whole-grid residual's order.
bool slab_pass_supported(const Geom &g);
void launch_tb_pass_slab(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                         const float *pin_b, float *pout_r, float *pout_b, int zlo, int zhi, bool pk,
                         cudaStream_t st);
int  residual_slab_tiles(const Geom &g, int z0, int z1, int *first, int *count);
int  launch_residual_slab(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                          const float *p_r, const float *p_b, int z0, int z1, double *partials, cudaStream_t st);
void launch_reduce_pairs(const double *partials, int n, double *out2, cudaStream_t st);
// d_r/d_b (may be null): the correction of a defect-correction solve, the
// pressure being p + d.
void launch_gradient(const Geom &g, const SolveParams &sp, float dt_over_rho_dx, const float *p_r,
                     const float *p_b, float *U, float *V, float *W, cudaStream_t st, const float *d_r = nullptr,
                     const float *d_b = nullptr);
// Defect-correction solve: rhs' = (b - A p) / scale into def and
// out2 = {||b - A p - A d||^2, ||b||^2}, b = scale rhs (FP64 stencils);
// returns the launches (2).  launch_fold: p = RN(p + d), d = the exact
// remainder.
int  launch_defect(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b, const float *p_r,
                   const float *p_b, const float *d_r, const float *d_b, float *def_r, float *def_b, double *partials,
                   int max_partials, double *out2, cudaStream_t st);
// The arrays of a defect-correction solve (build_solve_graph): its checks
// fold d into p and form a fresh defect instead of a plain residual.
struct DefectArrays {
    const float *rhs_r, *rhs_b;
    float *p_r, *p_b, *d_r, *d_b, *df_r, *df_b;
};
void launch_fold(const Geom &g, float *p_r, float *p_b, float *d_r, float *d_b, cudaStream_t st);
// Packed <-> natural layout.
void launch_pack(const Geom &g, const float *nat, float *red, float *black, cudaStream_t st);
void launch_unpack(const Geom &g, const float *red, const float *black, float *nat,
                   cudaStream_t st);

void launch_perlin(const float *pos3, int n, float scale, int seed, float *out, cudaStream_t st);

// Device-side state of a graph-run solve (see graph_solve.cu).
struct SolveCtl {
    int iters, checks, converged, pad;
    double r2, b2;                      // last ||r||^2, ||b||^2
    unsigned long long sweep_ns, t0;    // global-timer time inside sweep batches
    unsigned long long check_ns, t1;    // ... and inside the residual checks
};
cudaError_t build_solve_graph(const Geom &g, const SolveParams &sp, const float *rhs_r, const float *rhs_b,
                              float *p_r, float *p_b, double *partials, int n_partials, double *norm2,
                              SolveCtl *ctl, int chunk, int max_iter, double tol, int variant, cudaStream_t st,
                              cudaGraphExec_t *exec_out, int *body_kernels, int *prologue_kernels,
                              float *q_r = nullptr, float *q_b = nullptr, const DefectArrays *dfa = nullptr);

// -- batched solve over many grids (k_project.cu kernels, batch.cu graph) ---
struct BatchSim {
    Geom g;
    SolveParams sp;
    const float *rhs_r, *rhs_b;
    float *p_r, *p_b;
    float *q_r, *q_b;                   // the solver's temporal-blocking scratch pressure
    int max_iter;
    double tol;
};
// One temporal-blocking tile of a batch: grid `sim`, output rows
// [j0, j0 + ty) and planes [z0, z1); ty = batch_tb_rows(grid).
struct BatchTile {
    int sim, j0, z0, z1, ty;
};
struct BatchCtl {
    int iters, checks, converged, active;
    double r2, b2;
};
// The grids still running and their work-item offsets (device memory,
// capacity n grids).
struct BatchActive {
    int n;
    int *sim;
    long long *item0;
};
// Segment-kernel threads of one grid for KZ planes per thread (W % 8 == 0).
long long batch_sweep_items(const Geom &g, int kz);
// Persistent grid size (SMs x resident blocks) of the batched sweep.
int  batch_sweep_grid(int kz, int block);
// `sweeps` red+black sweeps over the grids listed in *act (built for this
// kz); nsims bounds its size.
void launch_batch_sweeps(const BatchSim *sims, const BatchActive *act, int nsims, int sweeps, int kz, int grid,
                         int block, cudaStream_t st);
// Temporal blocking in a batch: whether a grid's shape allows it, its tile
// rows and the dynamic shared memory of its tiles; `sweeps` (a multiple of
// 4) sweeps of every active grid as sweeps / 2 passes over the tiles (pk: the
// paired-FP32 stencil; the same bits).
bool batch_tb_supported(const Geom &g);
int  batch_tb_rows(const Geom &g);
size_t batch_tb_smem(const Geom &g);
void launch_batch_tb(const BatchSim *sims, const BatchTile *tiles, int ntiles, const BatchCtl *ctl, int sweeps,
                     size_t smem, bool pk, cudaStream_t st);
// FP64 residual of every active grid (grid s owns partial blocks
// [blk0[s], blk0[s+1]), residual_blocks(g_s) of them) and the per-grid
// continue/stop decision.  2 launches.
void launch_batch_check(const BatchSim *sims, const int *blk0, int nsims, int total_blocks, BatchCtl *ctl,
                        double *partials, int after_sweeps, int chunk, cudaStream_t st);

// Solver internals the batch uses (solver.cu).
void solver_batch_view(blz_solver *s, BatchSim *out, const blz_params **P);
void solver_flip_front(blz_solver *s);
void solver_add_launches(blz_solver *s, long long n);
cudaStream_t solver_stream(blz_solver *s);
const blz_params *solver_params(blz_solver *s);

// -- learned warm start: tensor-core convolution (unet_conv.cu) -------------
struct ConvDesc {
    int W, H, D;        // interior voxels (tensors carry a 1-voxel zero halo)
    int cin, cout;      // cin % 16 == 0; cout in {16, 32, 64, 128}
    int relu, out_f32;
    int out_stride;     // channels per output voxel (>= cout; 0: cout)
    int out_offset;     // first output channel written (multiple of 8)
};
int conv3d_smem_bytes(int cout);
}  // namespace blz
#include <cuda_bf16.h>
namespace blz {
// bias may be null; aux (BF16, same layout as y) masks the output to the
// voxels and channels where aux > 0 (the backward pass of a ReLU).
cudaError_t launch_conv3d(const ConvDesc &cd, const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias,
                          void *y, int *err, cudaStream_t st, const __nv_bfloat16 *aux = nullptr);

// 2x2x2 stride-2 transposed convolution on the tensor cores: x coarse W x H x
// D (padded channels-last, cin channels), w BF16 [8][cout][cin], output into
// channels [0, cout) of the fine tensor y (channel stride ys).  (cin, cout)
// in {(32, 16), (64, 32), (128, 64)}, else cudaErrorNotSupported.
cudaError_t launch_upconv_tc(int W, int H, int D, int cin, int cout, const __nv_bfloat16 *x,
                             const __nv_bfloat16 *w, const float *bias, __nv_bfloat16 *y, int ys, int *err,
                             cudaStream_t st);
// Data gradient of a 2x2x2 transposed convolution on the tensor cores: gx
// (coarse, channel stride cin) = (act > 0) * sum over parities of gy (fine,
// channel stride gs, channels [0, cout)) times the BF16 weights [8][cout][cin].
cudaError_t launch_upconv_dgrad_tc(int W, int H, int D, int cin, int cout, const __nv_bfloat16 *gy, int gs,
                                   const __nv_bfloat16 *w, const __nv_bfloat16 *act, __nv_bfloat16 *gx, int *err,
                                   cudaStream_t st);
// Weight gradient (no bias) of a 3x3x3 convolution (up = 0: x and gy at level
// W x H x D, dw [27][cout][cin]) or of a 2x2x2 transposed convolution (up = 1:
// x coarse at W x H x D, gy fine, dw [8][cout][cin]) on the tensor cores,
// added to dw.  Tensors are padded channels-last, passed at padded voxel 0,
// with BLZ_CONV_SLACK zero voxels on either side; gy zero on its halo.
cudaError_t launch_wgrad_tc(int up, int W, int H, int D, int cin, int cout, const __nv_bfloat16 *x, int xs,
                            const __nv_bfloat16 *gy, int gys, int gyoff, float *dw, int *err, cudaStream_t st);

// Sets the calling thread's error text (what blz_last_error(NULL) returns).
void set_thread_error(const char *msg);

// Solve parameters (scale, open faces, Dirichlet ghosts) of a parameter block.
SolveParams solve_params_of(const blz_params &P);

// Learned warm start (unet.cu), ordered on st, launches added to *launches:
// unet_correction computes the packed correction d (returned with a packed
// zero right-hand side); the caller sweeps p and d unet_smoothing(u) times;
// unet_combine adds alpha d with alpha minimising the residual norm.
int unet_correction(blz_unet *u, const blz_params &P, const float *rhs_r, const float *rhs_b, const float *p_r,
                    const float *p_b, cudaStream_t st, long long *launches, float **d_r, float **d_b,
                    const float **z_r, const float **z_b);
int unet_combine(blz_unet *u, const blz_params &P, const float *rhs_r, const float *rhs_b, float *p_r, float *p_b,
                 cudaStream_t st, long long *launches);
int unet_smoothing(const blz_unet *u);
int unet_prepare(blz_unet *u, const blz_params &P);
// The solver's attached network (null if none) and its warm start (solver.cu).
blz_unet *solver_warm(blz_solver *s);
int solver_warm_start(blz_solver *s, int variant, int *pre);
// BLZ_ERR_TIMEOUT if a tensor-core completion wait of the last warm start
// gave up (synchronises st).
int unet_timeout_flag(blz_unet *u, cudaStream_t st);

// -- advection ------------------------------------------------------------------
// D/Dn: the density scalar and its advected copy (null when not carried).
void launch_advect(const Geom &g, const float *T, const float *U, const float *V, const float *W,
                   float *Tn, float *Un, float *Vn, float *Wn, cudaStream_t st, int scheme,
                   const float *D = nullptr, float *Dn = nullptr);

} // namespace blz
