/*
 * blaze_b200.h — C ABI of the B200-native Blaze fluid step (libblaze_b200.so).
 *
 * Plain C: no CUDA, torch or C++ types cross this boundary; every buffer is a
 * pointer plus sizes implied by the grid dimensions.  Each entry point returns
 * BLZ_OK (0) or a negative BLZ_ERR_* code and never exits the process; the
 * text of the last failure is kept per solver (blz_last_error) or per thread
 * (blz_last_error(NULL)).
 *
 * Reference interface replaced (paths inside the Blaze project):
 *   class FluidSolver            src/FluidSolver.h:38-110
 *     FluidSolver(Timer*, SceneSettings*)   src/FluidSolver.cu:671-741  -> blz_create
 *     ~FluidSolver()                        src/FluidSolver.cu:743-768  -> blz_destroy
 *     addSource()                           src/FluidSolver.cu:770-821  -> blz_set_particles + blz_add_source
 *     step()                                src/FluidSolver.cu:858-955  -> blz_step
 *     project() (private)                   src/FluidSolver.cu:823-856  -> blz_project
 *     getTempGrid()                         src/FluidSolver.h:108       -> blz_field_ptr(BLZ_FIELD_T)
 *   struct SceneSettings (solver fields)    src/SceneSettings.h:32-71   -> blz_params
 *   Timer::iter / Timer::time               src/Timer.h:35-36           -> time argument of blz_step
 *   Parser::sourceParticleParse records     src/Parser.h:196-209        -> rec8 layout of blz_set_particles
 *   class RenderEngine           src/RenderEngine.h:46-95
 *     RenderEngine(Timer*, SceneSettings)   src/RenderEngine.cu:250-293 -> blz_render_create
 *     render(Grid**)                        src/RenderEngine.cu:306-365 -> blz_render / blz_render_solver
 *     writeToDisk()                         src/RenderEngine.cu:367-476 -> blz_render_write
 *   struct SceneSettings (renderer fields)  src/SceneSettings.h:73-107  -> blz_render_params
 *   checkCudaErrors -> exit()               src/utils/helper_cuda.h:577 -> negative return codes
 *
 * Grid layout (identical to the reference so fields can be exchanged as is):
 *   FP32, x fastest: index = i + j*w + k*w*h with (w,h,d) the field's own dims.
 *   T, p, rhs: (W, H, D)   U: (W+1, H, D)   V: (W, H+1, D)   W: (W, H, D+1).
 *   Object space flips y (grid j = 0 is the world top, yMax).
 */
#ifndef BLAZE_B200_H
#define BLAZE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BLZ_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define BLZ_OK            0
#define BLZ_ERR_CUDA     -1   /* a CUDA runtime call failed                 */
#define BLZ_ERR_ARG      -2   /* bad argument (dims, null pointer, field)   */
#define BLZ_ERR_TIMEOUT  -3   /* a bounded device wait gave up              */
#define BLZ_ERR_NAN      -4   /* non-finite value detected                  */
#define BLZ_ERR_NOCONV   -5   /* residual target not met within max_iter    */
#define BLZ_ERR_ALLOC    -6   /* device or host allocation failed           */
#define BLZ_ERR_STATE    -7   /* call not valid in the current state        */

/* ---- boundary-condition handling of the pressure solve ------------------ */
/* REF_COMPAT: the reference's Neumann-everywhere solve (the stencil counts
 *   in-domain neighbours only, FluidSolver.cu:536-561) and its boundary
 *   velocity copy after the gradient (FluidSolver.cu:626-668).
 * FREE_SURFACE: open faces (closed_bounds[f] == 0) carry a Dirichlet p = 0
 *   ghost in the stencil and in the gradient, so the projected field is
 *   discretely divergence free and the system is non-singular.             */
#define BLZ_BC_REF_COMPAT    0
#define BLZ_BC_FREE_SURFACE  1

/* ---- Gauss-Seidel ordering ----------------------------------------------- */
/* RB3D: colour (i+j+k)&1, all red cells then all black cells per sweep.
 * PLANE: the reference's schedule run race free (FluidSolver.cu:517-599):
 *   colour (i+j)&1, planes k = 0..D-1 in order, red then black per plane.  */
#define BLZ_GS_RB3D   0
#define BLZ_GS_PLANE  1

/* ---- fields -------------------------------------------------------------- */
#define BLZ_FIELD_T    0
#define BLZ_FIELD_U    1
#define BLZ_FIELD_V    2
#define BLZ_FIELD_W    3
#define BLZ_FIELD_P    4   /* pressure, T dims (stored colour packed inside) */
#define BLZ_FIELD_RHS  5   /* -div/dx with the wall fixes, T dims            */
#define BLZ_FIELD_DENSITY 6 /* smoke density scalar, T dims (density_field)  */

/* ---- solver parameters (SceneSettings' solver subset + new switches) ---- */
typedef struct blz_params {
    int   width, height, depth;   /* gridRes (T dims)                        */
    float dx, dt;
    float domain_min[3];          /* domainBboxMin (world)                   */
    float domain_max[3];          /* domainBboxMax (world)                   */
    int   closed_bounds[6];       /* xMin,xMax,yMin,yMax,zMin,zMax; 1 = wall */

    float density;                /* rho in the pressure scaling             */
    float gravity;                /* negative (world down)                   */
    float buoyancy;               /* beta (temperature)                      */
    float cooling_rate;
    float vorticity_conf;         /* epsilon                                 */
    float drag;

    int   wind_dir;               /* 0:+X 1:-X 2:+Z 3:-Z                     */
    float wind_amp, wind_speed, wind_turb_amp, wind_turb_scale;

    float turbulence_amp, turbulence_scale;
    float turb_mask_temp_ramp[2];
    float turb_mask_vel_ramp[2];

    /* pressure solve controls */
    int    max_iter;              /* maxIterSolve: sweep cap                 */
    double tol;                   /* relative FP64 residual target; <= 0 runs
                                     exactly max_iter sweeps (reference)     */
    int    check_every;           /* sweeps between residual checks (>= 1;
                                     0 counts as 1; < 0: chosen per solve
                                     from 20, 40, ..., 320 to minimise checks
                                     plus sweeps past convergence, given the
                                     previous solve's sweep count)          */
    int    bc_mode;               /* BLZ_BC_*                                */
    int    gs_order;              /* BLZ_GS_*                                */
    int    reset_pressure;        /* 1: p = 0 before every solve (the
                                     reference keeps p between frames)      */
    int    max_particles;         /* sourceMaxParticleCount                  */
    int    temporal_block;        /* 0: the autotuner may pick the two-sweeps-
                                     per-HBM-pass kernel; 1: unblocked
                                     sweeps only                             */
    int    device_loop;           /* 1: a residual-controlled solve runs as one
                                     CUDA graph whose conditional WHILE node
                                     decides on the device (no host round
                                     trip per check); needs max_iter to be a
                                     multiple of check_every                 */
    int    sweep_variant;         /* -1: autotune the sweep launch shape per
                                     grid size (first solve); >= 0: force one */
    int    advect_scheme;         /* BLZ_ADVECT_*: backtrace integrator       */
    /* Target mode only (no counterpart in the reference, whose buoyancy is
     * beta * T alone, FluidSolver.cu:142-156): a smoke density scalar on the
     * T grid, splatted from the particles like T, advected like T (tricubic,
     * clamped at 0), whose weight pulls down:
     * V += dt * (beta * T - buoyancy_alpha * rho) * g.                       */
    int    density_field;         /* 1: carry the density scalar            */
    float  buoyancy_alpha;        /* alpha (density)                         */
    /* 1: every solve works on the correction delta to the current pressure
     * p (defect correction): b - A p is formed in FP64 as the sweeps' right-
     * hand side, the sweeps (the same red-black Gauss-Seidel, so the same
     * iterates in exact arithmetic) run on delta, the gradient uses
     * p + delta difference by difference, and p = RN(p + delta) keeps the
     * exact remainder in delta for the next solve.  With p itself in FP32,
     * rounding bounds the relative residual below by about
     * 2e-7 ||p|| / ||b|| (1e-4 on smooth 256^3 pressures, more at 384^3);
     * the correction form removes that floor.  Not for batches.            */
    int    defect_correction;
} blz_params;

/* Backtrace integrators (FluidSolver.cu:392-456; the reference's step uses
 * RK3, the other two kernels exist there but are never launched).          */
#define BLZ_ADVECT_RK3    0
#define BLZ_ADVECT_EULER  1
#define BLZ_ADVECT_RK2    2

/* ---- per-step statistics ------------------------------------------------- */
typedef struct blz_step_stats {
    int    iterations;            /* GS sweeps run in the last solve         */
    int    converged;             /* 1 if tol was met (or tol <= 0)          */
    double residual;              /* ||b - A p||_2 (FP64) after the solve    */
    double rhs_norm;              /* ||b||_2 (FP64)                          */
    double rel_residual;          /* residual / rhs_norm (0 when b == 0)     */
    float  ms_source, ms_forces, ms_divergence, ms_solve, ms_gradient,
           ms_advect, ms_total;   /* device time per stage (CUDA events)     */
    float  ms_sweeps;             /* device time of the GS sweep launches
                                     alone (residual checks excluded)        */
    int    residual_checks;       /* FP64 residual evaluations in the solve  */
    int    sweep_variant;         /* sweep launch shape used (-1: one-cell)   */
    int    device_loop;           /* 1 if the solve ran as a device loop      */
    float  ms_checks;             /* device-loop solve: time inside the FP64
                                     residual checks (device global timer)   */
    float  ms_warm_start;         /* device time of the learned warm start
                                     (inside ms_solve; 0 without a network)  */
    int    warm_started;          /* 1 if a network set the initial pressure  */
    int    check_interval;        /* sweeps between residual checks used      */
} blz_step_stats;

typedef struct blz_solver blz_solver;

/* Fills *p with the reference's shipped-scene defaults (rho 0.1, g -9.8,
 * closed walls, RBGS in REF_COMPAT mode, 200 sweeps, no residual target). */
int  blz_default_params(blz_params *p);

/* FluidSolver::FluidSolver (FluidSolver.cu:671-741): allocates and zeroes all
 * fields on the current CUDA device.  dims must be >= 4; GS needs even W.   */
int  blz_create(const blz_params *p, blz_solver **out);
int  blz_destroy(blz_solver *s);

/* Optional caller stream (a cudaStream_t passed as void*).  NULL selects the
 * library-owned stream.  All later work of this solver is ordered on it.    */
int  blz_set_stream(blz_solver *s, void *cuda_stream);

/* Particle upload (Parser::sourceParticleParse, Parser.h:174-210): n records
 * of 8 host floats {pos.xyz (world), vel.xyz, pscale, temperature}.         */
int  blz_set_particles(blz_solver *s, const float *rec8, int n);

/* blz_set_particles with a density per particle (target mode): density[p]
 * is splatted into the density scalar by the same cubic pulse as the
 * temperature (blz_set_particles gives every particle density 1).  density
 * may be NULL (all 1).  No counterpart in the reference (its records carry
 * no density); BLZ_ERR_STATE unless the solver has density_field set.     */
int  blz_set_particles_ex(blz_solver *s, const float *rec8, const float *density, int n);

/* The device half of FluidSolver::addSource (FluidSolver.cu:796-816):
 * cubic-pulse splat of the uploaded particles, then front = splat wherever
 * |splat| > 1e-5 on T, U, V (negated, y flip) and W.                        */
int  blz_add_source(blz_solver *s);

/* FluidSolver::step (FluidSolver.cu:858-955): forces, projection, RK3
 * advection and buffer swap.  time = Timer::time (seconds).  stats may be
 * NULL.                                                                     */
int  blz_step(blz_solver *s, float time, blz_step_stats *stats);

/* Stage entry points (used by the step; exposed for stage-level parity).   */
int  blz_forces(blz_solver *s, float time);            /* cooldown..curl noise */
int  blz_project(blz_solver *s, blz_step_stats *st);   /* div, solve, gradient */
int  blz_divergence(blz_solver *s);
int  blz_solve(blz_solver *s, blz_step_stats *st);
int  blz_gradient(blz_solver *s);
int  blz_advect(blz_solver *s);                        /* + swap               */

/* Exactly n Gauss-Seidel sweeps (params' order and boundary handling) on the
 * current rhs and p, with no residual checks (the inner loop of
 * gs_solve_kernel, FluidSolver.cu:526-597, run n times).                    */
int  blz_sweeps(blz_solver *s, int n);

/* The current pressure system solved far past the FP32 floor: the iterate
 * is held in FP64 (red-black SOR with relaxation omega, FP64 residual checks
 * every 50 sweeps) until the FP64 relative residual is <= tol or max_sweeps
 * ran, then rounded once into p.  With the pressure stored in FP32 the
 * relative residual cannot go much below 2e-7 ||p|| / ||b|| (about 1e-4 on
 * smooth 256^3 pressures), so this is how converged pressures are obtained.
 * No counterpart in the reference and not a step of the fluid solve: it
 * computes the targets the learned warm start is trained on.  Allocates
 * 16 bytes per cell for the call; synchronises.                             */
int  blz_tight_solve(blz_solver *s, double tol, int max_sweeps, double omega, int *sweeps, double *rel_residual);

/* FP64 ||b - A p||_2 and ||b||_2 of the current rhs and p.                  */
int  blz_residual(blz_solver *s, double *res_norm, double *rhs_norm);

/* ---- z-slab decomposition of one grid's pressure solve --------------------
 * No counterpart in the reference (one GPU, FluidSolver.cu:517-599 solves
 * the whole grid).  Ranks (one process per GPU) each hold a solver of the
 * whole grid, run the step's other stages on the whole grid, and split the
 * solve into z slabs: each rank updates planes [z0, z1) only, and the caller
 * moves halo planes between ranks (blaze_b200/slab.py does both).  Slab
 * bounds are multiples of BLZ_SLAB_ALIGN (or D).  A pass over a slab reads
 * the black pressure on [z0 - BLZ_SLAB_HALO, z1 + BLZ_SLAB_HALO); the
 * residual of a slab reads p on planes z0 - 1 and z1.  The residual's
 * partial sums of all slabs, gathered into one array, reduce in the
 * whole-grid order, so the decomposed solve takes the same sweeps and gives
 * the same pressure, bit for bit, as blz_solve on one GPU (RB3D order, check
 * interval a multiple of 4, no defect correction).  All calls are
 * asynchronous on the solver's stream except blz_reduce_partials.           */
#define BLZ_SLAB_ALIGN 16
#define BLZ_SLAB_HALO  4
/* supported: the slab entry points apply to this solver (W % 8 == 0 with
 * the temporal-blocking pass, tiled residual, RB3D, no defect correction);
 * n_partials: FP64 pairs of the whole grid's residual; plane_floats: floats
 * per colour plane of the packed pressure (W/2 * H).                        */
int  blz_slab_info(blz_solver *s, int *supported, int *n_partials, long long *plane_floats);
/* Copies planes [z0, z1) of one colour (0 red, 1 black) of the pressure
 * (buf 0) or of the pass scratch (buf 1) to / from device memory of
 * (z1 - z0) * plane_floats floats.                                          */
int  blz_slab_get_planes(blz_solver *s, int buf, int colour, int z0, int z1, void *dst_dev);
int  blz_slab_set_planes(blz_solver *s, int buf, int colour, int z0, int z1, const void *src_dev);
/* One temporal-blocking pass (two red-black sweeps) over planes [z0, z1):
 * black input from the scratch (from_q = 1) or the pressure, both colours
 * written to the other buffer on [z0, z1) only.                             */
int  blz_slab_pass(blz_solver *s, int z0, int z1, int from_q);
/* The residual's FP64 partial sums over the tiles of planes [z0, z1) of p,
 * written to partials (device, n_partials pairs) at their whole-grid
 * indices [first, first + count).                                           */
int  blz_slab_residual(blz_solver *s, int z0, int z1, double *partials, int *first, int *count);
/* ||b - A p|| and ||b|| from a full array of partials (device), summed in
 * the whole-grid residual's order.  Synchronises the solver's stream.       */
int  blz_reduce_partials(blz_solver *s, const double *partials, double *res_norm, double *rhs_norm);

/* Field access in the reference layout.  on_device != 0: dst/src is a device
 * pointer of the field's size; otherwise host memory.                       */
int  blz_get_field(blz_solver *s, int field, float *dst, int on_device);
int  blz_set_field(blz_solver *s, int field, const float *src, int on_device);
size_t blz_field_size(const blz_solver *s, int field);  /* elements, 0 if bad */

/* Device pointer of a field's current front buffer (T, U, V, W).  This is the
 * buffer the reference's getTempGrid() Grid object reads via at(i,j,k); it
 * changes after every blz_step (front/back ping-pong).                      */
void *blz_field_ptr(blz_solver *s, int field);

/* Gradient noise of the wind and turbulence stages (the reference's
 * cudaNoise::perlinNoise, thirdparty/cuda-noise/cuda_noise.cuh:570-615)
 * evaluated on the current device at n host positions {x,y,z}; results go to
 * the host array out.  Lets callers check the noise without a solver.       */
int  blz_perlin(const float *pos3, int n, float scale, int seed, float *out);

/* The rest of the reference's noise library (thirdparty/cuda-noise/
 * cuda_noise.cuh), evaluated at positions {x,y,z}.  Ids 0-8 are the
 * library's basisFunction values (cuda_noise.cuh:13-23); the others are its
 * derived functions.  Each function reads the blz_noise_args fields named
 * beside it, with the library's argument meaning.                           */
#define BLZ_NOISE_CHECKER                  0   /* checker(scale, seed), 324-335          */
#define BLZ_NOISE_DISCRETE                 1   /* discreteNoise(scale, seed), 472-480    */
#define BLZ_NOISE_LINEARVALUE              2   /* linearValue(scale, seed), 482-515      */
#define BLZ_NOISE_FADEDVALUE               3   /* fadedValue(scale, seed), 517-550       */
#define BLZ_NOISE_CUBICVALUE               4   /* cubicValue(scale, seed), 552-568       */
#define BLZ_NOISE_PERLIN                   5   /* perlinNoise(scale, seed), 570-615      */
#define BLZ_NOISE_SIMPLEX                  6   /* simplexNoise(scale, seed), 230-321     */
#define BLZ_NOISE_WORLEY                   7   /* worleyNoise(scale, seed, size, min_num,
                                                  max_num, jitter), 395-436              */
#define BLZ_NOISE_SPOTS                    8   /* spots(... as worley, shape), 337-393   */
#define BLZ_NOISE_REPEATER_PERLIN          9   /* (scale, seed, octaves, lacunarity, decay), 620-633 */
#define BLZ_NOISE_REPEATER_PERLIN_BOUNDED 10   /* (... , threshold), 636-656             */
#define BLZ_NOISE_REPEATER_PERLIN_ABS     11   /* 659-673                                */
#define BLZ_NOISE_REPEATER_SIMPLEX        12   /* 676-690                                */
#define BLZ_NOISE_REPEATER_SIMPLEX_ABS    13   /* 693-707                                */
#define BLZ_NOISE_REPEATER_SIMPLEX_BOUNDED 14  /* (... , threshold), 710-731             */
#define BLZ_NOISE_REPEATER                15   /* repeater(... , basis), 734-779         */
#define BLZ_NOISE_FRACTAL_SIMPLEX         16   /* (scale, seed, du, octaves, lacunarity,
                                                  decay), 782-801                        */
#define BLZ_NOISE_TURBULENCE              17   /* (scale = scaleIn, scale_out, seed,
                                                  strength, basis, basis_out), 804-865   */
#define BLZ_NOISE_REPEATER_TURBULENCE     18   /* (as turbulence, octaves), 867-874      */
#define BLZ_NOISE_COUNT                   19

#define BLZ_SHAPE_STEP      0                  /* spots' profileShape, 26-30             */
#define BLZ_SHAPE_LINEAR    1
#define BLZ_SHAPE_QUADRATIC 2

typedef struct blz_noise_args {
    int   func;                 /* BLZ_NOISE_*                                     */
    int   seed;
    float scale;                /* turbulence: scaleIn                             */
    float scale_out;            /* turbulence: scaleOut                            */
    float size, jitter;         /* worley, spots                                   */
    int   min_num, max_num;     /* feature points per cell (worley, spots)        */
    int   shape;                /* spots: BLZ_SHAPE_*                              */
    int   octaves;              /* repeaters, fractal: n                           */
    float lacunarity, decay;
    float threshold;            /* bounded repeaters                               */
    float du;                   /* fractal simplex: smallest feature size          */
    float strength;             /* turbulence                                      */
    int   basis, basis_out;     /* repeater / turbulence bases (BLZ_NOISE_0..8)    */
} blz_noise_args;

/* Evaluates a->func at n positions pos3 into out (both device memory when
 * on_device, else host memory), on `stream` (NULL: the legacy default
 * stream) for device buffers.  Host buffers are copied through the device
 * and the call returns when out is written.  BLZ_ERR_ARG for an unknown
 * function or basis, octaves outside 0..64, min_num > max_num or n < 0.     */
int  blz_noise(const blz_noise_args *a, const float *pos3, long long n, float *out, int on_device, void *stream);

/* FP64 residual norms without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc (a host
 * application or plugin host that owns all device memory through its own
 * pool, or code that must not let an allocation synchronise the device).
 * Inputs are the caller's device arrays rhs and p in the reference layout
 * (T dims, as blz_get_field returns them); out2_dev receives {||b - A p||_2,
 * ||b||_2} (2 device doubles, b = rho dx^2/dt * rhs, A and the boundary
 * handling as in blz_params), on cuda_stream (NULL: the legacy default
 * stream).  Its scratch is a static 64 KiB device array (one FP64 pair per
 * z-plane), so depth must be <= 4096; larger grids return BLZ_ERR_ARG.
 * The first call on each device looks up that array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture.  All
 * calls share the array: calls that overlap on the GPU (other streams or
 * threads) race and must be serialised by the caller.                      */
int  blz_residual_noalloc(const blz_params *p, const float *rhs_dev, const float *p_dev,
                          double *out2_dev, void *cuda_stream);

/* ---- learned warm start: building blocks --------------------------------- */
/* Activation tensors of the warm-start network are BF16, channels last, with a
 * one-voxel zero halo: element (x,y,z,c) of a W x H x D x C tensor is at
 * ((((z+1)*(H+2) + (y+1))*(W+2) + (x+1))*C + c), and BLZ_CONV_SLACK zero
 * voxels precede and follow the (W+2)(H+2)(D+2) voxels.  No counterpart in
 * the reference (it has no learned components).                             */
#define BLZ_CONV_SLACK 256
typedef struct blz_conv_desc {
    int W, H, D;          /* interior voxels                                  */
    int cin, cout;        /* cin % 16 == 0; cout in {16, 32, 64, 128}         */
    int relu;             /* apply max(0, .) after the bias                   */
    int out_f32;          /* output FP32 instead of BF16 (same layout)        */
} blz_conv_desc;

/* y = conv3x3x3(x, w) + bias on the tcgen05 tensor cores (BF16 operands, FP32
 * accumulation in tensor memory).  x, y: device tensors in the layout above
 * (pointers to the first voxel, after the slack); w: device BF16
 * [27][cout][cin] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1); bias: device FP32
 * [cout].  Only interior voxels of y are written.  cuda_stream may be NULL.  */
int  blz_conv3d(const blz_conv_desc *d, const void *x, const void *w, const float *bias, void *y,
                void *cuda_stream);

/* ---- learned warm start: the network -------------------------------------- */
/* A 4-level 3-D U-Net (channels 16/32/64/128; per level two 3x3x3 convolutions
 * with ReLU; 2x2x2 average pooling; 2x2x2 stride-2 transposed convolutions;
 * skip concatenation [upsampled, skip]; a 1x1x1 head), BF16 activations, FP32
 * accumulation.  It maps, per cell, b = rho dx^2/dt * rhs, a Neumann-ghost
 * indicator, the previous pressure p and the residual r = b - A p (each over
 * its FP64 rms on the whole grid) to delta, and d = kappa * rms(r) * delta.
 * The solve may sweep p and d alike k times first (blz_unet_set_smoothing,
 * default 0; d with a zero right-hand side) and adds alpha M^k d, alpha
 * chosen by blz_unet_set_step (FP64 over the grid; default: minimising the
 * energy norm of the error, which never rises above the plain start's;
 * the residual-norm step keeps the smoothed residual at or below the plain
 * start's).  Parameters are one
 * FP32 array; layer l's
 * weights start at info[4] and its bias at info[5] (blz_unet_layer_info).
 * Weights of a 3x3x3 layer are [27][cout][cin] (tap as in blz_conv3d), of a
 * transposed convolution [8][cout][cin] (parity a + 2b + 4c for the fine
 * voxel (2x+a, 2y+b, 2z+c)), of the head [1][1][16].  Layer order: encoder
 * e0a e0b e1a e1b e2a e2b e3a e3b, decoder d2a d2b d1a d1b d0a d0b, transposed
 * u2 u1 u0, head.                                                            */
typedef struct blz_unet blz_unet;

/* info = {kind (0: 3x3x3, 1: transposed 2x2x2, 2: head), cin, cout, taps,
 * weight offset, bias offset}; BLZ_ERR_ARG past the last layer.             */
int  blz_unet_layer_info(int layer, long long info[6]);
/* Network for a width x height x depth crop (each a positive multiple of 8),
 * with all activations allocated on the current device; parameters zero.   */
int  blz_unet_create(int width, int height, int depth, blz_unet **out);
int  blz_unet_destroy(blz_unet *u);
long long blz_unet_num_params(const blz_unet *u);
long long blz_unet_kernel_launches(const blz_unet *u);
float blz_unet_last_alpha(const blz_unet *u);   /* alpha of the last warm start (synchronises) */
int  blz_unet_set_smoothing(blz_unet *u, int sweeps);   /* k above (>= 0)                  */
/* How alpha is chosen: ENERGY (default) minimises the energy norm
 * ||e - alpha M^k d||_A of the error, alpha = <M^k d, r> / <M^k d, A M^k d>
 * (A symmetric positive definite: at least one Dirichlet face); RESIDUAL
 * minimises the residual norm of the sum.                                  */
#define BLZ_WARM_STEP_RESIDUAL 0
#define BLZ_WARM_STEP_ENERGY   1
int  blz_unet_set_step(blz_unet *u, int mode);
int  blz_unet_set_params(blz_unet *u, const float *params, int on_device);   /* resets Adam */
int  blz_unet_get_params(const blz_unet *u, float *params, int on_device);
int  blz_unet_get_grads(const blz_unet *u, float *grads, int on_device);
int  blz_unet_set_kappa(blz_unet *u, float kappa);
/* Raw network output delta over the crop [origin, origin + dims) of the grid
 * that grid describes (dims and boundary handling), from device arrays rhs
 * and p in the reference layout; out: device FP32, crop dims, x fastest.    */
int  blz_unet_forward(blz_unet *u, const blz_params *grid, const int origin[3], const float *rhs,
                      const float *p, float *out, void *cuda_stream);
/* Loss and gradients of one training sample: L = mean over the crop of
 * (delta - (p_target - p) / (kappa rms(r)))^2.  Fills the parameter
 * gradients and loss[0] = L, loss[1] = mean target^2; synchronises.        */
int  blz_unet_loss_grad(blz_unet *u, const blz_params *grid, const int origin[3], const float *rhs,
                        const float *p, const float *p_target, double loss[2], void *cuda_stream);
/* Introspection for parity tests: padded shape {D+2, H+2, W+2, C} and FP32
 * host copy (halo included, no slack) of internal tensor `id`: activations
 * 0..17 in forward order (X0 e0a cat0 d0a d0b p1 e1a cat1 d1a d1b p2 e2a
 * cat2 d2a d2b p3 e3a e3b; a concat tensor holds [upsampled, skip]), then
 * the activation gradients 18..37 (g_d0b g_d0a g_cat0 g_e0b g_e0a g_p1 g_d1b
 * g_d1a g_cat1 g_e1b g_e1a g_p2 g_d2b g_d2a g_cat2 g_e2b g_e2a g_p3 g_e3b
 * g_e3a; g_x is dL/dx, masked by x's ReLU where x is an activation), which
 * exist after the first blz_unet_loss_grad.  Synchronises the device.      */
int  blz_unet_tensor_shape(const blz_unet *u, int id, int shape[4]);
int  blz_unet_get_tensor(const blz_unet *u, int id, float *out, long long capacity);
/* One Adam step (bias-corrected) with the gradients of the last loss_grad.  */
int  blz_unet_adam(blz_unet *u, float lr, float beta1, float beta2, float eps, void *cuda_stream);
/* Attach (or, with NULL, detach) a network whose dims equal the grid's: every
 * later solve of s starts from the network's warm start of the current
 * pressure and then sweeps to the same residual target.  The network stays
 * owned by the caller and must outlive the attachment.                     */
int  blz_set_warm_start(blz_solver *s, blz_unet *u);

/* ---- batched simulations ---------------------------------------------------- */
/* Many independent solvers (uneven grid sizes) stepped together.  No
 * counterpart in the reference, which runs one FluidSolver per process.  The
 * pressure solves of all grids share launches: each half sweep is one
 * persistent launch over every grid's work items, the FP64 residual one
 * launch over every grid's blocks plus one block per grid that decides,
 * exactly as that grid's own device-loop solve would, whether it goes on; a
 * CUDA graph with a conditional WHILE node loops until no grid goes on.  Each
 * grid's pressure, sweep count and residual equal those of its own solve bit
 * for bit.  A solver with a warm-start network attached (blz_set_warm_start)
 * is warm-started inside the batch exactly as alone, before the batched
 * loop; solvers of equal dims may share a network.  The sweep launch shape
 * is autotuned per batch.  When no grid's forces depend on time (no curl
 * noise, no moving wind noise), every frame is one graph launch.  Every
 * solver needs width % 8 == 0, 3-D red-black order, tol > 0, the same
 * check_every, max_iter a multiple of it, and defect_correction = 0.  The
 * batch puts all solvers on its own stream; while batched, step them only
 * through the batch (the solvers stay owned by the caller and must outlive
 * the batch, which returns them to their own streams when destroyed).      */
typedef struct blz_batch blz_batch;
int  blz_batch_create(blz_solver *const *solvers, int n, blz_batch **out);
int  blz_batch_destroy(blz_batch *b);
void *blz_batch_stream(blz_batch *b);                      /* the batch's cudaStream_t */
/* Sweep kernel of the batched solve: planes = -1 (default) autotunes between
 * the segment kernel (one sweep per pass over HBM) and temporal blocking (two
 * sweeps per pass, tiles of 8, 16 or 32 planes, scalar or paired-FP32
 * stencil); 0 forces the segment kernel; planes > 0 forces temporal blocking
 * with tiles of that many planes, paired != 0 with the paired-FP32 stencil
 * (BLZ_ERR_ARG unless check_every % 4 == 0 and every grid has width % 8 == 0
 * and width <= 384).  Every choice gives the same bits.  The stats'
 * sweep_variant reports the choice: the segment kernel's planes per thread
 * (1, 2, 4, 8), or 100 (scalar) or 200 (paired) + planes per tile.         */
int  blz_batch_set_sweep(blz_batch *b, int planes, int paired);
int  blz_batch_add_source(blz_batch *b);                   /* blz_add_source of every solver */
/* One frame of every solver: forces at times[i] (NULL: 0), divergence, the
 * batched solve, gradient, advection; stats[i] (may be NULL) gets solver i's
 * solve statistics.  Synchronises.                                          */
int  blz_batch_step(blz_batch *b, const float *times, blz_step_stats *stats);
/* The batched solve alone, after every solver's divergence.                 */
int  blz_batch_solve(blz_batch *b, blz_step_stats *stats);
long long blz_batch_kernel_launches(const blz_batch *b);
float blz_batch_last_ms(const blz_batch *b);             /* device ms of the last step/solve */

/* ---- volume renderer ---------------------------------------------------------- */
/* Replaces class RenderEngine (src/RenderEngine.h:46-95, RenderEngine.cu:
 * 50-365): the temperature field rendered as an emissive, absorbing and
 * single-scattering volume under directional lights, with an optional
 * blurred quarter-resolution multiple-scattering term.  The fields are the
 * renderer's part of SceneSettings (src/SceneSettings.h:73-107, parsed by
 * Parser.h:109-170); light_samples is parsed by the reference and unused by
 * its renderer, so it is not carried.                                      */
#define BLZ_MAX_LIGHTS 10
#define BLZ_MAX_RAMP   10

typedef struct blz_render_params {
    int   width, height;                       /* renderRes (pixels)                 */
    float cam_focal, cam_aperture;             /* cam.focal, cam.aperture            */
    float cam_u[3], cam_v[3], cam_w[3];        /* cam.rotMat rows                    */
    float cam_trans[3];                        /* cam.t (camera origin, world)       */
    float p_step, s_step, cutoff;              /* primarySampleRate, shadowSamplingRate,
                                                  cutoff                             */
    float density_scale, shadow_density_scale; /* densityScale, shadowDensityScale   */
    float absorption;                          /* absorption                         */
    float scattering[3], volume_color[3];      /* scatteringColor, volumeColor       */
    float gain;                                /* gain (shadow-ray falloff)          */
    float emission_scale;                      /* emissionScale                      */
    float temp_range[2];                       /* shaderTempRange                    */
    int   ramp_size;                           /* shaderColorRamp.count (1..10)      */
    float ramp_keys[BLZ_MAX_RAMP];
    float ramp_colors[BLZ_MAX_RAMP][3];
    float multi_scatter_scale;                 /* multiScatterScale (0: off)         */
    float multi_scatter_density_mask[2];
    float multi_scatter_color[3];
    int   multi_scatter_blur_iter;
    int   light_count;                         /* 0..10 directional lights           */
    float light_dir[BLZ_MAX_LIGHTS][3];
    float light_color[BLZ_MAX_LIGHTS][3];
    float light_intensity[BLZ_MAX_LIGHTS];
    float light_exposure[BLZ_MAX_LIGHTS];
} blz_render_params;

typedef struct blz_renderer blz_renderer;
/* RenderEngine(Timer*, SceneSettings) (RenderEngine.cu:250-293): `grid`
 * gives the T dims (each >= 4), dx and the domain box.                      */
int  blz_render_create(const blz_render_params *rp, const blz_params *grid, blz_renderer **out);
int  blz_render_destroy(blz_renderer *r);
int  blz_render_set_stream(blz_renderer *r, void *cuda_stream);
/* RenderEngine::render(Grid**) (RenderEngine.cu:306-365): renders the
 * temperature field `temp` (device memory, reference layout i + j*W + k*W*H,
 * the grid's dims) into the renderer's frame buffer.  Synchronises.        */
int  blz_render(blz_renderer *r, const float *temp);
/* The same for a solver's current temperature field.                        */
int  blz_render_solver(blz_renderer *r, blz_solver *s);
/* The frame buffer: width*height RGB float triples, row 0 at the top
 * (framebuffer[i + width*j] of RenderEngine.cu:185).                       */
int  blz_render_get_image(const blz_renderer *r, float *rgb, int on_device);
/* RenderEngine::writeToDisk (RenderEngine.cu:367-476): writes the frame
 * buffer to `path`, format by extension: .ppm (ASCII P3, 255.99 scaling as
 * the reference), .png (8-bit RGBA, clamped), .exr (32-bit float B, G, R
 * scanlines, uncompressed).                                                 */
int  blz_render_write(const blz_renderer *r, const char *path);
/* The writer alone, on any host RGB buffer (width*height float triples, row
 * 0 at the top); host code only, no GPU needed.                            */
int  blz_image_write(const char *path, const float *rgb, int width, int height);
/* Test hook: copies `temp` into the renderer's T volume and samples it at
 * n texel coordinates pos3 (device memory, x y z per sample) through the
 * renderer's filtered texture into out (device memory).                    */
int  blz_render_sample_temp(blz_renderer *r, const float *temp, const float *pos3, int n, float *out);
float blz_render_last_ms(const blz_renderer *r);          /* device ms of the last render */
long long blz_render_kernel_launches(const blz_renderer *r);
const char *blz_render_last_error(const blz_renderer *r);

/* Number of kernels this solver launched since creation.                    */
long long blz_kernel_launches(const blz_solver *s);

/* Last error text of s (or of the calling thread when s is NULL).           */
const char *blz_last_error(const blz_solver *s);

#ifdef __cplusplus
}
#endif
#endif /* BLAZE_B200_H */
