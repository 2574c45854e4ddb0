// render.cu — volume renderer of the temperature field and its image writers
// (reference src/RenderEngine.cu:50-476 with the device classes of
// Camera.h, Shader.h, Light.h, Ray.h, ColorRamp.h and Volume.h).
//
// Per frame:
//   1. T is copied into a 3-D CUDA array read through a texture object with
//      hardware trilinear filtering, clamped addressing and unnormalised
//      coordinates: the sampler the reference's images are defined by
//      (Volume.h:46-58), so a sample here is the reference's sample.
//   2. With multiple scattering on, T is averaged over 4^3 blocks above the
//      ramp's low temperature and blurred multi_scatter_blur_iter times with
//      the 3^3 [1 2 1]-type kernel (RenderEngine.cu:33-117), in linear memory
//      with clamped indices (the reference samples a texture at texel
//      centres, where trilinear filtering returns the texel itself), then
//      copied into its own filtered 3-D array.
//   3. One thread per pixel marches the camera ray through the domain box:
//      emission from the temperature ramp plus the scatter term, Beer-Lambert
//      extinction per step, and per light a shadow ray marched to the box
//      (RenderEngine.cu:130-231).  Samples in empty 8^3-texel cells skip
//      their texture fetch: the cell maximum proves that the reference's
//      cutoff test rejects them, so the march takes the same steps and keeps
//      the same samples.
// The camera, shader and light constants are formed in the kernel by the
// reference's own expressions (device constructors there), so both builds
// round them alike.  Every loop is bounded: a march never takes more steps
// than the domain diagonal allows (the reference's loops end at the box
// exit; a step too small to advance the ray would make them endless).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace blz {
namespace {

constexpr int kScatterRatio = 4;          // mScatterResRatio (RenderEngine.h:77)
constexpr int kMacro = 8;                 // texels per side of an empty-space cell

struct RenderArgs {
    int res_x, res_y;
    float3 cam_o, cam_u, cam_v, cam_w;
    float focal, aperture;
    float dx;
    float3 dmin, dmax, dsize;
    float p_step, s_step, cutoff;
    float density_scale, shadow_density_scale, absorption;
    float3 scattering, volume_color;
    float gain, emission_scale;
    float t_in, t_out;
    int ramp_n;
    float ramp_keys[BLZ_MAX_RAMP];
    float3 ramp_colors[BLZ_MAX_RAMP];
    float ms_scale, ms_mask0, ms_mask1;
    float3 ms_color;
    int n_lights;
    float3 l_dir[BLZ_MAX_LIGHTS], l_color[BLZ_MAX_LIGHTS];
    float l_intensity[BLZ_MAX_LIGHTS], l_exposure[BLZ_MAX_LIGHTS];
    int max_p_steps, max_s_steps;
    // Empty-space cells: mW x mH x mD cells of kMacro^3 texels, each holding
    // the largest texel under any sample whose coordinate falls in it (the
    // cell plus a one-texel apron).  A primary sample whose cell maximum is
    // below skip_p (shadow: skip_s) fails the reference's cutoff test for
    // sure, so its texture fetch is skipped; -inf disables the test.
    int mW, mH, mD;
    float skip_p, skip_s;
};

// Per-light and ramp tables, read with uniform loads (a kernel parameter
// array indexed by a loop counter would be copied to local memory).
struct Tables {
    float3 l_dir[BLZ_MAX_LIGHTS], l_illum[BLZ_MAX_LIGHTS];
    float ramp_keys[BLZ_MAX_RAMP];
    float3 ramp_colors[BLZ_MAX_RAMP];
};

__device__ __forceinline__ float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float sqlen(float3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
// The reference is built with fast math (its documented flags), so its
// exponentials and divisions are the approximate intrinsics; the renderer
// calls the same ones.
__device__ __forceinline__ float3 exp3(float3 a) { return f3(__expf(a.x), __expf(a.y), __expf(a.z)); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

struct Ray {
    float3 o, d, inv;
    int sx, sy, sz;
    float t0, t1;
};

__device__ __forceinline__ Ray make_ray(float3 o, float3 d) {
    Ray r;
    r.o = o;
    r.d = d;
    r.inv = f3(fdiv(1.0f, d.x), fdiv(1.0f, d.y), fdiv(1.0f, d.z));
    r.sx = r.inv.x < 0.0f; r.sy = r.inv.y < 0.0f; r.sz = r.inv.z < 0.0f;
    r.t0 = 0.0f;
    r.t1 = __int_as_float(0x7f800000);
    return r;
}

// Slab test of the ray against the domain box (RenderEngine.cu:119-157):
// on a hit, [t0, t1] is the part of the ray inside it, t0 clamped at 0.
__device__ bool box_hit(Ray &r, float3 lo, float3 hi) {
    const float bxs = r.sx ? hi.x : lo.x, bxe = r.sx ? lo.x : hi.x;
    const float bys = r.sy ? hi.y : lo.y, bye = r.sy ? lo.y : hi.y;
    const float bzs = r.sz ? hi.z : lo.z, bze = r.sz ? lo.z : hi.z;
    float tmin = (bxs - r.o.x) * r.inv.x;
    float tmax = (bxe - r.o.x) * r.inv.x;
    const float tymin = (bys - r.o.y) * r.inv.y;
    const float tymax = (bye - r.o.y) * r.inv.y;
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    const float tzmin = (bzs - r.o.z) * r.inv.z;
    const float tzmax = (bze - r.o.z) * r.inv.z;
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    r.t0 = fmaxf(tmin, 0.0f);
    r.t1 = tmax;
    return !(r.t1 < 0.0f);
}

// World position -> texel coordinates of T, y measured down from the top of
// the domain (Grid.h:292-296).
// inv_dx = fdiv(1, dx): the fast-math quotient x / dx is x times the
// approximate reciprocal of dx, formed once per thread here.
__device__ __forceinline__ float3 world_to_grid(const RenderArgs &a, float inv_dx, float3 p) {
    return f3((p.x - a.dmin.x) * inv_dx, (a.dsize.y - (p.y - a.dmin.y)) * inv_dx, (p.z - a.dmin.z) * inv_dx);
}

// Temperature ramp (ColorRamp.h:57-79): piecewise-linear over keys in
// [0, 1] after remapping [t_in, t_out].
__device__ float3 ramp_color(const RenderArgs &a, const Tables *__restrict__ tb, float temp) {
    const float x = fminf(fmaxf(fdiv(temp - a.t_in, a.t_out - a.t_in), 0.0f), 1.0f);
    if (a.ramp_n == 1) return tb->ramp_colors[0];
    int prev = 0, next = 0;
    for (int i = 0; i < a.ramp_n; ++i) {
        if (tb->ramp_keys[i] <= x) {
            prev = i;
        } else {
            next = i;
            break;
        }
    }
    const float range = tb->ramp_keys[next] - tb->ramp_keys[prev];
    const float blend = fdiv(x - tb->ramp_keys[prev], range);
    const float3 cp = tb->ramp_colors[prev], cn = tb->ramp_colors[next];
    return cp + blend * (cn - cp);
}

__device__ __forceinline__ float smooth_step(float e0, float e1, float x) {
    const float y = fmaxf(0.0f, fminf(fdiv(x - e0, e1 - e0), 1.0f));
    return y * y * (3.0f - (2.0f * y));
}

// One pixel per thread (RenderEngine.cu:159-231).
// Largest texel over each empty-space cell and its one-texel apron.
__global__ void k_macro_max(const float *__restrict__ T, int W, int H, int D, int mW, int mH, int mD,
                            float *__restrict__ out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= mW * mH * mD) return;
    const int mx = m % mW, my = (m / mW) % mH, mz = m / (mW * mH);
    const int x0 = max(mx * kMacro - 1, 0), x1 = min(mx * kMacro + kMacro, W - 1);
    const int y0 = max(my * kMacro - 1, 0), y1 = min(my * kMacro + kMacro, H - 1);
    const int z0 = max(mz * kMacro - 1, 0), z1 = min(mz * kMacro + kMacro, D - 1);
    float v = -INFINITY;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) v = fmaxf(v, __ldg(T + lin(x, y, z, W, H)));
    out[m] = v;
}

// The cell maximum at texel coordinates g: a point-filtered, clamped 3-D
// texture of the cells, sampled at g / kMacro (the texture unit forms floor
// and clamp; measured faster than forming the cell index in registers and
// reloading only on a change of cell).
__device__ __forceinline__ float macro_at(cudaTextureObject_t mtex, float3 g) {
    return tex3D<float>(mtex, g.x * (1.0f / kMacro), g.y * (1.0f / kMacro), g.z * (1.0f / kMacro));
}

// The tables; light intensities color * intensity * 2^exposure (Light.h:
// 44-47) are formed on the device as the reference's Light constructor does.
__global__ void k_tables_setup(RenderArgs a, Tables *__restrict__ tb) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int l = 0; l < a.n_lights; ++l) {
        tb->l_dir[l] = a.l_dir[l];
        tb->l_illum[l] = a.l_color[l] * a.l_intensity[l] * powf(2.0f, a.l_exposure[l]);
    }
    for (int i = 0; i < a.ramp_n; ++i) {
        tb->ramp_keys[i] = a.ramp_keys[i];
        tb->ramp_colors[i] = a.ramp_colors[i];
    }
}

__global__ void __launch_bounds__(64) k_render(RenderArgs a, cudaTextureObject_t temp_tex,
                                               cudaTextureObject_t scatter_tex, cudaTextureObject_t macro_tex,
                                               const Tables *__restrict__ tb, float *__restrict__ fb) {
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    if (i >= a.res_x || j >= a.res_y) return;
    float *out = fb + 3 * ((size_t)i + (size_t)a.res_x * j);
    out[0] = out[1] = out[2] = 0.0f;

    // camera (Camera.h:41-60)
    const float aspect = fdiv((float)a.res_x, (float)a.res_y);
    const float half_w = 0.5f * a.aperture;
    const float half_h = fdiv(half_w, aspect);
    const float3 top_left = a.cam_o - a.focal * a.cam_w - half_w * a.cam_u + half_h * a.cam_v;
    const float3 horiz = 2.0f * half_w * a.cam_u;
    const float3 vert = -2.0f * half_h * a.cam_v;
    const float3 v = top_left + fdiv(i + 0.5f, (float)a.res_x) * horiz + fdiv(j + 0.5f, (float)a.res_y) * vert - a.cam_o;
    const float3 dir = v * rsqrtf(dot3(v, v));
    Ray pr = make_ray(a.cam_o, dir);
    if (!box_hit(pr, a.dmin, a.dmax)) return;

    // shader constants (Shader.h:53-67)
    const float3 sa = a.scattering + f3(a.absorption, a.absorption, a.absorption);
    const float3 vs = a.volume_color * a.scattering;
    const float3 albedo = f3(fdiv(vs.x, sa.x), fdiv(vs.y, sa.y), fdiv(vs.z, sa.z));
    const float3 ext = (a.scattering + f3(a.absorption, a.absorption, a.absorption)) * -1.0f;
    const float3 one = f3(1.0f, 1.0f, 1.0f);
    const float inv_dx = fdiv(1.0f, a.dx);

    float3 lumi = f3(0.0f, 0.0f, 0.0f);
    float3 trans = f3(1.0f, 1.0f, 1.0f);
    int np = 0;
    for (float pt = pr.t0 + a.dx * 0.5f; pt <= pr.t1 && np < a.max_p_steps; pt += a.p_step, ++np) {
        const float3 ppos = pr.o + pt * pr.d;
        const float3 pg = world_to_grid(a, inv_dx, ppos);
        if (macro_at(macro_tex, pg) < a.skip_p) continue;
        const float temp = tex3D<float>(temp_tex, pg.x, pg.y, pg.z);
        const float density = temp * a.density_scale;
        if (density < a.cutoff) continue;
        // (the reference samples the scatter volume before this test; its
        // value is only used after it)
        const float scat = tex3D<float>(scatter_tex, pg.x / (float)kScatterRatio, pg.y / (float)kScatterRatio,
                                        pg.z / (float)kScatterRatio);

        float3 emission = f3(0.0f, 0.0f, 0.0f);
        if (a.emission_scale > 0.0f)
            emission = ramp_color(a, tb, temp) * a.emission_scale +
                       a.ms_color * scat * a.ms_scale * smooth_step(a.ms_mask0, a.ms_mask1, temp);
        const float3 dT = exp3(ext * density * a.p_step);

        for (int l = 0; l < a.n_lights; ++l) {
            // directional light (Light.h:37-54)
            Ray sr = make_ray(ppos, -1.0f * tb->l_dir[l]);
            box_hit(sr, a.dmin, a.dmax);
            float3 s_trans = f3(1.0f, 1.0f, 1.0f);
            int ns = 0;
            for (float st = sr.t0 + a.dx * 0.5f; st <= sr.t1 && ns < a.max_s_steps; st += a.s_step, ++ns) {
                const float3 sg = world_to_grid(a, inv_dx, sr.o + st * sr.d);
                if (macro_at(macro_tex, sg) < a.skip_s) continue;
                const float sd = tex3D<float>(temp_tex, sg.x, sg.y, sg.z) * a.density_scale * a.shadow_density_scale;
                if (sd < a.cutoff) continue;
                s_trans = s_trans * exp3((ext * sd * a.s_step) * fdiv(1.0f, 1.0f + st * a.gain));
                if (sqlen(s_trans) < a.cutoff) break;
            }
            lumi = lumi + albedo * s_trans * trans * tb->l_illum[l] * (one - dT);
        }
        lumi = lumi + trans * emission * (one - dT);
        trans = trans * dT;
        if (sqlen(trans) < a.cutoff) break;
    }
    out[0] = lumi.x;
    out[1] = lumi.y;
    out[2] = lumi.z;
}

// 4^3 block average of T above t_min (RenderEngine.cu:73-97).
__global__ void k_scatter_down(const float *__restrict__ T, int W, int H, int SW, int SH, int SD, float t_min,
                               float *__restrict__ out) {
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = threadIdx.z + blockIdx.z * blockDim.z;
    if (i >= SW || j >= SH || k >= SD) return;
    float acc = 0.0f;
    for (int io = 0; io < kScatterRatio; ++io)
        for (int jo = 0; jo < kScatterRatio; ++jo)
            for (int ko = 0; ko < kScatterRatio; ++ko) {
                const float t = __ldg(T + lin(i * kScatterRatio + io, j * kScatterRatio + jo,
                                              k * kScatterRatio + ko, W, H));
                acc += t > t_min ? t : 0.0f;
            }
    acc /= (float)(kScatterRatio * kScatterRatio * kScatterRatio);
    out[lin(i, j, k, SW, SH)] = acc;
}

// 3^3 blur with clamped neighbours (RenderEngine.cu:50-71): weights
// w[kk][jj][ii] / 28 summed in the reference's order (x fastest).
__constant__ float c_blur_w[27];

__global__ void k_scatter_blur(const float *__restrict__ in, int SW, int SH, int SD, float *__restrict__ out) {
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = threadIdx.z + blockIdx.z * blockDim.z;
    if (i >= SW || j >= SH || k >= SD) return;
    float acc = 0.0f;
    int idx = 0;
    for (int dk = -1; dk <= 1; ++dk)
        for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di, ++idx) {
                const int x = min(max(i + di, 0), SW - 1);
                const int y = min(max(j + dj, 0), SH - 1);
                const int z = min(max(k + dk, 0), SD - 1);
                acc += __ldg(in + lin(x, y, z, SW, SH)) * c_blur_w[idx];
            }
    out[lin(i, j, k, SW, SH)] = acc;
}

// Samples the T texture at n texel coordinates (a test hook for the
// sampler's parity with the oracle).
__global__ void k_sample(cudaTextureObject_t tex, const float *__restrict__ pos, int n, float *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = tex3D<float>(tex, pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]);
}

const float kBlurKernel[27] = {0, 1, 0, 1, 2, 1, 0, 1, 0,
                               1, 2, 1, 2, 4, 2, 1, 2, 1,
                               0, 1, 0, 1, 2, 1, 0, 1, 0};

} // namespace
} // namespace blz

using namespace blz;

struct blz_renderer {
    blz_render_params rp{};
    RenderArgs a{};
    int W = 0, H = 0, D = 0, SW = 0, SH = 0, SD = 0;
    int device = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    cudaArray_t t_arr = nullptr, s_arr = nullptr;
    cudaTextureObject_t t_tex = 0, s_tex = 0;
    float *s_buf[2] = {nullptr, nullptr};
    float *fb = nullptr;
    Tables *tables = nullptr;
    float *macro = nullptr;
    cudaArray_t m_arr = nullptr;
    cudaTextureObject_t m_tex = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float last_ms = 0.0f;
    long long launches = 0;
    std::string err;
};

static thread_local std::string g_render_err;

static int rfail(blz_renderer *r, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (r) r->err = buf;
    g_render_err = buf;
    return code;
}

#define RCK(r, x)                                                                               \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess)                                                                  \
            return rfail((r), BLZ_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_));       \
    } while (0)

static void render_release(blz_renderer *r) {
    if (!r) return;
    if (r->t_tex) cudaDestroyTextureObject(r->t_tex);
    if (r->s_tex) cudaDestroyTextureObject(r->s_tex);
    if (r->t_arr) cudaFreeArray(r->t_arr);
    if (r->s_arr) cudaFreeArray(r->s_arr);
    cudaFree(r->s_buf[0]);
    cudaFree(r->s_buf[1]);
    cudaFree(r->fb);
    cudaFree(r->tables);
    cudaFree(r->macro);
    if (r->m_tex) cudaDestroyTextureObject(r->m_tex);
    if (r->m_arr) cudaFreeArray(r->m_arr);
    if (r->e0) cudaEventDestroy(r->e0);
    if (r->e1) cudaEventDestroy(r->e1);
    if (r->own_stream && r->st) cudaStreamDestroy(r->st);
}

static int make_volume(blz_renderer *r, int w, int h, int d, cudaArray_t *arr, cudaTextureObject_t *tex,
                       cudaTextureFilterMode filter = cudaFilterModeLinear) {
    const cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float>();
    RCK(r, cudaMalloc3DArray(arr, &fmt, make_cudaExtent(w, h, d)));
    cudaResourceDesc res{};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = *arr;
    cudaTextureDesc td{};
    td.filterMode = filter;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    RCK(r, cudaCreateTextureObject(tex, &res, &td, nullptr));
    return BLZ_OK;
}

static int copy_to_volume(blz_renderer *r, const float *src, int w, int h, int d, cudaArray_t arr) {
    cudaMemcpy3DParms cp{};
    cp.srcPtr = make_cudaPitchedPtr(const_cast<float *>(src), (size_t)w * sizeof(float), w, h);
    cp.dstArray = arr;
    cp.extent = make_cudaExtent(w, h, d);
    cp.kind = cudaMemcpyDeviceToDevice;
    RCK(r, cudaMemcpy3DAsync(&cp, r->st));
    return BLZ_OK;
}

static float3 v3(const float *p) { return make_float3(p[0], p[1], p[2]); }

// ---- image writers (RenderEngine.cu:367-476) --------------------------------

static uint32_t crc32_of(const uint8_t *p, size_t n, uint32_t c = 0xffffffffu) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t v = i;
            for (int b = 0; b < 8; ++b) v = (v & 1) ? 0xedb88320u ^ (v >> 1) : v >> 1;
            table[i] = v;
        }
        init = true;
    }
    for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xff] ^ (c >> 8);
    return c;
}

static void put_be32(std::vector<uint8_t> &v, uint32_t x) {
    v.push_back(x >> 24); v.push_back(x >> 16); v.push_back(x >> 8); v.push_back(x);
}

static void png_chunk(std::vector<uint8_t> &out, const char *type, const std::vector<uint8_t> &data) {
    put_be32(out, (uint32_t)data.size());
    std::vector<uint8_t> td(type, type + 4);
    td.insert(td.end(), data.begin(), data.end());
    out.insert(out.end(), td.begin(), td.end());
    put_be32(out, crc32_of(td.data(), td.size()) ^ 0xffffffffu);
}

// 8-bit RGBA PNG, (int)(v * 255.0) clamped to [0, 255], alpha 255 (as the
// reference fills its buffer); the zlib stream uses stored deflate blocks.
static bool write_png(const char *path, const float *rgb, int w, int h) {
    std::vector<uint8_t> raw;
    raw.reserve((size_t)h * (1 + 4 * (size_t)w));
    for (int y = 0; y < h; ++y) {
        raw.push_back(0);                              // filter: none
        for (int x = 0; x < w; ++x) {
            const float *px = rgb + 3 * ((size_t)y * w + x);
            for (int c = 0; c < 3; ++c) {
                int v = (int)(px[c] * 255.0);
                raw.push_back((uint8_t)std::max(std::min(v, 255), 0));
            }
            raw.push_back(255);
        }
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    size_t off = 0;
    do {
        const size_t n = std::min<size_t>(65535, raw.size() - off);
        z.push_back(off + n == raw.size() ? 1 : 0);
        z.push_back(n & 0xff); z.push_back(n >> 8);
        z.push_back(~n & 0xff); z.push_back((~n >> 8) & 0xff);
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + n);
        off += n;
    } while (off < raw.size());
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) { a = (a + c) % 65521u; b = (b + a) % 65521u; }
    put_be32(z, (b << 16) | a);
    std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, w); put_be32(ihdr, h);
    ihdr.push_back(8); ihdr.push_back(6); ihdr.push_back(0); ihdr.push_back(0); ihdr.push_back(0);
    png_chunk(out, "IHDR", ihdr);
    png_chunk(out, "IDAT", z);
    png_chunk(out, "IEND", {});
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return std::fclose(f) == 0 && ok;
}

template <typename T> static void put_le(std::vector<uint8_t> &v, T x) {
    uint8_t b[sizeof(T)];
    std::memcpy(b, &x, sizeof(T));
    v.insert(v.end(), b, b + sizeof(T));
}

static void exr_attr(std::vector<uint8_t> &v, const char *name, const char *type, const std::vector<uint8_t> &val) {
    v.insert(v.end(), name, name + std::strlen(name) + 1);
    v.insert(v.end(), type, type + std::strlen(type) + 1);
    put_le<int32_t>(v, (int32_t)val.size());
    v.insert(v.end(), val.begin(), val.end());
}

// Single-part scanline OpenEXR, channels B, G, R as 32-bit float (the
// reference's channel set and order), no compression, one scanline per block.
static bool write_exr(const char *path, const float *rgb, int w, int h) {
    std::vector<uint8_t> v;
    put_le<uint32_t>(v, 20000630u);                    // magic 76 2f 31 01
    put_le<uint32_t>(v, 2u);                           // version 2, single-part scanline
    std::vector<uint8_t> ch;
    for (const char *n : {"B", "G", "R"}) {
        ch.insert(ch.end(), n, n + 2);
        put_le<int32_t>(ch, 2);                        // FLOAT
        ch.push_back(0); ch.push_back(0); ch.push_back(0); ch.push_back(0);
        put_le<int32_t>(ch, 1); put_le<int32_t>(ch, 1);
    }
    ch.push_back(0);
    exr_attr(v, "channels", "chlist", ch);
    exr_attr(v, "compression", "compression", {0});
    std::vector<uint8_t> box;
    put_le<int32_t>(box, 0); put_le<int32_t>(box, 0); put_le<int32_t>(box, w - 1); put_le<int32_t>(box, h - 1);
    exr_attr(v, "dataWindow", "box2i", box);
    exr_attr(v, "displayWindow", "box2i", box);
    exr_attr(v, "lineOrder", "lineOrder", {0});
    std::vector<uint8_t> one;
    put_le<float>(one, 1.0f);
    exr_attr(v, "pixelAspectRatio", "float", one);
    std::vector<uint8_t> ctr;
    put_le<float>(ctr, 0.0f); put_le<float>(ctr, 0.0f);
    exr_attr(v, "screenWindowCenter", "v2f", ctr);
    exr_attr(v, "screenWindowWidth", "float", one);
    v.push_back(0);
    const size_t table = v.size();
    const size_t line = 8 + 3 * 4 * (size_t)w;
    for (int y = 0; y < h; ++y) put_le<uint64_t>(v, (uint64_t)(table + 8 * (size_t)h + line * y));
    for (int y = 0; y < h; ++y) {
        put_le<int32_t>(v, y);
        put_le<int32_t>(v, (int32_t)(3 * 4 * w));
        for (int c : {2, 1, 0})
            for (int x = 0; x < w; ++x) put_le<float>(v, rgb[3 * ((size_t)y * w + x) + c]);
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v.data(), 1, v.size(), f) == v.size();
    return std::fclose(f) == 0 && ok;
}

// ASCII P3 with int(255.99 * v) per channel, unclamped (the reference's PPM).
static bool write_ppm(const char *path, const float *rgb, int w, int h) {
    FILE *f = std::fopen(path, "w");
    if (!f) return false;
    std::fprintf(f, "P3\n%d %d\n255\n", w, h);
    for (size_t i = 0; i < (size_t)w * h; ++i)
        std::fprintf(f, "%d %d %d\n", (int)(255.99 * rgb[3 * i]), (int)(255.99 * rgb[3 * i + 1]),
                     (int)(255.99 * rgb[3 * i + 2]));
    return std::fclose(f) == 0;
}

extern "C" {

const char *blz_render_last_error(const blz_renderer *r) { return r ? r->err.c_str() : g_render_err.c_str(); }

int blz_render_create(const blz_render_params *rp, const blz_params *grid, blz_renderer **out) {
    if (!rp || !grid || !out) return rfail(nullptr, BLZ_ERR_ARG, "null argument");
    *out = nullptr;
    if (grid->width < 4 || grid->height < 4 || grid->depth < 4)
        return rfail(nullptr, BLZ_ERR_ARG, "grid dims must be >= 4 (got %d x %d x %d)", grid->width, grid->height,
                     grid->depth);
    if (rp->width < 1 || rp->height < 1 || (long long)rp->width * rp->height > (1LL << 28))
        return rfail(nullptr, BLZ_ERR_ARG, "bad render resolution %d x %d", rp->width, rp->height);
    if (!(rp->p_step > 0.0f) || !(rp->s_step > 0.0f) || !(grid->dx > 0.0f))
        return rfail(nullptr, BLZ_ERR_ARG, "primary and shadow steps and dx must be positive");
    if (rp->ramp_size < 1 || rp->ramp_size > BLZ_MAX_RAMP)
        return rfail(nullptr, BLZ_ERR_ARG, "ramp_size must be 1..%d (got %d)", BLZ_MAX_RAMP, rp->ramp_size);
    if (rp->light_count < 0 || rp->light_count > BLZ_MAX_LIGHTS)
        return rfail(nullptr, BLZ_ERR_ARG, "light_count must be 0..%d (got %d)", BLZ_MAX_LIGHTS, rp->light_count);
    if (rp->multi_scatter_blur_iter < 0) return rfail(nullptr, BLZ_ERR_ARG, "negative multi_scatter_blur_iter");
    blz_renderer *r = new blz_renderer();
    r->rp = *rp;
    r->W = grid->width; r->H = grid->height; r->D = grid->depth;
    r->SW = r->W / kScatterRatio; r->SH = r->H / kScatterRatio; r->SD = r->D / kScatterRatio;
    cudaGetDevice(&r->device);
    RenderArgs &a = r->a;
    a.res_x = rp->width; a.res_y = rp->height;
    a.cam_o = v3(rp->cam_trans); a.cam_u = v3(rp->cam_u); a.cam_v = v3(rp->cam_v); a.cam_w = v3(rp->cam_w);
    a.focal = rp->cam_focal; a.aperture = rp->cam_aperture;
    a.dx = grid->dx;
    a.dmin = v3(grid->domain_min); a.dmax = v3(grid->domain_max);
    a.dsize = make_float3(a.dmax.x - a.dmin.x, a.dmax.y - a.dmin.y, a.dmax.z - a.dmin.z);
    a.p_step = rp->p_step; a.s_step = rp->s_step; a.cutoff = rp->cutoff;
    a.density_scale = rp->density_scale; a.shadow_density_scale = rp->shadow_density_scale;
    a.absorption = rp->absorption;
    a.scattering = v3(rp->scattering); a.volume_color = v3(rp->volume_color);
    a.gain = rp->gain; a.emission_scale = rp->emission_scale;
    a.t_in = rp->temp_range[0]; a.t_out = rp->temp_range[1];
    a.ramp_n = rp->ramp_size;
    for (int i = 0; i < rp->ramp_size; ++i) { a.ramp_keys[i] = rp->ramp_keys[i]; a.ramp_colors[i] = v3(rp->ramp_colors[i]); }
    a.ms_scale = rp->multi_scatter_scale;
    a.ms_mask0 = rp->multi_scatter_density_mask[0]; a.ms_mask1 = rp->multi_scatter_density_mask[1];
    a.ms_color = v3(rp->multi_scatter_color);
    a.n_lights = rp->light_count;
    for (int l = 0; l < rp->light_count; ++l) {
        a.l_dir[l] = v3(rp->light_dir[l]); a.l_color[l] = v3(rp->light_color[l]);
        a.l_intensity[l] = rp->light_intensity[l]; a.l_exposure[l] = rp->light_exposure[l];
    }
    // Step bounds: a ray inside the box covers at most its diagonal.
    const double diag = std::sqrt((double)a.dsize.x * a.dsize.x + (double)a.dsize.y * a.dsize.y +
                                  (double)a.dsize.z * a.dsize.z);
    a.max_p_steps = (int)std::min(1e8, std::ceil(diag / rp->p_step) + 16.0);
    a.max_s_steps = (int)std::min(1e8, std::ceil(diag / rp->s_step) + 16.0);
    a.mW = (r->W + kMacro - 1) / kMacro; a.mH = (r->H + kMacro - 1) / kMacro; a.mD = (r->D + kMacro - 1) / kMacro;
    // A filtered sample is a convex combination of the texels under it (its
    // corner weights are multiples of 1/256 that sum to one), so it is at most
    // the cell maximum; the 1e-4 margin covers the rounding of the sums.
    const float ds = rp->density_scale, dss = rp->density_scale * rp->shadow_density_scale;
    a.skip_p = ds > 0.0f ? rp->cutoff / (ds * 1.0001f) : -INFINITY;
    a.skip_s = dss > 0.0f ? rp->cutoff / (dss * 1.0001f) : -INFINITY;

    int rc = BLZ_OK;
    auto step = [&](cudaError_t e, const char *what) {
        if (rc == BLZ_OK && e != cudaSuccess) rc = rfail(r, BLZ_ERR_CUDA, "%s failed: %s", what, cudaGetErrorString(e));
    };
    step(cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking), "cudaStreamCreate");
    r->own_stream = r->st != nullptr;
    if (rc == BLZ_OK) rc = make_volume(r, r->W, r->H, r->D, &r->t_arr, &r->t_tex);
    if (rc == BLZ_OK) rc = make_volume(r, r->SW, r->SH, r->SD, &r->s_arr, &r->s_tex);
    const size_t sn = (size_t)r->SW * r->SH * r->SD;
    step(cudaMalloc(&r->s_buf[0], sn * sizeof(float)), "cudaMalloc(scatter)");
    step(cudaMalloc(&r->s_buf[1], sn * sizeof(float)), "cudaMalloc(scatter)");
    step(cudaMalloc(&r->fb, (size_t)3 * rp->width * rp->height * sizeof(float)), "cudaMalloc(frame buffer)");
    step(cudaMalloc(&r->tables, sizeof(Tables)), "cudaMalloc(tables)");
    step(cudaMalloc(&r->macro, (size_t)a.mW * a.mH * a.mD * sizeof(float)), "cudaMalloc(empty-space cells)");
    if (rc == BLZ_OK) rc = make_volume(r, a.mW, a.mH, a.mD, &r->m_arr, &r->m_tex, cudaFilterModePoint);
    if (rc == BLZ_OK) {
        k_tables_setup<<<1, 1, 0, r->st>>>(r->a, r->tables);
        step(cudaGetLastError(), "k_tables_setup");
        r->launches += 1;
    }
    step(cudaEventCreate(&r->e0), "cudaEventCreate");
    step(cudaEventCreate(&r->e1), "cudaEventCreate");
    // The scatter volume starts at zero (it is read, times a zero scale, when
    // multiple scattering is off).
    if (rc == BLZ_OK) step(cudaMemsetAsync(r->s_buf[0], 0, sn * sizeof(float), r->st), "cudaMemsetAsync");
    if (rc == BLZ_OK) rc = copy_to_volume(r, r->s_buf[0], r->SW, r->SH, r->SD, r->s_arr);
    if (rc == BLZ_OK) {
        float w[27], sum = 0.0f;
        for (float k : kBlurKernel) sum += k;
        for (int i = 0; i < 27; ++i) w[i] = kBlurKernel[i] / sum;
        step(cudaMemcpyToSymbolAsync(c_blur_w, w, sizeof w, 0, cudaMemcpyHostToDevice, r->st), "cudaMemcpyToSymbol");
    }
    if (rc == BLZ_OK) step(cudaStreamSynchronize(r->st), "cudaStreamSynchronize");
    if (rc != BLZ_OK) {
        g_render_err = r->err;
        render_release(r);
        delete r;
        return rc;
    }
    *out = r;
    return BLZ_OK;
}

int blz_render_destroy(blz_renderer *r) {
    if (!r) return BLZ_OK;
    if (r->st) cudaStreamSynchronize(r->st);
    render_release(r);
    delete r;
    return BLZ_OK;
}

int blz_render_set_stream(blz_renderer *r, void *cuda_stream) {
    if (!r) return rfail(nullptr, BLZ_ERR_ARG, "null renderer");
    RCK(r, cudaStreamSynchronize(r->st));
    if (r->own_stream) cudaStreamDestroy(r->st);
    r->st = static_cast<cudaStream_t>(cuda_stream);
    r->own_stream = false;
    return BLZ_OK;
}

int blz_render(blz_renderer *r, const float *temp) {
    if (!r || !temp) return rfail(r, BLZ_ERR_ARG, "null argument");
    RCK(r, cudaEventRecord(r->e0, r->st));
    int rc = copy_to_volume(r, temp, r->W, r->H, r->D, r->t_arr);
    if (rc != BLZ_OK) return rc;
    if (r->a.ms_scale > 0.0f) {
        const dim3 b(8, 8, 8);
        const dim3 g((r->SW + 7) / 8, (r->SH + 7) / 8, (r->SD + 7) / 8);
        k_scatter_down<<<g, b, 0, r->st>>>(temp, r->W, r->H, r->SW, r->SH, r->SD, r->rp.temp_range[0], r->s_buf[0]);
        int cur = 0;
        for (int it = 0; it < r->rp.multi_scatter_blur_iter; ++it) {
            k_scatter_blur<<<g, b, 0, r->st>>>(r->s_buf[cur], r->SW, r->SH, r->SD, r->s_buf[cur ^ 1]);
            cur ^= 1;
        }
        RCK(r, cudaGetLastError());
        r->launches += 1 + r->rp.multi_scatter_blur_iter;
        rc = copy_to_volume(r, r->s_buf[cur], r->SW, r->SH, r->SD, r->s_arr);
        if (rc != BLZ_OK) return rc;
    }
    const int nm = r->a.mW * r->a.mH * r->a.mD;
    k_macro_max<<<(nm + 127) / 128, 128, 0, r->st>>>(temp, r->W, r->H, r->D, r->a.mW, r->a.mH, r->a.mD, r->macro);
    RCK(r, cudaGetLastError());
    rc = copy_to_volume(r, r->macro, r->a.mW, r->a.mH, r->a.mD, r->m_arr);
    if (rc != BLZ_OK) return rc;
    const dim3 b(8, 8, 1);
    const dim3 g((r->a.res_x + 7) / 8, (r->a.res_y + 7) / 8, 1);
    k_render<<<g, b, 0, r->st>>>(r->a, r->t_tex, r->s_tex, r->m_tex, r->tables, r->fb);
    RCK(r, cudaGetLastError());
    r->launches += 2;
    RCK(r, cudaEventRecord(r->e1, r->st));
    RCK(r, cudaEventSynchronize(r->e1));
    RCK(r, cudaEventElapsedTime(&r->last_ms, r->e0, r->e1));
    return BLZ_OK;
}

int blz_render_solver(blz_renderer *r, blz_solver *s) {
    if (!r || !s) return rfail(r, BLZ_ERR_ARG, "null argument");
    const blz_params *P = solver_params(s);
    if (P->width != r->W || P->height != r->H || P->depth != r->D)
        return rfail(r, BLZ_ERR_ARG, "solver grid %d x %d x %d differs from the renderer's %d x %d x %d", P->width,
                     P->height, P->depth, r->W, r->H, r->D);
    RCK(r, cudaStreamSynchronize(solver_stream(s)));
    return blz_render(r, static_cast<const float *>(blz_field_ptr(s, BLZ_FIELD_T)));
}

int blz_render_get_image(const blz_renderer *r, float *rgb, int on_device) {
    blz_renderer *m = const_cast<blz_renderer *>(r);
    if (!r || !rgb) return rfail(m, BLZ_ERR_ARG, "null argument");
    const size_t n = (size_t)3 * r->a.res_x * r->a.res_y * sizeof(float);
    RCK(m, cudaMemcpyAsync(rgb, r->fb, n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->st));
    RCK(m, cudaStreamSynchronize(r->st));
    return BLZ_OK;
}

static int image_write(blz_renderer *r, const char *path, const float *rgb, int w, int h) {
    if (!path || !rgb || w < 1 || h < 1) return rfail(r, BLZ_ERR_ARG, "bad image arguments");
    const std::string p(path);
    const std::string ext = p.size() >= 4 ? p.substr(p.size() - 4) : std::string();
    if (ext != ".ppm" && ext != ".png" && ext != ".exr")
        return rfail(r, BLZ_ERR_ARG, "unknown image format of '%s' (.ppm, .png or .exr)", path);
    const bool ok = ext == ".ppm" ? write_ppm(path, rgb, w, h)
                  : ext == ".png" ? write_png(path, rgb, w, h)
                                  : write_exr(path, rgb, w, h);
    if (!ok) return rfail(r, BLZ_ERR_ARG, "cannot write '%s'", path);
    return BLZ_OK;
}

int blz_image_write(const char *path, const float *rgb, int width, int height) {
    return image_write(nullptr, path, rgb, width, height);
}

int blz_render_write(const blz_renderer *r, const char *path) {
    blz_renderer *m = const_cast<blz_renderer *>(r);
    if (!r || !path) return rfail(m, BLZ_ERR_ARG, "null argument");
    std::vector<float> rgb((size_t)3 * r->a.res_x * r->a.res_y);
    int rc = blz_render_get_image(r, rgb.data(), 0);
    if (rc != BLZ_OK) return rc;
    return image_write(m, path, rgb.data(), r->a.res_x, r->a.res_y);
}

float blz_render_last_ms(const blz_renderer *r) { return r ? r->last_ms : 0.0f; }

long long blz_render_kernel_launches(const blz_renderer *r) { return r ? r->launches : 0; }

int blz_render_sample_temp(blz_renderer *r, const float *temp, const float *pos3, int n, float *out) {
    if (!r || !temp || !pos3 || !out || n < 0) return rfail(r, BLZ_ERR_ARG, "null argument");
    if (n == 0) return BLZ_OK;
    int rc = copy_to_volume(r, temp, r->W, r->H, r->D, r->t_arr);
    if (rc != BLZ_OK) return rc;
    k_sample<<<(n + 255) / 256, 256, 0, r->st>>>(r->t_tex, pos3, n, out);
    RCK(r, cudaGetLastError());
    r->launches += 1;
    RCK(r, cudaStreamSynchronize(r->st));
    return BLZ_OK;
}

} // extern "C"
