// render_oracle.cpp — CPU oracle of Blaze's volume renderer.
//
// TEST INFRASTRUCTURE ONLY: loaded by the tests as the checker of the CUDA
// renderer (blaze_b200/csrc/render.cu), never by the product path.
//
// It restates, in plain single-threaded-per-pixel C++ (OpenMP over pixels),
// the reference's render pass (asiroisvigneux/Blaze src/RenderEngine.cu:
// 50-231 with Camera.h:41-60, Shader.h:53-71, Light.h:37-54, Ray.h:32-45,
// ColorRamp.h:57-79 and Grid.h:292-296) in FP32, the reference's type.
//
// The one piece the reference leaves to hardware is the texture sampler:
// tex3D<float> with linear filtering, clamped addressing and unnormalised
// coordinates (Volume.h:46-58).  CUDA documents it as trilinear
// interpolation between the texels around (x - 0.5, y - 0.5, z - 0.5) with
// the fractional weights held in 9-bit fixed point (8 fractional bits) and
// indices clamped to the volume.  tex_sample restates that in FP64 with the
// weight rule selectable (`quant`):
//   0  each axis fraction rounded to the nearest 1/256, weights multiplied
//      exactly;
//   1  each axis fraction truncated to 1/256;
//   2  exact fractions;
//   3  the rule measured on B200 texture units with in-bounds probes
//      (tests/test_gpu_render.py): each axis fraction rounded half up to
//      1/256; the eight corner weights are themselves multiples of 1/256 and
//      sum to exactly one: w_xz = round(wx * wz) per x-z corner, then
//      round(w_xz * wy) for the upper y corner and the rest of w_xz for the
//      lower; coordinates clamped to the texel-centre range first.  This
//      reproduces 99 % of the hardware's corner weights exactly; the others
//      differ by one 1/256 unit, so a sample is within 2 max|T| / 256.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/blaze_b200.h"

namespace {

struct V3 {
    float x, y, z;
};
inline V3 v3(float a, float b, float c) { return {a, b, c}; }
inline V3 v3p(const float *p) { return {p[0], p[1], p[2]}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float sqlen(V3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
inline V3 expv(V3 a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }

struct Volume {
    const float *a;
    int w, h, d;
    float at(int i, int j, int k) const {
        i = std::min(std::max(i, 0), w - 1);
        j = std::min(std::max(j, 0), h - 1);
        k = std::min(std::max(k, 0), d - 1);
        return a[(size_t)i + (size_t)w * ((size_t)j + (size_t)h * k)];
    }
};

double quantise(double f, int quant) {
    if (quant == 0) return std::nearbyint(f * 256.0) / 256.0;
    if (quant == 1) return std::floor(f * 256.0) / 256.0;
    return f;
}

float tex_sample_hw(const Volume &v, float x, float y, float z) {
    auto frac = [](double c, int n, int &i0) {
        c = std::min(std::max(c, 0.5), n - 0.5) - 0.5;
        const double f = std::floor(c);
        i0 = (int)f;
        return std::floor((c - f) * 256.0 + 0.5);      // 0..256
    };
    int i, j, k;
    const double a = frac(x, v.w, i), b = frac(y, v.h, j), c = frac(z, v.d, k);
    double s = 0.0;
    for (int dx = 0; dx < 2; ++dx)
        for (int dz = 0; dz < 2; ++dz) {
            const double wxz = std::floor((dx ? a : 256.0 - a) * (dz ? c : 256.0 - c) / 256.0 + 0.5);
            const double w1 = std::floor(wxz * b / 256.0 + 0.5);
            s += w1 / 256.0 * v.at(i + dx, j + 1, k + dz) + (wxz - w1) / 256.0 * v.at(i + dx, j, k + dz);
        }
    return (float)s;
}

float tex_sample(const Volume &v, float x, float y, float z, int quant) {
    if (quant == 3) return tex_sample_hw(v, x, y, z);
    const double xb = (double)x - 0.5, yb = (double)y - 0.5, zb = (double)z - 0.5;
    const double fi = std::floor(xb), fj = std::floor(yb), fk = std::floor(zb);
    const int i = (int)fi, j = (int)fj, k = (int)fk;
    const double a = quantise(xb - fi, quant), b = quantise(yb - fj, quant), c = quantise(zb - fk, quant);
    double s = 0.0;
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                const double w = (di ? a : 1.0 - a) * (dj ? b : 1.0 - b) * (dk ? c : 1.0 - c);
                s += w * v.at(i + di, j + dj, k + dk);
            }
    return (float)s;
}

struct Ray {
    V3 o, d, inv;
    int sx, sy, sz;
    float t0, t1;
};

Ray make_ray(V3 o, V3 d) {
    Ray r;
    r.o = o;
    r.d = d;
    r.inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    r.sx = r.inv.x < 0.0f; r.sy = r.inv.y < 0.0f; r.sz = r.inv.z < 0.0f;
    r.t0 = 0.0f;
    r.t1 = INFINITY;
    return r;
}

// RenderEngine.cu:119-157
bool box_hit(Ray &r, V3 lo, V3 hi) {
    const V3 b[2] = {lo, hi};
    float tmin = (b[r.sx].x - r.o.x) * r.inv.x;
    float tmax = (b[1 - r.sx].x - r.o.x) * r.inv.x;
    const float tymin = (b[r.sy].y - r.o.y) * r.inv.y;
    const float tymax = (b[1 - r.sy].y - r.o.y) * r.inv.y;
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    const float tzmin = (b[r.sz].z - r.o.z) * r.inv.z;
    const float tzmax = (b[1 - r.sz].z - r.o.z) * r.inv.z;
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    r.t0 = std::max(tmin, 0.0f);
    r.t1 = tmax;
    return !(r.t1 < 0.0f);
}

// ColorRamp.h:57-79
V3 ramp_color(const blz_render_params &rp, float temp) {
    const float x = std::min(std::max((temp - rp.temp_range[0]) / (rp.temp_range[1] - rp.temp_range[0]), 0.0f), 1.0f);
    if (rp.ramp_size == 1) return v3p(rp.ramp_colors[0]);
    int prev = 0, next = 0;
    for (int i = 0; i < rp.ramp_size; ++i) {
        if (rp.ramp_keys[i] <= x) {
            prev = i;
        } else {
            next = i;
            break;
        }
    }
    const float range = rp.ramp_keys[next] - rp.ramp_keys[prev];
    const float blend = (x - rp.ramp_keys[prev]) / range;
    const V3 a = v3p(rp.ramp_colors[prev]), b = v3p(rp.ramp_colors[next]);
    return a + blend * (b - a);
}

float smooth_step(float e0, float e1, float x) {
    const float y = std::max(0.0f, std::min((x - e0) / (e1 - e0), 1.0f));
    return y * y * (3.0f - (2.0f * y));
}

} // namespace

extern "C" {

void orc_tex_sample(const float *T, int W, int H, int D, const float *pos3, int n, float *out, int quant) {
    const Volume v{T, W, H, D};
    for (int t = 0; t < n; ++t) out[t] = tex_sample(v, pos3[3 * t], pos3[3 * t + 1], pos3[3 * t + 2], quant);
}

// The whole render pass into rgb (width*height*3, row 0 at the top).
void orc_render(const blz_render_params *rpp, const blz_params *grid, const float *T, float *rgb, int quant) {
    const blz_render_params &rp = *rpp;
    const int W = grid->width, H = grid->height, D = grid->depth;
    const Volume tv{T, W, H, D};
    // multiple-scattering volume (RenderEngine.cu:50-97, 320-345)
    const int SW = W / 4, SH = H / 4, SD = D / 4;
    std::vector<float> sc((size_t)SW * SH * SD, 0.0f), tmp(sc.size());
    if (rp.multi_scatter_scale > 0.0f) {
        for (int k = 0; k < SD; ++k)
            for (int j = 0; j < SH; ++j)
                for (int i = 0; i < SW; ++i) {
                    float acc = 0.0f;
                    for (int io = 0; io < 4; ++io)
                        for (int jo = 0; jo < 4; ++jo)
                            for (int ko = 0; ko < 4; ++ko) {
                                const float t = tv.at(4 * i + io, 4 * j + jo, 4 * k + ko);
                                acc += t > rp.temp_range[0] ? t : 0.0f;
                            }
                    sc[(size_t)i + (size_t)SW * (j + (size_t)SH * k)] = acc / 64.0f;
                }
        const float kern[27] = {0, 1, 0, 1, 2, 1, 0, 1, 0, 1, 2, 1, 2, 4, 2, 1, 2, 1, 0, 1, 0, 1, 2, 1, 0, 1, 0};
        float sum = 0.0f, w[27];
        for (float x : kern) sum += x;
        for (int i = 0; i < 27; ++i) w[i] = kern[i] / sum;
        for (int it = 0; it < rp.multi_scatter_blur_iter; ++it) {
            const Volume sv{sc.data(), SW, SH, SD};
            for (int k = 0; k < SD; ++k)
                for (int j = 0; j < SH; ++j)
                    for (int i = 0; i < SW; ++i) {
                        float acc = 0.0f;
                        int idx = 0;
                        for (int dk = -1; dk <= 1; ++dk)
                            for (int dj = -1; dj <= 1; ++dj)
                                for (int di = -1; di <= 1; ++di, ++idx)
                                    acc += sv.at(i + di, j + dj, k + dk) * w[idx];
                        tmp[(size_t)i + (size_t)SW * (j + (size_t)SH * k)] = acc;
                    }
            sc.swap(tmp);
        }
    }
    const Volume sv{sc.data(), SW, SH, SD};
    const V3 dmin = v3p(grid->domain_min), dmax = v3p(grid->domain_max), dsize = dmax - dmin;
    const float dx = grid->dx;
    const V3 cam_o = v3p(rp.cam_trans), cu = v3p(rp.cam_u), cv = v3p(rp.cam_v), cw = v3p(rp.cam_w);
    const float aspect = (float)rp.width / (float)rp.height;
    const float half_w = 0.5f * rp.cam_aperture, half_h = half_w / aspect;
    const V3 top_left = cam_o - rp.cam_focal * cw - half_w * cu + half_h * cv;
    const V3 horiz = 2.0f * half_w * cu, vert = -2.0f * half_h * cv;
    const V3 absv = v3(rp.absorption, rp.absorption, rp.absorption);
    const V3 scat = v3p(rp.scattering), vcol = v3p(rp.volume_color);
    const V3 albedo = (vcol * scat) / (scat + absv), ext = (scat + absv) * -1.0f, one = v3(1, 1, 1);
    auto w2g = [&](V3 p) { return v3((p.x - dmin.x) / dx, (dsize.y - (p.y - dmin.y)) / dx, (p.z - dmin.z) / dx); };
    const double diag = std::sqrt((double)dsize.x * dsize.x + (double)dsize.y * dsize.y + (double)dsize.z * dsize.z);
    const long max_p = (long)std::ceil(diag / rp.p_step) + 16, max_s = (long)std::ceil(diag / rp.s_step) + 16;
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 0; j < rp.height; ++j)
        for (int i = 0; i < rp.width; ++i) {
            float *out = rgb + 3 * ((size_t)i + (size_t)rp.width * j);
            out[0] = out[1] = out[2] = 0.0f;
            const V3 v = top_left + ((i + 0.5f) / rp.width) * horiz + ((j + 0.5f) / rp.height) * vert - cam_o;
            const V3 dir = v * (1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z));
            Ray pr = make_ray(cam_o, dir);
            if (!box_hit(pr, dmin, dmax)) continue;
            V3 lumi = v3(0, 0, 0), trans = v3(1, 1, 1);
            long np = 0;
            for (float pt = pr.t0 + dx * 0.5f; pt <= pr.t1 && np < max_p; pt += rp.p_step, ++np) {
                const V3 ppos = pr.o + pt * pr.d;
                const V3 pg = w2g(ppos);
                const float temp = tex_sample(tv, pg.x, pg.y, pg.z, quant);
                const float sct = tex_sample(sv, pg.x / 4.0f, pg.y / 4.0f, pg.z / 4.0f, quant);
                const float density = temp * rp.density_scale;
                if (density < rp.cutoff) continue;
                V3 emission = v3(0, 0, 0);
                if (rp.emission_scale > 0.0f)
                    emission = ramp_color(rp, temp) * rp.emission_scale +
                               v3p(rp.multi_scatter_color) * sct * rp.multi_scatter_scale *
                                   smooth_step(rp.multi_scatter_density_mask[0], rp.multi_scatter_density_mask[1], temp);
                const V3 dT = expv(ext * density * rp.p_step);
                for (int l = 0; l < rp.light_count; ++l) {
                    const V3 illum = v3p(rp.light_color[l]) * rp.light_intensity[l] * std::pow(2.0f, rp.light_exposure[l]);
                    Ray sr = make_ray(ppos, -1.0f * v3p(rp.light_dir[l]));
                    box_hit(sr, dmin, dmax);
                    V3 st_tr = v3(1, 1, 1);
                    long ns = 0;
                    for (float st = sr.t0 + dx * 0.5f; st <= sr.t1 && ns < max_s; st += rp.s_step, ++ns) {
                        const V3 sg = w2g(sr.o + st * sr.d);
                        const float sd = tex_sample(tv, sg.x, sg.y, sg.z, quant) * rp.density_scale * rp.shadow_density_scale;
                        if (sd < rp.cutoff) continue;
                        st_tr = st_tr * expv(ext * sd * rp.s_step / (1.0f + st * rp.gain));
                        if (sqlen(st_tr) < rp.cutoff) break;
                    }
                    lumi = lumi + albedo * st_tr * trans * illum * (one - dT);
                }
                lumi = lumi + trans * emission * (one - dT);
                trans = trans * dT;
                if (sqlen(trans) < rp.cutoff) break;
            }
            out[0] = lumi.x;
            out[1] = lumi.y;
            out[2] = lumi.z;
        }
}

} // extern "C"
