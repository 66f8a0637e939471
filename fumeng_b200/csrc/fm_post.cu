// Post-processing of a finished frame on the device: the reference's PostProcess chain
// (core/renderer.h:131-135) and the 8-bit conversion its RenderTarget::save_to_file does
// before the PNG write (render_target.h:26-31, image/image.cpp:98-109).
//
// Per-pixel steps (tone mapping, linear <-> sRGB) run as one kernel per run of
// consecutive per-pixel steps; the denoise step is an image-level filter between them.
// The arithmetic of the per-pixel steps is the reference's float build's: every
// operation explicitly rounded in the reference's order (no multiply-add is contracted),
// pow from the device's powf.  So the 8-bit outputs equal the reference's bytes for the
// same float input, up to the last bit of powf on the sRGB steps (a value whose
// 255 x lands within one float ulp of a rounding boundary can then differ by one code).
//
// Denoise: the reference calls Intel Open Image Denoise's "RT" filter with the albedo and
// normal images as guides (post/oidn_denoise.cpp:36-78).  That filter is a trained
// network that is not available here; this file runs a different, non-learned filter on
// the same inputs instead: the edge-avoiding a-trous wavelet filter (Dammertz, Sewtz,
// Hanika and Lensch, "Edge-Avoiding A-Trous Wavelet Transform for fast Global
// Illumination Filtering", HPG 2010), five passes of a 5x5 B3-spline kernel with taps
// 1, 2, 4, 8, 16 pixels apart, each tap weighted by its colour, normal and albedo
// distance to the centre.  Its output is not the reference's.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

namespace {

constexpr int kMaxPostSteps = 16;

struct PostChain {
    int n;
    int type[kMaxPostSteps];
    float lum[kMaxPostSteps];
};

// ToneMapping::FilmicCore (post/tonemapping.cpp:10-19), float, in the source's order.
FM_D float filmic_core(float x)
{
    const float A = 0.22f, B = 0.30f, C = 0.10f, D = 0.20f, E = 0.01f, F = 0.30f;
    const float num = __fadd_rn(__fmul_rn(x, __fadd_rn(__fmul_rn(A, x), __fmul_rn(C, B))), __fmul_rn(D, E));
    const float den = __fadd_rn(__fmul_rn(x, __fadd_rn(__fmul_rn(A, x), B)), __fmul_rn(D, F));
    return __fsub_rn(__fdiv_rn(num, den), __fdiv_rn(E, F));
}

// ToneMapping::Filmic (:21-25): FilmicCore(1.6 * value * lum) / FilmicCore(11.2).
FM_D float filmic(float v, float lum, float white)
{
    return __fdiv_rn(filmic_core(__fmul_rn(__fmul_rn(1.6f, v), lum)), white);
}

// LinearToSrgb / SrgbToLinear (core/utils.h:120-132), float.
FM_D float linear_to_srgb(float c)
{
    if (c <= 0.0031308f) return __fmul_rn(12.92f, c);
    return __fsub_rn(__fmul_rn(1.055f, powf(c, __fdiv_rn(1.0f, 2.4f))), 0.055f);
}

FM_D float srgb_to_linear(float c)
{
    if (c <= 0.04045f) return __fdiv_rn(__fmul_rn(c, 1.0f), 12.92f);
    return powf(__fdiv_rn(__fmul_rn(__fadd_rn(c, 0.055f), 1.0f), 1.055f), 2.4f);
}

__global__ void k_post_pointwise(float* __restrict__ rgb, int64_t n, PostChain chain, int first, int last)
{
    const float white = filmic_core(11.2f);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = rgb[i];
        for (int s = first; s < last; ++s) {
            if (chain.type[s] == FM_POST_TONEMAP)
                v = filmic(v, chain.lum[s], white);
            else if (chain.type[s] == FM_POST_LINEAR_TO_SRGB)
                v = linear_to_srgb(v);
            else if (chain.type[s] == FM_POST_SRGB_TO_LINEAR)
                v = srgb_to_linear(v);
        }
        rgb[i] = v;
    }
}

// RealToUInt8 (core/utils.h:134-137): Clamp(c, 0, 1) (utils.h:68-71), then
// round(255 c).  A NaN channel (left unchanged by the reference's Clamp, and undefined
// in its integer conversion) becomes 0.
__global__ void k_to_u8(const float* __restrict__ src, uint8_t* __restrict__ dst, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float c = src[i];
        c = c > 1.0f ? 1.0f : (c < 0.0f ? 0.0f : c);
        dst[i] = c == c ? (uint8_t)roundf(__fmul_rn(255.0f, c)) : (uint8_t)0;
    }
}

// One pass of the edge-avoiding a-trous filter at tap distance `step` (pixels).
// Weights: B3-spline h(dx) h(dy) with h = (1, 4, 6, 4, 1) / 16, times
//   exp(-|t(c_q) - t(c_p)|^2 / sc^2)          colour, t(c) = c / (1 + c) per channel
//   exp(-max(0, 1 - n_p . n_q) / sn^2)         normal (unit-normalised AOV means)
//   exp(-|a_q - a_p|^2 / sa^2)                 albedo
// with the colour scale halved at every pass (the finer detail has been removed).
__global__ void k_atrous(const float* __restrict__ in, float* __restrict__ out, const float* __restrict__ alb,
                         const float* __restrict__ nrm, int w, int h, int step, float sc, float sn, float sa)
{
    const float hk[5] = {1.0f / 16.0f, 4.0f / 16.0f, 6.0f / 16.0f, 4.0f / 16.0f, 1.0f / 16.0f};
    const int64_t npix = (int64_t)w * h;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % w), y = (int)(p / w);
        const f3 cp = f3{in[3 * p], in[3 * p + 1], in[3 * p + 2]};
        const f3 tp = f3{cp.x / (1.0f + fmaxf(cp.x, 0.0f)), cp.y / (1.0f + fmaxf(cp.y, 0.0f)),
                         cp.z / (1.0f + fmaxf(cp.z, 0.0f))};
        f3 np = f3{nrm[3 * p], nrm[3 * p + 1], nrm[3 * p + 2]};
        const float nl = length(np);
        np = nl > 0.0f ? np / nl : np;
        const f3 ap = f3{alb[3 * p], alb[3 * p + 1], alb[3 * p + 2]};
        f3 sum = mk(0.0f);
        float wsum = 0.0f;
        for (int dy = -2; dy <= 2; ++dy) {
            const int yy = y + dy * step;
            if (yy < 0 || yy >= h) continue;
            for (int dx = -2; dx <= 2; ++dx) {
                const int xx = x + dx * step;
                if (xx < 0 || xx >= w) continue;
                const int64_t q = (int64_t)yy * w + xx;
                const f3 cq = f3{in[3 * q], in[3 * q + 1], in[3 * q + 2]};
                const f3 tq = f3{cq.x / (1.0f + fmaxf(cq.x, 0.0f)), cq.y / (1.0f + fmaxf(cq.y, 0.0f)),
                                 cq.z / (1.0f + fmaxf(cq.z, 0.0f))};
                f3 nq = f3{nrm[3 * q], nrm[3 * q + 1], nrm[3 * q + 2]};
                const float ql = length(nq);
                nq = ql > 0.0f ? nq / ql : nq;
                const f3 aq = f3{alb[3 * q], alb[3 * q + 1], alb[3 * q + 2]};
                const f3 dc = tq - tp, da = aq - ap;
                const float wc = __expf(-dot(dc, dc) / (sc * sc));
                const float wn = __expf(-fmaxf(0.0f, 1.0f - dot(np, nq)) / (sn * sn));
                const float wa = __expf(-dot(da, da) / (sa * sa));
                const float wt = hk[dx + 2] * hk[dy + 2] * wc * wn * wa;
                if (!(wt > 0.0f) || !isfinite(cq.x + cq.y + cq.z)) continue;
                sum += cq * wt;
                wsum += wt;
            }
        }
        const f3 r = wsum > 0.0f ? sum / wsum : cp;
        out[3 * p] = r.x;
        out[3 * p + 1] = r.y;
        out[3 * p + 2] = r.z;
    }
}

}  // namespace

}  // namespace fm

using namespace fm;

extern "C" fm_status fm_postprocess(fm_ctx* ctx, int32_t width, int32_t height, const fm_post_step* steps,
                                    int32_t num_steps, float* rgb, const float* albedo, const float* normal,
                                    uint8_t* rgb8, uint8_t* albedo8, uint8_t* normal8, int32_t flags)
{
    if (!ctx) return FM_ERR_INVALID;
    if (width <= 0 || height <= 0 || (int64_t)width * height > ((int64_t)1 << 30) || num_steps < 0 ||
        num_steps > kMaxPostSteps || (num_steps > 0 && !steps) || !rgb)
        return set_error(ctx, FM_ERR_INVALID, "postprocess: bad arguments");
    PostChain chain{};
    chain.n = num_steps;
    bool denoise = false;
    for (int i = 0; i < num_steps; ++i) {
        const int t = steps[i].type;
        if (t != FM_POST_TONEMAP && t != FM_POST_LINEAR_TO_SRGB && t != FM_POST_SRGB_TO_LINEAR && t != FM_POST_DENOISE)
            return set_error(ctx, FM_ERR_INVALID, "postprocess: unknown step type");
        chain.type[i] = t;
        chain.lum[i] = steps[i].lum;
        denoise = denoise || t == FM_POST_DENOISE;
    }
    if (denoise && (!albedo || !normal))
        return set_error(ctx, FM_ERR_INVALID, "postprocess: the denoise step needs the albedo and normal images");
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = ctx->stream;
    const bool dev = (flags & FM_FLAG_DEVICE_PTRS) != 0;
    const int64_t n = (int64_t)width * height * 3;
    const size_t fbytes = (size_t)n * sizeof(float);
    // device copies when the caller's buffers are host memory, a ping-pong image for the
    // denoiser, and the 8-bit outputs
    const size_t need = (dev ? 0 : 3 * fbytes) + (denoise ? fbytes : 0) + (dev ? 0 : 3 * (size_t)n) + 1024;
    char* tmp = nullptr;
    FM_CUDA_TRY(ctx, cudaMallocAsync((void**)&tmp, need, s), "postprocess alloc");
    char* q = tmp;
    auto take = [&](size_t b) {
        char* r = q;
        q += (b + 255) / 256 * 256;
        return r;
    };
    float* d_rgb = rgb;
    const float* d_alb = albedo;
    const float* d_nrm = normal;
    uint8_t *d_rgb8 = rgb8, *d_alb8 = albedo8, *d_nrm8 = normal8;
    cudaError_t e = cudaSuccess;
    if (!dev) {
        d_rgb = reinterpret_cast<float*>(take(fbytes));
        float* a = albedo ? reinterpret_cast<float*>(take(fbytes)) : nullptr;
        float* nn = normal ? reinterpret_cast<float*>(take(fbytes)) : nullptr;
        e = cudaMemcpyAsync(d_rgb, rgb, fbytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && a) e = cudaMemcpyAsync(a, albedo, fbytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && nn) e = cudaMemcpyAsync(nn, normal, fbytes, cudaMemcpyHostToDevice, s);
        d_alb = a;
        d_nrm = nn;
        d_rgb8 = rgb8 ? reinterpret_cast<uint8_t*>(take((size_t)n)) : nullptr;
        d_alb8 = albedo8 && albedo ? reinterpret_cast<uint8_t*>(take((size_t)n)) : nullptr;
        d_nrm8 = normal8 && normal ? reinterpret_cast<uint8_t*>(take((size_t)n)) : nullptr;
    }
    float* pong = denoise ? reinterpret_cast<float*>(take(fbytes)) : nullptr;
    const int block = 256;
    const int grid = (int)std::min<int64_t>((n + block - 1) / block, (int64_t)ctx->num_sms * 16);
    const int pgrid = (int)std::min<int64_t>(((int64_t)width * height + block - 1) / block, (int64_t)ctx->num_sms * 16);
    int first = 0;
    for (int i = 0; i <= num_steps && e == cudaSuccess; ++i) {
        if (i < num_steps && chain.type[i] != FM_POST_DENOISE) continue;
        if (i > first) {
            k_post_pointwise<<<grid, block, 0, s>>>(d_rgb, n, chain, first, i);
            e = cudaGetLastError();
        }
        if (i < num_steps && e == cudaSuccess) {
            // five a-trous passes, ping-ponging between the image and `pong`; an odd number
            // of passes ends in `pong`, which is copied back
            float* src = d_rgb;
            float* dst = pong;
            for (int k = 0; k < 5 && e == cudaSuccess; ++k) {
                k_atrous<<<pgrid, block, 0, s>>>(src, dst, d_alb, d_nrm, width, height, 1 << k, 0.5f / (float)(1 << k),
                                                 0.35f, 0.1f);
                e = cudaGetLastError();
                std::swap(src, dst);
            }
            if (e == cudaSuccess && src != d_rgb) e = cudaMemcpyAsync(d_rgb, src, fbytes, cudaMemcpyDeviceToDevice, s);
        }
        first = i + 1;
    }
    if (e == cudaSuccess && d_rgb8) {
        k_to_u8<<<grid, block, 0, s>>>(d_rgb, d_rgb8, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && d_alb8 && d_alb) {
        k_to_u8<<<grid, block, 0, s>>>(d_alb, d_alb8, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && d_nrm8 && d_nrm) {
        k_to_u8<<<grid, block, 0, s>>>(d_nrm, d_nrm8, n);
        e = cudaGetLastError();
    }
    if (!dev && e == cudaSuccess) {
        e = cudaMemcpyAsync(rgb, d_rgb, fbytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && d_rgb8) e = cudaMemcpyAsync(rgb8, d_rgb8, (size_t)n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && d_alb8) e = cudaMemcpyAsync(albedo8, d_alb8, (size_t)n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && d_nrm8) e = cudaMemcpyAsync(normal8, d_nrm8, (size_t)n, cudaMemcpyDeviceToHost, s);
    }
    cudaFreeAsync(tmp, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(ctx, e, "postprocess");
    if (e2 != cudaSuccess) return cuda_error(ctx, e2, "postprocess");
    return FM_OK;
}
