// Environment-map importance tables, built on the device.
//
// Follows EnvImportanceSampler's construction (light/env_importance_sampler.h:28-65)
// and Distribution1D/2D (math/distribution_1d.cpp:5-29, distribution_2d.cpp:9-26):
//   lum[j][i]  = luminance(tex(texel centre)) * sin(pi * (j + 0.5) / H)
//   lumn       = lum / sum(lum) * W * H                      (mean 1)
//   row_j      = sum_i lumn[j][i] / W                        (Distribution1D::pdf_sum)
//   marg       = sum_j row_j / H                             (marginal pdf_sum)
//   sampling density of texel (i, j)  = lumn[j][i] / marg
//   density reported by EnvLight::Pdf = (lumn[j][i] / row_j) / marg
// All sums are FP64.  Sampling uses Vose alias tables (one per row for the
// conditional, one for the marginal) built from the same weights.
#include "fm_internal.h"
#include "fm_texture.cuh"

namespace fm {

namespace {

__global__ void k_env_lum(DevTexture tex, int w, int h, float* lum)
{
    const int n = w * h;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int i = q % w, j = q / w;
        const float du = 1.0f / (float)w, dv = 1.0f / (float)h;
        const float u0 = (float)i / (float)w, v0 = (float)j / (float)h;
        const float sin_theta = sinf(kPi * (v0 + 0.5f * dv));
        const f3 rad = tex_sample(tex, u0 + 0.5f * du, v0 + 0.5f * dv);
        lum[q] = luminance(rad) * sin_theta;
    }
}

__global__ void k_env_rowsum(const float* lum, int w, double* rowsum)
{
    __shared__ double s[256];
    const int j = blockIdx.x;
    double acc = 0.0;
    for (int i = threadIdx.x; i < w; i += blockDim.x) acc += (double)lum[(size_t)j * w + i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) rowsum[j] = s[0];
}

// totals[0] = sum of lum, totals[1] = marginal sum (of normalized row sums / H)
__global__ void k_env_totals(const double* rowsum, int w, int h, double* totals)
{
    __shared__ double s[256];
    double acc = 0.0;
    for (int j = threadIdx.x; j < h; j += blockDim.x) acc += rowsum[j];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) s[threadIdx.x] += s[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double total = s[0];
        totals[0] = total;
        // row_j = (rowsum_j / total * W * H) / W ; marg = sum_j row_j / H
        double m = 0.0;
        for (int j = 0; j < h; ++j) m += (rowsum[j] / total * (double)w * (double)h) / (double)w;
        totals[1] = m / (double)h;
    }
}

__global__ void k_env_pdfs(const float* lum, const double* rowsum, const double* totals, int w, int h,
                           float* pdf_sample, float* pdf_eval)
{
    const int n = w * h;
    const double total = totals[0], marg = totals[1];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int j = q / w;
        const double lumn = (double)lum[q] / total * (double)w * (double)h;
        const double row = rowsum[j] / total * (double)h;   // sum_i lumn / W
        pdf_sample[q] = (float)(lumn / marg);
        pdf_eval[q] = (float)((lumn / row) / marg);
    }
}

// Vose's alias method over n weights, sequential; `small`/`large` are scratch stacks.
FM_D void vose(const float* wts_f, const double* wts_d, int n, float* prob, int32_t* alias, int32_t* small,
               int32_t* large)
{
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += wts_f ? (double)wts_f[i] : wts_d[i];
    if (!(sum > 0.0)) {
        for (int i = 0; i < n; ++i) {
            prob[i] = 1.0f;
            alias[i] = i;
        }
        return;
    }
    // scaled weights are kept in prob as float while the stacks are processed in double
    int ns = 0, nl = 0;
    const double scale = (double)n / sum;
    for (int i = 0; i < n; ++i) {
        const double q = (wts_f ? (double)wts_f[i] : wts_d[i]) * scale;
        prob[i] = (float)q;
        if (q < 1.0) small[ns++] = i;
        else large[nl++] = i;
    }
    // remaining mass of the current large entries is tracked in double
    while (ns > 0 && nl > 0) {
        const int s = small[--ns];
        const int l = large[nl - 1];
        alias[s] = l;
        const double ql = ((double)prob[l] + (double)prob[s]) - 1.0;
        prob[l] = (float)ql;
        if (ql < 1.0) {
            --nl;
            small[ns++] = l;
        }
    }
    while (nl > 0) {
        const int l = large[--nl];
        prob[l] = 1.0f;
        alias[l] = l;
    }
    while (ns > 0) {
        const int s = small[--ns];
        prob[s] = 1.0f;
        alias[s] = s;
    }
}

__global__ void k_env_alias_rows(const float* lum, int w, int h, float* prob, int32_t* alias, int32_t* scratch)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= h) return;
    int32_t* small = scratch + (size_t)j * 2 * w;
    vose(lum + (size_t)j * w, nullptr, w, prob + (size_t)j * w, alias + (size_t)j * w, small, small + w);
}

__global__ void k_env_alias_marg(const double* rowsum, int h, float* prob, int32_t* alias, int32_t* scratch)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    vose(nullptr, rowsum, h, prob, alias, scratch, scratch + h);
}

// The same tables with one row per block (one warp): the row's weights, outputs and
// stacks live in shared memory while lane 0 runs Vose's method (its sequential loop is
// bound by memory latency), and the warp moves the row in and out.  Dynamic shared
// memory: 5 w 4-byte words.
__global__ void k_env_alias_rows_smem(const float* lum, int w, float* prob, int32_t* alias)
{
    extern __shared__ float4 smem_f4[];
    float* wt = reinterpret_cast<float*>(smem_f4);
    float* p = wt + w;
    int32_t* a = reinterpret_cast<int32_t*>(p + w);
    int32_t* stk = a + w;
    const size_t row = (size_t)blockIdx.x * w;
    for (int i = threadIdx.x; i < w; i += blockDim.x) wt[i] = lum[row + i];
    __syncwarp();
    if (threadIdx.x == 0) vose(wt, nullptr, w, p, a, stk, stk + w);
    __syncwarp();
    for (int i = threadIdx.x; i < w; i += blockDim.x) {
        prob[row + i] = p[i];
        alias[row + i] = a[i];
    }
}

// Marginal table in shared memory (24 h bytes: weights, probabilities, aliases, stacks).
__global__ void k_env_alias_marg_smem(const double* rowsum, int h, float* prob, int32_t* alias)
{
    extern __shared__ float4 smem_f4[];
    double* wt = reinterpret_cast<double*>(smem_f4);
    float* p = reinterpret_cast<float*>(wt + h);
    int32_t* a = reinterpret_cast<int32_t*>(p + h);
    int32_t* stk = a + h;
    for (int i = threadIdx.x; i < h; i += blockDim.x) wt[i] = rowsum[i];
    __syncwarp();
    if (threadIdx.x == 0) vose(nullptr, wt, h, p, a, stk, stk + h);
    __syncwarp();
    for (int i = threadIdx.x; i < h; i += blockDim.x) {
        prob[i] = p[i];
        alias[i] = a[i];
    }
}

// Dynamic shared memory a kernel may use: the default 48 KB, or up to the device's
// opt-in limit once requested.
template <class K>
bool smem_fits(K kernel, size_t bytes)
{
    if (bytes <= 48 * 1024) return true;
    int dev = 0, limit = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        bytes > (size_t)limit) {
        cudaGetLastError();
        return false;
    }
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

// grad[k][l][c] -= total_score * d log(sum lum)/d texel + row_score[k] * d log(rowsum_k)/d texel,
// with d lum[k][l] / d texel[k][l][c] = L_c * sin_k (lum as in k_env_lum).
__global__ void k_env_grad_spread(const float* lum, const double* rowsum, const double* totals, const double* row_score,
                                  const double* total_score, int w, int h, double* grad)
{
    const int n = w * h;
    const double total = totals[0], ts = total_score[0];
    const double Lc[3] = {0.2126, 0.7152, 0.0722};
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int j = q / w;
        const double sin_theta = (double)sinf(kPi * (((float)j + 0.5f) / (float)h));
        const double k_tot = total > 0.0 ? ts * sin_theta / total : 0.0;
        const double k_row = rowsum[j] > 0.0 ? row_score[j] * sin_theta / rowsum[j] : 0.0;
        for (int c = 0; c < 3; ++c) grad[3 * (size_t)q + c] -= (k_tot + k_row) * Lc[c];
    }
}

}  // namespace

fm_status env_grad_finalize(fm_ctx* ctx, const DevTexture& tex, const double* env_row, const double* env_total,
                            double* grad)
{
    const int w = tex.w, h = tex.h;
    const size_t n = (size_t)w * h;
    cudaStream_t st = ctx->stream;
    float* lum = nullptr;
    double *rowsum = nullptr, *totals = nullptr;
    FM_CUDA_TRY(ctx, cudaMallocAsync(&lum, n * sizeof(float), st), "env grad");
    FM_CUDA_TRY(ctx, cudaMallocAsync(&rowsum, h * sizeof(double), st), "env grad");
    FM_CUDA_TRY(ctx, cudaMallocAsync(&totals, 2 * sizeof(double), st), "env grad");
    const int grid = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    k_env_lum<<<grid, 256, 0, st>>>(tex, w, h, lum);
    k_env_rowsum<<<h, 256, 0, st>>>(lum, w, rowsum);
    k_env_totals<<<1, 256, 0, st>>>(rowsum, w, h, totals);
    k_env_grad_spread<<<grid, 256, 0, st>>>(lum, rowsum, totals, env_row, env_total, w, h, grad);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(lum, st);
    cudaFreeAsync(rowsum, st);
    cudaFreeAsync(totals, st);
    if (e != cudaSuccess) return cuda_error(ctx, e, "env grad");
    return FM_OK;
}

fm_status env_build_tables(fm_ctx* ctx, cudaStream_t st, fm_scene* scene, const DevTexture& tex, DevEnv& env)
{
    const int w = tex.w, h = tex.h;
    const size_t n = (size_t)w * h;
    float *lum = nullptr, *pdf_sample = nullptr, *pdf_eval = nullptr, *row_prob = nullptr, *marg_prob = nullptr;
    int32_t *row_alias = nullptr, *marg_alias = nullptr, *scratch = nullptr;
    double *rowsum = nullptr, *totals = nullptr;
    auto track = [&](void* p) { scene->allocations.push_back(p); };
    if (env.pdf_sample && env.w == w && env.h == h) {
        // rebuilding for new texel values: reuse the tables
        pdf_sample = const_cast<float*>(env.pdf_sample);
        pdf_eval = const_cast<float*>(env.pdf_eval);
        row_prob = const_cast<float*>(env.row_prob);
        row_alias = const_cast<int32_t*>(env.row_alias);
        marg_prob = const_cast<float*>(env.marg_prob);
        marg_alias = const_cast<int32_t*>(env.marg_alias);
    } else {
        FM_CUDA_TRY(ctx, cudaMallocAsync(&pdf_sample, n * sizeof(float), st), "env tables");
        track(pdf_sample);
        FM_CUDA_TRY(ctx, cudaMallocAsync(&pdf_eval, n * sizeof(float), st), "env tables");
        track(pdf_eval);
        FM_CUDA_TRY(ctx, cudaMallocAsync(&row_prob, n * sizeof(float), st), "env tables");
        track(row_prob);
        FM_CUDA_TRY(ctx, cudaMallocAsync(&row_alias, n * sizeof(int32_t), st), "env tables");
        track(row_alias);
        FM_CUDA_TRY(ctx, cudaMallocAsync(&marg_prob, h * sizeof(float), st), "env tables");
        track(marg_prob);
        FM_CUDA_TRY(ctx, cudaMallocAsync(&marg_alias, h * sizeof(int32_t), st), "env tables");
        track(marg_alias);
    }
    // temporaries
    FM_CUDA_TRY(ctx, cudaMallocAsync(&lum, n * sizeof(float), st), "env tables");
    FM_CUDA_TRY(ctx, cudaMallocAsync(&scratch, 2 * n * sizeof(int32_t), st), "env tables");
    FM_CUDA_TRY(ctx, cudaMallocAsync(&rowsum, h * sizeof(double), st), "env tables");
    FM_CUDA_TRY(ctx, cudaMallocAsync(&totals, 2 * sizeof(double), st), "env tables");
    k_env_lum<<<(int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, st>>>(tex, w, h, lum);
    k_env_rowsum<<<h, 256, 0, st>>>(lum, w, rowsum);
    k_env_totals<<<1, 256, 0, st>>>(rowsum, w, h, totals);
    k_env_pdfs<<<(int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, st>>>(lum, rowsum, totals, w, h,
                                                                                       pdf_sample, pdf_eval);
    const size_t row_smem = 5 * sizeof(float) * (size_t)w, marg_smem = 24 * (size_t)h;
    if (smem_fits(k_env_alias_rows_smem, row_smem))
        k_env_alias_rows_smem<<<h, 32, row_smem, st>>>(lum, w, row_prob, row_alias);
    else
        k_env_alias_rows<<<(h + 63) / 64, 64, 0, st>>>(lum, w, h, row_prob, row_alias, scratch);
    if (smem_fits(k_env_alias_marg_smem, marg_smem))
        k_env_alias_marg_smem<<<1, 32, marg_smem, st>>>(rowsum, h, marg_prob, marg_alias);
    else
        k_env_alias_marg<<<1, 1, 0, st>>>(rowsum, h, marg_prob, marg_alias, scratch);
    cudaFreeAsync(lum, st);
    cudaFreeAsync(scratch, st);
    cudaFreeAsync(rowsum, st);
    cudaFreeAsync(totals, st);
    FM_CUDA_TRY(ctx, cudaGetLastError(), "env tables");
    env.w = w;
    env.h = h;
    env.pdf_sample = pdf_sample;
    env.pdf_eval = pdf_eval;
    env.row_prob = row_prob;
    env.row_alias = row_alias;
    env.marg_prob = marg_prob;
    env.marg_alias = marg_alias;
    return FM_OK;
}

}  // namespace fm
