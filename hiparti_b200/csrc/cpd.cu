// cpd.cu -- CPD-ALS on the GPU, restating the loop of src/sptensor/cpd.c:32-160:
//
//   for it: for m:  M   = MTTKRP(X, A, m)
//                   A_m = M * (Hadamard_{k != m} A_k^T A_k)^{-1}
//                   lambda = it == 0 ? column 2-norms : max(column max, 1);  A_m /= lambda
//                   G_m = A_m^T A_m
//           fit = 1 - sqrt(||X||^2 + lambda^T (Hadamard_k G_k) lambda - 2 <X, M_{N-1} o A_{N-1} lambda>) / ||X||
//   final lambda: lambda_r *= prod_m ||A_m[:, r]||, columns normalised
//
// Precision: factors are stored in FP32 (or, in mixed mode, additionally as a
// BF16 copy that the MTTKRP gathers read); MTTKRP accumulates in FP32; Grams,
// their Hadamard product, the Cholesky factor and inverse, the row solve and
// the fit are FP64.  A Gram matrix that is not positive definite is inverted
// by Gauss-Jordan elimination with partial pivoting (the reference falls back
// to sgesv, src/matrix/matrix_solver.c:66-80); a singular one leaves the rows
// unsolved, as sgesv does when it fails.
//
// The fit uses the full symmetric Grams.  (The reference's KruskalTensorFit,
// src/ktensor/ktensor.c:105-147, reads the triangle of each Gram that its
// ssyrk_ call does not write, so its printed fit is not the model's fit.)
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <limits>

#include "checkpoint.cuh"
#include "spd.cuh"
#include "tensor.cuh"

namespace pti {

constexpr int kMaxCpdRank = 128;

// Gram accumulation: G += A^T A over rows [0, I).  If lambda is given the
// rows are first divided column-wise by lambda (and written back); if bf16 is
// given the (scaled) rows are also stored as BF16.  With round_bf16 the Gram
// is formed from the BF16-rounded values -- the ones the next MTTKRPs gather --
// so that an ALS step's right-hand side and normal matrix come from the same
// factors (with FP32 Grams beside BF16 gathers the normal equations are
// inconsistent, and inside an ALS swamp, where they are ill-conditioned, the
// solve amplifies that until the iteration diverges).  Dynamic shared
// memory: R*R doubles of accumulator + 32*R doubles of row tile.
__global__ void gram_kernel(float *A, uint32_t I, uint32_t R, uint32_t stride, const float *lambda,
                            __nv_bfloat16 *bf16, double *G, int round_bf16)
{
    extern __shared__ double sm[];
    double *acc = sm;
    double *tile = sm + (size_t)R * R;
    const uint32_t RR = R * R;
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) acc[e] = 0.0;
    for (uint64_t r0 = (uint64_t)blockIdx.x * 32; r0 < I; r0 += (uint64_t)gridDim.x * 32) {
        const uint32_t rows = (uint32_t)((I - r0) < 32 ? (I - r0) : 32);
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < 32 * stride; e += blockDim.x) {
            const uint32_t r = e / stride, c = e % stride;
            if (r >= rows) continue;
            float *p = A + (r0 + r) * stride + c;
            float v = *p;
            if (c >= R) {
                v = 0.f;
                if (lambda) *p = 0.f;
            } else if (lambda) {
                v = v / lambda[c];
                *p = v;
            }
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            if (bf16) bf16[(r0 + r) * stride + c] = h;
            if (c < R) tile[r * R + c] = round_bf16 ? (double)__bfloat162float(h) : (double)v;
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) {
            const uint32_t p = e / R, q = e % R;
            double s = 0.0;
            for (uint32_t r = 0; r < rows; ++r) s += tile[r * R + p] * tile[r * R + q];
            acc[e] += s;
        }
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) atomicAdd(G + e, acc[e]);
}

// One CTA: W = (Hadamard_{k != mode} G_k)^{-1}.  flag[0] = 1 if the Cholesky
// factorisation failed (fallback used), 2 if the matrix was singular
// (W = identity: rows left unsolved).  Ranks up to 32: the matrices sit in
// shared memory and one warp factors them (spd_inverse).
__global__ void gram_inverse_small_kernel(const double *G, uint32_t N, uint32_t R, uint32_t mode, double *W,
                                          int *flag)
{
    __shared__ double sV[32 * 32], sL[32 * 32], sLi[32 * 32], sW[32 * 32];
    const uint32_t RR = R * R;
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) {
        double v = 1.0;
        for (uint32_t k = 1; k < N; ++k) v *= G[(size_t)((mode + k) % N) * RR + e];
        sV[e] = v;
    }
    __syncthreads();
    const int f = spd_inverse(sV, sL, sLi, sW, R);
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) W[e] = sW[e];
    if (threadIdx.x == 0) flag[0] = f;
}

// The same for ranks above 32; work holds 3*R*R doubles in global memory.
__global__ void gram_inverse_kernel(const double *G, uint32_t N, uint32_t R, uint32_t mode, double *W,
                                    double *work, int *flag)
{
    const uint32_t RR = R * R;
    double *V = work, *L = work + RR, *Li = work + 2 * RR;
    __shared__ int s_bad;
    __shared__ double s_d;
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) {
        double v = 1.0;
        for (uint32_t k = 1; k < N; ++k) v *= G[(size_t)((mode + k) % N) * RR + e];
        V[e] = v;
        L[e] = 0.0;
        Li[e] = 0.0;
    }
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    // Cholesky V = L L^T, column by column
    for (uint32_t j = 0; j < R; ++j) {
        if (threadIdx.x == 0) {
            double d = V[j * R + j];
            for (uint32_t k = 0; k < j; ++k) d -= L[j * R + k] * L[j * R + k];
            if (!(d > 0.0)) s_bad = 1;
            s_d = d > 0.0 ? sqrt(d) : 1.0;
            L[j * R + j] = s_d;
        }
        __syncthreads();
        if (s_bad) break;
        for (uint32_t i = j + 1 + threadIdx.x; i < R; i += blockDim.x) {
            double s = V[i * R + j];
            for (uint32_t k = 0; k < j; ++k) s -= L[i * R + k] * L[j * R + k];
            L[i * R + j] = s / s_d;
        }
        __syncthreads();
    }
    if (!s_bad) {
        // Li = L^{-1}, one column per thread
        for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
            for (uint32_t i = c; i < R; ++i) {
                double s = (i == c) ? 1.0 : 0.0;
                for (uint32_t k = c; k < i; ++k) s -= L[i * R + k] * Li[k * R + c];
                Li[i * R + c] = s / L[i * R + i];
            }
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) {
            const uint32_t p = e / R, q = e % R;
            double s = 0.0;
            for (uint32_t k = max(p, q); k < R; ++k) s += Li[k * R + p] * Li[k * R + q];
            W[e] = s;
        }
        if (threadIdx.x == 0) flag[0] = 0;
        return;
    }
    // Gauss-Jordan with partial pivoting on [V | I]: L holds V, Li holds I.
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) {
        L[e] = V[e];
        Li[e] = (e / R == e % R) ? 1.0 : 0.0;
    }
    __shared__ uint32_t s_piv;
    __shared__ int s_sing;
    if (threadIdx.x == 0) s_sing = 0;
    __syncthreads();
    for (uint32_t j = 0; j < R && !s_sing; ++j) {
        if (threadIdx.x == 0) {
            uint32_t p = j;
            for (uint32_t i = j + 1; i < R; ++i)
                if (fabs(L[i * R + j]) > fabs(L[p * R + j])) p = i;
            s_piv = p;
            if (L[p * R + j] == 0.0) s_sing = 1;
        }
        __syncthreads();
        if (s_sing) break;
        const uint32_t p = s_piv;
        if (p != j)
            for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
                double t = L[j * R + c]; L[j * R + c] = L[p * R + c]; L[p * R + c] = t;
                t = Li[j * R + c]; Li[j * R + c] = Li[p * R + c]; Li[p * R + c] = t;
            }
        __syncthreads();
        const double piv = L[j * R + j];
        __syncthreads();
        for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
            L[j * R + c] /= piv;
            Li[j * R + c] /= piv;
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x) {
            const uint32_t i = e / R, c = e % R;
            if (i == j) continue;
            const double f = L[i * R + j];
            if (c != j) L[i * R + c] -= f * L[j * R + c];
            Li[i * R + c] -= f * Li[j * R + c];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < R; i += blockDim.x)
            if (i != j) L[i * R + j] = 0.0;
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < RR; e += blockDim.x)
        W[e] = s_sing ? ((e / R == e % R) ? 1.0 : 0.0) : Li[e];
    if (threadIdx.x == 0) flag[0] = s_sing ? 2 : 1;
}

// A[i, :] = M[i, :] * W (W symmetric), FP64 accumulation; pad columns zeroed.
// Accumulates per-column sums of squares (FP64) and maxima of the FP32 results.
__global__ void solve_rows_kernel(const float *M, const double *W, uint32_t I, uint32_t R, uint32_t stride, float *A,
                                  double *colsq, int *colmax)
{
    extern __shared__ double sm[];
    double *sW = sm;                         // R*R
    double *s_sq = sm + (size_t)R * R;       // R
    int *s_mx = reinterpret_cast<int *>(s_sq + R);  // R
    for (uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) sW[e] = W[e];
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        s_sq[c] = 0.0;
        s_mx[c] = 0;  // bits of +0.0f
    }
    __syncthreads();
    const uint64_t total = (uint64_t)I * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = e / stride;
        const uint32_t c = (uint32_t)(e % stride);
        if (c >= R) {
            A[e] = 0.f;
            continue;
        }
        const float *m = M + i * stride;
        double s = 0.0;
        for (uint32_t k = 0; k < R; ++k) s += (double)m[k] * sW[k * R + c];
        const float v = (float)s;
        A[e] = v;
        atomicAdd(&s_sq[c], (double)v * (double)v);
        if (v > 0.f) atomicMax(&s_mx[c], __float_as_int(v));
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        atomicAdd(&colsq[c], s_sq[c]);
        atomicMax(&colmax[c], s_mx[c]);
    }
}

// lambda from the column statistics: iteration 0 -> 2-norm
// (src/matrix/matrix.c:389-469), later -> max(column max, 1) (:472-553).
__global__ void lambda_kernel(const double *colsq, const int *colmax, uint32_t R, int use_2norm, float *lambda)
{
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        if (use_2norm) {
            lambda[c] = (float)sqrt(colsq[c]);
        } else {
            float v = __int_as_float(colmax[c]);
            lambda[c] = v < 1.f ? 1.f : v;
        }
    }
}

// inner += sum_i sum_r lambda_r A[i, r] M[i, r]; with Ab the factor is read
// from its BF16 copy (the values a BF16 iteration's MTTKRPs and Grams used,
// so that the fit is that of one model)
__global__ void inner_kernel(const float *A, const float *M, uint32_t I, uint32_t R, uint32_t stride,
                             const float *lambda, double *inner, const __nv_bfloat16 *Ab = nullptr)
{
    double s = 0.0;
    const uint64_t total = (uint64_t)I * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(e % stride);
        if (c < R) s += (double)(Ab ? __bfloat162float(Ab[e]) : A[e]) * (double)M[e] * (double)lambda[c];
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(inner, s);
}

__global__ void sumsq_kernel(const float *v, uint64_t n, double *out)
{
    double s = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += (double)v[i] * (double)v[i];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// fit = 1 - sqrt(normX2 + |lambda^T (Hadamard_k G_k) lambda| - 2 inner) / sqrt(normX2)
// (src/ktensor/ktensor.c:77-99: the square root is skipped if the residual is
// not positive).
__global__ void fit_kernel(const double *G, uint32_t N, uint32_t R, const float *lambda, const double *normX2,
                           const double *inner, double *fit_out)
{
    __shared__ double s_part[32];
    double s = 0.0;
    for (uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
        double v = 1.0;
        for (uint32_t k = 0; k < N; ++k) v *= G[(size_t)k * R * R + e];
        s += v * (double)lambda[e / R] * (double)lambda[e % R];
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double norm_mats = 0.0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) norm_mats += s_part[w];
        norm_mats = fabs(norm_mats);
        double residual = normX2[0] + norm_mats - 2.0 * inner[0];
        if (residual > 0.0) residual = sqrt(residual);
        fit_out[0] = 1.0 - residual / sqrt(normX2[0]);
    }
}

// Column 2-norms of A (FP64), for the final lambda.
__global__ void colsq_kernel(const float *A, uint32_t I, uint32_t R, uint32_t stride, double *colsq)
{
    extern __shared__ double s_sq[];
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) s_sq[c] = 0.0;
    __syncthreads();
    const uint64_t total = (uint64_t)I * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(e % stride);
        if (c < R) atomicAdd(&s_sq[c], (double)A[e] * (double)A[e]);
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) atomicAdd(&colsq[c], s_sq[c]);
}

// A[:, c] /= norm_c ; lambda_c *= norm_c (src/matrix/matrix.c:556-572)
__global__ void final_scale_kernel(float *A, uint32_t I, uint32_t R, uint32_t stride, const double *colsq,
                                   float *lambda, int update_lambda)
{
    const uint64_t total = (uint64_t)I * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(e % stride);
        if (c < R) A[e] = A[e] / (float)sqrt(colsq[c]);
    }
    if (update_lambda && blockIdx.x == 0)
        for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) lambda[c] *= (float)sqrt(colsq[c]);
}

// ---------------------------------------------------------------------------
// The ALS driver.
// ---------------------------------------------------------------------------
struct CpdOptions {
    uint32_t R = 0, niters = 0;
    double tol = 0.0;
    int precision = PTI_B200_F32;  // factors read by MTTKRP: F32 or BF16
    uint32_t fp32_sweeps = 1;      // closing iterations with FP32 factors (mixed mode)
    const char *ckpt_path = nullptr;  // checkpoint file (nullptr: none)
    uint32_t ckpt_every = 0;          // write after every ckpt_every iterations; always after the last
    bool resume = false;              // continue from ckpt_path when the file exists
    float *m_last = nullptr;          // device, ndims[N-1] x stride: receives the last MTTKRP output
};

struct CpdResult {
    std::vector<double> fits;
    uint32_t iters = 0;
    uint32_t resumed_from = 0;  // iterations restored from a checkpoint
    int solver_flags = 0;       // OR of gram_inverse flags seen
};

// A[m] (device, I_m x stride FP32) hold the initial factors on entry and the
// result on exit; lambda (device, R floats) receives the weights.  With a
// checkpoint file and `resume`, the loop state stored there replaces the
// initial factors and the loop continues after its last iteration.
int cpd_device(ptiB200Tensor *t, float *const *A, uint32_t stride, float *lambda, const CpdOptions &opt,
               CpdResult &res, cudaStream_t s)
{
    const char *mod = "B200 CPD-ALS";
    const uint32_t N = t->nmodes, R = opt.R;
    PTI_CHECK(R >= 1 && R <= (uint32_t)kMaxCpdRank, PTIERR_VALUE_ERROR, mod, "rank must be in [1, 128]");
    PTI_CHECK(stride >= R && stride % 8 == 0, PTIERR_SHAPE_MISMATCH, mod, "stride must be >= rank, multiple of 8");
    PTI_CHECK(opt.precision == PTI_B200_F32 || opt.precision == PTI_B200_BF16, PTIERR_VALUE_ERROR, mod,
              "bad precision");
    const uint32_t RR = R * R;
    uint32_t maxI = 0;
    for (uint32_t m = 0; m < N; ++m) maxI = std::max(maxI, t->ndims[m]);

    DevBuf M, G, W, work, stats, scal, Ab[kMaxModes];
    PTI_CUDA(M.alloc(padded((size_t)maxI * stride * 4), s), mod);
    PTI_CUDA(G.alloc(padded((size_t)N * RR * 8), s), mod);
    PTI_CUDA(W.alloc(padded((size_t)RR * 8), s), mod);
    PTI_CUDA(work.alloc(padded((size_t)3 * RR * 8), s), mod);
    PTI_CUDA(stats.alloc(padded((size_t)R * 12 + 64), s), mod);  // colsq (R doubles) + colmax (R ints)
    // scal: [0] normX2, [1] inner, [2..2+niters) fits ; flags after
    PTI_CUDA(scal.alloc(padded((size_t)(4 + opt.niters) * 8 + 64), s), mod);
    double *colsq = stats.as<double>();
    int *colmax = reinterpret_cast<int *>(colsq + R);
    double *normX2 = scal.as<double>(), *inner = normX2 + 1, *fits = normX2 + 2;
    int *flag = reinterpret_cast<int *>(fits + opt.niters + 1);
    const bool mixed = opt.precision == PTI_B200_BF16;
    if (mixed)
        for (uint32_t m = 0; m < N; ++m)
            PTI_CUDA(Ab[m].alloc(padded((size_t)t->ndims[m] * stride * 2), s), mod);

    // Resume: the stored loop state replaces the initial factors.  The row
    // pad columns are zeroed, as the solves leave them.
    CkptState st;
    bool have_ckpt = false;
    if (opt.resume && opt.ckpt_path) {
        bool missing = false;
        PTI_TRY(ckpt_read(opt.ckpt_path, st, &missing));
        have_ckpt = !missing;
    }
    if (have_ckpt) {
        bool same = st.nmodes == N && st.rank == R && st.nnz == t->nnz;
        for (uint32_t m = 0; same && m < N; ++m) same = st.ndims[m] == t->ndims[m];
        PTI_CHECK(same, PTIERR_SHAPE_MISMATCH, mod, "checkpoint is of another tensor shape or rank");
        PTI_CHECK(st.iters <= opt.niters, PTIERR_VALUE_ERROR, mod, "checkpoint holds more iterations than niters");
        for (uint32_t m = 0; m < N; ++m) {
            if (!t->ndims[m]) continue;
            PTI_CUDA(cudaMemsetAsync(A[m], 0, (size_t)t->ndims[m] * stride * 4, s), mod);
            PTI_CUDA(cudaMemcpy2DAsync(A[m], (size_t)stride * 4, st.factors[m].data(), (size_t)R * 4, (size_t)R * 4,
                                       t->ndims[m], cudaMemcpyHostToDevice, s),
                     mod);
        }
        PTI_CUDA(cudaMemcpyAsync(lambda, st.lambda.data(), (size_t)R * 4, cudaMemcpyHostToDevice, s), mod);
        if (st.iters)
            PTI_CUDA(cudaMemcpyAsync(fits, st.fits.data(), (size_t)st.iters * 8, cudaMemcpyHostToDevice, s), mod);
    }
    CkptWriter writer;
    if (opt.ckpt_path) PTI_TRY(writer.init(opt.ckpt_path, N, t->ndims.data(), t->nnz, R, opt.niters));

    const size_t gram_smem = (size_t)(RR + 32 * R) * 8;
    const size_t solve_smem = (size_t)RR * 8 + (size_t)R * 12;
    PTI_CUDA(cudaFuncSetAttribute(gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem), mod);
    PTI_CUDA(cudaFuncSetAttribute(solve_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem), mod);
    const unsigned sms = (unsigned)sm_count();
    auto rows_grid = [&](uint64_t items, unsigned per) {
        return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + per - 1) / per, sms * 4ull));
    };

    // Grams of every factor (cpd.c:65-72) and their BF16 copies; with
    // round_bf16 the Grams are of the BF16-rounded factors (gram_kernel)
    auto all_grams = [&](int round_bf16) -> int {
        PTI_CUDA(cudaMemsetAsync(G.ptr, 0, (size_t)N * RR * 8, s), mod);
        for (uint32_t m = 0; m < N; ++m)
            gram_kernel<<<rows_grid(t->ndims[m], 32), 256, gram_smem, s>>>(
                A[m], t->ndims[m], R, stride, nullptr, mixed ? Ab[m].as<__nv_bfloat16>() : nullptr,
                G.as<double>() + (size_t)m * RR, round_bf16);
        return 0;
    };
    const uint32_t it_first = have_ckpt ? st.iters : 0;
    bool grams_bf16 = mixed && it_first + opt.fp32_sweeps < opt.niters;
    PTI_TRY(all_grams(grams_bf16));
    PTI_CUDA(cudaMemsetAsync(scal.ptr, 0, 16, s), mod);
    if (t->nnz) sumsq_kernel<<<rows_grid(t->nnz, 256), 256, 0, s>>>(t->vals.as<float>(), t->nnz, normX2);
    PTI_CUDA(cudaGetLastError(), mod);

    if (have_ckpt) {
        // The sum of squares tells a different tensor of the same shape.
        double nx = 0.0;
        PTI_CUDA(cudaMemcpyAsync(&nx, normX2, 8, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
        PTI_CHECK(std::fabs(nx - st.normX2) <= 1e-6 * std::max(std::fabs(nx), std::fabs(st.normX2)),
                  PTIERR_VALUE_ERROR, mod, "checkpoint is of another tensor (sum of squared values differs)");
    }

    // W of a mode needs only the other modes' Grams, so it is computed on a
    // side stream while that mode's MTTKRP runs on s (fork at ev.g, join at
    // ev.w before the row solve)
    struct ForkEvents {
        cudaEvent_t g = nullptr, w = nullptr;
        ~ForkEvents()
        {
            if (g) cudaEventDestroy(g);
            if (w) cudaEventDestroy(w);
        }
    } ev;
    PTI_CUDA(cudaEventCreateWithFlags(&ev.g, cudaEventDisableTiming), mod);
    PTI_CUDA(cudaEventCreateWithFlags(&ev.w, cudaEventDisableTiming), mod);
    const cudaStream_t side = side_stream(1);

    std::vector<uint32_t> order(N);
    std::vector<const void *> fptr(N);
    res.fits.clear();
    res.resumed_from = have_ckpt ? st.iters : 0;
    double oldfit = have_ckpt && st.iters ? st.fits[st.iters - 1] : 0.0;
    bool converged = have_ckpt && (st.flags & kCkptConverged) && opt.tol > 0.0;
    uint32_t it = have_ckpt ? st.iters : 0;
    for (; it < opt.niters && !converged; ++it) {
        const bool use_bf16 = mixed && it + opt.fp32_sweeps < opt.niters;
        if (use_bf16 != grams_bf16) {  // the closing FP32 sweeps start: Grams of the FP32 factors
            grams_bf16 = use_bf16;
            PTI_TRY(all_grams(grams_bf16));
        }
        for (uint32_t k = 0; k < N; ++k)
            fptr[k] = use_bf16 ? (const void *)Ab[k].ptr : (const void *)A[k];
        for (uint32_t m = 0; m < N; ++m) {
            for (uint32_t i = 0; i < N; ++i) order[i] = (m + i) % N;
            PTI_CUDA(cudaEventRecord(ev.g, s), mod);
            PTI_CUDA(cudaStreamWaitEvent(side, ev.g, 0), mod);
            if (R <= 32)
                gram_inverse_small_kernel<<<1, 256, 0, side>>>(G.as<double>(), N, R, m, W.as<double>(), flag);
            else
                gram_inverse_kernel<<<1, 256, 0, side>>>(G.as<double>(), N, R, m, W.as<double>(), work.as<double>(),
                                                         flag);
            PTI_CUDA(cudaGetLastError(), mod);
            PTI_CUDA(cudaEventRecord(ev.w, side), mod);
            PTI_TRY(mttkrp_device(t, fptr.data(), use_bf16 ? PTI_B200_BF16 : PTI_B200_F32, R, stride, order.data(), m,
                                  M.as<float>(), s));
            PTI_CUDA(cudaStreamWaitEvent(s, ev.w, 0), mod);
            PTI_CUDA(cudaMemsetAsync(stats.ptr, 0, (size_t)R * 12, s), mod);
            solve_rows_kernel<<<rows_grid((uint64_t)t->ndims[m] * stride, 256), 256, solve_smem, s>>>(
                M.as<float>(), W.as<double>(), t->ndims[m], R, stride, A[m], colsq, colmax);
            lambda_kernel<<<1, 128, 0, s>>>(colsq, colmax, R, it == 0, lambda);
            PTI_CUDA(cudaMemsetAsync(G.as<double>() + (size_t)m * RR, 0, (size_t)RR * 8, s), mod);
            gram_kernel<<<rows_grid(t->ndims[m], 32), 256, gram_smem, s>>>(
                A[m], t->ndims[m], R, stride, lambda, mixed ? Ab[m].as<__nv_bfloat16>() : nullptr,
                G.as<double>() + (size_t)m * RR, use_bf16);
            PTI_CUDA(cudaGetLastError(), mod);
        }
        const uint32_t last = N - 1;
        PTI_CUDA(cudaMemsetAsync(inner, 0, 8, s), mod);
        inner_kernel<<<rows_grid((uint64_t)t->ndims[last] * stride, 256), 256, 0, s>>>(
            A[last], M.as<float>(), t->ndims[last], R, stride, lambda, inner,
            use_bf16 ? Ab[last].as<__nv_bfloat16>() : nullptr);
        fit_kernel<<<1, 256, 0, s>>>(G.as<double>(), N, R, lambda, normX2, inner, fits + it);
        PTI_CUDA(cudaGetLastError(), mod);
        if (opt.tol > 0.0) {
            double fit = 0.0;
            PTI_CUDA(cudaMemcpyAsync(&fit, fits + it, 8, cudaMemcpyDeviceToHost, s), mod);
            PTI_CUDA(cudaStreamSynchronize(s), mod);
            // cpd.c:144: stop when the fit changes by less than tol
            converged = it > 0 && std::fabs(fit - oldfit) < opt.tol;
            oldfit = fit;
        }
        if (opt.ckpt_path &&
            (converged || it + 1 == opt.niters || (opt.ckpt_every && (it + 1) % opt.ckpt_every == 0)))
            PTI_TRY(writer.save(A, stride, lambda, fits, normX2, it + 1, converged, s));
    }
    res.iters = it;
    if (opt.m_last && it > 0 && t->ndims[N - 1])
        PTI_CUDA(cudaMemcpyAsync(opt.m_last, M.ptr, (size_t)t->ndims[N - 1] * stride * 4, cudaMemcpyDeviceToDevice, s),
                 mod);
    // GetFinalLambda (matrix.c:556-572)
    for (uint32_t m = 0; m < N; ++m) {
        PTI_CUDA(cudaMemsetAsync(colsq, 0, (size_t)R * 8, s), mod);
        colsq_kernel<<<rows_grid((uint64_t)t->ndims[m] * stride, 256), 256, R * 8, s>>>(A[m], t->ndims[m], R, stride,
                                                                                        colsq);
        final_scale_kernel<<<rows_grid((uint64_t)t->ndims[m] * stride, 256), 256, 0, s>>>(A[m], t->ndims[m], R,
                                                                                          stride, colsq, lambda, 1);
    }
    PTI_CUDA(cudaGetLastError(), mod);
    res.fits.resize(it);
    int hflag = 0;
    if (it) PTI_CUDA(cudaMemcpyAsync(res.fits.data(), fits, it * 8, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    res.solver_flags = hflag;
    PTI_TRY(writer.finish());
    return 0;
}

int upload_coo(ptiB200Tensor *t, const ptiSparseTensor *X, cudaStream_t s);

namespace {

// Runs CPD-ALS on an uploaded tensor from the reference's initial factors
// (A[i][j] = i + j + 1, src/matrix/matrix.c:67-74) and copies the result into
// host rows (stride floats each) through `sink(m, device_ptr)`.
template <class Sink>
int host_cpd(ptiB200Tensor *t, uint32_t R, uint32_t niters, double tol, float *lambda_host, double *fit_out,
             Sink sink, cudaStream_t s)
{
    const char *mod = "B200 CPD-ALS";
    const uint32_t N = t->nmodes;
    const uint32_t stride = ((R - 1) / 8 + 1) * 8;
    DevBuf A[kMaxModes], lam;
    float *ptrs[kMaxModes];
    for (uint32_t m = 0; m < N; ++m) {
        const size_t n = (size_t)t->ndims[m] * stride;
        std::vector<float> h(n, 0.f);
        for (uint32_t i = 0; i < t->ndims[m]; ++i)
            for (uint32_t j = 0; j < R; ++j) h[(size_t)i * stride + j] = (float)(i + j + 1);
        PTI_CUDA(A[m].alloc(padded(n * 4), s), mod);
        PTI_CUDA(cudaMemcpyAsync(A[m].ptr, h.data(), n * 4, cudaMemcpyHostToDevice, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
        ptrs[m] = A[m].as<float>();
    }
    PTI_CUDA(lam.alloc(padded(R * 4), s), mod);
    CpdOptions opt;
    opt.R = R;
    opt.niters = niters;
    opt.tol = tol;
    CpdResult res;
    PTI_TRY(cpd_device(t, ptrs, stride, lam.as<float>(), opt, res, s));
    PTI_CUDA(cudaMemcpyAsync(lambda_host, lam.ptr, R * 4, cudaMemcpyDeviceToHost, s), mod);
    for (uint32_t m = 0; m < N; ++m) PTI_TRY(sink(m, A[m].as<float>(), stride));
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    *fit_out = res.iters ? res.fits.back() : 0.0;
    return 0;
}

int cpd_coo_entry(const ptiSparseTensor *X, ptiIndex R, ptiIndex niters, double tol, ptiKruskalTensor *k)
{
    const char *mod = "B200 CPD-ALS";
    PTI_CHECK(X && k && k->lambda, PTIERR_VALUE_ERROR, mod, "null tensor or Kruskal tensor");
    PTI_CHECK(R >= 1, PTIERR_VALUE_ERROR, mod, "rank must be positive");
    cudaStream_t s = sync_stream();
    ptiB200Tensor t;
    PTI_TRY(upload_coo(&t, X, s));
    const uint32_t N = X->nmodes;
    ptiMatrix **mats = static_cast<ptiMatrix **>(std::calloc(N + 1, sizeof(ptiMatrix *)));
    for (uint32_t m = 0; m <= N; ++m) mats[m] = static_cast<ptiMatrix *>(std::calloc(1, sizeof(ptiMatrix)));
    for (uint32_t m = 0; m < N; ++m) PTI_TRY(ptiNewMatrix(mats[m], X->ndims[m], R));
    auto sink = [&](uint32_t m, const float *d, uint32_t stride) -> int {
        PTI_CUDA(cudaMemcpyAsync(mats[m]->values, d, (size_t)X->ndims[m] * stride * 4, cudaMemcpyDeviceToHost, s),
                 mod);
        return 0;
    };
    double fit = 0.0;
    int r = host_cpd(&t, R, niters, tol, k->lambda, &fit, sink, s);
    if (r) {
        for (uint32_t m = 0; m <= N; ++m) {
            if (m < N) ptiFreeMatrix(mats[m]);
            std::free(mats[m]);
        }
        std::free(mats);
        return r;
    }
    // ktensor->factors = mats with mats[N] released (cpd.c:200-205)
    k->factors = mats;
    k->fit = fit;
    return 0;
}

int cpd_hicoo_entry(const ptiSparseTensorHiCOO *H, ptiIndex R, ptiIndex niters, double tol, ptiRankKruskalTensor *k)
{
    const char *mod = "B200 HiCOO CPD-ALS";
    PTI_CHECK(H && k && k->lambda, PTIERR_VALUE_ERROR, mod, "null tensor or Kruskal tensor");
    PTI_CHECK(R >= 1 && R <= 248, PTIERR_VALUE_ERROR, mod, "rank must be in [1, 248] for ptiRankMatrix");
    cudaStream_t s = sync_stream();
    ptiB200Tensor t;
    PTI_TRY(upload_hicoo(&t, H, s));
    const uint32_t N = H->nmodes;
    ptiRankMatrix **mats = static_cast<ptiRankMatrix **>(std::calloc(N + 1, sizeof(ptiRankMatrix *)));
    for (uint32_t m = 0; m <= N; ++m) mats[m] = static_cast<ptiRankMatrix *>(std::calloc(1, sizeof(ptiRankMatrix)));
    for (uint32_t m = 0; m < N; ++m) PTI_TRY(ptiNewRankMatrix(mats[m], H->ndims[m], (ptiElementIndex)R));
    auto sink = [&](uint32_t m, const float *d, uint32_t stride) -> int {
        PTI_CUDA(cudaMemcpyAsync(mats[m]->values, d, (size_t)H->ndims[m] * stride * 4, cudaMemcpyDeviceToHost, s),
                 mod);
        return 0;
    };
    double fit = 0.0;
    int r = host_cpd(&t, R, niters, tol, k->lambda, &fit, sink, s);
    if (r) {
        for (uint32_t m = 0; m <= N; ++m) {
            if (m < N) ptiFreeRankMatrix(mats[m]);
            std::free(mats[m]);
        }
        std::free(mats);
        return r;
    }
    k->factors = mats;
    k->fit = fit;
    return 0;
}

// ---------------------------------------------------------------------------
// The reference's dense ALS helpers and its ALS step with caller-seeded
// factors, as GPU calls on host matrices.  Each copies its operands to the
// device, runs there and copies the results back (the calls are small; a
// caller that keeps everything on the device uses ptiB200CpdAls).
// ---------------------------------------------------------------------------

// Grams as the reference keeps them: R x stride FP32, only the row-major
// upper triangle (i <= j) guaranteed written -- the part its ssyrk_('L') calls
// fill (src/sptensor/cpd.c:68,128).  out32 = the FP32 product of `count`
// Grams in the given order, mirrored to a full symmetric matrix
// (src/matrix/matrix.c:340-385); out64 = the same product in FP64 (R x R).
__global__ void tri_hadamard_kernel(const float *grams, uint32_t count, uint32_t R, uint32_t stride, float *out32,
                                    double *out64)
{
    for (uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
        const uint32_t i = e / R, j = e % R;
        const uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
        float v = 1.f;
        double w = 1.0;
        for (uint32_t k = 0; k < count; ++k) {
            const float gk = grams[(size_t)k * R * stride + (size_t)lo * stride + hi];
            v *= gk;
            w *= (double)gk;
        }
        if (out32) out32[(size_t)i * stride + j] = v;
        if (out64) out64[e] = w;
    }
}

// FP64 column statistics of a matrix: sums of squares and the largest
// positive entry (int bits of the FP32 value; 0 when there is none).
__global__ void colstat_kernel(const float *A, uint32_t I, uint32_t R, uint32_t stride, double *colsq, int *colmax)
{
    extern __shared__ double s_sq[];
    int *s_mx = reinterpret_cast<int *>(s_sq + R);
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        s_sq[c] = 0.0;
        s_mx[c] = 0;
    }
    __syncthreads();
    const uint64_t total = (uint64_t)I * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(e % stride);
        if (c >= R) continue;
        const float v = A[e];
        atomicAdd(&s_sq[c], (double)v * (double)v);
        if (v > 0.f) atomicMax(&s_mx[c], __float_as_int(v));
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        atomicAdd(&colsq[c], s_sq[c]);
        atomicMax(&colmax[c], s_mx[c]);
    }
}

// A[:, c] /= lambda[c] for the first R columns (pad columns untouched).
__global__ void div_cols_kernel(float *A, uint32_t I, uint32_t R, uint32_t stride, const float *lambda)
{
    const uint64_t total = (uint64_t)I * stride;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(e % stride);
        if (c < R) A[e] = A[e] / lambda[c];
    }
}

// |lambda^T (Hadamard_m G_m) lambda| over N Grams read from their row-major
// upper triangles (FP64), and the FP32 Hadamard product, full symmetric, into
// prod (the reference's scratch ata[nmodes], src/ktensor/ktensor.c:105-147).
__global__ void kruskal_normsq_kernel(const float *grams, uint32_t N, uint32_t R, uint32_t stride, const float *lambda,
                                      float *prod, double *out)
{
    __shared__ double s_part[32];
    double s = 0.0;
    for (uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
        const uint32_t i = e / R, j = e % R;
        const uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
        float v = 1.f;
        double w = 1.0;
        for (uint32_t k = 0; k < N; ++k) {
            const float gk = grams[(size_t)k * R * stride + (size_t)lo * stride + hi];
            v *= gk;
            w *= (double)gk;
        }
        if (prod) prod[(size_t)i * stride + j] = v;
        s += w * (double)lambda[i] * (double)lambda[j];
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += s_part[w];
        out[0] = fabs(t);
    }
}

namespace {

unsigned rows_grid_for(uint64_t items)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + 255) / 256, (uint64_t)sm_count() * 4));
}

// Device copy of the first `rows` rows (stride floats each) of host matrices,
// laid out one after another.
template <class Mat>
int upload_mats(DevBuf &buf, Mat *const *mats, const uint32_t *which, uint32_t count, uint32_t rows,
                uint32_t stride, cudaStream_t s, const char *mod)
{
    const size_t one = (size_t)rows * stride;
    PTI_CUDA(buf.alloc(padded(std::max<size_t>(1, count * one) * 4), s), mod);
    for (uint32_t k = 0; k < count; ++k)
        if (one)
            PTI_CUDA(cudaMemcpyAsync(buf.as<float>() + k * one, mats[which ? which[k] : k]->values, one * 4,
                                     cudaMemcpyHostToDevice, s),
                     mod);
    return 0;
}

// Grams aTa[0..nmodes] (R x R, one stride): same rank, stride and row count,
// as the reference asserts (src/matrix/matrix.c:345-348).
template <class Mat>
int check_grams(uint32_t nmodes, Mat **aTa, uint32_t upto, const char *mod)
{
    PTI_CHECK(aTa && nmodes >= 1, PTIERR_VALUE_ERROR, mod, "null matrices");
    for (uint32_t m = 0; m <= upto; ++m) PTI_CHECK(aTa[m] && aTa[m]->values, PTIERR_VALUE_ERROR, mod, "null matrix");
    const uint32_t R = aTa[0]->ncols, st = aTa[0]->stride;
    PTI_CHECK(R >= 1 && st >= R && aTa[0]->nrows >= R, PTIERR_SHAPE_MISMATCH, mod, "Gram must be rank x rank");
    for (uint32_t m = 1; m <= upto; ++m)
        PTI_CHECK((uint32_t)aTa[m]->ncols == R && (uint32_t)aTa[m]->stride == st && aTa[m]->nrows == aTa[0]->nrows,
                  PTIERR_SHAPE_MISMATCH, mod, "Grams differ in shape");
    return 0;
}

// ptiMatrixDotMulSeqTriangle, and with rhs the solve of ptiMatrixSolveNormals
// (src/matrix/matrix_solver.c:32-83): rhs <- rhs (Hadamard_{k != mode} aTa_k)^{-1}.
// aTa[nmodes] receives the FP32 Hadamard product, full symmetric.  The solve
// factors the FP64 product of the same Grams (Cholesky; Gauss-Jordan if it is
// not positive definite, as the reference falls back to sgesv; a singular
// matrix leaves rhs unchanged, as a failed sgesv does).
template <class Mat>
int normals(uint32_t mode, uint32_t nmodes, Mat **aTa, Mat *rhs, const char *mod)
{
    PTI_TRY(check_grams(nmodes, aTa, nmodes, mod));
    PTI_CHECK(mode < nmodes, PTIERR_VALUE_ERROR, mod, "mode out of range");
    const uint32_t R = aTa[0]->ncols, stride = aTa[0]->stride;
    if (rhs) {
        PTI_CHECK(rhs->values || rhs->nrows == 0, PTIERR_VALUE_ERROR, mod, "null right-hand side");
        PTI_CHECK((uint32_t)rhs->ncols == R && (uint32_t)rhs->stride == stride, PTIERR_SHAPE_MISMATCH, mod,
                  "right-hand side must have the Grams' rank and stride");
        PTI_CHECK(R <= (uint32_t)kMaxCpdRank, PTIERR_VALUE_ERROR, mod, "rank must be at most 128");
    }
    cudaStream_t s = sync_stream();
    std::vector<uint32_t> order;
    for (uint32_t m = 1; m < nmodes; ++m) order.push_back((mode + m) % nmodes);
    DevBuf grams, out32, out64;
    PTI_TRY(upload_mats(grams, aTa, order.data(), (uint32_t)order.size(), R, stride, s, mod));
    PTI_TRY(upload_mats(out32, aTa, &nmodes, 1, R, stride, s, mod));
    if (rhs) PTI_CUDA(out64.alloc(padded((size_t)R * R * 8), s), mod);
    tri_hadamard_kernel<<<1, 256, 0, s>>>(grams.as<float>(), (uint32_t)order.size(), R, stride, out32.as<float>(),
                                          rhs ? out64.as<double>() : nullptr);
    PTI_CUDA(cudaGetLastError(), mod);
    PTI_CUDA(cudaMemcpyAsync(aTa[nmodes]->values, out32.ptr, (size_t)R * stride * 4, cudaMemcpyDeviceToHost, s), mod);
    if (rhs && rhs->nrows) {
        const uint32_t I = rhs->nrows;
        DevBuf W, work, flag, Min, Aout, stats;
        PTI_CUDA(W.alloc(padded((size_t)R * R * 8), s), mod);
        PTI_CUDA(flag.alloc(64, s), mod);
        // the inverse kernels multiply the Grams of every mode but `mode`; with
        // the one product matrix as "mode 0 of two", that is the product itself
        if (R <= 32) {
            gram_inverse_small_kernel<<<1, 256, 0, s>>>(out64.as<double>(), 2, R, 1, W.as<double>(), flag.as<int>());
        } else {
            PTI_CUDA(work.alloc(padded((size_t)3 * R * R * 8), s), mod);
            gram_inverse_kernel<<<1, 256, 0, s>>>(out64.as<double>(), 2, R, 1, W.as<double>(), work.as<double>(),
                                                  flag.as<int>());
        }
        PTI_CUDA(Min.alloc(padded((size_t)I * stride * 4), s), mod);
        PTI_CUDA(Aout.alloc(padded((size_t)I * stride * 4), s), mod);
        PTI_CUDA(stats.alloc(padded((size_t)R * 12 + 64), s), mod);
        PTI_CUDA(cudaMemsetAsync(stats.ptr, 0, (size_t)R * 12, s), mod);
        PTI_CUDA(cudaMemcpyAsync(Min.ptr, rhs->values, (size_t)I * stride * 4, cudaMemcpyHostToDevice, s), mod);
        const size_t solve_smem = (size_t)R * R * 8 + (size_t)R * 12;
        PTI_CUDA(cudaFuncSetAttribute(solve_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem),
                 mod);
        solve_rows_kernel<<<rows_grid_for((uint64_t)I * stride), 256, solve_smem, s>>>(
            Min.as<float>(), W.as<double>(), I, R, stride, Aout.as<float>(), stats.as<double>(),
            reinterpret_cast<int *>(stats.as<double>() + R));
        PTI_CUDA(cudaGetLastError(), mod);
        int hflag = 0;
        PTI_CUDA(cudaMemcpyAsync(&hflag, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
        if (hflag != 2)
            PTI_CUDA(cudaMemcpyAsync(rhs->values, Aout.ptr, (size_t)I * stride * 4, cudaMemcpyDeviceToHost, s), mod);
    }
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

// ptiMatrix2Norm (use_2norm) / ptiMatrixMaxNorm (src/matrix/matrix.c:389-553):
// lambda = column 2-norms, or max(largest entry, 1); columns divided by it.
template <class Mat>
int col_normalize(Mat *A, float *lambda, int use_2norm, const char *mod)
{
    PTI_CHECK(A && lambda && (A->values || A->nrows == 0), PTIERR_VALUE_ERROR, mod, "null argument");
    const uint32_t I = A->nrows, R = A->ncols, stride = A->stride;
    PTI_CHECK(stride >= R, PTIERR_SHAPE_MISMATCH, mod, "stride below ncols");
    if (R == 0) return 0;
    cudaStream_t s = sync_stream();
    DevBuf dA, stats, lam;
    PTI_CUDA(dA.alloc(padded(std::max<size_t>(1, (size_t)I * stride) * 4), s), mod);
    PTI_CUDA(stats.alloc(padded((size_t)R * 12 + 64), s), mod);
    PTI_CUDA(lam.alloc(padded((size_t)R * 4), s), mod);
    PTI_CUDA(cudaMemsetAsync(stats.ptr, 0, (size_t)R * 12, s), mod);
    double *colsq = stats.as<double>();
    int *colmax = reinterpret_cast<int *>(colsq + R);
    if (I) {
        PTI_CUDA(cudaMemcpyAsync(dA.ptr, A->values, (size_t)I * stride * 4, cudaMemcpyHostToDevice, s), mod);
        colstat_kernel<<<rows_grid_for((uint64_t)I * stride), 256, (size_t)R * 12, s>>>(dA.as<float>(), I, R, stride,
                                                                                       colsq, colmax);
    }
    lambda_kernel<<<1, 128, 0, s>>>(colsq, colmax, R, use_2norm, lam.as<float>());
    if (I) div_cols_kernel<<<rows_grid_for((uint64_t)I * stride), 256, 0, s>>>(dA.as<float>(), I, R, stride,
                                                                              lam.as<float>());
    PTI_CUDA(cudaGetLastError(), mod);
    if (I) PTI_CUDA(cudaMemcpyAsync(A->values, dA.ptr, (size_t)I * stride * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaMemcpyAsync(lambda, lam.ptr, (size_t)R * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

// GetFinalLambda (src/matrix/matrix.c:556-572): every factor's columns to unit
// 2-norm, lambda multiplied by the norms.
template <class Mat>
int final_lambda(uint32_t rank, uint32_t nmodes, Mat **mats, float *lambda, const char *mod)
{
    PTI_CHECK(mats && lambda, PTIERR_VALUE_ERROR, mod, "null argument");
    cudaStream_t s = sync_stream();
    DevBuf lam, colsq;
    PTI_CUDA(lam.alloc(padded((size_t)rank * 4), s), mod);
    PTI_CUDA(colsq.alloc(padded((size_t)rank * 8), s), mod);
    PTI_CUDA(cudaMemcpyAsync(lam.ptr, lambda, (size_t)rank * 4, cudaMemcpyHostToDevice, s), mod);
    for (uint32_t m = 0; m < nmodes; ++m) {
        Mat *A = mats[m];
        PTI_CHECK(A && (uint32_t)A->ncols == rank && A->stride >= rank && (A->values || !A->nrows),
                  PTIERR_SHAPE_MISMATCH, mod, "factor must have `rank` columns");
        const uint32_t I = A->nrows, stride = A->stride;
        DevBuf dA;
        PTI_CUDA(dA.alloc(padded(std::max<size_t>(1, (size_t)I * stride) * 4), s), mod);
        PTI_CUDA(cudaMemsetAsync(colsq.ptr, 0, (size_t)rank * 8, s), mod);
        if (I) {
            PTI_CUDA(cudaMemcpyAsync(dA.ptr, A->values, (size_t)I * stride * 4, cudaMemcpyHostToDevice, s), mod);
            colsq_kernel<<<rows_grid_for((uint64_t)I * stride), 256, (size_t)rank * 8, s>>>(dA.as<float>(), I, rank,
                                                                                           stride, colsq.as<double>());
        }
        final_scale_kernel<<<rows_grid_for((uint64_t)std::max<uint32_t>(I, 1) * stride), 256, 0, s>>>(
            dA.as<float>(), I, rank, stride, colsq.as<double>(), lam.as<float>(), 1);
        PTI_CUDA(cudaGetLastError(), mod);
        if (I) PTI_CUDA(cudaMemcpyAsync(A->values, dA.ptr, (size_t)I * stride * 4, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
    }
    PTI_CUDA(cudaMemcpyAsync(lambda, lam.ptr, (size_t)rank * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

// lambda^T (Hadamard_m ata_m) lambda (src/ktensor/ktensor.c:105-147) from the
// Grams' row-major upper triangles -- the triangle the reference's ssyrk_
// calls write; its own loop reads the other one.  ata[nmodes] receives the
// FP32 Hadamard product.  NaN on bad arguments (last error set).
template <class Mat>
double kruskal_normsq(uint32_t nmodes, const float *lambda, Mat **ata, const char *mod)
{
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (!lambda || check_grams(nmodes, ata, nmodes, mod) != 0) {
        if (!lambda) complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__, "null lambda");
        return nan;
    }
    const uint32_t R = ata[0]->ncols, stride = ata[0]->stride;
    cudaStream_t s = sync_stream();
    DevBuf grams, prod, lam, out;
    double h = nan;
    if (upload_mats(grams, ata, (const uint32_t *)nullptr, nmodes, R, stride, s, mod) != 0 ||
        upload_mats(prod, ata, &nmodes, 1, R, stride, s, mod) != 0 || lam.alloc(padded((size_t)R * 4), s) != cudaSuccess ||
        out.alloc(64, s) != cudaSuccess) {
        complain(mod, PTIERR_CUDA_ERROR, __FILE__, __LINE__, "device allocation or copy failed");
        return nan;
    }
    cudaMemcpyAsync(lam.ptr, lambda, (size_t)R * 4, cudaMemcpyHostToDevice, s);
    kruskal_normsq_kernel<<<1, 256, 0, s>>>(grams.as<float>(), nmodes, R, stride, lam.as<float>(), prod.as<float>(),
                                            out.as<double>());
    cudaMemcpyAsync(ata[nmodes]->values, prod.ptr, (size_t)R * stride * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h, out.ptr, 8, cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        complain(mod, PTIERR_CUDA_ERROR + (int)e, __FILE__, __LINE__, cudaGetErrorString(e));
        return nan;
    }
    return h;
}

// sum_r lambda_r sum_i A_{N-1}[i, r] M[i, r], with M = mats[nmodes] the last
// MTTKRP output (src/ktensor/ktensor.c:152-240), FP64.
template <class Mat>
double kruskal_inner(uint32_t nmodes, const float *lambda, Mat **mats, const char *mod)
{
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (!mats || !lambda || nmodes < 1 || !mats[nmodes - 1] || !mats[nmodes] ||
        mats[nmodes - 1]->ncols != mats[nmodes]->ncols || mats[nmodes - 1]->stride != mats[nmodes]->stride) {
        complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__, "bad factor or MTTKRP matrix");
        return nan;
    }
    const uint32_t I = mats[nmodes - 1]->nrows, R = mats[nmodes - 1]->ncols, stride = mats[nmodes - 1]->stride;
    if (I == 0 || R == 0) return 0.0;
    cudaStream_t s = sync_stream();
    DevBuf A, M, lam, out;
    double h = nan;
    if (A.alloc(padded((size_t)I * stride * 4), s) != cudaSuccess ||
        M.alloc(padded((size_t)I * stride * 4), s) != cudaSuccess || lam.alloc(padded((size_t)R * 4), s) != cudaSuccess ||
        out.alloc(64, s) != cudaSuccess) {
        complain(mod, PTIERR_CUDA_ERROR, __FILE__, __LINE__, "device allocation failed");
        return nan;
    }
    cudaMemcpyAsync(A.ptr, mats[nmodes - 1]->values, (size_t)I * stride * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(M.ptr, mats[nmodes]->values, (size_t)I * stride * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(lam.ptr, lambda, (size_t)R * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(out.ptr, 0, 8, s);
    inner_kernel<<<rows_grid_for((uint64_t)I * stride), 256, 0, s>>>(A.as<float>(), M.as<float>(), I, R, stride,
                                                                     lam.as<float>(), out.as<double>());
    cudaMemcpyAsync(&h, out.ptr, 8, cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        complain(mod, PTIERR_CUDA_ERROR + (int)e, __FILE__, __LINE__, cudaGetErrorString(e));
        return nan;
    }
    return h;
}

// fit = 1 - sqrt(||X||^2 + norm - 2 inner) / ||X|| (src/ktensor/ktensor.c:77-99,
// the square root skipped when the residual is not positive)
double fit_from(double normX2, double norm_mats, double inner)
{
    double residual = normX2 + norm_mats - 2.0 * inner;
    if (residual > 0.0) residual = std::sqrt(residual);
    return 1.0 - residual / std::sqrt(normX2);
}

// The reference's ALS step on caller-seeded factors (CpdAlsStep,
// src/sptensor/cpd.c:32-160, and its HiCOO twin src/sptensor/hicoo/cpd.c:31):
// mats[0..N-1] hold the initial factors and receive the result (unit-norm
// columns, GetFinalLambda applied), lambda the weights, mats[N] the last
// MTTKRP output (mode N-1 of the last iteration).  Returns the last fit, NaN
// on error (last error set).
template <class Mat>
double cpd_step(ptiB200Tensor &t, uint32_t rank, uint32_t niters, double tol, Mat **mats, float *lambda,
                const char *mod)
{
    const double nan = std::numeric_limits<double>::quiet_NaN();
    const uint32_t N = t.nmodes;
    auto fail = [&](const char *why) {
        complain(mod, PTIERR_SHAPE_MISMATCH, __FILE__, __LINE__, why);
        return nan;
    };
    if (!mats || !lambda) return fail("null factors or lambda");
    for (uint32_t m = 0; m <= N; ++m)
        if (!mats[m] || !mats[m]->values) return fail("null factor matrix");
    const uint32_t stride = mats[0]->stride;
    for (uint32_t m = 0; m < N; ++m)
        if (mats[m]->nrows != t.ndims[m] || (uint32_t)mats[m]->ncols != rank || (uint32_t)mats[m]->stride != stride)
            return fail("factor m must be ndims[m] x rank, all with one stride");
    if ((uint32_t)mats[N]->stride != stride || std::max<uint32_t>(mats[N]->cap, mats[N]->nrows) < t.ndims[N - 1])
        return fail("mats[nmodes] must hold ndims[nmodes-1] rows of the factors' stride");
    cudaStream_t s = sync_stream();
    DevBuf A[kMaxModes], lam, Mlast;
    float *ptrs[kMaxModes];
    for (uint32_t m = 0; m < N; ++m) {
        const size_t n = (size_t)t.ndims[m] * stride;
        if (A[m].alloc(padded(std::max<size_t>(n, 1) * 4), s) != cudaSuccess ||
            (n && cudaMemcpyAsync(A[m].ptr, mats[m]->values, n * 4, cudaMemcpyHostToDevice, s) != cudaSuccess))
            return fail("device copy of the factors failed");
        ptrs[m] = A[m].as<float>();
    }
    if (lam.alloc(padded((size_t)rank * 4), s) != cudaSuccess ||
        Mlast.alloc(padded(std::max<size_t>(1, (size_t)t.ndims[N - 1] * stride) * 4), s) != cudaSuccess)
        return fail("device allocation failed");
    CpdOptions opt;
    opt.R = rank;
    opt.niters = niters;
    opt.tol = tol;
    opt.m_last = Mlast.as<float>();
    CpdResult res;
    if (cpd_device(&t, ptrs, stride, lam.as<float>(), opt, res, s) != 0) return nan;
    for (uint32_t m = 0; m < N; ++m)
        if (t.ndims[m])
            cudaMemcpyAsync(mats[m]->values, A[m].ptr, (size_t)t.ndims[m] * stride * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(lambda, lam.ptr, (size_t)rank * 4, cudaMemcpyDeviceToHost, s);
    if (res.iters && t.ndims[N - 1]) {
        cudaMemcpyAsync(mats[N]->values, Mlast.ptr, (size_t)t.ndims[N - 1] * stride * 4, cudaMemcpyDeviceToHost, s);
        mats[N]->nrows = t.ndims[N - 1];
    }
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        complain(mod, PTIERR_CUDA_ERROR + (int)e, __FILE__, __LINE__, cudaGetErrorString(e));
        return nan;
    }
    return res.iters ? res.fits.back() : 0.0;
}

double cpd_step_coo(const ptiSparseTensor *X, uint32_t rank, uint32_t niters, double tol, ptiMatrix **mats,
                    float *lambda)
{
    const char *mod = "CpdAlsStep";
    if (!X) {
        complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__, "null tensor");
        return std::numeric_limits<double>::quiet_NaN();
    }
    ptiB200Tensor t;
    if (upload_coo(&t, X, sync_stream()) != 0) return std::numeric_limits<double>::quiet_NaN();
    return cpd_step(t, rank, niters, tol, mats, lambda, mod);
}

double cpd_step_hicoo(const ptiSparseTensorHiCOO *H, uint32_t rank, uint32_t niters, double tol, ptiRankMatrix **mats,
                      float *lambda)
{
    const char *mod = "CpdAlsStepHiCOO";
    if (!H) {
        complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__, "null tensor");
        return std::numeric_limits<double>::quiet_NaN();
    }
    ptiB200Tensor t;
    if (upload_hicoo(&t, H, sync_stream()) != 0) return std::numeric_limits<double>::quiet_NaN();
    return cpd_step(t, rank, niters, tol, mats, lambda, mod);
}

double normsq_values(const float *vals, uint64_t nnz, const char *mod)
{
    if (nnz == 0) return 0.0;
    cudaStream_t s = sync_stream();
    DevBuf v, acc;
    double h = std::numeric_limits<double>::quiet_NaN();
    if (!vals || v.alloc(padded(nnz * 4), s) != cudaSuccess || acc.alloc(64, s) != cudaSuccess) {
        complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__, "null values or device allocation failed");
        return h;
    }
    cudaMemcpyAsync(v.ptr, vals, nnz * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(acc.ptr, 0, 8, s);
    sumsq_kernel<<<rows_grid_for(nnz), 256, 0, s>>>(v.as<float>(), nnz, acc.as<double>());
    cudaMemcpyAsync(&h, acc.ptr, 8, cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        complain(mod, PTIERR_CUDA_ERROR + (int)e, __FILE__, __LINE__, cudaGetErrorString(e));
        return std::numeric_limits<double>::quiet_NaN();
    }
    return h;
}

}  // namespace
}  // namespace
}  // namespace pti

extern "C" {

int ptiCpdAls(ptiSparseTensor const *const ptien, ptiIndex const rank, ptiIndex const niters, double const tol,
              ptiKruskalTensor *ktensor)
{
    return pti::cpd_coo_entry(ptien, rank, niters, tol, ktensor);
}
int ptiOmpCpdAls(ptiSparseTensor const *const ptien, ptiIndex const rank, ptiIndex const niters, double const tol,
                 const int tk, const int use_reduce, ptiKruskalTensor *ktensor)
{
    (void)tk;
    (void)use_reduce;
    return pti::cpd_coo_entry(ptien, rank, niters, tol, ktensor);
}
int ptiCudaCpdAls(ptiSparseTensor const *const ptien, ptiIndex const rank, ptiIndex const niters, double const tol,
                  ptiKruskalTensor *ktensor)
{
    return pti::cpd_coo_entry(ptien, rank, niters, tol, ktensor);
}
int ptiCpdAlsHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiIndex const rank, ptiIndex const niters,
                   double const tol, ptiRankKruskalTensor *ktensor)
{
    return pti::cpd_hicoo_entry(hitsr, rank, niters, tol, ktensor);
}
int ptiOmpCpdAlsHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiIndex const rank, ptiIndex const niters,
                      double const tol, const int tk, const int tb, int balanced, ptiRankKruskalTensor *ktensor)
{
    (void)tk;
    (void)tb;
    (void)balanced;
    return pti::cpd_hicoo_entry(hitsr, rank, niters, tol, ktensor);
}

int ptiB200CpdAls(ptiB200Tensor *t, ptiIndex rank, ptiIndex niters, double tol, int precision, ptiIndex fp32_sweeps,
                  float *const *dev_factors, ptiIndex stride, float *dev_lambda, double *fits, ptiIndex *iters_done,
                  void *stream)
{
    return ptiB200CpdAlsCheckpoint(t, rank, niters, tol, precision, fp32_sweeps, dev_factors, stride, dev_lambda,
                                   fits, iters_done, nullptr, 0, 0, stream);
}

int ptiB200CpdAlsCheckpoint(ptiB200Tensor *t, ptiIndex rank, ptiIndex niters, double tol, int precision,
                            ptiIndex fp32_sweeps, float *const *dev_factors, ptiIndex stride, float *dev_lambda,
                            double *fits, ptiIndex *iters_done, const char *ckpt_path, ptiIndex ckpt_every,
                            int resume, void *stream)
{
    using namespace pti;
    PTI_CHECK(t && dev_factors && dev_lambda, PTIERR_VALUE_ERROR, "B200 CPD-ALS", "null argument");
    PTI_CHECK(!resume || ckpt_path, PTIERR_VALUE_ERROR, "B200 CPD-ALS", "resume needs a checkpoint path");
    CpdOptions opt;
    opt.R = rank;
    opt.niters = niters;
    opt.tol = tol;
    opt.precision = precision;
    opt.fp32_sweeps = fp32_sweeps;
    opt.ckpt_path = ckpt_path && *ckpt_path ? ckpt_path : nullptr;
    opt.ckpt_every = ckpt_every;
    opt.resume = resume != 0;
    CpdResult res;
    PTI_TRY(cpd_device(t, dev_factors, stride, dev_lambda, opt, res, static_cast<cudaStream_t>(stream)));
    if (fits)
        for (uint32_t i = 0; i < res.iters; ++i) fits[i] = res.fits[i];
    if (iters_done) *iters_done = res.iters;
    return 0;
}

double SparseTensorFrobeniusNormSquared(ptiSparseTensor const *const ptien)
{
    return ptien ? pti::normsq_values(ptien->values.data, ptien->nnz, "SparseTensorFrobeniusNormSquared") : 0.0;
}

double SparseTensorFrobeniusNormSquaredHiCOO(ptiSparseTensorHiCOO const *const hitsr)
{
    return hitsr ? pti::normsq_values(hitsr->values.data, hitsr->nnz, "SparseTensorFrobeniusNormSquaredHiCOO") : 0.0;
}

int ptiMatrixDotMulSeqTriangle(ptiIndex const mode, ptiIndex const nmodes, ptiMatrix **mats)
{
    return pti::normals<ptiMatrix>(mode, nmodes, mats, nullptr, "ptiMatrixDotMulSeqTriangle");
}
int ptiRankMatrixDotMulSeqTriangle(ptiIndex const mode, ptiIndex const nmodes, ptiRankMatrix **mats)
{
    return pti::normals<ptiRankMatrix>(mode, nmodes, mats, nullptr, "ptiRankMatrixDotMulSeqTriangle");
}
int ptiMatrixSolveNormals(ptiIndex const mode, ptiIndex const nmodes, ptiMatrix **aTa, ptiMatrix *rhs)
{
    using namespace pti;
    PTI_CHECK(rhs, PTIERR_VALUE_ERROR, "ptiMatrixSolveNormals", "null right-hand side");
    return normals<ptiMatrix>(mode, nmodes, aTa, rhs, "ptiMatrixSolveNormals");
}
int ptiRankMatrixSolveNormals(ptiIndex const mode, ptiIndex const nmodes, ptiRankMatrix **aTa, ptiRankMatrix *rhs)
{
    using namespace pti;
    PTI_CHECK(rhs, PTIERR_VALUE_ERROR, "ptiRankMatrixSolveNormals", "null right-hand side");
    return normals<ptiRankMatrix>(mode, nmodes, aTa, rhs, "ptiRankMatrixSolveNormals");
}
int ptiMatrix2Norm(ptiMatrix *const A, ptiValue *const lambda)
{
    return pti::col_normalize(A, lambda, 1, "ptiMatrix2Norm");
}
int ptiRankMatrix2Norm(ptiRankMatrix *const A, ptiValue *const lambda)
{
    return pti::col_normalize(A, lambda, 1, "ptiRankMatrix2Norm");
}
int ptiMatrixMaxNorm(ptiMatrix *const A, ptiValue *const lambda)
{
    return pti::col_normalize(A, lambda, 0, "ptiMatrixMaxNorm");
}
int ptiRankMatrixMaxNorm(ptiRankMatrix *const A, ptiValue *const lambda)
{
    return pti::col_normalize(A, lambda, 0, "ptiRankMatrixMaxNorm");
}
void GetFinalLambda(ptiIndex const rank, ptiIndex const nmodes, ptiMatrix **mats, ptiValue *const lambda)
{
    pti::final_lambda(rank, nmodes, mats, lambda, "GetFinalLambda");
}
void GetRankFinalLambda(ptiElementIndex const rank, ptiIndex const nmodes, ptiRankMatrix **mats,
                        ptiValue *const lambda)
{
    pti::final_lambda<ptiRankMatrix>(rank, nmodes, mats, lambda, "GetRankFinalLambda");
}

double KruskalTensorFrobeniusNormSquared(ptiIndex const nmodes, ptiValue const *const lambda, ptiMatrix **ata)
{
    return pti::kruskal_normsq(nmodes, lambda, ata, "KruskalTensorFrobeniusNormSquared");
}
double KruskalTensorFrobeniusNormSquaredRank(ptiIndex const nmodes, ptiValue const *const lambda, ptiRankMatrix **ata)
{
    return pti::kruskal_normsq(nmodes, lambda, ata, "KruskalTensorFrobeniusNormSquaredRank");
}
double SparseKruskalTensorInnerProduct(ptiIndex const nmodes, ptiValue const *const lambda, ptiMatrix **mats)
{
    return pti::kruskal_inner(nmodes, lambda, mats, "SparseKruskalTensorInnerProduct");
}
double SparseKruskalTensorInnerProductRank(ptiIndex const nmodes, ptiValue const *const lambda, ptiRankMatrix **mats)
{
    return pti::kruskal_inner(nmodes, lambda, mats, "SparseKruskalTensorInnerProductRank");
}
double KruskalTensorFit(ptiSparseTensor const *const ptien, ptiValue const *const lambda, ptiMatrix **mats,
                        ptiMatrix **ata)
{
    if (!ptien) return std::numeric_limits<double>::quiet_NaN();
    const uint32_t N = ptien->nmodes;
    return pti::fit_from(SparseTensorFrobeniusNormSquared(ptien), KruskalTensorFrobeniusNormSquared(N, lambda, ata),
                         SparseKruskalTensorInnerProduct(N, lambda, mats));
}
double KruskalTensorFitHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiValue const *const lambda,
                             ptiRankMatrix **mats, ptiRankMatrix **ata)
{
    if (!hitsr) return std::numeric_limits<double>::quiet_NaN();
    const uint32_t N = hitsr->nmodes;
    return pti::fit_from(SparseTensorFrobeniusNormSquaredHiCOO(hitsr),
                         KruskalTensorFrobeniusNormSquaredRank(N, lambda, ata),
                         SparseKruskalTensorInnerProductRank(N, lambda, mats));
}

double CpdAlsStep(ptiSparseTensor const *const ptien, ptiIndex const rank, ptiIndex const niters, double const tol,
                  ptiMatrix **mats, ptiValue *const lambda)
{
    return pti::cpd_step_coo(ptien, rank, niters, tol, mats, lambda);
}
double OmpCpdAlsStep(ptiSparseTensor const *const ptien, ptiIndex const rank, ptiIndex const niters, double const tol,
                     const int tk, const int use_reduce, ptiMatrix **mats, ptiMatrix **copy_mats,
                     ptiValue *const lambda)
{
    (void)tk;
    (void)use_reduce;
    (void)copy_mats;
    return pti::cpd_step_coo(ptien, rank, niters, tol, mats, lambda);
}
double CpdAlsStepHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiIndex const rank, ptiIndex const niters,
                       double const tol, ptiRankMatrix **mats, ptiValue *const lambda)
{
    return pti::cpd_step_hicoo(hitsr, rank, niters, tol, mats, lambda);
}
double OmpCpdAlsStepHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiIndex const rank, ptiIndex const niters,
                          double const tol, const int tk, const int tb, const int *par_iters, ptiRankMatrix **mats,
                          ptiRankMatrix ***copy_mats, ptiValue *const lambda, int balanced)
{
    (void)tk;
    (void)tb;
    (void)par_iters;
    (void)copy_mats;
    (void)balanced;
    return pti::cpd_step_hicoo(hitsr, rank, niters, tol, mats, lambda);
}

}  // extern "C"
