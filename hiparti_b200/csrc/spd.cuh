// spd.cuh -- inverse of a small symmetric positive (semi)definite matrix in
// shared memory, by one CTA (the normal-equation solve of an ALS step).
#pragma once
#include <cstdint>

namespace pti {

// W = V^-1 for a symmetric R x R matrix (R <= 32) in FP64 shared memory, by
// the whole CTA.  Returns 0 (Cholesky), 1 (not positive definite: Gauss-Jordan
// elimination with partial pivoting, the counterpart of the reference's sgesv
// fallback, src/matrix/matrix_solver.c:66-80) or 2 (singular: W = identity, so
// the rows stay unsolved as when sgesv fails).
__device__ inline int spd_inverse(const double *V, double *L, double *Li, double *W, uint32_t R)
{
    __shared__ int s_bad, s_sing;
    __shared__ uint32_t s_piv;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint32_t RR = R * R;
    if (tid < 32) {
        // Cholesky V = L L^T by one warp: lane i owns row i of L
        int bad = 0;
        for (uint32_t j = 0; j < R; ++j) {
            double d = V[j * R + j];
            for (uint32_t k = 0; k < j; ++k) d -= L[j * R + k] * L[j * R + k];
            if (!(d > 0.0)) {
                bad = 1;
                break;
            }
            const double dj = sqrt(d);
            if (lane > j && lane < R) {
                double s = V[lane * R + j];
                for (uint32_t k = 0; k < j; ++k) s -= L[lane * R + k] * L[j * R + k];
                L[lane * R + j] = s / dj;
            }
            if (lane == j) L[j * R + j] = dj;
            __syncwarp();
        }
        if (lane == 0) s_bad = bad;
    }
    __syncthreads();
    if (!s_bad) {
        // Li = L^-1 (column c by thread c), then W = Li^T Li
        for (uint32_t c = tid; c < R; c += blockDim.x)
            for (uint32_t i = c; i < R; ++i) {
                double s = (i == c) ? 1.0 : 0.0;
                for (uint32_t k = c; k < i; ++k) s -= L[i * R + k] * Li[k * R + c];
                Li[i * R + c] = s / L[i * R + i];
            }
        __syncthreads();
        for (uint32_t e = tid; e < RR; e += blockDim.x) {
            const uint32_t p = e / R, q = e % R;
            double s = 0.0;
            for (uint32_t k = (p > q ? p : q); k < R; ++k) s += Li[k * R + p] * Li[k * R + q];
            W[e] = s;
        }
        __syncthreads();
        return 0;
    }
    // Gauss-Jordan on [V | I]: L holds V, Li holds I
    for (uint32_t e = tid; e < RR; e += blockDim.x) {
        L[e] = V[e];
        Li[e] = (e / R == e % R) ? 1.0 : 0.0;
    }
    if (tid == 0) s_sing = 0;
    __syncthreads();
    for (uint32_t j = 0; j < R; ++j) {
        if (tid == 0) {
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
            for (uint32_t c = tid; c < R; c += blockDim.x) {
                double t = L[j * R + c];
                L[j * R + c] = L[p * R + c];
                L[p * R + c] = t;
                t = Li[j * R + c];
                Li[j * R + c] = Li[p * R + c];
                Li[p * R + c] = t;
            }
        __syncthreads();
        const double piv = L[j * R + j];
        __syncthreads();
        for (uint32_t c = tid; c < R; c += blockDim.x) {
            L[j * R + c] /= piv;
            Li[j * R + c] /= piv;
        }
        __syncthreads();
        for (uint32_t e = tid; e < RR; e += blockDim.x) {
            const uint32_t i = e / R, c = e % R;
            if (i == j) continue;
            const double f = L[i * R + j];
            if (c != j) L[i * R + c] -= f * L[j * R + c];
            Li[i * R + c] -= f * Li[j * R + c];
        }
        __syncthreads();
        for (uint32_t i = tid; i < R; i += blockDim.x)
            if (i != j) L[i * R + j] = 0.0;
        __syncthreads();
    }
    const int sing = s_sing;
    for (uint32_t e = tid; e < RR; e += blockDim.x) W[e] = sing ? ((e / R == e % R) ? 1.0 : 0.0) : Li[e];
    __syncthreads();
    return sing ? 2 : 1;
}

}  // namespace pti
