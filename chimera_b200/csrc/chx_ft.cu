// chx_ft.cu -- windowed FT of a batch of spectra as a dense contraction (A5).
//
// chi(R_m) = sum_k chi(k) B(k, R_m), B = w(k) k^kw dk/sqrt(pi) e^{-2ikR}: the
// reference's resample -> window -> FFT -> slice (exafs_gpu/fourier.py:75-80)
// written as one [rows x nk] x [nk x 2 nR] product against a precomputed basis
// (real and imaginary columns interleaved), so any R grid can be used.
//
// precision 0: FP64 SIMT tiles (the accuracy reference on the device).
// precision 1: FP32 SIMT tiles.
// precision 2: split-BF16 three-product on the tcgen05 tensor cores with FP32
//              accumulation in tensor memory (chx_ft_tc.cu).
// precision 3: TF32, one tcgen05 product, FP32 accumulation (chx_ft_tc.cu).
#include <algorithm>
#include "chx_common.cuh"

namespace chx {

int ft_batch_tc(const double *chi, int rows, int nk, const double *basis, int nR, double *out,
                void *scratch, int64_t scratch_bytes, cudaStream_t st, bool tf32);
int64_t ft_batch_tc_scratch(int rows, int nk, int nR, bool tf32);
int ft_sums_tc(const double *chi, int rows, int nk, const double *basis, int nR,
               const double *target, const double *weight, double s0, double *out4,
               void *scratch, int64_t scratch_bytes, cudaStream_t st, bool tf32);
int64_t ft_sums_tc_scratch(int rows, int nk, int nR, bool tf32);

// 64 x 64 output tile per CTA, 256 threads, 4 x 4 outputs per thread
template <typename T>
__global__ void __launch_bounds__(256) k_ft_simt(const double *__restrict__ A, int rows, int nk,
                                                 const double *__restrict__ B, int ncol,
                                                 double *__restrict__ C) {
    constexpr int TM = 64, TN = 64, TK = 16;
    __shared__ T sa[TK][TM + 1];
    __shared__ T sb[TK][TN + 1];
    int r0 = blockIdx.y * TM, c0 = blockIdx.x * TN;
    int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    T acc[4][4] = {};
    for (int k0 = 0; k0 < nk; k0 += TK) {
        for (int q = threadIdx.x; q < TK * TM; q += 256) {
            int kk = q % TK, rr = q / TK;
            int gr = r0 + rr, gk = k0 + kk;
            sa[kk][rr] = (gr < rows && gk < nk) ? (T)A[(long)gr * nk + gk] : (T)0;
        }
        for (int q = threadIdx.x; q < TK * TN; q += 256) {
            int kk = q / TN, cc = q % TN;
            int gk = k0 + kk, gc = c0 + cc;
            sb[kk][cc] = (gk < nk && gc < ncol) ? (T)B[(long)gk * ncol + gc] : (T)0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sa[kk][tr + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sb[kk][tc + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int gr = r0 + tr + 16 * i, gc = c0 + tc + 16 * j;
            if (gr < rows && gc < ncol) C[(long)gr * ncol + gc] = (double)acc[i][j];
        }
}

}  // namespace chx

using namespace chx;

extern "C" {

int64_t chx_ft_batch_scratch_bytes(int rows, int nk, int nR, int precision) {
    if (rows <= 0 || nk <= 0 || nR <= 0) return -1;
    if (precision == 2 || precision == 3) return ft_batch_tc_scratch(rows, nk, nR, precision == 3);
    return 0;
}

int chx_ft_batch(const double *chi, int rows, int nk, const double *basis, int nR,
                 int precision, double *out, void *scratch, int64_t scratch_bytes,
                 void *stream) {
    CHX_REQUIRE(chi && basis && out && rows > 0 && nk > 0 && nR > 0, "ft_batch: bad arguments");
    cudaStream_t st = as_stream(stream);
    int ncol = 2 * nR;
    dim3 grid((ncol + 63) / 64, (rows + 63) / 64);
    if (precision == 0) {
        k_ft_simt<double><<<grid, 256, 0, st>>>(chi, rows, nk, basis, ncol, out);
    } else if (precision == 1) {
        k_ft_simt<float><<<grid, 256, 0, st>>>(chi, rows, nk, basis, ncol, out);
    } else if (precision == 2 || precision == 3) {
        return ft_batch_tc(chi, rows, nk, basis, nR, out, scratch, scratch_bytes, st,
                           precision == 3);
    } else {
        set_error("ft_batch: bad precision %d", precision);
        return CHX_ERR_ARG;
    }
    CHX_CHECK_LAUNCH("ft_batch");
    return CHX_OK;
}

int64_t chx_ft_window_sums_scratch_bytes(int rows, int nk, int nR, int precision) {
    if (rows <= 0 || nk <= 0 || nR <= 0 || (precision != 2 && precision != 3)) return -1;
    return ft_sums_tc_scratch(rows, nk, nR, precision == 3);
}

int chx_ft_window_sums(const double *chi, int rows, int nk, const double *basis, int nR,
                       const double *target, const double *weight, double s0, int precision,
                       double *sums, void *scratch, int64_t scratch_bytes, void *stream) {
    CHX_REQUIRE(chi && basis && target && weight && sums && rows > 0 && nk > 0 && nR > 0,
                "ft_window_sums: bad arguments");
    CHX_REQUIRE(precision == 2 || precision == 3,
                "ft_window_sums: precision %d (the fused form is 2 or 3)", precision);
    return ft_sums_tc(chi, rows, nk, basis, nR, target, weight, s0, sums, scratch,
                      scratch_bytes, as_stream(stream), precision == 3);
}

}  // extern "C"
