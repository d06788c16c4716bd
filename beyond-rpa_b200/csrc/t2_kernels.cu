// Device kernels of the direct-ring T2 chain (rpa_THC_CC_T2 / rpa_CC_T2_v5,
// src/rpa/rpa_CC_Doubles.f90:491-984):
//   * batched blocked forward substitution L X = B (the (1 + Pi_u)^{-1}
//     factors of rpa_CC_IM_v5 come from the Cholesky factors of the energy);
//   * guess-vector generation, column normalisation (rpa_CC_NormalizeColumns,
//     rpa_CC_Doubles.f90:80-91), scalings, gathers and column norms.
#include <algorithm>

#include "kernels.h"

namespace rpa {

namespace {

// ----------------------------------------------------------------- TRSM
constexpr int TB = 64;     // block of the blocked substitution
constexpr int TCOLS = 64;  // right-hand sides per CTA

// X_b(j0:j0+nb, cols) <- L_b(j0:j0+nb, j0:j0+nb)^{-1} X_b(j0:j0+nb, cols)
constexpr size_t kTrsmSmem = sizeof(double) * (TB * (TB + 1) + TB * (TCOLS + 1));

__global__ void __launch_bounds__(TCOLS) trsm_diag_kernel(const double* L, int64_t ldl, int64_t sL, double* X,
                                                          int64_t ldx, int64_t sX, int n, int ncols, int j0) {
  extern __shared__ double trsm_smem[];
  auto Ls = reinterpret_cast<double(*)[TB + 1]>(trsm_smem);
  auto Xs = reinterpret_cast<double(*)[TCOLS + 1]>(trsm_smem + TB * (TB + 1));
  const int b = blockIdx.y;
  const double* Lb = L + (int64_t)b * sL;
  double* Xb = X + (int64_t)b * sX;
  const int nb = min(TB, n - j0);
  const int c0 = blockIdx.x * TCOLS;
  const int t = threadIdx.x;
  for (int idx = t; idx < TB * TB; idx += blockDim.x) {
    const int r = idx % TB, c = idx / TB;
    Ls[r][c] = (r < nb && c <= r) ? Lb[(int64_t)(j0 + r) + ldl * (j0 + c)] : 0.0;
  }
  for (int idx = t; idx < TB * TCOLS; idx += blockDim.x) {
    const int r = idx % TB, c = idx / TB;  // a warp reads contiguous rows of one column
    Xs[r][c] = (r < nb && c0 + c < ncols) ? Xb[(int64_t)(j0 + r) + ldx * (c0 + c)] : 0.0;
  }
  __syncthreads();
  // thread t solves column t
  for (int r = 0; r < nb; ++r) {
    double s = Xs[r][t];
    for (int m = 0; m < r; ++m) s -= Ls[r][m] * Xs[m][t];
    Xs[r][t] = s / Ls[r][r];
  }
  __syncthreads();
  for (int idx = t; idx < TB * TCOLS; idx += blockDim.x) {
    const int r = idx % TB, c = idx / TB;
    if (r < nb && c0 + c < ncols) Xb[(int64_t)(j0 + r) + ldx * (c0 + c)] = Xs[r][c];
  }
}

// X_b(j0:j0+nb, cols) <- L_b(j0:j0+nb, j0:j0+nb)^{-T} X_b(j0:j0+nb, cols)  (backward substitution)
__global__ void __launch_bounds__(TCOLS) trsm_diag_trans_kernel(const double* L, int64_t ldl, int64_t sL, double* X,
                                                                int64_t ldx, int64_t sX, int n, int ncols, int j0) {
  extern __shared__ double trsm_smem[];
  auto Ls = reinterpret_cast<double(*)[TB + 1]>(trsm_smem);
  auto Xs = reinterpret_cast<double(*)[TCOLS + 1]>(trsm_smem + TB * (TB + 1));
  const int b = blockIdx.y;
  const double* Lb = L + (int64_t)b * sL;
  double* Xb = X + (int64_t)b * sX;
  const int nb = min(TB, n - j0);
  const int c0 = blockIdx.x * TCOLS;
  const int t = threadIdx.x;
  for (int idx = t; idx < TB * TB; idx += blockDim.x) {
    const int r = idx % TB, c = idx / TB;
    Ls[r][c] = (r < nb && c <= r) ? Lb[(int64_t)(j0 + r) + ldl * (j0 + c)] : 0.0;
  }
  for (int idx = t; idx < TB * TCOLS; idx += blockDim.x) {
    const int r = idx % TB, c = idx / TB;
    Xs[r][c] = (r < nb && c0 + c < ncols) ? Xb[(int64_t)(j0 + r) + ldx * (c0 + c)] : 0.0;
  }
  __syncthreads();
  for (int r = nb - 1; r >= 0; --r) {
    double s = Xs[r][t];
    for (int m = r + 1; m < nb; ++m) s -= Ls[m][r] * Xs[m][t];
    Xs[r][t] = s / Ls[r][r];
  }
  __syncthreads();
  for (int idx = t; idx < TB * TCOLS; idx += blockDim.x) {
    const int r = idx % TB, c = idx / TB;
    if (r < nb && c0 + c < ncols) Xb[(int64_t)(j0 + r) + ldx * (c0 + c)] = Xs[r][c];
  }
}

// Adjoint accumulation for a group of frequencies, one warp per column ai:
//   dR(:,ai) (+)= sum_k 2 alpha f_k c_k(ai) (Y_k - R)(:,ai)
//   dD(ai)   (+)= sum_k alpha f_k dc_k/dD(ai) R(:,ai)^T (Y_k - R)(:,ai)
// f_k = w_k/(2 pi), c = D/(D^2+u^2), dc/dD = (u^2-D^2)/(D^2+u^2)^2.
__global__ void __launch_bounds__(256) grad_accum_kernel(const double* R, int64_t ldR, const double* Y, int64_t ldy,
                                                         int64_t sY, int NQ, int64_t nov, const double* D,
                                                         GradGroup gg, double* dR, int64_t lddR, double* dD,
                                                         int first) {
  const int64_t a = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= nov) return;
  const double d = D[a];
  double cfac[16], dfac[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if (k < gg.n) {
      const double den = d * d + gg.u2[k];
      cfac[k] = 2.0 * gg.alpha * gg.f[k] * d / den;
      dfac[k] = gg.alpha * gg.f[k] * (gg.u2[k] - d * d) / (den * den);
    } else {
      cfac[k] = dfac[k] = 0.0;
    }
  }
  double dot = 0.0;
  for (int q = lane; q < NQ; q += 32) {
    const double r = R[(int64_t)q + ldR * a];
    double g = first ? 0.0 : dR[(int64_t)q + lddR * a];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      if (k < gg.n) {
        const double m = Y[(int64_t)k * sY + (int64_t)q + ldy * a] - r;
        g += cfac[k] * m;
        dot += dfac[k] * r * m;
      }
    }
    dR[(int64_t)q + lddR * a] = g;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, off);
  if (lane == 0) dD[a] = (first ? 0.0 : dD[a]) + dot;
}

// Y_b = R for every b (strided copy of a column-major matrix)
__global__ void replicate_kernel(const double* R, int64_t ldR, int NQ, int64_t nov, double* Y, int64_t ldy,
                                 int64_t sY, int nb) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)NQ * nov) return;
  const int64_t q = idx % NQ, a = idx / NQ;
  const double r = R[q + ldR * a];
  for (int b = 0; b < nb; ++b) Y[(int64_t)b * sY + q + ldy * a] = r;
}

// Sums of squares of the off-diagonal (out[0]) and diagonal (out[1]) entries: kOffBlocks
// CTAs write partial sums to out[2 ...], the last kernel adds them in a fixed order.
constexpr int kOffBlocks = 120;
__global__ void __launch_bounds__(256) offdiag_kernel(const double* A, int64_t lda, int n, double* out) {
  __shared__ double so[256], sd[256];
  double o = 0.0, d = 0.0;
  const int64_t total = (int64_t)n * n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx % n, j = idx / n;
    const double v = A[i + lda * j];
    if (i == j) d += v * v;
    else o += v * v;
  }
  so[threadIdx.x] = o;
  sd[threadIdx.x] = d;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      so[threadIdx.x] += so[threadIdx.x + s];
      sd[threadIdx.x] += sd[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 + 2 * blockIdx.x] = so[0];
    out[3 + 2 * blockIdx.x] = sd[0];
  }
}

__global__ void offdiag_final_kernel(double* out) {
  if (threadIdx.x != 0) return;
  double o = 0.0, d = 0.0;
  for (int b = 0; b < kOffBlocks; ++b) {
    o += out[2 + 2 * b];
    d += out[3 + 2 * b];
  }
  out[0] = o;
  out[1] = d;
}

// ----------------------------------------------------------------- vectors
// uniform [-1/2, 1/2) guess vectors (the reference: random_number - 1/2)
__global__ void fill_uniform_kernel(double* X, int64_t rows, int64_t cols, int64_t ldx, uint64_t seed) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * cols) return;
  const int64_t i = idx % rows, j = idx / rows;
  const uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)idx));
  X[i + ldx * j] = (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

// column norms^2 (one block per column, fixed-order reduction)
__global__ void __launch_bounds__(256) col_sqnorm_kernel(const double* X, int64_t rows, int64_t ldx, double* out) {
  __shared__ double sh[256];
  const int64_t j = blockIdx.x;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < rows; i += blockDim.x) {
    const double v = X[i + ldx * j];
    s += v * v;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = sh[0];
}

// X(:, j) *= colscale(j)  (colscale given as 1/sqrt(norm2) when inv_sqrt)
__global__ void scale_cols_kernel(double* X, int64_t rows, int64_t cols, int64_t ldx, const double* s, int inv_sqrt) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * cols) return;
  const int64_t i = idx % rows, j = idx / rows;
  const double f = inv_sqrt ? 1.0 / sqrt(s[j]) : s[j];
  X[i + ldx * j] *= f;
}

// Y(k*NQ + q, ai) = R(q, ai) * f_k(ai), f_k = -alpha D/(D^2+u_k^2) * sqrt(w_k)
__global__ void chi_scale_kernel(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D, ChiGroup cg,
                                 double* Y, int64_t ldy) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)NQ * nov;
  if (idx >= total) return;
  const int64_t q = idx % NQ, a = idx / NQ;
  const double d = D[a];
  const double r = R[q + ldR * a];
  for (int k = 0; k < cg.n; ++k) {
    const double f = -cg.alpha * d / (d * d + cg.u2[k]) * cg.sqrtw[k];
    Y[(int64_t)k * NQ + q + ldy * a] = r * f;
  }
}

// dst(:, j) = src(:, perm[j])
__global__ void gather_cols_kernel(const double* src, int64_t lds, double* dst, int64_t ldd, int64_t rows,
                                   int64_t cols, const int* perm, const double* colscale) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * cols) return;
  const int64_t i = idx % rows, j = idx / rows;
  const double f = colscale ? colscale[j] : 1.0;
  dst[i + ldd * j] = src[i + lds * perm[j]] * f;
}

// A <- (A + A^T)/2
__global__ void symmetrize_avg_kernel(double* A, int64_t lda, int n) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int64_t i = idx % n, j = idx / n;
  if (i <= j) return;
  const double v = 0.5 * (A[i + lda * j] + A[j + lda * i]);
  A[i + lda * j] = v;
  A[j + lda * i] = v;
}

__global__ void mbpt3_build_kernel(const double* Ukl, const double* Dkl, const double* Av, int n, double* Amat,
                                   double* Bmat, double* Bsym) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int64_t m = idx % n, k = idx / n;  // element (m, k)
  const double d = Dkl[idx], u = Ukl[idx];
  Amat[idx] = Av[m] * d + d * Av[k];
  Bmat[idx] = d + 2.0 * u + 4.0 * u * Av[k];
  // symmetric part: (B_mk + B_km)/2, with D and U symmetric
  Bsym[idx] = d + 2.0 * u + 2.0 * u * (Av[k] + Av[m]);
}

__global__ void lyap_scale_kernel(double* Y, const double* mu, int n, int* bad) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int64_t m = idx % n, k = idx / n;
  const double den = mu[m] + mu[k];
  if (!(den > 0.0)) {
    atomicAdd(bad, 1);
    Y[idx] = 0.0;
    return;
  }
  Y[idx] /= den;
}

// dst column map[2c+1] = src column map[2c] (columns of `rows` doubles, contiguous), c < ncols.
__global__ void copy_columns_kernel(const double* src, double* dst, const int64_t* map, int64_t ncols, int rows) {
  const int64_t c = blockIdx.y * (int64_t)gridDim.x + blockIdx.x;
  if (c >= ncols) return;
  const double* s = src + map[2 * c] * rows;
  double* d = dst + map[2 * c + 1] * rows;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) d[r] = s[r];
}

// C = A o B (element-wise, rows x cols, column-major)
__global__ void hadamard_kernel(const double* A, int64_t lda, const double* B, int64_t ldb, int rows, int cols,
                                double* C, int64_t ldc) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)rows * cols) return;
  const int64_t r = idx % rows, c = idx / rows;
  C[r + ldc * c] = A[r + lda * c] * B[r + ldb * c];
}

// Partial sums of sum_{r,c} w(r) A(r,c) B(r,c) (w optional): kDotBlocks CTAs each write one
// partial to out[blockIdx.x]; the caller adds them in a fixed order.
constexpr int kDotBlocks = kDotPartials;
__global__ void __launch_bounds__(256) dot_partials_kernel(const double* A, int64_t lda, const double* B, int64_t ldb,
                                                           int rows, int cols, const double* w, double* out) {
  __shared__ double red[256];
  const int64_t total = (int64_t)rows * cols;
  double acc = 0.0;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx % rows, c = idx / rows;
    const double v = A[r + lda * c] * B[r + ldb * c];
    acc += w ? w[r] * v : v;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// Khatri-Rao block of the THC factors: YX(g, a + nv*ii) = Xa(g, a) * Xi(g, i0 + ii), ii < ni
// (rpa_THC_Rkab / rpa_THC_Rkai, src/rpa/rpa_THC.f90:374-426).
__global__ void khatri_rao_kernel(const double* Xa, int64_t ldXa, const double* Xi, int64_t ldXi, int ngrid, int nv,
                                  int i0, int ni, double* YX) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)ngrid * nv * ni;
  if (idx >= total) return;
  const int64_t g = idx % ngrid, col = idx / ngrid;
  const int64_t a = col % nv, ii = col / nv;
  YX[idx] = Xa[g + ldXa * a] * Xi[g + ldXi * (i0 + ii)];
}

// Khatri-Rao block of an ai column range: YX(g, c) = Xa(g, a) Xi(g, i) for ai = ai0 + c = a + nv i.
__global__ void khatri_rao_cols_kernel(const double* Xa, int64_t ldXa, const double* Xi, int64_t ldXi, int ngrid,
                                       int nv, int64_t ai0, int64_t ncols, double* YX) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)ngrid * ncols) return;
  const int64_t g = idx % ngrid, ai = ai0 + idx / ngrid;
  const int64_t a = ai % nv, i = ai / nv;
  YX[idx] = Xa[g + ldXa * a] * Xi[g + ldXi * i];
}

// dst[j] += src[j] (first: dst[j] = src[j])
__global__ void add_into_kernel(double* dst, const double* src, int64_t n, int first) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) dst[j] = first ? src[j] : dst[j] + src[j];
}

// A(i, i) += s * (*fro2) for i < n  (fro2: a device scalar, e.g. ||Y||_F^2)
__global__ void add_diag_scaled_kernel(double* A, int64_t lda, int n, double s, const double* fro2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(int64_t)i * (lda + 1)] += s * fro2[0];
}

// B = A^T (A rows x cols, column-major), 32 x 32 tiles through shared memory.
__global__ void transpose_kernel(const double* A, int64_t lda, int rows, int cols, double* B, int64_t ldb) {
  __shared__ double tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + threadIdx.x, c = c0 + i;
    tile[i][threadIdx.x] = (r < rows && c < cols) ? A[r + lda * c] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + threadIdx.x, r = r0 + i;  // B(c, r) = A(r, c)
    if (c < cols && r < rows) B[c + ldb * r] = tile[threadIdx.x][i];
  }
}

inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_trsm_lower_left(const double* L, int64_t ldl, int64_t sL, double* X, int64_t ldx, int64_t sX,
                                   int n, int ncols, int batch, cudaStream_t stream) {
  cudaError_t e0 = cudaFuncSetAttribute(trsm_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem);
  if (e0 != cudaSuccess) return e0;
  for (int j0 = 0; j0 < n; j0 += TB) {
    trsm_diag_kernel<<<dim3((ncols + TCOLS - 1) / TCOLS, batch), TCOLS, kTrsmSmem, stream>>>(L, ldl, sL, X, ldx, sX,
                                                                                             n, ncols, j0);
    ++g_launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int nb = min(TB, n - j0);
    const int rest = n - j0 - nb;
    if (rest <= 0) break;
    GemmF64Args g{};
    g.M = rest;
    g.N = ncols;
    g.K = nb;
    g.A = L + (int64_t)(j0 + nb) + ldl * j0;
    g.a_m = 1;
    g.a_k = ldl;
    g.sA = sL;
    g.B = X + j0;
    g.b_k = 1;
    g.b_n = ldx;
    g.sB = sX;
    g.C = X + (j0 + nb);
    g.ldc = ldx;
    g.sC = sX;
    g.alpha = -1.0;
    g.beta = 1.0;
    g.batch = batch;
    e = launch_gemm_f64(g, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_trsm_lower_trans_left(const double* L, int64_t ldl, int64_t sL, double* X, int64_t ldx,
                                         int64_t sX, int n, int ncols, int batch, cudaStream_t stream) {
  cudaError_t e0 =
      cudaFuncSetAttribute(trsm_diag_trans_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem);
  if (e0 != cudaSuccess) return e0;
  const int nblk = (n + TB - 1) / TB;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int j0 = bi * TB;
    trsm_diag_trans_kernel<<<dim3((ncols + TCOLS - 1) / TCOLS, batch), TCOLS, kTrsmSmem, stream>>>(
        L, ldl, sL, X, ldx, sX, n, ncols, j0);
    ++g_launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (j0 == 0) break;
    const int nb = min(TB, n - j0);
    // X(0:j0, :) -= L(j0:j0+nb, 0:j0)^T X(j0:j0+nb, :)
    GemmF64Args g{};
    g.M = j0;
    g.N = ncols;
    g.K = nb;
    g.A = L + j0;  // A(m, k) = L(j0 + k, m)
    g.a_m = ldl;
    g.a_k = 1;
    g.sA = sL;
    g.B = X + j0;
    g.b_k = 1;
    g.b_n = ldx;
    g.sB = sX;
    g.C = X;
    g.ldc = ldx;
    g.sC = sX;
    g.alpha = -1.0;
    g.beta = 1.0;
    g.batch = batch;
    e = launch_gemm_f64(g, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_grad_accum(const double* R, int64_t ldR, const double* Y, int64_t ldy, int64_t sY, int NQ,
                              int64_t nov, const double* D, const GradGroup& gg, double* dR, int64_t lddR, double* dD,
                              bool first, cudaStream_t stream) {
  grad_accum_kernel<<<(unsigned)((nov + 7) / 8), 256, 0, stream>>>(R, ldR, Y, ldy, sY, NQ, nov, D, gg, dR, lddR, dD,
                                                                   first ? 1 : 0);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_replicate(const double* R, int64_t ldR, int NQ, int64_t nov, double* Y, int64_t ldy, int64_t sY,
                             int nb, cudaStream_t stream) {
  replicate_kernel<<<blocks_for((int64_t)NQ * nov), 256, 0, stream>>>(R, ldR, NQ, nov, Y, ldy, sY, nb);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_copy_columns(const double* src, double* dst, const int64_t* map, int64_t ncols, int rows,
                                cudaStream_t stream) {
  if (ncols <= 0) return cudaSuccess;
  const unsigned gx = (unsigned)std::min<int64_t>(ncols, 65535);
  const unsigned gy = (unsigned)((ncols + gx - 1) / gx);
  copy_columns_kernel<<<dim3(gx, gy), 128, 0, stream>>>(src, dst, map, ncols, rows);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_hadamard(const double* A, int64_t lda, const double* B, int64_t ldb, int rows, int cols,
                            double* C, int64_t ldc, cudaStream_t stream) {
  hadamard_kernel<<<blocks_for((int64_t)rows * cols), 256, 0, stream>>>(A, lda, B, ldb, rows, cols, C, ldc);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_dot_partials(const double* A, int64_t lda, const double* B, int64_t ldb, int rows, int cols,
                                const double* w, double* out, cudaStream_t stream) {
  dot_partials_kernel<<<kDotBlocks, 256, 0, stream>>>(A, lda, B, ldb, rows, cols, w, out);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_khatri_rao(const double* Xa, int64_t ldXa, const double* Xi, int64_t ldXi, int ngrid, int nv,
                              int i0, int ni, double* YX, cudaStream_t stream) {
  const int64_t total = (int64_t)ngrid * nv * ni;
  khatri_rao_kernel<<<blocks_for(total), 256, 0, stream>>>(Xa, ldXa, Xi, ldXi, ngrid, nv, i0, ni, YX);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_khatri_rao_cols(const double* Xa, int64_t ldXa, const double* Xi, int64_t ldXi, int ngrid, int nv,
                                   int64_t ai0, int64_t ncols, double* YX, cudaStream_t stream) {
  const int64_t total = (int64_t)ngrid * ncols;
  khatri_rao_cols_kernel<<<blocks_for(total), 256, 0, stream>>>(Xa, ldXa, Xi, ldXi, ngrid, nv, ai0, ncols, YX);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_add_into(double* dst, const double* src, int64_t n, bool first, cudaStream_t stream) {
  add_into_kernel<<<blocks_for(n), 256, 0, stream>>>(dst, src, n, first ? 1 : 0);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_add_diag_scaled(double* A, int64_t lda, int n, double s, const double* fro2,
                                  cudaStream_t stream) {
  add_diag_scaled_kernel<<<blocks_for(n), 256, 0, stream>>>(A, lda, n, s, fro2);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_transpose(const double* A, int64_t lda, int rows, int cols, double* B, int64_t ldb,
                             cudaStream_t stream) {
  dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(A, lda, rows, cols, B, ldb);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_mbpt3_build(const double* Ukl, const double* Dkl, const double* Avec, int n, double* Amat,
                               double* Bmat, double* Bsym, cudaStream_t stream) {
  mbpt3_build_kernel<<<blocks_for((int64_t)n * n), 256, 0, stream>>>(Ukl, Dkl, Avec, n, Amat, Bmat, Bsym);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_lyap_scale(double* Y, const double* mu, int n, int* bad, cudaStream_t stream) {
  lyap_scale_kernel<<<blocks_for((int64_t)n * n), 256, 0, stream>>>(Y, mu, n, bad);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_offdiag(const double* A, int64_t lda, int n, double* out, cudaStream_t stream) {
  offdiag_kernel<<<kOffBlocks, 256, 0, stream>>>(A, lda, n, out);
  offdiag_final_kernel<<<1, 32, 0, stream>>>(out);
  g_launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_fill_uniform(double* X, int64_t rows, int64_t cols, int64_t ldx, uint64_t seed,
                                cudaStream_t stream) {
  if (rows * cols == 0) return cudaSuccess;
  fill_uniform_kernel<<<blocks_for(rows * cols), 256, 0, stream>>>(X, rows, cols, ldx, seed);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_col_sqnorm(const double* X, int64_t rows, int64_t cols, int64_t ldx, double* out,
                              cudaStream_t stream) {
  if (cols == 0) return cudaSuccess;
  col_sqnorm_kernel<<<(unsigned)cols, 256, 0, stream>>>(X, rows, ldx, out);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_scale_cols(double* X, int64_t rows, int64_t cols, int64_t ldx, const double* s, bool inv_sqrt,
                              cudaStream_t stream) {
  if (rows * cols == 0) return cudaSuccess;
  scale_cols_kernel<<<blocks_for(rows * cols), 256, 0, stream>>>(X, rows, cols, ldx, s, inv_sqrt ? 1 : 0);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_chi_scale(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D, const ChiGroup& cg,
                             double* Y, int64_t ldy, cudaStream_t stream) {
  chi_scale_kernel<<<blocks_for((int64_t)NQ * nov), 256, 0, stream>>>(R, ldR, NQ, nov, D, cg, Y, ldy);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_gather_cols(const double* src, int64_t lds, double* dst, int64_t ldd, int64_t rows, int64_t cols,
                               const int* perm, const double* colscale, cudaStream_t stream) {
  if (rows * cols == 0) return cudaSuccess;
  gather_cols_kernel<<<blocks_for(rows * cols), 256, 0, stream>>>(src, lds, dst, ldd, rows, cols, perm, colscale);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_symmetrize_avg(double* A, int64_t lda, int n, cudaStream_t stream) {
  symmetrize_avg_kernel<<<blocks_for((int64_t)n * n), 256, 0, stream>>>(A, lda, n);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
