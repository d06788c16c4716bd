// FP64 log-det of 1 + Pi(u) by a batched, blocked, right-looking lower
// Cholesky, and the double-double trace / log sums of the energy.
//
// The reference takes ln|det(1+Pi)| from the diagonal of a Householder QR
// (real_LogDet, src/linear-algebra/real_linalg.f90:793-825, DGEQRF) and sums
// log|R_kk| and Tr Pi in REAL(16) (rpa_CC_EcRPA_Analytic,
// src/rpa/rpa_CC.f90:440-453).  1 + Pi is symmetric positive definite
// (Pi = R diag(alpha c) R^T with c > 0), so ln det = 2 sum ln L_kk of its
// Cholesky factor equals the QR value; the sums here are double-double.
// A non-positive pivot is reported as an error, never as a NaN energy.
#include <algorithm>

#include <cstdlib>

#include "kernels.h"

namespace rpa {

namespace {
constexpr int NB = kCholNB;  // Cholesky block size (64)
constexpr int NB2 = 256;     // outer block of the two-level schedule

// Factor the NB x NB diagonal block of each matrix (blockDim = 256): thread (r, q) = (t / 4,
// t % 4) keeps columns 16q .. 16q+15 of row r in registers; the column loop is unrolled by 16, so
// every register index is static.  Step j (one barrier): every thread forms the pivot d_j itself
// from what step j-1 published (the diagonal entry a_jj and l_{j,j-1}: d_j = a_jj - l_{j,j-1}^2,
// the same FMA the entry's owner applies), and the owners of column j publish the whole column,
// l_rj = a_rj / sqrt(d_j) below the pivot and zeros on and above it (double-buffered); every thread
// then subtracts l_rj l_cj from all 16 of its entries without a branch: the zeros leave the
// finished columns and the rows above the pivot unchanged, and entries above the diagonal (never
// stored) take whatever they get.  A block smaller than NB (the last of a matrix) is padded with
// the identity.  A non-positive or NaN pivot is replaced by 1 so that the factorization finishes,
// and reported.
//
// The inverse W = L^-1 of the block is then formed by columns, right-looking: thread (c, q) holds
// rows 16q .. 16q+15 of column c of W, the owner of row k scales it by 1 / L_kk and hands it to the
// column's other three threads by a shuffle.  W is stored transposed in the block's strict upper
// triangle, which the lower factorization never reads: W(k, c) at (c, k) for k > c.  The panel
// solve below reads it there; the diagonal of W, 1 / L_cc, it recomputes from the pivots.
constexpr int kPotrfThreads = 256;
constexpr int kLP = NB + 4;  // skewed pitch: index m at m + m / 16, so the four column blocks of a
                             // warp's rows fall in different banks
__device__ __forceinline__ int sk(int m) { return m + (m >> 4); }

__device__ __forceinline__ void potrf_diag_body(double* Az, int64_t ld, int n, int j0, double* Ldz, int* err) {
  __shared__ double col[2][kLP];
  __shared__ double dnx[2];
  __shared__ double LsT[NB][kLP];  // LsT[c][sk(r)] = L(r, c) below the diagonal, 0 elsewhere
  __shared__ double inv[NB];
  const int nbe = min(NB, n - j0);
  const int t = threadIdx.x;
  const int r = t >> 2, q = t & 3;
  double v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int c = 16 * q + i;
    v[i] = (c <= r && r < nbe) ? Az[(int64_t)(j0 + r) + ld * (int64_t)(j0 + c)] : (c == r ? 1.0 : 0.0);
  }
  if (t == 0) dnx[1] = v[0];
  __syncthreads();
  double dj = dnx[1];  // pivot of column 0
  double piv = 1.0;
  bool bad = false;
  for (int g = 0; g < 4; ++g) {
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      const int j = 16 * g + jj;
      const int buf = jj & 1;
      double d = dj;
      if (!(d > 0.0)) {  // the same value in every thread
        bad = true;
        d = 1.0;
      }
      // one reciprocal square root (1 ulp) instead of a square root and a division: the pivot
      // chain is the kernel's critical path
      const double ri = rsqrt(d);
      if (q == g) {
        double l = 0.0;
        if (r == j) {
          v[jj] = d * ri;
          piv = v[jj];
        } else if (r > j) {
          v[jj] *= ri;
          l = v[jj];
        }
        col[buf][sk(r)] = l;
      }
      if (r == j + 1 && q == ((j + 1) >> 4)) dnx[buf] = v[(jj + 1) & 15];
      __syncthreads();
      if (j + 1 < NB) {
        const double l1 = col[buf][sk(j + 1)];
        dj = fma(-l1, l1, dnx[buf]);
      }
      const double lr = col[buf][sk(r)];
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = fma(-lr, col[buf][sk(16 * q + i)], v[i]);
    }
  }
  if (bad && t == 0) atomicCAS(err, 0, (int)kDevNotSPD);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int c = 16 * q + i;
    LsT[c][sk(r)] = c < r ? v[i] : 0.0;
    if (c <= r && r < nbe) Az[(int64_t)(j0 + r) + ld * (int64_t)(j0 + c)] = v[i];
  }
  if (q == (r >> 4)) {  // the owner of the diagonal entry
    inv[r] = 1.0 / piv;
    if (r < nbe) Ldz[j0 + r] = piv;
  }
  __syncthreads();
  // column c = r of W: s[i] = W(16q + i, c), zero above the diagonal
  const int lane = t & 31;
  double s[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) s[i] = (16 * q + i == r) ? 1.0 : 0.0;
  for (int g = 0; g < 4; ++g) {
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      const int k = 16 * g + kk;
      double wk = s[kk] * inv[k];
      if (q == g) s[kk] = wk;
      wk = __shfl_sync(0xffffffffu, wk, (lane & ~3) | g);
#pragma unroll
      for (int i = 0; i < 16; ++i) s[i] = fma(-LsT[k][sk(16 * q + i)], wk, s[i]);
    }
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int m = 16 * q + i;
    if (m > r && m < nbe) Az[(int64_t)(j0 + r) + ld * (int64_t)(j0 + m)] = s[i];
  }
}

__global__ void __launch_bounds__(kPotrfThreads) potrf_diag_kernel(double* A, int64_t ld, int64_t stride, int n,
                                                                   int j0, double* Ldiag, int* err) {
  const int z = blockIdx.x;
  potrf_diag_body(A + (int64_t)z * stride, ld, n, j0, Ldiag + (int64_t)z * n, err);
}

// Panel solve: the rows below the diagonal block, X = A_p L^-T = A_p B with B = W^T upper
// triangular (strict part from the block's upper triangle, diagonal 1 / L_cc), on the FP64 tensor
// cores (DMMA m8n8k4, the fragment layout of dsyrk_f64.cu): 64 rows per CTA, 4 warps of 32 x 32
// outputs; warps of the first 32 columns stop at k = 32 (B(k, c) = 0 for k > c).  Every CTA reads
// all of its rows before it writes any, and no other CTA touches them.
constexpr int kTrsmRows = 64;
constexpr int kTrsmThreads = 128;
constexpr int kLdA = NB + 8;  // As[k][m]: fragment loads hit each bank pair twice
constexpr int kLdB = NB + 4;  // BsT[c][k]: likewise, and conflict-free fills
constexpr size_t kTrsmSmem = sizeof(double) * (size_t)NB * (kLdA + kLdB);

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void trsm_panel_body(double* Az, int64_t ld, int n, int j0, int rblock, const double* Ldz) {
  extern __shared__ __align__(16) double trsm_smem[];
  auto As = reinterpret_cast<double(*)[kLdA]>(trsm_smem);               // As[k][m] = A_p(m, k)
  auto BsT = reinterpret_cast<double(*)[kLdB]>(trsm_smem + NB * kLdA);  // BsT[c][k] = B(k, c)
  const int t = threadIdx.x;
  const int r0 = j0 + NB + rblock * kTrsmRows;
  const int rows = min(kTrsmRows, n - r0);
  // operands by asynchronous 8-byte copies (every load in flight at once), zeros and the
  // diagonal of B by plain stores to other addresses
  const int fi = t & (NB - 1), fc0 = t >> 6;
#pragma unroll
  for (int m = 0; m < NB / 2; ++m) {
    const int c = fc0 + 2 * m;
    if (fi < rows) cp_async8(&As[c][fi], Az + (int64_t)(r0 + fi) + ld * (int64_t)(j0 + c));
    else As[c][fi] = 0.0;
    if (fi < c) cp_async8(&BsT[c][fi], Az + (int64_t)(j0 + fi) + ld * (int64_t)(j0 + c));
    else if (fi > c) BsT[c][fi] = 0.0;
  }
  if (t < NB) BsT[t][t] = 1.0 / Ldz[j0 + t];
  cp_async_wait_all();
  __syncthreads();
  const int lane = t & 31, warp = t >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  auto kstep = [&](int ks) {
    const int kr = 4 * ks + (lane & 3);
    double af[4], bf[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) af[i] = As[kr][wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
    for (int j = 0; j < 4; ++j) bf[j] = BsT[wn * 32 + j * 8 + (lane >> 2)][kr];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
  };
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) kstep(ks);
  if (wn == 1) {  // B(k, c) = 0 for k > c: the first 32 columns stop at k = 32
#pragma unroll
    for (int ks = 8; ks < 16; ++ks) kstep(ks);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = wm * 32 + i * 8 + (lane >> 2);
    if (row >= rows) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int c = wn * 32 + j * 8 + 2 * (lane & 3) + v;
        Az[(int64_t)(r0 + row) + ld * (int64_t)(j0 + c)] = acc[i][j][v];
      }
  }
}

__global__ void __launch_bounds__(kTrsmThreads) trsm_panel_kernel(double* A, int64_t ld, int64_t stride, int n,
                                                                  int j0, const double* Ldiag) {
  const int z = blockIdx.y;
  trsm_panel_body(A + (int64_t)z * stride, ld, n, j0, blockIdx.x, Ldiag + (int64_t)z * n);
}

// ----------------------------------------------------------------- variable-size batches
__global__ void __launch_bounds__(kPotrfThreads) potrf_varlen_kernel(const MatDesc* mats, int j0, int* err) {
  const MatDesc md = mats[blockIdx.x];
  if (j0 >= md.n) return;
  potrf_diag_body(md.A, md.ld, md.n, j0, md.Ldiag, err);
}

__global__ void __launch_bounds__(kTrsmThreads) trsm_varlen_kernel(const MatDesc* mats, int j0) {
  const MatDesc md = mats[blockIdx.y];
  if (md.n - j0 - NB <= 0 || (int)blockIdx.x * kTrsmRows >= md.n - j0 - NB) return;
  trsm_panel_body(md.A, md.ld, md.n, j0, blockIdx.x, md.Ldiag);
}

// Shared-memory opt-in of the panel solve (> 48 KB), once per process.
cudaError_t trsm_smem_optin() {
  static const cudaError_t e = [] {
    cudaError_t r = cudaFuncSetAttribute(trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem);
    if (r == cudaSuccess)
      r = cudaFuncSetAttribute(trsm_varlen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem);
    return r;
  }();
  return e;
}

// Deterministic block reduction of double-double values (blockDim = 256).
__device__ dd block_reduce_dd(dd v) {
  __shared__ double sh[256], sl[256];
  sh[threadIdx.x] = v.hi;
  sl[threadIdx.x] = v.lo;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      dd o = dd_add_dd({sh[threadIdx.x], sl[threadIdx.x]}, {sh[threadIdx.x + s], sl[threadIdx.x + s]});
      sh[threadIdx.x] = o.hi;
      sl[threadIdx.x] = o.lo;
    }
    __syncthreads();
  }
  return {sh[0], sl[0]};
}

__global__ void __launch_bounds__(256) trace_shift_kernel(double* A, int64_t ld, int64_t stride, int n,
                                                          const double* diag, double* tr_dd) {
  const int z = blockIdx.x;
  double* Az = A + (int64_t)z * stride;
  dd acc{0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double* p = Az + (int64_t)i * (ld + 1);
    double v = diag ? diag[(int64_t)z * n + i] : *p;
    acc = dd_add(acc, v);
    *p = v + 1.0;
  }
  dd r = block_reduce_dd(acc);
  if (threadIdx.x == 0) {
    tr_dd[2 * z] = r.hi;
    tr_dd[2 * z + 1] = r.lo;
  }
}

__global__ void __launch_bounds__(256) logdet_sum_kernel(const double* Ldiag, int n, double* out_dd) {
  const int z = blockIdx.x;
  dd acc{0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc = dd_add(acc, 2.0 * log(Ldiag[(int64_t)z * n + i]));
  dd r = block_reduce_dd(acc);
  if (threadIdx.x == 0) {
    out_dd[2 * z] = r.hi;
    out_dd[2 * z + 1] = r.lo;
  }
}

__global__ void __launch_bounds__(256) trace_shift_varlen_kernel(const MatDesc* mats) {
  const MatDesc md = mats[blockIdx.x];
  dd acc{0.0, 0.0};
  for (int i = threadIdx.x; i < md.n; i += blockDim.x) {
    double* p = md.A + (int64_t)i * (md.ld + 1);
    const double v = *p;
    acc = dd_add(acc, v);
    *p = v + 1.0;
  }
  dd r = block_reduce_dd(acc);
  if (threadIdx.x == 0) {
    md.tr_dd[0] = r.hi;
    md.tr_dd[1] = r.lo;
  }
}

__global__ void __launch_bounds__(256) logdet_sum_varlen_kernel(const MatDesc* mats) {
  const MatDesc md = mats[blockIdx.x];
  dd acc{0.0, 0.0};
  for (int i = threadIdx.x; i < md.n; i += blockDim.x) acc = dd_add(acc, 2.0 * log(md.Ldiag[i]));
  dd r = block_reduce_dd(acc);
  if (threadIdx.x == 0) {
    md.ld_dd[0] = r.hi;
    md.ld_dd[1] = r.lo;
  }
}

__global__ void dai_kernel(const double* eps_o, const double* eps_v, int64_t no, int64_t nv, double* D) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= no * nv) return;
  const int64_t i = idx / nv, a = idx - i * nv;
  D[idx] = eps_v[a] - eps_o[i];
}

__global__ void symmetrize_kernel(double* A, int64_t ld, int64_t stride, int n) {
  __shared__ double tile[32][33];
  const int z = blockIdx.z;
  double* Az = A + (int64_t)z * stride;
  const int bx = blockIdx.x, by = blockIdx.y;  // destination tile: rows by*32, cols bx*32 (upper: rows < cols)
  if (by > bx) return;
  // read source tile (rows bx*32.., cols by*32..) which lies in the lower triangle
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = bx * 32 + threadIdx.x, c = by * 32 + j;
    tile[j][threadIdx.x] = (r < n && c < n) ? Az[(int64_t)r + ld * c] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = by * 32 + threadIdx.x, c = bx * 32 + j;  // destination (r, c) = source (c, r)
    if (r < n && c < n && r < c) Az[(int64_t)r + ld * c] = tile[threadIdx.x][j];
  }
}

__global__ void count_nonfinite_kernel(const double* x, int64_t n, int* count) {
  int local = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(x[i])) ++local;
  if (local) atomicAdd(count, local);
}

// Lower triangle (diagonal included) of nmat column-major n x n matrices: blockIdx.x strides over
// columns, blockIdx.y selects the matrix.  Entries above the diagonal are never read, so leftovers
// there (a reused buffer, a caller's unused upper half) cannot raise a false count.
__global__ void count_nonfinite_lower_kernel(const double* A, int64_t ld, int64_t stride, int n, int* count) {
  const double* a = A + (int64_t)blockIdx.y * stride;
  int local = 0;
  for (int c = blockIdx.x; c < n; c += gridDim.x) {
    const double* col = a + ld * (int64_t)c;
    for (int r = c + threadIdx.x; r < n; r += blockDim.x)
      if (!isfinite(col[r])) ++local;
  }
  if (local) atomicAdd(count, local);
}

// Rows 0 .. rows-1 of each column of a column-major array (blockIdx.x strides over the columns):
// a caller's padding rows between rows and ld are never read, so they cannot raise a false count.
__device__ __forceinline__ int count_nonfinite_cols_body(const double* A, int64_t ld, int64_t rows, int64_t cols) {
  int local = 0;
  for (int64_t c = blockIdx.x; c < cols; c += gridDim.x) {
    const double* col = A + ld * c;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x)
      if (!isfinite(col[r])) ++local;
  }
  return local;
}

__global__ void count_nonfinite_cols_kernel(const double* A, int64_t ld, int64_t rows, int64_t cols, int* count) {
  const int local = count_nonfinite_cols_body(A, ld, rows, cols);
  if (local) atomicAdd(count, local);
}

// Many arrays at once: blockIdx.y selects array ptrs[y] with (ld, rows, cols) = dims[3y .. 3y+2].
__global__ void count_nonfinite_multi_kernel(const double* const* ptrs, const int64_t* dims, int* count) {
  const int64_t* d = dims + 3 * (int64_t)blockIdx.y;
  const int local = count_nonfinite_cols_body(ptrs[blockIdx.y], d[0], d[1], d[2]);
  if (local) atomicAdd(count, local);
}

// Tile-tuner input: unit diagonal, off-diagonal entries uniform in (-1/(2n), 1/(2n)), so every
// off-diagonal row sum is below 1/2 and the matrix (and 1 + it) is symmetric positive definite.
__global__ void fill_spd_varlen_kernel(const MatDesc* mats, uint64_t seed) {
  const MatDesc md = mats[blockIdx.y];
  const double scale = 1.0 / (double)max(md.n, 1);
  for (int c = blockIdx.x; c < md.n; c += gridDim.x) {
    double* col = md.A + md.ld * (int64_t)c;
    for (int r = c + threadIdx.x; r < md.n; r += blockDim.x) {
      const uint64_t h = splitmix64(seed ^ splitmix64(((uint64_t)blockIdx.y << 40) ^ ((uint64_t)c << 20) ^ (uint64_t)r));
      col[r] = r == c ? 1.0 : ((double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5) * scale;
    }
  }
}

__global__ void copy_lower_kernel(const double* src, int64_t lds, int64_t strideS, double* dst, int64_t ldd,
                                  int64_t strideD, int n) {
  const int z = blockIdx.z;
  const int c = blockIdx.y;
  const double* s = src + (int64_t)z * strideS + lds * c;
  double* d = dst + (int64_t)z * strideD + ldd * c;
  for (int r = c + blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) d[r] = s[r];
}
}  // namespace

// Two-level blocked right-looking Cholesky: 64-wide column panels (diagonal
// factorization + panel solve + update of the rest of the outer block), then
// one rank-nb2 update of the trailing matrix per outer block.

// Default outer block width: NB2 unless RPA_B200_CHOL_NB2 (a multiple of NB) says otherwise.
int outer_block() {
  static int nb2 = [] {
    const char* e = std::getenv("RPA_B200_CHOL_NB2");
    const int v = e ? std::atoi(e) : NB2;
    return (v >= NB && v % NB == 0) ? v : NB2;
  }();
  return nb2;
}

LogdetPlan default_logdet_plan() { return LogdetPlan{outer_block(), 2}; }

bool valid_logdet_plan(const LogdetPlan& p) {
  return p.nb2 >= NB && p.nb2 <= 1024 && p.nb2 % NB == 0 && (p.tile_w == 2 || p.tile_w == 4);
}

// Lookahead (la non-null): after the panel of outer block t is factored, the trailing update is
// split into (a) the columns of block t+1, on the critical stream, and (b) everything right of
// block t+1, on la->rest.  Block t+1 (diagonal factorizations, panel solves, in-block updates:
// latency-bound launches) then runs beside (b) of block t, which touches disjoint columns; (a) of
// block t+1 waits for (b) of block t, whose columns it overlaps.
namespace {
struct LookaheadState {
  const Lookahead* la;
  cudaStream_t S;  // critical-path stream
  bool rest_pending = false;
  cudaError_t begin(cudaStream_t stream) {
    S = la ? la->crit : stream;
    if (!la) return cudaSuccess;
    cudaError_t e = cudaEventRecord(la->ev[0], stream);
    return e == cudaSuccess ? cudaStreamWaitEvent(la->crit, la->ev[0], 0) : e;
  }
  // before (a) of block t: (b) of block t-1 done; the panel of block t is final
  cudaError_t before_next_block() {
    cudaError_t e = cudaSuccess;
    if (rest_pending) e = cudaStreamWaitEvent(S, la->ev[2], 0);
    if (e == cudaSuccess) e = cudaEventRecord(la->ev[1], S);
    return e;
  }
  cudaError_t fork_rest() { return cudaStreamWaitEvent(la->rest, la->ev[1], 0); }
  cudaError_t rest_done() {
    rest_pending = true;
    return cudaEventRecord(la->ev[2], la->rest);
  }
  cudaError_t end(cudaStream_t stream) {
    if (!la) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (rest_pending) e = cudaStreamWaitEvent(S, la->ev[2], 0);
    if (e == cudaSuccess) e = cudaEventRecord(la->ev[3], S);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, la->ev[3], 0);
    return e;
  }
};

DsyrkArgs update_args(double* A, int64_t ld, int64_t stride, int nmat, int row0, int col0, int n, int ncols,
                      int kdim, int tile_w) {
  DsyrkArgs u{};
  u.A = A + (int64_t)row0 + ld * (int64_t)col0;
  u.lda = ld;
  u.strideA = stride;
  u.C = A + (int64_t)row0 + ld * (int64_t)row0;
  u.ldc = ld;
  u.strideC = stride;
  u.n = n;
  u.ncols = ncols;
  u.kdim = kdim;
  u.batch = nmat;
  u.D = nullptr;
  u.tile_w = tile_w;
  return u;
}
}  // namespace

cudaError_t launch_cholesky_lower(double* A, int64_t ld, int64_t stride, int n, int nmat, double* Ldiag, int* err,
                                  cudaStream_t stream, const LogdetPlan& plan, const Lookahead* la,
                                  const OzakiWork* oz) {
  if (!valid_logdet_plan(plan)) return cudaErrorInvalidValue;
  const int nb2 = plan.nb2;
  if (oz && (oz->S == 0 || oz->K != nb2)) oz = nullptr;
  if (cudaError_t e0 = trsm_smem_optin()) return e0;
  int obuf = 0;  // digit-plane buffer of the current outer block (alternates: the rest of block t's
                 // update may still read its planes while block t+1 is sliced)
  LookaheadState st{la, stream};
  cudaError_t e = st.begin(stream);
  if (e != cudaSuccess) return e;
  const cudaStream_t S = st.S;
  for (int J0 = 0; J0 < n; J0 += nb2) {
    const int J1 = min(n, J0 + nb2);
    for (int j0 = J0; j0 < J1; j0 += NB) {
      potrf_diag_kernel<<<nmat, kPotrfThreads, 0, S>>>(A, ld, stride, n, j0, Ldiag, err);
      ++g_launches;
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      const int below = n - j0 - NB;
      if (below <= 0) break;
      trsm_panel_kernel<<<dim3((below + kTrsmRows - 1) / kTrsmRows, nmat), kTrsmThreads, kTrsmSmem, S>>>(
          A, ld, stride, n, j0, Ldiag);
      ++g_launches;
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      const int ncols = J1 - (j0 + NB);  // columns of this outer block right of the panel
      if (ncols <= 0) continue;
      e = launch_dsyrk_lower(update_args(A, ld, stride, nmat, j0 + NB, j0, below, ncols, NB, plan.tile_w), S);
      if (e != cudaSuccess) return e;
    }
    const int trail = n - J1;
    if (trail <= 0) break;
    // full-width panels take the int8 route; a narrower last panel (n not a multiple of nb2) stays on DMMA
    const bool use_oz = oz && J1 - J0 == oz->K;
    if (use_oz && (e = launch_ozaki_slices(*oz, obuf, A, ld, stride, n, nmat, J1, J0, S)) != cudaSuccess) return e;
    auto update = [&](int row0, int nrows, int ncols, cudaStream_t s) {
      return use_oz ? launch_ozaki_update(*oz, obuf, A, ld, stride, n, nmat, row0, row0, nrows, ncols, err,
                                          oz->num_sms, s)
                    : launch_dsyrk_lower(update_args(A, ld, stride, nmat, row0, J0, nrows, ncols, J1 - J0,
                                                     plan.tile_w), s);
    };
    if (!la) {
      if ((e = update(J1, trail, trail, S)) != cudaSuccess) return e;
      obuf ^= 1;
      continue;
    }
    const int J2 = min(n, J1 + nb2);
    if ((e = st.before_next_block()) != cudaSuccess) return e;
    if ((e = update(J1, trail, J2 - J1, S)) != cudaSuccess) return e;
    if (n - J2 > 0) {
      if ((e = st.fork_rest()) != cudaSuccess) return e;
      if ((e = update(J2, n - J2, n - J2, la->rest)) != cudaSuccess) return e;
      if ((e = st.rest_done()) != cudaSuccess) return e;
    }
    obuf ^= 1;
  }
  return st.end(stream);
}

// Same schedule as launch_cholesky_lower over matrices of different orders:
// every step is launched for the largest order and matrices that are already
// finished (or too small for the step) leave at once.
cudaError_t launch_logdet_varlen(const MatDesc* mats, int nmat, int nmax, int* err, cudaStream_t stream,
                                 const LogdetPlan& plan, const Lookahead* la) {
  if (nmat <= 0) return cudaSuccess;
  if (!valid_logdet_plan(plan)) return cudaErrorInvalidValue;
  if (cudaError_t e0 = trsm_smem_optin()) return e0;
  trace_shift_varlen_kernel<<<nmat, 256, 0, stream>>>(mats);
  ++g_launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int nb2 = plan.nb2;
  LookaheadState st{la, stream};
  if ((e = st.begin(stream)) != cudaSuccess) return e;
  const cudaStream_t S = st.S;
  for (int J0 = 0; J0 < nmax; J0 += nb2) {
    const int J1 = std::min(nmax, J0 + nb2);
    for (int j0 = J0; j0 < J1; j0 += NB) {
      potrf_varlen_kernel<<<nmat, kPotrfThreads, 0, S>>>(mats, j0, err);
      ++g_launches;
      const int below = nmax - j0 - NB;
      if (below <= 0) break;
      trsm_varlen_kernel<<<dim3((below + kTrsmRows - 1) / kTrsmRows, nmat), kTrsmThreads, kTrsmSmem, S>>>(mats, j0);
      ++g_launches;
      e = launch_dsyrk_varlen(mats, nmat, 0, J0, j0, nb2, plan.tile_w, nmax, S);
      if (e != cudaSuccess) return e;
    }
    if (nmax - J1 <= 0) break;
    if (!la) {
      e = launch_dsyrk_varlen(mats, nmat, 1, J0, 0, nb2, plan.tile_w, nmax, S);
      if (e != cudaSuccess) return e;
      continue;
    }
    if ((e = st.before_next_block()) != cudaSuccess) return e;
    e = launch_dsyrk_varlen(mats, nmat, 2, J0, 0, nb2, plan.tile_w, nmax, S);
    if (e != cudaSuccess) return e;
    if (nmax - std::min(nmax, J1 + nb2) > 0) {
      if ((e = st.fork_rest()) != cudaSuccess) return e;
      e = launch_dsyrk_varlen(mats, nmat, 3, J0, 0, nb2, plan.tile_w, nmax, la->rest);
      if (e != cudaSuccess) return e;
      if ((e = st.rest_done()) != cudaSuccess) return e;
    }
  }
  if ((e = st.end(stream)) != cudaSuccess) return e;
  logdet_sum_varlen_kernel<<<nmat, 256, 0, stream>>>(mats);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_fill_spd_varlen(const MatDesc* mats, int nmat, int nmax, uint64_t seed, cudaStream_t stream) {
  if (nmat <= 0 || nmax <= 0) return cudaSuccess;
  fill_spd_varlen_kernel<<<dim3((unsigned)std::min(nmax, 1024), (unsigned)nmat), 256, 0, stream>>>(mats, seed);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_trace_shift(double* A, int64_t ld, int64_t stride, int n, int nmat, const double* diag,
                               double* tr_dd, cudaStream_t stream) {
  trace_shift_kernel<<<nmat, 256, 0, stream>>>(A, ld, stride, n, diag, tr_dd);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_logdet_sum(const double* Ldiag, int n, int nmat, double* logdet_dd, cudaStream_t stream) {
  logdet_sum_kernel<<<nmat, 256, 0, stream>>>(Ldiag, n, logdet_dd);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_dai(const double* eps_o, const double* eps_v, int64_t no, int64_t nv, double* D,
                       cudaStream_t stream) {
  const int64_t n = no * nv;
  if (n == 0) return cudaSuccess;
  dai_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(eps_o, eps_v, no, nv, D);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_symmetrize(double* A, int64_t ld, int64_t stride, int n, int nmat, cudaStream_t stream) {
  const int T = (n + 31) / 32;
  symmetrize_kernel<<<dim3(T, T, nmat), dim3(32, 8), 0, stream>>>(A, ld, stride, n);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_count_nonfinite(const double* x, int64_t n, int* count, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  int64_t blocks = (n + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  count_nonfinite_kernel<<<(unsigned)blocks, 256, 0, stream>>>(x, n, count);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_count_nonfinite_lower(const double* A, int64_t ld, int64_t stride, int n, int nmat, int* count,
                                         cudaStream_t stream) {
  if (n <= 0 || nmat <= 0) return cudaSuccess;
  const int cols = std::min(n, std::max(1, 4096 / nmat));
  count_nonfinite_lower_kernel<<<dim3((unsigned)cols, (unsigned)nmat), 256, 0, stream>>>(A, ld, stride, n, count);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_count_nonfinite_cols(const double* A, int64_t ld, int64_t rows, int64_t cols, int* count,
                                        cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>(cols, 4096);
  count_nonfinite_cols_kernel<<<(unsigned)blocks, 256, 0, stream>>>(A, ld, rows, cols, count);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_count_nonfinite_multi(const double* const* ptrs, const int64_t* dims, int narr, int blocks_per,
                                         int* count, cudaStream_t stream) {
  if (narr <= 0) return cudaSuccess;
  count_nonfinite_multi_kernel<<<dim3((unsigned)std::max(1, blocks_per), (unsigned)narr), 256, 0, stream>>>(ptrs, dims,
                                                                                                         count);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_copy_lower(const double* src, int64_t lds, int64_t strideS, double* dst, int64_t ldd,
                              int64_t strideD, int n, int nmat, cudaStream_t stream) {
  copy_lower_kernel<<<dim3((n + 255) / 256, n, nmat), 256, 0, stream>>>(src, lds, strideS, dst, ldd, strideD, n);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
