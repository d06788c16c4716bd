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
constexpr int NB = 64;  // Cholesky block size
constexpr int NB2 = 256;  // outer block of the two-level schedule

// Factor the NB x NB diagonal block of each matrix (blockDim = 256): thread (r, q) = (t / 4,
// t % 4) keeps columns q, q+4, ..., q+60 of row r in registers.  Step j: the owners of column j
// scale it by 1/sqrt(pivot) and publish it in shared memory (double-buffered); every thread
// subtracts l_rj l_cj from its columns c in (j, r]; the owner of entry (j+1, j+1) then takes its
// square root.  Two barriers per column and no shared-memory copy of the block.
__device__ __forceinline__ double reg_get(const double (&v)[NB / 4], int i) {
  double x = 0.0;
#pragma unroll
  for (int k = 0; k < NB / 4; ++k)
    if (k == i) x = v[k];
  return x;
}
__device__ __forceinline__ void reg_set(double (&v)[NB / 4], int i, double x) {
#pragma unroll
  for (int k = 0; k < NB / 4; ++k)
    if (k == i) v[k] = x;
}

__device__ __forceinline__ void potrf_diag_body(double* Az, int64_t ld, int n, int j0, double* Ldz, int* err) {
  __shared__ double col[2][NB];
  __shared__ double piv[NB], pinv[NB];
  const int nbe = min(NB, n - j0);
  const int t = threadIdx.x;
  const int r = t >> 2, q = t & 3;
  const bool live = r < nbe;
  double v[NB / 4];
#pragma unroll
  for (int i = 0; i < NB / 4; ++i) {
    const int c = q + 4 * i;
    v[i] = (live && c <= r) ? Az[(int64_t)(j0 + r) + ld * (int64_t)(j0 + c)] : 0.0;
  }
  bool bad = false;
  // owner of (j, j): square root of the updated pivot (a non-positive or NaN pivot is replaced
  // by 1 so that the factorization finishes; the error is reported)
  auto take_pivot = [&](int j) {
    double d = reg_get(v, j >> 2);
    if (!(d > 0.0)) {
      bad = true;
      d = 1.0;
    }
    // one reciprocal square root (1 ulp) instead of a square root and a division: the
    // pivot chain is the kernel's critical path
    const double ri = rsqrt(d);
    const double sq = d * ri;
    reg_set(v, j >> 2, sq);
    piv[j] = sq;
    pinv[j] = ri;
  };
  if (t == 0 && nbe > 0) take_pivot(0);
  __syncthreads();
  for (int j = 0; j < nbe; ++j) {
    const int buf = j & 1;
    if (live && r > j && q == (j & 3)) {
      const double l = reg_get(v, j >> 2) * pinv[j];
      reg_set(v, j >> 2, l);
      col[buf][r] = l;
    }
    __syncthreads();
    if (live && r > j) {
      const double lr = col[buf][r];
#pragma unroll
      for (int i = 0; i < NB / 4; ++i) {
        const int c = q + 4 * i;
        if (c > j && c <= r) v[i] -= lr * col[buf][c];
      }
      if (r == j + 1 && q == ((j + 1) & 3)) take_pivot(j + 1);
    }
    __syncthreads();
  }
  if (bad) atomicCAS(err, 0, (int)kDevNotSPD);
#pragma unroll
  for (int i = 0; i < NB / 4; ++i) {
    const int c = q + 4 * i;
    if (live && c <= r) Az[(int64_t)(j0 + r) + ld * (int64_t)(j0 + c)] = v[i];
  }
  if (t < nbe) Ldz[j0 + t] = piv[t];
}

__global__ void __launch_bounds__(256) potrf_diag_kernel(double* A, int64_t ld, int64_t stride, int n, int j0,
                                                         double* Ldiag, int* err) {
  const int z = blockIdx.x;
  potrf_diag_body(A + (int64_t)z * stride, ld, n, j0, Ldiag + (int64_t)z * n, err);
}

// Panel solve: rows below the diagonal block, X L_jj^T = A_panel, one row per thread.  Column c
// of X is final once it is scaled by 1/L_cc; it is then subtracted from the later columns of the
// row (right-looking within the row: 64 short dependency chains instead of one long one).
__device__ __forceinline__ void trsm_panel_body(double* Az, int64_t ld, int n, int j0, int rblock) {
  __shared__ double Ls[NB][NB + 1];
  __shared__ double inv[NB];
  const int t = threadIdx.x;
  for (int idx = t; idx < NB * NB; idx += blockDim.x) {
    const int r = idx % NB, c = idx / NB;
    Ls[r][c] = (r >= c) ? Az[(int64_t)(j0 + r) + ld * (int64_t)(j0 + c)] : 0.0;
  }
  __syncthreads();
  if (t < NB) inv[t] = 1.0 / Ls[t][t];
  __syncthreads();
  const int r = j0 + NB + rblock * blockDim.x + t;
  if (r >= n) return;
  double x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) x[c] = Az[(int64_t)r + ld * (int64_t)(j0 + c)];
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    x[c] *= inv[c];
#pragma unroll
    for (int m = c + 1; m < NB; ++m) x[m] -= x[c] * Ls[m][c];
  }
#pragma unroll
  for (int c = 0; c < NB; ++c) Az[(int64_t)r + ld * (int64_t)(j0 + c)] = x[c];
}

__global__ void __launch_bounds__(128) trsm_panel_kernel(double* A, int64_t ld, int64_t stride, int n, int j0) {
  trsm_panel_body(A + (int64_t)blockIdx.y * stride, ld, n, j0, blockIdx.x);
}

// ----------------------------------------------------------------- variable-size batches
__global__ void __launch_bounds__(256) potrf_varlen_kernel(const MatDesc* mats, int j0, int* err) {
  const MatDesc md = mats[blockIdx.x];
  if (j0 >= md.n) return;
  potrf_diag_body(md.A, md.ld, md.n, j0, md.Ldiag, err);
}

__global__ void __launch_bounds__(128) trsm_varlen_kernel(const MatDesc* mats, int j0) {
  const MatDesc md = mats[blockIdx.y];
  if (md.n - j0 - NB <= 0 || (int)(blockIdx.x * blockDim.x) >= md.n - j0 - NB) return;
  trsm_panel_body(md.A, md.ld, md.n, j0, blockIdx.x);
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

// Many arrays at once: blockIdx.y selects array (ptrs[y], counts[y]).
__global__ void count_nonfinite_multi_kernel(const double* const* ptrs, const int64_t* counts, int* count) {
  const double* x = ptrs[blockIdx.y];
  const int64_t n = counts[blockIdx.y];
  int local = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(x[i])) ++local;
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
  int obuf = 0;  // digit-plane buffer of the current outer block (alternates: the rest of block t's
                 // update may still read its planes while block t+1 is sliced)
  LookaheadState st{la, stream};
  cudaError_t e = st.begin(stream);
  if (e != cudaSuccess) return e;
  const cudaStream_t S = st.S;
  for (int J0 = 0; J0 < n; J0 += nb2) {
    const int J1 = min(n, J0 + nb2);
    for (int j0 = J0; j0 < J1; j0 += NB) {
      potrf_diag_kernel<<<nmat, 256, 0, S>>>(A, ld, stride, n, j0, Ldiag, err);
      ++g_launches;
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      const int below = n - j0 - NB;
      if (below <= 0) break;
      trsm_panel_kernel<<<dim3((below + 127) / 128, nmat), 128, 0, S>>>(A, ld, stride, n, j0);
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
      potrf_varlen_kernel<<<nmat, 256, 0, S>>>(mats, j0, err);
      ++g_launches;
      const int below = nmax - j0 - NB;
      if (below <= 0) break;
      trsm_varlen_kernel<<<dim3((below + 127) / 128, nmat), 128, 0, S>>>(mats, j0);
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

cudaError_t launch_count_nonfinite_multi(const double* const* ptrs, const int64_t* counts, int narr, int blocks_per,
                                         int* count, cudaStream_t stream) {
  if (narr <= 0) return cudaSuccess;
  count_nonfinite_multi_kernel<<<dim3((unsigned)std::max(1, blocks_per), (unsigned)narr), 256, 0, stream>>>(ptrs, counts,
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
