// Symmetric eigensolver on the GPU: the replacement of real_EVD
// (src/linear-algebra/real_linalg.f90:1501-1559), which calls LAPACK's
// divide-and-conquer dsyevd.  Same three stages, each shaped for the B200:
//
//  1. Householder reduction to tridiagonal form T = Q_H^T A Q_H (lower), in
//     panels of kNB columns: per column one single-CTA kernel (deferred update
//     of the column from the panel's V/W, reflector generation, finishing of
//     the previous column's w) and one multi-CTA matrix-vector product with
//     the trailing matrix (warp per column, coalesced); after each panel the
//     trailing matrix is updated by two FP64 DMMA GEMMs (A -= V W^T + W V^T).
//  2. Divide and conquer on T (Cuppen's tearing, rank-one merges):
//     leaves of <= 32 rows are solved by cyclic Jacobi, one warp per leaf;
//     every merge sorts the poles, deflates small z components and close
//     poles (Givens rotations), solves the secular equation by bisection in
//     coordinates relative to the nearest pole (warp per root), recomputes z
//     by the Loewner formula (Gu-Eisenstat) so the eigenvectors stay
//     orthogonal, and multiplies the children's eigenvectors by the rank-one
//     problem's eigenvectors with a DMMA GEMM.  All merges of one tree level
//     run in the same launches.
//  3. Back-transformation V = Q_H Z with compact-WY block reflectors
//     (I - V_b T_b V_b^T), three GEMMs per panel.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "kernels.h"

namespace rpa {

namespace {

constexpr int kNB = 32;    // panel width of the reduction and of the back-transformation
constexpr int kLeaf = 32;  // largest leaf of the divide-and-conquer tree
constexpr double kEps = 1.1102230246251565e-16;  // unit roundoff 2^-53

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; every thread gets the result.  red: >= 33 doubles of shared memory.
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    double t = lane < nw ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

__device__ double block_max(double v, double* red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    double t = lane < nw ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

// ---------------------------------------------------------------- stage 1: reduction

namespace cg = cooperative_groups;
constexpr int kCS = 8;    // CTAs per cluster of the per-column reduction step
constexpr int kCT = 512;  // threads per CTA

// Cluster-wide sum of cnt per-CTA partials (part[buf][0..cnt), written by the caller and
// followed by __syncthreads): after the cluster barrier every CTA adds the kCS partials in
// rank order through distributed shared memory, so all CTAs get identical totals in out.
// part is double-buffered: a CTA rewrites part[buf] only after the next barrier, which no CTA
// passes before every CTA has finished reading the previous buffer.
__device__ __forceinline__ void cluster_sum(cg::cluster_group& cl, double (*part)[2 * kNB], int& buf, int cnt,
                                            double* out) {
  cl.sync();
  if ((int)threadIdx.x < cnt) {
    double acc = 0.0;
    for (int k = 0; k < kCS; ++k) acc += cl.map_shared_rank(&part[buf][0], k)[threadIdx.x];
    out[threadIdx.x] = acc;
  }
  __syncthreads();
  buf ^= 1;
}

// One step of the panel reduction (panel starts at column p; Wp is n x kNB, ld n), run by one
// cluster of kCS CTAs; CTA `rank` owns rows [j+1 + rank*chunk, ...) of the active column.
//  fin >= 0: finish w of panel column fin from y = A_trailing v (the deferred update of the
//            trailing matrix by panel columns < fin is applied here), store W(:, fin).
//  nxt >= 0: bring column p+nxt up to date, generate its reflector (tau, d, e, V(:, p+nxt)).
__global__ void __cluster_dims__(kCS, 1, 1) __launch_bounds__(kCT)
    house_kernel(double* A, int n, int64_t mstride, double* V, double* Wp, int p, int fin, int nxt, const double* y,
                 double* tau, double* d, double* e) {
  cg::cluster_group cl = cg::this_cluster();
  {  // matrix of this cluster
    const int64_t z = (int64_t)blockIdx.x / kCS;
    A += mstride * z;
    V += mstride * z;
    Wp += (int64_t)n * kNB * z;
    y += (int64_t)n * z;
    tau += (int64_t)n * z;
    d += (int64_t)n * z;
    e += (int64_t)n * z;
  }
  const int rank = (int)cl.block_rank();
  __shared__ double part[2][2 * kNB];
  __shared__ double tot[2 * kNB];
  __shared__ double wj[kNB], vj[kNB];
  __shared__ double red[33];
  int buf = 0;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t ld = n;
  const int gt = rank * kCT + t;  // thread index within the cluster
  if (fin >= 0) {
    const int j = p + fin;
    const double* v = V + ld * j;
    const int m = n - 1 - j, chunk = (m + kCS - 1) / kCS;
    const int r0 = j + 1 + rank * chunk, r1 = min(n, r0 + chunk);
    // s1_c = V_c^T v (q = 2c), s2_c = W_c^T v (q = 2c + 1): warp per product over this CTA's rows
    for (int q = warp; q < 2 * fin; q += kCT / 32) {
      const int c = q >> 1;
      const double* col = (q & 1) ? (Wp + ld * c) : (V + ld * (p + c));
      double acc = 0.0;
      for (int r = r0 + lane; r < r1; r += 32) acc += col[r] * v[r];
      acc = warp_sum(acc);
      if (lane == 0) part[buf][q] = acc;
    }
    __syncthreads();
    cluster_sum(cl, part, buf, 2 * fin, tot);
    const double tj = tau[j];
    double* w = Wp + ld * fin;
    double pv = 0.0;
    for (int r = r0 + t; r < r1; r += kCT) {
      double val = y[r];
      for (int c = 0; c < fin; ++c) val -= V[r + ld * (p + c)] * tot[2 * c + 1] + Wp[r + ld * c] * tot[2 * c];
      val *= tj;
      w[r] = val;
      pv += val * v[r];
    }
    for (int r = gt; r <= j; r += kCS * kCT) w[r] = 0.0;
    pv = block_sum(pv, red);
    if (t == 0) part[buf][0] = pv;
    __syncthreads();
    cluster_sum(cl, part, buf, 1, tot);
    const double alpha = -0.5 * tj * tot[0];
    for (int r = r0 + t; r < r1; r += kCT) w[r] += alpha * v[r];
    cl.sync();  // W(:, fin) complete and visible to the whole cluster
  }
  if (nxt >= 0) {
    const int j = p + nxt;
    double* a = A + ld * j;
    const int m = n - j, chunk = (m + kCS - 1) / kCS;
    const int r0 = j + rank * chunk, r1 = min(n, r0 + chunk);
    if (t < nxt) {
      wj[t] = Wp[j + ld * t];
      vj[t] = V[j + ld * (p + t)];
    }
    __syncthreads();
    // deferred update of column j (rows >= j) from panel columns < nxt
    double ps = 0.0;
    for (int r = r0 + t; r < r1; r += kCT) {
      double val = a[r];
      for (int c = 0; c < nxt; ++c) val -= V[r + ld * (p + c)] * wj[c] + Wp[r + ld * c] * vj[c];
      a[r] = val;
      if (r >= j + 2) ps += val * val;
    }
    ps = block_sum(ps, red);
    if (t == 0) part[buf][0] = ps;
    __syncthreads();
    cluster_sum(cl, part, buf, 1, tot);  // its barrier also publishes the updated column
    const double sigma2 = tot[0];
    const double alpha = a[j + 1];
    double beta, tj, scale;
    if (sigma2 == 0.0) {
      beta = alpha;
      tj = 0.0;
      scale = 0.0;
    } else {
      beta = -copysign(sqrt(alpha * alpha + sigma2), alpha);
      tj = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    double* v = V + ld * j;
    for (int r = r0 + t; r < r1; r += kCT)
      if (r > j) v[r] = (r == j + 1) ? 1.0 : a[r] * scale;
    for (int r = gt; r <= j; r += kCS * kCT) v[r] = 0.0;
    if (rank == 0 && t == 0) {
      tau[j] = tj;
      d[j] = a[j];
      e[j] = beta;
    }
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// y(c) = sum_{r > j} A(r, c) v(r) for c > j: kGemvWarps warps per column (two columns per
// 256-thread block), each lane with four independent accumulators, partial sums added in a
// fixed order.  The trailing matrix is read once per column step, so the kernel must keep
// enough loads in flight to run at memory speed: one warp per column left it latency-bound.
constexpr int kGemvWarps = 4;
__global__ void __launch_bounds__(256) trailing_gemv_kernel(const double* A, int n, int64_t mstride, const double* v,
                                                            int j, double* y) {
  __shared__ double part[8];
  A += mstride * blockIdx.y;
  v += mstride * blockIdx.y;
  y += (int64_t)n * blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = j + 1 + (int)blockIdx.x * (8 / kGemvWarps) + warp / kGemvWarps;
  const int w = warp % kGemvWarps;
  double acc = 0.0;
  if (c < n) {
    const double* col = A + (int64_t)n * c;
    constexpr int S = 32 * kGemvWarps;  // rows between consecutive loads of one lane
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int r = j + 1 + w * 32 + lane;
    for (; r + 3 * S < n; r += 4 * S) {
      a0 += col[r] * v[r];
      a1 += col[r + S] * v[r + S];
      a2 += col[r + 2 * S] * v[r + 2 * S];
      a3 += col[r + 3 * S] * v[r + 3 * S];
    }
    for (; r < n; r += S) a0 += col[r] * v[r];
    acc = warp_sum((a0 + a1) + (a2 + a3));
  }
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (threadIdx.x < 8 / kGemvWarps) {
    const int cc = j + 1 + (int)blockIdx.x * (8 / kGemvWarps) + (int)threadIdx.x;
    if (cc < n) {
      double s = 0.0;
      for (int q = 0; q < kGemvWarps; ++q) s += part[threadIdx.x * kGemvWarps + q];
      y[cc] = s;
    }
  }
}

// ---------------------------------------------------------------- stage 3: back-transformation

// T (upper triangular, nb x nb, ld kNB) of the block reflector H_p ... H_{p+nb-1} = I - V T V^T,
// from G = V^T V (ld kNB): T(i,i) = tau_i, T(0:i, i) = -tau_i T(0:i, 0:i) G(0:i, i).
__global__ void build_t_kernel(const double* G, const double* tau, int nb, double* T, int n) {
  __shared__ double Gs[kNB][kNB + 1], Ts[kNB][kNB + 1], ts[kNB];
  G += (int64_t)kNB * kNB * blockIdx.x;  // one matrix of the batch per CTA
  T += (int64_t)kNB * kNB * blockIdx.x;
  tau += (int64_t)n * blockIdx.x;
  const int r = threadIdx.x;  // row of T
  for (int c = 0; c < kNB; ++c) {
    Gs[r][c] = (r < nb && c < nb) ? G[r + kNB * c] : 0.0;
    Ts[r][c] = 0.0;
  }
  ts[r] = r < nb ? tau[r] : 0.0;
  __syncwarp();
  for (int i = 0; i < nb; ++i) {
    double val = 0.0;
    if (r < i) {
      for (int c = r; c < i; ++c) val += Ts[r][c] * Gs[c][i];
      val *= -ts[i];
    } else if (r == i) {
      val = ts[i];
    }
    __syncwarp();
    Ts[r][i] = val;
    __syncwarp();
  }
  for (int c = 0; c < kNB; ++c) T[r + kNB * c] = Ts[r][c];
}

// ---------------------------------------------------------------- stage 2: divide and conquer

// Cuppen tearing: for every internal boundary b (between rows b-1 and b), d(b-1), d(b) -= |e(b-1)|.
__global__ void tear_kernel(double* d, const double* e, const int* bounds, int nb, int n, int nmat) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nb * nmat) return;
  const int64_t z = idx / nb;
  d += (int64_t)n * z;
  e += (int64_t)n * z;
  const int b = bounds[idx % nb];
  const double r = fabs(e[b - 1]);
  d[b - 1] -= r;
  d[b] -= r;
}

struct Leaf {
  int s, m;
};

// Leaf eigenproblems (tridiagonal, m <= 32) by cyclic two-sided Jacobi, one warp per leaf: the
// leaf is held densely in shared memory; each sweep is m'-1 rounds of m'/2 disjoint rotations
// (round-robin pairing, m' = m rounded up to even); lane l owns row/column l for the updates.
__global__ void __launch_bounds__(32) leaf_jacobi_kernel(const Leaf* leaves, const double* dIn, const double* eIn,
                                                         double* D, double* Q, int64_t ldq, int* err, int n,
                                                         int64_t mstride) {
  dIn += (int64_t)n * blockIdx.y;
  eIn += (int64_t)n * blockIdx.y;
  D += (int64_t)n * blockIdx.y;
  Q += mstride * blockIdx.y;
  constexpr int P = kLeaf + 1;
  __shared__ double a[kLeaf * P], z[kLeaf * P];  // a[r * P + c]
  __shared__ double rc[kLeaf / 2], rs[kLeaf / 2];
  __shared__ int rpi[kLeaf / 2], rqi[kLeaf / 2];
  const Leaf L = leaves[blockIdx.x];
  const int l = threadIdx.x, m = L.m;
  for (int c = 0; c < kLeaf; ++c) {
    double v = 0.0;
    if (l < m && c < m) {
      if (c == l) v = dIn[L.s + l];
      else if (c == l + 1) v = eIn[L.s + l];
      else if (c + 1 == l) v = eIn[L.s + c];
    }
    a[l * P + c] = v;
    z[l * P + c] = (l == c) ? 1.0 : 0.0;
  }
  __syncwarp();
  const int mp = (m + 1) & ~1;
  bool converged = (m <= 1);
  // a rotation is skipped when |a_pq| <= eps sqrt(|a_pp a_qq|); a sweep without rotations ends the solve
  for (int sweep = 0; sweep < 40 && !converged; ++sweep) {
    bool rotated = false;
    for (int r = 0; r < mp - 1; ++r) {
      if (l < mp / 2) {
        int p, q;
        if (l == 0) {
          p = r;
          q = mp - 1;
        } else {
          p = (r + l) % (mp - 1);
          q = (r - l + mp - 1) % (mp - 1);
        }
        if (p > q) {
          const int x = p;
          p = q;
          q = x;
        }
        double c = 1.0, sn = 0.0;
        bool did = false;
        if (q < m) {
          const double apq = a[p * P + q], app = a[p * P + p], aqq = a[q * P + q];
          if (apq != 0.0 && fabs(apq) > kEps * sqrt(fabs(app * aqq))) {
            const double th = (aqq - app) / (2.0 * apq);
            const double t = copysign(1.0, th) / (fabs(th) + sqrt(1.0 + th * th));
            c = 1.0 / sqrt(1.0 + t * t);
            sn = t * c;
            did = true;
          }
        }
        rotated |= did;
        rpi[l] = p;
        rqi[l] = did ? q : p;
        rc[l] = c;
        rs[l] = sn;
      }
      __syncwarp();
      // columns: A <- A J, Z <- Z J   (lane = row)
      for (int x = 0; x < mp / 2; ++x) {
        const int p = rpi[x], q = rqi[x];
        if (p == q) continue;
        const double c = rc[x], sn = rs[x];
        const double ap = a[l * P + p], aq = a[l * P + q];
        a[l * P + p] = c * ap - sn * aq;
        a[l * P + q] = sn * ap + c * aq;
        const double zp = z[l * P + p], zq = z[l * P + q];
        z[l * P + p] = c * zp - sn * zq;
        z[l * P + q] = sn * zp + c * zq;
      }
      __syncwarp();
      // rows: A <- J^T A   (lane = column)
      for (int x = 0; x < mp / 2; ++x) {
        const int p = rpi[x], q = rqi[x];
        if (p == q) continue;
        const double c = rc[x], sn = rs[x];
        const double ap = a[p * P + l], aq = a[q * P + l];
        a[p * P + l] = c * ap - sn * aq;
        a[q * P + l] = sn * ap + c * aq;
      }
      __syncwarp();
    }
    converged = !__any_sync(0xffffffffu, rotated);
  }
  if (!converged) {
    if (l == 0) atomicExch(err, 1);
    return;
  }
  if (l < m) {
    for (int c = 0; c < m; ++c) Q[(int64_t)(L.s + l) + ldq * (L.s + c)] = z[l * P + c];
    D[L.s + l] = a[l * P + l];
  }
}

struct Merge {
  int s, n1, n2;
  int64_t qp_off, uk_off;
};

// Per-merge scratch (offsets s for n-sized arrays, 2s for the sort keys).
struct DcScratch {
  double *keys, *ds, *zs, *dk, *zk, *ddef, *rc, *rs, *tau, *rho;
  int *kidx, *colS, *colk, *coldef, *rp, *ri, *org, *cnt;
};

// The scratch of matrix z of a batch (cnt and rho are indexed by merge + nm * z instead).
__device__ __forceinline__ DcScratch sc_at(DcScratch sc, int64_t z, int64_t n) {
  sc.keys += 2 * n * z;
  sc.kidx += 2 * n * z;
  sc.ds += n * z;
  sc.zs += n * z;
  sc.dk += n * z;
  sc.zk += n * z;
  sc.ddef += n * z;
  sc.rc += n * z;
  sc.rs += n * z;
  sc.tau += n * z;
  sc.colS += n * z;
  sc.colk += n * z;
  sc.coldef += n * z;
  sc.rp += n * z;
  sc.ri += n * z;
  sc.org += n * z;
  return sc;
}

// Sort the poles, form z from the children's boundary rows, deflate (one CTA per merge).
__global__ void __launch_bounds__(1024) merge_prepare_kernel(const Merge* merges, const double* D, const double* Q,
                                                             int64_t ldq, const double* e, DcScratch sc, int nfull,
                                                             int64_t mstride, int nm) {
  __shared__ double red[33];
  const Merge M = merges[blockIdx.x];
  const int64_t mz = blockIdx.x + (int64_t)nm * blockIdx.y;  // (merge, matrix)
  D += (int64_t)nfull * blockIdx.y;
  Q += mstride * blockIdx.y;
  e += (int64_t)nfull * blockIdx.y;
  sc = sc_at(sc, blockIdx.y, nfull);
  const int n = M.n1 + M.n2, s = M.s, t = threadIdx.x;
  int P = 1;
  while (P < n) P <<= 1;
  double* keys = sc.keys + 2 * (int64_t)s;
  int* kidx = sc.kidx + 2 * (int64_t)s;
  for (int i = t; i < P; i += blockDim.x) {
    keys[i] = i < n ? D[s + i] : INFINITY;
    kidx[i] = i;
  }
  __syncthreads();
  // bitonic sort (ascending) of (keys, kidx)
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = t; i < P / 2; i += blockDim.x) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool asc = ((lo & size) == 0);
        const double a = keys[lo], b = keys[hi];
        if ((a > b) == asc) {
          keys[lo] = b;
          keys[hi] = a;
          const int x = kidx[lo];
          kidx[lo] = kidx[hi];
          kidx[hi] = x;
        }
      }
      __syncthreads();
    }
  }
  const double eb = e[s + M.n1 - 1];
  const double sgn = eb >= 0.0 ? 1.0 : -1.0;
  const double rho = 2.0 * fabs(eb);
  const double inv_sqrt2 = 0.70710678118654752440;
  double mx = 0.0;
  for (int i = t; i < n; i += blockDim.x) {
    const int idx = kidx[i];
    const double dv = keys[i];
    const double zv = (idx < M.n1 ? Q[(int64_t)(s + M.n1 - 1) + ldq * (s + idx)]
                                  : sgn * Q[(int64_t)(s + M.n1) + ldq * (s + idx)]) *
                      inv_sqrt2;
    sc.ds[s + i] = dv;
    sc.zs[s + i] = zv;
    sc.colS[s + i] = idx;
    mx = fmax(mx, fabs(dv));
  }
  const double dmax = block_max(mx, red);
  if (t != 0) return;
  const double tol = 8.0 * kEps * fmax(dmax, rho);
  int k = 0, nd = 0, nr = 0;
  bool have = false;
  double pd = 0.0, pz = 0.0;
  int pcol = 0;
  for (int i = 0; i < n; ++i) {
    const double dt = sc.ds[s + i], zt = sc.zs[s + i];
    const int col = sc.colS[s + i];
    if (rho * fabs(zt) <= tol) {
      sc.ddef[s + nd] = dt;
      sc.coldef[s + nd] = col;
      ++nd;
      continue;
    }
    if (!have) {
      have = true;
      pd = dt;
      pz = zt;
      pcol = col;
      continue;
    }
    const double r = hypot(pz, zt);
    const double c = zt / r, sn = pz / r;
    if (fabs((dt - pd) * c * sn) <= tol) {
      sc.rp[s + nr] = pcol;
      sc.ri[s + nr] = col;
      sc.rc[s + nr] = c;
      sc.rs[s + nr] = sn;
      ++nr;
      sc.ddef[s + nd] = pd * c * c + dt * sn * sn;
      sc.coldef[s + nd] = pcol;
      ++nd;
      pd = pd * sn * sn + dt * c * c;
      pz = r;
      pcol = col;
    } else {
      sc.dk[s + k] = pd;
      sc.zk[s + k] = pz;
      sc.colk[s + k] = pcol;
      ++k;
      pd = dt;
      pz = zt;
      pcol = col;
    }
  }
  if (have) {
    sc.dk[s + k] = pd;
    sc.zk[s + k] = pz;
    sc.colk[s + k] = pcol;
    ++k;
  }
  sc.cnt[2 * mz] = k;
  sc.cnt[2 * mz + 1] = nr;
  sc.rho[mz] = rho;
}

// Apply the deflation rotations to the merge's block of Q (thread per row) and gather its
// columns as [non-deflated (k) | deflated] into Qp (n x n, ld n).
__global__ void merge_gather_kernel(const Merge* merges, double* Q, int64_t ldq, double* Qp_base, DcScratch sc,
                                    int nfull, int64_t mstride, int nm) {
  const Merge M = merges[blockIdx.y];
  const int n = M.n1 + M.n2, s = M.s;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t mz = blockIdx.y + (int64_t)nm * blockIdx.z;
  Q += mstride * blockIdx.z;
  Qp_base += mstride * blockIdx.z;
  sc = sc_at(sc, blockIdx.z, nfull);
  const int k = sc.cnt[2 * mz], nr = sc.cnt[2 * mz + 1];
  double* row = Q + (int64_t)(s + r) + ldq * s;  // row r of the block: row[ldq * col]
  for (int q = 0; q < nr; ++q) {
    const int64_t a = ldq * sc.rp[s + q], b = ldq * sc.ri[s + q];
    const double c = sc.rc[s + q], sn = sc.rs[s + q];
    const double x = row[a], y = row[b];
    row[a] = c * x - sn * y;
    row[b] = sn * x + c * y;
  }
  double* Qp = Qp_base + M.qp_off;
  for (int c = 0; c < k; ++c) Qp[r + (int64_t)n * c] = row[ldq * sc.colk[s + c]];
  for (int c = 0; c < n - k; ++c) Qp[r + (int64_t)n * (k + c)] = row[ldq * sc.coldef[s + c]];
}

// Roots of 1 + rho sum_i z_i^2 / (d_i - lambda) = 0 by bisection on tau = lambda - d_org, with
// d_org the pole nearer to the root (warp per root).
__global__ void __launch_bounds__(256) secular_kernel(const Merge* merges, DcScratch sc, int nfull, int nm) {
  const Merge M = merges[blockIdx.y];
  const int s = M.s;
  const int64_t mz = blockIdx.y + (int64_t)nm * blockIdx.z;
  sc = sc_at(sc, blockIdx.z, nfull);
  const int k = sc.cnt[2 * mz];
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (j >= k) return;
  const double rho = sc.rho[mz];
  const double* dk = sc.dk + s;
  const double* zk = sc.zk + s;
  double z2 = 0.0;
  for (int i = lane; i < k; i += 32) z2 += zk[i] * zk[i];
  z2 = warp_sum(z2);
  const double lo = dk[j];
  int org;
  double a, b;
  if (j < k - 1) {
    const double hi = dk[j + 1];
    const double mid = 0.5 * (lo + hi);
    double f = 0.0;
    for (int i = lane; i < k; i += 32) f += zk[i] * zk[i] / (dk[i] - mid);
    f = 1.0 + rho * warp_sum(f);
    if (f >= 0.0) {
      org = j;
      a = 0.0;
      b = mid - lo;
    } else {
      org = j + 1;
      a = mid - hi;
      b = 0.0;
    }
  } else {
    org = j;
    a = 0.0;
    b = rho * z2;
  }
  const double dorg = dk[org];
  double tau = 0.5 * (a + b);
  for (int it = 0; it < 400; ++it) {
    tau = 0.5 * (a + b);
    if (tau == a || tau == b) break;
    double f = 0.0;
    for (int i = lane; i < k; i += 32) f += zk[i] * zk[i] / ((dk[i] - dorg) - tau);
    f = 1.0 + rho * warp_sum(f);
    if (f > 0.0) b = tau;
    else if (f < 0.0) a = tau;
    else break;
  }
  if (lane == 0) {
    sc.tau[s + j] = tau;
    sc.org[s + j] = org;
  }
}

// Loewner formula: zhat_i = sign(z_i) sqrt(-prod_j (d_i - lambda_j) / prod_{j != i} (d_i - d_j) / rho);
// overwrites zk (the secular roots are already fixed).
__global__ void lowner_kernel(const Merge* merges, DcScratch sc, double* zhat, int nfull, int nm) {
  const Merge M = merges[blockIdx.y];
  const int s = M.s;
  const int64_t mz = blockIdx.y + (int64_t)nm * blockIdx.z;
  sc = sc_at(sc, blockIdx.z, nfull);
  zhat += (int64_t)nfull * blockIdx.z;
  const int k = sc.cnt[2 * mz];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  const double* dk = sc.dk + s;
  const double di = dk[i];
  double w = 1.0;
  for (int j = 0; j < k; ++j) {
    const double delta = (di - dk[sc.org[s + j]]) - sc.tau[s + j];
    w *= (j == i) ? delta : delta / (di - dk[j]);
  }
  zhat[s + i] = copysign(sqrt(fmax(-w, 0.0) / sc.rho[mz]), sc.zk[s + i]);
}

// Columns of the rank-one problem's eigenvectors, u_j(i) = zhat_i / (d_i - lambda_j) normalised
// (block per column), and the merged eigenvalues (non-deflated roots, then the deflated poles).
__global__ void __launch_bounds__(256) merge_vectors_kernel(const Merge* merges, DcScratch sc, const double* zhat,
                                                            double* Uk_base, double* D, int nfull, int64_t mstride,
                                                            int nm) {
  __shared__ double red[33];
  const Merge M = merges[blockIdx.y];
  const int n = M.n1 + M.n2, s = M.s;
  const int64_t mz = blockIdx.y + (int64_t)nm * blockIdx.z;
  sc = sc_at(sc, blockIdx.z, nfull);
  zhat += (int64_t)nfull * blockIdx.z;
  Uk_base += mstride * blockIdx.z;
  D += (int64_t)nfull * blockIdx.z;
  const int k = sc.cnt[2 * mz];
  const int j = blockIdx.x;
  if (j >= n) return;
  if (j >= k) {
    if (threadIdx.x == 0) D[s + j] = sc.ddef[s + (j - k)];
    return;
  }
  const double* dk = sc.dk + s;
  const double dorg = dk[sc.org[s + j]], tau = sc.tau[s + j];
  double* u = Uk_base + M.uk_off + (int64_t)k * j;
  double part = 0.0;
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    const double v = zhat[s + i] / ((dk[i] - dorg) - tau);
    u[i] = v;
    part += v * v;
  }
  const double inv = 1.0 / sqrt(block_sum(part, red));
  for (int i = threadIdx.x; i < k; i += blockDim.x) u[i] *= inv;
  if (threadIdx.x == 0) D[s + j] = dorg + tau;
}

// Deflated columns of every (merge, matrix): Q(block)(:, k ..) = Qp(:, k ..) (the rank-one
// problem's eigenvectors replace columns 0 .. k-1 through a GEMM).
__global__ void copy_deflated_kernel(const Merge* merges, const double* Qp_base, double* Q, int64_t ldq,
                                     const int* cnt, int64_t mstride, int nm) {
  const Merge M = merges[blockIdx.y];
  const int n = M.n1 + M.n2, s = M.s;
  const int64_t mz = blockIdx.y + (int64_t)nm * blockIdx.z;
  const int k = cnt[2 * mz];
  const int64_t total = (int64_t)n * (n - k);
  const double* Qp = Qp_base + mstride * blockIdx.z + M.qp_off;
  double* blk = Q + mstride * blockIdx.z + s + ldq * s;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx % n, c = k + idx / n;
    blk[r + ldq * c] = Qp[r + (int64_t)n * c];
  }
}

GemmF64Args gemm_args(int M, int N, int64_t K, const double* A, int64_t a_m, int64_t a_k, const double* B,
                      int64_t b_k, int64_t b_n, double* C, int64_t ldc, double alpha, double beta) {
  GemmF64Args g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = A;
  g.a_m = a_m;
  g.a_k = a_k;
  g.B = B;
  g.b_k = b_k;
  g.b_n = b_n;
  g.C = C;
  g.ldc = ldc;
  g.alpha = alpha;
  g.beta = beta;
  g.batch = 1;
  return g;
}

struct Node {
  int s, n, depth;
};

void build_tree(int s, int n, int depth, std::vector<Node>& nodes) {
  nodes.push_back({s, n, depth});
  if (n <= kLeaf) return;
  const int n1 = n / 2;
  build_tree(s, n1, depth + 1, nodes);
  build_tree(s + n1, n - n1, depth + 1, nodes);
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

size_t syevd_workspace_bytes(int n, int nmat) {
  const size_t nn = (size_t)n * n, B = (size_t)std::max(nmat, 1);
  size_t b = 0;
  b += 3 * align256(B * nn * 8);                    // V (Householder vectors), Qp, Uk
  b += align256(B * n * kNB * 8);                   // Wp
  b += 2 * align256(B * kNB * n * 8);               // Y, Y2
  b += 2 * align256(B * kNB * kNB * 8);             // G, T
  b += align256(std::max((size_t)16 * kNB * n, (size_t)64 * kNB * kNB) * 8);  // split-K partials (one matrix)
  b += 6 * align256(B * n * 8);                     // y, tau, d, e, zhat, D
  b += align256(B * 2 * n * 8) + align256(B * 2 * n * 4);  // sort keys
  b += 8 * align256(B * n * 8);                     // ds zs dk zk ddef rc rs tau
  b += 6 * align256(B * n * 4);                     // colS colk coldef rp ri org
  b += align256(B * n * 8) + align256(B * n * 4);   // rho, cnt (per merge and matrix)
  b += 2 * align256((size_t)n * sizeof(Merge)) + align256((size_t)n * sizeof(Leaf)) + align256((size_t)n * 4);
  b += align256((B * ((size_t)n / kLeaf + 2)) * (sizeof(GemmF64Args) + 8) + 64);  // grouped-GEMM descriptors
  return b + 4096 + 256;
}

size_t syevd_workspace_bytes(int n) { return syevd_workspace_bytes(n, 1); }

// Eigen-decompositions of nmat symmetric n x n matrices A_z = A + z n^2 (column-major, ld n;
// destroyed).  Z_z = Z + z n^2 receives the eigenvectors, evals (host, nmat x n) the eigenvalues in
// the order of the columns (not sorted).  Every stage runs all matrices in the same launches.
cudaError_t syevd_batched(double* A, int n, int nmat, double* Z, void* work, size_t work_bytes,
                          std::vector<double>& evals, bool& converged, cudaStream_t stream) {
  converged = false;
  if (n < 1 || nmat < 1) return cudaErrorInvalidValue;
  if (work_bytes < syevd_workspace_bytes(n, nmat)) return cudaErrorInvalidValue;
  const int64_t ld = n;
  const size_t nn = (size_t)n * n, B = (size_t)nmat;
  const int64_t ms = (int64_t)nn;  // matrix stride
  char* w = static_cast<char*>(work);
  auto take = [&](size_t bytes) {
    void* p = w;
    w += align256(bytes);
    return p;
  };
  double* V = (double*)take(B * nn * 8);
  double* Qp = (double*)take(B * nn * 8);
  double* Uk = (double*)take(B * nn * 8);
  double* Wp = (double*)take(B * n * kNB * 8);
  double* Y = (double*)take(B * kNB * n * 8);
  double* Y2 = (double*)take(B * kNB * n * 8);
  double* Gm = (double*)take(B * kNB * kNB * 8);
  double* Tb = (double*)take(B * kNB * kNB * 8);
  double* Pk = (double*)take(std::max((size_t)16 * kNB * n, (size_t)64 * kNB * kNB) * 8);
  double* y = (double*)take(B * n * 8);
  double* tau = (double*)take(B * n * 8);
  double* d = (double*)take(B * n * 8);
  double* e = (double*)take(B * n * 8);
  double* zhat = (double*)take(B * n * 8);
  double* D = (double*)take(B * n * 8);
  DcScratch sc;
  sc.keys = (double*)take(B * 2 * n * 8);
  sc.kidx = (int*)take(B * 2 * n * 4);
  sc.ds = (double*)take(B * n * 8);
  sc.zs = (double*)take(B * n * 8);
  sc.dk = (double*)take(B * n * 8);
  sc.zk = (double*)take(B * n * 8);
  sc.ddef = (double*)take(B * n * 8);
  sc.rc = (double*)take(B * n * 8);
  sc.rs = (double*)take(B * n * 8);
  sc.tau = (double*)take(B * n * 8);
  sc.colS = (int*)take(B * n * 4);
  sc.colk = (int*)take(B * n * 4);
  sc.coldef = (int*)take(B * n * 4);
  sc.rp = (int*)take(B * n * 4);
  sc.ri = (int*)take(B * n * 4);
  sc.org = (int*)take(B * n * 4);
  sc.rho = (double*)take(B * n * 8);
  sc.cnt = (int*)take(B * n * 4);
  Merge* dMerges = (Merge*)take((size_t)n * sizeof(Merge));
  Leaf* dLeaves = (Leaf*)take((size_t)n * sizeof(Leaf));
  int* dBounds = (int*)take((size_t)n * 4);
  const size_t desc_bytes = (B * ((size_t)n / kLeaf + 2)) * (sizeof(GemmF64Args) + 8) + 64;
  void* dDesc = take(desc_bytes);
  int* err_dev = (int*)take(sizeof(int));
  cudaError_t err;
#define SY_CHECK(x)                             \
  do {                                          \
    if ((err = (x)) != cudaSuccess) return err; \
  } while (0)
  auto batched = [&](GemmF64Args g, int64_t sA, int64_t sB, int64_t sC) {
    g.batch = nmat;
    g.sA = sA;
    g.sB = sB;
    g.sC = sC;
    return g;
  };

  // ---- stage 1: tridiagonal reduction (one 8-CTA cluster per matrix per column step)
  for (int p = 0; p <= n - 2; p += kNB) {
    const int nb = std::min(kNB, n - 1 - p);
    house_kernel<<<kCS * nmat, kCT, 0, stream>>>(A, n, ms, V, Wp, p, -1, 0, y, tau, d, e);
    ++g_launches;
    for (int i = 0; i < nb; ++i) {
      const int j = p + i;
      const int m = n - 1 - j;
      trailing_gemv_kernel<<<dim3((m + 8 / kGemvWarps - 1) / (8 / kGemvWarps), nmat), 256, 0, stream>>>(
          A, n, ms, V + ld * j, j, y);
      ++g_launches;
      house_kernel<<<kCS * nmat, kCT, 0, stream>>>(A, n, ms, V, Wp, p, i, i + 1 < nb ? i + 1 : -1, y, tau, d, e);
      ++g_launches;
    }
    SY_CHECK(cudaGetLastError());
    const int pe = p + nb;
    if (pe < n) {
      const int mt = n - pe;
      // A(pe:, pe:) -= V W^T + W V^T   (panel columns p..p+nb-1)
      SY_CHECK(launch_gemm_f64(batched(gemm_args(mt, mt, nb, V + pe + ld * p, 1, ld, Wp + pe, ld, 1, A + pe + ld * pe,
                                                 ld, -1.0, 1.0),
                                       ms, (int64_t)n * kNB, ms),
                               stream));
      SY_CHECK(launch_gemm_f64(batched(gemm_args(mt, mt, nb, Wp + pe, 1, ld, V + pe + ld * p, ld, 1, A + pe + ld * pe,
                                                 ld, -1.0, 1.0),
                                       (int64_t)n * kNB, ms, ms),
                               stream));
    }
  }
  SY_CHECK(cudaMemcpy2DAsync(d + (n - 1), (size_t)n * 8, A + (n - 1) + ld * (n - 1), nn * 8, 8, B,
                             cudaMemcpyDeviceToDevice, stream));

  // ---- stage 2: divide and conquer on (d, e), the same tree for every matrix
  SY_CHECK(cudaMemsetAsync(Z, 0, B * nn * 8, stream));
  SY_CHECK(cudaMemsetAsync(err_dev, 0, sizeof(int), stream));
  std::vector<Node> nodes;
  build_tree(0, n, 0, nodes);
  int maxdepth = 0;
  for (const Node& nd : nodes) maxdepth = std::max(maxdepth, nd.depth);
  std::vector<Leaf> leaves;
  std::vector<int> bounds;
  std::vector<std::vector<Merge>> levels(maxdepth + 1);
  for (const Node& nd : nodes) {
    if (nd.n <= kLeaf) {
      leaves.push_back({nd.s, nd.n});
    } else {
      const int n1 = nd.n / 2;
      bounds.push_back(nd.s + n1);
      levels[nd.depth].push_back({nd.s, n1, nd.n - n1, 0, 0});
    }
  }
  if (!bounds.empty()) {
    SY_CHECK(cudaMemcpyAsync(dBounds, bounds.data(), bounds.size() * 4, cudaMemcpyHostToDevice, stream));
    const int64_t tot = (int64_t)bounds.size() * nmat;
    tear_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, stream>>>(d, e, dBounds, (int)bounds.size(), n, nmat);
    ++g_launches;
  }
  SY_CHECK(cudaMemcpyAsync(dLeaves, leaves.data(), leaves.size() * sizeof(Leaf), cudaMemcpyHostToDevice, stream));
  leaf_jacobi_kernel<<<dim3((unsigned)leaves.size(), nmat), 32, 0, stream>>>(dLeaves, d, e, D, Z, ld, err_dev, n, ms);
  ++g_launches;
  SY_CHECK(cudaGetLastError());
  std::vector<int> cnt;
  for (int depth = maxdepth; depth >= 0; --depth) {
    std::vector<Merge>& mv = levels[depth];
    if (mv.empty()) continue;
    int64_t off = 0;
    int nmax = 0;
    for (Merge& m : mv) {
      const int nm = m.n1 + m.n2;
      m.qp_off = off;
      m.uk_off = off;
      off += (int64_t)nm * nm;
      nmax = std::max(nmax, nm);
    }
    const int nm_ = (int)mv.size();
    SY_CHECK(cudaMemcpyAsync(dMerges, mv.data(), mv.size() * sizeof(Merge), cudaMemcpyHostToDevice, stream));
    merge_prepare_kernel<<<dim3(nm_, nmat), 1024, 0, stream>>>(dMerges, D, Z, ld, e, sc, n, ms, nm_);
    merge_gather_kernel<<<dim3((nmax + 127) / 128, nm_, nmat), 128, 0, stream>>>(dMerges, Z, ld, Qp, sc, n, ms, nm_);
    secular_kernel<<<dim3((nmax + 7) / 8, nm_, nmat), 256, 0, stream>>>(dMerges, sc, n, nm_);
    lowner_kernel<<<dim3((nmax + 127) / 128, nm_, nmat), 128, 0, stream>>>(dMerges, sc, zhat, n, nm_);
    merge_vectors_kernel<<<dim3(nmax, nm_, nmat), 256, 0, stream>>>(dMerges, sc, zhat, Uk, D, n, ms, nm_);
    copy_deflated_kernel<<<dim3((unsigned)std::min<int64_t>(((int64_t)nmax * nmax + 255) / 256, 1024), nm_, nmat), 256,
                           0, stream>>>(dMerges, Qp, Z, ld, sc.cnt, ms, nm_);
    g_launches += 6;
    SY_CHECK(cudaGetLastError());
    cnt.resize(2 * (size_t)nm_ * nmat);
    SY_CHECK(cudaMemcpyAsync(cnt.data(), sc.cnt, cnt.size() * 4, cudaMemcpyDeviceToHost, stream));
    SY_CHECK(cudaStreamSynchronize(stream));  // mv and cnt must outlive their copies
    std::vector<GemmF64Args> probs;
    for (int z = 0; z < nmat; ++z)
      for (int q = 0; q < nm_; ++q) {
        const Merge& m = mv[q];
        const int nm = m.n1 + m.n2, k = cnt[2 * ((size_t)q + (size_t)nm_ * z)];
        if (k > 0)
          probs.push_back(gemm_args(nm, k, k, Qp + ms * z + m.qp_off, 1, nm, Uk + ms * z + m.uk_off, 1, k,
                                    Z + ms * z + m.s + ld * m.s, ld, 1.0, 0.0));
      }
    SY_CHECK(launch_gemm_f64_grouped(probs, dDesc, desc_bytes, stream));
  }

  // ---- stage 3: Z <- Q_H Z, panels in reverse order
  const int last_p = ((n - 2) / kNB) * kNB;
  for (int p = n >= 2 ? last_p : -1; p >= 0; p -= kNB) {
    const int nb = std::min(kNB, n - 1 - p);
    const int mr = n - 1 - p;  // rows p+1 .. n-1
    const double* Vb = V + (p + 1) + ld * p;
    GemmF64Args gg = gemm_args(nb, nb, mr, Vb, ld, 1, Vb, 1, ld, Gm, kNB, 1.0, 0.0);
    GemmF64Args gy = gemm_args(nb, n, mr, Vb, ld, 1, Z + (p + 1), 1, ld, Y, kNB, 1.0, 0.0);
    if (nmat == 1) {
      // G = V_b^T V_b and Y = V_b^T Z have few output tiles and K = mr: split K
      gg.splitk = std::max(1, std::min(64, mr / 256));
      gg.work = Pk;
      const int ytiles = (n + 63) / 64;  // about 600 CTA slots (148 SMs x 4), K chunks >= 256
      gy.splitk = std::max(1, std::min(16, std::min(mr / 256, 600 / ytiles)));
      gy.work = Pk;
    } else {
      gg = batched(gg, ms, ms, (int64_t)kNB * kNB);
      gy = batched(gy, ms, ms, (int64_t)kNB * n);
    }
    SY_CHECK(launch_gemm_f64(gg, stream));
    build_t_kernel<<<nmat, 32, 0, stream>>>(Gm, tau + p, nb, Tb, n);
    ++g_launches;
    SY_CHECK(launch_gemm_f64(gy, stream));
    SY_CHECK(launch_gemm_f64(batched(gemm_args(nb, n, nb, Tb, 1, kNB, Y, 1, kNB, Y2, kNB, 1.0, 0.0),
                                     (int64_t)kNB * kNB, (int64_t)kNB * n, (int64_t)kNB * n),
                             stream));
    SY_CHECK(launch_gemm_f64(batched(gemm_args(mr, n, nb, Vb, 1, ld, Y2, 1, kNB, Z + (p + 1), ld, -1.0, 1.0), ms,
                                     (int64_t)kNB * n, ms),
                             stream));
  }
  evals.resize(B * n);
  SY_CHECK(cudaMemcpyAsync(evals.data(), D, B * n * 8, cudaMemcpyDeviceToHost, stream));
  int herr = 0;
  SY_CHECK(cudaMemcpyAsync(&herr, err_dev, sizeof(int), cudaMemcpyDeviceToHost, stream));
  SY_CHECK(cudaStreamSynchronize(stream));
  converged = (herr == 0);  // a leaf's Jacobi iteration can fail to converge
  return cudaSuccess;
#undef SY_CHECK
}

cudaError_t syevd(double* A, int n, double* Z, void* work, size_t work_bytes, std::vector<double>& evals,
                  bool& converged, cudaStream_t stream) {
  return syevd_batched(A, n, 1, Z, work, work_bytes, evals, converged, stream);
}

}  // namespace rpa
