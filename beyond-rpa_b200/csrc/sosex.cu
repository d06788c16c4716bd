// SOSEX exchange contraction (rpa_CC_Exchange_SOSEX + rpa_CC_EcExchange1,
// src/rpa/rpa_CC_Exchange.f90:36-116):
//
//   E_x = -alpha * sum_{i>=j} (2 - delta_ij) sum_{Q,mu} B_mu W_ij(Q,mu) W_ji(Q,mu),
//   W_ij = R(:, :, i) U(:, :, j)^T   (sum over the virtual index a),
//
// with B = A (SOSEX) or A/(1-4A^2) (S^2 operator).  The reference forms
// W_ij and W_ji with two DGEMMs per occupied pair and reduces them with
// co_sum; here one CTA computes a 64 x 64 tile (Q, mu) of both W_ij and W_ji
// for one pair on the FP64 tensor-core path, multiplies them in registers
// and writes one partial sum (no W is stored; partials are reduced in a fixed
// order on the host, so the result is deterministic).
// R(Q, a + nv*i) is column-major with leading dimension ldR; U(a + nv*j, mu)
// is column-major (nov x NT) with leading dimension ldU (the Uaim layout of
// rpa_THC_CC_T2).
#include "kernels.h"

namespace rpa {

namespace {
constexpr int BM = 64;
constexpr int BK = 16;
constexpr int LDS = BM + 8;
constexpr int kThreads = 128;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void pair_decode(int p, int& i, int& j) {
  // p enumerates (i, j) with i >= j: p = i*(i+1)/2 + j
  int t = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while ((t + 1) * (t + 2) / 2 <= p) ++t;
  while (t * (t + 1) / 2 > p) --t;
  i = t;
  j = p - t * (t + 1) / 2;
}

// W_ij is formed from U1 and W_ji from U2 (U2 == U1 for SOSEX; U1 = U X for
// the Tr(XK) contraction of the MBPT3 exchange).
__global__ void __launch_bounds__(kThreads) sosex_kernel(const double* __restrict__ R, int64_t ldR, int NQ, int nv,
                                                         const double* __restrict__ U, int64_t ldU,
                                                         const double* __restrict__ U2, int64_t ldU2, int NT,
                                                         const double* __restrict__ Bmu, double* partial) {
  __shared__ double Ri[BK][LDS], Rj[BK][LDS], Uj[BK][LDS], Ui[BK][LDS];
  __shared__ double red[kThreads / 32];
  int i, j;
  pair_decode(blockIdx.x, i, j);
  const bool same = (U2 == U);
  const bool diag = (i == j) && same;  // W_ii W_ii: one accumulator suffices
  const int q0 = blockIdx.y * BM, m0 = blockIdx.z * BM;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int wm = warp >> 1, wn = warp & 1;

  double a1[4][4][2], a2[4][4][2];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) a1[x][y][0] = a1[x][y][1] = a2[x][y][0] = a2[x][y][1] = 0.0;

  for (int a0 = 0; a0 < nv; a0 += BK) {
    // R tiles: 16 columns (a) of 64 contiguous Q
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const int idx = t + kThreads * s;
      const int r = idx % BM, c = idx / BM;
      const int q = q0 + r, a = a0 + c;
      const bool ok = (q < NQ && a < nv);
      Ri[c][r] = ok ? R[(int64_t)q + ldR * ((int64_t)a + (int64_t)nv * i)] : 0.0;
      Rj[c][r] = (ok && !diag) ? R[(int64_t)q + ldR * ((int64_t)a + (int64_t)nv * j)] : 0.0;
    }
    // U tiles: rows a (contiguous) x 64 columns mu
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const int idx = t + kThreads * s;
      const int c = idx % BK, r = idx / BK;  // c: a (fast), r: mu
      const int mu = m0 + r, a = a0 + c;
      const bool ok = (mu < NT && a < nv);
      Uj[c][r] = ok ? U[((int64_t)a + (int64_t)nv * j) + ldU * mu] : 0.0;
      Ui[c][r] = (ok && !diag) ? U2[((int64_t)a + (int64_t)nv * i) + ldU2 * mu] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      const int kr = kk + (lane & 3);
      double fri[4], frj[4], fuj[4], fui[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        fri[x] = Ri[kr][wm * 32 + x * 8 + (lane >> 2)];
        frj[x] = Rj[kr][wm * 32 + x * 8 + (lane >> 2)];
      }
#pragma unroll
      for (int y = 0; y < 4; ++y) {
        fuj[y] = Uj[kr][wn * 32 + y * 8 + (lane >> 2)];
        fui[y] = Ui[kr][wn * 32 + y * 8 + (lane >> 2)];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) {
          dmma(a1[x][y][0], a1[x][y][1], fri[x], fuj[y]);
          if (!diag) dmma(a2[x][y][0], a2[x][y][1], frj[x], fui[y]);
        }
    }
    __syncthreads();
  }
  // Hadamard-reduce epilogue (out-of-range rows/columns hold zeros)
  double s = 0.0;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int mu = m0 + wn * 32 + y * 8 + 2 * (lane & 3) + v;
        const double b = (mu < NT) ? Bmu[mu] : 0.0;
        const double w2 = diag ? a1[x][y][v] : a2[x][y][v];
        s += b * a1[x][y][v] * w2;
      }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (t == 0) {
    double tot = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) tot += red[w];
    const int64_t idx = ((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * gridDim.z + blockIdx.z;
    partial[idx] = (i == j ? 1.0 : 2.0) * tot;
  }
}
}  // namespace

int64_t sosex_partials(int NQ, int no, int NT) {
  return (int64_t)no * (no + 1) / 2 * ((NQ + BM - 1) / BM) * ((NT + BM - 1) / BM);
}

cudaError_t launch_sosex(const double* R, int64_t ldR, int NQ, int no, int nv, const double* U, int64_t ldU,
                         const double* U2, int64_t ldU2, int NT, const double* Bmu, double* partial, int64_t* npartial,
                         cudaStream_t stream) {
  const int npairs = no * (no + 1) / 2;
  dim3 grid((unsigned)npairs, (unsigned)((NQ + BM - 1) / BM), (unsigned)((NT + BM - 1) / BM));
  *npartial = sosex_partials(NQ, no, NT);
  if (npairs == 0 || NT == 0) return cudaSuccess;
  sosex_kernel<<<grid, kThreads, 0, stream>>>(R, ldR, NQ, nv, U, ldU, U2 ? U2 : U, U2 ? ldU2 : ldU, NT, Bmu,
                                               partial);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
