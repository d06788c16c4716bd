// Internal launch interface between the C-ABI host layer (capi.cu) and the
// sm_100a kernels.  Not installed; the public ABI is include/rpa_b200.h.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "rpa_common.cuh"

namespace rpa {

// Kernel launches issued by this host thread (read and reset by the C-ABI layer).
extern thread_local int64_t g_launches;

// Frequencies handled by one scale/split launch (register-resident diagonal sums).
constexpr int kMaxKgLaunch = 16;

struct FreqGroup {
  int n;                       // number of frequencies in this launch
  double u2[kMaxKgLaunch];     // u_k^2
};

struct SplitPlan {
  int qtiles = 0;
  int nsplit = 0;
  int64_t ai_per_split = 0;
};

SplitPlan plan_scale_split(int NQ, int64_t nov, int num_sms);

// Store views of the split operands X_hi / X_lo written by the scale/split pass: 3-D (ai, Q, k)
// bf16 with row pitch `pitch` (a multiple of 8) and frequency stride pitch * NQ, boxes of 64 ai x
// 32 Q, 128-byte swizzle.  Returns cudaErrorInvalidValue when the driver rejects the map.
cudaError_t encode_split_store_map(PFN_cuTensorMapEncodeTiled_v12000 encode, CUtensorMap* m, void* base,
                                   int64_t nov, int NQ, int kg, int64_t pitch);

// One instance of a multi-instance scale/split launch.
struct SplitJob {
  CUtensorMap tm_hi, tm_lo;  // store views of this instance's X_hi / X_lo (encode_split_store_map)
  const double* R;
  int64_t ldR;
  int NQ;
  int64_t nov;
  const double* D;
  FreqGroup fg;
  double alpha;
  double* diag_part;
  int64_t ai_per_split;
  int nsplit;
  double* diag;  // [fg.n][NQ]
};
// work[b] = (job, q tile, ai split, 0); offsets[j] = sum_{i<j} fg.n * NQ of job i, total = sum.
// A bounded wait that expires records its code in *err.
cudaError_t launch_scale_split_multi(const SplitJob* jobs, const int4* work, int nwork, const int64_t* offsets,
                                     int njobs, int64_t total, int* err, cudaStream_t stream);

// X_k = sqrt(alpha c_k) R split into bf16 hi/lo rows (Q-major rows, ai contiguous, written
// through the store views tm_hi / tm_lo), plus the exact FP64 diagonal
// diag[k*NQ + Q] = sum_ai X_k(Q,ai)^2.
cudaError_t launch_scale_split(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                               const FreqGroup& fg, double alpha, const CUtensorMap* tm_hi, const CUtensorMap* tm_lo,
                               double* diag_part, double* diag, const SplitPlan& plan, int* err, cudaStream_t stream);
// The splits split0 .. split1-1 of the same pass (ai columns split*ai_per_split ..), without the
// diagonal reduction; launch_diag_reduce completes the diagonal once every split has run.
cudaError_t launch_scale_split_part(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                                    const FreqGroup& fg, double alpha, const CUtensorMap* tm_hi,
                                    const CUtensorMap* tm_lo, double* diag_part, const SplitPlan& plan, int split0,
                                    int split1, int* err, cudaStream_t stream);
cudaError_t launch_diag_reduce(const double* diag_part, const SplitPlan& plan, int kg, int NQ, double* diag,
                               cudaStream_t stream);

// ---------------------------------------------------------------- tcgen05 SYRK
struct SyrkTcArgs {
  int NQ;
  int64_t nov;
  int kg;            // frequencies in this launch
  double* Pi;        // output, lower triangle of Pi_k written (incl. diagonal)
  int64_t ldPi;
  int64_t piStride;  // elements between consecutive Pi_k
  const double* diag;  // exact diagonal [kg][NQ]; nullptr: the diagonal is left untouched
  int* err;
  int seg_chunks;    // 32-column chunks per accumulation segment (<= 0: no segmentation)
  // ai sub-range: 32-column chunks chunk0 .. chunk0 + ceil(nov_part / 32) - 1 of X (0, nov: all)
  int chunk0;
  int64_t nov_part;
  int accumulate;    // 1: Pi_k += the sub-range's contribution (FP64), 0: Pi_k = it
  // Optional L2 locality of a wave of persistent CTAs: every sync_every K chunks a producer
  // announces its progress in sync[wave * nmilestones + milestone] (zeroed before the launch)
  // and waits, bounded, until every CTA of its wave has passed milestone - sync_lag.  Purely a
  // performance device: a wait that runs out of time just stops synchronising.
  int* sync;
  int sync_every;
  int sync_lag;
};
// Counters needed by SyrkTcArgs::sync for a launch of this shape (0: no synchronisation).
int64_t syrk_tc_sync_words(int NQ, int kg, int64_t nov_part, int num_sms, int sync_every);
// Tensor maps: 3-D (ai, Q, k) bf16 views of X_hi / X_lo; A maps use a
// 128-row box, B maps a 256-row box, 32 ai per box, 64-byte swizzle.
cudaError_t launch_syrk_split_bf16(const CUtensorMap* tmA_hi, const CUtensorMap* tmA_lo, const CUtensorMap* tmB_hi,
                                   const CUtensorMap* tmB_lo, const SyrkTcArgs& a, int num_sms,
                                   cudaStream_t stream);
// One instance (fragment) of a multi-instance SYRK launch.
struct SyrkInst {
  CUtensorMap tmAh, tmAl, tmBh, tmBl;  // 3-D views of this instance's X_hi / X_lo
  double* Pi;
  int64_t ldPi, piStride;
  const double* diag;
  int NQ;
  int nchunks;  // ceil(nov / 32)
};
// sync (optional, zeroed, syrk_tc_multi_sync_words ints): wave milestones as in SyrkTcArgs; a unit
// shorter than max_chunks releases its wave's remaining milestones when it ends.
cudaError_t launch_syrk_split_bf16_multi(const SyrkInst* insts, const uint4* work, int nunits, int seg_chunks,
                                         int* err, int num_sms, cudaStream_t stream, int* sync = nullptr,
                                         int sync_every = 0, int sync_lag = 2, int max_chunks = 0);
int64_t syrk_tc_multi_sync_words(int nunits, int max_chunks, int num_sms, int sync_every);
// General split-BF16 GEMM on the same tensor-core pipeline (128 x 256 tiles over the full grid):
//   C(m, n) = alpha sum_k A(m, k) B(n, k) + beta C(m, n),  m < M, n < N, FP64 C (column-major, ldc),
// A = A_hi + A_lo (M rows, K contiguous) and B likewise (N rows): maps[4] = A_hi, A_lo (boxes of
// 32 x kSyrkTcTM) and B_hi, B_lo (32 x kSyrkTcTN), 3-D (K, rows, 1).  Rows of both must be padded
// to a multiple of 8 bf16 (16 bytes) with zeros beyond K.
struct GemmSplitArgs {
  int M, N;
  int64_t K;
  double* C;
  int64_t ldc;
  double alpha, beta;
  int seg_chunks;
  int* sync;  // optional wave milestones (zeroed, gemm_split_sync_words ints)
  int sync_every, sync_lag;
  int* err;
};
int64_t gemm_split_sync_words(int M, int N, int64_t K, int num_sms, int sync_every);
cudaError_t launch_gemm_split_bf16(const CUtensorMap* maps, const GemmSplitArgs& a, int num_sms,
                                   cudaStream_t stream);
int syrk_tc_blocks(int NQ);
// (tm, tn) of the lower-triangle 128 x 256 tiles in the kernel's unit order
void syrk_tc_block_coords(int NQ, std::vector<uint2>& out);
constexpr int kSyrkTcTM = 128;
constexpr int kSyrkTcTN = 256;
constexpr int kSyrkTcTK = 32;

// ---------------------------------------------------------------- FP64 (DMMA)
// C(lower) = alpha_scale * sum_k A(m,k) s(k) A(n,k) over k < kdim, or
// C(lower) -= sum_k A(m,k) A(n,k) (subtract mode).  A is column-major with
// leading dimension lda (rows contiguous).  Batched over `batch` matrices:
// A + z*strideA, C + z*strideC, and for scaled mode frequency z uses
// s(k) = alpha * D(k) / (D(k)^2 + u2[z]).
struct DsyrkArgs {
  const double* A;
  int64_t lda;
  int64_t strideA;
  double* C;
  int64_t ldc;
  int64_t strideC;
  int n;          // rows of C (order of the lower triangle)
  int ncols;      // columns of C updated (<= n; 0 means n): lower trapezoid
  int64_t kdim;   // contraction length
  int batch;
  // scaled mode
  const double* D;  // nullptr -> subtract mode
  double alpha;
  double u2[64];
  int tile_w;       // warps per CTA-tile side: 2 (64 x 64 tiles, 128 threads) or 4 (128 x 128, 512); 0 = 2
};
cudaError_t launch_dsyrk_lower(const DsyrkArgs& a, cudaStream_t stream);

// ---------------------------------------------------------------- log-det
// Batched lower Cholesky of nmat matrices (column-major, ld, stride),
// on entry A = 1 + Pi (lower triangle), on exit L; Ldiag[z*n + i] = L_ii.
// Tile plan of the blocked Cholesky: the outer block (columns per trailing update, a multiple
// of kCholNB) and the CTA tile of its FP64 SYRK updates (DsyrkArgs::tile_w).
constexpr int kCholNB = 64;  // inner block: diagonal factorization and panel solve
struct LogdetPlan {
  int nb2;
  int tile_w;
};
LogdetPlan default_logdet_plan();  // 256-column outer block (RPA_B200_CHOL_NB2 overrides), 64 x 64 tiles
bool valid_logdet_plan(const LogdetPlan& p);
// Lookahead schedule of the blocked Cholesky: the critical path (diagonal blocks, panel solves,
// the update of the next outer block) on `crit`, the update of the rest of the trailing matrix on
// `rest`; ev: 4 events without timing.  Both streams join the caller's stream before return.
struct Lookahead {
  cudaStream_t crit, rest;
  cudaEvent_t ev[4];
};
// FP64-accurate trailing updates on the int8 tensor cores (ozaki.cu): digit planes of the current
// panel (two buffers, alternating by outer block) and their tensor maps.
struct OzakiWork {
  int S = 0;  // digits per entry (7 or 8); 0: updates stay on DMMA
  int K = 0;  // panel width (the plan's outer block)
  int8_t* slices[2] = {nullptr, nullptr};
  int* expo[2] = {nullptr, nullptr};
  CUtensorMap mapA[2], mapB[2];
  int num_sms = 0;
};
int ozaki_slices_default();  // 0 (DMMA updates) unless RPA_B200_OZAKI_SLICES = 7 or 8
// Bytes of one of the two buffers for nmat matrices of order n, panel width K, S digits.
size_t ozaki_buffer_bytes(int n, int nmat, int K, int S);
cudaError_t ozaki_setup(OzakiWork& w, PFN_cuTensorMapEncodeTiled_v12000 encode, void* const buf[2], int n, int nmat,
                        int K, int S);
// Exponents and digit planes of rows r0 .. n-1 of the panel A(:, c0 .. c0 + K - 1), into buffer buf.
cudaError_t launch_ozaki_slices(const OzakiWork& w, int buf, const double* A, int64_t ld, int64_t stride, int n,
                                int nmat, int r0, int c0, cudaStream_t stream);
// C(r, c) -= sum_k P(r, k) P(c, k) over the C block rows row0 .. row0 + nrows - 1, columns col0 ..
// col0 + ncols - 1, entries with r >= c, P from buffer buf.
cudaError_t launch_ozaki_update(const OzakiWork& w, int buf, double* A, int64_t ld, int64_t stride, int n, int nmat,
                                int row0, int col0, int nrows, int ncols, int* err, int num_sms, cudaStream_t stream);

cudaError_t launch_cholesky_lower(double* A, int64_t ld, int64_t stride, int n, int nmat, double* Ldiag, int* err,
                                  cudaStream_t stream, const LogdetPlan& plan, const Lookahead* la = nullptr,
                                  const OzakiWork* oz = nullptr);
// tr[z] = sum_i A_z(i,i) (double-double, deterministic); then A_z(i,i) += 1.
// If `diag` is non-null the diagonal is first overwritten with diag[z*n+i].
cudaError_t launch_trace_shift(double* A, int64_t ld, int64_t stride, int n, int nmat, const double* diag,
                               double* tr_dd, cudaStream_t stream);
// logdet[z] = 2 sum_i log(Ldiag[z*n+i]) in double-double.
cudaError_t launch_logdet_sum(const double* Ldiag, int n, int nmat, double* logdet_dd, cudaStream_t stream);
// D(ai) = eps_v(a) - eps_o(i), ai = a + nv*i.
cudaError_t launch_dai(const double* eps_o, const double* eps_v, int64_t no, int64_t nv, double* D,
                       cudaStream_t stream);
// Copy lower triangle to upper (full symmetric square) for nmat matrices.
cudaError_t launch_symmetrize(double* A, int64_t ld, int64_t stride, int n, int nmat, cudaStream_t stream);
// Failure-detection self-test: one bounded wait on an mbarrier nobody arrives on, limit_ns long;
// it records kDevTimeoutSelfTest in *err when it expires.
cudaError_t launch_wait_timeout_selftest(int* err, unsigned long long limit_ns, cudaStream_t stream);
// Count non-finite entries of a device array (result accumulated into *count).
cudaError_t launch_count_nonfinite(const double* x, int64_t n, int* count, cudaStream_t stream);
// The same over the lower triangles (diagonal included) of nmat n x n matrices, ld and stride apart.
cudaError_t launch_count_nonfinite_lower(const double* A, int64_t ld, int64_t stride, int n, int nmat, int* count,
                                         cudaStream_t stream);
// The same over rows 0 .. rows-1 of cols columns of a column-major array, ld apart (rows from rows to
// ld - 1 are a caller's padding and are never read).
cudaError_t launch_count_nonfinite_cols(const double* A, int64_t ld, int64_t rows, int64_t cols, int* count,
                                        cudaStream_t stream);
// The same over narr such arrays: device arrays of pointers and of (ld, rows, cols) triples,
// blocks_per CTAs each.
cudaError_t launch_count_nonfinite_multi(const double* const* ptrs, const int64_t* dims, int narr, int blocks_per,
                                         int* count, cudaStream_t stream);
// Strided 2-D copy of a column-major matrix block (device to device).
cudaError_t launch_copy_lower(const double* src, int64_t lds, int64_t strideS, double* dst, int64_t ldd,
                              int64_t strideD, int n, int nmat, cudaStream_t stream);

// ---------------------------------------------------------------- generic FP64 GEMM
// C_b(m,n) = alpha * rowscale(m) * sum_k A_b(m,k) kscale_b(k) B_b(k,n) + beta * C_b(m,n)
struct GemmF64Args {
  int M, N;
  int64_t K;
  const double* A;
  int64_t a_m, a_k, sA;  // element strides of A (one of a_m, a_k should be 1)
  const double* B;
  int64_t b_k, b_n, sB;
  double* C;
  int64_t ldc, sC;       // C column-major
  double alpha, beta;
  const double* kscale;  // optional, per k (stride ks_stride per batch)
  int64_t ks_stride;
  const double* rowscale;  // optional, per m
  int batch;
  // split-K (batch must be 1): splitk partial products over K ranges go to work
  // (splitk * M * N doubles) and are summed in a fixed order by a second kernel
  int splitk;
  double* work;
};
cudaError_t launch_gemm_f64(const GemmF64Args& g, cudaStream_t stream);
// Independent problems (batch 1, no split-K; the first problem's operand layout picks the load
// mapping) in one launch; their descriptors
// are uploaded (stream-ordered) into dev_buf (probs.size() * sizeof(GemmF64Args) + 4 (n + 1) bytes).
cudaError_t launch_gemm_f64_grouped(const std::vector<GemmF64Args>& probs, void* dev_buf, size_t dev_bytes,
                                    cudaStream_t stream);
// The same with descriptors already on the device: tile_start_dev holds the nprob + 1 prefix sums
// of gemm_f64_tiles (ntiles = the last); a_m_unit / b_n_unit pick the load mapping.
cudaError_t launch_gemm_f64_grouped_dev(const GemmF64Args* probs_dev, const int* tile_start_dev, int nprob,
                                        int ntiles, bool a_m_unit, bool b_n_unit, cudaStream_t stream);
int gemm_f64_tiles(const GemmF64Args& g);

// ---------------------------------------------------------------- T2 chain
// Batched forward substitution L_b X_b = B_b in place (L lower, column-major).
cudaError_t launch_trsm_lower_left(const double* L, int64_t ldl, int64_t sL, double* X, int64_t ldx, int64_t sX,
                                   int n, int ncols, int batch, cudaStream_t stream);
// Batched backward substitution L_b^T X_b = B_b in place (L lower, column-major).
cudaError_t launch_trsm_lower_trans_left(const double* L, int64_t ldl, int64_t sL, double* X, int64_t ldx,
                                         int64_t sX, int n, int ncols, int batch, cudaStream_t stream);
// Adjoint of E_c for a group of <= 16 frequencies (f_k = w_k / 2pi).
struct GradGroup {
  int n;
  double alpha;
  double u2[16];
  double f[16];
};
cudaError_t launch_grad_accum(const double* R, int64_t ldR, const double* Y, int64_t ldy, int64_t sY, int NQ,
                              int64_t nov, const double* D, const GradGroup& gg, double* dR, int64_t lddR, double* dD,
                              bool first, cudaStream_t stream);
cudaError_t launch_replicate(const double* R, int64_t ldR, int NQ, int64_t nov, double* Y, int64_t ldy, int64_t sY,
                             int nb, cudaStream_t stream);
// out: 2 + 240 doubles (sums in out[0], out[1]; per-CTA partials after them)
cudaError_t launch_offdiag(const double* A, int64_t lda, int n, double* out, cudaStream_t stream);
cudaError_t launch_fill_uniform(double* X, int64_t rows, int64_t cols, int64_t ldx, uint64_t seed,
                                cudaStream_t stream);
cudaError_t launch_col_sqnorm(const double* X, int64_t rows, int64_t cols, int64_t ldx, double* out,
                              cudaStream_t stream);
cudaError_t launch_scale_cols(double* X, int64_t rows, int64_t cols, int64_t ldx, const double* s, bool inv_sqrt,
                              cudaStream_t stream);
struct ChiGroup {
  int n;
  double alpha;
  double u2[64];
  double sqrtw[64];
};
cudaError_t launch_chi_scale(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D, const ChiGroup& cg,
                             double* Y, int64_t ldy, cudaStream_t stream);
cudaError_t launch_gather_cols(const double* src, int64_t lds, double* dst, int64_t ldd, int64_t rows, int64_t cols,
                               const int* perm, const double* colscale, cudaStream_t stream);
cudaError_t launch_symmetrize_avg(double* A, int64_t lda, int n, cudaStream_t stream);

// SOSEX pair contraction: partial[tile] of -sum_{i>=j} (2 - delta_ij) sum_{Q,mu} B_mu W_ij W_ji,
// W_ij = R(:, :, i) U(:, :, j)^T; partials reduced on the host in fixed order.
// U2 (nullptr: U) forms W_ji.
cudaError_t launch_sosex(const double* R, int64_t ldR, int NQ, int no, int nv, const double* U, int64_t ldU,
                         const double* U2, int64_t ldU2, int NT, const double* Bmu, double* partial, int64_t* npartial,
                         cudaStream_t stream);
// dst column map[2c+1] <- src column map[2c] for c < ncols (columns of `rows` contiguous doubles).
cudaError_t launch_copy_columns(const double* src, double* dst, const int64_t* map, int64_t ncols, int rows,
                                cudaStream_t stream);
// C = A o B (element-wise).
cudaError_t launch_hadamard(const double* A, int64_t lda, const double* B, int64_t ldb, int rows, int cols,
                            double* C, int64_t ldc, cudaStream_t stream);
// out[0 .. kDotPartials) = per-CTA partial sums of sum_{r,c} w(r) A(r,c) B(r,c) (w may be nullptr).
constexpr int kDotPartials = 64;
cudaError_t launch_dot_partials(const double* A, int64_t lda, const double* B, int64_t ldb, int rows, int cols,
                                const double* w, double* out, cudaStream_t stream);
// YX(g, a + nv*ii) = Xa(g, a) Xi(g, i0 + ii) for ii < ni (YX: ngrid x nv*ni, ld ngrid).
// YX(g, c) = Xa(g, a) Xi(g, i) for the ai columns ai0 .. ai0 + ncols - 1 (ai = a + nv i), ld ngrid.
cudaError_t launch_khatri_rao_cols(const double* Xa, int64_t ldXa, const double* Xi, int64_t ldXi, int ngrid, int nv,
                                   int64_t ai0, int64_t ncols, double* YX, cudaStream_t stream);
// dst[j] += src[j] for j < n (first: dst[j] = src[j]).
cudaError_t launch_add_into(double* dst, const double* src, int64_t n, bool first, cudaStream_t stream);
cudaError_t launch_khatri_rao(const double* Xa, int64_t ldXa, const double* Xi, int64_t ldXi, int ngrid, int nv,
                              int i0, int ni, double* YX, cudaStream_t stream);
// A(i, i) += s * fro2[0]  (shift of a Gram matrix by a multiple of a device-side norm).
cudaError_t launch_add_diag_scaled(double* A, int64_t lda, int n, double s, const double* fro2,
                                  cudaStream_t stream);
// B = A^T (A: rows x cols, column-major).
cudaError_t launch_transpose(const double* A, int64_t lda, int rows, int cols, double* B, int64_t ldb,
                             cudaStream_t stream);
// MBPT3 exchange: A_mn = A_m D_mn + D_mn A_n, B_mn = D_mn + 2 U_mn + 4 U_mn A_n, Bs = (B + B^T)/2.
cudaError_t launch_mbpt3_build(const double* Ukl, const double* Dkl, const double* Avec, int n, double* Amat,
                               double* Bmat, double* Bsym, cudaStream_t stream);
// Y_mn /= (mu_m + mu_n); counts pairs with mu_m + mu_n <= 0 into *bad.
cudaError_t launch_lyap_scale(double* Y, const double* mu, int n, int* bad, cudaStream_t stream);
int64_t sosex_partials(int NQ, int no, int NT);

// ---------------------------------------------------------------- split-BF16 SOSEX (sosex_tc.cu)
// Operands split once into bf16 hi/lo rows of P = no * nvp columns (each occupied block padded
// to nvp = sosex_tc_nvp(nv), a multiple of 32): R -> NQ rows (launch_split_rows), U and U2 ->
// NT rows (launch_split_cols).  maps[6]: 3-D tensor maps (P, rows, 1) with 32 x 128 boxes of
// Rh, Rl, Uh, Ul, U2h, U2l.  partial: 16 FP64 values per unit, (2 - delta_ij) sum B W_ij W_ji.
struct SosexTcArgs {
  int NQ, no, nvp, NT;
  int nqt, nmt, nunits;  // 128-row Q tiles, 128-column mu tiles, pairs x nqt x nmt
  int same;              // U2 is U: the diagonal pairs need W_ii only
  int seg_chunks;        // 32-column chunks per TMEM accumulation segment
  const double* Bmu;
  double* partial;
  int* err;
};
int sosex_tc_nvp(int nv);
int64_t sosex_tc_units(int NQ, int no, int NT);
int64_t sosex_tc_partials(int NQ, int no, int NT);
cudaError_t launch_split_rows(const double* R, int64_t ldR, int NQ, int no, int nv, __nv_bfloat16* Xh,
                              __nv_bfloat16* Xl, cudaStream_t stream);
cudaError_t launch_split_cols(const double* U, int64_t ldU, int NT, int no, int nv, __nv_bfloat16* Xh,
                              __nv_bfloat16* Xl, cudaStream_t stream);
cudaError_t launch_sosex_split_bf16(const CUtensorMap* maps, const SosexTcArgs& a, int num_sms, cudaStream_t stream);
// out[b] = fixed-order sum of x[b*chunk .. (b+1)*chunk); *nout = number of chunks.
cudaError_t launch_chunk_sum(const double* x, int64_t n, int64_t chunk, double* out, int64_t* nout,
                             cudaStream_t stream);

// ---------------------------------------------------------------- variable-size batches
// One matrix of a batch of matrices of different orders (fragments).
struct MatDesc {
  double* A;       // column-major, lower triangle used
  int64_t ld;
  int n;
  double* Ldiag;   // n pivots L_ii
  double* tr_dd;   // 2 doubles: trace before the +1 shift (double-double)
  double* ld_dd;   // 2 doubles: 2 sum log L_ii (double-double)
};
// trace_shift + blocked Cholesky + log sums for nmat matrices of orders <= nmax.
cudaError_t launch_logdet_varlen(const MatDesc* mats, int nmat, int nmax, int* err, cudaStream_t stream,
                                 const LogdetPlan& plan, const Lookahead* la = nullptr);
// Overwrite the lower triangles of the matrices with a seeded, strictly diagonally dominant
// symmetric test matrix (unit diagonal, |off-diagonal row sums| < 1/2): the input of the tile tuner.
// One SYRK step of the variable-size schedule: mode 0 panel update, mode 1 trailing update,
// modes 2 and 3 the two halves of the trailing update under lookahead (the next outer block's
// columns; everything right of them).
cudaError_t launch_dsyrk_varlen(const MatDesc* mats, int nmat, int mode, int J0, int j0, int nb2, int tile_w,
                                int nmax, cudaStream_t stream);
cudaError_t launch_fill_spd_varlen(const MatDesc* mats, int nmat, int nmax, uint64_t seed, cudaStream_t stream);

// ---------------------------------------------------------------- symmetric eigensolver
// Householder tridiagonalisation + divide and conquer + WY back-transformation (syevd.cu).
size_t syevd_workspace_bytes(int n);
size_t syevd_workspace_bytes(int n, int nmat);
// nmat matrices of order n at stride n^2 (A destroyed), eigenvectors into Z at the same stride,
// evals (host) nmat x n; all matrices run in the same launches.
cudaError_t syevd_batched(double* A, int n, int nmat, double* Z, void* work, size_t work_bytes,
                          std::vector<double>& evals, bool& converged, cudaStream_t stream);
// A (n x n, ld n) is destroyed; Z (n x n, ld n) receives the eigenvectors and evals (host) the
// eigenvalues in the order of Z's columns; converged is false if a leaf solve failed.
// Synchronises the stream.
cudaError_t syevd(double* A, int n, double* Z, void* work, size_t work_bytes, std::vector<double>& evals,
                  bool& converged, cudaStream_t stream);

}  // namespace rpa
