// Dense and streaming kernels of the response operator: the Gamma bra-ket
// GEMMs on FP64 tensor cores (DMMA), the masked preconditioned CG steps, and
// small pointwise passes.
//
// Complex arrays of length npw are treated as real arrays of length 2*npw
// (Re, Im interleaved), exactly as WEST passes them to DGEMM at Gamma
// (glbrak.f90:37-40, apply_alpha_pc_to_m_wfcs.f90:65-72).
#include "wb_common.cuh"
#include <algorithm>

#include "wb_internal.h"

namespace wb {

WB_DEV void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// part[s][j][r] = sum_{k in split s} W[r][k] X[col j][k]        (A^T B, split K)
// CTA tile 32 r x 32 j, four warps interleave k in steps of 4 and are summed
// through shared memory at the end.
// ---------------------------------------------------------------------------
constexpr int TN_T = 32;
constexpr int TN_W = 4;

// PF: k steps between an operand load and the MMAs that use it (1 or 2: two
// pay at 64 projectors, cost at 208; same sums in the same order either way)
template <int PF>
__global__ void __launch_bounds__(32 * TN_W) k_gemm_tn(const double* __restrict__ W, long ldw, int M,
                                                       const double* __restrict__ X, long ldx,
                                                       const int* __restrict__ cols, int ncol_host, const int* dn,
                                                       int K, int kchunk, int ctas, double* __restrict__ part) {
  __shared__ double red[TN_W][TN_T * TN_T];
  const int ncol = dev_count(dn, ncol_host);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lr = lane >> 2, lk = lane & 3;
  const int r0 = blockIdx.x * TN_T, j0 = blockIdx.y * TN_T, split = blockIdx.z;
  if (j0 >= ncol) return;
  if (dn) {  // the split plan of this column count
    const int ns = gemm_tn_splits(M, ncol, K, ctas);
    if (split >= ns) return;
    kchunk = ((K + ns - 1) / ns + 15) / 16 * 16;
  }
  const int kb = split * kchunk, ke = min(K, kb + kchunk);
  const double* arow[4];
  bool aok[4];
  const double* bcol[4];
  bool bok[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = r0 + i * 8 + lr;
    aok[i] = r < M;
    arow[i] = W + (long)(aok[i] ? r : 0) * ldw;
    const int j = j0 + i * 8 + lr;
    bok[i] = j < ncol;
    const int c = bok[i] ? (cols ? cols[j] : j) : 0;
    bcol[i] = X + (long)c * ldx;
  }
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  auto load = [&](int k, double* a, double* b) {
    const int kk = k + lk;
    const bool kok = kk < ke;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      a[i] = (aok[i] && kok) ? __ldg(arow[i] + kk) : 0.0;
      b[i] = (bok[i] && kok) ? __ldg(bcol[i] + kk) : 0.0;
    }
  };
  auto mma_step = [&](const double* a, const double* b) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
  };
  constexpr int KS = 4 * TN_W;  // k advanced per step (the CTA's warps interleave k)
  const int k0 = kb + warp * 4;
  if constexpr (PF == 1) {      // the next step's operands load while this step's MMAs run
    double av[4], bv[4];
    load(k0, av, bv);
    for (int k = k0; k < ke; k += KS) {
      double an[4], bn[4];
      load(k + KS, an, bn);
      mma_step(av, bv);
#pragma unroll
      for (int i = 0; i < 4; ++i) { av[i] = an[i]; bv[i] = bn[i]; }
    }
  } else {                      // two steps ahead; two steps per trip, the buffers swap roles
    double a0[4], b0[4], a1[4], b1[4];
    load(k0, a0, b0);
    load(k0 + KS, a1, b1);
    for (int k = k0; k < ke; k += 2 * KS) {
      mma_step(a0, b0);         // step k, loaded two steps ago
      load(k + 2 * KS, a0, b0);
      if (k + KS >= ke) break;
      mma_step(a1, b1);         // step k + KS
      load(k + 3 * KS, a1, b1);
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int h = 0; h < 2; ++h) red[warp][(a * 8 + lr) * TN_T + b * 8 + 2 * lk + h] = acc[a][b][h];
  __syncthreads();
  for (int e = threadIdx.x; e < TN_T * TN_T; e += 32 * TN_W) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < TN_W; ++w) s += red[w][e];
    const int r = r0 + e / TN_T, j = j0 + e % TN_T;
    if (r < M && j < ncol) part[((long)split * ncol + j) * M + r] = s;
  }
}

size_t gemm_tn_part_doubles(int M, int nsys, int K, int ctas_max) {
  size_t best = 0;
  for (int t = 1; t <= (nsys + TN_T - 1) / TN_T; ++t) {
    const int n = std::min(nsys, t * TN_T);
    for (int c = 1; c <= ctas_max; ++c) best = std::max(best, (size_t)gemm_tn_splits(M, n, K, c) * n * M);
  }
  return best;
}

void gemm_tn(const double* W, long ldw, int M, const double* X, long ldx, const int* cols, int ncol, int K,
             int nsplit, double* part, cudaStream_t s, const int* dn, int ctas, int prefetch) {
  if (ncol <= 0 || M <= 0) return;
  if (dn) nsplit = gemm_tn_splits(M, 1, K, ctas);  // grid for the largest plan
  int kchunk = (K + nsplit - 1) / nsplit;
  kchunk = (kchunk + 15) / 16 * 16;
  dim3 grid((M + TN_T - 1) / TN_T, (ncol + TN_T - 1) / TN_T, nsplit);
  if (prefetch == 2)
    k_gemm_tn<2><<<grid, 32 * TN_W, 0, s>>>(W, ldw, M, X, ldx, cols, ncol, dn, K, kchunk, ctas, part);
  else
    k_gemm_tn<1><<<grid, 32 * TN_W, 0, s>>>(W, ldw, M, X, ldx, cols, ncol, dn, K, kchunk, ctas, part);
}

__global__ void __launch_bounds__(256) k_gamma_reduce(const double* __restrict__ part, int nsplit, int M,
                                                      int ncol_host, const int* dn, const double* __restrict__ W,
                                                      long ldw, const double* __restrict__ X, long ldx,
                                                      const int* __restrict__ cols, const double* __restrict__ D,
                                                      int nkb, double alpha, double* __restrict__ C, int K,
                                                      int ctas) {
  extern __shared__ double S[];
  const int ncol = dev_count(dn, ncol_host);
  const int j = blockIdx.x;
  if (j >= ncol) return;
  if (dn && ctas > 0) nsplit = gemm_tn_splits(M, ncol, K, ctas);
  const int col = cols ? cols[j] : j;
  const double x0 = X[(long)col * ldx];
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    double s = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) s += part[((long)sp * ncol + j) * M + r];
    S[r] = 2.0 * s - W[(long)r * ldw] * x0;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    double c;
    if (r < nkb) {
      c = 0.0;
      for (int q = 0; q < nkb; ++q) c = fma(D[r + (long)q * nkb], S[q], c);
    } else {
      c = alpha * S[r];
    }
    C[(long)j * M + r] = c;
  }
}

void gamma_reduce(const double* part, int nsplit, int M, int ncol, const double* W, long ldw, const double* X,
                  long ldx, const int* cols, const double* D, int nkb, double alpha, double* C, cudaStream_t s,
                  const int* dn, int K, int ctas) {
  if (ncol <= 0 || M <= 0) return;
  k_gamma_reduce<<<ncol, 256, sizeof(double) * M, s>>>(part, nsplit, M, ncol, dn, W, ldw, X, ldx, cols, D, nkb,
                                                        alpha, C, K, ctas);
}

// ---------------------------------------------------------------------------
// Y[col j][k] = beta Y[col j][k] + sum_r W[r][k] C[j][r]
// CTA: 4 warps x 32 rows of k, 32 columns j; inner loop over r in steps of 4.
// With beta != 0 (and 16-byte aligned rows of Y) the CTA's Y tile is copied
// into shared memory by cp.async at the start, so its DRAM latency overlaps
// the MMAs instead of stalling the epilogue.  Row stride 130 doubles: the four
// column groups of a half-warp's epilogue reads fall on disjoint banks.
// ---------------------------------------------------------------------------
constexpr int NN_YLD = 130;

WB_DEV void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

__global__ void __launch_bounds__(128) k_gemm_nn(const double* __restrict__ W, long ldw, int M,
                                                 const double* __restrict__ C, double* __restrict__ Y, long ldy,
                                                 const int* __restrict__ cols, int ncol_host, const int* dn, int K,
                                                 double beta, int stage_y) {
  __shared__ __align__(16) double ysh[32 * NN_YLD];
  const int ncol = dev_count(dn, ncol_host);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lr = lane >> 2, lk = lane & 3;
  const int kbase = blockIdx.x * 128;
  const int k0 = kbase + warp * 32, j0 = blockIdx.y * 32;
  if (j0 >= ncol) return;
  const bool pre = stage_y && beta != 0.0;
  if (pre) {  // Y[col(j0 + jl)][kbase + 2q, +1] -> ysh[jl][2q, +1]  (K is even: a pair never straddles K)
    for (int e = threadIdx.x; e < 32 * 64; e += 128) {
      const int jl = e >> 6, q = e & 63;
      const int j = j0 + jl, k = kbase + 2 * q;
      if (j < ncol && k < K) {
        const int col = cols ? cols[j] : j;
        cp_async16(ysh + jl * NN_YLD + 2 * q, Y + (long)col * ldy + k);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  }
  bool kok[4], jok[4];
  const double* crow[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    kok[i] = (k0 + i * 8 + lr) < K;
    const int j = j0 + i * 8 + lr;
    jok[i] = j < ncol;
    crow[i] = C + (long)(jok[i] ? j : 0) * M;
  }
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll 4
  for (int r = 0; r < M; r += 4) {
    const int rr = r + lk;
    const bool rok = rr < M;
    const double* wr = W + (long)(rok ? rr : 0) * ldw + k0 + lr;
    double av[4], bv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      av[i] = (rok && kok[i]) ? __ldg(wr + i * 8) : 0.0;
      bv[i] = (rok && jok[i]) ? __ldg(crow[i] + rr) : 0.0;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], av[a], bv[b]);
  }
  if (pre) {
    asm volatile("cp.async.wait_all;\n" ::);
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int jl = b * 8 + 2 * lk + h, j = j0 + jl;
      if (j >= ncol) continue;
      const int col = cols ? cols[j] : j;
      double* y = Y + (long)col * ldy;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int kl = warp * 32 + a * 8 + lr, k = kbase + kl;
        if (k >= K) continue;
        const double old = beta == 0.0 ? 0.0 : (pre ? ysh[jl * NN_YLD + kl] : y[k]);
        y[k] = beta * old + acc[a][b][h];
      }
    }
}

void gemm_nn(const double* W, long ldw, int M, const double* C, double* Y, long ldy, const int* cols, int ncol,
             int K, double beta, cudaStream_t s, const int* dn) {
  if (ncol <= 0 || M <= 0) return;
  const int stage_y = (K % 2 == 0) && (ldy % 2 == 0) && ((uintptr_t)Y % 16 == 0);
  dim3 grid((K + 127) / 128, (ncol + 31) / 32);
  k_gemm_nn<<<grid, 128, 0, s>>>(W, ldw, M, C, Y, ldy, cols, ncol, dn, K, beta, stage_y);
}

// ---------------------------------------------------------------------------
// pointwise passes
// ---------------------------------------------------------------------------
// aux(i, p) = dvg(perm(i), p) * sqvc(i)      (apply_operator.f90:49-53)
__global__ void k_permute_scale(const double2* __restrict__ dvg, long ld_in, const int* __restrict__ perm,
                                const double* __restrict__ sqvc, int npw, double2* __restrict__ aux, long ld_out) {
  const int p = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x)
    aux[(long)p * ld_out + i] = cscale(dvg[(long)p * ld_in + perm[i]], sqvc[i]);
}
void permute_scale(const double2* dvg, long ld_in, const int* perm, const double* sqvc, int npw, int m,
                   double2* aux, long ld_out, cudaStream_t s) {
  if (m <= 0) return;
  k_permute_scale<<<dim3((npw + 255) / 256, m), 256, 0, s>>>(dvg, ld_in, perm, sqvc, npw, aux, ld_out);
}

// 1 / max(1, g2kin / eprec_v) per band and G: the preconditioner of
// precondition_m_wfcts.f90:35-51 and linsolve_sternheimer_m_wfcts.f90:150-160,
// applied by multiplication.
__global__ void k_make_iprec(const double* __restrict__ g2kin, const double* __restrict__ eprec, int npw, int nocc,
                             double* __restrict__ iprec) {
  const int v = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x)
    iprec[(long)v * npw + i] = 1.0 / fmax(1.0, g2kin[i] / eprec[v]);
}
void make_iprec(const double* g2kin, const double* eprec, int npw, int nocc, double* iprec, cudaStream_t s) {
  k_make_iprec<<<dim3((npw + 255) / 256, nocc), 256, 0, s>>>(g2kin, eprec, npw, nocc, iprec);
}

// pf = f / max(1, g2kin / eprec)         (precondition_m_wfcts.f90:35-51)
__global__ void k_precondition(const double2* __restrict__ f, double2* __restrict__ pf,
                               const double* __restrict__ iprec, int nocc, int npw, long ld) {
  const int j = blockIdx.y;
  const double* ip = iprec + (long)(j % nocc) * npw;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x) {
    const double2 v = f[(long)j * ld + i];
    pf[(long)j * ld + i] = make_double2(v.x * ip[i], v.y * ip[i]);
  }
}
void precondition(const double2* f, double2* pf, const double* iprec, int nocc, int npw, int ncol, long ld,
                  cudaStream_t s) {
  if (ncol <= 0) return;
  k_precondition<<<dim3((npw + 255) / 256, ncol), 256, 0, s>>>(f, pf, iprec, nocc, npw, ld);
}

__global__ void k_sub_into(const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ out,
                           int npw, long ld) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x)
    out[(long)j * ld + i] = csub(a[(long)j * ld + i], b[(long)j * ld + i]);
}
void sub_into(const double2* a, const double2* b, double2* out, int npw, int ncol, long ld, cudaStream_t s) {
  if (ncol <= 0) return;
  k_sub_into<<<dim3((npw + 255) / 256, ncol), 256, 0, s>>>(a, b, out, npw, ld);
}

// T = g2kin P (Im at G=0 zeroed) - e P     (k_psi.f90:51-77 then :65-74 of
// apply_sternheimerop_to_m_wfcs.f90)
__global__ void k_kinetic_hpsi(const double2* __restrict__ P, double2* __restrict__ T,
                               const double* __restrict__ g2kin, const double* __restrict__ ecol,
                               const int* __restrict__ cols, const int* dn, int npw, long ld) {
  if ((int)blockIdx.y >= dev_count(dn, gridDim.y)) return;
  const int c = cols ? cols[blockIdx.y] : blockIdx.y;
  const double e = ecol[c];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x) {
    const double2 p = P[(long)c * ld + i];
    double2 h = cscale(p, g2kin[i]);
    if (i == 0) h.y = 0.0;
    T[(long)c * ld + i] = make_double2(fma(-e, p.x, h.x), fma(-e, p.y, h.y));
  }
}
void kinetic_hpsi(const double2* P, double2* T, const double* g2kin, const double* ecol, const int* cols, int ncol,
                  int npw, long ld, cudaStream_t s, const int* dn) {
  if (ncol <= 0) return;
  k_kinetic_hpsi<<<dim3((npw + 255) / 256, ncol), 256, 0, s>>>(P, T, g2kin, ecol, cols, dn, npw, ld);
}

// eprec_v = 1.35 sum_G |psi_v(G)|^2 g2kin(G)       (set_eprec.f90:40-53)
__global__ void __launch_bounds__(256) k_set_eprec(const double2* __restrict__ evc, const double* __restrict__ g2kin,
                                                   int npw, double* __restrict__ eprec) {
  __shared__ double red[8];
  const int v = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < npw; i += 256) {
    const double2 c = evc[(long)v * npw + i];
    s += (c.x * c.x + c.y * c.y) * g2kin[i];
  }
  s = block_sum<256>(s, red);
  if (threadIdx.x == 0) eprec[v] = 1.35 * s;
}
void set_eprec(const double2* evc, const double* g2kin, int npw, int nocc, double* eprec, cudaStream_t s) {
  k_set_eprec<<<nocc, 256, 0, s>>>(evc, g2kin, npw, eprec);
}

__global__ void k_fill_columns(const double* __restrict__ pb, int nocc, int nsys, double* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nsys; j += gridDim.x * blockDim.x) out[j] = pb[j % nocc];
}
void fill_columns(const double* per_band, int nocc, int nsys, double* out, cudaStream_t s) {
  k_fill_columns<<<(nsys + 255) / 256, 256, 0, s>>>(per_band, nocc, nsys, out);
}

__global__ void k_frac_coefficients(const double* __restrict__ C, int nocc, int nsys, int nfull,
                                    const double* __restrict__ occ, const double* __restrict__ et,
                                    double* __restrict__ fc) {
  const int nfrac = nocc - nfull;
  const long n = (long)nsys * nfrac;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const int j = (int)(e / nfrac), f = (int)(e % nfrac);
    const int i = j % nocc, r = nfull + f;
    double v = 0.0;
    const double docc = occ[i] - occ[r];
    if (r > i && fabs(docc) >= 1e-3) v = C[(long)j * nocc + r] * docc / occ[i] / (et[i] - et[r]);
    fc[e] = v;
  }
}
void frac_coefficients(const double* C, int nocc, int nsys, int nfull, const double* occ, const double* et,
                       double* fc, cudaStream_t s) {
  const long n = (long)nsys * (nocc - nfull);
  if (n <= 0) return;
  k_frac_coefficients<<<(int)std::min<long>((n + 255) / 256, 4096), 256, 0, s>>>(C, nocc, nsys, nfull, occ, et, fc);
}

// ---------------------------------------------------------------------------
// masked PCG (linsolve_sternheimer_m_wfcts.f90:146-330), one CTA per system
// ---------------------------------------------------------------------------
__global__ void k_cg_reset(unsigned char* conv, int nsys) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nsys; j += gridDim.x * blockDim.x) conv[j] = 0;
}
void cg_reset(unsigned char* conv, int nsys, cudaStream_t s) {
  k_cg_reset<<<(nsys + 255) / 256, 256, 0, s>>>(conv, nsys);
}

// h = g / max(1, g2kin/eprec); rho = <h|g>_Gamma; converged if rho < thr_j
// (thr_j = max(tr2 * rel_j, floor) when rel != nullptr, else tr2); otherwise
// P = -h + (rho / rho_prev) P  (P = -h at the first iteration).  C is the
// vector type (double2, or float2 in the mixed form); scalars are FP64.
template <class C>
__global__ void __launch_bounds__(256) k_cg_prec_rho(const int* __restrict__ act, const int* dn, const C* __restrict__ g,
                                                     C* __restrict__ P, const double* __restrict__ iprec, int nocc,
                                                     double* rho_prev, unsigned char* conv, int iter_host,
                                                     const int* iter_dev, double tr2, const double* __restrict__ rel,
                                                     double floor, int npw, long ld) {
  using T = real_t<C>;
  __shared__ double red[16];
  const int n = dev_count(dn, gridDim.x);
  const int iter = iter_dev ? *iter_dev : iter_host;
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const int j = act[b];
    const C* gj = g + (long)j * ld;
    C* pj = P + (long)j * ld;
    const double* ip = iprec + (long)(j % nocc) * npw;
    double t = 0.0, t0 = 0.0;
    for (int i = threadIdx.x; i < npw; i += 256) {
      const double w = ip[i];
      const C gv = gj[i];
      const double hx = (double)gv.x * w, hy = (double)gv.y * w;
      t = fma(hx, (double)gv.x, fma(hy, (double)gv.y, t));
      if (i == 0) t0 = hx * (double)gv.x;
    }
    const double2 s = block_sum2<256>(t, t0, red);
    const double rho = 2.0 * s.x - s.y;
    const double thr = rel ? fmax(tr2 * rel[j], floor) : tr2;
    if (rho < thr) {  // block-uniform
      if (threadIdx.x == 0) conv[j] = 1;
      continue;
    }
    const double beta = (iter == 1) ? 0.0 : rho / rho_prev[j];
    __syncthreads();
    if (threadIdx.x == 0) rho_prev[j] = rho;
    for (int i = threadIdx.x; i < npw; i += 256) {
      const double w = ip[i];
      const C gv = gj[i];
      const double hx = (double)gv.x * w, hy = (double)gv.y * w;
      if (iter == 1) {
        pj[i] = mkc<C>(T(-hx), T(-hy));
      } else {
        const C pv = pj[i];
        pj[i] = mkc<C>(T(fma(beta, (double)pv.x, -hx)), T(fma(beta, (double)pv.y, -hy)));
      }
    }
  }
}

// Grid of a per-system launch: one CTA per system; with a device count nmax
// bounds it (the CTAs beyond the count return at once).
static int sys_grid(int nmax, const int*) { return nmax; }

void cg_prec_rho(const int* act, int nact, const double2* g, double2* P, const double* iprec, int nocc,
                 double* rho_prev, unsigned char* conv, int iter, double tr2, int npw, long ld, cudaStream_t s,
                 const int* dn, const int* iter_dev) {
  if (nact <= 0) return;
  k_cg_prec_rho<double2><<<sys_grid(nact, dn), 256, 0, s>>>(act, dn, g, P, iprec, nocc, rho_prev, conv, iter, iter_dev,
                                                           tr2, nullptr, 0.0, npw, ld);
}
void cg_prec_rho32(const int* act, int nact, const float2* g, float2* P, const double* iprec, int nocc,
                   double* rho_prev, unsigned char* conv, int iter, double eta, const double* rel, double floor,
                   int npw, long ld, cudaStream_t s, const int* dn, const int* iter_dev) {
  if (nact <= 0) return;
  k_cg_prec_rho<float2><<<sys_grid(nact, dn), 256, 0, s>>>(act, dn, g, P, iprec, nocc, rho_prev, conv, iter, iter_dev,
                                                          eta, rel, floor, npw, ld);
}

// Active list in increasing system order (map_lbnd2ibnd, :356-382) and the
// Gamma FFT pairs (act[2k], act[2k+1]).
__global__ void __launch_bounds__(1024) k_cg_compact(const unsigned char* __restrict__ conv, int nsys_host,
                                                     const int* nsys_dev, int* __restrict__ act,
                                                     int2* __restrict__ items, int* __restrict__ nact_out) {
  const int nsys = dev_count(nsys_dev, nsys_host);
  __shared__ int wsum[32];
  __shared__ int base;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < nsys; c0 += 1024) {
    const int i = c0 + tid;
    const bool f = (i < nsys) && !conv[i];
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    const int pre = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    if (w == 0) {
      int v = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      wsum[lane] = v;  // inclusive
    }
    __syncthreads();
    const int off = base + (w > 0 ? wsum[w - 1] : 0) + pre;
    if (f) act[off] = i;
    __syncthreads();
    if (tid == 0) base += wsum[31];
    __syncthreads();
  }
  const int n = base;
  for (int k = tid; k < (n + 1) / 2; k += 1024)
    items[k] = make_int2(act[2 * k], (2 * k + 1 < n) ? act[2 * k + 1] : -1);
  if (tid == 0) *nact_out = n;
}
void cg_compact(const unsigned char* conv, int nsys, int* act, int2* items, int* nact_dev, int* nact_host,
                cudaStream_t s, const int* nsys_dev) {
  k_cg_compact<<<1, 1024, 0, s>>>(conv, nsys, nsys_dev, act, items, nact_dev);
  if (nact_host) cudaMemcpyAsync(nact_host, nact_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
}


// One PCG step after the operator, in one kernel: the update of iteration
// `iter` (a = <P|g>, c = <P|T> with the Gamma dot, x -= a/c P, g -= a/c T;
// linsolve_sternheimer_m_wfcts.f90:253-329) and, unless iter == maxiter,
// iteration iter + 1's preconditioning, rho, test and direction (as
// k_cg_prec_rho: h = M g, rho = <h|g>, P = -h + rho/rho_prev P).
// One CTA per system; the new g is preconditioned and its rho summed in the
// update's own pass, and the direction pass re-reads g (just written) and P
// (read twice already) from L2, so the vectors make fewer trips to DRAM than
// with two kernels with the active-list compaction between them.
template <class C, int NT>
__global__ void __launch_bounds__(NT) k_cg_step(const int* __restrict__ act, const int* dn, int nhost,
                                                C* __restrict__ x, C* __restrict__ g, C* __restrict__ P,
                                                const C* __restrict__ T, const double* __restrict__ iprec, int nocc,
                                                double* rho_prev, unsigned char* conv, int iter_host,
                                                const int* iter_dev, int maxiter, double tr2,
                                                const double* __restrict__ rel, double floor, int npw, long ld) {
  using R = real_t<C>;
  __shared__ double red[NT / 16];
  const int n = dev_count(dn, nhost);
  const int iter = iter_dev ? *iter_dev : iter_host;
  const bool prec = iter + 1 <= maxiter;  // the reference leaves its loop before this preconditioning otherwise
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const int j = act[b];
    const C* tj = T + (long)j * ld;
    C* pj = P + (long)j * ld;
    C* gj = g + (long)j * ld;
    C* xj = x + (long)j * ld;
    const double* ip = iprec + (long)(j % nocc) * npw;
    double a = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < npw; i += NT) {
      const C p = pj[i], gv = gj[i], tv = tj[i];
      double da = fma((double)p.x, (double)gv.x, (double)p.y * (double)gv.y);
      double dc = fma((double)p.x, (double)tv.x, (double)p.y * (double)tv.y);
      if (i == 0) { da -= 0.5 * (double)p.x * (double)gv.x; dc -= 0.5 * (double)p.x * (double)tv.x; }
      a += da;
      c += dc;
    }
    const double2 s = block_sum2<NT>(a, c, red);
    const R r = R((2.0 * s.x) / (2.0 * s.y));
    double tt = 0.0, t0 = 0.0;
    for (int i = threadIdx.x; i < npw; i += NT) {
      const C p = pj[i], tv = tj[i];
      const C xv = xj[i], gv = gj[i];
      xj[i] = mkc<C>(fma(-r, p.x, xv.x), fma(-r, p.y, xv.y));
      const C gn = mkc<C>(fma(-r, tv.x, gv.x), fma(-r, tv.y, gv.y));
      gj[i] = gn;
      if (prec) {
        const double w = ip[i];
        const double hx = (double)gn.x * w, hy = (double)gn.y * w;
        tt = fma(hx, (double)gn.x, fma(hy, (double)gn.y, tt));
        if (i == 0) t0 = hx * (double)gn.x;
      }
    }
    if (!prec) continue;
    const double2 s2 = block_sum2<NT>(tt, t0, red);
    const double rho = 2.0 * s2.x - s2.y;
    const double thr = rel ? fmax(tr2 * rel[j], floor) : tr2;
    if (rho < thr) {  // block-uniform
      if (threadIdx.x == 0) conv[j] = 1;
      continue;
    }
    const double beta = rho / rho_prev[j];  // iteration iter + 1 >= 2
    __syncthreads();
    if (threadIdx.x == 0) rho_prev[j] = rho;
    for (int i = threadIdx.x; i < npw; i += NT) {
      const double w = ip[i];
      const C gv = gj[i], pv = pj[i];
      const double hx = (double)gv.x * w, hy = (double)gv.y * w;
      pj[i] = mkc<C>(R(fma(beta, (double)pv.x, -hx)), R(fma(beta, (double)pv.y, -hy)));
    }
  }
}

// Launch shape of k_cg_step: a persistent grid of a few large CTAs per SM, each
// looping over systems, so the systems in flight (148 x 540 KB of FP64 vectors,
// 296 x 270 KB in FP32) keep their vectors in L2 between the kernel's three
// passes.  With one 256-thread CTA per system (1,200 systems in flight at c2)
// every pass re-read its vectors from DRAM: 1.22 MB read per FP64 system
// instead of 0.54 MB (ncu); the FP64 step went from 20.7 to 17.2 ms, the FP32
// one from 17.2 to 14.8 ms per c2 call.
static int sm_count() {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess || nsm <= 0)
      nsm = 148;
  }
  return nsm;
}
void cg_step(const int* act, int nact, double2* x, double2* g, double2* P, const double2* T, const double* iprec,
             int nocc, double* rho_prev, unsigned char* conv, int iter, int maxiter, double tr2, int npw, long ld,
             cudaStream_t s, const int* dn, const int* iter_dev) {
  if (nact <= 0) return;
  k_cg_step<double2, 1024><<<std::min(nact, sm_count()), 1024, 0, s>>>(
      act, dn, nact, x, g, P, T, iprec, nocc, rho_prev, conv, iter, iter_dev, maxiter, tr2, nullptr, 0.0, npw, ld);
}
void cg_step32(const int* act, int nact, float2* x, float2* g, float2* P, const float2* T, const double* iprec,
               int nocc, double* rho_prev, unsigned char* conv, int iter, int maxiter, double eta, const double* rel,
               double floor, int npw, long ld, cudaStream_t s, const int* dn, const int* iter_dev) {
  if (nact <= 0) return;
  k_cg_step<float2, 512><<<std::min(nact, 2 * sm_count()), 512, 0, s>>>(
      act, dn, nact, x, g, P, T, iprec, nocc, rho_prev, conv, iter, iter_dev, maxiter, eta, rel, floor, npw, ld);
}

// ---------------------------------------------------------------------------
// FP64 iterative refinement around the FP32 PCG (mixed form)
// ---------------------------------------------------------------------------
// R = B - T (FP64); rho = <M^-1 R|R>_Gamma; converged if rho < tr2 (the test of
// linsolve_sternheimer_m_wfcts.f90:215-216 on the true FP64 residual).
// Otherwise the FP32 correction solve starts from d = 0 with g = -R.
__global__ void __launch_bounds__(256) k_refine_residual(const int* __restrict__ act, const double2* __restrict__ B,
                                                         const double2* __restrict__ T,
                                                         const double* __restrict__ iprec, int nocc, double tr2,
                                                         unsigned char* conv, double* rho0, float2* __restrict__ g32,
                                                         float2* __restrict__ d32, int npw, long ld) {
  __shared__ double red[16];
  const int j = act[blockIdx.x];
  const double2* bj = B + (long)j * ld;
  const double2* tj = T + (long)j * ld;
  const double* ip = iprec + (long)(j % nocc) * npw;
  double t = 0.0, t0 = 0.0;
  for (int i = threadIdx.x; i < npw; i += 256) {
    const double2 b = bj[i], a = tj[i];
    const double rx = b.x - a.x, ry = b.y - a.y;
    const double w = ip[i];
    t = fma(rx * w, rx, fma(ry * w, ry, t));
    if (i == 0) t0 = rx * w * rx;
  }
  const double2 s = block_sum2<256>(t, t0, red);
  const double rho = 2.0 * s.x - s.y;
  const bool c = rho < tr2;
  if (threadIdx.x == 0) { conv[j] = c ? 1 : 0; rho0[j] = rho; }
  if (c) return;
  float2* gj = g32 + (long)j * ld;
  float2* dj = d32 + (long)j * ld;
  for (int i = threadIdx.x; i < npw; i += 256) {
    const double2 b = bj[i], a = tj[i];
    gj[i] = make_float2((float)(a.x - b.x), (float)(a.y - b.y));
    dj[i] = make_float2(0.f, 0.f);
  }
}
void refine_residual(const int* act, int nact, const double2* B, const double2* T, const double* iprec, int nocc,
                     double tr2, unsigned char* conv, double* rho0, float2* g32, float2* d32, int npw, long ld,
                     cudaStream_t s) {
  if (nact <= 0) return;
  k_refine_residual<<<nact, 256, 0, s>>>(act, B, T, iprec, nocc, tr2, conv, rho0, g32, d32, npw, ld);
}

// x += d for the listed columns
__global__ void k_refine_accumulate(const int* __restrict__ act, double2* __restrict__ X,
                                    const float2* __restrict__ d32, int npw, long ld) {
  const int j = act[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x) {
    const float2 d = d32[(long)j * ld + i];
    double2 x = X[(long)j * ld + i];
    X[(long)j * ld + i] = make_double2(x.x + (double)d.x, x.y + (double)d.y);
  }
}
void refine_accumulate(const int* act, int nact, double2* X, const float2* d32, int npw, long ld, cudaStream_t s) {
  if (nact <= 0) return;
  k_refine_accumulate<<<dim3((npw + 255) / 256, nact), 256, 0, s>>>(act, X, d32, npw, ld);
}

// FP32 T = g2kin P (Im at G=0 zeroed) - e P for the kinetic-only operator
__global__ void k_kinetic_hpsi32(const float2* __restrict__ P, float2* __restrict__ T, const float* __restrict__ g2kin,
                                 const float* __restrict__ ecol, const int* __restrict__ cols, const int* dn, int npw,
                                 long ld) {
  if ((int)blockIdx.y >= dev_count(dn, gridDim.y)) return;
  const int c = cols ? cols[blockIdx.y] : blockIdx.y;
  const float e = ecol[c];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x) {
    const float2 p = P[(long)c * ld + i];
    float2 h = make_float2(p.x * g2kin[i], p.y * g2kin[i]);
    if (i == 0) h.y = 0.f;
    T[(long)c * ld + i] = make_float2(fmaf(-e, p.x, h.x), fmaf(-e, p.y, h.y));
  }
}
void kinetic_hpsi32(const float2* P, float2* T, const float* g2kin, const float* ecol, const int* cols, int ncol,
                    int npw, long ld, cudaStream_t s, const int* dn) {
  if (ncol <= 0) return;
  k_kinetic_hpsi32<<<dim3((npw + 255) / 256, ncol), 256, 0, s>>>(P, T, g2kin, ecol, cols, dn, npw, ld);
}

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (float)a[i];
}
void to_float(const double* a, float* b, long n, cudaStream_t s) {
  if (n <= 0) return;
  k_to_float<<<(int)std::min<long>((n + 255) / 256, 4096), 256, 0, s>>>(a, b, n);
}

// ---------------------------------------------------------------------------
// FP32 bra-ket GEMMs of the inner solve (SIMT FFMA, shared-memory tiles)
// ---------------------------------------------------------------------------
// part[s][j][r] = sum_{k in split s} W[r][k] X[col j][k]; tile 64 r x 64 j, k step 16
__global__ void __launch_bounds__(256) k_gemm_tn_f32(const float* __restrict__ W, long ldw, int M,
                                                     const float* __restrict__ X, long ldx,
                                                     const int* __restrict__ cols, int ncol_host, const int* dn,
                                                     int K, int kchunk, float* __restrict__ part) {
  __shared__ float Ws[16][64 + 4];
  __shared__ float Xs[16][64 + 4];
  const int ncol = dev_count(dn, ncol_host);
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int r0 = blockIdx.x * 64, j0 = blockIdx.y * 64, split = blockIdx.z;
  if (j0 >= ncol) return;
  const int kb = split * kchunk, ke = min(K, kb + kchunk);
  float acc[4][4] = {};
  // loader: 64 rows x 8 float2 per operand, two per thread
  const int lrow = tid / 8, lk = (tid % 8) * 2;
  const float* wrow[2];
  const float* xrow[2];
  bool wok[2], xok[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = r0 + lrow + 32 * h;
    wok[h] = r < M;
    wrow[h] = W + (long)(wok[h] ? r : 0) * ldw;
    const int j = j0 + lrow + 32 * h;
    xok[h] = j < ncol;
    const int cj = xok[h] ? (cols ? cols[j] : j) : 0;
    xrow[h] = X + (long)cj * ldx;
  }
  for (int k0 = kb; k0 < ke; k0 += 16) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = k0 + lk;
      float2 wv = make_float2(0.f, 0.f), xv = make_float2(0.f, 0.f);
      if (wok[h] && k < ke) wv = *reinterpret_cast<const float2*>(wrow[h] + k);
      if (xok[h] && k < ke) xv = *reinterpret_cast<const float2*>(xrow[h] + k);
      Ws[lk][lrow + 32 * h] = wv.x; Ws[lk + 1][lrow + 32 * h] = wv.y;
      Xs[lk][lrow + 32 * h] = xv.x; Xs[lk + 1][lrow + 32 * h] = xv.y;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) { a[i] = Ws[kk][ty * 4 + i]; b[i] = Xs[kk][tx * 4 + i]; }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = fmaf(a[i], b[q], acc[i][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + ty * 4 + i, j = j0 + tx * 4 + q;
      if (r < M && j < ncol) part[((long)split * ncol + j) * M + r] = acc[i][q];
    }
}

int gemm_tn_splits32(int M, int ncol, int K) {
  const int tiles = ((M + 63) / 64) * ((ncol + 63) / 64);
  int ns = (2 * 148 * 2 + tiles - 1) / tiles;
  const int maxs = (K + 511) / 512;
  if (ns > maxs) ns = maxs;
  if (ns < 1) ns = 1;
  return ns;
}

void gemm_tn32(const float* W, long ldw, int M, const float* X, long ldx, const int* cols, int ncol, int K, int nsplit,
               float* part, cudaStream_t s, const int* dn) {
  if (ncol <= 0 || M <= 0) return;
  int kchunk = (K + nsplit - 1) / nsplit;
  kchunk = (kchunk + 15) / 16 * 16;
  dim3 grid((M + 63) / 64, (ncol + 63) / 64, nsplit);
  k_gemm_tn_f32<<<grid, 256, 0, s>>>(W, ldw, M, X, ldx, cols, ncol, dn, K, kchunk, part);
}

__global__ void __launch_bounds__(256) k_gamma_reduce32(const float* __restrict__ part, int nsplit, int M,
                                                        int ncol_host, const int* dn,
                                                        const float* __restrict__ W, long ldw,
                                                        const float* __restrict__ X, long ldx,
                                                        const int* __restrict__ cols, const float* __restrict__ D,
                                                        int nkb, float alpha, float* __restrict__ C, int K,
                                                        int umma_ctas) {
  extern __shared__ float Sf[];
  const int ncol = dev_count(dn, ncol_host);
  const int j = blockIdx.x;
  if (j >= ncol) return;
  if (dn && umma_ctas > 0) {  // the split plan of the tcgen05 bra-ket for this column count
    int per;
    umma_braket_plan(ncol, K, &nsplit, &per, umma_ctas);
  }
  const int col = cols ? cols[j] : j;
  const float x0 = X[(long)col * ldx];
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    float sum = 0.f;
    for (int sp = 0; sp < nsplit; ++sp) sum += part[((long)sp * ncol + j) * M + r];
    Sf[r] = 2.f * sum - W[(long)r * ldw] * x0;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    float c;
    if (r < nkb) {
      c = 0.f;
      for (int q = 0; q < nkb; ++q) c = fmaf(D[r + (long)q * nkb], Sf[q], c);
    } else {
      c = alpha * Sf[r];
    }
    C[(long)j * M + r] = c;
  }
}
void gamma_reduce32(const float* part, int nsplit, int M, int ncol, const float* W, long ldw, const float* X, long ldx,
                    const int* cols, const float* D, int nkb, float alpha, float* C, cudaStream_t s, const int* dn,
                    int K, int umma_ctas) {
  if (ncol <= 0 || M <= 0) return;
  k_gamma_reduce32<<<ncol, 256, sizeof(float) * M, s>>>(part, nsplit, M, ncol, dn, W, ldw, X, ldx, cols, D, nkb, alpha,
                                                        C, K, umma_ctas);
}

// Y[col j][k] += sum_r W[r][k] C[j][r]; tile 128 k x 32 j, r step 16
__global__ void __launch_bounds__(256) k_gemm_nn_f32(const float* __restrict__ W, long ldw, int M,
                                                     const float* __restrict__ C, float* __restrict__ Y, long ldy,
                                                     const int* __restrict__ cols, int ncol_host, const int* dn,
                                                     int K) {
  __shared__ float Ws[16][128 + 4];
  __shared__ float Cs[16][32 + 1];
  const int ncol = dev_count(dn, ncol_host);
  const int tid = threadIdx.x, tx = tid % 32, ty = tid / 32;
  const int k0 = blockIdx.x * 128, j0 = blockIdx.y * 32;
  if (j0 >= ncol) return;
  float acc[4][4] = {};  // [k i][j q]: k = k0 + tx*4 + i, j = j0 + ty*4 + q
  for (int rb = 0; rb < M; rb += 16) {
    for (int e = tid; e < 16 * 64; e += 256) {           // W tile: 16 r x 64 float2
      const int rr = e / 64, kk = (e % 64) * 2;
      const int r = rb + rr, k = k0 + kk;
      float2 v = make_float2(0.f, 0.f);
      if (r < M && k < K) v = *reinterpret_cast<const float2*>(W + (long)r * ldw + k);
      Ws[rr][kk] = v.x; Ws[rr][kk + 1] = v.y;
    }
    for (int e = tid; e < 16 * 32; e += 256) {           // C tile: 16 r x 32 j
      const int rr = e % 16, jj = e / 16;
      const int r = rb + rr, j = j0 + jj;
      Cs[rr][jj] = (r < M && j < ncol) ? C[(long)j * M + r] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < 16; ++rr) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) { a[i] = Ws[rr][tx * 4 + i]; b[i] = Cs[rr][ty * 4 + i]; }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = fmaf(a[i], b[q], acc[i][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int j = j0 + ty * 4 + q;
    if (j >= ncol) continue;
    const int col = cols ? cols[j] : j;
    float* y = Y + (long)col * ldy;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = k0 + tx * 4 + i;
      if (k < K) y[k] += acc[i][q];
    }
  }
}
void gemm_nn32_acc(const float* W, long ldw, int M, const float* C, float* Y, long ldy, const int* cols, int ncol, int K,
                   cudaStream_t s, const int* dn) {
  if (ncol <= 0 || M <= 0) return;
  dim3 grid((K + 127) / 128, (ncol + 31) / 32);
  k_gemm_nn_f32<<<grid, 256, 0, s>>>(W, ldw, M, C, Y, ldy, cols, ncol, dn, K);
}

// ---------------------------------------------------------------------------
// device-side loop control of the graph-captured PCG loops
// ---------------------------------------------------------------------------
// st[0] systems of the batch, st[1] iteration of the next pass, st[2] last
// iteration run, st[3] inner iterations run over all refinements (mixed form);
// st[4..5] active system-iterations and st[6..7] FFT boxes (64-bit counters).
__global__ void k_loop_init(int* st, int nsys, int reset_totals) {
  st[0] = nsys;
  st[1] = 1;
  st[2] = 0;
  if (reset_totals) {
    st[3] = 0;
    *reinterpret_cast<long long*>(st + 4) = 0;
    *reinterpret_cast<long long*>(st + 6) = 0;
  }
}
void loop_init(int* st, int nsys, bool reset_totals, cudaStream_t s) {
  k_loop_init<<<1, 1, 0, s>>>(st, nsys, reset_totals ? 1 : 0);
}

// End of one PCG pass (operator, update of iteration st[1] and the
// preconditioning of iteration st[1] + 1, active list): linsolve's loop over
// iter = 1..n_dfpt_maxiter, left when no system is active
// (linsolve_sternheimer_m_wfcts.f90:146,222); every FP32 correction solve of
// the mixed form is bounded the same way.  Sets the WHILE condition of the
// graph; for the FP64 loop (inner = 0) it leaves the reference's iteration
// count in st[2]: the passes that did work, plus the one whose test found no
// system left.
__global__ void k_loop_ctl(cudaGraphConditionalHandle h, const int* nact, int* st, int maxiter, int inner) {
  const int n = *nact, it = st[1];
  const bool more = n > 0 && it < maxiter;
  if (!inner && !more) st[2] = st[3] + (n == 0 ? 1 : 0);
  if (more) st[1] = it + 1;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}
void loop_ctl(cudaGraphConditionalHandle h, const int* nact, int* st, int maxiter, bool inner, cudaStream_t s) {
  k_loop_ctl<<<1, 1, 0, s>>>(h, nact, st, maxiter, inner ? 1 : 0);
}

// Start of a pass: counts the pass's work (st[3] passes with active systems,
// their active-system and FFT-item sums) and sets the SWITCH value: the
// smallest bucket k with min_items << k >= the active band-pair items (last
// bucket: the workspace capacity).
__global__ void k_loop_bucket(cudaGraphConditionalHandle h, const int* nact, int* st, int min_items, int nbuckets) {
  const int n = *nact;
  if (n > 0) {
    *reinterpret_cast<long long*>(st + 4) += n;
    *reinterpret_cast<long long*>(st + 6) += 2 * ((n + 1) / 2);
    st[3] += 1;
  }
  const int items = (n + 1) / 2;
  int k = 0;
  while (k < nbuckets - 1 && (min_items << k) < items) ++k;
  cudaGraphSetConditional(h, (unsigned)k);
}
void loop_bucket(cudaGraphConditionalHandle h, const int* nact, int* st, int min_items, int nbuckets, cudaStream_t s) {
  k_loop_bucket<<<1, 1, 0, s>>>(h, nact, st, min_items, nbuckets);
}

__global__ void k_count_unconverged(const unsigned char* __restrict__ conv, int nocc, int mb, int* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= mb) return;
  int n = 0;
  for (int v = 0; v < nocc; ++v) n += conv[(long)p * nocc + v] ? 0 : 1;
  out[p] = n;
}
void count_unconverged(const unsigned char* conv, int nocc, int mb, int* out, cudaStream_t s) {
  if (mb <= 0) return;
  k_count_unconverged<<<(mb + 127) / 128, 128, 0, s>>>(conv, nocc, mb, out);
}

}  // namespace wb
