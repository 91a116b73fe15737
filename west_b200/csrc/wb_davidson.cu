// PDEP Davidson eigensolver on one GPU (Wstat/davidson_diago.f90:31-437).
//
// The host loop follows davidson_diago_gamma step by step (the reference's
// driver is compiled Fortran; this is its C++ counterpart above the same
// device kernels).  The basis dvg/dng lives on the device in WEST's |G| order
// ([column][npw] complex, G = 0 first) and goes through apply_operator by
// column ranges, like the reference's mstart/mloc slices on one image.
// Device work: Gamma bra-kets for hr (build_hr_real) on the DMMA split-K
// GEMM, basis combinations (update_with_vr / refresh_with_vr) on the DMMA
// accumulation GEMM, modified Gram-Schmidt (do_mgs) as per-vector reductions
// and rank-1 updates, and Jacobi eigensolvers (diagox): cyclic in one CTA for
// bases up to 112, parallel two-sided block Jacobi over many CTAs above.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iterator>
#include <vector>

#include "wb_common.cuh"
#include "wb_ctx.h"

using namespace wb;

namespace {

// hr(col0 + j, rows) <- 2 sum_s part[s][j][r] - W_r(G0) X_j(G0)  (glbrak.f90:39-40)
__global__ void k_braket_to_hr(const double* __restrict__ part, int nsplit, int M, int ncol,
                               const double* __restrict__ W, long ldw, const double* __restrict__ X, long ldx,
                               double* __restrict__ hr, long ldh, int col0) {
  const int j = blockIdx.x;
  const double x0 = X[(long)j * ldx];
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    double s = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) s += part[((long)sp * ncol + j) * M + r];
    hr[(long)(col0 + j) * ldh + r] = 2.0 * s - W[(long)r * ldw] * x0;
  }
}

// Coefficients of update_with_vr_distr_real (wstat_tools.f90:1039-1072):
// C2[j][r] = vr(r, col0 + j), C1[j][r] = -ew(col0 + j) vr(r, col0 + j), r < nrow.
__global__ void k_vr_coef(const double* __restrict__ vr, long ldv, int nrow, int col0, int ncol,
                          const double* __restrict__ ew, double* __restrict__ c1, double* __restrict__ c2) {
  const int j = blockIdx.x;
  const double e = ew ? -ew[col0 + j] : 0.0;
  for (int r = threadIdx.x; r < nrow; r += blockDim.x) {
    const double v = vr[(long)(col0 + j) * ldv + r];
    c2[(long)j * nrow + r] = v;
    if (c1) c1[(long)j * nrow + r] = e * v;
  }
}

// Gamma self-product and normalisation of one column (do_mgs :1003-1031).
__global__ void __launch_bounds__(256) k_mgs_normalize(double2* __restrict__ a, int npw) {
  __shared__ double red[8];
  double s = 0.0;
  for (int i = threadIdx.x; i < npw; i += 256) {
    const double2 v = a[i];
    s = fma(v.x, v.x, fma(v.y, v.y, s));
  }
  s = block_sum<256>(s, red);
  const double anorm = 2.0 * s - a[0].x * a[0].x;
  const double sc = 1.0 / sqrt(anorm);
  for (int i = threadIdx.x; i < npw; i += 256) a[i] = cscale(a[i], sc);
}

// zbraket(j) = <vec|a_j>_Gamma for j in [j0, j0 + gridDim.x)  (do_mgs :1056-1085)
__global__ void __launch_bounds__(256) k_mgs_dots(const double2* __restrict__ a, long ld, int npw, int k, int j0,
                                                  double* __restrict__ dots) {
  __shared__ double red[8];
  const double2* vk = a + (long)k * ld;
  const double2* vj = a + (long)(j0 + blockIdx.x) * ld;
  double s = 0.0;
  for (int i = threadIdx.x; i < npw; i += 256) {
    const double2 p = vk[i], q = vj[i];
    s = fma(p.x, q.x, fma(p.y, q.y, s));
  }
  s = block_sum<256>(s, red);
  if (threadIdx.x == 0) dots[blockIdx.x] = 2.0 * s - vk[0].x * vj[0].x;
}

// a_j <- a_j - vec zbraket(j)   (ZGERU, do_mgs :1094)
__global__ void k_mgs_axpy(double2* __restrict__ a, long ld, int npw, int k, int j0, const double* __restrict__ dots) {
  const int jj = blockIdx.y;
  const double d = dots[jj];
  const double2* vk = a + (long)k * ld;
  double2* vj = a + (long)(j0 + jj) * ld;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npw; i += gridDim.x * blockDim.x) {
    const double2 p = vk[i];
    const double2 q = vj[i];
    vj[i] = make_double2(fma(-d, p.x, q.x), fma(-d, p.y, q.y));
  }
}

// Cyclic two-sided Jacobi on the upper triangle of hr[:n, :n] (what DSYEV 'U'
// reads in matdiago_dsy, Tools/linear_algebra_kernel.f90:84), round-robin
// ordering so each round rotates n/2 disjoint (p, q) planes in parallel,
// applying J^T A J block by block in one pass (two barriers per round).
// One CTA; A and V row-major in shared memory when in_smem (n <= kJacobiSmemN),
// else in global scratch.  Writes the nsel lowest eigenvalues to w and their
// eigenvectors to vr(:, 0:nsel) (ld ldv).
constexpr int kJacobiSmemN = 112;  // 2 n^2 doubles + pair tables within 227 KB

__host__ __device__ inline size_t jacobi_pairs_bytes(int n) {
  const int ne = n + (n & 1);
  return ((size_t)(ne / 2) * (2 * sizeof(double) + 2 * sizeof(int)) + sizeof(int) * n + 15) / 16 * 16;
}

__global__ void __launch_bounds__(1024) k_jacobi(const double* __restrict__ hr, long ldh, int n,
                                                 double* __restrict__ Ag, double* __restrict__ Vg,
                                                 int nsel, double* __restrict__ w, double* __restrict__ vr,
                                                 long ldv, int* __restrict__ sweeps_out, int in_smem) {
  extern __shared__ __align__(16) unsigned char shm[];
  const int ne = n + (n & 1);
  const int npairs = ne / 2;
  double* A = in_smem ? reinterpret_cast<double*>(shm + jacobi_pairs_bytes(n)) : Ag;
  double* V = in_smem ? A + (size_t)n * n : Vg;
  double* cs = reinterpret_cast<double*>(shm);           // [npairs] cos
  double* sn = cs + npairs;                                // [npairs] sin
  int* pp = reinterpret_cast<int*>(sn + npairs);           // [npairs]
  int* qq = pp + npairs;                                   // [npairs]
  int* idx = qq + npairs;                                  // [n]
  __shared__ double red[2][32];
  __shared__ int done;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e % n;
    A[e] = (i <= j) ? hr[(long)j * ldh + i] : hr[(long)i * ldh + j];
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e % n;
      const double v = A[e];
      if (i == j) dia = fma(v, v, dia); else off = fma(v, v, off);
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    if ((tid & 31) == 0) { red[0][tid >> 5] = off; red[1][tid >> 5] = dia; }
    __syncthreads();
    if (tid == 0) {
      double to = 0.0, td = 0.0;
      for (int i = 0; i < (nt + 31) / 32; ++i) { to += red[0][i]; td += red[1][i]; }
      done = (to <= 1e-30 * (td + to)) ? 1 : 0;   // off-diagonal Frobenius norm below 1e-15 of the total
    }
    __syncthreads();
    if (done) break;
    for (int r = 0; r < ne - 1; ++r) {
      for (int k = tid; k < npairs; k += nt) {
        const int a0 = (k == 0) ? 0 : 1 + ((k - 1 + r) % (ne - 1));
        const int kk = ne - 1 - k;
        const int b0 = 1 + ((kk - 1 + r) % (ne - 1));
        const int p = min(a0, b0), q = max(a0, b0);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[p * n + q];
          if (fabs(apq) > 1e-300) {
            const double tau = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        cs[k] = c; sn[k] = s; pp[k] = p; qq[k] = q;
      }
      __syncthreads();
      // A <- J^T A J in one pass: the round's planes are disjoint, so each 2x2
      // block (rows p1, q1 of plane k1; columns p2, q2 of plane k2) is owned by
      // one thread, which rotates its rows, then its columns (the same
      // arithmetic as a row pass followed by a column pass); V <- V J alongside
      for (int e = tid; e < npairs * npairs; e += nt) {
        const int k1 = e / npairs, k2 = e % npairs;
        const int p1 = pp[k1], q1 = qq[k1], p2 = pp[k2], q2 = qq[k2];
        const bool r2 = q1 < n, c2 = q2 < n;  // the padding index of odd n has no row / column
        const double ca = cs[k1], sa = sn[k1], cb = cs[k2], sb = sn[k2];
        const double a = A[p1 * n + p2];
        const double b = c2 ? A[p1 * n + q2] : 0.0;
        const double cc = r2 ? A[q1 * n + p2] : 0.0;
        const double d = (r2 && c2) ? A[q1 * n + q2] : 0.0;
        double ra = a, rb = b, rc = cc, rd = d;
        if (r2 && sa != 0.0) {
          ra = ca * a - sa * cc;
          rc = sa * a + ca * cc;
          rb = ca * b - sa * d;
          rd = sa * b + ca * d;
        }
        if (c2 && sb != 0.0) {
          A[p1 * n + p2] = cb * ra - sb * rb;
          A[p1 * n + q2] = sb * ra + cb * rb;
          if (r2) {
            A[q1 * n + p2] = cb * rc - sb * rd;
            A[q1 * n + q2] = sb * rc + cb * rd;
          }
        } else {
          A[p1 * n + p2] = ra;
          if (c2) A[p1 * n + q2] = rb;
          if (r2) {
            A[q1 * n + p2] = rc;
            if (c2) A[q1 * n + q2] = rd;
          }
        }
      }
      for (int e = tid; e < npairs * n; e += nt) {      // V <- V J; lanes run over the planes of a
        const int i = e / npairs, k = e % npairs;       // row (rows are n doubles apart: one bank)
        const int p = pp[k], q = qq[k];
        if (q >= n || sn[k] == 0.0) continue;
        const double c = cs[k], s = sn[k];
        const double vp = V[i * n + p], vq = V[i * n + q];
        V[i * n + p] = c * vp - s * vq;
        V[i * n + q] = s * vp + c * vq;
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    for (int i = 0; i < n; ++i) idx[i] = i;
    for (int i = 0; i < n; ++i) {                         // selection sort, ascending
      int best = i;
      for (int j = i + 1; j < n; ++j)
        if (A[idx[j] * n + idx[j]] < A[idx[best] * n + idx[best]]) best = j;
      const int t = idx[i]; idx[i] = idx[best]; idx[best] = t;
    }
    *sweeps_out = sweep;
  }
  __syncthreads();
  for (int e = tid; e < nsel * n; e += nt) {
    const int k = e / n, r = e % n;
    vr[(long)k * ldv + r] = V[r * n + idx[k]];
  }
  for (int k = tid; k < nsel; k += nt) w[k] = A[idx[k] * n + idx[k]];
}

// Rotation of plane (p, q) that zeroes A[p][q]: t = tan(theta) from
// cot(2 theta) = (a_qq - a_pp) / (2 a_pq), written as h sgn(d) / (|d| + sqrt(d^2 + h^2))
// with d = a_qq - a_pp and h = 2 a_pq (one square root and one division).
__device__ __forceinline__ void jacobi_rotation(const double* __restrict__ A, int ld, int p, int q, double& c,
                                                double& s) {
  const double apq = A[p * ld + q];
  c = 1.0;
  s = 0.0;
  if (fabs(apq) > 1e-300) {
    const double d = A[q * ld + q] - A[p * ld + p], h = 2.0 * apq;
    const double t = (d >= 0.0 ? h : -h) / (fabs(d) + sqrt(fma(d, d, h * h)));
    c = rsqrt(fma(t, t, 1.0));
    s = t * c;
  }
}

// The same cyclic Jacobi for n <= kJacobiFastN with one barrier per round.  The
// matrix is padded to ne = n + (n & 1) (the zero row and column of odd n never
// rotate).  Thread (k1, k2) of the npairs^2 threads owns the 2 x 2 block of
// planes k1, k2 and rows k2, k2 + npairs of plane k1's two columns of V
// (column-major, so a warp's lanes touch consecutive rows).  Each thread derives
// the rotations of its two planes from the previous round's matrix itself (the
// lanes of a warp share k1) and writes the next matrix to the other buffer, so no
// barrier separates the rotation parameters from the update; the planes of a
// thread advance through the round-robin ordering by increments.
constexpr int kJacobiFastN = 64;

__host__ __device__ inline size_t jacobi_fast_bytes(int n) {
  const int ne = n + (n & 1);
  return 3 * sizeof(double) * ne * ne + sizeof(int) * n;
}

__global__ void __launch_bounds__(1024) k_jacobi_fast(const double* __restrict__ hr, long ldh, int n, int nsel,
                                                      double* __restrict__ w, double* __restrict__ vr, long ldv,
                                                      int* __restrict__ sweeps_out) {
  extern __shared__ __align__(16) unsigned char shm[];
  const int ne = n + (n & 1), np = ne / 2, m = ne - 1;
  double* Ac = reinterpret_cast<double*>(shm);
  double* An = Ac + ne * ne;
  double* V = An + ne * ne;                          // V[col * ne + row]
  int* idx = reinterpret_cast<int*>(V + ne * ne);    // [n]
  __shared__ double red[2][32];
  __shared__ int done;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < ne * ne; e += nt) {
    const int i = e / ne, j = e % ne;
    double a = 0.0;
    if (i < n && j < n) a = (i <= j) ? hr[(long)j * ldh + i] : hr[(long)i * ldh + j];
    Ac[e] = a;
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  const bool act = tid < np * np;
  const int k1 = act ? tid / np : 0, k2 = act ? tid % np : 0;
  __syncthreads();
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int e = tid; e < ne * ne; e += nt) {
      const double v = Ac[e];
      if (e / ne == e % ne) dia = fma(v, v, dia); else off = fma(v, v, off);
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    if ((tid & 31) == 0) { red[0][tid >> 5] = off; red[1][tid >> 5] = dia; }
    __syncthreads();
    if (tid == 0) {
      double to = 0.0, td = 0.0;
      for (int i = 0; i < (nt + 31) / 32; ++i) { to += red[0][i]; td += red[1][i]; }
      done = (to <= 1e-30 * (td + to)) ? 1 : 0;   // off-diagonal Frobenius norm below 1e-15 of the total
    }
    __syncthreads();
    if (done) break;
    // plane k of round r: (1 + (k - 1 + r) mod m, or 0 for k = 0) and 1 + (m - 1 - k + r) mod m
    int xa1 = k1 > 0 ? k1 - 1 : 0, xb1 = m - 1 - k1;
    int xa2 = k2 > 0 ? k2 - 1 : 0, xb2 = m - 1 - k2;
    for (int r = 0; r < m; ++r) {
      if (act) {
        const int a1 = k1 > 0 ? 1 + xa1 : 0, b1 = 1 + xb1, a2 = k2 > 0 ? 1 + xa2 : 0, b2 = 1 + xb2;
        const int p1 = min(a1, b1), q1 = max(a1, b1), p2 = min(a2, b2), q2 = max(a2, b2);
        double ca, sa, cb, sb;
        jacobi_rotation(Ac, ne, p1, q1, ca, sa);
        jacobi_rotation(Ac, ne, p2, q2, cb, sb);
        const double a = Ac[p1 * ne + p2], b = Ac[p1 * ne + q2], cc = Ac[q1 * ne + p2], d = Ac[q1 * ne + q2];
        const double ra = ca * a - sa * cc, rc = sa * a + ca * cc;
        const double rb = ca * b - sa * d, rd = sa * b + ca * d;
        An[p1 * ne + p2] = cb * ra - sb * rb;
        An[q1 * ne + q2] = sb * rc + cb * rd;
        if (k1 == k2) {               // the plane's own pivot: zero by construction
          An[p1 * ne + q2] = 0.0;
          An[q1 * ne + p2] = 0.0;
        } else {
          An[p1 * ne + q2] = sb * ra + cb * rb;
          An[q1 * ne + p2] = cb * rc - sb * rd;
        }
        double* vp = V + p1 * ne;
        double* vq = V + q1 * ne;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int i = k2 + h * np;
          const double x = vp[i], y = vq[i];
          vp[i] = ca * x - sa * y;
          vq[i] = sa * x + ca * y;
        }
      }
      xa1 = xa1 + 1 == m ? 0 : xa1 + 1;
      xb1 = xb1 + 1 == m ? 0 : xb1 + 1;
      xa2 = xa2 + 1 == m ? 0 : xa2 + 1;
      xb2 = xb2 + 1 == m ? 0 : xb2 + 1;
      __syncthreads();
      double* t = Ac; Ac = An; An = t;
    }
  }
  for (int i = tid; i < n; i += nt) {   // rank of eigenvalue i (ascending, ties by index)
    const double li = Ac[i * ne + i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double lj = Ac[j * ne + j];
      rank += (lj < li || (lj == li && j < i)) ? 1 : 0;
    }
    if (rank < nsel) idx[rank] = i;
  }
  if (tid == 0) *sweeps_out = sweep;
  __syncthreads();
  for (int e = tid; e < nsel * n; e += nt) {
    const int k = e / n, r = e % n;
    vr[(long)k * ldv + r] = V[idx[k] * ne + r];
  }
  for (int k = tid; k < nsel; k += nt) w[k] = Ac[idx[k] * ne + idx[k]];
}

// ---------------------------------------------------------------------------
// Parallel two-sided block Jacobi for bases above kJacobiSmemN (up to 1024)
// ---------------------------------------------------------------------------
// The matrix (padded to npad = nb * kBJ with zero rows and columns, nb even) is
// cut into nb blocks of kBJ indices.  A sweep runs nb - 1 rounds of the same
// round-robin ordering as k_jacobi over blocks: in a round the nb / 2 disjoint
// block pairs P = I u J each diagonalise their 2 kBJ x 2 kBJ submatrix
// A[P, P] = U diag U^T in shared memory (one CTA per pair, the cyclic Jacobi
// above, to convergence), then A <- Q^T A Q and V <- V Q with Q =
// blockdiag(U_P), as independent tiles (pair x pair for A, rows x pair for V).
// Sweeps stop when the off-diagonal Frobenius norm is below 1e-14 of the whole:
// the rotations are applied as 32-term dot products, which leave rounding
// residues of about sqrt(n) eps ||A|| off the diagonal, so k_jacobi's 1e-15 is
// out of reach for large n; the eigenvalue error is second order in the
// off-diagonal norm, and the selected eigenvalues are recomputed at the end as
// Rayleigh quotients v^T hr v of the input matrix (first-order error in v only
// enters squared).  A pair whose off-diagonal block holds less than its share
// (1 / number of block pairs) of 1e-30 ||A||^2 keeps U = 1 and its tiles are
// left alone.  Padded indices carry no coupling, so they never rotate; they are
// excluded from the selection.
constexpr int kBJ = 16;
constexpr int kMaxBasis = 4096;
constexpr int kBJNormCtas = 1184;  // grid of the norm reduction (8 CTAs per SM)
constexpr int kBJ2 = 2 * kBJ;
constexpr int kBJThreads = 256;

__device__ __forceinline__ void bj_pair(int k, int r, int nb, int& I, int& J) {
  const int a0 = (k == 0) ? 0 : 1 + ((k - 1 + r) % (nb - 1));
  const int kk = nb - 1 - k;
  const int b0 = 1 + ((kk - 1 + r) % (nb - 1));
  I = min(a0, b0);
  J = max(a0, b0);
}
__device__ __forceinline__ int bj_glob(int l, int I, int J) { return l < kBJ ? I * kBJ + l : J * kBJ + (l - kBJ); }

__global__ void k_bj_init(const double* __restrict__ hr, long ldh, int n, int npad, double* __restrict__ A,
                          double* __restrict__ V) {
  const long nn = (long)npad * npad;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nn; e += (long)gridDim.x * blockDim.x) {
    const int i = (int)(e / npad), j = (int)(e % npad);
    double a = 0.0;
    if (i < n && j < n) a = (i <= j) ? hr[(long)j * ldh + i] : hr[(long)i * ldh + j];
    A[e] = a;
    V[e] = (i == j) ? 1.0 : 0.0;
  }
}

// per-CTA partial sums of the squared off-diagonal entries and of all entries
// (part[2 b], part[2 b + 1]); k_bj_norms_final adds them in a fixed order, so
// every run (and every rank of a sharded Davidson) takes the same decisions
__global__ void k_bj_norms(const double* __restrict__ A, int npad, double* __restrict__ part) {
  __shared__ double sh[2][32];
  double off = 0.0, tot = 0.0;
  const long nn = (long)npad * npad;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nn; e += (long)gridDim.x * blockDim.x) {
    const double v = A[e];
    tot = fma(v, v, tot);
    if (e / npad != e % npad) off = fma(v, v, off);
  }
  for (int o = 16; o > 0; o >>= 1) {
    off += __shfl_xor_sync(0xffffffffu, off, o);
    tot += __shfl_xor_sync(0xffffffffu, tot, o);
  }
  if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = off; sh[1][threadIdx.x >> 5] = tot; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double so = 0.0, st = 0.0;
    for (int i = 0; i < (int)blockDim.x / 32; ++i) { so += sh[0][i]; st += sh[1][i]; }
    part[2 * blockIdx.x] = so;
    part[2 * blockIdx.x + 1] = st;
  }
}
__global__ void k_bj_norms_final(const double* __restrict__ part, int nparts, double* __restrict__ red) {
  if (threadIdx.x == 0) {
    double so = 0.0, st = 0.0;
    for (int i = 0; i < nparts; ++i) { so += part[2 * i]; st += part[2 * i + 1]; }
    red[0] = so;
    red[1] = st;
  }
}

// k_bj_norms_final for the sweep loop of a CUDA graph: also counts the sweeps
// (first: the check before any) and sets the loop's WHILE condition to the
// host loop's test (continue while the off-diagonal norm exceeds 1e-14 of the
// whole and fewer than 40 sweeps ran).
__global__ void k_bj_norms_cond(const double* __restrict__ part, int nparts, double* __restrict__ red,
                                cudaGraphConditionalHandle h, int first) {
  if (threadIdx.x == 0) {
    double so = 0.0, st = 0.0;
    for (int i = 0; i < nparts; ++i) { so += part[2 * i]; st += part[2 * i + 1]; }
    red[0] = so;
    red[1] = st;
    int* sweep = reinterpret_cast<int*>(red + 2);
    const int sw = first ? 0 : *sweep + 1;
    *sweep = sw;
    cudaGraphSetConditional(h, (!(so <= 1e-28 * st) && sw < 40) ? 1u : 0u);
  }
}

// One CTA per block pair of round r: U_P (row-major, U[l][m]) of the pair's
// 2 kBJ x 2 kBJ submatrix, or the identity with skip[k] = 1.
__global__ void __launch_bounds__(kBJThreads) k_bj_solve(const double* __restrict__ A, int npad, int nb, int r,
                                                         const double* __restrict__ red, double* __restrict__ U,
                                                         int* __restrict__ skip, double skip_frac) {
  constexpr int n = kBJ2, npairs = kBJ2 / 2;
  __shared__ double S[n * n], Q[n * n];
  __shared__ double cs[npairs], sn[npairs];
  __shared__ int pp[npairs], qq[npairs];
  __shared__ double sh[2][kBJThreads / 32];
  __shared__ int done;
  const int tid = threadIdx.x, k = blockIdx.x;
  int I, J;
  bj_pair(k, r, nb, I, J);
  double offij = 0.0;
  for (int e = tid; e < n * n; e += kBJThreads) {
    const int i = e / n, j = e % n;
    const double v = A[(long)bj_glob(i, I, J) * npad + bj_glob(j, I, J)];
    S[e] = v;
    Q[e] = (i == j) ? 1.0 : 0.0;
    if (i < kBJ && j >= kBJ) offij = fma(v, v, offij);
  }
  for (int o = 16; o > 0; o >>= 1) offij += __shfl_xor_sync(0xffffffffu, offij, o);
  if ((tid & 31) == 0) sh[0][tid >> 5] = offij;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int i = 0; i < kBJThreads / 32; ++i) s += sh[0][i];
    done = (s <= skip_frac * red[1]) ? 1 : 0;
  }
  __syncthreads();
  double* Uk = U + (long)k * n * n;
  if (done) {
    for (int e = tid; e < n * n; e += kBJThreads) Uk[e] = Q[e];
    if (tid == 0) skip[k] = 1;
    return;
  }
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int e = tid; e < n * n; e += kBJThreads) {
      const double v = S[e];
      if (e / n == e % n) dia = fma(v, v, dia); else off = fma(v, v, off);
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    __syncthreads();
    if ((tid & 31) == 0) { sh[0][tid >> 5] = off; sh[1][tid >> 5] = dia; }
    __syncthreads();
    if (tid == 0) {
      double to = 0.0, td = 0.0;
      for (int i = 0; i < kBJThreads / 32; ++i) { to += sh[0][i]; td += sh[1][i]; }
      done = (to <= 1e-32 * (td + to)) ? 1 : 0;
    }
    __syncthreads();
    if (done) break;
    for (int rr = 0; rr < n - 1; ++rr) {
      if (tid < npairs) {
        const int kq = tid;
        const int a0 = (kq == 0) ? 0 : 1 + ((kq - 1 + rr) % (n - 1));
        const int kk = n - 1 - kq;
        const int b0 = 1 + ((kk - 1 + rr) % (n - 1));
        const int p = min(a0, b0), q = max(a0, b0);
        double c = 1.0, s = 0.0;
        const double apq = S[p * n + q];
        if (fabs(apq) > 1e-300) {
          const double tau = (S[q * n + q] - S[p * n + p]) / (2.0 * apq);
          const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        cs[kq] = c; sn[kq] = s; pp[kq] = p; qq[kq] = q;
      }
      __syncthreads();
      for (int e = tid; e < npairs * npairs; e += kBJThreads) {   // S <- J^T S J, 2x2 block per thread
        const int k1 = e / npairs, k2 = e % npairs;
        const int p1 = pp[k1], q1 = qq[k1], p2 = pp[k2], q2 = qq[k2];
        const double ca = cs[k1], sa = sn[k1], cb = cs[k2], sb = sn[k2];
        const double a = S[p1 * n + p2], b = S[p1 * n + q2], cc = S[q1 * n + p2], d = S[q1 * n + q2];
        const double ra = ca * a - sa * cc, rc = sa * a + ca * cc;
        const double rb = ca * b - sa * d, rd = sa * b + ca * d;
        S[p1 * n + p2] = cb * ra - sb * rb;
        S[q1 * n + q2] = sb * rc + cb * rd;
        if (k1 == k2 && sa != 0.0) {              // the plane's own pivot: zero by construction
          S[p1 * n + q2] = 0.0;
          S[q1 * n + p2] = 0.0;
        } else {
          S[p1 * n + q2] = sb * ra + cb * rb;
          S[q1 * n + p2] = cb * rc - sb * rd;
        }
      }
      for (int e = tid; e < npairs * n; e += kBJThreads) {         // Q <- Q J, lanes over the planes
        const int i = e / npairs, kq = e % npairs;
        const int p = pp[kq], q = qq[kq];
        const double c = cs[kq], s = sn[kq];
        const double vp = Q[i * n + p], vq = Q[i * n + q];
        Q[i * n + p] = c * vp - s * vq;
        Q[i * n + q] = s * vp + c * vq;
      }
      __syncthreads();
    }
  }
  for (int e = tid; e < n * n; e += kBJThreads) Uk[e] = Q[e];
  if (tid == 0) skip[k] = 0;
}

// A[P1, P2] <- U_P1^T A[P1, P2] U_P2 for the pair tile (blockIdx.x, blockIdx.y)
__global__ void __launch_bounds__(kBJThreads) k_bj_apply_a(double* __restrict__ A, int npad, int nb, int r,
                                                           const double* __restrict__ U,
                                                           const int* __restrict__ skip) {
  constexpr int n = kBJ2;
  const int k1 = blockIdx.x, k2 = blockIdx.y;
  if (skip[k1] && skip[k2]) return;
  __shared__ double U1[n * n], U2[n * n], T[n * n];
  int I1, J1, I2, J2;
  bj_pair(k1, r, nb, I1, J1);
  bj_pair(k2, r, nb, I2, J2);
  const int tid = threadIdx.x;
  for (int e = tid; e < n * n; e += kBJThreads) {
    U1[e] = U[(long)k1 * n * n + e];
    U2[e] = U[(long)k2 * n * n + e];
    T[e] = A[(long)bj_glob(e / n, I1, J1) * npad + bj_glob(e % n, I2, J2)];
  }
  __syncthreads();
  constexpr int PER = n * n / kBJThreads;
  double o[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {                 // (U1^T T)[i][j]
    const int e = tid + q * kBJThreads, i = e / n, j = e % n;
    double s = 0.0;
#pragma unroll 8
    for (int l = 0; l < n; ++l) s = fma(U1[l * n + i], T[l * n + j], s);
    o[q] = s;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; ++q) T[tid + q * kBJThreads] = o[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; ++q) {                 // (U1^T T U2)[i][j]
    const int e = tid + q * kBJThreads, i = e / n, j = e % n;
    double s = 0.0;
#pragma unroll 8
    for (int l = 0; l < n; ++l) s = fma(T[i * n + l], U2[l * n + j], s);
    A[(long)bj_glob(i, I1, J1) * npad + bj_glob(j, I2, J2)] = s;
  }
}

// V[rows, P] <- V[rows, P] U_P for rows [32 blockIdx.x, + 32) and pair blockIdx.y
__global__ void __launch_bounds__(kBJThreads) k_bj_apply_v(double* __restrict__ V, int npad, int nb, int r,
                                                           const double* __restrict__ U,
                                                           const int* __restrict__ skip) {
  constexpr int n = kBJ2;
  const int k = blockIdx.y, r0 = blockIdx.x * n;
  if (skip[k]) return;
  __shared__ double Uk[n * n], T[n * n];
  int I, J;
  bj_pair(k, r, nb, I, J);
  const int tid = threadIdx.x;
  for (int e = tid; e < n * n; e += kBJThreads) {
    Uk[e] = U[(long)k * n * n + e];
    T[e] = V[(long)(r0 + e / n) * npad + bj_glob(e % n, I, J)];
  }
  __syncthreads();
  constexpr int PER = n * n / kBJThreads;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = tid + q * kBJThreads, i = e / n, j = e % n;
    double s = 0.0;
#pragma unroll 8
    for (int l = 0; l < n; ++l) s = fma(T[i * n + l], Uk[l * n + j], s);
    V[(long)(r0 + i) * npad + bj_glob(j, I, J)] = s;
  }
}

// The nsel lowest of the n real eigenvalues (diag A, padding excluded) in
// ascending order into w, their eigenvectors (columns of V) into vr(:, 0:nsel).
__global__ void __launch_bounds__(1024) k_bj_select(const double* __restrict__ A, const double* __restrict__ V,
                                                    int n, int npad, int nsel, double* __restrict__ w,
                                                    double* __restrict__ vr, long ldv, int* __restrict__ idx) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double li = A[(long)i * npad + i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double lj = A[(long)j * npad + j];
      rank += (lj < li || (lj == li && j < i)) ? 1 : 0;
    }
    if (rank < nsel) { w[rank] = li; idx[rank] = i; }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nsel * n; e += blockDim.x) {
    const int k = e / n, rr = e % n;
    vr[(long)k * ldv + rr] = V[(long)rr * npad + idx[k]];
  }
}

// For each selected eigenvector v_k (vr column k): w[k] <- v^T hr v / v^T v and
// v <- v / |v|.  The many block rotations let the column norms of V drift by
// about 1e-12, which would scale every eigenvalue by as much.  hr is read from
// its upper triangle; one CTA per eigenvector.
__global__ void __launch_bounds__(256) k_bj_rayleigh(const double* __restrict__ hr, long ldh, int n,
                                                     double* __restrict__ vr, long ldv, double* __restrict__ w) {
  __shared__ double sv[4096];
  __shared__ double red[16];
  const int k = blockIdx.x;
  double* v = vr + (long)k * ldv;
  for (int i = threadIdx.x; i < n; i += 256) sv[i] = v[i];
  __syncthreads();
  double vhv = 0.0, vv = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) {    // row i of hr: (i, j) = hr[j ldh + i] for j >= i, hr[i ldh + j] below
    double hv = 0.0;
    const double* col = hr + (long)i * ldh;
    for (int j = 0; j < i; ++j) hv = fma(col[j], sv[j], hv);
    for (int j = i; j < n; ++j) hv = fma(hr[(long)j * ldh + i], sv[j], hv);
    vhv = fma(sv[i], hv, vhv);
    vv = fma(sv[i], sv[i], vv);
  }
  const double2 r = block_sum2<256>(vhv, vv, red);
  if (threadIdx.x == 0) w[k] = r.x / r.y;
  const double sc = 1.0 / sqrt(r.y);
  for (int i = threadIdx.x; i < n; i += 256) v[i] = sv[i] * sc;
}

// Scratch of the block Jacobi for bases up to nmax, in doubles.
size_t bj_doubles(int nmax) {
  int nb = (nmax + kBJ - 1) / kBJ;
  nb += nb & 1;
  const size_t npad = (size_t)nb * kBJ;
  return 2 * npad * npad + (size_t)(nb / 2) * kBJ2 * kBJ2 + 4 + nmax + nb + 2 * kBJNormCtas;
}

// One sweep: nb - 1 rounds of block-pair solves and tile rotations.
void bj_sweep(double* A, double* V, double* U, const double* red, int* skip, int npad, int nb, double skip_frac,
              cudaStream_t s) {
  const int npair = nb / 2;
  for (int r = 0; r < nb - 1; ++r) {
    k_bj_solve<<<npair, kBJThreads, 0, s>>>(A, npad, nb, r, red, U, skip, skip_frac);
    k_bj_apply_a<<<dim3(npair, npair), kBJThreads, 0, s>>>(A, npad, nb, r, U, skip);
    k_bj_apply_v<<<dim3(npad / kBJ2, npair), kBJThreads, 0, s>>>(V, npad, nb, r, U, skip);
  }
}

// Lowest nsel eigenpairs of the symmetric hr[:n, :n] (upper triangle, column
// major, ld ldh): w (device, ascending) and vr(:, 0:nsel) (device, ld ldv).
// scratch holds bj_doubles(n).  Run eagerly, the sweeps stop on norms read by
// the host (red_host: two doubles); while s is being captured into a CUDA graph
// they run inside a conditional WHILE node whose condition k_bj_norms_cond sets
// from the same test, the sweeps' kernels captured on the idle stream aux into
// the node's body (nodes added to the capture graph as cudaStreamGetCaptureInfo /
// cudaStreamUpdateCaptureDependencies provide).  Both forms launch the same
// kernels in the same order.
int block_jacobi(const double* hr, long ldh, int n, int nsel, double* w, double* vr, long ldv, double* scratch,
                 double* red_host, int* sweeps_out, cudaStream_t s, cudaStream_t aux) {
  int nb = (n + kBJ - 1) / kBJ;
  nb += nb & 1;
  const int npad = nb * kBJ, npair = nb / 2;
  double* A = scratch;
  double* V = A + (size_t)npad * npad;
  double* U = V + (size_t)npad * npad;
  double* red = U + (size_t)npair * kBJ2 * kBJ2;  // red[0..1] norms, red[2] the sweep count of the graph form
  double* npart = red + 4;                     // per-CTA partial norms
  int* iw = reinterpret_cast<int*>(npart + 2 * kBJNormCtas);  // skip flags, then the selection indices
  int* skip = iw;
  int* idx = iw + nb;
  const int g = std::min(kBJNormCtas, (int)(((long)npad * npad + 255) / 256));
  const double skip_frac = 1e-30 / (0.5 * nb * (nb - 1));
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  WB_CU(cudaStreamIsCapturing(s, &cs));
  int sweep = 0;
  if (cs == cudaStreamCaptureStatusActive) {
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    WB_CU(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    WB_CU(cudaGraphConditionalHandleCreate(&h, cg, 0, 0));
    k_bj_init<<<g, 256, 0, s>>>(hr, ldh, n, npad, A, V);
    k_bj_norms<<<g, 256, 0, s>>>(A, npad, npart);
    k_bj_norms_cond<<<1, 32, 0, s>>>(npart, g, red, h, 1);
    WB_CU(cudaGetLastError());
    WB_CU(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    WB_CU(cudaGraphAddNode(&wnode, cg, deps, nd, &wp));
    WB_CU(cudaStreamUpdateCaptureDependencies(s, &wnode, 1, cudaStreamSetCaptureDependencies));
    if (!aux) return fail(WB_ERR_ARG, "block Jacobi capture needs a second stream");
    cudaStream_t s2 = aux;
    cudaError_t e = cudaStreamBeginCaptureToGraph(s2, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      bj_sweep(A, V, U, red, skip, npad, nb, skip_frac, s2);
      k_bj_norms<<<g, 256, 0, s2>>>(A, npad, npart);
      k_bj_norms_cond<<<1, 32, 0, s2>>>(npart, g, red, h, 0);
      e = cudaGetLastError();
      cudaGraph_t bg = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(s2, &bg);
      if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return fail(WB_ERR_CUDA, std::string("block Jacobi sweep capture: ") + cudaGetErrorString(e));
    sweep = -1;  // counted on the device
  } else {
    k_bj_init<<<g, 256, 0, s>>>(hr, ldh, n, npad, A, V);
    for (;; ++sweep) {
      k_bj_norms<<<g, 256, 0, s>>>(A, npad, npart);
      k_bj_norms_final<<<1, 32, 0, s>>>(npart, g, red);
      WB_CU(cudaMemcpyAsync(red_host, red, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
      WB_CU(cudaStreamSynchronize(s));
      if (red_host[0] <= 1e-28 * red_host[1] || sweep == 40) break;
      bj_sweep(A, V, U, red, skip, npad, nb, skip_frac, s);
      WB_CU(cudaGetLastError());
    }
  }
  k_bj_select<<<1, 1024, 0, s>>>(A, V, n, npad, nsel, w, vr, ldv, idx);
  k_bj_rayleigh<<<nsel, 256, 0, s>>>(hr, ldh, n, vr, ldv, w);
  WB_CU(cudaGetLastError());
  *sweeps_out = sweep;
  return WB_OK;
}

// diagox_dsy (Wstat/wstat_tools.f90:48): the one-CTA shared-memory Jacobis up
// to kJacobiFastN and kJacobiSmemN, the block Jacobi above.  A and V: n^2 doubles each of
// global scratch (unused by the shared-memory path); bj: bj_doubles(n); aux: a
// second stream, needed when s is being captured and n > kJacobiSmemN.
int eigen_lowest(const double* hr, long ldh, int n, int nsel, double* w, double* vr, long ldv, double* A, double* V,
                 double* bj, int* sweeps, cudaStream_t s, cudaStream_t aux = nullptr) {
  if (n > kJacobiSmemN) {
    int sw = 0;
    double red[2];
    return block_jacobi(hr, ldh, n, nsel, w, vr, ldv, bj, red, &sw, s, aux);
  }
  if (n <= kJacobiFastN) {
    const int np = (n + 1) / 2;
    const int nt = std::max(32, (np * np + 31) / 32 * 32);
    k_jacobi_fast<<<1, nt, jacobi_fast_bytes(n), s>>>(hr, ldh, n, nsel, w, vr, ldv, sweeps);
    WB_CU(cudaGetLastError());
    return WB_OK;
  }
  const size_t shm = jacobi_pairs_bytes(n) + 2 * sizeof(double) * n * n;
  k_jacobi<<<1, 1024, shm, s>>>(hr, ldh, n, A, V, nsel, w, vr, ldv, sweeps, 1);
  WB_CU(cudaGetLastError());
  return WB_OK;
}

void jacobi_setup() {
  cudaFuncSetAttribute(k_jacobi_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)jacobi_fast_bytes(kJacobiFastN));
  cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(jacobi_pairs_bytes(kJacobiSmemN) + 2 * sizeof(double) * kJacobiSmemN * kJacobiSmemN));
}

// ---------------------------------------------------------------------------
// Iteration state on the device: st[0] = number of unconverged eigenpairs,
// st[1 + i] = conv(i), and ev(i) at dav_ev_offset(nvec) bytes.
// ---------------------------------------------------------------------------
inline size_t dav_ev_offset(int nvec) { return ((size_t)(1 + nvec) * sizeof(int) + 7) / 8 * 8; }
inline size_t dav_state_bytes(int nvec) { return dav_ev_offset(nvec) + sizeof(double) * nvec; }

// Reordering of davidson_diago.f90:273-296 (redistribute_vr_distr): the j-th
// unconverged index n (conv(n) = 0, ascending) moves vr(:, n) to vr(:, nbase + j)
// and ev(n) to w(nbase + j).  One CTA per new column; its first warp finds n by
// ballots over conv.  Sources (n < nvec <= nbase) and targets never overlap.
__global__ void __launch_bounds__(256) k_dav_shift(const int* __restrict__ st, const double* __restrict__ ev, int nvec,
                                                   int nbase, double* __restrict__ vr, long ldv, int nrow,
                                                   double* __restrict__ w) {
  const int* conv = st + 1;
  const int j = blockIdx.x;
  __shared__ int src;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int base = 0, found = -1;
    for (int n0 = 0; n0 < nvec && found < 0; n0 += 32) {
      const int n = n0 + lane;
      const unsigned b = __ballot_sync(0xffffffffu, n < nvec && conv[n] == 0);
      const int cnt = __popc(b);
      if (j < base + cnt) {
        unsigned bb = b;
        for (int t = 0; t < j - base; ++t) bb &= bb - 1;
        found = n0 + __ffs(bb) - 1;
      }
      base += cnt;
    }
    if (lane == 0) src = found;
  }
  __syncthreads();
  const int n = src;
  if (n < 0) return;
  if (threadIdx.x == 0) w[nbase + j] = ev[n];
  for (int r = threadIdx.x; r < nrow; r += blockDim.x) vr[(long)(nbase + j) * ldv + r] = vr[(long)n * ldv + r];
}

// Convergence test of davidson_diago.f90:346-347 on the new Ritz values w
// against ev (test = 1; the extra starting step only copies), then ev <- w and
// st[0] = number not converged.  One CTA.
__global__ void __launch_bounds__(256) k_dav_conv(const double* __restrict__ w, double* __restrict__ ev,
                                                  int* __restrict__ st, int nvec, double trev, double trev_rel,
                                                  int test) {
  int* conv = st + 1;
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
    const double e = w[i], o = ev[i];
    if (test) conv[i] = (fabs((e - o) / o) < trev_rel) && (fabs(e - o) < trev) ? 1 : 0;
    mine += conv[i] ? 0 : 1;
    ev[i] = e;
  }
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) st[0] = cnt;
}

constexpr size_t kMaxDavGraphs = 64;

// Runs body (stream work only) on s: eagerly without graphs, else from the
// cached executable of key, capturing and instantiating it on a miss.
template <class F>
int dav_graph(wb_ctx* c, cudaStream_t s, const std::vector<long long>& key, F body) {
  if (!c->use_graphs) return body();
  auto& gs = c->dav_graphs;
  for (size_t i = 0; i < gs.size(); ++i)
    if (gs[i].key == key) {
      std::rotate(gs.begin(), gs.begin() + i, gs.begin() + i + 1);
      WB_CU(cudaGraphLaunch(gs[0].exec, s));
      return WB_OK;
    }
  WB_CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const int rc = body();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(WB_ERR_CUDA, std::string("Davidson graph capture: ") + cudaGetErrorString(e));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return fail(WB_ERR_CUDA, std::string("Davidson graph instantiation: ") + cudaGetErrorString(ei));
  if (gs.size() >= kMaxDavGraphs) {
    cudaGraphExecDestroy(gs.back().exec);
    gs.pop_back();
  }
  gs.insert(gs.begin(), wb_ctx::DavGraph{key, ex});
  WB_CU(cudaGraphLaunch(ex, s));
  return WB_OK;
}

inline long long key_bits(double x) {
  long long b;
  std::memcpy(&b, &x, sizeof(b));
  return b;
}
inline long long key_ptr(const void* p) { return (long long)(intptr_t)p; }

struct Dav {
  wb_ctx* c;
  int npw, nvec, nvecx;
  long ld;
  double2 *dvg, *dng, *tmp;
  double *hr, *vr, *A, *V, *w, *part, *coef, *dots;
  int* sweeps;
  int nsplit;
  cudaStream_t s;
  cudaStream_t aux = nullptr;  // second stream of the block Jacobi's graph form
  int apply_calls = 0;
  long long applied = 0;

  // do_mgs on columns [start, end) (davidson_diago.f90:909): the columns before
  // start are orthonormal, so the new block is first projected against all of
  // them at once, twice (classical Gram-Schmidt with reorthogonalisation: the
  // Gamma bra-ket GEMM and the update GEMM), then orthonormalised column by
  // column inside the block.  Same result as the reference's column order up
  // to rounding; two GEMM passes instead of two launches per old column.
  int mgs(int start, int end) {
    if (start > 0 && end > start) {
      const int K = 2 * npw, nb = end - start;
      const double* B = reinterpret_cast<const double*>(dvg);
      double* X = reinterpret_cast<double*>(dvg + (long)start * ld);
      for (int pass = 0; pass < 2; ++pass) {
        gemm_tn(B, 2 * ld, start, X, 2 * ld, nullptr, nb, K, nsplit, part, s);
        gamma_reduce(part, nsplit, start, nb, B, 2 * ld, X, 2 * ld, nullptr, nullptr, 0, -1.0, coef, s);
        gemm_nn(B, 2 * ld, start, coef, X, 2 * ld, nullptr, nb, K, 1.0, s);
      }
    }
    for (int k = start; k < end; ++k) {
      k_mgs_normalize<<<1, 256, 0, s>>>(dvg + (long)k * ld, npw);
      const int j0 = k + 1;
      if (j0 >= end) continue;
      k_mgs_dots<<<end - j0, 256, 0, s>>>(dvg, ld, npw, k, j0, dots);
      k_mgs_axpy<<<dim3((npw + 255) / 256, end - j0), 256, 0, s>>>(dvg, ld, npw, k, j0, dots);
    }
    WB_CU(cudaGetLastError());
    return WB_OK;
  }
  double apply_s = 0.0;
  bool pending = false;  // an operator call whose batch is enqueued but not yet waited for
  // Completes a pending operator call: waits for the stream unless the caller
  // just did, folds in its counters and its time (events around the batch).
  int settle(bool waited) {
    if (!pending) return WB_OK;
    if (!waited) WB_CU(wb_wait(c));
    apply_settle(c);
    float ms = 0.f;
    WB_CU(cudaEventElapsedTime(&ms, c->dav_ev[0], c->dav_ev[1]));
    apply_s += 1e-3 * ms;
    pending = false;
    return WB_OK;
  }
  // The operator on columns col0 .. col0 + n - 1.  The library's own call is
  // only enqueued when it fits one batch: the steps after it follow on the same
  // stream, and one wait (after them) covers both.
  int apply(int col0, int n, double tr2) {
    const double* x = reinterpret_cast<const double*>(dvg + (long)col0 * ld);
    double* y = reinterpret_cast<double*>(dng + (long)col0 * ld);
    int rc = settle(false);  // its pinned staging is reused by this call
    if (rc) return rc;
    if (c->dav_apply) {
      const auto t0 = std::chrono::steady_clock::now();
      WB_CU(cudaStreamSynchronize(s));  // the hook runs on its own streams
      rc = c->dav_apply(c->dav_apply_user, col0, n, x, y, (int)ld, tr2);
      if (rc) return fail(rc, "Davidson operator hook failed (code " + std::to_string(rc) + ")");
      apply_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } else {
      for (cudaEvent_t& e : c->dav_ev)
        if (!e) WB_CU(cudaEventCreate(&e));
      WB_CU(cudaEventRecord(c->dav_ev[0], s));
      bool deferred = false;
      if ((rc = apply_deferred(c, n, x, (int)ld, y, (int)ld, tr2, &deferred))) return rc;
      WB_CU(cudaEventRecord(c->dav_ev[1], s));
      pending = true;
    }
    ++apply_calls;
    applied += n;
    return WB_OK;
  }
  int build_hr(int col0, int col1, int g_e) {  // hr(0:g_e, col0:col1) = <dvg|dng>
    const int ncol = col1 - col0, K = 2 * npw;
    const double* W = reinterpret_cast<const double*>(dvg);
    const double* X = reinterpret_cast<const double*>(dng + (long)col0 * ld);
    gemm_tn(W, 2 * ld, g_e, X, 2 * ld, nullptr, ncol, K, nsplit, part, s);
    k_braket_to_hr<<<ncol, 256, 0, s>>>(part, nsplit, g_e, ncol, W, 2 * ld, X, 2 * ld, hr, nvecx, col0);
    WB_CU(cudaGetLastError());
    return WB_OK;
  }
  double* bj = nullptr;  // block Jacobi scratch (bases above kJacobiSmemN)
  int* st = nullptr;     // device state (dav_ev_offset layout)
  double* ev = nullptr;
  unsigned char* host = nullptr;  // its pinned copy
  double trev = 0.0, trev_rel = 0.0;
  // Steps before the operator (davidson_diago.f90:273-306): move the
  // unconverged Ritz pairs behind the basis, update_with_vr_distr, do_mgs.
  int pre(int nbase, int notcnv) {
    const std::vector<long long> key = {0, nbase, notcnv, nvec, nvecx, ld, nsplit, key_ptr(dvg), key_ptr(dng),
                                        key_ptr(vr), key_ptr(w), key_ptr(coef), key_ptr(part), key_ptr(dots),
                                        key_ptr(st)};
    return dav_graph(c, s, key, [&]() -> int {
      k_dav_shift<<<notcnv, 256, 0, s>>>(st, ev, nvec, nbase, vr, nvecx, nvecx, w);
      const int K = 2 * npw;
      double* c1 = coef;
      double* c2 = coef + (size_t)nvecx * nvecx;
      k_vr_coef<<<notcnv, 256, 0, s>>>(vr, nvecx, nbase, nbase, notcnv, w, c1, c2);
      double* y = reinterpret_cast<double*>(dvg + (long)nbase * ld);
      gemm_nn(reinterpret_cast<const double*>(dvg), 2 * ld, nbase, c1, y, 2 * ld, nullptr, notcnv, K, 0.0, s);
      gemm_nn(reinterpret_cast<const double*>(dng), 2 * ld, nbase, c2, y, 2 * ld, nullptr, notcnv, K, 1.0, s);
      WB_CU(cudaGetLastError());
      return mgs(nbase, nbase + notcnv);
    });
  }
  // Steps after the operator (:331-347): build_hr of the new columns, diagox of
  // hr[:nbase + notcnv, :nbase + notcnv], the convergence test (test = 0: the
  // extra starting step, ev <- ew only) and the copy of the state to the host;
  // waits for it.
  int post(int nbase, int notcnv, int test) {
    const int n = nbase + notcnv;
    const std::vector<long long> key = {1, nbase, notcnv, test, nvec, nvecx, ld, nsplit, key_ptr(dvg), key_ptr(dng),
                                        key_ptr(hr), key_ptr(vr), key_ptr(A), key_ptr(V), key_ptr(w), key_ptr(part),
                                        key_ptr(bj), key_ptr(st), key_ptr(host), key_bits(trev), key_bits(trev_rel)};
    auto body = [&]() -> int {
      int rc = build_hr(nbase, n, n);
      if (rc) return rc;
      if ((rc = eigen_lowest(hr, nvecx, n, nvec, w, vr, nvecx, A, V, bj, sweeps, s, aux))) return rc;
      k_dav_conv<<<1, 256, 0, s>>>(w, ev, st, nvec, trev, trev_rel, test);
      WB_CU(cudaMemcpyAsync(host, st, dav_state_bytes(nvec), cudaMemcpyDeviceToHost, s));
      WB_CU(cudaGetLastError());
      return WB_OK;
    };
    const int rc = dav_graph(c, s, key, body);
    if (rc) return rc;
    WB_CU(wb_wait(c));
    return settle(true);
  }
  int unconverged() const { return reinterpret_cast<const int*>(host)[0]; }
  int conv_at(int i) const { return reinterpret_cast<const int*>(host)[1 + i]; }
  double ev_at(int i) const { return reinterpret_cast<const double*>(host + dav_ev_offset(nvec))[i]; }
  // host conv/ev -> device state (start and resumption)
  int upload(const std::vector<int>& conv_h, const std::vector<double>& ev_h) {
    int* hi = reinterpret_cast<int*>(host);
    int cnt = 0;
    for (int i = 0; i < nvec; ++i) { hi[1 + i] = conv_h[i]; cnt += conv_h[i] ? 0 : 1; }
    hi[0] = cnt;
    std::memcpy(host + dav_ev_offset(nvec), ev_h.data(), sizeof(double) * nvec);
    WB_CU(cudaMemcpyAsync(st, host, dav_state_bytes(nvec), cudaMemcpyHostToDevice, s));
    WB_CU(cudaStreamSynchronize(s));
    return WB_OK;
  }
  // out(:, 0:ncol) = basis(:, 0:nrow) vr(0:nrow, 0:ncol), via tmp
  int refresh(double2* basis, int nrow, int ncol) {
    const int K = 2 * npw;
    k_vr_coef<<<ncol, 256, 0, s>>>(vr, nvecx, nrow, 0, ncol, nullptr, nullptr, coef);
    gemm_nn(reinterpret_cast<const double*>(basis), 2 * ld, nrow, coef, reinterpret_cast<double*>(tmp), 2 * ld,
            nullptr, ncol, K, 0.0, s);
    WB_CU(cudaMemcpyAsync(basis, tmp, sizeof(double2) * ld * ncol, cudaMemcpyDeviceToDevice, s));
    WB_CU(cudaGetLastError());
    return WB_OK;
  }
};

}  // namespace

extern "C" int wb_davidson_set_apply(wb_ctx* c, wb_apply_fn fn, void* user) {
  if (!c) return fail(WB_ERR_ARG, "null context");
  c->dav_apply = fn;
  c->dav_apply_user = fn ? user : nullptr;
  return WB_OK;
}

extern "C" int wb_davidson(wb_ctx* c, const wb_davidson_params* p, const double* dvg0, int ld_dvg0, double* ev_out,
                           int* conv_out, double* pdep, int ld_pdep, wb_davidson_info* info) {
  if (!c || !p || !ev_out || (!dvg0 && !p->restart)) return fail(WB_ERR_ARG, "null argument");
  if ((p->n_steps_write_restart > 0 || p->restart) && !p->restart_dir)
    return fail(WB_ERR_ARG, "restart files need restart_dir");
  if (p->n_steps_write_restart < 0) return fail(WB_ERR_ARG, "n_steps_write_restart < 0");
  const int nvec = p->n_pdep_eigen, nvecx = p->n_pdep_basis;
  if (nvec < 1 || nvecx < 2 * nvec)
    return fail(WB_ERR_ARG, "need n_pdep_eigen >= 1 and n_pdep_basis >= 2 n_pdep_eigen (davidson_diago.f90:107)");
  if (nvecx > kMaxBasis)
    return fail(WB_ERR_UNSUPPORTED, "n_pdep_basis > " + std::to_string(kMaxBasis) + " is not provided");
  if (p->n_pdep_maxiter < 1) return fail(WB_ERR_ARG, "n_pdep_maxiter < 1");
  if ((dvg0 && ld_dvg0 < c->npw) || (pdep && ld_pdep < c->npw))
    return fail(WB_ERR_ARG, "leading dimension smaller than npw");
  const auto t0 = std::chrono::steady_clock::now();
  WB_CU(cudaSetDevice(c->device));
  jacobi_setup();
  WB_CU(cudaGetLastError());
  Dav d;
  d.c = c;
  d.npw = c->npw;
  d.ld = c->npw;
  d.nvec = nvec;
  d.nvecx = nvecx;
  d.s = c->stream;
  if (nvecx > kJacobiSmemN && c->use_graphs && !c->dav_aux)
    WB_CU(cudaStreamCreateWithFlags(&c->dav_aux, cudaStreamNonBlocking));
  d.aux = c->dav_aux;
  d.nsplit = gemm_tn_splits(nvecx, nvecx, 2 * c->npw);
  const size_t colb = sizeof(double2) * d.ld;
  if (c->dav_dvg.ensure(colb * nvecx) || c->dav_dng.ensure(colb * nvecx) || c->dav_tmp.ensure(colb * nvecx) ||
      c->dav_hr.ensure(sizeof(double) * nvecx * nvecx) || c->dav_vr.ensure(sizeof(double) * nvecx * nvecx) ||
      c->dav_A.ensure(sizeof(double) * nvecx * nvecx) || c->dav_V.ensure(sizeof(double) * nvecx * nvecx) ||
      c->dav_w.ensure(sizeof(double) * nvecx + 64) ||
      c->dav_part.ensure(sizeof(double) * (size_t)d.nsplit * nvecx * nvecx) ||
      c->dav_coef.ensure(sizeof(double) * 2 * nvecx * nvecx) || c->dav_dots.ensure(sizeof(double) * (nvecx + 1)) ||
      (nvecx > kJacobiSmemN && c->dav_bj.ensure(sizeof(double) * bj_doubles(nvecx))))
    return fail(WB_ERR_NOMEM, "device allocation of the Davidson basis failed");
  d.bj = c->dav_bj.as<double>();
  d.dvg = c->dav_dvg.as<double2>();
  d.dng = c->dav_dng.as<double2>();
  d.tmp = c->dav_tmp.as<double2>();
  d.hr = c->dav_hr.as<double>();
  d.vr = c->dav_vr.as<double>();
  d.A = c->dav_A.as<double>();
  d.V = c->dav_V.as<double>();
  d.w = c->dav_w.as<double>();
  d.sweeps = reinterpret_cast<int*>(d.w + nvecx);
  d.part = c->dav_part.as<double>();
  d.coef = c->dav_coef.as<double>();
  d.dots = c->dav_dots.as<double>();
  const size_t stb = dav_state_bytes(nvec);
  if (c->dav_st.ensure(stb)) return fail(WB_ERR_NOMEM, "device allocation of the Davidson state failed");
  if (c->dav_host_bytes < stb) {
    if (c->dav_host) cudaFreeHost(c->dav_host);
    c->dav_host = nullptr;
    c->dav_host_bytes = 0;
    if (cudaMallocHost(&c->dav_host, stb) != cudaSuccess) {
      cudaGetLastError();
      return fail(WB_ERR_NOMEM, "pinned host allocation of the Davidson state failed");
    }
    c->dav_host_bytes = stb;
  }
  d.st = c->dav_st.as<int>();
  d.ev = reinterpret_cast<double*>(c->dav_st.as<unsigned char>() + dav_ev_offset(nvec));
  d.host = static_cast<unsigned char*>(c->dav_host);
  d.trev = p->trev_pdep;
  d.trev_rel = p->trev_pdep_rel;
  cudaStream_t s = d.s;
  WB_CU(cudaMemsetAsync(d.dvg, 0, colb * nvecx, s));
  WB_CU(cudaMemsetAsync(d.dng, 0, colb * nvecx, s));
  WB_CU(cudaMemsetAsync(d.hr, 0, sizeof(double) * nvecx * nvecx, s));
  WB_CU(cudaMemsetAsync(d.vr, 0, sizeof(double) * nvecx * nvecx, s));
  std::vector<double> ew(nvecx, 0.0), ev(nvec, 0.0);
  std::vector<int> conv(nvec, 0);
  int nbase = nvec, notcnv = nvec, rc;
  int dav_iter = -2;
  // restart files (davidson_restart.f90): the state at the end of a step, the
  // basis columns [0, nbase) and hr/vr copied to the host
  auto checkpoint = [&]() -> int {
    DavRestart r;
    r.dav_iter = dav_iter;
    r.notcnv = notcnv;
    r.nbase = nbase;
    r.conv = conv;
    r.ev = ev;
    r.ew = ew;
    r.hr.resize((size_t)nvecx * nvecx);
    r.vr.resize((size_t)nvecx * nvecx);
    std::vector<double> hv((size_t)2 * d.ld * nbase), hn((size_t)2 * d.ld * nbase);
    WB_CU(cudaMemcpyAsync(hv.data(), d.dvg, colb * nbase, cudaMemcpyDeviceToHost, s));
    WB_CU(cudaMemcpyAsync(hn.data(), d.dng, colb * nbase, cudaMemcpyDeviceToHost, s));
    WB_CU(cudaMemcpyAsync(r.hr.data(), d.hr, sizeof(double) * r.hr.size(), cudaMemcpyDeviceToHost, s));
    WB_CU(cudaMemcpyAsync(r.vr.data(), d.vr, sizeof(double) * r.vr.size(), cudaMemcpyDeviceToHost, s));
    WB_CU(cudaStreamSynchronize(s));
    return dav_restart_write(p->restart_dir, r, nvec, nvecx, d.npw, hv.data(), hn.data(), d.ld);
  };
  const int nsw = p->n_steps_write_restart;
  if (p->restart) {                                                        // wstat_calculation 'R' (:154-159)
    DavRestart r;
    std::vector<double> hv((size_t)2 * d.ld * nvecx), hn((size_t)2 * d.ld * nvecx);
    if ((rc = dav_restart_read(p->restart_dir, r, nvec, nvecx, d.npw, hv.data(), hn.data(), d.ld))) return rc;
    WB_CU(cudaMemcpyAsync(d.dvg, hv.data(), colb * r.nbase, cudaMemcpyHostToDevice, s));
    WB_CU(cudaMemcpyAsync(d.dng, hn.data(), colb * r.nbase, cudaMemcpyHostToDevice, s));
    WB_CU(cudaMemcpyAsync(d.hr, r.hr.data(), sizeof(double) * r.hr.size(), cudaMemcpyHostToDevice, s));
    WB_CU(cudaMemcpyAsync(d.vr, r.vr.data(), sizeof(double) * r.vr.size(), cudaMemcpyHostToDevice, s));
    WB_CU(cudaStreamSynchronize(s));
    dav_iter = r.dav_iter;
    nbase = r.nbase;
    notcnv = r.notcnv;
    conv = r.conv;
    ev = r.ev;
    ew = r.ew;
  } else {                                                                 // from scratch (:161-199)
    WB_CU(cudaMemcpy2DAsync(d.dvg, colb, dvg0, sizeof(double2) * ld_dvg0, colb, nvec, cudaMemcpyHostToDevice, s));
    if ((rc = d.mgs(0, nvec))) return rc;
    if ((rc = d.apply(0, nvec, -1.0))) return rc;                          // lite solver
    dav_iter = -1;
    if (nsw == 1 && (rc = checkpoint())) return rc;
  }
  if ((rc = d.upload(conv, ev))) return rc;
  if (dav_iter == -1) {                                                    // extra starting step (:204-247)
    WB_CU(cudaMemcpyAsync(d.dvg, d.dng, colb * nvecx, cudaMemcpyDeviceToDevice, s));   // dvg = dng
    if ((rc = d.mgs(0, nvec))) return rc;
    if ((rc = d.apply(0, nvec, std::min(1e-4, 1e8 * p->tr2_dfpt)))) return rc;
    if ((rc = d.post(0, nvec, 0))) return rc;                              // build_hr, diagox, ev = ew
    for (int i = 0; i < nvec; ++i) ew[i] = ev[i] = d.ev_at(i);
    dav_iter = 0;
    if (nsw == 1 && (rc = checkpoint())) return rc;
  }
  bool refreshed = false;
  for (int kter = 1; kter <= p->n_pdep_maxiter; ++kter) {                 // :259
    ++dav_iter;
    for (int n = 0, np_ = 0; n < nvec; ++n)                               // :273-296, host copy of ew
      if (!conv[n]) ew[nbase + np_++] = ev[n];
    if ((rc = d.pre(nbase, notcnv))) return rc;                           // :273-306 on the device
    if ((rc = d.apply(nbase, notcnv, p->tr2_dfpt))) return rc;             // :324
    if ((rc = d.post(nbase, notcnv, 1))) return rc;                        // :331-347
    nbase += notcnv;
    notcnv = d.unconverged();
    for (int i = 0; i < nvec; ++i) {
      conv[i] = d.conv_at(i);
      ev[i] = ew[i] = d.ev_at(i);
    }
    if (notcnv == 0 || nbase + notcnv > nvecx || kter == p->n_pdep_maxiter) {
      if (notcnv == 0 || kter == p->n_pdep_maxiter) {
        if ((rc = d.refresh(d.dvg, nbase, nvec))) return rc;              // eigenvectors for the caller
        refreshed = true;
        if (notcnv == 0 && p->restart_dir && (nsw > 0 || p->restart))
          dav_restart_clear(p->restart_dir, nvecx);                       // :376
        break;
      }
      if ((rc = d.refresh(d.dvg, nbase, nvec))) return rc;                // :397-398
      if ((rc = d.refresh(d.dng, nbase, nvec))) return rc;
      nbase = nvec;
      std::vector<double> eye((size_t)nvecx * nvecx, 0.0), hd((size_t)nvecx * nvecx, 0.0);
      for (int i = 0; i < nbase; ++i) { hd[(size_t)i * nvecx + i] = ev[i]; eye[(size_t)i * nvecx + i] = 1.0; }
      WB_CU(cudaMemcpyAsync(d.hr, hd.data(), sizeof(double) * hd.size(), cudaMemcpyHostToDevice, s));
      WB_CU(cudaMemcpyAsync(d.vr, eye.data(), sizeof(double) * eye.size(), cudaMemcpyHostToDevice, s));
      WB_CU(cudaStreamSynchronize(s));
    }
    if (nsw > 0 && dav_iter % nsw == 0 && (rc = checkpoint())) return rc;  // :421-422
  }
  if (!refreshed && (rc = d.refresh(d.dvg, nbase, nvec))) return rc;
  if (pdep)
    WB_CU(cudaMemcpy2DAsync(pdep, sizeof(double2) * ld_pdep, d.dvg, colb, colb, nvec, cudaMemcpyDeviceToHost, s));
  WB_CU(cudaStreamSynchronize(s));
  std::memcpy(ev_out, ev.data(), sizeof(double) * nvec);
  if (conv_out) for (int i = 0; i < nvec; ++i) conv_out[i] = conv[i];
  if (info) {
    info->dav_iter = dav_iter;
    info->notcnv = notcnv;
    info->converged = notcnv == 0 ? 1 : 0;
    info->apply_calls = d.apply_calls;
    info->perturbations = d.applied;
    info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    info->seconds_apply = d.apply_s;
  }
  return WB_OK;
}

extern "C" int wb_diagox(wb_ctx* c, int nbase, int nvec, const double* hr, int ldh, double* ew, double* vr, int ldv) {
  if (!c || !hr || !ew || !vr) return fail(WB_ERR_ARG, "null argument");
  if (nbase < 1 || nvec < 1 || nvec > nbase) return fail(WB_ERR_ARG, "need 1 <= nvec <= nbase");
  if (nbase > kMaxBasis) return fail(WB_ERR_UNSUPPORTED, "nbase > " + std::to_string(kMaxBasis) + " is not provided");
  if (ldh < nbase || ldv < nbase) return fail(WB_ERR_ARG, "leading dimension smaller than nbase");
  WB_CU(cudaSetDevice(c->device));
  jacobi_setup();
  WB_CU(cudaGetLastError());
  const size_t nn = (size_t)nbase * nbase;
  const void* before[] = {c->dav_A.p, c->dav_V.p, c->dav_w.p, c->dav_bj.p};
  if (c->dav_A.ensure(sizeof(double) * nn) || c->dav_V.ensure(sizeof(double) * nn) ||
      c->dav_w.ensure(sizeof(double) * nbase + 64) ||
      (nbase > kJacobiSmemN && c->dav_bj.ensure(sizeof(double) * bj_doubles(nbase))))
    return fail(WB_ERR_NOMEM, "device allocation of the eigensolver scratch failed");
  const void* after[] = {c->dav_A.p, c->dav_V.p, c->dav_w.p, c->dav_bj.p};
  if (!std::equal(std::begin(before), std::end(before), std::begin(after)))
    c->dav_graphs_release();  // the Davidson's cached graphs point into the old buffers
  double* w = c->dav_w.as<double>();
  int rc = eigen_lowest(hr, ldh, nbase, nvec, w, vr, ldv, c->dav_A.as<double>(), c->dav_V.as<double>(),
                        c->dav_bj.as<double>(), reinterpret_cast<int*>(w + nbase), c->stream);
  if (rc) return rc;
  WB_CU(cudaMemcpyAsync(ew, w, sizeof(double) * nvec, cudaMemcpyDeviceToHost, c->stream));
  WB_CU(cudaStreamSynchronize(c->stream));
  return WB_OK;
}
