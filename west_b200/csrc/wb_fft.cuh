// Shared-memory / register FFT engine for the stick-and-plane 3D FFTs.
//
// A length-N line transform is split N = N1 * N2 (four-step):
//   step 1: N2 threads per line, each does an N1-point DFT in registers over
//           elements N2*n1 + n2, multiplies by W_N^(n2*k1) and writes back to
//           the same positions (thread-private, no barrier needed);
//   step 2: N1 threads per line, each reads N2 consecutive results, does an
//           N2-point DFT in registers and writes element k1 + N1*k2 (natural
//           order).  Reads and writes of one line overlap, so a barrier
//           separates them.
// The small DFTs (2, 3, 4, 5 and composites up to 16) are fully unrolled
// register code.  Twiddles come from a 2N-entry table in shared memory
// (computed on the host): entries [0, N) are W_N^j = exp(+2 pi i j / N) in
// natural order, entries [N, 2N) hold the step-1 factors W_N^(n2 k1) at
// N + k1 N2 + n2, so the lanes of one step read consecutive entries instead of
// entries k1 apart (a bank conflict).  DIR = +1 is QE's invfft sign, DIR = -1
// the fwfft sign.  No normalisation is applied here.
#pragma once
#include "wb_common.cuh"

namespace wb {

template <int N> struct FftSplit;
template <> struct FftSplit<16> { static constexpr int N1 = 4, N2 = 4; };
template <> struct FftSplit<20> { static constexpr int N1 = 4, N2 = 5; };
template <> struct FftSplit<24> { static constexpr int N1 = 4, N2 = 6; };
template <> struct FftSplit<32> { static constexpr int N1 = 8, N2 = 4; };
template <> struct FftSplit<36> { static constexpr int N1 = 4, N2 = 9; };
template <> struct FftSplit<40> { static constexpr int N1 = 8, N2 = 5; };
template <> struct FftSplit<48> { static constexpr int N1 = 8, N2 = 6; };
template <> struct FftSplit<60> { static constexpr int N1 = 12, N2 = 5; };
template <> struct FftSplit<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct FftSplit<72> { static constexpr int N1 = 8, N2 = 9; };
template <> struct FftSplit<80> { static constexpr int N1 = 8, N2 = 10; };
template <> struct FftSplit<96> { static constexpr int N1 = 8, N2 = 12; };
template <> struct FftSplit<100> { static constexpr int N1 = 10, N2 = 10; };
template <> struct FftSplit<108> { static constexpr int N1 = 12, N2 = 9; };
template <> struct FftSplit<120> { static constexpr int N1 = 12, N2 = 10; };

// Literal constants of the radix-3 and radix-5 butterflies.
constexpr double kS3 = 0.86602540378443864676;   // sin(2 pi / 3)
constexpr double kC51 = 0.30901699437494742410;  // cos(2 pi / 5)
constexpr double kC52 = -0.80901699437494742410; // cos(4 pi / 5)
constexpr double kS51 = 0.95105651629515357212;  // sin(2 pi / 5)
constexpr double kS52 = 0.58778525229247312917;  // sin(4 pi / 5)
// cos and sin of 2 pi k / 7, k = 1, 2, 3 (the radix-7 butterfly of the runtime-size path)
constexpr double kC71 = 0.62348980185873353053, kC72 = -0.22252093395631440429, kC73 = -0.90096886790241912624;
constexpr double kS71 = 0.78183148246802980871, kS72 = 0.97492791218182360702, kS73 = 0.43388373911755812048;

template <int R> struct Factor2;  // composite radices R = A * B
template <> struct Factor2<6> { static constexpr int A = 3, B = 2; };
template <> struct Factor2<8> { static constexpr int A = 4, B = 2; };
template <> struct Factor2<9> { static constexpr int A = 3, B = 3; };
template <> struct Factor2<10> { static constexpr int A = 5, B = 2; };
template <> struct Factor2<12> { static constexpr int A = 4, B = 3; };
template <> struct Factor2<16> { static constexpr int A = 4, B = 4; };

constexpr double kR2 = 0.70710678118654752440;   // sqrt(1/2)

// a * exp(DIR 2 pi i j / 8) for j = 1, 2, 3 (the inner twiddles of the radix-8
// DFT), from the exact forms (1 + i)/sqrt(2), i, (-1 + i)/sqrt(2)
template <int DIR, class C>
WB_DEV C tw8(C a, int j) {
  using T = real_t<C>;
  const T c = T(kR2);
  if (j == 2) return cmul_i<DIR>(a);
  const T s = a.x + a.y, d = a.x - a.y;
  if (j == 1) return DIR > 0 ? mkc<C>(c * d, c * s) : mkc<C>(c * s, -c * d);
  return DIR > 0 ? mkc<C>(-c * s, c * d) : mkc<C>(-c * d, -c * s);
}

// In-register DFT of size R: v[k] <- sum_n v[n] exp(DIR 2 pi i n k / R).
// NT is the length of the shared twiddle table twN (R divides NT).  C is
// double2 or float2.
template <int R, int DIR, int NT, class C>
WB_DEV void rdft(C* v, const C* twN) {
  using T = real_t<C>;
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 3) {
    C t1 = cadd(v[1], v[2]);
    C t2 = mkc<C>(v[0].x - T(0.5) * t1.x, v[0].y - T(0.5) * t1.y);
    C d = csub(v[1], v[2]);
    C t3 = cmul_i<DIR>(mkc<C>(T(kS3) * d.x, T(kS3) * d.y));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  } else if constexpr (R == 4) {
    C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    C c = cadd(v[1], v[3]), d = cmul_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  } else if constexpr (R == 5) {
    const T c51 = T(kC51), c52 = T(kC52), s51 = T(kS51), s52 = T(kS52);
    C x0 = v[0];
    C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    C a1 = mkc<C>(x0.x + c51 * t1.x + c52 * t2.x, x0.y + c51 * t1.y + c52 * t2.y);
    C a2 = mkc<C>(x0.x + c52 * t1.x + c51 * t2.x, x0.y + c52 * t1.y + c51 * t2.y);
    C b1 = cmul_i<DIR>(mkc<C>(s51 * t3.x + s52 * t4.x, s51 * t3.y + s52 * t4.y));
    C b2 = cmul_i<DIR>(mkc<C>(s52 * t3.x - s51 * t4.x, s52 * t3.y - s51 * t4.y));
    v[0] = cadd(x0, cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  } else if constexpr (R == 7) {
    // X_k = x0 + sum_{n=1..3} cos(2 pi n k / 7) t_n + i DIR sin(2 pi n k / 7) d_n,
    // t_n = x_n + x_{7-n}, d_n = x_n - x_{7-n}; X_{7-k} takes the opposite sine term
    const T c1 = T(kC71), c2 = T(kC72), c3 = T(kC73), s1 = T(kS71), s2 = T(kS72), s3 = T(kS73);
    const C x0 = v[0];
    const C t1 = cadd(v[1], v[6]), t2 = cadd(v[2], v[5]), t3 = cadd(v[3], v[4]);
    const C d1 = csub(v[1], v[6]), d2 = csub(v[2], v[5]), d3 = csub(v[3], v[4]);
    auto lin = [](C a, C b, C c, T ka, T kb, T kc) {
      return mkc<C>(ka * a.x + kb * b.x + kc * c.x, ka * a.y + kb * b.y + kc * c.y);
    };
    const C a1 = cadd(x0, lin(t1, t2, t3, c1, c2, c3)), b1 = cmul_i<DIR>(lin(d1, d2, d3, s1, s2, s3));
    const C a2 = cadd(x0, lin(t1, t2, t3, c2, c3, c1)), b2 = cmul_i<DIR>(lin(d1, d2, d3, s2, -s3, -s1));
    const C a3 = cadd(x0, lin(t1, t2, t3, c3, c1, c2)), b3 = cmul_i<DIR>(lin(d1, d2, d3, s3, -s1, s2));
    v[0] = cadd(x0, cadd(t1, cadd(t2, t3)));
    v[1] = cadd(a1, b1); v[6] = csub(a1, b1);
    v[2] = cadd(a2, b2); v[5] = csub(a2, b2);
    v[3] = cadd(a3, b3); v[4] = csub(a3, b3);
  } else {
    constexpr int A = Factor2<R>::A, B = Factor2<R>::B;
    C z[B][A];
#pragma unroll
    for (int b = 0; b < B; ++b) {
#pragma unroll
      for (int a = 0; a < A; ++a) z[b][a] = v[B * a + b];
      rdft<A, DIR, NT>(z[b], twN);
#pragma unroll
      for (int k1 = 1; k1 < A; ++k1)
        if (b > 0) {
          if constexpr (R == 8) z[b][k1] = tw8<DIR>(z[b][k1], k1);
          else z[b][k1] = ctw<DIR>(z[b][k1], twN[((b * k1) * (NT / R)) % NT]);
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      C t[B];
#pragma unroll
      for (int b = 0; b < B; ++b) t[b] = z[b][k1];
      rdft<B, DIR, NT>(t, twN);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
    }
  }
}

// Element layout of one line in shared memory.  Element e = N2*a + b is stored
// at (N2 + PAD)*a + b: with an odd block length, the N1 threads of step 2 (which
// read elements N2*k1 + n2) hit distinct banks, as do the N2 threads of step 1.
#define WB_HD __host__ __device__ __forceinline__
template <int N>
struct LinePad {
  static constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
  static constexpr int PAD = (N2 % 2 == 0) ? 1 : 0;
  static constexpr int LEN = N1 * (N2 + PAD);  // stored length of a line
  WB_HD static int off(int e) { return (e / N2) * (N2 + PAD) + (e % N2); }
  WB_HD static int off_blk(int a, int b) { return (N2 + PAD) * a + b; }
};

// Pruning for lines whose nonzero inputs (inverse) or needed outputs
// (forward) lie in [0, N/4) u [3N/4, N), as a wavefunction sphere does in a
// box sized for the density cutoff.  In step 1 element N2*n1 + n2 is live iff
// n1 is in the outer quarters (needs N1 % 4 == 0); in step 2 output
// k1 + N1*k2 is live iff k2 is in the outer quarters (needs N2 % 4 == 0).
// Dead inputs are compile-time zeros and dead outputs are never stored, so the
// compiler removes their arithmetic.
enum : int { PRUNE_NONE = 0, PRUNE_IN = 1, PRUNE_OUT = 2 };
template <int N>
struct Prune {
  static constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
  static constexpr bool IN_OK = (N1 % 4 == 0);
  static constexpr bool OUT_OK = (N2 % 4 == 0);
  WB_DEV static constexpr bool in_live(int n1) { return n1 < N1 / 4 || n1 >= N1 - N1 / 4; }
  WB_DEV static constexpr bool out_live(int k2) { return k2 < N2 / 4 || k2 >= N2 - N2 / 4; }
};

// Batched line FFTs in shared memory.  Line l starts at data + loff(l).
// Elements of a line are either padded-contiguous (PADDED, LinePad layout,
// element stride 1) or strided by es with no padding (columns of a plane,
// where consecutive threads take consecutive lines).  LINE_FAST puts
// consecutive threads on consecutive lines.  The two steps are separate so a
// kernel can fuse pointwise work between them; fft_lines runs both.  All
// functions must be called by all NT threads of the block.
template <int N, int DIR, int NT, bool LINE_FAST, bool PADDED, int PRUNE = PRUNE_NONE, class Off, class C>
WB_DEV void fft_step1(C* data, Off loff, int es, int nlines, const C* twN) {
  using LP = LinePad<N>;
  using PR = Prune<N>;
  constexpr bool PIN = (PRUNE == PRUNE_IN) && PR::IN_OK;
  constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
  const int tid = threadIdx.x;
  const int items1 = nlines * N2;
  for (int it = tid; it < items1; it += NT) {
    int line, n2;
    if (LINE_FAST) { line = it % nlines; n2 = it / nlines; }
    else { line = it / N2; n2 = it % N2; }
    C* p = data + loff(line);
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
      v[n1] = (PIN && !PR::in_live(n1)) ? mkc<C>(0, 0)
                                        : p[PADDED ? LP::off_blk(n1, n2) : (N2 * n1 + n2) * es];
    rdft<N1, DIR, N>(v, twN);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = ctw<DIR>(v[k1], twN[N + k1 * N2 + n2]);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) p[PADDED ? LP::off_blk(k1, n2) : (N2 * k1 + n2) * es] = v[k1];
  }
}

template <int N, int DIR, int NT, bool LINE_FAST, bool PADDED, int PRUNE = PRUNE_NONE, class Off, class C>
WB_DEV void fft_step2(C* data, Off loff, int es, int nlines, const C* twN) {
  using LP = LinePad<N>;
  using PR = Prune<N>;
  constexpr bool POUT = (PRUNE == PRUNE_OUT) && PR::OUT_OK;
  constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
  const int tid = threadIdx.x;
  constexpr int LPC = NT / N1;
  const int nchunks = (nlines + LPC - 1) / LPC;
  for (int c = 0; c < nchunks; ++c) {
    int line, k1;
    if (LINE_FAST) { line = c * LPC + tid % LPC; k1 = tid / LPC; }
    else { line = c * LPC + tid / N1; k1 = tid % N1; }
    const bool act = (tid < LPC * N1) && (line < nlines);
    C v[N2];
    C* p = data + (act ? loff(line) : 0);
    if (act) {
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) v[n2] = p[PADDED ? LP::off_blk(k1, n2) : (N2 * k1 + n2) * es];
      rdft<N2, DIR, N>(v, twN);
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2)
        if (!POUT || PR::out_live(k2)) p[PADDED ? LP::off(k1 + N1 * k2) : (k1 + N1 * k2) * es] = v[k2];
    }
  }
  __syncthreads();
}

template <int N, int DIR, int NT, bool LINE_FAST, bool PADDED, int PRUNE = PRUNE_NONE, class Off, class C>
WB_DEV void fft_lines(C* data, Off loff, int es, int nlines, const C* twN) {
  fft_step1<N, DIR, NT, LINE_FAST, PADDED, PRUNE>(data, loff, es, nlines, twN);
  __syncthreads();
  fft_step2<N, DIR, NT, LINE_FAST, PADDED, PRUNE>(data, loff, es, nlines, twN);
}

struct OffLinear {
  int stride;
  WB_DEV int operator()(int l) const { return l * stride; }
};
// Active columns of a padded plane: x in [0, xhi] and [N - (ncols - nlow), N).
template <int N>
struct OffCols {
  int nlow, ncols;
  WB_DEV int operator()(int l) const { return LinePad<N>::off(l < nlow ? l : N - ncols + l); }
};

// Plane of N x N complex values: rows are padded lines (LinePad), row stride RS.
template <int N>
struct Plane {
  static constexpr int RS = LinePad<N>::LEN;
  static constexpr int SIZE = N * RS;
  WB_HD static int row(int y) { return y * RS; }
  WB_HD static int at(int x, int y) { return y * RS + LinePad<N>::off(x); }
  // plane offset of the e-th element in row-major (y*N + x) order
  WB_HD static int at_lin(int e) { return at(e % N, e / N); }
};

// Plane of the fused local-potential kernel.  For N = 8 x 8 with 8-byte
// elements (FP32 complex) every group of 8 rows is shifted by GP = 8 more
// elements.  A half-warp of 8-byte accesses covers 16 bank slots (offset mod
// 16); the row stride 72 puts rows y and y+1 eight slots apart, and the group
// shift does the same for rows y and y+8, so the column passes can give each
// half-warp one aligned block of 8 columns in two rows 1 or 8 apart without a
// conflict (16-byte elements are served per quarter-warp, one row, and need
// no shift).
template <int N, class C>
struct FPlane {
  static constexpr int R = FftSplit<N>::N1;
  static constexpr int RS = LinePad<N>::LEN;
  static constexpr int GP = (sizeof(C) == 8 && R == 8 && FftSplit<N>::N2 == 8) ? 8 : 0;
  static constexpr int GS = R * RS + GP;  // stride between groups of R rows
  static constexpr int SIZE = N * RS + (N / R) * GP;
  // row y = R * a + b with b in [0, R)
  WB_HD static int row2(int a, int b) { return a * GS + b * RS; }
  WB_HD static int row(int y) { return row2(y / R, y % R); }
  WB_HD static int at(int x, int y) { return row(y) + LinePad<N>::off(x); }
  WB_HD static int at_lin(int e) { return at(e % N, e / N); }
};

}  // namespace wb
