// Internal interfaces between the west_b200 host code and its kernels.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace wb {

// Stick decomposition of the Gamma half sphere (built on the host from nl).
struct StickTab {
  int nsp;               // stick pairs; pair 0 is the (0,0) stick
  int nst;               // sticks in the buffer = 2 * nsp (stick 1 is a dummy)
  const int* sp_gstart;  // [nsp + 1] first internal G index of each pair
  const int2* g_qz;      // [npw] (2 * pair + side, signed z) of each internal G
  const int* st_pos;     // [nst] plane offset y*N + x of each stick, -1 = dummy
  int xhi;               // active plane columns: x in [0, xhi] and [N - (ncols - xhi - 1), N)
  int ncols;
  int prune;             // 1 if every |Miller index| < N/4 (sphere inside the outer quarters)
};

// Runtime-size transforms (boxes without a compiled edge: non-cubic boxes and
// the other 2, 3, 5, 7-smooth edges).  A line of length n is transformed in
// place by radix stages r[0..ns) (each 2, 3, 4, 5, 7 or 8): the inverse as
// decimation in frequency (natural input, output at digit-reversed positions),
// the forward as decimation in time over the same stages in reverse order
// (digit-reversed input, natural output).  Real-space data therefore sit at
// digit-reversed positions in every direction; they are only ever multiplied
// point by point, with V(r) stored in the same permuted layout.
constexpr int kRtMaxStages = 16;
struct RtPlan {
  int n, ns;
  int r[kRtMaxStages];
};
struct RtGeo {
  int nx, ny, nz;            // box edges, x fastest
  RtPlan px, py, pz;
  int ncols;                 // active x columns of a plane (the sticks' x values)
  int cs;                    // column stride of the shared-memory half plane (>= ny, odd)
  const int* colx;           // [ncols] box x index of active column c
  const int* spos;           // [nst] half-plane offset c * cs + (y mod ny) of each stick, -1 = dummy
  const double2 *twx, *twy, *twz;  // exp(+2 pi i j / n) per direction
  const float2 *twx32, *twy32, *twz32;
};
// radix stages of n (empty if n has a prime factor above 7)
RtPlan rt_plan(int n);
// box index in a direction of the value stored at position p by the inverse
int rt_digit_reverse(const RtPlan& pl, int p);
// shared memory of the runtime plane kernels for the given geometry and element size
size_t rt_plane_smem(const RtGeo& g, int elem_bytes, int* rows_per_chunk);

// Launches that take a device count (dcount != nullptr, CUDA-graph replays)
// size their grid for the host count as a maximum and read the number of
// systems from *dcount; items are pairs of systems.
struct FftArgs {
  int n;                 // box edge (0 when the runtime-size path runs)
  StickTab st;
  const double2* tw;     // [n] exp(+2 pi i j / n)
  cudaStream_t stream;
  const int* dcount = nullptr;
  int unfused = 0;       // 1: the two-pass plane kernel even where the fused one applies
  const RtGeo* rt = nullptr;  // runtime-size path when set
};

// FP32 twin of FftArgs for the mixed-precision inner solves.
struct FftArgs32 {
  int n;
  StickTab st;
  const float2* tw;
  cudaStream_t stream;
  const int* dcount = nullptr;
  int unfused = 0;
  const RtGeo* rt = nullptr;
};

// runtime-size counterparts of the fft_* entry points below (f.rt set)
void rt_zinv(const FftArgs& f, const double2* src, long ld, const int2* items, int nitems, double2* sticks);
void rt_zinv32(const FftArgs32& f, const float2* src, long ld, const int2* items, int nitems, float2* sticks);
void rt_zfwd_store(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dst, long ld);
void rt_zfwd_hpsi(const FftArgs& f, const double2* sticks, const int2* items, int nitems, const double2* P,
                  double2* T, long ld, const double* g2kin, const double* ecol);
void rt_zfwd_hpsi32(const FftArgs32& f, const float2* sticks, const int2* items, int nitems, const float2* P,
                    float2* T, long ld, const float* g2kin, const float* ecol);
void rt_zfwd_dng(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dng, long ld,
                 const int* perm, const double* sqvc);
void rt_plane_vloc(const FftArgs& f, double2* sticks, int nitems, const double* vs);
void rt_plane_vloc32(const FftArgs32& f, float2* sticks, int nitems, const float* vs);
void rt_plane_inv_box(const FftArgs& f, const double2* sticks, int nitems, double2* box);
void rt_plane_rhs(const FftArgs& f, const double2* evcr, const double2* dvbox, int npv, int mb, double2* sticks);
void rt_plane_drho(const FftArgs& f, const double2* dsticks, const double2* evcr, const double* occ, int nocc,
                   int mb, double2* acc, double scale, double2* osticks);
void rt_setup(const RtGeo& g);

bool fft_supported(int n);
// the fused one-pass plane kernel applies to this box and stick table
bool fft_fusable(int n, const StickTab& st);
// offset of plane element (x, y) in the shared-memory plane of the x-y pass
// kernels: the fused local-potential layout (fused) or the padded-row one,
// for elem_bytes 8 (FP32 complex) or 16 (FP64 complex)
int fft_plane_offset(int n, bool fused, int elem_bytes, int x, int y);

// Davidson restart hand-off in WEST's layout (Wstat/davidson_restart.f90):
// <dir>/summary.json (dav_iter, notcnv, nbase, conv, ev, ew), <dir>/hr_vr.dat
// (Fortran unformatted: hr then vr, n_pdep_basis^2 doubles each) and the basis
// <dir>/V<j>.dat, N<j>.dat (j = 000001.., pdep file format) for j <= nbase.
// dvg/dng are host arrays [ld, nbase] complex in WEST's G order.
struct DavRestart {
  int dav_iter = 0, notcnv = 0, nbase = 0;
  std::vector<int> conv;
  std::vector<double> ev, ew, hr, vr;
};
int dav_restart_write(const char* dir, const DavRestart& r, int nvec, int nvecx, int npw, const double* dvg,
                      const double* dng, long ld);
int dav_restart_read(const char* dir, DavRestart& r, int nvec, int nvecx, int npw, double* dvg, double* dng,
                     long ld);
void dav_restart_clear(const char* dir, int nvecx);
void fft_zinv32(const FftArgs32& f, const float2* src, long ld, const int2* items, int nitems, float2* sticks);
void fft_plane_vloc32(const FftArgs32& f, float2* sticks, int nitems, const float* vs);
void fft_zfwd_hpsi32(const FftArgs32& f, const float2* sticks, const int2* items, int nitems, const float2* P,
                     float2* T, long ld, const float* g2kin, const float* ecol);
void fft_setup(int n);
void fft_zinv(const FftArgs& f, const double2* src, long ld, const int2* items, int nitems, double2* sticks);
void fft_zfwd_store(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dst, long ld);
void fft_zfwd_hpsi(const FftArgs& f, const double2* sticks, const int2* items, int nitems, const double2* P,
                   double2* T, long ld, const double* g2kin, const double* ecol);
void fft_zfwd_dng(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dng, long ld,
                  const int* perm, const double* sqvc);
void fft_plane_vloc(const FftArgs& f, double2* sticks, int nitems, const double* vs);
void fft_plane_inv_box(const FftArgs& f, const double2* sticks, int nitems, double2* box);
void fft_plane_rhs(const FftArgs& f, const double2* evcr, const double2* dvbox, int npv, int mb, double2* sticks);
void fft_plane_drho(const FftArgs& f, const double2* dsticks, const double2* evcr, const double* occ, int nocc,
                    int mb, double2* acc, double scale, double2* osticks);

// ---- dense kernels (wb_la.cu) ----
// part[s][j][r] = sum_{k in split s} W[r*ldw + k] * X[col(j)*ldx + k]
// Split-K plans of the bra-ket GEMMs, host and device: a graph replay sizes its
// split grid for the largest plan and every CTA derives the plan of the device
// column count itself, so both paths split the same count the same way.
constexpr int kDmmaTile = 32;  // DMMA bra-ket CTA tile (rows and columns)
// split count of the DMMA bra-ket: about 2 * 148 * ctas_per_sm CTAs (4 warps each)
__host__ __device__ inline int gemm_tn_splits(int M, int ncol, int K, int ctas_per_sm = 2) {
  const int tiles = ((M + kDmmaTile - 1) / kDmmaTile) * ((ncol + kDmmaTile - 1) / kDmmaTile);
  int ns = (2 * 148 * ctas_per_sm + tiles - 1) / (tiles > 0 ? tiles : 1);
  const int maxs = (K + 511) / 512;
  if (ns > maxs) ns = maxs;
  if (ns < 1) ns = 1;
  return ns;
}
// part doubles for any column count up to nsys and any target up to ctas_max
size_t gemm_tn_part_doubles(int M, int nsys, int K, int ctas_max);
// with dn, ctas selects the device plan (nsplit is then ignored); prefetch: k
// steps between an operand load and its MMAs (1 or 2)
void gemm_tn(const double* W, long ldw, int M, const double* X, long ldx, const int* cols, int ncol, int K,
             int nsplit, double* part, cudaStream_t s, const int* dn = nullptr, int ctas = 2, int prefetch = 1);
// S = 2 sum_s part - W0 X0 (Gamma bra-ket, glbrak.f90:39-40), then
// C[j][r] = sum_{r'<nkb} D[r][r'] S[j][r'] for r < nkb, alpha S[j][r] otherwise
void gamma_reduce(const double* part, int nsplit, int M, int ncol, const double* W, long ldw, const double* X,
                  long ldx, const int* cols, const double* D, int nkb, double alpha, double* C, cudaStream_t s,
                  const int* dn = nullptr, int K = 0, int ctas = 0);
// Y[col(j)] = beta Y[col(j)] + W C[j]  over K real rows
void gemm_nn(const double* W, long ldw, int M, const double* C, double* Y, long ldy, const int* cols, int ncol,
             int K, double beta, cudaStream_t s, const int* dn = nullptr);

void permute_scale(const double2* dvg, long ld_in, const int* perm, const double* sqvc, int npw, int m,
                   double2* aux, long ld_out, cudaStream_t s);
// iprec[v][i] = 1 / max(1, g2kin[i] / eprec[v])
void make_iprec(const double* g2kin, const double* eprec, int npw, int nocc, double* iprec, cudaStream_t s);
// column j uses band j % nocc
void precondition(const double2* f, double2* pf, const double* iprec, int nocc, int npw, int ncol, long ld,
                  cudaStream_t s);
void sub_into(const double2* a, const double2* b, double2* out, int npw, int ncol, long ld, cudaStream_t s);
void kinetic_hpsi(const double2* P, double2* T, const double* g2kin, const double* ecol, const int* cols, int ncol,
                  int npw, long ld, cudaStream_t s, const int* dn = nullptr);
void set_eprec(const double2* evc, const double* g2kin, int npw, int nocc, double* eprec, cudaStream_t s);
void fill_columns(const double* per_band, int nocc, int nsys, double* out, cudaStream_t s);
// Fractional occupations (dfpt_module.f90:363-393): from C[j][r] = <psi_r|dV psi_i>
// (j = p nocc + i, r < nocc) the coefficients fc[j][f] of the bands r = nfull + f:
// 0 for r <= i or |occ_i - occ_r| < 1e-3, else C (occ_i - occ_r) / occ_i / (e_i - e_r)
void frac_coefficients(const double* C, int nocc, int nsys, int nfull, const double* occ, const double* et,
                       double* fc, cudaStream_t s);
void cg_reset(unsigned char* conv, int nsys, cudaStream_t s);
void cg_prec_rho(const int* act, int nact, const double2* g, double2* P, const double* iprec, int nocc,
                 double* rho_prev, unsigned char* conv, int iter, double tr2, int npw, long ld, cudaStream_t s,
                 const int* dn = nullptr, const int* iter_dev = nullptr);
// nact_host may be null (no host copy); nsys_dev, if given, overrides nsys
void cg_compact(const unsigned char* conv, int nsys, int* act, int2* items, int* nact_dev, int* nact_host,
                cudaStream_t s, const int* nsys_dev = nullptr);
// One PCG step after the operator: the update of iteration `iter` and, unless
// iter == maxiter, the preconditioning / rho / convergence test / direction of
// iteration iter + 1 (the iteration comes from *iter_dev when given).
void cg_step(const int* act, int nact, double2* x, double2* g, double2* P, const double2* T, const double* iprec,
             int nocc, double* rho_prev, unsigned char* conv, int iter, int maxiter, double tr2, int npw, long ld,
             cudaStream_t s, const int* dn = nullptr, const int* iter_dev = nullptr);
void cg_step32(const int* act, int nact, float2* x, float2* g, float2* P, const float2* T, const double* iprec,
               int nocc, double* rho_prev, unsigned char* conv, int iter, int maxiter, double eta, const double* rel,
               double floor, int npw, long ld, cudaStream_t s, const int* dn = nullptr,
               const int* iter_dev = nullptr);
void count_unconverged(const unsigned char* conv, int nocc, int mb, int* out, cudaStream_t s);
// loop state of the graph-captured PCG loops: int st[8] (wb_la.cu)
void loop_init(int* st, int nsys, bool reset_totals, cudaStream_t s);
void loop_ctl(cudaGraphConditionalHandle h, const int* nact, int* st, int maxiter, bool inner, cudaStream_t s);
void loop_bucket(cudaGraphConditionalHandle h, const int* nact, int* st, int min_items, int nbuckets, cudaStream_t s);

// ---- mixed form: FP32 inner PCG and FP64 refinement (wb_la.cu) ----
// inner test: rho < max(eta * rel[j], floor)
void cg_prec_rho32(const int* act, int nact, const float2* g, float2* P, const double* iprec, int nocc,
                   double* rho_prev, unsigned char* conv, int iter, double eta, const double* rel, double floor,
                   int npw, long ld, cudaStream_t s, const int* dn = nullptr, const int* iter_dev = nullptr);
void refine_residual(const int* act, int nact, const double2* B, const double2* T, const double* iprec, int nocc,
                     double tr2, unsigned char* conv, double* rho0, float2* g32, float2* d32, int npw, long ld,
                     cudaStream_t s);
void refine_accumulate(const int* act, int nact, double2* X, const float2* d32, int npw, long ld, cudaStream_t s);
void kinetic_hpsi32(const float2* P, float2* T, const float* g2kin, const float* ecol, const int* cols, int ncol,
                    int npw, long ld, cudaStream_t s, const int* dn = nullptr);
void to_float(const double* a, float* b, long n, cudaStream_t s);
int gemm_tn_splits32(int M, int ncol, int K);
void gemm_tn32(const float* W, long ldw, int M, const float* X, long ldx, const int* cols, int ncol, int K, int nsplit,
               float* part, cudaStream_t s, const int* dn = nullptr);
void gamma_reduce32(const float* part, int nsplit, int M, int ncol, const float* W, long ldw, const float* X, long ldx,
                    const int* cols, const float* D, int nkb, float alpha, float* C, cudaStream_t s,
                    const int* dn = nullptr, int K = 0, int umma_ctas = 0);
void gemm_nn32_acc(const float* W, long ldw, int M, const float* C, float* Y, long ldy, const int* cols, int ncol, int K,
                   cudaStream_t s, const int* dn = nullptr);

// split-BF16x3 tcgen05 GEMMs of the FP32 inner solve (wb_umma.cu)
bool umma_supported(int M);
int umma_np(int M);
void umma_setup();
__host__ __device__ inline void umma_braket_plan(int ncol, int K, int* nsplit, int* kb_per_split,
                                                 int ctas_per_sm = 2) {
  const int nkb = (K + 63) / 64;
  int tiles = (ncol + 127) / 128;
  if (tiles < 1) tiles = 1;
  int target = (ctas_per_sm * 148 + tiles - 1) / tiles;
  if (target < 1) target = 1;
  int per = (nkb + target - 1) / target;
  if (per < 2) per = 2;
  if (per > nkb) per = nkb;
  *kb_per_split = per;
  *nsplit = (nkb + per - 1) / per;
}
// part floats for any batch up to nsys and any ctas_per_sm up to kUmmaMaxCtas
constexpr int kUmmaMaxCtas = 3;
size_t umma_part_floats(int M, int nsys, int K);
size_t umma_braket_bytes(int M, int K);
size_t umma_update_bytes(int M, int K);
void umma_presplit(const double* W, long ldw, int M, int K, void* braket_tiles, void* update_tiles, cudaStream_t s);
// part[s][j][r] = sum over split s of W[r][k] X[cols[j]][k]; returns the number of splits
int umma_braket(const void* tiles, int M, const float* X, long ldx, const int* cols, int ncol, int K, float* part,
                int* err, cudaStream_t s, const int* dn = nullptr, int ctas_per_sm = 2);
// Y[cols[j]][k] += sum_r W[r][k] C[j][r]
// nj: systems per CTA (64 or 128; 0 = by projector count)
void umma_update(const void* tiles, int M, const float* C, float* Y, long ldy, const int* cols, int ncol, int K,
                 int* err, cudaStream_t s, const int* dn = nullptr, int nj = 0);

}  // namespace wb
