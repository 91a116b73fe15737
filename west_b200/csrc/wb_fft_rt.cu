// Runtime-size stick-and-plane FFTs: the path for boxes without a compiled
// edge (non-cubic boxes, and the 2, 3, 5, 7-smooth edges outside the compiled
// list).  Same decomposition and Gamma pack/unpack as wb_fft_kernels.cu (z
// passes over stick pairs, one z-plane per CTA for the x-y passes, the
// caller's pointwise work between the inverse and the forward transforms),
// with line lengths, radix stages and twiddles taken at run time.
//
// A line is transformed in place, one radix stage at a time over the whole
// CTA: the inverse (QE invfft sign) by decimation in frequency, which leaves
// the result at digit-reversed positions, the forward by decimation in time
// over the same stages in reverse order, which takes digit-reversed input and
// returns natural order.  No permutation pass is ever run: real-space data
// live at digit-reversed positions in all three directions, they are only
// multiplied point by point with each other and with V(r), which the host
// stores in the same permuted layout.
//
// The x-y pass keeps only the plane's active columns (the x values of the
// sticks) in shared memory, column-major with an odd column stride; rows are
// transformed in chunks of full length through a row scratch area.
#include <algorithm>

#include "wb_fft.cuh"
#include "wb_internal.h"

namespace wb {

RtPlan rt_plan(int n) {
  RtPlan p{};
  p.n = n;
  p.ns = 0;
  int m = n;
  for (int r : {8, 4, 2, 3, 5, 7})
    while (m % r == 0 && p.ns < kRtMaxStages) {
      p.r[p.ns++] = r;
      m /= r;
    }
  if (m != 1 || n < 2) p.ns = 0;
  return p;
}

int rt_digit_reverse(const RtPlan& pl, int p) {
  int block = pl.n, mult = 1, k = 0, rem = p;
  for (int s = 0; s < pl.ns; ++s) {
    const int R = pl.r[s], m = block / R;
    k += (rem / m) * mult;
    rem %= m;
    mult *= R;
    block = m;
  }
  return k;
}

constexpr int kRtZsg = 8;      // stick pairs per z-pass CTA
constexpr int kRtZnt = 128;
constexpr int kRtPnt = 256;
constexpr int kRtMaxRows = 16; // rows per chunk of the row passes

size_t rt_plane_smem(const RtGeo& g, int elem_bytes, int* rows_per_chunk) {
  const size_t base = (size_t)elem_bytes * (g.nx + g.ny + (size_t)g.ncols * g.cs);
  const size_t cap = 227u * 1024u;
  if (base + (size_t)elem_bytes * g.nx > cap) return 0;
  int rc = (int)std::min<size_t>((cap - base) / ((size_t)elem_bytes * g.nx), (size_t)kRtMaxRows);
  rc = std::min(rc, g.ny);
  if (rows_per_chunk) *rows_per_chunk = rc;
  return base + (size_t)elem_bytes * rc * g.nx;
}

template <class C>
WB_DEV const C* rt_table(const double2* t64, const float2* t32) {
  if constexpr (sizeof(C) == 16) return reinterpret_cast<const C*>(t64);
  else return reinterpret_cast<const C*>(t32);
}

// One butterfly of radix R over legs base + q m (element stride es): DIF does
// the R-point DFT then the twiddles W_L^(q j), DIT the twiddles then the DFT;
// L = m R, W_L^(q j) = tw[q j ts] with ts = n / L (q j < L, so no wrap).
template <int R, int DIR, bool DIF, class C>
WB_DEV void rt_bfly(C* p, int es, int base, int m, int j, int ts, const C* tw) {
  C v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = p[(base + q * m) * es];
  if (!DIF && j) {
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = ctw<DIR>(v[q], tw[q * j * ts]);
  }
  rdft<R, DIR, 8>(v, tw);  // R <= 8: exact constants, no table
  if (DIF && j) {
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = ctw<DIR>(v[q], tw[q * j * ts]);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) p[(base + q * m) * es] = v[q];
}

// nlines lines (line l starts at data + loff(l), element stride es), all
// threads of the CTA; ends with a barrier
template <int DIR, bool DIF, class C, class Off>
WB_DEV void rt_lines(C* data, Off loff, int es, int nlines, const RtPlan& pl, const C* tw) {
  const int n = pl.n;
  int blk = DIF ? n : 1;
  for (int st = 0; st < pl.ns; ++st) {
    const int s = DIF ? st : pl.ns - 1 - st;
    const int R = pl.r[s];
    const int m = DIF ? blk / R : blk;
    const int ts = n / (m * R);
    const int nb = n / R;
    for (int it = threadIdx.x; it < nlines * nb; it += blockDim.x) {
      const int line = it / nb, b = it - line * nb;
      const int bi = b / m, j = b - bi * m;
      C* p = data + loff(line);
      const int base = bi * m * R + j;
      switch (R) {
        case 2: rt_bfly<2, DIR, DIF>(p, es, base, m, j, ts, tw); break;
        case 3: rt_bfly<3, DIR, DIF>(p, es, base, m, j, ts, tw); break;
        case 4: rt_bfly<4, DIR, DIF>(p, es, base, m, j, ts, tw); break;
        case 5: rt_bfly<5, DIR, DIF>(p, es, base, m, j, ts, tw); break;
        case 7: rt_bfly<7, DIR, DIF>(p, es, base, m, j, ts, tw); break;
        default: rt_bfly<8, DIR, DIF>(p, es, base, m, j, ts, tw); break;
      }
    }
    __syncthreads();
    blk = DIF ? m : m * R;
  }
}

struct RtOff {
  int stride;
  WB_DEV int operator()(int l) const { return l * stride; }
};

template <class C>
WB_DEV C* rt_smem() {
  extern __shared__ __align__(16) unsigned char smraw[];
  return reinterpret_cast<C*>(smraw);
}

// ---------------------------------------------------------------------------
// z passes
// ---------------------------------------------------------------------------
template <class C>
__global__ void __launch_bounds__(kRtZnt) k_zinv_rt(const C* __restrict__ src, long ld,
                                                    const int2* __restrict__ items, StickTab st, RtGeo g,
                                                    C* __restrict__ out, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  const int N = g.nz, LS = N | 1;
  C* tw = rt_smem<C>();
  C* zb = tw + N;
  const C* twg = rt_table<C>(g.twz, g.twz32);
  const int q0 = blockIdx.x * kRtZsg, item = blockIdx.y;
  const int nq = min(kRtZsg, st.nsp - q0);
  const int2 it = items[item];
  const C* a = src + (long)it.x * ld;
  const C* b = src + (long)(it.y >= 0 ? it.y : it.x) * ld;
  const bool two = it.y >= 0;
  const int g0 = st.sp_gstart[q0], g1 = st.sp_gstart[q0 + nq];
  for (int i = threadIdx.x; i < N; i += kRtZnt) tw[i] = twg[i];
  for (int i = threadIdx.x; i < 2 * kRtZsg * LS; i += kRtZnt) zb[i] = mkc<C>(0, 0);
  __syncthreads();
  for (int gi = g0 + threadIdx.x; gi < g1; gi += kRtZnt) {
    const int2 qz = st.g_qz[gi];
    const C a1 = a[gi], a2 = two ? b[gi] : mkc<C>(0, 0);
    const C pos = mkc<C>(a1.x - a2.y, a1.y + a2.x);  // a1 + i a2
    const C neg = mkc<C>(a1.x + a2.y, a2.x - a1.y);  // conj(a1 - i a2)
    const int z = qz.y;
    if (qz.x < 2) {  // the (0,0) stick is its own mirror
      if (z != 0) { zb[(z + N) % N] = pos; zb[(N - z) % N] = neg; }
      else zb[0] = neg;  // G = 0: the -G store wins, as in the reference loop
    } else {
      const int l = qz.x - 2 * q0;
      zb[l * LS + (z + N) % N] = pos;
      zb[(l ^ 1) * LS + (N - z) % N] = neg;
    }
  }
  __syncthreads();
  rt_lines<+1, true>(zb, RtOff{LS}, 1, 2 * nq, g.pz, tw);
  const int ns = 2 * nq;
  C* o = out + (long)item * N * st.nst + 2 * q0;
  for (int e = threadIdx.x; e < ns * N; e += kRtZnt) {
    const int s = e % ns, pz = e / ns;
    o[(long)pz * st.nst + s] = zb[s * LS + pz];
  }
}

template <class C, class Epi>
__global__ void __launch_bounds__(kRtZnt) k_zfwd_rt(const C* __restrict__ sticks, const int2* __restrict__ items,
                                                    StickTab st, RtGeo g, Epi epi, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  using T = real_t<C>;
  const int N = g.nz, LS = N | 1;
  C* tw = rt_smem<C>();
  C* zb = tw + N;
  const C* twg = rt_table<C>(g.twz, g.twz32);
  const int q0 = blockIdx.x * kRtZsg, item = blockIdx.y;
  const int nq = min(kRtZsg, st.nsp - q0);
  const int ns = 2 * nq;
  const C* s0 = sticks + (long)item * N * st.nst + 2 * q0;
  for (int i = threadIdx.x; i < N; i += kRtZnt) tw[i] = twg[i];
  for (int e = threadIdx.x; e < ns * N; e += kRtZnt) {
    const int s = e % ns, pz = e / ns;
    zb[s * LS + pz] = s0[(long)pz * st.nst + s];
  }
  __syncthreads();
  rt_lines<-1, false>(zb, RtOff{LS}, 1, ns, g.pz, tw);
  const int2 it = items[item];
  const int g0 = st.sp_gstart[q0], g1 = st.sp_gstart[q0 + nq];
  for (int gi = g0 + threadIdx.x; gi < g1; gi += kRtZnt) {
    const int2 qz = st.g_qz[gi];
    const typename Epi::Pre pr = epi.pre(gi, it);
    const int z = qz.y;
    C ap, am;
    if (qz.x < 2) {
      ap = zb[(z + N) % N];
      am = zb[(N - z) % N];
    } else {
      const int l = qz.x - 2 * q0;
      ap = zb[l * LS + (z + N) % N];
      am = zb[(l ^ 1) * LS + (N - z) % N];
    }
    const C fp = mkc<C>(T(0.5) * (ap.x + am.x), T(0.5) * (ap.y + am.y));
    const C fm = mkc<C>(T(0.5) * (ap.x - am.x), T(0.5) * (ap.y - am.y));
    epi(gi, it, pr, mkc<C>(fp.x, fm.y), mkc<C>(fp.y, -fm.x));
  }
}

// ---------------------------------------------------------------------------
// x-y passes: half plane H[c][y] (active columns, stride cs) + row scratch
// ---------------------------------------------------------------------------
template <class C>
struct RtPlane {
  C *twx, *twy, *H, *Rb;
  WB_DEV RtPlane(const RtGeo& g) {
    twx = rt_smem<C>();
    twy = twx + g.nx;
    H = twy + g.ny;
    Rb = H + (size_t)g.ncols * g.cs;
  }
  WB_DEV void load_tw(const RtGeo& g) const {
    const C* tx = rt_table<C>(g.twx, g.twx32);
    const C* ty = rt_table<C>(g.twy, g.twy32);
    for (int i = threadIdx.x; i < g.nx; i += blockDim.x) twx[i] = tx[i];
    for (int i = threadIdx.x; i < g.ny; i += blockDim.x) twy[i] = ty[i];
  }
  // sticks -> H (zero elsewhere), then the inverse column transforms
  WB_DEV void sticks_in(const RtGeo& g, const StickTab& st, const C* __restrict__ sz) const {
    for (int e = threadIdx.x; e < g.ncols * g.cs; e += blockDim.x) H[e] = mkc<C>(0, 0);
    __syncthreads();
    for (int s = threadIdx.x; s < st.nst; s += blockDim.x) {
      const int p = g.spos[s];
      if (p >= 0) H[p] = sz[s];
    }
    __syncthreads();
    rt_lines<+1, true>(H, RtOff{g.cs}, 1, g.ncols, g.py, twy);
  }
  // forward column transforms, then H -> sticks
  WB_DEV void sticks_out(const RtGeo& g, const StickTab& st, C* __restrict__ sz) const {
    rt_lines<-1, false>(H, RtOff{g.cs}, 1, g.ncols, g.py, twy);
    for (int s = threadIdx.x; s < st.nst; s += blockDim.x) {
      const int p = g.spos[s];
      sz[s] = p >= 0 ? H[p] : mkc<C>(0, 0);
    }
  }
  // rows [y0, y0 + nr) of H -> Rb (full rows, zero at inactive x), inverse row transforms
  WB_DEV void rows_in(const RtGeo& g, int y0, int nr) const {
    for (int e = threadIdx.x; e < nr * g.nx; e += blockDim.x) Rb[e] = mkc<C>(0, 0);
    __syncthreads();
    for (int e = threadIdx.x; e < nr * g.ncols; e += blockDim.x) {
      const int r = e / g.ncols, c = e - r * g.ncols;
      Rb[r * g.nx + __ldg(g.colx + c)] = H[c * g.cs + y0 + r];
    }
    __syncthreads();
    rt_lines<+1, true>(Rb, RtOff{g.nx}, 1, nr, g.px, twx);
  }
  // forward row transforms of Rb, active columns back into H rows [y0, y0 + nr)
  WB_DEV void rows_out(const RtGeo& g, int y0, int nr) const {
    rt_lines<-1, false>(Rb, RtOff{g.nx}, 1, nr, g.px, twx);
    for (int e = threadIdx.x; e < nr * g.ncols; e += blockDim.x) {
      const int r = e / g.ncols, c = e - r * g.ncols;
      H[c * g.cs + y0 + r] = Rb[r * g.nx + __ldg(g.colx + c)];
    }
    __syncthreads();
  }
};

// psi -> V(r) psi(r) -> back, in place on the sticks of plane pz of item
template <class C>
__global__ void __launch_bounds__(kRtPnt) k_plane_vloc_rt(C* __restrict__ sticks, StickTab st, RtGeo g,
                                                          const real_t<C>* __restrict__ vs, int rc, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  const RtPlane<C> P(g);
  const int pz = blockIdx.x, item = blockIdx.y;
  C* sz = sticks + ((long)item * g.nz + pz) * st.nst;
  P.load_tw(g);
  P.sticks_in(g, st, sz);
  const real_t<C>* vz = vs + (long)pz * g.nx * g.ny;
  for (int y0 = 0; y0 < g.ny; y0 += rc) {
    const int nr = min(rc, g.ny - y0);
    P.rows_in(g, y0, nr);
    for (int e = threadIdx.x; e < nr * g.nx; e += blockDim.x) P.Rb[e] = cscale(P.Rb[e], vz[(long)y0 * g.nx + e]);
    __syncthreads();
    P.rows_out(g, y0, nr);
  }
  P.sticks_out(g, st, sz);
}

// sticks -> real-space box (permuted layout), no scaling
__global__ void __launch_bounds__(kRtPnt) k_plane_inv_box_rt(const double2* __restrict__ sticks, StickTab st,
                                                             RtGeo g, double2* __restrict__ box, int rc) {
  const RtPlane<double2> P(g);
  const int pz = blockIdx.x, item = blockIdx.y;
  P.load_tw(g);
  P.sticks_in(g, st, sticks + ((long)item * g.nz + pz) * st.nst);
  double2* o = box + ((long)item * g.nz + pz) * g.nx * g.ny;
  for (int y0 = 0; y0 < g.ny; y0 += rc) {
    const int nr = min(rc, g.ny - y0);
    P.rows_in(g, y0, nr);
    for (int e = threadIdx.x; e < nr * g.nx; e += blockDim.x) o[(long)y0 * g.nx + e] = P.Rb[e];
    __syncthreads();
  }
}

// RHS (dfpt_module.f90:245-260): (psi_v1 + i psi_v2)(r) dv_p(r) / N -> forward
// -> sticks, one CTA per (plane, perturbation) over the band pairs
__global__ void __launch_bounds__(kRtPnt) k_plane_rhs_rt(const double2* __restrict__ evcr,
                                                         const double2* __restrict__ dvbox, int npv, StickTab st,
                                                         RtGeo g, double2* __restrict__ sticks, int rc) {
  const RtPlane<double2> P(g);
  const int pz = blockIdx.x, p = blockIdx.y;
  const long plane = (long)g.nx * g.ny;
  const double inv = 1.0 / ((double)plane * g.nz);
  const double2* dv = dvbox + ((long)(p >> 1) * g.nz + pz) * plane;
  const bool hi = p & 1;
  P.load_tw(g);
  for (int k = 0; k < npv; ++k) {
    const double2* ps = evcr + ((long)k * g.nz + pz) * plane;
    for (int y0 = 0; y0 < g.ny; y0 += rc) {
      const int nr = min(rc, g.ny - y0);
      for (int e = threadIdx.x; e < nr * g.nx; e += blockDim.x) {
        const long o = (long)y0 * g.nx + e;
        const double2 d = dv[o];
        P.Rb[e] = cscale(ps[o], (hi ? d.y : d.x) * inv);
      }
      __syncthreads();
      P.rows_out(g, y0, nr);
    }
    const long item = (long)p * npv + k;
    P.sticks_out(g, st, sticks + (item * g.nz + pz) * st.nst);
    __syncthreads();
  }
}

// density response (dfpt_module.f90:403-423, :478): drho_p = sum_v occ_v
// psi_v(r) dpsi_v(r) for the two perturbations of pair pp, accumulated in the
// CTA's own slice of acc (one element per thread throughout), then
// (drho_p1 + i drho_p2) scale -> forward -> sticks
__global__ void __launch_bounds__(kRtPnt, 1) k_plane_drho_rt(const double2* __restrict__ dsticks,
                                                          const double2* __restrict__ evcr,
                                                          const double* __restrict__ occ, int nocc, int mb,
                                                          StickTab st, RtGeo g, double2* __restrict__ acc,
                                                          double scale, double2* __restrict__ osticks, int rc) {
  const RtPlane<double2> P(g);
  const int pz = blockIdx.x, pp = blockIdx.y;
  const int npv = (nocc + 1) / 2;
  const long plane = (long)g.nx * g.ny;
  double2* ac = acc + ((long)pp * g.nz + pz) * plane;
  P.load_tw(g);
  for (int pi = 0; pi < 2; ++pi) {
    const int p = 2 * pp + pi;
    if (p >= mb) {  // odd batch: the second density of the last pair is zero
      for (long e = threadIdx.x; e < plane; e += blockDim.x) ac[e].y = 0.0;
      continue;
    }
    for (int k = 0; k < npv; ++k) {
      const long item = (long)p * npv + k;
      P.sticks_in(g, st, dsticks + (item * g.nz + pz) * st.nst);
      const double o1 = occ[2 * k];
      const double o2 = (2 * k + 1 < nocc) ? occ[2 * k + 1] : 0.0;
      const double2* ps = evcr + ((long)k * g.nz + pz) * plane;
      for (int y0 = 0; y0 < g.ny; y0 += rc) {
        const int nr = min(rc, g.ny - y0);
        P.rows_in(g, y0, nr);
        for (int e = threadIdx.x; e < nr * g.nx; e += blockDim.x) {
          const long o = (long)y0 * g.nx + e;
          const double2 d = P.Rb[e], s = ps[o];
          const double v = fma(o1 * s.x, d.x, o2 * s.y * d.y);
          double* a = pi ? &ac[o].y : &ac[o].x;
          *a = (k == 0) ? v : *a + v;
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  for (int y0 = 0; y0 < g.ny; y0 += rc) {
    const int nr = min(rc, g.ny - y0);
    for (int e = threadIdx.x; e < nr * g.nx; e += blockDim.x) {
      const double2 a = ac[(long)y0 * g.nx + e];
      P.Rb[e] = make_double2(a.x * scale, a.y * scale);
    }
    __syncthreads();
    P.rows_out(g, y0, nr);
  }
  P.sticks_out(g, st, osticks + ((long)pp * g.nz + pz) * st.nst);
}

// ---------------------------------------------------------------------------
// epilogues of the forward z pass (the same operations as wb_fft_kernels.cu's)
// ---------------------------------------------------------------------------
struct RtEpiStore {
  double2* dst;
  long ld;
  struct Pre {};
  WB_DEV Pre pre(int, int2) const { return {}; }
  WB_DEV void operator()(int gi, int2 it, const Pre&, double2 b1, double2 b2) const {
    dst[(long)it.x * ld + gi] = b1;
    if (it.y >= 0) dst[(long)it.y * ld + gi] = b2;
  }
};

// T = (V psi + g2kin psi with Im(G=0) = 0) - e psi
template <class C>
struct RtEpiHpsi {
  using T = real_t<C>;
  const C* P;
  C* Tv;
  long ld;
  const T* g2kin;
  const T* ecol;
  struct Pre {
    C p1, p2;
    T k;
  };
  WB_DEV Pre pre(int gi, int2 it) const {
    Pre r;
    r.p1 = P[(long)it.x * ld + gi];
    r.p2 = it.y >= 0 ? P[(long)it.y * ld + gi] : mkc<C>(0, 0);
    r.k = g2kin[gi];
    return r;
  }
  WB_DEV void one(int gi, int c, C p, T k, C vp) const {
    C h = mkc<C>(fma(k, p.x, vp.x), fma(k, p.y, vp.y));
    if (gi == 0) h.y = T(0);
    const T e = ecol[c];
    Tv[(long)c * ld + gi] = mkc<C>(fma(-e, p.x, h.x), fma(-e, p.y, h.y));
  }
  WB_DEV void operator()(int gi, int2 it, const Pre& pr, C b1, C b2) const {
    one(gi, it.x, pr.p1, pr.k, b1);
    if (it.y >= 0) one(gi, it.y, pr.p2, pr.k, b2);
  }
};

// dng(perm(g), p) = sqvc(g) drho_G(g), G = 0 zeroed
struct RtEpiDng {
  double2* dng;
  long ld;
  const int* perm;
  const double* sqvc;
  struct Pre {
    double s;
    int r;
  };
  WB_DEV Pre pre(int gi, int2) const { return {(gi == 0) ? 0.0 : sqvc[gi], perm[gi]}; }
  WB_DEV void operator()(int, int2 it, const Pre& pr, double2 b1, double2 b2) const {
    const long r = pr.r;
    dng[(long)it.x * ld + r] = make_double2(pr.s * b1.x, pr.s * b1.y);
    if (it.y >= 0) dng[(long)it.y * ld + r] = make_double2(pr.s * b2.x, pr.s * b2.y);
  }
};

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <class C>
static size_t rt_zsmem(const RtGeo& g) { return sizeof(C) * (g.nz + 2 * kRtZsg * (g.nz | 1)); }
static dim3 rt_zgrid(const StickTab& st, int nitems) { return dim3((st.nsp + kRtZsg - 1) / kRtZsg, nitems); }

void rt_setup(const RtGeo& g) {
  const int z64 = (int)rt_zsmem<double2>(g), z32 = (int)rt_zsmem<float2>(g);
  const int p64 = (int)rt_plane_smem(g, 16, nullptr), p32 = (int)rt_plane_smem(g, 8, nullptr);
  cudaFuncSetAttribute(k_zinv_rt<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, z64);
  cudaFuncSetAttribute(k_zinv_rt<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, z32);
  cudaFuncSetAttribute(k_zfwd_rt<double2, RtEpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, z64);
  cudaFuncSetAttribute(k_zfwd_rt<double2, RtEpiHpsi<double2>>, cudaFuncAttributeMaxDynamicSharedMemorySize, z64);
  cudaFuncSetAttribute(k_zfwd_rt<float2, RtEpiHpsi<float2>>, cudaFuncAttributeMaxDynamicSharedMemorySize, z32);
  cudaFuncSetAttribute(k_zfwd_rt<double2, RtEpiDng>, cudaFuncAttributeMaxDynamicSharedMemorySize, z64);
  cudaFuncSetAttribute(k_plane_vloc_rt<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, p64);
  cudaFuncSetAttribute(k_plane_vloc_rt<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, p32);
  cudaFuncSetAttribute(k_plane_inv_box_rt, cudaFuncAttributeMaxDynamicSharedMemorySize, p64);
  cudaFuncSetAttribute(k_plane_rhs_rt, cudaFuncAttributeMaxDynamicSharedMemorySize, p64);
  cudaFuncSetAttribute(k_plane_drho_rt, cudaFuncAttributeMaxDynamicSharedMemorySize, p64);
}

template <class C, class F>
static void zinv_rt_t(const F& f, const C* src, long ld, const int2* items, int nitems, C* sticks) {
  if (nitems <= 0) return;
  k_zinv_rt<C><<<rt_zgrid(f.st, nitems), kRtZnt, rt_zsmem<C>(*f.rt), f.stream>>>(src, ld, items, f.st, *f.rt,
                                                                                  sticks, f.dcount);
}
template <class C, class F, class Epi>
static void zfwd_rt_t(const F& f, const C* sticks, const int2* items, int nitems, Epi epi) {
  if (nitems <= 0) return;
  k_zfwd_rt<C, Epi><<<rt_zgrid(f.st, nitems), kRtZnt, rt_zsmem<C>(*f.rt), f.stream>>>(sticks, items, f.st, *f.rt,
                                                                                      epi, f.dcount);
}
template <class C, class F>
static void vloc_rt_t(const F& f, C* sticks, int nitems, const real_t<C>* vs) {
  if (nitems <= 0) return;
  int rc = 1;
  const size_t sm = rt_plane_smem(*f.rt, sizeof(C), &rc);
  k_plane_vloc_rt<C><<<dim3(f.rt->nz, nitems), kRtPnt, sm, f.stream>>>(sticks, f.st, *f.rt, vs, rc, f.dcount);
}

void rt_zinv(const FftArgs& f, const double2* src, long ld, const int2* items, int nitems, double2* sticks) {
  zinv_rt_t<double2>(f, src, ld, items, nitems, sticks);
}
void rt_zinv32(const FftArgs32& f, const float2* src, long ld, const int2* items, int nitems, float2* sticks) {
  zinv_rt_t<float2>(f, src, ld, items, nitems, sticks);
}
void rt_zfwd_store(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dst, long ld) {
  zfwd_rt_t<double2>(f, sticks, items, nitems, RtEpiStore{dst, ld});
}
void rt_zfwd_hpsi(const FftArgs& f, const double2* sticks, const int2* items, int nitems, const double2* P,
                  double2* T, long ld, const double* g2kin, const double* ecol) {
  zfwd_rt_t<double2>(f, sticks, items, nitems, RtEpiHpsi<double2>{P, T, ld, g2kin, ecol});
}
void rt_zfwd_hpsi32(const FftArgs32& f, const float2* sticks, const int2* items, int nitems, const float2* P,
                    float2* T, long ld, const float* g2kin, const float* ecol) {
  zfwd_rt_t<float2>(f, sticks, items, nitems, RtEpiHpsi<float2>{P, T, ld, g2kin, ecol});
}
void rt_zfwd_dng(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dng, long ld,
                 const int* perm, const double* sqvc) {
  zfwd_rt_t<double2>(f, sticks, items, nitems, RtEpiDng{dng, ld, perm, sqvc});
}
void rt_plane_vloc(const FftArgs& f, double2* sticks, int nitems, const double* vs) {
  vloc_rt_t<double2>(f, sticks, nitems, vs);
}
void rt_plane_vloc32(const FftArgs32& f, float2* sticks, int nitems, const float* vs) {
  vloc_rt_t<float2>(f, sticks, nitems, vs);
}
void rt_plane_inv_box(const FftArgs& f, const double2* sticks, int nitems, double2* box) {
  if (nitems <= 0) return;
  int rc = 1;
  const size_t sm = rt_plane_smem(*f.rt, 16, &rc);
  k_plane_inv_box_rt<<<dim3(f.rt->nz, nitems), kRtPnt, sm, f.stream>>>(sticks, f.st, *f.rt, box, rc);
}
void rt_plane_rhs(const FftArgs& f, const double2* evcr, const double2* dvbox, int npv, int mb, double2* sticks) {
  if (mb <= 0) return;
  int rc = 1;
  const size_t sm = rt_plane_smem(*f.rt, 16, &rc);
  k_plane_rhs_rt<<<dim3(f.rt->nz, mb), kRtPnt, sm, f.stream>>>(evcr, dvbox, npv, f.st, *f.rt, sticks, rc);
}
void rt_plane_drho(const FftArgs& f, const double2* dsticks, const double2* evcr, const double* occ, int nocc,
                   int mb, double2* acc, double scale, double2* osticks) {
  if (mb <= 0) return;
  int rc = 1;
  const size_t sm = rt_plane_smem(*f.rt, 16, &rc);
  k_plane_drho_rt<<<dim3(f.rt->nz, (mb + 1) / 2), kRtPnt, sm, f.stream>>>(dsticks, evcr, occ, nocc, mb, f.st,
                                                                          *f.rt, acc, scale, osticks, rc);
}

}  // namespace wb
