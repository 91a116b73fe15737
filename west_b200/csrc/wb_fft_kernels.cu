// Stick-and-plane 3D FFTs of the Gamma-only response operator.
//
// The G sphere is cut into sticks along z.  A "stick pair" is the stick at
// (x, y) of the stored half sphere together with its mirror at (-x, -y), which
// holds the -G partners; the (0,0) stick is its own mirror.  Inside the
// library G vectors are ordered stick pair by stick pair, z ascending, so
// every stick pair reads one contiguous run of coefficients.
//
// One complex 3D FFT carries two real functions (FFT_kernel/fft_at_gamma.f90):
//   inverse: box(+G) = a1 + i a2, box(-G) = conj(a1 - i a2)          (:55-64)
//   forward: fp = (A(G) + A(-G))/2, fm = (A(G) - A(-G))/2,
//            b1 = (Re fp, Im fm), b2 = (Im fp, -Re fm)                 (:98-111)
// Both are fused into the z-pass kernels.  The x-y passes run one plane per
// CTA in shared memory, with the pointwise work of the caller (local
// potential, RHS product, density accumulation) fused between the inverse and
// forward transforms.
//
// Stick buffer layout: [item][z][stick], stick = 2q and 2q+1 for the two
// sticks of pair q; stick 1 (mirror slot of (0,0)) is a dummy that is never
// scattered.  g_qz of a stored G is (2q + side, z), side = which of the two
// sticks of the pair holds it.
#include <algorithm>
#include <type_traits>

#include "wb_fft.cuh"
#include "wb_internal.h"

namespace wb {

// z passes: 8 stick pairs per CTA of 128 threads (measured against 16/256 and
// 4/64 at 64^3: more, smaller CTAs overlap one CTA's loads with another's
// transform and stores; zfwd 0.30 instead of 0.34 us per FP64 item)
constexpr int ZSG = 8;
constexpr int ZNT = 128;
constexpr int PNT = 256;

// 2N-entry twiddle table: natural order, then the step-1 factors (wb_fft.cuh)
template <int N, class C>
WB_DEV void load_tw(C* tw, const C* twg) {
  constexpr int N2 = FftSplit<N>::N2;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    tw[i] = twg[i];
    tw[N + i] = twg[((i % N2) * (i / N2)) % N];
  }
}

// ---------------------------------------------------------------------------
// z pass, inverse: sphere coefficients of a pair of columns -> sticks
// ---------------------------------------------------------------------------
// One unit = stick pairs [ZSG qg, ZSG qg + ZSG) of band-pair item `item`.
// Shared memory of every unit: the twiddles (2N), then the work area.  A unit
// takes its pointers from the dynamic shared array itself so that a unit body
// compiled as a separate function still addresses shared memory directly.
template <class C>
WB_DEV C* smem_tw() {
  extern __shared__ __align__(16) unsigned char smraw[];
  return reinterpret_cast<C*>(smraw);
}

// Twiddles of one thread (2N entries over the block), held in registers so
// that their global loads are issued with the unit's other loads and stored
// to shared memory after the zero fill.
template <int N, class C>
struct TwRegs {
  static constexpr int PER = (2 * N + ZNT - 1) / ZNT;
  C v[PER];
  WB_DEV void load(const C* __restrict__ twg) {
    constexpr int N2 = FftSplit<N>::N2;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = threadIdx.x + ZNT * k;
      if (i < N) v[k] = twg[i];
      else if (i < 2 * N) v[k] = twg[(((i - N) % N2) * ((i - N) / N2)) % N];
    }
  }
  WB_DEV void store(C* tw) const {
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = threadIdx.x + ZNT * k;
      if (i < 2 * N) tw[i] = v[k];
    }
  }
};

// G coefficients prefetched per thread before the zero fill (the rest of a
// stick group's G vectors, if any, are read in a second loop).
constexpr int kZPre = 2;

template <int N, bool PR, class C>
__global__ void __launch_bounds__(ZNT) k_zinv(const C* __restrict__ src, long ld,
                                              const int2* __restrict__ items, StickTab st,
                                              C* __restrict__ out,
                                              const C* __restrict__ twg, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;  // beyond the device item count
  constexpr int LS = LinePad<N>::LEN | 1;  // odd line stride: conflict-free transposes
  using LP = LinePad<N>;
  C* tw = smem_tw<C>();
  C* zb = smem_tw<C>() + 2 * N;
  const int qg = blockIdx.x, item = blockIdx.y;
  const int q0 = qg * ZSG;
  const int nq = min(ZSG, st.nsp - q0);
  const int2 it = items[item];
  const C* a = src + (long)it.x * ld;
  const C* b = src + (long)(it.y >= 0 ? it.y : it.x) * ld;
  const bool two = it.y >= 0;
  const int g0 = st.sp_gstart[q0], g1 = st.sp_gstart[q0 + nq];
  TwRegs<N, C> twr;
  twr.load(twg);
  C pa[kZPre], pb[kZPre];
  int2 pq[kZPre];
#pragma unroll
  for (int k = 0; k < kZPre; ++k) {
    const int g = g0 + threadIdx.x + k * ZNT;
    if (g < g1) {
      pq[k] = st.g_qz[g];
      pa[k] = a[g];
      pb[k] = two ? b[g] : mkc<C>(0, 0);
    }
  }
  // zero what step 1 reads: with pruning only the live inputs (the sphere's z
  // lie in the outer quarters), otherwise the whole lines
  if constexpr (PR && Prune<N>::IN_OK) {
    constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2, NLIVE = N1 / 2;
    for (int e = threadIdx.x; e < 2 * ZSG * NLIVE * N2; e += ZNT) {
      const int l = e / (NLIVE * N2), r = e % (NLIVE * N2);
      const int h = r / N2, n2 = r % N2;
      const int n1 = h < NLIVE / 2 ? h : N1 - NLIVE + h;
      zb[l * LS + LP::off_blk(n1, n2)] = mkc<C>(0, 0);
    }
  } else {
    for (int i = threadIdx.x; i < 2 * ZSG * LS; i += ZNT) zb[i] = mkc<C>(0, 0);
  }
  twr.store(tw);
  __syncthreads();
  auto put = [&](int2 qz, C a1, C a2) {
    // pos = a1 + i a2 ; neg = conj(a1 - i a2)
    const C pos = mkc<C>(a1.x - a2.y, a1.y + a2.x);
    const C neg = mkc<C>(a1.x + a2.y, a2.x - a1.y);
    const int z = qz.y;
    if (qz.x < 2) {  // the (0,0) stick is its own mirror
      if (z != 0) { zb[LP::off((z + N) % N)] = pos; zb[LP::off((N - z) % N)] = neg; }
      else zb[0] = neg;  // G = 0: the -G store wins, as in the reference loop
    } else {
      const int l = qz.x - 2 * q0;  // slot of the stick holding G; its mirror is l ^ 1
      zb[l * LS + LP::off((z + N) % N)] = pos;
      zb[(l ^ 1) * LS + LP::off((N - z) % N)] = neg;
    }
  };
#pragma unroll
  for (int k = 0; k < kZPre; ++k)
    if (g0 + (int)threadIdx.x + k * ZNT < g1) put(pq[k], pa[k], pb[k]);
  for (int g = g0 + threadIdx.x + kZPre * ZNT; g < g1; g += ZNT)
    put(st.g_qz[g], a[g], two ? b[g] : mkc<C>(0, 0));
  __syncthreads();
  fft_lines<N, +1, ZNT, false, true, PR ? PRUNE_IN : PRUNE_NONE>(zb, OffLinear{LS}, 1, 2 * nq, tw);
  const int ns = 2 * nq;
  C* o = out + (long)item * N * st.nst + 2 * q0;
  for (int e = threadIdx.x; e < ns * N; e += ZNT) {
    const int s = e % ns, z = e / ns;
    o[(long)z * st.nst + s] = zb[s * LS + LinePad<N>::off(z)];
  }
}

// ---------------------------------------------------------------------------
// z pass, forward: sticks -> sphere with the Gamma unpack, then an epilogue
// ---------------------------------------------------------------------------
// The twiddles are loaded into registers with the sticks and stored after
// them.  An epilogue reads its per-G inputs through Epi::pre (prefetching them
// before the transform was measured slower: the extra registers cost more
// occupancy than the hidden latency gained).
template <int N, bool PR, class C, class Epi>
__global__ void __launch_bounds__(ZNT) k_zfwd(const C* __restrict__ sticks,
                                              const int2* __restrict__ items, StickTab st,
                                              const C* __restrict__ twg, Epi epi, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  constexpr int LS = LinePad<N>::LEN | 1;
  using LP = LinePad<N>;
  using T = real_t<C>;
  C* tw = smem_tw<C>();
  C* zb = smem_tw<C>() + 2 * N;
  const int qg = blockIdx.x, item = blockIdx.y;
  const int q0 = qg * ZSG;
  const int nq = min(ZSG, st.nsp - q0);
  const int ns = 2 * nq;
  const C* s0 = sticks + (long)item * N * st.nst + 2 * q0;
  TwRegs<N, C> twr;
  twr.load(twg);
  const int2 it = items[item];
  const int g0 = st.sp_gstart[q0], g1 = st.sp_gstart[q0 + nq];
  for (int e = threadIdx.x; e < ns * N; e += ZNT) {
    const int s = e % ns, z = e / ns;
    zb[s * LS + LinePad<N>::off(z)] = s0[(long)z * st.nst + s];
  }
  twr.store(tw);
  __syncthreads();
  fft_lines<N, -1, ZNT, false, true, PR ? PRUNE_OUT : PRUNE_NONE>(zb, OffLinear{LS}, 1, ns, tw);
  auto take = [&](int g, int2 qz, const typename Epi::Pre& pr) {
    const int z = qz.y;
    C ap, am;
    if (qz.x < 2) {
      ap = zb[LP::off((z + N) % N)];
      am = zb[LP::off((N - z) % N)];
    } else {
      const int l = qz.x - 2 * q0;
      ap = zb[l * LS + LP::off((z + N) % N)];
      am = zb[(l ^ 1) * LS + LP::off((N - z) % N)];
    }
    const C fp = mkc<C>(T(0.5) * (ap.x + am.x), T(0.5) * (ap.y + am.y));
    const C fm = mkc<C>(T(0.5) * (ap.x - am.x), T(0.5) * (ap.y - am.y));
    epi(g, it, pr, mkc<C>(fp.x, fm.y), mkc<C>(fp.y, -fm.x));
  };
  for (int g = g0 + threadIdx.x; g < g1; g += ZNT) take(g, st.g_qz[g], epi.pre(g, it));
}

struct EpiStore {
  double2* dst;
  long ld;
  struct Pre {};
  WB_DEV Pre pre(int, int2) const { return {}; }
  WB_DEV void operator()(int g, int2 it, const Pre&, double2 b1, double2 b2) const {
    dst[(long)it.x * ld + g] = b1;
    if (it.y >= 0) dst[(long)it.y * ld + g] = b2;
  }
};

// T = (V psi + g2kin psi with Im(G=0) = 0) - e psi   (h_psi then
// apply_sternheimerop_to_m_wfcs.f90:65-74; KB and alpha Pv follow as GEMMs)
template <class C>
struct EpiHpsiT {
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
  WB_DEV Pre pre(int g, int2 it) const {
    Pre r;
    r.p1 = P[(long)it.x * ld + g];
    r.p2 = it.y >= 0 ? P[(long)it.y * ld + g] : mkc<C>(0, 0);
    r.k = g2kin[g];
    return r;
  }
  WB_DEV void one(int g, int c, C p, T k, C vp) const {
    C h = mkc<C>(fma(k, p.x, vp.x), fma(k, p.y, vp.y));
    if (g == 0) h.y = T(0);
    const T e = ecol[c];
    Tv[(long)c * ld + g] = mkc<C>(fma(-e, p.x, h.x), fma(-e, p.y, h.y));
  }
  WB_DEV void operator()(int g, int2 it, const Pre& pr, C b1, C b2) const {
    one(g, it.x, pr.p1, pr.k, b1);
    if (it.y >= 0) one(g, it.y, pr.p2, pr.k, b2);
  }
};
using EpiHpsi = EpiHpsiT<double2>;
using EpiHpsi32 = EpiHpsiT<float2>;

// dng(perm(g), p) = sqvc(g) * drho_G(g), G = 0 zeroed
// (dfpt_module.f90:485-487,502-503 and apply_operator.f90:63-67)
struct EpiDng {
  double2* dng;
  long ld;
  const int* perm;
  const double* sqvc;
  struct Pre {
    double s;
    int r;
  };
  WB_DEV Pre pre(int g, int2) const { return {(g == 0) ? 0.0 : sqvc[g], perm[g]}; }
  WB_DEV void operator()(int g, int2 it, const Pre& pr, double2 b1, double2 b2) const {
    const double s = pr.s;
    const long r = pr.r;
    dng[(long)it.x * ld + r] = make_double2(s * b1.x, s * b1.y);
    if (it.y >= 0) dng[(long)it.y * ld + r] = make_double2(s * b2.x, s * b2.y);
  }
};

// ---------------------------------------------------------------------------
// x-y plane passes
// ---------------------------------------------------------------------------
// Zero what the inverse transforms read: with pruning (PR) only the active
// columns (which then are all x in [0, N/4) u [3N/4, N)) at live rows (y in
// the same quarters), otherwise the whole plane.
template <int N, bool PR, class C, class PL = Plane<N>, int NT = PNT>
WB_DEV void plane_zero(C* pl, const StickTab& st) {
  if constexpr (PR && Prune<N>::IN_OK) {
    constexpr int NL = 2 * (N / 4);
    const int nc = st.ncols, nlow = st.xhi + 1;
    for (int e = threadIdx.x; e < NL * nc; e += NT) {
      const int l = e % nc, r = e / nc;
      const int x = l < nlow ? l : N - nc + l;
      const int y = r < N / 4 ? r : N - NL + r;
      pl[PL::at(x, y)] = mkc<C>(0, 0);
    }
  } else {
    for (int e = threadIdx.x; e < PL::SIZE; e += NT) pl[e] = mkc<C>(0, 0);
  }
}
// stick positions are y*N + x in row-major plane order
template <int N, class C, class PL = Plane<N>, int NT = PNT>
WB_DEV void plane_scatter(C* pl, const C* __restrict__ sz, const int* __restrict__ pos, int nst) {
  for (int s = threadIdx.x; s < nst; s += NT) {
    const int p = pos[s];
    if (p >= 0) pl[PL::at_lin(p)] = sz[s];
  }
}
template <int N, class C, class PL = Plane<N>, int NT = PNT>
WB_DEV void plane_gather(const C* pl, C* __restrict__ sz, const int* __restrict__ pos, int nst) {
  for (int s = threadIdx.x; s < nst; s += NT) {
    const int p = pos[s];
    sz[s] = p >= 0 ? pl[PL::at_lin(p)] : mkc<C>(0, 0);
  }
}
// inverse transforms prune inputs, forward transforms prune outputs
template <int N, int DIR, bool PR, class C, int NT = PNT>
WB_DEV void plane_fft_cols(C* pl, const StickTab& st, const C* tw) {
  constexpr int P = !PR ? PRUNE_NONE : (DIR > 0 ? PRUNE_IN : PRUNE_OUT);
  fft_lines<N, DIR, NT, true, false, P>(pl, OffCols<N>{st.xhi + 1, st.ncols}, Plane<N>::RS, st.ncols, tw);
}
template <int N, int DIR, bool PR, class C, int NT = PNT>
WB_DEV void plane_fft_rows(C* pl, const C* tw) {
  constexpr int P = !PR ? PRUNE_NONE : (DIR > 0 ? PRUNE_IN : PRUNE_OUT);
  fft_lines<N, DIR, NT, false, true, P>(pl, OffLinear{Plane<N>::RS}, 1, N, tw);
}

// RHS and density kernels.  Up to 72^3 a thread keeps its share of the plane
// (N^2 / 256 doubles: dv(r) for the RHS, the band sum for the density) in
// registers across the band loop; from 80^3 on that share does not fit beside
// the 12- and 10-point transforms, so the RHS re-reads dv(r) and the density
// accumulates in the CTA's own slice of the global acc buffer, one element per
// thread throughout (148 such slices, 14 MB at 108^3, stay in L2).  The CTA
// may use up to 255 registers per thread (for the large boxes one CTA per SM,
// which their FP64 plane allows no more than anyway); two CTAs of 128
// registers spilled up to 976 B per thread.
template <int N>
constexpr bool rd_regs() { return N < 80; }
template <int N>
constexpr int rd_threads() { return 256; }
template <int N>
constexpr int rd_min_blocks() { return 1; }

// psi -> V(r) psi(r) / N^3 -> back, in place on the sticks (QE vloc_psi_gamma);
// one unit = plane z of item `item`
template <int N, bool PR, class C>
WB_DEV void plane_vloc_unit(C* __restrict__ sticks, const StickTab& st, const real_t<C>* __restrict__ vs, int z,
                            int item) {
  const C* tw = smem_tw<C>();
  C* pl = smem_tw<C>() + 2 * N;
  C* sz = sticks + ((long)item * N + z) * st.nst;
  plane_zero<N, PR>(pl, st);
  __syncthreads();
  plane_scatter<N>(pl, sz, st.st_pos, st.nst);
  __syncthreads();
  plane_fft_cols<N, +1, PR>(pl, st, tw);
  plane_fft_rows<N, +1, PR>(pl, tw);
  const real_t<C>* v = vs + (long)z * N * N;
  for (int e = threadIdx.x; e < N * N; e += PNT) {
    const int o = Plane<N>::at_lin(e);
    pl[o] = cscale(pl[o], v[e]);
  }
  __syncthreads();
  plane_fft_rows<N, -1, PR>(pl, tw);
  plane_fft_cols<N, -1, PR>(pl, st, tw);
  plane_gather<N>(pl, sz, st.st_pos, st.nst);
}

template <int N, bool PR, class C>
__global__ void __launch_bounds__(PNT) k_plane_vloc(C* __restrict__ sticks, StickTab st,
                                                    const real_t<C>* __restrict__ vs,
                                                    const C* __restrict__ twg, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  load_tw<N>(smem_tw<C>(), twg);
  plane_vloc_unit<N, PR, C>(sticks, st, vs, blockIdx.x, blockIdx.y);
}

// sticks -> full real-space box (complex: two real functions), no scaling
template <int N, bool PR>
__global__ void __launch_bounds__(PNT) k_plane_inv_box(const double2* __restrict__ sticks, StickTab st,
                                                       double2* __restrict__ box,
                                                       const double2* __restrict__ twg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* tw = reinterpret_cast<double2*>(smraw);
  double2* pl = tw + 2 * N;
  const int z = blockIdx.x, item = blockIdx.y;
  const double2* sz = sticks + ((long)item * N + z) * st.nst;
  load_tw<N>(tw, twg);
  plane_zero<N, PR>(pl, st);
  __syncthreads();
  plane_scatter<N>(pl, sz, st.st_pos, st.nst);
  __syncthreads();
  plane_fft_cols<N, +1, PR>(pl, st, tw);
  plane_fft_rows<N, +1, PR>(pl, tw);
  double2* o = box + ((long)item * N + z) * N * N;
  for (int e = threadIdx.x; e < N * N; e += PNT) o[e] = pl[Plane<N>::at_lin(e)];
}

// RHS of the Sternheimer equation, dfpt_module.f90:245-260:
// (psi_v1(r) + i psi_v2(r)) * dv_p(r) / N^3 -> forward -> sticks
// One CTA per (plane z, perturbation p) loops over the band pairs: dv_p(r) of
// the plane is read once into registers (thread t owns elements t + PNT q)
// instead of once per band pair, and the psi planes come from L2 (the grid of
// one CTA per band pair read 8.6 GB of boxes per c2 call; 1.7 against 2.1 ms).
template <int N, bool PR>
__global__ void __launch_bounds__(rd_threads<N>(), rd_min_blocks<N>()) k_plane_rhs(const double2* __restrict__ evcr,
                                                   const double2* __restrict__ dvbox, int npv,
                                                   StickTab st, double2* __restrict__ sticks,
                                                   const double2* __restrict__ twg) {
  constexpr int NT = rd_threads<N>();
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* tw = reinterpret_cast<double2*>(smraw);
  double2* pl = tw + 2 * N;
  const int z = blockIdx.x, p = blockIdx.y;
  load_tw<N>(tw, twg);
  constexpr bool REG = rd_regs<N>();
  constexpr int PER = REG ? (N * N + NT - 1) / NT : 1;
  constexpr double inv = 1.0 / ((double)N * N * N);
  const double2* dv = dvbox + ((long)(p >> 1) * N + z) * N * N;
  const bool hi = p & 1;
  double w[PER];
  if constexpr (REG) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = threadIdx.x + q * NT;
      w[q] = 0.0;
      if (e < N * N) {
        const double2 d = dv[e];
        w[q] = (hi ? d.y : d.x) * inv;
      }
    }
  }
  for (int k = 0; k < npv; ++k) {
    const double2* ps = evcr + ((long)k * N + z) * N * N;
    __syncthreads();  // the previous band pair's gather is done with the plane
    if constexpr (REG) {
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x + q * NT;
        if (e < N * N) pl[Plane<N>::at_lin(e)] = cscale(ps[e], w[q]);
      }
    } else {
      for (int e = threadIdx.x; e < N * N; e += NT) {
        const double2 d = dv[e];
        pl[Plane<N>::at_lin(e)] = cscale(ps[e], (hi ? d.y : d.x) * inv);
      }
    }
    __syncthreads();
    plane_fft_rows<N, -1, PR, double2, NT>(pl, tw);
    plane_fft_cols<N, -1, PR, double2, NT>(pl, st, tw);
    const long item = (long)p * npv + k;
    plane_gather<N, double2, Plane<N>, NT>(pl, sticks + (item * N + z) * st.nst, st.st_pos, st.nst);
  }
}

// Density response, dfpt_module.f90:403-423 and :478:
// drho_p(r) = sum_v occ_v psi_v(r) dpsi_v(r), two perturbations per CTA,
// then (drho_p1 + i drho_p2) * scale -> forward -> sticks.
// acc is per-CTA scratch in global memory ([pp][z][N*N] double2) that parks
// the first perturbation's density once; each element is owned by the thread
// that writes it.  The band sums run in registers (a read-modify-write of acc
// per band pair made the kernel DRAM-bound: 12.6 GB per c2 call); two CTAs per
// SM (a few hundred bytes of spills) beat one (2.5 against 2.9 ms per c2 call).
template <int N, bool PR>
__global__ void __launch_bounds__(rd_threads<N>(), rd_min_blocks<N>()) k_plane_drho(const double2* __restrict__ dsticks,
                                                    const double2* __restrict__ evcr,
                                                    const double* __restrict__ occ, int nocc,
                                                    int mb, StickTab st, double2* __restrict__ acc,
                                                    double scale, double2* __restrict__ osticks,
                                                    const double2* __restrict__ twg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* tw = reinterpret_cast<double2*>(smraw);
  double2* pl = tw + 2 * N;
  const int z = blockIdx.x, pp = blockIdx.y;
  const int npv = (nocc + 1) / 2;
  constexpr int NT = rd_threads<N>();
  load_tw<N>(tw, twg);
  // a perturbation's density of this plane is accumulated in registers (thread t
  // owns plane elements t + PNT q); the first of the two is parked in acc once
  double2* ac = acc + ((long)pp * N + z) * N * N;
  constexpr bool REG = rd_regs<N>();
  constexpr int PER = REG ? (N * N + NT - 1) / NT : 1;
  double a[PER];
  for (int pi = 0; pi < 2; ++pi) {
    const int p = 2 * pp + pi;
#pragma unroll
    for (int q = 0; q < PER; ++q) a[q] = 0.0;
    if constexpr (!REG) {  // the band sum of this perturbation in ac[].x (pi = 0) or ac[].y (pi = 1)
      for (int e = threadIdx.x; e < N * N; e += NT) {
        if (pi == 0) ac[e].x = 0.0;
        else ac[e].y = 0.0;
      }
    }
    for (int k = 0; p < mb && k < npv; ++k) {
      const long item = (long)p * npv + k;
      __syncthreads();
      plane_zero<N, PR, double2, Plane<N>, NT>(pl, st);
      __syncthreads();
      plane_scatter<N, double2, Plane<N>, NT>(pl, dsticks + (item * N + z) * st.nst, st.st_pos, st.nst);
      __syncthreads();
      plane_fft_cols<N, +1, PR, double2, NT>(pl, st, tw);
      plane_fft_rows<N, +1, PR, double2, NT>(pl, tw);
      const double o1 = occ[2 * k];
      const double o2 = (2 * k + 1 < nocc) ? occ[2 * k + 1] : 0.0;
      const double2* ps = evcr + ((long)k * N + z) * N * N;
      if constexpr (REG) {
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          const int e = threadIdx.x + q * NT;
          if (e < N * N) {
            const double2 d = pl[Plane<N>::at_lin(e)], s = ps[e];
            a[q] += fma(o1 * s.x, d.x, o2 * s.y * d.y);
          }
        }
      } else {
        for (int e = threadIdx.x; e < N * N; e += NT) {
          const double2 d = pl[Plane<N>::at_lin(e)], s = ps[e];
          const double v = fma(o1 * s.x, d.x, o2 * s.y * d.y);
          if (pi == 0) ac[e].x += v;
          else ac[e].y += v;
        }
      }
    }
    if (REG && pi == 0) {
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x + q * NT;
        if (e < N * N) ac[e].x = a[q];
      }
    }
  }
  __syncthreads();
  if constexpr (REG) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = threadIdx.x + q * NT;
      if (e < N * N) pl[Plane<N>::at_lin(e)] = make_double2(ac[e].x * scale, a[q] * scale);
    }
  } else {
    for (int e = threadIdx.x; e < N * N; e += NT) {
      const double2 v = ac[e];
      pl[Plane<N>::at_lin(e)] = make_double2(v.x * scale, v.y * scale);
    }
  }
  __syncthreads();
  plane_fft_rows<N, -1, PR, double2, NT>(pl, tw);
  plane_fft_cols<N, -1, PR, double2, NT>(pl, st, tw);
  plane_gather<N, double2, Plane<N>, NT>(pl, osticks + ((long)pp * N + z) * st.nst, st.st_pos, st.nst);
}

// Local potential for N1 == N2 boxes (64^3): the inverse-row second step, the
// V(r)/N^3 product and the forward-row first step run in registers of one
// thread (the outputs X[k1 + R k2] of the inverse are exactly the inputs
// x[R n1 + k1] of the forward step for n1 = k2), saving a shared-memory round
// trip of the whole plane.  The plane's sticks are loaded into registers
// before the zero fill so their latency overlaps it.  The plane uses the
// FPlane layout; the row threads keep their step-1 twiddles W^(q n2) in
// registers (every row item of a thread has the same n2 = tid % R).
constexpr int kFusedMaxSticksPerThread = 4;

template <int N, class C>
struct OffFRows {
  WB_DEV int operator()(int l) const { return FPlane<N, C>::row(l); }
};

// Column transforms of the fused plane.  For N = 64 (pruned: 32 active columns
// in the four aligned blocks x in [0,16) u [48,64)) thread t takes column
// 8 ((t / 16) % 4) + t % 8 of the active set and sub = 2 (t / 64) + (t / 8) % 2
// as its n2 (step 1) and k1 (step 2): a half-warp then covers one block of 8
// columns in two rows 1 (steps 1 and 2-out) or 8 (step 2-in) apart, which
// FPlane puts in disjoint bank slots.
template <int N, int DIR, int P, class C>
WB_DEV void fused_cols(C* pl, const StickTab& st, const C* tw) {
  using FP = FPlane<N, C>;
  if constexpr (N == 64 && PNT == 256) {
    constexpr int R = 8;
    using PR = Prune<N>;
    constexpr bool PIN = P == PRUNE_IN, POUT = P == PRUNE_OUT;
    const int tid = threadIdx.x;
    const int l = 8 * ((tid >> 4) & 3) + (tid & 7);
    const int x = l < 16 ? l : 32 + l;
    const int sub = 2 * (tid >> 6) + ((tid >> 3) & 1);
    C* p = pl + LinePad<N>::off(x);
    C v[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1)
      v[n1] = (PIN && !PR::in_live(n1)) ? mkc<C>(0, 0) : p[FP::row2(n1, sub)];
    rdft<R, DIR, N>(v, tw);
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) v[k1] = ctw<DIR>(v[k1], tw[N + k1 * R + sub]);
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) p[FP::row2(k1, sub)] = v[k1];
    __syncthreads();
#pragma unroll
    for (int n2 = 0; n2 < R; ++n2) v[n2] = p[FP::row2(sub, n2)];
    rdft<R, DIR, N>(v, tw);
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2)
      if (!POUT || PR::out_live(k2)) p[FP::row2(k2, sub)] = v[k2];
    __syncthreads();
  } else {
    static_assert(FP::GP == 0, "grouped plane rows need the N = 64 column mapping");
    fft_lines<N, DIR, PNT, true, false, P>(pl, OffCols<N>{st.xhi + 1, st.ncols}, FP::RS, st.ncols, tw);
  }
}

template <int N, class C, bool TWR>
WB_DEV void plane_vloc_fused_unit(C* __restrict__ sticks, const StickTab& st, const real_t<C>* __restrict__ vs, int z,
                                  int item, const C* __restrict__ twg) {
  C* tw = smem_tw<C>();
  C* pl = smem_tw<C>() + 2 * N;
  using T = real_t<C>;
  using FP = FPlane<N, C>;
  using PR = Prune<N>;
  constexpr int R = FftSplit<N>::N1;
  static_assert(FftSplit<N>::N1 == FftSplit<N>::N2, "fused rows need N1 == N2");
  static_assert(PNT % R == 0, "row threads keep one n2");
  constexpr int LPC = PNT / R;
  constexpr int NCH = (N + LPC - 1) / LPC;
  constexpr int MS = kFusedMaxSticksPerThread;
  using LP = LinePad<N>;
  const int tid = threadIdx.x;
  C* sz = sticks + ((long)item * N + z) * st.nst;
  C sv[MS];
  int sp[MS];
#pragma unroll
  for (int i = 0; i < MS; ++i) {
    const int s = tid + i * PNT;
    sp[i] = -1;
    if (s < st.nst) { sp[i] = st.st_pos[s]; sv[i] = sz[s]; }
  }
  const int k1 = tid % R;
  const bool rowthr = tid < LPC * R;
  const T* vz = vs + (long)z * N * N;
  load_tw<N>(tw, twg);
  plane_zero<N, true, C, FP>(pl, st);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MS; ++i)
    if (sp[i] >= 0) pl[FP::at_lin(sp[i])] = sv[i];
  C wr[R];
  if constexpr (TWR) {
#pragma unroll
    for (int q = 1; q < R; ++q) wr[q] = tw[N + q * R + k1];
  }
  __syncthreads();
  fused_cols<N, +1, PRUNE_IN, C>(pl, st, tw);
  // Rows: the R threads of a row are R consecutive lanes of one warp, and a warp
  // keeps its rows through all row steps, so the steps are separated by warp
  // barriers only.  Per row: inverse step 1 (pruned input, n2 = k1), inverse
  // step 2 + V(r) + forward step 1 in registers, forward step 2 (pruned output).
  static_assert(32 % R == 0, "a row's threads must share a warp");
#pragma unroll 1
  for (int c = 0; c < NCH; ++c) {
    const int y = c * LPC + tid / R;
    const bool act = rowthr && y < N;
    C* p = pl + FP::row(act ? y : 0);
    C v[R];
    if (act) {
#pragma unroll
      for (int n1 = 0; n1 < R; ++n1)
        v[n1] = (PR::IN_OK && !PR::in_live(n1)) ? mkc<C>(0, 0) : p[LP::off_blk(n1, k1)];
      rdft<R, +1, N>(v, tw);
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = ctw<+1>(v[q], TWR ? wr[q] : tw[N + q * R + k1]);
#pragma unroll
      for (int q = 0; q < R; ++q) p[LP::off_blk(q, k1)] = v[q];
    }
    __syncwarp();
    if (act) {
      T vr[R];                                      // V(r) of this row, loaded here to keep registers free
#pragma unroll
      for (int k2 = 0; k2 < R; ++k2) vr[k2] = __ldg(vz + y * N + k1 + R * k2);
#pragma unroll
      for (int n2 = 0; n2 < R; ++n2) v[n2] = p[LP::off_blk(k1, n2)];
      rdft<R, +1, N>(v, tw);                        // X[k1 + R k2], k2 = 0..R-1
#pragma unroll
      for (int k2 = 0; k2 < R; ++k2) v[k2] = cscale(v[k2], vr[k2]);
      rdft<R, -1, N>(v, tw);                        // forward step 1 over n1 = k2, thread n2 = k1
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = ctw<-1>(v[q], TWR ? wr[q] : tw[N + q * R + k1]);
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int q = 0; q < R; ++q) p[LP::off_blk(q, k1)] = v[q];
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int n2 = 0; n2 < R; ++n2) v[n2] = p[LP::off_blk(k1, n2)];
      rdft<R, -1, N>(v, tw);
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int k2 = 0; k2 < R; ++k2)
        if (!PR::OUT_OK || PR::out_live(k2)) p[LP::off(k1 + R * k2)] = v[k2];
    }
  }
  __syncthreads();
  fused_cols<N, -1, PRUNE_OUT, C>(pl, st, tw);
  plane_gather<N, C, FP>(pl, sz, st.st_pos, st.nst);
}

template <int N, class C>
__global__ void __launch_bounds__(PNT, 3) k_plane_vloc_fused(C* __restrict__ sticks, StickTab st,
                                                             const real_t<C>* __restrict__ vs,
                                                             const C* __restrict__ twg, const int* dn) {
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  plane_vloc_fused_unit<N, C, sizeof(C) == 8>(sticks, st, vs, blockIdx.x, blockIdx.y, twg);
}

// ---------------------------------------------------------------------------
// One-pass local-potential plane kernel for any split N = A x B (A = N1, B = N2)
// ---------------------------------------------------------------------------
// Rows: the inverse uses the split (A, B), the forward the transposed split
// (B, A).  The inverse's second step leaves X[k1 + A k2] (k2 = 0..B-1) in the
// thread owning k1, which is the input set {A n1' + n2'} of the forward's first
// step for n2' = k1: the inverse step 2, the V(r) product and the forward
// step 1 run in registers of one thread.  Each of the three row phases reads and
// writes the same plane positions per thread, so they need one block barrier
// between phases and none inside.  The forward's outputs k1' + B k2' are live
// (pruned transforms) iff k2' lies in the outer quarters of A, the condition of
// the inverse's live inputs, so A % 4 == 0 prunes both directions; the forward
// column pass uses the transposed split for the same reason.

// W_N^(n2 k1) for the step-1 twiddle of the split (S1, S2), k1 < S1, n2 < S2,
// from the second half of the table (built for FftSplit<N>)
template <int N, int S1, int S2, class C>
WB_DEV C tw_step1(const C* tw, int k1, int n2) {
  constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
  static_assert(S1 * S2 == N && (S1 == N1 || S1 == N2), "split of N");
  if constexpr (S1 == N1) return tw[N + k1 * N2 + n2];
  else return tw[N + n2 * N2 + k1];
}
template <int S>
WB_DEV constexpr bool outer_quarter(int i) { return i < S / 4 || i >= S - S / 4; }

// Line transforms with an explicit split N = S1 x S2 over lines whose element e
// sits at loff(l) + e es; consecutive threads take consecutive lines.  PIN:
// only inputs S2 n1 + n2 with n1 in the outer quarters of S1 are nonzero; POUT:
// only outputs k1 + S1 k2 with k2 in the outer quarters of S2 are stored.
template <int N, int S1, int S2, int DIR, int NT, bool PIN, bool POUT, class Off, class C>
WB_DEV void fft_lines_split(C* data, Off loff, int es, int nlines, const C* tw) {
  static_assert(!PIN || S1 % 4 == 0, "input pruning needs S1 % 4 == 0");
  static_assert(!POUT || S2 % 4 == 0, "output pruning needs S2 % 4 == 0");
  for (int it = threadIdx.x; it < nlines * S2; it += NT) {
    const int line = it % nlines, n2 = it / nlines;
    C* p = data + loff(line);
    C v[S1];
#pragma unroll
    for (int n1 = 0; n1 < S1; ++n1)
      v[n1] = (PIN && !outer_quarter<S1>(n1)) ? mkc<C>(0, 0) : p[(S2 * n1 + n2) * es];
    rdft<S1, DIR, N>(v, tw);
#pragma unroll
    for (int k1 = 1; k1 < S1; ++k1) v[k1] = ctw<DIR>(v[k1], tw_step1<N, S1, S2>(tw, k1, n2));
#pragma unroll
    for (int k1 = 0; k1 < S1; ++k1) p[(S2 * k1 + n2) * es] = v[k1];
  }
  __syncthreads();
  constexpr int LPC = NT / S1;
  const int nch = (nlines + LPC - 1) / LPC;
  for (int c = 0; c < nch; ++c) {
    const int line = c * LPC + (int)threadIdx.x % LPC, k1 = (int)threadIdx.x / LPC;
    const bool act = (int)threadIdx.x < LPC * S1 && line < nlines;
    C* p = data + (act ? loff(line) : 0);
    C v[S2];
    if (act) {
#pragma unroll
      for (int n2 = 0; n2 < S2; ++n2) v[n2] = p[(S2 * k1 + n2) * es];
      rdft<S2, DIR, N>(v, tw);
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int k2 = 0; k2 < S2; ++k2)
        if (!POUT || outer_quarter<S2>(k2)) p[(k1 + S1 * k2) * es] = v[k2];
    }
  }
  __syncthreads();
}

// Rows, phase 2: the inverse step 2 (B-point DFT of thread k1), V(r)/N^3 and the
// forward step 1 of the split (B, A) with its twiddles, written back in place.
template <int N, int NT, class C>
WB_DEV void rows_vloc_middle(C* pl, const C* tw, const real_t<C>* __restrict__ vz) {
  constexpr int A = FftSplit<N>::N1, B = FftSplit<N>::N2;
  using LP = LinePad<N>;
  using T = real_t<C>;
  for (int it = threadIdx.x; it < N * A; it += NT) {
    const int y = it / A, k1 = it % A;
    C* p = pl + Plane<N>::row(y);
    T vr[B];
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) vr[k2] = __ldg(vz + y * N + k1 + A * k2);
    C v[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) v[n2] = p[LP::off_blk(k1, n2)];
    rdft<B, +1, N>(v, tw);                          // X[k1 + A k2]
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) v[k2] = cscale(v[k2], vr[k2]);
    rdft<B, -1, N>(v, tw);                          // forward step 1, n2' = k1
#pragma unroll
    for (int q = 1; q < B; ++q) v[q] = ctw<-1>(v[q], tw_step1<N, B, A>(tw, q, k1));
#pragma unroll
    for (int q = 0; q < B; ++q) p[LP::off_blk(k1, q)] = v[q];
  }
}

// Threads per row in the row phases 1 and 3 (B of them work): A when A > B, so
// that a row's lanes never share a quarter-warp (FP64) or half-warp (FP32) with
// the next row's in a way that lands two on one bank (9-lane rows at 108^3 gave
// 2-way conflicts; 12-lane slots with the row stride 108 give none)
template <int N>
constexpr int row_slot() { return FftSplit<N>::N1 > FftSplit<N>::N2 ? FftSplit<N>::N1 : FftSplit<N>::N2; }

// Rows, phase 1: the inverse step 1 of the split (A, B): thread n2 < B of a row
// takes x = B n1 + n2 (pruned inputs in the outer quarters of A), A-point DFT,
// twiddles, back to the same positions.
template <int N, int NT, bool PIN, class C>
WB_DEV void rows_inverse_step1(C* pl, const C* tw) {
  constexpr int A = FftSplit<N>::N1, B = FftSplit<N>::N2, S = row_slot<N>();
  static_assert(!PIN || A % 4 == 0, "input pruning needs A % 4 == 0");
  using LP = LinePad<N>;
  for (int it = threadIdx.x; it < N * S; it += NT) {
    const int y = it / S, n2 = it % S;
    if (n2 >= B) continue;
    C* p = pl + Plane<N>::row(y);
    C v[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1)
      v[n1] = (PIN && !outer_quarter<A>(n1)) ? mkc<C>(0, 0) : p[LP::off_blk(n1, n2)];
    rdft<A, +1, N>(v, tw);
#pragma unroll
    for (int k1 = 1; k1 < A; ++k1) v[k1] = ctw<+1>(v[k1], tw_step1<N, A, B>(tw, k1, n2));
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) p[LP::off_blk(k1, n2)] = v[k1];
  }
}

// Rows, phase 3: the forward step 2 of the split (B, A): thread k1' < B takes
// Y[k1', n2'] from off_blk(n2', k1') and writes output k1' + B k2' to
// off_blk(k2', k1'), the positions it read.
template <int N, int NT, bool POUT, class C>
WB_DEV void rows_forward_step2(C* pl, const C* tw) {
  constexpr int A = FftSplit<N>::N1, B = FftSplit<N>::N2, S = row_slot<N>();
  static_assert(!POUT || A % 4 == 0, "output pruning of the transposed split needs A % 4 == 0");
  using LP = LinePad<N>;
  for (int it = threadIdx.x; it < N * S; it += NT) {
    const int y = it / S, k1 = it % S;
    if (k1 >= B) continue;
    C* p = pl + Plane<N>::row(y);
    C v[A];
#pragma unroll
    for (int n2 = 0; n2 < A; ++n2) v[n2] = p[LP::off_blk(n2, k1)];
    rdft<A, -1, N>(v, tw);
#pragma unroll
    for (int k2 = 0; k2 < A; ++k2)
      if (!POUT || outer_quarter<A>(k2)) p[LP::off_blk(k2, k1)] = v[k2];
  }
}

template <int N, class C>
static constexpr size_t psmem_c() { return sizeof(C) * (2 * N + Plane<N>::SIZE); }
// threads per CTA of the one-pass kernel: 512 in FP32 (two CTAs of 56
// registers per thread fit an SM up to 108^3) and in FP64 where the plane
// allows only one CTA per SM (from 80^3 up), 256 otherwise
template <int N, class C>
constexpr int gen_threads() {
  return (sizeof(C) == 8 || 2 * psmem_c<N, C>() > 227u * 1024u) ? 512 : 256;
}

template <int N, bool PR, class C>
__global__ void __launch_bounds__(gen_threads<N, C>(), sizeof(C) == 8 ? 2 : 1) k_plane_vloc_gen(C* __restrict__ sticks, StickTab st,
                                                                         const real_t<C>* __restrict__ vs,
                                                                         const C* __restrict__ twg, const int* dn) {
  constexpr int NT = gen_threads<N, C>();
  constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
  constexpr bool RP = PR && (N1 % 4 == 0);  // pruned rows and columns, both directions
  if (dn && (int)blockIdx.y >= dev_count<true>(dn, 0)) return;
  C* tw = smem_tw<C>();
  C* pl = smem_tw<C>() + 2 * N;
  const int z = blockIdx.x, item = blockIdx.y;
  C* sz = sticks + ((long)item * N + z) * st.nst;
  load_tw<N>(tw, twg);
  plane_zero<N, PR, C, Plane<N>, NT>(pl, st);
  __syncthreads();
  plane_scatter<N, C, Plane<N>, NT>(pl, sz, st.st_pos, st.nst);
  __syncthreads();
  const OffCols<N> cols{st.xhi + 1, st.ncols};
  fft_lines_split<N, N1, N2, +1, NT, RP, false>(pl, cols, Plane<N>::RS, st.ncols, tw);
  rows_inverse_step1<N, NT, RP>(pl, tw);
  __syncthreads();
  rows_vloc_middle<N, NT>(pl, tw, vs + (long)z * N * N);
  __syncthreads();
  rows_forward_step2<N, NT, RP>(pl, tw);
  __syncthreads();
  if constexpr (RP) fft_lines_split<N, N2, N1, -1, NT, false, true>(pl, cols, Plane<N>::RS, st.ncols, tw);
  else fft_lines_split<N, N1, N2, -1, NT, false, false>(pl, cols, Plane<N>::RS, st.ncols, tw);
  plane_gather<N, C, Plane<N>, NT>(pl, sz, st.st_pos, st.nst);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <int N, class C = double2>
static constexpr size_t zsmem() { return sizeof(C) * (2 * N + 2 * ZSG * (LinePad<N>::LEN | 1)); }
template <int N, class C = double2>
static constexpr size_t psmem() { return sizeof(C) * (2 * N + Plane<N>::SIZE); }
template <int N, class C>
static constexpr size_t fsmem() { return sizeof(C) * (2 * N + FPlane<N, C>::SIZE); }

template <int N>
struct FftN {
  static constexpr bool FUSABLE = FftSplit<N>::N1 == FftSplit<N>::N2 && Prune<N>::IN_OK && Prune<N>::OUT_OK;
  template <bool PR>
  static void setup_pr() {
    cudaFuncSetAttribute(k_zinv<N, PR, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N>());
    cudaFuncSetAttribute(k_zfwd<N, PR, double2, EpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N>());
    cudaFuncSetAttribute(k_zfwd<N, PR, double2, EpiHpsi>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N>());
    cudaFuncSetAttribute(k_zfwd<N, PR, double2, EpiDng>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N>());
    cudaFuncSetAttribute(k_plane_vloc<N, PR, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem<N>());
    cudaFuncSetAttribute(k_plane_inv_box<N, PR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem<N>());
    cudaFuncSetAttribute(k_plane_rhs<N, PR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem<N>());
    cudaFuncSetAttribute(k_plane_drho<N, PR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem<N>());
  }
  static void setup() {
    setup_pr<false>();
    setup_pr<true>();
    if constexpr (FUSABLE) {
      cudaFuncSetAttribute(k_plane_vloc_fused<N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)fsmem<N, double2>());
      cudaFuncSetAttribute(k_plane_vloc_fused<N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)fsmem<N, float2>());
    }
    cudaFuncSetAttribute(k_plane_vloc_gen<N, false, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)psmem_c<N, double2>());
    cudaFuncSetAttribute(k_plane_vloc_gen<N, true, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)psmem_c<N, double2>());
    cudaFuncSetAttribute(k_plane_vloc_gen<N, false, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)psmem_c<N, float2>());
    cudaFuncSetAttribute(k_plane_vloc_gen<N, true, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)psmem_c<N, float2>());
    for (int pr = 0; pr < 2; ++pr) {
      auto zi = pr ? k_zinv<N, true, float2> : k_zinv<N, false, float2>;
      auto zf = pr ? k_zfwd<N, true, float2, EpiHpsi32> : k_zfwd<N, false, float2, EpiHpsi32>;
      auto pv = pr ? k_plane_vloc<N, true, float2> : k_plane_vloc<N, false, float2>;
      cudaFuncSetAttribute(zi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N, float2>());
      cudaFuncSetAttribute(zf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N, float2>());
      cudaFuncSetAttribute(pv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem<N, float2>());
    }
  }
  static dim3 zgrid(const StickTab& st, int nitems) { return dim3((st.nsp + ZSG - 1) / ZSG, nitems); }
  // one-pass plane kernels: the register-row kernel for 8 x 8 and 4 x 4 splits
  // (pruned, sticks preloaded into registers), the generic one for every other
  // box and stick table
  static bool fused_square(const StickTab& st) {
    if constexpr (FUSABLE) return st.prune && st.nst <= kFusedMaxSticksPerThread * PNT;
    return false;
  }
  static bool fused(const StickTab&) { return true; }
  template <class F>
  static bool use_fused(const F& f) { return !f.unfused; }
  // Local-potential transforms of the PCG operator, FP64 (C = double2) or the
  // FP32 inner solves (C = float2): one CTA per (stick group or plane, item);
  // with a device count (graph replays) nitems is the bound the grid is sized
  // for and the CTAs beyond the device count return at once.
  template <class C, class F>
  static void zinv_t(const F& f, const C* src, long ld, const int2* items, int nitems, C* sticks) {
    if (nitems <= 0) return;
    constexpr size_t zs = zsmem<N, C>();
    if (f.st.prune)
      k_zinv<N, true, C><<<zgrid(f.st, nitems), ZNT, zs, f.stream>>>(src, ld, items, f.st, sticks, f.tw, f.dcount);
    else
      k_zinv<N, false, C><<<zgrid(f.st, nitems), ZNT, zs, f.stream>>>(src, ld, items, f.st, sticks, f.tw, f.dcount);
  }
  template <class C, class F>
  static void vloc_t(const F& f, C* sticks, int nitems, const real_t<C>* vs) {
    if (nitems <= 0) return;
    constexpr size_t ps = psmem<N, C>();
    const dim3 g(N, nitems);
    if (use_fused(f)) {
      if constexpr (FUSABLE) {
        if (fused_square(f.st)) {
          k_plane_vloc_fused<N, C><<<g, PNT, fsmem<N, C>(), f.stream>>>(sticks, f.st, vs, f.tw, f.dcount);
          return;
        }
      }
      constexpr int gnt = gen_threads<N, C>();
      if (f.st.prune)
        k_plane_vloc_gen<N, true, C><<<g, gnt, psmem_c<N, C>(), f.stream>>>(sticks, f.st, vs, f.tw, f.dcount);
      else
        k_plane_vloc_gen<N, false, C><<<g, gnt, psmem_c<N, C>(), f.stream>>>(sticks, f.st, vs, f.tw, f.dcount);
      return;
    }
    if (f.st.prune) k_plane_vloc<N, true, C><<<g, PNT, ps, f.stream>>>(sticks, f.st, vs, f.tw, f.dcount);
    else k_plane_vloc<N, false, C><<<g, PNT, ps, f.stream>>>(sticks, f.st, vs, f.tw, f.dcount);
  }
  template <class C, class F, class Epi>
  static void zfwd_t(const F& f, const C* sticks, const int2* items, int nitems, Epi epi) {
    if (nitems <= 0) return;
    constexpr size_t zs = zsmem<N, C>();
    if (f.st.prune)
      k_zfwd<N, true, C, Epi><<<zgrid(f.st, nitems), ZNT, zs, f.stream>>>(sticks, items, f.st, f.tw, epi, f.dcount);
    else
      k_zfwd<N, false, C, Epi><<<zgrid(f.st, nitems), ZNT, zs, f.stream>>>(sticks, items, f.st, f.tw, epi, f.dcount);
  }
  static void zinv32(const FftArgs32& f, const float2* src, long ld, const int2* items, int nitems, float2* sticks) {
    zinv_t<float2>(f, src, ld, items, nitems, sticks);
  }
  static void vloc32(const FftArgs32& f, float2* sticks, int nitems, const float* vs) {
    vloc_t<float2>(f, sticks, nitems, vs);
  }
  static void zfwd_hpsi32(const FftArgs32& f, const float2* sticks, const int2* items, int nitems, EpiHpsi32 epi) {
    zfwd_t<float2>(f, sticks, items, nitems, epi);
  }
  static void zinv(const FftArgs& f, const double2* src, long ld, const int2* items, int nitems, double2* sticks) {
    zinv_t<double2>(f, src, ld, items, nitems, sticks);
  }
  template <class Epi>
  static void zfwd(const FftArgs& f, const double2* sticks, const int2* items, int nitems, Epi epi) {
    zfwd_t<double2>(f, sticks, items, nitems, epi);
  }
  static void vloc(const FftArgs& f, double2* sticks, int nitems, const double* vs) {
    vloc_t<double2>(f, sticks, nitems, vs);
  }
  static void inv_box(const FftArgs& f, const double2* sticks, int nitems, double2* box) {
    if (nitems <= 0) return;
    const dim3 g(N, nitems);
    if (f.st.prune) k_plane_inv_box<N, true><<<g, PNT, psmem<N>(), f.stream>>>(sticks, f.st, box, f.tw);
    else k_plane_inv_box<N, false><<<g, PNT, psmem<N>(), f.stream>>>(sticks, f.st, box, f.tw);
  }
  static void rhs(const FftArgs& f, const double2* evcr, const double2* dvbox, int npv, int mb, double2* sticks) {
    if (mb <= 0) return;
    const dim3 g(N, mb);
    if (f.st.prune)
      k_plane_rhs<N, true><<<g, rd_threads<N>(), psmem<N>(), f.stream>>>(evcr, dvbox, npv, f.st, sticks, f.tw);
    else
      k_plane_rhs<N, false><<<g, rd_threads<N>(), psmem<N>(), f.stream>>>(evcr, dvbox, npv, f.st, sticks, f.tw);
  }
  static void drho(const FftArgs& f, const double2* dsticks, const double2* evcr, const double* occ, int nocc,
                   int mb, double2* acc, double scale, double2* osticks) {
    if (mb <= 0) return;
    const dim3 g(N, (mb + 1) / 2);
    if (f.st.prune)
      k_plane_drho<N, true><<<g, rd_threads<N>(), psmem<N>(), f.stream>>>(dsticks, evcr, occ, nocc, mb, f.st, acc,
                                                                          scale, osticks, f.tw);
    else
      k_plane_drho<N, false><<<g, rd_threads<N>(), psmem<N>(), f.stream>>>(dsticks, evcr, occ, nocc, mb, f.st, acc,
                                                                           scale, osticks, f.tw);
  }
};

#define WB_FOR_EACH_N(X) X(16) X(20) X(24) X(32) X(36) X(40) X(48) X(60) X(64) X(72) X(80) X(96) X(100) X(108)

bool fft_fusable(int n, const StickTab& st) {
  switch (n) {
#define X(n) case n: return FftN<n>::fused(st);
    WB_FOR_EACH_N(X)
#undef X
    default: return false;
  }
}

int fft_plane_offset(int n, bool fused, int elem_bytes, int x, int y) {
  switch (n) {
#define X(n)                                                                                  \
  case n:                                                                                     \
    if (!fused) return Plane<n>::at(x, y);                                                    \
    return elem_bytes == 8 ? FPlane<n, float2>::at(x, y) : FPlane<n, double2>::at(x, y);
    WB_FOR_EACH_N(X)
#undef X
    default: return 0;
  }
}

bool fft_supported(int n) {
  switch (n) {
#define X(n) case n: return true;
    WB_FOR_EACH_N(X)
#undef X
    default: return false;
  }
}

void fft_setup(int n) {
  switch (n) {
#define X(n) case n: FftN<n>::setup(); break;
    WB_FOR_EACH_N(X)
#undef X
    default: break;
  }
}

#define WB_DISPATCH(n, call) \
  switch (n) {               \
    WB_FOR_EACH_N(X)         \
    default: break;          \
  }

void fft_zinv(const FftArgs& f, const double2* src, long ld, const int2* items, int nitems, double2* sticks) {
  if (f.rt) return rt_zinv(f, src, ld, items, nitems, sticks);
#define X(n) case n: FftN<n>::zinv(f, src, ld, items, nitems, sticks); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_zfwd_store(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dst, long ld) {
  if (f.rt) return rt_zfwd_store(f, sticks, items, nitems, dst, ld);
#define X(n) case n: FftN<n>::zfwd(f, sticks, items, nitems, EpiStore{dst, ld}); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_zfwd_hpsi(const FftArgs& f, const double2* sticks, const int2* items, int nitems, const double2* P,
                   double2* T, long ld, const double* g2kin, const double* ecol) {
  if (f.rt) return rt_zfwd_hpsi(f, sticks, items, nitems, P, T, ld, g2kin, ecol);
#define X(n) case n: FftN<n>::zfwd(f, sticks, items, nitems, EpiHpsi{P, T, ld, g2kin, ecol}); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_zfwd_dng(const FftArgs& f, const double2* sticks, const int2* items, int nitems, double2* dng, long ld,
                  const int* perm, const double* sqvc) {
  if (f.rt) return rt_zfwd_dng(f, sticks, items, nitems, dng, ld, perm, sqvc);
#define X(n) case n: FftN<n>::zfwd(f, sticks, items, nitems, EpiDng{dng, ld, perm, sqvc}); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_zinv32(const FftArgs32& f, const float2* src, long ld, const int2* items, int nitems, float2* sticks) {
  if (f.rt) return rt_zinv32(f, src, ld, items, nitems, sticks);
#define X(n) case n: FftN<n>::zinv32(f, src, ld, items, nitems, sticks); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_plane_vloc32(const FftArgs32& f, float2* sticks, int nitems, const float* vs) {
  if (f.rt) return rt_plane_vloc32(f, sticks, nitems, vs);
#define X(n) case n: FftN<n>::vloc32(f, sticks, nitems, vs); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_zfwd_hpsi32(const FftArgs32& f, const float2* sticks, const int2* items, int nitems, const float2* P,
                     float2* T, long ld, const float* g2kin, const float* ecol) {
  if (f.rt) return rt_zfwd_hpsi32(f, sticks, items, nitems, P, T, ld, g2kin, ecol);
#define X(n) case n: FftN<n>::zfwd_hpsi32(f, sticks, items, nitems, EpiHpsi32{P, T, ld, g2kin, ecol}); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_plane_vloc(const FftArgs& f, double2* sticks, int nitems, const double* vs) {
  if (f.rt) return rt_plane_vloc(f, sticks, nitems, vs);
#define X(n) case n: FftN<n>::vloc(f, sticks, nitems, vs); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_plane_inv_box(const FftArgs& f, const double2* sticks, int nitems, double2* box) {
  if (f.rt) return rt_plane_inv_box(f, sticks, nitems, box);
#define X(n) case n: FftN<n>::inv_box(f, sticks, nitems, box); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_plane_rhs(const FftArgs& f, const double2* evcr, const double2* dvbox, int npv, int mb, double2* sticks) {
  if (f.rt) return rt_plane_rhs(f, evcr, dvbox, npv, mb, sticks);
#define X(n) case n: FftN<n>::rhs(f, evcr, dvbox, npv, mb, sticks); break;
  WB_DISPATCH(f.n, )
#undef X
}
void fft_plane_drho(const FftArgs& f, const double2* dsticks, const double2* evcr, const double* occ, int nocc,
                    int mb, double2* acc, double scale, double2* osticks) {
  if (f.rt) return rt_plane_drho(f, dsticks, evcr, occ, nocc, mb, acc, scale, osticks);
#define X(n) case n: FftN<n>::drho(f, dsticks, evcr, occ, nocc, mb, acc, scale, osticks); break;
  WB_DISPATCH(f.n, )
#undef X
}

}  // namespace wb
