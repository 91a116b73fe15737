// C ABI and host orchestration of the B200 response operator.
//
// The per-call pipeline replaces dfpt (DFPT_kernel/dfpt_module.f90:22-533) for
// a whole batch of perturbations at once instead of one perturbation at a
// time: all (perturbation, occupied band) Sternheimer systems run the masked
// PCG of linsolve_sternheimer_m_wfcts together, each with its own
// convergence mask, so every system follows exactly the reference's per-band
// iteration while the FFTs and GEMMs see thousands of columns per launch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "wb_ctx.h"

using namespace wb;

namespace wb {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

}  // namespace wb

namespace {

// Numbering of the stick pairs (pair 0 is (0,0)).  The plane kernels scatter
// and gather stick s of a plane from thread s % 256 of the CTA, so the order
// decides which plane offsets one warp instruction touches.  Pairs are taken
// in (y, x) order, each time the first one whose two sticks land on shared-
// memory bank slots not yet used by the current half-warp (8-byte elements,
// offset mod 16) and quarter-warp (16-byte elements, offset mod 8); when none
// fits, the next in order.
std::vector<std::pair<int, int>> stick_pair_order(int N, int prune, const std::map<std::pair<int, int>, int>& pairs) {
  const int nsp = (int)pairs.size();
  wb::StickTab shape{};
  shape.prune = prune;
  shape.nst = 2 * nsp;
  const bool fused = wb::fft_fusable(N, shape);
  std::vector<std::pair<int, int>> rest;
  for (auto& kv : pairs)
    if (kv.first.first != 0 || kv.first.second != 0) rest.push_back(kv.first);
  std::stable_sort(rest.begin(), rest.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
    return a.second != b.second ? a.second < b.second : a.first < b.first;
  });
  auto slots = [&](int x, int y, int& s16, int& s8) {
    s16 = wb::fft_plane_offset(N, fused, 8, (x + N) % N, (y + N) % N) % 16;
    s8 = wb::fft_plane_offset(N, fused, 16, (x + N) % N, (y + N) % N) % 8;
  };
  std::vector<std::pair<int, int>> order;
  order.reserve(nsp);
  order.push_back({0, 0});
  unsigned used16 = 0, used8 = 0;
  {
    int a16, a8;
    slots(0, 0, a16, a8);
    used16 = 1u << a16;
    used8 = 1u << a8;
  }
  std::vector<char> taken(rest.size(), 0);
  size_t first = 0;
  for (size_t n = 0; n < rest.size(); ++n) {
    const int lane = 2 * (int)order.size();
    if (lane % 16 == 0) used16 = 0;
    if (lane % 8 == 0) used8 = 0;
    while (taken[first]) ++first;
    size_t pick = first;
    int p16 = 0, p8 = 0, m16 = 0, m8 = 0;
    for (size_t i = first; i < rest.size(); ++i) {
      if (taken[i]) continue;
      int a16, a8, b16, b8;
      slots(rest[i].first, rest[i].second, a16, a8);
      slots(-rest[i].first, -rest[i].second, b16, b8);
      if (i == first) { p16 = a16; p8 = a8; m16 = b16; m8 = b8; }
      if (a16 != b16 && a8 != b8 && !(used16 >> a16 & 1) && !(used16 >> b16 & 1) && !(used8 >> a8 & 1) &&
          !(used8 >> b8 & 1)) {
        pick = i; p16 = a16; p8 = a8; m16 = b16; m8 = b8;
        break;
      }
    }
    taken[pick] = 1;
    used16 |= (1u << p16) | (1u << m16);
    used8 |= (1u << p8) | (1u << m8);
    order.push_back(rest[pick]);
  }
  return order;
}

template <class T>
int upload(const T* h, size_t n, DBuf& d);

int build_tables(wb_ctx* c, const wb_system* s, std::vector<int>& perm) {
  const int n1 = s->nr1, n2 = s->nr2, n3 = s->nr3, npw = s->npw;
  const long nnr = (long)n1 * n2 * n3;
  const bool rt = c->rt != 0;
  const int N = rt ? 0 : n1;  // the compiled (cubic) edge
  struct GInfo { int mx, my, mz, ref; };
  std::vector<GInfo> gi(npw);
  auto mill = [](int v, int n) { return v < (n + 1) / 2 ? v : v - n; };
  std::map<long, long> seen;
  for (int i = 0; i < npw; ++i) {
    const long b = (long)s->nl[i] - 1;
    if (b < 0 || b >= nnr) return fail(WB_ERR_ARG, "nl out of range at G " + std::to_string(i + 1));
    const int x = (int)(b % n1), y = (int)((b / n1) % n2), z = (int)(b / ((long)n1 * n2));
    gi[i] = {mill(x, n1), mill(y, n2), mill(z, n3), i};
    if (2 * std::abs(gi[i].mx) >= n1 || 2 * std::abs(gi[i].my) >= n2 || 2 * std::abs(gi[i].mz) >= n3)
      return fail(WB_ERR_ARG, "G sphere reaches the box edge (aliasing) at G " + std::to_string(i + 1));
    const long bm = (long)s->nlm[i] - 1;
    const long want = ((-gi[i].mx + n1) % n1) + (long)n1 * (((-gi[i].my + n2) % n2) + (long)n2 * ((-gi[i].mz + n3) % n3));
    if (bm != want) return fail(WB_ERR_ARG, "nlm is not the box index of -G at G " + std::to_string(i + 1));
    if (seen.count(b) || (i > 0 && seen.count(bm)))
      return fail(WB_ERR_ARG, "G and -G both stored (not a Gamma half sphere) at G " + std::to_string(i + 1));
    seen[b] = i;
  }
  if (gi[0].mx != 0 || gi[0].my != 0 || gi[0].mz != 0) return fail(WB_ERR_ARG, "first G vector must be G=0");
  // stick pairs: canonical stick (x > 0) or (x == 0, y > 0); (0,0) is pair 0
  auto canon = [](int x, int y, int& cx, int& cy, int& side) {
    if (x > 0 || (x == 0 && y > 0) || (x == 0 && y == 0)) { cx = x; cy = y; side = 0; }
    else { cx = -x; cy = -y; side = 1; }
  };
  std::map<std::pair<int, int>, int> pairs;
  pairs[{0, 0}] = 0;
  for (auto& g : gi) {
    int cx, cy, sd;
    canon(g.mx, g.my, cx, cy, sd);
    if (cx == 0 && cy == 0) continue;
    pairs.emplace(std::make_pair(cx, cy), 0);
  }
  const int nsp = (int)pairs.size();
  int mmax = 0;
  for (auto& g : gi) mmax = std::max({mmax, std::abs(g.mx), std::abs(g.my), std::abs(g.mz)});
  const int prune = (!rt && 4 * mmax < N && N % 4 == 0) ? 1 : 0;
  std::vector<std::pair<int, int>> pair_xy;
  if (!rt) {
    pair_xy = stick_pair_order(N, prune, pairs);
  } else {  // the runtime-size path: pairs in (y, x) order
    for (auto& kv : pairs) pair_xy.push_back(kv.first);
    std::stable_sort(pair_xy.begin() + 1, pair_xy.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
      return a.second != b.second ? a.second < b.second : a.first < b.first;
    });
  }
  for (int p = 1; p < nsp; ++p) pairs[pair_xy[p]] = p;
  std::vector<int> gq(npw), gside(npw);
  int xmax = 0;
  for (int i = 0; i < npw; ++i) {
    int cx, cy, sd;
    canon(gi[i].mx, gi[i].my, cx, cy, sd);
    gq[i] = pairs[{cx, cy}];
    gside[i] = (gq[i] == 0) ? 0 : sd;
    xmax = std::max(xmax, std::abs(gi[i].mx));
  }
  std::vector<int> order(npw);
  for (int i = 0; i < npw; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (gq[a] != gq[b]) return gq[a] < gq[b];
    const int za = gq[a] == 0 ? std::abs(gi[a].mz) : gi[a].mz;
    const int zb = gq[b] == 0 ? std::abs(gi[b].mz) : gi[b].mz;
    return za < zb;
  });
  perm.assign(order.begin(), order.end());  // internal -> reference
  std::vector<int> spg(nsp + 1, 0);
  std::vector<int2> gqz(npw);
  for (int i = 0; i < npw; ++i) {
    const int r = order[i];
    spg[gq[r] + 1]++;
    gqz[i] = make_int2(2 * gq[r] + gside[r], gi[r].mz);
  }
  for (int p = 0; p < nsp; ++p) spg[p + 1] += spg[p];
  const int nst = 2 * nsp;
  std::vector<int> stpos(nst, -1);
  if (!rt) {
    for (int p = 0; p < nsp; ++p) {
      const int x = pair_xy[p].first, y = pair_xy[p].second;
      stpos[2 * p] = ((y + N) % N) * N + ((x + N) % N);
      if (p > 0) stpos[2 * p + 1] = ((-y + N) % N) * N + ((-x + N) % N);
    }
  } else {
    // active columns: every x of a stick or its mirror, x in [-xmax, xmax]
    const int ncols = 2 * xmax + 1, cs = n2 | 1;
    std::vector<int> colx(ncols);
    for (int cidx = 0; cidx < ncols; ++cidx) colx[cidx] = (cidx - xmax + n1) % n1;
    auto col_of = [&](int x) { return x + xmax; };
    for (int p = 0; p < nsp; ++p) {
      const int x = pair_xy[p].first, y = pair_xy[p].second;
      stpos[2 * p] = col_of(x) * cs + (y + n2) % n2;
      if (p > 0) stpos[2 * p + 1] = col_of(-x) * cs + (-y + n2) % n2;
    }
    c->geo.ncols = ncols;
    c->geo.cs = cs;
    if (upload(colx.data(), colx.size(), c->rt_colx)) return fail(WB_ERR_NOMEM, "device allocation failed");
  }
  // device copies
  if (c->gqz.ensure(sizeof(int2) * npw) || c->spg.ensure(sizeof(int) * (nsp + 1)) ||
      c->stpos.ensure(sizeof(int) * nst) || c->perm.ensure(sizeof(int) * npw))
    return fail(WB_ERR_NOMEM, "device allocation of stick tables failed");
  WB_CU(cudaMemcpy(c->gqz.p, gqz.data(), sizeof(int2) * npw, cudaMemcpyHostToDevice));
  WB_CU(cudaMemcpy(c->spg.p, spg.data(), sizeof(int) * (nsp + 1), cudaMemcpyHostToDevice));
  WB_CU(cudaMemcpy(c->stpos.p, stpos.data(), sizeof(int) * nst, cudaMemcpyHostToDevice));
  WB_CU(cudaMemcpy(c->perm.p, perm.data(), sizeof(int) * npw, cudaMemcpyHostToDevice));
  c->st.nsp = nsp;
  c->st.nst = nst;
  c->st.sp_gstart = c->spg.as<int>();
  c->st.g_qz = c->gqz.as<int2>();
  c->st.st_pos = c->stpos.as<int>();
  c->st.xhi = xmax;
  c->st.ncols = 2 * xmax + 1;
  c->st.prune = prune;
  if (c->st.prune) {
    // pruned transforms read every x in the outer quarters, so those columns
    // are the active set (they are all zero-filled and transformed)
    c->st.xhi = N / 4 - 1;
    c->st.ncols = N / 2;
  }
  if (rt) {
    c->geo.colx = c->rt_colx.as<int>();
    c->geo.spos = c->stpos.as<int>();
  }
  return WB_OK;
}

// Upload a [ld, ncol] complex host array into internal order [ncol][npw].
int upload_cols(const double* h, int ld, int ncol, const std::vector<int>& perm, DBuf& d) {
  const int npw = (int)perm.size();
  std::vector<double2> tmp((size_t)npw * ncol);
  for (int j = 0; j < ncol; ++j)
    for (int i = 0; i < npw; ++i) {
      const double* src = h + 2 * ((size_t)j * ld + perm[i]);
      tmp[(size_t)j * npw + i] = make_double2(src[0], src[1]);
    }
  if (d.ensure(sizeof(double2) * tmp.size() + 16)) return fail(WB_ERR_NOMEM, "device allocation failed");
  WB_CU(cudaMemcpy(d.p, tmp.data(), sizeof(double2) * tmp.size(), cudaMemcpyHostToDevice));
  return WB_OK;
}

template <class T>
int upload(const T* h, size_t n, DBuf& d) {
  if (d.ensure(sizeof(T) * n + 16)) return fail(WB_ERR_NOMEM, "device allocation failed");
  WB_CU(cudaMemcpy(d.p, h, sizeof(T) * n, cudaMemcpyHostToDevice));
  return WB_OK;
}

// Accounts one pipeline stage: launches and work items always, device time
// when profiling is on.
struct Stage {
  wb_ctx* c;
  int st, e0 = -1;
  Stage(wb_ctx* c_, int st_, int launches, long long items) : c(c_), st(st_) {
    c->stats.stage_launches[st] += launches;
    c->stats.stage_items[st] += items;
    c->stats.launches += launches;
    if (c->prof & (1 << st)) {
      e0 = c->ev_get();
      if (e0 >= 0) cudaEventRecord(c->evpool[e0], c->stream);
    }
  }
  ~Stage() {
    if (e0 < 0) return;
    const int e1 = c->ev_get();
    if (e1 < 0) return;
    cudaEventRecord(c->evpool[e1], c->stream);
    c->marks.push_back({st, e0, e1});
  }
};

void resolve_marks(wb_ctx* c) {
  for (auto& mk : c->marks) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->evpool[mk.e0], c->evpool[mk.e1]) == cudaSuccess) c->stats.stage_ms[mk.stage] += ms;
  }
  c->marks.clear();
  c->evused = 0;
}

void pair_items(std::vector<int2>& it, int base, int n) {
  for (int k = 0; k < (n + 1) / 2; ++k) it.push_back(make_int2(base + 2 * k, (2 * k + 1 < n) ? base + 2 * k + 1 : -1));
}

size_t per_pert_bytes(const wb_ctx* c) {
  const size_t vec = sizeof(double2) * (size_t)c->npw * c->nocc;
  const size_t stk = sizeof(double2) * (size_t)c->nz * c->st.nst;
  const size_t mixed = c->precision == WB_PRECISION_MIXED ? 2 * vec + stk * (size_t)c->npv / 2 : 0;
  return mixed + 4 * vec                           // B, X, G, T (+ FP32 g, P, T, d and sticks)
         + stk * (size_t)c->npv                    // sticks (RHS / CG pairs / drho items)
         + sizeof(double2) * (size_t)c->nnr * 1    // dvbox + acc (one box per two perturbations each)
         + stk                                     // sticks2 (half per perturbation, rounded up)
         + sizeof(double) * (size_t)c->nocc * c->nproj * 9  // GEMM partials and coefficients
         + 2 * sizeof(double2) * (size_t)c->npw;   // aux, input/output staging
}

int choose_batch(wb_ctx* c, int m) {
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  const size_t budget = (size_t)(0.6 * (double)freeb);
  int mb = (int)std::max<size_t>(2, budget / std::max<size_t>(1, per_pert_bytes(c)));
  mb = std::min(mb, m);
  if (c->batch_cap > 0) mb = std::min(mb, c->batch_cap);
  return std::max(mb, 1);
}

int ensure_workspace(wb_ctx* c, int mb, long ld_in, long ld_out) {
  const size_t nsys = (size_t)std::max(mb * c->nocc, c->cap_nsys);
  c->cap_nsys = (int)nsys;
  mb = (int)(nsys / c->nocc);
  const size_t vec = sizeof(double2) * (size_t)c->npw * nsys;
  const size_t stk1 = sizeof(double2) * (size_t)c->nz * c->st.nst;
  const size_t mp = (mb + 1) / 2;
  const size_t nitems = std::max<size_t>({(nsys + 1) / 2, (size_t)mb * c->npv, mp, (size_t)c->npv});
  const int nsplit = gemm_tn_splits(c->nproj, (int)nsys, 2 * c->npw, 4);  // the tuner's largest target
  bool bad = false;
  bad |= c->dvg_in.ensure(sizeof(double2) * ld_in * mb + 16) != 0;
  bad |= c->dng_out.ensure(sizeof(double2) * ld_out * mb + 16) != 0;
  bad |= c->aux.ensure(sizeof(double2) * (size_t)c->npw * mb) != 0;
  bad |= c->dvbox.ensure(sizeof(double2) * (size_t)c->nnr * mp) != 0;
  bad |= c->B.ensure(vec) || c->X.ensure(vec) || c->G.ensure(vec) || c->T.ensure(vec);
  bad |= c->sticks.ensure(stk1 * nitems) != 0;
  bad |= c->sticks2.ensure(stk1 * mp) != 0;
  bad |= c->acc.ensure(sizeof(double2) * (size_t)c->nnr * mp) != 0;
  bad |= c->part.ensure(sizeof(double) * std::max((size_t)nsplit * nsys * c->nproj,
                                                   gemm_tn_part_doubles(c->nproj, (int)nsys, 2 * c->npw, 4))) != 0;
  bad |= c->C.ensure(sizeof(double) * nsys * c->nproj) != 0;
  bad |= c->rho.ensure(sizeof(double) * nsys) != 0;
  bad |= c->conv.ensure(nsys + 16) != 0;
  bad |= c->act.ensure(sizeof(int) * nsys) != 0;
  bad |= c->items.ensure(sizeof(int2) * (nsys / 2 + 1)) != 0;
  bad |= c->nact.ensure(sizeof(int) * 4) != 0;
  bad |= c->ecol.ensure(sizeof(double) * nsys) != 0;
  bad |= c->epcol.ensure(sizeof(double) * nsys) != 0;
  bad |= c->unconv.ensure(sizeof(int) * mb) != 0;
  bad |= c->items_pp.ensure(sizeof(int2) * mp) != 0;
  bad |= c->items_pk.ensure(sizeof(int2) * (size_t)mb * c->npv) != 0;
  if (c->nfull < c->nocc) bad |= c->fcoef.ensure(sizeof(double) * nsys * (c->nocc - c->nfull)) != 0;
  if (bad) return fail(WB_ERR_NOMEM, "device workspace allocation failed for a batch of " + std::to_string(mb));
  return WB_OK;
}

// T = (H - e + alpha Pv) X on columns cols[0..n) (pairs in items), K = 2 npw.
// ---------------------------------------------------------------------------
// autotuner: launch shapes timed on the first batch of each form
// ---------------------------------------------------------------------------
template <class F>
float time_ms(wb_ctx* c, F fn) {
  fn();  // warm-up
  float best = 3.4e38f;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(c->tev0, c->stream);
    fn();
    cudaEventRecord(c->tev1, c->stream);
    cudaEventSynchronize(c->tev1);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->tev0, c->tev1) == cudaSuccess) best = std::min(best, ms);
  }
  return best;
}

// FP64 form: split-K target of the DMMA bra-ket (1, 2 or 4 CTAs per SM) and
// the one-pass fused or two-pass plane kernel, timed on this batch's still
// unused buffers (X zeroed; sticks, part and the active list are rewritten
// by the batch afterwards).
// The two-pass plane kernel replaces the one-pass one only when it is clearly
// faster: at small boxes the two time within noise of each other, and a choice
// made by noise changed which kernel ran from one context to the next (and with
// it the rounding of every result).
constexpr float kPlaneSwitch = 0.9f;

int autotune64(wb_ctx* c, int nsys) {
  if (!c->tune.on || c->tune.done64) return WB_OK;
  c->tune.done64 = 1;
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = c->stream;
  const int K = 2 * c->npw;
  const long ld = c->npw;
  const int M = c->kinetic_only ? c->nocc : c->nproj;
  const double* W = c->W.as<double>() + (c->kinetic_only ? (size_t)c->nkb * K : 0);
  WB_CU(cudaMemsetAsync(c->X.p, 0, sizeof(double2) * ld * nsys, s));
  cg_reset(c->conv.as<unsigned char>(), nsys, s);
  cg_compact(c->conv.as<unsigned char>(), nsys, c->act.as<int>(), c->items.as<int2>(), c->nact.as<int>(), nullptr, s);
  float best = 3.4e38f;
  for (int ctas : {1, 2, 4}) {
    const int ns = gemm_tn_splits(M, nsys, K, ctas);
    const float ms = time_ms(c, [&] {
      gemm_tn(W, K, M, (const double*)c->X.p, 2 * ld, c->act.as<int>(), nsys, K, ns, c->part.as<double>(), s,
              nullptr, ctas, c->tune.dmma_pf);
    });
    if (ms < best) { best = ms; c->tune.dmma_ctas = ctas; }
  }
  if (!c->kinetic_only && fft_fusable(c->nr, c->st)) {
    FftArgs fa = c->fa;
    const int nit = (nsys + 1) / 2;
    fa.unfused = 0;
    const float tf = time_ms(c, [&] { fft_plane_vloc(fa, c->sticks.as<double2>(), nit, c->vs.as<double>()); });
    fa.unfused = 1;
    const float tu = time_ms(c, [&] { fft_plane_vloc(fa, c->sticks.as<double2>(), nit, c->vs.as<double>()); });
    c->tune.unfused64 = tu < kPlaneSwitch * tf ? 1 : 0;
  }
  WB_CU(cudaGetLastError());
  c->tune.ms += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return WB_OK;
}

// Mixed form: split-K target of the tcgen05 bra-ket (1..3 CTAs per SM), systems
// per CTA of the tcgen05 update (64 or 128) and the FP32 plane kernel variant,
// on the FP32 buffers before the inner solves use them.
int autotune32(wb_ctx* c, int nsys) {
  if (!c->tune.on || c->tune.done32) return WB_OK;
  c->tune.done32 = 1;
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = c->stream;
  const int K = 2 * c->npw;
  const long ld = c->npw;
  WB_CU(cudaMemsetAsync(c->P32.p, 0, sizeof(float2) * ld * nsys, s));
  WB_CU(cudaMemsetAsync(c->C32.p, 0, sizeof(float) * (size_t)nsys * c->umma_M, s));
  cg_reset(c->conv_in.as<unsigned char>(), nsys, s);
  cg_compact(c->conv_in.as<unsigned char>(), nsys, c->act_in.as<int>(), c->items_in.as<int2>(),
             c->nact_in.as<int>(), nullptr, s);
  if (c->umma) {
    float best = 3.4e38f;
    for (int ctas = 1; ctas <= kUmmaMaxCtas; ++ctas) {
      const float ms = time_ms(c, [&] {
        umma_braket(c->umma_braket_w.p, c->umma_M, (const float*)c->P32.p, 2 * ld, c->act_in.as<int>(), nsys, K,
                    c->part32.as<float>(), c->umma_err.as<int>(), s, nullptr, ctas);
      });
      if (ms < best) { best = ms; c->tune.umma_ctas = ctas; }
    }
    best = 3.4e38f;
    const int nrb = (umma_np(c->umma_M) + 63) / 64;
    for (int nj : {64, 128}) {
      if (nj == 128 && nrb > 2) continue;
      const float ms = time_ms(c, [&] {
        umma_update(c->umma_update_w.p, c->umma_M, c->C32.as<float>(), (float*)c->T32.p, 2 * ld, c->act_in.as<int>(),
                    nsys, K, c->umma_err.as<int>(), s, nullptr, nj);
      });
      if (ms < best) { best = ms; c->tune.update_nj = nj; }
    }
  }
  if (!c->kinetic_only && fft_fusable(c->nr, c->st)) {
    FftArgs32 fa = c->fa32;
    const int nit = (nsys + 1) / 2;
    fa.unfused = 0;
    const float tf = time_ms(c, [&] { fft_plane_vloc32(fa, c->sticks32.as<float2>(), nit, c->vs32.as<float>()); });
    fa.unfused = 1;
    const float tu = time_ms(c, [&] { fft_plane_vloc32(fa, c->sticks32.as<float2>(), nit, c->vs32.as<float>()); });
    c->tune.unfused32 = tu < kPlaneSwitch * tf ? 1 : 0;
  }
  WB_CU(cudaGetLastError());
  c->tune.ms += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return WB_OK;
}

// dn: device count of the listed columns (graph replays; n is then the maximum).
void apply_A(wb_ctx* c, const double2* Xv, double2* Tv, const int* cols, const int2* items, int n, int nsys,
             int nsplit, const int* dn = nullptr) {
  const long ld = c->npw;
  const int K = 2 * c->npw;
  cudaStream_t s = c->stream;
  FftArgs fa = c->fa;
  fa.dcount = dn;
  fa.unfused = c->tune.unfused64;
  const double* W = c->W.as<double>();
  int M = c->nproj, nkb = c->nkb;
  const double* Wsub = W;
  if (c->kinetic_only) {
    Stage g(c, WB_STAGE_VLOC_ZFWD, 1, n);
    kinetic_hpsi(Xv, Tv, c->g2kin.as<double>(), c->ecol.as<double>(), cols, n, c->npw, ld, s, dn);
    Wsub = W + (size_t)c->nkb * K;  // alpha Pv only
    M = c->nocc;
    nkb = 0;
  } else {
    const int nit = (n + 1) / 2;
    {
      Stage g(c, WB_STAGE_VLOC_ZINV, 1, nit);
      fft_zinv(fa, Xv, ld, items, nit, c->sticks.as<double2>());
    }
    {
      Stage g(c, WB_STAGE_VLOC_PLANE, 1, nit);
      fft_plane_vloc(fa, c->sticks.as<double2>(), nit, c->vs.as<double>());
    }
    {
      Stage g(c, WB_STAGE_VLOC_ZFWD, 1, nit);
      fft_zfwd_hpsi(fa, c->sticks.as<double2>(), items, nit, Xv, Tv, ld, c->g2kin.as<double>(),
                    c->ecol.as<double>());
    }
    c->stats.fft_boxes += 2 * nit;
  }
  {
    Stage g(c, WB_STAGE_GEMM_TN, 1, n);
    gemm_tn(Wsub, K, M, (const double*)Xv, 2 * ld, cols, n, K, nsplit, c->part.as<double>(), s, dn,
            c->tune.dmma_ctas, c->tune.dmma_pf);
  }
  {
    Stage g(c, WB_STAGE_GEMM_REDUCE, 1, n);
    gamma_reduce(c->part.as<double>(), nsplit, M, n, Wsub, K, (const double*)Xv, 2 * ld, cols, c->D.as<double>(),
                 nkb, c->alpha, c->C.as<double>(), s, dn, K, c->tune.dmma_ctas);
  }
  {
    Stage g(c, WB_STAGE_GEMM_NN, 1, n);
    gemm_nn(Wsub, K, M, c->C.as<double>(), (double*)Tv, 2 * ld, cols, n, K, 1.0, s, dn);
  }
  (void)nsys;
}

// ---------------------------------------------------------------------------
// mixed form: FP32 correction solves inside FP64 iterative refinement
// ---------------------------------------------------------------------------
constexpr double kInnerRhoReduction = 1e-10;  // inner PCG target: rho below 1e-10 of the outer residual's
constexpr int kMaxRefinements = 12;

int ensure_fp32(wb_ctx* c, int nsys, int nitems) {
  const int K = 2 * c->npw;
  if (!c->have32) {
    if (c->W32.ensure(sizeof(float) * (size_t)K * c->nproj + 16) || c->D32.ensure(sizeof(float) * std::max(1, c->nkb * c->nkb)) ||
        c->g2kin32.ensure(sizeof(float) * c->npw) || c->vs32.ensure(sizeof(float) * (size_t)c->nnr) ||
        c->tw32.ensure(sizeof(float2) * std::max(c->nr, 1)))
      return fail(WB_ERR_NOMEM, "device allocation of FP32 constants failed");
    if (c->rt) {
      if (c->twx32.ensure(sizeof(float2) * c->geo.nx) || c->twy32.ensure(sizeof(float2) * c->geo.ny) ||
          c->twz32.ensure(sizeof(float2) * c->geo.nz))
        return fail(WB_ERR_NOMEM, "device allocation of FP32 constants failed");
      to_float(c->twx.as<double>(), c->twx32.as<float>(), 2L * c->geo.nx, c->stream);
      to_float(c->twy.as<double>(), c->twy32.as<float>(), 2L * c->geo.ny, c->stream);
      to_float(c->twz.as<double>(), c->twz32.as<float>(), 2L * c->geo.nz, c->stream);
      c->geo.twx32 = c->twx32.as<float2>();
      c->geo.twy32 = c->twy32.as<float2>();
      c->geo.twz32 = c->twz32.as<float2>();
    }
    to_float(c->W.as<double>(), c->W32.as<float>(), (long)K * c->nproj, c->stream);
    if (c->nkb) to_float(c->D.as<double>(), c->D32.as<float>(), (long)c->nkb * c->nkb, c->stream);
    to_float(c->g2kin.as<double>(), c->g2kin32.as<float>(), c->npw, c->stream);
    to_float(c->vs.as<double>(), c->vs32.as<float>(), c->nnr, c->stream);
    if (!c->rt) to_float(c->tw.as<double>(), c->tw32.as<float>(), 2L * c->nr, c->stream);
    c->fa32.n = c->nr;
    c->fa32.st = c->st;
    c->fa32.tw = c->tw32.as<float2>();
    c->fa32.stream = c->stream;
    c->fa32.rt = c->rt ? &c->geo : nullptr;
    // the projector and Pv GEMMs on tensor cores: W split once into bf16 hi/lo tiles
    const int Msub = c->kinetic_only ? c->nocc : c->nproj;
    const double* Wsub = c->W.as<double>() + (c->kinetic_only ? (size_t)c->nkb * K : 0);
    if (umma_supported(Msub)) {
      if (c->umma_braket_w.ensure(umma_braket_bytes(Msub, K)) || c->umma_update_w.ensure(umma_update_bytes(Msub, K)) ||
          c->umma_err.ensure(sizeof(int)))
        return fail(WB_ERR_NOMEM, "device allocation of the bf16 projector tiles failed");
      umma_setup();
      umma_presplit(Wsub, K, Msub, K, c->umma_braket_w.p, c->umma_update_w.p, c->stream);
      WB_CU(cudaMemsetAsync(c->umma_err.p, 0, sizeof(int), c->stream));
      WB_CU(cudaGetLastError());
      c->umma = 1;
      c->umma_M = Msub;
    }
    c->have32 = 1;
  }
  const size_t vec = sizeof(float2) * (size_t)c->npw * nsys;
  const int nsplit = gemm_tn_splits32(c->nproj, nsys, K);
  size_t part_floats = (size_t)nsplit * nsys * c->nproj;
  if (c->umma) part_floats = std::max(part_floats, umma_part_floats(c->umma_M, nsys, K));
  bool bad = false;
  bad |= c->g32.ensure(vec) || c->P32.ensure(vec) || c->T32.ensure(vec) || c->d32.ensure(vec);
  bad |= c->sticks32.ensure(sizeof(float2) * (size_t)c->nz * c->st.nst * nitems) != 0;
  bad |= c->part32.ensure(sizeof(float) * part_floats) != 0;
  bad |= c->C32.ensure(sizeof(float) * (size_t)nsys * c->nproj) != 0;
  bad |= c->ecol32.ensure(sizeof(float) * nsys) || c->rho0.ensure(sizeof(double) * nsys) ||
         c->rho_in.ensure(sizeof(double) * nsys) || c->conv_in.ensure(nsys + 16) ||
         c->act_in.ensure(sizeof(int) * nsys) || c->items_in.ensure(sizeof(int2) * (nsys / 2 + 1)) ||
         c->nact_in.ensure(sizeof(int) * 4);
  if (bad) return fail(WB_ERR_NOMEM, "device workspace allocation failed for the mixed form");
  return WB_OK;
}

// FP32 T = (H - e + alpha Pv) P on the listed columns.
void apply_A32(wb_ctx* c, const float2* Pv, float2* Tv, const int* cols, const int2* items, int n, int nsplit,
               const int* dn = nullptr) {
  const long ld = c->npw;
  const int K = 2 * c->npw;
  cudaStream_t s = c->stream;
  FftArgs32 fa = c->fa32;
  fa.dcount = dn;
  fa.unfused = c->tune.unfused32;
  const float* W = c->W32.as<float>();
  int M = c->nproj, nkb = c->nkb;
  if (c->kinetic_only) {
    Stage g(c, WB_STAGE_VLOC_ZFWD, 1, n);
    kinetic_hpsi32(Pv, Tv, c->g2kin32.as<float>(), c->ecol32.as<float>(), cols, n, c->npw, ld, s, dn);
    W += (size_t)c->nkb * K;
    M = c->nocc;
    nkb = 0;
  } else {
    const int nit = (n + 1) / 2;
    {
      Stage g(c, WB_STAGE_VLOC_ZINV, 1, nit);
      fft_zinv32(fa, Pv, ld, items, nit, c->sticks32.as<float2>());
    }
    {
      Stage g(c, WB_STAGE_VLOC_PLANE, 1, nit);
      fft_plane_vloc32(fa, c->sticks32.as<float2>(), nit, c->vs32.as<float>());
    }
    {
      Stage g(c, WB_STAGE_VLOC_ZFWD, 1, nit);
      fft_zfwd_hpsi32(fa, c->sticks32.as<float2>(), items, nit, Pv, Tv, ld, c->g2kin32.as<float>(),
                      c->ecol32.as<float>());
    }
    c->stats.fft_boxes += 2 * nit;
  }
  {
    Stage g(c, WB_STAGE_GEMM_TN, 1, n);
    if (c->umma)
      nsplit = umma_braket(c->umma_braket_w.p, M, (const float*)Pv, 2 * ld, cols, n, K, c->part32.as<float>(),
                           c->umma_err.as<int>(), s, dn, c->tune.umma_ctas);
    else
      gemm_tn32(W, K, M, (const float*)Pv, 2 * ld, cols, n, K, nsplit, c->part32.as<float>(), s, dn);
  }
  {
    Stage g(c, WB_STAGE_GEMM_REDUCE, 1, n);
    gamma_reduce32(c->part32.as<float>(), nsplit, M, n, W, K, (const float*)Pv, 2 * ld, cols, c->D32.as<float>(), nkb,
                   (float)c->alpha, c->C32.as<float>(), s, dn, K, c->umma ? c->tune.umma_ctas : 0);
  }
  {
    Stage g(c, WB_STAGE_GEMM_NN, 1, n);
    if (c->umma)
      umma_update(c->umma_update_w.p, M, c->C32.as<float>(), (float*)Tv, 2 * ld, cols, n, K, c->umma_err.as<int>(), s,
                  dn, c->tune.update_nj);
    else
      gemm_nn32_acc(W, K, M, c->C32.as<float>(), (float*)Tv, 2 * ld, cols, n, K, s, dn);
  }
}

// ---------------------------------------------------------------------------
// CUDA graphs of the PCG loops
// ---------------------------------------------------------------------------
// One masked PCG pass (operator, update + the next iteration's prec/rho,
// compaction, loop control) is captured into the body of a conditional WHILE
// node, so the whole loop runs
// from one graph launch with its convergence test on the device.  The kernels
// take the active count from device memory and size their grids for the
// workspace capacity; the graph is rebuilt when a buffer, the capacity or tr2
// changes.  Stage profiling needs host-side events and runs the loop eagerly.
bool graph_mode(const wb_ctx* c) { return c->use_graphs && c->prof == 0; }

// The graph: WHILE { k_loop_bucket -> SWITCH(bucket) { one PCG pass sized for
// up to kMinBucketItems << k band-pair items } -> k_loop_ctl }.  Each branch
// launches the same kernels as the eager loop with grids for its bucket; the
// CTAs beyond the device count return at once, so at most half a grid idles.
constexpr int kMinBucketItems = 16;

template <class Pass>
int capture_loop(wb_ctx* c, wb_ctx::LoopCache& cache, std::vector<const void*> key, double tr2, int cap,
                 const int* dn, int* st, bool shared_budget, Pass pass) {
  for (int i = 0; i < 2; ++i) {
    const wb_ctx::LoopGraph& g = cache.slot[i];
    if (g.exec && g.key == key && g.tr2 == tr2) {
      cache.last = i;
      return WB_OK;
    }
  }
  cache.last = 1 - cache.last;  // replace the least recently used graph
  wb_ctx::LoopGraph& lg = cache.slot[cache.last];
  lg.release();
  const int cap_items = (cap + 1) / 2;
  int nb = 1;
  while ((kMinBucketItems << (nb - 1)) < cap_items) ++nb;
  cudaStream_t s = c->stream;
  const wb_stats saved = c->stats;
  cudaError_t e = cudaGraphCreate(&lg.graph, 0);
  cudaGraphConditionalHandle hw, hs;
  cudaGraphNodeParams wp = {};
  cudaGraphNode_t wnode, bnode, snode;
  cudaGraph_t body = nullptr;
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hw, lg.graph, 1, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    e = cudaGraphAddNode(&wnode, lg.graph, nullptr, 0, &wp);
  }
  if (e == cudaSuccess) {
    body = wp.conditional.phGraph_out[0];
    e = cudaGraphConditionalHandleCreate(&hs, body, 0, 0);
  }
  // 1. the bucket of this pass
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    loop_bucket(hs, dn, st, kMinBucketItems, nb, s);
    cudaGraph_t g1 = nullptr;
    e = cudaStreamEndCapture(s, &g1);
  }
  size_t nn = 1;
  if (e == cudaSuccess) e = cudaGraphGetNodes(body, &bnode, &nn);
  // 2. SWITCH over the buckets, one PCG pass per branch
  cudaGraphNodeParams sp = {};
  if (e == cudaSuccess) {
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = hs;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = (unsigned)nb;
    e = cudaGraphAddNode(&snode, body, &bnode, 1, &sp);
  }
  for (int k = 0; k < nb && e == cudaSuccess; ++k) {
    e = cudaStreamBeginCaptureToGraph(s, sp.conditional.phGraph_out[k], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) break;
    pass(std::min(cap, 2 * (kMinBucketItems << k)));
    cudaGraph_t gk = nullptr;
    e = cudaStreamEndCapture(s, &gk);
  }
  // 3. loop control after the pass
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s, body, &snode, nullptr, 1, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    loop_ctl(hw, dn, st, c->maxiter, shared_budget, s);
    cudaGraph_t g3 = nullptr;
    e = cudaStreamEndCapture(s, &g3);
  }
  c->stats = saved;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&lg.exec, lg.graph, 0);
  if (e != cudaSuccess) {
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(s, &junk);
    }
    cudaGetLastError();
    lg.release();
    return fail(WB_ERR_CUDA, std::string("capture of the PCG loop: ") + cudaGetErrorString(e));
  }
  lg.key = std::move(key);
  lg.tr2 = tr2;
  return WB_OK;
}

// Adds the device loop counters of a finished graph run to the call's stats.
void loop_stats(wb_ctx* c, int passes, int launches_per_pass) {
  const long long act = *reinterpret_cast<const long long*>(c->loop_host + 4);
  const long long boxes = *reinterpret_cast<const long long*>(c->loop_host + 6);
  c->stats.cg_active_sum += act;
  c->stats.fft_boxes += c->kinetic_only ? 0 : boxes;
  c->stats.launches += (long long)passes * launches_per_pass + 2;
}

// Solves (H - e_v + alpha Pv) x_v = b_v for all systems of the batch by FP64
// iterative refinement: FP64 residual r = b - A x, the reference's test
// <r|M^-1 r> < tr2, then an FP32 masked PCG for A d = r (restarted from d = 0,
// at most n_dfpt_maxiter passes like the reference's PCG) and x += d in FP64;
// at most kMaxRefinements residuals.  X holds the initial guess on entry
// (dfpt_module.f90:348) and the solution on exit.
int cg_mixed(wb_ctx* c, int mb, double tr2, int nsplit, int* iters_out) {
  cudaStream_t s = c->stream;
  const int npw = c->npw, nocc = c->nocc, nsys = mb * nocc;
  const long ld = npw;
  const int cap = std::max(c->cap_nsys, nsys);
  int rc = ensure_fp32(c, cap, std::max((cap + 1) / 2, 1));
  if (rc) return rc;
  rc = autotune32(c, nsys);
  if (rc) return rc;
  const bool graph = graph_mode(c);
  const int nsplit32 = gemm_tn_splits32(c->nproj, graph ? cap : nsys, 2 * npw);
  int* st = c->loopst.as<int>();
  if (graph) {
    // inner PCG pass on device counts, for every refinement
    std::vector<const void*> key = {c->g32.p,   c->P32.p,    c->T32.p,   c->d32.p,    c->sticks32.p, c->act_in.p,
                                    c->items_in.p, c->nact_in.p, c->conv_in.p, c->rho_in.p, c->rho0.p,
                                    c->part32.p, c->C32.p,    c->ecol32.p, st,          (const void*)(intptr_t)cap};
    const int* dn = c->nact_in.as<int>();
    rc = capture_loop(c, c->loop32, key, tr2, cap, dn, st, true, [&](int nmax) {
      apply_A32(c, c->P32.as<float2>(), c->T32.as<float2>(), c->act_in.as<int>(), c->items_in.as<int2>(), nmax,
                nsplit32, dn);
      cg_step32(c->act_in.as<int>(), nmax, c->d32.as<float2>(), c->g32.as<float2>(), c->P32.as<float2>(),
                c->T32.as<float2>(), c->iprec.as<double>(), nocc, c->rho_in.as<double>(),
                c->conv_in.as<unsigned char>(), 0, c->maxiter, kInnerRhoReduction, c->rho0.as<double>(), tr2, npw,
                ld, s, dn, st + 1);
      cg_compact(c->conv_in.as<unsigned char>(), cap, c->act_in.as<int>(), c->items_in.as<int2>(),
                 c->nact_in.as<int>(), nullptr, s, st);
    });
    if (rc) return rc;
    loop_init(st, nsys, true, s);
  }
  double2 *B = c->B.as<double2>(), *X = c->X.as<double2>(), *T = c->T.as<double2>();
  unsigned char* conv = c->conv.as<unsigned char>();
  int* act = c->act.as<int>();
  int2* items = c->items.as<int2>();
  unsigned char* cin = c->conv_in.as<unsigned char>();
  int* ain = c->act_in.as<int>();
  int2* iin = c->items_in.as<int2>();
  to_float(c->ecol.as<double>(), c->ecol32.as<float>(), nsys, s);
  cg_reset(conv, nsys, s);
  cg_compact(conv, nsys, act, items, c->nact.as<int>(), c->nact_host, s);
  int nact = nsys, inner_total = 0;
  for (int outer = 0; outer < kMaxRefinements; ++outer) {
    apply_A(c, X, T, act, items, nact, nsys, nsplit);                    // FP64 A x
    {
      Stage g(c, WB_STAGE_CG, 2, nact);
      refine_residual(act, nact, B, T, c->iprec.as<double>(), nocc, tr2, conv, c->rho0.as<double>(),
                      c->g32.as<float2>(), c->d32.as<float2>(), npw, ld, s);
      cg_compact(conv, nsys, act, items, c->nact.as<int>(), c->nact_host, s);
    }
    // the loop counters and the tensor-core GEMMs' error word ride along with the
    // active count: the loop always leaves at this wait, with no launch after it,
    // so the last copies are final
    if (graph) WB_CU(cudaMemcpyAsync(c->loop_host, st, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (c->umma) WB_CU(cudaMemcpyAsync(c->nact_host + 1, c->umma_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    WB_CU(wb_wait(c));
    nact = *c->nact_host;
    if (graph) inner_total = c->loop_host[3];
    if (nact == 0 || outer == kMaxRefinements - 1) break;
    c->stats.refinements += 1;
    WB_CU(cudaMemcpyAsync(cin, conv, nsys, cudaMemcpyDeviceToDevice, s));
    cg_compact(cin, nsys, ain, iin, c->nact_in.as<int>(), nullptr, s);
    int nin = nact;
    // each refinement restarts the FP32 PCG from d = 0 on the FP64 residual; its
    // preconditioning stops at rho < max(1e-10 rho_outer, tr2): the first
    // correction from x0 is the reference's own PCG (same Krylov space, same test)
    if (c->maxiter > 0) {
      Stage g(c, WB_STAGE_CG, 2, nin);
      cg_prec_rho32(ain, nin, c->g32.as<float2>(), c->P32.as<float2>(), c->iprec.as<double>(), nocc,
                    c->rho_in.as<double>(), cin, 1, kInnerRhoReduction, c->rho0.as<double>(), tr2, npw, ld, s);
      cg_compact(cin, nsys, ain, iin, c->nact_in.as<int>(), graph ? nullptr : c->nact_host, s);
    }
    if (graph && c->maxiter > 0) {
      loop_init(st, nsys, false, s);
      WB_CU(cudaGraphLaunch(c->loop32.cur(), s));
    }
    for (int it = 1; !graph && it <= c->maxiter; ++it) {
      WB_CU(cudaStreamSynchronize(s));
      nin = *c->nact_host;
      if (nin == 0) break;
      ++inner_total;
      c->stats.cg_active_sum += nin;
      apply_A32(c, c->P32.as<float2>(), c->T32.as<float2>(), ain, iin, nin, nsplit32);
      {
        Stage g(c, WB_STAGE_CG, 2, nin);
        cg_step32(ain, nin, c->d32.as<float2>(), c->g32.as<float2>(), c->P32.as<float2>(), c->T32.as<float2>(),
                  c->iprec.as<double>(), nocc, c->rho_in.as<double>(), cin, it, c->maxiter, kInnerRhoReduction,
                  c->rho0.as<double>(), tr2, npw, ld, s);
        cg_compact(cin, nsys, ain, iin, c->nact_in.as<int>(), c->nact_host, s);
      }
    }
    {
      Stage g(c, WB_STAGE_CG, 1, nact);
      refine_accumulate(act, nact, X, c->d32.as<float2>(), npw, ld, s);  // x += d (FP64)
    }
  }
  {
    Stage g(c, WB_STAGE_CG, 1, mb);
    count_unconverged(conv, nocc, mb, c->unconv.as<int>(), s);
  }
  if (graph) loop_stats(c, inner_total, c->kinetic_only ? 6 : 9);
  *iters_out = inner_total;
  if (c->umma) {  // a bounded wait of a tensor-core GEMM that ran out leaves its code here
    const int e = c->nact_host[1];
    if (e) {
      cudaMemsetAsync(c->umma_err.p, 0, sizeof(int), s);
      return fail(WB_ERR_CUDA, "tensor-core GEMM wait limit reached (code " + std::to_string(e) + ")");
    }
  }
  return WB_OK;
}

int run_batch(wb_ctx* c, int mb, const double2* dvg, long ld_in, double2* dng, long ld_out, double tr2) {
  cudaStream_t s = c->stream;
  const int npw = c->npw, nocc = c->nocc, npv = c->npv;
  const int nsys = mb * nocc;
  const long ld = npw;
  const int K = 2 * npw;
  const int mp = (mb + 1) / 2;
  // item tables: perturbation pairs and (perturbation, band pair)
  std::vector<int2> ipp, ipk;
  pair_items(ipp, 0, mb);
  for (int p = 0; p < mb; ++p) pair_items(ipk, p * nocc, nocc);
  {  // through the pinned staging area, after the unconverged counts' slots
    const size_t off = ((size_t)mb * sizeof(int) + 15) / 16 * 16;
    if (c->ensure_pin(off + sizeof(int2) * (ipp.size() + ipk.size())))
      return fail(WB_ERR_NOMEM, "pinned host allocation failed");
    int2* hp = reinterpret_cast<int2*>(c->pin + off);
    std::memcpy(hp, ipp.data(), sizeof(int2) * ipp.size());
    std::memcpy(hp + ipp.size(), ipk.data(), sizeof(int2) * ipk.size());
    WB_CU(cudaMemcpyAsync(c->items_pp.p, hp, sizeof(int2) * ipp.size(), cudaMemcpyHostToDevice, s));
    WB_CU(cudaMemcpyAsync(c->items_pk.p, hp + ipp.size(), sizeof(int2) * ipk.size(), cudaMemcpyHostToDevice, s));
  }
  double2* aux = c->aux.as<double2>();
  double2* B = c->B.as<double2>();
  double2* X = c->X.as<double2>();
  double2* G = c->G.as<double2>();
  double2* T = c->T.as<double2>();
  double2* stk = c->sticks.as<double2>();
  {
    Stage g(c, WB_STAGE_OTHER, 3, mb);
    fill_columns(c->et.as<double>(), nocc, nsys, c->ecol.as<double>(), s);
    fill_columns(c->eprec.as<double>(), nocc, nsys, c->epcol.as<double>(), s);
    // 1. aux = sqvc * dvg in internal order            (apply_operator.f90:49-53)
    permute_scale(dvg, ld_in, c->perm.as<int>(), c->sqvc.as<double>(), npw, mb, aux, ld, s);
  }
  {
    Stage g(c, WB_STAGE_RHS, 4, mp + (long long)mb * npv);
    // 2. dv(r) of perturbation pairs                   (dfpt_module.f90:235)
    fft_zinv(c->fa, aux, ld, c->items_pp.as<int2>(), mp, stk);
    fft_plane_inv_box(c->fa, stk, mp, c->dvbox.as<double2>());
    // 3. dvpsi = P_G[psi_v(r) dv(r)]                    (dfpt_module.f90:245-278)
    fft_plane_rhs(c->fa, c->evcr.as<double2>(), c->dvbox.as<double2>(), npv, mb, stk);
    fft_zfwd_store(c->fa, stk, c->items_pk.as<int2>(), mb * npv, B, ld);
  }
  c->stats.fft_boxes += mp + (long long)mb * npv;
  // 4. dvpsi <- -Pc dvpsi = -dvpsi + evc (evc^T dvpsi)  (dfpt_module.f90:346)
  const double* Wevc = c->W.as<double>() + (size_t)c->nkb * K;
  int rc0 = autotune64(c, nsys);
  if (rc0) return rc0;
  const int nsplit = gemm_tn_splits(c->nproj, nsys, K, c->tune.dmma_ctas);
  {
    Stage g(c, WB_STAGE_OTHER, 4, nsys);
    gemm_tn(Wevc, K, nocc, (const double*)B, 2 * ld, nullptr, nsys, K, nsplit, c->part.as<double>(), s);
    gamma_reduce(c->part.as<double>(), nsplit, nocc, nsys, Wevc, K, (const double*)B, 2 * ld, nullptr, nullptr, 0,
                 1.0, c->C.as<double>(), s);
    // fractional occupations: <psi_j|dV psi_i> of the partly occupied bands j, scaled
    // (dfpt_module.f90:328-337,363-393); C is reused by the PCG, so they are kept apart
    if (c->nfull < nocc)
      frac_coefficients(c->C.as<double>(), nocc, nsys, c->nfull, c->occ.as<double>(), c->et.as<double>(),
                        c->fcoef.as<double>(), s);
    gemm_nn(Wevc, K, nocc, c->C.as<double>(), (double*)B, 2 * ld, nullptr, nsys, K, -1.0, s);
    // 5. dpsi = precondition(dvpsi)                    (dfpt_module.f90:348)
    precondition(B, X, c->iprec.as<double>(), nocc, npw, nsys, ld, s);
  }
  // 6. PCG                                           (dfpt_module.f90:350-361)
  int iters = 0;
  if (tr2 >= 0.0 && c->precision == WB_PRECISION_MIXED) {
    int rc = cg_mixed(c, mb, tr2, nsplit, &iters);
    if (rc) return rc;
  } else if (tr2 >= 0.0) {
    unsigned char* conv = c->conv.as<unsigned char>();
    int* act = c->act.as<int>();
    int2* items = c->items.as<int2>();
    {
      Stage g(c, WB_STAGE_CG, 2, nsys);
      cg_reset(conv, nsys, s);
      cg_compact(conv, nsys, act, items, c->nact.as<int>(), c->nact_host, s);
    }
    apply_A(c, X, T, act, items, nsys, nsys, nsplit);            // :127
    {
      Stage g(c, WB_STAGE_CG, 1, nsys);
      sub_into(T, B, G, npw, nsys, ld, s);                       // :130-138
    }
    int nact = nsys;
    const bool graph = graph_mode(c) && c->maxiter > 0;
    if (c->maxiter > 0) {                                        // iteration 1: prec, rho, test (:146-222)
      Stage g(c, WB_STAGE_CG, 2, nsys);
      cg_prec_rho(act, nsys, G, B, c->iprec.as<double>(), nocc, c->rho.as<double>(), conv, 1, tr2, npw, ld, s);
      cg_compact(conv, nsys, act, items, c->nact.as<int>(), graph ? nullptr : c->nact_host, s);
    }
    if (graph) {                                                 // :146-330 as one graph launch
      const int cap = c->cap_nsys;
      const int nsplit_cap = gemm_tn_splits(c->nproj, cap, K, c->tune.dmma_ctas);
      int* st = c->loopst.as<int>();
      const int* dn = c->nact.as<int>();
      std::vector<const void*> key = {B, X, G, T, c->sticks.p, act, items, dn, conv, c->rho.p, c->part.p, c->C.p,
                                      c->ecol.p, st, (const void*)(intptr_t)cap};
      int rc = capture_loop(c, c->loop64, key, tr2, cap, dn, st, false, [&](int nmax) {
        apply_A(c, B, T, act, items, nmax, cap, nsplit_cap, dn);
        cg_step(act, nmax, X, G, B, T, c->iprec.as<double>(), nocc, c->rho.as<double>(), conv, 0, c->maxiter, tr2,
                npw, ld, s, dn, st + 1);
        cg_compact(conv, cap, act, items, c->nact.as<int>(), nullptr, s, st);
      });
      if (rc) return rc;
      loop_init(st, nsys, true, s);
      WB_CU(cudaGraphLaunch(c->loop64.cur(), s));
      WB_CU(cudaMemcpyAsync(c->loop_host, st, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
      // read after the batch's final wait (pending_loop_stats): no host round
      // trip between the PCG graph and the density stage
      c->loop_pending = c->kinetic_only ? 6 : 9;
    }
    for (int it = 1; !graph && it <= c->maxiter; ++it) {        // :146
      WB_CU(cudaStreamSynchronize(s));
      nact = *c->nact_host;
      iters = it;
      if (nact == 0) break;                                      // :222
      c->stats.cg_active_sum += nact;
      apply_A(c, B, T, act, items, nact, nsys, nsplit);          // :251
      {
        Stage g(c, WB_STAGE_CG, 2, nact);
        // :253-329, then iteration it + 1's :146-222
        cg_step(act, nact, X, G, B, T, c->iprec.as<double>(), nocc, c->rho.as<double>(), conv, it, c->maxiter, tr2,
                npw, ld, s);
        cg_compact(conv, nsys, act, items, c->nact.as<int>(), c->nact_host, s);
      }
    }
    {
      Stage g(c, WB_STAGE_CG, 1, mb);
      count_unconverged(conv, nocc, mb, c->unconv.as<int>(), s);
    }
  } else {
    WB_CU(cudaMemsetAsync(c->unconv.p, 0, sizeof(int) * mb, s));
  }
  c->stats.cg_iterations = std::max(c->stats.cg_iterations, iters);
  if (c->nfull < nocc) {                                // dpsi += evc_frac psi_dvpsi (dfpt_module.f90:397-398)
    Stage g(c, WB_STAGE_OTHER, 1, nsys);
    gemm_nn(Wevc + (size_t)c->nfull * K, K, nocc - c->nfull, c->fcoef.as<double>(), (double*)X, 2 * ld, nullptr, nsys,
            K, 1.0, s);
  }
  // 7. drho and dng                                   (dfpt_module.f90:403-487)
  {
    Stage g(c, WB_STAGE_DRHO, 3, (long long)mb * npv + mp);
    fft_zinv(c->fa, X, ld, c->items_pk.as<int2>(), mb * npv, stk);
    const double scale = 2.0 * c->wk / c->omega / (double)c->nnr;
    fft_plane_drho(c->fa, stk, c->evcr.as<double2>(), c->occ.as<double>(), nocc, mb, c->acc.as<double2>(), scale,
                   c->sticks2.as<double2>());
    fft_zfwd_dng(c->fa, c->sticks2.as<double2>(), c->items_pp.as<int2>(), mp, dng, ld_out, c->perm.as<int>(),
                 c->sqvc.as<double>());
  }
  c->stats.fft_boxes += (long long)mb * npv + mp;
  // to the pinned staging area; the caller reads it after its wait
  WB_CU(cudaMemcpyAsync(c->pin, c->unconv.p, sizeof(int) * mb, cudaMemcpyDeviceToHost, s));
  return WB_OK;
}

}  // namespace

// The FP64 PCG graph's counters of a finished batch (copied by the batch to
// pinned memory) into the call's stats.
void wb::apply_settle(wb_ctx* c) {
  if (!c->loop_pending) return;
  c->stats.cg_iterations = std::max(c->stats.cg_iterations, c->loop_host[2]);
  loop_stats(c, c->loop_host[3], c->loop_pending);
  c->loop_pending = 0;
}

namespace {

// With defer (device buffers, one batch, no stage profiling) the call returns
// right after enqueuing the batch: no wait, no unconverged counts, no ms_total;
// the caller waits on the context's stream later and then calls apply_settle.
int apply_impl(wb_ctx* c, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng, double tr2, int iq,
               int* unconverged, bool on_device, bool* deferred = nullptr) {
  g_err.clear();
  if (!c) return fail(WB_ERR_ARG, "null context");
  if (m < 0) return fail(WB_ERR_ARG, "m < 0");
  if (iq != 1) return fail(WB_ERR_UNSUPPORTED, "only iq = 1 (Gamma) is provided");
  if (m > 0 && (!dvg || !dng)) return fail(WB_ERR_ARG, "null dvg or dng");
  if (ld_dvg < c->npw || ld_dng < c->npw) return fail(WB_ERR_ARG, "leading dimension smaller than npw");
  if (std::isnan(tr2)) return fail(WB_ERR_ARG, "tr2 is NaN");
  WB_CU(cudaSetDevice(c->device));
  c->stats = wb_stats{};
  c->marks.clear();
  c->evused = 0;
  c->loop_pending = 0;
  c->stats.m = m;
  if (m == 0) return WB_OK;
  cudaStream_t s = c->stream;
  WB_CU(cudaEventRecord(c->ev0, s));
  const int mb = choose_batch(c, m);
  const bool defer = deferred && on_device && mb >= m && !c->prof;
  if (deferred) *deferred = defer;
  int rc = ensure_workspace(c, mb, on_device ? 1 : ld_dvg, on_device ? 1 : ld_dng);
  if (rc) return rc;
  std::vector<int> unc(m, 0);
  for (int p0 = 0; p0 < m; p0 += mb) {
    const int nb = std::min(mb, m - p0);
    const double2* din;
    double2* dout;
    if (on_device) {
      din = reinterpret_cast<const double2*>(dvg) + (size_t)p0 * ld_dvg;
      dout = reinterpret_cast<double2*>(dng) + (size_t)p0 * ld_dng;
    } else {
      WB_CU(cudaMemcpyAsync(c->dvg_in.p, dvg + 2 * (size_t)p0 * ld_dvg, sizeof(double2) * (size_t)ld_dvg * nb,
                            cudaMemcpyHostToDevice, s));
      din = c->dvg_in.as<double2>();
      dout = c->dng_out.as<double2>();
    }
    // rows >= npw of dng are zero (apply_operator.f90:44, dng = 0)
    if (ld_dng > c->npw)
      WB_CU(cudaMemset2DAsync(dout + c->npw, sizeof(double2) * ld_dng, 0, sizeof(double2) * (ld_dng - c->npw), nb, s));
    rc = run_batch(c, nb, din, ld_dvg, dout, ld_dng, tr2);
    if (rc) return rc;
    if (!on_device)
      WB_CU(cudaMemcpyAsync(dng + 2 * (size_t)p0 * ld_dng, c->dng_out.p, sizeof(double2) * (size_t)ld_dng * nb,
                            cudaMemcpyDeviceToHost, s));
    if (defer) return WB_OK;
    WB_CU(wb_wait(c));
    apply_settle(c);
    std::memcpy(unc.data() + p0, c->pin, sizeof(int) * nb);
  }
  WB_CU(cudaEventRecord(c->ev1, s));
  WB_CU(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->stats.ms_total = ms;
  resolve_marks(c);
  WB_CU(cudaGetLastError());
  if (unconverged) std::memcpy(unconverged, unc.data(), sizeof(int) * m);
  return WB_OK;
}

}  // namespace

int wb::apply_deferred(wb_ctx* c, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng, double tr2,
                       bool* deferred) {
  return apply_impl(c, m, dvg, ld_dvg, dng, ld_dng, tr2, 1, nullptr, true, deferred);
}

extern "C" {

int wb_version(void) { return 100; }

const char* wb_last_error(void) { return g_err.c_str(); }

int wb_ctx_create(wb_ctx** out, const wb_system* s, int device) {
  g_err.clear();
  if (!out || !s) return fail(WB_ERR_ARG, "null argument");
  *out = nullptr;
  if (s->npw <= 0 || s->npwx < s->npw) return fail(WB_ERR_ARG, "need 0 < npw <= npwx");
  if (s->nr1 < 2 || s->nr2 < 2 || s->nr3 < 2) return fail(WB_ERR_ARG, "FFT box edges must be >= 2");
  // compiled kernels for the listed cubic edges; every other box runs the
  // runtime-size transforms, which need 2, 3, 5, 7-smooth edges
  const bool compiled = s->nr1 == s->nr2 && s->nr1 == s->nr3 && fft_supported(s->nr1);
  if (!compiled)
    for (int e : {s->nr1, s->nr2, s->nr3})
      if (rt_plan(e).ns == 0)
        return fail(WB_ERR_UNSUPPORTED, "FFT edge " + std::to_string(e) + " has a prime factor above 7");
  if (s->nbnd_occ <= 0 || s->nkb < 0) return fail(WB_ERR_ARG, "bad nbnd_occ or nkb");
  if (s->gstart != 2) return fail(WB_ERR_UNSUPPORTED, "gstart must be 2 (G=0 on this process)");
  if (s->n_dfpt_maxiter < 0) return fail(WB_ERR_ARG, "n_dfpt_maxiter < 0");
  if (!s->nl || !s->nlm || !s->g2kin || !s->vrs || !s->evc || !s->et || !s->occupation || !s->sqvc ||
      (s->nkb > 0 && (!s->vkb || !s->deeq)))
    return fail(WB_ERR_ARG, "null system array");
  if (!(s->omega > 0.0)) return fail(WB_ERR_ARG, "omega must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return fail(WB_ERR_CUDA, "no CUDA device " + std::to_string(device));
  }
  wb_ctx* c = new wb_ctx();
  c->device = device;
  auto bail = [&](int code) {
    wb_ctx_destroy(c);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(fail(WB_ERR_CUDA, "cudaSetDevice failed"));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaMallocHost(&c->nact_host, sizeof(int) * 4) != cudaSuccess ||
      cudaMallocHost(&c->loop_host, sizeof(int) * 8) != cudaSuccess || c->loopst.ensure(sizeof(int) * 8) != 0 ||
      cudaEventCreate(&c->tev0) != cudaSuccess || cudaEventCreate(&c->tev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->wait_ev, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(WB_ERR_CUDA, "stream/event creation failed"));
  c->npw = s->npw;
  c->rt = compiled ? 0 : 1;
  c->nr = compiled ? s->nr1 : 0;
  c->nz = s->nr3;
  c->nnr = s->nr1 * s->nr2 * s->nr3;
  if (c->rt) {
    c->geo.nx = s->nr1;
    c->geo.ny = s->nr2;
    c->geo.nz = s->nr3;
    c->geo.px = rt_plan(s->nr1);
    c->geo.py = rt_plan(s->nr2);
    c->geo.pz = rt_plan(s->nr3);
  }
  c->nocc = s->nbnd_occ;
  c->nkb = s->nkb;
  c->nproj = s->nkb + s->nbnd_occ;
  c->npv = (s->nbnd_occ + 1) / 2;
  c->maxiter = s->n_dfpt_maxiter;
  c->kinetic_only = s->l_kinetic_only;
  c->omega = s->omega;
  c->wk = s->wk;
  c->alpha = s->alpha_pv;
  // FP64 bra-ket operand prefetch: two k steps ahead for few projectors (64 at
  // the c2 cell: 4.3 -> 3.3 ms per m = 16 call), one for many (208 at the 108^3
  // cell, where the extra registers cost more: 222 -> 242 ms)
  c->tune.dmma_pf = c->nproj <= 96 ? 2 : 1;
  // fractional occupations (Tools/set_nbndocc.f90:58-69): nbnd_occ_full is the
  // highest band occupied above 1 - docc_thr; the correction of dfpt_module.f90:
  // 363-398 needs non-degenerate energies wherever the occupations differ (:387)
  for (int b = 0; b < c->nocc; ++b)
    if (s->occupation[b] > 1.0 - 1e-3) c->nfull = b + 1;
  for (int i = 0; i < c->nocc; ++i)
    for (int r = std::max(i + 1, c->nfull); r < c->nocc; ++r)
      if (std::fabs(s->occupation[i] - s->occupation[r]) >= 1e-3 && std::fabs(s->et[i] - s->et[r]) < 1e-3)
        return bail(fail(WB_ERR_ARG, "fractional occupation degenerate orbitals (bands " + std::to_string(i + 1) +
                                         " and " + std::to_string(r + 1) + ")"));
  std::vector<int> perm;
  int rc = build_tables(c, s, perm);
  if (rc) return bail(rc);
  const int N = c->nr, npw = c->npw;
  // twiddles exp(+2 pi i j / n), accurate host values
  auto twiddles = [](int n) {
    std::vector<double2> t(n);
    for (int j = 0; j < n; ++j) {
      const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
      t[j] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return t;
  };
  std::vector<double> g2(npw), sq(npw);
  for (int i = 0; i < npw; ++i) { g2[i] = s->g2kin[perm[i]]; sq[i] = s->sqvc[perm[i]]; }
  std::vector<double> vsc(c->nnr);
  if (!c->rt) {
    for (int i = 0; i < c->nnr; ++i) vsc[i] = s->vrs[i] / (double)c->nnr;
    if ((rc = upload(twiddles(N).data(), N, c->tw))) return bail(rc);
  } else {
    // V(r) / N at the digit-reversed positions the runtime transforms leave real space in
    const int nx = s->nr1, ny = s->nr2, nz = s->nr3;
    std::vector<int> rx(nx), ry(ny), rz(nz);
    for (int p = 0; p < nx; ++p) rx[p] = rt_digit_reverse(c->geo.px, p);
    for (int p = 0; p < ny; ++p) ry[p] = rt_digit_reverse(c->geo.py, p);
    for (int p = 0; p < nz; ++p) rz[p] = rt_digit_reverse(c->geo.pz, p);
    for (int pz = 0; pz < nz; ++pz)
      for (int py = 0; py < ny; ++py)
        for (int px = 0; px < nx; ++px)
          vsc[((size_t)pz * ny + py) * nx + px] = s->vrs[((size_t)rz[pz] * ny + ry[py]) * nx + rx[px]] / (double)c->nnr;
    if ((rc = upload(twiddles(nx).data(), nx, c->twx)) || (rc = upload(twiddles(ny).data(), ny, c->twy)) ||
        (rc = upload(twiddles(nz).data(), nz, c->twz)))
      return bail(rc);
    c->geo.twx = c->twx.as<double2>();
    c->geo.twy = c->twy.as<double2>();
    c->geo.twz = c->twz.as<double2>();
    if (rt_plane_smem(c->geo, 16, nullptr) == 0)
      return bail(fail(WB_ERR_UNSUPPORTED, "the x-y plane of this box does not fit in shared memory"));
  }
  if ((rc = upload(g2.data(), npw, c->g2kin)) ||
      (rc = upload(sq.data(), npw, c->sqvc)) || (rc = upload(vsc.data(), c->nnr, c->vs)) ||
      (rc = upload(s->et, c->nocc, c->et)) || (rc = upload(s->occupation, c->nocc, c->occ)))
    return bail(rc);
  if ((rc = upload_cols(s->evc, s->npwx, c->nocc, perm, c->evc))) return bail(rc);
  // W = [vkb | evc] as real columns of length 2 npw
  {
    std::vector<double2> w((size_t)npw * c->nproj);
    for (int j = 0; j < c->nproj; ++j) {
      const double* src = j < c->nkb ? s->vkb + 2 * (size_t)j * s->npwx : s->evc + 2 * (size_t)(j - c->nkb) * s->npwx;
      for (int i = 0; i < npw; ++i) w[(size_t)j * npw + i] = make_double2(src[2 * perm[i]], src[2 * perm[i] + 1]);
    }
    if ((rc = upload(w.data(), w.size(), c->W))) return bail(rc);
    std::vector<double> dd(std::max(1, c->nkb * c->nkb), 0.0);
    if (c->nkb) std::memcpy(dd.data(), s->deeq, sizeof(double) * c->nkb * c->nkb);
    if ((rc = upload(dd.data(), dd.size(), c->D))) return bail(rc);
  }
  if (c->rt) rt_setup(c->geo);
  else fft_setup(N);
  c->fa.n = N;
  c->fa.st = c->st;
  c->fa.tw = c->tw.as<double2>();
  c->fa.stream = c->stream;
  c->fa.rt = c->rt ? &c->geo : nullptr;
  // eprec (set_eprec.f90) and psi_v(r) for all occupied bands, in pairs
  if (c->eprec.ensure(sizeof(double) * c->nocc) || c->evcr.ensure(sizeof(double2) * (size_t)c->nnr * c->npv) ||
      c->iota_items.ensure(sizeof(int2) * c->npv) ||
      c->sticks.ensure(sizeof(double2) * (size_t)c->nz * c->st.nst * c->npv))
    return bail(fail(WB_ERR_NOMEM, "device allocation failed"));
  set_eprec(c->evc.as<double2>(), c->g2kin.as<double>(), npw, c->nocc, c->eprec.as<double>(), c->stream);
  if (c->iprec.ensure(sizeof(double) * (size_t)npw * c->nocc)) return bail(fail(WB_ERR_NOMEM, "device allocation failed"));
  make_iprec(c->g2kin.as<double>(), c->eprec.as<double>(), npw, c->nocc, c->iprec.as<double>(), c->stream);
  std::vector<int2> ib;
  pair_items(ib, 0, c->nocc);
  if (cudaMemcpy(c->iota_items.p, ib.data(), sizeof(int2) * ib.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(WB_ERR_CUDA, "upload failed"));
  fft_zinv(c->fa, c->evc.as<double2>(), npw, c->iota_items.as<int2>(), c->npv, c->sticks.as<double2>());
  fft_plane_inv_box(c->fa, c->sticks.as<double2>(), c->npv, c->evcr.as<double2>());
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return bail(fail(WB_ERR_CUDA, std::string("context setup: ") + cudaGetErrorString(e)));
  *out = c;
  return WB_OK;
}

int wb_ctx_destroy(wb_ctx* c) {
  if (!c) return WB_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DBuf* bufs[] = {&c->perm, &c->gqz, &c->spg, &c->stpos, &c->tw, &c->g2kin, &c->sqvc, &c->vs, &c->evc, &c->W,
                  &c->D, &c->eprec, &c->et, &c->occ, &c->evcr, &c->iprec, &c->dvg_in, &c->dng_out, &c->aux, &c->dvbox, &c->B,
                  &c->X, &c->G, &c->T, &c->sticks, &c->sticks2, &c->acc, &c->part, &c->C, &c->rho, &c->conv,
                  &c->act, &c->items, &c->nact, &c->ecol, &c->epcol, &c->unconv, &c->items_pp, &c->items_pk,
                  &c->iota_items, &c->fcoef, &c->rt_colx, &c->twx, &c->twy, &c->twz, &c->twx32, &c->twy32, &c->twz32, &c->dav_dvg, &c->dav_dng, &c->dav_tmp, &c->dav_hr, &c->dav_vr, &c->dav_A,
                  &c->dav_V, &c->dav_w, &c->dav_part, &c->dav_coef, &c->dav_dots, &c->dav_bj, &c->dav_st, &c->W32, &c->D32, &c->g2kin32,
                  &c->vs32, &c->tw32, &c->g32, &c->P32, &c->T32, &c->d32, &c->sticks32, &c->part32, &c->C32,
                  &c->ecol32, &c->rho0, &c->rho_in, &c->conv_in, &c->act_in, &c->items_in, &c->nact_in,
                  &c->umma_braket_w, &c->umma_update_w, &c->umma_err};
  c->loop64.release();
  c->loop32.release();
  c->dav_graphs_release();
  if (c->dav_host) cudaFreeHost(c->dav_host);
  if (c->dav_aux) cudaStreamDestroy(c->dav_aux);
  for (cudaEvent_t e : c->dav_ev)
    if (e) cudaEventDestroy(e);
  for (DBuf* b : bufs) b->release();
  c->loopst.release();
  if (c->nact_host) cudaFreeHost(c->nact_host);
  if (c->loop_host) cudaFreeHost(c->loop_host);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->tev0) cudaEventDestroy(c->tev0);
  if (c->tev1) cudaEventDestroy(c->tev1);
  if (c->wait_ev) cudaEventDestroy(c->wait_ev);
  if (c->pin) cudaFreeHost(c->pin);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return WB_OK;
}

int wb_apply_operator(wb_ctx* c, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng, double tr2, int iq,
                      int* unconverged) {
  return apply_impl(c, m, dvg, ld_dvg, dng, ld_dng, tr2, iq, unconverged, false);
}

int wb_apply_operator_device(wb_ctx* c, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng, double tr2,
                             int iq, int* unconverged) {
  return apply_impl(c, m, dvg, ld_dvg, dng, ld_dng, tr2, iq, unconverged, true);
}

int wb_set_precision(wb_ctx* c, int mode) {
  if (!c) return fail(WB_ERR_ARG, "null context");
  if (mode == WB_PRECISION_FP64 || mode == WB_PRECISION_MIXED) { c->precision = mode; return WB_OK; }
  return fail(WB_ERR_ARG, "unknown precision mode");
}

int wb_set_batch(wb_ctx* c, int maxp) {
  if (!c) return fail(WB_ERR_ARG, "null context");
  if (maxp < 0) return fail(WB_ERR_ARG, "negative batch");
  c->batch_cap = maxp;
  return WB_OK;
}

int wb_set_profiling(wb_ctx* c, int stage_mask) {
  if (!c) return fail(WB_ERR_ARG, "null context");
  if (stage_mask < 0 || stage_mask > WB_PROFILE_ALL) return fail(WB_ERR_ARG, "profiling mask out of range");
  c->prof = stage_mask;
  return WB_OK;
}

int wb_apply_operator_multi(int nctx, wb_ctx* const* ctx, const int* m, const double* const* dvg, const int* ld_dvg,
                            double* const* dng, const int* ld_dng, double tr2, int iq, int* const* unconverged,
                            int on_device) {
  g_err.clear();
  if (nctx < 0 || (nctx > 0 && (!ctx || !m || !dvg || !ld_dvg || !dng || !ld_dng)))
    return fail(WB_ERR_ARG, "null argument");
  for (int i = 0; i < nctx; ++i)
    for (int j = 0; j < i; ++j)
      if (ctx[i] == ctx[j]) return fail(WB_ERR_ARG, "a context appears twice");
  std::vector<int> rc(nctx, WB_OK);
  std::vector<std::string> msg(nctx);
  std::vector<std::thread> th;
  th.reserve(nctx);
  for (int i = 0; i < nctx; ++i)
    th.emplace_back([&, i] {
      rc[i] = apply_impl(ctx[i], m[i], dvg[i], ld_dvg[i], dng[i], ld_dng[i], tr2, iq,
                         unconverged ? unconverged[i] : nullptr, on_device != 0);
      msg[i] = g_err;
    });
  for (auto& t : th) t.join();
  for (int i = 0; i < nctx; ++i)
    if (rc[i] != WB_OK) return fail(rc[i], "system " + std::to_string(i) + ": " + msg[i]);
  return WB_OK;
}

int wb_get_tuning(const wb_ctx* c, wb_tuning* out) {
  if (!c || !out) return fail(WB_ERR_ARG, "null argument");
  out->autotune = c->tune.on;
  out->tuned_fp64 = c->tune.done64;
  out->tuned_mixed = c->tune.done32;
  out->dmma_ctas_per_sm = c->tune.dmma_ctas;
  out->dmma_prefetch = c->tune.dmma_pf;
  out->tc_braket_ctas_per_sm = c->tune.umma_ctas;
  out->tc_update_systems = c->tune.update_nj;
  out->plane_fused_fp64 = fft_fusable(c->nr, c->st) && !c->tune.unfused64;
  out->plane_fused_mixed = fft_fusable(c->nr, c->st) && !c->tune.unfused32;
  out->tuning_ms = c->tune.ms;
  return WB_OK;
}

int wb_set_autotune(wb_ctx* c, int enable) {
  if (!c) return fail(WB_ERR_ARG, "null context");
  c->tune.on = enable ? 1 : 0;
  return WB_OK;
}

int wb_set_graphs(wb_ctx* c, int enable) {
  if (!c) return fail(WB_ERR_ARG, "null context");
  c->use_graphs = enable ? 1 : 0;
  return WB_OK;
}

int wb_get_stats(const wb_ctx* c, wb_stats* out) {
  if (!c || !out) return fail(WB_ERR_ARG, "null argument");
  *out = c->stats;
  return WB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of wb_apply_operator_device.
//
// For callers that must not allocate device memory while they run: a host
// code that has handed all of its GPU memory to its own pool allocator, a
// real-time or latency-bound loop that cannot afford the implicit device
// synchronisation of cudaMalloc/cudaFree, or a caller whose allocation
// policy forbids allocations after set-up.  Every per-call buffer (stick
// buffers, PCG vectors, GEMM partial sums, density accumulators, index
// tables) is carved out of one file-scope __device__ array of
// WB_NOALLOC_SCRATCH_BYTES; the context's constant data was allocated once by
// wb_ctx_create.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[WB_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array for the context's device, looked up on
// the context's first allocation-free call, with that device current, and kept
// in the context: the address belongs to the CUDA context the library's module
// is loaded in, so a context created later (after a cudaDeviceReset, say) makes
// its own lookup.  A failed lookup is not kept; the next call tries again.  The
// host-side name g_noalloc_scratch is only a stand-in for the symbol: it must
// never be passed to a kernel.
int noalloc_scratch(wb_ctx* c, unsigned char** out) {
  if (!c->noalloc_base) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return fail(WB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    c->noalloc_base = p;
  }
  *out = static_cast<unsigned char*>(c->noalloc_base);
  return WB_OK;
}

// Bump carver over the scratch array (256-byte aligned pieces).  With a null
// base it only measures.
struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += sizeof(T) * n;
    return p;
  }
};

struct NoallocWs {
  double2 *aux, *dvbox, *B, *X, *G, *T, *sticks, *sticks2, *acc;
  double *part, *C, *rho, *ecol, *epcol;
  unsigned char* conv;
  int *act, *nact, *unconv;
  int2 *items, *items_pp, *items_pk;
  int nsplit;
};

void noalloc_layout(const wb_ctx* c, int mb, Carve& cv, NoallocWs& w) {
  const size_t nsys = (size_t)mb * c->nocc;
  const size_t npw = c->npw;
  const size_t stk1 = (size_t)c->nz * c->st.nst;
  const size_t mp = ((size_t)mb + 1) / 2;
  const size_t nitems = std::max<size_t>({(nsys + 1) / 2, (size_t)mb * c->npv, mp});
  w.nsplit = gemm_tn_splits(c->nproj, (int)nsys, 2 * c->npw);
  w.aux = cv.take<double2>(npw * mb);
  w.dvbox = cv.take<double2>((size_t)c->nnr * mp);
  w.B = cv.take<double2>(npw * nsys);
  w.X = cv.take<double2>(npw * nsys);
  w.G = cv.take<double2>(npw * nsys);
  w.T = cv.take<double2>(npw * nsys);
  w.sticks = cv.take<double2>(stk1 * nitems);
  w.sticks2 = cv.take<double2>(stk1 * mp);
  w.acc = cv.take<double2>((size_t)c->nnr * mp);
  w.part = cv.take<double>((size_t)w.nsplit * nsys * c->nproj);
  w.C = cv.take<double>(nsys * c->nproj);
  w.rho = cv.take<double>(nsys);
  w.ecol = cv.take<double>(nsys);
  w.epcol = cv.take<double>(nsys);
  w.conv = cv.take<unsigned char>(nsys);
  w.act = cv.take<int>(nsys);
  w.nact = cv.take<int>(4);
  w.unconv = cv.take<int>(mb);
  w.items = cv.take<int2>(nsys / 2 + 1);
  w.items_pp = cv.take<int2>(mp);
  w.items_pk = cv.take<int2>((size_t)mb * c->npv);
}

__global__ void k_noalloc_items(int2* __restrict__ pp, int2* __restrict__ pk, int mb, int nocc, int npv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int mp = (mb + 1) / 2;
  if (i < mp) pp[i] = make_int2(2 * i, (2 * i + 1 < mb) ? 2 * i + 1 : -1);
  if (i < mb * npv) {
    const int p = i / npv, k = i % npv;
    pk[i] = make_int2(p * nocc + 2 * k, (2 * k + 1 < nocc) ? p * nocc + 2 * k + 1 : -1);
  }
}

// (H - e + alpha Pv) on the listed columns, with workspace from the scratch array.
void noalloc_apply_A(wb_ctx* c, const NoallocWs& w, const double2* Xv, double2* Tv, const int* cols,
                     const int2* items, int n) {
  const long ld = c->npw;
  const int K = 2 * c->npw;
  cudaStream_t s = c->stream;
  const double* Wsub = c->W.as<double>();
  int M = c->nproj, nkb = c->nkb;
  if (c->kinetic_only) {
    kinetic_hpsi(Xv, Tv, c->g2kin.as<double>(), w.ecol, cols, n, c->npw, ld, s);
    Wsub = c->W.as<double>() + (size_t)c->nkb * K;
    M = c->nocc;
    nkb = 0;
  } else {
    const int nit = (n + 1) / 2;
    fft_zinv(c->fa, Xv, ld, items, nit, w.sticks);
    fft_plane_vloc(c->fa, w.sticks, nit, c->vs.as<double>());
    fft_zfwd_hpsi(c->fa, w.sticks, items, nit, Xv, Tv, ld, c->g2kin.as<double>(), w.ecol);
  }
  gemm_tn(Wsub, K, M, (const double*)Xv, 2 * ld, cols, n, K, w.nsplit, w.part, s);
  gamma_reduce(w.part, w.nsplit, M, n, Wsub, K, (const double*)Xv, 2 * ld, cols, c->D.as<double>(), nkb, c->alpha,
               w.C, s);
  gemm_nn(Wsub, K, M, w.C, (double*)Tv, 2 * ld, cols, n, K, 1.0, s);
}

int noalloc_run(wb_ctx* c, const NoallocWs& w, int mb, const double2* dvg, long ld_in, double2* dng, long ld_out,
                double tr2, int* unconv_host) {
  cudaStream_t s = c->stream;
  const int npw = c->npw, nocc = c->nocc, npv = c->npv;
  const int nsys = mb * nocc;
  const long ld = npw;
  const int K = 2 * npw;
  const int mp = (mb + 1) / 2;
  const int nit = std::max(mp, mb * npv);
  k_noalloc_items<<<(nit + 255) / 256, 256, 0, s>>>(w.items_pp, w.items_pk, mb, nocc, npv);
  fill_columns(c->et.as<double>(), nocc, nsys, w.ecol, s);
  fill_columns(c->eprec.as<double>(), nocc, nsys, w.epcol, s);
  permute_scale(dvg, ld_in, c->perm.as<int>(), c->sqvc.as<double>(), npw, mb, w.aux, ld, s);
  fft_zinv(c->fa, w.aux, ld, w.items_pp, mp, w.sticks);
  fft_plane_inv_box(c->fa, w.sticks, mp, w.dvbox);
  fft_plane_rhs(c->fa, c->evcr.as<double2>(), w.dvbox, npv, mb, w.sticks);
  fft_zfwd_store(c->fa, w.sticks, w.items_pk, mb * npv, w.B, ld);
  const double* Wevc = c->W.as<double>() + (size_t)c->nkb * K;
  gemm_tn(Wevc, K, nocc, (const double*)w.B, 2 * ld, nullptr, nsys, K, w.nsplit, w.part, s);
  gamma_reduce(w.part, w.nsplit, nocc, nsys, Wevc, K, (const double*)w.B, 2 * ld, nullptr, nullptr, 0, 1.0, w.C, s);
  gemm_nn(Wevc, K, nocc, w.C, (double*)w.B, 2 * ld, nullptr, nsys, K, -1.0, s);
  precondition(w.B, w.X, c->iprec.as<double>(), nocc, npw, nsys, ld, s);
  int iters = 0;
  if (tr2 >= 0.0) {
    cg_reset(w.conv, nsys, s);
    cg_compact(w.conv, nsys, w.act, w.items, w.nact, c->nact_host, s);
    noalloc_apply_A(c, w, w.X, w.T, w.act, w.items, nsys);
    sub_into(w.T, w.B, w.G, npw, nsys, ld, s);
    int nact = nsys;
    if (c->maxiter > 0) {
      cg_prec_rho(w.act, nact, w.G, w.B, c->iprec.as<double>(), nocc, w.rho, w.conv, 1, tr2, npw, ld, s);
      cg_compact(w.conv, nsys, w.act, w.items, w.nact, c->nact_host, s);
    }
    for (int it = 1; it <= c->maxiter; ++it) {
      WB_CU(cudaStreamSynchronize(s));
      nact = *c->nact_host;
      iters = it;
      if (nact == 0) break;
      c->stats.cg_active_sum += nact;
      noalloc_apply_A(c, w, w.B, w.T, w.act, w.items, nact);
      cg_step(w.act, nact, w.X, w.G, w.B, w.T, c->iprec.as<double>(), nocc, w.rho, w.conv, it, c->maxiter, tr2, npw,
              ld, s);
      cg_compact(w.conv, nsys, w.act, w.items, w.nact, c->nact_host, s);
    }
    count_unconverged(w.conv, nocc, mb, w.unconv, s);
  } else {
    WB_CU(cudaMemsetAsync(w.unconv, 0, sizeof(int) * mb, s));
  }
  c->stats.cg_iterations = std::max(c->stats.cg_iterations, iters);
  fft_zinv(c->fa, w.X, ld, w.items_pk, mb * npv, w.sticks);
  const double scale = 2.0 * c->wk / c->omega / (double)c->nnr;
  fft_plane_drho(c->fa, w.sticks, c->evcr.as<double2>(), c->occ.as<double>(), nocc, mb, w.acc, scale, w.sticks2);
  fft_zfwd_dng(c->fa, w.sticks2, w.items_pp, mp, dng, ld_out, c->perm.as<int>(), c->sqvc.as<double>());
  if (unconv_host) WB_CU(cudaMemcpyAsync(unconv_host, w.unconv, sizeof(int) * mb, cudaMemcpyDeviceToHost, s));
  WB_CU(cudaStreamSynchronize(s));
  WB_CU(cudaGetLastError());
  return WB_OK;
}

}  // namespace

extern "C" int wb_apply_operator_device_noalloc(wb_ctx* c, int m, const double* dvg, int ld_dvg, double* dng,
                                                int ld_dng, double tr2, int iq, int* unconverged) {
  g_err.clear();
  if (!c) return fail(WB_ERR_ARG, "null context");
  if (m < 0) return fail(WB_ERR_ARG, "m < 0");
  if (iq != 1) return fail(WB_ERR_UNSUPPORTED, "only iq = 1 (Gamma) is provided");
  if (m > 0 && (!dvg || !dng)) return fail(WB_ERR_ARG, "null dvg or dng");
  if (ld_dvg < c->npw || ld_dng < c->npw) return fail(WB_ERR_ARG, "leading dimension smaller than npw");
  if (std::isnan(tr2)) return fail(WB_ERR_ARG, "tr2 is NaN");
  if (c->precision != WB_PRECISION_FP64)
    return fail(WB_ERR_UNSUPPORTED, "the allocation-free entry point runs the FP64 form only");
  if (c->nfull < c->nocc)
    return fail(WB_ERR_UNSUPPORTED, "the allocation-free entry point has no fractional occupations");
  // the four PCG vectors alone must fit: this bounds m before any int product
  // of the layout (m * nbnd_occ systems, m * band pairs) is formed
  if (4.0 * sizeof(double2) * (double)m * c->nocc * c->npw > (double)WB_NOALLOC_SCRATCH_BYTES)
    return fail(WB_ERR_ARG, "m = " + std::to_string(m) + " perturbations do not fit the allocation-free entry "
                "point's scratch of " + std::to_string((size_t)WB_NOALLOC_SCRATCH_BYTES) +
                " bytes (WB_NOALLOC_SCRATCH_BYTES): use fewer perturbations per call");
  Carve probe{nullptr};
  NoallocWs w{};
  noalloc_layout(c, std::max(m, 1), probe, w);
  if (probe.off > (size_t)WB_NOALLOC_SCRATCH_BYTES)
    return fail(WB_ERR_ARG, "this call needs " + std::to_string(probe.off) + " bytes of scratch; the allocation-free "
                "entry point has " + std::to_string((size_t)WB_NOALLOC_SCRATCH_BYTES) +
                " (WB_NOALLOC_SCRATCH_BYTES): use fewer perturbations per call");
  WB_CU(cudaSetDevice(c->device));
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(c, &base);
  if (rc) return rc;
  c->stats = wb_stats{};
  c->stats.m = m;
  if (m == 0) return WB_OK;
  Carve cv{base};
  noalloc_layout(c, m, cv, w);
  if (ld_dng > c->npw)
    WB_CU(cudaMemset2DAsync(reinterpret_cast<double2*>(dng) + c->npw, sizeof(double2) * ld_dng, 0,
                            sizeof(double2) * (ld_dng - c->npw), m, c->stream));
  return noalloc_run(c, w, m, reinterpret_cast<const double2*>(dvg), ld_dvg, reinterpret_cast<double2*>(dng), ld_dng,
                     tr2, unconverged);
}
