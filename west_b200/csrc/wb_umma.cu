// Split-BF16x3 tensor-core GEMMs (tcgen05, sm_100a) of the FP32 inner solves.
//
// The two dense contractions of the Sternheimer operator on Gamma
// (apply_sternheimerop_to_m_wfcs.f90:65-74 with QE's calbec/add_vuspsi and
// apply_alpha_pv_to_m_wfcs.f90:65-72; glbrak.f90:39-40 for the bra-ket):
//   bra-ket  part[s][j][r] = sum_{k in split s} W[r][k] X[col j][k]
//   update   Y[col j][k]  += sum_r W[r][k] C[j][r]
// with W = [vkb | evc] as real pairs (K = 2 npw rows).  Every FP32 operand x
// is split into bf16 hi = rn(x) and lo = rn(x - hi); a product is
// hi*hi + hi*lo + lo*hi, accumulated in FP32 in tensor memory (TMEM).
//
// W is constant: it is split once into bf16 tiles already in the UMMA
// K-major 128-byte-swizzled layout and streamed into shared memory with
// cp.async.bulk.  X and C change every iteration: the CTA's threads load them
// as FP32, split them and store the swizzled bf16 tiles themselves.  One
// thread issues tcgen05.mma (M = 128, N = projectors or systems, K = 16);
// tcgen05.commit arrives on an mbarrier that releases the shared buffers and
// the accumulator to the epilogue warps (tcgen05.ld).  Every wait is bounded:
// on time-out the kernel records a code in *err, skips the rest of its work,
// frees its TMEM and returns.
#include <cuda_bf16.h>

#include <cstdint>

#include "wb_internal.h"

namespace wb {
namespace {

constexpr int kThreads = 256;
constexpr int kRows = 128;                 // MMA M
constexpr int kTile = kRows * 128;         // one 128 x 64 bf16 swizzled tile: 16 KB
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Byte offset of 16-byte chunk ch (0..7, eight bf16 along K) of row r in a
// K-major tile with 128-byte rows, 8-row groups 1024 bytes apart and the
// 128-byte swizzle (chunk ^= row % 8).
__host__ __device__ __forceinline__ uint32_t sw128(int r, int ch) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((ch ^ (r & 7)) << 4));
}

// UMMA shared-memory descriptor of a K-major SWIZZLE_128B tile starting at
// shared address a: start >> 4, leading offset 1 (unused by this layout),
// stride offset 1024 B between 8-row groups, version 1, layout type 2.
__device__ __forceinline__ uint64_t sdesc(uint32_t a) {
  return (uint64_t)((a >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete, at most kWaitNs.
__device__ bool mbar_wait(uint64_t* b, uint32_t parity, int* err, int code) {
  if (mbar_test(b, parity)) return true;
  const uint64_t t0 = globaltimer();
  while (!mbar_test(b, parity)) {
    if (globaltimer() - t0 > kWaitNs) {
      atomicExch(err, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {  // one full warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {  // one full warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (one full warp).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {  // a at the lower address
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
// Eight FP32 values -> their bf16 hi parts and bf16 lo parts (x - hi).
__device__ __forceinline__ void split8(const float (&x)[8], uint4& hi, uint4& lo) {
  float h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    h[i] = __bfloat162float(__float2bfloat16_rn(x[i]));
    l[i] = x[i] - h[i];
  }
  hi = make_uint4(pack2(h[0], h[1]), pack2(h[2], h[3]), pack2(h[4], h[5]), pack2(h[6], h[7]));
  lo = make_uint4(pack2(l[0], l[1]), pack2(l[2], l[3]), pack2(l[4], l[5]), pack2(l[6], l[7]));
}
// The same from FP64 (the constant W): lo = rn(w - hi) with w exact.
__device__ __forceinline__ void split8(const double (&x)[8], uint4& hi, uint4& lo) {
  float h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    h[i] = __bfloat162float(__double2bfloat16(x[i]));
    l[i] = (float)(x[i] - (double)h[i]);
  }
  hi = make_uint4(pack2(h[0], h[1]), pack2(h[2], h[3]), pack2(h[4], h[5]), pack2(h[6], h[7]));
  lo = make_uint4(pack2(l[0], l[1]), pack2(l[2], l[3]), pack2(l[4], l[5]), pack2(l[6], l[7]));
}

__host__ __device__ constexpr uint32_t tmem_cols(int n) {
  return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : n <= 256 ? 256u : 512u;
}

// ---------------------------------------------------------------------------
// setup: W (FP64, [M][K] with row stride ldw) -> swizzled bf16 hi/lo tiles
// ---------------------------------------------------------------------------
// bra-ket B operand: per 64-wide k block kb, [hi: NP rows x 128 B][lo: same]
__global__ void k_presplit_braket(const double* __restrict__ W, long ldw, int M, int K, int NP, int nkb,
                                  unsigned char* __restrict__ out) {
  const long n = (long)nkb * NP * 8;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const int ch = (int)(e & 7), r = (int)((e >> 3) % NP), kb = (int)(e / (8L * NP));
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = kb * 64 + ch * 8 + i;
      x[i] = (r < M && k < K) ? W[(long)r * ldw + k] : 0.0;
    }
    uint4 hi, lo;
    split8(x, hi, lo);
    unsigned char* base = out + (size_t)kb * NP * 256;
    *reinterpret_cast<uint4*>(base + sw128(r, ch)) = hi;
    *reinterpret_cast<uint4*>(base + (size_t)NP * 128 + sw128(r, ch)) = lo;
  }
}

// update A operand: per 128-row k tile kt and 64-wide r block rb,
// [hi: 128 rows (k) x 128 B (r)][lo: same]
__global__ void k_presplit_update(const double* __restrict__ W, long ldw, int M, int K, int nrb, int nkt,
                                  unsigned char* __restrict__ out) {
  const long n = (long)nkt * nrb * kRows * 8;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const int ch = (int)(e & 7), row = (int)((e >> 3) % kRows);
    const long tile = e / (8L * kRows);
    const int rb = (int)(tile % nrb), kt = (int)(tile / nrb);
    const int k = kt * kRows + row;
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = rb * 64 + ch * 8 + i;
      x[i] = (r < M && k < K) ? W[(long)r * ldw + k] : 0.0;
    }
    uint4 hi, lo;
    split8(x, hi, lo);
    unsigned char* base = out + (size_t)tile * 2 * kTile;
    *reinterpret_cast<uint4*>(base + sw128(row, ch)) = hi;
    *reinterpret_cast<uint4*>(base + kTile + sw128(row, ch)) = lo;
  }
}

// ---------------------------------------------------------------------------
// bra-ket: 128 systems x NP projectors per CTA, split over K, two stages
// ---------------------------------------------------------------------------
struct BraketArgs {
  const float* X;
  long ldx;
  const int* cols;
  int ncol, K;
  const unsigned char* Wt;  // k_presplit_braket tiles
  int NP, M, kb_per_split, nkb;
  float* part;
  int* err;
  const int* dn;  // device count of columns (graph replays) or null
  int ctas;       // split target of the device plan (with dn)
};

__host__ __device__ constexpr int braket_stage_bytes(int NP) { return 2 * kTile + NP * 256; }

__global__ void __launch_bounds__(kThreads, 2) k_braket_umma(BraketArgs a) {
  extern __shared__ unsigned char sm_raw[];
  const uint32_t pad = (1024u - (smem_addr(sm_raw) & 1023u)) & 1023u;
  unsigned char* sm = sm_raw + pad;
  const int SB = braket_stage_bytes(a.NP);
  uint64_t* wfull = reinterpret_cast<uint64_t*>(sm + 2 * SB);
  uint64_t* mdone = wfull + 2;
  uint32_t* slot = reinterpret_cast<uint32_t*>(mdone + 2);
  volatile int* abort_f = reinterpret_cast<volatile int*>(slot + 1);

  const int ncol = a.dn ? *a.dn : a.ncol;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int j0 = blockIdx.x * kRows;
  if (j0 >= ncol) return;  // before any TMEM or barrier state
  if (a.dn) {              // the split plan of this column count
    int ns;
    umma_braket_plan(ncol, a.K, &ns, &a.kb_per_split, a.ctas);
    if ((int)blockIdx.y >= ns) return;
  }
  const int kb0 = blockIdx.y * a.kb_per_split;
  const int nk = min(a.nkb, kb0 + a.kb_per_split) - kb0;
  const uint32_t ncols = tmem_cols(a.NP);
  if (warp == 0) tmem_alloc(slot, ncols);
  if (tid == 0) {
    mbar_init(&wfull[0], 1);
    mbar_init(&wfull[1], 1);
    mbar_init(&mdone[0], 1);
    mbar_init(&mdone[1], 1);
    *abort_f = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;

  // producer map: 4 passes of 32 rows, eight threads per row, eight k each
  const int ch = tid & 7;
  const float* xr[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int j = j0 + p * 32 + (tid >> 3);
    xr[p] = j < ncol ? a.X + (long)(a.cols ? a.cols[j] : j) * a.ldx : nullptr;
  }
  float v[4][8];
  auto load = [&](int kb) {
    const int k = kb * 64 + ch * 8;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      if (xr[p] && k + 8 <= a.K) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 t = __ldg(reinterpret_cast<const float2*>(xr[p] + k) + q);
          v[p][2 * q] = t.x;
          v[p][2 * q + 1] = t.y;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[p][i] = (xr[p] && k + i < a.K) ? __ldg(xr[p] + k + i) : 0.f;
      }
    }
  };
  auto store = [&](int s) {
    unsigned char* ah = sm + s * SB;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      uint4 hi, lo;
      split8(v[p], hi, lo);
      const uint32_t o = sw128(p * 32 + (tid >> 3), ch);
      *reinterpret_cast<uint4*>(ah + o) = hi;
      *reinterpret_cast<uint4*>(ah + kTile + o) = lo;
    }
  };

  const uint32_t idesc = idesc_bf16(kRows, a.NP);
  const uint32_t wbytes = (uint32_t)a.NP * 256u;
  uint32_t mph = 0u, wph = 0u;  // phase parity per stage, bit s
  load(kb0);
  for (int it = 0; it < nk; ++it) {
    const int s = it & 1;
    if (it >= 2 && !*abort_f) {  // the MMAs that read stage s two blocks ago
      if (!mbar_wait(&mdone[s], (mph >> s) & 1u, a.err, 1)) *abort_f = 1;
      mph ^= 1u << s;
    }
    if (tid == 0 && !*abort_f) {
      mbar_expect_tx(&wfull[s], wbytes);
      bulk_g2s(sm + s * SB + 2 * kTile, a.Wt + (size_t)(kb0 + it) * wbytes, wbytes, &wfull[s]);
    }
    store(s);
    if (it + 1 < nk) load(kb0 + it + 1);
    fence_async_smem();
    __syncthreads();
    if (tid == 0 && !*abort_f) {
      if (!mbar_wait(&wfull[s], (wph >> s) & 1u, a.err, 2)) *abort_f = 1;
      wph ^= 1u << s;
      if (!*abort_f) {
        tc_fence_after();
        const uint32_t ah = smem_addr(sm + s * SB), al = ah + kTile, bh = ah + 2 * kTile, bl = bh + a.NP * 128;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t o = q * 32;
          mma_bf16(tmem, sdesc(ah + o), sdesc(bh + o), idesc, (it | q) != 0);
          mma_bf16(tmem, sdesc(ah + o), sdesc(bl + o), idesc, 1u);
          mma_bf16(tmem, sdesc(al + o), sdesc(bh + o), idesc, 1u);
        }
        mma_commit(&mdone[s]);
      }
    }
  }
  // the commits of the last two blocks
  for (int it = max(0, nk - 2); it < nk && !*abort_f; ++it) {
    const int s = it & 1;
    if (!mbar_wait(&mdone[s], (mph >> s) & 1u, a.err, 3)) *abort_f = 1;
    mph ^= 1u << s;
  }
  __syncthreads();
  const bool ok = !*abort_f;
  tc_fence_after();
  if (ok && warp < 4) {
    const int j = j0 + warp * 32 + lane;
    float* dst = a.part + ((long)blockIdx.y * ncol + j) * a.M;
    for (int c0 = 0; c0 < a.NP; c0 += 16) {
      float d[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, d);
      if (j < ncol) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (c0 + i < a.M) dst[c0 + i] = d[i];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, ncols);
  }
}

// ---------------------------------------------------------------------------
// update: 128 k rows x NJ systems per CTA, K of the MMA = projectors
// ---------------------------------------------------------------------------
struct UpdateArgs {
  const unsigned char* Wt;  // k_presplit_update tiles
  int NP, nrb;
  const float* C;
  int M;
  float* Y;
  long ldy;
  const int* cols;
  int ncol, K, NJ;
  int* err;
  const int* dn;
};

__host__ __device__ constexpr int update_smem_bytes(int nrb, int NJ) { return nrb * 2 * kTile + nrb * NJ * 256 + 64 + 1024; }

__global__ void __launch_bounds__(kThreads, 3) k_update_umma(UpdateArgs a) {
  extern __shared__ unsigned char sm_raw[];
  const uint32_t pad = (1024u - (smem_addr(sm_raw) & 1023u)) & 1023u;
  unsigned char* sm = sm_raw + pad;
  const int NJ = a.NJ, nrb = a.nrb;
  unsigned char* At = sm;                          // nrb x [hi, lo] x 16 KB
  unsigned char* Bt = sm + nrb * 2 * kTile;        // nrb x [hi, lo] x NJ x 128 B
  uint64_t* afull = reinterpret_cast<uint64_t*>(Bt + nrb * NJ * 256);
  uint64_t* done = afull + 1;
  uint32_t* slot = reinterpret_cast<uint32_t*>(done + 1);

  const int ncol = a.dn ? *a.dn : a.ncol;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k0 = blockIdx.x * kRows, jt0 = blockIdx.y * NJ;
  if (jt0 >= ncol) return;  // before any TMEM or barrier state
  const uint32_t ncols = tmem_cols(NJ);
  if (warp == 0) tmem_alloc(slot, ncols);
  if (tid == 0) {
    mbar_init(afull, 1);
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  if (tid == 0) {
    mbar_expect_tx(afull, (uint32_t)(nrb * 2 * kTile));
    const unsigned char* src = a.Wt + (size_t)blockIdx.x * nrb * 2 * kTile;
    for (int t = 0; t < 2 * nrb; ++t) bulk_g2s(At + t * kTile, src + (size_t)t * kTile, kTile, afull);
  }
  // C tile (NJ systems x 64 nrb projectors), split into bf16 hi/lo
  for (int e = tid; e < NJ * nrb * 8; e += kThreads) {
    const int ch = e & 7, row = (e >> 3) % NJ, rb = e / (8 * NJ);
    const int j = jt0 + row, r0 = rb * 64 + ch * 8;
    float x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (j < ncol && r0 + i < a.M) ? __ldg(a.C + (long)j * a.M + r0 + i) : 0.f;
    uint4 hi, lo;
    split8(x, hi, lo);
    unsigned char* b = Bt + rb * NJ * 256;
    *reinterpret_cast<uint4*>(b + sw128(row, ch)) = hi;
    *reinterpret_cast<uint4*>(b + NJ * 128 + sw128(row, ch)) = lo;
  }
  fence_async_smem();
  __syncthreads();
  __shared__ int abort_s;
  if (tid == 0) {
    abort_s = 0;
    if (!mbar_wait(afull, 0, a.err, 4)) {
      abort_s = 1;
    } else {
      tc_fence_after();
      const uint32_t idesc = idesc_bf16(kRows, NJ);
      const uint32_t a0 = smem_addr(At), b0 = smem_addr(Bt);
      for (int q = 0; q < a.NP / 16; ++q) {
        const int rb = q >> 2;
        const uint32_t o = (q & 3) * 32;
        const uint32_t ah = a0 + rb * 2 * kTile, al = ah + kTile;
        const uint32_t bh = b0 + rb * NJ * 256, bl = bh + NJ * 128;
        mma_bf16(tmem, sdesc(ah + o), sdesc(bh + o), idesc, q != 0);
        mma_bf16(tmem, sdesc(ah + o), sdesc(bl + o), idesc, 1u);
        mma_bf16(tmem, sdesc(al + o), sdesc(bh + o), idesc, 1u);
      }
      mma_commit(done);
    }
  }
  __syncthreads();
  // epilogue map: warp w reads TMEM lanes 32 (w % 4) .. +31 (k rows) and half
  // w / 4 of the NJ columns (systems), 16 columns per tcgen05.ld
  const int lq = warp & 3, half = warp >> 2;
  const int k = k0 + lq * 32 + lane;
  const int cbeg = half * (NJ / 2), cend = cbeg + NJ / 2;
  int ycol[16];  // column of Y per TMEM column, -1 outside the matrix
  float yv[16];
  // Y of the first 16 columns is read while the MMAs run
  auto load_y = [&](int c0) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int j = jt0 + c0 + i;
      ycol[i] = (j < ncol && k < a.K) ? (a.cols ? a.cols[j] : j) : -1;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) yv[i] = ycol[i] >= 0 ? a.Y[(long)ycol[i] * a.ldy + k] : 0.f;
  };
  load_y(cbeg);
  bool ok = !abort_s;
  if (ok && !mbar_wait(done, 0, a.err, 5)) ok = false;
  // a thread that timed out skips its own stores; the warp stays converged for tcgen05.ld
  ok = __all_sync(0xffffffffu, ok);
  tc_fence_after();
  if (ok) {
    for (int c0 = cbeg; c0 < cend; c0 += 16) {
      float d[16];
      tmem_ld16(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)c0, d);
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (ycol[i] >= 0) a.Y[(long)ycol[i] * a.ldy + k] = yv[i] + d[i];
      if (c0 + 16 < cend) load_y(c0 + 16);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, ncols);
  }
}

int update_nj(int nrb) { return nrb <= 2 ? 128 : 64; }

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool umma_supported(int M) { return M >= 1 && M <= 256; }

int umma_np(int M) { return (M + 15) / 16 * 16; }

size_t umma_part_floats(int M, int nsys, int K) {
  size_t best = 0;
  for (int t = 1; t <= (nsys + kRows - 1) / kRows; ++t) {
    const int n = std::min(nsys, t * kRows);
    for (int c = 1; c <= kUmmaMaxCtas; ++c) {
      int ns, per;
      umma_braket_plan(n, K, &ns, &per, c);
      best = std::max(best, (size_t)ns * n * M);
    }
  }
  return best;
}

size_t umma_braket_bytes(int M, int K) { return (size_t)((K + 63) / 64) * umma_np(M) * 256; }
size_t umma_update_bytes(int M, int K) {
  return (size_t)((K + kRows - 1) / kRows) * ((umma_np(M) + 63) / 64) * 2 * kTile;
}

void umma_presplit(const double* W, long ldw, int M, int K, void* braket_tiles, void* update_tiles,
                   cudaStream_t s) {
  const int NP = umma_np(M), nkb = (K + 63) / 64, nrb = (NP + 63) / 64, nkt = (K + kRows - 1) / kRows;
  k_presplit_braket<<<1024, 256, 0, s>>>(W, ldw, M, K, NP, nkb, static_cast<unsigned char*>(braket_tiles));
  k_presplit_update<<<1024, 256, 0, s>>>(W, ldw, M, K, nrb, nkt, static_cast<unsigned char*>(update_tiles));
}

static size_t braket_smem(int NP) { return 2 * (size_t)braket_stage_bytes(NP) + 64 + 1024; }

void umma_setup() {
  cudaFuncSetAttribute(k_braket_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)braket_smem(256));
  cudaFuncSetAttribute(k_update_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, update_smem_bytes(4, 64));
}

int umma_braket(const void* tiles, int M, const float* X, long ldx, const int* cols, int ncol, int K, float* part,
                int* err, cudaStream_t s, const int* dn, int ctas_per_sm) {
  if (ncol <= 0) return 1;
  BraketArgs a{};
  a.X = X;
  a.ldx = ldx;
  a.cols = cols;
  a.ncol = ncol;
  a.K = K;
  a.Wt = static_cast<const unsigned char*>(tiles);
  a.NP = umma_np(M);
  a.M = M;
  a.nkb = (K + 63) / 64;
  int nsplit;
  a.ctas = std::min(std::max(ctas_per_sm, 1), kUmmaMaxCtas);
  // a device count launches the largest plan's split grid (one column)
  umma_braket_plan(dn ? 1 : ncol, K, &nsplit, &a.kb_per_split, a.ctas);
  a.part = part;
  a.err = err;
  a.dn = dn;
  const dim3 grid((ncol + kRows - 1) / kRows, nsplit);
  k_braket_umma<<<grid, kThreads, braket_smem(a.NP), s>>>(a);
  return nsplit;
}

void umma_update(const void* tiles, int M, const float* C, float* Y, long ldy, const int* cols, int ncol, int K,
                 int* err, cudaStream_t s, const int* dn, int nj) {
  if (ncol <= 0) return;
  UpdateArgs a{};
  a.Wt = static_cast<const unsigned char*>(tiles);
  a.NP = umma_np(M);
  a.nrb = (a.NP + 63) / 64;
  a.C = C;
  a.M = M;
  a.Y = Y;
  a.ldy = ldy;
  a.cols = cols;
  a.ncol = ncol;
  a.K = K;
  a.NJ = (nj == 64 || (nj == 128 && a.nrb <= 2)) ? nj : update_nj(a.nrb);
  a.err = err;
  a.dn = dn;
  const dim3 grid((K + kRows - 1) / kRows, (ncol + a.NJ - 1) / a.NJ);
  k_update_umma<<<grid, kThreads, update_smem_bytes(a.nrb, a.NJ), s>>>(a);
}

}  // namespace wb
