// Legendre contraction on tcgen05 tensor cores, split-BF16 with FP32
// accumulation (DINO_PREC_BF16X3).
//
// Every FP32 operand x is split into x_hi = bf16(x) and x_lo = bf16(x - x_hi);
// each product is formed as hi*hi + hi*lo + lo*hi (the lo*lo term, ~2^-16
// relative, is dropped) and accumulated in FP32 in tensor memory.  The
// Legendre tables are split from their FP64 values.
//
// Per zonal wavenumber m the contraction is a GEMM
//   inverse:  D[r, j]  = sum_{l'} X_p[r, l'] P_p[j, l']   (K = l', N = j)
//   forward:  D[r, l'] = sum_j  G_p[r, j]  P_p[l', j]     (K = j,  N = l')
// with r = (field, cos/sin) rows, p the parity of l - m (the N/S fold),
// l = m + 2 l' + p, and G_0 / G_1 the symmetric / antisymmetric latitude
// folds.  All operands are K-major bf16 in HBM, loaded by TMA (no multicast)
// into 128-byte-swizzled shared memory tiles; one thread issues
// tcgen05.mma (M = 128, N = latitudes or l', K = 16 per instruction) into two
// TMEM accumulators (one per parity); four warps read them back with
// tcgen05.ld and write the unfolded FP32 result.  Only the K steps and N
// columns that the triangular (m, l) range needs are issued.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dino_internal.cuh"

namespace dino {

typedef __nv_bfloat16 bf16;

struct TcTables {
  int Kp = 0;   // inverse K extent (l'), multiple of 64
  int Np = 0;   // inverse N (latitudes), multiple of 16
  int Kj = 0;   // forward K extent (latitudes), multiple of 64
  int Nf = 0;   // forward N (l'), multiple of 16
  int cap = 0;  // fields per launch
  int Rp = 0;   // rows per (m, parity) slab of the A operands
  bf16 *Bih = nullptr, *Bil = nullptr, *Bfh = nullptr, *Bfl = nullptr;
  bf16 *Aih = nullptr, *Ail = nullptr, *Afh = nullptr, *Afl = nullptr;
  CUtensorMap tAih, tAil, tBih, tBil, tAfh, tAfl, tBfh, tBfl;
  int* d_err = nullptr;
  int stages_inv = 0, stages_fwd = 0;
  size_t smem_inv = 0, smem_fwd = 0;
  // N sub-ranges per (m, row tile) CTA and their width (B tile rows).
  int nsplit_inv = 1, nsplit_fwd = 1, Nsub_inv = 0, Nsub_fwd = 0;
  // Autotuning record: candidates tried and the chosen launch time.
  int tuned_fields = 0, tried_inv = 0, tried_fwd = 0;
  float us_inv = 0.f, us_fwd = 0.f;
};

__host__ __device__ __forceinline__ int round_up(int x, int m) { return (x + m - 1) / m * m; }

// ---------------------------------------------------------------------------
// Operand preparation
// ---------------------------------------------------------------------------

// FP64 recurrence (as in plan.cu) written as split bf16 into the inverse
// table [m][p][j][Kp] and the forward table [m][p][l'][Kj].
__global__ void tc_table_kernel(int lw, int L, int Jh, const double* __restrict__ x,
                                int Kp, int Np, int Kj, int Nf,
                                bf16* __restrict__ Bih, bf16* __restrict__ Bil,
                                bf16* __restrict__ Bfh, bf16* __restrict__ Bfl) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int m = blockIdx.y;
  if (j >= Jh || m >= lw) return;
  double xj = x[j];
  double y = sqrt(1.0 - xj * xj);
  double diag = 1.0 / sqrt(2.0);
  for (int mm = 1; mm <= m; ++mm) diag = -sqrt(1.0 + 1.0 / (2.0 * mm)) * y * diag;
  double p2 = 0.0, p1 = diag;
  double m2 = (double)m * m;
  for (int k = 0; k < L - m; ++k) {
    double cur;
    if (k == 0) {
      cur = diag;
    } else {
      double mk2 = (double)(m + k) * (m + k);
      double mkp2 = (double)(m + k - 1) * (m + k - 1);
      double a = sqrt((4.0 * mk2 - 1.0) / (mk2 - m2));
      double b = sqrt((mkp2 - m2) / (4.0 * mkp2 - 1.0));
      cur = a * (xj * p1 - b * p2);
      p2 = p1;
      p1 = cur;
    }
    bf16 hi = __double2bfloat16(cur);
    bf16 lo = __double2bfloat16(cur - (double)__bfloat162float(hi));
    int p = k & 1, kk = k >> 1;
    size_t ii = ((size_t)(m * 2 + p) * Np + j) * Kp + kk;
    size_t fi = ((size_t)(m * 2 + p) * Nf + kk) * Kj + j;
    Bih[ii] = hi;
    Bil[ii] = lo;
    Bfh[fi] = hi;
    Bfl[fi] = lo;
  }
}

__device__ __forceinline__ void split_bf16(float v, bf16& hi, bf16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

__device__ __forceinline__ void tc_row_map(int m, int r, int& b, int& row) {
  if (m == 0) {
    b = r;
    row = 0;
  } else {
    b = r >> 1;
    row = 2 * m - 1 + (r & 1);
  }
}

// Eight consecutive split values as one 16-byte store of each half.
__device__ __forceinline__ void store_split8(const float (&v)[8], bf16* hi, bf16* lo) {
  __align__(16) bf16 h[8];
  __align__(16) bf16 l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) split_bf16(v[i], h[i], l[i]);
  *reinterpret_cast<uint4*>(hi) = *reinterpret_cast<const uint4*>(h);
  *reinterpret_cast<uint4*>(lo) = *reinterpret_cast<const uint4*>(l);
}

// Modal rows -> A[m][p][r][kk] = x[b][row][m + 2 kk + p], zero-padded to the
// next multiple of 64 in kk.  A thread converts 8 consecutive kk of both
// parities (16 consecutive l, read as one contiguous run) and writes them as
// 16-byte stores.
__global__ void tc_split_inverse_kernel(Segs in, int nf, int M, int L, int Rp,
                                        int Kp, int roff, bf16* __restrict__ Ah,
                                        bf16* __restrict__ Al) {
  const int m = blockIdx.y;
  const int rows = (m == 0) ? nf : 2 * nf;
  const int Lm = L - m;
  const int gw = round_up((Lm + 1) >> 1, 64) / 8;  // 8-kk groups per row
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)rows * gw) return;
  const int g = idx % gw;
  const int r = idx / gw;
  int b, row;
  tc_row_map(m, r, b, row);
  const float* xr = seg_field(in, b, (size_t)M * L) + (size_t)row * L + m;
  const int k0 = 16 * g;
  float ev[8], od[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int ke = k0 + 2 * i, ko = ke + 1;
    ev[i] = (ke < Lm) ? xr[ke] : 0.f;
    od[i] = (ko < Lm) ? xr[ko] : 0.f;
  }
  const size_t o0 = ((size_t)(m * 2) * Rp + roff + r) * Kp + 8 * g;
  const size_t o1 = ((size_t)(m * 2 + 1) * Rp + roff + r) * Kp + 8 * g;
  store_split8(ev, Ah + o0, Al + o0);
  store_split8(od, Ah + o1, Al + o1);
}

// Weighted Fourier coefficients G[b][row][j] -> symmetric (p = 0) and
// antisymmetric (p = 1) latitude folds, split into A[m][p][r][j].  A thread
// folds 8 consecutive latitudes against their mirrors and writes 16-byte
// stores.
__global__ void tc_fold_forward_kernel(const float* __restrict__ G, int nf, int M,
                                       int J, int Jh, int Rp, int Kj, int roff,
                                       bf16* __restrict__ Ah, bf16* __restrict__ Al) {
  const int m = blockIdx.y;
  const int rows = (m == 0) ? nf : 2 * nf;
  const int gw = Kj / 8;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)rows * gw) return;
  const int g = idx % gw;
  const int r = idx / gw;
  int b, row;
  tc_row_map(m, r, b, row);
  const float* gr = G + ((size_t)b * M + row) * J;
  const int j0 = 8 * g;
  float sv[8], dv[8];
  if (j0 + 8 <= Jh && (J & 3) == 0) {
    // Aligned fast path: j0..j0+7 and J-8-j0..J-1-j0 are float4 pairs.
    const float4 a0 = *reinterpret_cast<const float4*>(gr + j0);
    const float4 a1 = *reinterpret_cast<const float4*>(gr + j0 + 4);
    const float4 b0 = *reinterpret_cast<const float4*>(gr + J - 8 - j0);
    const float4 b1 = *reinterpret_cast<const float4*>(gr + J - 4 - j0);
    const float d[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float e[8] = {b1.w, b1.z, b1.y, b1.x, b0.w, b0.z, b0.y, b0.x};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      sv[i] = d[i] + e[i];
      dv[i] = d[i] - e[i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int j = j0 + i;
      float s = 0.f, d = 0.f;
      if (j < Jh) {
        const float g1 = gr[j];
        const int jm = J - 1 - j;
        const float g2 = (jm != j) ? gr[jm] : 0.f;
        s = g1 + g2;
        d = g1 - g2;
      }
      sv[i] = s;
      dv[i] = d;
    }
  }
  const size_t o0 = ((size_t)(m * 2) * Rp + roff + r) * Kj + j0;
  const size_t o1 = ((size_t)(m * 2 + 1) * Rp + roff + r) * Kj + j0;
  store_split8(sv, Ah + o0, Al + o0);
  store_split8(dv, Ah + o1, Al + o1);
}

// ---------------------------------------------------------------------------
// tcgen05 / TMA / mbarrier primitives (inline PTX)
// ---------------------------------------------------------------------------

constexpr int kTcThreads = 128;
constexpr int kMaxStages = 4;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity; gives up after kWaitLimitNs,
// records `code` in *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          int* err, int code) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_test(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) {
      atomicCAS(err, 0, code);
      return false;
    }
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm,
                                            uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), leading offset unused for swizzled K-major.
__device__ __forceinline__ uint64_t umma_desc_sw128(const void* p) {
  uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= 1ull << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= 1ull << 46;
  d |= 2ull << 61;
  return d;
}

// kind::f16 instruction descriptor: D = F32, A = B = BF16, both K-major,
// M = 128, N = n.
__device__ __forceinline__ uint32_t umma_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
        "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------
// The contraction kernel
// ---------------------------------------------------------------------------

struct TcArgs {
  int nf, M, L, J, Jh;
  int Rp;        // A slab rows
  int roff;      // first A slab row of this launch (operand-slab half)
  int Nrows;     // rows of one (m, parity) B table (Np or Nf)
  int Nsub;      // B tile rows = N columns of this CTA (blockIdx.z-th range)
  int stages;
  int tmem_cols; // allocated TMEM columns (power of two)
  float* out;    // inverse: Fourier [nf][M][J]; forward: modal [nf][M][L]
  int* err;
};

template <bool kForward>
__global__ void __launch_bounds__(kTcThreads, 2)
legendre_tc_kernel(const __grid_constant__ CUtensorMap tAh,
                   const __grid_constant__ CUtensorMap tAl,
                   const __grid_constant__ CUtensorMap tBh,
                   const __grid_constant__ CUtensorMap tBl, TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kMaxStages];
  __shared__ __align__(8) uint64_t empty_bar[kMaxStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_slot;

  const int m = blockIdx.y;
  const int tile = blockIdx.x;
  const int rows = (m == 0) ? a.nf : 2 * a.nf;
  if (tile * 128 >= rows) return;  // uniform for the CTA

  const int Lm = a.L - m;
  const int n_par[2] = {(Lm + 1) >> 1, Lm >> 1};
  // This CTA's N range: latitudes (inverse) or l' (forward) lo .. lo+Nsub-1.
  const int lo = blockIdx.z * a.Nsub;
  int kblk[2], ksteps[2], ncols[2], cnt[2];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    if (!kForward) {
      kblk[p] = (n_par[p] + 63) / 64;
      ksteps[p] = (n_par[p] + 15) / 16;
      ncols[p] = a.Nsub;
      cnt[p] = n_par[p];
    } else {
      cnt[p] = max(0, min(n_par[p] - lo, a.Nsub));
      kblk[p] = cnt[p] ? (a.Jh + 63) / 64 : 0;
      ksteps[p] = (a.Jh + 15) / 16;
      ncols[p] = round_up(cnt[p] > 0 ? cnt[p] : 16, 16);
    }
  }
  // Uniform early exits: no output column in this range.
  if (kForward && cnt[0] == 0) return;
  if (!kForward && lo >= a.Jh) return;
  const int nblocks = kblk[0] + kblk[1];
  const uint32_t tile_a = 128u * 128u;             // 128 rows x 64 bf16
  const uint32_t tile_b = (uint32_t)a.Nsub * 128u;  // Nsub rows x 64 bf16
  const uint32_t stage_bytes = 2 * tile_a + 2 * tile_b;
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* base = smem_raw + pad;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < a.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const int acc_cols = a.Nsub;  // parity p accumulates at column p * Nsub

  if (threadIdx.x == 0) {
    // TMA producer.
    for (int i = 0; i < nblocks; ++i) {
      const int s = i % a.stages;
      const int use = i / a.stages;
      if (use > 0 && !mbar_wait(&empty_bar[s], (use - 1) & 1, a.err, 1)) break;
      const int p = (i < kblk[0]) ? 0 : 1;
      const int k = (p == 0) ? i : i - kblk[0];
      uint8_t* st = base + (size_t)s * stage_bytes;
      mbar_expect_tx(&full_bar[s], stage_bytes);
      const int ya = (m * 2 + p) * a.Rp + a.roff + tile * 128;
      const int yb = (m * 2 + p) * a.Nrows + lo;
      tma_load_2d(st, &tAh, &full_bar[s], k * 64, ya);
      tma_load_2d(st + tile_a, &tAl, &full_bar[s], k * 64, ya);
      tma_load_2d(st + 2 * tile_a, &tBh, &full_bar[s], k * 64, yb);
      tma_load_2d(st + 2 * tile_a + tile_b, &tBl, &full_bar[s], k * 64, yb);
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer: hi*hi + hi*lo + lo*hi per K step of 16.
    for (int i = 0; i < nblocks; ++i) {
      const int s = i % a.stages;
      const int use = i / a.stages;
      if (!mbar_wait(&full_bar[s], use & 1, a.err, 2)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int p = (i < kblk[0]) ? 0 : 1;
      const int k = (p == 0) ? i : i - kblk[0];
      const int steps = min(4, ksteps[p] - k * 4);
      const uint32_t d = tmem + (uint32_t)(p * acc_cols);
      const uint32_t idesc = umma_idesc_bf16(ncols[p]);
      uint8_t* st = base + (size_t)s * stage_bytes;
      const uint64_t dah = umma_desc_sw128(st);
      const uint64_t dal = umma_desc_sw128(st + tile_a);
      const uint64_t dbh = umma_desc_sw128(st + 2 * tile_a);
      const uint64_t dbl = umma_desc_sw128(st + 2 * tile_a + tile_b);
      for (int q = 0; q < steps; ++q) {
        const uint64_t off = (uint64_t)(2 * q);  // 32 bytes per K step, in 16 B units
        const uint32_t acc = (k > 0 || q > 0) ? 1u : 0u;
        umma_bf16(d, dah + off, dbh + off, idesc, acc);
        umma_bf16(d, dah + off, dbl + off, idesc, 1u);
        umma_bf16(d, dal + off, dbh + off, idesc, 1u);
      }
      umma_commit(&empty_bar[s]);
    }
    // Arrives once every MMA issued above has completed.
    umma_commit(&done_bar);
  }
  __syncwarp();
  bool ok = mbar_wait(&done_bar, 0, a.err, 3);
  ok = __all_sync(0xffffffffu, ok);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok) {
    // Epilogue.  Each warp owns TMEM lanes (rows) 32w .. 32w+31; a thread
    // reads its row's accumulator columns, the warp stages a 32-row block in
    // shared memory (the drained pipeline buffers) and writes it back with
    // row-contiguous, coalesced stores.
    constexpr int kStride = 36;  // floats per staged row (16-byte multiple)
    float* stage = reinterpret_cast<float*>(base) + warp * 32 * kStride;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    const int row0 = tile * 128 + warp * 32;  // first row of this warp
    if (!kForward) {
      const bool vec = (a.J & 3) == 0;
      for (int c = 0; c < a.Nsub / 16; ++c) {
        float e[16], od[16];
        tmem_ld16(lane_base + c * 16, e);
        if (n_par[1] > 0) {
          tmem_ld16(lane_base + acc_cols + c * 16, od);
        } else {
#pragma unroll
          for (int t = 0; t < 16; ++t) od[t] = 0.f;
        }
        // stage[r][t] = E + O at j = 16c + t; stage[r][16 + t] = E - O at
        // j = J - 16(c+1) + t (the mirrored block, ascending).
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          stage[lane * kStride + t] = e[t] + od[t];
          stage[lane * kStride + 16 + (15 - t)] = e[t] - od[t];
        }
        __syncwarp();
        const int jb = lo + 16 * c;
        const int jm = a.J - jb - 16;
        // 4 threads per row, 8 rows per pass, 4 passes; two half-blocks.
        for (int pass = 0; pass < 8; ++pass) {
          const int half = pass >> 2;                 // 0: direct, 1: mirror
          const int r = (pass & 3) * 8 + (lane >> 2);  // staged row
          const int q = lane & 3;                      // float4 within 16
          const int rr = row0 + r;
          if (rr < rows) {
            int b, row;
            tc_row_map(m, rr, b, row);
            float* o = a.out + ((size_t)b * a.M + row) * a.J;
            const float* src = stage + r * kStride + half * 16 + q * 4;
            const int j = (half ? jm : jb) + q * 4;
            if (vec && jb + 16 <= a.Jh && (half == 0 || jm >= a.Jh)) {
              *reinterpret_cast<float4*>(o + j) =
                  *reinterpret_cast<const float4*>(src);
            } else {
#pragma unroll
              for (int e2 = 0; e2 < 4; ++e2) {
                const int jj = j + e2;
                // direct half covers j < Jh; mirrored half covers j >= J - Jh
                // except the self-mirrored middle row of an odd J.
                if (half == 0) {
                  if (jj < a.Jh) o[jj] = src[e2];
                } else {
                  const int jsrc = a.J - 1 - jj;  // its direct index
                  if (jsrc >= 0 && jsrc < a.Jh && jsrc != jj) o[jj] = src[e2];
                }
              }
            }
          }
        }
        __syncwarp();
      }
    } else {
      // Structural zeros l < m (first N range only), one row at a time.
      for (int r = 0; r < 32 && lo == 0; ++r) {
        const int rr = row0 + r;
        if (rr >= rows) break;
        int b, row;
        tc_row_map(m, rr, b, row);
        float* o = a.out + ((size_t)b * a.M + row) * a.L;
        for (int l = lane; l < m; l += 32) o[l] = 0.f;
      }
      const int nchunks = (max(cnt[0], cnt[1]) + 15) / 16;
      for (int c = 0; c < nchunks; ++c) {
        float e[16], od[16];
        tmem_ld16(lane_base + c * 16, e);
        if (cnt[1] > 0) {
          tmem_ld16(lane_base + acc_cols + c * 16, od);
        } else {
#pragma unroll
          for (int t = 0; t < 16; ++t) od[t] = 0.f;
        }
        // Interleave parities: l = m + 32c + 2t + p.
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          stage[lane * kStride + 2 * t] = e[t];
          stage[lane * kStride + 2 * t + 1] = od[t];
        }
        __syncwarp();
        const int lbase = m + 2 * (lo + 16 * c);
        for (int r = 0; r < 32; ++r) {
          const int rr = row0 + r;
          if (rr >= rows) break;
          const int l = lbase + lane;
          const int lp = lo + 16 * c + (lane >> 1);
          const bool keep = (lane & 1) ? (lp < n_par[1]) : (lp < n_par[0]);
          if (keep && l < a.L) {
            int b, row;
            tc_row_map(m, rr, b, row);
            a.out[((size_t)b * a.M + row) * a.L + l] = stage[r * kStride + lane];
          }
        }
        __syncwarp();
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(a.tmem_cols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

static int make_map(CUtensorMap* tm, const bf16* ptr, int inner, long long rows,
                    int box_rows) {
  auto fn = encode_fn();
  DINO_REQUIRE(fn != nullptr, DINO_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  DINO_REQUIRE(((uintptr_t)ptr & 15) == 0, DINO_ERR_ARG, "TMA base must be 16-byte aligned");
  DINO_REQUIRE(inner % 64 == 0 && box_rows >= 8 && box_rows <= 256, DINO_ERR_ARG,
               "bad TMA box");
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(bf16)};
  cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  cuuint32_t elem[2] = {1u, 1u};
  CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)ptr, dims, strides, box,
                  elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return DINO_ERR_CUDA;
  }
  return DINO_OK;
}

// ---------------------------------------------------------------------------
// Autotuning of the tensor-core launch shape
// ---------------------------------------------------------------------------

constexpr size_t kTcSmemLimit = 220 * 1024;

int tc_status(dino_plan* p);

static int tmem_cols_for(int cols);

// One candidate shape for a direction: the (m, row tile) CTA's N range is
// split into nsplit ranges of Nsub rows, with a pipeline `stages` deep.
struct TcShape {
  int nsplit, Nsub, stages;
  size_t smem;
};

static void tc_candidates(int nfull, std::vector<TcShape>* out) {
  int last_nsub = -1;
  for (int nsplit : {1, 2, 4}) {
    const int nsub = round_up((nfull + nsplit - 1) / nsplit, 16);
    if (nsub == last_nsub || (nsplit > 1 && nsub * (nsplit - 1) >= nfull)) continue;
    last_nsub = nsub;
    if (tmem_cols_for(2 * nsub) > 512) continue;
    const size_t stage = 2 * 128 * 128 + 2 * (size_t)nsub * 128;
    for (int stages = 2; stages <= kMaxStages; ++stages) {
      const size_t smem = stage * stages + 1024;
      if (smem > kTcSmemLimit) break;
      out->push_back({nsplit, nsub, stages, smem});
    }
  }
}

template <bool kForward>
static int tc_time_shape(dino_plan* p, TcTables* t, const TcShape& c, int nf, float* out,
                         cudaEvent_t e0, cudaEvent_t e1, float* us) {
  const size_t lw2 = (size_t)p->lw * 2;
  CUtensorMap bh, bl;
  if (!kForward) {
    DINO_TRY(make_map(&bh, t->Bih, t->Kp, (long long)lw2 * t->Np, c.Nsub));
    DINO_TRY(make_map(&bl, t->Bil, t->Kp, (long long)lw2 * t->Np, c.Nsub));
  } else {
    DINO_TRY(make_map(&bh, t->Bfh, t->Kj, (long long)lw2 * t->Nf, c.Nsub));
    DINO_TRY(make_map(&bl, t->Bfl, t->Kj, (long long)lw2 * t->Nf, c.Nsub));
  }
  TcArgs a{};
  a.nf = nf;
  a.M = p->M;
  a.L = p->L;
  a.J = p->J;
  a.Jh = p->Jh;
  a.Rp = t->Rp;
  a.Nrows = kForward ? t->Nf : t->Np;
  a.Nsub = c.Nsub;
  a.stages = c.stages;
  a.tmem_cols = tmem_cols_for(2 * c.Nsub);
  a.out = out;
  a.err = t->d_err;
  dim3 grid(ceil_div(2 * nf, 128), p->lw, c.nsplit);
  const CUtensorMap& ah = kForward ? t->tAfh : t->tAih;
  const CUtensorMap& al = kForward ? t->tAfl : t->tAil;
  constexpr int kReps = 3;
  for (int r = 0; r <= kReps; ++r) {
    if (r == 1) DINO_CHECK_CUDA(cudaEventRecord(e0, 0));
    legendre_tc_kernel<kForward><<<grid, kTcThreads, c.smem, 0>>>(ah, al, bh, bl, a);
    DINO_TRY(check_launch("legendre_tc (autotune)"));
  }
  DINO_CHECK_CUDA(cudaEventRecord(e1, 0));
  DINO_CHECK_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  DINO_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  *us = 1e3f * ms / kReps;
  return DINO_OK;
}

// Times every candidate shape of both directions on this plan's tables with
// an L2-sized batch (the chunk the transforms launch) and keeps the fastest.
static int tc_autotune(dino_plan* p, TcTables* t) {
  const size_t per_field = (size_t)p->M * p->J * sizeof(float);
  int nf = (int)((48ull << 20) / (per_field ? per_field : 1));
  nf = nf < 1 ? 1 : nf;
  nf = nf > t->cap ? t->cap : nf;
  t->tuned_fields = nf;
  float* fwd_out = nullptr;
  DINO_CHECK_CUDA(cudaMalloc(&fwd_out, sizeof(float) * (size_t)nf * p->M * p->L));
  cudaEvent_t e0, e1;
  DINO_CHECK_CUDA(cudaEventCreate(&e0));
  DINO_CHECK_CUDA(cudaEventCreate(&e1));
  auto tune = [&](bool forward) -> int {
    std::vector<TcShape> cands;
    tc_candidates(forward ? t->Nf : t->Np, &cands);
    float best = 1e30f;
    TcShape pick = cands.front();
    for (const TcShape& c : cands) {
      float us = 0.f;
      const int rc = forward ? tc_time_shape<true>(p, t, c, nf, fwd_out, e0, e1, &us)
                             : tc_time_shape<false>(p, t, c, nf, p->d_work, e0, e1, &us);
      if (rc != DINO_OK) return rc;
      if (us < best) {
        best = us;
        pick = c;
      }
    }
    const size_t lw2 = (size_t)p->lw * 2;
    if (forward) {
      t->nsplit_fwd = pick.nsplit;
      t->Nsub_fwd = pick.Nsub;
      t->stages_fwd = pick.stages;
      t->smem_fwd = pick.smem;
      t->us_fwd = best;
      t->tried_fwd = (int)cands.size();
      DINO_TRY(make_map(&t->tBfh, t->Bfh, t->Kj, (long long)lw2 * t->Nf, pick.Nsub));
      DINO_TRY(make_map(&t->tBfl, t->Bfl, t->Kj, (long long)lw2 * t->Nf, pick.Nsub));
    } else {
      t->nsplit_inv = pick.nsplit;
      t->Nsub_inv = pick.Nsub;
      t->stages_inv = pick.stages;
      t->smem_inv = pick.smem;
      t->us_inv = best;
      t->tried_inv = (int)cands.size();
      DINO_TRY(make_map(&t->tBih, t->Bih, t->Kp, (long long)lw2 * t->Np, pick.Nsub));
      DINO_TRY(make_map(&t->tBil, t->Bil, t->Kp, (long long)lw2 * t->Np, pick.Nsub));
    }
    return DINO_OK;
  };
  int rc = tune(false);
  if (rc == DINO_OK) rc = tune(true);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(fwd_out);
  if (rc != DINO_OK) return rc;
  return tc_status(p);
}

std::string tc_describe(dino_plan* p) {
  TcTables* t = p->tc;
  if (!t) return "";
  char buf[512];
  snprintf(buf, sizeof(buf),
           "tcgen05 split-BF16 Legendre autotuned on %d fields: inverse %d N ranges of "
           "%d rows, %d stages (%.1f us, %d shapes tried); forward %d N ranges of %d rows, "
           "%d stages (%.1f us, %d shapes tried)",
           t->tuned_fields, t->nsplit_inv, t->Nsub_inv, t->stages_inv, t->us_inv,
           t->tried_inv, t->nsplit_fwd, t->Nsub_fwd, t->stages_fwd, t->us_fwd, t->tried_fwd);
  return buf;
}

int tc_tables_build(dino_plan* p) {
  DINO_REQUIRE(p->Jh <= 256, DINO_ERR_UNSUPPORTED,
               "tensor-core path supports at most 512 latitudes");
  DINO_REQUIRE((p->L + 1) / 2 <= 256, DINO_ERR_UNSUPPORTED,
               "tensor-core path supports at most 512 total wavenumbers");
  TcTables* t = new TcTables();
  p->tc = t;
  const int half_l = (p->L + 1) / 2;
  t->Kp = round_up(half_l, 64);
  t->Np = round_up(p->Jh, 16);
  t->Kj = round_up(p->Jh, 64);
  t->Nf = round_up(half_l, 16);
  // Fields per launch: A operands at most ~256 MiB each direction.
  const size_t per_field = (size_t)p->lw * 2 * 2 * (t->Kp + t->Kj) * 2 * sizeof(bf16);
  int cap = (int)((512ull << 20) / (per_field ? per_field : 1));
  if (cap > p->max_fields) cap = p->max_fields;
  if (cap < 1) cap = 1;
  t->cap = cap;
  t->Rp = round_up(2 * cap, 128);
  const size_t lw2 = (size_t)p->lw * 2;
  const size_t nBi = lw2 * t->Np * t->Kp, nBf = lw2 * t->Nf * t->Kj;
  const size_t nAi = lw2 * t->Rp * t->Kp, nAf = lw2 * t->Rp * t->Kj;
  DINO_CHECK_CUDA(cudaMalloc(&t->Bih, nBi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Bil, nBi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Bfh, nBf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Bfl, nBf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Aih, nAi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Ail, nAi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Afh, nAf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->Afl, nAf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Bih, 0, nBi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Bil, 0, nBi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Bfh, 0, nBf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Bfl, 0, nBf * sizeof(bf16)));
  // The A slabs are rewritten by every call; zero them once so that rows
  // past a short batch hold finite values.
  DINO_CHECK_CUDA(cudaMemset(t->Aih, 0, nAi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Ail, 0, nAi * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Afh, 0, nAf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMemset(t->Afl, 0, nAf * sizeof(bf16)));
  DINO_CHECK_CUDA(cudaMalloc(&t->d_err, sizeof(int)));
  DINO_CHECK_CUDA(cudaMemset(t->d_err, 0, sizeof(int)));
  dim3 grid(ceil_div(p->Jh, 128), p->lw);
  tc_table_kernel<<<grid, 128>>>(p->lw, p->L, p->Jh, p->d_x64, t->Kp, t->Np, t->Kj, t->Nf,
                                 t->Bih, t->Bil, t->Bfh, t->Bfl);
  DINO_TRY(check_launch("tc_table"));
  const long long rowsA = (long long)lw2 * t->Rp;
  DINO_TRY(make_map(&t->tAih, t->Aih, t->Kp, rowsA, 128));
  DINO_TRY(make_map(&t->tAil, t->Ail, t->Kp, rowsA, 128));
  DINO_TRY(make_map(&t->tAfh, t->Afh, t->Kj, rowsA, 128));
  DINO_TRY(make_map(&t->tAfl, t->Afl, t->Kj, rowsA, 128));
  DINO_CHECK_CUDA(cudaFuncSetAttribute(legendre_tc_kernel<false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kTcSmemLimit));
  DINO_CHECK_CUDA(cudaFuncSetAttribute(legendre_tc_kernel<true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kTcSmemLimit));
  DINO_CHECK_CUDA(cudaDeviceSynchronize());
  return tc_autotune(p, t);
}

void tc_tables_free(dino_plan* p) {
  TcTables* t = p->tc;
  if (!t) return;
  cudaFree(t->Bih);
  cudaFree(t->Bil);
  cudaFree(t->Bfh);
  cudaFree(t->Bfl);
  cudaFree(t->Aih);
  cudaFree(t->Ail);
  cudaFree(t->Afh);
  cudaFree(t->Afl);
  cudaFree(t->d_err);
  delete t;
  p->tc = nullptr;
}

static int tmem_cols_for(int cols) {
  int c = 32;
  while (c < cols) c *= 2;
  return c;
}

// Rows of one operand-slab half (a multiple of the 128-row MMA tile).
static int tc_slot_rows(const TcTables* t) { return (t->Rp / 2) / 128 * 128; }

int tc_slot_fields(dino_plan* p) {
  return p->tc ? tc_slot_rows(p->tc) / 2 : (1 << 30);
}

int tc_legendre_inverse(dino_plan* p, const Segs& in, float* out, int nf,
                        cudaStream_t st, int slot) {
  TcTables* t = p->tc;
  DINO_REQUIRE(t, DINO_ERR_ARG, "plan has no tensor-core tables");
  const size_t ms = (size_t)p->M * p->L, fs = (size_t)p->M * p->J;
  const int cap = slot < 0 ? t->cap : tc_slot_rows(t) / 2;
  const int roff = slot > 0 ? tc_slot_rows(t) : 0;
  DINO_REQUIRE(cap >= 1, DINO_ERR_UNSUPPORTED, "operand slab too small for two slots");
  for (int f0 = 0; f0 < nf; f0 += cap) {
    const int n = nf - f0 < cap ? nf - f0 : cap;
    Segs sub = seg_offset(in, f0, n, ms);
    const int max_rows = 2 * n;
    dim3 g1((unsigned)(((size_t)max_rows * (t->Kp / 8) + 255) / 256), p->lw);
    tc_split_inverse_kernel<<<g1, 256, 0, st>>>(sub, n, p->M, p->L, t->Rp, t->Kp, roff,
                                                t->Aih, t->Ail);
    DINO_TRY(check_launch("tc_split_inverse"));
    TcArgs a{};
    a.nf = n;
    a.M = p->M;
    a.L = p->L;
    a.J = p->J;
    a.Jh = p->Jh;
    a.Rp = t->Rp;
    a.roff = roff;
    a.Nrows = t->Np;
    a.Nsub = t->Nsub_inv;
    a.stages = t->stages_inv;
    a.tmem_cols = tmem_cols_for(2 * t->Nsub_inv);
    a.out = out + f0 * fs;
    a.err = t->d_err;
    dim3 g2(ceil_div(max_rows, 128), p->lw, t->nsplit_inv);
    legendre_tc_kernel<false><<<g2, kTcThreads, t->smem_inv, st>>>(t->tAih, t->tAil, t->tBih,
                                                                   t->tBil, a);
    DINO_TRY(check_launch("legendre_tc_inverse"));
  }
  return DINO_OK;
}

int tc_legendre_forward(dino_plan* p, const float* G, float* out, int nf,
                        cudaStream_t st, int slot) {
  TcTables* t = p->tc;
  DINO_REQUIRE(t, DINO_ERR_ARG, "plan has no tensor-core tables");
  const size_t ms = (size_t)p->M * p->L, fs = (size_t)p->M * p->J;
  const int cap = slot < 0 ? t->cap : tc_slot_rows(t) / 2;
  const int roff = slot > 0 ? tc_slot_rows(t) : 0;
  DINO_REQUIRE(cap >= 1, DINO_ERR_UNSUPPORTED, "operand slab too small for two slots");
  for (int f0 = 0; f0 < nf; f0 += cap) {
    const int n = nf - f0 < cap ? nf - f0 : cap;
    const int max_rows = 2 * n;
    dim3 g1((unsigned)(((size_t)max_rows * (t->Kj / 8) + 255) / 256), p->lw);
    tc_fold_forward_kernel<<<g1, 256, 0, st>>>(G + f0 * fs, n, p->M, p->J, p->Jh, t->Rp, t->Kj,
                                               roff, t->Afh, t->Afl);
    DINO_TRY(check_launch("tc_fold_forward"));
    TcArgs a{};
    a.nf = n;
    a.M = p->M;
    a.L = p->L;
    a.J = p->J;
    a.Jh = p->Jh;
    a.Rp = t->Rp;
    a.roff = roff;
    a.Nrows = t->Nf;
    a.Nsub = t->Nsub_fwd;
    a.stages = t->stages_fwd;
    a.tmem_cols = tmem_cols_for(2 * t->Nsub_fwd);
    a.out = out + f0 * ms;
    a.err = t->d_err;
    dim3 g2(ceil_div(max_rows, 128), p->lw, t->nsplit_fwd);
    legendre_tc_kernel<true><<<g2, kTcThreads, t->smem_fwd, st>>>(t->tAfh, t->tAfl, t->tBfh,
                                                                  t->tBfl, a);
    DINO_TRY(check_launch("legendre_tc_forward"));
  }
  return DINO_OK;
}

int tc_status(dino_plan* p) {
  if (!p->tc) return DINO_OK;
  int err = 0;
  DINO_CHECK_CUDA(cudaMemcpy(&err, p->tc->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    set_error("a tensor-core wait gave up (code " + std::to_string(err) + ")");
    return DINO_ERR_TIMEOUT;
  }
  return DINO_OK;
}

}  // namespace dino

extern "C" int dino_plan_describe(dino_plan* p, char* buf, size_t len) {
  DINO_REQUIRE(p && buf && len > 0, DINO_ERR_ARG, "dino_plan_describe: null argument");
  char head[256];
  snprintf(head, sizeof(head),
           "grid %d x %d nodes, %d x %d modal, Legendre %s, batch capacity %d fields",
           p->I, p->J, p->M, p->L,
           p->precision == DINO_PREC_BF16X3 ? "split-BF16 (tcgen05)" : "FP32 (SIMT)",
           p->max_fields);
  std::string s = head;
  const std::string tc = dino::tc_describe(p);
  if (!tc.empty()) s += "; " + tc;
  snprintf(buf, len, "%s", s.c_str());
  return DINO_OK;
}

extern "C" int dino_plan_status(dino_plan* p) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_plan_status: null argument");
  DINO_CHECK_CUDA(cudaDeviceSynchronize());
  return dino::tc_status(p);
}
