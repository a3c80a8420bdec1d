// Legendre contraction on tcgen05 tensor cores, split-BF16 (DINO_PREC_BF16X3)
// or split-TF32 (DINO_PREC_TF32X3) with FP32 accumulation.
//
// Every FP32 operand x is split into x_hi = round(x) and x_lo = round(x - x_hi)
// in the operand format (bf16: 8 significant bits, tf32: 11); each product is
// formed as hi*hi + hi*lo + lo*hi (the lo*lo term, ~2^-16 relative for bf16
// and ~2^-22 for tf32, is dropped) and accumulated in FP32 in tensor memory.
// The Legendre tables are split from their FP64 values.  A tile row holds
// one K block of 32 entries, swizzled over its width (64 bytes of bf16, 128
// bytes of tf32), and one MMA instruction consumes 32 bytes of K (16 or 8
// entries).
//
// Per zonal wavenumber m the contraction is a GEMM
//   inverse:  D[r, j]  = sum_{l'} X_p[r, l'] P_p[j, l']   (K = l', N = j)
//   forward:  D[r, l'] = sum_j  G_p[r, j]  P_p[l', j]     (K = j,  N = l')
// with r = (field, cos/sin) rows, p the parity of l - m (the N/S fold),
// l = m + 2 l' + p, and G_0 / G_1 the symmetric / antisymmetric latitude
// folds.  The tables P_p are K-major split operands in HBM, loaded by TMA (no
// multicast) into swizzled shared memory tiles; the A operand is
// produced in the same layout by six warps of the CTA straight from the FP32
// modal coefficients (inverse) or Fourier coefficients (forward): one read of
// the source gives both parities, folded and split.  One thread issues
// tcgen05.mma (M = 128, N = latitudes or l', 32 bytes of K per instruction) into two
// TMEM accumulators (one per parity); all eight warps read them back with
// tcgen05.ld and write the unfolded FP32 result.  Only the K steps and N
// columns that the triangular (m, l) range needs are issued.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dino_internal.cuh"

namespace dino {

typedef __nv_bfloat16 bf16;

struct TcTables {
  int tf32 = 0; // operand format: 0 bf16 (2-byte entries), 1 tf32 (4-byte)
  int Kp = 0;   // inverse K extent (l'), multiple of the K block
  int Np = 0;   // inverse N (latitudes), multiple of 16
  int Kj = 0;   // forward K extent (latitudes), multiple of the K block
  int Nf = 0;   // forward N (l'), multiple of 16
  void *Bih = nullptr, *Bil = nullptr, *Bfh = nullptr, *Bfl = nullptr;
  int* d_err = nullptr;
  // Launch shape of each m group of each direction, chosen by the
  // autotuner: N sub-ranges per (m, row tile) CTA and their width (B tile
  // rows), pipeline depth, and the B tensor maps for that width.
  struct Shape {
    int m0 = 0, m1 = 0;
    int nsplit = 1, Nsub = 0, stages = 0;
    size_t smem = 0;
    float us = 0.f;
    int tried = 0;
    CUtensorMap bh, bl;
  };
  static constexpr int kMaxGroups = 2;
  Shape inv[kMaxGroups], fwd[kMaxGroups];
  int ngroups_inv = 1, ngroups_fwd = 1;
  // Autotuning record: the chunk size and each direction's total time.
  int tuned_fields = 0;
  float us_inv = 0.f, us_fwd = 0.f;
  // Total time of the two-group arrangement (0 when not tried).
  float us_inv_split = 0.f, us_fwd_split = 0.f;
  // The FP32 SIMT contraction, timed beside the tensor-core shapes; a
  // direction whose SIMT launch is faster at the tuned size runs SIMT (more
  // accurate than either split form, so the precision contract holds).
  float us_simt_inv = 0.f, us_simt_fwd = 0.f;
  int simt_inv = 0, simt_fwd = 0;
};

__host__ __device__ __forceinline__ int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Operand formats.  kKB: K entries per swizzled tile row (one K block per
// pipeline stage); kStep: K entries per MMA instruction (32 bytes); kChunk: K
// entries per 16-byte chunk of a row; kFmt: the instruction descriptor's A / B
// format code; kUnroll: producer tasks loaded before any is converted;
// kSepAcc: the hi*lo + lo*hi corrections accumulate in TMEM accumulators of
// their own, added to the hi*hi sums in FP32 by the epilogue.
//
// Each MMA instruction adds its products into the FP32 accumulator with a
// rounding of its own, about one unit in the last place of the accumulator.
// With exact accumulation the tf32 split would be ~1e-7 accurate (2^-22 per
// term), so there these roundings dominate: the separate accumulators leave
// one per K step on the large sums instead of three.  The bf16 split (~4e-6,
// its dropped lo*lo term) dominates the roundings, so one accumulator serves.
//
// kRowBytes: bytes of one tile row (one K block), swizzled over its own
// width (64 or 128 bytes); kLayout: the UMMA descriptor's code for that
// swizzle.  Split-BF16 K blocks are 32 entries (64-byte rows), which halves a
// pipeline stage against 128-byte rows, so that two CTAs share an SM at the
// widest N range that fits TMEM twice (128 columns per accumulator).
struct OpBf16 {
  typedef bf16 T;
  static constexpr int kKB = 32, kStep = 16, kChunk = 8, kUnroll = 3;
  static constexpr int kRowBytes = 64;
  static constexpr uint64_t kLayout = 4;  // SWIZZLE_64B
  static constexpr uint32_t kFmt = 1;  // BF16
  static constexpr bool kSepAcc = false;
};
struct OpTf32 {
  typedef float T;  // tf32 in an FP32 container (low 13 mantissa bits zero)
  static constexpr int kKB = 32, kStep = 8, kChunk = 4, kUnroll = 6;
  static constexpr int kRowBytes = 128;
  static constexpr uint64_t kLayout = 2;  // SWIZZLE_128B
  static constexpr uint32_t kFmt = 2;  // TF32
  static constexpr bool kSepAcc = true;
};

// Row bytes of a plan's operand format (host side).
constexpr int tc_row_bytes(int tf32) { return tf32 ? OpTf32::kRowBytes : OpBf16::kRowBytes; }

// TMEM accumulators (each Nsub columns) per CTA: one per parity, twice that
// with separate correction accumulators.
__host__ __device__ constexpr int tc_accumulators(bool sep) { return sep ? 4 : 2; }

// ---------------------------------------------------------------------------
// Operand preparation
// ---------------------------------------------------------------------------

// x rounded to tf32 (10 stored mantissa bits), to nearest, ties away from zero.
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void split_table(double v, bf16& hi, bf16& lo) {
  hi = __double2bfloat16(v);
  lo = __double2bfloat16(v - (double)__bfloat162float(hi));
}

__device__ __forceinline__ void split_table(double v, float& hi, float& lo) {
  hi = tf32_rna((float)v);
  lo = tf32_rna((float)(v - (double)hi));
}

// FP64 recurrence (as in plan.cu) written as split operands into the inverse
// table [m][p][j][Kp] and the forward table [m][p][l'][Kj].
template <class T>
__global__ void tc_table_kernel(int lw, int L, int Jh, const double* __restrict__ x,
                                int Kp, int Np, int Kj, int Nf,
                                T* __restrict__ Bih, T* __restrict__ Bil,
                                T* __restrict__ Bfh, T* __restrict__ Bfl) {
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
    T hi, lo;
    split_table(cur, hi, lo);
    int p = k & 1, kk = k >> 1;
    size_t ii = ((size_t)(m * 2 + p) * Np + j) * Kp + kk;
    size_t fi = ((size_t)(m * 2 + p) * Nf + kk) * Kj + j;
    Bih[ii] = hi;
    Bil[ii] = lo;
    Bfh[fi] = hi;
    Bfl[fi] = lo;
  }
}

// ---------------------------------------------------------------------------
// tcgen05 / TMA / mbarrier primitives (inline PTX)
// ---------------------------------------------------------------------------

constexpr int kTcThreads = 256;
constexpr int kTcProducers = 192;  // warps 2-7
constexpr int kMaxStages = 6;
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// True once the phase with the given parity has completed; the hardware may
// suspend the thread for a while before answering false (try_wait), so a
// waiting warp does not spin on the issue slots.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity; gives up after limit_ns
// (kWaitLimitNs in the contraction kernels), records `code` in *err and
// returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          int* err, int code,
                                          unsigned long long limit_ns = kWaitLimitNs) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_test(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) {
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

// TMA tensor store of a shared-memory box (bulk async-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* tm, const void* src, int x,
                                             int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<uint64_t>(tm)),
      "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
      : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Waits until at most N of this thread's committed bulk groups still read
// their shared-memory source.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Waits until this thread's bulk groups have completed.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, rows of Op::kRowBytes swizzled
// over their width, 8-row groups 8 * kRowBytes apart (SBO), leading offset
// unused for swizzled K-major.
template <class Op>
__device__ __forceinline__ uint64_t umma_desc(const void* p) {
  uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= 1ull << 16;
  d |= (uint64_t)((8 * Op::kRowBytes) >> 4) << 32;
  d |= 1ull << 46;
  d |= Op::kLayout << 61;
  return d;
}

// Instruction descriptor: D = F32 (bits 4-5), A and B in the operand format
// (bits 7-9, 10-12), both K-major, N = n (bits 17-22, n / 8), M = 128 (bits
// 24-28, M / 16).
template <class Op>
__device__ __forceinline__ uint32_t umma_idesc(int n) {
  return (1u << 4) | (Op::kFmt << 7) | (Op::kFmt << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

// D (+)= A B^T for one 32-byte K step: kind::f16 for bf16, kind::tf32.
template <class Op>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b,
                                     uint32_t idesc, uint32_t accumulate) {
  if constexpr (Op::kFmt == OpBf16::kFmt) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
  }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// Issues a 16-column TMEM load (32 lanes x 32 bits); the values are valid
// after tmem_wait16 / tmem_tie16 on the same registers.
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
        "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// Waits for this thread's TMEM loads; the register operands order every
// later use of r after the wait.
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// Orders the uses of a second load's registers after a preceding tmem_wait16
// (volatile asm statements keep their order).
__device__ __forceinline__ void tmem_tie16(uint32_t (&r)[16]) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]));
}

// Both parities' 16 columns at c0 (parity 1 only when `odd`), one wait.
__device__ __forceinline__ void tmem_ld_pair(uint32_t c0, uint32_t c1, bool odd,
                                             float (&e)[16], float (&o)[16]) {
  uint32_t re[16], ro[16];
  tmem_ld16_issue(c0, re);
  if (odd) tmem_ld16_issue(c1, ro);
  tmem_wait16(re);
  if (odd) tmem_tie16(ro);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    e[i] = __uint_as_float(re[i]);
    o[i] = odd ? __uint_as_float(ro[i]) : 0.f;
  }
}

// Chunk c (16 columns) of both parities' results: accumulator p at column
// p * ncol, and with separate corrections their sums with accumulator 2 + p.
template <class Op>
__device__ __forceinline__ void tc_ld_acc(uint32_t base, int ncol, int c, bool odd,
                                          float (&e)[16], float (&o)[16]) {
  const uint32_t c0 = base + (uint32_t)(c * 16);
  if constexpr (Op::kSepAcc) {
    uint32_t r0[16], r1[16], r2[16], r3[16];
    tmem_ld16_issue(c0, r0);
    tmem_ld16_issue(c0 + 2 * ncol, r2);
    if (odd) {
      tmem_ld16_issue(c0 + ncol, r1);
      tmem_ld16_issue(c0 + 3 * ncol, r3);
    }
    tmem_wait16(r0);
    tmem_tie16(r2);
    if (odd) {
      tmem_tie16(r1);
      tmem_tie16(r3);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      e[i] = __uint_as_float(r0[i]) + __uint_as_float(r2[i]);
      o[i] = odd ? __uint_as_float(r1[i]) + __uint_as_float(r3[i]) : 0.f;
    }
  } else {
    tmem_ld_pair(c0, c0 + ncol, odd, e, o);
  }
}


// v[q] for a q known only at run time, by selects (no local-memory copy).
__device__ __forceinline__ float4 pick4(const float4 (&v)[4], int q) {
  const float4 a = (q & 1) ? v[1] : v[0];
  const float4 b = (q & 1) ? v[3] : v[2];
  return (q & 2) ? b : a;
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

// Forward epilogue: stores one staged chunk (32 interleaved l = lbase + lane
// of the rows row0 .. row0 + 31, stage[r][stride]) of the modal output.  Rows are
// (field, cos / sin of m) pairs for m > 0 (row0 even), fields for m = 0, so
// each row's address follows from the previous one by a fixed step.
__device__ __forceinline__ void fwd_store_chunk(float* out, int M, int L, int m, int rows,
                                                int row0, const float* stage, int stride,
                                                int lbase, bool keep, int lane) {
  const int l = lbase + lane;
  if (!keep || l >= L) return;
  const size_t ML = (size_t)M * L;
  const int rmax = min(32, rows - row0);
  if (m == 0) {
    float* o = out + (size_t)row0 * ML + l;
#pragma unroll 4
    for (int r = 0; r < rmax; ++r, o += ML) *o = stage[r * stride + lane];
  } else {
    float* o = out + (size_t)(row0 >> 1) * ML + (size_t)(2 * m - 1) * L + l;
#pragma unroll 4
    for (int r = 0; r < rmax; r += 2, o += ML) {
      o[0] = stage[r * stride + lane];
      if (r + 1 < rmax) o[L] = stage[(r + 1) * stride + lane];
    }
  }
}

// Byte offset of 16-byte chunk c of row r in a K-major tile of
// Op::kRowBytes rows swizzled over their width: the layout that TMA writes
// for CU_TENSOR_MAP_SWIZZLE_128B / _64B and the UMMA descriptor (umma_desc)
// reads.  128-byte rows: chunk c ^ (r mod 8); 64-byte rows: c ^ (r / 2 mod 4)
// (the address bits 4-6 or 4-5 XOR bits 7-9 or 7-8).
template <class Op>
__device__ __forceinline__ uint32_t sw_off(int r, int c) {
  if constexpr (Op::kRowBytes == 128)
    return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
  else
    return (uint32_t)(r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
}

// hi = bf16x2(x0, x1) and lo = bf16x2 of the remainders x - hi, each rounded
// to nearest: one packed conversion per pair for each half.
__device__ __forceinline__ void split_pair(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = reinterpret_cast<const uint32_t&>(h);
  lo = reinterpret_cast<const uint32_t&>(l);
}

// Splits Op::kChunk values v[s0], v[s0 + st], ... (8 for bf16, 4 for tf32)
// into hi / lo and writes them as one 16-byte chunk of each tile (shared
// memory).
template <class Op, int N>
__device__ __forceinline__ void put_split(const float (&v)[N], int s0, int st,
                                          uint8_t* hi, uint8_t* lo, uint32_t off) {
  uint32_t h[4], l[4];
  if constexpr (Op::kFmt == OpBf16::kFmt) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      split_pair(v[s0 + (2 * i) * st], v[s0 + (2 * i + 1) * st], h[i], l[i]);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float x = v[s0 + i * st];
      const float xh = tf32_rna(x);
      h[i] = __float_as_uint(xh);
      l[i] = __float_as_uint(tf32_rna(x - xh));
    }
  }
  *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// ---------------------------------------------------------------------------
// The contraction kernel
// ---------------------------------------------------------------------------

struct TcArgs {
  int nf, M, L, J, Jh;
  int Nrows;     // rows of one (m, parity) B table (Np or Nf)
  int Nsub;      // B tile rows = N columns of this CTA (blockIdx.z-th range)
  int stages;
  int tmem_cols; // allocated TMEM columns (power of two)
  int vec;       // inverse: rows of the modal input start 16-byte aligned
  int tma_out;   // inverse: full 16-latitude blocks leave by TMA tensor stores
  Segs in;       // inverse: modal coefficients [nf][M][L]
  const float* G;  // forward: weighted Fourier coefficients [nf][M][J]
  float* out;    // inverse: Fourier [nf][M][J]; forward: modal [nf][M][L]
  int* err;
  int m0;        // first zonal wavenumber of the launch (blockIdx.y = m - m0)
};

// Pipeline order of the (K block, parity) stages: block k's parity 0, then
// its parity 1 while k < kb1 (kb1 = K blocks of parity 1 <= those of parity 0).
__device__ __forceinline__ void tc_seq(int i, int kb1, int& k, int& p) {
  if (i < 2 * kb1) {
    k = i >> 1;
    p = i & 1;
  } else {
    k = i - kb1;
    p = 0;
  }
}

// A operand of K block k for this CTA's 128 rows, both parities from one
// read of the FP32 source, written split into the stage tiles t0 (parity 0)
// and t1 (parity 1, null when absent): hi at t, lo at t + 16 KB.  With
// B = Op::kKB (K entries per block) and C = Op::kChunk (per 16-byte chunk):
//   inverse: A_p[r][kk] = x[b][row][m + 2 (B k + kk) + p]  (0 past l = L - 1)
//   forward: A_p[r][jj] = G[j] + (-1)^p G[J - 1 - j], j = B k + jj  (0 past Jh)
// A task is one (row, 16-byte chunk); each thread loads Op::kUnroll tasks
// before converting any, so that enough bytes are in flight to cover the
// latency.
template <class Op>
constexpr int kTcTasks = 128 * (Op::kRowBytes / 16);
// Tasks per producer thread in flight in the inverse: all of a split-BF16 K
// block's (512 / 192 -> 3), so each K block costs one round trip to memory.
template <class Op>
constexpr int kInvUnroll = Op::kUnroll;

// Inverse: a task covers the 2C consecutive l = m + l0 .. m + l0 + 2C - 1
// (both parities).  S = m mod 4 places them at entries S .. S + 2C - 1 of a
// window of W = 2C + 4 floats that starts 16-byte aligned (W / 4 float4).
template <class Op, int S>
__device__ __forceinline__ void tc_produce_inverse(const TcArgs& a, int m, int tile, int rows,
                                                   int k, uint8_t* t0, uint8_t* t1, int pt) {
  constexpr uint32_t kTile = 128u * Op::kRowBytes;
  constexpr int C = Op::kChunk, W = 2 * C + 4, U = kInvUnroll<Op>;
  for (int q0 = pt; q0 < kTcTasks<Op>; q0 += U * kTcProducers) {
    float w[U][W];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kTcProducers;
#pragma unroll
      for (int e = 0; e < W; ++e) w[u][e] = 0.f;
      if (q >= kTcTasks<Op>) continue;
      constexpr int CH = Op::kRowBytes / 16;  // chunks per tile row
      const int r = q / CH, c = q % CH;
      const int rr = tile * 128 + r;
      if (rr >= rows) continue;
      int b, row;
      tc_row_map(m, rr, b, row);
      const int l0 = 2 * Op::kKB * k + 2 * C * c;  // relative to l = m
      const int lim = (a.L - m) - l0;             // valid entries from l0
      const float* src = seg_field(a.in, b, (size_t)a.M * a.L) + (size_t)row * a.L + m + l0;
      if (a.vec && lim >= W) {
        const float4* w4 = reinterpret_cast<const float4*>(src - S);
#pragma unroll
        for (int i = 0; i < W / 4; ++i) {
          const float4 t = __ldg(w4 + i);
          w[u][4 * i] = t.x;
          w[u][4 * i + 1] = t.y;
          w[u][4 * i + 2] = t.z;
          w[u][4 * i + 3] = t.w;
        }
      } else {
#pragma unroll
        for (int e = 0; e < 2 * C; ++e) w[u][e + S] = (e < lim) ? __ldg(src + e) : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kTcProducers;
      if (q >= kTcTasks<Op>) continue;
      const uint32_t off = sw_off<Op>(q / (Op::kRowBytes / 16), q % (Op::kRowBytes / 16));
      // Entries S .. S+2C-1: even l - m are parity 0, odd ones parity 1.
      put_split<Op>(w[u], S, 2, t0, t0 + kTile, off);
      if (t1) put_split<Op>(w[u], S + 1, 2, t1, t1 + kTile, off);
    }
  }
}

// Inverse, rows at any alignment (L not a multiple of 4, or a segment that
// starts off a 16-byte boundary): the same tasks, each read as W / 4 float4 of
// the 16-byte-aligned window that holds its 2C entries, R = the entries'
// misalignment (0..3, per task), and shifted into place with two rounds of
// selects; a task whose window would cross the end of its row reads its
// entries one by one.  The window ends inside the row, and it starts on the
// 16-byte boundary at or before the task's first entry: inside the caller's
// allocation, which starts on a 256-byte boundary (device allocations do).
template <class Op>
__device__ __forceinline__ void tc_produce_inverse_any(const TcArgs& a, int m, int tile,
                                                       int rows, int k, uint8_t* t0,
                                                       uint8_t* t1, int pt) {
  constexpr uint32_t kTile = 128u * Op::kRowBytes;
  constexpr int C = Op::kChunk, W = 2 * C + 4, U = kInvUnroll<Op>;
  for (int q0 = pt; q0 < kTcTasks<Op>; q0 += U * kTcProducers) {
    float w[U][W];
    int sh[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kTcProducers;
#pragma unroll
      for (int e = 0; e < W; ++e) w[u][e] = 0.f;
      sh[u] = 0;
      if (q >= kTcTasks<Op>) continue;
      constexpr int CH = Op::kRowBytes / 16;  // chunks per tile row
      const int r = q / CH, c = q % CH;
      const int rr = tile * 128 + r;
      if (rr >= rows) continue;
      int b, row;
      tc_row_map(m, rr, b, row);
      const int l0 = 2 * Op::kKB * k + 2 * C * c;  // relative to l = m
      const int lim = (a.L - m) - l0;             // valid entries from l0
      const float* src = seg_field(a.in, b, (size_t)a.M * a.L) + (size_t)row * a.L + m + l0;
      const int R = (int)((reinterpret_cast<uintptr_t>(src) >> 2) & 3);
      if (lim >= W - R) {
        const float4* w4 = reinterpret_cast<const float4*>(src - R);
#pragma unroll
        for (int i = 0; i < W / 4; ++i) {
          const float4 t = __ldg(w4 + i);
          w[u][4 * i] = t.x;
          w[u][4 * i + 1] = t.y;
          w[u][4 * i + 2] = t.z;
          w[u][4 * i + 3] = t.w;
        }
        sh[u] = R;
      } else {
#pragma unroll
        for (int e = 0; e < 2 * C; ++e) w[u][e] = (e < lim) ? __ldg(src + e) : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kTcProducers;
      if (q >= kTcTasks<Op>) continue;
      // o[e] = w[sh + e]: shift by 1, then by 2.
      float y[2 * C + 2], o[2 * C];
#pragma unroll
      for (int i = 0; i < 2 * C + 2; ++i) y[i] = (sh[u] & 1) ? w[u][i + 1] : w[u][i];
#pragma unroll
      for (int e = 0; e < 2 * C; ++e) o[e] = (sh[u] & 2) ? y[e + 2] : y[e];
      const uint32_t off = sw_off<Op>(q / (Op::kRowBytes / 16), q % (Op::kRowBytes / 16));
      put_split<Op>(o, 0, 2, t0, t0 + kTile, off);
      if (t1) put_split<Op>(o, 1, 2, t1, t1 + kTile, off);
    }
  }
}

// Forward: a task covers the C latitudes j0 .. j0 + C - 1 and their mirrors.
template <class Op>
__device__ __forceinline__ void tc_produce_forward(const TcArgs& a, int m, int tile, int rows,
                                                   int k, uint8_t* t0, uint8_t* t1, int pt) {
  constexpr uint32_t kTile = 128u * Op::kRowBytes;
  constexpr int C = Op::kChunk, U = Op::kUnroll;
  const bool vec = (a.J & 3) == 0;
  for (int q0 = pt; q0 < kTcTasks<Op>; q0 += U * kTcProducers) {
    float d[U][C], e[U][C];  // G[j0 + t], G[J - 1 - j0 - t]
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kTcProducers;
#pragma unroll
      for (int t = 0; t < C; ++t) d[u][t] = e[u][t] = 0.f;
      if (q >= kTcTasks<Op>) continue;
      constexpr int CH = Op::kRowBytes / 16;  // chunks per tile row
      const int r = q / CH, c = q % CH;
      const int rr = tile * 128 + r;
      if (rr >= rows) continue;
      int b, row;
      tc_row_map(m, rr, b, row);
      const float* gr = a.G + ((size_t)b * a.M + row) * a.J;
      const int j0 = Op::kKB * k + C * c;
      if (vec && j0 + C <= a.Jh) {
        // j0 + 4i .. j0 + 4i + 3 and J - 4(i+1) - j0 .. J - 1 - 4i - j0 are
        // float4 (J and j0 are multiples of 4).
#pragma unroll
        for (int i = 0; i < C / 4; ++i) {
          const float4 f = __ldg(reinterpret_cast<const float4*>(gr + j0 + 4 * i));
          const float4 g = __ldg(reinterpret_cast<const float4*>(gr + a.J - 4 * (i + 1) - j0));
          d[u][4 * i] = f.x; d[u][4 * i + 1] = f.y; d[u][4 * i + 2] = f.z; d[u][4 * i + 3] = f.w;
          e[u][4 * i] = g.w; e[u][4 * i + 1] = g.z; e[u][4 * i + 2] = g.y; e[u][4 * i + 3] = g.x;
        }
      } else {
#pragma unroll
        for (int t = 0; t < C; ++t) {
          const int j = j0 + t;
          if (j < a.Jh) {
            const int jm = a.J - 1 - j;
            d[u][t] = __ldg(gr + j);
            e[u][t] = (jm != j) ? __ldg(gr + jm) : 0.f;
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kTcProducers;
      if (q >= kTcTasks<Op>) continue;
      const uint32_t off = sw_off<Op>(q / (Op::kRowBytes / 16), q % (Op::kRowBytes / 16));
      float sv[C], dv[C];
#pragma unroll
      for (int t = 0; t < C; ++t) {
        sv[t] = d[u][t] + e[u][t];
        dv[t] = d[u][t] - e[u][t];
      }
      put_split<Op>(sv, 0, 1, t0, t0 + kTile, off);
      if (t1) put_split<Op>(dv, 0, 1, t1, t1 + kTile, off);
    }
  }
}

// L2 prefetches of the rows of K block k: block 0's before the CTA's set-up
// barrier (barrier init, TMEM allocation), so that the set-up overlaps their
// latency, and block k + 1's as the producers start block k, so that its
// memory latency overlaps block k's conversion and stage waits.  Every
// address lies inside its row.
__device__ __forceinline__ void prefetch_l2(const float* p) {
  asm volatile("prefetch.L2 [%0];" ::"l"(p));
}

template <bool kForward, class Op>
__device__ __forceinline__ void tc_prefetch_block(const TcArgs& a, int m, int tile, int rows,
                                                  int k, int pt) {
  constexpr int kPts = kForward ? 4 : 3;  // addresses per row
  for (int q = pt; q < 128 * kPts; q += kTcProducers) {
    const int r = q / kPts, e = q - r * kPts;
    const int rr = tile * 128 + r;
    if (rr >= rows) continue;
    int b, row;
    tc_row_map(m, rr, b, row);
    if (kForward) {
      const float* gr = a.G + ((size_t)b * a.M + row) * a.J;
      const int j0 = Op::kKB * k;
      const int w = min(Op::kKB, a.Jh - j0);  // >= 1 for k < kblk
      const int j = e == 0 ? j0 : e == 1 ? j0 + w - 1 : e == 2 ? a.J - j0 - w : a.J - 1 - j0;
      prefetch_l2(gr + j);
    } else {
      const int l0 = 2 * Op::kKB * k;  // relative to l = m
      const float* src = seg_field(a.in, b, (size_t)a.M * a.L) + (size_t)row * a.L + m + l0;
      const int last = min(2 * Op::kKB, a.L - m - l0) - 1;  // >= 0 for k < kblk
      const int off = e == 0 ? 0 : e == 1 ? min(32, last) : last;
      prefetch_l2(src + off);
    }
  }
}

template <bool kForward, class Op>
__device__ __forceinline__ void tc_produce(const TcArgs& a, int m, int tile, int rows, int k,
                                           uint8_t* t0, uint8_t* t1, int pt) {
  if (kForward) {
    tc_produce_forward<Op>(a, m, tile, rows, k, t0, t1, pt);
  } else if (!a.vec) {
    tc_produce_inverse_any<Op>(a, m, tile, rows, k, t0, t1, pt);
  } else {
    switch (m & 3) {
      case 0: tc_produce_inverse<Op, 0>(a, m, tile, rows, k, t0, t1, pt); break;
      case 1: tc_produce_inverse<Op, 1>(a, m, tile, rows, k, t0, t1, pt); break;
      case 2: tc_produce_inverse<Op, 2>(a, m, tile, rows, k, t0, t1, pt); break;
      default: tc_produce_inverse<Op, 3>(a, m, tile, rows, k, t0, t1, pt); break;
    }
  }
}

// Warp roles: warp 0 lane 0 loads the B tables by TMA, warp 1 allocates TMEM
// and its lane 0 issues the MMAs, warps 2-7 produce the A tiles; all eight
// warps drain TMEM in the epilogue (warp w reads lane quarter w mod 4 and
// every other 16-column chunk).
template <bool kForward, class Op>
__global__ void __launch_bounds__(kTcThreads, 2)
legendre_tc_kernel(const __grid_constant__ CUtensorMap tBh,
                   const __grid_constant__ CUtensorMap tBl,
                   const __grid_constant__ CUtensorMap tO2,
                   const __grid_constant__ CUtensorMap tO1, const __grid_constant__ TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kMaxStages];
  __shared__ __align__(8) uint64_t empty_bar[kMaxStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_slot;

  const int m = a.m0 + blockIdx.y;
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
      kblk[p] = (n_par[p] + Op::kKB - 1) / Op::kKB;
      ksteps[p] = (n_par[p] + Op::kStep - 1) / Op::kStep;
      ncols[p] = a.Nsub;
      cnt[p] = n_par[p];
    } else {
      cnt[p] = max(0, min(n_par[p] - lo, a.Nsub));
      kblk[p] = cnt[p] ? (a.Jh + Op::kKB - 1) / Op::kKB : 0;
      ksteps[p] = (a.Jh + Op::kStep - 1) / Op::kStep;
      ncols[p] = round_up(cnt[p] > 0 ? cnt[p] : 16, 16);
    }
  }
  // Uniform early exits: no output column in this range.
  if (kForward && cnt[0] == 0) return;
  if (!kForward && lo >= a.Jh) return;
  const int nblocks = kblk[0] + kblk[1];
  const uint32_t tile_a = 128u * Op::kRowBytes;             // 128 rows x one K block
  const uint32_t tile_b = (uint32_t)a.Nsub * Op::kRowBytes;  // Nsub rows x one K block
  const uint32_t stage_bytes = 2 * tile_a + 2 * tile_b;
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t* base = smem_raw + pad;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < a.stages; ++s) {
      // One arrive with the B bytes (TMA) and one per producer thread.
      mbar_init(&full_bar[s], 1 + kTcProducers);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // The first stages' table tiles, before the set-up barrier (this thread
    // initialised the barriers; every stage is free).
    for (int i = 0; i < min(a.stages, nblocks); ++i) {
      int k, p;
      tc_seq(i, kblk[1], k, p);
      uint8_t* st = base + (size_t)i * stage_bytes;
      mbar_expect_tx(&full_bar[i], 2 * tile_b);
      const int yb = (m * 2 + p) * a.Nrows + lo;
      tma_load_2d(st + 2 * tile_a, &tBh, &full_bar[i], k * Op::kKB, yb);
      tma_load_2d(st + 2 * tile_a + tile_b, &tBl, &full_bar[i], k * Op::kKB, yb);
    }
  } else if (warp >= 2) {
    tc_prefetch_block<kForward, Op>(a, m, tile, rows, 0, threadIdx.x - 64);
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
  // Parity p accumulates at column p * Nsub (its corrections, when separate,
  // at (2 + p) * Nsub).
  const int acc_cols = a.Nsub;

  if (threadIdx.x == 0) {
    // B producer (TMA); the first min(stages, nblocks) were issued above.
    for (int i = min(a.stages, nblocks); i < nblocks; ++i) {
      const int s = i % a.stages;
      const int use = i / a.stages;
      if (use > 0 && !mbar_wait(&empty_bar[s], (use - 1) & 1, a.err, 1)) break;
      int k, p;
      tc_seq(i, kblk[1], k, p);
      uint8_t* st = base + (size_t)s * stage_bytes;
      mbar_expect_tx(&full_bar[s], 2 * tile_b);
      const int yb = (m * 2 + p) * a.Nrows + lo;
      tma_load_2d(st + 2 * tile_a, &tBh, &full_bar[s], k * Op::kKB, yb);
      tma_load_2d(st + 2 * tile_a + tile_b, &tBl, &full_bar[s], k * Op::kKB, yb);
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer: hi*hi + hi*lo + lo*hi per 32-byte K step.
    for (int i = 0; i < nblocks; ++i) {
      const int s = i % a.stages;
      const int use = i / a.stages;
      if (!mbar_wait(&full_bar[s], use & 1, a.err, 2)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int k, p;
      tc_seq(i, kblk[1], k, p);
      constexpr int kSPB = Op::kKB / Op::kStep;  // MMA K steps per K block
      const int steps = min(kSPB, (p ? ksteps[1] : ksteps[0]) - k * kSPB);
      const uint32_t d = tmem + (uint32_t)(p * acc_cols);
      // Corrections: their own accumulator, or the same one.
      const uint32_t dc = Op::kSepAcc ? tmem + (uint32_t)((2 + p) * acc_cols) : d;
      const uint32_t idesc = umma_idesc<Op>(p ? ncols[1] : ncols[0]);
      uint8_t* st = base + (size_t)s * stage_bytes;
      const uint64_t dah = umma_desc<Op>(st);
      const uint64_t dal = umma_desc<Op>(st + tile_a);
      const uint64_t dbh = umma_desc<Op>(st + 2 * tile_a);
      const uint64_t dbl = umma_desc<Op>(st + 2 * tile_a + tile_b);
      for (int q = 0; q < steps; ++q) {
        const uint64_t off = (uint64_t)(2 * q);  // 32 bytes per K step, in 16 B units
        const uint32_t acc = (k > 0 || q > 0) ? 1u : 0u;
        umma<Op>(d, dah + off, dbh + off, idesc, acc);
        umma<Op>(dc, dah + off, dbl + off, idesc, Op::kSepAcc ? acc : 1u);
        umma<Op>(dc, dal + off, dbh + off, idesc, 1u);
      }
      umma_commit(&empty_bar[s]);
    }
    // Arrives once every MMA issued above has completed.
    umma_commit(&done_bar);
  } else if (warp >= 2) {
    // A producers: block k's parities go to consecutive stages.
    const int pt = threadIdx.x - 64;
    for (int k = 0; k < kblk[0]; ++k) {
      const bool two = k < kblk[1];
      const int i0 = two ? 2 * k : k + kblk[1];
      const int s0 = i0 % a.stages, u0 = i0 / a.stages;
      const int s1 = (i0 + 1) % a.stages, u1 = (i0 + 1) / a.stages;
      if (u0 > 0 && !mbar_wait(&empty_bar[s0], (u0 - 1) & 1, a.err, 4)) break;
      if (two && u1 > 0 && !mbar_wait(&empty_bar[s1], (u1 - 1) & 1, a.err, 4)) break;
      uint8_t* t0 = base + (size_t)s0 * stage_bytes;
      uint8_t* t1 = two ? base + (size_t)s1 * stage_bytes : nullptr;
      if (k + 1 < kblk[0]) tc_prefetch_block<kForward, Op>(a, m, tile, rows, k + 1, pt);
      tc_produce<kForward, Op>(a, m, tile, rows, k, t0, t1, pt);
      // Make the generic-proxy stores visible to the tensor cores.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full_bar[s0]);
      if (two) mbar_arrive(&full_bar[s1]);
    }
    if (kForward) {
      // The structural zeros l < m of this tile's rows, while the MMAs of
      // the last K blocks run.  The rows are dealt out over the N ranges
      // that have columns (the others have returned), warps 2-7 take
      // alternate rows and lanes consecutive l.
      const int nact = min((int)gridDim.z, (n_par[0] + a.Nsub - 1) / a.Nsub);
      const int pw = pt >> 5;
      for (int r = (int)blockIdx.z + nact * pw; r < 128; r += nact * (kTcProducers / 32)) {
        const int rr = tile * 128 + r;
        if (rr >= rows) break;
        int b, row;
        tc_row_map(m, rr, b, row);
        float* o = a.out + ((size_t)b * a.M + row) * a.L;
        for (int l = lane; l < m; l += 32) o[l] = 0.f;
      }
    }
  }
  __syncwarp();
  bool ok = mbar_wait(&done_bar, 0, a.err, 3);
  ok = __all_sync(0xffffffffu, ok);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok) {
    // Epilogue.  Warp w reads TMEM lanes (rows) 32 (w mod 4) .. +31, stages a
    // 32-row block in shared memory (the drained pipeline buffers) and writes
    // it back with row-contiguous, coalesced stores; the two warps of a lane
    // quarter take alternate 16-column chunks.
    constexpr int kStride = 36;  // floats per staged row (16-byte multiple)
    constexpr int kFwdStride = 34;  // forward: floats per staged row (8-byte multiple)
    const int quarter = warp & 3, half = warp >> 2;
    // Each warp owns 8 KB of the drained pipeline buffers: two TMA-store
    // buffers (a direct and a mirrored 32 x 16 block each, the box layout of
    // tO2 / tO1), which the row-store path reuses as its staging area.
    float* wbuf = reinterpret_cast<float*>(base) + warp * 2048;
    float* stage = wbuf;
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
    const int row0 = tile * 128 + quarter * 32;  // first row of this warp
    if (!kForward) {
      const bool vec = (a.J & 3) == 0;
      int nb = 0;  // TMA-stored chunks of this warp (buffer nb & 1)
      for (int c = half; c < a.Nsub / 16; c += 2) {
        float e[16], od[16];
        tc_ld_acc<Op>(lane_base, acc_cols, c, n_par[1] > 0, e, od);
        const int jb = lo + 16 * c;
        const int jm = a.J - jb - 16;
        if (a.tma_out && jb + 16 <= a.Jh && jm >= a.Jh) {
          // Direct block j = jb .. jb+15 and mirrored block j = jm .. jm+15,
          // both ascending, 16 floats per staged row.
          float* sd = wbuf + (nb & 1) * 1024;
          float* sm = sd + 512;
          if (lane == 0) bulk_wait_read<1>();  // this buffer's store two chunks ago
          __syncwarp();
          float4* d4 = reinterpret_cast<float4*>(sd + lane * 16);
          float4* m4 = reinterpret_cast<float4*>(sm + lane * 16);
          float4 dv[4], mv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            dv[i] = make_float4(e[4 * i] + od[4 * i], e[4 * i + 1] + od[4 * i + 1],
                                e[4 * i + 2] + od[4 * i + 2], e[4 * i + 3] + od[4 * i + 3]);
            mv[i] = make_float4(e[15 - 4 * i] - od[15 - 4 * i], e[14 - 4 * i] - od[14 - 4 * i],
                                e[13 - 4 * i] - od[13 - 4 * i], e[12 - 4 * i] - od[12 - 4 * i]);
          }
          // A staged row is 64 bytes: at store i lane L writes its float4
          // (i + L / 2) mod 4, so each 8-lane phase covers all 32 banks once.
          const int rot = (lane >> 1) & 3;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int q = (i + rot) & 3;
            d4[q] = pick4(dv, q);
            m4[q] = pick4(mv, q);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            // Rows (field, cos / sin of m) are the box's (z, y); fields past
            // nf fall outside the tensor and are not written.
            if (m == 0) {
              tma_store_3d(&tO1, sd, jb, 0, row0);
              tma_store_3d(&tO1, sm, jm, 0, row0);
            } else {
              tma_store_3d(&tO2, sd, jb, 2 * m - 1, row0 >> 1);
              tma_store_3d(&tO2, sm, jm, 2 * m - 1, row0 >> 1);
            }
            bulk_commit();
          }
          ++nb;
          continue;
        }
        // Row-store path: the staging area is this warp's TMA buffers, so
        // their stores must have read them.
        if (lane == 0 && nb > 0) bulk_wait_read<0>();
        __syncwarp();
        // stage[r][t] = E + O at j = 16c + t; stage[r][16 + t] = E - O at
        // j = J - 16(c+1) + t (the mirrored block, ascending).
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          stage[lane * kStride + t] = e[t] + od[t];
          stage[lane * kStride + 16 + (15 - t)] = e[t] - od[t];
        }
        __syncwarp();
        // 4 threads per row, 8 rows per pass, 4 passes; two half-blocks.
        for (int pass = 0; pass < 8; ++pass) {
          const int hb = pass >> 2;                    // 0: direct, 1: mirror
          const int r = (pass & 3) * 8 + (lane >> 2);  // staged row
          const int q = lane & 3;                      // float4 within 16
          const int rr = row0 + r;
          if (rr < rows) {
            int b, row;
            tc_row_map(m, rr, b, row);
            float* o = a.out + ((size_t)b * a.M + row) * a.J;
            const float* src = stage + r * kStride + hb * 16 + q * 4;
            const int j = (hb ? jm : jb) + q * 4;
            if (vec && jb + 16 <= a.Jh && (hb == 0 || jm >= a.Jh)) {
              *reinterpret_cast<float4*>(o + j) =
                  *reinterpret_cast<const float4*>(src);
            } else {
#pragma unroll
              for (int e2 = 0; e2 < 4; ++e2) {
                const int jj = j + e2;
                // direct half covers j < Jh; mirrored half covers j >= J - Jh
                // except the self-mirrored middle row of an odd J.
                if (hb == 0) {
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
      // The stores have read their shared-memory source before the CTA (and
      // its shared memory) ends; their global writes complete with the grid.
      if (lane == 0 && nb > 0) bulk_wait_read<0>();
      __syncwarp();
    } else {
      const int nchunks = (max(cnt[0], cnt[1]) + 15) / 16;
      for (int c = half; c < nchunks; c += 2) {
        float e[16], od[16];
        tc_ld_acc<Op>(lane_base, acc_cols, c, cnt[1] > 0, e, od);
        // Interleave parities: l = m + 32c + 2t + p.  Rows kFwdStride = 34
        // floats apart: each half-warp's 8-byte stores cover all 32 banks.
#pragma unroll
        for (int t = 0; t < 16; ++t)
          *reinterpret_cast<float2*>(stage + lane * kFwdStride + 2 * t) = make_float2(e[t], od[t]);
        __syncwarp();
        const int lp = lo + 16 * c + (lane >> 1);
        const bool keep = (lane & 1) ? (lp < n_par[1]) : (lp < n_par[0]);
        fwd_store_chunk(a.out, a.M, a.L, m, rows, row0, stage, kFwdStride, m + 2 * (lo + 16 * c),
                        keep, lane);
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

// Table [rows][inner] of bf16 (tf32 = 0) or tf32-in-FP32 (tf32 = 1) entries;
// the box is one K block (kRowBytes) of box_rows rows, swizzled for the MMA.
static int make_map(CUtensorMap* tm, const void* ptr, int tf32, int inner, long long rows,
                    int box_rows) {
  auto fn = encode_fn();
  const int esz = tf32 ? 4 : 2;
  const int rb = tc_row_bytes(tf32);
  const int kb = rb / esz;
  DINO_REQUIRE(fn != nullptr, DINO_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  DINO_REQUIRE(((uintptr_t)ptr & 15) == 0, DINO_ERR_ARG, "TMA base must be 16-byte aligned");
  DINO_REQUIRE(inner % kb == 0 && box_rows >= 8 && box_rows <= 256, DINO_ERR_ARG,
               "bad TMA box");
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)inner * esz};
  cuuint32_t box[2] = {(cuuint32_t)kb, (cuuint32_t)box_rows};
  cuuint32_t elem[2] = {1u, 1u};
  CUresult r = fn(tm, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                  2, (void*)ptr, dims, strides, box,
                  elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  rb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return DINO_ERR_CUDA;
  }
  return DINO_OK;
}

// FP32 output tensor [nf][M][J] for the inverse epilogue's TMA stores: box
// 16 latitudes x box_y rows x box_z fields.  Returns false (row stores are
// used instead) when the layout does not allow tensor stores.
static bool make_out_map(CUtensorMap* tm, const float* out, int J, int M, int nf, int box_y,
                         int box_z) {
  auto fn = encode_fn();
  if (!fn || (J & 3) != 0 || ((uintptr_t)out & 15) != 0 || nf < 1) return false;
  cuuint64_t dims[3] = {(cuuint64_t)J, (cuuint64_t)M, (cuuint64_t)nf};
  cuuint64_t strides[2] = {(cuuint64_t)J * sizeof(float), (cuuint64_t)M * J * sizeof(float)};
  cuuint32_t box[3] = {16u, (cuuint32_t)box_y, (cuuint32_t)box_z};
  cuuint32_t elem[3] = {1u, 1u, 1u};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)out, dims, strides, box, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Both output maps of an inverse launch; sets a.tma_out.
static void tc_out_maps(const dino_plan* p, TcArgs* a, float* out, int nf, CUtensorMap* o2,
                        CUtensorMap* o1) {
  memset(o2, 0, sizeof(*o2));
  memset(o1, 0, sizeof(*o1));
  a->tma_out = make_out_map(o2, out, p->J, p->M, nf, 2, 16) &&
               make_out_map(o1, out, p->J, p->M, nf, 1, 32);
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

// N range widths: the full range split in 1, 2 or 4, and 128 and 64
// columns (an accumulator pair of 128 columns is the widest that lets two
// CTAs share TMEM); depths from 2 stages while the shared memory fits.  The
// epilogue stages its output in the drained pipeline buffers, 8 KB per warp.
static void tc_candidates(int nfull, int accs, int row_bytes, std::vector<TcShape>* out) {
  std::vector<int> widths;
  for (int nsplit : {1, 2, 4}) widths.push_back(round_up((nfull + nsplit - 1) / nsplit, 16));
  for (int w : {128, 64})
    if (w < nfull) widths.push_back(w);
  std::vector<int> seen;
  for (int nsub : widths) {
    bool dup = false;
    for (int w : seen) dup |= (w == nsub);
    if (dup || tmem_cols_for(accs * nsub) > 512) continue;
    seen.push_back(nsub);
    const int nsplit = (nfull + nsub - 1) / nsub;
    const size_t stage = 2 * 128 * (size_t)row_bytes + 2 * (size_t)nsub * row_bytes;
    for (int stages = 2; stages <= kMaxStages; ++stages) {
      const size_t smem = std::max(stage * stages, (size_t)kTcThreads / 32 * 8192) + 1024;
      if (smem > kTcSmemLimit) break;
      out->push_back({nsplit, nsub, stages, smem});
    }
  }
}

// Modal rows start 16-byte aligned in every segment (the inverse producer's
// float4 path).
static int tc_vec_input(const dino_plan* p, const Segs& in) {
  if (p->L % 4 != 0) return 0;
  for (int i = 0; i < in.n; ++i)
    if (((uintptr_t)in.ptr[i] & 15) != 0) return 0;
  return 1;
}

static TcArgs tc_args(const dino_plan* p, const TcTables* t, bool forward, int nf) {
  TcArgs a{};
  a.nf = nf;
  a.M = p->M;
  a.L = p->L;
  a.J = p->J;
  a.Jh = p->Jh;
  a.Nrows = forward ? t->Nf : t->Np;
  a.err = t->d_err;
  return a;
}

// A launch's shape fields in the kernel arguments.
static void tc_set_shape(const TcTables* t, int m0, int nsub, int stages, TcArgs* a) {
  a->m0 = m0;
  a->Nsub = nsub;
  a->stages = stages;
  a->tmem_cols = tmem_cols_for(tc_accumulators(t->tf32) * nsub);
}

// One launch of the contraction in the plan's operand format.
template <bool kForward>
static void tc_launch(const TcTables* t, dim3 grid, size_t smem, cudaStream_t st,
                      const CUtensorMap& bh, const CUtensorMap& bl, const CUtensorMap& o2,
                      const CUtensorMap& o1, const TcArgs& a) {
  if (t->tf32)
    legendre_tc_kernel<kForward, OpTf32><<<grid, kTcThreads, smem, st>>>(bh, bl, o2, o1, a);
  else
    legendre_tc_kernel<kForward, OpBf16><<<grid, kTcThreads, smem, st>>>(bh, bl, o2, o1, a);
}

template <bool kForward>
static int tc_time_shape(dino_plan* p, TcTables* t, const TcShape& c, int m0, int m1, int nf,
                         const float* src, float* out, cudaEvent_t e0, cudaEvent_t e1,
                         float* us) {
  const size_t lw2 = (size_t)p->lw * 2;
  CUtensorMap bh, bl;
  if (!kForward) {
    DINO_TRY(make_map(&bh, t->Bih, t->tf32, t->Kp, (long long)lw2 * t->Np, c.Nsub));
    DINO_TRY(make_map(&bl, t->Bil, t->tf32, t->Kp, (long long)lw2 * t->Np, c.Nsub));
  } else {
    DINO_TRY(make_map(&bh, t->Bfh, t->tf32, t->Kj, (long long)lw2 * t->Nf, c.Nsub));
    DINO_TRY(make_map(&bl, t->Bfl, t->tf32, t->Kj, (long long)lw2 * t->Nf, c.Nsub));
  }
  TcArgs a = tc_args(p, t, kForward, nf);
  tc_set_shape(t, m0, c.Nsub, c.stages, &a);
  a.out = out;
  CUtensorMap o2, o1;
  memset(&o2, 0, sizeof(o2));
  memset(&o1, 0, sizeof(o1));
  if (kForward) {
    a.G = src;
  } else {
    a.in = one_seg(src, nf);
    a.vec = tc_vec_input(p, a.in);
    tc_out_maps(p, &a, out, nf, &o2, &o1);
  }
  dim3 grid(ceil_div(2 * nf, 128), m1 - m0, c.nsplit);
  constexpr int kReps = 10;
  for (int r = 0; r <= kReps; ++r) {
    if (r == 1) DINO_CHECK_CUDA(cudaEventRecord(e0, 0));
    tc_launch<kForward>(t, grid, c.smem, 0, bh, bl, o2, o1, a);
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
// the chunk that the transforms launch for large batches, and keeps the
// fastest.
static int tc_autotune(dino_plan* p, TcTables* t) {
  // The chunk that a large batch is transformed in.
  const int nf = l2_chunk(p, 1 << 20, p->max_fields);
  t->tuned_fields = nf;
  // Zero inputs: modal [nf][M][L] here, Fourier [nf][M][J] in the workspace.
  float* modal = nullptr;
  const size_t modal_bytes = sizeof(float) * (size_t)nf * p->M * p->L;
  DINO_CHECK_CUDA(cudaMalloc(&modal, modal_bytes));
  DINO_CHECK_CUDA(cudaMemset(modal, 0, modal_bytes));
  DINO_CHECK_CUDA(cudaMemset(p->d_work, 0, sizeof(float) * (size_t)nf * p->M * p->J));
  cudaEvent_t e0, e1;
  DINO_CHECK_CUDA(cudaEventCreate(&e0));
  DINO_CHECK_CUDA(cudaEventCreate(&e1));
  // Launch shapes are tuned for the whole m range in one launch and for two
  // m groups (low and high zonal wavenumbers: the triangle's short high-m
  // rows, with few l' for the forward and few K steps for the inverse,
  // favour other splits and depths than the long low-m rows), each group in
  // a launch of its own; per direction the faster arrangement is kept.
  auto tune_groups = [&](bool forward, int ngroups, TcTables::Shape* out,
                         float* total) -> int {
    const size_t lw2 = (size_t)p->lw * 2;
    *total = 0.f;
    for (int gi = 0; gi < ngroups; ++gi) {
      TcTables::Shape& sh = out[gi];
      sh.m0 = gi * p->lw / ngroups;
      sh.m1 = (gi + 1) * p->lw / ngroups;
      // The group's widest N range: l' of its lowest m (forward), or the
      // latitudes (inverse).
      const int nfull = forward ? round_up((p->L - sh.m0 + 1) / 2, 16) : t->Np;
      std::vector<TcShape> cands;
      tc_candidates(nfull, tc_accumulators(t->tf32), tc_row_bytes(t->tf32), &cands);
      // DINO_B200_TC_SHAPE="inv:NSUBxSTAGES,fwd:NSUBxSTAGES" keeps only the
      // named candidates (a profiler's serialised launches make its own
      // timings pick unrepresentative shapes).
      if (const char* want = std::getenv("DINO_B200_TC_SHAPE")) {
        const char* key = std::strstr(want, forward ? "fwd:" : "inv:");
        int wn = 0, ws = 0;
        if (key && std::sscanf(key + 4, "%dx%d", &wn, &ws) == 2) {
          std::vector<TcShape> keep;
          for (const TcShape& c : cands)
            if (c.Nsub == wn && c.stages == ws) keep.push_back(c);
          if (!keep.empty()) cands.swap(keep);
        }
      }
      float best = 1e30f;
      TcShape pick = cands.front();
      for (const TcShape& c : cands) {
        float us = 0.f;
        const int rc =
            forward ? tc_time_shape<true>(p, t, c, sh.m0, sh.m1, nf, p->d_work, modal, e0, e1, &us)
                    : tc_time_shape<false>(p, t, c, sh.m0, sh.m1, nf, modal, p->d_work, e0, e1,
                                           &us);
        if (rc != DINO_OK) return rc;
        if (std::getenv("DINO_B200_TC_DEBUG"))
          std::fprintf(stderr, "tc tune %s m %d-%d nsplit %d nsub %d stages %d smem %zu: %.1f us\n",
                       forward ? "fwd" : "inv", sh.m0, sh.m1, c.nsplit, c.Nsub, c.stages, c.smem, us);
        if (us < best) {
          best = us;
          pick = c;
        }
      }
      sh.nsplit = pick.nsplit;
      sh.Nsub = pick.Nsub;
      sh.stages = pick.stages;
      sh.smem = pick.smem;
      sh.us = best;
      sh.tried = (int)cands.size();
      *total += best;
      if (forward) {
        DINO_TRY(make_map(&sh.bh, t->Bfh, t->tf32, t->Kj, (long long)lw2 * t->Nf, pick.Nsub));
        DINO_TRY(make_map(&sh.bl, t->Bfl, t->tf32, t->Kj, (long long)lw2 * t->Nf, pick.Nsub));
      } else {
        DINO_TRY(make_map(&sh.bh, t->Bih, t->tf32, t->Kp, (long long)lw2 * t->Np, pick.Nsub));
        DINO_TRY(make_map(&sh.bl, t->Bil, t->tf32, t->Kp, (long long)lw2 * t->Np, pick.Nsub));
      }
    }
    return DINO_OK;
  };
  auto tune = [&](bool forward) -> int {
    TcTables::Shape* dst = forward ? t->fwd : t->inv;
    float one = 0.f;
    DINO_TRY(tune_groups(forward, 1, dst, &one));
    int ngroups = 1;
    float best = one;
    // DINO_B200_TC_M_GROUPS=1 or 2 forces the arrangement (tests of both);
    // a forced shape (DINO_B200_TC_SHAPE) is one launch.
    const char* force = std::getenv("DINO_B200_TC_M_GROUPS");
    const int forced = force ? std::atoi(force) : (std::getenv("DINO_B200_TC_SHAPE") ? 1 : 0);
    if (p->lw >= 32 && forced != 1) {
      TcTables::Shape two[TcTables::kMaxGroups];
      float t2 = 0.f;
      DINO_TRY(tune_groups(forward, 2, two, &t2));
      if (t2 < one || forced == 2) {
        for (int gi = 0; gi < 2; ++gi) dst[gi] = two[gi];
        ngroups = 2;
        best = t2;
      }
      (forward ? t->us_fwd_split : t->us_inv_split) = t2;
    }
    (forward ? t->ngroups_fwd : t->ngroups_inv) = ngroups;
    (forward ? t->us_fwd : t->us_inv) = best;
    return DINO_OK;
  };
  // The FP32 SIMT contraction on the same sizes (10 timed launches after one
  // warm-up, like the tensor-core shapes).
  auto time_simt = [&](bool forward, float* us) -> int {
    constexpr int kReps = 10;
    for (int r = 0; r <= kReps; ++r) {
      if (r == 1) DINO_CHECK_CUDA(cudaEventRecord(e0, 0));
      if (forward)
        DINO_TRY(legendre_forward_fp32(p, p->d_work, modal, nf, 0));
      else
        DINO_TRY(legendre_inverse_fp32(p, one_seg(modal, nf), p->d_work, nf, 0));
    }
    DINO_CHECK_CUDA(cudaEventRecord(e1, 0));
    DINO_CHECK_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    DINO_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *us = 1e3f * ms / kReps;
    return DINO_OK;
  };
  int rc = tune(false);
  if (rc == DINO_OK) rc = tune(true);
  if (rc == DINO_OK) rc = time_simt(false, &t->us_simt_inv);
  if (rc == DINO_OK) rc = time_simt(true, &t->us_simt_fwd);
  // DINO_B200_TENSOR_CORES_ONLY=1 keeps the tensor-core form whatever the
  // timings (the tests of the tensor-core kernels on small grids use it).
  const char* only = std::getenv("DINO_B200_TENSOR_CORES_ONLY");
  const bool tc_only = (only && only[0] == '1') || std::getenv("DINO_B200_TC_SHAPE");
  t->simt_inv = !tc_only && t->us_simt_inv < t->us_inv ? 1 : 0;
  t->simt_fwd = !tc_only && t->us_simt_fwd < t->us_fwd ? 1 : 0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(modal);
  if (rc != DINO_OK) return rc;
  return tc_status(p);
}

bool tc_use_simt(const dino_plan* p, bool forward) {
  const TcTables* t = p->tc;
  return t && (forward ? t->simt_fwd : t->simt_inv);
}

std::string tc_describe(dino_plan* p) {
  TcTables* t = p->tc;
  if (!t) return "";
  auto dir = [&](const char* name, const TcTables::Shape* g, int ng, float us, float split,
                 float simt, int used) {
    std::string out = name;
    for (int gi = 0; gi < ng; ++gi) {
      char b[160];
      snprintf(b, sizeof(b), "%s m %d-%d: %d N ranges of %d rows, %d stages (%.1f us, %d shapes)",
               gi ? ";" : "", g[gi].m0, g[gi].m1 - 1, g[gi].nsplit, g[gi].Nsub, g[gi].stages,
               g[gi].us, g[gi].tried);
      out += b;
    }
    char b[160];
    snprintf(b, sizeof(b), "; %.1f us (two m groups: %.1f us), FP32 SIMT %.1f us%s", us, split,
             simt, used ? ", faster: used" : "");
    return out + b;
  };
  char head[128];
  snprintf(head, sizeof(head), "tcgen05 %s Legendre autotuned on %d fields (shapes tried per m range): ",
           t->tf32 ? "split-TF32" : "split-BF16", t->tuned_fields);
  return std::string(head) +
         dir("inverse", t->inv, t->ngroups_inv, t->us_inv, t->us_inv_split, t->us_simt_inv,
             t->simt_inv) +
         " | " +
         dir("forward", t->fwd, t->ngroups_fwd, t->us_fwd, t->us_fwd_split, t->us_simt_fwd,
             t->simt_fwd);
}

int tc_tables_build(dino_plan* p) {
  DINO_REQUIRE(p->Jh <= 256, DINO_ERR_UNSUPPORTED,
               "tensor-core path supports at most 512 latitudes");
  DINO_REQUIRE((p->L + 1) / 2 <= 256, DINO_ERR_UNSUPPORTED,
               "tensor-core path supports at most 512 total wavenumbers");
  TcTables* t = new TcTables();
  p->tc = t;
  t->tf32 = p->precision == DINO_PREC_TF32X3;
  const int kb = t->tf32 ? OpTf32::kKB : OpBf16::kKB;
  const size_t esz = t->tf32 ? sizeof(float) : sizeof(bf16);
  const int half_l = (p->L + 1) / 2;
  t->Kp = round_up(half_l, kb);
  t->Np = round_up(p->Jh, 16);

  t->Kj = round_up(p->Jh, kb);
  t->Nf = round_up(half_l, 16);
  const size_t lw2 = (size_t)p->lw * 2;
  const size_t nBi = lw2 * t->Np * t->Kp, nBf = lw2 * t->Nf * t->Kj;
  DINO_CHECK_CUDA(cudaMalloc(&t->Bih, nBi * esz));
  DINO_CHECK_CUDA(cudaMalloc(&t->Bil, nBi * esz));
  DINO_CHECK_CUDA(cudaMalloc(&t->Bfh, nBf * esz));
  DINO_CHECK_CUDA(cudaMalloc(&t->Bfl, nBf * esz));
  DINO_CHECK_CUDA(cudaMemset(t->Bih, 0, nBi * esz));
  DINO_CHECK_CUDA(cudaMemset(t->Bil, 0, nBi * esz));
  DINO_CHECK_CUDA(cudaMemset(t->Bfh, 0, nBf * esz));
  DINO_CHECK_CUDA(cudaMemset(t->Bfl, 0, nBf * esz));
  DINO_CHECK_CUDA(cudaMalloc(&t->d_err, sizeof(int)));
  DINO_CHECK_CUDA(cudaMemset(t->d_err, 0, sizeof(int)));
  dim3 grid(ceil_div(p->Jh, 128), p->lw);
  if (t->tf32) {
    tc_table_kernel<float><<<grid, 128>>>(
        p->lw, p->L, p->Jh, p->d_x64, t->Kp, t->Np, t->Kj, t->Nf, (float*)t->Bih,
        (float*)t->Bil, (float*)t->Bfh, (float*)t->Bfl);
  } else {
    tc_table_kernel<bf16><<<grid, 128>>>(p->lw, p->L, p->Jh, p->d_x64, t->Kp, t->Np, t->Kj,
                                         t->Nf, (bf16*)t->Bih, (bf16*)t->Bil, (bf16*)t->Bfh,
                                         (bf16*)t->Bfl);
  }
  DINO_TRY(check_launch("tc_table"));
  if (t->tf32) {
    DINO_CHECK_CUDA(cudaFuncSetAttribute(legendre_tc_kernel<false, OpTf32>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmemLimit));
    DINO_CHECK_CUDA(cudaFuncSetAttribute(legendre_tc_kernel<true, OpTf32>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmemLimit));
  } else {
    DINO_CHECK_CUDA(cudaFuncSetAttribute(legendre_tc_kernel<false, OpBf16>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmemLimit));
    DINO_CHECK_CUDA(cudaFuncSetAttribute(legendre_tc_kernel<true, OpBf16>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmemLimit));
  }
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
  cudaFree(t->d_err);
  delete t;
  p->tc = nullptr;
}

static int tmem_cols_for(int cols) {
  int c = 32;
  while (c < cols) c *= 2;
  return c;
}

int tc_legendre_inverse(dino_plan* p, const Segs& in, float* out, int nf,
                        cudaStream_t st) {
  TcTables* t = p->tc;
  DINO_REQUIRE(t, DINO_ERR_ARG, "plan has no tensor-core tables");
  if (nf == 0) return DINO_OK;
  TcArgs a = tc_args(p, t, false, nf);
  a.in = in;
  a.vec = tc_vec_input(p, in);
  a.out = out;
  CUtensorMap o2, o1;
  tc_out_maps(p, &a, out, nf, &o2, &o1);
  for (int gi = 0; gi < t->ngroups_inv; ++gi) {
    const TcTables::Shape& sh = t->inv[gi];
    tc_set_shape(t, sh.m0, sh.Nsub, sh.stages, &a);
    dim3 grid(ceil_div(2 * nf, 128), sh.m1 - sh.m0, sh.nsplit);
    tc_launch<false>(t, grid, sh.smem, st, sh.bh, sh.bl, o2, o1, a);
    DINO_TRY(check_launch("legendre_tc_inverse"));
  }
  return DINO_OK;
}

int tc_legendre_forward(dino_plan* p, const float* G, float* out, int nf,
                        cudaStream_t st) {
  TcTables* t = p->tc;
  DINO_REQUIRE(t, DINO_ERR_ARG, "plan has no tensor-core tables");
  if (nf == 0) return DINO_OK;
  TcArgs a = tc_args(p, t, true, nf);
  a.G = G;
  a.out = out;
  CUtensorMap unused;  // the forward epilogue uses row stores
  memset(&unused, 0, sizeof(unused));
  for (int gi = 0; gi < t->ngroups_fwd; ++gi) {
    const TcTables::Shape& sh = t->fwd[gi];
    tc_set_shape(t, sh.m0, sh.Nsub, sh.stages, &a);
    dim3 grid(ceil_div(2 * nf, 128), sh.m1 - sh.m0, sh.nsplit);
    tc_launch<true>(t, grid, sh.smem, st, sh.bh, sh.bl, unused, unused, a);
    DINO_TRY(check_launch("legendre_tc_forward"));
  }
  return DINO_OK;
}

// Reads (and clears) the plan's device error flag.
int tc_status(dino_plan* p) {
  if (!p->tc) return DINO_OK;
  int err = 0;
  DINO_CHECK_CUDA(cudaMemcpy(&err, p->tc->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    DINO_CHECK_CUDA(cudaMemset(p->tc->d_err, 0, sizeof(int)));
    set_error("a tensor-core wait gave up (code " + std::to_string(err) + ")");
    return DINO_ERR_TIMEOUT;
  }
  return DINO_OK;
}

// One CTA whose thread 0 waits, through the contraction kernels' bounded
// wait, on an mbarrier that nothing ever completes: the wait gives up after
// limit_ns and records kWaitCheckCode in *err.  The failure path of a
// stalled pipeline, exercised without a fault.
constexpr int kWaitCheckCode = 5;

__global__ void tc_wait_check_kernel(int* err, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_wait(&bar, 0, err, kWaitCheckCode, limit_ns);
  }
}

}  // namespace dino

extern "C" int dino_plan_describe(dino_plan* p, char* buf, size_t len) {
  DINO_REQUIRE(p && buf && len > 0, DINO_ERR_ARG, "dino_plan_describe: null argument");
  char head[256];
  snprintf(head, sizeof(head),
           "grid %d x %d nodes, %d x %d modal, Legendre %s, batch capacity %d fields",
           p->I, p->J, p->M, p->L,
           p->precision == DINO_PREC_BF16X3   ? "split-BF16 (tcgen05)"
           : p->precision == DINO_PREC_TF32X3 ? "split-TF32 (tcgen05)"
                                              : "FP32 (SIMT)",
           p->max_fields);
  std::string s = head;
  const std::string tc = dino::tc_describe(p);
  if (!tc.empty()) s += "; " + tc;
  snprintf(buf, len, "%s", s.c_str());
  return DINO_OK;
}

extern "C" int dino_plan_check_wait_timeout(dino_plan* p, int64_t limit_ns, void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_plan_check_wait_timeout: null argument");
  DINO_REQUIRE(p->tc, DINO_ERR_UNSUPPORTED,
               "dino_plan_check_wait_timeout: the plan has no tensor-core kernels");
  DINO_REQUIRE(limit_ns >= 1000000 && limit_ns <= 10000000000LL, DINO_ERR_ARG,
               "dino_plan_check_wait_timeout: limit must be 1 ms .. 10 s");
  dino::tc_wait_check_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(
      p->tc->d_err, (unsigned long long)limit_ns);
  return dino::check_launch("tc_wait_check");
}

extern "C" int dino_plan_status(dino_plan* p) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_plan_status: null argument");
  DINO_CHECK_CUDA(cudaDeviceSynchronize());
  return dino::tc_status(p);
}

