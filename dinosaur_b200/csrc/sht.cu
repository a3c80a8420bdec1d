// Spherical-harmonic transform pair on one B200: per-m Legendre contraction
// over Gaussian latitude (N/S folded, FP32 SIMT form here; tensor-core form in
// legendre_tc.cu) and a real FFT over longitude in shared memory.
//
// Semantics follow RealSphericalHarmonics.inverse_transform / transform
// (dinosaur/spherical_harmonic.py:262-280):
//   inverse:  px[b,m,j] = sum_l p[m,j,l] x[b,m,l];  out[b,i,j] = sum_m f[i,m] px[b,m,j]
//   forward:  fwx[b,m,j] = sum_i f[i,m] w[j] z[b,i,j];  out[b,m,l] = sum_j p[m,j,l] fwx[b,m,j]
// with f the unit-norm real Fourier basis (fourier.py:24-60) and p the
// normalised associated Legendre functions duplicated over +-m rows.
//
// Folding: Gauss nodes are mirror symmetric and p[m, J-1-j, l] =
// (-1)^(l-m) p[m, j, l], so each contraction splits into even and odd (l-m)
// halves over Jh = ceil(J/2) latitudes, halving the arithmetic.

#include <cmath>

#include <algorithm>

#include "dino_internal.cuh"

namespace dino {

// ---------------------------------------------------------------------------
// Legendre contraction, FP32 SIMT
// ---------------------------------------------------------------------------

constexpr int kLegTB = 128;  // (field, cos/sin) rows per CTA
constexpr int kLegTN = 32;   // latitudes (inverse) or l values (forward) per CTA
constexpr int kLegKC = 16;   // contraction chunk
constexpr int kLegThreads = 128;

// Row r of the m-slice: m == 0 has one row per field (cos), m > 0 has two.
__device__ __forceinline__ void row_map(int m, int r, int& b, int& row) {
  if (m == 0) {
    b = r;
    row = 0;
  } else {
    b = r >> 1;
    row = 2 * m - 1 + (r & 1);
  }
}

// Each thread stages 4 rows x 4 contraction indices of a 128 x 16 operand
// chunk: rows (tid / 4) + 32 i, indices 4 (tid % 4) .. + 3.  Row pointers are
// resolved once per CTA; the next chunk is prefetched into registers while
// the current one is consumed from shared memory.

// out_fourier[b][row][j] for all j from modal rows (inverse contraction).
__global__ void __launch_bounds__(kLegThreads)
legendre_inverse_simt(Segs in, float* __restrict__ out, int B, int M, int L,
                      int J, int Jh, const float* __restrict__ ptab,
                      const int64_t* __restrict__ ptab_off) {
  const int m = blockIdx.z;
  const int rows = (m == 0) ? B : 2 * B;
  const int r0 = blockIdx.y * kLegTB;
  if (r0 >= rows) return;
  const int j0 = blockIdx.x * kLegTN;
  const int Lm = L - m;
  const float* P = ptab + ptab_off[m];

  __shared__ __align__(16) float Xs[kLegKC][kLegTB + 4];
  __shared__ __align__(16) float Ps[kLegKC][kLegTN];

  const int tid = threadIdx.x;
  const int tx = tid & 7;   // 8 groups of 4 latitudes
  const int ty = tid >> 3;  // 16 groups of 8 rows
  const int lq = tid & 3;   // load quarter (4 contraction indices)
  const float* xrow[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = r0 + (tid >> 2) + 32 * i;
    xrow[i] = nullptr;
    if (r < rows) {
      int b, row;
      row_map(m, r, b, row);
      xrow[i] = seg_field(in, b, (size_t)M * L) + (size_t)row * L + m;
    }
  }
  const int pk = tid >> 3, pj = (tid & 7) * 4;  // P chunk: 16 x 32 as float4
  float xv[4][4];
  float4 pv;
  auto fetch = [&](int kc) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = kc + lq * 4 + e;
        xv[i][e] = (xrow[i] && k < Lm) ? xrow[i][k] : 0.f;
      }
    const int k = kc + pk;
    const int j = j0 + pj;
    // Vector load only when the row start is 16-byte aligned (Jh % 4 == 0;
    // the per-m table offsets are multiples of Jh).
    if ((Jh & 3) == 0 && k < Lm && j + 3 < Jh) {
      pv = *reinterpret_cast<const float4*>(P + (size_t)k * Jh + j);
    } else {
      float t[4];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        t[e] = (k < Lm && j + e < Jh) ? P[(size_t)k * Jh + j + e] : 0.f;
      pv = make_float4(t[0], t[1], t[2], t[3]);
    }
  };

  float accE[8][4], accO[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int t = 0; t < 4; ++t) accE[i][t] = accO[i][t] = 0.f;

  fetch(0);
  for (int kc = 0; kc < Lm; kc += kLegKC) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int e = 0; e < 4; ++e) Xs[lq * 4 + e][(tid >> 2) + 32 * i] = xv[i][e];
    *reinterpret_cast<float4*>(&Ps[pk][pj]) = pv;
    __syncthreads();
    if (kc + kLegKC < Lm) fetch(kc + kLegKC);
#pragma unroll
    for (int kk = 0; kk < kLegKC; kk += 2) {
      float4 xa = *reinterpret_cast<const float4*>(&Xs[kk][ty * 8]);
      float4 xb = *reinterpret_cast<const float4*>(&Xs[kk][ty * 8 + 4]);
      float4 pp = *reinterpret_cast<const float4*>(&Ps[kk][tx * 4]);
      float xe[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
      float pe[4] = {pp.x, pp.y, pp.z, pp.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int t = 0; t < 4; ++t) accE[i][t] = fmaf(xe[i], pe[t], accE[i][t]);
      xa = *reinterpret_cast<const float4*>(&Xs[kk + 1][ty * 8]);
      xb = *reinterpret_cast<const float4*>(&Xs[kk + 1][ty * 8 + 4]);
      pp = *reinterpret_cast<const float4*>(&Ps[kk + 1][tx * 4]);
      float xo[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
      float po[4] = {pp.x, pp.y, pp.z, pp.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int t = 0; t < 4; ++t) accO[i][t] = fmaf(xo[i], po[t], accO[i][t]);
    }
  }

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int r = r0 + ty * 8 + i;
    if (r >= rows) continue;
    int b, row;
    row_map(m, r, b, row);
    float* o = out + ((size_t)b * M + row) * J;
    const int jv = j0 + tx * 4;
    if ((J & 3) == 0 && jv + 3 < Jh) {
      // Row starts are 16-byte aligned; the mirrored block J-4-jv.. is too.
      *reinterpret_cast<float4*>(o + jv) =
          make_float4(accE[i][0] + accO[i][0], accE[i][1] + accO[i][1],
                      accE[i][2] + accO[i][2], accE[i][3] + accO[i][3]);
      *reinterpret_cast<float4*>(o + (J - 4 - jv)) =
          make_float4(accE[i][3] - accO[i][3], accE[i][2] - accO[i][2],
                      accE[i][1] - accO[i][1], accE[i][0] - accO[i][0]);
      continue;
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      int j = jv + t;
      if (j >= Jh) continue;
      o[j] = accE[i][t] + accO[i][t];
      int jm = J - 1 - j;
      if (jm != j) o[jm] = accE[i][t] - accO[i][t];
    }
  }
}

// out_modal[b][row][l] = sum_j p[m,j,l] G[b][row][j] (forward contraction);
// writes zeros for l < m.  A CTA covers 128 rows and TN values of l (64 for
// long l ranges, 32 for short ones, which keeps more CTAs per SM): thread
// (tx, ty) accumulates rows 8 ty .. 8 ty + 7 at l - m = k0 + tx + 8 t,
// t < TN / 8, all of one parity, so it reads only the symmetric (even) or
// antisymmetric (odd) latitude fold.  Folds and table chunks are fetched with
// float4 loads where the rows allow.
template <int TN>
__global__ void __launch_bounds__(kLegThreads)
legendre_forward_simt(const float* __restrict__ G, float* __restrict__ out,
                      int B, int M, int L, int J, int Jh,
                      const float* __restrict__ ptab,
                      const int64_t* __restrict__ ptab_off) {
  const int m = blockIdx.z;
  const int rows = (m == 0) ? B : 2 * B;
  const int r0 = blockIdx.y * kLegTB;
  if (r0 >= rows) return;
  const int Lm = L - m;
  constexpr int TT = TN / 8;           // l values per thread
  constexpr int PV = TN / 8;           // table values fetched per thread and chunk
  constexpr int PT = kLegKC / PV;      // threads per table row
  const int k0 = blockIdx.x * TN;  // l - m offset of this tile
  const int tid = threadIdx.x;
  const int tx = tid & 7;
  const int ty = tid >> 3;

  if (blockIdx.x == 0 && m > 0) {
    // Structural zeros l < m of the rows handled by this CTA.
    for (int idx = tid; idx < kLegTB * m; idx += kLegThreads) {
      int rl = idx / m, l = idx % m;
      int r = r0 + rl;
      if (r < rows) {
        int b, row;
        row_map(m, r, b, row);
        out[((size_t)b * M + row) * L + l] = 0.f;
      }
    }
  }
  if (k0 >= Lm) return;
  const float* P = ptab + ptab_off[m];

  __shared__ __align__(16) float Ss[kLegKC][kLegTB + 4];
  __shared__ __align__(16) float Ds[kLegKC][kLegTB + 4];
  __shared__ float Ps[kLegKC][TN + 1];

  const int lq = tid & 3;
  const float* grow[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = r0 + (tid >> 2) + 32 * i;
    grow[i] = nullptr;
    if (r < rows) {
      int b, row;
      row_map(m, r, b, row);
      grow[i] = G + ((size_t)b * M + row) * J;
    }
  }
  // Row starts are 16-byte aligned when J % 4 == 0 (then so are j and the
  // mirrored J - 4 - j for j a multiple of 4).
  const bool vec = (J & 3) == 0;
  // P chunk TN (l) x 16 (j): thread loads l = tid / PT, j = PV (tid % PT) ..
  const int pl_ = tid / PT, pjq = (tid % PT) * PV;
  float sv[4][4], dv[4][4], pvr[PV];
  auto fetch = [&](int jc) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = jc + lq * 4;
      float g1[4] = {0.f, 0.f, 0.f, 0.f}, g2[4] = {0.f, 0.f, 0.f, 0.f};
      if (grow[i]) {
        if (vec && j + 4 <= Jh) {
          const float4 d = *reinterpret_cast<const float4*>(grow[i] + j);
          const float4 e = *reinterpret_cast<const float4*>(grow[i] + J - 4 - j);
          g1[0] = d.x; g1[1] = d.y; g1[2] = d.z; g1[3] = d.w;
          g2[0] = e.w; g2[1] = e.z; g2[2] = e.y; g2[3] = e.x;
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (j + e < Jh) {
              g1[e] = grow[i][j + e];
              const int jm = J - 1 - (j + e);
              g2[e] = (jm != j + e) ? grow[i][jm] : 0.f;
            }
          }
        }
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        sv[i][e] = g1[e] + g2[e];
        dv[i][e] = g1[e] - g2[e];
      }
    }
    const int k = k0 + pl_;
    const int j = jc + pjq;
    const float* pr = P + (size_t)k * Jh + j;
    if ((Jh & 3) == 0 && k < Lm && j + PV <= Jh) {
      // Table rows start 16-byte aligned (the per-m offsets are multiples of
      // Jh).
#pragma unroll
      for (int q = 0; q < PV / 4; ++q) {
        const float4 v = *reinterpret_cast<const float4*>(pr + 4 * q);
        pvr[4 * q] = v.x;
        pvr[4 * q + 1] = v.y;
        pvr[4 * q + 2] = v.z;
        pvr[4 * q + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int e = 0; e < PV; ++e) pvr[e] = (k < Lm && j + e < Jh) ? pr[e] : 0.f;
    }
  };

  float acc[8][TT];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int t = 0; t < TT; ++t) acc[i][t] = 0.f;

  fetch(0);
  for (int jc = 0; jc < Jh; jc += kLegKC) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        Ss[lq * 4 + e][(tid >> 2) + 32 * i] = sv[i][e];
        Ds[lq * 4 + e][(tid >> 2) + 32 * i] = dv[i][e];
      }
#pragma unroll
    for (int e = 0; e < PV; ++e) Ps[pjq + e][pl_] = pvr[e];
    __syncthreads();
    if (jc + kLegKC < Jh) fetch(jc + kLegKC);
    const float* fold = (tx & 1) ? &Ds[0][0] : &Ss[0][0];
#pragma unroll
    for (int jj = 0; jj < kLegKC; ++jj) {
      float4 fa = *reinterpret_cast<const float4*>(fold + jj * (kLegTB + 4) + ty * 8);
      float4 fb = *reinterpret_cast<const float4*>(fold + jj * (kLegTB + 4) + ty * 8 + 4);
      float f8[8] = {fa.x, fa.y, fa.z, fa.w, fb.x, fb.y, fb.z, fb.w};
      float pw[TT];
#pragma unroll
      for (int t = 0; t < TT; ++t) pw[t] = Ps[jj][tx + 8 * t];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int t = 0; t < TT; ++t) acc[i][t] = fmaf(f8[i], pw[t], acc[i][t]);
    }
  }

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int r = r0 + ty * 8 + i;
    if (r >= rows) continue;
    int b, row;
    row_map(m, r, b, row);
    float* o = out + ((size_t)b * M + row) * L + m;
#pragma unroll
    for (int t = 0; t < TT; ++t) {
      int k = k0 + tx + 8 * t;
      if (k < Lm) o[k] = acc[i][t];
    }
  }
}

// The FP32 SIMT inverse contraction regardless of the plan's precision.
int legendre_inverse_fp32(dino_plan* p, const Segs& in, float* out, int nf,
                          cudaStream_t st) {
  NvtxRange range("inv_legendre");
  dim3 grid(ceil_div(p->Jh, kLegTN), ceil_div(2 * nf, kLegTB), p->lw);
  legendre_inverse_simt<<<grid, kLegThreads, 0, st>>>(
      in, out, nf, p->M, p->L, p->J, p->Jh, p->d_ptab, p->d_ptab_off);
  return check_launch("legendre_inverse_simt");
}

int legendre_inverse(dino_plan* p, const Segs& in, float* out, int nf,
                     cudaStream_t st) {
  NvtxRange range("inv_legendre");
  if (p->precision != DINO_PREC_FP32 && !tc_use_simt(p, false))
    return tc_legendre_inverse(p, in, out, nf, st);
  dim3 grid(ceil_div(p->Jh, kLegTN), ceil_div(2 * nf, kLegTB), p->lw);
  legendre_inverse_simt<<<grid, kLegThreads, 0, st>>>(
      in, out, nf, p->M, p->L, p->J, p->Jh, p->d_ptab, p->d_ptab_off);
  return check_launch("legendre_inverse_simt");
}

int legendre_forward(dino_plan* p, const float* G, float* out, int nf,
                     cudaStream_t st) {
  NvtxRange range("fwd_legendre");
  if (p->precision != DINO_PREC_FP32 && !tc_use_simt(p, true))
    return tc_legendre_forward(p, G, out, nf, st);
  return legendre_forward_fp32(p, G, out, nf, st);
}

// The FP32 SIMT forward contraction regardless of the plan's precision.
int legendre_forward_fp32(dino_plan* p, const float* G, float* out, int nf,
                          cudaStream_t st) {
  if (p->L > 64) {
    dim3 grid(ceil_div(p->L, 64), ceil_div(2 * nf, kLegTB), p->lw);
    legendre_forward_simt<64><<<grid, kLegThreads, 0, st>>>(
        G, out, nf, p->M, p->L, p->J, p->Jh, p->d_ptab, p->d_ptab_off);
  } else {
    dim3 grid(ceil_div(p->L, 32), ceil_div(2 * nf, kLegTB), p->lw);
    legendre_forward_simt<32><<<grid, kLegThreads, 0, st>>>(
        G, out, nf, p->M, p->L, p->J, p->Jh, p->d_ptab, p->d_ptab_off);
  }
  return check_launch("legendre_forward_simt");
}

// ---------------------------------------------------------------------------
// Real FFT over longitude (power-of-two I = 2N), shared-memory Stockham
// radix-4/2 on the half-length complex sequence z[n] = x[2n] + i x[2n+1].
// ---------------------------------------------------------------------------

constexpr int kFftJS = 16;       // latitudes (columns) per CTA
constexpr int kFftThreads = 256;
static_assert(kFftThreads % kFftJS == 0, "a thread keeps one FFT column in every pass");

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// Multiply by +i (kSign = +1) or -i (kSign = -1).
template <int kSign>
__device__ __forceinline__ float2 cmul_i(float2 a) {
  return kSign > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// exp(2 pi i k / 16), k = 0..7 (the 16th roots of unity used by the
// register DFTs; cos/sin of multiples of pi/8).
__device__ __forceinline__ float2 root16(int k) {
  constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f;
  constexpr float h = 0.70710678118654757f;
  switch (k & 7) {
    case 0: return make_float2(1.f, 0.f);
    case 1: return make_float2(c1, s1);
    case 2: return make_float2(h, h);
    case 3: return make_float2(s1, c1);
    case 4: return make_float2(0.f, 1.f);
    case 5: return make_float2(-s1, c1);
    case 6: return make_float2(-h, h);
    default: return make_float2(-c1, s1);
  }
}

// exp(kSign 2 pi i k / 16) for any k >= 0.
template <int kSign>
__device__ __forceinline__ float2 w16(int k) {
  float2 w = root16(k & 7);
  if (k & 8) w = make_float2(-w.x, -w.y);
  return kSign < 0 ? cconj(w) : w;
}

// Multiplies by exp(kSign 2 pi i k / 16) for a compile-time k: multiples of
// 4 are sign swaps (no multiply), the others one complex multiply.
template <int K, int kSign>
__device__ __forceinline__ float2 twiddle16(float2 a) {
  constexpr int k = K & 15;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (k == 4) {
    return cmul_i<kSign>(a);
  } else if constexpr (k == 8) {
    return make_float2(-a.x, -a.y);
  } else if constexpr (k == 12) {
    return cmul_i<-kSign>(a);
  } else {
    return cmul(a, w16<kSign>(k));
  }
}

// DFT of length 4: X_k = sum_q v_q exp(kSign 2 pi i q k / 4).
template <int kSign>
__device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d) {
  const float2 s0 = cadd(a, c), d0 = csub(a, c);
  const float2 s1 = cadd(b, d), d1 = cmul_i<kSign>(csub(b, d));
  a = cadd(s0, s1);
  c = csub(s0, s1);
  b = cadd(d0, d1);
  d = csub(d0, d1);
}

// In-register DFT of length R (power of two <= 16), natural order in and
// out: v_s <- sum_q v_q exp(kSign 2 pi i q s / R).  Lengths 4 and 16 use
// DFT-4 butterflies (16 = 4 x 4 with the twiddles of multiples of 4 as sign
// swaps); 2 and 8 split once more by two.
template <int R, int kSign>
__device__ __forceinline__ void dft_reg(float2* v) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    dft4<kSign>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 16) {
    // q = 4 q1 + q2, s = s1 + 4 s2: DFT-4 over q1 for each q2, twiddle
    // W16^(q2 s1), DFT-4 over q2 for each s1.
    float2 y[16];
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2) {
      float2 a = v[q2], b = v[4 + q2], c = v[8 + q2], d = v[12 + q2];
      dft4<kSign>(a, b, c, d);
      y[4 * q2] = a;      // s1 = 0
      y[4 * q2 + 1] = b;  // s1 = 1
      y[4 * q2 + 2] = c;  // s1 = 2
      y[4 * q2 + 3] = d;  // s1 = 3
    }
    y[5] = twiddle16<1, kSign>(y[5]);
    y[6] = twiddle16<2, kSign>(y[6]);
    y[7] = twiddle16<3, kSign>(y[7]);
    y[9] = twiddle16<2, kSign>(y[9]);
    y[10] = twiddle16<4, kSign>(y[10]);
    y[11] = twiddle16<6, kSign>(y[11]);
    y[13] = twiddle16<3, kSign>(y[13]);
    y[14] = twiddle16<6, kSign>(y[14]);
    y[15] = twiddle16<9, kSign>(y[15]);
#pragma unroll
    for (int s1 = 0; s1 < 4; ++s1) {
      float2 a = y[s1], b = y[4 + s1], c = y[8 + s1], d = y[12 + s1];
      dft4<kSign>(a, b, c, d);
      v[s1] = a;
      v[s1 + 4] = b;
      v[s1 + 8] = c;
      v[s1 + 12] = d;
    }
  } else {
    // R = 8: even / odd halves, then W8^k = W16^(2k) on the odd half.
    constexpr int H = R / 2;
    float2 e[H], o[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    dft_reg<H, kSign>(e);
    dft_reg<H, kSign>(o);
    const float2 t0 = o[0];
    const float2 t1 = twiddle16<2, kSign>(o[1]);
    const float2 t2 = twiddle16<4, kSign>(o[2]);
    const float2 t3 = twiddle16<6, kSign>(o[3]);
    v[0] = cadd(e[0], t0);
    v[4] = csub(e[0], t0);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);
    v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
  }
}

// One radix-R Stockham pass over N points for kFftJS columns.  load(n, c)
// returns element n of column c; store(n, c, v) writes output element n.
// Every thread issues all of its loads before its first store; kSync puts a
// barrier between the two, so that the pass may run in place on one shared
// buffer.
template <int N, int R, int kSign, bool kSync, class Load, class Store>
__device__ __forceinline__ void stockham_pass(int Ns, const float2* twn,
                                              Load load, Store store) {
  constexpr int Q = N / R;
  constexpr int kTotal = Q * kFftJS;
  constexpr int kItems = (kTotal + kFftThreads - 1) / kFftThreads;
  const int stride = N / (Ns * R);
  float2 v[kItems][R];
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int item = threadIdx.x + it * kFftThreads;
    if (item < kTotal) {
      const int c = item % kFftJS, j = item / kFftJS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = load(j + r * Q, c);
    }
  }
  if (kSync) __syncthreads();
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int item = threadIdx.x + it * kFftThreads;
    if (item < kTotal) {
      const int c = item % kFftJS, j = item / kFftJS;
      const int k = j % Ns;
      if (k) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = twn[r * k * stride];
          if (kSign < 0) w = cconj(w);
          v[it][r] = cmul(v[it][r], w);
        }
      }
      dft_reg<R, kSign>(v[it]);
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) store(base + r * Ns, c, v[it][r]);
    }
  }
}

// Radix schedule (at most three passes) for each supported N.
template <int N> struct FftRadix;
template <> struct FftRadix<8> { static constexpr int r1 = 8, r2 = 1, r3 = 1; };
template <> struct FftRadix<16> { static constexpr int r1 = 16, r2 = 1, r3 = 1; };
template <> struct FftRadix<32> { static constexpr int r1 = 8, r2 = 4, r3 = 1; };
template <> struct FftRadix<64> { static constexpr int r1 = 8, r2 = 8, r3 = 1; };
template <> struct FftRadix<128> { static constexpr int r1 = 16, r2 = 8, r3 = 1; };
template <> struct FftRadix<256> { static constexpr int r1 = 16, r2 = 16, r3 = 1; };
template <> struct FftRadix<512> { static constexpr int r1 = 8, r2 = 8, r3 = 8; };

// Shared memory of both kernels: one N x kFftJS complex buffer and the two
// N-entry twiddle tables.
template <int N>
constexpr size_t fft_smem_bytes() {
  return sizeof(float2) * ((size_t)N * kFftJS + 2 * N);
}

// Runs all passes on the one shared buffer S: the first pass reads via
// `first` (in place when kFirstInS), the last writes via `last`; the passes
// between run in place.
// kLastInS: the last pass writes back into S (in place, so its loads finish
// before its stores).
template <int N, int kSign, bool kFirstInS, bool kLastInS = false, class First, class Last>
__device__ __forceinline__ void fft_passes(float2* S, const float2* twn, First first,
                                           Last last) {
  using Rd = FftRadix<N>;
  auto s_load = [S](int n, int c) { return S[n * kFftJS + c]; };
  auto s_store = [S](int n, int c, float2 v) { S[n * kFftJS + c] = v; };
  if constexpr (Rd::r2 == 1) {
    stockham_pass<N, Rd::r1, kSign, kFirstInS || kLastInS>(1, twn, first, last);
  } else if constexpr (Rd::r3 == 1) {
    stockham_pass<N, Rd::r1, kSign, kFirstInS>(1, twn, first, s_store);
    __syncthreads();
    stockham_pass<N, Rd::r2, kSign, kLastInS>(Rd::r1, twn, s_load, last);
  } else {
    stockham_pass<N, Rd::r1, kSign, kFirstInS>(1, twn, first, s_store);
    __syncthreads();
    stockham_pass<N, Rd::r2, kSign, true>(Rd::r1, twn, s_load, s_store);
    __syncthreads();
    stockham_pass<N, Rd::r3, kSign, kLastInS>(Rd::r1 * Rd::r2, twn, s_load, last);
  }
}

// Copies a rows x kFftJS tile (row stride J floats) into shared memory
// (row stride kFftJS): 16-byte asynchronous copies when rows start 16-byte
// aligned and the tile is full, else scalar loads with zero fill past ncol.
template <int kMaxRows>
__device__ __forceinline__ void stage_tile(const float* __restrict__ src, int rows,
                                           int J, int ncol, float* dst) {
  if ((J & 3) == 0 && ncol == kFftJS && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    constexpr int kQ = kFftJS / 4;  // float4 per row
    // 16-byte asynchronous copies (cp.async): every copy of the thread is in
    // flight at once and none holds a register; the caller's barrier follows
    // the wait below.
    constexpr int kChunks = (kMaxRows * kQ + kFftThreads - 1) / kFftThreads;
#pragma unroll
    for (int i = 0; i < kChunks; ++i) {
      const int t = threadIdx.x + i * kFftThreads;
      const int r = t / kQ, q = t % kQ;
      if (r < rows) {
        const float* g = src + (size_t)r * J + 4 * q;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(reinterpret_cast<float4*>(dst) + t)),
                     "l"(g)
                     : "memory");
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else {
    for (int t = threadIdx.x; t < rows * kFftJS; t += kFftThreads) {
      const int r = t / kFftJS, c = t % kFftJS;
      dst[t] = (c < ncol) ? src[(size_t)r * J + c] : 0.f;
    }
  }
}

// Fourier coefficients F[b][row][j] -> nodal[b][i][j] (optionally scaled by
// wq[j], which gives the adjoint of the weighted forward transform).
// Z[k] = (X[k] + conj X[N-k]) + i w_I^k (X[k] - conj X[N-k]), then
// z = IDFT_N(Z) and x[2n] = Re z[n], x[2n+1] = Im z[n].  The coefficient tile
// (at most 2N - 1 rows of kFftJS floats) is staged in the shared buffer, Z is
// formed in registers in two halves and written back over it, the passes run
// in place and a per-column copy writes the nodal rows.  Up to N = 256 the
// kernel fits 48 registers, so five CTAs (36 KB of shared memory each) share
// an SM.
template <int N>
__global__ void __launch_bounds__(kFftThreads, N <= 256 ? 5 : 3)
rfft_inverse_kernel(const float* __restrict__ F, float* __restrict__ out,
                    int M, int lw, int J, const float2* __restrict__ tw_n,
                    const float2* __restrict__ tw_i,
                    const float* __restrict__ wq) {
  extern __shared__ float2 sm[];
  float2* S = sm;
  float2* twn = S + N * kFftJS;
  float2* twi = twn + N;
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int j0 = blockIdx.x * kFftJS;
  const int ncol = min(kFftJS, J - j0);
  for (int t = tid; t < N; t += kFftThreads) {
    twn[t] = tw_n[t];
    twi[t] = tw_i[t];
  }
  const float* Fb = F + (size_t)b * M * J + j0;
  const int rows = min(M, 2 * min(lw, N) - 1);  // rows X() reads; <= 2N - 1
  const float* src = reinterpret_cast<const float*>(S);
  stage_tile<2 * N>(Fb, rows, J, ncol, reinterpret_cast<float*>(S));
  __syncthreads();
  const float inv_sqrt_2pi = 0.3989422804014327f;
  const float half_inv_sqrt_pi = 0.28209479177387814f;
  auto X = [&](int k, int c) -> float2 {
    if (c >= ncol || k >= lw || k >= N) return make_float2(0.f, 0.f);
    if (k == 0) return make_float2(src[c] * inv_sqrt_2pi, 0.f);
    return make_float2(src[(2 * k - 1) * kFftJS + c] * half_inv_sqrt_pi,
                       -src[(2 * k) * kFftJS + c] * half_inv_sqrt_pi);
  };
  // Pairs (k, N - k), k = 0..N/2; k = 0 pairs with the (zero) Nyquist term.
  // A thread keeps one column (c = tid mod kFftJS) and takes
  // k = tid / kFftJS + kRowsPerPass * it.  Z[k] overwrites the staged rows
  // 2k and 2k + 1 and Z[N - k] the rows 2(N - k) and 2(N - k) + 1, so the
  // items run in two halves (k < kSplit, then the rest), each loading all of
  // its X before any of its Z is written: the first half's Z rows are ones
  // that the second half no longer reads, except row 2 kSplit - 1 of
  // Z[kSplit - 1], which is written after the second half's loads.  Half
  // the X values are live at a time.
  constexpr int kRowsPerPass = kFftThreads / kFftJS;
  constexpr int kItems = (N / 2 + 1 + kRowsPerPass - 1) / kRowsPerPass;
  constexpr int kItA = kItems / 2;
  constexpr int kSplit = kItA * kRowsPerPass;
  const int cz = tid % kFftJS, k0 = tid / kFftJS;
  auto z_pair = [&](int k, float2 xk, float2 xn, bool write_k) {
    const float2 xnc = cconj(xn), xkc = cconj(xk);
    const float2 zk = cadd(cadd(xk, xnc), cmul_i<1>(cmul(twi[k], csub(xk, xnc))));
    if (write_k) S[k * kFftJS + cz] = zk;
    if (k > 0 && k < N / 2 + (N & 1)) {
      const int kn = N - k;
      S[kn * kFftJS + cz] =
          cadd(cadd(xn, xkc), cmul_i<1>(cmul(twi[kn], csub(xn, xkc))));
    }
    return zk;
  };
  float2 held = make_float2(0.f, 0.f);  // Z[kSplit - 1], written last
  bool hold = false;
  if constexpr (kItA > 0) {
    float2 xk[kItA], xn[kItA];
#pragma unroll
    for (int it = 0; it < kItA; ++it) {
      const int k = k0 + it * kRowsPerPass;
      xk[it] = X(k, cz);
      xn[it] = (k == 0) ? make_float2(0.f, 0.f) : X(N - k, cz);
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kItA; ++it) {
      const int k = k0 + it * kRowsPerPass;
      const bool last_row = (k == kSplit - 1);
      const float2 zk = z_pair(k, xk[it], xn[it], !last_row);
      if (last_row) {
        held = zk;
        hold = true;
      }
    }
  }
  {
    constexpr int kItB = kItems - kItA;
    float2 xk[kItB], xn[kItB];
#pragma unroll
    for (int it = 0; it < kItB; ++it) {
      const int k = kSplit + k0 + it * kRowsPerPass;
      if (k <= N / 2) {
        xk[it] = X(k, cz);
        xn[it] = (k == 0) ? make_float2(0.f, 0.f) : X(N - k, cz);
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kItB; ++it) {
      const int k = kSplit + k0 + it * kRowsPerPass;
      if (k <= N / 2) z_pair(k, xk[it], xn[it], true);
    }
    if (hold) S[(kSplit - 1) * kFftJS + cz] = held;
  }
  __syncthreads();
  float* ob = out + (size_t)b * (2 * N) * J + j0;
  auto first = [S](int n, int c) { return S[n * kFftJS + c]; };
  // The last pass writes z back into S; then each thread copies its column
  // (c = tid mod kFftJS, the same in every pass) out as rows 2n (Re z[n])
  // and 2n + 1 (Im z[n]) with its weight read once.  Keeping the global
  // stores out of the pass keeps its register count down.
  auto last = [S](int n, int c, float2 v) { S[n * kFftJS + c] = v; };
  fft_passes<N, 1, true, true>(S, twn, first, last);
  __syncthreads();
  const int cth = tid % kFftJS;
  if (cth < ncol) {
    const float sc = wq ? wq[j0 + cth] : 1.f;
    float* oc = ob + cth;
    for (int n = tid / kFftJS; n < N; n += kFftThreads / kFftJS) {
      const float2 v = S[n * kFftJS + cth];
      oc[2 * n * J] = v.x * sc;
      oc[(2 * n + 1) * J] = v.y * sc;
    }
  }
}

// nodal[b][i][j] -> F[b][row][j] (times wq[j] when given: the forward SHT's
// quadrature weights; without: the adjoint of the inverse transform).
template <int N>
__global__ void __launch_bounds__(kFftThreads)
rfft_forward_kernel(const float* __restrict__ x, float* __restrict__ F, int M,
                    int lw, int J, const float2* __restrict__ tw_n,
                    const float2* __restrict__ tw_i,
                    const float* __restrict__ wq) {
  extern __shared__ float2 sm[];
  float2* S = sm;
  float2* twn = S + N * kFftJS;
  float2* twi = twn + N;
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int j0 = blockIdx.x * kFftJS;
  const int ncol = min(kFftJS, J - j0);
  for (int t = tid; t < N; t += kFftThreads) {
    twn[t] = tw_n[t];
    twi[t] = tw_i[t];
  }
  const float* xb = x + (size_t)b * (2 * N) * J + j0;
  // The nodal tile (2N rows of kFftJS floats) is staged by asynchronous
  // copies; the first pass reads it in place.
  stage_tile<2 * N>(xb, 2 * N, J, ncol, reinterpret_cast<float*>(S));
  __syncthreads();
  const float* Sf = reinterpret_cast<const float*>(S);
  auto first = [Sf](int n, int c) {
    return make_float2(Sf[2 * n * kFftJS + c], Sf[(2 * n + 1) * kFftJS + c]);
  };
  auto last = [S](int n, int c, float2 v) { S[n * kFftJS + c] = v; };
  fft_passes<N, -1, true>(S, twn, first, last);
  __syncthreads();
  float* Fb = F + (size_t)b * M * J + j0;
  const float inv_sqrt_2pi = 0.3989422804014327f;
  const float inv_sqrt_pi = 0.5641895835477563f;
  // X[k] and X[N - k] from the same two values of Z: with
  // s = (Z[k] + conj Z[N-k]) / 2 and d = (Z[k] - conj Z[N-k]) / 2,
  // X[k] = s + e^{-2 pi i k / I} (-i d), and X[N-k] likewise with Z[k] and
  // Z[N-k] exchanged.  A thread keeps one column (c = tid mod kFftJS) and
  // takes k = tid / kFftJS + kFftJS q for k <= N / 2.
  const int c = tid % kFftJS;
  if (c < ncol) {
    const float w = wq ? wq[j0 + c] : 1.f;
    const float a0 = w * inv_sqrt_2pi, a1 = w * inv_sqrt_pi;
    float* Fc = Fb + c;
    for (int k = tid / kFftJS; k <= N / 2; k += kFftThreads / kFftJS) {
      const int kn = (N - k) & (N - 1);  // N - k; 0 for k = 0
      const float2 zk = S[k * kFftJS + c];
      const float2 zn = S[kn * kFftJS + c];
      if (k < lw) {
        const float2 zc = cconj(zn);
        const float2 s2 = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
        const float2 d2 = make_float2(0.5f * (zk.x - zc.x), 0.5f * (zk.y - zc.y));
        const float2 xk = cadd(s2, cmul(cconj(twi[k]), cmul_i<-1>(d2)));
        if (k == 0) {
          Fc[0] = xk.x * a0;
        } else {
          Fc[(2 * k - 1) * J] = xk.x * a1;
          Fc[2 * k * J] = -xk.y * a1;
        }
      }
      if (k > 0 && k < N / 2 && kn < lw) {
        const float2 zc = cconj(zk);
        const float2 s2 = make_float2(0.5f * (zn.x + zc.x), 0.5f * (zn.y + zc.y));
        const float2 d2 = make_float2(0.5f * (zn.x - zc.x), 0.5f * (zn.y - zc.y));
        const float2 xn = cadd(s2, cmul(cconj(twi[kn]), cmul_i<-1>(d2)));
        Fc[(2 * kn - 1) * J] = xn.x * a1;
        Fc[2 * kn * J] = -xn.y * a1;
      }
    }
  }
}

// Generic longitude transforms by direct summation with the FP32 real basis
// f[i][row] (any I, any lw <= I).
__global__ void dft_inverse_kernel(const float* __restrict__ F,
                                   float* __restrict__ out, int M, int I, int J,
                                   const float* __restrict__ f,
                                   const float* __restrict__ wq) {
  int j = blockIdx.x * 32 + threadIdx.x;
  int i = blockIdx.y * 8 + threadIdx.y;
  int b = blockIdx.z;
  if (j >= J || i >= I) return;
  const float* Fb = F + (size_t)b * M * J + j;
  const float* fi = f + (size_t)i * M;
  float acc = 0.f;
  for (int r = 0; r < M; ++r) acc = fmaf(fi[r], Fb[(size_t)r * J], acc);
  if (wq) acc *= wq[j];
  out[((size_t)b * I + i) * J + j] = acc;
}

__global__ void dft_forward_kernel(const float* __restrict__ x,
                                   float* __restrict__ F, int M, int I, int J,
                                   const float* __restrict__ f,
                                   const float* __restrict__ wq) {
  int j = blockIdx.x * 32 + threadIdx.x;
  int r = blockIdx.y * 8 + threadIdx.y;
  int b = blockIdx.z;
  if (j >= J || r >= M) return;
  const float* xb = x + (size_t)b * I * J + j;
  float acc = 0.f;
  for (int i = 0; i < I; ++i) acc = fmaf(f[(size_t)i * M + r], xb[(size_t)i * J], acc);
  if (wq) acc *= wq[j];
  F[((size_t)b * M + r) * J + j] = acc;
}

template <int N>
static int configure_rfft() {
  // Kernel attributes are set once per device, outside any stream capture
  // (sht_prepare runs this at plan creation on the plan's device).
  static PerDeviceOnce once;
  return once.run([] {
    const int smem = (int)fft_smem_bytes<N>();
    DINO_CHECK_CUDA(cudaFuncSetAttribute(rfft_inverse_kernel<N>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    DINO_CHECK_CUDA(cudaFuncSetAttribute(rfft_forward_kernel<N>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return DINO_OK;
  });
}

template <int N>
static int launch_rfft(dino_plan* p, const float* in, float* out, int nf,
                       bool inverse, const float* wq, cudaStream_t st) {
  const size_t smem = fft_smem_bytes<N>();
  if (!p) return configure_rfft<N>();
  DINO_TRY(configure_rfft<N>());
  dim3 grid(ceil_div(p->J, kFftJS), nf);
  if (inverse) {
    rfft_inverse_kernel<N><<<grid, kFftThreads, smem, st>>>(
        in, out, p->M, p->lw, p->J, p->d_tw_n, p->d_tw_i, wq);
    return check_launch("rfft_inverse");
  }
  rfft_forward_kernel<N><<<grid, kFftThreads, smem, st>>>(
      in, out, p->M, p->lw, p->J, p->d_tw_n, p->d_tw_i, wq);
  return check_launch("rfft_forward");
}

static int rfft_dispatch_n(int n, dino_plan* p, const float* in, float* out,
                           int nf, bool inverse, const float* wq,
                           cudaStream_t st) {
  switch (n) {
    case 8: return launch_rfft<8>(p, in, out, nf, inverse, wq, st);
    case 16: return launch_rfft<16>(p, in, out, nf, inverse, wq, st);
    case 32: return launch_rfft<32>(p, in, out, nf, inverse, wq, st);
    case 64: return launch_rfft<64>(p, in, out, nf, inverse, wq, st);
    case 128: return launch_rfft<128>(p, in, out, nf, inverse, wq, st);
    case 256: return launch_rfft<256>(p, in, out, nf, inverse, wq, st);
    case 512: return launch_rfft<512>(p, in, out, nf, inverse, wq, st);
  }
  set_error("internal: unsupported FFT length");
  return DINO_ERR_UNSUPPORTED;
}

static int rfft_dispatch(dino_plan* p, const float* in, float* out, int nf,
                         bool inverse, const float* wq, cudaStream_t st) {
  return rfft_dispatch_n(p->N, p, in, out, nf, inverse, wq, st);
}

int sht_prepare(dino_plan* p) {
  if (!p->fft_pow2) return DINO_OK;
  return rfft_dispatch_n(p->N, nullptr, nullptr, nullptr, 0, true, nullptr, 0);
}

int fourier_inverse(dino_plan* p, const float* F, float* nodal, int nf,
                    bool weighted_adjoint, cudaStream_t st) {
  NvtxRange range("inv_fourier");
  const float* wq = weighted_adjoint ? p->d_wq : nullptr;
  if (p->fft_pow2) return rfft_dispatch(p, F, nodal, nf, true, wq, st);
  dim3 grid(ceil_div(p->J, 32), ceil_div(p->I, 8), nf);
  dft_inverse_kernel<<<grid, dim3(32, 8), 0, st>>>(F, nodal, p->M, p->I, p->J,
                                                    p->d_fbasis, wq);
  return check_launch("dft_inverse");
}

int fourier_forward(dino_plan* p, const float* nodal, float* F, int nf,
                    bool weighted, cudaStream_t st) {
  NvtxRange range("fwd_fourier");
  const float* wq = weighted ? p->d_wq : nullptr;
  if (p->fft_pow2) return rfft_dispatch(p, nodal, F, nf, false, wq, st);
  dim3 grid(ceil_div(p->J, 32), ceil_div(p->M, 8), nf);
  dft_forward_kernel<<<grid, dim3(32, 8), 0, st>>>(nodal, F, p->M, p->I, p->J,
                                                    p->d_fbasis, wq);
  return check_launch("dft_forward");
}

// ---------------------------------------------------------------------------
// Transform drivers (chunked by workspace capacity)
// ---------------------------------------------------------------------------

// Fields per launch such that the intermediate Fourier coefficients of one
// chunk (fields x M x J floats) stay resident in L2 between the Legendre and
// FFT kernels; chunks are balanced, and on the tensor-core path whole
// 128-row MMA tiles (64 fields) where the cap allows.
int l2_chunk(dino_plan* p, int nf, int work_fields) {
  const size_t per_field = (size_t)p->M * p->J * sizeof(float);
  int cap = (int)((48ull << 20) / (per_field ? per_field : 1));
  if (cap < 1) cap = 1;
  if (cap > work_fields) cap = work_fields;
  if (p->precision != DINO_PREC_FP32 && cap >= 64) {
    cap = cap / 64 * 64;
    const int chunks = (nf + cap - 1) / cap;
    const int even = (nf + chunks - 1) / chunks;
    return std::min(cap, (even + 63) / 64 * 64);
  }
  const int chunks = (nf + cap - 1) / cap;
  return (nf + chunks - 1) / chunks;
}

// Chunks alternate between the caller's stream and the plan's side stream
// when two of them fit in the workspace: each stream has its own half, both
// chunks' intermediates stay in L2, and one chunk's kernels fill the SMs the
// other leaves idle in its waves' tails.  The side stream forks from and joins back into the
// caller's stream with events, so the pattern also records into CUDA graphs.
struct ChunkRun {
  dino_plan* p;
  cudaStream_t st;
  float* work;
  size_t work_stride;  // floats per half
  bool dual = false;

  ChunkRun(dino_plan* p_, cudaStream_t st_, float* work_, int chunk, int nf,
           int work_fields)
      : p(p_), st(st_), work(work_), work_stride((size_t)chunk * p_->M * p_->J) {
    dual = p->side && nf > chunk && 2 * chunk <= work_fields;
  }
  int begin() {
    if (!dual) return DINO_OK;
    DINO_CHECK_CUDA(cudaEventRecord(p->ev_fork, st));
    DINO_CHECK_CUDA(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    return DINO_OK;
  }
  int slot(int c) const { return dual ? (c & 1) : -1; }
  cudaStream_t stream(int c) const { return slot(c) == 1 ? p->side : st; }
  float* buf(int c) const { return work + (slot(c) == 1 ? work_stride : 0); }
  int end() {
    if (!dual) return DINO_OK;
    DINO_CHECK_CUDA(cudaEventRecord(p->ev_join, p->side));
    DINO_CHECK_CUDA(cudaStreamWaitEvent(st, p->ev_join, 0));
    return DINO_OK;
  }
};

int sht_inverse_segs(dino_plan* p, const Segs& in, float* out, int nf,
                     float* work, int work_fields, cudaStream_t st) {
  const size_t ms = (size_t)p->M * p->L, ns = (size_t)p->I * p->J;
  const int chunk = l2_chunk(p, nf, work_fields);
  ChunkRun run(p, st, work, chunk, nf, work_fields);
  DINO_TRY(run.begin());
  for (int c = 0, f0 = 0; f0 < nf; ++c, f0 += chunk) {
    int n = nf - f0 < chunk ? nf - f0 : chunk;
    Segs sub = seg_offset(in, f0, n, ms);
    DINO_TRY(legendre_inverse(p, sub, run.buf(c), n, run.stream(c)));
    DINO_TRY(fourier_inverse(p, run.buf(c), out + f0 * ns, n, false, run.stream(c)));
  }
  return run.end();
}

int sht_forward_to(dino_plan* p, const float* nodal, float* out, int nf,
                   float* work, int work_fields, cudaStream_t st) {
  const size_t ms = (size_t)p->M * p->L, ns = (size_t)p->I * p->J;
  const int chunk = l2_chunk(p, nf, work_fields);
  ChunkRun run(p, st, work, chunk, nf, work_fields);
  DINO_TRY(run.begin());
  for (int c = 0, f0 = 0; f0 < nf; ++c, f0 += chunk) {
    int n = nf - f0 < chunk ? nf - f0 : chunk;
    DINO_TRY(fourier_forward(p, nodal + f0 * ns, run.buf(c), n, true, run.stream(c)));
    DINO_TRY(legendre_forward(p, run.buf(c), out + f0 * ms, n, run.stream(c)));
  }
  return run.end();
}

// Adjoint of the inverse transform: unweighted forward Fourier, then the
// forward contraction.  Adjoint of the forward transform: the inverse
// contraction, then the inverse Fourier synthesis scaled by w[j].  Chunked
// like the transforms themselves (work holds work_fields x M x J floats).
int sht_inverse_adjoint_to(dino_plan* p, const float* nodal_ct, float* modal_ct,
                           int nf, float* work, int work_fields, cudaStream_t st) {
  const size_t ms = (size_t)p->M * p->L, ns = (size_t)p->I * p->J;
  const int chunk = l2_chunk(p, nf, work_fields);
  ChunkRun run(p, st, work, chunk, nf, work_fields);
  DINO_TRY(run.begin());
  for (int c = 0, f0 = 0; f0 < nf; ++c, f0 += chunk) {
    int n = nf - f0 < chunk ? nf - f0 : chunk;
    DINO_TRY(fourier_forward(p, nodal_ct + f0 * ns, run.buf(c), n, false, run.stream(c)));
    DINO_TRY(legendre_forward(p, run.buf(c), modal_ct + f0 * ms, n, run.stream(c)));
  }
  return run.end();
}

int sht_forward_adjoint_to(dino_plan* p, const float* modal_ct, float* nodal_ct,
                           int nf, float* work, int work_fields, cudaStream_t st) {
  const size_t ms = (size_t)p->M * p->L, ns = (size_t)p->I * p->J;
  const int chunk = l2_chunk(p, nf, work_fields);
  ChunkRun run(p, st, work, chunk, nf, work_fields);
  DINO_TRY(run.begin());
  for (int c = 0, f0 = 0; f0 < nf; ++c, f0 += chunk) {
    int n = nf - f0 < chunk ? nf - f0 : chunk;
    DINO_TRY(legendre_inverse(p, one_seg(modal_ct + f0 * ms, n), run.buf(c), n,
                              run.stream(c)));
    DINO_TRY(fourier_inverse(p, run.buf(c), nodal_ct + f0 * ns, n, true, run.stream(c)));
  }
  return run.end();
}

static int sht_inverse_adjoint(dino_plan* p, const float* nodal_ct,
                               float* modal_ct, int nf, cudaStream_t st) {
  return sht_inverse_adjoint_to(p, nodal_ct, modal_ct, nf, p->d_work,
                                p->max_fields, st);
}

static int sht_forward_adjoint(dino_plan* p, const float* modal_ct,
                               float* nodal_ct, int nf, cudaStream_t st) {
  return sht_forward_adjoint_to(p, modal_ct, nodal_ct, nf, p->d_work,
                                p->max_fields, st);
}

// ---------------------------------------------------------------------------
// FastSphericalHarmonics modal layout (spherical_harmonic.py:411-621)
// ---------------------------------------------------------------------------

// Rows of the Fast layout are m = 0, 0 (imaginary, always zero), 1, -1, 2,
// -2, ... (:486-497): the Real layout [M = 2 lw - 1][L] with a zero row
// inserted at index 1.  to_fast: [M][L] -> [M + 1][L]; else the inverse
// (which drops row 1).
__global__ void modal_relayout_kernel(const float* __restrict__ in,
                                      float* __restrict__ out, int M, int L,
                                      int to_fast) {
  const int rows_in = to_fast ? M : M + 1, rows_out = to_fast ? M + 1 : M;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)rows_out * L) return;
  const int r = idx / L, l = idx % L;
  const float* src = in + (size_t)blockIdx.y * rows_in * L;
  float v;
  if (to_fast)
    v = (r == 0) ? src[l] : (r == 1 ? 0.f : src[(size_t)(r - 1) * L + l]);
  else
    v = src[(size_t)(r == 0 ? 0 : r + 1) * L + l];
  out[(size_t)blockIdx.y * rows_out * L + idx] = v;
}

int modal_relayout(dino_plan* p, bool to_fast, const float* in, float* out, int nf,
                   cudaStream_t st) {
  const int rows_out = to_fast ? p->M + 1 : p->M;
  dim3 grid(ceil_div(rows_out * p->L, 256), nf);
  modal_relayout_kernel<<<grid, 256, 0, st>>>(in, out, p->M, p->L, to_fast ? 1 : 0);
  return check_launch("modal_relayout");
}

// ---------------------------------------------------------------------------
// Spectral operators (spherical_harmonic.py:1033-1102)
// ---------------------------------------------------------------------------

// Spectral operators; `transpose` applies the transposed (adjoint) map.
// cos_lat_d_dlat: out[l] = ta[l+1] x[l+1] + tb[l-1] x[l-1]
//   transpose:    out[l] = ta[l] x[l-1] + tb[l] x[l+1]
// d_dlon is antisymmetric; the Laplacians and the clip are diagonal.
__global__ void modal_op_kernel(int op, int transpose,
                                const float* __restrict__ in,
                                float* __restrict__ out, int nf, int M, int L,
                                int lw, const float* __restrict__ deriv,
                                const float* __restrict__ lap,
                                const float* __restrict__ invlap, int clip_n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)nf * M * L;
  if (idx >= total) return;
  int l = idx % L;
  int row = (idx / L) % M;
  size_t base = idx - l - (size_t)row * L;  // start of this field
  int m = (row + 1) / 2;
  const float* x = in + base;
  float v = 0.f;
  switch (op) {
    case DINO_OP_D_DLON: {
      float s = transpose ? -1.f : 1.f;
      if (row == 0) v = 0.f;
      else if (row & 1) v = s * m * x[(size_t)(row + 1) * L + l];
      else v = -s * m * x[(size_t)(row - 1) * L + l];
      break;
    }
    case DINO_OP_COS_LAT_D_DLAT:
    case DINO_OP_SEC_LAT_D_DLAT_COS2: {
      const float* ta = deriv + (op == DINO_OP_COS_LAT_D_DLAT ? 0 : 2) * (size_t)lw * L;
      const float* tb = ta + (size_t)lw * L;
      const float* xr = x + (size_t)row * L;
      const float* tam = ta + (size_t)m * L;
      const float* tbm = tb + (size_t)m * L;
      if (!transpose) {
        if (l + 1 < L) v += tam[l + 1] * xr[l + 1];
        if (l >= 1) v += tbm[l - 1] * xr[l - 1];
      } else {
        if (l >= 1) v += tam[l] * xr[l - 1];
        if (l + 1 < L) v += tbm[l] * xr[l + 1];
      }
      break;
    }
    case DINO_OP_LAPLACIAN:
      v = x[(size_t)row * L + l] * lap[l];
      break;
    case DINO_OP_INVERSE_LAPLACIAN:
      v = x[(size_t)row * L + l] * invlap[l];
      break;
    case DINO_OP_CLIP:
      v = (l < L - clip_n) ? x[(size_t)row * L + l] : 0.f;
      break;
  }
  out[idx] = v;
}

int modal_op(dino_plan* p, int op, const float* in, float* out, int nf, int arg,
             cudaStream_t st) {
  const int transpose = (op & 8) ? 1 : 0;
  op &= 7;
  DINO_REQUIRE(op >= DINO_OP_D_DLON && op <= DINO_OP_CLIP, DINO_ERR_ARG,
               "unknown modal operator");
  DINO_REQUIRE(op != DINO_OP_CLIP || arg > 0, DINO_ERR_ARG,
               "`n` must be >= 0");
  DINO_REQUIRE(in != out, DINO_ERR_ARG, "modal_op: in and out must differ");
  size_t total = (size_t)nf * p->M * p->L;
  if (total == 0) return DINO_OK;
  modal_op_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
      op, transpose, in, out, nf, p->M, p->L, p->lw, p->d_deriv, p->d_lap,
      p->d_invlap, arg);
  return check_launch("modal_op");
}

}  // namespace dino

using namespace dino;

extern "C" {

int dino_sht_inverse(dino_plan* p, const float* modal, float* nodal, int32_t nf,
                     void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_sht_inverse: null plan");
  DINO_REQUIRE(nf >= 0, DINO_ERR_SHAPE, "nfields must be >= 0");
  if (nf == 0) return DINO_OK;  // buffers may be null for an empty batch
  DINO_REQUIRE(modal && nodal, DINO_ERR_ARG, "dino_sht_inverse: null argument");
  return sht_inverse_segs(p, one_seg(modal, nf), nodal, nf, p->d_work,
                          p->max_fields, (cudaStream_t)stream);
}

int dino_sht_forward(dino_plan* p, const float* nodal, float* modal, int32_t nf,
                     void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_sht_forward: null plan");
  DINO_REQUIRE(nf >= 0, DINO_ERR_SHAPE, "nfields must be >= 0");
  if (nf == 0) return DINO_OK;
  DINO_REQUIRE(modal && nodal, DINO_ERR_ARG, "dino_sht_forward: null argument");
  return sht_forward_to(p, nodal, modal, nf, p->d_work, p->max_fields,
                        (cudaStream_t)stream);
}

int dino_sht_inverse_adjoint(dino_plan* p, const float* nodal_ct,
                             float* modal_ct, int32_t nf, void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "null plan");
  DINO_REQUIRE(nf >= 0, DINO_ERR_SHAPE, "nfields must be >= 0");
  if (nf == 0) return DINO_OK;
  DINO_REQUIRE(nodal_ct && modal_ct, DINO_ERR_ARG, "null argument");
  return sht_inverse_adjoint(p, nodal_ct, modal_ct, nf, (cudaStream_t)stream);
}

int dino_sht_forward_adjoint(dino_plan* p, const float* modal_ct,
                             float* nodal_ct, int32_t nf, void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "null plan");
  DINO_REQUIRE(nf >= 0, DINO_ERR_SHAPE, "nfields must be >= 0");
  if (nf == 0) return DINO_OK;
  DINO_REQUIRE(nodal_ct && modal_ct, DINO_ERR_ARG, "null argument");
  return sht_forward_adjoint(p, modal_ct, nodal_ct, nf, (cudaStream_t)stream);
}

int dino_sht_phase(dino_plan* p, int32_t phase, const float* in, float* out,
                   int32_t nf, void* stream) {
  DINO_REQUIRE(p && in && out, DINO_ERR_ARG, "dino_sht_phase: null argument");
  DINO_REQUIRE(nf >= 0 && nf <= p->max_fields, DINO_ERR_SHAPE,
               "nfields must be in [0, max_fields]");
  if (nf == 0) return DINO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  switch (phase) {
    case DINO_PHASE_LEGENDRE_INVERSE:
      return legendre_inverse(p, one_seg(in, nf), out, nf, st);
    case DINO_PHASE_FOURIER_INVERSE:
      return fourier_inverse(p, in, out, nf, false, st);
    case DINO_PHASE_FOURIER_FORWARD:
      return fourier_forward(p, in, out, nf, true, st);
    case DINO_PHASE_LEGENDRE_FORWARD:
      return legendre_forward(p, in, out, nf, st);
  }
  set_error("unknown transform phase");
  return DINO_ERR_ARG;
}

int dino_modal_op(dino_plan* p, int32_t op, const float* in, float* out,
                  int32_t nf, int32_t arg, void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_modal_op: null plan");
  DINO_REQUIRE(nf >= 0, DINO_ERR_SHAPE, "nfields must be >= 0");
  if (nf == 0) return DINO_OK;
  DINO_REQUIRE(in && out, DINO_ERR_ARG, "dino_modal_op: null argument");
  return modal_op(p, op, in, out, nf, arg, (cudaStream_t)stream);
}

int dino_modal_relayout(dino_plan* p, int32_t to_fast, const float* in, float* out,
                        int32_t nfields, void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_modal_relayout: null plan");
  DINO_REQUIRE(nfields >= 0 && nfields <= 65535, DINO_ERR_SHAPE, "nfields out of range");
  if (nfields == 0) return DINO_OK;
  DINO_REQUIRE(in && out, DINO_ERR_ARG, "dino_modal_relayout: null argument");
  DINO_REQUIRE(in != out, DINO_ERR_ARG, "dino_modal_relayout: in and out must differ");
  return modal_relayout(p, to_fast != 0, in, out, nfields, (cudaStream_t)stream);
}

}  // extern "C"
