// Primitive equations on sigma levels: explicit tendencies, implicit terms,
// implicit inverse and the imex_rk_sil3 step with a per-l step filter.
//
// Follows PrimitiveEquationsSigma (dinosaur/primitive_equations.py:835-1458),
// compute_diagnostic_state_sigma (:168-225), HeldSuarezForcingSigma
// (dinosaur/held_suarez.py:47-167), imex_runge_kutta / imex_rk_sil3
// (dinosaur/time_integration.py:329-405) and the exponential step filter
// (:427-455).  Data stays in HBM in the packed, kind-major state layout
// described in include/dino_b200.h; one explicit evaluation is
//   modal pre-pass -> inverse SHT -> fused nodal column kernel ->
//   forward SHT -> modal post-pass,
// and each RK stage is an elementwise combine over all planes plus one
// per-(m, l) kernel for the implicit solve, the implicit terms of the
// solution, the final combination and the filter.

#include <cmath>
#include <cstring>
#include <deque>
#include <initializer_list>
#include <vector>

#include "dino_internal.cuh"

namespace dino {

constexpr int kMaxTracers = 4;

// ---------------------------------------------------------------------------
// Object
// ---------------------------------------------------------------------------

// One per-l operator of the implicit part (see pe_matrix_build_kernel).
struct MatEntry {
  int kind = 0;
  double eta = 0;
  std::vector<double> filter;  // folded-in step filter (kMatFinal), else empty
  bool transposed = false;     // the transpose of the operator of `kind`
  float* d = nullptr;          // [L][nin][RP]: operator^T, rows zero-padded
  int R = 0, nin = 0, RP = 0;  // rows, columns (inputs), padded rows
};

struct FilterCacheEntry {
  std::vector<double> host;
  float* d_filter;
};

struct GraphEntry {
  float* state = nullptr;
  double dt = 0;
  float* filter = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

}  // namespace dino

struct dino_pe {
  dino_plan* plan = nullptr;
  int K = 0, mem = 0, nT = 0, hum = -1, vadv = 1, hs = 0, tref_varies = 0;
  int M = 0, L = 0, I = 0, J = 0;
  size_t ML = 0, IJ = 0;
  double R = 0, Rv = 0, Cpv = 0, kappa = 0, g = 0, Omega = 0;
  double hs_p0 = 0, hs_sigma_b = 0, hs_kf = 0, hs_ka = 0, hs_ks = 0,
         hs_minT = 0, hs_maxT = 0, hs_dTy = 0, hs_dThz = 0;
  // Host copies (FP64).
  std::vector<double> dsig, c2c, alpha, tref, sumsig, sigma, G, H;
  // The implicit operator's ln ps column and ln ps row: R T_ref and the
  // sigma thickness on sigma levels; on hybrid levels the Simmons-Burridge
  // pressure-gradient coefficient and da / p_s_ref + db at p_s_ref.
  std::vector<double> imp_col, imp_row;
  // Hybrid sigma-pressure levels (vertical_scheme 1).
  int hybrid = 0, hum_hyb = -1;
  double ps_ref = 0;
  float* d_hyb = nullptr;  // per-level constants of pe_nodal_hybrid_kernel
  // Device constants.
  float* d_levpack = nullptr;  // per-level constants, packed per level (kLevPack)
  int sms = 148;               // multiprocessors of the device
  float* d_lat = nullptr;   // per-latitude constants: sec2, f, sin2, cos2
  float* d_orog = nullptr;  // modal orography [M][L]
  // Field bookkeeping (planes).
  int n_state = 0, n_inv = 0, n_fwd = 0, n_aux = 0;
  // Plane bases inside the nodal buffer / forward buffers.
  int p_u = 0, p_v = 0, p_gqx = 0, p_gqy = 0, p_gx = 0, p_gy = 0,
      p_laplnps = 0, p_lnps = 0;
  int o_Au = 0, o_Av = 0, o_KE = 0, o_uT = 0, o_vT = 0, o_Tn = 0, o_tr = 0,
      o_vh = 0, o_gh = 0, o_dh = 0, o_hsT = 0, o_lnps = 0;
  // Work buffers.
  float* d_aux = nullptr;
  float* d_nodal = nullptr;
  float* d_fwd_in = nullptr;
  float* d_fwd_out = nullptr;
  float* d_work = nullptr;
  int work_fields = 0;
  float* d_f[3] = {nullptr, nullptr, nullptr};
  float* d_g[2] = {nullptr, nullptr};
  float* d_Y = nullptr;
  float* d_ystar = nullptr;  // Y* of the current stage (implicit planes)
  // l-major operands of the per-l implicit products: [L][2n][Cp].
  int Cp = 0;
  float* d_lm_in = nullptr;
  float* d_lm_out = nullptr;
  // Adjoint work (allocated by the first VJP call).
  float* d_xbar_n = nullptr;  // nodal cotangents, n_inv planes
  float* d_xbar_m = nullptr;  // their modal adjoint, n_inv planes
  float* d_adj[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int* d_flag = nullptr;
  std::deque<dino::MatEntry> mat_cache;  // stable element addresses
  std::vector<dino::FilterCacheEntry> filter_cache;
  dino::GraphEntry graph;
};

namespace dino {

// Offsets into the host-side per-level arrays (floats) from which the packed
// table (kLevPack) is built; every array has K entries (c2ci and trefdiff
// hold 0 at K - 1).
struct LevOff {
  int dsig, c2ci, alpha, tref, sumsig, sigma, kv, trefdiff, logsp0;
  int total;
};

static LevOff lev_offsets(int K) {
  LevOff o;
  o.dsig = 0;
  o.c2ci = K;
  o.alpha = 2 * K;
  o.tref = 3 * K;
  o.sumsig = 4 * K;
  o.sigma = 5 * K;
  o.kv = 6 * K;
  o.trefdiff = 7 * K;  // (Tref[k+1]-Tref[k]) * c2ci[k]
  o.logsp0 = 8 * K;    // log(sigma_k / p0) (Held-Suarez)
  o.total = 9 * K;
  return o;
}

// Plane index helpers: kind base p, member mb, level k.
__device__ __forceinline__ size_t pl(int p, int mb, int K, int k) {
  return (size_t)p + (size_t)mb * K + k;
}

// ---------------------------------------------------------------------------
// Modal pre-pass: u cos, v cos, cos grad ln ps (+ humidity gradient, lap ln ps)
// (get_cos_lat_vector, spherical_harmonic.py:1164-1178; cos_lat_grad :1104-1111;
//  primitive_equations.py:168-225, :861-963)
// ---------------------------------------------------------------------------

struct PrepArgs {
  const float* state;
  float* aux;
  int K, mem, nT, hum;
  int M, L, lw;
  int p_div, p_vort, p_lnps, p_hum;  // state planes
  int a_u, a_v, a_gqx, a_gqy, a_gx, a_gy, a_laplnps;  // aux planes (-1 = unused)
  // Hybrid levels: ln p_s without its l = 0 coefficient (-1 = unused).
  int a_lnpsdev = -1;
  const float* deriv;
  const float* lap;
  const float* invlap;
  float inv_radius;
};

// The modal-point geometry of (row, l), loaded once and reused for every
// level: the d/dlon partner row and factor, and the cos_lat_d_dlat (tab 0) or
// sec_lat_d_dlat_cos2 (tab 2) recurrence coefficients at l + 1 and l - 1
// (optionally times a per-l scaling s, folded in).
struct ModalNbr {
  int row, l, L;
  int dl_row;
  float dl_fac;
  float a1, b1;  // coefficients of x[l + 1] and x[l - 1] (0 when out of range)

  __device__ ModalNbr(int row_, int l_, int L_, int lw, const float* deriv, int tab,
                      const float* s)
      : row(row_), l(l_), L(L_) {
    const int m = (row + 1) >> 1;
    if (row == 0) {
      dl_row = 0;
      dl_fac = 0.f;
    } else if (row & 1) {
      dl_row = row + 1;
      dl_fac = (float)m;
    } else {
      dl_row = row - 1;
      dl_fac = -(float)m;
    }
    const float* ta = deriv + (size_t)tab * lw * L + (size_t)m * L;
    const float* tb = ta + (size_t)lw * L;
    a1 = (l + 1 < L) ? ta[l + 1] * (s ? s[l + 1] : 1.f) : 0.f;
    b1 = (l >= 1) ? tb[l - 1] * (s ? s[l - 1] : 1.f) : 0.f;
  }
  __device__ float dlon(const float* x) const {
    return dl_fac * x[(size_t)dl_row * L + l];
  }
  __device__ float dlat(const float* x) const {
    const float* xr = x + (size_t)row * L + l;
    float v = 0.f;
    if (l + 1 < L) v += a1 * xr[1];
    if (l >= 1) v += b1 * xr[-1];
    return v;
  }
};

// Threads cover (row, l) with l fastest; each walks kPlanesPerThread of the
// (member, level) planes, reusing its operator coefficients.
constexpr int kModalTX = 32, kModalTY = 8, kPlanesPerThread = 8;

__global__ void __launch_bounds__(kModalTX * kModalTY) pe_prep_kernel(PrepArgs a) {
  const int l = blockIdx.x * kModalTX + threadIdx.x;
  const int row = blockIdx.y * kModalTY + threadIdx.y;
  if (l >= a.L || row >= a.M) return;
  const size_t ML = (size_t)a.M * a.L;
  const size_t idx = (size_t)row * a.L + l;
  const float ir = a.inv_radius;
  // u, v from vorticity / divergence through the inverse Laplacian (scaled
  // coefficients); unscaled ones for the humidity and ln ps gradients.
  const ModalNbr ns(row, l, a.L, a.lw, a.deriv, 0, a.invlap);
  const ModalNbr nu(row, l, a.L, a.lw, a.deriv, 0, nullptr);
  const float il = a.invlap[l];
  const int q0 = blockIdx.z * kPlanesPerThread;
  const int q1 = min(q0 + kPlanesPerThread, a.K * a.mem);
  for (int q = q0; q < q1; ++q) {
    const int mb = q / a.K, k = q - mb * a.K;
    const float* vort = a.state + pl(a.p_vort, mb, a.K, k) * ML;
    const float* div = a.state + pl(a.p_div, mb, a.K, k) * ML;
    // psi = lap^-1 vort, chi = lap^-1 div (l = 0 -> 0)
    const float dchi = ns.dlon(div) * il;
    const float dpsi = ns.dlon(vort) * il;
    const float cchi = ns.dlat(div);
    const float cpsi = ns.dlat(vort);
    a.aux[pl(a.a_u, mb, a.K, k) * ML + idx] = (dchi - cpsi) * ir;
    a.aux[pl(a.a_v, mb, a.K, k) * ML + idx] = (cchi + dpsi) * ir;
    if (a.hum >= 0) {
      const float* qh = a.state + pl(a.p_hum, mb, a.K, k) * ML;
      a.aux[pl(a.a_gqx, mb, a.K, k) * ML + idx] = nu.dlon(qh) * ir;
      a.aux[pl(a.a_gqy, mb, a.K, k) * ML + idx] = nu.dlat(qh) * ir;
    }
    if (k == 0) {
      const float* lnps = a.state + ((size_t)a.p_lnps + mb) * ML;
      a.aux[((size_t)a.a_gx + mb) * ML + idx] = nu.dlon(lnps) * ir;
      a.aux[((size_t)a.a_gy + mb) * ML + idx] = nu.dlat(lnps) * ir;
      if (a.hum >= 0)
        a.aux[((size_t)a.a_laplnps + mb) * ML + idx] = lnps[idx] * a.lap[l];
      if (a.a_lnpsdev >= 0)
        a.aux[((size_t)a.a_lnpsdev + mb) * ML + idx] = idx == 0 ? 0.f : lnps[idx];
    }
  }
}

static dim3 modal_grid(int M, int L, int planes) {
  return dim3(ceil_div(L, kModalTX), ceil_div(M, kModalTY),
              ceil_div(planes, kPlanesPerThread));
}

// ---------------------------------------------------------------------------
// Fused nodal column kernel (all explicit nodal products of one evaluation)
// ---------------------------------------------------------------------------

struct NodalArgs {
  const float* nod;
  float* fwd;
  int K, mem, nT, hum, vadv, hs, tref_varies;
  int I, J;
  int p_vort, p_div, p_temp, p_tr, p_u, p_v, p_gqx, p_gqy, p_gx, p_gy,
      p_laplnps, p_lnps;
  int o_Au, o_Av, o_KE, o_uT, o_vT, o_Tn, o_tr, o_vh, o_gh, o_dh, o_hsT,
      o_lnps;
  const float* levpack;  // [K][kLevPack] per-level coefficients
  const float* lat;  // [4][J]: sec2, coriolis, sin^2, cos^2
  float R, kappa, Rv_over_R, Cpv_over_Cp, Rv_minus_R;
  float hs_p0, hs_ka, hs_ks, hs_sigma_b, hs_minT, hs_maxT, hs_dTy, hs_dThz;
};

// Packed per-level coefficients (16 floats, four float4 per level):
//   0 dsig, 1 1/dsig, 2 sumsig, 3 tref,
//   4 c2ci (0 at K-1), 5 c2ci[k-1] (0 at 0), 6 alpha, 7 alpha[k-1] (0 at 0),
//   8 Rayleigh kv, 9 Held-Suarez cutoff, 10 (sigma/p0)^kappa, 11 log(sigma/p0),
//   12 trefdiff (0 at K-1), 13 trefdiff[k-1] (0 at 0), 14-15 unused.
constexpr int kLevPack = 16;

template <int V>
__device__ __forceinline__ void ld_vec(float (&x)[V], const float* p) {
  static_assert(V == 1 || V == 2, "one or two columns per thread");
  if constexpr (V == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    x[0] = t.x; x[1] = t.y;
  } else {
    x[0] = *p;
  }
}

template <int V>
__device__ __forceinline__ void st_vec(float* p, const float (&x)[V]) {
  if constexpr (V == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(x[0], x[1]);
  } else {
    *p = x[0];
  }
}

// One thread per (V adjacent columns, chunk of levels): blockDim =
// (kNodalCols, C), chunk c holding levels [c K / C, (c + 1) K / C).  The
// column totals and the prefix sums that sigma-dot needs come from per-chunk
// partial sums exchanged through shared memory, so a thread walks K / C
// levels.  A chunk's running sums are its partial sum formed in the same
// order, so the sigma-dot of a half level shared by two chunks is the same in
// both.  V columns share each address computation and level coefficient (the
// latitude count J is a multiple of V, so they lie on one meridian).
// kTracers = false compiles out the tracer windows (dry states).
constexpr int kNodalCols = 32, kNodalMaxChunks = 4;

template <bool kTracers, int V>
__global__ void __launch_bounds__(kNodalCols * kNodalMaxChunks)
    pe_nodal_kernel(NodalArgs a) {
  extern __shared__ float4 s_lev[];  // [K][kLevPack / 4]
  __shared__ float s_e[kNodalMaxChunks][kNodalCols * V];
  __shared__ float s_f[kNodalMaxChunks][kNodalCols * V];
  __shared__ float s_g[kTracers ? kNodalMaxChunks : 1][kNodalCols * V];
  const int tx = threadIdx.x, c = threadIdx.y, C = blockDim.y;
  const int K = a.K;
  for (int i = c * kNodalCols + tx; i < K * (kLevPack / 4); i += kNodalCols * C)
    s_lev[i] = reinterpret_cast<const float4*>(a.levpack)[i];
  __syncthreads();
  // Offsets within one kind's planes are 32-bit (K * I * J < 2^31, checked
  // on the host); tracer kinds stay 64-bit apart.
  const unsigned IJ = (unsigned)a.I * (unsigned)a.J;
  const unsigned col = (blockIdx.x * kNodalCols + tx) * V;
  const bool active = col < IJ;
  const int mb = blockIdx.y;
  const int k0 = (c * K) / C, k1 = ((c + 1) * K) / C;
  const int nT = kTracers ? a.nT : 0;
  const int hum = kTracers ? a.hum : -1;
  const int j = active ? (int)(col % (unsigned)a.J) : 0;
  float sec2[V], fcor[V];
  ld_vec(sec2, a.lat + j);
  ld_vec(fcor, a.lat + a.J + j);
  // Level-0 pointers of these columns for each kind; level k is at [k * IJ].
  auto in = [&](int p) { return a.nod + pl(p, mb, K, 0) * IJ + col; };
  auto out = [&](int p) { return a.fwd + pl(p, mb, K, 0) * IJ + col; };
  const float* Pu = in(a.p_u);
  const float* Pv = in(a.p_v);
  const float* Pd = in(a.p_div);
  const float* Pz = in(a.p_vort);
  const float* PT = in(a.p_temp);
  // Tracer planes are a.mem * K apart.
  const size_t tstride = (size_t)a.mem * K * IJ;
  const float* Pq = in(a.p_tr);
  const float* Ph = Pq + (hum >= 0 ? hum : 0) * tstride;
  const float rv1 = a.Rv_over_R - 1.f;
  float gx[V], gy[V];

  // Pass 1: this chunk's share of the column totals of u.grad(ln ps) and of
  // (div + u.grad ln ps), both weighted by the layer thickness
  // (cumulative_sigma_integral, last level), and (moist) of the geopotential
  // suffix sum of the virtual-temperature difference.
  float pe_[V], pf_[V], pg_[V];
#pragma unroll
  for (int i = 0; i < V; ++i) pe_[i] = pf_[i] = pg_[i] = 0.f;
  if (active) {
    ld_vec(gx, a.nod + ((size_t)a.p_gx + mb) * IJ + col);
    ld_vec(gy, a.nod + ((size_t)a.p_gy + mb) * IJ + col);
    for (int k = k0; k < k1; ++k) {
      const unsigned o = (unsigned)k * IJ;
      const float ds = s_lev[4 * k].x;
      float u[V], v[V], d[V];
      ld_vec(u, Pu + o);
      ld_vec(v, Pv + o);
      ld_vec(d, Pd + o);
#pragma unroll
      for (int i = 0; i < V; ++i) {
        const float ugl = (u[i] * gx[i] + v[i] * gy[i]) * sec2[i];
        pe_[i] += ugl * ds;
        pf_[i] += (d[i] + ugl) * ds;
      }
    }
    if (hum >= 0) {
      for (int k = max(k0, 1); k < k1; ++k) {
        const unsigned o = (unsigned)k * IJ;
        const float4 c1 = s_lev[4 * k + 1];
        const float tr = s_lev[4 * k].w;
        float h[V], T[V];
        ld_vec(h, Ph + o);
        ld_vec(T, PT + o);
#pragma unroll
        for (int i = 0; i < V; ++i) pg_[i] += (c1.z + c1.w) * (h[i] * (T[i] + tr) * rv1);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < V; ++i) {
    s_e[c][tx * V + i] = pe_[i];
    s_f[c][tx * V + i] = pf_[i];
    if (kTracers) s_g[c][tx * V + i] = pg_[i];
  }
  __syncthreads();
  if (!active) return;
  float Fe[V], Ff[V], pre_e[V], pre_f[V];
#pragma unroll
  for (int i = 0; i < V; ++i) {
    Fe[i] = Ff[i] = pre_e[i] = pre_f[i] = 0.f;
    for (int cc = 0; cc < C; ++cc) {
      if (cc == c) {
        pre_e[i] = Fe[i];
        pre_f[i] = Ff[i];
      }
      Fe[i] += s_e[cc][tx * V + i];
      Ff[i] += s_f[cc][tx * V + i];
    }
  }

  // Moist: geopotential of the virtual-temperature difference, G @ td with
  // G[k][h] = R alpha_k (h = k), R (alpha_h + alpha_{h-1}) (h > k): a suffix
  // sum evaluated bottom-up (get_geopotential_weights_sigma, :306-338).
  if (hum >= 0) {
    float suffix[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
      suffix[i] = 0.f;
      for (int cc = C - 1; cc > c; --cc) suffix[i] += s_g[cc][tx * V + i];
    }
    float* Ogh = out(a.o_gh);
    for (int k = k1 - 1; k >= k0; --k) {
      const unsigned o = (unsigned)k * IJ;
      const float4 c1 = s_lev[4 * k + 1];
      const float tr = s_lev[4 * k].w;
      float h[V], T[V], g[V];
      ld_vec(h, Ph + o);
      ld_vec(T, PT + o);
#pragma unroll
      for (int i = 0; i < V; ++i) {
        const float td = h[i] * (T[i] + tr) * rv1;
        g[i] = a.R * (c1.z * td + suffix[i]);
        suffix[i] += (c1.z + c1.w) * td;
      }
      st_vec(Ogh + o, g);
    }
  }

  float* OAu = out(a.o_Au);
  float* OAv = out(a.o_Av);
  float* OKE = out(a.o_KE);
  float* OuT = out(a.o_uT);
  float* OvT = out(a.o_vT);
  float* OTn = out(a.o_Tn);
  float* Otr = out(a.o_tr);
  // Per-column Held-Suarez factors: T_eq = max(T_min, (sigma/p0)^kappa
  // ps^kappa (A0 - B0 log(sigma/p0))) and k_T = k_a + (k_s - k_a) cutoff cos^4.
  float hs_e[V], hs_A0[V], hs_B0[V], hs_dk[V];
  if (a.hs) {
    float lnps_n[V], sin2[V], cos2[V];
    ld_vec(lnps_n, a.nod + ((size_t)a.p_lnps + mb) * IJ + col);
    ld_vec(sin2, a.lat + 2 * a.J + j);
    ld_vec(cos2, a.lat + 3 * a.J + j);
#pragma unroll
    for (int i = 0; i < V; ++i) {
      hs_e[i] = expf(a.kappa * lnps_n[i]);
      hs_A0[i] = a.hs_maxT - a.hs_dTy * sin2[i] - a.hs_dThz * lnps_n[i] * cos2[i];
      hs_B0[i] = a.hs_dThz * cos2[i];
      hs_dk[i] = (a.hs_ks - a.hs_ka) * (cos2[i] * cos2[i]);
    }
  }
  float laplnps[V];
  if (hum >= 0) ld_vec(laplnps, a.nod + ((size_t)a.p_laplnps + mb) * IJ + col);

  // Pass 2: everything else, streaming over the chunk's levels top-down with
  // a window of (k-1, k, k+1) for the vertically advected fields.  The level
  // coefficients hold zero for the half levels outside the column, and the
  // window reads level K-1 again in place of a level K, so the boundary terms
  // vanish without branches.
  const unsigned o0 = (unsigned)k0 * IJ;
  const unsigned om = k0 > 0 ? o0 - IJ : o0;
  float u_p[V], v_p[V], T_p[V], u_c[V], v_c[V], T_c[V];
  ld_vec(u_p, Pu + om);
  ld_vec(v_p, Pv + om);
  ld_vec(T_p, PT + om);
  ld_vec(u_c, Pu + o0);
  ld_vec(v_c, Pv + o0);
  ld_vec(T_c, PT + o0);
  float q_p[kTracers ? kMaxTracers : 1][V], q_c[kTracers ? kMaxTracers : 1][V];
  if (kTracers) {
#pragma unroll
    for (int t = 0; t < kMaxTracers; ++t) {
      if (t < nT) {
        ld_vec(q_p[t], Pq + t * tstride + om);
        ld_vec(q_c[t], Pq + t * tstride + o0);
      }
    }
  }
  // Prefix sums through level k (fe, ff) and k - 1 (fe_prev, ff_prev).
  float loc_e[V], loc_f[V], fe_prev[V], ff_prev[V], sd_up_f[V], sd_up_e[V];
  {
    const float ssu = k0 > 0 ? s_lev[4 * (k0 - 1)].z : 0.f;
#pragma unroll
    for (int i = 0; i < V; ++i) {
      loc_e[i] = loc_f[i] = 0.f;
      fe_prev[i] = pre_e[i];
      ff_prev[i] = pre_f[i];
      // sigma-dot at k0 - 1/2 (0 at the top)
      sd_up_f[i] = k0 > 0 ? ssu * Ff[i] - pre_f[i] : 0.f;
      sd_up_e[i] = k0 > 0 ? ssu * Fe[i] - pre_e[i] : 0.f;
    }
  }

  for (int k = k0; k < k1; ++k) {
    const unsigned o = (unsigned)k * IJ;
    const unsigned on = (k + 1 < K) ? o + IJ : o;
    const float4 c0 = s_lev[4 * k], c1 = s_lev[4 * k + 1];
    const float4 c2 = s_lev[4 * k + 2], c3 = s_lev[4 * k + 3];
    const float ds = c0.x, inv_ds = c0.y, ss = c0.z, tr = c0.w;
    const float ci_dn = c1.x, ci_up = c1.y, al = c1.z, al_up = c1.w;
    float u_n[V], v_n[V], T_n[V], zeta[V], div[V];
    ld_vec(u_n, Pu + on);
    ld_vec(v_n, Pv + on);
    ld_vec(T_n, PT + on);
    ld_vec(zeta, Pz + o);
    ld_vec(div, Pd + o);
    float q_n[kTracers ? kMaxTracers : 1][V];
    if (kTracers) {
#pragma unroll
      for (int t = 0; t < kMaxTracers; ++t)
        if (t < nT) ld_vec(q_n[t], Pq + t * tstride + on);
    }
    float gqx[V], gqy[V];
    if (hum >= 0) {
      ld_vec(gqx, a.nod + pl(a.p_gqx, mb, K, 0) * IJ + col + o);
      ld_vec(gqy, a.nod + pl(a.p_gqy, mb, K, 0) * IJ + col + o);
    }
    float rAu[V], rAv[V], rKE[V], ruT[V], rvT[V], rTn[V], rhs[V], rvh[V], rdh[V];
    float sdn_f[V], sdn_e[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
      const float ugl = (u_c[i] * gx[i] + v_c[i] * gy[i]) * sec2[i];
      loc_e[i] += ugl * ds;
      loc_f[i] += (div[i] + ugl) * ds;
      const float fe = pre_e[i] + loc_e[i];
      const float ff = pre_f[i] + loc_f[i];
      const float sd_dn_f = ss * Ff[i] - ff;  // sigma-dot at k + 1/2
      const float sd_dn_e = ss * Fe[i] - fe;
      sdn_f[i] = sd_dn_f;
      sdn_e[i] = sd_dn_e;
      // centered_vertical_advection(w, x)[k] = -0.5 (w_{k+1/2} dx_{k+1/2} +
      // w_{k-1/2} dx_{k-1/2}) (sigma_coordinates.py:344-405).
      auto vadv = [&](float xp, float xc, float xn) {
        return -0.5f * (sd_dn_f * ((xn - xc) * ci_dn) + sd_up_f[i] * ((xc - xp) * ci_up));
      };
      float q_h = 0.f;
      if (kTracers && hum >= 0) {
#pragma unroll
        for (int t = 0; t < kMaxTracers; ++t)
          if (t == hum) q_h = q_c[t][i];
      }
      // curl_and_div_tendencies (:1001-1059)
      const float adj = (hum >= 0) ? 1.f + rv1 * q_h : 1.f;
      const float rt = a.R * T_c[i] * adj;
      float sdu = 0.f, sdv = 0.f;
      if (a.vadv) {
        sdu = -vadv(u_p[i], u_c[i], u_n[i]);
        sdv = -vadv(v_p[i], v_c[i], v_n[i]);
      }
      const float tv = zeta[i] + fcor[i];
      float Au = -v_c[i] * tv * sec2[i] + (sdu + rt * gx[i]) * sec2[i];
      float Av = u_c[i] * tv * sec2[i] + (sdv + rt * gy[i]) * sec2[i];
      if (a.hs) {
        // Rayleigh drag folded in: curl/div of -(-kv u / cos^2).
        Au += c2.x * u_c[i] * sec2[i];
        Av += c2.x * v_c[i] * sec2[i];
      }
      rAu[i] = Au;
      rAv[i] = Av;
      rKE[i] = (u_c[i] * u_c[i] + v_c[i] * v_c[i]) * sec2[i] * 0.5f;
      ruT[i] = u_c[i] * T_c[i] * sec2[i];
      rvT[i] = v_c[i] * T_c[i] * sec2[i];
      // Temperature: horizontal nodal term, vertical advection, adiabatic.
      float Tn = T_c[i] * div[i];
      if (a.vadv) Tn += vadv(T_p[i], T_c[i], T_n[i]);
      if (a.tref_varies) Tn += -0.5f * (sd_dn_e * c3.x + sd_up_e[i] * c3.y);
      const float ge = (al * fe + al_up * fe_prev[i]) * inv_ds;
      const float gf = (al * ff + al_up * ff_prev[i]) * inv_ds;
      const float mean_part = tr * (ugl - ge);
      float var_part;
      if (hum < 0) {
        var_part = T_c[i] * (ugl - gf);
      } else {
        const float den = 1.f + (a.Cpv_over_Cp - 1.f) * q_h;
        const float tv_var = T_c[i] * ((1.f + rv1 * q_h) / den);
        const float tv_ref = tr * (((a.Rv_over_R - a.Cpv_over_Cp) * q_h) / den);
        var_part = (tv_var + tv_ref) * (ugl - gf);
      }
      rTn[i] = Tn + a.kappa * (mean_part + var_part);
      if (hum >= 0) {
        const float coef = tr * a.Rv_minus_R;
        rvh[i] = coef * sec2[i] * (gx[i] * gqy[i] - gy[i] * gqx[i]);
        rdh[i] = coef * sec2[i] * (gqx[i] * gx[i] + gqy[i] * gy[i]) +
                 q_h * laplnps[i] * tr * a.Rv_minus_R;
      }
      if (a.hs) {
        // held_suarez.py:105-120, :138-151, with log(p / p0) = log(sigma / p0)
        // + ln ps, so (p / p0)^kappa = (sigma / p0)^kappa ps^kappa.
        const float kt = a.hs_ka + hs_dk[i] * c2.y;
        float teq = c2.z * hs_e[i] * (hs_A0[i] - hs_B0[i] * c2.w);
        teq = fmaxf(a.hs_minT, teq);
        rhs[i] = -kt * (tr + T_c[i] - teq);
      }
      fe_prev[i] = fe;
      ff_prev[i] = ff;
    }
    st_vec(OAu + o, rAu);
    st_vec(OAv + o, rAv);
    st_vec(OKE + o, rKE);
    st_vec(OuT + o, ruT);
    st_vec(OvT + o, rvT);
    st_vec(OTn + o, rTn);
    if (hum >= 0) {
      st_vec(a.fwd + pl(a.o_vh, mb, K, 0) * IJ + col + o, rvh);
      st_vec(a.fwd + pl(a.o_dh, mb, K, 0) * IJ + col + o, rdh);
    }
    if (a.hs) st_vec(a.fwd + pl(a.o_hsT, mb, K, 0) * IJ + col + o, rhs);
    // Tracers: u q, v q (times sec^2) and q div + vertical advection.
    if (kTracers) {
#pragma unroll
      for (int t = 0; t < kMaxTracers; ++t) {
        if (t >= nT) break;
        float* ob = Otr + 3 * t * tstride;
        float fu[V], fv[V], fq[V];
#pragma unroll
        for (int i = 0; i < V; ++i) {
          fu[i] = u_c[i] * q_c[t][i] * sec2[i];
          fv[i] = v_c[i] * q_c[t][i] * sec2[i];
          float qn = q_c[t][i] * div[i];
          if (a.vadv)
            qn += -0.5f * (sdn_f[i] * ((q_n[t][i] - q_c[t][i]) * ci_dn) +
                           sd_up_f[i] * ((q_c[t][i] - q_p[t][i]) * ci_up));
          fq[i] = qn;
        }
        st_vec(ob + o, fu);
        st_vec(ob + tstride + o, fv);
        st_vec(ob + 2 * tstride + o, fq);
      }
    }
    // Advance the window.
#pragma unroll
    for (int i = 0; i < V; ++i) {
      sd_up_f[i] = sdn_f[i];
      sd_up_e[i] = sdn_e[i];
      u_p[i] = u_c[i]; v_p[i] = v_c[i]; T_p[i] = T_c[i];
      u_c[i] = u_n[i]; v_c[i] = v_n[i]; T_c[i] = T_n[i];
    }
    if (kTracers) {
#pragma unroll
      for (int t = 0; t < kMaxTracers; ++t)
#pragma unroll
        for (int i = 0; i < V; ++i) {
          q_p[t][i] = q_c[t][i];
          q_c[t][i] = q_n[t][i];
        }
    }
  }
  if (c == 0) {
    float l[V];
#pragma unroll
    for (int i = 0; i < V; ++i) l[i] = -Fe[i];
    st_vec(a.fwd + ((size_t)a.o_lnps + mb) * IJ + col, l);
  }
}

// ---------------------------------------------------------------------------
// Nodal column kernel on hybrid sigma-pressure levels (Simmons & Burridge)
// ---------------------------------------------------------------------------

// Per-level constants of pe_nodal_hybrid_kernel, kHybPack floats per level k
// (0 = top), all at the reference surface pressure p_s_ref except a, b:
//   0 a_{k-1/2}  1 b_{k-1/2}  2 da_k  3 db_k  4 T_ref,k  5 alpha_k
//   6 log(p_{k+1/2} / p_{k-1/2})  7 s_k = W_k p_s / max(dp_k, 1e-6 p_s)
//   8 p_{k-1/2}  9 dp_k  10 W_k = log-ratio_k b_{k-1/2} + alpha_k db_k
//   11 1 / dp_k  12 1 / P_{k-1/2}  13 b_{k-1/2} / P_{k-1/2}
// (P = max(p, 1e-6 p_s_ref), the floored interface pressure), followed by
// a, b, p, 1 / P and b / P of the lowest interface.
constexpr int kHybPack = 16;
constexpr int kHybTail = 5;
constexpr int kHybThreads = 128;

struct HybridArgs {
  const float* nod;         // nodal inverse-transform planes
  float* fwd;               // nodal forward-transform planes
  const float* lev;         // [K][kHybPack], a_K, b_K, p_K
  const float* lat;         // sec^2 [J], 2 Omega sin [J]
  const float* lnps_modal;  // modal ln p_s of the state, [mem][M][L]
  unsigned ML;
  int K, mem, nT, hum, vadv, tref_varies, I, J;
  int p_vort, p_div, p_temp, p_tr, p_u, p_v, p_gx, p_gy, p_lnps;
  int o_Au, o_Av, o_KE, o_uT, o_vT, o_Tn, o_tr, o_lnps;
  float R, kappa, ps_ref, Rv_over_R, Cpv_over_Cp;
  double ln_ps_ref, inv_y00;  // FP64: their difference below is ~1e-2 of each
};

// One thread per column (member blockIdx.y): the nodal explicit terms of
// PrimitiveEquationsHybrid (primitive_equations.py:1536-1603, :2058-2360).
//
// FP32 accuracy.  Nodal ln p_s is ~45 (nondimensional pressure ~3e19) with
// variations of ~1e-3, beyond FP32's resolution of ~4e-6 there; so ln p_s
// arrives as the transform of its coefficients without the l = 0 term (the
// p_lnps plane) plus that term's nodal value c_00 / (2 sqrt(pi)), and
// p_s = p_s_ref exp(rel) with rel = ln(p_s / p_s_ref) formed from them.  The
// pressure-gradient and geopotential residuals subtract terms at p_s_ref
// from terms at p_s; they are written as the reference value plus
// deviations proportional to p_s - p_s_ref (the log pressure ratios through
// log1p, alpha, W and W p_s / dp), so nothing large cancels.  The geopotential
// residual omits its horizontally uniform part R (sum_{j>k} T_ref,j lr_j +
// alpha_k T_ref,k) at p_s_ref, which the Laplacian of the divergence
// tendency removes.
//
// Passes over the levels:
//   A+B (bottom-up): column totals of the layer mass-flux divergences
//     D_k = dp_k div_k + db_k p_s (v . grad ln p_s) and of their advective
//     part, the ln p_s tendency, and kinetic energy plus the geopotential
//     residual (get_geopotential_diff_hybrid, :1628-1675) through suffix sums.
//   C (top-down): mass fluxes M_{k+1/2} = -sum_{r<=k} D_r + b_{k+1/2} sum D
//     at both interfaces of the level, vertical advection
//     (hybrid_vertical_advection, :1941-1958), the pressure-gradient
//     residual (:1826-1856), the temperature tendency with the omega / p
//     terms (:2124-2224, whose integrands are the same D_k) and the tracers.
// Outputs use the planes of pe_nodal_kernel, so the modal post-pass is shared.
__global__ void __launch_bounds__(kHybThreads) pe_nodal_hybrid_kernel(HybridArgs a) {
  extern __shared__ float s_hyb[];
  const int K = a.K;
  for (int i = threadIdx.x; i < K * kHybPack + kHybTail; i += blockDim.x) s_hyb[i] = a.lev[i];
  // log1p(x) of this column's K + 1 interfaces, computed in the bottom-up
  // pass and reused top-down (interface i at s_l1[i * blockDim.x + tid]).
  float* s_l1 = s_hyb + K * kHybPack + kHybTail;
  __syncthreads();
  const unsigned IJ = (unsigned)a.I * (unsigned)a.J;
  const unsigned col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= IJ) return;
  const int mb = blockIdx.y;
  const int mK = a.mem * K;
  const int j = (int)(col % (unsigned)a.J);
  const float sec2 = a.lat[j];
  const float fcor = a.lat[a.J + j];
  // The inputs are read-only for the kernel's duration: read-only loads may
  // run ahead of the output stores.
  auto ld = [&](int base, int k) -> float {
    return __ldg(a.nod + ((size_t)base + (size_t)mb * K + k) * IJ + col);
  };
  auto st = [&](int base, int k, float v) {
    a.fwd[((size_t)base + (size_t)mb * K + k) * IJ + col] = v;
  };
  auto lev = [&](int k, int i) -> float { return s_hyb[k * kHybPack + i]; };
  auto a_if = [&](int i) -> float { return i < K ? lev(i, 0) : s_hyb[K * kHybPack]; };
  auto b_if = [&](int i) -> float { return i < K ? lev(i, 1) : s_hyb[K * kHybPack + 1]; };
  auto pr_if = [&](int i) -> float { return i < K ? lev(i, 8) : s_hyb[K * kHybPack + 2]; };
  auto ipr_if = [&](int i) -> float { return i < K ? lev(i, 12) : s_hyb[K * kHybPack + 3]; };
  auto bpr_if = [&](int i) -> float { return i < K ? lev(i, 13) : s_hyb[K * kHybPack + 4]; };
  const float gx = __ldg(a.nod + ((size_t)a.p_gx + mb) * IJ + col);
  const float gy = __ldg(a.nod + ((size_t)a.p_gy + mb) * IJ + col);
  const float psr = a.ps_ref;
  // The uniform part c_00 / (2 sqrt(pi)) - ln p_s_ref in FP64: both terms
  // are ~45 and their FP32 roundings would be ~5e-6 of a difference ~1e-2.
  const float rel = (float)((double)a.lnps_modal[(size_t)mb * a.ML] * a.inv_y00 - a.ln_ps_ref) +
                    __ldg(a.nod + ((size_t)a.p_lnps + mb) * IJ + col);
  const float ps = psr * expf(rel);
  const float dps = psr * expm1f(rel);  // p_s - p_s_ref
  const float floor_s = 1e-6f * ps, floor_r = 1e-6f * psr;
  const int hum = a.hum;
  auto hum_at = [&](int k) -> float { return hum >= 0 ? ld(a.p_tr + hum * mK, k) : 0.f; };
  // Virtual-temperature factor 1 + (R_v / R - 1) q.
  auto adj_of = [&](float q) -> float { return hum >= 0 ? 1.f + (a.Rv_over_R - 1.f) * q : 1.f; };
  // (P_i - P_i,ref) / P_i,ref of the floored interface pressure max(p, 1e-6 p_s).
  // Unfloored: b dps / P_ref; floored both ways: dps / p_s_ref.
  const float inv_psr = 1.f / psr;
  auto x_if = [&](int i) -> float {
    const float p = a_if(i) + b_if(i) * ps, pr = pr_if(i);
    if (p >= floor_s && pr >= floor_r) return dps * bpr_if(i);
    if (p < floor_s && pr < floor_r) return dps * inv_psr;
    return (fmaxf(p, floor_s) - fmaxf(pr, floor_r)) * ipr_if(i);
  };
  // Level k at this column, given log1p(x) of its upper and lower interfaces
  // (each interface's value is carried to the next level): deviations of the
  // log ratio and alpha (_get_vertical_discretization_coeffs, :1507-1533), W
  // and s - s_ref = W p_s / dp - (W p_s / dp)_ref.
  struct Lev {
    float dlr, dal, W, ds;
  };
  auto level = [&](int k, float l1_up, float l1_dn) -> Lev {
    Lev o;
    o.dlr = l1_dn - l1_up;
    const float da = lev(k, 2), db = lev(k, 3), dpr = lev(k, 9), idpr = lev(k, 11);
    const float dp = da + db * ps;
    const float idp = 1.f / dp;
    const float r = (a_if(k) + b_if(k) * ps) * idp;
    const float dr = dps * (b_if(k) * da - a_if(k) * db) * (idp * idpr);
    o.dal = -(dr * lev(k, 6) + r * o.dlr);
    const float dW = o.dlr * b_if(k) + o.dal * db;
    o.W = lev(k, 10) + dW;
    if (dp >= floor_s && dpr >= floor_r)
      o.ds = lev(k, 10) * da * dps * (idp * idpr) + dW * ps * idp;
    else
      o.ds = o.W * ps / fmaxf(dp, floor_s) - lev(k, 7);
    return o;
  };

  // Pass A+B (bottom-up): the column totals and the ln p_s tendency, and
  // KE + R (sum_{j>k} t_j ((adj_j - 1) lr_ref,j + adj_j dlr_j)
  //         + t_k ((adj_k - 1) alpha_ref,k + adj_k dalpha_k)), t = T' + T_ref.
  float totF = 0.f, totE = 0.f;
  {
    float lp_a = 0.f, lp_b = 0.f, suf = 0.f;
    const float inv_ps_diff = -dps / ps / psr;  // 1 / p_s - 1 / p_s_ref
    float l1_dn = log1pf(x_if(K));
    s_l1[K * blockDim.x + threadIdx.x] = l1_dn;
    // Level k's inputs were loaded during level k + 1 (one level ahead).
    float u_x = ld(a.p_u, K - 1), v_x = ld(a.p_v, K - 1), d_x = ld(a.p_div, K - 1),
          T_x = ld(a.p_temp, K - 1), q_x = hum_at(K - 1);
    for (int k = K - 1; k >= 0; --k) {
      const float u = u_x, v = v_x, d = d_x, T = T_x, q = q_x;
      if (k > 0) {
        u_x = ld(a.p_u, k - 1);
        v_x = ld(a.p_v, k - 1);
        d_x = ld(a.p_div, k - 1);
        T_x = ld(a.p_temp, k - 1);
        q_x = hum_at(k - 1);
      }
      const float da = lev(k, 2), db = lev(k, 3);
      const float udg = (u * gx + v * gy) * sec2;
      const float dp = da + db * ps;
      const float DE = db * ps * udg;
      totF += dp * d + DE;
      totE += DE;
      lp_a += d * da * inv_ps_diff;
      lp_b += udg * db;
      const float l1_up = log1pf(x_if(k));
      s_l1[k * blockDim.x + threadIdx.x] = l1_up;
      const Lev L = level(k, l1_up, l1_dn);
      l1_dn = l1_up;
      const float t = T + lev(k, 4);
      const float adj = adj_of(q);
      const float ke = (u * u + v * v) * sec2 * 0.5f;
      st(a.o_KE, k, ke + a.R * (suf + t * ((adj - 1.f) * lev(k, 5) + adj * L.dal)));
      suf += t * ((adj - 1.f) * lev(k, 6) + adj * L.dlr);
    }
    a.fwd[((size_t)a.o_lnps + mb) * IJ + col] = -(lp_a + lp_b);
  }

  // Pass C.
  float cumF = 0.f, cumE = 0.f;  // sum_{r<k} D_r
  float fF_prev = 0.f, fE_prev = 0.f, alr_prev = 0.f;
  float u_p = 0.f, v_p = 0.f, T_p = 0.f, u_c = ld(a.p_u, 0), v_c = ld(a.p_v, 0),
        T_c = ld(a.p_temp, 0);
  float q_p[kMaxTracers], q_c[kMaxTracers];
#pragma unroll
  for (int t = 0; t < kMaxTracers; ++t) {
    q_p[t] = 0.f;
    q_c[t] = t < a.nT ? ld(a.p_tr + t * mK, 0) : 0.f;
  }
  float l1_up = s_l1[threadIdx.x];
  // zeta, div of level k and u, v, T of level k + 1 were loaded during
  // level k - 1.
  float zeta_x = ld(a.p_vort, 0), d_x = ld(a.p_div, 0);
  float u_x = K > 1 ? ld(a.p_u, 1) : 0.f, v_x = K > 1 ? ld(a.p_v, 1) : 0.f,
        T_x = K > 1 ? ld(a.p_temp, 1) : 0.f;
  for (int k = 0; k < K; ++k) {
    const bool has_up = k > 0, has_dn = k + 1 < K;
    const float u_n = u_x, v_n = v_x, T_n = T_x;
    const float zeta = zeta_x, d = d_x;
    if (has_dn) {
      zeta_x = ld(a.p_vort, k + 1);
      d_x = ld(a.p_div, k + 1);
      if (k + 2 < K) {
        u_x = ld(a.p_u, k + 2);
        v_x = ld(a.p_v, k + 2);
        T_x = ld(a.p_temp, k + 2);
      } else {
        u_x = v_x = T_x = 0.f;
      }
    }
    const float da = lev(k, 2), db = lev(k, 3), tr = lev(k, 4), alr = lev(k, 5);
    const float udg = (u_c * gx + v_c * gy) * sec2;
    const float dp = da + db * ps;
    const float DE = db * ps * udg;
    const float DF = dp * d + DE;
    // Mass fluxes at the level's upper (k - 1/2) and lower (k + 1/2) interfaces.
    const float MF_up = -cumF + b_if(k) * totF, MF_dn = -(cumF + DF) + b_if(k + 1) * totF;
    const float ME_up = -cumE + b_if(k) * totE, ME_dn = -(cumE + DE) + b_if(k + 1) * totE;
    const float inv_dp = 1.f / dp;
    // hybrid_vertical_advection(M, x)_k; only interior interfaces carry flux.
    auto vadv = [&](float mu, float md, float xp, float xc, float xn) -> float {
      const float fu = has_up ? mu * (xc - xp) : 0.f;
      const float fd = has_dn ? md * (xn - xc) : 0.f;
      return -0.5f * (fu + fd) * inv_dp;
    };
    const float l1_dn = s_l1[(k + 1) * blockDim.x + threadIdx.x];
    const Lev L = level(k, l1_up, l1_dn);
    l1_up = l1_dn;
    float q_h = 0.f;  // selected without a dynamic index (keeps q_c in registers)
#pragma unroll
    for (int t2 = 0; t2 < kMaxTracers; ++t2)
      if (t2 == hum) q_h = q_c[t2];
    const float adj = adj_of(q_h);
    const float t = T_c + tr;
    // Pressure-gradient residual C_k(T, p_s) adj - C_k(T_ref, p_s_ref)
    // = R (t adj (s - s_ref) + (t (adj - 1) + T') s_ref).
    const float pgf = a.R * (t * adj * L.ds + (t * (adj - 1.f) + T_c) * lev(k, 7));
    float sdu = 0.f, sdv = 0.f;
    if (a.vadv) {
      sdu = -vadv(MF_up, MF_dn, u_p, u_c, u_n);
      sdv = -vadv(MF_up, MF_dn, v_p, v_c, v_n);
    }
    const float tv = zeta + fcor;
    st(a.o_Au, k, -v_c * tv * sec2 + (sdu + pgf * gx) * sec2);
    st(a.o_Av, k, u_c * tv * sec2 + (sdv + pgf * gy) * sec2);
    st(a.o_uT, k, u_c * T_c * sec2);
    st(a.o_vT, k, v_c * T_c * sec2);
    // Temperature: T' div, vertical advection, omega / p terms
    // (_t_omega_over_p_hybrid, :2032-2056, with alpha at p_s_ref).
    float Tn = T_c * d;
    if (a.vadv) Tn += vadv(MF_up, MF_dn, T_p, T_c, T_n);
    if (a.tref_varies) {
      const float tr_up = has_up ? lev(k - 1, 4) : 0.f;
      const float tr_dn = has_dn ? lev(k + 1, 4) : 0.f;
      Tn += vadv(ME_up, ME_dn, tr_up, tr, tr_dn);
    }
    const float fF = cumF + DF, fE = cumE + DE;
    const float gF = (alr * fF + alr_prev * fF_prev) * inv_dp;
    const float gE = (alr * fE + alr_prev * fE_prev) * inv_dp;
    const float sudg = udg * ps * L.W * (dp >= floor_s ? inv_dp : 1.f / floor_s);
    const float mean_part = tr * (sudg - gE);
    float var_part;
    if (hum < 0) {
      var_part = T_c * (sudg - gF);
    } else {
      const float den = 1.f + (a.Cpv_over_Cp - 1.f) * q_h;
      const float tvar = T_c * ((1.f + (a.Rv_over_R - 1.f) * q_h) / den);
      const float tref_q = tr * (((a.Rv_over_R - a.Cpv_over_Cp) * q_h) / den);
      var_part = (tvar + tref_q) * (sudg - gF);
    }
    st(a.o_Tn, k, Tn + a.kappa * (mean_part + var_part));
    // Tracers: u q, v q (times sec^2) and q div + vertical advection.
#pragma unroll
    for (int t2 = 0; t2 < kMaxTracers; ++t2) {
      if (t2 >= a.nT) break;
      const float q_n = has_dn ? ld(a.p_tr + t2 * mK, k + 1) : 0.f;
      const int ob = a.o_tr + 3 * t2 * mK;
      st(ob, k, u_c * q_c[t2] * sec2);
      st(ob + mK, k, v_c * q_c[t2] * sec2);
      float qn = q_c[t2] * d;
      if (a.vadv) qn += vadv(MF_up, MF_dn, q_p[t2], q_c[t2], q_n);
      st(ob + 2 * mK, k, qn);
      q_p[t2] = q_c[t2];
      q_c[t2] = q_n;
    }
    cumF += DF;
    cumE += DE;
    fF_prev = fF;
    fE_prev = fE;
    alr_prev = alr;
    u_p = u_c; v_p = v_c; T_p = T_c;
    u_c = u_n; v_c = v_n; T_c = T_n;
  }
}

// ---------------------------------------------------------------------------
// Modal post-pass: curl/div, Laplacians, horizontal advection divergence,
// orography, humidity corrections, clip of the top wavenumber.
// ---------------------------------------------------------------------------

struct PostArgs {
  const float* fm;  // forward outputs (modal)
  float* tend;      // packed state layout
  const float* orog;
  int K, mem, nT, hum, hs;
  int M, L, lw;
  int o_Au, o_Av, o_KE, o_uT, o_vT, o_Tn, o_tr, o_vh, o_gh, o_dh, o_hsT,
      o_lnps;
  int p_vort, p_div, p_temp, p_tr, p_lnps;
  const float* deriv;
  const float* lap;
  float inv_radius, gravity;
};

__global__ void __launch_bounds__(kModalTX * kModalTY) pe_post_kernel(PostArgs a) {
  const int l = blockIdx.x * kModalTX + threadIdx.x;
  const int row = blockIdx.y * kModalTY + threadIdx.y;
  if (l >= a.L || row >= a.M) return;
  const size_t ML = (size_t)a.M * a.L;
  const size_t idx = (size_t)row * a.L + l;
  const int K = a.K;
  const bool clip = (l == a.L - 1);
  const float lam = a.lap[l];
  const float ir = a.inv_radius;
  const float orog = a.gravity * lam * a.orog[idx];
  const ModalNbr nb(row, l, a.L, a.lw, a.deriv, 2, nullptr);
  const int q0 = blockIdx.z * kPlanesPerThread;
  const int q1 = min(q0 + kPlanesPerThread, K * a.mem);
  for (int q = q0; q < q1; ++q) {
    const int mb = q / K, k = q - mb * K;
#define FM(p) (a.fm + pl(p, mb, K, k) * ML)
#define OUT(p) a.tend[pl(p, mb, K, k) * ML + idx]
    const float* Au = FM(a.o_Au);
    const float* Av = FM(a.o_Av);
    float vort = -(nb.dlon(Av) - nb.dlat(Au)) * ir;
    float div = -(nb.dlon(Au) + nb.dlat(Av)) * ir;
    div += -lam * FM(a.o_KE)[idx] - orog;
    if (a.hum >= 0) {
      vort += FM(a.o_vh)[idx];
      div += -lam * FM(a.o_gh)[idx] - FM(a.o_dh)[idx];
    }
    float temp = FM(a.o_Tn)[idx] - (nb.dlon(FM(a.o_uT)) + nb.dlat(FM(a.o_vT))) * ir;
    if (clip) {
      vort = 0.f;
      div = 0.f;
      temp = 0.f;
    }
    if (a.hs) temp += FM(a.o_hsT)[idx];
    OUT(a.p_vort) = vort;
    OUT(a.p_div) = div;
    OUT(a.p_temp) = temp;
    for (int t = 0; t < a.nT; ++t) {
      const int ob = a.o_tr + 3 * t * a.mem * K;
      float qv = FM(ob + 2 * a.mem * K)[idx] -
                 (nb.dlon(FM(ob)) + nb.dlat(FM(ob + a.mem * K))) * ir;
      OUT(a.p_tr + t * a.mem * K) = clip ? 0.f : qv;
    }
    if (k == 0) {
      const float lnps = a.fm[((size_t)a.o_lnps + mb) * ML + idx];
      a.tend[((size_t)a.p_lnps + mb) * ML + idx] = clip ? 0.f : lnps;
    }
#undef FM
#undef OUT
  }
}

// ---------------------------------------------------------------------------
// Adjoint of the explicit terms (the VJP of explicit_terms,
// primitive_equations.py:1126-1194): the transposed post-pass, the forward
// transform's adjoint, the VJP of the nodal column kernel (recomputing its
// inputs), the inverse transform's adjoint and the transposed pre-pass.
// ---------------------------------------------------------------------------

// Transposed post-pass: tendency cotangents (packed state layout) ->
// cotangents of the forward-transform outputs.  d/dlon is antisymmetric
// (its transpose is -d/dlon); the top total wavenumber of every clipped
// tendency has a zero cotangent.
struct PostAdjArgs {
  const float* tbar;
  float* fbar;
  int K, mem, nT, hum, hs;
  int M, L, lw;
  int o_Au, o_Av, o_KE, o_uT, o_vT, o_Tn, o_tr, o_vh, o_gh, o_dh, o_hsT,
      o_lnps;
  int p_vort, p_div, p_temp, p_tr, p_lnps;
  const float* deriv;
  const float* lap;
  float inv_radius;
};

// Transposed operators at (row, l): d/dlon^T = -d/dlon, and
// (D^T y)[l] = ta[l] y[l-1] + tb[l] y[l+1] with y taken as zero at l >= lclip
// (the clipped top wavenumber of a tendency cotangent).
struct ModalNbrT {
  int row, l, L;
  int dl_row;
  float dl_fac;
  float a0, b0;  // coefficients of y[l - 1] and y[l + 1] (0 when out of range)

  __device__ ModalNbrT(int row_, int l_, int L_, int lw, const float* deriv, int tab,
                       int lclip)
      : row(row_), l(l_), L(L_) {
    const int m = (row + 1) >> 1;
    if (row == 0) {
      dl_row = 0;
      dl_fac = 0.f;
    } else if (row & 1) {
      dl_row = row + 1;
      dl_fac = (float)m;
    } else {
      dl_row = row - 1;
      dl_fac = -(float)m;
    }
    const float* ta = deriv + (size_t)tab * lw * L + (size_t)m * L;
    const float* tb = ta + (size_t)lw * L;
    a0 = (l >= 1 && l - 1 < lclip) ? ta[l] : 0.f;
    b0 = (l + 1 < lclip) ? tb[l] : 0.f;
  }
  // d/dlon (the transpose is its negative).
  __device__ float dlon(const float* x) const {
    return dl_fac * x[(size_t)dl_row * L + l];
  }
  __device__ float dlat_t(const float* y) const {
    const float* yr = y + (size_t)row * L + l;
    float v = 0.f;
    if (a0 != 0.f) v += a0 * yr[-1];
    if (b0 != 0.f) v += b0 * yr[1];
    return v;
  }
};

__global__ void __launch_bounds__(kModalTX * kModalTY) pe_post_adjoint_kernel(PostAdjArgs a) {
  const int l = blockIdx.x * kModalTX + threadIdx.x;
  const int row = blockIdx.y * kModalTY + threadIdx.y;
  if (l >= a.L || row >= a.M) return;
  const size_t ML = (size_t)a.M * a.L;
  const size_t idx = (size_t)row * a.L + l;
  const int K = a.K;
  const int Lc = a.L - 1;
  const bool keep = l < Lc;
  const float ir = a.inv_radius;
  const float lam = a.lap[l];
  const ModalNbrT nb(row, l, a.L, a.lw, a.deriv, 2, Lc);
  const int q0 = blockIdx.z * kPlanesPerThread;
  const int q1 = min(q0 + kPlanesPerThread, K * a.mem);
  for (int q = q0; q < q1; ++q) {
    const int mb = q / K, k = q - mb * K;
#define TB(p) (a.tbar + pl(p, mb, K, k) * ML)
#define FB(p) a.fbar[pl(p, mb, K, k) * ML + idx]
    const float* vb = TB(a.p_vort);
    const float* db = TB(a.p_div);
    const float* Tb = TB(a.p_temp);
    const float vc = keep ? vb[idx] : 0.f;
    const float dc = keep ? db[idx] : 0.f;
    const float Tc = keep ? Tb[idx] : 0.f;
    const float dlon_v = keep ? nb.dlon(vb) : 0.f;
    const float dlon_d = keep ? nb.dlon(db) : 0.f;
    const float dlon_T = keep ? nb.dlon(Tb) : 0.f;
    FB(a.o_Au) = (nb.dlat_t(vb) + dlon_d) * ir;
    FB(a.o_Av) = (dlon_v - nb.dlat_t(db)) * ir;
    FB(a.o_KE) = -lam * dc;
    if (a.hum >= 0) {
      FB(a.o_vh) = vc;
      FB(a.o_gh) = -lam * dc;
      FB(a.o_dh) = -dc;
    }
    FB(a.o_Tn) = Tc;
    FB(a.o_uT) = dlon_T * ir;
    FB(a.o_vT) = -nb.dlat_t(Tb) * ir;
    if (a.hs) FB(a.o_hsT) = Tb[idx];
    for (int t = 0; t < a.nT; ++t) {
      const int ob = a.o_tr + 3 * t * a.mem * K;
      const float* qb = TB(a.p_tr + t * a.mem * K);
      FB(ob) = (keep ? nb.dlon(qb) : 0.f) * ir;
      FB(ob + a.mem * K) = -nb.dlat_t(qb) * ir;
      FB(ob + 2 * a.mem * K) = keep ? qb[idx] : 0.f;
    }
    if (k == 0)
      a.fbar[((size_t)a.o_lnps + mb) * ML + idx] =
          keep ? a.tbar[((size_t)a.p_lnps + mb) * ML + idx] : 0.f;
#undef TB
#undef FB
  }
}

// VJP of pe_nodal_kernel for one column.  Pass 0 forms the column totals;
// pass 1 runs bottom-up with a (k, k+1) window: each half level k+1/2 takes
// the cotangents of the centred vertical advection of u, v, T' and the
// tracers (and of the reference-temperature term), and the cumulative sigma
// sums become suffix sums of their cotangents; pass 2 adds the cotangents of
// the column totals, which reach every level.
struct NodalAdjArgs {
  NodalArgs f;        // forward arguments; f.nod holds the forward inputs
  const float* fbar;  // cotangents of the nodal outputs (forward-input layout)
  float* xbar;        // cotangents of the nodal inputs (nodal-buffer layout)
};

// Five CTAs per SM (96 registers, no spills).  The per-level coefficients
// come from the packed table in shared memory (kLevPack, as in
// pe_nodal_kernel); plane offsets are 32-bit (the nodal and forward-input
// buffers hold fewer than 2^32 floats, checked on the host).
__global__ void __launch_bounds__(128, 5) pe_nodal_adjoint_kernel(NodalAdjArgs A) {
  extern __shared__ float4 s_lev[];  // [K][kLevPack / 4]
  const NodalArgs& a = A.f;
  const int K = a.K;
  for (int i = threadIdx.x; i < K * (kLevPack / 4); i += blockDim.x)
    s_lev[i] = reinterpret_cast<const float4*>(a.levpack)[i];
  __syncthreads();
  const unsigned IJ = (unsigned)a.I * (unsigned)a.J;
  const unsigned col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= IJ) return;
  const int mb = blockIdx.y;
  const int j = (int)(col % (unsigned)a.J);
  const float sec2 = a.lat[j];
  const float fcor = a.lat[a.J + j];
  // Per-level coefficients (see kLevPack).
  auto dsig = [&](int k) { return s_lev[4 * k].x; };
  auto invds = [&](int k) { return s_lev[4 * k].y; };
  auto sumsig = [&](int k) { return s_lev[4 * k].z; };
  auto tref = [&](int k) { return s_lev[4 * k].w; };
  auto c2ci = [&](int k) { return s_lev[4 * k + 1].x; };
  auto alpha = [&](int k) { return s_lev[4 * k + 1].z; };
  auto alpha_up = [&](int k) { return s_lev[4 * k + 1].w; };
  auto trd = [&](int k) { return s_lev[4 * k + 3].x; };
  const float* nod = a.nod;
  const float* fb = A.fbar;
  float* xb = A.xbar;
  const unsigned mK = (unsigned)mb * (unsigned)K;
#define NOD(p, k) nod[((unsigned)(p) + mK + (unsigned)(k)) * IJ + col]
#define FB(p, k) fb[((unsigned)(p) + mK + (unsigned)(k)) * IJ + col]
#define XB(p, k) xb[((unsigned)(p) + mK + (unsigned)(k)) * IJ + col]
  const bool moist = a.hum >= 0;
  const float gx = nod[((unsigned)a.p_gx + mb) * IJ + col];
  const float gy = nod[((unsigned)a.p_gy + mb) * IJ + col];
  const float ra = a.Rv_over_R - 1.f;
  const float rb = a.Cpv_over_Cp - 1.f;
  const float rc = a.Rv_over_R - a.Cpv_over_Cp;
  const float kap = a.kappa;

  // Pass 0: column totals.
  float Fe = 0.f, Ff = 0.f, Su = 0.f, Sv = 0.f, Gh = 0.f;
  for (int k = 0; k < K; ++k) {
    const float u = NOD(a.p_u, k), v = NOD(a.p_v, k), d = NOD(a.p_div, k);
    const float ugl = (u * gx + v * gy) * sec2;
    const float ds = dsig(k);
    Fe += ugl * ds;
    Ff += (d + ugl) * ds;
    Su += u * ds;
    Sv += v * ds;
    if (moist) Gh += FB(a.o_gh, k);
  }
  float laplnps = 0.f;
  if (moist) laplnps = nod[((unsigned)a.p_laplnps + mb) * IJ + col];
  float lnps_n = 0.f, sin2 = 0.f, cos2 = 0.f, hs_e = 0.f;
  if (a.hs) {
    lnps_n = nod[((unsigned)a.p_lnps + mb) * IJ + col];
    sin2 = a.lat[2 * a.J + j];
    cos2 = a.lat[3 * a.J + j];
    hs_e = expf(kap * lnps_n);  // ps^kappa; (p / p0)^kappa = (sigma / p0)^kappa ps^kappa
  }

  float gxb = 0.f, gyb = 0.f, laplnpsb = 0.f, lnpsb = 0.f;
  float Feb = -fb[((unsigned)a.o_lnps + mb) * IJ + col], Ffb = 0.f;
  // Window: values of level k+1.
  float u_n = 0.f, v_n = 0.f, T_n = 0.f;
  float Vu_n = 0.f, Vv_n = 0.f, VT_n = 0.f, Tnb_n = 0.f;
  float ub_n = 0.f, vb_n = 0.f, Tb_n = 0.f;
  float q_n[kMaxTracers], Vq_n[kMaxTracers], qb_n[kMaxTracers];
#pragma unroll
  for (int t = 0; t < kMaxTracers; ++t) q_n[t] = Vq_n[t] = qb_n[t] = 0.f;
  float carry_fe = 0.f, carry_ff = 0.f;  // from ge/gf of level k+1
  float Se = 0.f, Sf = 0.f, SGh = 0.f;   // suffix sums
  float fe = Fe, ff = Ff;                // prefix sums through level k

  for (int k = K - 1; k >= 0; --k) {
    const bool has_next = k + 1 < K;
    const float u = NOD(a.p_u, k), v = NOD(a.p_v, k), d = NOD(a.p_div, k);
    const float z = NOD(a.p_vort, k), T = NOD(a.p_temp, k);
    float q[kMaxTracers];
    float q_h = 0.f;
#pragma unroll
    for (int t = 0; t < kMaxTracers; ++t) {
      q[t] = (t < a.nT) ? NOD(a.p_tr + t * a.mem * K, k) : 0.f;
      if (t == a.hum) q_h = q[t];
    }
    const float ugl = (u * gx + v * gy) * sec2;
    const float fe_k = fe, ff_k = ff;
    const float fe_km = fe_k - ugl * dsig(k);
    const float ff_km = ff_k - (d + ugl) * dsig(k);
    const float inv_ds = invds(k);
    const float trk = tref(k);

    const float Aub = FB(a.o_Au, k), Avb = FB(a.o_Av, k), KEb = FB(a.o_KE, k);
    const float uTb = FB(a.o_uT, k), vTb = FB(a.o_vT, k), Tnb = FB(a.o_Tn, k);
    const float adj = moist ? 1.f + ra * q_h : 1.f;
    const float rt = a.R * T * adj;
    const float tv = z + fcor;
    const float zb = sec2 * (-v * Aub + u * Avb);
    float ub = tv * sec2 * Avb + u * sec2 * KEb + T * sec2 * uTb;
    float vb = -tv * sec2 * Aub + v * sec2 * KEb + T * sec2 * vTb;
    if (a.hs) {
      const float kv = s_lev[4 * k + 2].x;
      ub += kv * sec2 * Aub;
      vb += kv * sec2 * Avb;
    }
    const float rtb = sec2 * (gx * Aub + gy * Avb);
    float Tb = a.R * adj * rtb + u * sec2 * uTb + v * sec2 * vTb + d * Tnb;
    float qhb = moist ? a.R * T * ra * rtb : 0.f;
    gxb += rt * sec2 * Aub;
    gyb += rt * sec2 * Avb;
    float db = T * Tnb;
    // Adiabatic term kappa (Tref (ugl - ge) + P (ugl - gf)).
    const float gf = (alpha(k) * ff_k + alpha_up(k) * ff_km) * inv_ds;
    float uglb = kap * trk * Tnb;
    const float geb = -kap * trk * Tnb;
    float gfb;
    if (!moist) {
      Tb += kap * (ugl - gf) * Tnb;
      uglb += kap * T * Tnb;
      gfb = -kap * T * Tnb;
    } else {
      const float den = 1.f + rb * q_h;
      const float P = (T * (1.f + ra * q_h) + trk * rc * q_h) / den;
      Tb += kap * (ugl - gf) * Tnb * (1.f + ra * q_h) / den;
      qhb += kap * (ugl - gf) * Tnb * (T * (ra - rb) + trk * rc) / (den * den);
      uglb += kap * P * Tnb;
      gfb = -kap * P * Tnb;
    }
    // Tracers.
    float qb[kMaxTracers], Vq[kMaxTracers];
#pragma unroll
    for (int t = 0; t < kMaxTracers; ++t) {
      qb[t] = 0.f;
      Vq[t] = 0.f;
      if (t < a.nT) {
        const int ob = a.o_tr + 3 * t * a.mem * K;
        const float uqb = FB(ob, k), vqb = FB(ob + a.mem * K, k);
        const float qnb = FB(ob + 2 * a.mem * K, k);
        ub += q[t] * sec2 * uqb;
        vb += q[t] * sec2 * vqb;
        qb[t] = u * sec2 * uqb + v * sec2 * vqb + d * qnb;
        db += q[t] * qnb;
        Vq[t] = a.vadv ? qnb : 0.f;
      }
    }
    if (moist) {
      const float gqx = NOD(a.p_gqx, k), gqy = NOD(a.p_gqy, k);
      const float vhb = FB(a.o_vh, k), dhb = FB(a.o_dh, k), ghb = FB(a.o_gh, k);
      const float coef = trk * a.Rv_minus_R;
      gxb += coef * sec2 * (gqy * vhb + gqx * dhb);
      gyb += coef * sec2 * (-gqx * vhb + gqy * dhb);
      XB(a.p_gqx, k) = coef * sec2 * (-gy * vhb + gx * dhb);
      XB(a.p_gqy, k) = coef * sec2 * (gx * vhb + gy * dhb);
      qhb += laplnps * coef * dhb;
      laplnpsb += q_h * coef * dhb;
      // Geopotential of the virtual-temperature difference.
      SGh += ghb;
      const float above = Gh - SGh;  // sum of the cotangents of levels < k
      const float tdb = a.R * alpha(k) * ghb +
                        (k > 0 ? a.R * (alpha(k) + alpha_up(k)) * above : 0.f);
      qhb += (T + trk) * ra * tdb;
      Tb += q_h * ra * tdb;
#pragma unroll
      for (int t = 0; t < kMaxTracers; ++t)
        if (t == a.hum) qb[t] += qhb;
    }
    if (a.hs) {
      const float hsTb = FB(a.o_hsT, k);
      const float4 c2 = s_lev[4 * k + 2];  // kv, cutoff, (sigma/p0)^kappa, log(sigma/p0)
      const float kt = a.hs_ka + (a.hs_ks - a.hs_ka) * (c2.y * cos2 * cos2);
      const float lp = c2.w + lnps_n;  // log(p / p0)
      const float pk = c2.z * hs_e;
      const float B = a.hs_maxT - a.hs_dTy * sin2 - a.hs_dThz * lp * cos2;
      Tb += -kt * hsTb;
      if (pk * B > a.hs_minT) lnpsb += kt * hsTb * pk * (kap * B - a.hs_dThz * cos2);
    }
    const float Vu = a.vadv ? -sec2 * Aub : 0.f;
    const float Vv = a.vadv ? -sec2 * Avb : 0.f;
    const float VT = a.vadv ? Tnb : 0.f;
    float fe_b = alpha(k) * inv_ds * geb + carry_fe;
    float ff_b = alpha(k) * inv_ds * gfb + carry_ff;
    if (has_next) {
      // Half level k+1/2.
      const float c = c2ci(k);
      const float ssk = sumsig(k);
      if (a.vadv) {
        const float wf = ssk * Ff - ff_k;
        float wfb = 0.f;
        auto half = [&](float xc, float xn, float Vc, float Vn, float& xbc, float& xbn) {
          const float vs = Vc + Vn;
          wfb += -0.5f * c * (xn - xc) * vs;
          const float Db = -0.5f * wf * vs;
          xbn += c * Db;
          xbc -= c * Db;
        };
        half(u, u_n, Vu, Vu_n, ub, ub_n);
        half(v, v_n, Vv, Vv_n, vb, vb_n);
        half(T, T_n, VT, VT_n, Tb, Tb_n);
#pragma unroll
        for (int t = 0; t < kMaxTracers; ++t)
          if (t < a.nT) half(q[t], q_n[t], Vq[t], Vq_n[t], qb[t], qb_n[t]);
        ff_b -= wfb;
        Ffb += ssk * wfb;
      }
      if (a.tref_varies) {
        const float web = -0.5f * trd(k) * (Tnb + Tnb_n);
        fe_b -= web;
        Feb += ssk * web;
      }
      // Level k+1 has all its contributions.
      XB(a.p_u, k + 1) = ub_n;
      XB(a.p_v, k + 1) = vb_n;
      XB(a.p_temp, k + 1) = Tb_n;
#pragma unroll
      for (int t = 0; t < kMaxTracers; ++t)
        if (t < a.nT) XB(a.p_tr + t * a.mem * K, k + 1) = qb_n[t];
    }
    Se += fe_b;
    Sf += ff_b;
    uglb += dsig(k) * (Se + Sf);
    db += dsig(k) * Sf;
    ub += gx * sec2 * uglb;
    vb += gy * sec2 * uglb;
    gxb += u * sec2 * uglb;
    gyb += v * sec2 * uglb;
    XB(a.p_vort, k) = zb;
    XB(a.p_div, k) = db;
    carry_fe = alpha_up(k) * inv_ds * geb;
    carry_ff = alpha_up(k) * inv_ds * gfb;
    u_n = u; v_n = v; T_n = T;
    Vu_n = Vu; Vv_n = Vv; VT_n = VT; Tnb_n = Tnb;
    ub_n = ub; vb_n = vb; Tb_n = Tb;
#pragma unroll
    for (int t = 0; t < kMaxTracers; ++t) {
      q_n[t] = q[t];
      Vq_n[t] = Vq[t];
      qb_n[t] = qb[t];
    }
    fe = fe_km;
    ff = ff_km;
  }
  XB(a.p_u, 0) = ub_n;
  XB(a.p_v, 0) = vb_n;
  XB(a.p_temp, 0) = Tb_n;
#pragma unroll
  for (int t = 0; t < kMaxTracers; ++t)
    if (t < a.nT) XB(a.p_tr + t * a.mem * K, 0) = qb_n[t];

  // Pass 2: cotangents of the column totals.
  const float Ftb = Feb + Ffb;
  for (int k = 0; k < K; ++k) {
    const float ds = dsig(k);
    XB(a.p_u, k) += gx * sec2 * ds * Ftb;
    XB(a.p_v, k) += gy * sec2 * ds * Ftb;
    XB(a.p_div, k) += ds * Ffb;
  }
  gxb += sec2 * Ftb * Su;
  gyb += sec2 * Ftb * Sv;
  xb[((unsigned)a.p_gx + mb) * IJ + col] = gxb;
  xb[((unsigned)a.p_gy + mb) * IJ + col] = gyb;
  if (moist) xb[((unsigned)a.p_laplnps + mb) * IJ + col] = laplnpsb;
  if (a.hs) xb[((unsigned)a.p_lnps + mb) * IJ + col] = lnpsb;
#undef NOD
#undef FB
#undef XB
}

// Transposed pre-pass: modal cotangents of the inverse-transform inputs
// (nodal-buffer plane order) -> cotangent of the packed state.
struct PrepAdjArgs {
  const float* xbar;
  float* sbar;
  int K, mem, nT, hum, hs;
  int M, L, lw;
  int p_u, p_v, p_gqx, p_gqy, p_gx, p_gy, p_laplnps, p_lnps;
  int s_lnps;
  const float* deriv;
  const float* lap;
  const float* invlap;
  float inv_radius;
};

__global__ void __launch_bounds__(kModalTX * kModalTY) pe_prep_adjoint_kernel(PrepAdjArgs a) {
  const int l = blockIdx.x * kModalTX + threadIdx.x;
  const int row = blockIdx.y * kModalTY + threadIdx.y;
  if (l >= a.L || row >= a.M) return;
  const size_t ML = (size_t)a.M * a.L;
  const size_t idx = (size_t)row * a.L + l;
  const int K = a.K;
  const int mK = a.mem * K;
  const float ir = a.inv_radius;
  const float s = a.invlap[l] * ir;
  const ModalNbrT nb(row, l, a.L, a.lw, a.deriv, 0, a.L);
  const int q0 = blockIdx.z * kPlanesPerThread;
  const int q1 = min(q0 + kPlanesPerThread, K * a.mem);
  for (int q = q0; q < q1; ++q) {
    const int mb = q / K, k = q - mb * K;
    const float* ub = a.xbar + pl(a.p_u, mb, K, k) * ML;
    const float* vb = a.xbar + pl(a.p_v, mb, K, k) * ML;
    const size_t pz = pl(0, mb, K, k) * ML + idx;
    a.sbar[pz] = a.xbar[pz] + s * (-nb.dlat_t(ub) - nb.dlon(vb));
    const size_t pd = pl(mK, mb, K, k) * ML + idx;
    a.sbar[pd] = a.xbar[pd] + s * (-nb.dlon(ub) + nb.dlat_t(vb));
    const size_t pt = pl(2 * mK, mb, K, k) * ML + idx;
    a.sbar[pt] = a.xbar[pt];
    for (int t = 0; t < a.nT; ++t) {
      const size_t pq = pl((3 + t) * mK, mb, K, k) * ML + idx;
      float v = a.xbar[pq];
      if (t == a.hum) {
        const float* gqxb = a.xbar + pl(a.p_gqx, mb, K, k) * ML;
        const float* gqyb = a.xbar + pl(a.p_gqy, mb, K, k) * ML;
        v += ir * (-nb.dlon(gqxb) + nb.dlat_t(gqyb));
      }
      a.sbar[pq] = v;
    }
    if (k == 0) {
      const float* gxb = a.xbar + ((size_t)a.p_gx + mb) * ML;
      const float* gyb = a.xbar + ((size_t)a.p_gy + mb) * ML;
      float v = a.hs ? a.xbar[((size_t)a.p_lnps + mb) * ML + idx] : 0.f;
      v += ir * (-nb.dlon(gxb) + nb.dlat_t(gyb));
      if (a.hum >= 0) v += a.lap[l] * a.xbar[((size_t)a.p_laplnps + mb) * ML + idx];
      a.sbar[((size_t)a.s_lnps + mb) * ML + idx] = v;
    }
  }
}

// out = sum_t c_t x_t over the packed state, with coefficients ci on the
// implicit planes (div, T', ln ps) and ce on the others; `filt` (per l)
// scales the result on the other planes; `only` restricts the planes written
// (0: all, 1: implicit, 2: others).
struct LinCombArgs {
  const float* x[6];
  float ci[6], ce[6];
  int nx;
  const float* filt;
  float* out;
  int mK, nT, L, only;
  size_t ML;
};

__global__ void pe_lincomb_kernel(LinCombArgs a) {
  const int plane = blockIdx.y;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.ML) return;
  const bool imp = (plane >= a.mK && plane < 3 * a.mK) || plane >= (3 + a.nT) * a.mK;
  if ((a.only == 1 && !imp) || (a.only == 2 && imp)) return;
  const size_t p = (size_t)plane * a.ML + idx;
  float v = 0.f;
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    const float c = imp ? a.ci[t] : a.ce[t];
    if (t < a.nx && c != 0.f) v = fmaf(c, a.x[t][p], v);
  }
  if (!imp && a.filt) v *= a.filt[idx % a.L];
  a.out[p] = v;
}

// ---------------------------------------------------------------------------
// Per-l operators of the implicit part, composed in FP64 on the GPU.
//
// On the stacked vector (div[K], T'[K], ln ps) of total wavenumber l the
// implicit terms are y -> L_l y (primitive_equations.py:1196-1249):
//   div rows  -lam_l (G T' + R Tref ln ps)
//   T' rows   -H div
//   ln ps     -dsig . div
// and implicit_inverse(eta) applies (I - eta L_l)^-1 (_get_implicit_term_
// matrix_sigma, :544-598, and :1251-1330).  The builder inverts I - eta L_l by
// Gauss-Jordan elimination with partial pivoting in FP64 (one CTA per l) and
// writes one FP32 operator per l, transposed ([column k][row r]) with rows
// zero-padded to the apply kernel's row tile:
//   kMatL      L_l
//   kMatInv    (I - eta L_l)^-1
//   kMatInvG   [(I - eta L_l)^-1 ; L_l (I - eta L_l)^-1]: the solution and its
//              implicit terms from one product
//   kMatFinal  f_l (I + eta L_l (I - eta L_l)^-1): the last SIL3 stage,
//              Y* + eta G(Y) with Y = (I - eta L_l)^-1 Y*, times the filter
// ---------------------------------------------------------------------------

enum MatKind { kMatL = 0, kMatInv = 1, kMatInvG = 2, kMatFinal = 3 };

constexpr int kMaxLevels = 48;

struct MatBuildArgs {
  int K, kind, RP, nin, transposed;
  double eta;
  const double* G;       // K x K
  const double* H;       // K x K
  const double* lcol;    // K: the ln ps column of L's divergence rows
  const double* trow;    // K: L's ln ps row (d ln ps / dt = -trow . div)
  const double* lam;     // L
  const double* filter;  // L, or null
  float* out;            // [L][n][RP]
  int* flag;
};

__global__ void pe_matrix_build_kernel(MatBuildArgs a) {
  extern __shared__ double aug[];  // n x 2n
  __shared__ double factor[2 * kMaxLevels + 1];
  __shared__ int piv;
  const int l = blockIdx.x;
  const int K = a.K, n = 2 * K + 1, n2 = 2 * n;
  const int tid = threadIdx.x, nt = blockDim.x;
  const double lm = a.lam[l];
  const double eta = a.eta;
  float* o = a.out + (size_t)l * a.nin * a.RP;
  auto Lrc = [&](int r, int c) -> double {
    if (r < K) {
      if (c < K) return 0.0;
      if (c < 2 * K) return -lm * a.G[r * K + (c - K)];
      return -lm * a.lcol[r];
    }
    if (r < 2 * K) return c < K ? -a.H[(r - K) * K + c] : 0.0;
    return c < K ? -a.trow[c] : 0.0;
  };
  if (a.kind == kMatL) {
    for (int e = tid; e < a.nin * a.RP; e += nt) {
      const int c = e / a.RP, r = e - c * a.RP;
      o[e] = r < n ? (float)(a.transposed ? Lrc(c, r) : Lrc(r, c)) : 0.f;
    }
    return;
  }
  for (int e = tid; e < n * n2; e += nt) {
    const int r = e / n2, c = e - r * n2;
    aug[e] = c >= n ? ((c - n == r) ? 1.0 : 0.0)
                    : ((r == c) ? 1.0 : 0.0) - eta * Lrc(r, c);
  }
  __syncthreads();
  for (int col = 0; col < n; ++col) {
    if (tid == 0) {
      int best = col;
      double bv = fabs(aug[col * n2 + col]);
      for (int r = col + 1; r < n; ++r) {
        const double v = fabs(aug[r * n2 + col]);
        if (v > bv) {
          bv = v;
          best = r;
        }
      }
      piv = best;
      if (!(bv > 0.0)) atomicExch(a.flag, 1);
    }
    __syncthreads();
    if (piv != col) {
      for (int c = tid; c < n2; c += nt) {
        const double t = aug[col * n2 + c];
        aug[col * n2 + c] = aug[piv * n2 + c];
        aug[piv * n2 + c] = t;
      }
    }
    __syncthreads();
    const double inv_p = 1.0 / aug[col * n2 + col];
    __syncthreads();
    for (int c = tid; c < n2; c += nt) aug[col * n2 + c] *= inv_p;
    for (int r = tid; r < n; r += nt) factor[r] = aug[r * n2 + col];
    __syncthreads();
    for (int e = tid; e < n * n2; e += nt) {
      const int r = e / n2, c = e - r * n2;
      if (r != col) aug[e] -= factor[r] * aug[col * n2 + c];
    }
    __syncthreads();
  }
  auto inv = [&](int r, int c) { return aug[r * n2 + n + c]; };
  auto l_inv = [&](int r, int c) -> double {
    double s = 0.0;
    if (r < K) {
      for (int j = 0; j < K; ++j) s += a.G[r * K + j] * inv(K + j, c);
      return -lm * (s + a.lcol[r] * inv(2 * K, c));
    }
    if (r < 2 * K) {
      for (int j = 0; j < K; ++j) s += a.H[(r - K) * K + j] * inv(j, c);
      return -s;
    }
    for (int j = 0; j < K; ++j) s += a.trow[j] * inv(j, c);
    return -s;
  };
  const double f = a.filter ? a.filter[l] : 1.0;
  // Entry (r, c) of the operator of `kind` (r < n, or r < 2n for kMatInvG).
  auto op = [&](int r, int c) -> double {
    if (a.kind == kMatInv) return inv(r, c);
    if (a.kind == kMatInvG) return r < n ? inv(r, c) : l_inv(r - n, c);
    return f * (((r == c) ? 1.0 : 0.0) + eta * l_inv(r, c));
  };
  const int rows = a.kind == kMatInvG ? 2 * n : n;
  for (int e = tid; e < a.nin * a.RP; e += nt) {
    const int c = e / a.RP, r = e - c * a.RP;
    double v = 0.0;
    if (a.transposed) {
      if (r < n && c < rows) v = op(c, r);
    } else if (r < rows) {
      v = op(r, c);
    }
    if (!isfinite(v)) atomicExch(a.flag, 2);
    o[e] = (float)v;
  }
}

// ---------------------------------------------------------------------------
// IMEX stage: an elementwise combine and a per-(m, l) implicit solve
// ---------------------------------------------------------------------------

// Y* = y0 + sum_t fc_t f_t + sum_t gc_t g_t over every plane of the packed
// state (g terms exist on the divergence, temperature and ln ps planes only).
// Planes without an implicit part (vorticity, tracers) are final after the
// combine: they go to `out` (times the per-l filter when given); the
// implicit planes go to `ystar` for the solve.
struct CombineArgs {
  const float* y0;
  const float* f[3];
  float fc[3];
  int nf;
  const float* g[2];
  float gc[2];
  int ng;
  const float* filter;
  float* out;
  float* ystar;
  int mK, nT, L;
  size_t ML;
};

__global__ void pe_combine_kernel(CombineArgs a) {
  const int plane = blockIdx.y;
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.ML) return;
  const bool implicit_plane =
      (plane >= a.mK && plane < 3 * a.mK) || plane >= (3 + a.nT) * a.mK;
  const size_t p = (size_t)plane * a.ML + idx;
  float v = a.y0[p];
#pragma unroll
  for (int t = 0; t < 3; ++t)
    if (t < a.nf) v = fmaf(a.fc[t], a.f[t][p], v);
  if (implicit_plane) {
#pragma unroll
    for (int t = 0; t < 2; ++t)
      if (t < a.ng) v = fmaf(a.gc[t], a.g[t][p], v);
    a.ystar[p] = v;
  } else {
    if (a.filter) v *= a.filter[idx % a.L];
    a.out[p] = v;
  }
}

// Per-(l, column) application of an implicit operator: for every total
// wavenumber l, Out[R x C] = A_l[R x nin] Ys[nin x C], where the C = members * M
// columns are the (member, m-row) pairs and Ys stacks the n = 2K+1 implicit
// planes (div, T', ln ps) of src (and, for nin = 2n, those of src2).
//
// The state keeps l fastest ([plane][row][l]), so the operands go through an
// l-major copy Y[l][k][c] (columns padded to Cp, a multiple of 64): a tiled
// shared-memory transpose in (pe_lm_gather_kernel), the per-l product on
// contiguous rows (pe_apply_kernel), and a tiled transpose out
// (pe_lm_scatter_kernel) -- every global access is a full 128-byte row.

struct LmArgs {
  const float* src;   // gather: stacked planes [0, n), scaled by s1
  const float* src2;  // gather: stacked planes [n, 2n), scaled by s2
  float s1, s2;
  float* out;         // scatter: rows [0, n)
  float* out2;        // scatter: rows [n, 2n)
  float* lm;          // gather output / scatter input: [L][nk][Cp]
  int nk, n, K, M, L, C, Cp;
  int p_div, p_temp, p_lnps;
  size_t ML;
};

__device__ __forceinline__ size_t stacked_plane(const LmArgs& a, int i, int mb) {
  if (i < a.K) return pl(a.p_div, mb, a.K, i);
  if (i < 2 * a.K) return pl(a.p_temp, mb, a.K, i - a.K);
  return (size_t)a.p_lnps + mb;
}

// One 32 (rows of one member) x 32 (l) tile of stacked plane k per CTA (256
// threads): blockIdx.y enumerates (member, row tile), so a tile never spans
// two members and the column c = member * M + row needs no division.
__global__ void __launch_bounds__(256) pe_lm_gather_kernel(LmArgs a) {
  __shared__ float tile[32][33];
  const int k = blockIdx.z;
  const int row_tiles = (a.M + 31) / 32;
  const int mb = blockIdx.y / row_tiles;
  const int row0 = (blockIdx.y - mb * row_tiles) * 32;
  const int l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const bool first = k < a.n;
  const int kk = first ? k : k - a.n;
  const float sc = first ? a.s1 : a.s2;
  const float* src = (first ? a.src : a.src2) + stacked_plane(a, kk, mb) * a.ML;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rr = ty + 8 * i, row = row0 + rr, l = l0 + tx;
    tile[rr][tx] = (row < a.M && l < a.L) ? sc * src[(size_t)row * a.L + l] : 0.f;
  }
  __syncthreads();
  const int row = row0 + tx;
  if (row >= a.M) return;
  float* dst = a.lm + (size_t)k * a.Cp + (size_t)mb * a.M + row;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int ll = ty + 8 * i, l = l0 + ll;
    if (l < a.L) dst[(size_t)l * a.nk * a.Cp] = tile[tx][ll];
  }
}

// Row r of the l-major product back into the state layout (rows [0, n) to
// out, [n, 2n) to out2), tiled like the gather.
__global__ void __launch_bounds__(256) pe_lm_scatter_kernel(LmArgs a) {
  __shared__ float tile[32][33];
  const int r = blockIdx.z;
  const int row_tiles = (a.M + 31) / 32;
  const int mb = blockIdx.y / row_tiles;
  const int row0 = (blockIdx.y - mb * row_tiles) * 32;
  const int l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  {
    const int row = row0 + tx;
    const float* srcp = a.lm + (size_t)r * a.Cp + (size_t)mb * a.M + row;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int ll = ty + 8 * i, l = l0 + ll;
      tile[ll][tx] = (l < a.L && row < a.M) ? srcp[(size_t)l * a.nk * a.Cp] : 0.f;
    }
  }
  __syncthreads();
  float* dst = (r < a.n ? a.out : a.out2) +
               stacked_plane(a, r < a.n ? r : r - a.n, mb) * a.ML;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rr = ty + 8 * i, row = row0 + rr, l = l0 + tx;
    if (row < a.M && l < a.L) dst[(size_t)row * a.L + l] = tile[tx][rr];
  }
}

struct ApplyArgs {
  const float* A;     // [L][nin][RP]: operator^T per l
  const float* ylm;   // [L][nin][Cp]
  float* olm;         // [L][R][Cp]
  int R, nin, RP, Cp;
};

constexpr int kApplyCols = 128;
constexpr int kApplyMaxTR = 9;

// A CTA takes one l, 128 columns and 16*TR rows of A_l: it stages A_l^T and
// the operand rows in shared memory and each thread accumulates a TR x 8
// register tile, columns 4 cg .. 4 cg + 3 and 64 + 4 cg .. 64 + 4 cg + 3
// (two conflict-free float4 operand reads per k, broadcast A reads, float4
// stores).
template <int TR>
__global__ void __launch_bounds__(256) pe_apply_kernel(ApplyArgs a) {
  constexpr int RPT = 16 * TR;
  constexpr int Q4 = kApplyCols / 4;  // float4 per operand row
  extern __shared__ __align__(16) float smem[];
  const int nin = a.nin;
  float* At = smem;                    // [nin][RPT]
  float* Ys = At + (size_t)nin * RPT;  // [nin][kApplyCols]
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * kApplyCols;
  const int l = blockIdx.y;
  const int r0 = blockIdx.z * RPT;
  {
    const float* Ag = a.A + (size_t)l * nin * a.RP + r0;
    constexpr int Q = RPT / 4;
    for (int e = tid; e < nin * Q; e += 256) {
      const int k = e / Q, q = e - k * Q;
      reinterpret_cast<float4*>(At)[e] =
          reinterpret_cast<const float4*>(Ag + (size_t)k * a.RP)[q];
    }
    const float* Yg = a.ylm + (size_t)l * nin * a.Cp + c0;
    for (int e = tid; e < nin * Q4; e += 256) {
      const int k = e / Q4, q = e - k * Q4;
      reinterpret_cast<float4*>(Ys)[e] =
          reinterpret_cast<const float4*>(Yg + (size_t)k * a.Cp)[q];
    }
  }
  __syncthreads();
  const int cg = tid & 15, rg = tid >> 4;
  float acc[TR][8];
#pragma unroll
  for (int i = 0; i < TR; ++i)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[i][c] = 0.f;
  const float* ar = At + rg * TR;
  const float4* yr = reinterpret_cast<const float4*>(Ys) + cg;
#pragma unroll 2
  for (int k = 0; k < nin; ++k) {
    const float4 y0 = yr[k * Q4];
    const float4 y1 = yr[k * Q4 + 16];
#pragma unroll
    for (int i = 0; i < TR; ++i) {
      const float av = ar[k * RPT + i];
      acc[i][0] = fmaf(av, y0.x, acc[i][0]);
      acc[i][1] = fmaf(av, y0.y, acc[i][1]);
      acc[i][2] = fmaf(av, y0.z, acc[i][2]);
      acc[i][3] = fmaf(av, y0.w, acc[i][3]);
      acc[i][4] = fmaf(av, y1.x, acc[i][4]);
      acc[i][5] = fmaf(av, y1.y, acc[i][5]);
      acc[i][6] = fmaf(av, y1.z, acc[i][6]);
      acc[i][7] = fmaf(av, y1.w, acc[i][7]);
    }
  }
  float* og = a.olm + (size_t)l * a.R * a.Cp + c0 + cg * 4;
#pragma unroll
  for (int i = 0; i < TR; ++i) {
    const int r = r0 + rg * TR + i;
    if (r < a.R) {
      float* o = og + (size_t)r * a.Cp;
      *reinterpret_cast<float4*>(o) = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
      *reinterpret_cast<float4*>(o + 64) =
          make_float4(acc[i][4], acc[i][5], acc[i][6], acc[i][7]);
    }
  }
}

// Rows per thread for an operator of R rows (one row tile while R <= 144).
static int apply_tr(int R) {
  int tr = (R + 15) / 16;
  return tr > kApplyMaxTR ? kApplyMaxTR : tr;
}

static size_t apply_smem(int n, int tr) {
  return sizeof(float) * (size_t)n * (16 * tr + kApplyCols);
}

template <int TR>
static int apply_attr() {
  DINO_CHECK_CUDA(cudaFuncSetAttribute(pe_apply_kernel<TR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)apply_smem(2 * (2 * kMaxLevels + 1), TR)));
  return DINO_OK;
}

// Sets the shared-memory attribute of every instantiation once per device
// (kept out of graph capture).
static int prepare_apply() {
  static PerDeviceOnce once;
  return once.run([] {
    DINO_TRY(apply_attr<1>());
    DINO_TRY(apply_attr<2>());
    DINO_TRY(apply_attr<3>());
    DINO_TRY(apply_attr<4>());
    DINO_TRY(apply_attr<5>());
    DINO_TRY(apply_attr<6>());
    DINO_TRY(apply_attr<7>());
    DINO_TRY(apply_attr<8>());
    DINO_TRY(apply_attr<9>());
    return DINO_OK;
  });
}

template <int TR>
static void apply_launch(dim3 grid, size_t smem, cudaStream_t st, const ApplyArgs& a) {
  pe_apply_kernel<TR><<<grid, 256, smem, st>>>(a);
}

static int launch_apply(dino_pe* pe, const MatEntry* m, const float* src,
                        float* out, float* out2, cudaStream_t st,
                        const float* src2 = nullptr, float s1 = 1.f, float s2 = 1.f) {
  LmArgs g{};
  g.src = src;
  g.src2 = src2;
  g.s1 = s1;
  g.s2 = s2;
  g.out = out;
  g.out2 = out2;
  g.n = 2 * pe->K + 1;
  g.K = pe->K;
  g.M = pe->M;
  g.L = pe->L;
  g.C = pe->mem * pe->M;
  g.Cp = pe->Cp;
  g.p_div = pe->mem * pe->K;
  g.p_temp = 2 * pe->mem * pe->K;
  g.p_lnps = (3 + pe->nT) * pe->mem * pe->K;
  g.ML = pe->ML;
  const dim3 tiles(ceil_div(pe->L, 32), ceil_div(pe->M, 32) * pe->mem);
  g.lm = pe->d_lm_in;
  g.nk = m->nin;
  pe_lm_gather_kernel<<<dim3(tiles.x, tiles.y, m->nin), 256, 0, st>>>(g);
  DINO_TRY(check_launch("pe_lm_gather"));
  ApplyArgs a{};
  a.A = m->d;
  a.ylm = pe->d_lm_in;
  a.olm = pe->d_lm_out;
  a.R = m->R;
  a.nin = m->nin;
  a.RP = m->RP;
  a.Cp = pe->Cp;
  const int tr = apply_tr(m->R);
  const int rpt = 16 * tr;
  dim3 grid(pe->Cp / kApplyCols, pe->L, ceil_div(m->R, rpt));
  const size_t smem = apply_smem(a.nin, tr);
  switch (tr) {
    case 1: apply_launch<1>(grid, smem, st, a); break;
    case 2: apply_launch<2>(grid, smem, st, a); break;
    case 3: apply_launch<3>(grid, smem, st, a); break;
    case 4: apply_launch<4>(grid, smem, st, a); break;
    case 5: apply_launch<5>(grid, smem, st, a); break;
    case 6: apply_launch<6>(grid, smem, st, a); break;
    case 7: apply_launch<7>(grid, smem, st, a); break;
    case 8: apply_launch<8>(grid, smem, st, a); break;
    default: apply_launch<9>(grid, smem, st, a); break;
  }
  DINO_TRY(check_launch("pe_apply"));
  g.lm = pe->d_lm_out;
  g.nk = m->R;
  pe_lm_scatter_kernel<<<dim3(tiles.x, tiles.y, m->R), 256, 0, st>>>(g);
  return check_launch("pe_lm_scatter");
}

struct Term {
  float c;
  const float* x;
};

static int launch_combine(dino_pe* pe, const float* y0,
                          std::initializer_list<Term> f,
                          std::initializer_list<Term> g, const float* filter,
                          float* out, cudaStream_t st) {
  CombineArgs a{};
  a.y0 = y0;
  for (const Term& t : f) {
    a.fc[a.nf] = t.c;
    a.f[a.nf++] = t.x;
  }
  for (const Term& t : g) {
    a.gc[a.ng] = t.c;
    a.g[a.ng++] = t.x;
  }
  a.filter = filter;
  a.out = out;
  a.ystar = pe->d_ystar;
  a.mK = pe->mem * pe->K;
  a.nT = pe->nT;
  a.L = pe->L;
  a.ML = pe->ML;
  dim3 grid(ceil_div((int)pe->ML, 256), pe->n_state);
  pe_combine_kernel<<<grid, 256, 0, st>>>(a);
  return check_launch("pe_combine");
}

static int get_matrix(dino_pe* pe, int kind, double eta, const double* host_filter,
                      const MatEntry** out, bool transposed = false) {
  const int K = pe->K, L = pe->L, n = 2 * K + 1;
  if (kind == kMatL) eta = 0.0;
  if (kind != kMatFinal) host_filter = nullptr;
  for (auto& e : pe->mat_cache) {
    if (e.kind != kind || e.eta != eta || e.transposed != transposed) continue;
    if (host_filter ? (e.filter.size() == (size_t)L &&
                       std::memcmp(e.filter.data(), host_filter, sizeof(double) * L) == 0)
                    : e.filter.empty()) {
      *out = &e;
      return DINO_OK;
    }
  }
  DINO_REQUIRE(K <= kMaxLevels, DINO_ERR_UNSUPPORTED, "implicit operators support up to 48 levels");
  DINO_TRY(prepare_apply());
  MatEntry m;
  m.kind = kind;
  m.eta = eta;
  if (host_filter) m.filter.assign(host_filter, host_filter + L);
  m.transposed = transposed;
  m.R = (kind == kMatInvG && !transposed) ? 2 * n : n;
  m.nin = (kind == kMatInvG && transposed) ? 2 * n : n;
  const int rpt = 16 * apply_tr(m.R);
  m.RP = ceil_div(m.R, rpt) * rpt;
  std::vector<double> lam(L);
  for (int l = 0; l < L; ++l)
    lam[l] = -(double)l * (l + 1) / (pe->plan->radius * pe->plan->radius);
  std::vector<double> consts;
  consts.insert(consts.end(), pe->G.begin(), pe->G.end());
  consts.insert(consts.end(), pe->H.begin(), pe->H.end());
  consts.insert(consts.end(), pe->imp_col.begin(), pe->imp_col.end());
  consts.insert(consts.end(), pe->imp_row.begin(), pe->imp_row.end());
  consts.insert(consts.end(), lam.begin(), lam.end());
  if (host_filter) consts.insert(consts.end(), host_filter, host_filter + L);
  double* dc = nullptr;
  auto build = [&]() -> int {
    DINO_CHECK_CUDA(cudaMalloc(&dc, sizeof(double) * consts.size()));
    DINO_CHECK_CUDA(cudaMemcpy(dc, consts.data(), sizeof(double) * consts.size(),
                               cudaMemcpyHostToDevice));
    DINO_CHECK_CUDA(cudaMalloc(&m.d, sizeof(float) * (size_t)L * m.nin * m.RP));
    DINO_CHECK_CUDA(cudaMemset(pe->d_flag, 0, sizeof(int)));
    MatBuildArgs b{};
    b.K = K;
    b.kind = kind;
    b.RP = m.RP;
    b.nin = m.nin;
    b.transposed = transposed ? 1 : 0;
    b.eta = eta;
    b.G = dc;
    b.H = dc + K * K;
    b.lcol = dc + 2 * K * K;
    b.trow = dc + 2 * K * K + K;
    b.lam = dc + 2 * K * K + 2 * K;
    b.filter = host_filter ? dc + 2 * K * K + 2 * K + L : nullptr;
    b.out = m.d;
    b.flag = pe->d_flag;
    const size_t smem = sizeof(double) * n * 2 * n;
    DINO_CHECK_CUDA(cudaFuncSetAttribute(pe_matrix_build_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    pe_matrix_build_kernel<<<L, 256, smem>>>(b);
    DINO_TRY(check_launch("pe_matrix_build"));
    int flag = 0;
    DINO_CHECK_CUDA(cudaMemcpy(&flag, pe->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    DINO_REQUIRE(flag == 0, DINO_ERR_NAN,
                 "implicit matrix is singular or its inverse is not finite");
    return DINO_OK;
  };
  const int rc = build();
  cudaFree(dc);
  if (rc != DINO_OK) {
    cudaFree(m.d);
    return rc;
  }
  pe->mat_cache.push_back(std::move(m));
  *out = &pe->mat_cache.back();
  return DINO_OK;
}

static int get_filter(dino_pe* pe, const double* host, float** out) {
  *out = nullptr;
  if (!host) return DINO_OK;
  for (auto& e : pe->filter_cache) {
    if (std::memcmp(e.host.data(), host, sizeof(double) * pe->L) == 0) {
      *out = e.d_filter;
      return DINO_OK;
    }
  }
  std::vector<float> f(pe->L);
  for (int l = 0; l < pe->L; ++l) f[l] = (float)host[l];
  float* d;
  DINO_CHECK_CUDA(cudaMalloc(&d, sizeof(float) * pe->L));
  DINO_CHECK_CUDA(cudaMemcpy(d, f.data(), sizeof(float) * pe->L, cudaMemcpyHostToDevice));
  pe->filter_cache.push_back({std::vector<double>(host, host + pe->L), d});
  *out = d;
  return DINO_OK;
}

// Modal pre-pass and inverse transforms: the nodal inputs of the column
// kernel in pe->d_nodal.
static int pe_nodal_inputs(dino_pe* pe, const float* state, cudaStream_t st) {
  dino_plan* p = pe->plan;
  const int K = pe->K, mem = pe->mem;
  const int mK = mem * K;
  // 1. modal pre-pass
  {
    PrepArgs a{};
    a.state = state;
    a.aux = pe->d_aux;
    a.K = K;
    a.mem = mem;
    a.nT = pe->nT;
    a.hum = pe->hum;
    a.M = pe->M;
    a.L = pe->L;
    a.lw = p->lw;
    a.p_vort = 0;
    a.p_div = mK;
    a.p_lnps = (3 + pe->nT) * mK;
    a.p_hum = pe->hum >= 0 ? (3 + pe->hum) * mK : 0;
    int q = 0;
    a.a_u = q; q += mK;
    a.a_v = q; q += mK;
    if (pe->hum >= 0) {
      a.a_gqx = q; q += mK;
      a.a_gqy = q; q += mK;
    }
    a.a_gx = q; q += mem;
    a.a_gy = q; q += mem;
    if (pe->hum >= 0) {
      a.a_laplnps = q; q += mem;
    }
    if (pe->hybrid) {
      a.a_lnpsdev = q; q += mem;
    }
    a.deriv = p->d_deriv;
    a.lap = p->d_lap;
    a.invlap = p->d_invlap;
    a.inv_radius = (float)(1.0 / p->radius);
    pe_prep_kernel<<<modal_grid(pe->M, pe->L, K * mem), dim3(kModalTX, kModalTY), 0, st>>>(a);
    DINO_TRY(check_launch("pe_prep"));
  }
  // 2. inverse SHT of [state kinds][aux][ln ps (Held-Suarez)]
  {
    Segs s{};
    s.n = 0;
    s.start[0] = 0;
    int acc = 0;
    s.ptr[s.n] = state;
    acc += (3 + pe->nT) * mK;
    s.start[++s.n] = acc;
    s.ptr[s.n] = pe->d_aux;
    acc += pe->n_aux;
    s.start[++s.n] = acc;
    if (pe->hs) {
      s.ptr[s.n] = state + (size_t)(3 + pe->nT) * mK * pe->ML;
      acc += mem;
      s.start[++s.n] = acc;
    }
    DINO_TRY(sht_inverse_segs(p, s, pe->d_nodal, pe->n_inv, pe->d_work,
                              pe->work_fields, st));
  }
  return DINO_OK;
}

// Level chunks per column for pe_nodal_kernel: the fewest (1, 2 or 4) that
// give about two waves of 16 warps per SM, keeping four or more levels a chunk.
static int nodal_chunks(const dino_pe* pe, int V) {
  const int64_t warps = (int64_t)ceil_div((int)(pe->IJ / V), kNodalCols) * pe->mem;
  int C = 1;
  while (2 * C <= kNodalMaxChunks && warps * C < 16LL * pe->sms && pe->K >= 8 * C) C *= 2;
  return C;
}

// Adjacent columns per thread for pe_nodal_kernel: two for dry states where
// the latitude count is even (122 registers; four need 188 and run slower),
// one with tracers (whose windows two columns would double).
static int nodal_vec(const dino_pe* pe) {
  return (pe->nT == 0 && pe->J % 2 == 0) ? 2 : 1;
}

static size_t nodal_smem(int K) { return (size_t)K * kLevPack * sizeof(float); }

// Opts every pe_nodal_kernel form into the level table's shared memory.
static int nodal_prepare(int K) {
  const size_t smem = nodal_smem(K);
  if (smem <= 48 * 1024) return DINO_OK;
  const int n = (int)smem;
  DINO_CHECK_CUDA(cudaFuncSetAttribute(pe_nodal_kernel<false, 1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, n));
  DINO_CHECK_CUDA(cudaFuncSetAttribute(pe_nodal_kernel<false, 2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, n));
  DINO_CHECK_CUDA(cudaFuncSetAttribute(pe_nodal_kernel<true, 1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, n));
  DINO_CHECK_CUDA(cudaFuncSetAttribute(pe_nodal_adjoint_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, n));
  return DINO_OK;
}

static NodalArgs make_nodal_args(dino_pe* pe);

static int launch_nodal_hybrid(dino_pe* pe, const float* state, cudaStream_t st) {
  const int K = pe->K, mK = pe->mem * K;
  HybridArgs a{};
  a.nod = pe->d_nodal;
  a.fwd = pe->d_fwd_in;
  a.lev = pe->d_hyb;
  a.lat = pe->d_lat;
  a.lnps_modal = state + (size_t)(3 + pe->nT) * mK * pe->ML;
  a.ML = (unsigned)pe->ML;
  a.K = K;
  a.mem = pe->mem;
  a.nT = pe->nT;
  a.hum = pe->hum_hyb;
  a.vadv = pe->vadv;
  a.tref_varies = pe->tref_varies;
  a.I = pe->I;
  a.J = pe->J;
  a.p_vort = 0;
  a.p_div = mK;
  a.p_temp = 2 * mK;
  a.p_tr = 3 * mK;
  a.p_u = pe->p_u;
  a.p_v = pe->p_v;
  a.p_gx = pe->p_gx;
  a.p_gy = pe->p_gy;
  a.p_lnps = pe->p_lnps;
  a.o_Au = pe->o_Au;
  a.o_Av = pe->o_Av;
  a.o_KE = pe->o_KE;
  a.o_uT = pe->o_uT;
  a.o_vT = pe->o_vT;
  a.o_Tn = pe->o_Tn;
  a.o_tr = pe->o_tr;
  a.o_lnps = pe->o_lnps;
  a.R = (float)pe->R;
  a.kappa = (float)pe->kappa;
  a.ps_ref = (float)pe->ps_ref;
  a.ln_ps_ref = std::log(pe->ps_ref);
  // The constant field 1 has the modal coefficient 2 sqrt(pi) at l = m = 0.
  a.inv_y00 = 0.5 / std::sqrt(3.14159265358979323846);
  a.Rv_over_R = (float)(pe->Rv / pe->R);
  a.Cpv_over_Cp = (float)(pe->Cpv / (pe->R / pe->kappa));
  const dim3 grid(ceil_div((int)pe->IJ, kHybThreads), pe->mem);
  const size_t smem = sizeof(float) * ((size_t)K * kHybPack + kHybTail +
                                       (size_t)(K + 1) * kHybThreads);
  pe_nodal_hybrid_kernel<<<grid, kHybThreads, smem, st>>>(a);
  return check_launch("pe_nodal_hybrid");
}
static int launch_nodal(dino_pe* pe, const float* state, cudaStream_t st) {
  if (pe->hybrid) return launch_nodal_hybrid(pe, state, st);
  const NodalArgs a = make_nodal_args(pe);
  const int V = nodal_vec(pe);
  const dim3 grid(ceil_div((int)(pe->IJ / V), kNodalCols), pe->mem);
  const dim3 block(kNodalCols, nodal_chunks(pe, V));
  const size_t smem = nodal_smem(pe->K);
  if (pe->nT > 0)
    pe_nodal_kernel<true, 1><<<grid, block, smem, st>>>(a);
  else if (V == 2)
    pe_nodal_kernel<false, 2><<<grid, block, smem, st>>>(a);
  else
    pe_nodal_kernel<false, 1><<<grid, block, smem, st>>>(a);
  return check_launch("pe_nodal");
}

static NodalArgs make_nodal_args(dino_pe* pe) {
  const int K = pe->K, mem = pe->mem;
  const int mK = mem * K;
  NodalArgs a{};
  {
    a.nod = pe->d_nodal;
    a.fwd = pe->d_fwd_in;
    a.K = K;
    a.mem = mem;
    a.nT = pe->nT;
    a.hum = pe->hum;
    a.vadv = pe->vadv;
    a.hs = pe->hs;
    a.tref_varies = pe->tref_varies;
    a.I = pe->I;
    a.J = pe->J;
    a.p_vort = 0;
    a.p_div = mK;
    a.p_temp = 2 * mK;
    a.p_tr = 3 * mK;
    a.p_u = pe->p_u;
    a.p_v = pe->p_v;
    a.p_gqx = pe->p_gqx;
    a.p_gqy = pe->p_gqy;
    a.p_gx = pe->p_gx;
    a.p_gy = pe->p_gy;
    a.p_laplnps = pe->p_laplnps;
    a.p_lnps = pe->p_lnps;
    a.o_Au = pe->o_Au;
    a.o_Av = pe->o_Av;
    a.o_KE = pe->o_KE;
    a.o_uT = pe->o_uT;
    a.o_vT = pe->o_vT;
    a.o_Tn = pe->o_Tn;
    a.o_tr = pe->o_tr;
    a.o_vh = pe->o_vh;
    a.o_gh = pe->o_gh;
    a.o_dh = pe->o_dh;
    a.o_hsT = pe->o_hsT;
    a.o_lnps = pe->o_lnps;
    a.levpack = pe->d_levpack;
    a.lat = pe->d_lat;
    a.R = (float)pe->R;
    a.kappa = (float)pe->kappa;
    a.Rv_over_R = (float)(pe->Rv / pe->R);
    a.Cpv_over_Cp = (float)(pe->Cpv / (pe->R / pe->kappa));
    a.Rv_minus_R = (float)(pe->Rv - pe->R);
    a.hs_p0 = (float)pe->hs_p0;
    a.hs_ka = (float)pe->hs_ka;
    a.hs_ks = (float)pe->hs_ks;
    a.hs_sigma_b = (float)pe->hs_sigma_b;
    a.hs_minT = (float)pe->hs_minT;
    a.hs_maxT = (float)pe->hs_maxT;
    a.hs_dTy = (float)pe->hs_dTy;
    a.hs_dThz = (float)pe->hs_dThz;
  }
  return a;
}

static int pe_explicit_impl(dino_pe* pe, const float* state, float* tend,
                            cudaStream_t st) {
  dino_plan* p = pe->plan;
  const int K = pe->K, mem = pe->mem;
  const int mK = mem * K;
  DINO_TRY(pe_nodal_inputs(pe, state, st));
  // 3. fused nodal column kernel
  {
    DINO_TRY(launch_nodal(pe, state, st));
  }
  // 4. forward SHT
  DINO_TRY(sht_forward_to(p, pe->d_fwd_in, pe->d_fwd_out, pe->n_fwd, pe->d_work,
                          pe->work_fields, st));
  // 5. modal post-pass
  {
    PostArgs a{};
    a.fm = pe->d_fwd_out;
    a.tend = tend;
    a.orog = pe->d_orog;
    a.K = K;
    a.mem = mem;
    a.nT = pe->nT;
    a.hum = pe->hum;
    a.hs = pe->hs;
    a.M = pe->M;
    a.L = pe->L;
    a.lw = p->lw;
    a.o_Au = pe->o_Au;
    a.o_Av = pe->o_Av;
    a.o_KE = pe->o_KE;
    a.o_uT = pe->o_uT;
    a.o_vT = pe->o_vT;
    a.o_Tn = pe->o_Tn;
    a.o_tr = pe->o_tr;
    a.o_vh = pe->o_vh;
    a.o_gh = pe->o_gh;
    a.o_dh = pe->o_dh;
    a.o_hsT = pe->o_hsT;
    a.o_lnps = pe->o_lnps;
    a.p_vort = 0;
    a.p_div = mK;
    a.p_temp = 2 * mK;
    a.p_tr = 3 * mK;
    a.p_lnps = (3 + pe->nT) * mK;
    a.deriv = p->d_deriv;
    a.lap = p->d_lap;
    a.inv_radius = (float)(1.0 / p->radius);
    a.gravity = (float)pe->g;
    pe_post_kernel<<<modal_grid(pe->M, pe->L, K * mem), dim3(kModalTX, kModalTY), 0, st>>>(a);
    DINO_TRY(check_launch("pe_post"));
  }
  return DINO_OK;
}

// One filtered imex_rk_sil3 step in place (time_integration.py:329-405 with
// the SIL3 tableau a_ex = [[1/3], [1/6, 1/2], [1/2, -1/2, 1]],
// a_im = [[1/6, 1/6], [1/3, 0, 1/3], [3/8, 0, 3/8, 1/4]]):
//   f0 = F(y), g0 = G(y)
//   Y1 = (1 - dt/6 G)^-1 (y + dt/3 f0 + dt/6 g0),            f1 = F(Y1)
//   Y2 = (1 - dt/3 G)^-1 (y + dt/6 f0 + dt/2 f1 + dt/3 g0),  f2 = F(Y2), g2 = G(Y2)
//   Y3* = y + dt/2 f0 - dt/2 f1 + dt f2 + 3dt/8 g0 + 3dt/8 g2
//   y_next = filter(Y3* + dt/4 G((1 - dt/4 G)^-1 Y3*))
// Each stage is one elementwise combine plus one per-l operator product.
struct StepMats {
  const MatEntry* L;      // G
  const MatEntry* inv1;   // (1 - dt/6 G)^-1
  const MatEntry* invg2;  // (1 - dt/3 G)^-1 and G of the result
  const MatEntry* fin3;   // filter (1 + dt/4 G (1 - dt/4 G)^-1)
};

static int get_step_mats(dino_pe* pe, double dt, const double* host_filter,
                         StepMats* m) {
  DINO_TRY(get_matrix(pe, kMatL, 0.0, nullptr, &m->L));
  DINO_TRY(get_matrix(pe, kMatInv, dt / 6.0, nullptr, &m->inv1));
  DINO_TRY(get_matrix(pe, kMatInvG, dt / 3.0, nullptr, &m->invg2));
  DINO_TRY(get_matrix(pe, kMatFinal, dt / 4.0, host_filter, &m->fin3));
  return DINO_OK;
}

static int pe_step_once(dino_pe* pe, float* y, double dt, const float* filt,
                        const StepMats& m, cudaStream_t st) {
  DINO_TRY(pe_explicit_impl(pe, y, pe->d_f[0], st));
  DINO_TRY(launch_apply(pe, m.L, y, pe->d_g[0], nullptr, st));
  DINO_TRY(launch_combine(pe, y, {{(float)(dt / 3.0), pe->d_f[0]}},
                          {{(float)(dt / 6.0), pe->d_g[0]}}, nullptr, pe->d_Y, st));
  DINO_TRY(launch_apply(pe, m.inv1, pe->d_ystar, pe->d_Y, nullptr, st));
  DINO_TRY(pe_explicit_impl(pe, pe->d_Y, pe->d_f[1], st));
  DINO_TRY(launch_combine(
      pe, y, {{(float)(dt / 6.0), pe->d_f[0]}, {(float)(dt * 0.5), pe->d_f[1]}},
      {{(float)(dt / 3.0), pe->d_g[0]}}, nullptr, pe->d_Y, st));
  DINO_TRY(launch_apply(pe, m.invg2, pe->d_ystar, pe->d_Y, pe->d_g[1], st));
  DINO_TRY(pe_explicit_impl(pe, pe->d_Y, pe->d_f[2], st));
  DINO_TRY(launch_combine(
      pe, y,
      {{(float)(dt * 0.5), pe->d_f[0]}, {(float)(dt * -0.5), pe->d_f[1]},
       {(float)dt, pe->d_f[2]}},
      {{(float)(dt * 0.375), pe->d_g[0]}, {(float)(dt * 0.375), pe->d_g[1]}},
      filt, y, st));
  DINO_TRY(launch_apply(pe, m.fin3, pe->d_ystar, y, nullptr, st));
  return DINO_OK;
}


// ---------------------------------------------------------------------------
// Reverse mode
// ---------------------------------------------------------------------------

static int pe_ensure_adjoint(dino_pe* pe) {
  if (pe->d_xbar_n) return DINO_OK;
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_xbar_n, sizeof(float) * pe->n_inv * pe->IJ));
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_xbar_m, sizeof(float) * pe->n_inv * pe->ML));
  for (auto*& b : pe->d_adj)
    DINO_CHECK_CUDA(cudaMalloc(&b, sizeof(float) * pe->n_state * pe->ML));
  return DINO_OK;
}

// state_ct = (d explicit_terms / d state)^T tend_ct at `state`.
static int pe_explicit_vjp_impl(dino_pe* pe, const float* state, const float* tbar,
                                float* sbar, cudaStream_t st) {
  dino_plan* p = pe->plan;
  const int K = pe->K, mem = pe->mem, mK = mem * K;
  DINO_TRY(pe_nodal_inputs(pe, state, st));
  {
    PostAdjArgs a{};
    a.tbar = tbar;
    a.fbar = pe->d_fwd_out;
    a.K = K;
    a.mem = mem;
    a.nT = pe->nT;
    a.hum = pe->hum;
    a.hs = pe->hs;
    a.M = pe->M;
    a.L = pe->L;
    a.lw = p->lw;
    a.o_Au = pe->o_Au;
    a.o_Av = pe->o_Av;
    a.o_KE = pe->o_KE;
    a.o_uT = pe->o_uT;
    a.o_vT = pe->o_vT;
    a.o_Tn = pe->o_Tn;
    a.o_tr = pe->o_tr;
    a.o_vh = pe->o_vh;
    a.o_gh = pe->o_gh;
    a.o_dh = pe->o_dh;
    a.o_hsT = pe->o_hsT;
    a.o_lnps = pe->o_lnps;
    a.p_vort = 0;
    a.p_div = mK;
    a.p_temp = 2 * mK;
    a.p_tr = 3 * mK;
    a.p_lnps = (3 + pe->nT) * mK;
    a.deriv = p->d_deriv;
    a.lap = p->d_lap;
    a.inv_radius = (float)(1.0 / p->radius);
    pe_post_adjoint_kernel<<<modal_grid(pe->M, pe->L, K * mem), dim3(kModalTX, kModalTY), 0,
                             st>>>(a);
    DINO_TRY(check_launch("pe_post_adjoint"));
  }
  DINO_TRY(sht_forward_adjoint_to(p, pe->d_fwd_out, pe->d_fwd_in, pe->n_fwd,
                                  pe->d_work, pe->work_fields, st));
  {
    NodalAdjArgs a{};
    a.f = make_nodal_args(pe);
    a.fbar = pe->d_fwd_in;
    a.xbar = pe->d_xbar_n;
    dim3 grid(ceil_div((int)pe->IJ, 128), mem);
    pe_nodal_adjoint_kernel<<<grid, 128, nodal_smem(K), st>>>(a);
    DINO_TRY(check_launch("pe_nodal_adjoint"));
  }
  DINO_TRY(sht_inverse_adjoint_to(p, pe->d_xbar_n, pe->d_xbar_m, pe->n_inv,
                                  pe->d_work, pe->work_fields, st));
  {
    PrepAdjArgs a{};
    a.xbar = pe->d_xbar_m;
    a.sbar = sbar;
    a.K = K;
    a.mem = mem;
    a.nT = pe->nT;
    a.hum = pe->hum;
    a.hs = pe->hs;
    a.M = pe->M;
    a.L = pe->L;
    a.lw = p->lw;
    a.p_u = pe->p_u;
    a.p_v = pe->p_v;
    a.p_gqx = pe->p_gqx;
    a.p_gqy = pe->p_gqy;
    a.p_gx = pe->p_gx;
    a.p_gy = pe->p_gy;
    a.p_laplnps = pe->p_laplnps;
    a.p_lnps = pe->p_lnps;
    a.s_lnps = (3 + pe->nT) * mK;
    a.deriv = p->d_deriv;
    a.lap = p->d_lap;
    a.invlap = p->d_invlap;
    a.inv_radius = (float)(1.0 / p->radius);
    pe_prep_adjoint_kernel<<<modal_grid(pe->M, pe->L, K * mem), dim3(kModalTX, kModalTY), 0,
                             st>>>(a);
    DINO_TRY(check_launch("pe_prep_adjoint"));
  }
  return DINO_OK;
}

struct LinTerm {
  const float* x;
  float ci, ce;
};

static int launch_lincomb(dino_pe* pe, std::initializer_list<LinTerm> terms,
                          const float* filt, float* out, int only, cudaStream_t st) {
  LinCombArgs a{};
  for (const LinTerm& t : terms) {
    a.x[a.nx] = t.x;
    a.ci[a.nx] = t.ci;
    a.ce[a.nx] = t.ce;
    ++a.nx;
  }
  a.filt = filt;
  a.out = out;
  a.mK = pe->mem * pe->K;
  a.nT = pe->nT;
  a.L = pe->L;
  a.only = only;
  a.ML = pe->ML;
  dim3 grid(ceil_div((int)pe->ML, 256), pe->n_state);
  pe_lincomb_kernel<<<grid, 256, 0, st>>>(a);
  return check_launch("pe_lincomb");
}

struct StepMatsT {
  const MatEntry* L;      // G^T
  const MatEntry* inv1;   // ((1 - dt/6 G)^-1)^T
  const MatEntry* invg2;  // [(1 - dt/3 G)^-1 ; G (1 - dt/3 G)^-1]^T
  const MatEntry* fin3;   // (filter (1 + dt/4 G (1 - dt/4 G)^-1))^T
};

static int get_step_mats_t(dino_pe* pe, double dt, const double* host_filter,
                           StepMatsT* m) {
  DINO_TRY(get_matrix(pe, kMatL, 0.0, nullptr, &m->L, true));
  DINO_TRY(get_matrix(pe, kMatInv, dt / 6.0, nullptr, &m->inv1, true));
  DINO_TRY(get_matrix(pe, kMatInvG, dt / 3.0, nullptr, &m->invg2, true));
  DINO_TRY(get_matrix(pe, kMatFinal, dt / 4.0, host_filter, &m->fin3, true));
  return DINO_OK;
}

// VJP of one filtered SIL3 step at y: in_ct = (d step / d y)^T out_ct.  The
// stage states Y1, Y2 are recomputed from y; the reverse sweep follows the
// forward tableau (see pe_step_once):
//   Z3 = Fin3^T out_ct (implicit planes), filter * out_ct (others)
//   V2 = F'(Y2)^T (dt Z3);           Z2 = [Inv2; G Inv2]^T [V2; 3dt/8 Z3]
//   V1 = F'(Y1)^T (dt/2 (Z2 - Z3));  Z1 = Inv1^T V1
//   V0 = F'(y)^T (dt/2 Z3 + dt/6 Z2 + dt/3 Z1)
//   in_ct = Z1 + Z2 + Z3 + V0 + G^T (3dt/8 Z3 + dt/3 Z2 + dt/6 Z1)
// (Inv_i act on the implicit planes only; elsewhere they are the identity.)
static int pe_step_vjp_impl(dino_pe* pe, const float* y, const float* out_ct,
                            float* in_ct, double dt, const float* filt,
                            const StepMats& m, const StepMatsT& mt, cudaStream_t st) {
  float* Y1 = pe->d_adj[0];
  float* Y2 = pe->d_adj[1];
  float* Z1 = pe->d_adj[2];
  float* Z2 = pe->d_adj[3];
  float* Z3 = pe->d_adj[4];
  float* V = pe->d_adj[5];
  const float fdt = (float)dt;
  // Stage states.
  DINO_TRY(pe_explicit_impl(pe, y, pe->d_f[0], st));
  DINO_TRY(launch_apply(pe, m.L, y, pe->d_g[0], nullptr, st));
  DINO_TRY(launch_combine(pe, y, {{(float)(dt / 3.0), pe->d_f[0]}},
                          {{(float)(dt / 6.0), pe->d_g[0]}}, nullptr, Y1, st));
  DINO_TRY(launch_apply(pe, m.inv1, pe->d_ystar, Y1, nullptr, st));
  DINO_TRY(pe_explicit_impl(pe, Y1, pe->d_f[1], st));
  DINO_TRY(launch_combine(
      pe, y, {{(float)(dt / 6.0), pe->d_f[0]}, {(float)(dt * 0.5), pe->d_f[1]}},
      {{(float)(dt / 3.0), pe->d_g[0]}}, nullptr, Y2, st));
  DINO_TRY(launch_apply(pe, m.invg2, pe->d_ystar, Y2, pe->d_g[1], st));
  // Reverse sweep.
  float* C = pe->d_f[0];
  DINO_TRY(launch_apply(pe, mt.fin3, out_ct, Z3, nullptr, st));
  DINO_TRY(launch_lincomb(pe, {{out_ct, 0.f, 1.f}}, filt, Z3, 2, st));
  DINO_TRY(launch_lincomb(pe, {{Z3, fdt, fdt}}, nullptr, C, 0, st));
  DINO_TRY(pe_explicit_vjp_impl(pe, Y2, C, V, st));
  DINO_TRY(launch_apply(pe, mt.invg2, V, Z2, nullptr, st, Z3, 1.f,
                        (float)(dt * 0.375)));
  DINO_TRY(launch_lincomb(pe, {{V, 0.f, 1.f}}, nullptr, Z2, 2, st));
  const float h = (float)(dt * 0.5);
  DINO_TRY(launch_lincomb(pe, {{Z3, -h, -h}, {Z2, h, h}}, nullptr, C, 0, st));
  DINO_TRY(pe_explicit_vjp_impl(pe, Y1, C, V, st));
  DINO_TRY(launch_apply(pe, mt.inv1, V, Z1, nullptr, st));
  DINO_TRY(launch_lincomb(pe, {{V, 0.f, 1.f}}, nullptr, Z1, 2, st));
  const float c3 = (float)(dt * 0.5), c2 = (float)(dt / 6.0), c1 = (float)(dt / 3.0);
  DINO_TRY(launch_lincomb(pe, {{Z3, c3, c3}, {Z2, c2, c2}, {Z1, c1, c1}}, nullptr, C,
                          0, st));
  DINO_TRY(pe_explicit_vjp_impl(pe, y, C, V, st));
  float* Gb = pe->d_f[1];
  float* Tt = pe->d_f[2];
  DINO_TRY(launch_lincomb(pe,
                          {{Z3, (float)(dt * 0.375), 0.f},
                           {Z2, (float)(dt / 3.0), 0.f},
                           {Z1, (float)(dt / 6.0), 0.f}},
                          nullptr, Gb, 1, st));
  DINO_TRY(launch_apply(pe, mt.L, Gb, Tt, nullptr, st));
  DINO_TRY(launch_lincomb(pe,
                          {{Z1, 1.f, 1.f}, {Z2, 1.f, 1.f}, {Z3, 1.f, 1.f},
                           {V, 1.f, 1.f}, {Tt, 1.f, 0.f}},
                          nullptr, in_ct, 0, st));
  return DINO_OK;
}

template <typename T>
static int upload_vec(T** dst, const std::vector<T>& v) {
  DINO_CHECK_CUDA(cudaMalloc((void**)dst, sizeof(T) * (v.empty() ? 1 : v.size())));
  if (!v.empty())
    DINO_CHECK_CUDA(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return DINO_OK;
}

static void pe_free(dino_pe* pe) {
  if (!pe) return;
  if (pe->graph.exec) cudaGraphExecDestroy(pe->graph.exec);
  if (pe->graph.graph) cudaGraphDestroy(pe->graph.graph);
  for (auto& e : pe->mat_cache) cudaFree(e.d);
  for (auto& e : pe->filter_cache) cudaFree(e.d_filter);
  cudaFree(pe->d_levpack);
  cudaFree(pe->d_hyb);
  cudaFree(pe->d_lat);
  cudaFree(pe->d_orog);
  cudaFree(pe->d_aux);
  cudaFree(pe->d_nodal);
  cudaFree(pe->d_fwd_in);
  cudaFree(pe->d_fwd_out);
  cudaFree(pe->d_work);
  for (auto* f : pe->d_f) cudaFree(f);
  for (auto* g : pe->d_g) cudaFree(g);
  cudaFree(pe->d_Y);
  cudaFree(pe->d_ystar);
  cudaFree(pe->d_lm_in);
  cudaFree(pe->d_lm_out);
  cudaFree(pe->d_xbar_n);
  cudaFree(pe->d_xbar_m);
  for (auto* b : pe->d_adj) cudaFree(b);
  cudaFree(pe->d_flag);
  delete pe;
}

static int pe_build(dino_pe* pe, const dino_pe_desc* d) {
  dino_plan* p = pe->plan;
  const int K = pe->K, mem = pe->mem, nT = pe->nT, J = pe->J;
  const int mK = mem * K;
  pe->dsig.assign(d->layer_thickness, d->layer_thickness + K);
  pe->c2c.assign(d->inv_center_to_center, d->inv_center_to_center + (K > 1 ? K - 1 : 0));
  pe->alpha.assign(d->sigma_ratios, d->sigma_ratios + K);
  pe->tref.assign(d->reference_temperature, d->reference_temperature + K);
  pe->sigma.assign(d->sigma_centers, d->sigma_centers + K);
  pe->G.assign(d->geopotential_weights, d->geopotential_weights + K * K);
  pe->H.assign(d->temperature_weights, d->temperature_weights + K * K);
  pe->sumsig.resize(K);
  double acc = 0.0;
  for (int k = 0; k < K; ++k) {
    acc += pe->dsig[k];
    pe->sumsig[k] = acc;
  }
  pe->tref_varies = 0;
  for (int k = 1; k < K; ++k)
    if (pe->tref[k] != pe->tref[0]) pe->tref_varies = 1;
  pe->imp_col.resize(K);
  pe->imp_row.resize(K);
  for (int k = 0; k < K; ++k) {
    pe->imp_col[k] = d->implicit_lnps_column ? d->implicit_lnps_column[k] : pe->R * pe->tref[k];
    pe->imp_row[k] = d->implicit_thickness ? d->implicit_thickness[k] : pe->dsig[k];
  }
  if (pe->hybrid) {
    // pe_nodal_hybrid_kernel's level constants at p_s_ref, in FP64: alpha and
    // the log pressure ratio as _get_vertical_discretization_coeffs_numpy
    // (primitive_equations.py:1483-1504) forms them, W and W p_s / dp
    // (_get_pgf_lps_coefficient_numpy, :1859-1887).
    const double* A = d->hybrid_a_boundaries;
    const double* B = d->hybrid_b_boundaries;
    const double psr = pe->ps_ref;
    std::vector<float> hp((size_t)K * kHybPack + kHybTail, 0.f);
    for (int k = 0; k < K; ++k) {
      const double pu = A[k] + B[k] * psr, pd = A[k + 1] + B[k + 1] * psr;
      DINO_REQUIRE(pd - pu > 0, DINO_ERR_ARG, "Pressure must decrease monotonically with height.");
      const double lr = std::log(std::max(pd, 1e-6 * psr) / std::max(pu, 1e-6 * psr));
      const double al = 1.0 - (pu / (pd - pu)) * lr;
      const double da = A[k + 1] - A[k], db = B[k + 1] - B[k];
      const double dp = da + db * psr;
      const double W = lr * B[k] + al * db;
      float* q = hp.data() + (size_t)k * kHybPack;
      q[0] = (float)A[k];
      q[1] = (float)B[k];
      q[2] = (float)da;
      q[3] = (float)db;
      q[4] = (float)pe->tref[k];
      q[5] = (float)al;
      q[6] = (float)lr;
      q[7] = (float)(W * psr / std::max(dp, 1e-6 * psr));
      q[8] = (float)pu;
      q[9] = (float)dp;
      q[10] = (float)W;
      q[11] = (float)(1.0 / dp);
      q[12] = (float)(1.0 / std::max(pu, 1e-6 * psr));
      q[13] = (float)(B[k] / std::max(pu, 1e-6 * psr));
    }
    const double pK = A[K] + B[K] * psr;
    hp[(size_t)K * kHybPack] = (float)A[K];
    hp[(size_t)K * kHybPack + 1] = (float)B[K];
    hp[(size_t)K * kHybPack + 2] = (float)pK;
    hp[(size_t)K * kHybPack + 3] = (float)(1.0 / std::max(pK, 1e-6 * psr));
    hp[(size_t)K * kHybPack + 4] = (float)(B[K] / std::max(pK, 1e-6 * psr));
    DINO_TRY(upload_vec(&pe->d_hyb, hp));
  }

  // Level constants.
  LevOff lo = lev_offsets(K);
  std::vector<float> lev(lo.total, 0.f);
  for (int k = 0; k < K; ++k) {
    lev[lo.dsig + k] = (float)pe->dsig[k];
    lev[lo.alpha + k] = (float)pe->alpha[k];
    lev[lo.tref + k] = (float)pe->tref[k];
    lev[lo.sumsig + k] = (float)pe->sumsig[k];
    lev[lo.sigma + k] = (float)pe->sigma[k];
    double cut = (pe->sigma[k] - pe->hs_sigma_b) / (1.0 - pe->hs_sigma_b);
    lev[lo.kv + k] = (float)(pe->hs_kf * (cut > 0 ? cut : 0.0));
    if (pe->hs_p0 > 0) lev[lo.logsp0 + k] = (float)std::log(pe->sigma[k] / pe->hs_p0);
    if (k + 1 < K) {
      // center_to_center arrives already as the reference's 1/x operand.
      lev[lo.c2ci + k] = (float)pe->c2c[k];
      lev[lo.trefdiff + k] = (float)((pe->tref[k + 1] - pe->tref[k]) * pe->c2c[k]);
    }
  }
  // The same constants packed per level for pe_nodal_kernel (kLevPack).
  std::vector<float> pack((size_t)K * kLevPack, 0.f);
  for (int k = 0; k < K; ++k) {
    float* q = pack.data() + (size_t)k * kLevPack;
    const double cut = std::max(0.0, (pe->sigma[k] - pe->hs_sigma_b) / (1.0 - pe->hs_sigma_b));
    q[0] = lev[lo.dsig + k];
    q[1] = (float)(1.0 / pe->dsig[k]);
    q[2] = lev[lo.sumsig + k];
    q[3] = lev[lo.tref + k];
    q[4] = lev[lo.c2ci + k];
    q[5] = k > 0 ? lev[lo.c2ci + k - 1] : 0.f;
    q[6] = lev[lo.alpha + k];
    q[7] = k > 0 ? lev[lo.alpha + k - 1] : 0.f;
    q[8] = lev[lo.kv + k];
    q[9] = (float)cut;
    if (pe->hs_p0 > 0) {
      const double lsp = std::log(pe->sigma[k] / pe->hs_p0);
      q[10] = (float)std::exp(pe->kappa * lsp);
      q[11] = (float)lsp;
    }
    q[12] = lev[lo.trefdiff + k];
    q[13] = k > 0 ? lev[lo.trefdiff + k - 1] : 0.f;
  }
  DINO_TRY(upload_vec(&pe->d_levpack, pack));
  DINO_TRY(nodal_prepare(K));
  {
    int dev = 0;
    DINO_CHECK_CUDA(cudaGetDevice(&dev));
    DINO_CHECK_CUDA(cudaDeviceGetAttribute(&pe->sms, cudaDevAttrMultiProcessorCount, dev));
  }
  // Latitude constants: sec^2, Coriolis 2 Omega sin, sin^2, cos^2.
  std::vector<float> lat(4 * J);
  for (int j = 0; j < J; ++j) {
    double s = p->h_x64[j];
    lat[j] = (float)(1.0 / (1.0 - s * s));
    lat[J + j] = (float)(2.0 * pe->Omega * s);
    double latr = std::asin(s);
    lat[2 * J + j] = (float)(std::sin(latr) * std::sin(latr));
    lat[3 * J + j] = (float)(std::cos(latr) * std::cos(latr));
  }
  DINO_TRY(upload_vec(&pe->d_lat, lat));
  {
    std::vector<float> orog(pe->ML, 0.f);
    if (d->orography_modal) std::memcpy(orog.data(), d->orography_modal, sizeof(float) * pe->ML);
    DINO_TRY(upload_vec(&pe->d_orog, orog));
  }

  // Field bookkeeping.
  const bool moist = pe->hum >= 0;
  pe->n_state = (3 + nT) * mK + mem;
  // Hybrid levels add ln p_s without its l = 0 term to the aux planes.
  pe->n_aux = 2 * mK + (moist ? 2 * mK : 0) + 2 * mem + (moist ? mem : 0) +
              (pe->hybrid ? mem : 0);
  pe->n_inv = (3 + nT) * mK + pe->n_aux + (pe->hs ? mem : 0);
  {
    int q = (3 + nT) * mK;  // nodal planes follow the inverse field order
    pe->p_u = q; q += mK;
    pe->p_v = q; q += mK;
    if (moist) {
      pe->p_gqx = q; q += mK;
      pe->p_gqy = q; q += mK;
    }
    pe->p_gx = q; q += mem;
    pe->p_gy = q; q += mem;
    if (moist) {
      pe->p_laplnps = q; q += mem;
    }
    if (pe->hybrid || pe->hs) {
      // hybrid: the deviation plane (aux); Held-Suarez: ln p_s itself
      pe->p_lnps = q; q += mem;
    }
  }
  {
    int q = 0;
    pe->o_Au = q; q += mK;
    pe->o_Av = q; q += mK;
    pe->o_KE = q; q += mK;
    pe->o_uT = q; q += mK;
    pe->o_vT = q; q += mK;
    pe->o_Tn = q; q += mK;
    pe->o_tr = q; q += 3 * nT * mK;
    if (moist) {
      pe->o_vh = q; q += mK;
      pe->o_gh = q; q += mK;
      pe->o_dh = q; q += mK;
    }
    if (pe->hs) {
      pe->o_hsT = q; q += mK;
    }
    pe->o_lnps = q; q += mem;
    pe->n_fwd = q;
  }
  const size_t ML = pe->ML, IJ = pe->IJ;
  // The nodal kernels address these buffers with 32-bit offsets.
  DINO_REQUIRE((uint64_t)pe->n_inv * IJ < (1ull << 32) && (uint64_t)pe->n_fwd * IJ < (1ull << 32),
               DINO_ERR_UNSUPPORTED, "nodal buffers must hold fewer than 2^32 values");
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_aux, sizeof(float) * pe->n_aux * ML));
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_nodal, sizeof(float) * pe->n_inv * IJ));
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_fwd_in, sizeof(float) * pe->n_fwd * IJ));
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_fwd_out, sizeof(float) * pe->n_fwd * ML));
  pe->work_fields = pe->n_inv > pe->n_fwd ? pe->n_inv : pe->n_fwd;
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_work, sizeof(float) * (size_t)pe->work_fields * p->M * p->J));
  for (auto*& f : pe->d_f) DINO_CHECK_CUDA(cudaMalloc(&f, sizeof(float) * pe->n_state * ML));
  for (auto*& g : pe->d_g) DINO_CHECK_CUDA(cudaMalloc(&g, sizeof(float) * pe->n_state * ML));
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_Y, sizeof(float) * pe->n_state * ML));
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_ystar, sizeof(float) * pe->n_state * ML));
  pe->Cp = ceil_div(pe->mem * pe->M, kApplyCols) * kApplyCols;
  {
    const size_t lm = (size_t)pe->L * 2 * (2 * K + 1) * pe->Cp;
    DINO_CHECK_CUDA(cudaMalloc(&pe->d_lm_in, sizeof(float) * lm));
    DINO_CHECK_CUDA(cudaMalloc(&pe->d_lm_out, sizeof(float) * lm));
    DINO_CHECK_CUDA(cudaMemset(pe->d_lm_in, 0, sizeof(float) * lm));
    DINO_CHECK_CUDA(cudaMemset(pe->d_lm_out, 0, sizeof(float) * lm));
  }
  DINO_CHECK_CUDA(cudaMalloc(&pe->d_flag, sizeof(int)));
  DINO_CHECK_CUDA(cudaDeviceSynchronize());
  return DINO_OK;
}

}  // namespace dino

using namespace dino;

extern "C" {

int dino_pe_create(dino_plan* plan, const dino_pe_desc* d, dino_pe** out) {
  DINO_REQUIRE(plan && d && out, DINO_ERR_ARG, "dino_pe_create: null argument");
  *out = nullptr;
  DINO_REQUIRE(d->layers >= 1 && d->layers <= 48, DINO_ERR_UNSUPPORTED,
               "layers must be in [1, 48]");
  DINO_REQUIRE(d->members >= 1, DINO_ERR_ARG, "members must be >= 1");
  DINO_REQUIRE(d->n_tracers >= 0 && d->n_tracers <= kMaxTracers,
               DINO_ERR_UNSUPPORTED, "at most 4 tracers are supported");
  DINO_REQUIRE(d->humidity_tracer >= -1 && d->humidity_tracer < d->n_tracers,
               DINO_ERR_ARG, "humidity_tracer out of range");
  DINO_REQUIRE(d->layer_thickness && d->inv_center_to_center && d->sigma_ratios &&
                   d->reference_temperature && d->geopotential_weights &&
                   d->temperature_weights && d->sigma_centers,
               DINO_ERR_ARG, "dino_pe_create: missing vertical arrays");
  DINO_REQUIRE(!(d->held_suarez && d->n_tracers > 0), DINO_ERR_UNSUPPORTED,
               "Held-Suarez forcing composes with tracer-free states only");
  DINO_REQUIRE(d->vertical_scheme == 0 || d->vertical_scheme == 1, DINO_ERR_ARG,
               "vertical_scheme must be 0 (sigma) or 1 (hybrid)");
  if (d->vertical_scheme == 1) {
    DINO_REQUIRE(d->hybrid_a_boundaries && d->hybrid_b_boundaries &&
                     d->implicit_lnps_column && d->implicit_thickness,
                 DINO_ERR_ARG, "dino_pe_create: missing hybrid-level arrays");
    DINO_REQUIRE(d->reference_surface_pressure > 0, DINO_ERR_ARG,
                 "`reference_surface_pressure` must be positive.");
    DINO_REQUIRE(!d->held_suarez, DINO_ERR_UNSUPPORTED,
                 "Held-Suarez forcing is defined on sigma levels only");
  }
  DINO_REQUIRE((int64_t)d->layers * plan->I * plan->J < ((int64_t)1 << 31),
               DINO_ERR_UNSUPPORTED, "layers x nodal points must be below 2^31");
  dino_pe* pe = new dino_pe();
  pe->plan = plan;
  pe->K = d->layers;
  pe->mem = d->members;
  pe->nT = d->n_tracers;
  pe->hum = d->humidity_tracer;
  pe->hybrid = d->vertical_scheme == 1 ? 1 : 0;
  if (pe->hybrid) {
    // Humidity enters the hybrid column kernel only; the sigma-form moist
    // planes (humidity gradients, corrections) stay off.
    pe->hum_hyb = pe->hum;
    pe->hum = -1;
    pe->ps_ref = d->reference_surface_pressure;
  }
  pe->vadv = d->include_vertical_advection ? 1 : 0;
  pe->hs = d->held_suarez ? 1 : 0;
  pe->M = plan->M;
  pe->L = plan->L;
  pe->I = plan->I;
  pe->J = plan->J;
  pe->ML = (size_t)pe->M * pe->L;
  pe->IJ = (size_t)pe->I * pe->J;
  pe->R = d->R;
  pe->Rv = d->R_vapor;
  pe->Cpv = d->Cp_vapor;
  pe->kappa = d->kappa;
  pe->g = d->gravity;
  pe->Omega = d->angular_velocity;
  pe->hs_p0 = d->hs_p0;
  pe->hs_sigma_b = d->hs_sigma_b;
  pe->hs_kf = d->hs_kf;
  pe->hs_ka = d->hs_ka;
  pe->hs_ks = d->hs_ks;
  pe->hs_minT = d->hs_minT;
  pe->hs_maxT = d->hs_maxT;
  pe->hs_dTy = d->hs_dTy;
  pe->hs_dThz = d->hs_dThz;
  int rc = pe_build(pe, d);
  if (rc != DINO_OK) {
    pe_free(pe);
    return rc;
  }
  *out = pe;
  return DINO_OK;
}

int dino_pe_destroy(dino_pe* pe) {
  pe_free(pe);
  return DINO_OK;
}

int dino_pe_counts(const dino_pe* pe, int32_t* counts) {
  DINO_REQUIRE(pe && counts, DINO_ERR_ARG, "dino_pe_counts: null argument");
  counts[0] = pe->n_state;
  counts[1] = pe->n_aux;
  counts[2] = pe->n_inv;
  counts[3] = pe->n_fwd;
  counts[4] = pe->mem * (2 * pe->K + 1);
  return DINO_OK;
}

int64_t dino_pe_state_size(const dino_pe* pe) {
  if (!pe) return -1;
  return (int64_t)pe->n_state * (int64_t)pe->ML;
}

int dino_pe_explicit(dino_pe* pe, const float* state, float* tend, void* stream) {
  DINO_REQUIRE(pe && state && tend, DINO_ERR_ARG, "dino_pe_explicit: null argument");
  DINO_REQUIRE(state != tend, DINO_ERR_ARG, "dino_pe_explicit: in and out must differ");
  return pe_explicit_impl(pe, state, tend, (cudaStream_t)stream);
}

int dino_pe_implicit(dino_pe* pe, const float* state, float* out, void* stream) {
  DINO_REQUIRE(pe && state && out, DINO_ERR_ARG, "dino_pe_implicit: null argument");
  DINO_REQUIRE(state != out, DINO_ERR_ARG, "dino_pe_implicit: in and out must differ");
  cudaStream_t st = (cudaStream_t)stream;
  // Vorticity and tracers have no implicit terms.
  DINO_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(float) * pe->n_state * pe->ML, st));
  const MatEntry* m = nullptr;
  DINO_TRY(get_matrix(pe, kMatL, 0.0, nullptr, &m));
  return launch_apply(pe, m, state, out, nullptr, st);
}

int dino_pe_implicit_inverse(dino_pe* pe, const float* state, float* out,
                             double eta, void* stream) {
  DINO_REQUIRE(pe && state && out, DINO_ERR_ARG, "dino_pe_implicit_inverse: null argument");
  DINO_REQUIRE(std::isfinite(eta), DINO_ERR_ARG, "step_size must be finite");
  const MatEntry* m = nullptr;
  DINO_TRY(get_matrix(pe, kMatInv, eta, nullptr, &m));
  cudaStream_t st = (cudaStream_t)stream;
  if (out != state) {
    // Vorticity and tracer planes pass through unchanged.
    const size_t mK = (size_t)pe->mem * pe->K;
    DINO_CHECK_CUDA(cudaMemcpyAsync(out, state, sizeof(float) * mK * pe->ML,
                                    cudaMemcpyDeviceToDevice, st));
    if (pe->nT > 0)
      DINO_CHECK_CUDA(cudaMemcpyAsync(out + 3 * mK * pe->ML, state + 3 * mK * pe->ML,
                                      sizeof(float) * pe->nT * mK * pe->ML,
                                      cudaMemcpyDeviceToDevice, st));
  }
  return launch_apply(pe, m, state, out, nullptr, st);
}

int dino_pe_step(dino_pe* pe, float* state, double dt, const double* host_filter,
                 int32_t n_steps, void* stream) {
  DINO_REQUIRE(pe && state, DINO_ERR_ARG, "dino_pe_step: null argument");
  DINO_REQUIRE(n_steps >= 0, DINO_ERR_ARG, "n_steps must be >= 0");
  StepMats mats;
  DINO_TRY(get_step_mats(pe, dt, host_filter, &mats));
  float* filt = nullptr;
  DINO_TRY(get_filter(pe, host_filter, &filt));
  for (int s = 0; s < n_steps; ++s)
    DINO_TRY(pe_step_once(pe, state, dt, filt, mats, (cudaStream_t)stream));
  return DINO_OK;
}

int dino_pe_step_graph(dino_pe* pe, float* state, double dt,
                       const double* host_filter, int32_t n_steps,
                       void* stream) {
  DINO_REQUIRE(pe && state, DINO_ERR_ARG, "dino_pe_step_graph: null argument");
  DINO_REQUIRE(n_steps >= 0, DINO_ERR_ARG, "n_steps must be >= 0");
  cudaStream_t st = (cudaStream_t)stream;
  StepMats mats;
  DINO_TRY(get_step_mats(pe, dt, host_filter, &mats));
  float* filt = nullptr;
  DINO_TRY(get_filter(pe, host_filter, &filt));
  GraphEntry& g = pe->graph;
  if (!(g.exec && g.state == state && g.dt == dt && g.filter == filt)) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = GraphEntry{};
    DINO_TRY(sht_prepare(pe->plan));
    DINO_TRY(prepare_apply());
    // Capture on a private stream so that the caller's stream (possibly the
    // legacy default stream) is never put in capture mode.
    cudaStream_t cap;
    DINO_CHECK_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    DINO_CHECK_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = pe_step_once(pe, state, dt, filt, mats, cap);
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (rc != DINO_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    DINO_CHECK_CUDA(ce);
    DINO_CHECK_CUDA(cudaGraphInstantiate(&g.exec, graph, 0));
    g.graph = graph;
    g.state = state;
    g.dt = dt;
    g.filter = filt;
  }
  for (int s = 0; s < n_steps; ++s) DINO_CHECK_CUDA(cudaGraphLaunch(g.exec, st));
  return DINO_OK;
}

int dino_pe_trajectory(dino_pe* pe, float* state, double dt, const double* host_filter,
                       int32_t outer_steps, int32_t inner_steps, int32_t start_with_input,
                       float* frames, void* stream) {
  DINO_REQUIRE(pe && state, DINO_ERR_ARG, "dino_pe_trajectory: null argument");
  DINO_REQUIRE(outer_steps >= 0 && inner_steps >= 1, DINO_ERR_ARG,
               "dino_pe_trajectory: need outer_steps >= 0 and inner_steps >= 1");
  if (outer_steps == 0) return DINO_OK;
  const size_t n = (size_t)pe->n_state * pe->ML;
  DINO_REQUIRE(frames, DINO_ERR_ARG, "dino_pe_trajectory: null frames");
  DINO_REQUIRE(frames + n * outer_steps <= state || state + n <= frames, DINO_ERR_ARG,
               "dino_pe_trajectory: frames must not overlap the state");
  cudaStream_t st = (cudaStream_t)stream;
  // Every frame: the captured step graph replayed inner_steps times and one
  // device-to-device copy of the packed state into its slot, all queued on
  // the stream; the host never waits.
  for (int f = 0; f < outer_steps; ++f) {
    float* slot = frames + (size_t)f * n;
    if (start_with_input)
      DINO_CHECK_CUDA(cudaMemcpyAsync(slot, state, n * sizeof(float),
                                      cudaMemcpyDeviceToDevice, st));
    DINO_TRY(dino_pe_step_graph(pe, state, dt, host_filter, inner_steps, stream));
    if (!start_with_input)
      DINO_CHECK_CUDA(cudaMemcpyAsync(slot, state, n * sizeof(float),
                                      cudaMemcpyDeviceToDevice, st));
  }
  return DINO_OK;
}

int dino_pe_explicit_vjp(dino_pe* pe, const float* state, const float* tend_ct,
                         float* state_ct, void* stream) {
  DINO_REQUIRE(pe && state && tend_ct && state_ct, DINO_ERR_ARG,
               "dino_pe_explicit_vjp: null argument");
  DINO_REQUIRE(!pe->hybrid, DINO_ERR_UNSUPPORTED,
               "the explicit-term VJP is built for sigma levels only");
  DINO_REQUIRE(state_ct != state && state_ct != tend_ct, DINO_ERR_ARG,
               "dino_pe_explicit_vjp: state_ct must not alias the inputs");
  DINO_TRY(pe_ensure_adjoint(pe));
  DINO_TRY(sht_prepare(pe->plan));
  return pe_explicit_vjp_impl(pe, state, tend_ct, state_ct, (cudaStream_t)stream);
}

int dino_pe_implicit_vjp(dino_pe* pe, const float* out_ct, float* in_ct, void* stream) {
  DINO_REQUIRE(pe && out_ct && in_ct, DINO_ERR_ARG, "dino_pe_implicit_vjp: null argument");
  DINO_REQUIRE(out_ct != in_ct, DINO_ERR_ARG, "dino_pe_implicit_vjp: in and out must differ");
  cudaStream_t st = (cudaStream_t)stream;
  DINO_CHECK_CUDA(cudaMemsetAsync(in_ct, 0, sizeof(float) * pe->n_state * pe->ML, st));
  const MatEntry* m = nullptr;
  DINO_TRY(get_matrix(pe, kMatL, 0.0, nullptr, &m, true));
  return launch_apply(pe, m, out_ct, in_ct, nullptr, st);
}

int dino_pe_implicit_inverse_vjp(dino_pe* pe, const float* out_ct, float* in_ct,
                                 double eta, void* stream) {
  DINO_REQUIRE(pe && out_ct && in_ct, DINO_ERR_ARG,
               "dino_pe_implicit_inverse_vjp: null argument");
  DINO_REQUIRE(std::isfinite(eta), DINO_ERR_ARG, "step_size must be finite");
  const MatEntry* m = nullptr;
  DINO_TRY(get_matrix(pe, kMatInv, eta, nullptr, &m, true));
  cudaStream_t st = (cudaStream_t)stream;
  if (out_ct != in_ct)
    DINO_TRY(launch_lincomb(pe, {{out_ct, 0.f, 1.f}}, nullptr, in_ct, 2, st));
  return launch_apply(pe, m, out_ct, in_ct, nullptr, st);
}

int dino_pe_step_vjp(dino_pe* pe, const float* state, const float* out_ct,
                     float* in_ct, double dt, const double* host_filter,
                     void* stream) {
  DINO_REQUIRE(pe && state && out_ct && in_ct, DINO_ERR_ARG,
               "dino_pe_step_vjp: null argument");
  DINO_REQUIRE(!pe->hybrid, DINO_ERR_UNSUPPORTED,
               "the step VJP is built for sigma levels only");
  DINO_REQUIRE(in_ct != state, DINO_ERR_ARG, "dino_pe_step_vjp: in_ct must not alias state");
  DINO_TRY(pe_ensure_adjoint(pe));
  DINO_TRY(sht_prepare(pe->plan));
  StepMats m;
  DINO_TRY(get_step_mats(pe, dt, host_filter, &m));
  StepMatsT mt;
  DINO_TRY(get_step_mats_t(pe, dt, host_filter, &mt));
  float* filt = nullptr;
  DINO_TRY(get_filter(pe, host_filter, &filt));
  return pe_step_vjp_impl(pe, state, out_ct, in_ct, dt, filt, m, mt,
                          (cudaStream_t)stream);
}

}  // extern "C"

