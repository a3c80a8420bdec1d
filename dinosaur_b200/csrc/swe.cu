// Shallow-water equations on the sphere: explicit tendencies, implicit terms
// and the closed-form implicit inverse (ShallowWaterEquations,
// dinosaur/shallow_water.py:121-230).
//
// Packed state, kind-major: [vorticity: members*K][divergence][potential]
// planes of [M][L].  One explicit evaluation is
//   modal pre-pass (u cos, v cos, clipped vorticity and potential)
//   -> inverse SHT -> nodal products (u (zeta + f), u phi, kinetic energy)
//   -> forward SHT -> modal post-pass (div/curl, Laplacian, the layer
//   pressure coupling through the density ratios, clip of the top l).

#include <cmath>
#include <vector>

#include "dino_internal.cuh"

struct dino_swe {
  dino_plan* plan = nullptr;
  int K = 0, mem = 0, M = 0, L = 0, I = 0, J = 0;
  size_t ML = 0, IJ = 0;
  float* d_dens = nullptr;   // K x K density ratios (shallow_water.py:71-86)
  float* d_phiref = nullptr; // K reference potentials
  float* d_orog = nullptr;   // [M][L] modal orography (zeros when absent)
  float* d_lat = nullptr;    // [2][J]: sec^2(lat), 2 Omega sin(lat)
  float* d_aux = nullptr;    // [u][v][zeta clipped][phi clipped]: 4 mK planes
  float* d_nodal = nullptr;  // their nodal values
  float* d_fwd_in = nullptr; // [b_u][b_v][g_u][g_v][e]: 5 mK nodal planes
  float* d_fwd_out = nullptr;
  float* d_work = nullptr;
  int work_fields = 0;
};

namespace dino {
namespace {

struct SwePrepArgs {
  const float* state;
  float* aux;
  int K, mem, M, L, lw;
  const float* deriv;
  const float* invlap;
  float inv_radius;
};

// get_cos_lat_vector(vorticity, divergence, grid) with its default clip
// (spherical_harmonic.py:1164-1178) and clip_wavenumbers of vorticity and
// potential before their inverse transforms (shallow_water.py:60-62).
__global__ void swe_prep_kernel(SwePrepArgs a) {
  const size_t ML = (size_t)a.M * a.L;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ML) return;
  const int l = idx % a.L, row = idx / a.L;
  const size_t mK = (size_t)a.mem * a.K;
  const size_t plane = (size_t)blockIdx.z * a.K + blockIdx.y;  // member, level
  const float* vort = a.state + plane * ML;
  const float* div = a.state + (mK + plane) * ML;
  const float* phi = a.state + (2 * mK + plane) * ML;
  const bool keep = l < a.L - 1;
  float u = 0.f, v = 0.f;
  if (keep) {
    const float dchi = d_dlon_at(div, row, l, a.L) * a.invlap[l];
    const float dpsi = d_dlon_at(vort, row, l, a.L) * a.invlap[l];
    const float cchi = dlat_at(div, a.invlap, row, l, a.L, a.lw, a.deriv, 0);
    const float cpsi = dlat_at(vort, a.invlap, row, l, a.L, a.lw, a.deriv, 0);
    u = (dchi - cpsi) * a.inv_radius;
    v = (cchi + dpsi) * a.inv_radius;
  }
  a.aux[plane * ML + idx] = u;
  a.aux[(mK + plane) * ML + idx] = v;
  a.aux[(2 * mK + plane) * ML + idx] = keep ? vort[idx] : 0.f;
  a.aux[(3 * mK + plane) * ML + idx] = keep ? phi[idx] : 0.f;
}

struct SweNodalArgs {
  const float* nod;  // [u][v][zeta][phi]
  float* fwd;        // [b_u][b_v][g_u][g_v][e]
  int J;
  size_t IJ, mK;
  const float* lat;
};

// shallow_water.py:170-177: b = u (zeta + f) sec^2, g = u phi sec^2,
// e = |u|^2 sec^2 / 2 on the nodal grid.
__global__ void swe_nodal_kernel(SweNodalArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.IJ) return;
  const size_t plane = blockIdx.y;
  const int j = idx % a.J;
  const float sec2 = a.lat[j];
  const float f = a.lat[a.J + j];
  const size_t s = a.mK * a.IJ, o = plane * a.IJ + idx;
  const float u = a.nod[o], v = a.nod[s + o];
  const float tv = a.nod[2 * s + o] + f;
  const float phi = a.nod[3 * s + o];
  a.fwd[o] = u * tv * sec2;
  a.fwd[s + o] = v * tv * sec2;
  a.fwd[2 * s + o] = u * phi * sec2;
  a.fwd[3 * s + o] = v * phi * sec2;
  a.fwd[4 * s + o] = (u * u + v * v) * sec2 * 0.5f;
}

struct SwePostArgs {
  const float* fm;     // modal [b_u][b_v][g_u][g_v][e]
  const float* state;  // for the potential
  float* tend;
  const float* dens;   // K x K
  const float* orog;
  int K, mem, M, L, lw;
  const float* deriv;
  const float* lap;
  float inv_radius;
};

// shallow_water.py:186-205.  p = D phi + orography (the layers' pressure
// coupling); vorticity -div_cos_lat(b); divergence -lap(p + e) +
// curl_cos_lat(b); potential -div_cos_lat(g); every tendency clipped.
__global__ void swe_post_kernel(SwePostArgs a) {
  const size_t ML = (size_t)a.M * a.L;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ML) return;
  const int l = idx % a.L, row = idx / a.L;
  const int k = blockIdx.y, mb = blockIdx.z, K = a.K;
  const size_t mK = (size_t)a.mem * K;
  const size_t plane = (size_t)mb * K + k;
  float* out_z = a.tend + plane * ML;
  float* out_d = a.tend + (mK + plane) * ML;
  float* out_p = a.tend + (2 * mK + plane) * ML;
  if (l == a.L - 1) {
    out_z[idx] = 0.f;
    out_d[idx] = 0.f;
    out_p[idx] = 0.f;
    return;
  }
  const float* bu = a.fm + plane * ML;
  const float* bv = a.fm + (mK + plane) * ML;
  const float* gu = a.fm + (2 * mK + plane) * ML;
  const float* gv = a.fm + (3 * mK + plane) * ML;
  const float* e = a.fm + (4 * mK + plane) * ML;
  const float ir = a.inv_radius;
  float p = a.orog[idx];
  for (int b = 0; b < K; ++b)
    p = fmaf(a.dens[k * K + b], a.state[(2 * mK + (size_t)mb * K + b) * ML + idx], p);
  const float div_b = (d_dlon_at(bu, row, l, a.L) +
                       dlat_at(bv, nullptr, row, l, a.L, a.lw, a.deriv, 2)) * ir;
  const float curl_b = (d_dlon_at(bv, row, l, a.L) -
                        dlat_at(bu, nullptr, row, l, a.L, a.lw, a.deriv, 2)) * ir;
  const float div_g = (d_dlon_at(gu, row, l, a.L) +
                       dlat_at(gv, nullptr, row, l, a.L, a.lw, a.deriv, 2)) * ir;
  out_z[idx] = -div_b;
  out_d[idx] = -a.lap[l] * (p + e[idx]) + curl_b;
  out_p[idx] = -div_g;
}

struct SweImplicitArgs {
  const float* in;
  float* out;
  const float* phiref;
  const float* lap;
  float eta;
  int mode;  // 0: implicit terms, 1: implicit inverse
  int K, mem, L;
  size_t ML;
};

// shallow_water.py:207-230, elementwise per (layer, m, l).
__global__ void swe_implicit_kernel(SweImplicitArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.ML) return;
  const int l = idx % a.L;
  const int k = blockIdx.y, mb = blockIdx.z;
  const size_t mK = (size_t)a.mem * a.K;
  const size_t plane = (size_t)mb * a.K + k;
  const size_t oz = plane * a.ML + idx, od = (mK + plane) * a.ML + idx,
               op = (2 * mK + plane) * a.ML + idx;
  const float z = a.in[oz], d = a.in[od], p = a.in[op];
  const float lam = a.lap[l], ref = a.phiref[k];
  if (a.mode == 0) {
    a.out[oz] = 0.f;
    a.out[od] = -lam * p;
    a.out[op] = -ref * d;
  } else {
    const float s = 1.f / (1.f - a.eta * a.eta * ref * lam);
    a.out[oz] = z;
    a.out[od] = s * (d - a.eta * lam * p);
    a.out[op] = s * (-a.eta * ref * d + p);
  }
}

template <typename T>
int upload(T** dst, const std::vector<T>& v) {
  DINO_CHECK_CUDA(cudaMalloc(dst, sizeof(T) * v.size()));
  DINO_CHECK_CUDA(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return DINO_OK;
}

void swe_free(dino_swe* s) {
  if (!s) return;
  cudaFree(s->d_dens);
  cudaFree(s->d_phiref);
  cudaFree(s->d_orog);
  cudaFree(s->d_lat);
  cudaFree(s->d_aux);
  cudaFree(s->d_nodal);
  cudaFree(s->d_fwd_in);
  cudaFree(s->d_fwd_out);
  cudaFree(s->d_work);
  delete s;
}

int swe_build(dino_swe* s, const dino_swe_desc* d) {
  dino_plan* p = s->plan;
  const int K = s->K;
  std::vector<float> dens(K * K), ref(K), lat(2 * p->J);
  // D[i][j] = min(rho_j / rho_i, 1) with a zero diagonal: the pressure on
  // layer i from the layers j (shallow_water.py:71-86).
  for (int i = 0; i < K; ++i) {
    for (int j = 0; j < K; ++j) {
      const double r = d->densities ? d->densities[j] / d->densities[i] : 1.0;
      dens[i * K + j] = (i == j) ? 0.f : (float)(r < 1.0 ? r : 1.0);
    }
    ref[i] = (float)d->reference_potential[i];
  }
  for (int j = 0; j < p->J; ++j) {
    const double x = p->h_x64[j];
    lat[j] = (float)(1.0 / (1.0 - x * x));
    lat[p->J + j] = (float)(2.0 * d->angular_velocity * x);
  }
  DINO_TRY(upload(&s->d_dens, dens));
  DINO_TRY(upload(&s->d_phiref, ref));
  DINO_TRY(upload(&s->d_lat, lat));
  std::vector<float> orog(s->ML, 0.f);
  if (d->orography_modal)
    for (size_t i = 0; i < s->ML; ++i) orog[i] = d->orography_modal[i];
  DINO_TRY(upload(&s->d_orog, orog));
  const size_t mK = (size_t)s->mem * K;
  DINO_CHECK_CUDA(cudaMalloc(&s->d_aux, sizeof(float) * 4 * mK * s->ML));
  DINO_CHECK_CUDA(cudaMalloc(&s->d_nodal, sizeof(float) * 4 * mK * s->IJ));
  DINO_CHECK_CUDA(cudaMalloc(&s->d_fwd_in, sizeof(float) * 5 * mK * s->IJ));
  DINO_CHECK_CUDA(cudaMalloc(&s->d_fwd_out, sizeof(float) * 5 * mK * s->ML));
  s->work_fields = (int)(5 * mK);
  DINO_CHECK_CUDA(cudaMalloc(&s->d_work, sizeof(float) * 5 * mK * p->M * p->J));
  return DINO_OK;
}

int swe_explicit_impl(dino_swe* s, const float* state, float* tend, cudaStream_t st) {
  dino_plan* p = s->plan;
  const int K = s->K, mem = s->mem;
  const int mK = mem * K;
  {
    SwePrepArgs a{state, s->d_aux, K, mem, s->M, s->L, p->lw, p->d_deriv, p->d_invlap,
                  (float)(1.0 / p->radius)};
    dim3 grid(ceil_div((int)s->ML, 256), K, mem);
    swe_prep_kernel<<<grid, 256, 0, st>>>(a);
    DINO_TRY(check_launch("swe_prep"));
  }
  DINO_TRY(sht_inverse_segs(p, one_seg(s->d_aux, 4 * mK), s->d_nodal, 4 * mK, s->d_work,
                            s->work_fields, st));
  {
    SweNodalArgs a{s->d_nodal, s->d_fwd_in, s->J, s->IJ, (size_t)mK, s->d_lat};
    dim3 grid(ceil_div((int)s->IJ, 256), mK);
    swe_nodal_kernel<<<grid, 256, 0, st>>>(a);
    DINO_TRY(check_launch("swe_nodal"));
  }
  DINO_TRY(sht_forward_to(p, s->d_fwd_in, s->d_fwd_out, 5 * mK, s->d_work,
                          s->work_fields, st));
  {
    SwePostArgs a{s->d_fwd_out, state, tend, s->d_dens, s->d_orog, K, mem, s->M, s->L,
                  p->lw, p->d_deriv, p->d_lap, (float)(1.0 / p->radius)};
    dim3 grid(ceil_div((int)s->ML, 256), K, mem);
    swe_post_kernel<<<grid, 256, 0, st>>>(a);
    DINO_TRY(check_launch("swe_post"));
  }
  return DINO_OK;
}

int swe_implicit_impl(dino_swe* s, const float* in, float* out, int mode, double eta,
                      cudaStream_t st) {
  SweImplicitArgs a{in, out, s->d_phiref, s->plan->d_lap, (float)eta, mode, s->K, s->mem,
                    s->L, s->ML};
  dim3 grid(ceil_div((int)s->ML, 256), s->K, s->mem);
  swe_implicit_kernel<<<grid, 256, 0, st>>>(a);
  return check_launch("swe_implicit");
}

}  // namespace
}  // namespace dino

using namespace dino;

extern "C" {

int dino_swe_create(dino_plan* plan, const dino_swe_desc* d, dino_swe** out) {
  DINO_REQUIRE(plan && d && out, DINO_ERR_ARG, "dino_swe_create: null argument");
  DINO_REQUIRE(d->layers >= 1 && d->layers <= 256, DINO_ERR_UNSUPPORTED,
               "layers must be in [1, 256]");
  DINO_REQUIRE(d->members >= 1, DINO_ERR_ARG, "members must be >= 1");
  DINO_REQUIRE(d->reference_potential != nullptr, DINO_ERR_ARG,
               "dino_swe_create: missing reference potential");
  if (d->densities)
    for (int i = 0; i < d->layers; ++i)
      DINO_REQUIRE(d->densities[i] > 0, DINO_ERR_ARG, "densities must be positive");
  dino_swe* s = new dino_swe();
  s->plan = plan;
  s->K = d->layers;
  s->mem = d->members;
  s->M = plan->M;
  s->L = plan->L;
  s->I = plan->I;
  s->J = plan->J;
  s->ML = (size_t)s->M * s->L;
  s->IJ = (size_t)s->I * s->J;
  const int rc = swe_build(s, d);
  if (rc != DINO_OK) {
    swe_free(s);
    return rc;
  }
  *out = s;
  return DINO_OK;
}

int dino_swe_destroy(dino_swe* s) {
  swe_free(s);
  return DINO_OK;
}

int64_t dino_swe_state_size(const dino_swe* s) {
  return s ? (int64_t)3 * s->mem * s->K * (int64_t)s->ML : -1;
}

int dino_swe_explicit(dino_swe* s, const float* state, float* out, void* stream) {
  DINO_REQUIRE(s && state && out, DINO_ERR_ARG, "dino_swe_explicit: null argument");
  DINO_REQUIRE(state != out, DINO_ERR_ARG, "dino_swe_explicit: in and out must differ");
  return swe_explicit_impl(s, state, out, (cudaStream_t)stream);
}

int dino_swe_implicit(dino_swe* s, const float* state, float* out, void* stream) {
  DINO_REQUIRE(s && state && out, DINO_ERR_ARG, "dino_swe_implicit: null argument");
  return swe_implicit_impl(s, state, out, 0, 0.0, (cudaStream_t)stream);
}

int dino_swe_implicit_inverse(dino_swe* s, const float* state, float* out, double eta,
                              void* stream) {
  DINO_REQUIRE(s && state && out, DINO_ERR_ARG, "dino_swe_implicit_inverse: null argument");
  DINO_REQUIRE(std::isfinite(eta), DINO_ERR_ARG, "step_size must be finite");
  return swe_implicit_impl(s, state, out, 1, eta, (cudaStream_t)stream);
}

}  // extern "C"
