// Transform plans: FP64 Gauss-Legendre nodes and associated-Legendre tables
// built on the GPU, host-built FP64 constants rounded to FP32, workspace.
//
// Follows dinosaur/associated_legendre.py:23-114 (normalised recurrence,
// Gauss nodes) and dinosaur/fourier.py:24-60 (real Fourier basis) of the
// reference; the tables are laid out for the kernels in sht.cu.

#include <cmath>
#include <cstring>
#include <mutex>

#include "dino_internal.cuh"

namespace dino {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int check_launch(const char* what) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_error(std::string("kernel launch failed (") + what +
              "): " + cudaGetErrorString(err));
    return DINO_ERR_CUDA;
  }
  return DINO_OK;
}

Segs seg_offset(const Segs& s, int first, int count, size_t stride) {
  // Fields [first, first + count) of a segment list, rebased to start at 0.
  Segs out{};
  out.n = 0;
  out.start[0] = 0;
  for (int i = 0; i < s.n; ++i) {
    int lo = s.start[i], hi = s.start[i + 1];
    int a = lo > first ? lo : first;
    int b = hi < first + count ? hi : first + count;
    if (a >= b) continue;
    out.ptr[out.n] = s.ptr[i] + (size_t)(a - lo) * stride;
    out.start[out.n] = a - first;
    out.start[out.n + 1] = b - first;
    out.n++;
  }
  return out;
}

// ---------------------------------------------------------------------------
// FP64 table kernels
// ---------------------------------------------------------------------------

// Gauss-Legendre nodes (ascending) and weights by Newton's method on P_J,
// evaluated with the three-term recurrence in FP64.  Nodes are computed for
// the lower half and mirrored so that x[J-1-j] == -x[j] exactly.
__global__ void gauss_nodes_kernel(int J, double* __restrict__ x,
                                   double* __restrict__ w) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int half = (J + 1) / 2;
  if (j >= half) return;
  const double pi = 3.14159265358979323846;
  double xr = -cos(pi * (j + 0.75) / (J + 0.5));
  if ((J & 1) && j == J / 2) xr = 0.0;
  double dp = 1.0;
  for (int iter = 0; iter < 100; ++iter) {
    double p0 = 1.0, p1 = xr;
    for (int n = 2; n <= J; ++n) {
      double p2 = ((2.0 * n - 1.0) * xr * p1 - (n - 1.0) * p0) / n;
      p0 = p1;
      p1 = p2;
    }
    dp = J * (xr * p1 - p0) / (xr * xr - 1.0);
    double dx = p1 / dp;
    xr -= dx;
    // Quadratic convergence: once the update is below 1e-15 one more step
    // reaches round-off (a tighter absolute test may never be met).
    if (fabs(dx) < 1e-15) {
      p0 = 1.0;
      p1 = xr;
      for (int n = 2; n <= J; ++n) {
        double p2 = ((2.0 * n - 1.0) * xr * p1 - (n - 1.0) * p0) / n;
        p0 = p1;
        p1 = p2;
      }
      xr -= p1 / (J * (xr * p1 - p0) / (xr * xr - 1.0));
      break;
    }
  }
  {
    // Final derivative at the converged root for the weight.
    double p0 = 1.0, p1 = xr;
    for (int n = 2; n <= J; ++n) {
      double p2 = ((2.0 * n - 1.0) * xr * p1 - (n - 1.0) * p0) / n;
      p0 = p1;
      p1 = p2;
    }
    dp = J * (xr * p1 - p0) / (xr * xr - 1.0);
  }
  double wr = 2.0 / ((1.0 - xr * xr) * dp * dp);
  x[j] = xr;
  w[j] = wr;
  if (J - 1 - j != j) {
    x[J - 1 - j] = -xr;
    w[J - 1 - j] = wr;
  }
}

// Normalised associated Legendre functions P_l^m(x_j) for j < Jh, stored as
// FP32 at ptab[off[m] + (l - m) * Jh + j].  One thread per (m, j).
__global__ void legendre_table_kernel(int lw, int L, int Jh,
                                      const double* __restrict__ x,
                                      const int64_t* __restrict__ off,
                                      float* __restrict__ ptab) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int m = blockIdx.y;
  if (j >= Jh || m >= lw) return;
  double xj = x[j];
  double y = sqrt(1.0 - xj * xj);
  double diag = 1.0 / sqrt(2.0);
  for (int mm = 1; mm <= m; ++mm) diag = -sqrt(1.0 + 1.0 / (2.0 * mm)) * y * diag;
  float* out = ptab + off[m];
  double p2 = 0.0, p1 = diag;
  out[j] = (float)diag;
  double m2 = (double)m * m;
  for (int k = 1; k < L - m; ++k) {
    double mk2 = (double)(m + k) * (m + k);
    double mkp2 = (double)(m + k - 1) * (m + k - 1);
    double a = sqrt((4.0 * mk2 - 1.0) / (mk2 - m2));
    double b = sqrt((mkp2 - m2) / (4.0 * mkp2 - 1.0));
    double cur = a * (xj * p1 - b * p2);
    out[(size_t)k * Jh + j] = (float)cur;
    p2 = p1;
    p1 = cur;
  }
}

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

template <typename T>
static int upload(T** dst, const std::vector<T>& src) {
  DINO_CHECK_CUDA(cudaMalloc((void**)dst, sizeof(T) * (src.empty() ? 1 : src.size())));
  if (!src.empty())
    DINO_CHECK_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(),
                               cudaMemcpyHostToDevice));
  return DINO_OK;
}

static void plan_free(dino_plan* p) {
  if (!p) return;
  if (p->side) {
    cudaStreamSynchronize(p->side);
    cudaStreamDestroy(p->side);
  }
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  tc_tables_free(p);
  cudaFree(p->d_x64);
  cudaFree(p->d_w64);
  cudaFree(p->d_wq);
  cudaFree(p->d_ptab);
  cudaFree(p->d_ptab_off);
  cudaFree(p->d_fbasis);
  cudaFree(p->d_tw_n);
  cudaFree(p->d_tw_i);
  cudaFree(p->d_deriv);
  cudaFree(p->d_lap);
  cudaFree(p->d_invlap);
  cudaFree(p->d_work);
  delete p;
}

static int plan_build(dino_plan* p, const dino_grid_desc* d) {
  const int lw = p->lw, L = p->L, I = p->I, J = p->J, M = p->M, Jh = p->Jh;
  DINO_CHECK_CUDA(cudaGetDevice(&p->device));

  // Nodes and weights (FP64).
  DINO_CHECK_CUDA(cudaMalloc(&p->d_x64, sizeof(double) * J));
  DINO_CHECK_CUDA(cudaMalloc(&p->d_w64, sizeof(double) * J));
  if (p->spacing == DINO_SPACING_GAUSS) {
    int half = (J + 1) / 2;
    gauss_nodes_kernel<<<ceil_div(half, 128), 128>>>(J, p->d_x64, p->d_w64);
    DINO_TRY(check_launch("gauss_nodes"));
  } else {
    DINO_REQUIRE(d->host_nodes && d->host_weights, DINO_ERR_ARG,
                 "non-Gauss latitude spacing needs host_nodes/host_weights");
    DINO_CHECK_CUDA(cudaMemcpy(p->d_x64, d->host_nodes, sizeof(double) * J,
                               cudaMemcpyHostToDevice));
    DINO_CHECK_CUDA(cudaMemcpy(p->d_w64, d->host_weights, sizeof(double) * J,
                               cudaMemcpyHostToDevice));
  }
  p->h_x64.resize(J);
  p->h_w64.resize(J);
  DINO_CHECK_CUDA(cudaMemcpy(p->h_x64.data(), p->d_x64, sizeof(double) * J,
                             cudaMemcpyDeviceToHost));
  DINO_CHECK_CUDA(cudaMemcpy(p->h_w64.data(), p->d_w64, sizeof(double) * J,
                             cudaMemcpyDeviceToHost));
  if (p->spacing != DINO_SPACING_GAUSS) {
    // The folded table assumes mirror-symmetric nodes.
    for (int j = 0; j < J; ++j) {
      if (std::fabs(p->h_x64[j] + p->h_x64[J - 1 - j]) > 1e-12) {
        set_error("latitude nodes must be symmetric about the equator");
        return DINO_ERR_UNSUPPORTED;
      }
    }
  }

  // Quadrature weights including the longitude weight 2 pi / I.
  {
    std::vector<float> wq(J);
    const double wf = 2.0 * M_PI / I;
    for (int j = 0; j < J; ++j) wq[j] = (float)(wf * p->h_w64[j]);
    DINO_TRY(upload(&p->d_wq, wq));
  }

  // Folded Legendre table (FP64 recurrence on the GPU, stored FP32).
  {
    p->h_ptab_off.resize(lw + 1);
    int64_t off = 0;
    for (int m = 0; m < lw; ++m) {
      p->h_ptab_off[m] = off;
      off += (int64_t)(L - m) * Jh;
    }
    p->h_ptab_off[lw] = off;
    DINO_TRY(upload(&p->d_ptab_off, p->h_ptab_off));
    DINO_CHECK_CUDA(cudaMalloc(&p->d_ptab, sizeof(float) * (off > 0 ? off : 1)));
    dim3 grid(ceil_div(Jh, 128), lw);
    legendre_table_kernel<<<grid, 128>>>(lw, L, Jh, p->d_x64, p->d_ptab_off,
                                         p->d_ptab);
    DINO_TRY(check_launch("legendre_table"));
  }

  // Real Fourier basis (fourier.py:24-60) for the generic DFT path.
  {
    std::vector<float> f((size_t)I * M);
    for (int i = 0; i < I; ++i) {
      double lam = 2.0 * M_PI * i / I;
      f[(size_t)i * M] = (float)(1.0 / std::sqrt(2.0 * M_PI));
      for (int k = 1; k < lw; ++k) {
        f[(size_t)i * M + 2 * k - 1] = (float)(std::cos(k * lam) / std::sqrt(M_PI));
        f[(size_t)i * M + 2 * k] = (float)(std::sin(k * lam) / std::sqrt(M_PI));
      }
    }
    DINO_TRY(upload(&p->d_fbasis, f));
  }

  // Twiddles for the power-of-two real FFT path.
  p->N = I / 2;
  p->fft_pow2 = (I % 2 == 0) && is_pow2(p->N) && p->N >= 8 && p->N <= 512 &&
                lw <= p->N;
  if (p->fft_pow2) {
    std::vector<float2> tn(p->N), ti(p->N);
    for (int k = 0; k < p->N; ++k) {
      double an = 2.0 * M_PI * k / p->N, ai = 2.0 * M_PI * k / I;
      tn[k] = make_float2((float)std::cos(an), (float)std::sin(an));
      ti[k] = make_float2((float)std::cos(ai), (float)std::sin(ai));
    }
    DINO_TRY(upload(&p->d_tw_n, tn));
    DINO_TRY(upload(&p->d_tw_i, ti));
  }

  // Derivative recurrence weights (spherical_harmonic.py:1063-1102) and
  // Laplacian eigenvalues (:1010-1046), FP64 on the host, stored FP32.
  {
    std::vector<float> dv((size_t)4 * lw * L);
    for (int m = 0; m < lw; ++m) {
      for (int l = 0; l < L; ++l) {
        double mask = (m <= l) ? 1.0 : 0.0;
        double a = (l == 0) ? 0.0
                            : std::sqrt(mask * ((double)l * l - (double)m * m) /
                                        (4.0 * l * l - 1.0));
        double b = (l == L - 1)
                       ? 0.0
                       : std::sqrt(mask * ((double)(l + 1) * (l + 1) - (double)m * m) /
                                   (4.0 * (l + 1) * (l + 1) - 1.0));
        size_t o = (size_t)m * L + l;
        dv[o] = (float)((l + 1) * a);
        dv[(size_t)lw * L + o] = (float)(-l * b);
        dv[(size_t)2 * lw * L + o] = (float)((l - 1) * a);
        dv[(size_t)3 * lw * L + o] = (float)(-(l + 2) * b);
      }
    }
    DINO_TRY(upload(&p->d_deriv, dv));
    std::vector<float> lap(L), inv(L);
    for (int l = 0; l < L; ++l) {
      double e = -(double)l * (l + 1) / (p->radius * p->radius);
      lap[l] = (float)e;
      inv[l] = (l == 0) ? 0.f : (float)(1.0 / e);
    }
    DINO_TRY(upload(&p->d_lap, lap));
    DINO_TRY(upload(&p->d_invlap, inv));
  }

  // Workspace for the intermediate Fourier coefficients.
  DINO_CHECK_CUDA(cudaMalloc(&p->d_work, sizeof(float) * (size_t)p->max_fields * M * J));
  // Side stream and fork/join events for alternating chunks.
  DINO_CHECK_CUDA(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
  DINO_CHECK_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
  DINO_CHECK_CUDA(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));

  if (p->precision != DINO_PREC_FP32) DINO_TRY(tc_tables_build(p));
  DINO_CHECK_CUDA(cudaDeviceSynchronize());
  return DINO_OK;
}

}  // namespace dino

using namespace dino;

extern "C" {

int dino_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return DINO_ERR_ARG;
  std::snprintf(buf, len, "%s", dino::g_last_error.c_str());
  return DINO_OK;
}

const char* dino_version(void) { return "dino_b200 0.1 sm_100a"; }

int dino_plan_create(const dino_grid_desc* d, int32_t max_fields,
                     int32_t precision, dino_plan** out) {
  DINO_REQUIRE(d && out, DINO_ERR_ARG, "dino_plan_create: null argument");
  *out = nullptr;
  DINO_REQUIRE(d->longitude_wavenumbers >= 1 && d->total_wavenumbers >= 1 &&
                   d->longitude_nodes >= 1 && d->latitude_nodes >= 1,
               DINO_ERR_SHAPE, "dino_plan_create: sizes must be positive");
  DINO_REQUIRE(d->longitude_wavenumbers <= d->total_wavenumbers, DINO_ERR_SHAPE,
               "Expected n_m <= n_l (longitude_wavenumbers <= total_wavenumbers)");
  DINO_REQUIRE(d->longitude_nodes >= d->longitude_wavenumbers, DINO_ERR_SHAPE,
               "`real_basis` requires nodes >= wavenumbers");
  DINO_REQUIRE(d->latitude_spacing >= 0 && d->latitude_spacing <= 2,
               DINO_ERR_ARG, "unknown latitude spacing");
  DINO_REQUIRE(precision == DINO_PREC_FP32 || precision == DINO_PREC_BF16X3 ||
                   precision == DINO_PREC_TF32X3,
               DINO_ERR_ARG, "unknown precision");
  DINO_REQUIRE(max_fields >= 1, DINO_ERR_ARG, "max_fields must be >= 1");
  dino_plan* p = new dino_plan();
  p->lw = d->longitude_wavenumbers;
  p->L = d->total_wavenumbers;
  p->I = d->longitude_nodes;
  p->J = d->latitude_nodes;
  p->M = 2 * p->lw - 1;
  p->Jh = (p->J + 1) / 2;
  p->spacing = d->latitude_spacing;
  p->precision = precision;
  p->max_fields = max_fields;
  p->radius = d->radius;
  int rc = plan_build(p, d);
  if (rc != DINO_OK) {
    plan_free(p);
    return rc;
  }
  *out = p;
  return DINO_OK;
}

int dino_plan_destroy(dino_plan* p) {
  plan_free(p);
  return DINO_OK;
}

int dino_plan_nodes(const dino_plan* p, double* x, double* w) {
  DINO_REQUIRE(p && x && w, DINO_ERR_ARG, "dino_plan_nodes: null argument");
  std::memcpy(x, p->h_x64.data(), sizeof(double) * p->J);
  std::memcpy(w, p->h_w64.data(), sizeof(double) * p->J);
  return DINO_OK;
}

int dino_plan_legendre_column(const dino_plan* p, int32_t m, int32_t l,
                              double* out) {
  DINO_REQUIRE(p && out, DINO_ERR_ARG, "null argument");
  DINO_REQUIRE(m >= 0 && m < p->lw && l >= 0 && l < p->L, DINO_ERR_SHAPE,
               "(m, l) out of range");
  if (l < m) {
    for (int j = 0; j < p->J; ++j) out[j] = 0.0;
    return DINO_OK;
  }
  std::vector<float> col(p->Jh);
  DINO_CHECK_CUDA(cudaMemcpy(col.data(),
                             p->d_ptab + p->h_ptab_off[m] + (int64_t)(l - m) * p->Jh,
                             sizeof(float) * p->Jh, cudaMemcpyDeviceToHost));
  double sign = ((l - m) & 1) ? -1.0 : 1.0;
  for (int j = 0; j < p->Jh; ++j) {
    out[j] = col[j];
    out[p->J - 1 - j] = sign * col[j];
  }
  return DINO_OK;
}

}  // extern "C"
