// Internal declarations shared by the dino_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dino_b200.h"

namespace dino {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------

void set_error(const std::string& msg);

struct Status {
  int code = DINO_OK;
};

#define DINO_CHECK_CUDA(expr)                                             \
  do {                                                                    \
    cudaError_t err_ = (expr);                                            \
    if (err_ != cudaSuccess) {                                            \
      ::dino::set_error(std::string(#expr) + ": " +                       \
                        cudaGetErrorString(err_));                        \
      return DINO_ERR_CUDA;                                               \
    }                                                                     \
  } while (0)

#define DINO_REQUIRE(cond, code, msg)        \
  do {                                       \
    if (!(cond)) {                           \
      ::dino::set_error(msg);                \
      return (code);                         \
    }                                        \
  } while (0)

#define DINO_TRY(expr)          \
  do {                          \
    int rc_ = (expr);           \
    if (rc_ != DINO_OK) return rc_; \
  } while (0)

// Checks the launch status of the last kernel (does not synchronize).
int check_launch(const char* what);

// An NVTX range over the enclosing scope, so that profilers group the
// kernels a phase launches under the reference's names for its phases
// (inv_legendre, inv_fourier, fwd_fourier, fwd_legendre: the named calls of
// spherical_harmonic.py:265-279).  Costs nothing without an attached tool.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Runs a set-up step (returning a status) once per device and process, with
// that device current.  Kernel attributes such as the dynamic shared-memory
// limit belong to the device's context, so every device that launches the
// kernel needs its own call.  Safe to call from several host threads.
class PerDeviceOnce {
 public:
  template <class F>
  int run(F&& fn) {
    int dev = 0;
    DINO_CHECK_CUDA(cudaGetDevice(&dev));
    DINO_REQUIRE(dev >= 0 && dev < 64, DINO_ERR_ARG, "device index out of range");
    const uint64_t bit = 1ull << dev;
    std::lock_guard<std::mutex> lock(mu_);
    if (done_ & bit) return DINO_OK;
    DINO_TRY(fn());
    done_ |= bit;
    return DINO_OK;
  }

 private:
  std::mutex mu_;
  uint64_t done_ = 0;
};

// ---------------------------------------------------------------------------
// Field segments: a batch of fields gathered from up to kMaxSegs contiguous
// runs of [M][L] (or [I][J]) planes.
// ---------------------------------------------------------------------------

constexpr int kMaxSegs = 4;

struct Segs {
  const float* ptr[kMaxSegs];
  int start[kMaxSegs + 1];
  int n;
};

inline Segs one_seg(const float* p, int count) {
  Segs s{};
  s.ptr[0] = p;
  s.start[0] = 0;
  s.start[1] = count;
  s.n = 1;
  return s;
}

__device__ __forceinline__ const float* seg_field(const Segs& s, int b,
                                                  size_t stride) {
  int i = 0;
  while (i + 1 < s.n && b >= s.start[i + 1]) ++i;
  return s.ptr[i] + (size_t)(b - s.start[i]) * stride;
}

Segs seg_offset(const Segs& s, int first, int count, size_t stride);

// ---------------------------------------------------------------------------
// Transform plan
// ---------------------------------------------------------------------------

struct TcTables;  // tensor-core operand tables (legendre_tc.cu)

}  // namespace dino

struct dino_plan {
  // Shapes.
  int lw = 0, L = 0, I = 0, J = 0, M = 0, Jh = 0, N = 0;
  int spacing = 0, precision = 0, max_fields = 0, device = 0;
  double radius = 1.0;
  bool fft_pow2 = false;
  // FP64 nodes and weights (device and host copies).
  double* d_x64 = nullptr;
  double* d_w64 = nullptr;
  std::vector<double> h_x64, h_w64;
  // FP32 tables.
  float* d_wq = nullptr;       // J: Gauss weight * 2pi / I
  float* d_ptab = nullptr;     // folded Legendre table, [m][l-m][Jh]
  int64_t* d_ptab_off = nullptr;  // lw + 1 offsets into d_ptab
  std::vector<int64_t> h_ptab_off;
  float* d_fbasis = nullptr;   // [I][M] real Fourier basis (generic DFT path)
  float2* d_tw_n = nullptr;    // N twiddles exp(+2 pi i k / N)
  float2* d_tw_i = nullptr;    // N twiddles exp(+2 pi i k / I)
  float* d_deriv = nullptr;    // 4 tables [lw][L]: (l+1)a, -l b, (l-1)a, -(l+2)b
  float* d_lap = nullptr;      // L: -l(l+1)/r^2
  float* d_invlap = nullptr;   // L: inverse, 0 at l = 0
  // Workspace: intermediate Fourier coefficients [max_fields][M][J].
  float* d_work = nullptr;
  dino::TcTables* tc = nullptr;
  // Second stream for alternating L2-sized chunks, with fork/join events.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

namespace dino {

// ---------------------------------------------------------------------------
// Modal operators at one (row, l) of a [M][L] plane (real layout: rows
// m = 0, +1, -1, ...; deriv holds the recurrence tables of the plan).
// ---------------------------------------------------------------------------

// d/dlon: the cos/sin pair of each m swaps with a factor +-m.
__device__ __forceinline__ float d_dlon_at(const float* x, int row, int l,
                                           int L) {
  if (row == 0) return 0.f;
  int m = (row + 1) >> 1;
  return (row & 1) ? m * x[(size_t)(row + 1) * L + l]
                   : -m * x[(size_t)(row - 1) * L + l];
}

// cos_lat_d_dlat (tab = 0) or sec_lat_d_dlat_cos2 (tab = 2) at (row, l) of a
// plane x scaled elementwise by s[l] (s = nullptr: no scaling).
__device__ __forceinline__ float dlat_at(const float* x, const float* s,
                                         int row, int l, int L, int lw,
                                         const float* deriv, int tab) {
  int m = (row + 1) >> 1;
  const float* ta = deriv + (size_t)tab * lw * L + (size_t)m * L;
  const float* tb = ta + (size_t)lw * L;
  const float* xr = x + (size_t)row * L;
  float v = 0.f;
  if (l + 1 < L) v += ta[l + 1] * (s ? s[l + 1] * xr[l + 1] : xr[l + 1]);
  if (l >= 1) v += tb[l - 1] * (s ? s[l - 1] * xr[l - 1] : xr[l - 1]);
  return v;
}

// sht.cu
int sht_inverse_segs(dino_plan* p, const Segs& in, float* out_nodal, int nfields,
                     float* work, int work_fields, cudaStream_t st);
int sht_forward_to(dino_plan* p, const float* nodal, float* out_modal,
                   int nfields, float* work, int work_fields, cudaStream_t st);
int sht_inverse_adjoint_to(dino_plan* p, const float* nodal_ct, float* modal_ct,
                           int nfields, float* work, int work_fields, cudaStream_t st);
int sht_forward_adjoint_to(dino_plan* p, const float* modal_ct, float* nodal_ct,
                           int nfields, float* work, int work_fields, cudaStream_t st);
// Fields per chunk of a chunked transform of nf fields (sht.cu).
int l2_chunk(dino_plan* p, int nf, int work_fields);
int legendre_inverse(dino_plan* p, const Segs& in, float* out_fourier,
                     int nfields, cudaStream_t st);
int legendre_forward(dino_plan* p, const float* fourier, float* out_modal,
                     int nfields, cudaStream_t st);
int fourier_inverse(dino_plan* p, const float* fourier, float* nodal,
                    int nfields, bool weighted_adjoint, cudaStream_t st);
int fourier_forward(dino_plan* p, const float* nodal, float* fourier,
                    int nfields, bool weighted, cudaStream_t st);
int modal_op(dino_plan* p, int op, const float* in, float* out, int nfields,
             int arg, cudaStream_t st);
// Sets kernel attributes ahead of stream capture.
int sht_prepare(dino_plan* p);
// FP32 SIMT inverse Legendre contraction for any plan (no precision dispatch).
std::string tc_describe(dino_plan* p);  // legendre_tc.cu
int legendre_inverse_fp32(dino_plan* p, const Segs& in, float* out, int nf,
                          cudaStream_t st);
// FP32 SIMT forward Legendre contraction for any plan.
int legendre_forward_fp32(dino_plan* p, const float* fourier, float* out, int nf,
                          cudaStream_t st);
// Whether a tensor-core plan's autotuner found the FP32 SIMT contraction of
// this direction faster at its chunk size (legendre_tc.cu).
bool tc_use_simt(const dino_plan* p, bool forward);

// legendre_tc.cu
int tc_tables_build(dino_plan* p);
void tc_tables_free(dino_plan* p);
int tc_legendre_inverse(dino_plan* p, const Segs& in, float* out_fourier,
                        int nfields, cudaStream_t st);
int tc_legendre_forward(dino_plan* p, const float* fourier, float* out_modal,
                        int nfields, cudaStream_t st);

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace dino
