// Allocation-free inverse spherical-harmonic transform.
//
// Some callers may not allocate device memory when they call into this
// library: a handler running inside a framework that owns the GPU's memory
// pool, or a time-critical loop that cannot accept cudaMalloc's implicit
// device synchronisation.  dino_sht_inverse_noalloc serves them: it runs the
// FP32 inverse transform (Legendre contraction, then the longitude FFT) with
// the intermediate Fourier coefficients in the fixed device array below
// instead of the plan's workspace, and calls no cudaMalloc, cudaFree or
// allocating library routine.

#include <mutex>

#include "dino_internal.cuh"

namespace dino {

// Scratch for the intermediate coefficients [nfields][M][J]; 16 MiB on every
// GPU that loads the library, held until the process exits.  In host code
// this name is only a stand-in: kernels receive the device address obtained
// from cudaGetSymbolAddress.  Every element a call reads is first written by
// the same call, so nothing has to be cleared between calls.
static __device__ __align__(256) float g_noalloc_scratch[DINO_NOALLOC_SCRATCH_FLOATS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
float* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).  The plan's tables live on the
// plan's device, so that device must be the current one.
int scratch_for_current_device(const dino_plan* p, float** out) {
  int dev = 0;
  DINO_CHECK_CUDA(cudaGetDevice(&dev));
  DINO_REQUIRE(dev == p->device, DINO_ERR_ARG,
               "dino_sht_inverse_noalloc: the plan belongs to device " +
                   std::to_string(p->device) + " but device " + std::to_string(dev) +
                   " is current");
  DINO_REQUIRE(dev >= 0 && dev < kMaxDevices, DINO_ERR_UNSUPPORTED,
               "dino_sht_inverse_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (err != cudaSuccess || ptr == nullptr) {
      set_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                cudaGetErrorString(err));
      return DINO_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<float*>(ptr);
  }
  *out = g_scratch_ptr[dev];
  return DINO_OK;
}

}  // namespace
}  // namespace dino

using namespace dino;

extern "C" int dino_sht_inverse_noalloc(dino_plan* p, const float* modal,
                                        float* nodal, int32_t nf,
                                        void* stream) {
  DINO_REQUIRE(p, DINO_ERR_ARG, "dino_sht_inverse_noalloc: null plan");
  DINO_REQUIRE(nf >= 0, DINO_ERR_SHAPE, "nfields must be >= 0");
  if (nf == 0) return DINO_OK;  // an empty batch is a no-op; buffers may be NULL
  DINO_REQUIRE(modal && nodal, DINO_ERR_ARG,
               "dino_sht_inverse_noalloc: null buffer");
  const long long need = (long long)nf * p->M * p->J;
  if (need > (long long)DINO_NOALLOC_SCRATCH_FLOATS) {
    set_error("dino_sht_inverse_noalloc: nfields * M * J = " +
              std::to_string(need) + " floats exceeds the fixed scratch of " +
              std::to_string((long long)DINO_NOALLOC_SCRATCH_FLOATS) +
              " floats; pass at most " +
              std::to_string((long long)DINO_NOALLOC_SCRATCH_FLOATS /
                             ((long long)p->M * p->J)) +
              " fields per call");
    return DINO_ERR_SHAPE;
  }
  float* scratch = nullptr;
  DINO_TRY(scratch_for_current_device(p, &scratch));
  cudaStream_t st = (cudaStream_t)stream;
  DINO_TRY(legendre_inverse_fp32(p, one_seg(modal, nf), scratch, nf, st));
  return fourier_inverse(p, scratch, nodal, nf, false, st);
}
