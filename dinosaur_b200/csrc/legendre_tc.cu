// Tensor-core (tcgen05) Legendre contraction: placeholder until the
// split-BF16 kernels land; plans requesting DINO_PREC_BF16X3 are refused.
#include "dino_internal.cuh"

namespace dino {

int tc_tables_build(dino_plan* p) {
  (void)p;
  set_error("DINO_PREC_BF16X3 is not available in this build");
  return DINO_ERR_UNSUPPORTED;
}
void tc_tables_free(dino_plan* p) { (void)p; }
int tc_legendre_inverse(dino_plan*, const Segs&, float*, int, cudaStream_t) {
  set_error("DINO_PREC_BF16X3 is not available in this build");
  return DINO_ERR_UNSUPPORTED;
}
int tc_legendre_forward(dino_plan*, const float*, float*, int, cudaStream_t) {
  set_error("DINO_PREC_BF16X3 is not available in this build");
  return DINO_ERR_UNSUPPORTED;
}

}  // namespace dino
