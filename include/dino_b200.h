/*
 * dino_b200 -- C ABI of the B200-native spectral dynamical-core step.
 *
 * Every entry point returns an int status (DINO_OK = 0) and never throws;
 * dino_last_error() returns a thread-local message for the last failure.
 * Pointers named d_* are device pointers; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream).  Array layouts follow the reference:
 *   nodal  [fields][longitude I][latitude J]  (latitude fastest, ascending sin)
 *   modal  [fields][M = 2*lw-1][L = tw]       (rows m = 0, +1, -1, +2, -2, ...)
 * Objects (plans, equations) are immutable after creation except for internal
 * caches and may be shared by threads that use distinct streams; calls that
 * share a workspace must not overlap in time (one stream per object).
 *
 * Reference interfaces replaced (neuralgcm/dinosaur 1.3.6, file:line):
 *   dino_plan_create        Grid.spherical_harmonics / RealSphericalHarmonics.basis
 *                           (dinosaur/spherical_harmonic.py:935-949, :219-260),
 *                           associated_legendre.evaluate / gauss_legendre_nodes
 *                           (dinosaur/associated_legendre.py:70-114)
 *   dino_sht_inverse        Grid.to_nodal -> RealSphericalHarmonics.inverse_transform
 *                           (dinosaur/spherical_harmonic.py:1017-1023, :262-269)
 *   dino_sht_forward        Grid.to_modal -> RealSphericalHarmonics.transform
 *                           (dinosaur/spherical_harmonic.py:1025-1031, :271-280)
 *   dino_sht_*_adjoint      the VJPs JAX derives for the two einsum pairs above
 *   dino_modal_op           Grid.d_dlon / cos_lat_d_dlat / sec_lat_d_dlat_cos2 /
 *                           laplacian / inverse_laplacian / clip_wavenumbers
 *                           (dinosaur/spherical_harmonic.py:1033-1102)
 *   dino_pe_create          PrimitiveEquationsSigma.__init__ + weight matrices
 *                           (dinosaur/primitive_equations.py:283-598, :697-724)
 *   dino_pe_explicit        PrimitiveEquationsSigma.explicit_terms (:1126-1194)
 *   dino_pe_implicit        PrimitiveEquationsSigma.implicit_terms (:1196-1249)
 *   dino_pe_implicit_inverse PrimitiveEquationsSigma.implicit_inverse, 'split'
 *                           (:1251-1330)
 *   dino_pe_step            step_with_filters(imex_rk_sil3(eq, dt), [filter])
 *                           repeated n times (dinosaur/time_integration.py:375-405,
 *                           :427-455, :494-520)
 */
#ifndef DINO_B200_H_
#define DINO_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DINO_API __attribute__((visibility("default")))
#else
#define DINO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define DINO_OK 0
#define DINO_ERR_ARG 1         /* bad argument (null pointer, bad enum)      */
#define DINO_ERR_SHAPE 2       /* inconsistent sizes                         */
#define DINO_ERR_CUDA 3        /* a CUDA runtime call failed                 */
#define DINO_ERR_TIMEOUT 4     /* a bounded device wait gave up              */
#define DINO_ERR_NAN 5         /* non-finite value where the reference asserts */
#define DINO_ERR_UNSUPPORTED 6 /* configuration not supported by this build  */

/* Latitude spacings (spherical_harmonic.py:43-47). */
#define DINO_SPACING_GAUSS 0
#define DINO_SPACING_EQUIANGULAR 1
#define DINO_SPACING_EQUIANGULAR_WITH_POLES 2

/* Legendre-contraction arithmetic. */
#define DINO_PREC_FP32 0    /* SIMT FP32 FMA (plain form)                          */
#define DINO_PREC_BF16X3 1  /* tcgen05 kind::f16, hi*hi + hi*lo + lo*hi, FP32 accum */
#define DINO_PREC_TF32X3 2  /* tcgen05 kind::tf32, hi*hi + hi*lo + lo*hi, FP32 accum */

/* Modal operators for dino_modal_op. */
#define DINO_OP_D_DLON 0
#define DINO_OP_COS_LAT_D_DLAT 1
#define DINO_OP_SEC_LAT_D_DLAT_COS2 2
#define DINO_OP_LAPLACIAN 3
#define DINO_OP_INVERSE_LAPLACIAN 4
#define DINO_OP_CLIP 5

typedef struct dino_grid_desc {
  int32_t longitude_wavenumbers; /* lw: m in [0, lw)                 */
  int32_t total_wavenumbers;     /* tw = L: l in [0, tw)             */
  int32_t longitude_nodes;       /* I                                */
  int32_t latitude_nodes;        /* J                                */
  int32_t latitude_spacing;      /* DINO_SPACING_*                   */
  int32_t reserved;
  double radius;                 /* sphere radius (nondimensional)   */
  /* Optional host arrays (length J) of sin(latitude) nodes and weights for
   * non-Gauss spacings; NULL for Gauss nodes, which are built on the GPU. */
  const double* host_nodes;
  const double* host_weights;
} dino_grid_desc;

typedef struct dino_plan dino_plan;
typedef struct dino_pe dino_pe;

/* Copies the last error message of this thread into buf (NUL-terminated). */
DINO_API int dino_last_error(char* buf, size_t len);
/* Library version string, e.g. "dino_b200 0.1 sm_100a". */
DINO_API const char* dino_version(void);

/* Builds a transform plan on the current device: FP64 Gauss nodes/weights and
 * associated-Legendre tables computed on the GPU, rounded to the working
 * precision; a workspace for up to max_fields fields per call. */
DINO_API int dino_plan_create(const dino_grid_desc* desc, int32_t max_fields,
                     int32_t precision, dino_plan** out);
DINO_API int dino_plan_destroy(dino_plan* plan);
/* Copies the FP64 sin(latitude) nodes and quadrature weights (length J). */
DINO_API int dino_plan_nodes(const dino_plan* plan, double* host_sin_lat,
                    double* host_weights);
/* Copies the FP32 Legendre table entry p[m, j, l] for one (m, l) over all j
 * into host_out (length J); used by tests. */
DINO_API int dino_plan_legendre_column(const dino_plan* plan, int32_t m, int32_t l,
                              double* host_out);

/* A one-line description of the plan (shapes, Legendre form, and for the
 * tensor-core forms the launch shapes its autotuner chose at creation and
 * their measured times), NUL-terminated and truncated to len bytes.  No
 * counterpart in the reference. */
DINO_API int dino_plan_describe(dino_plan* plan, char* buf, size_t len);

/* Synchronizes the device and reports whether any bounded device-side wait
 * of this plan's kernels gave up (DINO_ERR_TIMEOUT, after which the flag is
 * cleared); DINO_OK otherwise.  Replaces the reference's reliance on XLA
 * raising at dispatch; no direct counterpart. */
DINO_API int dino_plan_status(dino_plan* plan);

/* Diagnostic of the failure path (no counterpart in the reference): launches
 * one CTA on `stream` whose bounded wait, the routine every tensor-core
 * pipeline wait uses, waits on an mbarrier that nothing completes; after
 * limit_ns (1 ms .. 10 s) it gives up and records a code in the plan's device
 * error flag, so that the next dino_plan_status returns DINO_ERR_TIMEOUT.
 * The context stays usable.  Tensor-core plans only (else
 * DINO_ERR_UNSUPPORTED). */
DINO_API int dino_plan_check_wait_timeout(dino_plan* plan, int64_t limit_ns,
                                          void* stream);

/* Allocation-free inverse transform (no counterpart in the reference).
 * Same result as dino_sht_inverse on an FP32 plan, but the intermediate
 * Fourier coefficients live in a fixed array of DINO_NOALLOC_SCRATCH_FLOATS
 * floats (16 MiB) inside the library, held on every GPU that loads it, instead
 * of the plan's workspace; the call performs no device allocation or free.
 * It is meant for callers that may not allocate device memory at call time,
 * for example a handler inside a framework that owns the GPU's memory pool,
 * or a loop that cannot afford cudaMalloc's implicit device synchronization.
 * The plan must already exist (its tables are read, not written) and its
 * device must be the current one (otherwise DINO_ERR_ARG).  nfields = 0 is a
 * no-op with NULL buffers allowed.  Limits and
 * rules: nfields * M * J <= DINO_NOALLOC_SCRATCH_FLOATS, otherwise
 * DINO_ERR_SHAPE; the Legendre contraction always runs in FP32; the first
 * call on a device looks the array up (cudaGetSymbolAddress) and sets kernel
 * attributes, so make that first call before any stream capture; all calls on
 * a device share the one array, so calls that overlap on the GPU (different
 * streams or threads) race and must be serialised by the caller. */
#define DINO_NOALLOC_SCRATCH_FLOATS (4 * 1024 * 1024)
DINO_API int dino_sht_inverse_noalloc(dino_plan* plan, const float* d_modal,
                                      float* d_nodal, int32_t nfields,
                                      void* stream);

/* modal [nfields][M][L] -> nodal [nfields][I][J].  For every batch entry
 * point, nfields = 0 is a no-op and its buffers may then be NULL. */
DINO_API int dino_sht_inverse(dino_plan* plan, const float* d_modal, float* d_nodal,
                     int32_t nfields, void* stream);
/* nodal [nfields][I][J] -> modal [nfields][M][L]. */
DINO_API int dino_sht_forward(dino_plan* plan, const float* d_nodal, float* d_modal,
                     int32_t nfields, void* stream);
/* Transposes of the two maps above: nodal cotangent -> modal cotangent and
 * modal cotangent -> nodal cotangent. */
DINO_API int dino_sht_inverse_adjoint(dino_plan* plan, const float* d_nodal_ct,
                             float* d_modal_ct, int32_t nfields, void* stream);
DINO_API int dino_sht_forward_adjoint(dino_plan* plan, const float* d_modal_ct,
                             float* d_nodal_ct, int32_t nfields, void* stream);
/* One phase of the transform pair, for profiling and composition:
 *   DINO_PHASE_LEGENDRE_INVERSE  modal [nf][M][L] -> Fourier [nf][M][J]
 *   DINO_PHASE_FOURIER_INVERSE   Fourier [nf][M][J] -> nodal [nf][I][J]
 *   DINO_PHASE_FOURIER_FORWARD   nodal [nf][I][J] -> weighted Fourier [nf][M][J]
 *   DINO_PHASE_LEGENDRE_FORWARD  weighted Fourier [nf][M][J] -> modal [nf][M][L]
 * nf must not exceed the plan's max_fields. */
#define DINO_PHASE_LEGENDRE_INVERSE 0
#define DINO_PHASE_FOURIER_INVERSE 1
#define DINO_PHASE_FOURIER_FORWARD 2
#define DINO_PHASE_LEGENDRE_FORWARD 3
DINO_API int dino_sht_phase(dino_plan* plan, int32_t phase, const float* d_in,
                            float* d_out, int32_t nfields, void* stream);
/* One spectral operator (DINO_OP_*) on modal [nfields][M][L]; `arg` is the
 * number of wavenumbers to clip for DINO_OP_CLIP and is ignored otherwise. */
DINO_API int dino_modal_op(dino_plan* plan, int32_t op, const float* d_in, float* d_out,
                  int32_t nfields, int32_t arg, void* stream);

/* Primitive equations on sigma levels.  Packed state layout (device, FP32),
 * kind-major so each kind is contiguous over members and levels:
 *   [vorticity  members*K][divergence members*K][temperature members*K]
 *   [tracer_0 members*K]...[tracer_{n-1} members*K][log_ps members]
 * each entry one modal [M][L] plane. */
typedef struct dino_pe_desc {
  int32_t layers;              /* K                                        */
  int32_t members;             /* ensemble members in one launch           */
  int32_t n_tracers;
  int32_t humidity_tracer;     /* index of specific humidity, -1 if dry    */
  int32_t include_vertical_advection;
  int32_t held_suarez;         /* 1: add HeldSuarezForcingSigma tendencies */
  const double* sigma_boundaries;     /* host, K+1 (the reference's dtype) */
  const double* sigma_centers;        /* host, K                           */
  const double* layer_thickness;      /* host, K                           */
  const double* inv_center_to_center; /* host, K-1: 1/(sigma[k+1]-sigma[k]) as the
                                         reference forms it (in the sigma dtype) */
  const double* reference_temperature;/* host, K                           */
  const double* geopotential_weights; /* host, K*K (G, includes R)         */
  const double* temperature_weights;  /* host, K*K (H)                     */
  const double* sigma_ratios;         /* host, K (alpha)                   */
  const float* orography_modal;       /* host, M*L (modal orography)       */
  double angular_velocity, gravity, R, R_vapor, Cp_vapor, kappa;
  /* Held-Suarez constants (nondimensional), used when held_suarez = 1. */
  double hs_p0, hs_sigma_b, hs_kf, hs_ka, hs_ks, hs_minT, hs_maxT, hs_dTy,
      hs_dThz;
  /* Vertical coordinate: 0 sigma levels (PrimitiveEquationsSigma), 1 hybrid
   * sigma-pressure levels p = a + b p_s (PrimitiveEquationsHybrid,
   * primitive_equations.py:1961-2533; no Held-Suarez, no explicit-term or
   * step VJP).  For hybrid levels geopotential_weights and
   * temperature_weights hold the hybrid G and H at p_s_ref, and the
   * sigma-only arrays above are placeholders of their sizes (layer_thickness
   * must be positive). */
  int32_t vertical_scheme;
  const double* hybrid_a_boundaries;  /* host, K+1, nondimensional pressure  */
  const double* hybrid_b_boundaries;  /* host, K+1                           */
  double reference_surface_pressure;  /* nondimensional p_s_ref              */
  /* The implicit operator's ln ps column c and ln ps row w
   * (d div_k/dt = -lap(sum_j G_kj T_j + c_k ln ps), d ln ps/dt = -sum_k w_k
   * div_k); NULL gives the sigma values R T_ref and layer_thickness.  Hybrid:
   * the pressure-gradient coefficient at p_s_ref and da / p_s_ref + db. */
  const double* implicit_lnps_column; /* host, K, or NULL                    */
  const double* implicit_thickness;   /* host, K, or NULL                    */
} dino_pe_desc;

DINO_API int dino_pe_create(dino_plan* plan, const dino_pe_desc* desc, dino_pe** out);
DINO_API int dino_pe_destroy(dino_pe* pe);
/* Size in floats of one packed state. */
DINO_API int64_t dino_pe_state_size(const dino_pe* pe);
/* Plane counts of the engine's work, for traffic accounting (no counterpart
 * in the reference): counts[0] state planes, [1] modal auxiliary planes made
 * by the pre-pass, [2] fields of the inverse transform, [3] fields of the
 * forward transform, [4] implicit planes (members x (2K + 1)); each plane
 * is one [M][L] (modal) or [I][J] (nodal) array. */
DINO_API int dino_pe_counts(const dino_pe* pe, int32_t* counts);
DINO_API int dino_pe_explicit(dino_pe* pe, const float* d_state, float* d_tendency,
                     void* stream);
DINO_API int dino_pe_implicit(dino_pe* pe, const float* d_state, float* d_out,
                     void* stream);
DINO_API int dino_pe_implicit_inverse(dino_pe* pe, const float* d_state, float* d_out,
                             double step_size, void* stream);
/* Advances d_state in place by n_steps of imex_rk_sil3 with time step dt,
 * followed each step by multiplication with the per-l filter scaling
 * (host array of length L, e.g. the exponential step filter; NULL = none). */
DINO_API int dino_pe_step(dino_pe* pe, float* d_state, double dt,
                 const double* host_filter, int32_t n_steps, void* stream);
/* Captures one filtered step into a CUDA graph (created on first use for this
 * (dt, filter)); dino_pe_step_graph then replays it n_steps times. */
DINO_API int dino_pe_step_graph(dino_pe* pe, float* d_state, double dt,
                       const double* host_filter, int32_t n_steps,
                       void* stream);
/* trajectory_from_step(step, outer_steps, inner_steps, start_with_input)
 * (dinosaur/time_integration.py:523-564) for the filtered SIL3 step: advances
 * d_state in place by outer_steps x inner_steps steps and writes outer_steps
 * frames of the packed state (dino_pe_state_size floats each) to d_frames:
 * the state after each block of inner_steps steps, or before it when
 * start_with_input is nonzero.  The steps replay the captured step graph and
 * each frame is a device-to-device copy on the same stream, so the host
 * issues the whole rollout without waiting.  d_frames must not overlap
 * d_state. */
DINO_API int dino_pe_trajectory(dino_pe* pe, float* d_state, double dt,
                                const double* host_filter, int32_t outer_steps,
                                int32_t inner_steps, int32_t start_with_input,
                                float* d_frames, void* stream);

/* Converts modal arrays between the Real layout ([M = 2 lw - 1][L], rows
 * m = 0, 1, -1, ...) and the FastSphericalHarmonics layout ([2 lw][L], rows
 * m = 0, 0 (imaginary, zero), 1, -1, ...; spherical_harmonic.py:411-621):
 * to_fast = 1 inserts the zero row, 0 drops it.  in and out must differ. */
DINO_API int dino_modal_relayout(dino_plan* plan, int32_t to_fast,
                                 const float* d_in, float* d_out,
                                 int32_t nfields, void* stream);

/* ---- Shallow-water equations (shallow_water.py:121-230) ------------------
 * Packed state, kind-major: [vorticity: members*layers][divergence]
 * [potential] planes of [M][L] in the plan's real modal layout. */
typedef struct dino_swe dino_swe;

typedef struct dino_swe_desc {
  int32_t layers;                    /* K */
  int32_t members;                   /* ensemble members, >= 1 */
  const double* reference_potential; /* [K] mean geopotential per layer */
  const double* densities;           /* [K] from the top, or NULL (all 1) */
  const float* orography_modal;      /* [M][L] or NULL */
  double angular_velocity;           /* nondimensional Omega */
} dino_swe_desc;

/* ShallowWaterEquations(coords, physics_specs, orography,
 * reference_potential, densities) (shallow_water.py:121-140). */
DINO_API int dino_swe_create(dino_plan* plan, const dino_swe_desc* desc,
                             dino_swe** out);
DINO_API int dino_swe_destroy(dino_swe* swe);
DINO_API int64_t dino_swe_state_size(const dino_swe* swe);
/* explicit_terms (shallow_water.py:158-205); out must not alias state. */
DINO_API int dino_swe_explicit(dino_swe* swe, const float* d_state,
                               float* d_out, void* stream);
/* implicit_terms (:207-213). */
DINO_API int dino_swe_implicit(dino_swe* swe, const float* d_state,
                               float* d_out, void* stream);
/* implicit_inverse(state, eta), closed form per l (:215-230); in place
 * allowed. */
DINO_API int dino_swe_implicit_inverse(dino_swe* swe, const float* d_state,
                                       float* d_out, double eta, void* stream);

/* ---- Reverse mode (vector-Jacobian products) ----------------------------
 * The reference differentiates its step with jax.vjp / jax.grad through the
 * JAX einsums of explicit_terms, implicit_terms and implicit_inverse
 * (primitive_equations.py:1126-1330) and the imex_rk_sil3 stages
 * (time_integration.py:329-405); these entries are the hand-written
 * equivalents on the packed state layout.  Each allocates the adjoint work
 * buffers of `pe` on first use. */

/* d_state_ct = (d explicit_terms / d state)^T d_tend_ct at d_state.
 * d_state_ct must not alias the inputs. */
DINO_API int dino_pe_explicit_vjp(dino_pe* pe, const float* d_state,
                                  const float* d_tend_ct, float* d_state_ct,
                                  void* stream);
/* d_in_ct = G^T d_out_ct for the linear implicit_terms G (buffers differ). */
DINO_API int dino_pe_implicit_vjp(dino_pe* pe, const float* d_out_ct,
                                  float* d_in_ct, void* stream);
/* d_in_ct = ((1 - eta G)^-1)^T d_out_ct (in place allowed). */
DINO_API int dino_pe_implicit_inverse_vjp(dino_pe* pe, const float* d_out_ct,
                                          float* d_in_ct, double eta,
                                          void* stream);
/* VJP of one filtered SIL3 step taken from d_state (not modified):
 * d_in_ct = (d step / d state)^T d_out_ct.  The stage states are recomputed
 * from d_state, so a rollout's backward pass needs only the per-step input
 * states (per-step checkpointing).  d_in_ct may alias d_out_ct. */
DINO_API int dino_pe_step_vjp(dino_pe* pe, const float* d_state,
                              const float* d_out_ct, float* d_in_ct, double dt,
                              const double* host_filter, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DINO_B200_H_ */
