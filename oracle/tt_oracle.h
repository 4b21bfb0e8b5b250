/*
 * ORACLE -- test infrastructure only.
 *
 * CPU double-precision restatement of ToyTrace's forward path tracer with next-event
 * estimation (`--algo pt`).  It exists to check the CUDA product path: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and never as the
 * thing measured or shipped.  See tt_oracle.cpp for the per-function reference citations.
 *
 * Parity status: the reference itself cannot be built here (Embree, Eigen, TBB, Boost,
 * yaml-cpp, pcg32 and others are absent), so this restatement is pinned against the
 * reference's own known-answer tests (spectral round trips, reflect/refract, intersector
 * tests, RNG) and golden tables extracted from the reference source text
 * (tests/golden/).  Exact Embree hit ids and exact RNG streams are unpinned; image parity
 * is statistical.
 */
#ifndef TT_ORACLE_H
#define TT_ORACLE_H

#include <stdint.h>
#include "../include/toytrace_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_scene or_scene;

or_scene* or_create(const tt_scene_desc* scene, const tt_params* params);
void or_destroy(or_scene* s);
const char* or_last_error(void);

/* rays: n*8 doubles (org, tnear, dir, tfar). brute_force!=0 tests every triangle. */
int or_intersect(or_scene* s, const double* rays, int n, int brute_force,
                 int32_t* prim, double* t, double* u, double* v);
int or_occluded(or_scene* s, const double* rays, int n, uint8_t* occluded);

/* Renders spp samples per pixel for pixels [pixel_begin, pixel_end) with global sample
 * numbers sample_offset .. sample_offset+spp-1.  Adds into accum / light_accum (npix*3)
 * and *splat_count (number of samples inserted).  nthreads <= 0: hardware threads. */
int or_render(or_scene* s, int spp, uint64_t seed, int sample_offset, int pixel_begin,
              int pixel_end, int nthreads, double* accum, double* light_accum,
              uint64_t* splat_count);

/* Shader sampling on a z-up surface (see tt_sample_bsdf_batch). */
int or_sample_bsdf(or_scene* s, int material, const double* wi, const int32_t* lambda_idx,
                   int n, uint64_t seed, double* out_dir, double* out_value, double* out_pdf);
int or_eval_bsdf(or_scene* s, int material, const double* wi, const int32_t* lambda_idx,
                 const double* dirs, int n, double* out_value, double* out_pdf);

/* Known-answer helpers. */
void or_rgb_to_spectrum(const double* rgb, double* spectrum36);
void or_spectrum_to_rgb(const double* spectrum36, double* rgb);
void or_selection_to_rgb(const double* val3, const int32_t* idx3, double* rgb);
void or_rgb_to_selection(const double* rgb, const int32_t* idx3, double* val3);
void or_reflected(const double* wi, const double* n, double* out);
int or_refracted(const double* wi, const double* n, double eta_i_over_t, double* out);
void or_half_vector(const double* wi, const double* wo, double* out);
int or_half_vector_refracted(const double* wi, const double* wo, double eta, double* out);
double or_fresnel(double cos_i, double eta_i_over_t);
void or_pcg32_stream(uint64_t initstate, uint64_t initseq, int n, uint32_t* out);
double or_pcg32_nextdouble_first(uint64_t initstate, uint64_t initseq);
int or_uniform_int_stream(uint64_t initstate, uint64_t initseq, int a, int b, int n, int32_t* out);
void or_tables(double* smits7x36, double* m3x36, double* sun36);
/* Environment light evaluation for tests: radiance of all env lights into direction
 * dir_out (the direction the light travels) and the NEE pdf (TotalEnv EvaluatePdf). */
int or_eval_env(or_scene* s, const double* dir_out, const int32_t* lambda_idx, double* value3, double* pdf);
int or_scene_info(or_scene* s, double* bbox6, int32_t* counts4);
int or_medium_walk(or_scene* s, const double* org3, const double* dir3, double tfar, int max, int32_t* media,
                   double* ts, int32_t* initial);
int or_transmittance(or_scene* s, const double* org3, const double* dir3, double length, const int32_t* idx,
                     uint64_t seed, double* T3, double* coeff3);
int or_track(or_scene* s, const double* org3, const double* dir3, const int32_t* idx, int n, uint64_t seed,
             double* out);
int or_atmosphere_query(or_scene* s, int medium, const double* pos3, const double* org3, const double* dir3,
                        double length, const int32_t* idx, double* out);
int or_medium_phase_sample(or_scene* s, int medium, const double* pos3, const double* wi3, const int32_t* idx, int n,
                           uint64_t seed, double* dirs, double* value3, double* pdf);
int or_phase_sample(int kind, double g, const double* wi3, int n, uint64_t seed, double* dirs, double* pdf,
                    double* value);
/* Quasi-random sampler: SobolSequence(point, dim) for n points (dim < 4096); the generator
 * matrix (32 columns) for given Joe-Kuo parameters; and the draws of QuasiRandomSequence
 * for a pixel and point: `ops` holds per draw 0 = Uniform01, 1 = UniformUnitSquare,
 * 2 + id = SetSubsequenceId(id) (no output). */
int or_sobol(int dim, int n, const uint32_t* points, double* out);
void or_sobol_matrix(int s, int a, const uint16_t* m, uint32_t* out32);
int or_qmc_draws(int px, int py, uint32_t point, int n_ops, const int32_t* ops, uint64_t pcg_seed, double* out);

#ifdef __cplusplus
}
#endif

#endif
