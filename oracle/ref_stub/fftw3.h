/* Stand-in for the FFTW3 single-precision API, used only to compile the
 * reference Radia CPU module as a test oracle.  The reference calls FFTW only
 * from its particle-trajectory code, which the oracle never exercises; every
 * entry point here aborts so an accidental call cannot go unnoticed. */
#ifndef ORACLE_FFTW3_STUB_H
#define ORACLE_FFTW3_STUB_H
#include <stdio.h>
#include <stdlib.h>
typedef float fftwf_complex[2];
typedef struct oracle_fftwf_plan_s *fftwf_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
static inline void oracle_fftw_absent(const char *f)
{ fprintf(stderr, "oracle build has no FFTW: %s called\n", f); abort(); }
static inline void *fftwf_malloc(size_t n) { (void)n; oracle_fftw_absent("fftwf_malloc"); return 0; }
static inline void fftwf_free(void *p) { (void)p; oracle_fftw_absent("fftwf_free"); }
static inline fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *i, fftwf_complex *o, int s, unsigned f)
{ (void)n; (void)i; (void)o; (void)s; (void)f; oracle_fftw_absent("fftwf_plan_dft_1d"); return 0; }
static inline fftwf_plan fftwf_plan_dft_2d(int a, int b, fftwf_complex *i, fftwf_complex *o, int s, unsigned f)
{ (void)a; (void)b; (void)i; (void)o; (void)s; (void)f; oracle_fftw_absent("fftwf_plan_dft_2d"); return 0; }
static inline void fftwf_destroy_plan(fftwf_plan p) { (void)p; oracle_fftw_absent("fftwf_destroy_plan"); }
static inline void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *i, fftwf_complex *o)
{ (void)p; (void)i; (void)o; oracle_fftw_absent("fftwf_execute_dft"); }
#endif
