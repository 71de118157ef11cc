/* Declarations of the FFTW3 single-precision calls Radia's core names.  The
 * image has no FFTW, and the core calls it only from its particle-trajectory
 * module (radptrj.cpp), which the relaxation path never reaches: each call
 * here prints what was called and aborts, so a call cannot go unnoticed. */
#ifndef RADB200_SHIM_FFTW3_H
#define RADB200_SHIM_FFTW3_H
#include <stdio.h>
#include <stdlib.h>
typedef float fftwf_complex[2];
typedef struct radb200_fftwf_plan_s *fftwf_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
static inline void radb200_no_fftw(const char *f)
{ fprintf(stderr, "radia built without FFTW: %s called\n", f); abort(); }
static inline void *fftwf_malloc(size_t n) { (void)n; radb200_no_fftw("fftwf_malloc"); return 0; }
static inline void fftwf_free(void *p) { (void)p; radb200_no_fftw("fftwf_free"); }
static inline fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *i, fftwf_complex *o, int s, unsigned f)
{ (void)n; (void)i; (void)o; (void)s; (void)f; radb200_no_fftw("fftwf_plan_dft_1d"); return 0; }
static inline fftwf_plan fftwf_plan_dft_2d(int a, int b, fftwf_complex *i, fftwf_complex *o, int s, unsigned f)
{ (void)a; (void)b; (void)i; (void)o; (void)s; (void)f; radb200_no_fftw("fftwf_plan_dft_2d"); return 0; }
static inline void fftwf_destroy_plan(fftwf_plan p) { (void)p; radb200_no_fftw("fftwf_destroy_plan"); }
static inline void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *i, fftwf_complex *o)
{ (void)p; (void)i; (void)o; radb200_no_fftw("fftwf_execute_dft"); }
#endif
