// Stand-in for fftw3.h: only the types named by engine headers; no FFT is run.
#ifndef RTM_SHIM_FFTW3_H
#define RTM_SHIM_FFTW3_H
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;
#endif
