// Stand-in for fftw3.h: the types the engine headers name and the
// single-precision 1-D r2c / c2r / r2r calls FdEngine_r2c and FdEngine_r2r
// make, computed as plain sums in double by the definitions FFTW documents
// (ref_shim.cpp).
#ifndef RTM_SHIM_FFTW3_H
#define RTM_SHIM_FFTW3_H
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
typedef enum {
  FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
  FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
  FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;
typedef fftw_r2r_kind fftwf_r2r_kind;
fftwf_plan fftwf_plan_r2r_1d(int n, float *in, float *out, fftwf_r2r_kind kind, unsigned flags);
void fftwf_execute_r2r(const fftwf_plan p, float *in, float *out);
void fftwf_destroy_plan(fftwf_plan p);
#endif
