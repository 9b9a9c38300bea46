/* Stand-in for the FFTW declarations the reference's headers name
 * (common/fftwHao/include/fftw_hao.h); FFTW is not on the AFQMC walker-step
 * path and fftw_hao.cpp is not built.  Oracle reference build only. */
#pragma once
typedef double fftw_complex[2];
typedef struct or_fftw_plan_s *fftw_plan;
