// Stand-in for the absent libFFTV/baseinc.h (test infrastructure for oracle/_ref).
#ifndef RTM_SHIM_FFTV_BASEINC_H
#define RTM_SHIM_FFTV_BASEINC_H
#endif
