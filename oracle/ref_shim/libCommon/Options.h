// Stand-in for the absent libCommon/Options.h (test infrastructure for oracle/_ref).
#ifndef RTM_SHIM_OPTIONS_H
#define RTM_SHIM_OPTIONS_H
#endif
