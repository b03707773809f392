/* Oracle build shim (test infrastructure only): see ppl.h. */
#ifndef ORACLE_SHIM_PPLTASKS_H_
#define ORACLE_SHIM_PPLTASKS_H_
#include "ppl.h"
#endif
