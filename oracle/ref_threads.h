// Force-included ahead of the reference sources when the oracle builds them
// (test infrastructure only).  The reference hard-codes its OpenMP thread
// count as a macro, THREADS_NUM_USED = 16 (cpp/paramSetting.hpp:11).  The
// header is pulled in first here (it is `#pragma once`, so the sources' own
// `#include "../paramSetting.hpp"` is then skipped) and the macro is
// redefined to a run-time query, so the compiled reference uses the number of
// host cores the process may run on, or CBMV_REF_THREADS when that is set.
#pragma once
#include "paramSetting.hpp"
#undef THREADS_NUM_USED
#ifdef __cplusplus
extern "C"
#endif
int cbmv_ref_threads(void);
#define THREADS_NUM_USED (cbmv_ref_threads())
