// FP64 kernels compiled with -fmad=false: every multiply and add rounds separately, as the
// reference's x86-64 build does, so results compare bitwise with the CPU restatement.
#define PIP_FLAVOUR exact
#define PIP_RCP 0
#define PIP_LAUNCHERS launchers_exact
#include "pip_step_impl.cuh"
