// FP64 kernels with FMA contraction (the default drop-in build).
#define PIP_FLAVOUR fast
#define PIP_RCP 1
#define PIP_LAUNCHERS launchers_fast
#include "pip_step_impl.cuh"
