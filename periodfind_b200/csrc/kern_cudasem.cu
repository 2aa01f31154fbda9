// kern_cudasem.cu -- fold kernels with the arithmetic of the reference's
// CUDA build.  Compiled with -use_fast_math, exactly as the reference
// compiles periodfind/cuda/*.cu (setup.py:129).
#define PF_SEM_CPU_TU 0
#define PF_KNS sem_cuda
#define PF_SUFFIX cudasem
#include "pf_launch.h"
#include "pf_fold.cuh"
#include "pf_bin.cuh"
#include "pf_fpw.cuh"
#include "pf_lsrec.cuh"
#include "pf_binwarp.cuh"
#include "pf_kern_dispatch.inc"
