// kern_cpusem.cu -- fold kernels with the arithmetic of the reference's CPU
// path (rust/src/*.rs): compiled with IEEE divides and square roots, no
// flush-to-zero and no multiply-add contraction.
#define PF_SEM_CPU_TU 1
#define PF_KNS sem_cpu
#define PF_SUFFIX cpusem
#include "pf_launch.h"
#include "pf_fold.cuh"
#include "pf_bin.cuh"
#include "pf_fpw.cuh"
#include "pf_lsrec.cuh"
#include "pf_binwarp.cuh"
#include "pf_kern_dispatch.inc"
