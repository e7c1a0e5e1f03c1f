// FP64 production path: same kernels with FMA contraction enabled (launchers
// other than the stage kernels, and the Ops tables of the fp64 and mixed variants).
#define JB_NS fast
#define JB_FAST 1
#define JB_NS_NAME "fp64"
#define JB_OPS_NAME fast_ops
#define JB_PART JB_PART_MAIN
#include "jb_variant.inc"
