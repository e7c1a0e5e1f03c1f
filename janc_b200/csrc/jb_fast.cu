// FP64 production path: same kernels with FMA contraction enabled.
#define JB_NS fast
#define JB_FAST 1
#define JB_NS_NAME "fp64"
#define JB_OPS_NAME fast_ops
#include "jb_variant.inc"
