// FP64 path, FMA contraction: flux-splitting stage launchers.
#define JB_NS fast
#define JB_FAST 1
#define JB_NS_NAME "fp64"
#define JB_OPS_NAME fast_ops
#define JB_PART JB_PART_FLUX64
#include "jb_variant.inc"
