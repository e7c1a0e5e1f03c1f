// FP64 path, FMA contraction: the block-structured AMR stage and chemistry
// launchers (also used by the mixed variant, whose blocks stay float64).
#define JB_NS fast
#define JB_FAST 1
#define JB_NS_NAME "fp64"
#define JB_OPS_NAME fast_ops
#define JB_PART JB_PART_AMR
#include "jb_variant.inc"
