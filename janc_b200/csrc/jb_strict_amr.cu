// FP64 path with the reference's rounding (-fmad=false): the block-structured
// AMR stage and chemistry launchers.
#define JB_NS strict
#define JB_FAST 0
#define JB_NS_NAME "fp64_strict"
#define JB_OPS_NAME strict_ops
#define JB_PART JB_PART_AMR
#include "jb_variant.inc"
