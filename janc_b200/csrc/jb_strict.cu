// FP64 path with the reference's rounding: compiled with -fmad=false so that
// no multiply-add pair is contracted and each expression rounds as NumPy/XLA
// float64 does.  Transcendentals (exp, log, pow) are CUDA's.  Launchers
// other than the stage kernels, and the variant's Ops table.
#define JB_NS strict
#define JB_FAST 0
#define JB_NS_NAME "fp64_strict"
#define JB_OPS_NAME strict_ops
#define JB_PART JB_PART_MAIN
#include "jb_variant.inc"
