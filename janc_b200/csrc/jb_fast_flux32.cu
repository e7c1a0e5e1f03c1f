// Mixed path: float32 flux-splitting stage launchers and the 2D x-sweep / y-run kernels.
#define JB_NS fast
#define JB_FAST 1
#define JB_NS_NAME "fp64"
#define JB_OPS_NAME fast_ops
#define JB_PART JB_PART_FLUX32
#include "jb_variant.inc"
