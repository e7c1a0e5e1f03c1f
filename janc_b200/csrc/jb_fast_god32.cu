// Mixed path: Godunov stage launchers with float32 reconstruction.
#define JB_NS fast
#define JB_FAST 1
#define JB_NS_NAME "fp64"
#define JB_OPS_NAME fast_ops
#define JB_PART JB_PART_GOD32
#include "jb_variant.inc"
