// update_aux without any device allocation.
//
// Some callers of this library cannot allocate device memory themselves: the
// solver embedded as a plugin in a host application that reserves all device
// memory up front and forbids allocations after start-up, or a call made from
// inside another runtime's operator (for example an XLA custom call) whose
// device memory belongs to that runtime's allocator.  jb_create() allocates a
// workspace with cudaMalloc, so those callers cannot use a handle.  This entry
// point runs the same temperature solve as jb_update_aux() with its scratch
// (the six Halley-iterate planes and the reduction slots) taken from one
// file-scope __device__ array instead.
//
// The array is sized for JB_NOALLOC_MAX_CELLS cells (about 3.1 MB); every GPU
// that loads the library keeps it until the process exits.  All calls share
// it: calls whose kernels overlap on the GPU (different streams, or several
// host threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/janc_b200.h"
#include "jb_ops.h"

namespace {

constexpr int kMaxDevices = 64;

// [0, 256): reduction slots; then JB_NCAND planes of JB_NOALLOC_MAX_CELLS doubles
constexpr size_t kSlotBytes = 256;
constexpr size_t kScratchBytes = kSlotBytes + sizeof(double) * (size_t)JB_NCAND * JB_NOALLOC_MAX_CELLS;
static_assert(sizeof(jb_slots) <= kSlotBytes, "slots must fit the reserved prefix");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_lock;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (host code only
// sees a stand-in for the symbol).  Outside stream capture it is looked up
// on every call, so a device reset, after which the module can load at
// another address, never leaves a stale pointer; during a capture the
// address of this device's last uncaptured call is used (capture makes no
// lookup, which could load the module).
int scratch_address(cudaStream_t st, void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return JB_ERR_CUDA;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return JB_ERR_CUDA;
  std::lock_guard<std::mutex> guard(g_lock);
  if (cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return JB_ERR_CUDA;
    g_addr[dev] = p;
  } else if (!g_addr[dev]) {
    return JB_ERR_ARG;  // the first call on a device must not be captured
  }
  *out = g_addr[dev];
  return JB_OK;
}

}  // namespace

extern "C" int jb_update_aux_noalloc(const jb_mech_params* mech, int dim, int nx, int ny,
                                     int precision, const double* U, const double* aux_in,
                                     double* aux_out, void* stream) {
  if (!mech || !U || !aux_in || !aux_out) return JB_ERR_ARG;
  if (dim != 1 && dim != 2) return JB_ERR_ARG;
  if (dim == 1) ny = 1;
  if (nx < 1 || ny < 1) return JB_ERR_ARG;
  const long long ncell = (long long)nx * ny;
  if (ncell > JB_NOALLOC_MAX_CELLS) return JB_ERR_ARG;  // larger grids need jb_create
  if (mech->ns != 9 || mech->nr != 8 || mech->nreac != 19) return JB_ERR_UNSUPPORTED;
  // JB_PREC_MIXED is refused: its temperature solve is the fp64 one, and a
  // caller asking for it gets the fp64 result by passing JB_PREC_FP64
  if (precision != JB_PREC_STRICT && precision != JB_PREC_FP64) return JB_ERR_UNSUPPORTED;
  cudaStream_t st = (cudaStream_t)stream;
  void* base = nullptr;
  if (int rc = scratch_address(st, &base)) return rc;
  jb_mech_params m = *mech;
  jb::derive_mech(m);
  jb_grid g = {};
  g.nx = nx;
  g.ny = ny;
  g.nv = dim == 2 ? 12 : 11;
  g.nY = dim == 2 ? 4 : 3;
  g.ncell = ncell;
  g.dx = 1.0;
  g.dy = 1.0;
  g.idx = 1.0;
  g.idy = 1.0;
  g.inj_block_p = 1.0;
  g.lstrip = nx > ny ? nx : ny;
  jb_slots* slots = reinterpret_cast<jb_slots*>(base);
  double* cand = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kSlotBytes);
  const jb::Ops& o = precision == JB_PREC_STRICT ? jb::strict_ops : jb::fast_ops;
  // the slots keep the previous call's contents: clear them first
  if (o.slots_reset(slots, st) != cudaSuccess) return JB_ERR_CUDA;
  if (o.halley(dim, m, g, U, aux_in, cand, slots, 0, st) != cudaSuccess) return JB_ERR_CUDA;
  // cand planes are addressed with the grid's own cell count, so only the
  // first JB_NCAND * ncell doubles are touched
  if (o.select(dim, true, false, false, m, g, U, nullptr, cand, aux_out, nullptr, slots, 0, 0, nullptr, st) !=
      cudaSuccess)
    return JB_ERR_CUDA;
  return JB_OK;
}
