// Allocation-free Hilbert keys + sort.
//
// Some callers of this library cannot call cudaMalloc: a simulation that
// hands the solver device arrays from its own pool or arena allocator and
// forbids any other allocation (so its memory budget stays fixed for the
// whole run), or code that runs inside a region where allocating would stall
// or break it (a stream-ordered pipeline that must not synchronise, a host
// callback).  tpm_hilbert_sort_noalloc serves them: the caller passes the
// inputs and outputs, and every intermediate buffer the radix sort needs
// (ping-pong copies, per-tile digit counts, the digit histogram) and the
// bounding-box scratch live in one file-scope __device__ array below.  That
// array is sized for TPM_NOALLOC_MAX_PARTICLES and, like every __device__
// variable, is held on each GPU that loads this library until the process
// exits.  All calls share it, so two calls whose work overlaps on the GPU
// (different streams, or different host threads on one device) race and
// corrupt each other's results; callers serialise them.
#include <mutex>

#include "../../include/treepm_b200.h"
#include "common.cuh"
#include "sort.cuh"
#include "tree.cuh"

namespace {

constexpr int64_t NOALLOC_MAX = TPM_NOALLOC_MAX_PARTICLES;
// bounding box words + TreeParams, then the radix-sort scratch
constexpr size_t NOALLOC_PARAMS_BYTES = 512;
// the sort's own sizing rule at the largest accepted n, so every n <= NOALLOC_MAX fits
constexpr size_t NOALLOC_SORT_BYTES = tpm::radix_sort_scratch_bytes(NOALLOC_MAX);
static_assert(NOALLOC_SORT_BYTES >= tpm::radix_sort_scratch_bytes(NOALLOC_MAX - 1),
              "scratch sizing must grow with n");
constexpr size_t NOALLOC_BYTES = NOALLOC_PARAMS_BYTES + NOALLOC_SORT_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of g_noalloc_scratch per device ordinal.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and reused.
constexpr int MAX_DEVICES = 64;
unsigned char* g_scratch_addr[MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

unsigned char* scratch_for_current_device(int dev) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    TPM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int tpm_hilbert_sort_noalloc(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n,
                                        double box_size, uint64_t* keys_out, uint32_t* order_out, void* stream) {
  if (n < 0 || (n > 0 && (!qx || !qy || !qz || !keys_out || !order_out))) return TPM_ERR_INVALID_ARGUMENT;
  if (n > NOALLOC_MAX) return TPM_ERR_TOO_LARGE;
  if (!(box_size > 0.0)) return TPM_ERR_INVALID_ARGUMENT;
  if (n == 0) return TPM_OK;
  try {
    int dev = 0;
    TPM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return TPM_ERR_INVALID_ARGUMENT;
    unsigned char* base = scratch_for_current_device(dev);
    cudaStream_t s = (cudaStream_t)stream;
    tpm::TreeBuffers t{};
    t.bbox = (uint32_t*)base;
    t.params = (tpm::TreeParams*)(base + 64);
    tpm::Particles p{};
    p.qx = const_cast<uint32_t*>(qx);
    p.qy = const_cast<uint32_t*>(qy);
    p.qz = const_cast<uint32_t*>(qz);
    // bounding box of the positions (sfc.rs:250-280), keys in input order,
    // values = input indices
    tpm::launch_bbox_root(p, n, box_size, t, s);
    tpm::launch_hilbert_keys(p, n, box_size, t.params, keys_out, order_out, s);
    // stable sort: equal keys keep ascending input index
    tpm::radix_sort_u64_all_passes(keys_out, order_out, n, base + NOALLOC_PARAMS_BYTES, NOALLOC_SORT_BYTES, s);
  } catch (const tpm::Error& e) {
    return e.code ? e.code : TPM_ERR_CUDA;
  }
  return TPM_OK;
}
