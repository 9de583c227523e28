// qbxfmm_apply_noalloc: the whole apply for callers that cannot allocate device
// memory.
//
// Some callers of this library cannot call cudaMalloc: a host code whose own memory
// manager owns every device allocation and hands libraries only the buffers they
// read and write, or code running where allocating is not permitted.  Such a caller
// passes only the density and the output; the apply's intermediate arrays
// (tree-order strengths, box multipoles and locals, QBX expansions, potentials by
// target kind, the error word) live in a file-scope device array of fixed size,
// QBXFMM_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library keeps until
// the process exits.
//
// Rules of use:
//   * The first call on a device resolves the array's device address
//     (cudaGetSymbolAddress, with that device current); make that first call before
//     any stream capture.
//   * All calls on a device share the one array and it keeps the previous call's
//     contents; the apply clears everything it accumulates into.  Calls whose work
//     overlaps on the GPU (other streams, other host threads) race on the array:
//     serialize them.
//   * Problems whose intermediate arrays exceed the array are rejected with
//     QBXFMM_ERR_ARG before anything is launched.
//   * The translations use the per-pair kernels (the translation-class matrices need
//     more memory than the array holds).
#include <mutex>
#include <string>

#include "../../include/qbxfmm_api.h"
#include "kernels.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[QBXFMM_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

size_t round256(size_t n) { return (n + 255) / 256 * 256; }

}  // namespace

namespace qbx {
int plan_base_workspace_sizes(const qbxfmm_plan* p, size_t* sizes6);
int set_last_error(int code, const std::string& msg);
}  // namespace qbx

extern "C" int qbxfmm_apply_noalloc(const qbxfmm_plan* plan, const qbxfmm_upsample* up,
                                    const void* density, void* out, void* stream)
{
  if (!plan || !up || !density || !out)
    return qbx::set_last_error(QBXFMM_ERR_ARG, "null argument");
  size_t sz[6];
  if (int rc = qbx::plan_base_workspace_sizes(plan, sz)) return rc;
  size_t need = 256;   // error word
  for (int i = 0; i < 6; ++i) need += round256(sz[i]);
  if (need > (size_t)QBXFMM_NOALLOC_SCRATCH_BYTES)
    return qbx::set_last_error(
        QBXFMM_ERR_ARG, "qbxfmm_apply_noalloc: the problem needs " + std::to_string(need) +
                            " bytes of scratch, the built-in maximum is " +
                            std::to_string((size_t)QBXFMM_NOALLOC_SCRATCH_BYTES) +
                            " bytes; use qbxfmm_apply with a caller-owned workspace");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return qbx::set_last_error(QBXFMM_ERR_ARG, "device ordinal out of range");
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess)
        return qbx::set_last_error(QBXFMM_ERR_CUDA,
                                   std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_ptr[dev] = ptr;
    }
    base = static_cast<unsigned char*>(g_scratch_ptr[dev]);
  }
  qbxfmm_workspace ws;
  size_t off = 0;
  void* bufs[6];
  for (int i = 0; i < 6; ++i) {
    bufs[i] = base + off;
    off += round256(sz[i]);
  }
  ws.strengths = bufs[0];
  ws.mpoles = bufs[1];
  ws.locals = bufs[2];
  ws.qbx_exps = bufs[3];
  ws.pot_nonqbx = bufs[4];
  ws.pot_tree = bufs[5];
  ws.error_word = reinterpret_cast<int32_t*>(base + off);
  ws.translations = nullptr;
  ws.pair_scratch = nullptr;
  return qbxfmm_apply(plan, up, &ws, density, out, stream);
}
