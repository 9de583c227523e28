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
// Layout of the array: the error word in the first 256 bytes, then the six
// intermediate arrays, each starting on a 256-byte boundary.
//
// Rules of use:
//   * The plan's device must be the current device.  The first call on a device
//     resolves the array's device address (cudaGetSymbolAddress, with that device
//     current); make that first call before any stream capture.  cudaDeviceReset is
//     not supported between calls (a new context holds a new copy of the array).
//   * All calls on a device share the one array and it keeps the previous call's
//     contents; the apply clears everything it accumulates into.  Calls whose work
//     overlaps on the GPU (other streams, other host threads) race on the array:
//     serialize them.
//   * Problems whose intermediate arrays exceed the array are rejected with
//     QBXFMM_ERR_ARG before anything is launched, and so are 3D Helmholtz plans,
//     whose translation tables are a caller-owned buffer of qbxfmm_apply.
//   * Kernels that meet an out-of-range list entry set the error word and skip the
//     entry; qbxfmm_noalloc_error_word reads it back.
#include <mutex>
#include <string>

#include "../../include/qbxfmm_api.h"
#include "kernels.h"

namespace qbx {
int plan_base_workspace_sizes(const qbxfmm_plan* p, size_t* sizes6);
int set_last_error(int code, const std::string& msg);
int plan_device(const qbxfmm_plan* p);
bool plan_needs_translation_tables(const qbxfmm_plan* p);
}  // namespace qbx

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[QBXFMM_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr size_t kErrorWordBytes = 256;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

size_t round256(size_t n) { return (n + 255) / 256 * 256; }

int current_device(int* dev)
{
  cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (*dev < 0 || *dev >= kMaxDevices)
    return qbx::set_last_error(QBXFMM_ERR_ARG, "device ordinal out of range");
  return QBXFMM_OK;
}

}  // namespace

extern "C" int qbxfmm_apply_noalloc(const qbxfmm_plan* plan, const qbxfmm_upsample* up,
                                    const void* density, void* out, void* stream)
{
  if (!plan || !up || !density || !out)
    return qbx::set_last_error(QBXFMM_ERR_ARG, "null argument");
  if (qbx::plan_needs_translation_tables(plan))
    return qbx::set_last_error(
        QBXFMM_ERR_ARG,
        "qbxfmm_apply_noalloc: 3D Helmholtz plans are not supported (their rotation and "
        "translation tables live in a caller-owned buffer); use qbxfmm_apply");
  size_t sz[6];
  if (int rc = qbx::plan_base_workspace_sizes(plan, sz)) return rc;
  size_t need = kErrorWordBytes;
  for (int i = 0; i < 6; ++i) need += round256(sz[i]);
  if (need > (size_t)QBXFMM_NOALLOC_SCRATCH_BYTES)
    return qbx::set_last_error(
        QBXFMM_ERR_ARG, "qbxfmm_apply_noalloc: the problem needs " + std::to_string(need) +
                            " bytes of scratch, the built-in maximum is " +
                            std::to_string((size_t)QBXFMM_NOALLOC_SCRATCH_BYTES) +
                            " bytes; use qbxfmm_apply with a caller-owned workspace");
  int dev = 0;
  if (int rc = current_device(&dev)) return rc;
  if (dev != qbx::plan_device(plan))
    return qbx::set_last_error(QBXFMM_ERR_ARG,
                               "qbxfmm_apply_noalloc: the current device (" + std::to_string(dev) +
                                   ") is not the plan's device (" +
                                   std::to_string(qbx::plan_device(plan)) + ")");
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess)
        return qbx::set_last_error(QBXFMM_ERR_CUDA,
                                   std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_ptr[dev] = ptr;
    }
    base = static_cast<unsigned char*>(g_scratch_ptr[dev]);
  }
  qbxfmm_workspace ws;
  size_t off = kErrorWordBytes;
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
  ws.error_word = reinterpret_cast<int32_t*>(base);
  ws.translations = nullptr;
  ws.pair_scratch = nullptr;
  return qbxfmm_apply(plan, up, &ws, density, out, stream);
}

extern "C" int qbxfmm_noalloc_error_word(int32_t* host_out, void* stream)
{
  if (!host_out) return qbx::set_last_error(QBXFMM_ERR_ARG, "null argument");
  int dev = 0;
  if (int rc = current_device(&dev)) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyFromSymbolAsync(host_out, g_noalloc_scratch, sizeof(int32_t), 0,
                                            cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA,
                               std::string("qbxfmm_noalloc_error_word: ") + cudaGetErrorString(e));
  return QBXFMM_OK;
}
