// noalloc.cu -- getm_tracer_vdiff_noalloc: the implicit vertical-diffusion solve of a tracer with
// no context and no device allocation of any kind.
//
// Who needs it. getm_tracer_vdiff takes its two Thomas-coefficient scratch arrays from a context,
// which allocates them with cudaMalloc on first use (and frees and re-allocates them when a larger
// domain comes along). Some callers cannot accept that:
//   * a host model that hands over raw device pointers and keeps no context object, e.g. a
//     Fortran time loop that calls one C function per tracer and owns nothing else on the device;
//   * a caller whose device memory is already committed to the model state and to other
//     components on the same GPU, where an allocation half-way through a run may fail;
//   * a caller that keeps other streams busy: cudaFree (which a context runs when it grows its
//     scratch) waits for the whole device, which stalls that overlapped work.
// This entry point uses instead a scratch array with static storage in this file. Its size is
// fixed when the library is built, so the call itself never allocates, and it fails with
// GETM_ERR_TOO_LARGE rather than asking for more.
//
// The results are those of getm_tracer_vdiff: the same kernel (k_vdiff, FP64, no contracted
// multiply-adds) runs with the same arguments; only the scratch pointers differ.
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "launch.h"

namespace {

constexpr long long kMaxCells = GETM_VDIFF_NOALLOC_MAX_CELLS;

// Thomas coefficients ru (first half) and qu (second half) of every column, indexed like a 3D
// field of the domain. Nothing here has to start at zero: in one call every thread writes the
// elements of its own column before it reads them back, and reads nothing else.
static __device__ __align__(256) double g_vdiff_scratch[2 * kMaxCells];

// Device address of g_vdiff_scratch, looked up with the device current and kept per device
// together with the identity of the CUDA context it was looked up in. The module holding the
// array is loaded into each context anew, so after a device reset (cudaDeviceReset, which ends the
// primary context) the array may sit at another address: a call in a context other than the cached
// one looks the address up again. Context identities come from the driver (cuCtxGetCurrent,
// cuCtxGetId) through cudaGetDriverEntryPoint, so the library needs no link to libcuda.
constexpr int kMaxDevices = 64;
struct ScratchAddr {
  unsigned long long ctx_id = 0;  // 0: not looked up yet (context ids start at 1)
  double* p = nullptr;
};
ScratchAddr g_scratch_addr[kMaxDevices];
std::mutex g_setup_mutex;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// The id of the calling thread's current context (0 when none is current or the driver cannot
// tell).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
  if (get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

int scratch_on_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return GETM_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return GETM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  ScratchAddr& e = g_scratch_addr[dev];
  unsigned long long id = current_context_id();
  if (e.p && id != 0 && id == e.ctx_id) {
    *out = e.p;
    return GETM_OK;
  }
  // set-up in this context: the runtime makes the device's primary context current if no
  // context is, and loads the module holding the array if it has not been loaded yet
  void* addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_vdiff_scratch) != cudaSuccess || !addr) {
    cudaGetLastError();
    return GETM_ERR_CUDA;
  }
  if (id == 0) id = current_context_id();
  e.ctx_id = id;  // 0 if the driver cannot name the context: then every call looks the address up
  e.p = static_cast<double*>(addr);
  *out = e.p;
  return GETM_OK;
}

}  // namespace

extern "C" int getm_tracer_vdiff_noalloc(const getm_domain* dom, void* stream, double dt, double cnpar,
                                         double avmol, double* S, const double* hn, const double* nuh,
                                         const int32_t* az, const double* src) {
  using namespace gb;
  if (!dom || !S || !hn || !nuh || !az) return GETM_ERR_ARG;
  if (dom->imax < dom->imin || dom->jmax < dom->jmin || dom->kmax < 0) return GETM_ERR_ARG;
  const long long ni = (long long)dom->imax - dom->imin + 1 + 2 * HALO;
  const long long nj = (long long)dom->jmax - dom->jmin + 1 + 2 * HALO;
  // the scratch is indexed like a 3D field: sk * (kmax + 1) elements per coefficient. The sizes
  // are compared by division before any product is formed, so that no caller-given value can
  // overflow a product past the limit.
  if (dom->sj < ni || dom->sk < dom->sj) return GETM_ERR_ARG;
  if (dom->sk > kMaxCells / ((long long)dom->kmax + 1)) return GETM_ERR_TOO_LARGE;
  if (dom->sj > dom->sk / nj) return GETM_ERR_ARG;  // sk < sj * nj (sk <= kMaxCells here)
  if (dom->kmax <= 1) return GETM_OK;  // no interior interface: the solve leaves S unchanged
  double* scr = nullptr;
  int rc = scratch_on_current_device(&scr);
  if (rc) return rc;
  const Dev d = to_dev(*dom);
  rc = run_vdiff<double>(d, (cudaStream_t)stream, dt, cnpar, avmol, S, hn, nuh, az, src, scr, scr + kMaxCells);
  return rc ? GETM_ERR_CUDA : GETM_OK;
}
