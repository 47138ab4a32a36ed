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
#include <atomic>
#include <mutex>

#include "common.cuh"
#include "launch.h"

namespace {

constexpr long long kMaxCells = GETM_VDIFF_NOALLOC_MAX_CELLS;

// Thomas coefficients ru (first half) and qu (second half) of every column, indexed like a 3D
// field of the domain. Nothing here has to start at zero: in one call every thread writes the
// elements of its own column before it reads them back, and reads nothing else.
static __device__ __align__(256) double g_vdiff_scratch[2 * kMaxCells];

// Device address of g_vdiff_scratch, looked up once per device (with that device current).
constexpr int kMaxDevices = 64;
std::atomic<double*> g_scratch_addr[kMaxDevices];
std::mutex g_setup_mutex;

int scratch_on_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return GETM_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return GETM_ERR_UNSUPPORTED;
  double* p = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_scratch_addr[dev].load(std::memory_order_relaxed);
    if (!p) {
      void* addr = nullptr;
      if (cudaGetSymbolAddress(&addr, g_vdiff_scratch) != cudaSuccess || !addr) {
        cudaGetLastError();
        return GETM_ERR_CUDA;
      }
      p = static_cast<double*>(addr);
      g_scratch_addr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return GETM_OK;
}

}  // namespace

extern "C" int getm_tracer_vdiff_noalloc(const getm_domain* dom, void* stream, double dt, double cnpar,
                                         double avmol, double* S, const double* hn, const double* nuh,
                                         const int32_t* az, const double* src) {
  using namespace gb;
  if (!dom || !S || !hn || !nuh || !az) return GETM_ERR_ARG;
  if (dom->imax < dom->imin || dom->jmax < dom->jmin || dom->kmax < 0) return GETM_ERR_ARG;
  const long long ni = dom->imax - dom->imin + 1 + 2 * HALO;
  const long long nj = dom->jmax - dom->jmin + 1 + 2 * HALO;
  if (dom->sj < ni || dom->sk < dom->sj * nj) return GETM_ERR_ARG;
  // the scratch is indexed like a 3D field: sk * (kmax + 1) elements per coefficient
  if (dom->sk * (long long)(dom->kmax + 1) > kMaxCells) return GETM_ERR_TOO_LARGE;
  if (dom->kmax <= 1) return GETM_OK;  // no interior interface: the solve leaves S unchanged
  double* scr = nullptr;
  int rc = scratch_on_current_device(&scr);
  if (rc) return rc;
  const Dev d = to_dev(*dom);
  rc = run_vdiff<double>(d, (cudaStream_t)stream, dt, cnpar, avmol, S, hn, nuh, az, src, scr, scr + kMaxCells);
  return rc ? GETM_ERR_CUDA : GETM_OK;
}
