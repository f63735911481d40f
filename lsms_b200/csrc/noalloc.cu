// b200tau_solve_dense_noalloc: the dense tau00 solve without any device allocation.
//
// Some callers cannot call cudaMalloc: applications whose device memory is owned by another
// allocator (a host program that reserves the GPU's memory up front for its own pool, so an
// allocation inside this library would fail or fragment that pool), and latency-critical callers
// that cannot afford the implicit device synchronisation of cudaMalloc/cudaFree.  For them this
// entry runs the same FP64 solve as b200tau_solve_dense (block elimination, one refinement step)
// on device buffers the caller passes, with all scratch memory in one file-scope __device__
// array of fixed size, so nothing is allocated and no context is needed.
//
// Limits: n <= kNoAllocMaxN (512) and b <= 32.  The scratch array (about 8.9 MB) is part of the
// library image and stays resident on every GPU that loads the library until the process exits.
// Every call uses the same array and leaves its contents behind; the call clears what has to
// start at zero (pivot, convergence and error flags).  Calls whose work overlaps on the GPU (two
// host threads, or two streams, at the same time on the same device) race on the array and give
// wrong results: serialise them.
//
// The device address of the array is looked up with cudaGetSymbolAddress once per device, by the
// first call made while that device is current; that first call should therefore come before any
// stream capture.  Host code never passes the array's name to a kernel (in host code the name is
// a host-side stand-in, not a device address).

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/b200tau.h"
#include "common.cuh"

using namespace b200;

namespace {

constexpr int kNoAllocMaxN = 512;   // largest n accepted (a multiple of 64: ld == kNoAllocMaxN)
constexpr int kNoAllocLd = kNoAllocMaxN;
constexpr size_t kMatBytes = sizeof(double2) * (size_t)kNoAllocLd * kNoAllocLd;      // 4 MiB
constexpr size_t kVecBytes = sizeof(double2) * (size_t)kNoAllocLd * kMaxB;           // 256 KiB
constexpr size_t kOffM = 0;
constexpr size_t kOffF = kOffM + kMatBytes;
constexpr size_t kOffX = kOffF + kMatBytes;
constexpr size_t kOffR = kOffX + kVecBytes;
constexpr size_t kOffY = kOffR + kVecBytes;
constexpr size_t kOffJob = kOffY + kVecBytes;                                          // JobDev record
constexpr size_t kOffFlags = kOffJob + 512;                                             // info, conv, err
constexpr size_t kScratchBytes = kOffFlags + 256;
static_assert(sizeof(JobDev) <= 512, "JobDev record must fit its scratch slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lookup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
cudaError_t scratch_address(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_lookup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int b200tau_solve_dense_noalloc(const double *m, int n, int ldm, const double *t0, int b,
                                           double *tau00, void *stream) {
  if (!m || !t0 || !tau00) return B200TAU_ERR_ARG;
  if (n < 1 || b < 1 || b > n || b > kMaxB || ldm < n) return B200TAU_ERR_ARG;
  if (n > kNoAllocMaxN) return B200TAU_ERR_ARG;  // beyond the fixed scratch array
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char *base = nullptr;
  if (scratch_address(&base) != cudaSuccess) return B200TAU_ERR_CUDA;
  double2 *M = reinterpret_cast<double2 *>(base + kOffM);
  double2 *F = reinterpret_cast<double2 *>(base + kOffF);
  JobDev *dJ = reinterpret_cast<JobDev *>(base + kOffJob);
  int *flags = reinterpret_cast<int *>(base + kOffFlags);  // [0] info, [1] conv, [2] err
  const int ld = kNoAllocLd;
  const int r = n - b;
  const size_t es = sizeof(double2);
  const double2 *dm = reinterpret_cast<const double2 *>(m);
  // reorder into the central-site-last layout: [Mrr Mr0; M0r M00] <- [M00 M0r; Mr0 Mrr]
  cudaError_t e = cudaSuccess;
  if (r > 0) {
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(M, ld * es, dm + b + (size_t)b * ldm, ldm * es, r * es, r, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(M + (size_t)r * ld, ld * es, dm + b, ldm * es, r * es, b, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(M + r, ld * es, dm + (size_t)b * ldm, ldm * es, b * es, r, cudaMemcpyDeviceToDevice, s);
  }
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(M + r + (size_t)r * ld, ld * es, dm, ldm * es, b * es, b, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = launch_copy_to_factor(kFactorFP64, M, F, n, ld, s);
  JobDev J;
  std::memset(&J, 0, sizeof(J));
  J.M = M;
  J.F = F;
  J.X = reinterpret_cast<double2 *>(base + kOffX);
  J.R = reinterpret_cast<double2 *>(base + kOffR);
  J.Y = reinterpret_cast<double2 *>(base + kOffY);
  J.conv = flags + 1;
  J.N = n;
  J.n = r;
  J.b = b;
  J.ld = ld;
  J.t0 = reinterpret_cast<const double2 *>(t0);
  J.t0_ld = b;
  J.out = reinterpret_cast<double2 *>(tau00);  // b x b, written by the last kernel
  J.out_mode = 1;
  J.err = flags + 2;
  // the JobDev record is copied from a pageable host object; the runtime stages pageable
  // host-to-device copies before the call returns, so the stack object may go out of scope
  if (e == cudaSuccess) e = cudaMemcpyAsync(dJ, &J, sizeof(J), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, 3 * sizeof(int), s);
  long launches = 0;
  if (e == cudaSuccess) e = launch_eliminate(kFactorFP64, dJ, 1, r, n, flags, s, &launches, nullptr, nullptr, flags + 2);
  if (e == cudaSuccess) e = launch_solve_refine(kFactorFP64, dJ, 1, r, n, b, 1, 1, b, flags, s, &launches);
  if (e != cudaSuccess) return B200TAU_ERR_CUDA;
  int host_flags[3] = {0, 0, 0};
  if (cudaMemcpyAsync(host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return B200TAU_ERR_CUDA;
  if (host_flags[0] != 0) return B200TAU_ERR_SINGULAR;
  if (host_flags[2] != 0) return B200TAU_ERR_TIMEOUT;
  return B200TAU_OK;
}
