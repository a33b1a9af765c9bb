// energy_spectrum for callers that cannot allocate device memory.
//
// hit_energy_spectrum needs a plan, and a plan allocates its tables and its
// reduction scratch with cudaMalloc on first use.  Some callers cannot do
// that: a handler that runs while its stream is being captured into a CUDA
// graph (cudaMalloc/cudaFree are not stream operations and cudaFree
// synchronises the device), an XLA custom call, which must take every device
// buffer from XLA, or a process whose device memory is already reserved by
// another allocator.  hit_energy_spectrum_noalloc serves them: the caller
// passes the state and the two outputs, the wavenumbers are recomputed from
// indices, and the per-block partial sums live in g_spectrum_scratch below, a
// fixed 4 MiB array that the CUDA module holds on every GPU that loads this
// library until the process exits.
//
// Set-up: the first call on a device (with that device current) looks up the
// device address of the array with cudaGetSymbolAddress and caches it with the
// context it was looked up in; make that first call before any stream capture.
// A call that finds another context current on the device (the old one was
// torn down, e.g. by cudaDeviceReset) looks the address up again, so a stale
// address of a module that no longer exists is never used.  Every later call reuses the
// same array, so calls whose kernels overlap on the GPU (different streams, or
// different host threads) race on it and must be ordered by the caller.
// Nothing in the array has to start at zero: every block overwrites all of its
// partial slots before the finishing kernel reads them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "hit3d.h"
#include "kernels.h"

namespace hit {
int record_error(int code, const std::string& msg);
}

using namespace hit;

namespace {

constexpr int kScratchDoubles = 1 << 19;  // 4 MiB of float64 partial sums
constexpr int kBlocks = 148;              // one block per SM

static __device__ __align__(256) double g_spectrum_scratch[kScratchDoubles];

std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};

// The calling thread's current driver context, through the runtime's driver
// entry point (no link to the driver library); nullptr if unavailable.
CUcontext current_context() {
  typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<CtxGetCurrentFn>(p);
    cudaGetLastError();
    return (CtxGetCurrentFn) nullptr;
  }();
  CUcontext c = nullptr;
  if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
  return c;
}

__device__ __forceinline__ int freq_i(int i, int n) { return i < n / 2 ? i : i - n; }

template <typename T> __device__ __forceinline__ int shell_index(T k2, T k0);
template <> __device__ __forceinline__ int shell_index<float>(float k2, float k0) {
  return (int)floorf(__fadd_rn(__fdiv_rn(__fsqrt_rn(k2), k0), 0.5f));
}
template <> __device__ __forceinline__ int shell_index<double>(double k2, double k0) {
  return (int)floor(__dadd_rn(__ddiv_rn(__dsqrt_rn(k2), k0), 0.5));
}

// Per-block shell sums of w |u_c|^2, wavenumbers (T)(2 pi / L * n) formed in
// double from the indices exactly as the plan's host tables are.
template <typename T>
__global__ void __launch_bounds__(NT) k_spectrum_static(const V2<T>* __restrict__ u, int Nx, int Ny, int Nz, double ax,
                                                        double ay, double az, T k0, int nshell, double* scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* bins = reinterpret_cast<double*>(smem_raw);
  for (int s = threadIdx.x; s < 3 * nshell; s += NT) bins[s] = 0.0;
  __syncthreads();
  const int Nzh = Nz / 2 + 1;
  const long long nmodes = (long long)Nx * Ny * Nzh;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nmodes; m += (long long)gridDim.x * NT) {
    const int k = (int)(m % Nzh);
    const long long r = m / Nzh;
    const int fy = (int)(r % Ny), fx = (int)(r / Ny);
    const T kx = (T)(ax * (double)freq_i(fx, Nx)), ky = (T)(ay * (double)freq_i(fy, Ny)), kz = (T)(az * (double)k);
    const int s = shell_index<T>(k2_of(kx, ky, kz), k0);
    if (s < 0 || s >= nshell) continue;
    const double w = (k == 0 || ((Nz & 1) == 0 && k == Nz / 2)) ? 1.0 : 2.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const V2<T> v = u[c * nmodes + m];
      const double a2 = (double)v.x * v.x + (double)v.y * v.y;
      if (a2 != 0.0) atomicAdd(&bins[c * nshell + s], w * a2);
    }
  }
  __syncthreads();
  double* out = scratch + (long long)blockIdx.x * 3 * nshell;
  for (int s = threadIdx.x; s < 3 * nshell; s += NT) out[s] = bins[s];
}

// Kahan sum of the block partials per (component, shell) -> spectra.
__global__ void k_spectrum_static_finish(const double* __restrict__ scratch, int nblocks, int nshell, double inv,
                                         double* E, double* Ec) {
  const int s = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nshell) return;
  double tot = 0.0;
  for (int c = 0; c < 3; ++c) {
    double sum = 0.0, comp = 0.0;
    for (int b = 0; b < nblocks; ++b) {
      const double y = scratch[(long long)b * 3 * nshell + c * nshell + s] - comp;
      const double t = sum + y;
      comp = (t - sum) - y;
      sum = t;
    }
    const double v = sum * inv;
    if (Ec) Ec[c * (nshell - 1) + s - 1] = v;
    tot += v;
  }
  if (E) E[s - 1] = tot;
}

bool size_ok(int n) { return n >= 4 && n <= 1024 && (n & (n - 1)) == 0; }

}  // namespace

extern "C" int hit_energy_spectrum_noalloc(int nx, int ny, int nz, double lx, double ly, double lz, int dtype,
                                           const void* u_hat, double* E_dev, double* Ecomp_dev, void* stream) {
  if (!u_hat || (!E_dev && !Ecomp_dev)) return record_error(HIT_E_INVALID, "NULL input or no output requested");
  if (!size_ok(nx) || !size_ok(ny) || !size_ok(nz))
    return record_error(HIT_E_UNSUPPORTED, "hit_energy_spectrum_noalloc: grid sizes must be powers of two in [4, 1024], got " +
                                               std::to_string(nx) + "x" + std::to_string(ny) + "x" + std::to_string(nz));
  if (dtype != HIT_DTYPE_F32 && dtype != HIT_DTYPE_F64) return record_error(HIT_E_UNSUPPORTED, "dtype must be F32 or F64");
  if (!(lx > 0) || !(ly > 0) || !(lz > 0)) return record_error(HIT_E_INVALID, "box lengths must be positive");
  const int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  const int smax = (int)std::ceil(std::sqrt(3.0) * nmax / 2.0) + 1;
  const int nshell = smax + 1;
  const long long need = (long long)kBlocks * 3 * nshell;
  if (need > kScratchDoubles)
    return record_error(HIT_E_UNSUPPORTED, "hit_energy_spectrum_noalloc: " + std::to_string(need) +
                                               " partial sums exceed the static scratch of " +
                                               std::to_string(kScratchDoubles) + " doubles");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return record_error(HIT_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return record_error(HIT_E_UNSUPPORTED, "device index beyond 63");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const CUcontext ctx = current_context();
    if (!g_scratch_addr[dev] || ctx != g_scratch_ctx[dev]) {
      g_scratch_addr[dev] = nullptr;
      e = cudaGetSymbolAddress(&g_scratch_addr[dev], g_spectrum_scratch);
      if (e != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        return record_error(HIT_E_CUDA, std::string("cudaGetSymbolAddress(g_spectrum_scratch): ") + cudaGetErrorString(e));
      }
      g_scratch_ctx[dev] = current_context();  // the runtime has made the device's primary context current
    }
    scratch = g_scratch_addr[dev];
  }
  const double two_pi = 2.0 * M_PI;
  const double ax = two_pi / lx, ay = two_pi / ly, az = two_pi / lz;
  const double n = (double)nx * ny * nz;
  const double inv = 1.0 / (2.0 * n * n);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = sizeof(double) * 3 * nshell;
  double* sp = static_cast<double*>(scratch);
  if (dtype == HIT_DTYPE_F32)
    k_spectrum_static<float><<<kBlocks, NT, smem, st>>>(static_cast<const float2*>(u_hat), nx, ny, nz, ax, ay, az,
                                                        (float)(2.0 * M_PI / lx), nshell, sp);
  else
    k_spectrum_static<double><<<kBlocks, NT, smem, st>>>(static_cast<const double2*>(u_hat), nx, ny, nz, ax, ay, az,
                                                         2.0 * M_PI / lx, nshell, sp);
  e = cudaGetLastError();
  if (e != cudaSuccess) return record_error(HIT_E_CUDA, std::string("k_spectrum_static: ") + cudaGetErrorString(e));
  k_spectrum_static_finish<<<(nshell + NT - 1) / NT, NT, 0, st>>>(sp, kBlocks, nshell, inv, E_dev, Ecomp_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) return record_error(HIT_E_CUDA, std::string("k_spectrum_static_finish: ") + cudaGetErrorString(e));
  return HIT_OK;
}
