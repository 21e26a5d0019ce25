// noalloc.cu -- the FP64 direct-sum force checker without any allocation.
//
// bonsai_direct_fp64 (treecode.cu) keeps its partial sums in buffers that the
// handle allocates with cudaMalloc.  Some callers cannot allocate device
// memory: code that runs inside another framework whose allocator owns all of
// the GPU's memory, or a timing-critical loop that must not pay cudaMalloc's
// implicit device-wide synchronisation.  bonsai_direct_fp64_noalloc serves
// them: the caller passes device pointers for the inputs and the output, and
// the only scratch (the per-slice partial sums) is the file-scope array below,
// which every process that loads the library holds on every GPU it uses until
// exit.
//
// Limits and sharing:
//   * capacity kNoAllocDoubles doubles (2 MiB): ns <= 65536 samples; larger
//     requests return BONSAI_ERR_TOO_LARGE without launching anything;
//   * sample indices must lie in [0, n); the kernel reads no particle for an
//     index outside that range and writes a NaN row for it instead;
//   * with include_self the i == j term is summed, so eps2 must be > 0 (at
//     eps2 = 0 that term is 0/0): eps2 <= 0 with include_self returns
//     BONSAI_ERR_ARG;
//   * all calls share the array.  Every entry a call reads is written by the
//     same call first, so nothing has to start at zero, but two calls whose
//     kernels overlap on the GPU (different streams, or different host
//     threads) race on it and give wrong results: serialise them;
//   * every call looks up the array's device address with
//     cudaGetSymbolAddress on the current device (nothing is cached, so a
//     device reset or a new context is harmless).  The first call on a device
//     may load the library's device code there; make it before any stream
//     capture on that device.
#include "../../include/bonsai_b200.h"
#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr int kNoAllocDoubles = 1 << 18;  // 2 MiB of FP64 partial sums
constexpr int kNoAllocMaxSamples = kNoAllocDoubles / 4;

static __device__ __align__(256) double g_direct_scratch[kNoAllocDoubles];

// The array's address on the current device.  Host code cannot pass the
// symbol itself to a kernel: on the host it only names a stand-in, not device
// memory.
int scratch_for_current_device(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_direct_scratch);
  if (e != cudaSuccess) return -(int)e - 1000;
  *out = static_cast<double*>(p);
  return 0;
}

}  // namespace

extern "C" int bonsai_direct_fp64_noalloc(const float* d_pos4, int n, const int* d_sample, int ns, double eps2,
                                          int include_self, double* d_out, void* stream) {
  if (!d_pos4 || !d_sample || !d_out || n < 1 || ns < 1 || !(eps2 >= 0.0)) return BONSAI_ERR_ARG;
  if (include_self && !(eps2 > 0.0)) return BONSAI_ERR_ARG;  // the i == j term would be 0/0
  if (ns > kNoAllocMaxSamples) return BONSAI_ERR_TOO_LARGE;
  double* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  int dev = 0, nsm = 0;
  BONSAI_CUDA_TRY(cudaGetDevice(&dev));
  BONSAI_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  // slices of the sources: enough blocks to fill the GPU, bounded by the scratch
  int nsplit = (nsm * 8 * 256) / ns;
  nsplit = nsplit < 1 ? 1 : (nsplit > 512 ? 512 : nsplit);
  while ((long long)nsplit * ns * 4 > kNoAllocDoubles) nsplit--;
  bonsai::launch_direct_fp64(reinterpret_cast<const float4*>(d_pos4), n, d_sample, ns, eps2, include_self, scratch,
                             nsplit, d_out, static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e - 1000;
}
