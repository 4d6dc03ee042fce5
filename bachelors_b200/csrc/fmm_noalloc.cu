// Direct Biot-Savart sum for callers that cannot allocate device memory.
//
// fmm_direct (the plan-based entry point) packs the sources into plan-owned device buffers
// before it sums. Some callers cannot let a library allocate: their device memory is owned by
// another allocator (a framework's caching pool that has reserved the GPU), or they run latency
// critical host loops in which a cudaMalloc, which may synchronise the device or fail, is not
// acceptable. fmm_direct_B_noalloc computes the same FP32 sum from caller-owned device inputs
// and output and keeps its only scratch, the packed sources, in a fixed array in device memory
// that the library image carries; it never calls cudaMalloc, cudaFree or an allocating library
// routine.
//
// The array (g_noallocSources, NOALLOC_MAX_SOURCES sources, 8 MiB) belongs to this file's device
// module. Under CUDA's lazy module loading (the default) the module, and with it the array, is
// loaded onto a device by the first call made with that device current, when the array's address
// is looked up (cudaGetSymbolAddress); from then on it stays on that device until the process
// exits. That first call can therefore allocate the array's device memory and synchronise, and it
// fails (FMM_E_CUDA, with the runtime's reason) when another allocator has already reserved all of
// the device's memory: make it once per device before the caller's allocator reserves the GPU,
// outside latency-critical loops and before any stream capture. Later calls allocate nothing. All calls share the array and it keeps the
// previous call's contents: each call overwrites the entries it reads before reading them, so
// nothing needs clearing, but calls whose work overlaps on the GPU (other streams, or other
// host threads) race on it and must be serialised by the caller.
#include <mutex>

#include "fmm_internal.cuh"

namespace fmm {

constexpr int64_t NOALLOC_MAX_SOURCES = int64_t(1) << 18;

// packed sources: positions [0, MAX), strengths w J [MAX, 2 MAX)
static __device__ __align__(256) float4 g_noallocSources[2 * NOALLOC_MAX_SOURCES];

namespace {

std::mutex g_noallocMutex;
float4* g_noallocPtr[64] = {};

__global__ void kPackSourcesNoalloc(const float* __restrict__ xyz, const float* __restrict__ w,
                                    const float* __restrict__ J, int n, float4* __restrict__ scratch)
{
   int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i >= n) return;
   float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
   float jx, jy, jz;
   if(J) { jx = J[3 * i]; jy = J[3 * i + 1]; jz = J[3 * i + 2]; }
   else
   {
      // the reference's azimuthal direction perp(q) / |perp(q)|, zero on the axis
      float l = sqrtf(x * x + y * y);
      jx = l != 0.f ? -y / l : 0.f;
      jy = l != 0.f ? x / l : 0.f;
      jz = 0.f;
   }
   scratch[i] = make_float4(x, y, z, 0.f);
   scratch[NOALLOC_MAX_SOURCES + i] = make_float4(w[i] * jx, w[i] * jy, w[i] * jz, 0.f);
}

template <int NT>
__global__ void __launch_bounds__(NT) kDirectNoalloc(const float4* __restrict__ scratch, int n,
                                                     const float* __restrict__ tgt, int m, float scaleB,
                                                     float* __restrict__ outB)
{
   __shared__ float4 Sp[NT], Sq[NT];
   const int ti = blockIdx.x * NT + threadIdx.x;
   const bool active = ti < m;
   float x = 0.f, y = 0.f, z = 0.f;
   if(active) { x = tgt[3 * int64_t(ti)]; y = tgt[3 * int64_t(ti) + 1]; z = tgt[3 * int64_t(ti) + 2]; }
   float B[3] = {0.f, 0.f, 0.f};
   for(int sb = 0; sb < n; sb += NT)
   {
      const int cnt = min(NT, n - sb);
      __syncthreads();
      if(threadIdx.x < cnt)
      {
         Sp[threadIdx.x] = scratch[sb + threadIdx.x];
         Sq[threadIdx.x] = scratch[NOALLOC_MAX_SOURCES + sb + threadIdx.x];
      }
      __syncthreads();
      if(active)
         for(int i = 0; i < cnt; i++)
         {
            const float dx = x - Sp[i].x, dy = y - Sp[i].y, dz = z - Sp[i].z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if(r2 == 0.f) continue;
            const float ri = rsqrtf(r2);
            const float ri3 = ri * ri * ri;
            B[0] += (Sq[i].y * dz - Sq[i].z * dy) * ri3;
            B[1] += (Sq[i].z * dx - Sq[i].x * dz) * ri3;
            B[2] += (Sq[i].x * dy - Sq[i].y * dx) * ri3;
         }
   }
   if(active)
      for(int d = 0; d < 3; d++) outB[3 * int64_t(ti) + d] = B[d] * scaleB;
}

// Device address of the static scratch array on the current device, looked up once per device.
fmm_status noallocScratch(float4** out)
{
   int dev = 0;
   FMM_CUDA(cudaGetDevice(&dev));
   if(dev < 0 || dev >= 64) return setError(FMM_E_INVALID, "fmm_direct_B_noalloc: device %d out of range", dev);
   std::lock_guard<std::mutex> lock(g_noallocMutex);
   if(!g_noallocPtr[dev])
   {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noallocSources);
      if(e != cudaSuccess || !p)
      {
         cudaGetLastError();
         return setError(FMM_E_CUDA,
                         "fmm_direct_B_noalloc: loading the library's scratch array onto device %d failed (%s); "
                         "make the first call on each device before another allocator reserves its memory",
                         dev, cudaGetErrorString(e));
      }
      g_noallocPtr[dev] = static_cast<float4*>(p);
   }
   *out = g_noallocPtr[dev];
   return FMM_OK;
}

}  // namespace
}  // namespace fmm

extern "C" fmm_status fmm_direct_B_noalloc(const float* xyz, const float* w, const float* J, int64_t n,
                                           const float* tgt, int64_t m, double current, float* out_B, void* stream)
{
   using namespace fmm;
   if(n < 0 || m < 0) return setError(FMM_E_INVALID, "fmm_direct_B_noalloc: negative size");
   if(n > NOALLOC_MAX_SOURCES)
      return setError(FMM_E_LIMIT, "fmm_direct_B_noalloc: %lld sources exceed the limit of %lld", (long long)n,
                      (long long)NOALLOC_MAX_SOURCES);
   if(m > (int64_t(1) << 31) - 1) return setError(FMM_E_LIMIT, "fmm_direct_B_noalloc: too many targets");
   if((n > 0 && (!xyz || !w)) || (m > 0 && (!tgt || !out_B)))
      return setError(FMM_E_INVALID, "fmm_direct_B_noalloc: null pointer");
   if(m == 0) return FMM_OK;
   float4* scratch = nullptr;
   FMM_TRY(noallocScratch(&scratch));
   cudaStream_t st = static_cast<cudaStream_t>(stream);
   if(n > 0)
   {
      kPackSourcesNoalloc<<<int((n + 255) / 256), 256, 0, st>>>(xyz, w, J, int(n), scratch);
      FMM_CHECK_LAUNCH();
   }
   constexpr int NT = 128;
   const float scaleB = float(REF_MU0 / (4 * REF_PI) * current);
   kDirectNoalloc<NT><<<int((m + NT - 1) / NT), NT, 0, st>>>(scratch, int(n), tgt, int(m), scaleB, out_B);
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}
