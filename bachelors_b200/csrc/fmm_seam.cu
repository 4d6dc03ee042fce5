// The reference's kernel-caller seam, kernels::translateAll* (FMM/FMMGPU/translation_algorithms.hpp:8-61),
// as B200 kernels behind extern "C" entry points:
//   fmm_translate_all                 <- translateAllCPU / translateAllGPU
//   fmm_translate_all_matrix          <- translateAllCPUMatrixBLAS / translateAllGPUMatrixCuBLAS (both overloads)
//   fmm_translate_all_matrix_complex  <- translateAllCPUMatrix / translateAllGPUMatrix
// These are the building blocks the reference's M2M "Layers" and "Matrices" algorithms call
// (multipole_solver.cpp:304-322,381-404, fast_multipole_solver.cpp:335-352). The solver in this
// library does not use them (its M2M/L2L run on precomputed box-size-scaled operators); they exist
// so that code written against the reference's seam links against this library unchanged.
#include "fmm_internal.cuh"

namespace fmm {
namespace {

// The reference's 1/sqrt(2) literal (math.hpp:16); its real<->complex views use it.
constexpr double SEAM_R_SQRT_2 = 0.70710678118;

__host__ __device__ constexpr int seamIdx(int l, int m) { return l * l + l + m; }

// (-1)^((|m - mu| + |mu| - |m|) / 2), the sign of the reference's multipoleTranslationFactor
// (multipole_translator.cpp:143-146); the exponent is a non-negative integer.
__device__ inline int seamSign(int m, int mu)
{
   return (((abs(m - mu) + abs(mu) - abs(m)) >> 1) & 1) ? -1 : 1;
}

// Complex view of a real-form entry (l, m != 0) as the reference reads it (kernels.cuh:84-112):
// s (h[l,|m|] + i sign(m) h[l,-|m|]).
template <class T>
__device__ inline void seamView(const T* h, int l, int m, T s, T& re, T& im)
{
   const int am = abs(m);
   re = h[seamIdx(l, am)] * s;
   im = h[seamIdx(l, -am)] * (m > 0 ? s : -s);
}

// One CTA per item (grid-stride): the translation harmonics a[L] and the three components of
// the expansion b[L][3] are staged in shared memory (b transposed to [3][L]); each thread owns
// output pairs (l, +-m) and accumulates the three components in registers.
template <class T>
__global__ void kTranslateAll(T* __restrict__ result, const T* __restrict__ a, const T* __restrict__ b,
                              int64_t count, int p)
{
   extern __shared__ __align__(16) unsigned char seamSmem[];
   const int L = (p + 1) * (p + 1);
   const int npairs = (p + 1) * (p + 2) / 2;
   T* sa = reinterpret_cast<T*>(seamSmem);
   T* sb = sa + L;
   const T s = T(SEAM_R_SQRT_2);
   for(int64_t item = blockIdx.x; item < count; item += gridDim.x)
   {
      const T* ai = a + item * L;
      const T* bi = b + item * 3 * L;
      for(int k = threadIdx.x; k < L; k += blockDim.x) sa[k] = ai[k];
      for(int j = threadIdx.x; j < 3 * L; j += blockDim.x) sb[(j % 3) * L + j / 3] = bi[j];
      __syncthreads();
      for(int pi = threadIdx.x; pi < npairs; pi += blockDim.x)
      {
         int l = 0;
         while((l + 1) * (l + 2) / 2 <= pi) l++;
         const int m = pi - l * (l + 1) / 2;
         T* ri = result + item * 3 * L;
         if(m == 0)
         {
            T z[3] = {0, 0, 0};
            for(int lam = 0; lam <= l; lam++)
            {
               const int dl = l - lam;
               const int mm = min(lam, dl);
               for(int mu = -mm; mu <= mm; mu++)
               {
                  const T f = T(seamSign(0, mu)) * sa[seamIdx(dl, mu)];
                  for(int c = 0; c < 3; c++) z[c] += sb[c * L + seamIdx(lam, mu)] * f;
               }
            }
            for(int c = 0; c < 3; c++) ri[3 * seamIdx(l, 0) + c] = z[c];
            continue;
         }
         T re[3] = {0, 0, 0}, im[3] = {0, 0, 0};
         for(int lam = 0; lam <= l; lam++)
         {
            const int dl = l - lam;
            for(int mu = -lam; mu <= lam; mu++)
            {
               T Bre[3], Bim[3];
               for(int c = 0; c < 3; c++)
               {
                  if(mu == 0)
                  {
                     Bre[c] = sb[c * L + seamIdx(lam, 0)];
                     Bim[c] = 0;
                  }
                  else
                     seamView(sb + c * L, lam, mu, s, Bre[c], Bim[c]);
               }
               const int dm = m - mu;
               if(abs(dm) <= dl)
               {
                  T Are, Aim;
                  if(dm == 0) { Are = sa[seamIdx(dl, 0)]; Aim = 0; }
                  else seamView(sa, dl, dm, s, Are, Aim);
                  const T f = T(seamSign(m, mu));
                  for(int c = 0; c < 3; c++)
                  {
                     re[c] += (Bre[c] * Are - Bim[c] * Aim) * f;
                     im[c] += (Bre[c] * Aim + Bim[c] * Are) * f;
                  }
               }
               const int dn = -m - mu;
               if(abs(dn) <= dl)
               {
                  T Are, Aim;
                  if(dn == 0) { Are = sa[seamIdx(dl, 0)]; Aim = 0; }
                  else seamView(sa, dl, dn, s, Are, Aim);
                  const T f = T(seamSign(-m, mu));
                  for(int c = 0; c < 3; c++)
                  {
                     re[c] += (Bre[c] * Are - Bim[c] * Aim) * f;
                     im[c] -= (Bre[c] * Aim + Bim[c] * Are) * f;
                  }
               }
            }
         }
         for(int c = 0; c < 3; c++)
         {
            ri[3 * seamIdx(l, m) + c] = re[c] * s;
            ri[3 * seamIdx(l, -m) + c] = im[c] * s;
         }
      }
      __syncthreads();
   }
}

// Multiply-accumulate for the real and complex (re, im) element types.
__device__ inline void mac(float& c, float a, float b) { c = fmaf(a, b, c); }
__device__ inline void mac(double& c, double a, double b) { c = fma(a, b, c); }
__device__ inline void mac(float2& c, float2 a, float2 b)
{
   c.x = fmaf(a.x, b.x, c.x);
   c.x = fmaf(-a.y, b.y, c.x);
   c.y = fmaf(a.x, b.y, c.y);
   c.y = fmaf(a.y, b.x, c.y);
}
__device__ inline void mac(double2& c, double2 a, double2 b)
{
   c.x = fma(a.x, b.x, c.x);
   c.x = fma(-a.y, b.y, c.x);
   c.y = fma(a.x, b.y, c.y);
   c.y = fma(a.y, b.x, c.y);
}

// C[i][j] = sum_k A[i][k] B[k][j] for i < M, j, k < L, all row-major; blockIdx.z selects one of
// several products that share B (A and C advance by M * L). 64 x 64 output tile per CTA,
// 16-deep K slices through shared memory, 4 x 4 outputs per thread.
constexpr int GBM = 64, GBN = 64, GBK = 16;
template <class V>
__global__ void __launch_bounds__(256) kRowGemm(V* __restrict__ C, const V* __restrict__ A, const V* __restrict__ B,
                                               int64_t M, int L)
{
   __shared__ V As[GBK][GBM];
   __shared__ V Bs[GBK][GBN];
   const int64_t i0 = int64_t(blockIdx.x) * GBM;
   const int j0 = blockIdx.y * GBN;
   A += int64_t(blockIdx.z) * M * L;
   C += int64_t(blockIdx.z) * M * L;
   const int tid = threadIdx.x;
   const int ty = tid / 16, tx = tid % 16;
   V acc[4][4];
   for(int r = 0; r < 4; r++)
      for(int c = 0; c < 4; c++) acc[r][c] = V{};
   for(int k0 = 0; k0 < L; k0 += GBK)
   {
      for(int e = tid; e < GBM * GBK; e += 256)
      {
         const int row = e / GBK, kk = e % GBK;
         const int64_t gi = i0 + row;
         const int gk = k0 + kk;
         As[kk][row] = (gi < M && gk < L) ? A[gi * L + gk] : V{};
      }
      for(int e = tid; e < GBK * GBN; e += 256)
      {
         const int kk = e / GBN, col = e % GBN;
         const int gk = k0 + kk, gj = j0 + col;
         Bs[kk][col] = (gk < L && gj < L) ? B[int64_t(gk) * L + gj] : V{};
      }
      __syncthreads();
#pragma unroll
      for(int kk = 0; kk < GBK; kk++)
      {
         V av[4], bv[4];
#pragma unroll
         for(int r = 0; r < 4; r++) av[r] = As[kk][ty * 4 + r];
#pragma unroll
         for(int c = 0; c < 4; c++) bv[c] = Bs[kk][tx * 4 + c];
#pragma unroll
         for(int r = 0; r < 4; r++)
#pragma unroll
            for(int c = 0; c < 4; c++) mac(acc[r][c], av[r], bv[c]);
      }
      __syncthreads();
   }
   for(int r = 0; r < 4; r++)
   {
      const int64_t gi = i0 + ty * 4 + r;
      if(gi >= M) continue;
      for(int c = 0; c < 4; c++)
      {
         const int gj = j0 + tx * 4 + c;
         if(gj < L) C[gi * L + gj] = acc[r][c];
      }
   }
}

// Runs `launch(a_dev, b_dev, result_dev)` on device or host buffers. Host buffers are staged
// through stream-ordered allocations that are freed before returning; the call then waits for
// the result. Device buffers are used in place and the call returns without waiting.
template <class F>
fmm_status withBuffers(const char* who, int on_device, cudaStream_t st, const void* a, size_t aBytes,
                       const void* b, size_t bBytes, void* result, size_t rBytes, F launch)
{
   if(on_device)
   {
      launch(a, b, result);
      cudaError_t e = cudaGetLastError();
      if(e != cudaSuccess) return setError(FMM_E_CUDA, "%s: %s", who, cudaGetErrorString(e));
      return FMM_OK;
   }
   void *da = nullptr, *db = nullptr, *dr = nullptr;
   cudaError_t e = cudaMallocAsync(&da, std::max<size_t>(aBytes, 16), st);
   if(e == cudaSuccess) e = cudaMallocAsync(&db, std::max<size_t>(bBytes, 16), st);
   if(e == cudaSuccess) e = cudaMallocAsync(&dr, std::max<size_t>(rBytes, 16), st);
   if(e == cudaSuccess && aBytes) e = cudaMemcpyAsync(da, a, aBytes, cudaMemcpyHostToDevice, st);
   if(e == cudaSuccess && bBytes) e = cudaMemcpyAsync(db, b, bBytes, cudaMemcpyHostToDevice, st);
   if(e == cudaSuccess)
   {
      launch(da, db, dr);
      e = cudaGetLastError();
   }
   if(e == cudaSuccess && rBytes) e = cudaMemcpyAsync(result, dr, rBytes, cudaMemcpyDeviceToHost, st);
   const fmm_status bad = e == cudaErrorMemoryAllocation ? FMM_E_OOM : FMM_E_CUDA;
   const cudaError_t first = e;
   if(da) cudaFreeAsync(da, st);
   if(db) cudaFreeAsync(db, st);
   if(dr) cudaFreeAsync(dr, st);
   cudaError_t es = cudaStreamSynchronize(st);
   if(first != cudaSuccess)
   {
      cudaGetLastError();
      return setError(bad, "%s: %s", who, cudaGetErrorString(first));
   }
   if(es != cudaSuccess) return setError(FMM_E_CUDA, "%s: %s", who, cudaGetErrorString(es));
   return FMM_OK;
}

constexpr int SEAM_MAX_ORDER = 32;
constexpr int SEAM_MAX_GRID = 148 * 64;

template <class T>
void launchTranslateAll(T* r, const T* a, const T* b, int64_t count, int p, cudaStream_t st)
{
   if(count == 0) return;
   const int L = (p + 1) * (p + 1);
   const int npairs = (p + 1) * (p + 2) / 2;
   const int threads = std::min(256, std::max(32, (npairs + 31) / 32 * 32));
   const int grid = int(std::min<int64_t>(count, SEAM_MAX_GRID));
   kTranslateAll<T><<<grid, threads, 4 * L * sizeof(T), st>>>(r, a, b, count, p);
}

template <class V>
void launchRowGemm(V* C, const V* A, const V* B, int64_t M, int L, int64_t batch, cudaStream_t st)
{
   if(M == 0 || L == 0 || batch == 0) return;
   dim3 grid(unsigned((M + GBM - 1) / GBM), unsigned((L + GBN - 1) / GBN), unsigned(batch));
   kRowGemm<V><<<grid, 256, 0, st>>>(C, A, B, M, L);
}

}  // namespace
}  // namespace fmm

using namespace fmm;

extern "C" {

fmm_status fmm_translate_all(void* result, const void* harmonics, const void* expansions, int64_t count, int order,
                             int precision, int on_device, void* stream)
{
   if(count < 0 || order < 0 || order > SEAM_MAX_ORDER || (precision != FMM_FP32 && precision != FMM_FP64))
      return setError(FMM_E_INVALID, "fmm_translate_all: bad count/order/precision");
   if(count > 0 && (!result || !harmonics || !expansions))
      return setError(FMM_E_INVALID, "fmm_translate_all: null pointer");
   if(count == 0) return FMM_OK;
   const size_t es = precision == FMM_FP64 ? 8 : 4;
   const size_t L = size_t(order + 1) * (order + 1);
   cudaStream_t st = (cudaStream_t)stream;
   return withBuffers("fmm_translate_all", on_device, st, harmonics, es * L * count, expansions, es * 3 * L * count,
                      result, es * 3 * L * count, [&](const void* a, const void* b, void* r) {
                         if(precision == FMM_FP64)
                            launchTranslateAll<double>((double*)r, (const double*)a, (const double*)b, count, order, st);
                         else
                            launchTranslateAll<float>((float*)r, (const float*)a, (const float*)b, count, order, st);
                      });
}

fmm_status fmm_translate_all_matrix(void* result, const void* a, const void* b, int64_t count, int order,
                                    int64_t batch, int precision, int on_device, void* stream)
{
   if(count < 0 || order < 0 || batch < 0 || batch > 65535 || (precision != FMM_FP32 && precision != FMM_FP64))
      return setError(FMM_E_INVALID, "fmm_translate_all_matrix: bad count/order/batch/precision");
   const int64_t L = int64_t(order + 1) * (order + 1);
   if(L > (1 << 20) || (count + GBM - 1) / GBM > INT32_MAX)
      return setError(FMM_E_LIMIT, "fmm_translate_all_matrix: size beyond the kernel's grid");
   if(count == 0 || batch == 0) return FMM_OK;
   if(!result || !a || !b) return setError(FMM_E_INVALID, "fmm_translate_all_matrix: null pointer");
   const size_t es = precision == FMM_FP64 ? 8 : 4;
   cudaStream_t st = (cudaStream_t)stream;
   return withBuffers("fmm_translate_all_matrix", on_device, st, a, es * L * count * batch, b, es * L * L, result,
                      es * L * count * batch, [&](const void* da, const void* db, void* dr) {
                         if(precision == FMM_FP64)
                            launchRowGemm<double>((double*)dr, (const double*)da, (const double*)db, count, int(L), batch, st);
                         else
                            launchRowGemm<float>((float*)dr, (const float*)da, (const float*)db, count, int(L), batch, st);
                      });
}

fmm_status fmm_translate_all_matrix_complex(void* result, const void* a, const void* b, int64_t count, int order,
                                            int precision, int on_device, void* stream)
{
   if(count < 0 || order < 0 || (precision != FMM_FP32 && precision != FMM_FP64))
      return setError(FMM_E_INVALID, "fmm_translate_all_matrix_complex: bad count/order/precision");
   const int64_t L = int64_t(order + 1) * (order + 1);
   if(L > (1 << 20) || (count + GBM - 1) / GBM > INT32_MAX)
      return setError(FMM_E_LIMIT, "fmm_translate_all_matrix_complex: size beyond the kernel's grid");
   if(count == 0) return FMM_OK;
   if(!result || !a || !b) return setError(FMM_E_INVALID, "fmm_translate_all_matrix_complex: null pointer");
   const size_t es = precision == FMM_FP64 ? 16 : 8;
   cudaStream_t st = (cudaStream_t)stream;
   return withBuffers("fmm_translate_all_matrix_complex", on_device, st, a, es * L * count, b, es * L * L, result,
                      es * L * count, [&](const void* da, const void* db, void* dr) {
                         if(precision == FMM_FP64)
                            launchRowGemm<double2>((double2*)dr, (const double2*)da, (const double2*)db, count, int(L), 1, st);
                         else
                            launchRowGemm<float2>((float2*)dr, (const float2*)da, (const float2*)db, count, int(L), 1, st);
                      });
}

}  // extern "C"
