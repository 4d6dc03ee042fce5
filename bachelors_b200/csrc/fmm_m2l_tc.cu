// M2L on the 5th-generation tensor cores (tcgen05, sm_100a), split-BF16 x3.
//
// The M2L step of the reference (FastMultipoleSolver::accountFarInteractions ->
// MultipoleTranslator::multipoleToLocalWithComplex, FMM/FMMGPU/fast_multipole_solver.cpp:258-276,
// multipole_translator.cpp:148-199) translates, for every (target box, source box) pair of the
// interaction lists, the source multipole into the target local expansion. With box-size scaled
// expansions the translation depends only on the offset o between the boxes (316 offsets), so
// a target box's local expansion is  L~_t = sum_o T_o M~_{t+o}: a sum of GEMMs.
//
// One CTA owns 42 consecutive target boxes = 126 rows (box, component) of a 128-row tile and
// all (p+1)^2 output coefficients (TMEM columns). For each offset with at least one source in
// the tile it accumulates  D[128 x N] += A_o[128 x K] * T_o^T[K x N]  where the rows of A_o are
// the gathered source multipoles. Operands are split x = hi + lo in bf16 and the three products
// hi*hi + hi*lo + lo*hi are accumulated in FP32 in tensor memory.
//
// Warp roles (320 threads):
//   warp 0      TMEM allocation; lane 0 issues the tcgen05.mma instructions
//   warp 1      lane 0 streams the pre-swizzled operator image with cp.async.bulk (no multicast)
//   warps 2..9  gather source rows (FP32), split to bf16 hi/lo, store in the SW128 K-major layout
//   warps 2..5  epilogue: tcgen05.ld of the accumulator, store of the local expansions
// Stages hold one 64-wide K chunk of A (hi, lo) and of T_o (hi, lo); two stages rotate through
// mbarriers (full: producers + bulk-copy bytes, empty: tcgen05.commit). Every wait is bounded by
// a 2 s global-timer limit; on expiry the CTA records FMM timeout in the error word and stops.
#include <cuda_bf16.h>

#include "fmm_internal.cuh"

namespace fmm {

namespace tc {

constexpr int TT = 42;               // target boxes per tile
constexpr int ROWS = 128;            // MMA M
constexpr int KC = 64;               // K chunk (one 128-byte swizzle atom of bf16)
constexpr int NPROD = 256;           // producer threads
constexpr int NTHREADS = 320;
constexpr uint64_t TIMEOUT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t globalTimer()
{
   uint64_t t;
   asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
   return t;
}

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbarArrive(uint32_t bar)
{
   asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbarArriveExpectTx(uint32_t bar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint32_t bar, uint32_t parity)
{
   uint32_t ok;
   asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
   return ok != 0;
}

// Bounded wait; returns false (and raises the error word) when the limit expires.
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity, int* err, volatile int* abortFlag)
{
   if(mbarTryWait(bar, parity)) return true;
   const uint64_t t0 = globalTimer();
   while(true)
   {
      if(mbarTryWait(bar, parity)) return true;
      if(*abortFlag) return false;
      if(globalTimer() - t0 > TIMEOUT_NS)
      {
         atomicOr(err, ERR_TIMEOUT);
         *abortFlag = 1;
         return false;
      }
   }
}

__device__ __forceinline__ void bulkLoad(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr)
{
   uint64_t d = 0;
   d |= uint64_t((addr >> 4) & 0x3FFF);          // start address
   d |= uint64_t(1) << 16;                        // leading byte offset (unused for swizzled K-major)
   d |= uint64_t(1024 >> 4) << 32;                // stride byte offset
   d |= uint64_t(1) << 46;                        // descriptor version for sm_100
   d |= uint64_t(2) << 61;                        // SWIZZLE_128B
   return d;
}

// Instruction descriptor: bf16 x bf16 -> f32, A and B K-major, shape M x N.
__host__ __device__ constexpr uint32_t instrDescBf16(int M, int N)
{
   return (1u << 4)                  // D format F32
          | (1u << 7)                // A format BF16
          | (1u << 10)               // B format BF16
          | (uint32_t(N >> 3) << 17) // N
          | (uint32_t(M >> 4) << 24);  // M
}

__device__ __forceinline__ void mmaBf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accumulate)
{
   asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dTmem), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mmaCommit(uint32_t bar)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmemLd16(uint32_t addr, float* v)
{
   uint32_t r[16];
   asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for(int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) (k < 64, bf16) inside a SW128 K-major block of 128-byte rows.
__host__ __device__ constexpr uint32_t swz(uint32_t row, uint32_t k)
{
   return row * 128u + ((((k >> 3) ^ (row & 7u)) & 7u) << 4) + ((k & 7u) << 1);
}

}  // namespace tc

// Operator image for the tensor-core M2L: for every offset slot and K chunk, the hi block then
// the lo block, each N rows (output coefficients, N = Lp) x 64 bf16 (input coefficients) in
// the SW128 K-major layout, zero outside the (p+1)^2 x (p+1)^2 operator.
__global__ void kPrepM2LImage(const double* __restrict__ op64, int L, int N, int nChunks, __nv_bfloat16* img)
{
   const int64_t blockElems = int64_t(N) * tc::KC;             // one hi or lo block
   const int64_t total = int64_t(316) * nChunks * 2 * blockElems;
   for(int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
   {
      int64_t r = e;
      const int kk = int(r % tc::KC); r /= tc::KC;
      const int n = int(r % N); r /= N;
      const int half = int(r % 2); r /= 2;
      const int c = int(r % nChunks);
      const int o = int(r / nChunks);
      const int k = c * tc::KC + kk;
      double x = (n < L && k < L) ? op64[(int64_t(o) * L + n) * L + k] : 0.0;
      __nv_bfloat16 hi = __float2bfloat16_rn(float(x));
      __nv_bfloat16 v = half == 0 ? hi : __float2bfloat16_rn(float(x - double(__bfloat162float(hi))));
      uint8_t* blk = reinterpret_cast<uint8_t*>(img) + ((int64_t(o) * nChunks + c) * 2 + half) * blockElems * 2;
      *reinterpret_cast<__nv_bfloat16*>(blk + tc::swz(uint32_t(n), uint32_t(kk))) = v;
   }
}

__global__ void __launch_bounds__(tc::NTHREADS, 1)
kM2LTc(int firstNode, int nNodes, const int* __restrict__ vtab, int Lp, int nChunks,
       const uint8_t* __restrict__ img, const float* __restrict__ M, float* __restrict__ Lc, int* err)
{
   using namespace tc;
   extern __shared__ uint8_t smraw[];
   const int N = Lp;                                  // output columns (<= 320)
   const uint32_t aBytes = ROWS * 128;                // one A block (hi or lo), 16 KB
   const uint32_t bBytes = uint32_t(N) * 128;         // one B block (hi or lo)
   const uint32_t stageBytes = 2 * aBytes + 2 * bBytes;
   // 1024-byte aligned stage area, then the control block
   const uint32_t rawAddr = smemAddr(smraw);
   const uint32_t base = (rawAddr + 1023u) & ~1023u;
   uint8_t* sbase = smraw + (base - rawAddr);
   uint8_t* ctrl = sbase + 2 * stageBytes;
   uint64_t* bars = reinterpret_cast<uint64_t*>(ctrl);          // full[2], empty[2], done
   uint32_t* tmemBase = reinterpret_cast<uint32_t*>(ctrl + 64);
   volatile int* abortFlag = reinterpret_cast<volatile int*>(ctrl + 68);
   uint32_t* present = reinterpret_cast<uint32_t*>(ctrl + 72);  // 10 words: offsets present in the tile
   int* itemOffset = reinterpret_cast<int*>(ctrl + 128);        // compacted present offsets [316]

   const int tid = threadIdx.x;
   const int warp = tid >> 5, lane = tid & 31;
   const int t0 = firstNode + blockIdx.x * TT;
   const int tEnd = min(t0 + TT, firstNode + nNodes);
   const uint32_t fullBar0 = smemAddr(&bars[0]), emptyBar0 = smemAddr(&bars[2]), doneBar = smemAddr(&bars[4]);

   if(tid < 10) present[tid] = 0;
   if(tid == 0)
   {
      *abortFlag = 0;
      mbarInit(fullBar0, NPROD + 1);
      mbarInit(fullBar0 + 8, NPROD + 1);
      mbarInit(emptyBar0, 1);
      mbarInit(emptyBar0 + 8, 1);
      mbarInit(doneBar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if(warp == 0)
   {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(tmemBase)),
                   "r"(512));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   __syncthreads();
   // which offsets have a source for some box of the tile
   for(int e = tid; e < TT * 316; e += NTHREADS)
   {
      const int t = t0 + e / 316, o = e % 316;
      if(t < tEnd && vtab[int64_t(t) * 316 + o] >= 0) atomicOr(&present[o >> 5], 1u << (o & 31));
   }
   fenceBeforeSync();
   __syncthreads();
   fenceAfterSync();
   // compact the present offsets (same list for every role)
   if(tid == 0)
   {
      int k = 0;
      for(int o = 0; o < 316; o++)
         if(present[o >> 5] & (1u << (o & 31))) itemOffset[k++] = o;
      itemOffset[316] = k;
   }
   __syncthreads();
   const int nOff = itemOffset[316];
   const int nItems = nOff * nChunks;
   const uint32_t tmem = *tmemBase;

   if(warp == 0)
   {
      if(lane == 0)
      {
         const uint32_t idA = instrDescBf16(ROWS, 256);
         const int nB = N - 256;                      // 48 for p = 16; <= 0 for smaller orders
         const uint32_t idB = nB > 0 ? instrDescBf16(ROWS, nB) : 0u;
         const uint32_t idFull = instrDescBf16(ROWS, N <= 256 ? N : 256);
         bool first = true;
         for(int it = 0; it < nItems; it++)
         {
            const int s = it & 1;
            if(!mbarWait(fullBar0 + 8 * s, (it >> 1) & 1, err, abortFlag)) break;
            fenceAfterSync();
            const uint32_t st = base + s * stageBytes;
            const uint32_t aHi = st, aLo = st + aBytes, bHi = st + 2 * aBytes, bLo = bHi + bBytes;
#pragma unroll
            for(int ks = 0; ks < KC / 16; ks++)
            {
               const uint32_t koff = ks * 32;
               const uint32_t a[3] = {aHi + koff, aHi + koff, aLo + koff};
               const uint32_t b[3] = {bHi + koff, bLo + koff, bHi + koff};
#pragma unroll
               for(int pass = 0; pass < 3; pass++)
               {
                  const uint32_t acc = first ? 0u : 1u;
                  mmaBf16(tmem, smemDesc(a[pass]), smemDesc(b[pass]), N <= 256 ? idFull : idA, acc);
                  if(nB > 0) mmaBf16(tmem + 256, smemDesc(a[pass]), smemDesc(b[pass] + 256 * 128), idB, acc);
                  first = false;
               }
            }
            mmaCommit(emptyBar0 + 8 * s);
         }
         mmaCommit(doneBar);
      }
      __syncwarp();
   }
   else if(warp == 1)
   {
      if(lane == 0)
      {
         for(int it = 0; it < nItems; it++)
         {
            const int s = it & 1;
            if(it >= 2 && !mbarWait(emptyBar0 + 8 * s, ((it >> 1) - 1) & 1, err, abortFlag)) break;
            const int o = itemOffset[it / nChunks], c = it % nChunks;
            const uint8_t* src = img + (int64_t(o) * nChunks + c) * 2 * bBytes;
            const uint32_t dst = base + s * stageBytes + 2 * aBytes;
            mbarArriveExpectTx(fullBar0 + 8 * s, 2 * bBytes);
            bulkLoad(dst, src, 2 * bBytes, fullBar0 + 8 * s);
         }
      }
      __syncwarp();
   }
   else
   {
      // producers: two threads per row, 32 K-elements each
      const int ptid = tid - 64;
      const int row = ptid >> 1, half = ptid & 1;
      const int tgt = t0 + row / 3, comp = row % 3;
      const bool rowValid = row < 3 * TT && tgt < tEnd;
      for(int it = 0; it < nItems; it++)
      {
         const int s = it & 1;
         if(it >= 2 && !mbarWait(emptyBar0 + 8 * s, ((it >> 1) - 1) & 1, err, abortFlag)) break;
         const int o = itemOffset[it / nChunks], c = it % nChunks;
         int src = -1;
         if(rowValid) src = vtab[int64_t(tgt) * 316 + o];
         uint8_t* aHi = sbase + s * stageBytes;
         uint8_t* aLo = aHi + aBytes;
         const int k0 = c * KC + half * 32;
#pragma unroll
         for(int q = 0; q < 4; q++)
         {
            float v[8];
            const int k = k0 + 8 * q;
            if(src >= 0 && k < Lp)
            {
               const float4* p = reinterpret_cast<const float4*>(M + (int64_t(src) * 3 + comp) * Lp + k);
               const float4 x0 = __ldg(p), x1 = __ldg(p + 1);
               v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w; v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
            }
            else
            {
#pragma unroll
               for(int i = 0; i < 8; i++) v[i] = 0.f;
            }
            uint32_t hw[4], lw[4];
#pragma unroll
            for(int i = 0; i < 4; i++)
            {
               const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * i]), h1 = __float2bfloat16_rn(v[2 * i + 1]);
               const __nv_bfloat16 l0 = __float2bfloat16_rn(v[2 * i] - __bfloat162float(h0));
               const __nv_bfloat16 l1 = __float2bfloat16_rn(v[2 * i + 1] - __bfloat162float(h1));
               hw[i] = uint32_t(__bfloat16_as_ushort(h0)) | (uint32_t(__bfloat16_as_ushort(h1)) << 16);
               lw[i] = uint32_t(__bfloat16_as_ushort(l0)) | (uint32_t(__bfloat16_as_ushort(l1)) << 16);
            }
            const uint32_t off = swz(uint32_t(row), uint32_t(half * 32 + 8 * q));
            *reinterpret_cast<uint4*>(aHi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4*>(aLo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
         }
         fenceProxyAsync();
         mbarArrive(fullBar0 + 8 * s);
      }
      // epilogue on warps 2..5: TMEM lanes 32 (warp % 4) .. + 31
      if(warp < 6)
      {
         const bool ok = mbarWait(doneBar, 0, err, abortFlag);
         fenceAfterSync();
         const int lanes = 32 * (warp & 3);
         const int r = lanes + lane;
         const int et = t0 + r / 3, ec = r % 3;
         const bool valid = r < 3 * TT && et < tEnd;
         float* out = Lc + (int64_t(et) * 3 + ec) * Lp;
         for(int c0 = 0; c0 < N; c0 += 16)
         {
            float v[16];
            if(ok && nItems > 0) tmemLd16(tmem + (uint32_t(lanes) << 16) + uint32_t(c0), v);
            else
               for(int i = 0; i < 16; i++) v[i] = 0.f;
            if(valid)
               for(int i = 0; i < 16; i++) out[c0 + i] = v[i];
         }
      }
   }
   fenceBeforeSync();
   __syncthreads();
   if(warp == 0)
   {
      // the accumulator must be idle before it is released, also after an aborted pipeline
      if(lane == 0 && nItems > 0) mbarWait(doneBar, 0, err, abortFlag);
      __syncwarp();
      fenceAfterSync();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
   }
}

fmm_status m2lTensorCore(Plan& P, cudaStream_t st)
{
   if(P.cfg.m2l_mode != FMM_M2L_BF16X3)
      return setError(FMM_E_INVALID, "tensor-core M2L: only the BF16X3 mode is built");
   const int L = P.L, Lp = P.Lp;
   if(Lp > 320) return setError(FMM_E_INVALID, "tensor-core M2L supports p <= 16");
   if(Lp % 16) return setError(FMM_E_INVALID, "tensor-core M2L needs 16-aligned coefficient rows");
   const int nChunks = (L + tc::KC - 1) / tc::KC;
   const size_t imgBytes = size_t(316) * nChunks * 2 * size_t(Lp) * 128;
   if(P.opImgOrder != P.p)
   {
      FMM_TRY(P.opM2Lbf.reserve(imgBytes));
      kPrepM2LImage<<<4096, 256, 0, st>>>((const double*)P.opM2L64.ptr, L, Lp, nChunks, (__nv_bfloat16*)P.opM2Lbf.ptr);
      FMM_TRY(launched(P, "kPrepM2LImage", st));
      P.opImgOrder = P.p;
   }
   const int first = 1;
   const int count = int(P.tree.nNodes - 1);
   if(count <= 0) return FMM_OK;
   const int blocks = (count + tc::TT - 1) / tc::TT;
   const size_t stageBytes = 2 * tc::ROWS * 128 + 2 * size_t(Lp) * 128;
   const size_t smem = 1024 + 2 * stageBytes + 128 + 4 * 320;
   FMM_CUDA(cudaFuncSetAttribute(kM2LTc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
   FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
   kM2LTc<<<blocks, tc::NTHREADS, smem, st>>>(first, count, P.lists.vtab, Lp, nChunks, (const uint8_t*)P.opM2Lbf.ptr,
                                             (const float*)P.mult.ptr, (float*)P.local.ptr, P.err);
   FMM_TRY(launched(P, "kM2LTc", st));
   int herr = 0;
   FMM_CUDA(cudaMemcpyAsync(&herr, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
   FMM_CUDA(cudaStreamSynchronize(st));
   if(herr & ERR_TIMEOUT) return setError(FMM_E_TIMEOUT, "tensor-core M2L: a pipeline wait timed out");
   return FMM_OK;
}

}  // namespace fmm
