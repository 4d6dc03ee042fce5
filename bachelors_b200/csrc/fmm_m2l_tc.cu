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
// the gathered source multipoles. Operands are split into bf16 pieces: x = hi + lo with the three
// products hi*hi + hi*lo + lo*hi (BF16X3), or x = hi + mid + lo with the six products down to
// 2^-16 relative (BF16X6); all are accumulated in FP32 in tensor memory.
//
// Warp roles (448 threads):
//   warp 0      TMEM allocation; lane 0 issues the tcgen05.mma instructions
//   warp 1      lane 0 streams the pre-swizzled operator image with cp.async.bulk (no multicast)
//   warps 2..9  gather source rows (FP32), split to bf16 pieces, store in the swizzled K-major layout
//   warps 10-13 drain: every few offsets tcgen05.ld the accumulator and add it to the FP32 local
//               expansions in global memory (the tensor-core accumulation truncates; long chains
//               into one TMEM value lose accuracy), then release TMEM for a fresh accumulation
// Stages hold one K chunk of every piece of A and of T_o; two stages rotate through mbarriers
// (full: producers + bulk-copy bytes, empty: tcgen05.commit). Every wait is bounded by
// a 2 s global-timer limit; on expiry the CTA records FMM timeout in the error word and stops.
#include <cstdlib>

#include <cuda_bf16.h>

#include "fmm_internal.cuh"

namespace fmm {

namespace tc {

constexpr int TT = 42;               // target boxes per tile
constexpr int ROWS = 128;            // MMA M
// (the K chunk width depends on the number of bf16 pieces, see Layout)
constexpr int NPROD = 256;           // producer threads
constexpr int NTHREADS = 448;
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


// Operand layout for NP bf16 pieces per value (2: hi + lo, 3: hi + mid + lo). With two pieces a K
// chunk is 64 elements in 128-byte rows (SW128, 108 KB per stage); with three it is 32 elements in
// 64-byte rows (SW64, 83 KB per stage); two stages in both. (Four SW64 stages of two pieces were
// measured slower than two SW128 stages: more barrier round trips per offset.)
template <int NP> struct Layout;
template <> struct Layout<2>
{
   static constexpr int KC = 64, RB = 128, SBO = 1024, SWZ = 2, NSTAGE = 2;
   __host__ __device__ static constexpr uint32_t off(uint32_t row, uint32_t k)
   { return row * 128u + ((((k >> 3) ^ (row & 7u)) & 7u) << 4) + ((k & 7u) << 1); }
};
template <> struct Layout<3>
{
   static constexpr int KC = 32, RB = 64, SBO = 512, SWZ = 4, NSTAGE = 2;
   __host__ __device__ static constexpr uint32_t off(uint32_t row, uint32_t k)
   { return row * 64u + ((((k >> 3) ^ ((row >> 1) & 3u)) & 3u) << 4) + ((k & 7u) << 1); }
};

// Shared-memory matrix descriptor: K-major, swizzled rows, 8-row groups SBO bytes apart.
template <int NP>
__device__ __forceinline__ uint64_t smemDescT(uint32_t addr)
{
   uint64_t d = 0;
   d |= uint64_t((addr >> 4) & 0x3FFF);               // start address
   d |= uint64_t(1) << 16;                             // leading byte offset (unused when swizzled)
   d |= uint64_t(Layout<NP>::SBO >> 4) << 32;         // stride byte offset
   d |= uint64_t(1) << 46;                             // descriptor version for sm_100
   d |= uint64_t(Layout<NP>::SWZ) << 61;              // swizzle mode
   return d;
}

// Split of x into NP bf16 pieces, each the round-to-nearest of the remaining residual.
template <int NP>
__device__ __forceinline__ void splitBf16(double x, __nv_bfloat16* piece)
{
   double r = x;
#pragma unroll
   for(int i = 0; i < NP; i++)
   {
      piece[i] = __float2bfloat16_rn(float(r));
      r -= double(__bfloat162float(piece[i]));
   }
}

}  // namespace tc

// Operator image for the tensor-core M2L: for every offset slot and K chunk, the NP piece blocks
// (hi first), each N rows (output coefficients, N = Lp) x KC bf16 (input coefficients) in the
// swizzled K-major layout, zero outside the (p+1)^2 x (p+1)^2 operator.
template <int NP>
__global__ void kPrepM2LImage(const double* __restrict__ op64, int L, int N, int nChunks, uint8_t* img)
{
   using Lay = tc::Layout<NP>;
   const int64_t blockBytes = int64_t(N) * Lay::RB;
   const int64_t total = int64_t(316) * nChunks * int64_t(N) * Lay::KC;
   for(int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
   {
      int64_t r = e;
      const int kk = int(r % Lay::KC); r /= Lay::KC;
      const int n = int(r % N); r /= N;
      const int c = int(r % nChunks);
      const int o = int(r / nChunks);
      const int k = c * Lay::KC + kk;
      const double x = (n < L && k < L) ? op64[(int64_t(o) * L + n) * L + k] : 0.0;
      __nv_bfloat16 piece[NP];
      tc::splitBf16<NP>(x, piece);
      uint8_t* blk = img + (int64_t(o) * nChunks + c) * NP * blockBytes;
#pragma unroll
      for(int i = 0; i < NP; i++)
         *reinterpret_cast<__nv_bfloat16*>(blk + i * blockBytes + Lay::off(uint32_t(n), uint32_t(kk))) = piece[i];
   }
}

template <int NP>
__global__ void __launch_bounds__(tc::NTHREADS, 1)
kM2LTc(const int* __restrict__ targets, int nTargets, const int* __restrict__ vtab, int Lp, int nChunks,
       const uint8_t* __restrict__ img, const float* __restrict__ M, float* __restrict__ Lc, int drainEvery, int* err)
{
   using namespace tc;
   using Lay = Layout<NP>;
   constexpr int KCH = Lay::KC;
   constexpr int NPASS = NP == 2 ? 3 : 6;
   // (A piece, B piece) of every product kept: hi*hi, hi*lo, lo*hi  /  down to 2^-16 with three pieces
   constexpr int PA[6] = {0, 0, 1, 1, 0, 2};
   constexpr int PB[6] = {0, 1, 0, 1, 2, 0};
   constexpr int PA2[3] = {0, 0, 1};
   constexpr int PB2[3] = {0, 1, 0};
   extern __shared__ uint8_t smraw[];
   const int N = Lp;                                   // output columns (<= 320)
   const uint32_t aBytes = ROWS * Lay::RB;             // one A piece
   const uint32_t bBytes = uint32_t(N) * Lay::RB;      // one B piece
   const uint32_t stageBytes = NP * (aBytes + bBytes);
   const uint32_t rawAddr = smemAddr(smraw);
   const uint32_t base = (rawAddr + 1023u) & ~1023u;
   uint8_t* sbase = smraw + (base - rawAddr);
   constexpr int NS = Lay::NSTAGE;
   uint8_t* ctrl = sbase + NS * stageBytes;
   uint64_t* bars = reinterpret_cast<uint64_t*>(ctrl);          // full[NS], empty[NS], done, drainFull, drainEmpty
   uint32_t* tmemBase = reinterpret_cast<uint32_t*>(ctrl + 128);
   volatile int* abortFlag = reinterpret_cast<volatile int*>(ctrl + 132);
   uint32_t* present = reinterpret_cast<uint32_t*>(ctrl + 136); // 10 words: offsets present in the tile
   int* itemOffset = reinterpret_cast<int*>(ctrl + 192);        // compacted present offsets [316] + count
   int* tileNode = itemOffset + 320;                            // the tile's target boxes [TT]

   const int tid = threadIdx.x;
   const int warp = tid >> 5, lane = tid & 31;
   const int first = blockIdx.x * TT;
   const int nTile = min(TT, nTargets - first);
   const uint32_t fullBar0 = smemAddr(&bars[0]), emptyBar0 = smemAddr(&bars[NS]), doneBar = smemAddr(&bars[2 * NS]);
   const uint32_t drainFull = smemAddr(&bars[2 * NS + 1]), drainEmpty = smemAddr(&bars[2 * NS + 2]);

   if(tid < 10) present[tid] = 0;
   if(tid < TT) tileNode[tid] = tid < nTile ? targets[first + tid] : -1;
   if(tid == 0)
   {
      *abortFlag = 0;
      for(int s = 0; s < NS; s++)
      {
         mbarInit(fullBar0 + 8 * s, NPROD + 1);
         mbarInit(emptyBar0 + 8 * s, 1);
      }
      mbarInit(doneBar, 1);
      mbarInit(drainFull, 1);
      mbarInit(drainEmpty, 128);
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
      const int t = tileNode[e / 316], o = e % 316;
      if(t >= 0 && vtab[int64_t(t) * 316 + o] >= 0) atomicOr(&present[o >> 5], 1u << (o & 31));
   }
   fenceBeforeSync();
   __syncthreads();
   fenceAfterSync();
   if(tid == 0)
   {
      // far offsets first: the smaller contributions enter the accumulator before the large ones
      int k = 0;
      for(int i = 0; i < 316; i++)
      {
         const int o = d_m2lFarFirst[i];
         if(present[o >> 5] & (1u << (o & 31))) itemOffset[k++] = o;
      }
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
         const int nB = N - 256;                       // second MMA's width (48 at p = 16)
         const uint32_t idA = instrDescBf16(ROWS, N <= 256 ? N : 256);
         const uint32_t idB = nB > 0 ? instrDescBf16(ROWS, nB) : 0u;
         bool firstMma = true;
         int drains = 0;
         for(int it = 0; it < nItems; it++)
         {
            const int s = it % NS;
            if(!mbarWait(fullBar0 + 8 * s, (it / NS) & 1, err, abortFlag)) break;
            fenceAfterSync();
            const uint32_t st = base + s * stageBytes;
            const uint32_t aSt = st, bSt = st + NP * aBytes;
#pragma unroll
            for(int ks = 0; ks < KCH / 16; ks++)
            {
               const uint32_t koff = ks * 32;
#pragma unroll
               for(int pass = 0; pass < NPASS; pass++)
               {
                  const int pa = NP == 2 ? PA2[pass] : PA[pass];
                  const int pb = NP == 2 ? PB2[pass] : PB[pass];
                  const uint32_t a = aSt + pa * aBytes + koff;
                  const uint32_t b = bSt + pb * bBytes + koff;
                  const uint32_t acc = firstMma ? 0u : 1u;
                  mmaBf16(tmem, smemDescT<NP>(a), smemDescT<NP>(b), idA, acc);
                  if(nB > 0) mmaBf16(tmem + 256, smemDescT<NP>(a), smemDescT<NP>(b + 256 * Lay::RB), idB, acc);
                  firstMma = false;
               }
            }
            mmaCommit(emptyBar0 + 8 * s);
            // every drainEvery offsets (and after the last) hand the accumulator to the drain warps
            // and start a fresh one: the tensor cores' FP32 accumulation truncates, so long chains
            // of accumulations into one TMEM value drift; the running sum is kept in FP32 instead
            if(it % nChunks == nChunks - 1)
            {
               const int oi = it / nChunks;
               if((oi + 1) % drainEvery == 0 || oi == nOff - 1)
               {
                  mmaCommit(drainFull);
                  if(oi != nOff - 1)
                  {
                     if(!mbarWait(drainEmpty, drains & 1, err, abortFlag)) break;
                     fenceAfterSync();
                  }
                  drains++;
                  firstMma = true;
               }
            }
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
            const int s = it % NS;
            if(it >= NS && !mbarWait(emptyBar0 + 8 * s, (it / NS - 1) & 1, err, abortFlag)) break;
            const int o = itemOffset[it / nChunks], c = nChunks - 1 - it % nChunks;
            const uint8_t* src = img + (int64_t(o) * nChunks + c) * NP * bBytes;
            const uint32_t dst = base + s * stageBytes + NP * aBytes;
            mbarArriveExpectTx(fullBar0 + 8 * s, NP * bBytes);
            bulkLoad(dst, src, NP * bBytes, fullBar0 + 8 * s);
         }
      }
      __syncwarp();
   }
   else if(warp >= 10)
   {
      // drain warps 10..13: TMEM lanes 32 (warp % 4) .. + 31, one accumulator row per thread
      const int lanes = 32 * (warp & 3);
      const int r = lanes + lane;
      const int et = r < 3 * TT ? tileNode[r / 3] : -1, ec = r % 3;
      float* out = Lc + (int64_t(et) * 3 + ec) * Lp;
      const int nDrains = (nOff + drainEvery - 1) / drainEvery;
      // The running sum lives in the (zero-initialised) local expansions: fire-and-forget FP32
      // vector adds, rounded to nearest. Each row has one writer, this thread, and same-address
      // operations of one thread stay in program order, so the result is deterministic.
      for(int d = 0; d < nDrains; d++)
      {
         if(!mbarWait(drainFull, d & 1, err, abortFlag)) break;
         fenceAfterSync();
         for(int c0 = 0; c0 < N; c0 += 16)
         {
            float v[16];
            tmemLd16(tmem + (uint32_t(lanes) << 16) + uint32_t(c0), v);
            if(et >= 0)
            {
               float4* o4 = reinterpret_cast<float4*>(out + c0);
#pragma unroll
               for(int i = 0; i < 4; i++) atomicAdd(o4 + i, make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
            }
         }
         fenceBeforeSync();
         mbarArrive(drainEmpty);
      }
   }
   else
   {
      // producers (warps 2..9): two threads per row, KCH / 2 K-elements each
      constexpr int PER = KCH / 2;
      const int ptid = tid - 64;
      const int row = ptid >> 1, half = ptid & 1;
      const int slot = row / 3, comp = row % 3;
      const int tgt = row < 3 * TT ? tileNode[slot] : -1;
      for(int it = 0; it < nItems; it++)
      {
         const int s = it % NS;
         if(it >= NS && !mbarWait(emptyBar0 + 8 * s, (it / NS - 1) & 1, err, abortFlag)) break;
         const int o = itemOffset[it / nChunks], c = nChunks - 1 - it % nChunks;
         const int src = tgt >= 0 ? vtab[int64_t(tgt) * 316 + o] : -1;
         uint8_t* aSt = sbase + s * stageBytes;
         const int k0 = c * KCH + half * PER;
#pragma unroll
         for(int q = 0; q < PER / 8; q++)
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
            uint32_t w[NP][4];
#pragma unroll
            for(int i = 0; i < 4; i++)
            {
               __nv_bfloat16 p0[NP], p1[NP];
               // FP32 residuals are exact here: each piece removes the leading bits of the remainder
               float r0 = v[2 * i], r1 = v[2 * i + 1];
#pragma unroll
               for(int j = 0; j < NP; j++)
               {
                  p0[j] = __float2bfloat16_rn(r0);
                  p1[j] = __float2bfloat16_rn(r1);
                  r0 -= __bfloat162float(p0[j]);
                  r1 -= __bfloat162float(p1[j]);
                  w[j][i] = uint32_t(__bfloat16_as_ushort(p0[j])) | (uint32_t(__bfloat16_as_ushort(p1[j])) << 16);
               }
            }
            const uint32_t off = Lay::off(uint32_t(row), uint32_t(half * PER + 8 * q));
#pragma unroll
            for(int j = 0; j < NP; j++)
               *reinterpret_cast<uint4*>(aSt + j * aBytes + off) = make_uint4(w[j][0], w[j][1], w[j][2], w[j][3]);
         }
         fenceProxyAsync();
         mbarArrive(fullBar0 + 8 * s);
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

template <int NP>
static fmm_status launchM2LTc(Plan& P, cudaStream_t st)
{
   using Lay = tc::Layout<NP>;
   const int L = P.L, Lp = P.Lp;
   const int nChunks = (L + Lay::KC - 1) / Lay::KC;
   const size_t imgBytes = size_t(316) * nChunks * NP * size_t(Lp) * Lay::RB;
   const int tag = P.p * 8 + NP;
   if(P.opImgOrder != tag)
   {
      FMM_TRY(P.opM2Lbf.reserve(imgBytes));
      kPrepM2LImage<NP><<<4096, 256, 0, st>>>((const double*)P.opM2L64.ptr, L, Lp, nChunks, (uint8_t*)P.opM2Lbf.ptr);
      FMM_TRY(launched(P, "kPrepM2LImage", st));
      P.opImgOrder = tag;
   }
   const int count = P.nM2LTargets;
   if(count <= 0) return FMM_OK;
   const int blocks = (count + tc::TT - 1) / tc::TT;
   const size_t stageBytes = NP * (size_t(tc::ROWS) + size_t(Lp)) * Lay::RB;
   const size_t smem = 1024 + Lay::NSTAGE * stageBytes + 192 + 4 * (320 + 64);
   if(smem > 232448) return setError(FMM_E_INVALID, "tensor-core M2L: %zu bytes of shared memory needed", smem);
   FMM_CUDA(cudaFuncSetAttribute(kM2LTc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
   FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
   int drainEvery = 8;
   if(const char* e = getenv("FMM_TC_DRAIN")) drainEvery = std::max(1, atoi(e));
   kM2LTc<NP><<<blocks, tc::NTHREADS, smem, st>>>((const int*)P.m2lTargets.ptr, count, P.lists.vtab, Lp, nChunks,
                                                 (const uint8_t*)P.opM2Lbf.ptr, (const float*)P.mult.ptr,
                                                 (float*)P.local.ptr, drainEvery, P.err);
   FMM_TRY(launched(P, "kM2LTc", st));
   if(P.capturing) return FMM_OK;  // inside a graph capture the error word is checked after the launch
   int herr = 0;
   FMM_CUDA(cudaMemcpyAsync(&herr, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
   FMM_CUDA(cudaStreamSynchronize(st));
   if(herr & ERR_TIMEOUT) return setError(FMM_E_TIMEOUT, "tensor-core M2L: a pipeline wait timed out");
   return FMM_OK;
}

fmm_status m2lTensorCore(Plan& P, cudaStream_t st)
{
   if(P.Lp > 320) return setError(FMM_E_INVALID, "tensor-core M2L supports p <= 16");
   if(P.Lp % 16) return setError(FMM_E_INVALID, "tensor-core M2L needs 16-aligned coefficient rows");
   if(P.cfg.m2l_mode == FMM_M2L_BF16X3) return launchM2LTc<2>(P, st);
   if(P.cfg.m2l_mode == FMM_M2L_BF16X6) return launchM2LTc<3>(P, st);
   return setError(FMM_E_INVALID, "tensor-core M2L: the TF32 mode is not built");
}

}  // namespace fmm
