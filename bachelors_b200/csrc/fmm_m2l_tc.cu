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
// 2^-16 relative (BF16X6), or one TF32 product of operands rounded to 11 significant bits (TF32,
// kind::tf32, 4-byte elements); all are accumulated in FP32 in tensor memory.
//
// Warp roles (576 threads):
//   warp 0      TMEM allocation; lane 0 issues the tcgen05.mma instructions
//   warp 1      lane 0 streams the pre-swizzled operator image with cp.async.bulk (no multicast)
//   warps 2..9  gather the source rows, already split into bf16 pieces once per solve
//               (kSplitMultipoles), with 16-byte cp.async copies into the swizzled K-major layout
//   warps 10-17 drain: every few offsets tcgen05.ld the accumulator and add it to FP32 running
//               sums (the tensor-core accumulation truncates; long chains into one TMEM value lose
//               accuracy), then release the accumulator for a fresh accumulation. The running sums
//               live in the tensor-memory columns the accumulator leaves free (208 of 512 at
//               p = 16, all of them at p <= 12), then (drainMode 3) 32 more in the drain threads'
//               registers, the rest in the local expansions in global memory. Each TMEM lane
//               quadrant has two drain warps, one per half of the columns
// Stages hold one K chunk of every piece of A and of T_o; two stages rotate through mbarriers
// (full: the producers' arrivals, op: the operator bulk copy's bytes, empty: tcgen05.commit).
// Every pipeline wait is bounded by a global-timer limit (2 s unless the plan sets another); on
// expiry the CTA records a timeout in the error word and every role leaves its loop. Before the
// CTA exits it still waits, whatever the abort flag says and again with a 2 s bound, for the
// asynchronous work it started: the producers for their cp.async copies, warp 1 for its bulk
// copies (the last phase of each stage's op barrier), warp 0 for its MMAs (tcgen05.commit to
// the done barrier); only then is the tensor memory freed.
#include <cstdlib>

#include <cuda_bf16.h>

#include "fmm_internal.cuh"

namespace fmm {

namespace tc {

constexpr int TT = 42;               // target boxes per tile
constexpr int ROWS = 128;            // MMA M
// (the K chunk width depends on the number of bf16 pieces, see Layout)
constexpr int NPROD = 256;           // producer threads
constexpr int NTHREADS = 576;
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

// The same test, but a thread whose phase has not completed is suspended in hardware until it does or
// until about suspendNs nanoseconds have passed: a waiting role then takes no issue slots from the
// MMA-issuing warp that shares its scheduler (spinning roles slowed every MMA by half).
__device__ __forceinline__ bool mbarTryWaitSleep(uint32_t bar, uint32_t parity, uint32_t suspendNs)
{
   uint32_t ok;
   asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(suspendNs)
      : "memory");
   return ok != 0;
}

// Bounded pipeline wait; returns false when another role of the CTA has given up, or (raising
// the error word and the CTA's abort flag) when limitNs expires.
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity, int* err, volatile int* abortFlag,
                                         uint64_t limitNs)
{
   if(mbarTryWait(bar, parity)) return true;
   const uint64_t t0 = globalTimer();
   // suspended tests of at most ~1 us (never beyond the limit) between the checks of the limit and the flag
   const uint32_t hint = uint32_t(limitNs < 1000 ? limitNs : 1000);
   while(true)
   {
      if(mbarTryWaitSleep(bar, parity, hint)) return true;
      if(*abortFlag) return false;
      if(globalTimer() - t0 > limitNs)
      {
         atomicOr(err, ERR_TIMEOUT);
         *abortFlag = 1;
         return false;
      }
   }
}

// Wait for asynchronous work this CTA issued itself (bulk copies, MMAs) before it releases the
// shared and tensor memory that work writes: the abort flag is ignored, since such work always
// completes; the 2 s bound only keeps a broken device from holding the CTA forever.
__device__ __forceinline__ bool mbarWaitIssued(uint32_t bar, uint32_t parity, int* err)
{
   if(mbarTryWait(bar, parity)) return true;
   const uint64_t t0 = globalTimer();
   while(true)
   {
      if(mbarTryWaitSleep(bar, parity, 1000)) return true;
      if(globalTimer() - t0 > TIMEOUT_NS)
      {
         atomicOr(err, ERR_TIMEOUT);
         return false;
      }
   }
}

// 16-byte global -> shared copy; srcBytes = 0 writes zeros without reading.
__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, uint32_t srcBytes)
{
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Arrive on the mbarrier once every cp.async this thread issued so far has landed (counts as one of
// the barrier's expected arrivals); the thread itself does not wait.
__device__ __forceinline__ void cpAsyncArriveNoinc(uint32_t bar)
{
   asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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

// Instruction descriptor: tf32 x tf32 -> f32, A and B K-major, shape M x N.
__host__ __device__ constexpr uint32_t instrDescTf32(int M, int N)
{
   return (1u << 4)                  // D format F32
          | (2u << 7)                // A format TF32
          | (2u << 10)               // B format TF32
          | (uint32_t(N >> 3) << 17) // N
          | (uint32_t(M >> 4) << 24);  // M
}

__device__ __forceinline__ void mmaTf32(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accumulate)
{
   asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dTmem), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate));
}

// x rounded to tf32 (10 explicit mantissa bits, round to nearest, ties away), as its fp32 bit pattern
__device__ __forceinline__ uint32_t toTf32(float x)
{
   uint32_t r;
   asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
   return r;
}

__device__ __forceinline__ void mmaCommit(uint32_t bar)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 16 columns of FP32 from tensor memory; no wait (tcgen05.wait::ld before use).
__device__ __forceinline__ void tmemLd16NoWait(uint32_t addr, uint32_t* r)
{
   asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
__device__ __forceinline__ void tmemWaitLd() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 32 lanes x 8 columns of FP32, no wait
__device__ __forceinline__ void tmemLd8NoWait(uint32_t addr, uint32_t* r)
{
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(addr));
}
__device__ __forceinline__ void tmemSt16(uint32_t addr, const uint32_t* r)
{
   asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
      ::"r"(addr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void tmemWaitSt() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

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


// Operand layout of one K chunk of KCW bf16 elements per row: 64 elements in 128-byte rows
// (128-byte swizzle) or 32 elements in 64-byte rows (64-byte swizzle). An A stage holds NP slots of
// 128 rows, a B stage the operator rows of one pipeline item; the numbers of stages are what fits in
// shared memory (three A and two B stages with 64-wide chunks of two pieces at p = 16).
// ES: element bytes; KSTEP: K elements per MMA instruction (32 bytes for both element types).
template <int KCW> struct Layout;
template <> struct Layout<64>
{
   static constexpr int KC = 64, RB = 128, SBO = 1024, SWZ = 2, ES = 2, KSTEP = 16;
   static constexpr bool TF32 = false;
   __host__ __device__ static constexpr uint32_t off(uint32_t row, uint32_t k)
   { return row * 128u + ((((k >> 3) ^ (row & 7u)) & 7u) << 4) + ((k & 7u) << 1); }
};
template <> struct Layout<32>
{
   static constexpr int KC = 32, RB = 64, SBO = 512, SWZ = 4, ES = 2, KSTEP = 16;
   static constexpr bool TF32 = false;
   __host__ __device__ static constexpr uint32_t off(uint32_t row, uint32_t k)
   { return row * 64u + ((((k >> 3) ^ ((row >> 1) & 3u)) & 3u) << 4) + ((k & 7u) << 1); }
};
// tf32 operands: 32 elements of 4 bytes per 128-byte row, 128-byte swizzle
struct LayoutTf32
{
   static constexpr int KC = 32, RB = 128, SBO = 1024, SWZ = 2, ES = 4, KSTEP = 8;
   static constexpr bool TF32 = true;
   __host__ __device__ static constexpr uint32_t off(uint32_t row, uint32_t k)
   { return row * 128u + ((((k >> 2) ^ (row & 7u)) & 7u) << 4) + ((k & 3u) << 2); }
};
constexpr int MAXSTAGE = 6;

// Shared-memory matrix descriptor: K-major, swizzled rows, 8-row groups SBO bytes apart.
template <class Lay>
__device__ __forceinline__ uint64_t smemDescT(uint32_t addr)
{
   uint64_t d = 0;
   d |= uint64_t((addr >> 4) & 0x3FFF);               // start address
   d |= uint64_t(1) << 16;                             // leading byte offset (unused when swizzled)
   d |= uint64_t(Lay::SBO >> 4) << 32;                // stride byte offset
   d |= uint64_t(1) << 46;                             // descriptor version for sm_100
   d |= uint64_t(Lay::SWZ) << 61;                     // swizzle mode
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
template <int NP, class Lay>
__global__ void kPrepM2LImage(const double* __restrict__ op64, int nOps, int L, int N, int nChunks, uint8_t* img)
{
   const int64_t blockBytes = int64_t(N) * Lay::RB;
   const int64_t total = int64_t(nOps) * nChunks * int64_t(N) * Lay::KC;
   for(int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
   {
      int64_t r = e;
      const int kk = int(r % Lay::KC); r /= Lay::KC;
      const int n = int(r % N); r /= N;
      const int c = int(r % nChunks);
      const int o = int(r / nChunks);
      const int k = c * Lay::KC + kk;
      const double x = (n < L && k < L) ? op64[(int64_t(o) * L + n) * L + k] : 0.0;
      uint8_t* blk = img + (int64_t(o) * nChunks + c) * NP * blockBytes;
      if constexpr(Lay::TF32)
         *reinterpret_cast<uint32_t*>(blk + Lay::off(uint32_t(n), uint32_t(kk))) = tc::toTf32(float(x));
      else
      {
         __nv_bfloat16 piece[NP];
         tc::splitBf16<NP>(x, piece);
#pragma unroll
         for(int i = 0; i < NP; i++)
            *reinterpret_cast<__nv_bfloat16*>(blk + i * blockBytes + Lay::off(uint32_t(n), uint32_t(kk))) = piece[i];
      }
   }
}

// The multipoles split into NP bf16 pieces, once per solve: Mbf[node][comp][piece][Lp], each
// piece the round-to-nearest of the remaining FP32 residual (exact: every piece removes the
// leading bits of the remainder).
// Output columns each 16-wide K step of the M2L needs: with the degree cutoff l + lambda <= P, the
// inputs of a K step (degrees >= lambda_min) only reach outputs of degree <= P - lambda_min,
// which are the first (P - lambda_min + 1)^2 columns (rounded up to 16). Step 0 is always full.
// The correction products (hi*lo, lo*hi, and the smaller ones of BF16X6) of a K step reach only the
// outputs of degree <= C - lambda_min (nc, C <= P, rounded up to 16 as well): with box-size scaled
// expansions a term of degrees (l, lambda) scales like q^(l + lambda) (q < 1 with the distance of the
// offset), so far beyond degree C the hi*hi product's 2^-9 relative rounding is below the result's
// accuracy, and those terms need no correction passes.
constexpr int MAXKSTEPS = 64;   // K steps of one row (38 at p = 16 with 8-element TF32 steps)
constexpr int MAXITEMS = 16;    // pipeline items of one offset (K chunks: 10 at p = 16 with 32-wide chunks)
// Pipeline items of one offset: item i carries K chunks first[i] .. first[i] + count[i] - 1. A chunk with
// correction products travels alone, its NP pieces in the stage's NP slots; chunks without any (their
// first, widest K step has none) travel up to NP per stage, chunk first + j's leading piece in slot j.
// The chunks stay in increasing K order, so an accumulation still starts with chunk 0's full-width MMA.
struct M2LCols
{
   int n[MAXKSTEPS];    // output columns of the leading product (hi * hi)
   int nc[MAXKSTEPS];   // output columns of the correction products, <= n
   int first[MAXITEMS];
   int count[MAXITEMS];
   int bOff[MAXITEMS][3];   // byte offsets / 16 of the item's operator slots in its B stage
   int nItems;              // items per offset
};

// Control area after the stages: barriers, the accumulator's address, the abort flag, the offsets present,
// then the per-tile tables (16-bit where they fit, so that a third A stage fits at p = 16)
constexpr int CTRL_HEAD = 256;
constexpr int REC = 24;   // 16-bit fields per item record (ItemRec), 48 bytes
constexpr int CTRL_BYTES = CTRL_HEAD + 2 * 320 + 4 * 64 + 2 * REC * MAXITEMS;

// An item's record in shared memory, read with one vector load per 8 fields: first chunk, chunks, the B
// slots' offsets / 16 [NP], the output columns of every K step of its chunks [NP][K steps per chunk] (0 beyond
// the item's chunks and past the last coefficient), the correction products' columns [K steps per chunk] (0
// unless the item is one chunk).
template <int NP, int KPC>
struct ItemRec
{
   static constexpr int FIRST = 0, COUNT = 1, BOFF = 2, NCOL = 2 + NP, NCOR = 2 + NP + NP * KPC;
   static constexpr int WORDS = (NCOR + KPC + 7) / 8;   // 16-byte words read
   static_assert(WORDS * 8 <= REC, "item record too small");
   int4 q[WORDS];
   __device__ __forceinline__ void load(const int4* tab, int item)
   {
#pragma unroll
      for(int w = 0; w < WORDS; w++) q[w] = tab[(REC / 8) * item + w];
   }
   // field k (a constant once the callers' loops are unrolled)
   __device__ __forceinline__ int operator[](int k) const
   {
      const int4& v4 = q[k >> 3];
      const int w = (k >> 1) & 3;
      const int v = w == 0 ? v4.x : w == 1 ? v4.y : w == 2 ? v4.z : v4.w;
      return (v >> (16 * (k & 1))) & 0xFFFF;
   }
};

template <int NP, bool TF32>
__global__ void kSplitMultipoles(const float* __restrict__ M, int64_t rows, int Lp, uint8_t* __restrict__ Mout)
{
   __nv_bfloat16* Mbf = reinterpret_cast<__nv_bfloat16*>(Mout);
   const int64_t total = rows * Lp;
   for(int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
   {
      const int64_t row = e / Lp;
      const int k = int(e % Lp);
      float r = M[e];
      if constexpr(TF32)
         reinterpret_cast<uint32_t*>(Mout)[e] = tc::toTf32(r);   // one piece
      else
      {
#pragma unroll
         for(int j = 0; j < NP; j++)
         {
            const __nv_bfloat16 b = __float2bfloat16_rn(r);
            Mbf[(row * NP + j) * Lp + k] = b;
            r -= __bfloat162float(b);
         }
      }
   }
}

// First column of the kept tail (keepTail, N > 256): the drains sum the columns that the tensor memory beside the
// accumulator (512 - N) and 32 registers per row hold; the columns after them, the top degrees, accumulate
// through the whole tile. Without a tail: N.
__host__ __device__ constexpr int tailSplit(int keepTail, int N)
{
   return !(keepTail && N > 256) ? N : (((512 - N + 32) & ~15) < 256 ? ((512 - N + 32) & ~15) : 256);
}

// Whether the accumulator is drained after the oi-th of nOff offsets: every dNear offsets, and, when
// dFar differs, every dFar offsets through the first (far) half of the offsets, which ends with a drain.
// Offsets run far first, so the first half holds the small contributions: the tensor core's accumulation
// error grows with the magnitude accumulated, and longer chains there cost little accuracy.
__device__ __forceinline__ bool drainAfter(int oi, int nOff, int dNear, int dFar)
{
   if(oi == nOff - 1) return true;
   if(dFar == dNear) return (oi + 1) % dNear == 0;
   const int half = nOff / 2;
   if(oi < half) return (oi + 1) % dFar == 0 || oi == half - 1;
   return (oi + 1 - half) % dNear == 0;
}

// drainAfter as a running schedule, asked once per offset in order, without divisions (the MMA-issuing
// thread runs it once per offset, on the pipeline's critical path)
struct DrainSchedule
{
   int run = 0, half, nOff, dNear, dFar;
   __device__ DrainSchedule(int n, int dn, int df) : half(dn == df ? -1 : n / 2), nOff(n), dNear(dn), dFar(df) {}
   __device__ __forceinline__ bool after(int oi)
   {
      const int limit = oi < half ? dFar : dNear;
      const bool d = oi == nOff - 1 || oi == half - 1 || run + 1 == limit;
      run = d ? 0 : run + 1;
      return d;
   }
};

// Position in the pipeline kept by increments (no divisions in the loops): the A stage sa and the B stage
// sb with the parities of their current uses, the item c of the current offset and the offset's index oi.
struct PipeCursor
{
   int sa = 0, pha = 0, sb = 0, phb = 0, c = 0, oi = 0;
   __device__ __forceinline__ void next(int NA, int NB, int nPer)
   {
      if(++sa == NA) { sa = 0; pha ^= 1; }
      if(++sb == NB) { sb = 0; phb ^= 1; }
      if(++c == nPer) { c = 0; ++oi; }
   }
};

// 18 warps: five of them share one SM sub-partition's 16K registers, so 96 per thread at most.
// PIECES: the final outputs are also stored as operand pieces (Mout); the M2M's form.
template <int NP, class Lay, bool PIECES = false>
__global__ void __maxnreg__(96)
kM2LTc(const int* __restrict__ targets, int nTargets, const int* __restrict__ vtab, int nOps, int L, int Lp,
       int nChunks, const uint8_t* __restrict__ img, const uint8_t* __restrict__ Mbf, float* __restrict__ Lc,
       int addOut, uint8_t* __restrict__ Mout, int drainEvery, int drainFar, int drainItems, int nStagesA, int nStagesB,
       uint32_t bStage, int drainMode, int keepTail,
       const M2LCols cols, unsigned long long* counters, int* err, uint64_t waitNs, int asyncArrive,
       unsigned long long* prof)
{
   // prof (developer switch): SM cycles per role, summed over CTAs, see TcProf
   const long long tStart = prof ? clock64() : 0;
   using namespace tc;
   constexpr int KCH = Lay::KC;
   constexpr int NPASS = NP == 1 ? 1 : (NP == 2 ? 3 : 6);
   // (A piece, B piece) of every product kept: hi*hi, hi*lo, lo*hi  /  down to 2^-16 with three pieces
   constexpr int PA[6] = {0, 0, 1, 1, 0, 2};
   constexpr int PB[6] = {0, 1, 0, 1, 2, 0};
   constexpr int PA2[3] = {0, 0, 1};
   constexpr int PB2[3] = {0, 1, 0};
   extern __shared__ uint8_t smraw[];
   const int N = Lp;                                   // output columns (<= 320)
   const uint32_t aBytes = ROWS * Lay::RB;             // one A piece
   const uint32_t bBytes = uint32_t(N) * Lay::RB;      // one operator block (all N rows of a piece)
   const uint32_t aStage = NP * aBytes;
   const uint32_t rawAddr = smemAddr(smraw);
   const uint32_t base = (rawAddr + 1023u) & ~1023u;
   uint8_t* sbase = smraw + (base - rawAddr);
   // two rings: NA stages of the gathered multipole pieces (A), NB <= NA stages of operator rows (B)
   const int NA = nStagesA, NB = nStagesB;
   const uint32_t bRing = base + NA * aStage;
   uint8_t* ctrl = sbase + NA * aStage + NB * bStage;
   // full[NA], empty[NA], done, drainFull, drainEmpty, op[NB]: at most 3 MAXSTAGE + 3 = 21 barriers
   uint64_t* bars = reinterpret_cast<uint64_t*>(ctrl);
   uint32_t* tmemBase = reinterpret_cast<uint32_t*>(ctrl + 192);
   volatile int* abortFlag = reinterpret_cast<volatile int*>(ctrl + 196);
   uint32_t* present = reinterpret_cast<uint32_t*>(ctrl + 200); // 10 words: offsets present in the tile
   int* offCount = reinterpret_cast<int*>(ctrl + 240);          // offsets present
   uint16_t* itemOffset = reinterpret_cast<uint16_t*>(ctrl + CTRL_HEAD); // compacted present offsets [316]
   int* tileNode = reinterpret_cast<int*>(ctrl + CTRL_HEAD + 2 * 320);    // the tile's target boxes [TT]
   uint16_t* recTab = reinterpret_cast<uint16_t*>(tileNode + 64);          // item records [MAXITEMS][REC]
   const int4* rec4 = reinterpret_cast<const int4*>(recTab);
   constexpr int KPC = Lay::KC / Lay::KSTEP;                               // K steps per chunk
   using Rec = ItemRec<NP, KPC>;

   const int tid = threadIdx.x;
   const int warp = tid >> 5, lane = tid & 31;
   const int first = blockIdx.x * TT;
   const int nTile = min(TT, nTargets - first);
   const uint32_t fullBar0 = smemAddr(&bars[0]), emptyBar0 = smemAddr(&bars[NA]), doneBar = smemAddr(&bars[2 * NA]);
   const uint32_t drainFull = smemAddr(&bars[2 * NA + 1]), drainEmpty = smemAddr(&bars[2 * NA + 2]);
   const uint32_t opBar0 = smemAddr(&bars[2 * NA + 3]);

   if(tid < 10) present[tid] = 0;
   if(tid < TT) tileNode[tid] = tid < nTile ? targets[first + tid] : -1;
   if(tid == 0)
   {
      for(int i = 0; i < cols.nItems; i++)
      {
         uint16_t* r = recTab + REC * i;
         const int c0 = cols.first[i], m = cols.count[i];
         for(int k = 0; k < REC; k++) r[k] = 0;
         r[Rec::FIRST] = uint16_t(c0);
         r[Rec::COUNT] = uint16_t(m);
         for(int j = 0; j < NP; j++)
         {
            r[Rec::BOFF + j] = uint16_t(cols.bOff[i][j]);
            if(j < m)
               for(int ks = 0; ks < KPC; ks++) r[Rec::NCOL + KPC * j + ks] = uint16_t(cols.n[(c0 + j) * KPC + ks]);
         }
         if(m == 1)
            for(int ks = 0; ks < KPC; ks++) r[Rec::NCOR + ks] = uint16_t(cols.nc[c0 * KPC + ks]);
      }
   }
   if(tid == 0)
   {
      *abortFlag = 0;
      for(int s = 0; s < NA; s++)
      {
         mbarInit(fullBar0 + 8 * s, NPROD);
         mbarInit(emptyBar0 + 8 * s, 1);
      }
      for(int s = 0; s < NB; s++) mbarInit(opBar0 + 8 * s, 1);
      mbarInit(doneBar, 1);
      mbarInit(drainFull, 1);
      mbarInit(drainEmpty, 256);
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
   for(int e = tid; e < TT * nOps; e += NTHREADS)
   {
      const int t = tileNode[e / nOps], o = e % nOps;
      if(t >= 0 && vtab[int64_t(t) * nOps + o] >= 0) atomicOr(&present[o >> 5], 1u << (o & 31));
   }
   fenceBeforeSync();
   __syncthreads();
   fenceAfterSync();
   if(tid == 0)
   {
      // M2L: far offsets first, so the smaller contributions enter the accumulator before the large
      // ones; the 8 child octants of M2M / L2L in order
      int k = 0;
      for(int i = 0; i < nOps; i++)
      {
         const int o = nOps == 316 ? d_m2lFarFirst[i] : i;
         if(present[o >> 5] & (1u << (o & 31))) itemOffset[k++] = uint16_t(o);
      }
      *offCount = k;
      // work accounting: pipeline items and tile-offset pairs
      if(counters)
      {
         atomicAdd(counters, (unsigned long long)(k * cols.nItems));
         atomicAdd(counters + 1, (unsigned long long)k);
      }
   }
   __syncthreads();
   const int nOff = *offCount;
   const int nPer = cols.nItems;                       // items per offset
   const int nItems = nOff * nPer;
   const uint32_t tmem = *tmemBase;
   if(prof && tid == 0)
   {
      atomicAdd(prof + 10, (unsigned long long)(clock64() - tStart));
      atomicAdd(prof + 11, (unsigned long long)nItems);
   }

   if(warp == 0)
   {
      if(lane == 0)
      {
         bool firstMma = true;
         bool tailFirst = true;   // keepTail: the columns >= split accumulate through the whole tile
         // an MMA covers at most 256 columns; a wider K step is split at 256, with keepTail where the kept
         // columns start
         const int split = keepTail ? tailSplit(1, N) : 256;
         int drains = 0;
         long long tw0 = 0, tw1 = 0, tw2 = 0;
         long long tIssue[6] = {0, 0, 0, 0, 0, 0};   // per K chunk: from the stage's arrival to the commit
         const long long tl = prof ? clock64() : 0;
         DrainSchedule sched(nOff, drainEvery, drainFar);
         PipeCursor cur;
         int sinceDrain = 0;
         // item records are read one item ahead: the loads land while the thread waits for the stages
         Rec next;
         next.load(rec4, 0);
         for(int it = 0; it < nItems; it++, cur.next(NA, NB, nPer))
         {
            const Rec rc = next;
            {
               next.load(rec4, cur.c + 1 == nPer ? 0 : cur.c + 1);
            }
            const int m = rc[Rec::COUNT];
            long long t0 = prof ? clock64() : 0;
            if(!mbarWait(fullBar0 + 8 * cur.sa, cur.pha, err, abortFlag, waitNs)) break;
            long long t1 = prof ? clock64() : 0;
            if(!mbarWait(opBar0 + 8 * cur.sb, cur.phb, err, abortFlag, waitNs)) break;
            long long t2 = 0;
            if(prof)
            {
               t2 = clock64();
               tw0 += t1 - t0;
               tw1 += t2 - t1;
            }
            // the producers' cp.async writes (generic proxy), observed through the barrier, before
            // the tensor core reads the stage (async proxy)
            if(asyncArrive) fenceProxyAsync();
            fenceAfterSync();
            const uint32_t aSt = base + cur.sa * aStage, bSt = bRing + cur.sb * bStage;
            // descriptors of the stages; an MMA's operand is the stage's descriptor plus the slot's
            // byte offset / 16 (the start-address field, bits 0-13, holds every shared-memory address)
            const uint64_t dA = smemDescT<Lay>(aSt), dB = smemDescT<Lay>(bSt);
#pragma unroll
            for(int j = 0; j < NP; j++)
            {
               if(j >= m) break;
#pragma unroll
               for(int ks = 0; ks < KPC; ks++)
               {
                  const uint32_t koff = ks * 32;
                  // this K step's output columns in one MMA (<= 256) or two (split at 256 or at the kept
                  // tail); the correction products over the first nCor of them (a chunk alone: j = 0). K steps
                  // past the last coefficient (the last chunk is partly padding) have no columns.
                  const int nCol = rc[Rec::NCOL + KPC * j + ks];
                  if(nCol == 0) break;
                  const int nCor = rc[Rec::NCOR + ks];
#pragma unroll
                  for(int pass = 0; pass < NPASS; pass++)
                  {
                     const int w = pass == 0 ? nCol : nCor;
                     if(w == 0) break;
                     const int nA = min(w, split), nB = w - nA;
                     const uint32_t idA = Lay::TF32 ? instrDescTf32(ROWS, nA) : instrDescBf16(ROWS, nA);
                     const uint32_t idB = Lay::TF32 ? instrDescTf32(ROWS, nB > 0 ? nB : 16) : instrDescBf16(ROWS, nB > 0 ? nB : 16);
                     // piece slots: pa, pb for a chunk alone, slot j (pass 0 only) for a shared stage
                     const int pa = j + (NP == 1 ? 0 : (NP == 2 ? PA2[pass] : PA[pass]));
                     const int pb = j + (NP == 1 ? 0 : (NP == 2 ? PB2[pass] : PB[pass]));
                     const uint64_t da = dA + ((pa * aBytes + koff) >> 4);
                     const uint64_t db = dB + uint64_t(rc[Rec::BOFF + pb]) + (koff >> 4);
                     const uint32_t acc = firstMma ? 0u : 1u;
                     const uint32_t accT = keepTail ? (tailFirst ? 0u : 1u) : acc;
                     if constexpr(Lay::TF32)
                     {
                        mmaTf32(tmem, da, db, idA, acc);
                        if(nB > 0) mmaTf32(tmem + nA, da, db + ((nA * Lay::RB) >> 4), idB, accT);
                     }
                     else
                     {
                        mmaBf16(tmem, da, db, idA, acc);
                        if(nB > 0) mmaBf16(tmem + nA, da, db + ((nA * Lay::RB) >> 4), idB, accT);
                     }
                     firstMma = false;
                     if(nB > 0) tailFirst = false;
                  }
               }
            }
            mmaCommit(emptyBar0 + 8 * cur.sa);
            if(prof && cur.c < 6) tIssue[cur.c] += clock64() - t2;
            // every drainEvery offsets (and after the last) hand the accumulator to the drain warps
            // and start a fresh one: the tensor cores' FP32 accumulation truncates, so long chains
            // of accumulations into one TMEM value drift; the running sum is kept in FP32 instead
            // (drainItems > 0: every drainItems pipeline items instead, for full-width operators only:
            // a fresh accumulation must start with an MMA that writes every column)
            bool drainNow;
            if(drainItems > 0)
            {
               drainNow = ++sinceDrain == drainItems || it == nItems - 1;
               if(drainNow) sinceDrain = 0;
            }
            else
               drainNow = cur.c == nPer - 1 && sched.after(cur.oi);
            {
               if(drainNow)
               {
                  mmaCommit(drainFull);
                  if(it != nItems - 1)
                  {
                     const long long t3 = prof ? clock64() : 0;
                     if(!mbarWait(drainEmpty, drains & 1, err, abortFlag, waitNs)) break;
                     if(prof) tw2 += clock64() - t3;
                     fenceAfterSync();
                  }
                  drains++;
                  firstMma = true;
               }
            }
         }
         mmaCommit(doneBar);
         if(prof)
         {
            atomicAdd(prof + 0, (unsigned long long)tw0);
            atomicAdd(prof + 1, (unsigned long long)tw1);
            atomicAdd(prof + 2, (unsigned long long)tw2);
            atomicAdd(prof + 3, (unsigned long long)(clock64() - tl));
            for(int c = 0; c < 6; c++) atomicAdd(prof + 16 + c, (unsigned long long)tIssue[c]);
         }
      }
      __syncwarp();
   }
   else if(warp == 1)
   {
      if(lane == 0)
      {
         int issued = 0;
         long long twe = 0;
         PipeCursor cur;
         for(int it = 0; it < nItems; it++, cur.next(NA, NB, nPer))
         {
            const int s = cur.sb;
            const long long t0 = prof ? clock64() : 0;
            // the B stage's previous use, item it - NB, must have been consumed: its MMAs completed when
            // the empty barrier of its A stage completed its use (it - NB) / NA. (That barrier cannot
            // complete a later use first: item it - NB + NA >= it needs this item's operator rows.)
            if(it >= NB)
            {
               const int prev = it - NB;
               if(!mbarWait(emptyBar0 + 8 * (prev % NA), (prev / NA) & 1, err, abortFlag, waitNs)) break;
            }
            if(prof) twe += clock64() - t0;
            const int o = itemOffset[cur.oi];
            Rec rc;
            rc.load(rec4, cur.c);
            const int c0 = rc[Rec::FIRST], m = rc[Rec::COUNT];
            const uint32_t dst = bRing + s * bStage;
            // only the operator rows (output columns) a chunk's widest K step uses: of the leading
            // piece for the hi * hi product, of the others for the correction products. A chunk alone
            // fills the slots with its pieces, chunks sharing the stage their leading pieces.
            uint32_t bytes[NP];
            uint32_t tx = 0;
#pragma unroll
            for(int j = 0; j < NP; j++)
            {
               bytes[j] = m == 1 ? uint32_t(j == 0 ? rc[Rec::NCOL] : rc[Rec::NCOR]) * Lay::RB
                                 : uint32_t(rc[Rec::NCOL + KPC * j]) * Lay::RB;   // (0 for j >= m)
               tx += bytes[j];
            }
            mbarArriveExpectTx(opBar0 + 8 * s, tx);
#pragma unroll
            for(int j = 0; j < NP; j++)
            {
               const uint8_t* src = m == 1 ? img + ((int64_t(o) * nChunks + c0) * NP + j) * bBytes
                                           : img + (int64_t(o) * nChunks + c0 + j) * NP * bBytes;
               if(bytes[j]) bulkLoad(dst + 16u * uint32_t(rc[Rec::BOFF + j]), src, bytes[j], opBar0 + 8 * s);
            }
            issued = it + 1;
         }
         // the copies in flight write this CTA's shared memory: wait for them before it can exit. A stage
         // is reused only after the MMAs consumed its previous item, which waited for that item's copy, so
         // only the last item issued on each stage can still be in flight.
         for(int s = 0; s < NB && s < issued; s++)
         {
            const int last = s + ((issued - 1 - s) / NB) * NB;
            mbarWaitIssued(opBar0 + 8 * s, (last / NB) & 1, err);
         }
         if(prof) atomicAdd(prof + 4, (unsigned long long)twe);
      }
      __syncwarp();
   }
   else if(warp >= 10)
   {
      // drain warps 10..17: warp w reads TMEM lanes 32 (w % 4) .. + 31 (one accumulator row per
      // thread) and half of the columns of every part below (warps 10-13 the first half)
      const int lanes = 32 * (warp & 3);
      const int half = (warp - 10) >> 2;
      const int r = lanes + lane;
      const int et = r < 3 * TT ? tileNode[r / 3] : -1, ec = r % 3;
      float* out = Lc + (int64_t(et) * 3 + ec) * Lp;
      const uint32_t tAcc = tmem + (uint32_t(lanes) << 16);
      int nDrains = 0;
      if(drainItems > 0) nDrains = (nItems + drainItems - 1) / drainItems;
      else
         for(int oi = 0; oi < nOff; oi++) nDrains += drainAfter(oi, nOff, drainEvery, drainFar) ? 1 : 0;
      // The running sum is FP32, rounded to nearest, and has one writer per row and column (this
      // thread); the locals start at zero and no other CTA touches these rows, so the result is
      // deterministic. Its columns live in three parts:
      //   [0, nS)    in the tensor memory the accumulator leaves free (columns N .. 511), drainMode >= 2
      //   [nS, nR)   in this thread's registers (RHALF columns per half), drainMode 3
      //   [nR, nT)   in the local expansions: fire-and-forget vector atomics (drainMode 0) or
      //              load-add-store, the first drain storing (drainMode >= 1)
      // With keepTail the columns [nT, N) (the top degrees, whose terms are the smallest; the columns the
      // tensor memory and the registers cannot hold) are not drained: their accumulation runs through the
      // whole tile in tensor memory and the last drain writes it.
      constexpr int RHALF = 16;
      const int nT = tailSplit(keepTail, N);
      const int nS = drainMode >= 2 ? (min(nT, 512 - N) & ~15) : 0;
      const int nR = drainMode == 3 ? min(nT, nS + 2 * RHALF) : nS;
      // [a, b) split at a multiple of 16 columns; this warp's half
      auto split = [&](int a, int b, int& lo, int& hi) {
         const int mid = min(b, a + ((((b - a) >> 1) + 15) & ~15));
         lo = half ? mid : a;
         hi = half ? b : mid;
      };
      int sLo, sHi, gLo, gHi;
      split(0, nS, sLo, sHi);
      const int rLo = nS + half * RHALF;
      const int rHi = min(nR, rLo + RHALF);
      split(nR, nT, gLo, gHi);
      const uint32_t tSum = tAcc + uint32_t(N);
      float rsum[RHALF];
#pragma unroll
      for(int i = 0; i < RHALF; i++) rsum[i] = 0.f;
      long long twd = 0;
      const long long tdl = prof ? clock64() : 0;
      for(int d = 0; d < nDrains; d++)
      {
         const long long t0 = prof ? clock64() : 0;
         if(!mbarWait(drainFull, d & 1, err, abortFlag, waitNs)) break;
         if(prof) twd += clock64() - t0;
         fenceAfterSync();
         const bool last = d == nDrains - 1;
         // tensor-memory part: S += acc (d > 0) or S = acc; the last drain writes S + acc to the locals
         for(int c0 = sLo; c0 < sHi; c0 += 16)
         {
            uint32_t a[16], sv[16];
            tmemLd16NoWait(tAcc + uint32_t(c0), a);
            if(d > 0) tmemLd16NoWait(tSum + uint32_t(c0), sv);
            tmemWaitLd();
#pragma unroll
            for(int i = 0; i < 16; i++)
               sv[i] = d > 0 ? __float_as_uint(__uint_as_float(sv[i]) + __uint_as_float(a[i])) : a[i];
            if(last)
            {
               if(et >= 0)
               {
                  float4* o4 = reinterpret_cast<float4*>(out + c0);
#pragma unroll
                  for(int i = 0; i < 4; i++)
                  {
                     float4 v = make_float4(__uint_as_float(sv[4 * i]), __uint_as_float(sv[4 * i + 1]),
                                            __uint_as_float(sv[4 * i + 2]), __uint_as_float(sv[4 * i + 3]));
                     if(addOut)
                     {
                        const float4 w = o4[i];
                        v = make_float4(w.x + v.x, w.y + v.y, w.z + v.z, w.w + v.w);
                     }
                     o4[i] = v;
                     if(PIECES) storePieces4(Mout, int64_t(et) * 3 + ec, c0 + 4 * i, Lp, Lay::TF32 ? 1 : NP, v);
                  }
               }
            }
            else
               tmemSt16(tSum + uint32_t(c0), sv);
         }
         if(sHi > sLo && !last) tmemWaitSt();
         // register part
#pragma unroll
         for(int j = 0; j < RHALF / 16; j++)
         {
            const int c0 = rLo + 16 * j;
            if(c0 >= rHi) break;
            uint32_t a[16];
            tmemLd16NoWait(tAcc + uint32_t(c0), a);
            tmemWaitLd();
#pragma unroll
            for(int i = 0; i < 16; i++) rsum[16 * j + i] = (d > 0 ? rsum[16 * j + i] : 0.f) + __uint_as_float(a[i]);
            if(last && et >= 0)
            {
               float4* o4 = reinterpret_cast<float4*>(out + c0);
#pragma unroll
               for(int i = 0; i < 4; i++)
               {
                  float4 v = make_float4(rsum[16 * j + 4 * i], rsum[16 * j + 4 * i + 1], rsum[16 * j + 4 * i + 2],
                                         rsum[16 * j + 4 * i + 3]);
                  if(addOut)
                  {
                     const float4 w = o4[i];
                     v = make_float4(w.x + v.x, w.y + v.y, w.z + v.z, w.w + v.w);
                  }
                  o4[i] = v;
                  if(PIECES) storePieces4(Mout, int64_t(et) * 3 + ec, c0 + 4 * i, Lp, Lay::TF32 ? 1 : NP, v);
               }
            }
         }
         // global part, 16 columns per step (with addOut the first drain adds to the values already there
         // as well); the running sums load while the accumulator does. The last drain also writes the
         // kept columns [nT, N) the same way: their accumulator, plus the values there with addOut.
         int tLo = 0, tHi = 0;
         if(last) split(nT, N, tLo, tHi);
         for(int part = 0; part < 2; part++)
         {
            const int lo = part ? tLo : gLo, hi = part ? tHi : gHi;
            const bool rmw = drainMode != 0 && (part ? addOut != 0 : (d > 0 || addOut)) && et >= 0;
            for(int c0 = lo; c0 < hi; c0 += 16)
            {
               uint32_t u[16];
               float4 old[4];
               float4* o4 = reinterpret_cast<float4*>(out + c0);
               tmemLd16NoWait(tAcc + uint32_t(c0), u);
               if(rmw)
               {
#pragma unroll
                  for(int i = 0; i < 4; i++) old[i] = o4[i];
               }
               tmemWaitLd();
               if(et < 0) continue;
#pragma unroll
               for(int i = 0; i < 4; i++)
               {
                  const float4 v = make_float4(__uint_as_float(u[4 * i]), __uint_as_float(u[4 * i + 1]),
                                               __uint_as_float(u[4 * i + 2]), __uint_as_float(u[4 * i + 3]));
                  if(drainMode == 0) atomicAdd(o4 + i, v);
                  else
                  {
                     const float4 f = rmw ? make_float4(old[i].x + v.x, old[i].y + v.y, old[i].z + v.z, old[i].w + v.w) : v;
                     o4[i] = f;
                     // (Mout is only given with drainMode != 0: atomics leave the final value unknown here)
                     if(PIECES && last) storePieces4(Mout, int64_t(et) * 3 + ec, c0 + 4 * i, Lp, Lay::TF32 ? 1 : NP, f);
                  }
               }
            }
         }
         fenceBeforeSync();
         mbarArrive(drainEmpty);
      }
      if(prof && warp == 10 && lane == 0)
      {
         atomicAdd(prof + 23, (unsigned long long)nDrains);
         atomicAdd(prof + 7, (unsigned long long)twd);
         atomicAdd(prof + 8, (unsigned long long)(clock64() - tdl));
      }
   }
   else
   {
      // producers (warps 2..9): two threads per row, KCH / 2 K-elements (KCH / 8 chunks of 16 bytes)
      // of every piece each. Item it - 1 is signalled as soon as its copies have landed, then the
      // copies of item it are issued once its stage is free: one item's gather is in flight while
      // the tensor cores work on the previous one, and issuing never delays a signal.
      constexpr int PER = KCH / 2;                   // K elements per thread and chunk
      constexpr int EPC = 16 / Lay::ES;              // elements per 16-byte copy
      const int ptid = tid - 64;
      const int row = ptid >> 1, half = ptid & 1;
      const int slot = row / 3, comp = row % 3;
      const int tgt = row < 3 * TT ? tileNode[slot] : -1;
      int src = (tgt >= 0 && nItems > 0) ? vtab[int64_t(tgt) * nOps + itemOffset[0]] : -1;
      int srcNext = -1;
      int pending = -1;   // stage of the item whose copies are still to be signalled (synchronous form)
      long long twp = 0;
      const long long tpl = prof ? clock64() : 0;
      PipeCursor cur;
      for(int it = 0; it < nItems; it++, cur.next(NA, NB, nPer))
      {
         const int s = cur.sa;
         const int oi = cur.oi, c = cur.c;
         if(c == 0 && oi + 1 < nOff)
            srcNext = tgt >= 0 ? vtab[int64_t(tgt) * nOps + itemOffset[oi + 1]] : -1;
         if(pending >= 0)
         {
            // (synchronous form: this thread waits for its previous item's copies, then arrives)
            cpAsyncWaitAll();
            fenceProxyAsync();
            mbarArrive(fullBar0 + 8 * pending);
            pending = -1;
         }
         const long long t0 = prof ? clock64() : 0;
         if(it >= NA && !mbarWait(emptyBar0 + 8 * s, cur.pha ^ 1, err, abortFlag, waitNs)) break;
         if(prof) twp += clock64() - t0;
         const uint32_t aSt = base + s * aStage;
         Rec rc;
         rc.load(rec4, c);
         const int c0 = rc[Rec::FIRST], m = rc[Rec::COUNT];
         const uint8_t* rowp = Mbf + ((int64_t(src >= 0 ? src : 0) * 3 + comp) * NP) * Lp * Lay::ES;
         // a chunk alone: its pieces into the slots, the ones after the leading piece only when its first
         // (widest) K step has correction products; chunks sharing the stage: chunk c0 + j's leading
         // piece into slot j
         const int nSlots = m == 1 ? (rc[Rec::NCOR] > 0 ? NP : 1) : m;
#pragma unroll
         for(int q = 0; q < PER / EPC; q++)
         {
            const uint32_t off = Lay::off(uint32_t(row), uint32_t(half * PER + EPC * q));
#pragma unroll
            for(int j = 0; j < NP; j++)
            {
               if(j >= nSlots) break;
               const int k = (m == 1 ? c0 : c0 + j) * KCH + half * PER + EPC * q;
               const int piece = m == 1 ? j : 0;
               const uint32_t bytes = (src >= 0 && k < Lp) ? 16u : 0u;
               cpAsync16(aSt + j * aBytes + off, rowp + (int64_t(piece) * Lp + (bytes ? k : 0)) * Lay::ES, bytes);
            }
         }
         if(asyncArrive)
            // the barrier completes when every producer's copies of this item have landed, while the
            // thread goes on with the next free stage: up to NA items in flight
            cpAsyncArriveNoinc(fullBar0 + 8 * s);
         else
         {
            cpAsyncCommit();
            pending = s;
         }
         if(c == nPer - 1) src = srcNext;
      }
      cpAsyncWaitAll();
      if(pending >= 0 && !*abortFlag)
      {
         fenceProxyAsync();
         mbarArrive(fullBar0 + 8 * pending);
      }
      if(prof && tid == 64)
      {
         atomicAdd(prof + 5, (unsigned long long)twp);
         atomicAdd(prof + 6, (unsigned long long)(clock64() - tpl));
      }
   }
   fenceBeforeSync();
   __syncthreads();
   if(warp == 0)
   {
      // the accumulator must be idle before it is released, also after an aborted pipeline: the
      // commit to doneBar arrives once every MMA issued before it has completed
      if(lane == 0 && nItems > 0) mbarWaitIssued(doneBar, 0, err);
      __syncwarp();
      fenceAfterSync();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
   }
   if(prof && tid == 0) atomicAdd(prof + 9, (unsigned long long)(clock64() - tStart));
}

// The pipeline items of one offset (M2LCols): a K chunk with correction products travels alone; with
// share, runs of chunks without any travel up to NP per stage.
static fmm_status planItems(M2LCols& cols, int nChunks, int stepsPerChunk, int NP, bool share)
{
   if(nChunks > MAXITEMS) return setError(FMM_E_INVALID, "tensor-core pipeline: %d K chunks exceed the item table", nChunks);
   auto hiOnly = [&](int c) {
      for(int ks = 0; ks < stepsPerChunk; ks++)
         if(cols.nc[c * stepsPerChunk + ks] > 0) return false;
      return true;
   };
   int n = 0;
   for(int c = 0; c < nChunks;)
   {
      int m = 1;
      if(share && hiOnly(c))
         while(m < NP && c + m < nChunks && hiOnly(c + m)) m++;
      cols.first[n] = c;
      cols.count[n] = m;
      n++;
      c += m;
   }
   cols.nItems = n;
   return FMM_OK;
}

// The operator slots of every item in its B stage (M2LCols::bOff), the B stage size, and the stage counts of
// the two rings within the shared memory: two B stages (more while A stages outnumber them) and as many A
// stages as the rest holds.
struct StagePlan
{
   int na, nb;
   uint32_t bStage;
   size_t smem;
};
static constexpr size_t SMEM_BUDGET = 232448;   // the opt-in dynamic shared memory of one block

static fmm_status planStages(M2LCols& cols, int NP, int stepsPerChunk, int rowBytes, const char* what, StagePlan& sp)
{
   uint32_t bStage = 1024;
   for(int i = 0; i < cols.nItems; i++)
   {
      const int c0 = cols.first[i], m = cols.count[i];
      uint32_t off = 0;
      for(int j = 0; j < 3; j++) cols.bOff[i][j] = 0;
      for(int j = 0; j < NP; j++)
      {
         cols.bOff[i][j] = int(off / 16);
         int rows = 0;
         if(m == 1) rows = j == 0 ? cols.n[c0 * stepsPerChunk] : cols.nc[c0 * stepsPerChunk];
         else if(j < m) rows = cols.n[(c0 + j) * stepsPerChunk];
         off += uint32_t(rows) * uint32_t(rowBytes);
      }
      bStage = std::max(bStage, off);
   }
   bStage = (bStage + 1023u) & ~1023u;
   const size_t aStage = size_t(NP) * tc::ROWS * rowBytes;
   const size_t fixed = 1024 + CTRL_BYTES;
   if(fixed + 2 * (aStage + bStage) > SMEM_BUDGET)
      return setError(FMM_E_INVALID, "%s: stages of %zu + %u bytes do not fit twice", what, aStage, bStage);
   int nb = 2;
   const int na = int(std::min<size_t>(tc::MAXSTAGE, (SMEM_BUDGET - fixed - nb * size_t(bStage)) / aStage));
   while(nb < na && fixed + na * aStage + (nb + 1) * size_t(bStage) <= SMEM_BUDGET) nb++;
   sp = {na, nb, bStage, fixed + na * aStage + nb * size_t(bStage)};
   return FMM_OK;
}

template <int NP, class Lay>
static fmm_status launchM2LTc(Plan& P, cudaStream_t st)
{
   const int L = P.L, Lp = P.Lp;
   const int nChunks = (L + Lay::KC - 1) / Lay::KC;
   const size_t imgBytes = size_t(316) * nChunks * NP * size_t(Lp) * Lay::RB;
   const int tag = ((P.p * 8 + NP) * 128 + Lay::KC) * 2 + (Lay::TF32 ? 1 : 0);
   if(P.opImgOrder != tag)
   {
      FMM_TRY(P.opM2Lbf.reserve(imgBytes));
      kPrepM2LImage<NP, Lay><<<4096, 256, 0, st>>>((const double*)P.opM2L64.ptr, 316, L, Lp, nChunks,
                                                   (uint8_t*)P.opM2Lbf.ptr);
      FMM_TRY(launched(P, "kPrepM2LImage", st));
      P.opImgOrder = tag;
   }
   const int count = P.nM2LTargets;
   if(count <= 0) return FMM_OK;
   const int blocks = (count + tc::TT - 1) / tc::TT;
   FMM_TRY(P.tcCounters.reserve(2 * sizeof(unsigned long long)));
   FMM_CUDA(cudaMemsetAsync(P.tcCounters.ptr, 0, 2 * sizeof(unsigned long long), st));
   P.tcTiles = blocks;
   // the degree cutoff: 0 -> p + 8, negative -> none (l + lambda <= 2p, the full operator)
   const int cut = P.cfg.m2l_tc_degree_cutoff == 0 ? P.p + 8 : (P.cfg.m2l_tc_degree_cutoff < 0 ? 2 * P.p
                                                                : std::max(P.cfg.m2l_tc_degree_cutoff, P.p));
   // correction products: by default for l + lambda <= 10 and lambda <= 5. The size of the terms they correct
   // falls with l + lambda whatever p is (box-size scaled bases). At p = 16 (2^24 torus) the corrections of all
   // terms give rel-L2 7.61e-7 in 245 ms of M2L, these 7.44e-7 in 162 ms: fewer accumulations into the tensor
   // core's truncating FP32 accumulator outweigh the tiny terms they corrected.
   const int corrSet = P.tcCorrCut == -2 ? 10 : P.tcCorrCut;
   const int corr = corrSet < 0 ? -1 : std::min(cut, corrSet);
   M2LCols cols{};
   if(nChunks * (Lay::KC / Lay::KSTEP) > MAXKSTEPS)
      return setError(FMM_E_INVALID, "tensor-core M2L: %d K steps exceed the column table", nChunks * (Lay::KC / Lay::KSTEP));
   for(int g = 0; g < nChunks * (Lay::KC / Lay::KSTEP); g++)
   {
      const int k = Lay::KSTEP * g;
      int lmin = 0;
      while((lmin + 1) * (lmin + 1) <= k) lmin++;
      int n = cut - lmin >= 0 ? std::min(L, (cut - lmin + 1) * (cut - lmin + 1)) : 0;
      n = std::min(Lp, (n + 15) / 16 * 16);
      cols.n[g] = k < L ? n : 0;
      // correction products: up to degree corr - lambda_min (corr < 0: as the leading product), and only for
      // K steps whose lowest input degree is at most P.tcCorrLam (when >= 0)
      int nc = corr - lmin >= 0 ? std::min(L, (corr - lmin + 1) * (corr - lmin + 1)) : 0;
      if(P.tcCorrLam >= 0 && lmin > P.tcCorrLam) nc = 0;
      nc = std::min(Lp, (nc + 15) / 16 * 16);
      cols.nc[g] = corr < 0 ? cols.n[g] : std::min(cols.n[g], nc);
   }
   FMM_TRY(planItems(cols, nChunks, Lay::KC / Lay::KSTEP, NP, P.tcPair != 0));
   StagePlan sp;
   FMM_TRY(planStages(cols, NP, Lay::KC / Lay::KSTEP, Lay::RB, "tensor-core M2L", sp));
   // (the attribute is the budget, not this launch's size: the translations share the kernel and a graph
   // replays every launch with its own size)
   FMM_CUDA(cudaFuncSetAttribute(kM2LTc<NP, Lay>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_BUDGET)));
   const int64_t rows = P.tree.nNodes * 3;
   // developer switch FMM_TC_PROF=1: per-role SM cycles of this launch, printed to stderr
   unsigned long long* prof = nullptr;
   if(P.tcProf)
   {
      FMM_TRY(P.tcProfBuf.reserve(24 * sizeof(unsigned long long)));
      prof = (unsigned long long*)P.tcProfBuf.ptr;
      FMM_CUDA(cudaMemsetAsync(prof, 0, 24 * sizeof(unsigned long long), st));
   }
   // the tensor-core M2M leaves every source level's multipoles split in this format
   if(P.multBfTag != NP * 2 + (Lay::TF32 ? 1 : 0))
   {
      FMM_TRY(P.multBf.reserve(size_t(Lay::ES) * rows * NP * Lp));
      kSplitMultipoles<NP, Lay::TF32><<<148 * 16, 256, 0, st>>>((const float*)P.mult.ptr, rows, Lp, (uint8_t*)P.multBf.ptr);
      FMM_TRY(launched(P, "kSplitMultipoles", st));
   }
   kM2LTc<NP, Lay><<<blocks, tc::NTHREADS, sp.smem, st>>>((const int*)P.m2lTargets.ptr, count, P.lists.vtab, 316, L, Lp,
                                                      nChunks, (const uint8_t*)P.opM2Lbf.ptr, (const uint8_t*)P.multBf.ptr,
                                                      (float*)P.local.ptr, 0, nullptr, (NP == 2 ? P.tcDrainEvery : std::max(1, P.tcDrainEvery / 2)),
                                                      (NP == 2 ? P.tcDrainFar : std::max(1, P.tcDrainFar / 2)), 0, sp.na, sp.nb, sp.bStage, P.tcDrainMode, P.tcKeepTail, cols, (unsigned long long*)P.tcCounters.ptr, P.pipeErr, P.tcWaitNs, P.tcAsyncArrive,
                                                      prof);
   FMM_TRY(launched(P, "kM2LTc", st));
   if(prof)
   {
      unsigned long long h[24];
      FMM_CUDA(cudaMemcpyAsync(h, prof, sizeof(h), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      const double b = double(blocks), it = double(h[11]) / b;
      fprintf(stderr,
              "kM2LTc profile, SM cycles per CTA (%d CTAs, %.0f items each): total %.0f, prologue %.0f | MMA thread: "
              "loop %.0f, wait producers %.0f, wait operator %.0f, wait drain %.0f | operator thread: wait stage %.0f "
              "| producer: loop %.0f, wait stage %.0f | drain: loop %.0f, wait accumulator %.0f\n",
              blocks, it, h[9] / b, h[10] / b, h[3] / b, h[0] / b, h[1] / b, h[2] / b, h[4] / b, h[6] / b, h[5] / b,
              h[8] / b, h[7] / b);
      fprintf(stderr, "kM2LTc profile, drains per CTA %.1f\n", double(h[23]) / b);
      fprintf(stderr, "kM2LTc profile, MMA thread cycles per item from the stage's arrival to its commit, by item:");
      for(int c = 0; c < std::min(cols.nItems, 6); c++) fprintf(stderr, " %.0f", h[16 + c] * double(cols.nItems) / double(h[11]));
      fprintf(stderr, "\n");
   }
   // a timed-out wait raises the pipeline error word, which the calling phase reads once at its end
   return FMM_OK;
}

// M2M and L2L on the same kernel, one launch per level, with the 8 child-octant operators in place
// of the 316 offsets. M2M: the targets are the level's parents, vtabUp gives each parent's child
// with sources per octant, the children's multipoles are split into pieces first (so after the
// upward pass every level >= 1 is split and the M2L reuses it), and the parents' multipoles are
// stored. L2L: the targets are the next level's nodes with targets sorted by octant (one operator
// per tile), vtabDn gives each one's parent, the parents' locals are split first, and the result
// is added to the children's locals (addOut). Full output width: the triangular structure (M2M
// outputs of degree l take inputs of degree <= l, L2L the reverse) is not a prefix of the columns.
template <int NP, class Lay>
static fmm_status translateTc(Plan& P, cudaStream_t st, bool up)
{
   const int L = P.L, Lp = P.Lp;
   const int nChunks = (L + Lay::KC - 1) / Lay::KC;
   const int tag = ((P.p * 8 + NP) * 128 + Lay::KC) * 2 + (Lay::TF32 ? 1 : 0);
   const size_t imgBytes = size_t(8) * nChunks * NP * size_t(Lp) * Lay::RB;
   if(P.opTrImgTag != tag)
   {
      FMM_TRY(P.opM2Mbf.reserve(imgBytes));
      FMM_TRY(P.opL2Lbf.reserve(imgBytes));
      kPrepM2LImage<NP, Lay><<<1024, 256, 0, st>>>((const double*)P.opM2M64.ptr, 8, L, Lp, nChunks,
                                                   (uint8_t*)P.opM2Mbf.ptr);
      FMM_TRY(launched(P, "kPrepM2LImage", st));
      kPrepM2LImage<NP, Lay><<<1024, 256, 0, st>>>((const double*)P.opL2L64.ptr, 8, L, Lp, nChunks,
                                                   (uint8_t*)P.opL2Lbf.ptr);
      FMM_TRY(launched(P, "kPrepM2LImage", st));
      P.opTrImgTag = tag;
   }
   M2LCols cols{};
   const int nSteps = nChunks * (Lay::KC / Lay::KSTEP);
   if(nSteps > MAXKSTEPS) return setError(FMM_E_INVALID, "tensor-core translation: %d K steps exceed the column table", nSteps);
   for(int g = 0; g < nSteps; g++) cols.n[g] = cols.nc[g] = Lay::KSTEP * g < L ? Lp : 0;
   // every chunk alone in its stage: the drains every drainItems items need full-width chunks
   FMM_TRY(planItems(cols, nChunks, Lay::KC / Lay::KSTEP, NP, false));
   StagePlan sp;
   FMM_TRY(planStages(cols, NP, Lay::KC / Lay::KSTEP, Lay::RB, "tensor-core translation", sp));
   const size_t smem = sp.smem;
   FMM_CUDA(cudaFuncSetAttribute(kM2LTc<NP, Lay>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_BUDGET)));
   FMM_CUDA(cudaFuncSetAttribute(kM2LTc<NP, Lay, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_BUDGET)));
   const int64_t rows = P.tree.nNodes * 3;
   FMM_TRY(P.multBf.reserve(size_t(Lay::ES) * rows * NP * Lp));
   const int drainEvery = NP == 2 ? P.tcDrainEvery : std::max(1, P.tcDrainEvery / 2);
   const size_t pieceRow = size_t(Lay::ES) * NP * Lp;   // bytes of one split row
   const Tree& t = P.tree;
   auto split = [&](const float* src, int lvl) -> fmm_status {
      const int64_t r0 = int64_t(t.levelStart[lvl]) * 3, r1 = int64_t(t.levelStart[lvl + 1]) * 3;
      if(r1 <= r0) return FMM_OK;
      kSplitMultipoles<NP, Lay::TF32><<<std::min<int64_t>(148 * 16, (r1 - r0) * Lp / 256 + 1), 256, 0, st>>>(
         src + r0 * Lp, r1 - r0, Lp, (uint8_t*)P.multBf.ptr + r0 * pieceRow);
      return launched(P, "kSplitMultipoles", st);
   };
   if(up)
   {
      // the warp P2M already wrote the leaves in this piece format: then every parent's pieces come out
      // of its M2M launch (Mout) and no level is split separately
      const int tag = NP * 2 + (Lay::TF32 ? 1 : 0);
      const bool fused = P.p2mPiecesTag == tag && P.tcDrainMode != 0;
      for(int level = t.nLevels - 2; level >= 0; level--)
      {
         const int a = P.parStart[level], b = P.parStart[level + 1];
         if(b <= a) continue;
         if(!fused) FMM_TRY(split((const float*)P.mult.ptr, level + 1));
         auto kern = fused ? kM2LTc<NP, Lay, true> : kM2LTc<NP, Lay, false>;
         kern<<<(b - a + tc::TT - 1) / tc::TT, tc::NTHREADS, smem, st>>>(
            (const int*)P.parList.ptr + a, b - a, (const int*)P.vtabUp.ptr, 8, L, Lp, nChunks,
            (const uint8_t*)P.opM2Mbf.ptr, (const uint8_t*)P.multBf.ptr, (float*)P.mult.ptr, 0,
            (uint8_t*)P.multBf.ptr, drainEvery, drainEvery, P.tcTrDrainItems, sp.na, sp.nb, sp.bStage, P.tcDrainMode, 0, cols, nullptr, P.pipeErr, P.tcWaitNs, P.tcAsyncArrive, nullptr);
         FMM_TRY(launched(P, "kM2LTc<M2M>", st));
      }
      P.multBfTag = NP * 2 + (Lay::TF32 ? 1 : 0);
   }
   else
   {
      for(int level = 0; level + 1 < t.nLevels; level++)
      {
         const int a = P.l2lStart[8 * (level + 1)], b = P.l2lStart[8 * (level + 2)];
         if(b <= a) continue;
         FMM_TRY(split((const float*)P.local.ptr, level));
         kM2LTc<NP, Lay><<<(b - a + tc::TT - 1) / tc::TT, tc::NTHREADS, smem, st>>>(
            (const int*)P.l2lTargets.ptr + a, b - a, (const int*)P.vtabDn.ptr, 8, L, Lp, nChunks,
            (const uint8_t*)P.opL2Lbf.ptr, (const uint8_t*)P.multBf.ptr, (float*)P.local.ptr, 1, nullptr, drainEvery, drainEvery,
            P.tcTrDrainItems, sp.na, sp.nb, sp.bStage,
            P.tcDrainMode, 0, cols, nullptr, P.pipeErr, P.tcWaitNs, P.tcAsyncArrive, nullptr);
         FMM_TRY(launched(P, "kM2LTc<L2L>", st));
      }
      P.multBfTag = -1;
   }
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

static fmm_status translateTensorCore(Plan& P, cudaStream_t st, bool up)
{
   if(P.Lp > 320 || P.Lp % 16) return setError(FMM_E_INVALID, "tensor-core translation supports p <= 16");
   using tc::Layout;
   // pieces: 0 follows the M2L mode; 3 is BF16X6, whose products carry the full FP32 significand
   const int np = up ? P.tcTrPiecesUp : P.tcTrPiecesDn;
   if(np == 3) return P.tcKChunk == 64 ? translateTc<3, Layout<64>>(P, st, up) : translateTc<3, Layout<32>>(P, st, up);
   if(np == 2) return P.tcKChunk == 32 ? translateTc<2, Layout<32>>(P, st, up) : translateTc<2, Layout<64>>(P, st, up);
   if(P.cfg.m2l_mode == FMM_M2L_BF16X3)
      return P.tcKChunk == 32 ? translateTc<2, Layout<32>>(P, st, up) : translateTc<2, Layout<64>>(P, st, up);
   if(P.cfg.m2l_mode == FMM_M2L_BF16X6)
      return P.tcKChunk == 64 ? translateTc<3, Layout<64>>(P, st, up) : translateTc<3, Layout<32>>(P, st, up);
   return translateTc<1, tc::LayoutTf32>(P, st, up);
}

int m2mPieces(const Plan& P)
{
   if(P.tcTrPiecesUp == 2 || P.tcTrPiecesUp == 3) return P.tcTrPiecesUp;
   if(P.cfg.m2l_mode == FMM_M2L_BF16X3) return 2;
   if(P.cfg.m2l_mode == FMM_M2L_BF16X6) return 3;
   return 1;
}

fmm_status m2mTensorCore(Plan& P, cudaStream_t st) { return translateTensorCore(P, st, true); }
fmm_status l2lTensorCore(Plan& P, cudaStream_t st) { return translateTensorCore(P, st, false); }

fmm_status m2lTensorCore(Plan& P, cudaStream_t st)
{
   if(P.Lp > 320) return setError(FMM_E_INVALID, "tensor-core M2L supports p <= 16");
   if(P.Lp % 16) return setError(FMM_E_INVALID, "tensor-core M2L needs 16-aligned coefficient rows");
   using tc::Layout;
   if(P.cfg.m2l_mode == FMM_M2L_BF16X3)
      return P.tcKChunk == 32 ? launchM2LTc<2, Layout<32>>(P, st) : launchM2LTc<2, Layout<64>>(P, st);
   if(P.cfg.m2l_mode == FMM_M2L_BF16X6)
      return P.tcKChunk == 64 ? launchM2LTc<3, Layout<64>>(P, st) : launchM2LTc<3, Layout<32>>(P, st);
   return launchM2LTc<1, tc::LayoutTf32>(P, st);
}

}  // namespace fmm
