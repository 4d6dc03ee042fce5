// Host-side plan state and error plumbing shared by the library's translation units.
#pragma once
#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <vector>

#include "../../include/fmmcuda.h"
#include "fmm_common.cuh"

namespace fmm {

// Four consecutive coefficients (columns col .. col + 3 of multipole row `row`) stored as the tensor-core
// operand pieces: np = 1 one tf32 word each (round to nearest, ties away), np = 2 or 3 bf16 pieces, each the
// round-to-nearest of the FP32 residual left by the previous ones (the residuals are exact in FP32).
// Layout: [row][piece][Lp], 4 bytes an element for tf32 and 2 for bf16 (the tensor-core M2L's Mbf).
__device__ __forceinline__ void storePieces4(uint8_t* out, int64_t row, int col, int Lp, int np, float4 v)
{
   if(np == 1)
   {
      uint32_t w[4];
      const float x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for(int i = 0; i < 4; i++) asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(w[i]) : "f"(x[i]));
      *reinterpret_cast<uint4*>(out + (row * Lp + col) * 4) = make_uint4(w[0], w[1], w[2], w[3]);
      return;
   }
   float r[4] = {v.x, v.y, v.z, v.w};
   for(int j = 0; j < np; j++)
   {
      __nv_bfloat16 b[4];
#pragma unroll
      for(int i = 0; i < 4; i++)
      {
         b[i] = __float2bfloat16_rn(r[i]);
         r[i] -= __bfloat162float(b[i]);
      }
      uint2 pk;
      pk.x = uint32_t(__bfloat16_as_ushort(b[0])) | (uint32_t(__bfloat16_as_ushort(b[1])) << 16);
      pk.y = uint32_t(__bfloat16_as_ushort(b[2])) | (uint32_t(__bfloat16_as_ushort(b[3])) << 16);
      *reinterpret_cast<uint2*>(out + ((row * np + j) * Lp + col) * 2) = pk;
   }
}

fmm_status setError(fmm_status s, const char* fmt, ...);

#define FMM_TRY(expr)                                   \
   do                                                   \
   {                                                    \
      fmm_status _s = (expr);                           \
      if(_s != FMM_OK) return _s;                       \
   } while(0)

#define FMM_CUDA(expr)                                                                          \
   do                                                                                           \
   {                                                                                            \
      cudaError_t _e = (expr);                                                                  \
      if(_e != cudaSuccess)                                                                     \
         return ::fmm::setError(_e == cudaErrorMemoryAllocation ? FMM_E_OOM : FMM_E_CUDA,        \
                                "%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
   } while(0)

#define FMM_CHECK_LAUNCH() FMM_CUDA(cudaGetLastError())

// device error flags set by list builders and bounded waits
enum : int {
   ERR_LIST_A = 1,
   ERR_LIST_X = 2,
   ERR_LIST_COL = 4,
   ERR_LIST_V = 8,
   ERR_DFS = 16,
   ERR_TIMEOUT = 32,
};

extern __constant__ int d_m2lIndex[NOFF];   // offset index (0..342) -> M2L slot (0..315) or -1
extern __constant__ int d_m2lOffset[316];   // M2L slot -> offset index
extern __constant__ int d_m2lFarFirst[316]; // M2L slots by decreasing offset length

// A growable device allocation.
struct DevBuf
{
   void* ptr = nullptr;
   size_t bytes = 0;
   fmm_status reserve(size_t want)
   {
      if(want <= bytes) return FMM_OK;
      if(ptr) cudaFree(ptr);
      ptr = nullptr;
      bytes = 0;
      size_t b = std::max<size_t>(want, 256);
      cudaError_t e = cudaMalloc(&ptr, b);
      if(e != cudaSuccess)
      {
         cudaGetLastError();
         return setError(FMM_E_OOM, "cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(e));
      }
      bytes = b;
      return FMM_OK;
   }
   void release()
   {
      if(ptr) cudaFree(ptr);
      ptr = nullptr;
      bytes = 0;
   }
};

struct RootBox
{
   double center[3];
   double H;
   double lo[3];
   double scale;
};

struct Lists
{
   int* col;      // [node][COLCAP]
   int* ncol;
   int* acoarse;  // [node][ACAP]
   int* na;
   int* xl;       // [node][XCAP]
   int* nx;
   int* vtab;     // [node][316], source node or -1
   int* nv;
};

struct Plan
{
   fmm_config cfg;
   int p = 0, L = 0, Lp = 0;
   bool fp64 = false;
   // inputs (device copies, element type float or double)
   DevBuf srcXYZb, srcWb, srcJb, tgtXYZb;
   void* srcXYZ = nullptr; void* srcW = nullptr; void* srcJ = nullptr; void* tgtXYZ = nullptr;
   bool hasJ = false;
   // the BEM problem (fmm_set_bem_sources): J = B x n and sigma = B . n per source, the plan's strengths
   // then carry w J and w sigma (fmm_bem.cu)
   bool bem = false;
   DevBuf srcSigmab;
   void* srcSigma = nullptr;
   int64_t n = 0, m = 0;
   // independent problems ("coils"): coil c owns sources [srcOff[c], srcOff[c+1]) and targets
   // [tgtOff[c], tgtOff[c+1]); one coil by default. Each coil is a root of the forest; node keys
   // carry the coil index above the Morton bits, so keys of different coils never mix.
   int nCoils = 1;
   bool batch = false;                   // set by fmm_batch_set_coils
   std::vector<int> srcOff, tgtOff;      // host copies, nCoils + 1 entries each
   DevBuf segb;                          // device copies: srcOff then tgtOff
   int maxLevel = MAXLEVEL;              // deepest level the keys resolve
   int coilBits = 0;                     // key bits above the Morton bits
   // tree
   RootBox* root = nullptr;              // [nCoils]
   DevBuf rootb, sKeys, tKeys, sIdx, tIdx, sPos, sQ, tPos, cubTmp, scratch, lvlBounds, lvlCnt, lvlOff;
   DevBuf nodeBufs[12];
   int64_t nodeCap = 0;
   Tree tree{};
   DevBuf listBufs[8];
   int64_t listCap = 0;
   Lists lists{};
   DevBuf p2pOff, p2pList;
   DevBuf nearCounts;                    // [leaves, direct pairs] of the last tree (kNearCounts)
   int nP2P = 0;
   int64_t nV = 0;
   DevBuf parList;                      // nodes with children, in node order (M2M / L2L tiles)
   std::vector<int> parStart;           // parList index where each level's parents start [nLevels + 1]
   DevBuf m2lTargets, m2lKeys;          // boxes with an M2L list, grouped by octant
   int nM2LTargets = 0;
   // tensor-core M2M / L2L: per node and child octant, the child with sources (vtabUp, indexed by the
   // parent) and the parent of a child with targets (vtabDn, indexed by the child); the nodes with
   // targets below the roots sorted by (level, octant), and where each level starts in that list
   DevBuf vtabUp, vtabDn, l2lTargets, l2lKeys;
   std::vector<int> l2lStart;            // [8 level + octant], up to [8 nLevels]
   DevBuf opM2Mbf, opL2Lbf;              // their operator images
   int opTrImgTag = -1;
   int p2mPiecesTag = -1;                // the piece format kP2MWarp also wrote the leaves in (-1: none)
   int multBfTag = -1;                   // pieces/format multBf holds the multipoles of every node in
                                         // (levels >= 1), -1 when it holds anything else
   int tcTranslate = 1;                  // M2M (1) / L2L (2) on the tensor cores in tensor-core M2L plans
   int tcTrDrainItems = 0;               // their drains: every this many pipeline items (0: per drainEvery offsets)
   int tcTrPiecesUp = 0, tcTrPiecesDn = 3;   // their bf16 pieces (0: as the M2L mode)
   int l2lChildMajor = 1;                // CUDA-core L2L over the sorted child lists (kL2LChild)
   bool tcTranslations(int which = 3) const
   {
      return !fp64 && cfg.m2l_mode != FMM_M2L_SIMT && (tcTranslate & which) != 0;
   }
   int* err = nullptr;                   // tree build: list-capacity flags
   int* pipeErr = nullptr;               // tensor-core pipelines: ERR_TIMEOUT; cleared when a solve (or a
                                         // phase called on its own) starts and read once when it ends
   int* hostErr = nullptr;               // pinned host word the pipeline error is read into
   uint64_t tcWaitNs = 2000000000ull;    // limit of one tensor-core pipeline wait (fmm_set_wait_limit)
   DevBuf errb;
   // expansions [node][3][Lp] and outputs
   DevBuf mult, local, outB, outA;
   // operator tables (scaled basis): FP64 masters and the working-precision copies
   DevBuf opM2M64, opL2L64, opM2L64;     // [8][L][L], [8][L][L], [316][L][L] FP64 row-major
   DevBuf opM2Mw, opL2Lw, opM2Lw;        // transposed working copies, see fmm_kernels.cu
   DevBuf curlTab;                       // L2P: the curl expansion as <= 4 terms of the local, see kL2PWarp
   std::vector<unsigned char> curlHost;  // its host copy (kept alive for the asynchronous upload)
   DevBuf opM2Lbf;                       // bf16 hi/lo split for the tensor-core M2L
   DevBuf multBf;                        // multipoles split into bf16 pieces for the tensor-core M2L
   int opOrder = -1;
   // tensor-core M2L tile choices (autotuned per order and leaf capacity, or set by environment)
   int tcKChunk = 0;                     // K chunk width 32 or 64 (0: 64 for BF16X3, 32 for BF16X6)
   int tcDrainFar = 8;                   // the same through the first (far) half of a tile's offsets
   int tcDrainEvery = 8;                 // offsets accumulated in tensor memory between drains (BF16X6,
                                         // with twice the accumulations per offset, drains twice as often)
   int tcProf = 0;                       // FMM_TC_PROF=1: per-role cycle counts of the M2L launch to stderr
   DevBuf tcProfBuf;
   int tcCorrLam = 5;                    // ... and only in K steps whose lowest input degree is <= this (-1: any)
   int tcAsyncArrive = 0;                // tensor-core pipelines: 0: each producer waits for its copies, fences
                                         // and arrives; 1: producers arrive through cp.async.mbarrier and
                                         // the MMA thread fences (up to NS items in flight, but the MMA
                                         // thread loses ~400-600 cycles per item after such a barrier:
                                         // M2L 159 ms against 137 ms at 2^24)
   int tcKeepTail = 1;                   // tensor-core M2L: accumulator columns >= 256 (the top degrees) are
                                         // drained once per tile, not with the others
   int tcPair = 1;                       // tensor-core M2L: K chunks without correction products travel
                                         // up to NP per pipeline stage (0: one chunk per stage)
   int tcCorrCut = -2;                   // tensor-core M2L: correction products only for l + lambda <= this
                                         // (-1: every term the degree cutoff keeps; -2: 10)
   int tcDrainMode = 3;                  // 0: vector atomics, 1: load-add-store, 2: running sums in TMEM + 1,
                                         // 3: as 2 with 32 more columns in the drain threads' registers
   int listsWarp = 1;                    // interaction lists: 0 a thread per node (kListsLevel), 2 a warp per
                                         // node (kListsLevelWarp), 1 a warp for single-coil plans
   bool tgtIsSrc = false;                // the targets are the sources (fmm_set_targets_to_sources since the
                                         // last set_sources / set_targets)
   int treePersistent = 1;               // every tree level in one cooperative launch (kBuildLevels)
   DevBuf levelState;                    // its barrier, work queues and level starts
   int tcGroup = 2;                      // M2L target boxes grouped by octant, then 0: in node order,
                                         // 1: by list length, 2: by partner pattern (rarest offsets first)
   int simtKc = 16;                      // its K chunk (16 or 32)
   int simtTiled = 1;                    // FP32 CUDA-core M2L: register-tiled kernel (0: the row-broadcast form)
   int l2pSplit = 1;                     // 1: L2P in kL2PWarp, then the near field; 0: both in kL2PNear
   int nearTile = 256;                   // near-field source tile, points (128 or 256)
   int p2mChunk = 0;                     // P2M: 0 one warp per leaf; 16 or 32: one block per leaf, that many
                                         // recurrence steps reduced per shared tile
   DevBuf tcCounters;                    // [items, tile-offset pairs] of the last tensor-core M2L
   int64_t tcTiles = 0;
   int opImgOrder = -1;                  // order the tensor-core operator image was built for
   // state
   bool treeReady = false, upReady = false, downReady = false;
   fmm_stats stats{};
   cudaEvent_t ev[8];
   bool eventsMade = false;

   int64_t launches = 0;      // kernels this plan launched (all phases, cumulative)
   bool debugSync = false;    // FMM_DEBUG_SYNC=1: synchronise and check after every launch

   // CUDA graph of upward + downward + evaluation for the current tree (fmm_graph_capture)
   bool capturing = false;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t graphExec = nullptr;
   int graphWant = 0;
   void dropGraph()
   {
      if(graphExec) cudaGraphExecDestroy(graphExec);
      if(graph) cudaGraphDestroy(graph);
      graphExec = nullptr;
      graph = nullptr;
      graphWant = 0;
   }

   // adjoint: a plan on the swapped point sets, and staging for host inputs / outputs
   Plan* adj = nullptr;
   DevBuf adjG, adjOut;
   DevBuf tcPts, tcOut;                  // fmm_treecode: staging of host query points and results
   bool adjointDone = false;

   // fmm_set_sources_async: the host inputs cross the bus on copyStream while the solve runs; the
   // source points first (evPos), then weights and current directions (evInputs). Work that reads them
   // waits on the events (a wait on a completed event costs nothing), so the tree build starts once the
   // points are in and the strengths are gathered at its end.
   cudaStream_t copyStream = nullptr;
   cudaEvent_t evPrev = nullptr, evPos = nullptr, evInputs = nullptr;
   bool inputsAsync = false;
   fmm_status waitSourcePoints(cudaStream_t st) { return waitCopy(st, evPos); }
   fmm_status waitSourceInputs(cudaStream_t st) { return waitCopy(st, evInputs); }
   fmm_status waitCopy(cudaStream_t st, cudaEvent_t ev)
   {
      const cudaError_t e = inputsAsync ? cudaStreamWaitEvent(st, ev, 0) : cudaSuccess;
      if(e != cudaSuccess) return setError(FMM_E_CUDA, "waiting for the source copies: %s", cudaGetErrorString(e));
      return FMM_OK;
   }

   fmm_status init(const fmm_config& c);
   void release();
   fmm_status ensureNodes(int64_t cap, cudaStream_t st = 0);
   fmm_status ensureLists(int64_t cap);
};

// Bookkeeping after every kernel launch: counts it, surfaces launch errors, and in debug mode
// synchronises so a fault is attributed to the kernel that raised it.
inline fmm_status launched(Plan& P, const char* name, cudaStream_t st)
{
   P.launches++;
   cudaError_t e = cudaGetLastError();
   if(e == cudaSuccess && P.debugSync) e = cudaStreamSynchronize(st);
   if(e != cudaSuccess)
      return setError(e == cudaErrorMemoryAllocation ? FMM_E_OOM : FMM_E_CUDA, "kernel %s: %s", name,
                      cudaGetErrorString(e));
   return FMM_OK;
}

template <class T> fmm_status buildTreeT(Plan& P, cudaStream_t st);
template <class T> fmm_status upwardT(Plan& P, cudaStream_t st);
template <class T> fmm_status downwardT(Plan& P, cudaStream_t st);
template <class T> fmm_status evaluateT(Plan& P, double current, int want, cudaStream_t st);
template <class T> fmm_status directT(Plan& P, double current, int want, cudaStream_t st);
fmm_status buildOperators(Plan& P, cudaStream_t st);
fmm_status initOffsetTables();
fmm_status m2lTensorCore(Plan& P, cudaStream_t st);
fmm_status m2mTensorCore(Plan& P, cudaStream_t st);
int m2mPieces(const Plan& P);   // operand pieces of the tensor-core M2M: 1 (tf32), 2 or 3 (bf16)
fmm_status l2lTensorCore(Plan& P, cudaStream_t st);
template <class T> fmm_status regatherStrengthsT(Plan& P, cudaStream_t st);
template <class T> fmm_status scaleCopyT(Plan& P, const void* src, void* dst, int64_t count, double scale, cudaStream_t st);
template <class T> fmm_status adjointT(Plan& P, Plan& A, double current, const void* g, void* dJ, void* dx, cudaStream_t st);
template <class T> fmm_status adjointDirectT(Plan& P, double current, const void* g, void* dJ, void* dx, cudaStream_t st);
template <class T> fmm_status bemPrepareT(Plan& P, const void* B, const void* nrm, cudaStream_t st);
template <class T> fmm_status bemP2MT(Plan& P, cudaStream_t st);
template <class T> fmm_status bemNearT(Plan& P, cudaStream_t st);
template <class T> fmm_status bemDirectT(Plan& P, cudaStream_t st);
template <class T>
fmm_status treecodeT(Plan& P, double current, int want, const void* pts, int64_t m, void* outB, void* outA, int flags,
                     cudaStream_t st);

}  // namespace fmm
