// C ABI of libfmmcuda.so (declared in include/fmmcuda.h): plan lifetime, input staging,
// phase sequencing, timing and error reporting.
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <string>

#include "fmm_internal.cuh"

namespace fmm {

// addingKernel (FMMCUDADLL/kernels.cuh:6-11): c = a + b
__global__ void kAdd(const float* a, const float* b, float* c, int64_t n)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i < n) c[i] = a[i] + b[i];
}

fmm_status directFp64Subset(Plan& P, double current, const double* tgtDev, int k, double* outDev, cudaStream_t st);

namespace {
thread_local std::string g_lastError;

// autotuned choices per (device, order, leaf capacity, target leaf capacity, precision, M2L mode)
std::mutex g_tuneMutex;
std::map<std::array<int, 6>, fmm_tuning> g_tuned;

std::array<int, 6> tuneKey(const fmm_config& c)
{
   return {c.device, c.order, c.leaf_capacity, c.target_leaf_capacity, c.precision, c.m2l_mode};
}
}

fmm_status setError(fmm_status s, const char* fmt, ...)
{
   char buf[1024];
   va_list ap;
   va_start(ap, fmt);
   vsnprintf(buf, sizeof(buf), fmt, ap);
   va_end(ap);
   g_lastError = buf;
   return s;
}

fmm_status Plan::ensureNodes(int64_t cap, cudaStream_t st)
{
   if(cap <= nodeCap) return FMM_OK;
   // grow every per-node array, keeping the contents
   const size_t es[12] = {8, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4};
   for(int b = 0; b < 12; b++)
   {
      DevBuf nb;
      FMM_TRY(nb.reserve(es[b] * cap));
      if(nodeBufs[b].ptr && nodeCap > 0)
         FMM_CUDA(cudaMemcpyAsync(nb.ptr, nodeBufs[b].ptr, es[b] * nodeCap, cudaMemcpyDeviceToDevice, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      nodeBufs[b].release();
      nodeBufs[b] = nb;
   }
   nodeCap = cap;
   tree.key = (uint64_t*)nodeBufs[0].ptr;
   tree.level = (int*)nodeBufs[1].ptr;
   tree.ix = (int*)nodeBufs[2].ptr;
   tree.iy = (int*)nodeBufs[3].ptr;
   tree.iz = (int*)nodeBufs[4].ptr;
   tree.s0 = (int*)nodeBufs[5].ptr;
   tree.s1 = (int*)nodeBufs[6].ptr;
   tree.t0 = (int*)nodeBufs[7].ptr;
   tree.t1 = (int*)nodeBufs[8].ptr;
   tree.parent = (int*)nodeBufs[9].ptr;
   tree.child0 = (int*)nodeBufs[10].ptr;
   tree.nchild = (int*)nodeBufs[11].ptr;
   return FMM_OK;
}

fmm_status Plan::init(const fmm_config& c)
{
   cfg = c;
   p = c.order;
   L = nharm(p);
   Lp = padded(L);
   fp64 = c.precision == FMM_FP64;
   const char* dbg = getenv("FMM_DEBUG_SYNC");
   debugSync = dbg && dbg[0] == '1';
   {
      std::lock_guard<std::mutex> lock(g_tuneMutex);
      auto it = g_tuned.find(tuneKey(c));
      if(it != g_tuned.end())
      {
         tcKChunk = it->second.m2l_k_chunk;
         nearTile = it->second.near_tile;
         p2mChunk = it->second.p2m_chunk;
      }
   }
   if(const char* e = getenv("FMM_TC_KC")) tcKChunk = atoi(e) == 32 ? 32 : 64;
   if(const char* e = getenv("FMM_TC_DRAIN")) tcDrainEvery = std::max(1, atoi(e));
   tcDrainFar = tcDrainEvery;
   if(const char* e = getenv("FMM_TC_DRAINFAR")) tcDrainFar = std::max(1, atoi(e));
   if(const char* e = getenv("FMM_TC_CORR")) tcCorrCut = atoi(e);
   if(const char* e = getenv("FMM_TC_CORRLAM")) tcCorrLam = atoi(e);
   if(const char* e = getenv("FMM_TC_ASYNC")) tcAsyncArrive = atoi(e) != 0;
   if(const char* e = getenv("FMM_TC_PAIR")) tcPair = atoi(e) != 0;
   if(const char* e = getenv("FMM_TREE_PERSISTENT")) treePersistent = atoi(e) != 0;
   if(const char* e = getenv("FMM_LISTS_WARP")) listsWarp = std::min(2, std::max(0, atoi(e)));
   if(const char* e = getenv("FMM_TC_KEEPTAIL")) tcKeepTail = atoi(e) != 0;
   if(const char* e = getenv("FMM_TC_PROF")) tcProf = atoi(e) != 0;
   if(const char* e = getenv("FMM_TC_CUTOFF")) cfg.m2l_tc_degree_cutoff = atoi(e);
   if(const char* e = getenv("FMM_TC_DRAINMODE")) tcDrainMode = std::min(3, std::max(0, atoi(e)));
   if(const char* e = getenv("FMM_TC_GROUP")) tcGroup = std::min(2, std::max(0, atoi(e)));
   if(const char* e = getenv("FMM_L2P_SPLIT")) l2pSplit = atoi(e) != 0;
   if(const char* e = getenv("FMM_SIMT_TILED")) simtTiled = std::min(2, std::max(0, atoi(e)));
   if(const char* e = getenv("FMM_SIMT_KC")) simtKc = atoi(e) == 32 ? 32 : 16;
   if(const char* e = getenv("FMM_TC_TRANSLATE")) tcTranslate = atoi(e) & 3;
   if(const char* e = getenv("FMM_TC_TRDRAIN")) tcTrDrainItems = std::max(0, atoi(e));
   if(const char* e = getenv("FMM_L2L_CHILD")) l2lChildMajor = atoi(e) != 0;
   if(const char* e = getenv("FMM_TC_TRNP_UP")) tcTrPiecesUp = std::min(3, std::max(0, atoi(e)));
   if(const char* e = getenv("FMM_TC_TRNP_DN")) tcTrPiecesDn = std::min(3, std::max(0, atoi(e)));

   FMM_TRY(rootb.reserve(sizeof(RootBox)));
   FMM_TRY(errb.reserve(2 * sizeof(int)));
   FMM_TRY(initOffsetTables());
   root = (RootBox*)rootb.ptr;
   err = (int*)errb.ptr;
   pipeErr = err + 1;
   FMM_CUDA(cudaMemset(errb.ptr, 0, 2 * sizeof(int)));
   FMM_CUDA(cudaMallocHost((void**)&hostErr, sizeof(int)));
   *hostErr = 0;
   for(int i = 0; i < 8; i++) cudaEventCreate(&ev[i]);
   eventsMade = true;
   return FMM_OK;
}

void Plan::release()
{
   dropGraph();
   if(copyStream)
   {
      // copies of fmm_set_sources_async still in flight write into buffers freed below
      cudaStreamSynchronize(copyStream);
      cudaStreamDestroy(copyStream);
      cudaEventDestroy(evPrev);
      cudaEventDestroy(evPos);
      cudaEventDestroy(evInputs);
      copyStream = nullptr;
      evPrev = evPos = evInputs = nullptr;
   }
   inputsAsync = false;
   if(adj)
   {
      adj->release();
      delete adj;
      adj = nullptr;
   }
   DevBuf* bufs[] = {&srcXYZb, &srcWb, &srcJb, &tgtXYZb, &rootb, &sKeys, &tKeys, &sIdx, &tIdx, &sPos, &sQ, &tPos,
                     &cubTmp, &scratch, &lvlBounds, &lvlCnt, &lvlOff, &p2pOff, &p2pList, &parList, &m2lTargets, &m2lKeys, &errb,
                     &mult, &local, &outB, &outA, &opM2M64, &opL2L64, &opM2L64, &opM2Mw, &opL2Lw, &opM2Lw, &opM2Lbf, &multBf, &tcCounters,
                     &adjG, &adjOut, &tcPts, &tcOut, &srcSigmab, &nearCounts, &tcProfBuf, &levelState, &curlTab, &vtabUp, &vtabDn, &l2lTargets, &l2lKeys, &opM2Mbf, &opL2Lbf};
   for(DevBuf* b : bufs) b->release();
   for(auto& b : nodeBufs) b.release();
   for(auto& b : listBufs) b.release();
   if(hostErr) cudaFreeHost(hostErr);
   hostErr = nullptr;
   err = pipeErr = nullptr;
   if(eventsMade)
      for(int i = 0; i < 8; i++) cudaEventDestroy(ev[i]);
   eventsMade = false;
}

fmm_status Plan::ensureLists(int64_t cap)
{
   if(cap <= listCap) return FMM_OK;
   const size_t per[8] = {COLCAP, 1, ACAP, 1, XCAP, 1, 316, 1};
   for(int b = 0; b < 8; b++) FMM_TRY(listBufs[b].reserve(sizeof(int) * per[b] * cap));
   listCap = cap;
   lists.col = (int*)listBufs[0].ptr;
   lists.ncol = (int*)listBufs[1].ptr;
   lists.acoarse = (int*)listBufs[2].ptr;
   lists.na = (int*)listBufs[3].ptr;
   lists.xl = (int*)listBufs[4].ptr;
   lists.nx = (int*)listBufs[5].ptr;
   lists.vtab = (int*)listBufs[6].ptr;
   lists.nv = (int*)listBufs[7].ptr;
   return FMM_OK;
}

}  // namespace fmm

using namespace fmm;

struct fmm_plan
{
   Plan P;
};

namespace {

struct DeviceGuard
{
   int prev = -1;
   explicit DeviceGuard(int dev)
   {
      cudaGetDevice(&prev);
      if(prev != dev) cudaSetDevice(dev);
   }
   ~DeviceGuard()
   {
      int cur = -1;
      cudaGetDevice(&cur);
      if(prev >= 0 && cur != prev) cudaSetDevice(prev);
   }
};

fmm_status copyIn(DevBuf& buf, const void* src, size_t bytes, int onDevice, cudaStream_t st, void** out)
{
   FMM_TRY(buf.reserve(bytes));
   if(bytes) FMM_CUDA(cudaMemcpyAsync(buf.ptr, src, bytes, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
   *out = buf.ptr;
   return FMM_OK;
}

fmm_status copyOut(void* dst, const DevBuf& buf, size_t bytes, int onDevice, cudaStream_t st)
{
   if(!dst || !bytes) return FMM_OK;
   FMM_CUDA(cudaMemcpyAsync(dst, buf.ptr, bytes, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
   if(!onDevice) FMM_CUDA(cudaStreamSynchronize(st));
   return FMM_OK;
}

// The tensor-core pipelines' error word: cleared on the stream when a solve (or a phase called on
// its own) starts, read once when it ends, so the phases between queue their kernels without a
// host wait.
fmm_status pipeBegin(Plan& P, cudaStream_t st)
{
   FMM_CUDA(cudaMemsetAsync(P.pipeErr, 0, sizeof(int), st));
   return FMM_OK;
}

fmm_status pipeCheck(Plan& P, cudaStream_t st, const char* what)
{
   FMM_CUDA(cudaMemcpyAsync(P.hostErr, P.pipeErr, sizeof(int), cudaMemcpyDeviceToHost, st));
   FMM_CUDA(cudaStreamSynchronize(st));
   if(*P.hostErr & ERR_TIMEOUT)
      return setError(FMM_E_TIMEOUT, "%s: a tensor-core pipeline wait timed out (limit %.3g s)", what,
                      double(P.tcWaitNs) * 1e-9);
   return FMM_OK;
}

fmm_status upwardPhase(Plan& P, cudaStream_t st)
{
   FMM_TRY(P.fp64 ? upwardT<double>(P, st) : upwardT<float>(P, st));
   cudaEventRecord(P.ev[2], st);
   P.upReady = true;
   P.downReady = false;
   return FMM_OK;
}

fmm_status downwardPhase(Plan& P, cudaStream_t st)
{
   FMM_TRY(P.fp64 ? downwardT<double>(P, st) : downwardT<float>(P, st));
   cudaEventRecord(P.ev[4], st);
   P.downReady = true;
   return FMM_OK;
}

double elapsed(cudaEvent_t a, cudaEvent_t b)
{
   float ms = 0;
   if(cudaEventElapsedTime(&ms, a, b) != cudaSuccess) { cudaGetLastError(); return 0; }
   return ms;
}

}  // namespace

extern "C" {

const char* fmm_version(void) { return "bachelors_b200 fmmcuda 0.1 (sm_100a)"; }

const char* fmm_last_error_string(void) { return g_lastError.c_str(); }

void fmm_default_config(fmm_config* cfg)
{
   if(!cfg) return;
   std::memset(cfg, 0, sizeof(*cfg));
   cfg->order = 10;
   cfg->leaf_capacity = 64;
   cfg->precision = FMM_FP32;
   cfg->m2l_mode = FMM_M2L_SIMT;
   cfg->m2l_truncate = 0;
   cfg->device = 0;
   cfg->root_half_width = 0;
}

fmm_status fmm_plan_create(const fmm_config* cfg, fmm_plan** plan)
{
   if(!cfg || !plan) return setError(FMM_E_INVALID, "fmm_plan_create: null argument");
   *plan = nullptr;
   if(cfg->order < 1 || cfg->order > MAXORDER)
      return setError(FMM_E_INVALID, "order %d outside 1..%d", cfg->order, MAXORDER);
   if(cfg->leaf_capacity < 1) return setError(FMM_E_INVALID, "leaf_capacity must be >= 1");
   if(cfg->precision != FMM_FP32 && cfg->precision != FMM_FP64)
      return setError(FMM_E_INVALID, "unknown precision %d", cfg->precision);
   if(cfg->m2l_mode < FMM_M2L_SIMT || cfg->m2l_mode > FMM_M2L_BF16X6)
      return setError(FMM_E_INVALID, "unknown m2l_mode %d", cfg->m2l_mode);
   int ndev = 0;
   cudaError_t e = cudaGetDeviceCount(&ndev);
   if(e != cudaSuccess || ndev == 0)
   {
      cudaGetLastError();
      return setError(FMM_E_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
   }
   if(cfg->device < 0 || cfg->device >= ndev) return setError(FMM_E_INVALID, "device %d out of range", cfg->device);
   DeviceGuard g(cfg->device);
   fmm_plan* h = new fmm_plan();
   fmm_status s = h->P.init(*cfg);
   if(s != FMM_OK) { delete h; return s; }
   *plan = h;
   return FMM_OK;
}

fmm_status fmm_plan_destroy(fmm_plan* plan)
{
   if(!plan) return FMM_OK;
   DeviceGuard g(plan->P.cfg.device);
   plan->P.release();
   delete plan;
   return FMM_OK;
}

fmm_status fmm_set_sources(fmm_plan* plan, const void* xyz, const void* w, const void* J, int64_t n, int on_device,
                           void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   if(n < 0 || n > (int64_t(1) << 31) - 1) return setError(FMM_E_INVALID, "source count %lld out of range", (long long)n);
   if(n > 0 && (!xyz || !w)) return setError(FMM_E_INVALID, "null source coordinates or weights");
   Plan& P = plan->P;
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(P.waitSourceInputs(st));   // copies of an earlier fmm_set_sources_async into the same buffers
   FMM_TRY(copyIn(P.srcXYZb, xyz, es * 3 * n, on_device, st, &P.srcXYZ));
   FMM_TRY(copyIn(P.srcWb, w, es * n, on_device, st, &P.srcW));
   P.hasJ = J != nullptr;
   if(P.hasJ) FMM_TRY(copyIn(P.srcJb, J, es * 3 * n, on_device, st, &P.srcJ));
   if(!on_device) FMM_CUDA(cudaStreamSynchronize(st));
   P.inputsAsync = false;
   P.bem = false;
   P.n = n;
   P.tgtIsSrc = false;
   P.treeReady = P.upReady = P.downReady = false;
   P.dropGraph();
   return FMM_OK;
}

fmm_status fmm_set_sources_async(fmm_plan* plan, const void* xyz, const void* w, const void* J, int64_t n, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   if(n < 0 || n > (int64_t(1) << 31) - 1) return setError(FMM_E_INVALID, "source count %lld out of range", (long long)n);
   if(n > 0 && (!xyz || !w)) return setError(FMM_E_INVALID, "null source coordinates or weights");
   Plan& P = plan->P;
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   // page-locked host memory only: a pageable buffer would be copied by the driver before the call returns
   const void* ptrs[3] = {xyz, w, J};
   for(const void* p : ptrs)
   {
      if(!p || n == 0) continue;
      cudaPointerAttributes a;
      const cudaError_t e = cudaPointerGetAttributes(&a, p);
      if(e != cudaSuccess || a.type != cudaMemoryTypeHost)
      {
         cudaGetLastError();
         return setError(FMM_E_INVALID, "fmm_set_sources_async: the inputs must be page-locked host memory");
      }
   }
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(P.srcXYZb.reserve(es * 3 * n));
   FMM_TRY(P.srcWb.reserve(es * n));
   P.hasJ = J != nullptr;
   if(P.hasJ) FMM_TRY(P.srcJb.reserve(es * 3 * n));
   if(!P.copyStream)
   {
      FMM_CUDA(cudaStreamCreateWithFlags(&P.copyStream, cudaStreamNonBlocking));
      FMM_CUDA(cudaEventCreateWithFlags(&P.evPrev, cudaEventDisableTiming));
      FMM_CUDA(cudaEventCreateWithFlags(&P.evPos, cudaEventDisableTiming));
      FMM_CUDA(cudaEventCreateWithFlags(&P.evInputs, cudaEventDisableTiming));
   }
   // the copies follow the work queued on `stream` so far (it may still read the previous sources)
   FMM_CUDA(cudaEventRecord(P.evPrev, st));
   FMM_CUDA(cudaStreamWaitEvent(P.copyStream, P.evPrev, 0));
   if(n) FMM_CUDA(cudaMemcpyAsync(P.srcXYZb.ptr, xyz, es * 3 * n, cudaMemcpyHostToDevice, P.copyStream));
   FMM_CUDA(cudaEventRecord(P.evPos, P.copyStream));
   if(n) FMM_CUDA(cudaMemcpyAsync(P.srcWb.ptr, w, es * n, cudaMemcpyHostToDevice, P.copyStream));
   if(n && P.hasJ) FMM_CUDA(cudaMemcpyAsync(P.srcJb.ptr, J, es * 3 * n, cudaMemcpyHostToDevice, P.copyStream));
   FMM_CUDA(cudaEventRecord(P.evInputs, P.copyStream));
   P.srcXYZ = P.srcXYZb.ptr;
   P.srcW = P.srcWb.ptr;
   if(P.hasJ) P.srcJ = P.srcJb.ptr;
   P.inputsAsync = true;
   P.bem = false;
   P.n = n;
   P.tgtIsSrc = false;
   P.treeReady = P.upReady = P.downReady = false;
   P.dropGraph();
   return FMM_OK;
}

fmm_status fmm_set_bem_sources(fmm_plan* plan, const void* xyz, const void* w, const void* B, const void* normal,
                               int64_t n, int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   if(n < 0 || n > (int64_t(1) << 31) - 1) return setError(FMM_E_INVALID, "source count %lld out of range", (long long)n);
   if(n > 0 && (!xyz || !w || !B || !normal)) return setError(FMM_E_INVALID, "fmm_set_bem_sources: null argument");
   Plan& P = plan->P;
   if(P.batch) return setError(FMM_E_INVALID, "fmm_set_bem_sources: not available on a batched plan");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(copyIn(P.srcXYZb, xyz, es * 3 * n, on_device, st, &P.srcXYZ));
   FMM_TRY(copyIn(P.srcWb, w, es * n, on_device, st, &P.srcW));
   FMM_TRY(P.srcJb.reserve(std::max<size_t>(es * 3 * n, 16)));
   FMM_TRY(P.srcSigmab.reserve(std::max<size_t>(es * n, 16)));
   P.srcJ = P.srcJb.ptr;
   P.srcSigma = P.srcSigmab.ptr;
   P.n = n;
   P.tgtIsSrc = false;
   P.hasJ = true;
   P.bem = true;
   // B and the normals (staged when on the host) become J = B x n and sigma = B . n
   const void* dB = B;
   const void* dN = normal;
   DevBuf stage;
   if(!on_device && n > 0)
   {
      FMM_TRY(stage.reserve(2 * es * 3 * n));
      cudaError_t e = cudaMemcpyAsync(stage.ptr, B, es * 3 * n, cudaMemcpyHostToDevice, st);
      if(e == cudaSuccess)
         e = cudaMemcpyAsync((char*)stage.ptr + es * 3 * n, normal, es * 3 * n, cudaMemcpyHostToDevice, st);
      if(e != cudaSuccess)
      {
         stage.release();
         return setError(FMM_E_CUDA, "fmm_set_bem_sources: %s", cudaGetErrorString(e));
      }
      dB = stage.ptr;
      dN = (char*)stage.ptr + es * 3 * n;
   }
   fmm_status s = P.fp64 ? bemPrepareT<double>(P, dB, dN, st) : bemPrepareT<float>(P, dB, dN, st);
   if(!on_device || stage.ptr)
   {
      cudaError_t e = cudaStreamSynchronize(st);
      if(s == FMM_OK && e != cudaSuccess) s = setError(FMM_E_CUDA, "fmm_set_bem_sources: %s", cudaGetErrorString(e));
   }
   stage.release();
   P.inputsAsync = false;
   P.treeReady = P.upReady = P.downReady = false;
   P.dropGraph();
   return s;
}

fmm_status fmm_set_targets(fmm_plan* plan, const void* xyz, int64_t m, int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   if(m < 0 || m > (int64_t(1) << 31) - 1) return setError(FMM_E_INVALID, "target count %lld out of range", (long long)m);
   if(m > 0 && !xyz) return setError(FMM_E_INVALID, "null target coordinates");
   Plan& P = plan->P;
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(copyIn(P.tgtXYZb, xyz, es * 3 * m, on_device, st, &P.tgtXYZ));
   if(!on_device) FMM_CUDA(cudaStreamSynchronize(st));
   P.m = m;
   P.tgtIsSrc = false;
   P.treeReady = P.upReady = P.downReady = false;
   P.dropGraph();
   return FMM_OK;
}

fmm_status fmm_set_targets_to_sources(fmm_plan* plan, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(P.n > 0 && !P.srcXYZ) return setError(FMM_E_INVALID, "fmm_set_targets_to_sources: no sources set");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourcePoints(st));   // fmm_set_sources_async copies in flight
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   const size_t bytes = es * 3 * size_t(P.n);
   FMM_TRY(P.tgtXYZb.reserve(std::max<size_t>(bytes, 16)));
   if(bytes) FMM_CUDA(cudaMemcpyAsync(P.tgtXYZb.ptr, P.srcXYZ, bytes, cudaMemcpyDeviceToDevice, st));
   P.tgtXYZ = P.tgtXYZb.ptr;
   P.m = P.n;
   P.tgtIsSrc = true;
   P.treeReady = P.upReady = P.downReady = false;
   P.dropGraph();
   return FMM_OK;
}

fmm_status fmm_build_tree(fmm_plan* plan, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(P.n + P.m == 0) return setError(FMM_E_INVALID, "no sources or targets set");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   P.dropGraph();
   cudaEventRecord(P.ev[0], st);
   FMM_TRY(P.fp64 ? buildTreeT<double>(P, st) : buildTreeT<float>(P, st));
   cudaEventRecord(P.ev[1], st);
   P.treeReady = true;
   P.upReady = P.downReady = false;
   return FMM_OK;
}

fmm_status fmm_upward(fmm_plan* plan, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.treeReady) return setError(FMM_E_INVALID, "fmm_upward: tree not built");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(pipeBegin(P, st));
   FMM_TRY(upwardPhase(P, st));
   return pipeCheck(P, st, "fmm_upward");
}

fmm_status fmm_downward(fmm_plan* plan, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.upReady) return setError(FMM_E_INVALID, "fmm_downward: multipoles are not ready");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(pipeBegin(P, st));
   FMM_TRY(downwardPhase(P, st));
   return pipeCheck(P, st, "fmm_downward");
}

fmm_status fmm_evaluate(fmm_plan* plan, double current, int want, void* out_B, void* out_A, int on_device,
                        void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.downReady) return setError(FMM_E_INVALID, "fmm_evaluate: local expansions are not ready");
   if(want < 1 || want > 3) return setError(FMM_E_INVALID, "want must be 1, 2 or 3");
   if(P.bem && want != 2)
      return setError(FMM_E_INVALID, "a plan with BEM sources evaluates the BEM integral into out_A (want = 2)");
   if(((want & 1) && !out_B) || ((want & 2) && !out_A)) return setError(FMM_E_INVALID, "null output buffer");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   size_t bytes = es * 3 * std::max<int64_t>(P.m, 1);
   bool directB = on_device && (want & 1);
   bool directA = on_device && (want & 2);
   // write straight into device outputs; stage host outputs through plan buffers
   DevBuf ob, oa;
   if(directB) { ob.ptr = out_B; ob.bytes = bytes; }
   else if(want & 1) { FMM_TRY(P.outB.reserve(bytes)); ob = P.outB; }
   if(directA) { oa.ptr = out_A; oa.bytes = bytes; }
   else if(want & 2) { FMM_TRY(P.outA.reserve(bytes)); oa = P.outA; }
   DevBuf saveB = P.outB, saveA = P.outA;
   P.outB = ob;
   P.outA = oa;
   fmm_status s = P.fp64 ? evaluateT<double>(P, current, want, st) : evaluateT<float>(P, current, want, st);
   P.outB = saveB;
   P.outA = saveA;
   FMM_TRY(s);
   cudaEventRecord(P.ev[5], st);
   if(!on_device)
   {
      if(want & 1) FMM_TRY(copyOut(out_B, P.outB, es * 3 * P.m, 0, st));
      if(want & 2) FMM_TRY(copyOut(out_A, P.outA, es * 3 * P.m, 0, st));
   }
   return FMM_OK;
}

fmm_status fmm_solve(fmm_plan* plan, double current, int want, void* out_B, void* out_A, int on_device, void* stream)
{
   if(plan && plan->P.bem && want != 2)
      return setError(FMM_E_INVALID, "a plan with BEM sources evaluates the BEM integral into out_A (want = 2)");
   FMM_TRY(fmm_build_tree(plan, stream));
   Plan& P = plan->P;
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   // upward, M2L and downward are queued without a host wait; the pipeline error word is read
   // once, after the evaluation
   FMM_TRY(pipeBegin(P, st));
   FMM_TRY(upwardPhase(P, st));
   FMM_TRY(downwardPhase(P, st));
   FMM_TRY(fmm_evaluate(plan, current, want, out_B, out_A, on_device, stream));
   return pipeCheck(P, st, "fmm_solve");
}

fmm_status fmm_direct(fmm_plan* plan, double current, int want, void* out_B, void* out_A, int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(want < 1 || want > 3) return setError(FMM_E_INVALID, "want must be 1, 2 or 3");
   if(((want & 1) && !out_B) || ((want & 2) && !out_A)) return setError(FMM_E_INVALID, "null output buffer");
   if(P.bem && want != 2)
      return setError(FMM_E_INVALID, "a plan with BEM sources sums the BEM integral into out_A (want = 2)");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   if(!P.treeReady) FMM_TRY(fmm_build_tree(plan, stream));
   size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   size_t bytes = es * 3 * std::max<int64_t>(P.m, 1);
   FMM_TRY(P.outB.reserve(bytes));
   FMM_TRY(P.outA.reserve(bytes));
   FMM_TRY(P.fp64 ? directT<double>(P, current, want, st) : directT<float>(P, current, want, st));
   if(want & 1) FMM_TRY(copyOut(out_B, P.outB, es * 3 * P.m, on_device, st));
   if(want & 2) FMM_TRY(copyOut(out_A, P.outA, es * 3 * P.m, on_device, st));
   return FMM_OK;
}

fmm_status fmm_direct_fp64_subset(fmm_plan* plan, double current, const double* tgt, int64_t k, double* out_B)
{
   if(!plan || (k > 0 && (!tgt || !out_B))) return setError(FMM_E_INVALID, "null argument");
   Plan& P = plan->P;
   if(P.batch)
      return setError(FMM_E_INVALID, "fmm_direct_fp64_subset: explicit targets belong to no coil of a batched plan");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = 0;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   if(!P.treeReady) FMM_TRY(fmm_build_tree(plan, nullptr));
   DevBuf t, o;
   FMM_TRY(t.reserve(sizeof(double) * 3 * std::max<int64_t>(k, 1)));
   fmm_status s = o.reserve(sizeof(double) * 3 * std::max<int64_t>(k, 1));
   if(s != FMM_OK) { t.release(); return s; }
   cudaMemcpyAsync(t.ptr, tgt, sizeof(double) * 3 * k, cudaMemcpyHostToDevice, st);
   s = directFp64Subset(P, current, (const double*)t.ptr, int(k), (double*)o.ptr, st);
   if(s == FMM_OK)
   {
      cudaError_t e = cudaMemcpyAsync(out_B, o.ptr, sizeof(double) * 3 * k, cudaMemcpyDeviceToHost, st);
      if(e == cudaSuccess) e = cudaStreamSynchronize(st);
      if(e != cudaSuccess) s = setError(FMM_E_CUDA, "fmm_direct_fp64_subset: %s", cudaGetErrorString(e));
   }
   t.release();
   o.release();
   return s;
}

fmm_status fmm_adjoint(fmm_plan* plan, double current, const void* dL_dB, void* dL_dJ, void* dL_dx, int on_device,
                       void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(P.n == 0 || P.m == 0) return setError(FMM_E_INVALID, "fmm_adjoint: sources and targets must be set");
   if(P.bem) return setError(FMM_E_INVALID, "fmm_adjoint: not available for BEM sources");
   if(!dL_dB || (!dL_dJ && !dL_dx)) return setError(FMM_E_INVALID, "fmm_adjoint: null argument");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   if(!P.adj)
   {
      fmm_config c = P.cfg;
      // roles swap: the forward targets are the adjoint sources
      c.leaf_capacity = P.cfg.target_leaf_capacity > 0 ? P.cfg.target_leaf_capacity : P.cfg.leaf_capacity;
      c.target_leaf_capacity = P.cfg.leaf_capacity;
      P.adj = new Plan();
      fmm_status s = P.adj->init(c);
      if(s != FMM_OK) { P.adj->release(); delete P.adj; P.adj = nullptr; return s; }
   }
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   P.adj->tcWaitNs = P.tcWaitNs;
   // the coils keep their pairing with the roles swapped
   P.adj->nCoils = P.nCoils;
   P.adj->batch = P.batch;
   P.adj->srcOff = P.tgtOff;
   P.adj->tgtOff = P.srcOff;
   const void* gDev = dL_dB;
   void* dJ = dL_dJ;
   void* dx = dL_dx;
   if(!on_device)
   {
      FMM_TRY(P.adjG.reserve(es * 3 * P.m));
      FMM_CUDA(cudaMemcpyAsync(P.adjG.ptr, dL_dB, es * 3 * P.m, cudaMemcpyHostToDevice, st));
      gDev = P.adjG.ptr;
      FMM_TRY(P.adjOut.reserve(2 * es * 3 * P.n));
      dJ = dL_dJ ? P.adjOut.ptr : nullptr;
      dx = dL_dx ? (char*)P.adjOut.ptr + es * 3 * P.n : nullptr;
   }
   cudaEventRecord(P.ev[6], st);
   FMM_TRY(pipeBegin(*P.adj, st));
   FMM_TRY(P.fp64 ? adjointT<double>(P, *P.adj, current, gDev, dJ, dx, st)
                  : adjointT<float>(P, *P.adj, current, gDev, dJ, dx, st));
   cudaEventRecord(P.ev[7], st);
   FMM_TRY(pipeCheck(*P.adj, st, "fmm_adjoint"));
   P.adjointDone = true;
   if(!on_device)
   {
      if(dL_dJ) FMM_CUDA(cudaMemcpyAsync(dL_dJ, dJ, es * 3 * P.n, cudaMemcpyDeviceToHost, st));
      if(dL_dx) FMM_CUDA(cudaMemcpyAsync(dL_dx, dx, es * 3 * P.n, cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
   }
   return FMM_OK;
}

fmm_status fmm_treecode(fmm_plan* plan, double current, int want, const void* pts, int64_t m, void* out_B, void* out_A,
                        int flags, int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.upReady) return setError(FMM_E_INVALID, "fmm_treecode: multipoles are not ready (fmm_build_tree, fmm_upward)");
   if(P.batch) return setError(FMM_E_INVALID, "fmm_treecode: a query point belongs to no coil of a batched plan");
   if(want < 1 || want > 3) return setError(FMM_E_INVALID, "want must be 1, 2 or 3");
   if(flags & ~(FMM_TREECODE_REFERENCE_NEAR | FMM_TREECODE_FD_CURL))
      return setError(FMM_E_INVALID, "fmm_treecode: unknown flags 0x%x", flags);
   if(P.bem && want != 2)
      return setError(FMM_E_INVALID, "fmm_treecode: a plan with BEM sources evaluates the BEM integral (want = 2)");
   if(m < 0 || m > (int64_t(1) << 31) - 1) return setError(FMM_E_INVALID, "query count %lld out of range", (long long)m);
   if(m > 0 && (!pts || ((want & 1) && !out_B) || ((want & 2) && !out_A)))
      return setError(FMM_E_INVALID, "fmm_treecode: null argument");
   if(m == 0) return FMM_OK;
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   const size_t bytes = es * 3 * size_t(m);
   const void* dPts = pts;
   void* dB = out_B;
   void* dA = out_A;
   if(!on_device)
   {
      FMM_TRY(P.tcPts.reserve(bytes));
      FMM_TRY(P.tcOut.reserve(2 * bytes));
      FMM_CUDA(cudaMemcpyAsync(P.tcPts.ptr, pts, bytes, cudaMemcpyHostToDevice, st));
      dPts = P.tcPts.ptr;
      dB = (want & 1) ? P.tcOut.ptr : nullptr;
      dA = (want & 2) ? (char*)P.tcOut.ptr + bytes : nullptr;
   }
   FMM_TRY(P.fp64 ? treecodeT<double>(P, current, want, dPts, m, dB, dA, flags, st)
                  : treecodeT<float>(P, current, want, dPts, m, dB, dA, flags, st));
   if(!on_device)
   {
      if(want & 1) FMM_CUDA(cudaMemcpyAsync(out_B, dB, bytes, cudaMemcpyDeviceToHost, st));
      if(want & 2) FMM_CUDA(cudaMemcpyAsync(out_A, dA, bytes, cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
   }
   return FMM_OK;
}

fmm_status fmm_adjoint_direct(fmm_plan* plan, double current, const void* dL_dB, void* dL_dJ, void* dL_dx,
                              int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!dL_dB || (!dL_dJ && !dL_dx)) return setError(FMM_E_INVALID, "fmm_adjoint_direct: null argument");
   if(P.bem) return setError(FMM_E_INVALID, "fmm_adjoint_direct: not available for BEM sources");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   const void* gDev = dL_dB;
   void* dJ = dL_dJ;
   void* dx = dL_dx;
   if(!on_device)
   {
      FMM_TRY(P.adjG.reserve(es * 3 * std::max<int64_t>(P.m, 1)));
      if(P.m) FMM_CUDA(cudaMemcpyAsync(P.adjG.ptr, dL_dB, es * 3 * P.m, cudaMemcpyHostToDevice, st));
      gDev = P.adjG.ptr;
      FMM_TRY(P.adjOut.reserve(2 * es * 3 * std::max<int64_t>(P.n, 1)));
      dJ = dL_dJ ? P.adjOut.ptr : nullptr;
      dx = dL_dx ? (char*)P.adjOut.ptr + es * 3 * P.n : nullptr;
   }
   if(P.n)
   {
      if(dJ) FMM_CUDA(cudaMemsetAsync(dJ, 0, es * 3 * P.n, st));
      if(dx) FMM_CUDA(cudaMemsetAsync(dx, 0, es * 3 * P.n, st));
   }
   FMM_TRY(P.fp64 ? adjointDirectT<double>(P, current, gDev, dJ, dx, st)
                  : adjointDirectT<float>(P, current, gDev, dJ, dx, st));
   if(!on_device)
   {
      if(dL_dJ && P.n) FMM_CUDA(cudaMemcpyAsync(dL_dJ, dJ, es * 3 * P.n, cudaMemcpyDeviceToHost, st));
      if(dL_dx && P.n) FMM_CUDA(cudaMemcpyAsync(dL_dx, dx, es * 3 * P.n, cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
   }
   return FMM_OK;
}

fmm_status fmm_get_tuning(const fmm_plan* plan, fmm_tuning* out)
{
   if(!plan || !out) return setError(FMM_E_INVALID, "null argument");
   const Plan& P = plan->P;
   std::memset(out, 0, sizeof(*out));
   out->m2l_k_chunk = P.tcKChunk ? P.tcKChunk : (P.cfg.m2l_mode == FMM_M2L_BF16X6 ? 32 : 64);
   out->near_tile = P.nearTile;
   out->p2m_chunk = P.p2mChunk;
   return FMM_OK;
}

fmm_status fmm_set_tuning(fmm_plan* plan, const fmm_tuning* in)
{
   if(!plan || !in) return setError(FMM_E_INVALID, "null argument");
   if((in->m2l_k_chunk != 32 && in->m2l_k_chunk != 64) || (in->near_tile != 128 && in->near_tile != 256) ||
      (in->p2m_chunk != 0 && in->p2m_chunk != 16 && in->p2m_chunk != 32))
      return setError(FMM_E_INVALID, "fmm_set_tuning: m2l_k_chunk 32|64, near_tile 128|256, p2m_chunk 0|16|32");
   Plan& P = plan->P;
   P.tcKChunk = in->m2l_k_chunk;
   P.nearTile = in->near_tile;
   P.p2mChunk = in->p2m_chunk;
   P.dropGraph();
   return FMM_OK;
}

fmm_status fmm_autotune(fmm_plan* plan, fmm_tuning* out, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.downReady) return setError(FMM_E_INVALID, "fmm_autotune: run fmm_solve first (the tuner times the plan's data)");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   P.dropGraph();
   FMM_TRY(pipeBegin(P, st));
   cudaEvent_t e0, e1;
   FMM_CUDA(cudaEventCreate(&e0));
   cudaError_t ce = cudaEventCreate(&e1);
   if(ce != cudaSuccess)
   {
      cudaEventDestroy(e0);
      return setError(FMM_E_CUDA, "fmm_autotune: %s", cudaGetErrorString(ce));
   }
   fmm_status s = FMM_OK;
   // best of two runs of one phase, in milliseconds
   auto timePhase = [&](auto&& phase, double& ms) -> fmm_status {
      ms = 1e300;
      for(int r = 0; r < 2; r++)
      {
         cudaEventRecord(e0, st);
         FMM_TRY(phase());
         cudaEventRecord(e1, st);
         FMM_CUDA(cudaEventSynchronize(e1));
         float t = 0;
         cudaEventElapsedTime(&t, e0, e1);
         ms = std::min(ms, double(t));
      }
      return FMM_OK;
   };
   auto up = [&]() { return P.fp64 ? upwardT<double>(P, st) : upwardT<float>(P, st); };
   auto down = [&]() { return P.fp64 ? downwardT<double>(P, st) : downwardT<float>(P, st); };
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   auto near = [&]() { return P.fp64 ? evaluateT<double>(P, 1.0, 1, st) : evaluateT<float>(P, 1.0, 1, st); };
   fmm_tuning best{};
   do
   {
      s = P.outB.reserve(es * 3 * std::max<int64_t>(P.m, 1));
      if(s != FMM_OK) break;
      // P2M variant
      double bestMs = 1e300;
      for(int cv : {0, 16, 32})
      {
         P.p2mChunk = cv;
         double ms;
         if((s = timePhase(up, ms)) != FMM_OK) break;
         if(ms < bestMs) { bestMs = ms; best.p2m_chunk = cv; best.ms_upward = ms; }
      }
      if(s != FMM_OK) break;
      P.p2mChunk = best.p2m_chunk;
      // tensor-core M2L K chunk (CUDA-core and FP64 plans have one shape)
      bestMs = 1e300;
      const bool tc = !P.fp64 && P.cfg.m2l_mode != FMM_M2L_SIMT;
      for(int kc : {64, 32})
      {
         if(!tc && kc == 32) continue;
         P.tcKChunk = kc;
         double ms;
         if((s = timePhase(down, ms)) != FMM_OK) break;
         if(ms < bestMs) { bestMs = ms; best.m2l_k_chunk = kc; best.ms_downward = ms; }
      }
      if(s != FMM_OK) break;
      P.tcKChunk = best.m2l_k_chunk;
      // leave the plan's locals from a run of the chosen variant
      if((s = down()) != FMM_OK) break;
      // near-field tile
      bestMs = 1e300;
      for(int ts : {256, 128})
      {
         P.nearTile = ts;
         double ms;
         if((s = timePhase(near, ms)) != FMM_OK) break;
         if(ms < bestMs) { bestMs = ms; best.near_tile = ts; best.ms_near = ms; }
      }
      if(s != FMM_OK) break;
      P.nearTile = best.near_tile;
      FMM_CUDA(cudaStreamSynchronize(st));
   } while(false);
   cudaEventDestroy(e0);
   cudaEventDestroy(e1);
   FMM_TRY(s);
   FMM_TRY(pipeCheck(P, st, "fmm_autotune"));
   {
      std::lock_guard<std::mutex> lock(g_tuneMutex);
      g_tuned[tuneKey(P.cfg)] = best;
   }
   if(out) *out = best;
   return FMM_OK;
}

fmm_status fmm_batch_set_coils(fmm_plan* plan, int64_t ncoils, const int64_t* src_offsets, const int64_t* tgt_offsets)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(ncoils == 0)
   {
      P.batch = false;
      P.nCoils = 1;
   }
   else
   {
      if(P.bem) return setError(FMM_E_INVALID, "fmm_batch_set_coils: not available for BEM sources");
      if(ncoils < 0 || ncoils > FMM_MAX_COILS)
         return setError(FMM_E_INVALID, "fmm_batch_set_coils: %lld coils outside 0..%d", (long long)ncoils, FMM_MAX_COILS);
      if(!src_offsets || !tgt_offsets) return setError(FMM_E_INVALID, "fmm_batch_set_coils: null offsets");
      if(src_offsets[0] != 0 || tgt_offsets[0] != 0 || src_offsets[ncoils] != P.n || tgt_offsets[ncoils] != P.m)
         return setError(FMM_E_INVALID, "fmm_batch_set_coils: offsets must run from 0 to the source (%lld) and "
                                        "target (%lld) counts; set sources and targets first",
                         (long long)P.n, (long long)P.m);
      for(int64_t c = 0; c < ncoils; c++)
         if(src_offsets[c + 1] < src_offsets[c] || tgt_offsets[c + 1] < tgt_offsets[c])
            return setError(FMM_E_INVALID, "fmm_batch_set_coils: offsets decrease at coil %lld", (long long)c);
      P.srcOff.assign(src_offsets, src_offsets + ncoils + 1);
      P.tgtOff.assign(tgt_offsets, tgt_offsets + ncoils + 1);
      P.nCoils = int(ncoils);
      P.batch = true;
   }
   P.treeReady = P.upReady = P.downReady = false;
   P.dropGraph();
   return FMM_OK;
}

fmm_status fmm_batch_partition(int64_t ncoils, const int64_t* src_offsets, const int64_t* tgt_offsets, int nparts,
                               int* part)
{
   if(ncoils < 0 || ncoils > FMM_MAX_COILS || nparts < 1)
      return setError(FMM_E_INVALID, "fmm_batch_partition: %lld coils, %d parts", (long long)ncoils, nparts);
   if(ncoils > 0 && (!src_offsets || !tgt_offsets || !part)) return setError(FMM_E_INVALID, "fmm_batch_partition: null argument");
   std::vector<std::pair<int64_t, int64_t>> work(static_cast<size_t>(ncoils));   // (-work, coil): decreasing work, then coil
   for(int64_t c = 0; c < ncoils; c++)
   {
      const int64_t ns = src_offsets[c + 1] - src_offsets[c], nt = tgt_offsets[c + 1] - tgt_offsets[c];
      if(ns < 0 || nt < 0) return setError(FMM_E_INVALID, "fmm_batch_partition: offsets decrease at coil %lld", (long long)c);
      work[size_t(c)] = {-(ns + nt), c};
   }
   std::sort(work.begin(), work.end());
   std::vector<int64_t> load(static_cast<size_t>(nparts), 0);
   for(const auto& wc : work)
   {
      int best = 0;
      for(int q = 1; q < nparts; q++)
         if(load[size_t(q)] < load[size_t(best)]) best = q;
      part[wc.second] = best;
      load[size_t(best)] -= wc.first;
   }
   return FMM_OK;
}

fmm_status fmm_update_sources(fmm_plan* plan, const void* w, const void* J, int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.treeReady) return setError(FMM_E_INVALID, "fmm_update_sources: the tree is not built");
   if(P.n > 0 && !w) return setError(FMM_E_INVALID, "fmm_update_sources: null weights");
   if(P.bem) return setError(FMM_E_INVALID, "fmm_update_sources: set BEM sources again with fmm_set_bem_sources");
   if((J != nullptr) != P.hasJ)
      return setError(FMM_E_INVALID, "fmm_update_sources: J must be given exactly when the sources were set with J");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(st));   // fmm_set_sources_async copies in flight
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   if(P.n)
   {
      FMM_CUDA(cudaMemcpyAsync(P.srcW, w, es * P.n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
      if(J)
         FMM_CUDA(cudaMemcpyAsync(P.srcJ, J, es * 3 * P.n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  st));
   }
   FMM_TRY(P.fp64 ? regatherStrengthsT<double>(P, st) : regatherStrengthsT<float>(P, st));
   if(!on_device) FMM_CUDA(cudaStreamSynchronize(st));
   P.upReady = P.downReady = false;
   return FMM_OK;
}

fmm_status fmm_graph_capture(fmm_plan* plan, int want, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   const bool tcMode = !P.fp64 && P.cfg.m2l_mode != FMM_M2L_SIMT;
   if(!P.treeReady || P.opOrder != P.p || (tcMode && P.opImgOrder < 0))
      return setError(FMM_E_INVALID, "fmm_graph_capture: run fmm_solve first");
   if(want < 1 || want > 3) return setError(FMM_E_INVALID, "want must be 1, 2 or 3");
   DeviceGuard g(P.cfg.device);
   P.dropGraph();
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(P.outB.reserve(es * 3 * std::max<int64_t>(P.m, 1)));
   FMM_TRY(P.outA.reserve(es * 3 * std::max<int64_t>(P.m, 1)));
   // warm the lazily built state (operator image, buffers) eagerly, then capture on a private stream
   cudaStream_t user = (cudaStream_t)stream;
   FMM_TRY(P.waitSourceInputs(user));   // fmm_set_sources_async copies in flight
   FMM_CUDA(cudaStreamSynchronize(user));
   cudaStream_t cs = nullptr;
   FMM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
   fmm_status s = FMM_OK;
   cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
   if(e != cudaSuccess) s = setError(FMM_E_CUDA, "fmm_graph_capture: %s", cudaGetErrorString(e));
   else
   {
      P.capturing = true;
      s = P.fp64 ? upwardT<double>(P, cs) : upwardT<float>(P, cs);
      if(s == FMM_OK) s = P.fp64 ? downwardT<double>(P, cs) : downwardT<float>(P, cs);
      if(s == FMM_OK) s = P.fp64 ? evaluateT<double>(P, 1.0, want, cs) : evaluateT<float>(P, 1.0, want, cs);
      P.capturing = false;
      cudaGraph_t gr = nullptr;
      e = cudaStreamEndCapture(cs, &gr);
      if(s == FMM_OK && e != cudaSuccess) s = setError(FMM_E_CUDA, "fmm_graph_capture: %s", cudaGetErrorString(e));
      if(s == FMM_OK)
      {
         e = cudaGraphInstantiate(&P.graphExec, gr, 0);
         if(e != cudaSuccess) s = setError(FMM_E_CUDA, "fmm_graph_capture: instantiate: %s", cudaGetErrorString(e));
         P.graph = gr;
      }
      else if(gr)
         cudaGraphDestroy(gr);
   }
   cudaGetLastError();
   cudaStreamDestroy(cs);
   if(s != FMM_OK)
   {
      P.dropGraph();
      return s;
   }
   P.graphWant = want;
   return FMM_OK;
}

fmm_status fmm_graph_launch(fmm_plan* plan, double current, void* out_B, void* out_A, int on_device, void* stream)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   Plan& P = plan->P;
   if(!P.graphExec) return setError(FMM_E_INVALID, "fmm_graph_launch: no captured graph (fmm_graph_capture)");
   if(((P.graphWant & 1) && !out_B) || ((P.graphWant & 2) && !out_A))
      return setError(FMM_E_INVALID, "fmm_graph_launch: null output buffer");
   DeviceGuard g(P.cfg.device);
   cudaStream_t st = (cudaStream_t)stream;
   const size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(pipeBegin(P, st));
   FMM_CUDA(cudaGraphLaunch(P.graphExec, st));
   const int64_t cnt = 3 * P.m;
   if(on_device)
   {
      if(P.graphWant & 1) FMM_TRY(P.fp64 ? scaleCopyT<double>(P, P.outB.ptr, out_B, cnt, current, st)
                                         : scaleCopyT<float>(P, P.outB.ptr, out_B, cnt, current, st));
      if(P.graphWant & 2) FMM_TRY(P.fp64 ? scaleCopyT<double>(P, P.outA.ptr, out_A, cnt, current, st)
                                         : scaleCopyT<float>(P, P.outA.ptr, out_A, cnt, current, st));
      return FMM_OK;
   }
   // host outputs: scale in place on the device, copy back, and check the error word
   if(P.graphWant & 1) FMM_TRY(P.fp64 ? scaleCopyT<double>(P, P.outB.ptr, P.outB.ptr, cnt, current, st)
                                      : scaleCopyT<float>(P, P.outB.ptr, P.outB.ptr, cnt, current, st));
   if(P.graphWant & 2) FMM_TRY(P.fp64 ? scaleCopyT<double>(P, P.outA.ptr, P.outA.ptr, cnt, current, st)
                                      : scaleCopyT<float>(P, P.outA.ptr, P.outA.ptr, cnt, current, st));
   if(P.graphWant & 1) FMM_CUDA(cudaMemcpyAsync(out_B, P.outB.ptr, es * cnt, cudaMemcpyDeviceToHost, st));
   if(P.graphWant & 2) FMM_CUDA(cudaMemcpyAsync(out_A, P.outA.ptr, es * cnt, cudaMemcpyDeviceToHost, st));
   return pipeCheck(P, st, "fmm_graph_launch");
}

fmm_status fmm_set_wait_limit(fmm_plan* plan, double seconds)
{
   if(!plan) return setError(FMM_E_INVALID, "null plan");
   if(!(seconds > 0) || seconds > 60)
      return setError(FMM_E_INVALID, "fmm_set_wait_limit: %g s outside (0, 60]", seconds);
   Plan& P = plan->P;
   P.tcWaitNs = std::max<uint64_t>(1, uint64_t(seconds * 1e9));
   P.dropGraph();   // a captured graph holds the old limit
   return FMM_OK;
}

fmm_status fmm_get_stats(const fmm_plan* plan, fmm_stats* stats)
{
   if(!plan || !stats) return setError(FMM_E_INVALID, "null argument");
   const Plan& P = plan->P;
   DeviceGuard g(P.cfg.device);
   fmm_stats s{};
   if(P.downReady) cudaEventSynchronize(P.ev[5]);
   s.ms_tree = elapsed(P.ev[0], P.ev[1]);
   s.ms_upward = elapsed(P.ev[1], P.ev[2]);
   s.ms_m2l = elapsed(P.ev[2], P.ev[3]);
   s.ms_downward = elapsed(P.ev[2], P.ev[4]);
   s.ms_near = elapsed(P.ev[4], P.ev[5]);
   s.ms_total = elapsed(P.ev[0], P.ev[5]);
   if(P.adjointDone)
   {
      cudaEventSynchronize(P.ev[7]);
      s.ms_adjoint = elapsed(P.ev[6], P.ev[7]);
   }
   s.nodes = P.tree.nNodes;
   s.levels = P.tree.nLevels;
   s.p2p_pairs = P.nP2P;
   s.v_pairs = P.nV;
   if(P.treeReady && P.nearCounts.ptr)
   {
      unsigned long long c[2] = {0, 0};
      if(cudaMemcpy(c, P.nearCounts.ptr, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess)
      {
         s.leaves = int64_t(c[0]);
         s.p2p_interactions = int64_t(c[1]);
      }
   }
   s.n_sources = P.n;
   s.n_targets = P.m;
   s.coils = P.nCoils;
   s.m2l_tiles = 0;
   s.m2l_tile_offsets = 0;
   if(P.downReady && P.tcTiles > 0 && P.tcCounters.ptr && !P.fp64 && P.cfg.m2l_mode != FMM_M2L_SIMT)
   {
      unsigned long long c[2] = {0, 0};
      cudaEventSynchronize(P.ev[4]);
      if(cudaMemcpy(c, P.tcCounters.ptr, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess)
      {
         s.m2l_tiles = P.tcTiles;
         s.m2l_tile_offsets = int64_t(c[1]);
      }
      else cudaGetLastError();
   }
   *stats = s;
   return FMM_OK;
}

fmm_status fmm_get_operator(fmm_plan* plan, int kind, int index, double* out)
{
   if(!plan || !out) return setError(FMM_E_INVALID, "null argument");
   Plan& P = plan->P;
   DeviceGuard g(P.cfg.device);
   if(kind < 0 || kind > 2) return setError(FMM_E_INVALID, "kind must be 0, 1 or 2");
   const int L = P.L;
   int slot = index;
   if(kind == 2)
   {
      int ox = index % 7 - 3, oy = (index / 7) % 7 - 3, oz = index / 49 - 3;
      if(index < 0 || index >= NOFF || (abs(ox) <= 1 && abs(oy) <= 1 && abs(oz) <= 1))
         return setError(FMM_E_INVALID, "offset index %d is not an M2L offset", index);
      int k = 0;
      for(int o = 0; o < index; o++)
      {
         int ax = o % 7 - 3, ay = (o / 7) % 7 - 3, az = o / 49 - 3;
         if(!(abs(ax) <= 1 && abs(ay) <= 1 && abs(az) <= 1)) k++;
      }
      slot = k;
   }
   else if(index < 0 || index > 7) return setError(FMM_E_INVALID, "octant must be 0..7");
   FMM_TRY(buildOperators(P, 0));
   const DevBuf& b = kind == 0 ? P.opM2M64 : kind == 1 ? P.opL2L64 : P.opM2L64;
   FMM_CUDA(cudaMemcpy(out, (const double*)b.ptr + int64_t(slot) * L * L, sizeof(double) * L * L,
                       cudaMemcpyDeviceToHost));
   return FMM_OK;
}


fmm_status fmm_add_vectors(const float* a, const float* b, float* c, int64_t n)
{
   if(n < 0 || (n > 0 && (!a || !b || !c))) return setError(FMM_E_INVALID, "fmm_add_vectors: bad arguments");
   if(n == 0) return FMM_OK;
   DevBuf da, db, dc;
   fmm_status s = da.reserve(sizeof(float) * n);
   if(s == FMM_OK) s = db.reserve(sizeof(float) * n);
   if(s == FMM_OK) s = dc.reserve(sizeof(float) * n);
   if(s == FMM_OK)
   {
      cudaError_t e = cudaMemcpy(da.ptr, a, sizeof(float) * n, cudaMemcpyHostToDevice);
      if(e == cudaSuccess) e = cudaMemcpy(db.ptr, b, sizeof(float) * n, cudaMemcpyHostToDevice);
      if(e == cudaSuccess)
      {
         kAdd<<<int((n + 255) / 256), 256>>>((const float*)da.ptr, (const float*)db.ptr, (float*)dc.ptr, n);
         e = cudaGetLastError();
      }
      if(e == cudaSuccess) e = cudaMemcpy(c, dc.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost);
      if(e != cudaSuccess) s = setError(FMM_E_CUDA, "fmm_add_vectors: %s", cudaGetErrorString(e));
   }
   da.release();
   db.release();
   dc.release();
   return s;
}

}  // extern "C"
