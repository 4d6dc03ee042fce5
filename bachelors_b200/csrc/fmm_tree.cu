// Device octree and interaction lists.
//
// Replaces the reference's pointer octrees and its dual-tree map building
// (FMM/FMMGPU/quadrature_octree.cpp:23-97, calculation_point_octree.cpp:26-97,
// fast_multipole_solver.cpp:105-184) with one Morton-ordered octree over sources and targets,
// built level by level on the device:
//   keys      Morton codes, up to 21 bits per axis, x in the lowest bit of each triple, with
//             the coil index above them when several independent coils share the plan
//   sort      CUB radix sort of (key, index) for sources and for targets
//   nodes     one root per coil (its own bounding cube); a node at level l holds the points
//             whose key prefix matches; it splits when it holds more than `cap` sources or more
//             than `capT` targets (and l < the deepest key level); its children are the non-empty
//             octants, found by binary search in the sorted keys
//   lists     Col (same-level adjacent), A (coarser adjacent leaves), X (coarser non-adjacent
//             leaves), V (same-level M2L sources, dense table over the 316 offsets), and for
//             each target leaf the CSR list of source nodes whose points it sums directly.
#include <cub/cub.cuh>

#include "fmm_internal.cuh"

namespace fmm {

// ------------------------------------------------------------------------------ bounding box
template <class T>
__global__ void kBBox(const T* __restrict__ a, int64_t na, const T* __restrict__ b, int64_t nb, double* partial)
{
   double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
   int64_t n = na + nb;
   for(int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
   {
      const T* p = i < na ? a + 3 * i : b + 3 * (i - na);
      for(int d = 0; d < 3; d++)
      {
         double v = double(p[d]);
         lo[d] = fmin(lo[d], v);
         hi[d] = fmax(hi[d], v);
      }
   }
   typedef cub::BlockReduce<double, 256> BR;
   __shared__ typename BR::TempStorage tmp;
   for(int d = 0; d < 3; d++)
   {
      double l = BR(tmp).Reduce(lo[d], cub::Min());
      __syncthreads();
      double h = BR(tmp).Reduce(hi[d], cub::Max());
      __syncthreads();
      if(threadIdx.x == 0) { partial[6 * blockIdx.x + d] = l; partial[6 * blockIdx.x + 3 + d] = h; }
   }
}

// Root cube around a bounding box: center = (lo + hi) / 2, H = max half extent * (1 + 2^-20) + 1e-300;
// keys resolve 2^maxLevel cells per axis.
__device__ void setRootBox(const double lo[3], const double hi[3], int maxLevel, RootBox* root)
{
   double H = 0;
   for(int d = 0; d < 3; d++)
   {
      root->center[d] = 0.5 * (lo[d] + hi[d]);
      H = fmax(H, hi[d] - lo[d]);
   }
   H = 0.5 * H;
   H = __dadd_rn(__dmul_rn(H, 1.0 + 9.5367431640625e-07), 1e-300);
   root->H = H;
   for(int d = 0; d < 3; d++) root->lo[d] = root->center[d] - H;
   root->scale = double(int64_t(1) << maxLevel) / (2.0 * H);
}

__global__ void kRootFromBBox(const double* partial, int nblocks, int maxLevel, RootBox* root)
{
   if(threadIdx.x != 0 || blockIdx.x != 0) return;
   double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
   for(int b = 0; b < nblocks; b++)
      for(int d = 0; d < 3; d++)
      {
         lo[d] = fmin(lo[d], partial[6 * b + d]);
         hi[d] = fmax(hi[d], partial[6 * b + 3 + d]);
      }
   setRootBox(lo, hi, maxLevel, root);
}

__global__ void kRootFromConfig(double cx, double cy, double cz, double H, int maxLevel, RootBox* root)
{
   if(threadIdx.x != 0 || blockIdx.x != 0) return;
   root->center[0] = cx; root->center[1] = cy; root->center[2] = cz;
   root->H = H;
   for(int d = 0; d < 3; d++) root->lo[d] = root->center[d] - H;
   root->scale = double(int64_t(1) << maxLevel) / (2.0 * H);
}

// One block per coil: the cube around that coil's sources and targets (an empty coil gets a unit cube).
template <class T>
__global__ void kRootsPerCoil(const T* __restrict__ src, const T* __restrict__ tgt, const int* __restrict__ srcOff,
                              const int* __restrict__ tgtOff, int maxLevel, RootBox* roots)
{
   const int c = blockIdx.x;
   const int64_t sa = srcOff[c], sn = srcOff[c + 1] - sa, ta = tgtOff[c], tn = tgtOff[c + 1] - ta;
   double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
   for(int64_t i = threadIdx.x; i < sn + tn; i += blockDim.x)
   {
      const T* p = i < sn ? src + 3 * (sa + i) : tgt + 3 * (ta + i - sn);
      for(int d = 0; d < 3; d++)
      {
         double v = double(p[d]);
         lo[d] = fmin(lo[d], v);
         hi[d] = fmax(hi[d], v);
      }
   }
   typedef cub::BlockReduce<double, 256> BR;
   __shared__ typename BR::TempStorage tmp;
   __shared__ double blo[3], bhi[3];
   for(int d = 0; d < 3; d++)
   {
      double l = BR(tmp).Reduce(lo[d], cub::Min());
      __syncthreads();
      double h = BR(tmp).Reduce(hi[d], cub::Max());
      __syncthreads();
      if(threadIdx.x == 0) { blo[d] = l; bhi[d] = h; }
   }
   if(threadIdx.x != 0) return;
   if(sn + tn == 0)
      for(int d = 0; d < 3; d++) { blo[d] = -1; bhi[d] = 1; }
   setRootBox(blo, bhi, maxLevel, roots + c);
}

// ------------------------------------------------------------------------------ Morton keys
__device__ __forceinline__ uint64_t spread3(uint64_t v)
{
   v &= 0x1fffff;
   v = (v | v << 32) & 0x1f00000000ffffull;
   v = (v | v << 16) & 0x1f0000ff0000ffull;
   v = (v | v << 8) & 0x100f00f00f00f00full;
   v = (v | v << 4) & 0x10c30c30c30c30c3ull;
   v = (v | v << 2) & 0x1249249249249249ull;
   return v;
}

__device__ __forceinline__ int64_t quantize(double x, double lo, double scale, int maxLevel)
{
   double u = floor(__dmul_rn(__dsub_rn(x, lo), scale));
   u = fmax(u, 0.0);
   u = fmin(u, double((int64_t(1) << maxLevel) - 1));
   return int64_t(u);
}

// Key of point i: its coil (the segment of `off` that holds i) above the Morton code of its
// cell in that coil's root cube.
template <class T>
__global__ void kKeys(const T* __restrict__ xyz, int64_t n, const RootBox* __restrict__ roots,
                      const int* __restrict__ off, int nCoils, int maxLevel, uint64_t* keys, int* idx)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i >= n) return;
   int lo = 0, hi = nCoils;  // largest c with off[c] <= i
   while(hi - lo > 1)
   {
      int mid = (lo + hi) >> 1;
      if(off[mid] <= i) lo = mid;
      else hi = mid;
   }
   const RootBox& rb = roots[lo];
   int64_t ux = quantize(double(xyz[3 * i]), rb.lo[0], rb.scale, maxLevel);
   int64_t uy = quantize(double(xyz[3 * i + 1]), rb.lo[1], rb.scale, maxLevel);
   int64_t uz = quantize(double(xyz[3 * i + 2]), rb.lo[2], rb.scale, maxLevel);
   keys[i] = (uint64_t(lo) << (3 * maxLevel)) | spread3(uint64_t(ux)) | (spread3(uint64_t(uy)) << 1) |
             (spread3(uint64_t(uz)) << 2);
   idx[i] = int(i);
}

template <class T>
__global__ void kGatherSources(const T* __restrict__ xyz, const T* __restrict__ w, const T* __restrict__ J,
                               const T* __restrict__ sigma, const int* __restrict__ order, int64_t n,
                               typename Vec4<T>::type* pos, typename Vec4<T>::type* q)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i >= n) return;
   int64_t s = order[i];
   T x = xyz[3 * s], y = xyz[3 * s + 1], z = xyz[3 * s + 2];
   T jx, jy, jz;
   if(J) { jx = J[3 * s]; jy = J[3 * s + 1]; jz = J[3 * s + 2]; }
   else
   {
      // perp(q).normalized() (FMM/FMMGPU/vector3.cu:154-204): (-y, x, 0) / |(-y, x, 0)|
      T l = sqrt(x * x + y * y);
      if(l != T(0)) { jx = -y / l; jy = x / l; }
      else { jx = T(0); jy = T(0); }
      jz = T(0);
   }
   // (pos or q null: that half only, for strengths that arrive after the points)
   if(pos) pos[i] = {x, y, z, T(0)};
   if(!q) return;
   T ww = w[s];
   // the fourth lane carries w sigma for BEM sources (fmm_bem.cu), zero otherwise
   q[i] = {ww * jx, ww * jy, ww * jz, sigma ? ww * sigma[s] : T(0)};
}

template <class T>
__global__ void kGatherTargets(const T* __restrict__ xyz, const int* __restrict__ order, int64_t m,
                               typename Vec4<T>::type* pos)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i >= m) return;
   int64_t s = order[i];
   pos[i] = {xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2], T(0)};
}

// ------------------------------------------------------------------------------ nodes
// Root c spans its coil's segments of the sorted sources and targets (the sort is by coil first).
__global__ void kInitRoots(Tree t, int nCoils, const int* __restrict__ srcOff, const int* __restrict__ tgtOff)
{
   int c = blockIdx.x * blockDim.x + threadIdx.x;
   if(c >= nCoils) return;
   t.key[c] = uint64_t(c); t.level[c] = 0; t.ix[c] = t.iy[c] = t.iz[c] = 0;
   t.s0[c] = srcOff[c]; t.s1[c] = srcOff[c + 1]; t.t0[c] = tgtOff[c]; t.t1[c] = tgtOff[c + 1];
   t.parent[c] = -1; t.child0[c] = -1; t.nchild[c] = 0;
}

__device__ __forceinline__ int lowerBound(const uint64_t* __restrict__ keys, int a, int b, uint64_t v)
{
   while(a < b)
   {
      int mid = (a + b) >> 1;
      if(keys[mid] < v) a = mid + 1;
      else b = mid;
   }
   return a;
}

// Node i (the j-th of its level): decide the split and find the 8 children's ranges (bounds row j);
// returns the number of non-empty children.
__device__ int childBounds(Tree& t, int i, int j, int level, int maxLevel, int cap, int capT,
                           const uint64_t* __restrict__ skeys, const uint64_t* __restrict__ tkeys, int* bounds)
{
   int s0 = t.s0[i], s1 = t.s1[i], t0 = t.t0[i], t1 = t.t1[i];
   t.child0[i] = -1;
   t.nchild[i] = 0;
   if(!((s1 - s0 > cap || t1 - t0 > capT) && level < maxLevel)) return 0;
   uint64_t key = t.key[i];
   int shift = 3 * (maxLevel - level - 1);
   int sb[9], tb[9];
   for(int c = 0; c < 8; c++)
   {
      uint64_t bound = ((key << 3) + uint64_t(c)) << shift;
      sb[c] = c == 0 ? s0 : lowerBound(skeys, s0, s1, bound);
      tb[c] = c == 0 ? t0 : lowerBound(tkeys, t0, t1, bound);
   }
   sb[8] = s1; tb[8] = t1;
   int k = 0;
   for(int c = 0; c < 8; c++)
   {
      bounds[18 * j + c] = sb[c];
      bounds[18 * j + 9 + c] = tb[c];
      if(sb[c + 1] - sb[c] + tb[c + 1] - tb[c] > 0) k++;
   }
   bounds[18 * j + 8] = s1;
   bounds[18 * j + 17] = t1;
   return k;
}

// For nodes [a, b) of `level`: decide the split and find the 8 children's ranges.
__global__ void kCountChildren(Tree t, int a, int b, int level, int maxLevel, int cap, int capT,
                               const uint64_t* __restrict__ skeys, const uint64_t* __restrict__ tkeys, int* bounds,
                               int* cnt)
{
   int i = a + blockIdx.x * blockDim.x + threadIdx.x;
   if(i >= b) return;
   cnt[i - a] = childBounds(t, i, i - a, level, maxLevel, cap, capT, skeys, tkeys, bounds);
}

// The k children of node i (the j-th of its level), numbered from c0.
__device__ void makeChildrenOf(Tree& t, int i, int j, int level, int c0, int k, const int* __restrict__ bounds)
{
   t.child0[i] = c0;
   t.nchild[i] = k;
   const int* sb = bounds + 18 * j;
   const int* tb = sb + 9;
   uint64_t key = t.key[i];
   int n = 0;
   for(int c = 0; c < 8; c++)
   {
      if(sb[c + 1] - sb[c] + tb[c + 1] - tb[c] == 0) continue;
      int ch = c0 + n++;
      t.key[ch] = (key << 3) | uint64_t(c);
      t.level[ch] = level + 1;
      t.ix[ch] = 2 * t.ix[i] + (c & 1);
      t.iy[ch] = 2 * t.iy[i] + ((c >> 1) & 1);
      t.iz[ch] = 2 * t.iz[i] + ((c >> 2) & 1);
      t.s0[ch] = sb[c]; t.s1[ch] = sb[c + 1];
      t.t0[ch] = tb[c]; t.t1[ch] = tb[c + 1];
      t.parent[ch] = i;
      t.child0[ch] = -1;
      t.nchild[ch] = 0;
   }
}

__global__ void kMakeChildren(Tree t, int a, int b, int level, int next, const int* __restrict__ bounds,
                              const int* __restrict__ cnt, const int* __restrict__ off)
{
   int i = a + blockIdx.x * blockDim.x + threadIdx.x;
   if(i >= b) return;
   int j = i - a;
   if(cnt[j] == 0) return;
   makeChildrenOf(t, i, j, level, next + off[j], cnt[j], bounds);
}

// ------------------------------------------------------------------------------ persistent level build
// All levels in one cooperative launch (every block resident). Per level the blocks take work items of LB_T
// consecutive nodes from the level's queue (an atomic counter, so items start in order). An item counts its
// nodes' children, publishes its total, finds the children numbered before it by a decoupled look-back over
// the items before it (each has already published at least its own total), and builds its children at once.
// One grid barrier per level; the last item publishes the next level's range, and the host reads the level
// starts once, after the launch, instead of once per level.
constexpr int LB_T = 256;

struct LevelBuildState
{
   unsigned bar[64];             // grid barrier: arrivals in bar[0], generation in bar[32] (another cache line)
   int grab[MAXLEVEL];           // per level: next work item
   int levelStart[MAXLEVEL + 2];
   int nLevels;
   int overflow;                 // a level did not fit in the node arrays
};

__device__ __forceinline__ int ldAcquire(const int* p)
{
   int v;
   asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ unsigned ldAcquireU(const unsigned* p)
{
   unsigned v;
   asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ unsigned long long ldAcquireU64(const unsigned long long* p)
{
   unsigned long long v;
   asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ void stReleaseU64(unsigned long long* p, unsigned long long v)
{
   asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t treeTimer()
{
   uint64_t t;
   asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
   return t;
}

// Grid barrier of a cooperative launch: arrivals in bar[0], generation in bar[32] (its own cache line, so the
// waiting blocks' polls do not contend with the arrivals). Bounded: a block that waits longer than limitNs
// raises ERR_TIMEOUT and every thread of it returns false.
__device__ bool gridBarrier(unsigned* bar, int* err, uint64_t limitNs)
{
   __shared__ int ok;
   __syncthreads();
   if(threadIdx.x == 0)
   {
      ok = 1;
      const unsigned g = ldAcquireU(bar + 32);
      __threadfence();
      if(atomicAdd(bar, 1u) == gridDim.x - 1)
      {
         atomicExch(bar, 0u);
         __threadfence();
         atomicAdd(bar + 32, 1u);
      }
      else
      {
         const uint64_t t0 = treeTimer();
         while(ldAcquireU(bar + 32) == g)
         {
            if(treeTimer() - t0 > limitNs)
            {
               atomicOr(err, ERR_TIMEOUT);
               ok = 0;
               break;
            }
            __nanosleep(200);
         }
      }
      __threadfence();
   }
   __syncthreads();
   return ok != 0;
}

// Look-back words, one per work item: (level + 1) << 40 | state << 32 | value, state 1 = the item's own
// total, 2 = its total plus everything before it; a word of another level reads as "not yet".
__device__ __forceinline__ unsigned long long lbWord(int level, int state, int value)
{
   return (unsigned long long)(level + 1) << 40 | (unsigned long long)state << 32 | unsigned(value);
}

__global__ void __launch_bounds__(LB_T, 6) kBuildLevels(Tree t, int maxLevel, int cap, int capT,
                                                        const uint64_t* __restrict__ skeys,
                                                        const uint64_t* __restrict__ tkeys, int* bounds,
                                                        unsigned long long* look, int64_t capNodes,
                                                        LevelBuildState* S, int* err, uint64_t limitNs)
{
   typedef cub::BlockScan<int, LB_T> Scan;
   __shared__ typename Scan::TempStorage scanTmp;
   __shared__ int item, before, failed;
   const int tid = threadIdx.x;
   int nLev = 1;
   if(tid == 0) failed = 0;
   for(int level = 0; level < maxLevel; level++)
   {
      const int a = ldAcquire(&S->levelStart[level]), b = ldAcquire(&S->levelStart[level + 1]);
      if(b <= a) break;
      const int nItems = (b - a + LB_T - 1) / LB_T;
      while(true)
      {
         if(tid == 0) item = atomicAdd(&S->grab[level], 1);
         __syncthreads();
         const int it = item;
         if(it >= nItems) break;
         const int i = a + it * LB_T + tid;
         const int k = i < b ? childBounds(t, i, i - a, level, maxLevel, cap, capT, skeys, tkeys, bounds) : 0;
         int ex, total;
         Scan(scanTmp).ExclusiveSum(k, ex, total);
         if(tid == 0)
         {
            // publish this item's total, then add up the items before it
            int sum = 0;
            if(it == 0) stReleaseU64(&look[0], lbWord(level, 2, total));
            else
            {
               stReleaseU64(&look[it], lbWord(level, 1, total));
               const uint64_t t0 = treeTimer();
               for(int j = it - 1; j >= 0;)
               {
                  const unsigned long long w = ldAcquireU64(&look[j]);
                  const int st = int(w >> 32) & 0xFF;
                  if(int(w >> 40) == level + 1 && st != 0)
                  {
                     sum += int(unsigned(w));
                     if(st == 2) break;
                     j--;
                     continue;
                  }
                  if(treeTimer() - t0 > limitNs)
                  {
                     atomicOr(err, ERR_TIMEOUT);
                     failed = 1;
                     break;
                  }
               }
               stReleaseU64(&look[it], lbWord(level, 2, sum + total));
            }
            before = sum;
            // children that would not fit are not built; the host grows the arrays and builds again
            if(int64_t(b) + sum + total > capNodes) S->overflow = 1;
            if(it == nItems - 1) S->levelStart[level + 2] = int(std::min<int64_t>(int64_t(b) + sum + total, capNodes));
         }
         __syncthreads();
         const int64_t c0 = int64_t(b) + before + ex;
         if(k > 0 && c0 + k <= capNodes) makeChildrenOf(t, i, i - a, level, int(c0), k, bounds);
         __syncthreads();
      }
      if(!gridBarrier(S->bar, err, limitNs) || failed) return;
      if(ldAcquire(&S->overflow)) break;
      const int nb = ldAcquire(&S->levelStart[level + 2]);
      if(nb == b) break;   // no children: the tree ends here
      nLev = level + 2;
   }
   if(blockIdx.x == 0 && tid == 0) S->nLevels = nLev;
}

// ------------------------------------------------------------------------------ lists
__device__ __forceinline__ bool adjacentNodes(const Tree& t, int a, int b)
{
   int la = t.level[a], lb = t.level[b];
   int c = la <= lb ? a : b, f = la <= lb ? b : a;
   int sh = abs(lb - la);
   int64_t s = int64_t(1) << sh;
   int64_t ci[3] = {t.ix[c], t.iy[c], t.iz[c]}, fi[3] = {t.ix[f], t.iy[f], t.iz[f]};
   for(int d = 0; d < 3; d++)
      if(fi[d] < ci[d] * s - 1 || fi[d] > (ci[d] + 1) * s) return false;
   return true;
}

// Each root is its own only colleague: nothing links different coils.
__global__ void kInitRootLists(Lists L, int nCoils)
{
   int c = blockIdx.x * blockDim.x + threadIdx.x;
   if(c >= nCoils) return;
   L.col[int64_t(c) * COLCAP] = c; L.ncol[c] = 1; L.na[c] = 0; L.nx[c] = 0; L.nv[c] = 0;
   for(int k = 0; k < 316; k++) L.vtab[int64_t(c) * 316 + k] = -1;
}

// One thread per node D of a level >= 1; the parent's lists are complete.
__global__ void kListsLevel(Tree t, Lists L, int a, int b, int* err)
{
   int D = a + blockIdx.x * blockDim.x + threadIdx.x;
   if(D >= b) return;
   int P = t.parent[D];
   int ncol = 0, na = 0, nx = 0, nv = 0;
   int* vt = L.vtab + int64_t(D) * 316;   // preset to -1 for the whole tree before the levels
   const bool hasT = t.t1[D] > t.t0[D];
   auto coarse = [&](int S) {
      if(adjacentNodes(t, S, D))
      {
         if(na < ACAP) L.acoarse[int64_t(D) * ACAP + na] = S;
         else atomicOr(err, ERR_LIST_A);
         na++;
      }
      else
      {
         if(nx < XCAP) L.xl[int64_t(D) * XCAP + nx] = S;
         else atomicOr(err, ERR_LIST_X);
         nx++;
      }
   };
   for(int k = 0; k < L.ncol[P]; k++)
   {
      int C = L.col[int64_t(P) * COLCAP + k];
      int nc = t.nchild[C];
      if(nc == 0) { coarse(C); continue; }
      int c0 = t.child0[C];
      for(int e = 0; e < nc; e++)
      {
         int c = c0 + e;
         if(adjacentNodes(t, c, D))
         {
            if(ncol < COLCAP) L.col[int64_t(D) * COLCAP + ncol] = c;
            else atomicOr(err, ERR_LIST_COL);
            ncol++;
         }
         else if(hasT && t.s1[c] > t.s0[c])
         {
            int ox = t.ix[c] - t.ix[D], oy = t.iy[c] - t.iy[D], oz = t.iz[c] - t.iz[D];
            int o = d_m2lIndex[offsetIndex(ox, oy, oz)];
            if(o >= 0) { vt[o] = c; nv++; }
            else atomicOr(err, ERR_LIST_V);
         }
      }
   }
   for(int k = 0; k < L.na[P]; k++) coarse(L.acoarse[int64_t(P) * ACAP + k]);
   L.ncol[D] = min(ncol, COLCAP);
   L.na[D] = min(na, ACAP);
   L.nx[D] = min(nx, XCAP);
   L.nv[D] = nv;
}

// kListsLevel with one warp per node D: the lanes take the parent's colleagues (at most 27), their child counts
// make a list of candidate slots (a leaf colleague is one slot, otherwise one per child), and each pass
// classifies 32 candidates at once. Entries are appended by ballots in candidate order, so the colleague, A and
// X lists come out exactly as in kListsLevel (the V table is indexed by offset).
constexpr int LW_WARPS = 8;

__global__ void __launch_bounds__(32 * LW_WARPS) kListsLevelWarp(Tree t, Lists L, int a, int b, int* err)
{
   __shared__ int sC[LW_WARPS][32], sNc[LW_WARPS][32], sC0[LW_WARPS][32], sEx[LW_WARPS][33];
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
   const int D = a + blockIdx.x * LW_WARPS + w;
   if(D >= b) return;
   const int P = t.parent[D];
   int* vt = L.vtab + int64_t(D) * 316;   // preset to -1 for the whole tree before the levels
   const bool hasT = t.t1[D] > t.t0[D];
   const unsigned below = (1u << lane) - 1u;
   int ncol = 0, na = 0, nx = 0, nv = 0;
   // append this lane's entry (if any) to a list in lane order; returns the list's new length
   auto append = [&](bool has, int node, int* list, int cap, int count, int errBit) {
      const unsigned m = __ballot_sync(0xffffffffu, has);
      if(has)
      {
         const int pos = count + __popc(m & below);
         if(pos < cap) list[pos] = node;
         else atomicOr(err, errBit);
      }
      return count + __popc(m);
   };
   const int ncP = L.ncol[P];
   int C = -1, nc = 0, c0 = 0;
   if(lane < ncP)
   {
      C = L.col[int64_t(P) * COLCAP + lane];
      nc = t.nchild[C];
      c0 = t.child0[C];
   }
   const int slots = lane < ncP ? (nc > 0 ? nc : 1) : 0;
   int incl = slots;
   for(int d = 1; d < 32; d <<= 1)
   {
      const int v = __shfl_up_sync(0xffffffffu, incl, d);
      if(lane >= d) incl += v;
   }
   const int total = __shfl_sync(0xffffffffu, incl, 31);
   sC[w][lane] = C;
   sNc[w][lane] = nc;
   sC0[w][lane] = c0;
   sEx[w][lane] = incl - slots;
   if(lane == 0) sEx[w][32] = total;
   __syncwarp();
   int* colD = L.col + int64_t(D) * COLCAP;
   int* aD = L.acoarse + int64_t(D) * ACAP;
   int* xD = L.xl + int64_t(D) * XCAP;
   for(int base = 0; base < total; base += 32)
   {
      const int q = base + lane;
      bool isCol = false, isA = false, isX = false;
      int node = -1;
      if(q < total)
      {
         // the colleague owning slot q: the last lane j < ncP with sEx[j] <= q
         int lo = 0, hi = ncP;
         while(hi - lo > 1)
         {
            const int mid = (lo + hi) >> 1;
            if(sEx[w][mid] <= q) lo = mid;
            else hi = mid;
         }
         if(sNc[w][lo] == 0)
         {
            node = sC[w][lo];
            isA = adjacentNodes(t, node, D);
            isX = !isA;
         }
         else
         {
            node = sC0[w][lo] + (q - sEx[w][lo]);
            if(adjacentNodes(t, node, D)) isCol = true;
            else if(hasT && t.s1[node] > t.s0[node])
            {
               const int ox = t.ix[node] - t.ix[D], oy = t.iy[node] - t.iy[D], oz = t.iz[node] - t.iz[D];
               const int o = d_m2lIndex[offsetIndex(ox, oy, oz)];
               if(o >= 0)
               {
                  vt[o] = node;
                  nv++;
               }
               else atomicOr(err, ERR_LIST_V);
            }
         }
      }
      ncol = append(isCol, node, colD, COLCAP, ncol, ERR_LIST_COL);
      na = append(isA, node, aD, ACAP, na, ERR_LIST_A);
      nx = append(isX, node, xD, XCAP, nx, ERR_LIST_X);
   }
   // the parent's coarser adjacent leaves, after the colleagues' entries (as in kListsLevel)
   const int naP = L.na[P];
   for(int base = 0; base < naP; base += 32)
   {
      const int k = base + lane;
      bool isA = false, isX = false;
      int node = -1;
      if(k < naP)
      {
         node = L.acoarse[int64_t(P) * ACAP + k];
         isA = adjacentNodes(t, node, D);
         isX = !isA;
      }
      na = append(isA, node, aD, ACAP, na, ERR_LIST_A);
      nx = append(isX, node, xD, XCAP, nx, ERR_LIST_X);
   }
   for(int d = 16; d > 0; d >>= 1) nv += __shfl_xor_sync(0xffffffffu, nv, d);
   if(lane == 0)
   {
      L.ncol[D] = min(ncol, COLCAP);
      L.na[D] = min(na, ACAP);
      L.nx[D] = min(nx, XCAP);
      L.nv[D] = nv;
   }
}

// Statistics of the finished tree: out[0] += leaves, out[1] += direct (target, source) pairs the near
// field evaluates (targets of a leaf x points of its direct-list nodes, the self pairs included).
__global__ void kNearCounts(Tree t, int nNodes, const int* __restrict__ off, const int* __restrict__ list,
                            unsigned long long* out)
{
   unsigned long long leaves = 0, pairs = 0;
   for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < nNodes; n += gridDim.x * blockDim.x)
   {
      if(t.nchild[n] != 0) continue;
      leaves++;
      const int nt = t.t1[n] - t.t0[n];
      if(nt == 0) continue;
      long long ns = 0;
      for(int e = off[n]; e < off[n + 1]; e++)
      {
         const int S = list[e];
         ns += t.s1[S] - t.s0[S];
      }
      pairs += (unsigned long long)nt * (unsigned long long)ns;
   }
   for(int d = 16; d > 0; d >>= 1)
   {
      leaves += __shfl_down_sync(0xffffffffu, leaves, d);
      pairs += __shfl_down_sync(0xffffffffu, pairs, d);
   }
   if((threadIdx.x & 31) == 0)
   {
      atomicAdd(out, leaves);
      atomicAdd(out + 1, pairs);
   }
}

// Direct-interaction source nodes of every target leaf (count pass when out == nullptr).
__global__ void kP2PLists(Tree t, Lists L, int nNodes, const int* __restrict__ off, int* cnt, int* out, int* err)
{
   int T = blockIdx.x * blockDim.x + threadIdx.x;
   if(T >= nNodes) return;
   if(t.nchild[T] != 0 || t.t1[T] == t.t0[T]) { if(!out) cnt[T] = 0; return; }
   int k = 0;
   int base = out ? off[T] : 0;
   auto emit = [&](int S) {
      if(t.s1[S] == t.s0[S]) return;
      if(out) out[base + k] = S;
      k++;
   };
   // same-level leaf colleagues (including T itself) and coarser adjacent leaves
   for(int e = 0; e < L.ncol[T]; e++)
   {
      int C = L.col[int64_t(T) * COLCAP + e];
      if(t.nchild[C] == 0) emit(C);
   }
   for(int e = 0; e < L.na[T]; e++) emit(L.acoarse[int64_t(T) * ACAP + e]);
   // finer nodes below non-leaf colleagues: adjacent leaves, and non-adjacent nodes whose parent
   // is adjacent (the duals of A and X)
   int stack[256];
   int sp = 0;
   for(int e = 0; e < L.ncol[T]; e++)
   {
      int C = L.col[int64_t(T) * COLCAP + e];
      int nc = t.nchild[C];
      for(int c = 0; c < nc; c++)
      {
         if(sp < 256) stack[sp++] = t.child0[C] + c;
         else atomicOr(err, ERR_DFS);
      }
   }
   while(sp > 0)
   {
      int Q = stack[--sp];
      if(adjacentNodes(t, Q, T))
      {
         int nc = t.nchild[Q];
         if(nc == 0) emit(Q);
         else
            for(int c = 0; c < nc; c++)
            {
               if(sp < 256) stack[sp++] = t.child0[Q] + c;
               else atomicOr(err, ERR_DFS);
            }
      }
      else emit(Q);
   }
   // coarser non-adjacent leaves of T and of its ancestors
   for(int a = T; a >= 0; a = t.parent[a])
      for(int e = 0; e < L.nx[a]; e++) emit(L.xl[int64_t(a) * XCAP + e]);
   if(!out) cnt[T] = k;
}

// Keys that group the boxes with an M2L list by their octant in the parent (boxes without one
// sort last): boxes of one octant can only see the 189 offsets that octant allows, so tiles of
// same-octant boxes leave fewer rows of the tensor-core M2L empty.
__global__ void kM2LTargetKeys(Tree t, Lists L, int nNodes, int byCount, unsigned* keys, int* vals, int* count)
{
   int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i >= nNodes) return;
   bool has = L.nv[i] > 0;
   // octant, then (optionally) the list length, longest first: boxes with full neighbourhoods fill
   // whole tiles, sparse boundary boxes share tiles with each other
   const unsigned sub = byCount ? unsigned(316 - min(L.nv[i], 316)) : 0u;
   keys[i] = has ? (unsigned(t.key[i] & 7) << 9) | sub : (8u << 9);
   vals[i] = i;
   if(has) atomicAdd(count, 1);
}

// M2L target order by partner pattern: a tile's cost is the number of offsets any of its 42 boxes has a
// partner at, so boxes with similar sets of offsets should share tiles. The key of a box is its octant, then
// its offset bits with the rarest offsets first (the most telling ones): offsets counted over all boxes
// (kOffsetCounts), ranked in one block (kOffsetRanks), and each box's bits of ranks 0-60 and 61-124 packed
// into two 64-bit words (kM2LMaskKeys) that two stable radix sorts order (word 1, then word 0).
__global__ void kOffsetCounts(Lists L, int nNodes, unsigned* counts)
{
   // one warp per box row at a time: the row's 316 entries as 10 coalesced loads in flight; lane l counts
   // offsets l + 32 k in registers and adds them to the totals once
   const int lane = threadIdx.x & 31;
   const int warp = int((blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5);
   const int nWarps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
   unsigned c[10];
#pragma unroll
   for(int k = 0; k < 10; k++) c[k] = 0;
   for(int i = warp; i < nNodes; i += nWarps)
   {
      const int* vt = L.vtab + int64_t(i) * 316;
      int v[10];
#pragma unroll
      for(int k = 0; k < 10; k++) v[k] = lane + 32 * k < 316 ? vt[lane + 32 * k] : -1;
#pragma unroll
      for(int k = 0; k < 10; k++) c[k] += v[k] >= 0 ? 1u : 0u;
   }
#pragma unroll
   for(int k = 0; k < 10; k++)
      if(lane + 32 * k < 316 && c[k]) atomicAdd(&counts[lane + 32 * k], c[k]);
}
// rank[o]: the position of offset o in increasing count order (ties by index); one block of 320 threads
__global__ void kOffsetRanks(const unsigned* __restrict__ counts, int* rank)
{
   const int o = threadIdx.x;
   if(o >= 316) return;
   const unsigned c = counts[o];
   int r = 0;
   for(int q = 0; q < 316; q++)
   {
      const unsigned d = counts[q];
      r += (d < c || (d == c && q < o)) ? 1 : 0;
   }
   rank[o] = r;
}
// word 0: octant (bits 63..61), ranks 0..60 (bits 60..0); word 1: ranks 61..124 (bits 63..0). Boxes without
// M2L partners sort last. A warp per box at a time (grid-stride): the lanes read the box's table row together
// (10 coalesced loads in flight) and OR their bits into the two words; the boxes with partners are counted
// per block, one atomic each.
__global__ void kM2LMaskKeys(Tree t, Lists L, int nNodes, const int* __restrict__ rank, unsigned long long* k0,
                             unsigned long long* k1, int* vals, int* count)
{
   __shared__ int rk[316];
   __shared__ int blockCount;
   for(int o = threadIdx.x; o < 316; o += blockDim.x) rk[o] = rank[o];
   if(threadIdx.x == 0) blockCount = 0;
   __syncthreads();
   const int lane = threadIdx.x & 31;
   const int warp = int((blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5);
   const int nWarps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
   int mine = 0;
   for(int i = warp; i < nNodes; i += nWarps)
   {
      if(L.nv[i] <= 0)
      {
         if(lane == 0)
         {
            vals[i] = i;
            k0[i] = ~0ull;
            k1[i] = ~0ull;
         }
         continue;
      }
      unsigned long long w0 = 0, w1 = 0;
      const int* vt = L.vtab + int64_t(i) * 316;
      int v[10];
#pragma unroll
      for(int k = 0; k < 10; k++) v[k] = lane + 32 * k < 316 ? vt[lane + 32 * k] : -1;
#pragma unroll
      for(int k = 0; k < 10; k++)
      {
         if(v[k] < 0) continue;
         const int r = rk[lane + 32 * k];
         if(r < 61) w0 |= 1ull << (60 - r);
         else if(r < 125) w1 |= 1ull << (124 - r);
      }
      for(int d = 16; d > 0; d >>= 1)
      {
         w0 |= __shfl_xor_sync(0xffffffffu, w0, d);
         w1 |= __shfl_xor_sync(0xffffffffu, w1, d);
      }
      if(lane == 0)
      {
         mine++;
         vals[i] = i;
         k0[i] = w0 | (unsigned long long)(t.key[i] & 7) << 61;
         k1[i] = w1;
      }
   }
   if(lane == 0 && mine) atomicAdd(&blockCount, mine);
   __syncthreads();
   if(threadIdx.x == 0 && blockCount) atomicAdd(count, blockCount);
}
__global__ void kGatherKeys(const unsigned long long* __restrict__ k0, const int* __restrict__ order, int n,
                            unsigned long long* out)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i < n) out[i] = k0[order[i]];
}

// Nodes with children, compacted in node order (so each level's parents are contiguous), and the
// compacted index where each level starts.
__global__ void kParentFlags(Tree t, int nNodes, int* flags)
{
   int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i < nNodes) flags[i] = t.nchild[i] > 0 ? 1 : 0;
}
__global__ void kParentScatter(const int* __restrict__ flags, const int* __restrict__ pos, int nNodes, int* parList)
{
   int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i < nNodes && flags[i]) parList[pos[i]] = i;
}
__global__ void kParentLevelStarts(Tree t, const int* __restrict__ pos, int* out)
{
   int l = threadIdx.x;
   if(l <= t.nLevels) out[l] = pos[t.levelStart[l]];
}

// Tensor-core M2M / L2L tables (both preset to -1): up[parent][octant] = the child with sources,
// dn[child][octant of the child] = its parent, for children with targets.
__global__ void kTranslateTables(Tree t, int nNodes, int* __restrict__ up, int* __restrict__ dn)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i >= nNodes) return;
   const int par = t.parent[i];
   if(par < 0) return;
   const int o = int(t.key[i] & 7);
   if(t.s1[i] > t.s0[i]) up[int64_t(par) * 8 + o] = i;
   if(t.t1[i] > t.t0[i]) dn[int64_t(i) * 8 + o] = par;
}
// Keys (level, octant) of the nodes with targets below the roots; the rest sort last.
__global__ void kL2LTargetKeys(Tree t, int nNodes, unsigned* keys, int* vals)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if(i >= nNodes) return;
   const bool has = t.parent[i] >= 0 && t.t1[i] > t.t0[i];
   keys[i] = has ? (unsigned(t.level[i]) << 3) | unsigned(t.key[i] & 7) : unsigned(MAXLEVEL + 2) << 3;
   vals[i] = i;
}
// out[8 l + o] = the first sorted position whose (level, octant) is >= (l, o), up to (nLevels, 0).
__global__ void kL2LLevelStarts(const unsigned* __restrict__ keys, int n, int nLevels, int* out)
{
   const int lo8 = threadIdx.x;
   if(lo8 > 8 * nLevels) return;
   int lo = 0, hi = n;
   while(lo < hi)
   {
      const int mid = (lo + hi) >> 1;
      if(keys[mid] < unsigned(lo8)) lo = mid + 1;
      else hi = mid;
   }
   out[lo8] = lo;
}

// ------------------------------------------------------------------------------ host driver
__global__ void kInitLevelState(LevelBuildState* S, int nRoots)
{
   const int i = threadIdx.x;
   S->bar[i] = 0;
   if(i < MAXLEVEL) S->grab[i] = 0;
   if(i < MAXLEVEL + 2) S->levelStart[i] = i == 1 ? nRoots : 0;
   if(i == 0)
   {
      S->nLevels = 0;
      S->overflow = 0;
   }
}

// Every level of the forest in one cooperative launch (kBuildLevels), the node arrays grown and the build
// repeated when a level would not fit; one host wait for the level starts.
static fmm_status buildLevelsPersistent(Plan& P, cudaStream_t st, int64_t& capNodes, int K, const int* dSrcOff,
                                        const int* dTgtOff, const uint64_t* sk, const uint64_t* tk, int capS, int capT,
                                        int& nLevels, int64_t& total)
{
   int dev = 0, nSM = 0, perSM = 0;
   FMM_CUDA(cudaGetDevice(&dev));
   FMM_CUDA(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, dev));
   FMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kBuildLevels, LB_T, 0));
   if(perSM < 1) return setError(FMM_E_CUDA, "kBuildLevels: no resident block");
   // up to 4 blocks per SM (measured: the batch's level build took 10.3 ms of tree phase with 4, 10.4 with all
   // 6 resident)
   const int grid = nSM * std::min(perSM, 4);
   FMM_TRY(P.levelState.reserve(sizeof(LevelBuildState)));
   LevelBuildState* S = (LevelBuildState*)P.levelState.ptr;
   for(int attempt = 0; attempt < 8; attempt++)
   {
      FMM_TRY(P.ensureNodes(capNodes, st));
      Tree& t = P.tree;
      FMM_TRY(P.lvlBounds.reserve(sizeof(int) * 18 * size_t(capNodes)));
      // look-back words of every item of a level (levels never hold more than capNodes nodes); a word
      // carries its level, so the words of one level never pass for another's
      FMM_TRY(P.lvlOff.reserve(sizeof(unsigned long long) * size_t(capNodes / LB_T + 2)));
      FMM_CUDA(cudaMemsetAsync(P.lvlOff.ptr, 0, sizeof(unsigned long long) * size_t(capNodes / LB_T + 2), st));
      kInitRoots<<<(K + 255) / 256, 256, 0, st>>>(t, K, dSrcOff, dTgtOff);
      FMM_TRY(launched(P, "kInitRoots", st));
      kInitLevelState<<<1, 64, 0, st>>>(S, K);
      FMM_TRY(launched(P, "kInitLevelState", st));
      FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
      int maxLevel = P.maxLevel;
      int* bounds = (int*)P.lvlBounds.ptr;
      unsigned long long* look = (unsigned long long*)P.lvlOff.ptr;
      int* err = P.err;
      uint64_t limit = P.tcWaitNs;
      void* args[] = {&t, &maxLevel, &capS, &capT, &sk, &tk, &bounds, &look, &capNodes, &S, &err, &limit};
      FMM_CUDA(cudaLaunchCooperativeKernel((const void*)kBuildLevels, dim3(grid), dim3(LB_T), args, 0, st));
      FMM_TRY(launched(P, "kBuildLevels", st));
      LevelBuildState h;
      int herr = 0;
      FMM_CUDA(cudaMemcpyAsync(&h, S, sizeof(h), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaMemcpyAsync(&herr, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
      if(herr & ERR_TIMEOUT) return setError(FMM_E_TIMEOUT, "kBuildLevels: a grid barrier timed out");
      if(h.overflow)
      {
         // (the arrays keep the grown size, so later builds of this plan start from it)
         capNodes *= 2;
         continue;
      }
      nLevels = h.nLevels;
      for(int l = 0; l <= nLevels; l++) t.levelStart[l] = h.levelStart[l];
      total = h.levelStart[nLevels];
      return FMM_OK;
   }
   return setError(FMM_E_LIMIT, "kBuildLevels: node capacity did not converge");
}

template <class T>
fmm_status buildTreeT(Plan& P, cudaStream_t st)
{
   const int64_t n = P.n, m = P.m;
   const int threads = 256;
   // coils: one by default; the key keeps ceil(log2(coils)) bits above the Morton bits
   const int K = P.nCoils;
   if(!P.batch)
   {
      P.srcOff.assign({0, int(n)});
      P.tgtOff.assign({0, int(m)});
   }
   if(int(P.srcOff.size()) != K + 1 || int(P.tgtOff.size()) != K + 1 || P.srcOff[K] != n || P.tgtOff[K] != m)
      return setError(FMM_E_INVALID, "coil offsets do not match the source/target counts (%lld, %lld); "
                                     "call fmm_batch_set_coils after setting sources and targets",
                      (long long)n, (long long)m);
   P.coilBits = 0;
   while((int64_t(1) << P.coilBits) < K) P.coilBits++;
   P.maxLevel = std::min(MAXLEVEL, (63 - P.coilBits) / 3);
   FMM_TRY(P.waitSourcePoints(st));   // points copied by fmm_set_sources_async
   FMM_TRY(P.segb.reserve(sizeof(int) * 2 * (K + 1)));
   int* dSrcOff = (int*)P.segb.ptr;
   int* dTgtOff = dSrcOff + K + 1;
   FMM_CUDA(cudaMemcpyAsync(dSrcOff, P.srcOff.data(), sizeof(int) * (K + 1), cudaMemcpyHostToDevice, st));
   FMM_CUDA(cudaMemcpyAsync(dTgtOff, P.tgtOff.data(), sizeof(int) * (K + 1), cudaMemcpyHostToDevice, st));
   // root cubes
   FMM_TRY(P.rootb.reserve(sizeof(RootBox) * K));
   P.root = (RootBox*)P.rootb.ptr;
   if(P.batch)
   {
      kRootsPerCoil<T><<<K, 256, 0, st>>>((const T*)P.srcXYZ, (const T*)P.tgtXYZ, dSrcOff, dTgtOff, P.maxLevel,
                                          P.root);
      FMM_TRY(launched(P, "kRootsPerCoil", st));
   }
   else if(P.cfg.root_half_width > 0)
   {
      kRootFromConfig<<<1, 1, 0, st>>>(P.cfg.root_center[0], P.cfg.root_center[1], P.cfg.root_center[2],
                                       P.cfg.root_half_width, P.maxLevel, P.root);
      FMM_TRY(launched(P, "kRootFromConfig", st));
   }
   else
   {
      int nb = int(std::min<int64_t>(1024, (n + m + threads - 1) / threads));
      nb = std::max(nb, 1);
      FMM_TRY(P.scratch.reserve(sizeof(double) * 6 * nb));
      kBBox<T><<<nb, threads, 0, st>>>((const T*)P.srcXYZ, n, (const T*)P.tgtXYZ, m, (double*)P.scratch.ptr);
      FMM_TRY(launched(P, "kBBox", st));
      kRootFromBBox<<<1, 1, 0, st>>>((const double*)P.scratch.ptr, nb, P.maxLevel, P.root);
      FMM_TRY(launched(P, "kRootFromBBox", st));
   }
   FMM_CHECK_LAUNCH();
   // keys and sort
   FMM_TRY(P.sKeys.reserve(2 * sizeof(uint64_t) * n));
   FMM_TRY(P.tKeys.reserve(2 * sizeof(uint64_t) * m));
   FMM_TRY(P.sIdx.reserve(2 * sizeof(int) * n));
   FMM_TRY(P.tIdx.reserve(2 * sizeof(int) * m));
   uint64_t* sk = (uint64_t*)P.sKeys.ptr;
   uint64_t* tk = (uint64_t*)P.tKeys.ptr;
   int* si = (int*)P.sIdx.ptr;
   int* ti = (int*)P.tIdx.ptr;
   if(n) {
      kKeys<T><<<(n + threads - 1) / threads, threads, 0, st>>>((const T*)P.srcXYZ, n, P.root, dSrcOff, K,
                                                                P.maxLevel, sk + n, si + n);
      FMM_TRY(launched(P, "kKeys", st));
   }
   // targets that are the sources (fmm_set_targets_to_sources, one coil): their keys, order and sorted
   // positions are the sources', copied instead of computed and sorted again
   const bool same = P.tgtIsSrc && K == 1 && m == n && !P.bem;
   if(m && !same) {
      kKeys<T><<<(m + threads - 1) / threads, threads, 0, st>>>((const T*)P.tgtXYZ, m, P.root, dTgtOff, K,
                                                                P.maxLevel, tk + m, ti + m);
      FMM_TRY(launched(P, "kKeys", st));
   }
   FMM_CHECK_LAUNCH();
   const int keyBits = 3 * P.maxLevel + P.coilBits;
   size_t need = 0, tmp = 0;
   cub::DeviceRadixSort::SortPairs(nullptr, tmp, sk + n, sk, si + n, si, int(n), 0, keyBits, st);
   need = std::max(need, tmp);
   cub::DeviceRadixSort::SortPairs(nullptr, tmp, tk + m, tk, ti + m, ti, int(m), 0, keyBits, st);
   need = std::max(need, tmp);
   FMM_TRY(P.cubTmp.reserve(need));
   tmp = P.cubTmp.bytes;
   if(n) FMM_CUDA(cub::DeviceRadixSort::SortPairs(P.cubTmp.ptr, tmp, sk + n, sk, si + n, si, int(n), 0, keyBits, st));
   tmp = P.cubTmp.bytes;
   if(m && !same) FMM_CUDA(cub::DeviceRadixSort::SortPairs(P.cubTmp.ptr, tmp, tk + m, tk, ti + m, ti, int(m), 0, keyBits, st));
   if(m && same)
   {
      FMM_CUDA(cudaMemcpyAsync(tk, sk, sizeof(uint64_t) * m, cudaMemcpyDeviceToDevice, st));
      FMM_CUDA(cudaMemcpyAsync(ti, si, sizeof(int) * m, cudaMemcpyDeviceToDevice, st));
   }
   if(P.debugSync) FMM_CUDA(cudaStreamSynchronize(st));
   // sorted point data
   typedef typename Vec4<T>::type V4;
   FMM_TRY(P.sPos.reserve(sizeof(V4) * std::max<int64_t>(n, 1)));
   FMM_TRY(P.sQ.reserve(sizeof(V4) * std::max<int64_t>(n, 1)));
   FMM_TRY(P.tPos.reserve(sizeof(V4) * std::max<int64_t>(m, 1)));
   if(n)
   {
      // strengths still crossing the bus (fmm_set_sources_async): gathered at the end of the build
      kGatherSources<T><<<(n + threads - 1) / threads, threads, 0, st>>>(
         (const T*)P.srcXYZ, (const T*)P.srcW, (const T*)(P.hasJ ? P.srcJ : nullptr),
         (const T*)(P.bem ? P.srcSigma : nullptr), si, n, (V4*)P.sPos.ptr,
         P.inputsAsync ? nullptr : (V4*)P.sQ.ptr);
      FMM_TRY(launched(P, "kGatherSources", st));
   }
   if(m && same)
      // (the sorted sources' (x, y, z, 0): the fourth lane is zero for sources that are not BEM sources)
      FMM_CUDA(cudaMemcpyAsync(P.tPos.ptr, P.sPos.ptr, sizeof(V4) * m, cudaMemcpyDeviceToDevice, st));
   else if(m) {
      kGatherTargets<T><<<(m + threads - 1) / threads, threads, 0, st>>>((const T*)P.tgtXYZ, ti, m, (V4*)P.tPos.ptr);
      FMM_TRY(launched(P, "kGatherTargets", st));
   }
   FMM_CHECK_LAUNCH();

   // nodes, level by level (at least the capacity an earlier build of this plan grew to)
   int64_t capNodes = std::max<int64_t>(1024, 2 * (n + m) / std::max(1, P.cfg.leaf_capacity) + 64 + 2 * K);
   capNodes = std::max<int64_t>(capNodes, P.nodeCap);
   FMM_TRY(P.ensureNodes(capNodes));
   Tree& t = P.tree;
   const int capS = P.cfg.leaf_capacity;
   const int capT = P.cfg.target_leaf_capacity > 0 ? P.cfg.target_leaf_capacity : P.cfg.leaf_capacity;
   int nLevels = 1;
   int64_t total = K;
   bool built = false;
   if(P.treePersistent)
   {
      int coop = 0, dev = 0;
      FMM_CUDA(cudaGetDevice(&dev));
      FMM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
      if(coop)
      {
         FMM_TRY(buildLevelsPersistent(P, st, capNodes, K, dSrcOff, dTgtOff, sk, tk, capS, capT, nLevels, total));
         built = true;
      }
   }
   if(!built)
   {
   kInitRoots<<<(K + 255) / 256, 256, 0, st>>>(t, K, dSrcOff, dTgtOff);
   FMM_TRY(launched(P, "kInitRoots", st));
   t.levelStart[0] = 0;
   t.levelStart[1] = K;
   for(int level = 0; level < P.maxLevel; level++)
   {
      int a = t.levelStart[level], b = t.levelStart[level + 1];
      int cnt = b - a;
      if(cnt == 0) break;
      FMM_TRY(P.lvlBounds.reserve(sizeof(int) * 18 * cnt));
      FMM_TRY(P.lvlCnt.reserve(sizeof(int) * (cnt + 1)));
      FMM_TRY(P.lvlOff.reserve(sizeof(int) * (cnt + 1)));
      int* bounds = (int*)P.lvlBounds.ptr;
      int* cc = (int*)P.lvlCnt.ptr;
      int* off = (int*)P.lvlOff.ptr;
      kCountChildren<<<(cnt + threads - 1) / threads, threads, 0, st>>>(t, a, b, level, P.maxLevel, capS, capT, sk, tk,
                                                                        bounds, cc);
      FMM_TRY(launched(P, "kCountChildren", st));
      FMM_CHECK_LAUNCH();
      tmp = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tmp, cc, off, cnt + 1, st);
      FMM_TRY(P.cubTmp.reserve(tmp));
      tmp = P.cubTmp.bytes;
      // cnt[cnt] must be 0 for the total to land in off[cnt]
      FMM_CUDA(cudaMemsetAsync(cc + cnt, 0, sizeof(int), st));
      FMM_CUDA(cub::DeviceScan::ExclusiveSum(P.cubTmp.ptr, tmp, cc, off, cnt + 1, st));
      if(P.debugSync) FMM_CUDA(cudaStreamSynchronize(st));
      int nextCount = 0;
      FMM_CUDA(cudaMemcpyAsync(&nextCount, off + cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      if(nextCount == 0) break;
      if(total + nextCount > capNodes)
      {
         capNodes = std::max<int64_t>(2 * capNodes, total + nextCount);
         FMM_TRY(P.ensureNodes(capNodes, st));
      }
      kMakeChildren<<<(cnt + threads - 1) / threads, threads, 0, st>>>(t, a, b, level, int(total), bounds, cc, off);
      FMM_TRY(launched(P, "kMakeChildren", st));
      FMM_CHECK_LAUNCH();
      total += nextCount;
      t.levelStart[level + 2] = int(total);
      nLevels = level + 2;
   }
   }
   t.nNodes = total;
   t.nLevels = nLevels;

   // lists
   FMM_TRY(P.ensureLists(total));
   Lists& Ls = P.lists;
   FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
   // every node's M2L table starts empty: one fill here instead of 316 strided stores per node
   FMM_CUDA(cudaMemsetAsync(Ls.vtab, 0xff, sizeof(int) * 316 * size_t(total), st));
   kInitRootLists<<<(K + 255) / 256, 256, 0, st>>>(Ls, K);
   FMM_TRY(launched(P, "kInitRootLists", st));
   for(int level = 1; level < nLevels; level++)
   {
      int a = t.levelStart[level], b = t.levelStart[level + 1];
      // one warp per box pays where boxes have many candidates (a dense single coil: 11.1 -> 10.0 ms of tree
      // phase at 2^24) and not where most have few (the 256 small coils of the batch: 11.6 -> 13.4 ms)
      if(P.listsWarp == 2 || (P.listsWarp == 1 && K == 1))
      {
         kListsLevelWarp<<<(b - a + LW_WARPS - 1) / LW_WARPS, 32 * LW_WARPS, 0, st>>>(t, Ls, a, b, P.err);
         FMM_TRY(launched(P, "kListsLevelWarp", st));
      }
      else
      {
         kListsLevel<<<(b - a + 127) / 128, 128, 0, st>>>(t, Ls, a, b, P.err);
         FMM_TRY(launched(P, "kListsLevel", st));
      }
   }
   FMM_CHECK_LAUNCH();
   int nn = int(total);
   FMM_TRY(P.p2pOff.reserve(sizeof(int) * (nn + 1)));
   FMM_TRY(P.lvlCnt.reserve(sizeof(int) * (nn + 1)));
   int* pc = (int*)P.lvlCnt.ptr;
   int* po = (int*)P.p2pOff.ptr;
   kP2PLists<<<(nn + 127) / 128, 128, 0, st>>>(t, Ls, nn, nullptr, pc, nullptr, P.err);
   FMM_TRY(launched(P, "kP2PLists", st));
   FMM_CUDA(cudaMemsetAsync(pc + nn, 0, sizeof(int), st));
   tmp = 0;
   cub::DeviceScan::ExclusiveSum(nullptr, tmp, pc, po, nn + 1, st);
   FMM_TRY(P.cubTmp.reserve(tmp));
   tmp = P.cubTmp.bytes;
   FMM_CUDA(cub::DeviceScan::ExclusiveSum(P.cubTmp.ptr, tmp, pc, po, nn + 1, st));
   int nP2P = 0;
   FMM_CUDA(cudaMemcpyAsync(&nP2P, po + nn, sizeof(int), cudaMemcpyDeviceToHost, st));
   // number of M2L (V-list) pairs
   FMM_TRY(P.scratch.reserve(sizeof(long long)));
   tmp = 0;
   cub::DeviceReduce::Sum(nullptr, tmp, Ls.nv, (long long*)P.scratch.ptr, nn, st);
   FMM_TRY(P.cubTmp.reserve(tmp));
   tmp = P.cubTmp.bytes;
   FMM_CUDA(cub::DeviceReduce::Sum(P.cubTmp.ptr, tmp, Ls.nv, (long long*)P.scratch.ptr, nn, st));
   long long nV = 0;
   FMM_CUDA(cudaMemcpyAsync(&nV, P.scratch.ptr, sizeof(long long), cudaMemcpyDeviceToHost, st));
   int herr = 0;
   FMM_CUDA(cudaMemcpyAsync(&herr, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
   FMM_CUDA(cudaStreamSynchronize(st));
   if(herr) return setError(FMM_E_LIMIT, "interaction list capacity exceeded (code %d)", herr);
   FMM_TRY(P.p2pList.reserve(sizeof(int) * std::max(nP2P, 1)));
   kP2PLists<<<(nn + 127) / 128, 128, 0, st>>>(t, Ls, nn, po, nullptr, (int*)P.p2pList.ptr, P.err);
   FMM_TRY(launched(P, "kP2PLists", st));
   FMM_CHECK_LAUNCH();
   P.nP2P = nP2P;
   P.nV = nV;
   FMM_TRY(P.nearCounts.reserve(2 * sizeof(unsigned long long)));
   FMM_CUDA(cudaMemsetAsync(P.nearCounts.ptr, 0, 2 * sizeof(unsigned long long), st));
   kNearCounts<<<148 * 4, 256, 0, st>>>(t, nn, po, (const int*)P.p2pList.ptr, (unsigned long long*)P.nearCounts.ptr);
   FMM_TRY(launched(P, "kNearCounts", st));
   FMM_CHECK_LAUNCH();
   // parents per level for the M2M / L2L GEMMs
   {
      int* flags = (int*)P.lvlCnt.ptr;   // nn + 1 ints, free again once the direct lists are counted
      FMM_TRY(P.lvlOff.reserve(sizeof(int) * (nn + 1)));
      int* pos = (int*)P.lvlOff.ptr;
      FMM_TRY(P.parList.reserve(sizeof(int) * std::max(nn, 1)));
      kParentFlags<<<(nn + 255) / 256, 256, 0, st>>>(t, nn, flags);
      FMM_TRY(launched(P, "kParentFlags", st));
      FMM_CUDA(cudaMemsetAsync(flags + nn, 0, sizeof(int), st));
      tmp = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tmp, flags, pos, nn + 1, st);
      FMM_TRY(P.cubTmp.reserve(tmp));
      tmp = P.cubTmp.bytes;
      FMM_CUDA(cub::DeviceScan::ExclusiveSum(P.cubTmp.ptr, tmp, flags, pos, nn + 1, st));
      kParentScatter<<<(nn + 255) / 256, 256, 0, st>>>(flags, pos, nn, (int*)P.parList.ptr);
      FMM_TRY(launched(P, "kParentScatter", st));
      FMM_TRY(P.scratch.reserve(sizeof(int) * (MAXLEVEL + 2)));
      t.levelStart[nLevels] = nn;
      kParentLevelStarts<<<1, 32, 0, st>>>(t, pos, (int*)P.scratch.ptr);
      FMM_TRY(launched(P, "kParentLevelStarts", st));
      P.parStart.assign(nLevels + 1, 0);
      FMM_CUDA(cudaMemcpyAsync(P.parStart.data(), P.scratch.ptr, sizeof(int) * (nLevels + 1), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
   }
   // M2L targets grouped by octant, then (tcGroup 2) by partner pattern
   if(P.tcGroup == 2)
   {
      FMM_TRY(P.m2lTargets.reserve(2 * sizeof(int) * nn));
      // three key arrays of nn words (word 0, word 1, word 0 in word-1 order), sorted copies, and the
      // offset counts and ranks
      FMM_TRY(P.m2lKeys.reserve(sizeof(unsigned long long) * (4 * size_t(nn) + 2) + 2 * sizeof(int) * 320));
      unsigned long long* k0 = (unsigned long long*)P.m2lKeys.ptr;
      unsigned long long* k1 = k0 + nn;
      unsigned long long* k2 = k1 + nn;
      unsigned long long* k3 = k2 + nn;
      unsigned* counts = (unsigned*)(k3 + nn + 2);
      int* rank = (int*)(counts + 320);
      int* vv = (int*)P.m2lTargets.ptr;
      FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
      FMM_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned) * 320, st));
      kOffsetCounts<<<148 * 4, 256, 0, st>>>(Ls, nn, counts);
      FMM_TRY(launched(P, "kOffsetCounts", st));
      kOffsetRanks<<<1, 320, 0, st>>>(counts, rank);
      FMM_TRY(launched(P, "kOffsetRanks", st));
      kM2LMaskKeys<<<148 * 8, 256, 0, st>>>(t, Ls, nn, rank, k0, k1, vv + nn, P.err);
      FMM_TRY(launched(P, "kM2LMaskKeys", st));
      // stable LSD order: by word 1, then by word 0
      tmp = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tmp, k1, k3, vv + nn, vv, nn, 0, 64, st);
      FMM_TRY(P.cubTmp.reserve(tmp));
      tmp = P.cubTmp.bytes;
      FMM_CUDA(cub::DeviceRadixSort::SortPairs(P.cubTmp.ptr, tmp, k1, k3, vv + nn, vv, nn, 0, 64, st));
      kGatherKeys<<<(nn + 255) / 256, 256, 0, st>>>(k0, vv, nn, k2);
      FMM_TRY(launched(P, "kGatherKeys", st));
      tmp = P.cubTmp.bytes;
      FMM_CUDA(cub::DeviceRadixSort::SortPairs(P.cubTmp.ptr, tmp, k2, k3, vv, vv + nn, nn, 0, 64, st));
      // the final order is in vv + nn: move it to the front
      FMM_CUDA(cudaMemcpyAsync(vv, vv + nn, sizeof(int) * nn, cudaMemcpyDeviceToDevice, st));
      int cntT = 0;
      FMM_CUDA(cudaMemcpyAsync(&cntT, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      P.nM2LTargets = cntT;
      FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
   }
   else
   {
      FMM_TRY(P.m2lTargets.reserve(2 * sizeof(int) * nn));
      FMM_TRY(P.m2lKeys.reserve(2 * sizeof(unsigned) * nn));
      unsigned* kk = (unsigned*)P.m2lKeys.ptr;
      int* vv = (int*)P.m2lTargets.ptr;
      FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
      kM2LTargetKeys<<<(nn + 255) / 256, 256, 0, st>>>(t, Ls, nn, P.tcGroup == 1, kk + nn, vv + nn, P.err);
      FMM_TRY(launched(P, "kM2LTargetKeys", st));
      tmp = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tmp, kk + nn, kk, vv + nn, vv, nn, 0, 13, st);
      FMM_TRY(P.cubTmp.reserve(tmp));
      tmp = P.cubTmp.bytes;
      FMM_CUDA(cub::DeviceRadixSort::SortPairs(P.cubTmp.ptr, tmp, kk + nn, kk, vv + nn, vv, nn, 0, 13, st));
      int cntT = 0;
      FMM_CUDA(cudaMemcpyAsync(&cntT, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      P.nM2LTargets = cntT;
      FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
   }
   P.multBfTag = -1;
   // M2M / L2L tables: the L2L child lists always (both L2L forms use them), the octant tables
   // for the tensor-core forms
   {
      if(P.tcTranslations())
      {
         FMM_TRY(P.vtabUp.reserve(sizeof(int) * 8 * size_t(nn)));
         FMM_TRY(P.vtabDn.reserve(sizeof(int) * 8 * size_t(nn)));
         FMM_CUDA(cudaMemsetAsync(P.vtabUp.ptr, 0xff, sizeof(int) * 8 * size_t(nn), st));
         FMM_CUDA(cudaMemsetAsync(P.vtabDn.ptr, 0xff, sizeof(int) * 8 * size_t(nn), st));
         kTranslateTables<<<(nn + 255) / 256, 256, 0, st>>>(t, nn, (int*)P.vtabUp.ptr, (int*)P.vtabDn.ptr);
         FMM_TRY(launched(P, "kTranslateTables", st));
      }
      FMM_TRY(P.l2lTargets.reserve(2 * sizeof(int) * nn));
      FMM_TRY(P.l2lKeys.reserve(2 * sizeof(unsigned) * nn));
      unsigned* kk = (unsigned*)P.l2lKeys.ptr;
      int* vv = (int*)P.l2lTargets.ptr;
      kL2LTargetKeys<<<(nn + 255) / 256, 256, 0, st>>>(t, nn, kk + nn, vv + nn);
      FMM_TRY(launched(P, "kL2LTargetKeys", st));
      tmp = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tmp, kk + nn, kk, vv + nn, vv, nn, 0, 8, st);
      FMM_TRY(P.cubTmp.reserve(tmp));
      tmp = P.cubTmp.bytes;
      FMM_CUDA(cub::DeviceRadixSort::SortPairs(P.cubTmp.ptr, tmp, kk + nn, kk, vv + nn, vv, nn, 0, 8, st));
      FMM_TRY(P.scratch.reserve(sizeof(int) * 8 * (MAXLEVEL + 2)));
      kL2LLevelStarts<<<1, 8 * (MAXLEVEL + 2), 0, st>>>(kk, nn, nLevels, (int*)P.scratch.ptr);
      FMM_TRY(launched(P, "kL2LLevelStarts", st));
      P.l2lStart.assign(8 * nLevels + 1, 0);
      FMM_CUDA(cudaMemcpyAsync(P.l2lStart.data(), P.scratch.ptr, sizeof(int) * (8 * nLevels + 1), cudaMemcpyDeviceToHost, st));
      FMM_CUDA(cudaStreamSynchronize(st));
      FMM_CHECK_LAUNCH();
   }
   if(P.inputsAsync && n)
   {
      typedef typename Vec4<T>::type V4;
      FMM_TRY(P.waitSourceInputs(st));
      kGatherSources<T><<<(n + threads - 1) / threads, threads, 0, st>>>(
         (const T*)P.srcXYZ, (const T*)P.srcW, (const T*)(P.hasJ ? P.srcJ : nullptr), nullptr,
         (const int*)P.sIdx.ptr, n, nullptr, (V4*)P.sQ.ptr);
      FMM_TRY(launched(P, "kGatherSources", st));
      FMM_CHECK_LAUNCH();
   }
   return FMM_OK;
}

template fmm_status buildTreeT<float>(Plan&, cudaStream_t);
template fmm_status buildTreeT<double>(Plan&, cudaStream_t);

}  // namespace fmm
