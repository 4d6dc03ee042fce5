// The BEM problem (the reference's Problem::BEM: FastMultipoleSolver::calcBEM,
// FMM/FMMGPU/fast_multipole_solver.cpp:233-250, with the P2M math::calcBEMIntegralContribution,
// integration.cpp:295-353, and the direct math::calcBEMIntegral, integration.cpp:191-215).
//
// A BEM quadrature holds a point q, a weight w, a field value B and a surface normal n. Its kernel at x is
//   K(x) = w [(B . n) d + d x (B x n)] / |d|^3,   d = q - x,
// and the integral is sum_q K(x) / (4 pi). With sigma = w (B . n) and s = w (B x n) the kernel is
// sigma d / |d|^3 + d x s / |d|^3: each component is the potential of point dipoles
// (d / |d|^3 = -grad_q 1/|x - q|), so a box's multipole is
//   M_k = -sum_q [sigma grad R_k(q - c) + grad R_k(q - c) x s]
// and the field sum_k M_k I_k(x - c) / (4 pi): the Biot-Savart pipeline's vector expansions, M2M, M2L and
// L2L serve unchanged; the P2M, the near field and the direct sum are the BEM's own. The plan keeps s as
// its sources' strength vector (w J with J = B x n) and sigma in the strength stream's fourth lane.
#include "fmm_internal.cuh"

namespace fmm {

namespace {

template <class T>
struct Dual
{
   T v, x, y, z;
};
template <class T> __device__ __forceinline__ Dual<T> dSub(Dual<T> a, Dual<T> b) { return {a.v - b.v, a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> __device__ __forceinline__ Dual<T> dAdd(Dual<T> a, Dual<T> b) { return {a.v + b.v, a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> __device__ __forceinline__ Dual<T> dScale(Dual<T> a, T s) { return {a.v * s, a.x * s, a.y * s, a.z * s}; }
template <class T> __device__ __forceinline__ Dual<T> dMul(Dual<T> a, Dual<T> b)
{
   return {a.v * b.v, a.x * b.v + a.v * b.x, a.y * b.v + a.v * b.y, a.z * b.v + a.v * b.z};
}

template <class T>
__global__ void kBemPrepare(const T* __restrict__ B, const T* __restrict__ nrm, int64_t n, T* __restrict__ J,
                            T* __restrict__ sigma)
{
   const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i >= n) return;
   const T bx = B[3 * i], by = B[3 * i + 1], bz = B[3 * i + 2];
   const T nx = nrm[3 * i], ny = nrm[3 * i + 1], nz = nrm[3 * i + 2];
   J[3 * i] = by * nz - bz * ny;
   J[3 * i + 1] = bz * nx - bx * nz;
   J[3 * i + 2] = bx * ny - by * nx;
   sigma[i] = bx * nx + by * ny + bz * nz;
}

// One warp per leaf with sources; lanes own points, 32 at a time. Each lane runs the regular-harmonic
// recurrence (fmm_common.cuh visitRegular) on dual numbers for its point, in the leaf's scaled
// coordinates u = (q - c) / h; the warp sums each coefficient's three components over its points by
// shuffles and lane 0 keeps the running sum in shared memory. A box of side h stores M~_l = M_l / h^l;
// grad_q R_l(q - c) = h^(l-1) grad_u R_l(u), so M~_k = -(1/h) sum_q [sigma g + g x s], g = grad_u R_k(u).
constexpr int BEM_P2M_WARPS = 4;

template <class T>
__global__ void __launch_bounds__(32 * BEM_P2M_WARPS) kP2MBem(Tree t, const RootBox* __restrict__ rootp, int p,
                                                              int Lp, const typename Vec4<T>::type* __restrict__ spos,
                                                              const typename Vec4<T>::type* __restrict__ sq,
                                                              T* __restrict__ mult)
{
   extern __shared__ __align__(16) unsigned char smraw[];
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int64_t node = int64_t(blockIdx.x) * BEM_P2M_WARPS + warp;
   const int L = nharm(p);
   double* acc = reinterpret_cast<double*>(smraw) + size_t(warp) * 3 * L;
   if(node >= t.nNodes) return;
   if(t.nchild[node] != 0 || t.s1[node] == t.s0[node]) return;
   for(int e = lane; e < 3 * L; e += 32) acc[e] = 0.0;
   __syncwarp();
   const RootBox rb = rootp[rootOf(t, int(node))];
   const int level = t.level[node];
   const double h = 2.0 * rb.H / double(int64_t(1) << level);
   const double cx = rb.center[0] - rb.H + (double(t.ix[node]) + 0.5) * h;
   const double cy = rb.center[1] - rb.H + (double(t.iy[node]) + 0.5) * h;
   const double cz = rb.center[2] - rb.H + (double(t.iz[node]) + 0.5) * h;
   const T sq2 = T(1.4142135623730950488);
   for(int base = t.s0[node]; base < t.s1[node]; base += 32)
   {
      const int i = base + lane;
      const bool on = i < t.s1[node];
      T ux = T(0), uy = T(0), uz = T(0), sg = T(0), s0 = T(0), s1 = T(0), s2 = T(0);
      if(on)
      {
         const auto q = spos[i];
         const auto s = sq[i];
         ux = T((double(q.x) - cx) / h);
         uy = T((double(q.y) - cy) / h);
         uz = T((double(q.z) - cz) / h);
         s0 = s.x; s1 = s.y; s2 = s.z; sg = s.w;
      }
      const Dual<T> X{ux, T(1), T(0), T(0)}, Y{uy, T(0), T(1), T(0)}, Z{uz, T(0), T(0), T(1)};
      const Dual<T> R2{ux * ux + uy * uy + uz * uz, T(2) * ux, T(2) * uy, T(2) * uz};
      Dual<T> dre{T(1), T(0), T(0), T(0)}, dim{T(0), T(0), T(0), T(0)};   // S_m^m
      // the contribution of gradient g of one real harmonic to the three components: -(sigma g + g x s)
      auto emit = [&](int k, Dual<T> r) {
         T v[3];
         v[0] = -(sg * r.x + (r.y * s2 - r.z * s1));
         v[1] = -(sg * r.y + (r.z * s0 - r.x * s2));
         v[2] = -(sg * r.z + (r.x * s1 - r.y * s0));
#pragma unroll
         for(int c = 0; c < 3; c++)
         {
            double w = double(v[c]);
#pragma unroll
            for(int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if(lane == 0) acc[c * L + k] += w;
         }
      };
      for(int m = 0; m <= p; m++)
      {
         if(m > 0)
         {
            const T f = T(1) / T(2 * m);
            const Dual<T> nre = dScale(dSub(dMul(dre, X), dMul(dim, Y)), f);
            const Dual<T> nim = dScale(dAdd(dMul(dre, Y), dMul(dim, X)), f);
            dre = nre; dim = nim;
         }
         Dual<T> are = dre, aim = dim, bre{T(0), T(0), T(0), T(0)}, bim{T(0), T(0), T(0), T(0)};
         for(int l = m; l <= p; l++)
         {
            const T s = (l & 1) ? T(-1) : T(1);
            if(m == 0) emit(l * l + l, dScale(are, s));
            else
            {
               emit(l * l + l + m, dScale(are, s * sq2));
               emit(l * l + l - m, dScale(aim, s * sq2));
            }
            if(l == p) break;
            Dual<T> cre, cim;
            if(l == m)
            {
               cre = dMul(Z, are);
               cim = dMul(Z, aim);
            }
            else
            {
               const T inv = T(1) / T((l - m + 1) * (l + m + 1));
               const T a = T(2 * l + 1) * inv;
               cre = dSub(dScale(dMul(Z, are), a), dScale(dMul(R2, bre), inv));
               cim = dSub(dScale(dMul(Z, aim), a), dScale(dMul(R2, bim), inv));
            }
            bre = are; bim = aim; are = cre; aim = cim;
         }
      }
   }
   __syncwarp();
   const double ih = 1.0 / h;
   for(int e = lane; e < 3 * L; e += 32)
      mult[node * 3 * Lp + (e / L) * Lp + e % L] = T(acc[e] * ih);
}

// the BEM kernel of source (q, sigma, s) at x, accumulated into K: sigma d / |d|^3 + d x s / |d|^3, d = q - x
template <class V4>
__device__ __forceinline__ void bemKernel(double x, double y, double z, const V4& q, const V4& s, double K[3])
{
   const double dx = double(q.x) - x, dy = double(q.y) - y, dz = double(q.z) - z;
   const double r2 = dx * dx + dy * dy + dz * dz;
   if(r2 == 0.0) return;
   const double ri = 1.0 / sqrt(r2), ri3 = ri * ri * ri;
   const double sg = double(s.w);
   K[0] += (sg * dx + (dy * double(s.z) - dz * double(s.y))) * ri3;
   K[1] += (sg * dy + (dz * double(s.x) - dx * double(s.z))) * ri3;
   K[2] += (sg * dz + (dx * double(s.y) - dy * double(s.x))) * ri3;
}

// Near field of the BEM problem: one block per target leaf; each thread adds to its targets' far field
// (written unscaled by the L2P into out) the direct sum over the leaf's direct-list source boxes, and
// scales the total by 1 / (4 pi).
template <class T>
__global__ void __launch_bounds__(128) kBemNear(Tree t, const typename Vec4<T>::type* __restrict__ tpos,
                                                const typename Vec4<T>::type* __restrict__ spos,
                                                const typename Vec4<T>::type* __restrict__ sq,
                                                const int* __restrict__ p2pOff, const int* __restrict__ p2pList,
                                                const int* __restrict__ tOrder, double scale, T* __restrict__ out)
{
   const int node = blockIdx.x;
   if(t.nchild[node] != 0 || t.t1[node] == t.t0[node]) return;
   const int e0 = p2pOff[node], e1 = p2pOff[node + 1];
   for(int ti = t.t0[node] + threadIdx.x; ti < t.t1[node]; ti += blockDim.x)
   {
      const auto xp = tpos[ti];
      const double x = double(xp.x), y = double(xp.y), z = double(xp.z);
      const int64_t o = tOrder[ti];
      double K[3] = {double(out[3 * o]), double(out[3 * o + 1]), double(out[3 * o + 2])};
      for(int e = e0; e < e1; e++)
      {
         const int sn = p2pList[e];
         for(int i = t.s0[sn]; i < t.s1[sn]; i++) bemKernel(x, y, z, spos[i], sq[i], K);
      }
      for(int c = 0; c < 3; c++) out[3 * o + c] = T(K[c] * scale);
   }
}

// Direct BEM integral (math::calcBEMIntegral) at every target: one thread per target over all sources.
template <class T>
__global__ void __launch_bounds__(128) kDirectBem(const typename Vec4<T>::type* __restrict__ spos,
                                                  const typename Vec4<T>::type* __restrict__ sq, int n,
                                                  const T* __restrict__ tgt, int64_t m, double scale, T* __restrict__ out)
{
   __shared__ typename Vec4<T>::type Sp[128], Sq[128];
   const int64_t ti = blockIdx.x * int64_t(128) + threadIdx.x;
   const bool active = ti < m;
   const double x = active ? double(tgt[3 * ti]) : 0.0, y = active ? double(tgt[3 * ti + 1]) : 0.0,
                z = active ? double(tgt[3 * ti + 2]) : 0.0;
   double K[3] = {0, 0, 0};
   for(int sb = 0; sb < n; sb += 128)
   {
      const int cnt = min(128, n - sb);
      __syncthreads();
      if(threadIdx.x < cnt)
      {
         Sp[threadIdx.x] = spos[sb + threadIdx.x];
         Sq[threadIdx.x] = sq[sb + threadIdx.x];
      }
      __syncthreads();
      if(active)
         for(int i = 0; i < cnt; i++) bemKernel(x, y, z, Sp[i], Sq[i], K);
   }
   if(active)
      for(int c = 0; c < 3; c++) out[3 * ti + c] = T(K[c] * scale);
}

}  // namespace

template <class T>
fmm_status bemPrepareT(Plan& P, const void* B, const void* nrm, cudaStream_t st)
{
   if(P.n == 0) return FMM_OK;
   kBemPrepare<T><<<int((P.n + 255) / 256), 256, 0, st>>>((const T*)B, (const T*)nrm, P.n, (T*)P.srcJ, (T*)P.srcSigma);
   return launched(P, "kBemPrepare", st);
}

template <class T>
fmm_status bemP2MT(Plan& P, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   const int64_t N = P.tree.nNodes;
   const size_t shm = sizeof(double) * 3 * size_t(P.L) * BEM_P2M_WARPS;
   FMM_CUDA(cudaFuncSetAttribute(kP2MBem<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
   kP2MBem<T><<<int((N + BEM_P2M_WARPS - 1) / BEM_P2M_WARPS), 32 * BEM_P2M_WARPS, shm, st>>>(
      P.tree, P.root, P.p, P.Lp, (const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, (T*)P.mult.ptr);
   return launched(P, "kP2MBem", st);
}

template <class T>
fmm_status bemNearT(Plan& P, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   const int64_t N = P.tree.nNodes;
   kBemNear<T><<<int(N), 128, 0, st>>>(P.tree, (const V4*)P.tPos.ptr, (const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr,
                                       (const int*)P.p2pOff.ptr, (const int*)P.p2pList.ptr, (const int*)P.tIdx.ptr,
                                       1.0 / (4 * REF_PI), (T*)P.outA.ptr);
   return launched(P, "kBemNear", st);
}

template <class T>
fmm_status bemDirectT(Plan& P, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   if(P.m == 0) return FMM_OK;
   kDirectBem<T><<<int((P.m + 127) / 128), 128, 0, st>>>((const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, int(P.n),
                                                        (const T*)P.tgtXYZ, P.m, 1.0 / (4 * REF_PI), (T*)P.outA.ptr);
   return launched(P, "kDirectBem", st);
}

template fmm_status bemPrepareT<float>(Plan&, const void*, const void*, cudaStream_t);
template fmm_status bemPrepareT<double>(Plan&, const void*, const void*, cudaStream_t);
template fmm_status bemP2MT<float>(Plan&, cudaStream_t);
template fmm_status bemP2MT<double>(Plan&, cudaStream_t);
template fmm_status bemNearT<float>(Plan&, cudaStream_t);
template fmm_status bemNearT<double>(Plan&, cudaStream_t);
template fmm_status bemDirectT<float>(Plan&, cudaStream_t);
template fmm_status bemDirectT<double>(Plan&, cudaStream_t);

}  // namespace fmm
