// Treecode evaluation on the plan's source tree (the reference's MultipoleSolver::calcA / calcB(current,
// point), FMM/FMMGPU/multipole_solver.cpp:686-700, descending with QuadratureOctreeNode::calcA / calcRot,
// quadrature_octree.cpp:171-258).
//
// For each query point x the source tree is walked from its root: a box whose half-diagonal r and
// distance d from its centre satisfy 4 r^2 < d^2 contributes through its multipole (the reference's
// acceptance test), any other box through its children; a leaf that fails the test is summed directly
// (by default) or contributes nothing (FMM_TREECODE_REFERENCE_NEAR, as the reference, which loses
// 10-19 % near its sources). With box-size scaled multipoles (a box of side h keeps M~_l = M_l / h^l)
// a box's potential at x is (1/h) sum_k M~_k I_k(u), u = (x - c) / h; its gradient, for B = curl A,
// comes from the same irregular-harmonic recurrence run on dual numbers (value and three partial
// derivatives), or by central differences of A with step 1e-3 as the reference does
// (FMM_TREECODE_FD_CURL).
//
// One thread per query point, an explicit stack of boxes in local memory.
#include "fmm_internal.cuh"

namespace fmm {

namespace {

// value and gradient (d/dx, d/dy, d/dz) of a scalar
template <class T>
struct Dual
{
   T v, x, y, z;
};
template <class T> __device__ __forceinline__ Dual<T> dAdd(Dual<T> a, Dual<T> b) { return {a.v + b.v, a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> __device__ __forceinline__ Dual<T> dSub(Dual<T> a, Dual<T> b) { return {a.v - b.v, a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> __device__ __forceinline__ Dual<T> dScale(Dual<T> a, T s) { return {a.v * s, a.x * s, a.y * s, a.z * s}; }
template <class T> __device__ __forceinline__ Dual<T> dMul(Dual<T> a, Dual<T> b)
{
   return {a.v * b.v, a.x * b.v + a.v * b.x, a.y * b.v + a.v * b.y, a.z * b.v + a.v * b.z};
}
// acc += s a
template <class T> __device__ __forceinline__ void dAxpy(Dual<T>& acc, T s, Dual<T> a)
{
   acc.v += s * a.v; acc.x += s * a.x; acc.y += s * a.y; acc.z += s * a.z;
}

constexpr int TC_STACK = 192;   // 7 siblings a level x 21 levels + the root, with room to spare
constexpr int TC_NT = 128;

// sum_k M~[c][k] I_k(u) for the three components c, with gradients with respect to u, in the standard
// real irregular convention (I_l^0 = (-1)^l Re T_l^0, I_l^{+-m} = (-1)^l sqrt2 {Re, Im} T_l^m, T the
// complex irregular harmonic of fmm_common.cuh, whose recurrence this runs on dual numbers).
template <class T, bool GRAD>
__device__ void irregularSum(int p, int Lp, const T* __restrict__ M, T ux, T uy, T uz, Dual<T> acc[3])
{
   const T sq2 = T(1.4142135623730950488);
   const Dual<T> X{ux, T(1), T(0), T(0)}, Y{uy, T(0), T(1), T(0)}, Z{uz, T(0), T(0), T(1)};
   const T r2 = ux * ux + uy * uy + uz * uz;
   const T i2 = T(1) / r2, ir = sqrt(i2);
   // 1 / r^2 and 1 / r as duals
   const Dual<T> IR2{i2, -T(2) * ux * i2 * i2, -T(2) * uy * i2 * i2, -T(2) * uz * i2 * i2};
   const T ir3 = ir * i2;
   Dual<T> dre{ir, -ux * ir3, -uy * ir3, -uz * ir3}, dim{T(0), T(0), T(0), T(0)};   // T_m^m
   for(int c = 0; c < 3; c++) acc[c] = {T(0), T(0), T(0), T(0)};
   for(int m = 0; m <= p; m++)
   {
      if(m > 0)
      {
         // T_m^m = (2m - 1) (x + i y) T_{m-1}^{m-1} / r^2
         const T f = T(2 * m - 1);
         const Dual<T> nre = dMul(dSub(dMul(X, dre), dMul(Y, dim)), IR2);
         const Dual<T> nim = dMul(dAdd(dMul(X, dim), dMul(Y, dre)), IR2);
         dre = dScale(nre, f);
         dim = dScale(nim, f);
      }
      Dual<T> are = dre, aim = dim, bre{T(0), T(0), T(0), T(0)}, bim{T(0), T(0), T(0), T(0)};
      for(int l = m; l <= p; l++)
      {
         const T s = (l & 1) ? T(-1) : T(1);
         if(m == 0)
         {
            const int k = l * l + l;
            for(int c = 0; c < 3; c++) dAxpy(acc[c], s * M[c * Lp + k], are);
         }
         else
         {
            const int kp = l * l + l + m, km = l * l + l - m;
            for(int c = 0; c < 3; c++)
            {
               dAxpy(acc[c], s * sq2 * M[c * Lp + kp], are);
               dAxpy(acc[c], s * sq2 * M[c * Lp + km], aim);
            }
         }
         if(l == p) break;
         Dual<T> cre, cim;
         if(l == m)
         {
            const T f = T(2 * m + 1);
            cre = dScale(dMul(dMul(Z, are), IR2), f);
            cim = dScale(dMul(dMul(Z, aim), IR2), f);
         }
         else
         {
            const T f = T(2 * l + 1), g = T((l + m) * (l - m));
            cre = dMul(dSub(dScale(dMul(Z, are), f), dScale(bre, g)), IR2);
            cim = dMul(dSub(dScale(dMul(Z, aim), f), dScale(bim, g)), IR2);
         }
         bre = are; bim = aim; are = cre; aim = cim;
      }
   }
   (void)GRAD;
}

template <class T>
__global__ void __launch_bounds__(TC_NT) kTreecode(Tree t, const RootBox* __restrict__ rootp, int p, int Lp,
                                                   const T* __restrict__ mult, const typename Vec4<T>::type* __restrict__ spos,
                                                   const typename Vec4<T>::type* __restrict__ sq, const T* __restrict__ pts,
                                                   int64_t m, int flags, T scaleB, T scaleA, int want, int bem,
                                                   T* __restrict__ outB, T* __restrict__ outA, int* err)
{
   const int64_t qi = blockIdx.x * int64_t(TC_NT) + threadIdx.x;
   if(qi >= m) return;
   const bool refNear = flags & 1, fdCurl = flags & 2;
   const RootBox rb = rootp[0];
   const double x = double(pts[3 * qi]), y = double(pts[3 * qi + 1]), z = double(pts[3 * qi + 2]);
   double A[3] = {0, 0, 0}, G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // A_c and dA_c / dx_j
   double Bn[3] = {0, 0, 0};                                              // direct near-field B
   int stack[TC_STACK];
   int top = 0;
   for(int r = t.levelStart[0]; r < t.levelStart[1]; r++) stack[top++] = r;
   const T eps = T(1e-3);   // the reference's math::eps for the central differences
   while(top > 0)
   {
      const int node = stack[--top];
      const int level = t.level[node];
      const double h = 2.0 * rb.H / double(int64_t(1) << level);
      const double cx = rb.center[0] - rb.H + (double(t.ix[node]) + 0.5) * h;
      const double cy = rb.center[1] - rb.H + (double(t.iy[node]) + 0.5) * h;
      const double cz = rb.center[2] - rb.H + (double(t.iz[node]) + 0.5) * h;
      const double dx = x - cx, dy = y - cy, dz = z - cz;
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double r2 = 3.0 * 0.25 * h * h;   // half-diagonal^2: three half-widths h / 2
      if(4.0 * r2 < d2)
      {
         const T* M = mult + int64_t(node) * 3 * Lp;
         const double ih = 1.0 / h;
         if(!fdCurl)
         {
            Dual<T> acc[3];
            irregularSum<T, true>(p, Lp, M, T(dx * ih), T(dy * ih), T(dz * ih), acc);
            for(int c = 0; c < 3; c++)
            {
               A[c] += double(acc[c].v) * ih;
               G[c][0] += double(acc[c].x) * ih * ih;
               G[c][1] += double(acc[c].y) * ih * ih;
               G[c][2] += double(acc[c].z) * ih * ih;
            }
         }
         else
         {
            Dual<T> acc[3];
            irregularSum<T, false>(p, Lp, M, T(dx * ih), T(dy * ih), T(dz * ih), acc);
            for(int c = 0; c < 3; c++) A[c] += double(acc[c].v) * ih;
            if(want & 1)
               for(int j = 0; j < 3; j++)
               {
                  Dual<T> ap[3], am[3];
                  const double e = double(eps) * ih;
                  irregularSum<T, false>(p, Lp, M, T(dx * ih + (j == 0 ? e : 0.0)), T(dy * ih + (j == 1 ? e : 0.0)),
                                         T(dz * ih + (j == 2 ? e : 0.0)), ap);
                  irregularSum<T, false>(p, Lp, M, T(dx * ih - (j == 0 ? e : 0.0)), T(dy * ih - (j == 1 ? e : 0.0)),
                                         T(dz * ih - (j == 2 ? e : 0.0)), am);
                  for(int c = 0; c < 3; c++) G[c][j] += double(ap[c].v - am[c].v) * ih / (2.0 * double(eps));
               }
         }
         continue;
      }
      const int nc = t.nchild[node];
      if(nc == 0)
      {
         if(refNear) continue;
         // direct sum over the leaf's sources (coincident points skipped)
         for(int i = t.s0[node]; i < t.s1[node]; i++)
         {
            const auto q = spos[i];
            const auto s = sq[i];
            const double ex = x - double(q.x), ey = y - double(q.y), ez = z - double(q.z);
            const double e2 = ex * ex + ey * ey + ez * ez;
            if(e2 == 0.0) continue;
            const double ri = 1.0 / sqrt(e2), ri3 = ri * ri * ri;
            if(bem)
            {
               // the BEM kernel sigma d / |d|^3 + d x s / |d|^3 with d = q - x = -(ex, ey, ez) (fmm_bem.cu)
               const double sg = double(s.w);
               A[0] -= (sg * ex + (ey * double(s.z) - ez * double(s.y))) * ri3;
               A[1] -= (sg * ey + (ez * double(s.x) - ex * double(s.z))) * ri3;
               A[2] -= (sg * ez + (ex * double(s.y) - ey * double(s.x))) * ri3;
               continue;
            }
            Bn[0] += (double(s.y) * ez - double(s.z) * ey) * ri3;
            Bn[1] += (double(s.z) * ex - double(s.x) * ez) * ri3;
            Bn[2] += (double(s.x) * ey - double(s.y) * ex) * ri3;
            A[0] += double(s.x) * ri;
            A[1] += double(s.y) * ri;
            A[2] += double(s.z) * ri;
         }
         continue;
      }
      if(top + nc > TC_STACK)
      {
         atomicOr(err, ERR_DFS);
         break;
      }
      const int c0 = t.child0[node];
      for(int c = 0; c < nc; c++) stack[top++] = c0 + c;
   }
   if(want & 1)
   {
      const double B0 = G[2][1] - G[1][2] + Bn[0];
      const double B1 = G[0][2] - G[2][0] + Bn[1];
      const double B2 = G[1][0] - G[0][1] + Bn[2];
      outB[3 * qi] = T(B0 * double(scaleB));
      outB[3 * qi + 1] = T(B1 * double(scaleB));
      outB[3 * qi + 2] = T(B2 * double(scaleB));
   }
   if(want & 2)
      for(int c = 0; c < 3; c++) outA[3 * qi + c] = T(A[c] * double(scaleA));
}

}  // namespace

template <class T>
fmm_status treecodeT(Plan& P, double current, int want, const void* pts, int64_t m, void* outB, void* outA, int flags,
                     cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   if(m == 0) return FMM_OK;
   // A (and, for BEM sources, the BEM integral) times current / (4 pi), as MultipoleSolver::calcA
   // (multipole_solver.cpp:686-692) scales both
   const T scaleB = T(REF_MU0 / (4 * REF_PI) * current), scaleA = T(1.0 / (4 * REF_PI) * current);
   FMM_CUDA(cudaMemsetAsync(P.err, 0, sizeof(int), st));
   const int blocks = int((m + TC_NT - 1) / TC_NT);
   kTreecode<T><<<blocks, TC_NT, 0, st>>>(P.tree, P.root, P.p, P.Lp, (const T*)P.mult.ptr, (const V4*)P.sPos.ptr,
                                          (const V4*)P.sQ.ptr, (const T*)pts, m, flags, scaleB, scaleA, want, P.bem ? 1 : 0, (T*)outB,
                                          (T*)outA, P.err);
   FMM_TRY(launched(P, "kTreecode", st));
   int herr = 0;
   FMM_CUDA(cudaMemcpyAsync(&herr, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
   FMM_CUDA(cudaStreamSynchronize(st));
   if(herr) return setError(FMM_E_LIMIT, "fmm_treecode: the descent stack overflowed (code %d)", herr);
   return FMM_OK;
}

template fmm_status treecodeT<float>(Plan&, double, int, const void*, int64_t, void*, void*, int, cudaStream_t);
template fmm_status treecodeT<double>(Plan&, double, int, const void*, int64_t, void*, void*, int, cudaStream_t);

}  // namespace fmm
