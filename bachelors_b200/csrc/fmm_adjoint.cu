// Adjoint (transposed) FMM: gradients of a loss of B with respect to the current densities J and
// the source positions. No counterpart in the reference, which has no gradients.
//
// With g_t = dLoss/dB(x_t) and c = mu0 I / (4 pi), the forward sum B_t = c sum_q w_q J_q x (x_t - q)/r^3
// gives
//   dLoss/dJ_q = c w_q C(q),        C(y) = sum_t g_t x (y - x_t) / |y - x_t|^3
//   dLoss/dq   = c w_q grad_y (J_q . C(y)) at y = q   (+ c w_q (dJ/dq)^T C(q) for the azimuthal J)
// C is itself a Biot-Savart field: the targets act as sources of strength g_t and the source points
// as targets, so the adjoint is one FMM on the swapped point sets (same tree when the two leaf
// capacities agree), evaluated with first and second derivatives of the local expansions: C = curl A
// and grad C from the coefficient-space derivative identities applied twice. Near pairs are summed
// directly with the exact kernel derivative  a / r^3 - 3 (e . a) e / r^5,  e = q - x_t, a = J_q x g_t.
#include "fmm_internal.cuh"

namespace fmm {

template <class T>
__device__ inline T coefAtA(const T* Lv, int l, int m)
{
   return (abs(m) <= l) ? Lv[hidx(l, m)] : T(0);
}

// Coefficient of R_{l'}^{mu} in d/dx_j (sum_k V_k R_k), j = 0 (x), 1 (y), 2 (z); l = l' + 1.
// (Same identities as the forward L2P.)
template <class T>
__device__ inline T gradCoeffA(const T* Lv, int j, int lp, int mu)
{
   const int l = lp + 1;
   const T h = T(0.5), r2 = T(0.70710678118654752440);
   if(j == 2) return -coefAtA(Lv, l, mu);
   if(j == 0)
   {
      if(mu == 0) return -r2 * coefAtA(Lv, l, 1);
      if(mu == 1) return -h * coefAtA(Lv, l, 2) + r2 * coefAtA(Lv, l, 0);
      if(mu >= 2) return -h * coefAtA(Lv, l, mu + 1) + h * coefAtA(Lv, l, mu - 1);
      if(mu == -1) return -h * coefAtA(Lv, l, -2);
      return -h * coefAtA(Lv, l, mu - 1) + h * coefAtA(Lv, l, mu + 1);
   }
   if(mu == 0) return -r2 * coefAtA(Lv, l, -1);
   if(mu == 1) return -h * coefAtA(Lv, l, -2);
   if(mu >= 2) return -h * coefAtA(Lv, l, -(mu + 1)) - h * coefAtA(Lv, l, -(mu - 1));
   if(mu == -1) return h * coefAtA(Lv, l, 2) + r2 * coefAtA(Lv, l, 0);
   return h * coefAtA(Lv, l, 1 - mu) + h * coefAtA(Lv, l, -mu - 1);
}

__device__ inline void lmOf(int k, int& l, int& m)
{
   l = int(sqrtf(float(k)));
   while(l * l > k) l--;
   while((l + 1) * (l + 1) <= k) l++;
   m = k - l * l - l;
}

// One block per leaf of the adjoint tree holding targets (= forward sources). Outputs in the
// forward source input order.
template <class T, int NT>
__global__ void __launch_bounds__(NT) kAdjointEval(Tree t, const RootBox* __restrict__ rootp, int p, int Lp,
                                                   const T* __restrict__ Lc,
                                                   const typename Vec4<T>::type* __restrict__ tpos,
                                                   const typename Vec4<T>::type* __restrict__ spos,
                                                   const typename Vec4<T>::type* __restrict__ sq,
                                                   const int* __restrict__ p2pOff, const int* __restrict__ p2pList,
                                                   const int* __restrict__ tOrder, const T* __restrict__ fw,
                                                   const T* __restrict__ fJ, double scale, T* __restrict__ dJ,
                                                   T* __restrict__ dx)
{
   typedef typename Vec4<T>::type V4;
   extern __shared__ __align__(32) unsigned char smraw[];
   const int node = blockIdx.x;
   if(t.nchild[node] != 0 || t.t1[node] == t.t0[node]) return;
   const int L = nharm(p), L1 = nharm(p - 1), L2 = nharm(p - 2 >= 0 ? p - 2 : 0);
   T* Ls = (T*)smraw;          // [3][L]   local expansion of A (adjoint vector potential)
   T* Cs = Ls + 3 * L;         // [3][L1]  expansion of C = curl A
   T* Ds = Cs + 3 * L1;        // [3][3][L2] expansions of d C_c / d x_j
   const size_t coefBytes = (sizeof(T) * (3 * L + 3 * L1 + 9 * L2) + 31) & ~size_t(31);
   V4* Sp = (V4*)(smraw + coefBytes);
   V4* Sq = Sp + NT;
   for(int e = threadIdx.x; e < 3 * L; e += NT) Ls[e] = Lc[int64_t(node) * 3 * Lp + (e / L) * Lp + e % L];
   __syncthreads();
   for(int e = threadIdx.x; e < 3 * L1; e += NT)
   {
      const int c = e / L1, k = e % L1;
      int lp, mu;
      lmOf(k, lp, mu);
      const int cp = (c + 2) % 3, cm = (c + 1) % 3, jp = (c + 1) % 3, jm = (c + 2) % 3;
      Cs[e] = gradCoeffA(Ls + cp * L, jp, lp, mu) - gradCoeffA(Ls + cm * L, jm, lp, mu);
   }
   __syncthreads();
   if(p >= 2)
      for(int e = threadIdx.x; e < 9 * L2; e += NT)
      {
         const int cj = e / L2, k = e % L2;
         const int c = cj / 3, j = cj % 3;
         int lp, mu;
         lmOf(k, lp, mu);
         Ds[e] = gradCoeffA(Cs + c * L1, j, lp, mu);
      }
   __syncthreads();
   const RootBox rb = rootp[rootOf(t, node)];
   double ctr[3], h;
   {
      const int lev = t.level[node];
      h = 2.0 * rb.H / double(int64_t(1) << lev);
      ctr[0] = rb.center[0] - rb.H + (double(t.ix[node]) + 0.5) * h;
      ctr[1] = rb.center[1] - rb.H + (double(t.iy[node]) + 0.5) * h;
      ctr[2] = rb.center[2] - rb.H + (double(t.iz[node]) + 0.5) * h;
   }
   const T ih2 = T(1.0 / (h * h)), ih3 = T(1.0 / (h * h * h));
   const int t0 = t.t0[node], t1 = t.t1[node];
   const int e0 = p2pOff[node], e1 = p2pOff[node + 1];
   for(int base = t0; base < t1; base += NT)
   {
      const int ti = base + threadIdx.x;
      const bool active = ti < t1;
      const V4 x = active ? tpos[ti] : V4{T(0), T(0), T(0), T(0)};
      const int o = active ? tOrder[ti] : 0;
      T Jq[3] = {T(0), T(0), T(0)};
      if(active)
      {
         if(fJ) { Jq[0] = fJ[3 * o]; Jq[1] = fJ[3 * o + 1]; Jq[2] = fJ[3 * o + 2]; }
         else
         {
            const T l = sqrt(x.x * x.x + x.y * x.y);
            if(l != T(0)) { Jq[0] = -x.y / l; Jq[1] = x.x / l; }
         }
      }
      T C[3] = {T(0), T(0), T(0)}, D[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
      if(active)
      {
         const T ux = T((double(x.x) - ctr[0]) / h), uy = T((double(x.y) - ctr[1]) / h), uz = T((double(x.z) - ctr[2]) / h);
         const T sq2 = T(1.4142135623730950488);
         visitRegular<T>(p - 1, ux, uy, uz, [&](int l, int m, T re, T im) {
            const T s = (l & 1) ? T(-1) : T(1);
            T r0, r1;
            if(m == 0) { r0 = s * re; r1 = T(0); }
            else { r0 = s * sq2 * re; r1 = s * sq2 * im; }
            const int k0 = hidx(l, m), k1 = hidx(l, -m);
            for(int c = 0; c < 3; c++)
            {
               C[c] += Cs[c * L1 + k0] * r0;
               if(m) C[c] += Cs[c * L1 + k1] * r1;
            }
            if(l <= p - 2)
               for(int c = 0; c < 3; c++)
                  for(int j = 0; j < 3; j++)
                  {
                     const T* dv = Ds + (3 * c + j) * L2;
                     D[c][j] += dv[k0] * r0;
                     if(m) D[c][j] += dv[k1] * r1;
                  }
         });
      }
      double Cd[3], Gd[3];
      for(int c = 0; c < 3; c++) Cd[c] = double(C[c] * ih2);
      for(int j = 0; j < 3; j++) Gd[j] = double((Jq[0] * D[0][j] + Jq[1] * D[1][j] + Jq[2] * D[2][j]) * ih3);
      // near field: adjoint sources are the forward targets with strength g
      for(int e = e0; e < e1; e++)
      {
         const int S = p2pList[e];
         const int a0 = t.s0[S], a1 = t.s1[S];
         for(int sb = a0; sb < a1; sb += NT)
         {
            const int cnt = min(NT, a1 - sb);
            __syncthreads();
            if(threadIdx.x < cnt) { Sp[threadIdx.x] = spos[sb + threadIdx.x]; Sq[threadIdx.x] = sq[sb + threadIdx.x]; }
            __syncthreads();
            if(active)
            {
               T pc[3] = {T(0), T(0), T(0)}, pg[3] = {T(0), T(0), T(0)};
               for(int i = 0; i < cnt; i++)
               {
                  const V4 y = Sp[i], g = Sq[i];
                  const T ex = x.x - y.x, ey = x.y - y.y, ez = x.z - y.z;
                  const T r2 = ex * ex + ey * ey + ez * ez;
                  if(r2 == T(0)) continue;
                  T ri;
                  if constexpr(sizeof(T) == 4) ri = rsqrtf(r2);
                  else ri = rsqrt(r2);
                  const T ri2 = ri * ri, ri3 = ri2 * ri, ri5 = ri3 * ri2;
                  pc[0] += (g.y * ez - g.z * ey) * ri3;
                  pc[1] += (g.z * ex - g.x * ez) * ri3;
                  pc[2] += (g.x * ey - g.y * ex) * ri3;
                  const T ax = Jq[1] * g.z - Jq[2] * g.y, ay = Jq[2] * g.x - Jq[0] * g.z, az = Jq[0] * g.y - Jq[1] * g.x;
                  const T ea3 = T(3) * (ex * ax + ey * ay + ez * az) * ri5;
                  pg[0] += ax * ri3 - ea3 * ex;
                  pg[1] += ay * ri3 - ea3 * ey;
                  pg[2] += az * ri3 - ea3 * ez;
               }
               for(int d = 0; d < 3; d++) { Cd[d] += double(pc[d]); Gd[d] += double(pg[d]); }
            }
         }
      }
      if(active)
      {
         if(!fJ)
         {
            // derivative of the azimuthal direction (-y, x, 0) / rho
            const double X = double(x.x), Y = double(x.y), rho2 = X * X + Y * Y;
            if(rho2 > 0)
            {
               const double ir = 1.0 / (rho2 * sqrt(rho2));
               Gd[0] += (X * Y * Cd[0] + Y * Y * Cd[1]) * ir;
               Gd[1] += (-X * X * Cd[0] - X * Y * Cd[1]) * ir;
            }
         }
         const double s = scale * double(fw[o]);
         for(int d = 0; d < 3; d++)
         {
            if(dJ) dJ[3 * int64_t(o) + d] = T(s * Cd[d]);
            if(dx) dx[3 * int64_t(o) + d] = T(s * Gd[d]);
         }
      }
   }
}

// Direct-sum adjoint, one thread per source (input order); the targets and their g stream through
// shared memory in tiles; C and grad(J . C) accumulate in FP64. blockIdx.y selects a coil: its
// sources [srcOff[c], srcOff[c+1]) see only its targets [tgtOff[c], tgtOff[c+1]).
template <class T, int NT>
__global__ void __launch_bounds__(NT) kAdjointDirect(const T* __restrict__ sxyz, const T* __restrict__ sw,
                                                     const T* __restrict__ sJ, const T* __restrict__ txyz,
                                                     const T* __restrict__ g, const int* __restrict__ srcOff,
                                                     const int* __restrict__ tgtOff, double scale, T* __restrict__ dJ,
                                                     T* __restrict__ dx)
{
   __shared__ double Tx[NT][3], Tg[NT][3];
   const int c = blockIdx.y;
   const int sBeg = srcOff[c], sEnd = srcOff[c + 1], tBeg = tgtOff[c], tEnd = tgtOff[c + 1];
   if(sBeg + int(blockIdx.x) * NT >= sEnd) return;
   const int q = sBeg + blockIdx.x * NT + threadIdx.x;
   const bool active = q < sEnd;
   double X = 0, Y = 0, Z = 0, j[3] = {0, 0, 0};
   if(active)
   {
      X = double(sxyz[3 * q]); Y = double(sxyz[3 * q + 1]); Z = double(sxyz[3 * q + 2]);
      if(sJ) { j[0] = double(sJ[3 * q]); j[1] = double(sJ[3 * q + 1]); j[2] = double(sJ[3 * q + 2]); }
      else
      {
         const double rho = sqrt(X * X + Y * Y);
         if(rho > 0) { j[0] = -Y / rho; j[1] = X / rho; }
      }
   }
   double C[3] = {0, 0, 0}, G[3] = {0, 0, 0};
   for(int tb = tBeg; tb < tEnd; tb += NT)
   {
      const int cnt = min(NT, tEnd - tb);
      __syncthreads();
      if(threadIdx.x < cnt)
         for(int d = 0; d < 3; d++)
         {
            Tx[threadIdx.x][d] = double(txyz[3 * (tb + threadIdx.x) + d]);
            Tg[threadIdx.x][d] = double(g[3 * (tb + threadIdx.x) + d]);
         }
      __syncthreads();
      if(!active) continue;
      for(int i = 0; i < cnt; i++)
      {
         const double ex = X - Tx[i][0], ey = Y - Tx[i][1], ez = Z - Tx[i][2];
         const double r2 = ex * ex + ey * ey + ez * ez;
         if(r2 == 0) continue;
         const double ri = 1.0 / sqrt(r2), ri3 = ri * ri * ri, ri5 = ri3 * ri * ri;
         const double gx = Tg[i][0], gy = Tg[i][1], gz = Tg[i][2];
         C[0] += (gy * ez - gz * ey) * ri3;
         C[1] += (gz * ex - gx * ez) * ri3;
         C[2] += (gx * ey - gy * ex) * ri3;
         const double ax = j[1] * gz - j[2] * gy, ay = j[2] * gx - j[0] * gz, az = j[0] * gy - j[1] * gx;
         const double ea3 = 3.0 * (ex * ax + ey * ay + ez * az) * ri5;
         G[0] += ax * ri3 - ea3 * ex;
         G[1] += ay * ri3 - ea3 * ey;
         G[2] += az * ri3 - ea3 * ez;
      }
   }
   if(!active) return;
   if(!sJ)
   {
      // derivative of the azimuthal direction (-y, x, 0) / rho
      const double rho2 = X * X + Y * Y;
      if(rho2 > 0)
      {
         const double ir = 1.0 / (rho2 * sqrt(rho2));
         G[0] += (X * Y * C[0] + Y * Y * C[1]) * ir;
         G[1] += (-X * X * C[0] - X * Y * C[1]) * ir;
      }
   }
   const double s = scale * double(sw[q]);
   for(int d = 0; d < 3; d++)
   {
      if(dJ) dJ[3 * int64_t(q) + d] = T(s * C[d]);
      if(dx) dx[3 * int64_t(q) + d] = T(s * G[d]);
   }
}

template <class T>
fmm_status adjointDirectT(Plan& P, double current, const void* g, void* dJ, void* dx, cudaStream_t st)
{
   constexpr int NT = 128;
   const int K = P.nCoils;
   if(!P.batch)
   {
      P.srcOff.assign({0, int(P.n)});
      P.tgtOff.assign({0, int(P.m)});
   }
   if(int(P.srcOff.size()) != K + 1 || P.srcOff[K] != P.n || P.tgtOff[K] != P.m)
      return setError(FMM_E_INVALID, "coil offsets do not match the source/target counts");
   FMM_TRY(P.segb.reserve(sizeof(int) * 2 * (K + 1)));
   int* so = (int*)P.segb.ptr;
   int* to = so + K + 1;
   FMM_CUDA(cudaMemcpyAsync(so, P.srcOff.data(), sizeof(int) * (K + 1), cudaMemcpyHostToDevice, st));
   FMM_CUDA(cudaMemcpyAsync(to, P.tgtOff.data(), sizeof(int) * (K + 1), cudaMemcpyHostToDevice, st));
   int maxS = 0;
   for(int c = 0; c < K; c++) maxS = std::max(maxS, P.srcOff[c + 1] - P.srcOff[c]);
   if(maxS == 0) return FMM_OK;
   const double scale = REF_MU0 / (4 * REF_PI) * current;
   kAdjointDirect<T, NT><<<dim3((maxS + NT - 1) / NT, K), NT, 0, st>>>(
      (const T*)P.srcXYZ, (const T*)P.srcW, P.hasJ ? (const T*)P.srcJ : nullptr, (const T*)P.tgtXYZ, (const T*)g, so,
      to, scale, (T*)dJ, (T*)dx);
   FMM_TRY(launched(P, "kAdjointDirect", st));
   return FMM_OK;
}

template fmm_status adjointDirectT<float>(Plan&, double, const void*, void*, void*, cudaStream_t);
template fmm_status adjointDirectT<double>(Plan&, double, const void*, void*, void*, cudaStream_t);

template <class T>
__global__ void kFill(T* a, int64_t n, T v)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i < n) a[i] = v;
}

template <class T>
fmm_status adjointT(Plan& P, Plan& A, double current, const void* g, void* dJ, void* dx, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   const size_t es = sizeof(T);
   // adjoint problem: sources = forward targets with unit weight and "current" g; targets = forward sources
   FMM_TRY(A.srcXYZb.reserve(es * 3 * std::max<int64_t>(P.m, 1)));
   FMM_TRY(A.srcWb.reserve(es * std::max<int64_t>(P.m, 1)));
   FMM_TRY(A.srcJb.reserve(es * 3 * std::max<int64_t>(P.m, 1)));
   FMM_TRY(A.tgtXYZb.reserve(es * 3 * std::max<int64_t>(P.n, 1)));
   if(P.m) FMM_CUDA(cudaMemcpyAsync(A.srcXYZb.ptr, P.tgtXYZ, es * 3 * P.m, cudaMemcpyDeviceToDevice, st));
   if(P.m) FMM_CUDA(cudaMemcpyAsync(A.srcJb.ptr, g, es * 3 * P.m, cudaMemcpyDeviceToDevice, st));
   if(P.n) FMM_CUDA(cudaMemcpyAsync(A.tgtXYZb.ptr, P.srcXYZ, es * 3 * P.n, cudaMemcpyDeviceToDevice, st));
   if(P.m)
   {
      kFill<T><<<int((P.m + 255) / 256), 256, 0, st>>>((T*)A.srcWb.ptr, P.m, T(1));
      FMM_TRY(launched(A, "kFill", st));
   }
   A.srcXYZ = A.srcXYZb.ptr; A.srcW = A.srcWb.ptr; A.srcJ = A.srcJb.ptr; A.tgtXYZ = A.tgtXYZb.ptr;
   A.hasJ = true;
   A.n = P.m;
   A.m = P.n;
   FMM_TRY(buildTreeT<T>(A, st));
   FMM_TRY(upwardT<T>(A, st));
   FMM_TRY(downwardT<T>(A, st));
   constexpr int NT = 64;
   const int p = A.p;
   const int L = nharm(p), L1 = nharm(p - 1), L2 = nharm(p >= 2 ? p - 2 : 0);
   size_t shm = ((sizeof(T) * (3 * L + 3 * L1 + 9 * L2) + 31) & ~size_t(31)) + 2 * sizeof(V4) * NT;
   FMM_CUDA(cudaFuncSetAttribute(kAdjointEval<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
   const double scale = REF_MU0 / (4 * REF_PI) * current;
   kAdjointEval<T, NT><<<int(A.tree.nNodes), NT, shm, st>>>(
      A.tree, A.root, p, A.Lp, (const T*)A.local.ptr, (const V4*)A.tPos.ptr, (const V4*)A.sPos.ptr,
      (const V4*)A.sQ.ptr, (const int*)A.p2pOff.ptr, (const int*)A.p2pList.ptr, (const int*)A.tIdx.ptr,
      (const T*)P.srcW, P.hasJ ? (const T*)P.srcJ : nullptr, scale, (T*)dJ, (T*)dx);
   FMM_TRY(launched(A, "kAdjointEval", st));
   return FMM_OK;
}

template fmm_status adjointT<float>(Plan&, Plan&, double, const void*, void*, void*, cudaStream_t);
template fmm_status adjointT<double>(Plan&, Plan&, double, const void*, void*, void*, cudaStream_t);

}  // namespace fmm
