// FMM kernels for sm_100a: translation-operator tables (FP64), P2M, M2M, M2L (CUDA-core
// form), L2L, and the fused L2P + direct near field.
//
// Every expansion is stored box-size scaled: a node of side h keeps M~_l = M_l / h^l and
// L~_l = L_l h^(l+1). With that scaling the M2M, L2L and M2L operators do not depend on the
// level: 8 M2M and 8 L2L operators (one per child octant) and 316 M2L operators (one per
// offset o in [-3,3]^3 outside [-1,1]^3), all built once per order in FP64.
//
// Reference counterparts (FMM/FMMGPU/):
//   P2M   math::calcIntegralContribution                     integration.cpp:137-161
//   M2M   MultipoleTranslator::translateMultipoleWithComplex  multipole_translator.cpp:3-32,111-125,143-146
//   M2L   multipoleToLocalWithComplex (l + lambda <= p)       multipole_translator.cpp:148-199
//   L2L   translateLocalWithComplex                          multipole_translator.cpp:201-255
//   L2P   CalculationPointOctreeNode::calcA / calcRot        calculation_point_octree.cpp:192-275
//         (B from analytic gradients here, finite differences there)
//   near  bioSavartLaplaceFunction                           integration.cpp:113-120
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include <cuda_bf16.h>

#include <cub/cub.cuh>

#include "fmm_internal.cuh"

namespace fmm {

__constant__ int d_m2lIndex[NOFF];
__constant__ int d_m2lOffset[316];
__constant__ int d_m2lFarFirst[316];

// Constant memory is per device context: fill it once on every device that uses the library.
fmm_status initOffsetTables()
{
   static bool done[64] = {false};
   int dev = 0;
   FMM_CUDA(cudaGetDevice(&dev));
   if(dev < 64 && done[dev]) return FMM_OK;
   int idx[NOFF], off[316];
   int k = 0;
   for(int oz = -3; oz <= 3; oz++)
      for(int oy = -3; oy <= 3; oy++)
         for(int ox = -3; ox <= 3; ox++)
         {
            int o = offsetIndex(ox, oy, oz);
            if(abs(ox) <= 1 && abs(oy) <= 1 && abs(oz) <= 1) idx[o] = -1;
            else { idx[o] = k; off[k] = o; k++; }
         }
   int far[316];
   for(int i = 0; i < 316; i++) far[i] = i;
   auto len2 = [&](int slot) {
      int o = off[slot];
      int ox = o % 7 - 3, oy = (o / 7) % 7 - 3, oz = o / 49 - 3;
      return ox * ox + oy * oy + oz * oz;
   };
   std::stable_sort(far, far + 316, [&](int a, int b) { return len2(a) > len2(b); });
   FMM_CUDA(cudaMemcpyToSymbol(d_m2lFarFirst, far, sizeof(far)));
   FMM_CUDA(cudaMemcpyToSymbol(d_m2lIndex, idx, sizeof(idx)));
   FMM_CUDA(cudaMemcpyToSymbol(d_m2lOffset, off, sizeof(off)));
   if(dev < 64) done[dev] = true;
   return FMM_OK;
}

// ====================================================================================
// Operator tables. Entry (i, j) of a translation in the real basis, derived from the
// reference's complex form res(l,m) = sum a(lambda,mu) G(l,m,lambda,mu) between the
// realToComplex / complexToReal conversions (harmonics.cpp:340-379), with exact 1/sqrt2.
// ====================================================================================
struct C2 { double re, im; };

__device__ inline C2 cplxOf(const double* H, int n, int k)
{
   const double s = 0.70710678118654752440;
   if(k == 0) return {H[hidx(n, 0)], 0.0};
   int a = abs(k);
   return {s * H[hidx(n, a)], (k > 0 ? s : -s) * H[hidx(n, -a)]};
}

__device__ inline double signPow(int t) { int e = (-t) / 2; return (e & 1) ? -1.0 : 1.0; }

// kind 0 = M2M, 1 = L2L, 2 = M2L. H = real harmonics of the translation (regular for
// M2M / L2L, irregular to order `lim` for M2L).
__device__ C2 translationG(int kind, int l, int m, int lam, int mu, const double* H, int lim)
{
   if(kind == 0)
   {
      int dl = l - lam, dm = m - mu;
      if(dl < 0 || abs(dm) > dl) return {0, 0};
      C2 b = cplxOf(H, dl, dm);
      double f = signPow(abs(m) - abs(m - mu) - abs(mu));
      return {b.re * f, b.im * f};
   }
   if(kind == 1)
   {
      int dl = lam - l, dm = m - mu;
      if(dl < 0 || abs(dm) > dl) return {0, 0};
      C2 b = cplxOf(H, dl, dm);
      double f = signPow(abs(mu) - abs(m - mu) - abs(m)) * (((lam + l) & 1) ? -1.0 : 1.0);
      return {b.re * f, b.im * f};
   }
   int dl = l + lam, dm = m - mu;
   if(dl > lim) return {0, 0};
   C2 b = cplxOf(H, dl, dm);
   double f = signPow(abs(m - mu) - abs(m) - abs(mu)) * ((lam & 1) ? -1.0 : 1.0);
   return {b.re * f, b.im * f};
}

__device__ double operatorEntry(int kind, int i, int j, const double* H, int lim)
{
   const double s = 0.70710678118654752440;
   int l = int(sqrt(double(i))); while(l * l > i) l--; while((l + 1) * (l + 1) <= i) l++;
   int mi = i - l * l - l;
   int lam = int(sqrt(double(j))); while(lam * lam > j) lam--; while((lam + 1) * (lam + 1) <= j) lam++;
   int mj = j - lam * lam - lam;
   // complex input of the unit real vector e_j
   int mus[2]; C2 as[2]; int nin;
   if(mj == 0) { mus[0] = 0; as[0] = {1, 0}; nin = 1; }
   else if(mj > 0) { mus[0] = mj; as[0] = {s, 0}; mus[1] = -mj; as[1] = {s, 0}; nin = 2; }
   else { mus[0] = -mj; as[0] = {0, s}; mus[1] = mj; as[1] = {0, -s}; nin = 2; }
   auto res = [&](int m) {
      C2 r = {0, 0};
      for(int e = 0; e < nin; e++)
      {
         C2 g = translationG(kind, l, m, lam, mus[e], H, lim);
         r.re += as[e].re * g.re - as[e].im * g.im;
         r.im += as[e].re * g.im + as[e].im * g.re;
      }
      return r;
   };
   if(mi == 0) return res(0).re;
   if(mi > 0) return s * (res(mi).re + res(-mi).re);
   return s * (res(-mi).im - res(mi).im);
}

// One block per operator. op < 8: M2M octant, op < 16: L2L octant, else M2L slot.
__global__ void kBuildOperators(int p, int lim, int first, int count, double* m2m, double* l2l, double* m2l)
{
   extern __shared__ double Hs[];
   int op = first + blockIdx.x;
   if(blockIdx.x >= count) return;
   int L = nharm(p);
   int kind = op < 8 ? 0 : (op < 16 ? 1 : 2);
   if(threadIdx.x == 0)
   {
      if(kind < 2)
      {
         int oct = op & 7;
         double t[3] = {((oct & 1) - 0.5) * 0.5, (((oct >> 1) & 1) - 0.5) * 0.5, (((oct >> 2) & 1) - 0.5) * 0.5};
         if(kind == 1) { t[0] = -t[0]; t[1] = -t[1]; t[2] = -t[2]; }
         realRegular<double>(p, t[0], t[1], t[2], Hs);
      }
      else
      {
         int o = d_m2lOffset[op - 16];
         int ox = o % 7 - 3, oy = (o / 7) % 7 - 3, oz = o / 49 - 3;
         realIrregular<double>(lim, double(ox), double(oy), double(oz), Hs);
      }
   }
   __syncthreads();
   double* out = kind == 0 ? m2m + int64_t(op) * L * L : kind == 1 ? l2l + int64_t(op - 8) * L * L
                                                                   : m2l + int64_t(op - 16) * L * L;
   for(int e = threadIdx.x; e < L * L; e += blockDim.x)
   {
      int i = e / L, j = e % L;
      double v = operatorEntry(kind, i, j, Hs, lim);
      int li = int(sqrt(double(i))); while(li * li > i) li--; while((li + 1) * (li + 1) <= i) li++;
      int lj = int(sqrt(double(j))); while(lj * lj > j) lj--; while((lj + 1) * (lj + 1) <= j) lj++;
      if(kind == 0) v = ldexp(v, -lj);        // scaled M2M: columns times 2^-lambda
      else if(kind == 1) v = ldexp(v, -(li + 1));  // scaled L2L: rows times 2^-(l+1)
      out[e] = v;
   }
}

// Working copies: transposed [op][j (input)][k (output, padded to Lp)] in T.
template <class T>
__global__ void kTransposeOps(const double* __restrict__ src, int nops, int L, int Lp, T* dst)
{
   int64_t total = int64_t(nops) * L * Lp;
   for(int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
   {
      int k = int(e % Lp);
      int64_t r = e / Lp;
      int j = int(r % L);
      int op = int(r / L);
      dst[e] = k < L ? T(src[(int64_t(op) * L + k) * L + j]) : T(0);
   }
}

// The gradient coefficients of kL2PNear's gradCoeff as terms: its value is sum_i c[i] Lv[idx[i]]
// (the same case analysis, for tables).
struct GradTerms
{
   int n;
   int idx[2];
   double c[2];
};
inline GradTerms gradTerms(int j, int lp, int mu)
{
   const int l = lp + 1;
   const double h = 0.5, r2 = 0.70710678118654752440;
   GradTerms g{0, {0, 0}, {0.0, 0.0}};
   auto add = [&](double c, int m) {
      if(std::abs(m) <= l) { g.idx[g.n] = hidx(l, m); g.c[g.n] = c; g.n++; }
   };
   if(j == 2) add(-1.0, mu);
   else if(j == 0)
   {
      if(mu == 0) add(-r2, 1);
      else if(mu == 1) { add(-h, 2); add(r2, 0); }
      else if(mu >= 2) { add(-h, mu + 1); add(h, mu - 1); }
      else if(mu == -1) add(-h, -2);
      else { add(-h, mu - 1); add(h, mu + 1); }
   }
   else
   {
      if(mu == 0) add(-r2, -1);
      else if(mu == 1) add(-h, -2);
      else if(mu >= 2) { add(-h, -(mu + 1)); add(-h, -(mu - 1)); }
      else if(mu == -1) { add(h, 2); add(r2, 0); }
      else { add(h, 1 - mu); add(h, -mu - 1); }
   }
   return g;
}
// One entry of the L2P curl table: curl-expansion coefficient k' (degree <= p - 1), component c,
// with the real-basis factor (-1)^l' (sqrt2 for m != 0) folded in, as <= 4 terms of the local
// expansion row [3][Lp] of a box. Entries are [k'][4]; the fourth of each k' is empty.
template <class T>
struct CurlEntry
{
   int idx[4];
   T c[4];
};

fmm_status buildOperators(Plan& P, cudaStream_t st)
{
   if(P.opOrder == P.p) return FMM_OK;
   FMM_TRY(initOffsetTables());
   const int p = P.p, L = P.L, Lp = P.Lp;
   const int lim = P.cfg.m2l_truncate ? p : 2 * p;
   FMM_TRY(P.opM2M64.reserve(sizeof(double) * 8 * L * L));
   FMM_TRY(P.opL2L64.reserve(sizeof(double) * 8 * L * L));
   FMM_TRY(P.opM2L64.reserve(sizeof(double) * 316 * L * L));
   size_t shm = sizeof(double) * nharm(std::max(lim, p));
   kBuildOperators<<<16 + 316, 256, shm, st>>>(p, lim, 0, 16 + 316, (double*)P.opM2M64.ptr, (double*)P.opL2L64.ptr,
                                               (double*)P.opM2L64.ptr);
   FMM_TRY(launched(P, "kBuildOperators", st));
   FMM_CHECK_LAUNCH();
   size_t es = P.fp64 ? sizeof(double) : sizeof(float);
   FMM_TRY(P.opM2Mw.reserve(es * 8 * L * Lp));
   FMM_TRY(P.opL2Lw.reserve(es * 8 * L * Lp));
   FMM_TRY(P.opM2Lw.reserve(es * 316 * L * Lp));
   if(P.fp64)
   {
      kTransposeOps<double><<<1024, 256, 0, st>>>((const double*)P.opM2M64.ptr, 8, L, Lp, (double*)P.opM2Mw.ptr);
      FMM_TRY(launched(P, "kTransposeOps", st));
      kTransposeOps<double><<<1024, 256, 0, st>>>((const double*)P.opL2L64.ptr, 8, L, Lp, (double*)P.opL2Lw.ptr);
      FMM_TRY(launched(P, "kTransposeOps", st));
      kTransposeOps<double><<<4096, 256, 0, st>>>((const double*)P.opM2L64.ptr, 316, L, Lp, (double*)P.opM2Lw.ptr);
      FMM_TRY(launched(P, "kTransposeOps", st));
   }
   else
   {
      kTransposeOps<float><<<1024, 256, 0, st>>>((const double*)P.opM2M64.ptr, 8, L, Lp, (float*)P.opM2Mw.ptr);
      FMM_TRY(launched(P, "kTransposeOps", st));
      kTransposeOps<float><<<1024, 256, 0, st>>>((const double*)P.opL2L64.ptr, 8, L, Lp, (float*)P.opL2Lw.ptr);
      FMM_TRY(launched(P, "kTransposeOps", st));
      kTransposeOps<float><<<4096, 256, 0, st>>>((const double*)P.opM2L64.ptr, 316, L, Lp, (float*)P.opM2Lw.ptr);
      FMM_TRY(launched(P, "kTransposeOps", st));
   }
   FMM_CHECK_LAUNCH();
   // the L2P curl table in the plan's precision
   {
      const int Lb = nharm(p - 1);
      const size_t esz = P.fp64 ? sizeof(CurlEntry<double>) : sizeof(CurlEntry<float>);
      P.curlHost.assign(esz * 4 * Lb, 0);
      for(int k = 0; k < Lb; k++)
      {
         int lp = 0;
         while((lp + 1) * (lp + 1) <= k) lp++;
         const int mu = k - lp * lp - lp;
         const double f = ((lp & 1) ? -1.0 : 1.0) * (mu != 0 ? 1.4142135623730950488 : 1.0);
         for(int c = 0; c < 3; c++)
         {
            // B_x = dAz/dy - dAy/dz, B_y = dAx/dz - dAz/dx, B_z = dAy/dx - dAx/dy
            const int cp = (c + 2) % 3, cm = (c + 1) % 3, jp = (c + 1) % 3, jm = (c + 2) % 3;
            const GradTerms gp = gradTerms(jp, lp, mu), gm = gradTerms(jm, lp, mu);
            int idx[4] = {0, 0, 0, 0};
            double cf[4] = {0, 0, 0, 0};
            int n = 0;
            for(int i = 0; i < gp.n; i++) { idx[n] = cp * Lp + gp.idx[i]; cf[n] = f * gp.c[i]; n++; }
            for(int i = 0; i < gm.n; i++) { idx[n] = cm * Lp + gm.idx[i]; cf[n] = -f * gm.c[i]; n++; }
            unsigned char* dst = P.curlHost.data() + esz * (4 * k + c);
            if(P.fp64)
            {
               CurlEntry<double> e;
               for(int i = 0; i < 4; i++) { e.idx[i] = idx[i]; e.c[i] = cf[i]; }
               memcpy(dst, &e, sizeof(e));
            }
            else
            {
               CurlEntry<float> e;
               for(int i = 0; i < 4; i++) { e.idx[i] = idx[i]; e.c[i] = float(cf[i]); }
               memcpy(dst, &e, sizeof(e));
            }
         }
      }
      FMM_TRY(P.curlTab.reserve(P.curlHost.size()));
      FMM_CUDA(cudaMemcpyAsync(P.curlTab.ptr, P.curlHost.data(), P.curlHost.size(), cudaMemcpyHostToDevice, st));
   }
   P.opOrder = p;
   P.opImgOrder = -1;
   return FMM_OK;
}

// ====================================================================================
// M2M and L2L as tiled GEMMs over the parents of one level. A block takes 32 parents (96 rows:
// parent x component) and 64 output coefficients; for each child octant o it streams the rows
// (children's multipoles, or the parents' locals) and the operator T_o through shared memory in
// K slices of 32, 6 x 4 outputs per thread. Operator elements are loaded once per tile instead of
// once per parent. K is limited to the triangle each translation needs: an output of degree l
// takes inputs of degree <= l (M2M) or >= l (L2L).
//   M2M: parent = sum_o T_o child_o          (one writer per parent: stored)
//   L2L: child_o += T_o parent               (one writer per child: load-add-store)
// ====================================================================================
constexpr int TG_P = 32, TG_ROWS = 96, TG_N = 64, TG_K = 32;

__device__ __forceinline__ void load4(const float* p, float* v)
{
   const float4 x = *reinterpret_cast<const float4*>(p);
   v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void load4(const double* p, double* v)
{
   const double2 x = reinterpret_cast<const double2*>(p)[0], y = reinterpret_cast<const double2*>(p)[1];
   v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
__device__ __forceinline__ void load2(const float* p, float* v)
{
   const float2 x = *reinterpret_cast<const float2*>(p);
   v[0] = x.x; v[1] = x.y;
}
__device__ __forceinline__ void load2(const double* p, double* v)
{
   const double2 x = *reinterpret_cast<const double2*>(p);
   v[0] = x.x; v[1] = x.y;
}

__device__ __forceinline__ int degreeOf(int k)
{
   int l = int(sqrtf(float(k)));
   while(l * l > k) l--;
   while((l + 1) * (l + 1) <= k) l++;
   return l;
}

template <class T, bool UP>
__global__ void __launch_bounds__(256, 2) kTranslateLevel(Tree t, const int* __restrict__ parList, int pBeg, int pEnd,
                                                          int p, int Lp, const T* __restrict__ opw, T* __restrict__ X)
{
   __shared__ __align__(16) T As[TG_K][TG_ROWS + 1];
   __shared__ __align__(16) T Bs[TG_K][TG_N];
   __shared__ int childOf[TG_P][8];
   __shared__ int parentOf[TG_P];
   const int tid = threadIdx.x;
   const int L = nharm(p);
   const int pt0 = pBeg + blockIdx.x * TG_P;
   const int n0 = blockIdx.y * TG_N;
   if(tid < TG_P)
   {
      const int par = pt0 + tid < pEnd ? parList[pt0 + tid] : -1;
      parentOf[tid] = par;
      for(int o = 0; o < 8; o++) childOf[tid][o] = -1;
      if(par >= 0)
      {
         const int c0 = t.child0[par], nc = t.nchild[par];
         for(int c = 0; c < nc; c++)
         {
            const int ch = c0 + c;
            // M2M needs children with sources, L2L children with targets
            const bool use = UP ? t.s1[ch] > t.s0[ch] : t.t1[ch] > t.t0[ch];
            if(use) childOf[tid][int(t.key[ch] & 7)] = ch;
         }
      }
   }
   __syncthreads();
   const int lLo = degreeOf(min(n0, L - 1)), lHi = degreeOf(min(n0 + TG_N - 1, L - 1));
   const int kLo = UP ? 0 : lLo * lLo;
   const int kHi = UP ? (lHi + 1) * (lHi + 1) : L;
   const int tr = tid >> 4, tc = tid & 15;
   T acc[6][4];
#pragma unroll
   for(int i = 0; i < 6; i++)
#pragma unroll
      for(int j = 0; j < 4; j++) acc[i][j] = T(0);
   // steps (octant o, K slice) in order; each step's rows and operator slice are loaded into
   // registers one step ahead, so the global loads overlap the previous step's arithmetic.
   // Element q of a thread: row (tid / 32) + 8 q at K offset tid % 32 (k fastest across a warp:
   // coalesced row reads), and operator row (tid / 64) + 4 q at column tid % 64.
   const int nK = (kHi - kLo + TG_K - 1) / TG_K;
   const int nSteps = 8 * nK;
   constexpr int QA = TG_K * TG_ROWS / 256, QB = TG_K * TG_N / 256;
   T ra[QA], rb[QB];
   const int aK = tid & 31, aR = tid >> 5;
   const int bN = tid & 63, bK = tid >> 6;
   auto load = [&](int step) {
      const int o = step / nK, k0 = kLo + (step % nK) * TG_K;
      const T* op = opw + int64_t(o) * L * Lp + n0 + bN;
      const bool aIn = k0 + aK < kHi;
#pragma unroll
      for(int q = 0; q < QA; q++)
      {
         const int r = aR + 8 * q;
         const int i = r / 3, c = r - 3 * i;
         const int src = UP ? childOf[i][o] : parentOf[i];
         ra[q] = (src >= 0 && aIn) ? X[(int64_t(src) * 3 + c) * Lp + k0 + aK] : T(0);
      }
      const bool bIn = n0 + bN < Lp;
#pragma unroll
      for(int q = 0; q < QB; q++)
      {
         const int k = k0 + bK + 4 * q;
         rb[q] = (k < kHi && bIn) ? op[int64_t(k) * Lp] : T(0);
      }
   };
   if(nSteps > 0) load(0);
   for(int step = 0; step < nSteps; step++)
   {
      __syncthreads();
#pragma unroll
      for(int q = 0; q < QA; q++) As[aK][aR + 8 * q] = ra[q];
#pragma unroll
      for(int q = 0; q < QB; q++) Bs[bK + 4 * q][bN] = rb[q];
      __syncthreads();
      if(step + 1 < nSteps) load(step + 1);
#pragma unroll 8
      for(int kk = 0; kk < TG_K; kk++)
      {
         T a[6], b[4];
#pragma unroll
         for(int i = 0; i < 6; i++) a[i] = As[kk][tr * 6 + i];
         load4(&Bs[kk][tc * 4], b);
#pragma unroll
         for(int i = 0; i < 6; i++)
#pragma unroll
            for(int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
      }
      if(!UP && step % nK == nK - 1)
      {
         // this octant's children: child += acc, then a fresh accumulator for the next octant
         const int o = step / nK;
#pragma unroll
         for(int i = 0; i < 6; i++)
         {
            const int r = tr * 6 + i, pi = r / 3, c = r % 3;
            const int ch = childOf[pi][o];
            if(ch >= 0)
               for(int j = 0; j < 4; j++)
               {
                  const int n = n0 + tc * 4 + j;
                  if(n < Lp) X[(int64_t(ch) * 3 + c) * Lp + n] += acc[i][j];
               }
#pragma unroll
            for(int j = 0; j < 4; j++) acc[i][j] = T(0);
         }
      }
   }
   if(UP)
   {
#pragma unroll
      for(int i = 0; i < 6; i++)
      {
         const int r = tr * 6 + i, pi = r / 3, c = r % 3;
         const int par = parentOf[pi];
         if(par < 0 || t.s1[par] == t.s0[par]) continue;
         for(int j = 0; j < 4; j++)
         {
            const int n = n0 + tc * 4 + j;
            if(n < Lp) X[(int64_t(par) * 3 + c) * Lp + n] = acc[i][j];
         }
      }
   }
}

// ====================================================================================
// Geometry helpers
// ====================================================================================
__device__ __forceinline__ void nodeCenter(const RootBox& rb, int level, int ix, int iy, int iz, double c[3], double& h)
{
   h = 2.0 * rb.H / double(int64_t(1) << level);
   c[0] = rb.center[0] - rb.H + (double(ix) + 0.5) * h;
   c[1] = rb.center[1] - rb.H + (double(iy) + 0.5) * h;
   c[2] = rb.center[2] - rb.H + (double(iz) + 0.5) * h;
}

// ====================================================================================
// P2M: one block of NT threads per leaf holding sources, one source point per thread. Each
// thread runs the harmonic recurrence of its point as explicit state in registers (RegularIter,
// the visit order of visitRegular). Every CV visits the block reduces the values of those
// visits over its points through a small shared tile (the values of a visit are the same
// coefficient for every thread, so the tile's columns are coefficients) and adds them to the
// leaf's multipole, kept in shared memory until the end. Leaves with more than NT points take
// their points NT at a time.
// ====================================================================================
template <class T>
struct RegularIter
{
   T x, y, z, r2;
   T dre, dim;       // S_m^m
   T are, aim;       // S_l^m (the current visit)
   T bre, bim;       // S_{l-1}^m
   int l, m, p;
   __device__ __forceinline__ void start(int p_, T x_, T y_, T z_)
   {
      p = p_; x = x_; y = y_; z = z_; r2 = x * x + y * y + z * z;
      dre = T(1); dim = T(0); are = T(1); aim = T(0); bre = T(0); bim = T(0); l = 0; m = 0;
   }
   // moves to the next (l, m) of the visit order: l = m..p for m = 0..p
   __device__ __forceinline__ void next()
   {
      if(l < p)
      {
         T cre, cim;
         if(l == m) { cre = z * are; cim = z * aim; }
         else
         {
            const T inv = T(1) / T((l - m + 1) * (l + m + 1));
            const T a = T(2 * l + 1) * inv;
            cre = a * z * are - inv * r2 * bre;
            cim = a * z * aim - inv * r2 * bim;
         }
         bre = are; bim = aim; are = cre; aim = cim;
         l++;
      }
      else
      {
         m++;
         const T s = T(1) / T(2 * m);
         const T nre = (dre * x - dim * y) * s;
         const T nim = (dre * y + dim * x) * s;
         dre = nre; dim = nim;
         are = dre; aim = dim; bre = T(0); bim = T(0);
         l = m;
      }
   }
};

template <class T, int NT, int CV>
__global__ void __launch_bounds__(NT) kP2M(Tree t, const RootBox* __restrict__ rootp,
                                           const typename Vec4<T>::type* __restrict__ pos,
                                           const typename Vec4<T>::type* __restrict__ q, int p, int Lp, T* __restrict__ M)
{
   __shared__ T R[NT][2 * CV + 1];   // the chunk's real-basis values per point (odd stride)
   __shared__ T Q[NT][3];            // w J per point
   __shared__ int kOf[2 * CV];       // coefficient index of each column of R (-1: none)
   extern __shared__ unsigned char smraw[];
   T* Macc = (T*)smraw;              // [3][Lp] the leaf's multipole
   const int node = blockIdx.x;
   if(t.nchild[node] != 0) return;
   const int s0 = t.s0[node], s1 = t.s1[node];
   if(s1 == s0) return;
   const int tid = threadIdx.x;
   const int L = nharm(p);
   const int nVisits = (p + 1) * (p + 2) / 2;
   for(int e = tid; e < 3 * Lp; e += NT) Macc[e] = T(0);
   const RootBox rb = rootp[rootOf(t, node)];
   double c[3], h;
   nodeCenter(rb, t.level[node], t.ix[node], t.iy[node], t.iz[node], c, h);
   const double ih = 1.0 / h;
   const T sq2 = T(1.4142135623730950488);
   for(int base = s0; base < s1; base += NT)
   {
      const int cnt = min(NT, s1 - base);
      RegularIter<T> it;
      T qx = T(0), qy = T(0), qz = T(0);
      if(tid < cnt)
      {
         const auto xp = pos[base + tid];
         const auto w = q[base + tid];
         it.start(p, T((double(xp.x) - c[0]) * ih), T((double(xp.y) - c[1]) * ih), T((double(xp.z) - c[2]) * ih));
         qx = w.x; qy = w.y; qz = w.z;
      }
      else
         it.start(p, T(0), T(0), T(0));
      Q[tid][0] = qx; Q[tid][1] = qy; Q[tid][2] = qz;
      int vl = 0, vm = 0;   // (l, m) of the chunk's first visit, tracked uniformly by every thread
      for(int v0 = 0; v0 < nVisits; v0 += CV)
      {
         const int nv = min(CV, nVisits - v0);
         // this thread's values for visits v0 .. v0 + nv - 1, and the columns' coefficients
         int cl = vl, cm = vm;
         for(int j = 0; j < nv; j++)
         {
            const T sgn = (it.l & 1) ? T(-1) : T(1);
            if(it.m == 0) { R[tid][2 * j] = sgn * it.are; R[tid][2 * j + 1] = T(0); }
            else { R[tid][2 * j] = sgn * sq2 * it.are; R[tid][2 * j + 1] = sgn * sq2 * it.aim; }
            if(tid == 0)
            {
               kOf[2 * j] = hidx(cl, cm);
               kOf[2 * j + 1] = cm > 0 ? hidx(cl, -cm) : -1;
            }
            if(v0 + j + 1 < nVisits) it.next();
            if(cl < p) cl++;
            else { cm++; cl = cm; }
         }
         vl = cl; vm = cm;
         __syncthreads();
         // reduce over the points: output (column, component) pairs split over the threads
         for(int o = tid; o < 2 * nv * 3; o += NT)
         {
            const int col = o / 3, comp = o - 3 * col;
            const int k = kOf[col];
            if(k < 0) continue;
            T acc = T(0);
            for(int i = 0; i < cnt; i++) acc += Q[i][comp] * R[i][col];
            Macc[comp * Lp + k] += acc;
         }
         __syncthreads();
      }
   }
   T* out = M + int64_t(node) * 3 * Lp;
   for(int e = tid; e < 3 * Lp; e += NT) out[e] = (e % Lp) < L ? Macc[e] : T(0);
}

// ====================================================================================
// P2M, one warp per leaf. Lane (u, c), u < U = p / 2 + 1, c < 3, owns component c of the
// complex coefficients S_l^m of the two orders m_a = u and m_b = p - u (p + 2 values; p / 2 + 1
// when m_a = m_b), so the U units cover every order once and the 3 U <= 27 lanes have equal
// work. The leaf's points go 32 at a time: lane j scales point j to the box and writes its
// diagonal values S_m^m (m = 0..p, the recurrence's first step) to shared memory; then every lane
// walks the points in order, running the l-recurrence of m_a and then of m_b and adding
// q_c S_l^m into registers. Step j of a lane uses the coefficients (a, b, e) of its table row:
//   S_j = a z S_{j-1} - b r^2 S_{j-2} + e S_{m_b}^{m_b}
// with e = 1, a = b = 0 at the step that starts the m_b chain and b = 0 at the first step of
// each chain, so no lane branches. At the end the real coefficients (-1)^l sqrt2 (Re, Im) S_l^m
// (m > 0) and (-1)^l S_l^0 go through shared memory to one coalesced store of the leaf's
// multipole.
// ====================================================================================
constexpr int P2MW_WARPS = 4;
constexpr int P2MW_STEPS = MAXORDER + 2;

template <class T>
inline size_t p2mWarpSmem(int p, int Lp)
{
   const size_t perWarp = 32 * 8 + std::max<size_t>(size_t(32) * 2 * (p + 1), size_t(3) * Lp);
   return sizeof(T) * (size_t(P2MW_STEPS) * 32 * 4 + P2MW_WARPS * perWarp);
}

template <class T>
__global__ void __launch_bounds__(32 * P2MW_WARPS) kP2MWarp(Tree t, const RootBox* __restrict__ rootp,
                                                          const typename Vec4<T>::type* __restrict__ pos,
                                                          const typename Vec4<T>::type* __restrict__ q, int p,
                                                          int Lp, T* __restrict__ M, uint8_t* __restrict__ Mpieces,
                                                          int np)
{
   typedef typename Vec4<T>::type V4;
   extern __shared__ __align__(16) unsigned char smraw[];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int U = p / 2 + 1;
   // the step table, [step][lane] (a, b, e, 0)
   V4* AB = (V4*)smraw;
   const size_t perWarp = 32 * 8 + max(32 * 2 * (p + 1), 3 * Lp);
   T* Pt = (T*)(AB + P2MW_STEPS * 32) + warp * perWarp;   // [32][8] point: u, r^2, q
   T* Ds = Pt + 32 * 8;                                  // [32][p + 1] (re, im) of S_m^m; later [3][Lp]
   const int u = lane % U, c = min(lane / U, 2);
   const int ma = u, mb = p - u;
   const int na = p + 1 - ma;                            // terms of the m_a chain
   for(int e = threadIdx.x; e < P2MW_STEPS * 32; e += 32 * P2MW_WARPS)
   {
      const int j = e / 32, ln = e % 32;
      const int uu = ln % U;
      const int a0 = uu, b0 = p - uu, n0 = p + 1 - a0;
      const int n = n0 + (b0 != a0 ? p + 1 - b0 : 0);
      T a = T(0), b = T(0), ee = T(0);
      if(j == n0 && j < n) ee = T(1);
      else if(j > 0 && j < n)
      {
         const int m = j < n0 ? a0 : b0;
         const int l = j < n0 ? a0 + j - 1 : b0 + (j - n0) - 1;
         const T inv = T(1) / T((l - m + 1) * (l + m + 1));
         a = T(2 * l + 1) * inv;
         b = l == m ? T(0) : inv;
      }
      AB[e] = V4{a, b, ee, T(0)};
   }
   __syncthreads();
   const int node = blockIdx.x * P2MW_WARPS + warp;
   if(node >= t.nNodes || t.nchild[node] != 0) return;
   const int s0 = t.s0[node], s1 = t.s1[node];
   if(s1 == s0) return;
   const RootBox rb = rootp[rootOf(t, node)];
   double cen[3], h;
   nodeCenter(rb, t.level[node], t.ix[node], t.iy[node], t.iz[node], cen, h);
   const double ih = 1.0 / h;
   T accR[P2MW_STEPS], accI[P2MW_STEPS];
#pragma unroll
   for(int j = 0; j < P2MW_STEPS; j++) { accR[j] = T(0); accI[j] = T(0); }
   for(int base = s0; base < s1; base += 32)
   {
      const int cnt = min(32, s1 - base);
      if(lane < cnt)
      {
         const V4 xp = pos[base + lane], w = q[base + lane];
         const T x = T((double(xp.x) - cen[0]) * ih), y = T((double(xp.y) - cen[1]) * ih),
                 z = T((double(xp.z) - cen[2]) * ih);
         T* pt = Pt + lane * 8;
         pt[0] = x; pt[1] = y; pt[2] = z; pt[3] = x * x + y * y + z * z;
         pt[4] = w.x; pt[5] = w.y; pt[6] = w.z;
         T dre = T(1), dim = T(0);
         T* d = Ds + lane * 2 * (p + 1);
         d[0] = dre; d[1] = dim;
         for(int m = 1; m <= p; m++)
         {
            const T sc = T(1) / T(2 * m);
            const T nre = (dre * x - dim * y) * sc;
            const T nim = (dre * y + dim * x) * sc;
            dre = nre; dim = nim;
            d[2 * m] = dre; d[2 * m + 1] = dim;
         }
      }
      __syncwarp();
      // two points per pass (independent recurrences sharing the table loads); an odd count's
      // partner is a zero-strength point at the box centre
      for(int i = 0; i < cnt; i += 2)
      {
         const bool two = i + 1 < cnt;
         const T* pt = Pt + i * 8;
         const T* d = Ds + i * 2 * (p + 1);
         const T z = pt[2], r2 = pt[3], qc = pt[4 + c];
         const T z2 = two ? pt[8 + 2] : T(0), r22 = two ? pt[8 + 3] : T(0), qc2 = two ? pt[8 + 4 + c] : T(0);
         const T* d2 = d + 2 * (p + 1);
         T are = d[2 * ma], aim = d[2 * ma + 1];
         const T bdr = d[2 * mb], bdi = d[2 * mb + 1];
         T are2 = two ? d2[2 * ma] : T(0), aim2 = two ? d2[2 * ma + 1] : T(0);
         const T bdr2 = two ? d2[2 * mb] : T(0), bdi2 = two ? d2[2 * mb + 1] : T(0);
         T bre = T(0), bim = T(0), bre2 = T(0), bim2 = T(0);
         accR[0] += qc * are + qc2 * are2;
         accI[0] += qc * aim + qc2 * aim2;
#pragma unroll
         for(int j = 1; j < P2MW_STEPS; j++)
         {
            if(j > p + 1) break;
            const V4 k = AB[j * 32 + lane];
            const T az = k.x * z, br = k.y * r2;
            const T az2 = k.x * z2, br2 = k.y * r22;
            const T cre = k.z * bdr + (az * are - br * bre);
            const T cim = k.z * bdi + (az * aim - br * bim);
            const T cre2 = k.z * bdr2 + (az2 * are2 - br2 * bre2);
            const T cim2 = k.z * bdi2 + (az2 * aim2 - br2 * bim2);
            bre = are; bim = aim; are = cre; aim = cim;
            bre2 = are2; bim2 = aim2; are2 = cre2; aim2 = cim2;
            accR[j] += qc * are + qc2 * are2;
            accI[j] += qc * aim + qc2 * aim2;
         }
      }
      __syncwarp();
   }
   // real coefficients through shared memory, then one coalesced store
   T* Mst = Ds;
   for(int e = lane; e < 3 * Lp; e += 32)
      if(e % Lp >= (p + 1) * (p + 1)) Mst[e] = T(0);
   if(lane < 3 * U)
   {
      const int nb = mb != ma ? p + 1 - mb : 0;
      const T sq2 = T(1.4142135623730950488);
#pragma unroll
      for(int j = 0; j < P2MW_STEPS; j++)
      {
         if(j >= na + nb) break;
         const int m = j < na ? ma : mb;
         const int l = j < na ? ma + j : mb + (j - na);
         const T sg = (l & 1) ? T(-1) : T(1);
         T* mc = Mst + c * Lp;
         if(m == 0) mc[hidx(l, 0)] = sg * accR[j];
         else
         {
            mc[hidx(l, m)] = sg * sq2 * accR[j];
            mc[hidx(l, -m)] = sg * sq2 * accI[j];
         }
      }
   }
   __syncwarp();
   T* out = M + int64_t(node) * 3 * Lp;
   for(int e = lane; e < 3 * Lp; e += 32) out[e] = Mst[e];
   // the same coefficients as tensor-core operand pieces (the M2M's and M2L's input format), so the
   // upward pass needs no separate split of the leaves
   if constexpr(sizeof(T) == 4)
      if(Mpieces)
         for(int e4 = lane; e4 < 3 * Lp / 4; e4 += 32)
         {
            const int e = 4 * e4;
            const float4 v = make_float4(Mst[e], Mst[e + 1], Mst[e + 2], Mst[e + 3]);
            storePieces4(Mpieces, int64_t(node) * 3 + e / Lp, e % Lp, Lp, np, v);
         }
}

// ====================================================================================
// M2M, one level: one block per node of the level with children; the parent sums the
// translated multipoles of its children. Output coefficient k of degree l only needs input
// coefficients j < (l+1)^2.
// ====================================================================================

// ====================================================================================
// L2L, one level: one block per node of the level holding targets; adds the parent's
// translated local expansion. Output coefficient of degree l needs inputs of degree >= l.
// ====================================================================================

// ====================================================================================
// L2L, one level, child-major: the level's children with targets come sorted by octant, and a
// block takes 32 children of one octant (blockIdx.z), so every row of its tile uses the same
// operator T_o and none is computed for a child that does not exist. Rows are the parents' locals
// (parent x component), gathered; the K range per 64-column group is the L2L triangle (inputs of
// degree >= the output's); the result is added to the children's locals (one writer per child).
// ====================================================================================
struct L2LSeg
{
   int start[9];   // the octants' ranges in the sorted child list
};

template <class T>
__global__ void __launch_bounds__(256, 2) kL2LChild(Tree t, const int* __restrict__ list, L2LSeg seg, int p, int Lp,
                                                    const T* __restrict__ opw, T* __restrict__ X)
{
   const int o = blockIdx.z;
   const int s0 = seg.start[o] + blockIdx.x * TG_P, s1 = seg.start[o + 1];
   if(s0 >= s1) return;
   // rows padded by two: the transposed stores meet two-way bank conflicts, and each thread reads its
   // six rows as three aligned pairs
   __shared__ __align__(16) T As[TG_K][TG_ROWS + 2];
   __shared__ __align__(16) T Bs[TG_K][TG_N];
   __shared__ int childOf[TG_P], parentOf[TG_P];
   const int tid = threadIdx.x;
   const int L = nharm(p);
   const int n0 = blockIdx.y * TG_N;
   if(tid < TG_P)
   {
      const int ch = s0 + tid < s1 ? list[s0 + tid] : -1;
      childOf[tid] = ch;
      parentOf[tid] = ch >= 0 ? t.parent[ch] : -1;
   }
   __syncthreads();
   const int lLo = degreeOf(min(n0, L - 1));
   const int kLo = lLo * lLo, kHi = L;
   const int tr = tid >> 4, tc = tid & 15;
   T acc[6][4];
#pragma unroll
   for(int i = 0; i < 6; i++)
#pragma unroll
      for(int j = 0; j < 4; j++) acc[i][j] = T(0);
   const int nK = (kHi - kLo + TG_K - 1) / TG_K;
   constexpr int QA = TG_K * TG_ROWS / 256, QB = TG_K * TG_N / 256;
   T ra[QA], rb[QB];
   const int aK = tid & 31, aR = tid >> 5;
   const int bN = tid & 63, bK = tid >> 6;
   const T* op = opw + int64_t(o) * L * Lp + n0 + bN;
   const bool bIn = n0 + bN < Lp;
   auto load = [&](int step) {
      const int k0 = kLo + step * TG_K;
      const bool aIn = k0 + aK < kHi;
#pragma unroll
      for(int q = 0; q < QA; q++)
      {
         const int r = aR + 8 * q;
         const int i = r / 3, c = r - 3 * i;
         const int src = parentOf[i];
         ra[q] = (src >= 0 && aIn) ? X[(int64_t(src) * 3 + c) * Lp + k0 + aK] : T(0);
      }
#pragma unroll
      for(int q = 0; q < QB; q++)
      {
         const int k = k0 + bK + 4 * q;
         rb[q] = (k < kHi && bIn) ? op[int64_t(k) * Lp] : T(0);
      }
   };
   if(nK > 0) load(0);
   for(int step = 0; step < nK; step++)
   {
      __syncthreads();
#pragma unroll
      for(int q = 0; q < QA; q++) As[aK][aR + 8 * q] = ra[q];
#pragma unroll
      for(int q = 0; q < QB; q++) Bs[bK + 4 * q][bN] = rb[q];
      __syncthreads();
      if(step + 1 < nK) load(step + 1);
#pragma unroll 8
      for(int kk = 0; kk < TG_K; kk++)
      {
         T a[6], b[4];
#pragma unroll
         for(int i = 0; i < 6; i += 2) load2(&As[kk][tr * 6 + i], a + i);
         load4(&Bs[kk][tc * 4], b);
#pragma unroll
         for(int i = 0; i < 6; i++)
#pragma unroll
            for(int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
      }
   }
#pragma unroll
   for(int i = 0; i < 6; i++)
   {
      const int r = tr * 6 + i, ci = r / 3, c = r % 3;
      const int ch = childOf[ci];
      if(ch < 0) continue;
      for(int j = 0; j < 4; j++)
      {
         const int n = n0 + tc * 4 + j;
         if(n < Lp) X[(int64_t(ch) * 3 + c) * Lp + n] += acc[i][j];
      }
   }
}

// ====================================================================================
// M2L on the CUDA cores (FP32 or FP64 FMA). A block owns TT target boxes from the octant-grouped
// list of boxes with an M2L list (3 TT rows: box x component) and all output coefficients; it
// walks only the offsets present in its tile and, per offset, the K chunks of the operator. The
// gathered source rows and the operator slice of an item are brought to shared memory with
// cp.async, double-buffered so that the next item's copies run under this item's arithmetic.
// Warp w owns rows RPT w .. RPT w + RPT - 1 (its A reads are broadcasts), lane c the columns
// c + 32 n. With the degree cutoff l + lambda <= P, a K chunk whose lowest input degree is
// lambda_min only reaches the first (P - lambda_min + 1)^2 columns; the rest are skipped.
// ====================================================================================
constexpr int SM_NC = 10;              // 10 x 32 = 320 >= Lp for p <= 16

template <class T> struct SimtShape;
template <> struct SimtShape<float> { static constexpr int RPT = 12, KC = 32; };
template <> struct SimtShape<double> { static constexpr int RPT = 6, KC = 16; };

struct SimtCols
{
   int n[32];   // output columns of each K chunk (0: chunk unused)
};

__device__ __forceinline__ void cpAsync16Simt(void* dst, const void* src, uint32_t srcBytes)
{
   const uint32_t d = uint32_t(__cvta_generic_to_shared(dst));
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(srcBytes) : "memory");
}

template <class T>
__global__ void __launch_bounds__(256) kM2LSimt(const int* __restrict__ targets, int nTargets,
                                                const int* __restrict__ vtab, int p, int Lp, int nChunks,
                                                const SimtCols cols, const T* __restrict__ opw,
                                                const T* __restrict__ M, T* __restrict__ Lc)
{
   constexpr int RPT = SimtShape<T>::RPT, KC = SimtShape<T>::KC;
   constexpr int ROWS = 8 * RPT, TT = ROWS / 3;
   constexpr int NCOL = 32 * SM_NC;
   extern __shared__ __align__(16) unsigned char smraw[];
   T* As = (T*)smraw;                       // [2][ROWS][KC]
   T* Bs = As + 2 * ROWS * KC;              // [2][KC][NCOL]
   __shared__ int tileNode[TT];
   __shared__ uint32_t present[10];
   __shared__ int offs[316];
   __shared__ int nOffS;
   __shared__ int colTab[32];
   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   const int L = nharm(p);
   const int first = blockIdx.x * TT;
   if(tid < TT) tileNode[tid] = first + tid < nTargets ? targets[first + tid] : -1;
   if(tid < 10) present[tid] = 0;
   if(tid == 0)
   {
#pragma unroll
      for(int g = 0; g < 32; g++) colTab[g] = cols.n[g];
   }
   __syncthreads();
   for(int e = tid; e < TT * 316; e += 256)
   {
      const int t = tileNode[e / 316], o = e % 316;
      if(t >= 0 && vtab[int64_t(t) * 316 + o] >= 0) atomicOr(&present[o >> 5], 1u << (o & 31));
   }
   __syncthreads();
   if(tid == 0)
   {
      int k = 0;
      for(int o = 0; o < 316; o++)
         if(present[o >> 5] & (1u << (o & 31))) offs[k++] = o;
      nOffS = k;
   }
   __syncthreads();
   const int nItems = nOffS * nChunks;
   // copies of item it into buffer b: source rows (A) and operator rows k0 .. k0 + KC (B)
   auto issue = [&](int it, int b) {
      const int o = offs[it / nChunks], c = it % nChunks;
      const int k0 = c * KC;
      const int nCol = colTab[c];
      T* A = As + b * ROWS * KC;
      T* B = Bs + b * KC * NCOL;
      constexpr int ACH = KC * int(sizeof(T)) / 16;          // 16-byte chunks per row
      for(int e = tid; e < ROWS * ACH; e += 256)
      {
         const int r = e / ACH, q = e % ACH;
         const int t = tileNode[r / 3];
         const int src = t >= 0 ? vtab[int64_t(t) * 316 + o] : -1;
         // K positions past the row (k0 + KC can exceed Lp) are zero-filled, never read
         const int k = k0 + q * (16 / int(sizeof(T)));
         const bool in = src >= 0 && k < Lp;
         const T* g = M + (int64_t(in ? src : 0) * 3 + r % 3) * Lp + (in ? k : 0);
         cpAsync16Simt(A + r * KC + q * (16 / int(sizeof(T))), g, in ? 16u : 0u);
      }
      constexpr int BCH = NCOL * int(sizeof(T)) / 16;        // 16-byte chunks per operator row
      const T* op = opw + int64_t(o) * L * Lp;
      for(int e = tid; e < KC * BCH; e += 256)
      {
         const int kk = e / BCH, q = e % BCH;
         const int col = q * (16 / int(sizeof(T)));
         const int k = k0 + kk;
         const bool in = k < L && col < nCol;
         cpAsync16Simt(B + kk * NCOL + col, op + (in ? int64_t(k) * Lp + col : 0), in ? 16u : 0u);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
   };
   T acc[RPT][SM_NC];
#pragma unroll
   for(int r = 0; r < RPT; r++)
#pragma unroll
      for(int n = 0; n < SM_NC; n++) acc[r][n] = T(0);
   if(nItems > 0) issue(0, 0);
   for(int it = 0; it < nItems; it++)
   {
      const int b = it & 1;
      if(it + 1 < nItems)
      {
         issue(it + 1, b ^ 1);
         asm volatile("cp.async.wait_group 1;" ::: "memory");
      }
      else
         asm volatile("cp.async.wait_group 0;" ::: "memory");
      __syncthreads();
      const T* A = As + b * ROWS * KC + warp * RPT * KC;
      const T* B = Bs + b * KC * NCOL + lane;
      const int nCol = colTab[it % nChunks];
#pragma unroll 2
      for(int kk = 0; kk < KC; kk++)
      {
         T a[RPT], bv[SM_NC];
#pragma unroll
         for(int r = 0; r < RPT; r++) a[r] = A[r * KC + kk];
#pragma unroll
         for(int n = 0; n < SM_NC; n++) bv[n] = 32 * n < nCol ? B[kk * NCOL + 32 * n] : T(0);
#pragma unroll
         for(int r = 0; r < RPT; r++)
#pragma unroll
            for(int n = 0; n < SM_NC; n++)
               if(32 * n < nCol) acc[r][n] += a[r] * bv[n];
      }
      __syncthreads();
   }
#pragma unroll
   for(int r = 0; r < RPT; r++)
   {
      const int row = RPT * warp + r;
      const int node = tileNode[row / 3];
      if(node < 0) continue;
#pragma unroll
      for(int n = 0; n < SM_NC; n++)
      {
         const int col = lane + 32 * n;
         if(col < Lp) Lc[(int64_t(node) * 3 + row % 3) * Lp + col] = col < L ? acc[r][n] : T(0);
      }
   }
}

// ====================================================================================
// M2L on the CUDA cores in FP32, register-tiled (the plain FP32 form of FP32 plans). The same GEMM
// sum as kM2LTc: a tile of 42 target boxes = 126 rows (box, component) of a 128-row block, and for each
// offset present in the tile and each 16-wide K chunk C[128 x 160] += A_o[128 x 16] T_o[16 x 160], with
// C the block's 160 output columns (two column blocks cover the 304 of p = 16; the second skips the K
// chunks whose degree cutoff ends below its first column). Thread (ty, tx) of 256 owns rows 8 ty .. + 7
// and the column pairs 2 tx + 32 j (j < 5): per K element it reads its 8 rows as two 16-byte loads from a
// transposed copy of A and its 10 columns as five 8-byte loads, for 80 FMAs. A (gathered source rows)
// and the operator slice arrive by cp.async, double-buffered.
// ====================================================================================
constexpr int ST_TT = 42, ST_ROWS = 128, ST_CB = 160, ST_TPAD = ST_ROWS + 4;

template <int KC>
constexpr size_t simtTiledSmem()
{
   return sizeof(float) * (2 * ST_ROWS * KC + KC * ST_TPAD + 2 * KC * ST_CB);
}

template <int MINB, int ST_KC>
__global__ void __launch_bounds__(256, MINB) kM2LSimtTiled(const int* __restrict__ targets, int nTargets,
                                                        const int* __restrict__ vtab, int L, int Lp, int nChunks,
                                                        const SimtCols cols, const float* __restrict__ opw,
                                                        const float* __restrict__ M, float* __restrict__ Lc)
{
   extern __shared__ __align__(16) float smf[];
   // gathered rows, row-major (cp.async target) [2][ROWS][KC]; the current item's rows, K-major [KC][TPAD];
   // the operator slice [2][KC][CB]
   float (*As)[ST_ROWS][ST_KC] = reinterpret_cast<float (*)[ST_ROWS][ST_KC]>(smf);
   float (*At)[ST_TPAD] = reinterpret_cast<float (*)[ST_TPAD]>(smf + 2 * ST_ROWS * ST_KC);
   float (*Bs)[ST_KC][ST_CB] = reinterpret_cast<float (*)[ST_KC][ST_CB]>(smf + 2 * ST_ROWS * ST_KC + ST_KC * ST_TPAD);
   __shared__ int tileNode[ST_TT];
   __shared__ uint32_t present[10];
   __shared__ int offs[316];
   __shared__ int nOffS;
   __shared__ int chunkList[32], nChunkS;
   const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
   const int first = blockIdx.x * ST_TT;
   const int cb = blockIdx.y, col0 = cb * ST_CB;
   if(tid < ST_TT) tileNode[tid] = first + tid < nTargets ? targets[first + tid] : -1;
   if(tid < 10) present[tid] = 0;
   __syncthreads();
   for(int e = tid; e < ST_TT * 316; e += 256)
   {
      const int t = tileNode[e / 316], o = e % 316;
      if(t >= 0 && vtab[int64_t(t) * 316 + o] >= 0) atomicOr(&present[o >> 5], 1u << (o & 31));
   }
   __syncthreads();
   if(tid == 0)
   {
      int k = 0;
      for(int o = 0; o < 316; o++)
         if(present[o >> 5] & (1u << (o & 31))) offs[k++] = o;
      nOffS = k;
      // the K chunks that reach this column block (the degree cutoff narrows later chunks)
      int nc = 0;
      for(int c = 0; c < nChunks; c++)
         if(cols.n[c] > col0) chunkList[nc++] = c;
      nChunkS = nc;
   }
   __syncthreads();
   const int nCh = nChunkS, nOff = nOffS, nItems = nOff * nCh;
   // A: 128 rows x KC floats in 16-byte chunks; thread tid copies chunks (tid & 3) + 4 i of rows tid >> 2
   // and (tid >> 2) + 64 for every item, so it keeps those rows' source boxes for the current offset and
   // loads the next offset's one offset ahead (the V table read is off the copies' critical path)
   const int rA = tid >> 2, qA = tid & 3;
   int tA[2];
   for(int h = 0; h < 2; h++)
   {
      const int r = rA + 64 * h;
      tA[h] = r < 3 * ST_TT ? tileNode[r / 3] : -1;
   }
   int srcCur[2] = {-1, -1}, srcNxt[2] = {-1, -1};
   int oiCur = -1;
   auto loadSrc = [&](int oi, int* out) {
      const int o = offs[oi];
      for(int h = 0; h < 2; h++) out[h] = tA[h] >= 0 ? vtab[int64_t(tA[h]) * 316 + o] : -1;
   };
   auto issue = [&](int it, int b) {
      const int oi = it / nCh;
      const int o = offs[oi], c = chunkList[it - oi * nCh];
      const int k0 = c * ST_KC;
      if(oi != oiCur)
      {
         if(oi == oiCur + 1 && oiCur >= 0) { srcCur[0] = srcNxt[0]; srcCur[1] = srcNxt[1]; }
         else loadSrc(oi, srcCur);
         oiCur = oi;
         if(oi + 1 < nOff) loadSrc(oi + 1, srcNxt);
      }
      for(int h = 0; h < 2; h++)
#pragma unroll
         for(int i = 0; i < ST_KC / 16; i++)
         {
            const int r = rA + 64 * h, src = srcCur[h];
            const int q = qA + 4 * i, k = k0 + 4 * q;
            const bool in = src >= 0 && k < Lp;
            const float* g = M + (int64_t(in ? src : 0) * 3 + r % 3) * Lp + (in ? k : 0);
            cpAsync16Simt(&As[b][r][4 * q], g, in ? 16u : 0u);
         }
      // B: 16 K rows x 160 columns = 640 chunks
      const float* op = opw + int64_t(o) * L * Lp;
      const int nCol = cols.n[c];
      for(int e = tid; e < ST_KC * (ST_CB / 4); e += 256)
      {
         const int kk = e / (ST_CB / 4), q = e % (ST_CB / 4);
         const int col = col0 + 4 * q, k = k0 + kk;
         const bool in = k < L && col < nCol;
         cpAsync16Simt(&Bs[b][kk][4 * q], op + (in ? int64_t(k) * Lp + col : 0), in ? 16u : 0u);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
   };
   float acc[8][10];
#pragma unroll
   for(int r = 0; r < 8; r++)
#pragma unroll
      for(int n = 0; n < 10; n++) acc[r][n] = 0.f;
   if(nItems > 0) issue(0, 0);
   for(int it = 0; it < nItems; it++)
   {
      const int b = it & 1;
      if(it + 1 < nItems)
      {
         issue(it + 1, b ^ 1);
         asm volatile("cp.async.wait_group 1;" ::: "memory");
      }
      else
         asm volatile("cp.async.wait_group 0;" ::: "memory");
      __syncthreads();
      // transpose this item's rows into At[k][row]
#pragma unroll
      for(int q = 0; q < (ST_ROWS * ST_KC) / 256; q++)
      {
         const int e = tid + 256 * q;
         const int r = e / ST_KC, k = e % ST_KC;
         At[k][r] = As[b][r][k];
      }
      __syncthreads();
#pragma unroll 4
      for(int k = 0; k < ST_KC; k++)
      {
         const float4 a0 = *reinterpret_cast<const float4*>(&At[k][8 * ty]);
         const float4 a1 = *reinterpret_cast<const float4*>(&At[k][8 * ty + 4]);
         const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
         float bv[10];
#pragma unroll
         for(int j = 0; j < 5; j++)
         {
            const float2 v = *reinterpret_cast<const float2*>(&Bs[b][k][2 * tx + 32 * j]);
            bv[2 * j] = v.x;
            bv[2 * j + 1] = v.y;
         }
#pragma unroll
         for(int r = 0; r < 8; r++)
#pragma unroll
            for(int n = 0; n < 10; n++) acc[r][n] = fmaf(a[r], bv[n], acc[r][n]);
      }
      __syncthreads();
   }
#pragma unroll
   for(int r = 0; r < 8; r++)
   {
      const int row = 8 * ty + r;
      if(row >= 3 * ST_TT) continue;
      const int node = tileNode[row / 3];
      if(node < 0) continue;
      float* out = Lc + (int64_t(node) * 3 + row % 3) * Lp;
#pragma unroll
      for(int j = 0; j < 5; j++)
      {
         const int col = col0 + 2 * tx + 32 * j;
         if(col < Lp) out[col] = col < L ? acc[r][2 * j] : 0.f;
         if(col + 1 < Lp) out[col + 1] = col + 1 < L ? acc[r][2 * j + 1] : 0.f;
      }
   }
}

// ====================================================================================
// L2P + near field: one block per target leaf. The local expansion is turned into the
// expansion of B = curl A (order p - 1) in shared memory, evaluated per target by the
// harmonic recurrence, then the direct sum over the leaf's source list is added.
//
// Real-basis derivatives used for the curl (R = regular harmonics, standard convention):
//   d/dz R_l^{+-m} = -R_{l-1}^{+-m}
//   d/dx, d/dy move m by one; see gradCoeff below.
// ====================================================================================
template <class T>
__device__ inline T coefAt(const T* Lv, int l, int m)
{
   return (abs(m) <= l) ? Lv[hidx(l, m)] : T(0);
}

// Coefficient of R_{l'}^{mu} in d/dx_j (sum_k L_k R_k), j = 0 (x), 1 (y), 2 (z); l = l' + 1.
template <class T>
__device__ inline T gradCoeff(const T* Lv, int j, int lp, int mu)
{
   const int l = lp + 1;
   const T h = T(0.5), r2 = T(0.70710678118654752440);
   if(j == 2) return -coefAt(Lv, l, mu);
   if(j == 0)
   {
      if(mu == 0) return -r2 * coefAt(Lv, l, 1);
      if(mu == 1) return -h * coefAt(Lv, l, 2) + r2 * coefAt(Lv, l, 0);
      if(mu >= 2) return -h * coefAt(Lv, l, mu + 1) + h * coefAt(Lv, l, mu - 1);
      if(mu == -1) return -h * coefAt(Lv, l, -2);
      return -h * coefAt(Lv, l, mu - 1) + h * coefAt(Lv, l, mu + 1);
   }
   if(mu == 0) return -r2 * coefAt(Lv, l, -1);
   if(mu == 1) return -h * coefAt(Lv, l, -2);
   if(mu >= 2) return -h * coefAt(Lv, l, -(mu + 1)) - h * coefAt(Lv, l, -(mu - 1));
   if(mu == -1) return h * coefAt(Lv, l, 2) + r2 * coefAt(Lv, l, 0);
   return h * coefAt(Lv, l, 1 - mu) + h * coefAt(Lv, l, -mu - 1);
}

// 1/sqrt(x) by the PTX approximate reciprocal square root (flushes subnormal inputs to zero).
__device__ __forceinline__ float rsqrtApprox(float x)
{
   float y;
   asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
   return y;
}
// Packed FP32 pairs (sm_100 f32x2 arithmetic): two floats in one 64-bit register, low half first.
typedef unsigned long long f2p;
__device__ __forceinline__ f2p pk2(float a, float b)
{
   f2p r;
   asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
   return r;
}
__device__ __forceinline__ void upk2(f2p v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2p sub2(f2p a, f2p b)
{
   f2p d;
   asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
   return d;
}
__device__ __forceinline__ f2p mul2(f2p a, f2p b)
{
   f2p d;
   asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
   return d;
}
__device__ __forceinline__ f2p fma2(f2p a, f2p b, f2p c)
{
   f2p d;
   asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
   return d;
}
__device__ __forceinline__ void cpAsync4(void* dst, const void* src, uint32_t srcBytes)
{
   const uint32_t d = uint32_t(__cvta_generic_to_shared(dst));
   asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(srcBytes) : "memory");
}
// Bytes of one near-field source tile of TS points: FP32 tiles hold source pairs
// [x0 x1 y0 y1 z0 z1 wx0 wx1 wy0 wy1 wz0 wz1] (24 bytes a point), FP64 tiles two [TS] arrays of
// (x, y, z, -) and (wx, wy, wz, -).
template <class T>
__host__ __device__ constexpr int nearTileBytes(int TS)
{
   return sizeof(T) == 4 ? 24 * TS : 2 * 4 * int(sizeof(T)) * TS;
}

// Largest 1/r whose cube is finite in T, for the coincident-pair cap of the near field.
template <class T> __device__ __forceinline__ T riCap();
template <> __device__ __forceinline__ float riCap<float>() { return 6.0e12f; }
template <> __device__ __forceinline__ double riCap<double>() { return 1.0e100; }

// L2P alone, one warp per target leaf, one target per lane (32 at a time). The leaf's curl
// expansion (and, for A, its local expansion) is stored as [k] (x, y, z, 0) with the real-basis
// factors (-1)^l sqrt2 folded in, so each visited harmonic costs one broadcast 16-byte shared
// load and three FMAs per coefficient. The recurrence's coefficients come from a table shared by
// the block (visit order: m outer, l inner): 1/(2m) at l = m, else the (a, b) of
// S_l^m = a z S_{l-1}^m - b r^2 S_{l-2}^m, so no lane divides. The far field is written to the
// outputs unscaled; kL2PNear<..., FAR = false> adds the near field and applies the scale.
constexpr int L2PW_WARPS = 4;

template <class T, bool WANTA>
inline size_t l2pWarpSmem(int p)
{
   const int L = nharm(p), Lb = nharm(p - 1), nV = (p + 1) * (p + 2) / 2;
   const size_t perWarp = size_t(4) * Lb + (WANTA ? size_t(4) * L : 0) + size_t(3) * padded(L);
   return sizeof(T) * (size_t(4) * nV + L2PW_WARPS * perWarp);
}

template <class T, bool WANTA>
__global__ void __launch_bounds__(32 * L2PW_WARPS) kL2PWarp(Tree t, const RootBox* __restrict__ rootp, int p,
                                                          int Lp, const T* __restrict__ Lc,
                                                          const typename Vec4<T>::type* __restrict__ tpos,
                                                          const int* __restrict__ tOrder,
                                                          const CurlEntry<T>* __restrict__ curl, int want,
                                                          T* __restrict__ outB, T* __restrict__ outA)
{
   typedef typename Vec4<T>::type V4;
   extern __shared__ __align__(16) unsigned char smraw[];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int L = nharm(p), Lb = nharm(p - 1);
   const int q = WANTA ? p : p - 1;                     // highest degree visited
   const int nV = (p + 1) * (p + 2) / 2;                // table: degrees 0..p
   V4* tab = (V4*)smraw;
   const int perWarp = 4 * Lb + (WANTA ? 4 * L : 0) + 3 * Lp;
   T* wbase = (T*)(tab + nV) + warp * perWarp;
   V4* Cs = (V4*)wbase;                                 // [Lb] curl expansion
   V4* As = Cs + Lb;                                    // [L] local expansion (WANTA)
   T* Ls = wbase + 4 * Lb + (WANTA ? 4 * L : 0);        // [3][Lp] the box's local row
   for(int v = threadIdx.x; v < nV; v += 32 * L2PW_WARPS)
   {
      int m = 0, r = v;
      while(r >= p + 1 - m) { r -= p + 1 - m; m++; }
      const int l = m + r;
      T a = T(0), b = T(0);
      if(l == m) a = m > 0 ? T(1) / T(2 * m) : T(1);
      else
      {
         const int lp = l - 1;
         const T inv = T(1) / T((lp - m + 1) * (lp + m + 1));
         a = T(2 * lp + 1) * inv;
         b = lp == m ? T(0) : inv;
      }
      tab[v] = V4{a, b, T(0), T(0)};
   }
   __syncthreads();
   const int node = blockIdx.x * L2PW_WARPS + warp;
   if(node >= t.nNodes || t.nchild[node] != 0) return;
   const int t0 = t.t0[node], t1 = t.t1[node];
   if(t1 == t0) return;
   // the box's local row staged with 16-byte loads (Lp is a multiple of 16), all issued at once
   {
      typedef typename Vec4<T>::type V4g;
      const V4g* src = reinterpret_cast<const V4g*>(Lc + int64_t(node) * 3 * Lp);
      V4g* dst = reinterpret_cast<V4g*>(Ls);
#pragma unroll 4
      for(int e = lane; e < 3 * Lp / 4; e += 32) dst[e] = src[e];
   }
   __syncwarp();
   const T* lc = Ls;
   // the curl expansion from the table: each entry <= 4 terms of the box's local row
#pragma unroll 4
   for(int e = lane; e < 4 * Lb; e += 32)
   {
      const CurlEntry<T> ce = curl[e];
      ((T*)Cs)[e] = ce.c[0] * lc[ce.idx[0]] + ce.c[1] * lc[ce.idx[1]] + ce.c[2] * lc[ce.idx[2]] +
                    ce.c[3] * lc[ce.idx[3]];
   }
   if(WANTA)
   {
      const T sq2 = T(1.4142135623730950488);
      for(int e = lane; e < 4 * L; e += 32)
      {
         const int k = e >> 2, c = e & 3;
         int l = int(sqrtf(float(k)));
         while(l * l > k) l--;
         while((l + 1) * (l + 1) <= k) l++;
         const int mu = k - l * l - l;
         const T f = ((l & 1) ? T(-1) : T(1)) * (mu != 0 ? sq2 : T(1));
         ((T*)As)[e] = c < 3 ? f * lc[c * Lp + k] : T(0);
      }
   }
   __syncwarp();
   const RootBox rb = rootp[rootOf(t, node)];
   double cen[3], h;
   nodeCenter(rb, t.level[node], t.ix[node], t.iy[node], t.iz[node], cen, h);
   const T ih = T(1.0 / h), ih2 = T(1.0 / (h * h));
   // G lanes per target when the leaf is small (G = 4 up to 8 targets, 2 up to 16): group g of the
   // W = 32 / G lanes visits the orders m = g, g + G, ..., and the groups' sums meet by shuffles
   const int nt = t1 - t0;
   const int G = nt <= 8 ? 4 : (nt <= 16 ? 2 : 1), W = 32 / G;
   const int g = lane / W, jl = lane % W;
   auto vStart = [&](int m) { return m * (p + 1) - m * (m - 1) / 2; };   // first visit of order m
   for(int base = t0; base < t1; base += W)
   {
      const int ti = base + jl;
      const bool act = ti < t1;
      const V4 x = act ? tpos[ti] : V4{T(0), T(0), T(0), T(0)};
      const T ux = T((double(x.x) - cen[0]) / h), uy = T((double(x.y) - cen[1]) / h),
              uz = T((double(x.z) - cen[2]) / h);
      const T r2 = ux * ux + uy * uy + uz * uz;
      T B0 = T(0), B1 = T(0), B2 = T(0), A0 = T(0), A1 = T(0), A2 = T(0);
      T dre = T(1), dim = T(0);   // S_m^m, advanced to this group's first order
      for(int j = 1; j <= g; j++)
      {
         const T sc = tab[vStart(j)].x;
         const T nre = (dre * ux - dim * uy) * sc;
         const T nim = (dre * uy + dim * ux) * sc;
         dre = nre; dim = nim;
      }
      // S_l^0 stays real (the imaginary parts are zero), so order 0 needs no case of its own: its
      // k1 = k0 term adds zero
      // the contribution of one visited harmonic (l, m): coefficients k0 = hidx(l, m), k1 = hidx(l, -m)
      auto visit = [&](int l, int k0, int k1, T are, T aim) {
         if(!WANTA || l < p)
         {
            const V4 c0 = Cs[k0], c1 = Cs[k1];
            B0 += c0.x * are + c1.x * aim; B1 += c0.y * are + c1.y * aim; B2 += c0.z * are + c1.z * aim;
         }
         if(WANTA)
         {
            const V4 a0 = As[k0], a1 = As[k1];
            A0 += a0.x * are + a1.x * aim; A1 += a0.y * are + a1.y * aim; A2 += a0.z * are + a1.z * aim;
         }
      };
      // S_{j-1}^{j-1} -> S_j^j
      auto diag = [&](T& re, T& im, int j) {
         const T sc = tab[vStart(j)].x;
         const T nre = (re * ux - im * uy) * sc;
         const T nim = (re * uy + im * ux) * sc;
         re = nre; im = nim;
      };
      // orders m and m2 = m + G walked together: two independent recurrences in flight per lane
      for(int m = g; m <= q; m += 2 * G)
      {
         const int m2 = m + G;
         const bool two = m2 <= q;
         T e2re = dre, e2im = dim;   // S_{m2}^{m2}
         for(int j = m + 1; j <= m2 && j <= q; j++) diag(e2re, e2im, j);
         int v = vStart(m), v2 = two ? vStart(m2) : 0;
         T are = dre, aim = dim, bre = T(0), bim = T(0);
         T are2 = e2re, aim2 = e2im, bre2 = T(0), bim2 = T(0);
         int k0 = m * m + 2 * m, k1 = m * m, k02 = m2 * m2 + 2 * m2, k12 = m2 * m2;
         visit(m, k0, k1, are, aim);
         v++;
         if(two)
         {
            visit(m2, k02, k12, are2, aim2);
            v2++;
         }
         const int n2 = two ? q - m2 : 0;   // steps both orders take
#pragma unroll 2
         for(int st = 1; st <= n2; st++, v++, v2++)
         {
            const int l = m + st, l2 = m2 + st;
            const V4 ab = tab[v], ab2 = tab[v2];
            k0 += 2 * l; k1 += 2 * l; k02 += 2 * l2; k12 += 2 * l2;
            const T az = ab.x * uz, br = ab.y * r2, az2 = ab2.x * uz, br2 = ab2.y * r2;
            const T cre = az * are - br * bre, cim = az * aim - br * bim;
            const T cre2 = az2 * are2 - br2 * bre2, cim2 = az2 * aim2 - br2 * bim2;
            bre = are; bim = aim; are = cre; aim = cim;
            bre2 = are2; bim2 = aim2; are2 = cre2; aim2 = cim2;
            visit(l, k0, k1, are, aim);
            visit(l2, k02, k12, are2, aim2);
         }
         // the rest of order m (all of it when m2 > q)
#pragma unroll 4
         for(int l = m + n2 + 1; l <= q; l++, v++)
         {
            const V4 ab = tab[v];
            k0 += 2 * l; k1 += 2 * l;
            const T az = ab.x * uz, br = ab.y * r2;
            const T cre = az * are - br * bre, cim = az * aim - br * bim;
            bre = are; bim = aim; are = cre; aim = cim;
            visit(l, k0, k1, are, aim);
         }
         // S_m^m -> S_{m+2G}^{m+2G}
         dre = e2re; dim = e2im;
         for(int j = m2 + 1; j <= m2 + G && j <= q; j++) diag(dre, dim, j);
      }
      for(int off = 16; off >= W; off >>= 1)
      {
         B0 += __shfl_down_sync(0xffffffffu, B0, off);
         B1 += __shfl_down_sync(0xffffffffu, B1, off);
         B2 += __shfl_down_sync(0xffffffffu, B2, off);
         if(WANTA)
         {
            A0 += __shfl_down_sync(0xffffffffu, A0, off);
            A1 += __shfl_down_sync(0xffffffffu, A1, off);
            A2 += __shfl_down_sync(0xffffffffu, A2, off);
         }
      }
      if(act && g == 0)
      {
         const int o = tOrder[ti];
         if(want & 1)
         {
            outB[3 * int64_t(o)] = B0 * ih2; outB[3 * int64_t(o) + 1] = B1 * ih2; outB[3 * int64_t(o) + 2] = B2 * ih2;
         }
         if(WANTA)
         {
            outA[3 * int64_t(o)] = A0 * ih; outA[3 * int64_t(o) + 1] = A1 * ih; outA[3 * int64_t(o) + 2] = A2 * ih;
         }
      }
   }
}

// L2P and the direct near field: one block of NT threads per target leaf. The far field comes from
// the leaf's local expansion (analytic curl, one target per thread). The near field packs the
// points of the leaf's direct-interaction source nodes into shared tiles of TS points; when the
// leaf has fewer targets than threads, the G = NT / targets thread groups each take every G-th
// source of a tile and their partial sums are added in a fixed order at the end. Each thread
// sums one tile in T and the tile sums in FP64, so no single-precision chain is longer than a tile.
template <class T, int NT, int TS, int NE, bool WANTA, bool FAR>
__global__ void __launch_bounds__(NT, FAR ? 1 : (sizeof(T) == 4 ? (WANTA ? 12 : 16) : 8)) kL2PNear(Tree t, const RootBox* __restrict__ rootp, int p, int Lp,
                                               const T* __restrict__ Lc,
                                               const typename Vec4<T>::type* __restrict__ tpos,
                                               const typename Vec4<T>::type* __restrict__ spos,
                                               const typename Vec4<T>::type* __restrict__ sq,
                                               const int* __restrict__ p2pOff, const int* __restrict__ p2pList,
                                               const int* __restrict__ tOrder, T scaleB, T scaleA, int want,
                                               T* __restrict__ outB, T* __restrict__ outA)
{
   typedef typename Vec4<T>::type V4;
   extern __shared__ __align__(32) unsigned char smraw[];
   const int node = blockIdx.x;
   if(t.nchild[node] != 0 || t.t1[node] == t.t0[node]) return;
   const int tid = threadIdx.x;
   const int L = nharm(p);
   const int Lb = nharm(p - 1);
   T* Ls = (T*)smraw;          // [3][L] local
   T* Cs = Ls + 3 * L;         // [3][Lb] curl expansion
   // source tiles start on a 32-byte boundary after the two coefficient arrays (none without FAR)
   const size_t coefBytes = FAR ? (sizeof(T) * (3 * L + 3 * Lb) + 31) & ~size_t(31) : 0;
   unsigned char* tiles = smraw + coefBytes;                          // two source tiles
   double* red = (double*)(tiles + 2 * nearTileBytes<T>(TS));        // [6][NT] group partial sums
   typedef cub::BlockScan<int, NT> ScanT;
   __shared__ typename ScanT::TempStorage scanTmp;
   __shared__ int ePre[NE + 1];        // prefix sums of the batch's source counts
   __shared__ int eSrc[NE];            // first sorted source of each batch entry
   if(FAR)
   {
   for(int e = tid; e < 3 * L; e += NT) Ls[e] = Lc[int64_t(node) * 3 * Lp + (e / L) * Lp + e % L];
   __syncthreads();
   for(int e = tid; e < 3 * Lb; e += NT)
   {
      const int c = e / Lb, k = e % Lb;
      int lp = int(sqrtf(float(k)));
      while(lp * lp > k) lp--;
      while((lp + 1) * (lp + 1) <= k) lp++;
      const int mu = k - lp * lp - lp;
      // B_x = dAz/dy - dAy/dz, B_y = dAx/dz - dAz/dx, B_z = dAy/dx - dAx/dy
      const int cp = (c + 2) % 3, cm = (c + 1) % 3;   // (z,y) for x; (x,z) for y; (y,x) for z
      const int jp = (c + 1) % 3, jm = (c + 2) % 3;
      Cs[e] = gradCoeff(Ls + cp * L, jp, lp, mu) - gradCoeff(Ls + cm * L, jm, lp, mu);
   }
   __syncthreads();
   }
   const RootBox rb = rootp[rootOf(t, node)];
   double c[3], h;
   nodeCenter(rb, t.level[node], t.ix[node], t.iy[node], t.iz[node], c, h);
   const T ih = T(1.0 / h), ih2 = T(1.0 / (h * h));
   const int t0 = t.t0[node], t1 = t.t1[node];
   const int e0 = p2pOff[node], e1 = p2pOff[node + 1];
   constexpr bool wantA = WANTA;
   for(int base = t0; base < t1; base += NT)
   {
      const int nt = min(NT, t1 - base);     // targets in this pass
      const int G = NT / nt;                 // thread groups sharing a tile's sources
      const int tt = tid % nt, g = tid / nt;
      const bool inGroup = g < G;
      const int ti = base + tt;
      V4 x = inGroup ? tpos[ti] : V4{T(0), T(0), T(0), T(0)};
      double Bd[3] = {0, 0, 0}, Ad[3] = {0, 0, 0};
      if(!FAR && inGroup && g == 0)
      {
         // the far field, already evaluated by kL2PWarp into the outputs (unscaled)
         const int o = tOrder[ti];
         if(want & 1) for(int d = 0; d < 3; d++) Bd[d] = double(outB[3 * int64_t(o) + d]);
         if(WANTA) for(int d = 0; d < 3; d++) Ad[d] = double(outA[3 * int64_t(o) + d]);
      }
      if(FAR && inGroup && g == 0)
      {
         T B[3] = {T(0), T(0), T(0)}, A[3] = {T(0), T(0), T(0)};
         const T ux = T((double(x.x) - c[0]) / h), uy = T((double(x.y) - c[1]) / h), uz = T((double(x.z) - c[2]) / h);
         const T sq2 = T(1.4142135623730950488);
         visitRegular<T>(p, ux, uy, uz, [&](int l, int m, T re, T im) {
            const T s = (l & 1) ? T(-1) : T(1);
            T r0, r1;
            if(m == 0) { r0 = s * re; r1 = T(0); }
            else { r0 = s * sq2 * re; r1 = s * sq2 * im; }
            if(l < p)
            {
               const int k0 = hidx(l, m), k1 = hidx(l, -m);
               for(int d = 0; d < 3; d++)
               {
                  B[d] += Cs[d * Lb + k0] * r0;
                  if(m) B[d] += Cs[d * Lb + k1] * r1;
               }
            }
            if(wantA)
            {
               const int k0 = hidx(l, m), k1 = hidx(l, -m);
               for(int d = 0; d < 3; d++)
               {
                  A[d] += Ls[d * L + k0] * r0;
                  if(m) A[d] += Ls[d * L + k1] * r1;
               }
            }
         });
         for(int d = 0; d < 3; d++) { Bd[d] = double(B[d] * ih2); Ad[d] = double(A[d] * ih); }
      }
      // near field over packed tiles of the direct-list source nodes
      auto tileSum = [&](int n, int b) {
         if(!inGroup) return;
         T pb[3] = {T(0), T(0), T(0)}, pa[3] = {T(0), T(0), T(0)};
         if constexpr(sizeof(T) == 4)
         {
            // two sources per step in packed f32x2 arithmetic; the cross product's two products are
            // accumulated in separate sums (no negation in the packed FMA)
            const ulonglong2* tq = (const ulonglong2*)(tiles + b * nearTileBytes<T>(TS));
            const int nPairs = (n + 1) >> 1;
            const f2p X = pk2(x.x, x.x), Y = pk2(x.y, x.y), Z = pk2(x.z, x.z);
            f2p sxp = 0, sxn = 0, syp = 0, syn = 0, szp = 0, szn = 0, ax = 0, ay = 0, az = 0;
#pragma unroll 2
            for(int P = g; P < nPairs; P += G)
            {
               const ulonglong2 q0 = tq[3 * P], q1 = tq[3 * P + 1], q2 = tq[3 * P + 2];
               const f2p DX = sub2(X, q0.x), DY = sub2(Y, q0.y), DZ = sub2(Z, q1.x);
               f2p R2 = mul2(DX, DX);
               R2 = fma2(DY, DY, R2);
               R2 = fma2(DZ, DZ, R2);
               float r2a, r2b;
               upk2(R2, r2a, r2b);
               float ria = rsqrtApprox(r2a), rib = rsqrtApprox(r2b);
               // coincident pair (the target itself) and the empty slot of an odd tile: no
               // contribution. For B the capped 1/r (whose cube still fits a float) meets a zero
               // difference vector or a zero weight; A needs the explicit test.
               if constexpr(WANTA)
               {
                  ria = r2a > 0.f ? ria : 0.f;
                  rib = r2b > 0.f ? rib : 0.f;
               }
               else
               {
                  ria = fminf(ria, riCap<float>());
                  rib = fminf(rib, riCap<float>());
               }
               const f2p RI = pk2(ria, rib);
               const f2p RI3 = mul2(mul2(RI, RI), RI);
               const f2p UX = mul2(q1.y, RI3), UY = mul2(q2.x, RI3), UZ = mul2(q2.y, RI3);
               sxp = fma2(UY, DZ, sxp); sxn = fma2(UZ, DY, sxn);
               syp = fma2(UZ, DX, syp); syn = fma2(UX, DZ, syn);
               szp = fma2(UX, DY, szp); szn = fma2(UY, DX, szn);
               if constexpr(WANTA)
               {
                  ax = fma2(q1.y, RI, ax); ay = fma2(q2.x, RI, ay); az = fma2(q2.y, RI, az);
               }
            }
            float u0, u1, v0, v1;
            upk2(sxp, u0, u1); upk2(sxn, v0, v1); pb[0] = (u0 + u1) - (v0 + v1);
            upk2(syp, u0, u1); upk2(syn, v0, v1); pb[1] = (u0 + u1) - (v0 + v1);
            upk2(szp, u0, u1); upk2(szn, v0, v1); pb[2] = (u0 + u1) - (v0 + v1);
            if constexpr(WANTA)
            {
               upk2(ax, u0, u1); pa[0] = u0 + u1;
               upk2(ay, u0, u1); pa[1] = u0 + u1;
               upk2(az, u0, u1); pa[2] = u0 + u1;
            }
         }
         else
         {
            const V4* tp = (const V4*)(tiles + b * nearTileBytes<T>(TS));
            const V4* tq = tp + TS;
#pragma unroll 4
            for(int i = g; i < n; i += G)
            {
               const V4 y = tp[i], w = tq[i];
               const T dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
               const T r2 = dx * dx + dy * dy + dz * dz;
               T ri = rsqrt(r2);
               if constexpr(WANTA) ri = r2 > T(0) ? ri : T(0);
               else ri = min(ri, riCap<T>());
               const T ri3 = ri * ri * ri;
               pb[0] += (w.y * dz - w.z * dy) * ri3;
               pb[1] += (w.z * dx - w.x * dz) * ri3;
               pb[2] += (w.x * dy - w.y * dx) * ri3;
               if(wantA) { pa[0] += w.x * ri; pa[1] += w.y * ri; pa[2] += w.z * ri; }
            }
         }
         for(int d = 0; d < 3; d++) { Bd[d] += double(pb[d]); Ad[d] += double(pa[d]); }
      };
      // the list in batches of NE entries: their point ranges are read together into shared memory
      // and prefix-summed, so every tile position finds its source by a shared-memory search and
      // all of a tile's loads are independent
      for(int eb = e0; eb < e1; eb += NE)
      {
         const int ne = min(NE, e1 - eb);
         int sz[NE / NT];
#pragma unroll
         for(int r = 0; r < NE / NT; r++)
         {
            const int k = tid * (NE / NT) + r;
            int a = 0, n = 0;
            if(k < ne)
            {
               const int S = p2pList[eb + k];
               a = t.s0[S];
               n = t.s1[S] - a;
            }
            if(k < NE) eSrc[k] = a;
            sz[r] = n;
         }
         int total;
         ScanT(scanTmp).ExclusiveSum(sz, sz, total);
#pragma unroll
         for(int r = 0; r < NE / NT; r++) ePre[tid * (NE / NT) + r] = sz[r];
         if(tid == 0) ePre[NE] = total;
         __syncthreads();
         // tiles double-buffered: tile k + 1's copies (cp.async) are in flight while tile k is summed
         auto issueTile = [&](int pos, int b) {
            const int n = min(TS, total - pos);
            const int nf = sizeof(T) == 4 ? (n + 1) & ~1 : n;   // FP32: the odd tile's last pair slot zero-filled
            unsigned char* tb = tiles + b * nearTileBytes<T>(TS);
            for(int j = tid; j < nf; j += NT)
            {
               const bool in = j < n;
               int src = 0;
               if(in)
               {
                  const int qpos = pos + j;
                  int lo = 0, hi = ne;  // last entry with ePre <= qpos
                  while(hi - lo > 1)
                  {
                     const int mid = (lo + hi) >> 1;
                     if(ePre[mid] <= qpos) lo = mid;
                     else hi = mid;
                  }
                  src = eSrc[lo] + (qpos - ePre[lo]);
               }
               if constexpr(sizeof(T) == 4)
               {
                  float* d = (float*)tb + 12 * (j >> 1) + (j & 1);
                  const float* ps = (const float*)(spos + src);
                  const float* qs = (const float*)(sq + src);
                  const uint32_t by = in ? 4u : 0u;
                  cpAsync4(d, ps, by); cpAsync4(d + 2, ps + 1, by); cpAsync4(d + 4, ps + 2, by);
                  cpAsync4(d + 6, qs, by); cpAsync4(d + 8, qs + 1, by); cpAsync4(d + 10, qs + 2, by);
               }
               else
               {
                  V4* tp = (V4*)tb;
#pragma unroll
                  for(int h = 0; h < int(sizeof(V4)) / 16; h++)
                  {
                     cpAsync16Simt((char*)(tp + j) + 16 * h, (const char*)(spos + src) + 16 * h, 16u);
                     cpAsync16Simt((char*)(tp + TS + j) + 16 * h, (const char*)(sq + src) + 16 * h, 16u);
                  }
               }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
         };
         const int nTiles = (total + TS - 1) / TS;
         if(nTiles > 0) issueTile(0, 0);
         for(int k = 0; k < nTiles; k++)
         {
            if(k + 1 < nTiles)
            {
               issueTile((k + 1) * TS, (k + 1) & 1);
               asm volatile("cp.async.wait_group 1;" ::: "memory");
            }
            else
               asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncthreads();
            tileSum(min(TS, total - k * TS), k & 1);
            __syncthreads();
         }
      }
      // add the groups' partial sums in group order
      if(G > 1)
      {
         for(int d = 0; d < 3; d++) { red[d * NT + tid] = Bd[d]; red[(3 + d) * NT + tid] = Ad[d]; }
         __syncthreads();
         if(g == 0)
            for(int gg = 1; gg < G; gg++)
               for(int d = 0; d < 3; d++)
               {
                  Bd[d] += red[d * NT + gg * nt + tt];
                  Ad[d] += red[(3 + d) * NT + gg * nt + tt];
               }
         __syncthreads();
      }
      if(g == 0)
      {
         const int o = tOrder[ti];
         if(want & 1) for(int d = 0; d < 3; d++) outB[3 * int64_t(o) + d] = T(Bd[d] * double(scaleB));
         if(want & 2) for(int d = 0; d < 3; d++) outA[3 * int64_t(o) + d] = T(Ad[d] * double(scaleA));
      }
   }
}

// ====================================================================================
// Direct sums over all sources (fmm_direct): one thread per target, sources staged through
// shared memory.
// ====================================================================================
template <class T, class U, int NT>
__global__ void __launch_bounds__(NT) kDirect(const typename Vec4<T>::type* __restrict__ spos,
                                              const typename Vec4<T>::type* __restrict__ sq, int n,
                                              const U* __restrict__ tgt, int m, const int* __restrict__ sseg,
                                              const int* __restrict__ tseg, U scaleB, U scaleA, int want,
                                              U* __restrict__ outB, U* __restrict__ outA)
{
   __shared__ U Sp[NT][4];
   __shared__ U Sq[NT][3];
   // blockIdx.y selects a coil: its targets [tseg[c], tseg[c+1]) see only its sources
   // [sseg[c], sseg[c+1]); without segments every target sees every source
   const int c = blockIdx.y;
   const int tBeg = tseg ? tseg[c] : 0, tEnd = tseg ? tseg[c + 1] : m;
   const int sBeg = sseg ? sseg[c] : 0, sEnd = sseg ? sseg[c + 1] : n;
   const int ti = tBeg + blockIdx.x * NT + threadIdx.x;
   if(tBeg + int(blockIdx.x) * NT >= tEnd) return;
   const bool active = ti < tEnd;
   U x = 0, y = 0, z = 0;
   if(active) { x = tgt[3 * int64_t(ti)]; y = tgt[3 * int64_t(ti) + 1]; z = tgt[3 * int64_t(ti) + 2]; }
   U B[3] = {0, 0, 0}, A[3] = {0, 0, 0};
   for(int sb = sBeg; sb < sEnd; sb += NT)
   {
      const int cnt = min(NT, sEnd - sb);
      __syncthreads();
      if(threadIdx.x < cnt)
      {
         const auto a = spos[sb + threadIdx.x];
         const auto b = sq[sb + threadIdx.x];
         Sp[threadIdx.x][0] = U(a.x); Sp[threadIdx.x][1] = U(a.y); Sp[threadIdx.x][2] = U(a.z);
         Sq[threadIdx.x][0] = U(b.x); Sq[threadIdx.x][1] = U(b.y); Sq[threadIdx.x][2] = U(b.z);
      }
      __syncthreads();
      if(active)
         for(int i = 0; i < cnt; i++)
         {
            const U dx = x - Sp[i][0], dy = y - Sp[i][1], dz = z - Sp[i][2];
            const U r2 = dx * dx + dy * dy + dz * dz;
            if(r2 == U(0)) continue;
            U ri;
            if constexpr(sizeof(U) == 4) ri = rsqrtf(r2);
            else ri = U(1) / sqrt(r2);
            const U ri3 = ri * ri * ri;
            B[0] += (Sq[i][1] * dz - Sq[i][2] * dy) * ri3;
            B[1] += (Sq[i][2] * dx - Sq[i][0] * dz) * ri3;
            B[2] += (Sq[i][0] * dy - Sq[i][1] * dx) * ri3;
            A[0] += Sq[i][0] * ri; A[1] += Sq[i][1] * ri; A[2] += Sq[i][2] * ri;
         }
   }
   if(active)
   {
      if(want & 1) for(int d = 0; d < 3; d++) outB[3 * int64_t(ti) + d] = B[d] * scaleB;
      if(want & 2) for(int d = 0; d < 3; d++) outA[3 * int64_t(ti) + d] = A[d] * scaleA;
   }
}

// ====================================================================================
// Host drivers
// ====================================================================================
template <class T>
fmm_status upwardT(Plan& P, cudaStream_t st)
{
   FMM_TRY(buildOperators(P, st));
   const int64_t N = P.tree.nNodes;
   const int Lp = P.Lp;
   FMM_TRY(P.mult.reserve(sizeof(T) * N * 3 * Lp));
   FMM_CUDA(cudaMemsetAsync(P.mult.ptr, 0, sizeof(T) * N * 3 * Lp, st));
   typedef typename Vec4<T>::type V4;
   constexpr int NT = 64;
   const size_t shm = sizeof(T) * 3 * Lp;
   if(P.bem)
   {
      // dipole multipoles of the BEM sources (fmm_bem.cu); the translations below are the same
      P.p2mPiecesTag = -1;
      FMM_TRY(bemP2MT<T>(P, st));
   }
   else if(P.p2mChunk == 0)
   {
      const size_t shw = p2mWarpSmem<T>(P.p, Lp);
      if(shw > 48 * 1024)
         FMM_CUDA(cudaFuncSetAttribute(kP2MWarp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shw)));
      // tensor-core M2M plans: the leaves' multipoles also leave as the M2M's operand pieces
      int np = 0;
      if(sizeof(T) == 4 && P.tcTranslations(1) && P.tcDrainMode != 0) np = m2mPieces(P);
      if(np)
         FMM_TRY(P.multBf.reserve(size_t(np == 1 ? 4 : 2 * np) * size_t(N) * 3 * Lp));
      kP2MWarp<T><<<int((N + P2MW_WARPS - 1) / P2MW_WARPS), 32 * P2MW_WARPS, shw, st>>>(
         P.tree, P.root, (const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, P.p, Lp, (T*)P.mult.ptr,
         np ? (uint8_t*)P.multBf.ptr : nullptr, np);
      P.p2mPiecesTag = np ? (np == 1 ? 3 : 2 * np) : -1;
   }
   else
   {
      P.p2mPiecesTag = -1;
      if(P.p2mChunk == 32)
         kP2M<T, NT, 32><<<int(N), NT, shm, st>>>(P.tree, P.root, (const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, P.p,
                                                 Lp, (T*)P.mult.ptr);
      else
         kP2M<T, NT, 16><<<int(N), NT, shm, st>>>(P.tree, P.root, (const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, P.p,
                                                 Lp, (T*)P.mult.ptr);
   }
   FMM_TRY(launched(P, "kP2M", st));
   FMM_CHECK_LAUNCH();
   if(P.tcTranslations(1)) return m2mTensorCore(P, st);
   const int nCol = (Lp + TG_N - 1) / TG_N;
   for(int level = P.tree.nLevels - 2; level >= 0; level--)
   {
      const int a = P.parStart[level], b = P.parStart[level + 1];
      if(b <= a) continue;
      kTranslateLevel<T, true><<<dim3((b - a + TG_P - 1) / TG_P, nCol), 256, 0, st>>>(
         P.tree, (const int*)P.parList.ptr, a, b, P.p, Lp, (const T*)P.opM2Mw.ptr, (T*)P.mult.ptr);
      FMM_TRY(launched(P, "kTranslateLevel<M2M>", st));
   }
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

template <class T>
fmm_status m2lSimt(Plan& P, cudaStream_t st)
{
   const int count = P.nM2LTargets;
   if(count <= 0) return FMM_OK;
   constexpr int RPT = SimtShape<T>::RPT, KC = SimtShape<T>::KC;
   constexpr int TT = 8 * RPT / 3;
   const int L = P.L, Lp = P.Lp;
   const int nChunks = (L + KC - 1) / KC;
   if(Lp > 32 * SM_NC || nChunks > 32) return setError(FMM_E_INVALID, "CUDA-core M2L supports p <= 16");
   // degree cutoff (see fmm_config.m2l_tc_degree_cutoff): FP32 plans default to p + 8, FP64 plans
   // to the full operator
   const int c = P.cfg.m2l_tc_degree_cutoff;
   const int cut = c < 0 || (c == 0 && P.fp64) ? 2 * P.p : (c == 0 ? P.p + 8 : std::max(c, P.p));
   SimtCols cols{};
   for(int g = 0; g < nChunks; g++)
   {
      const int k = KC * g;
      int lmin = 0;
      while((lmin + 1) * (lmin + 1) <= k) lmin++;
      const int n = cut - lmin >= 0 ? std::min(L, (cut - lmin + 1) * (cut - lmin + 1)) : 0;
      cols.n[g] = std::min(Lp, (n + 3) / 4 * 4);
   }
   if(sizeof(T) == 4 && P.simtTiled)
   {
      // FP32: the register-tiled kernel, K chunks of 16 (or 32) with the same degree cutoff
      const int ST_KC = P.simtKc;
      SimtCols c16{};
      const int n16 = (L + ST_KC - 1) / ST_KC;
      if(n16 > 32) return setError(FMM_E_INVALID, "CUDA-core M2L supports p <= 16");
      for(int g = 0; g < n16; g++)
      {
         const int k = ST_KC * g;
         int lmin = 0;
         while((lmin + 1) * (lmin + 1) <= k) lmin++;
         const int n = cut - lmin >= 0 ? std::min(L, (cut - lmin + 1) * (cut - lmin + 1)) : 0;
         c16.n[g] = std::min(Lp, (n + 3) / 4 * 4);
      }
      const dim3 grid((count + ST_TT - 1) / ST_TT, (Lp + ST_CB - 1) / ST_CB);
      // two blocks per SM (registers capped at 128) or one with all the registers it wants
      auto kern = P.simtTiled == 2 ? (ST_KC == 32 ? kM2LSimtTiled<1, 32> : kM2LSimtTiled<1, 16>)
                                   : (ST_KC == 32 ? kM2LSimtTiled<2, 32> : kM2LSimtTiled<2, 16>);
      const size_t smemT = ST_KC == 32 ? simtTiledSmem<32>() : simtTiledSmem<16>();
      FMM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemT)));
      kern<<<grid, 256, smemT, st>>>((const int*)P.m2lTargets.ptr, count, P.lists.vtab, L, Lp, n16, c16,
                                     (const float*)P.opM2Lw.ptr, (const float*)P.mult.ptr, (float*)P.local.ptr);
      FMM_TRY(launched(P, "kM2LSimtTiled", st));
      FMM_CHECK_LAUNCH();
      return FMM_OK;
   }
   const size_t smem = sizeof(T) * 2 * (size_t(8 * RPT) * KC + size_t(KC) * 32 * SM_NC);
   FMM_CUDA(cudaFuncSetAttribute(kM2LSimt<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
   const int blocks = (count + TT - 1) / TT;
   kM2LSimt<T><<<blocks, 256, smem, st>>>((const int*)P.m2lTargets.ptr, count, P.lists.vtab, P.p, Lp, nChunks, cols,
                                          (const T*)P.opM2Lw.ptr, (const T*)P.mult.ptr, (T*)P.local.ptr);
   FMM_TRY(launched(P, "kM2LSimt", st));
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

template <class T>
fmm_status downwardT(Plan& P, cudaStream_t st)
{
   const int64_t N = P.tree.nNodes;
   const int Lp = P.Lp;
   FMM_TRY(P.local.reserve(sizeof(T) * N * 3 * Lp));
   FMM_CUDA(cudaMemsetAsync(P.local.ptr, 0, sizeof(T) * N * 3 * Lp, st));
   if(sizeof(T) == 4 && P.cfg.m2l_mode != FMM_M2L_SIMT) FMM_TRY(m2lTensorCore(P, st));
   else FMM_TRY(m2lSimt<T>(P, st));
   if(P.eventsMade && !P.capturing) cudaEventRecord(P.ev[3], st);
   if(P.tcTranslations(2)) return l2lTensorCore(P, st);
   const int nCol = (Lp + TG_N - 1) / TG_N;
   if(P.l2lChildMajor)
   {
      for(int level = 0; level + 1 < P.tree.nLevels; level++)
      {
         L2LSeg seg;
         int maxTiles = 0;
         for(int o = 0; o <= 8; o++) seg.start[o] = P.l2lStart[8 * (level + 1) + o];
         for(int o = 0; o < 8; o++) maxTiles = std::max(maxTiles, (seg.start[o + 1] - seg.start[o] + TG_P - 1) / TG_P);
         if(maxTiles == 0) continue;
         kL2LChild<T><<<dim3(maxTiles, nCol, 8), 256, 0, st>>>(P.tree, (const int*)P.l2lTargets.ptr, seg, P.p, Lp,
                                                                (const T*)P.opL2Lw.ptr, (T*)P.local.ptr);
         FMM_TRY(launched(P, "kL2LChild", st));
      }
      FMM_CHECK_LAUNCH();
      return FMM_OK;
   }
   for(int level = 0; level + 1 < P.tree.nLevels; level++)
   {
      const int a = P.parStart[level], b = P.parStart[level + 1];
      if(b <= a) continue;
      kTranslateLevel<T, false><<<dim3((b - a + TG_P - 1) / TG_P, nCol), 256, 0, st>>>(
         P.tree, (const int*)P.parList.ptr, a, b, P.p, Lp, (const T*)P.opL2Lw.ptr, (T*)P.local.ptr);
      FMM_TRY(launched(P, "kTranslateLevel<L2L>", st));
   }
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

template <class T>
fmm_status evaluateT(Plan& P, double current, int want, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   const int64_t N = P.tree.nNodes;
   const int L = P.L, Lb = nharm(P.p - 1);
   constexpr int NT = 64, NE = 128;
   const int TS = P.nearTile == 128 ? 128 : 256;
   const bool split = P.l2pSplit != 0;
   const size_t coef = split ? 0 : (sizeof(T) * (3 * L + 3 * Lb) + 31) & ~size_t(31);
   size_t shm = coef + 2 * size_t(nearTileBytes<T>(TS)) + sizeof(double) * 6 * NT;
   T scaleB = T(REF_MU0 / (4 * REF_PI) * current), scaleA = T(1.0 / (4 * REF_PI) * current);
   if(P.bem)
   {
      // BEM: the far field sum_k L_k R_k (the A form of the L2P), then the BEM kernel's near field and
      // the 1 / (4 pi) of calcBEM (fast_multipole_solver.cpp:233-250; no current factor there)
      const size_t sh = l2pWarpSmem<T, true>(P.p);
      if(sh > 48 * 1024) FMM_CUDA(cudaFuncSetAttribute(kL2PWarp<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh)));
      kL2PWarp<T, true><<<int((N + L2PW_WARPS - 1) / L2PW_WARPS), 32 * L2PW_WARPS, sh, st>>>(
         P.tree, P.root, P.p, P.Lp, (const T*)P.local.ptr, (const V4*)P.tPos.ptr, (const int*)P.tIdx.ptr,
         (const CurlEntry<T>*)P.curlTab.ptr, 2, (T*)P.outB.ptr, (T*)P.outA.ptr);
      FMM_TRY(launched(P, "kL2PWarp", st));
      return bemNearT<T>(P, st);
   }
   if(split)
   {
      auto runL2P = [&](auto kernel, size_t sh) -> fmm_status {
         if(sh > 48 * 1024) FMM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sh)));
         kernel<<<int((N + L2PW_WARPS - 1) / L2PW_WARPS), 32 * L2PW_WARPS, sh, st>>>(
            P.tree, P.root, P.p, P.Lp, (const T*)P.local.ptr, (const V4*)P.tPos.ptr, (const int*)P.tIdx.ptr,
            (const CurlEntry<T>*)P.curlTab.ptr, want, (T*)P.outB.ptr, (T*)P.outA.ptr);
         return FMM_OK;
      };
      if(want & 2) FMM_TRY(runL2P(kL2PWarp<T, true>, l2pWarpSmem<T, true>(P.p)));
      else FMM_TRY(runL2P(kL2PWarp<T, false>, l2pWarpSmem<T, false>(P.p)));
      FMM_TRY(launched(P, "kL2PWarp", st));
   }
   auto run = [&](auto kernel) -> fmm_status {
      FMM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
      kernel<<<int(N), NT, shm, st>>>(P.tree, P.root, P.p, P.Lp, (const T*)P.local.ptr, (const V4*)P.tPos.ptr,
                                      (const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, (const int*)P.p2pOff.ptr,
                                      (const int*)P.p2pList.ptr, (const int*)P.tIdx.ptr, scaleB, scaleA, want,
                                      (T*)P.outB.ptr, (T*)P.outA.ptr);
      return FMM_OK;
   };
   if(split)
   {
      if(TS == 128)
      {
         if(want & 2) FMM_TRY(run(kL2PNear<T, NT, 128, NE, true, false>));
         else FMM_TRY(run(kL2PNear<T, NT, 128, NE, false, false>));
      }
      else
      {
         if(want & 2) FMM_TRY(run(kL2PNear<T, NT, 256, NE, true, false>));
         else FMM_TRY(run(kL2PNear<T, NT, 256, NE, false, false>));
      }
   }
   else if(TS == 128)
   {
      if(want & 2) FMM_TRY(run(kL2PNear<T, NT, 128, NE, true, true>));
      else FMM_TRY(run(kL2PNear<T, NT, 128, NE, false, true>));
   }
   else
   {
      if(want & 2) FMM_TRY(run(kL2PNear<T, NT, 256, NE, true, true>));
      else FMM_TRY(run(kL2PNear<T, NT, 256, NE, false, true>));
   }
   FMM_TRY(launched(P, "kL2PNear", st));
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

template <class T>
fmm_status directT(Plan& P, double current, int want, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   constexpr int NT = 128;
   T scaleB = T(REF_MU0 / (4 * REF_PI) * current), scaleA = T(1.0 / (4 * REF_PI) * current);
   if(P.bem) return bemDirectT<T>(P, st);
   int maxT = 0;
   for(int c = 0; c < P.nCoils; c++) maxT = std::max(maxT, P.tgtOff[c + 1] - P.tgtOff[c]);
   const int blocks = (maxT + NT - 1) / NT;
   if(blocks == 0) return FMM_OK;
   const int* seg = (const int*)P.segb.ptr;   // srcOff then tgtOff, uploaded by the tree build
   kDirect<T, T, NT><<<dim3(blocks, P.nCoils), NT, 0, st>>>((const V4*)P.sPos.ptr, (const V4*)P.sQ.ptr, int(P.n),
                                                           (const T*)P.tgtXYZ, int(P.m), seg, seg + P.nCoils + 1,
                                                           scaleB, scaleA, want, (T*)P.outB.ptr, (T*)P.outA.ptr);
   FMM_TRY(launched(P, "kDirect", st));
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

fmm_status directFp64Subset(Plan& P, double current, const double* tgtDev, int k, double* outDev, cudaStream_t st)
{
   constexpr int NT = 128;
   int blocks = (k + NT - 1) / NT;
   if(blocks == 0) return FMM_OK;
   double scaleB = REF_MU0 / (4 * REF_PI) * current;
   if(P.fp64)
   {
      kDirect<double, double, NT><<<blocks, NT, 0, st>>>((const double4*)P.sPos.ptr, (const double4*)P.sQ.ptr,
                                                         int(P.n), tgtDev, k, nullptr, nullptr, scaleB, 0.0, 1,
                                                         outDev, nullptr);
      FMM_TRY(launched(P, "kDirect", st));
   }
   else
   {
      kDirect<float, double, NT><<<blocks, NT, 0, st>>>((const float4*)P.sPos.ptr, (const float4*)P.sQ.ptr, int(P.n),
                                                        tgtDev, k, nullptr, nullptr, scaleB, 0.0, 1, outDev, nullptr);
      FMM_TRY(launched(P, "kDirect", st));
   }
   FMM_CHECK_LAUNCH();
   return FMM_OK;
}

// New strengths w J for the same source positions, in the tree's sorted order.
template <class T>
__global__ void kRegatherStrengths(const T* __restrict__ xyz, const T* __restrict__ w, const T* __restrict__ J,
                                   const T* __restrict__ sigma, const int* __restrict__ order, int64_t n,
                                   typename Vec4<T>::type* q)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i >= n) return;
   int64_t s = order[i];
   T jx, jy, jz;
   if(J) { jx = J[3 * s]; jy = J[3 * s + 1]; jz = J[3 * s + 2]; }
   else
   {
      const T x = xyz[3 * s], y = xyz[3 * s + 1];
      const T l = sqrt(x * x + y * y);
      jx = l != T(0) ? -y / l : T(0);
      jy = l != T(0) ? x / l : T(0);
      jz = T(0);
   }
   const T ww = w[s];
   q[i] = {ww * jx, ww * jy, ww * jz, sigma ? ww * sigma[s] : T(0)};
}

template <class T>
__global__ void kScaleCopy(const T* __restrict__ src, T* __restrict__ dst, int64_t count, T scale)
{
   int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(i < count) dst[i] = src[i] * scale;
}

template <class T>
fmm_status regatherStrengthsT(Plan& P, cudaStream_t st)
{
   typedef typename Vec4<T>::type V4;
   if(P.n == 0) return FMM_OK;
   kRegatherStrengths<T><<<int((P.n + 255) / 256), 256, 0, st>>>((const T*)P.srcXYZ, (const T*)P.srcW,
                                                                 (const T*)(P.hasJ ? P.srcJ : nullptr),
                                                                 (const T*)(P.bem ? P.srcSigma : nullptr),
                                                                 (const int*)P.sIdx.ptr, P.n, (V4*)P.sQ.ptr);
   FMM_TRY(launched(P, "kRegatherStrengths", st));
   return FMM_OK;
}

template <class T>
fmm_status scaleCopyT(Plan& P, const void* src, void* dst, int64_t count, double scale, cudaStream_t st)
{
   if(count == 0) return FMM_OK;
   kScaleCopy<T><<<int((count + 255) / 256), 256, 0, st>>>((const T*)src, (T*)dst, count, T(scale));
   FMM_TRY(launched(P, "kScaleCopy", st));
   return FMM_OK;
}

template fmm_status regatherStrengthsT<float>(Plan&, cudaStream_t);
template fmm_status regatherStrengthsT<double>(Plan&, cudaStream_t);
template fmm_status scaleCopyT<float>(Plan&, const void*, void*, int64_t, double, cudaStream_t);
template fmm_status scaleCopyT<double>(Plan&, const void*, void*, int64_t, double, cudaStream_t);

template fmm_status upwardT<float>(Plan&, cudaStream_t);
template fmm_status upwardT<double>(Plan&, cudaStream_t);
template fmm_status downwardT<float>(Plan&, cudaStream_t);
template fmm_status downwardT<double>(Plan&, cudaStream_t);
template fmm_status evaluateT<float>(Plan&, double, int, cudaStream_t);
template fmm_status evaluateT<double>(Plan&, double, int, cudaStream_t);
template fmm_status directT<float>(Plan&, double, int, cudaStream_t);
template fmm_status directT<double>(Plan&, double, int, cudaStream_t);

}  // namespace fmm
