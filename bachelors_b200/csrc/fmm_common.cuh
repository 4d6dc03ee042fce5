// Shared device-side definitions of the B200 FMM: constants, node layout, solid-harmonic
// recurrences and small helpers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fmm {

constexpr int MAXLEVEL = 21;          // Morton depth (21 bits per axis in a 63-bit key)
constexpr int MAXORDER = 16;          // largest expansion order p
constexpr int NOFF = 343;             // offsets in [-3,3]^3; 316 of them are M2L offsets
constexpr int COLCAP = 27;            // same-level adjacent nodes (incl. self)
constexpr int ACAP = 32;              // coarser adjacent leaves (at most 26 by geometry)
constexpr int XCAP = 64;              // coarser non-adjacent leaves (at most 53)

// The reference's literals (FMM/FMMGPU/math.hpp:12-13).
constexpr double REF_PI = 3.14159265359;
constexpr double REF_MU0 = 1.2566370614e-6;

__host__ __device__ constexpr int nharm(int p) { return (p + 1) * (p + 1); }
__host__ __device__ constexpr int hidx(int l, int m) { return l * l + l + m; }
// Coefficient rows are padded to a multiple of 16 elements (bf16 MMA K-steps and 16-byte rows).
__host__ __device__ constexpr int padded(int L) { return (L + 15) & ~15; }
__host__ __device__ inline int offsetIndex(int ox, int oy, int oz) { return (ox + 3) + 7 * (oy + 3) + 49 * (oz + 3); }

// Device forest, structure of arrays. Level-0 nodes are the roots, one per coil (independent
// problem); nodes are numbered level by level, by key within a level; children of a node are
// contiguous. A node's key is (coil << 3 level) | (its Morton path below the root).
struct Tree
{
   int64_t nNodes;
   int nLevels;                 // levels 0..nLevels-1 are populated
   int levelStart[MAXLEVEL + 2];
   // per node
   uint64_t* key;
   int* level;
   int* ix; int* iy; int* iz;
   int* s0; int* s1; int* t0; int* t1;
   int* parent;
   int* child0;
   int* nchild;
};

// Root (coil) index of a node.
__device__ __forceinline__ int rootOf(const Tree& t, int node)
{
   return int(t.key[node] >> (3 * t.level[node]));
}

// ---------------------------------------------------------------------------------------
// Solid harmonics by Cartesian recurrence (no square roots or divisions by r).
//
// For m >= 0 the complex regular harmonic S_l^m = r^l P_l^m(cos t) e^{i m f} / (l + m)!
// (P_l^m without the Condon-Shortley phase) satisfies
//   S_0^0 = 1,  S_m^m = S_{m-1}^{m-1} (x + i y) / (2m),  S_{m+1}^m = z S_m^m,
//   S_{l+1}^m = ((2l + 1) z S_l^m - r^2 S_{l-1}^m) / ((l - m + 1)(l + m + 1)).
// The reference's real regular harmonics (FMM/FMMGPU/harmonics.cpp:79-199) are
//   R_l^0 = (-1)^l S_l^0,  R_l^m = (-1)^l sqrt2 Re S_l^m,  R_l^-m = (-1)^l sqrt2 Im S_l^m.
// The irregular T_l^m = (l - m)! P_l^m(cos t) e^{i m f} / r^{l+1} satisfies
//   T_0^0 = 1/r,  T_m^m = (2m - 1)(x + i y) T_{m-1}^{m-1} / r^2,  T_{m+1}^m = (2m + 1) z T_m^m / r^2,
//   T_{l+1}^m = ((2l + 1) z T_l^m - (l + m)(l - m) T_{l-1}^m) / r^2,
// and I_l^{0,m,-m} follow with the same (-1)^l sqrt2 Re / Im factors.
//
// visitRegular walks (m, l) with m outer and l inner, holding O(1) state, and calls
// f(l, m, re, im) with the complex S_l^m; callers apply the real-basis factors.
// ---------------------------------------------------------------------------------------
template <class T, class F>
__device__ __forceinline__ void visitRegular(int p, T x, T y, T z, F&& f)
{
   const T r2 = x * x + y * y + z * z;
   T dre = T(1), dim = T(0);  // S_m^m
   for(int m = 0; m <= p; m++)
   {
      if(m > 0)
      {
         const T s = T(1) / T(2 * m);
         const T nre = (dre * x - dim * y) * s;
         const T nim = (dre * y + dim * x) * s;
         dre = nre; dim = nim;
      }
      T are = dre, aim = dim;   // S_l^m
      T bre = T(0), bim = T(0); // S_{l-1}^m
      f(m, m, are, aim);
      for(int l = m; l < p; l++)
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
         f(l + 1, m, are, aim);
      }
   }
}

// Fills out[(p+1)^2] with the real regular harmonics R_k(x, y, z) (standard convention).
template <class T>
__device__ inline void realRegular(int p, T x, T y, T z, T* out)
{
   const T sq2 = T(1.4142135623730950488);
   visitRegular<T>(p, x, y, z, [&](int l, int m, T re, T im) {
      const T s = (l & 1) ? T(-1) : T(1);
      if(m == 0) out[hidx(l, 0)] = s * re;
      else { out[hidx(l, m)] = s * sq2 * re; out[hidx(l, -m)] = s * sq2 * im; }
   });
}

// Fills out[(q+1)^2] with the real irregular harmonics I_k(x, y, z) up to order q.
template <class T>
__device__ inline void realIrregular(int q, T x, T y, T z, T* out)
{
   const T sq2 = T(1.4142135623730950488);
   const T r2 = x * x + y * y + z * z;
   const T ir2 = T(1) / r2;
   T dre = T(1) / sqrt(r2), dim = T(0);  // T_m^m
   for(int m = 0; m <= q; m++)
   {
      if(m > 0)
      {
         const T s = T(2 * m - 1) * ir2;
         const T nre = (dre * x - dim * y) * s;
         const T nim = (dre * y + dim * x) * s;
         dre = nre; dim = nim;
      }
      T are = dre, aim = dim, bre = T(0), bim = T(0);
      for(int l = m; l <= q; l++)
      {
         const T s = (l & 1) ? T(-1) : T(1);
         if(m == 0) out[hidx(l, 0)] = s * are;
         else { out[hidx(l, m)] = s * sq2 * are; out[hidx(l, -m)] = s * sq2 * aim; }
         if(l == q) break;
         T cre, cim;
         if(l == m) { cre = T(2 * m + 1) * z * are * ir2; cim = T(2 * m + 1) * z * aim * ir2; }
         else
         {
            const T c = T((l + m) * (l - m));
            cre = (T(2 * l + 1) * z * are - c * bre) * ir2;
            cim = (T(2 * l + 1) * z * aim - c * bim) * ir2;
         }
         bre = are; bim = aim; are = cre; aim = cim;
      }
   }
}

template <class T> struct Vec4;
template <> struct Vec4<float> { typedef float4 type; };
template <> struct Vec4<double> { typedef double4 type; };

}  // namespace fmm
