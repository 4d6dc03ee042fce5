// extern "C" entry points over the reference FMM (FMM/FMMGPU of iamwhoamianamy/bachelors),
// compiled together with the reference's own translation units by build_ref.sh.
// Test infrastructure only: it exposes the reference's operators and its FastMultipoleSolver
// CPU pipeline to ctypes so that golden vectors can be generated from the reference itself
// and the reference can be timed as the CPU baseline. Every interface takes and returns
// double; the reference computes in its compile-time `real` (float or double).
//
// Reference functions wrapped (paths relative to FMM/FMMGPU/):
//   Harmonics::calcRegularSolidHarmonics / calcIrregularSolidHarmonics   harmonics.cpp:79-125
//   math::calcIntegralContribution (P2M, J = perp(q).normalized())        integration.cpp:137-161
//   MultipoleTranslator::translateMultipoleWithComplex (M2M)              multipole_translator.cpp:111-125
//   MultipoleTranslator::multipoleToLocalWithComplex (M2L, l+lambda<=p)   multipole_translator.cpp:178-193
//   MultipoleTranslator::translateLocalWithComplex (L2L)                  multipole_translator.cpp:234-249
//   mult(local, regular) (A from a local expansion)                       calculation_point_octree.cpp:192-212
//   math::calcBioSavartLaplace (direct sum)                               integration.cpp:101-120
//   kernels::translateAllCPU, translateAllCPUMatrixBLAS                   translation_algorithms_cpu.cpp:9-135
//   Torus (hexahedra -> 5 tetrahedra) + math::tetrahedraToQuadratures     torus.cpp:9-117, integration.cpp:163-187
//   FastMultipoleSolver full B / A pipeline                               fast_multipole_solver.cpp:12-231
//   math::calcBEMIntegral, calcBEMIntegralContribution (BEM problem)     integration.cpp:191-215, 295-353
//   MultipoleSolver treecode B (single source tree, no locals)           multipole_solver.cpp:20-139, 686-700
#include <chrono>
#include <cstdint>
#include <cstring>
#include <array>
#include <unordered_map>
#include <vector>

#include "fast_multipole_solver.hpp"
#include "multipole_solver.hpp"
#include "harmonics.hpp"
#include "integration.hpp"
#include "multipole_translator.hpp"
#include "translation_algorithms.hpp"
#include "torus.hpp"
#include "basis_quadratures.hpp"
#include "bem_quadrature.hpp"

namespace {
HarmonicSeries<Vector3> toSeries(int order, const double* in)
{
   HarmonicSeries<Vector3> s(order);
   for(int k = 0; k < (order + 1) * (order + 1); k++)
      s.getHarmonic(k) = Vector3(real(in[3 * k]), real(in[3 * k + 1]), real(in[3 * k + 2]));
   return s;
}
void fromSeries(const HarmonicSeries<Vector3>& s, double* out)
{
   for(size_t k = 0; k < s.elemCount(); k++)
   {
      out[3 * k] = s.getHarmonic(k).x;
      out[3 * k + 1] = s.getHarmonic(k).y;
      out[3 * k + 2] = s.getHarmonic(k).z;
   }
}
struct KeyHash
{
   size_t operator()(const std::array<real, 3>& a) const
   {
      size_t h = 1469598103934665603ull;
      for(real v : a)
      {
         uint64_t bits = 0;
         std::memcpy(&bits, &v, sizeof(real));
         h = (h ^ bits) * 1099511628211ull;
      }
      return h;
   }
};
// BEM quadratures from rows (x, y, z, weight, Bx, By, Bz, nx, ny, nz).
std::vector<BEMQuadrature> bemQuadratures(int n, const double* q)
{
   std::vector<BEMQuadrature> r;
   r.reserve(n);
   for(int i = 0; i < n; i++)
   {
      const double* e = q + 10 * i;
      r.emplace_back(Vector3(real(e[0]), real(e[1]), real(e[2])), real(1), real(e[3]),
                     Vector3(real(e[4]), real(e[5]), real(e[6])), Vector3(real(e[7]), real(e[8]), real(e[9])));
   }
   return r;
}
double seconds(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b)
{
   return std::chrono::duration<double>(b - a).count();
}
}

extern "C" {

int ref_real_bytes() { return int(sizeof(real)); }

int ref_order() { return FMM_ORDER; }

void ref_regular(int order, const double* xyz, double* out)
{
   auto h = Harmonics::calcRegularSolidHarmonics(order, Vector3(real(xyz[0]), real(xyz[1]), real(xyz[2])));
   for(size_t k = 0; k < h.elemCount(); k++) out[k] = h.getHarmonic(int(k));
}

void ref_irregular(int order, const double* xyz, double* out)
{
   auto h = Harmonics::calcIrregularSolidHarmonics(order, Vector3(real(xyz[0]), real(xyz[1]), real(xyz[2])));
   for(size_t k = 0; k < h.elemCount(); k++) out[k] = h.getHarmonic(int(k));
}

// P2M about `center` of n quadratures (x, y, z, weight); out is (p+1)^2 x 3, AoS [k][xyz].
void ref_p2m(int order, int n, const double* xyzw, const double* center, double* out)
{
   std::vector<Quadrature> q(n);
   for(int i = 0; i < n; i++)
      q[i] = Quadrature(Vector3(real(xyzw[4 * i]), real(xyzw[4 * i + 1]), real(xyzw[4 * i + 2])),
                        real(xyzw[4 * i + 3]), real(1));
   auto res = math::calcIntegralContribution(q, order, Vector3(real(center[0]), real(center[1]), real(center[2])));
   fromSeries(res, out);
}

void ref_m2m(int order, const double* in, const double* t, double* out)
{
   auto res = MultipoleTranslator::translateMultipoleWithComplex(toSeries(order, in),
                                                                Vector3(real(t[0]), real(t[1]), real(t[2])));
   fromSeries(res, out);
}

void ref_m2l(int order, const double* in, const double* t, double* out)
{
   auto res = MultipoleTranslator::multipoleToLocalWithComplex(toSeries(order, in),
                                                              Vector3(real(t[0]), real(t[1]), real(t[2])));
   fromSeries(res, out);
}

void ref_l2l(int order, const double* in, const double* t, double* out)
{
   auto res = MultipoleTranslator::translateLocalWithComplex(toSeries(order, in),
                                                            Vector3(real(t[0]), real(t[1]), real(t[2])));
   fromSeries(res, out);
}

// kernels::translateAllCPU over `count` items: result[i] = M2M of the vector expansion b[i]
// ((order+1)^2 x 3, AoS) by the real regular harmonics a[i] ((order+1)^2).
void ref_translate_all(int count, int order, const double* a, const double* b, double* result)
{
   const size_t L = size_t(order + 1) * (order + 1);
   std::vector<real> ar(L * count);
   std::vector<Vector3> br(L * count), res(L * count);
   for(size_t i = 0; i < L * count; i++)
   {
      ar[i] = real(a[i]);
      br[i] = Vector3(real(b[3 * i]), real(b[3 * i + 1]), real(b[3 * i + 2]));
   }
   kernels::translateAllCPU(res.data(), ar.data(), br.data(), size_t(count), size_t(order));
   for(size_t i = 0; i < L * count; i++)
   {
      result[3 * i] = res[i].x; result[3 * i + 1] = res[i].y; result[3 * i + 2] = res[i].z;
   }
}

// kernels::translateAllCPUMatrixBLAS: column-major C (L x count) = B (L x L) * A (L x count).
void ref_translate_all_matrix(int count, int order, const double* a, const double* b, double* result)
{
   const size_t L = size_t(order + 1) * (order + 1);
   std::vector<real> ar(a, a + L * count), br(b, b + L * L), res(L * count);
   kernels::translateAllCPUMatrixBLAS(res.data(), ar.data(), br.data(), size_t(count), size_t(order));
   for(size_t i = 0; i < L * count; i++) result[i] = res[i];
}

// The reference's tetrahedral torus quadratures (Torus(radius, width, nL, nW, nH) split into
// tetrahedra, each carrying the basis rule read from the two text files): xyzw[4 k], k = number of
// tetrahedra x rule points. Returns k; with out == nullptr only counts.
int ref_torus_quadratures(double radius, double width, int nL, int nW, int nH, const char* ruleX, const char* ruleW,
                          double* out)
{
   Torus torus(real(radius), real(width), nL, nW, nH);
   BasisQuadratures bq;
   bq.initFromTXT(ruleX, ruleW);
   auto q = math::tetrahedraToQuadratures(torus.tetrahedra, bq);
   if(out)
      for(size_t i = 0; i < q.size(); i++)
      {
         out[4 * i] = q[i].x; out[4 * i + 1] = q[i].y; out[4 * i + 2] = q[i].z; out[4 * i + 3] = q[i].weight;
      }
   return int(q.size());
}

// math::calcBEMIntegral at m points over n BEM quadratures (rows as bemQuadratures): out[3m].
void ref_bem_direct(int n, const double* q, int m, const double* pts, double* out)
{
   const std::vector<BEMQuadrature> bq = bemQuadratures(n, q);
   for(int j = 0; j < m; j++)
   {
      Vector3 r = math::calcBEMIntegral(Vector3(real(pts[3 * j]), real(pts[3 * j + 1]), real(pts[3 * j + 2])), bq);
      out[3 * j] = r.x; out[3 * j + 1] = r.y; out[3 * j + 2] = r.z;
   }
}

// math::calcBEMIntegralContribution (the BEM P2M, central differences of the regular harmonics) about
// `center`: out[(p+1)^2][3].
void ref_bem_p2m(int order, int n, const double* q, const double* center, double* out)
{
   std::vector<BEMQuadrature> bq = bemQuadratures(n, q);
   std::vector<Quadrature*> ptrs(n);
   for(int i = 0; i < n; i++) ptrs[i] = &bq[i];
   auto res = math::calcBEMIntegralContribution(ptrs, order, Vector3(real(center[0]), real(center[1]), real(center[2])));
   fromSeries(res, out);
}

// The reference's treecode: MultipoleSolver over n quadratures (x, y, z, weight; J the azimuthal default)
// with leaf capacity `cap`, leaf P2M, complex-translation M2M, then calcB(current, point) at m points:
// out[3m]. The source tree's root is the reference's fixed box (centre 0, half-width 3).
void ref_treecode_B(int n, const double* xyzw, int m, const double* pts, int cap, double current, double* out)
{
   std::vector<Quadrature> q(n);
   for(int i = 0; i < n; i++)
      q[i] = Quadrature(Vector3(real(xyzw[4 * i]), real(xyzw[4 * i + 1]), real(xyzw[4 * i + 2])),
                        real(xyzw[4 * i + 3]), real(1));
   MultipoleSolver solver(q, Problem::BioSavartLaplace, size_t(cap));
   solver.calcMultipoleExpansionsAtLeaves();
   solver.calclMultipoleExpansions(M2MAlg::ComplexTranslation, Device::CPU);
   for(int j = 0; j < m; j++)
   {
      Vector3 b = solver.calcB(real(current), Vector3(real(pts[3 * j]), real(pts[3 * j + 1]), real(pts[3 * j + 2])));
      out[3 * j] = b.x; out[3 * j + 1] = b.y; out[3 * j + 2] = b.z;
   }
}

// A(x) = sum_k local_k * R_k(d), d = x - center (no 1/(4 pi) or current factor).
void ref_eval_local(int order, const double* local, const double* d, double* out3)
{
   auto r = Harmonics::calcRegularSolidHarmonics(order, Vector3(real(d[0]), real(d[1]), real(d[2])));
   Vector3 a = mult(toSeries(order, local), r);
   out3[0] = a.x; out3[1] = a.y; out3[2] = a.z;
}

// Direct Biot-Savart B at m points from n quadratures (x, y, z, weight), J = perp(q).normalized().
void ref_direct_B(int n, const double* xyzw, int m, const double* pts, double current, double* outB)
{
   std::vector<Quadrature> q(n);
   for(int i = 0; i < n; i++)
      q[i] = Quadrature(Vector3(real(xyzw[4 * i]), real(xyzw[4 * i + 1]), real(xyzw[4 * i + 2])),
                        real(xyzw[4 * i + 3]), real(1));
#pragma omp parallel for schedule(dynamic, 16)
   for(int j = 0; j < m; j++)
   {
      Vector3 b = math::calcBioSavartLaplace(real(current), Vector3(real(pts[3 * j]), real(pts[3 * j + 1]),
                                                                    real(pts[3 * j + 2])), q);
      outB[3 * j] = b.x; outB[3 * j + 1] = b.y; outB[3 * j + 2] = b.z;
   }
}

// The reference's production FMM pipeline (Matrices M2M on the CPU, complex M2L and L2L,
// finite-difference curl). Results are returned in input order. times[0..4] receive the
// seconds spent in: trees, P2M, M2M, lists+M2L+L2L, evaluation. Returns the number of
// targets the reference produced a value for (all of them unless it dropped some).
int ref_fmm(int n, const double* xyzw, int m, const double* pts, int capS, int capT, double current,
            int wantB, double* out, double* times)
{
   std::vector<Quadrature> q(n);
   for(int i = 0; i < n; i++)
      q[i] = Quadrature(Vector3(real(xyzw[4 * i]), real(xyzw[4 * i + 1]), real(xyzw[4 * i + 2])),
                        real(xyzw[4 * i + 3]), real(1));
   std::vector<Vector3> p(m);
   std::unordered_map<std::array<real, 3>, int, KeyHash> index;
   index.reserve(size_t(m) * 2);
   for(int j = 0; j < m; j++)
   {
      p[j] = Vector3(real(pts[3 * j]), real(pts[3 * j + 1]), real(pts[3 * j + 2]));
      index[{p[j].x, p[j].y, p[j].z}] = j;
   }
   auto t0 = std::chrono::steady_clock::now();
   FastMultipoleSolver solver(q, p, Problem::BioSavartLaplace, size_t(capS), size_t(capT));
   auto t1 = std::chrono::steady_clock::now();
   solver.calcMultipoleExpansionsAtLeaves();
   auto t2 = std::chrono::steady_clock::now();
   solver.calclMultipoleExpansions(M2MAlg::Matrices, Device::CPU);
   auto t3 = std::chrono::steady_clock::now();
   solver.calcLocalMultipoleExpansions(M2LAlg::ComplexTranslation, Device::CPU);
   auto t4 = std::chrono::steady_clock::now();
   auto res = wantB ? solver.calcB(real(current)) : solver.calcA(real(current));
   auto t5 = std::chrono::steady_clock::now();
   if(times)
   {
      times[0] = seconds(t0, t1); times[1] = seconds(t1, t2); times[2] = seconds(t2, t3);
      times[3] = seconds(t3, t4); times[4] = seconds(t4, t5);
   }
   int found = 0;
   for(auto& [pt, v] : res)
   {
      auto it = index.find({pt.x, pt.y, pt.z});
      if(it == index.end()) continue;
      int j = it->second;
      out[3 * j] = v.x; out[3 * j + 1] = v.y; out[3 * j + 2] = v.z;
      found++;
   }
   return found;
}

}
