/*
 * fmm_facade.hpp: header-only C++ facade over the C ABI (fmmcuda.h) that keeps the reference's
 * C++ names and signatures, so that code written against iamwhoamianamy/bachelors links against
 * libfmmcuda.so after swapping includes:
 *
 *   Vector3, Quadrature, real                 FMM/FMMGPU/vector3.cuh:8-57, quadrature.hpp:4-10, real.hpp
 *   Problem, M2MAlg, Device, M2LAlg           FMM/FMMGPU/multipole_solver_enums.hpp:3-30
 *   MultipoleSolver                           FMM/FMMGPU/multipole_solver.hpp:12-48
 *   FastMultipoleSolver                       FMM/FMMGPU/fast_multipole_solver.hpp:13-49
 *   math::calcBioSavartLaplace                FMM/FMMGPU/integration.hpp:46-49
 *   kernels::addVectors, kernels::translateAll*   FMMCUDADLL/kernel_callers.hpp:5-10,
 *                                             FMM/FMMGPU/translation_algorithms.hpp:8-61
 *
 * `real` is float unless FMM_REAL_IS_DOUBLE is defined (the reference's REAL_IS_FLOAT /
 * REAL_IS_DOUBLE switch). Differences a caller sees:
 *   - the algorithm and device enums are accepted and ignored (one GPU algorithm);
 *   - calcA / calcB(current) return (point, value) pairs in the caller's point order, not tree order;
 *   - errors throw std::runtime_error carrying fmm_last_error_string(); nothing exits the process;
 *   - the expansion order is a constructor argument (default 10, the reference's harmonicOrder);
 *   - leaf capacities keep the reference's meaning "a box holding this many points splits": the plan's
 *     leaves hold at most capacity - 1 points;
 *   - MultipoleSolver::calcA / calcB(current, point) (the reference's single-tree treecode,
 *     multipole_solver.cpp:686-700) run the device treecode (fmm_treecode) on the plan's tree and
 *     multipoles: the reference's acceptance test, with close leaves summed directly and B from the analytic
 *     curl (treecodeFlags = FMM_TREECODE_REFERENCE_NEAR | FMM_TREECODE_FD_CURL gives the reference's
 *     choices); the root cube is the sources' bounding cube unless config() sets one (the reference's is
 *     centre 0, half-width 3, and drops sources outside it);
 *   - Problem::BEM takes BEMQuadrature sources (fmm_set_bem_sources); FastMultipoleSolver::calcBEM sums close
 *     boxes directly (the reference drops close leaves) and the tree's root is a cube around the sources
 *     (the reference's BEM root is the box of half-widths 1.1, 1.1, 1.6 at the origin);
 * The solvers keep references to the caller's vectors, as the reference does
 * (multipole_solver.cpp:27-32, fast_multipole_solver.hpp:16): they must outlive the solver. The
 * data is copied to the GPU when the first phase runs.
 *
 * Define FMM_FACADE_NO_GLOBAL_NAMES to keep everything inside namespace fmm (by default the
 * reference's global names Vector3, Quadrature, real, MultipoleSolver, FastMultipoleSolver,
 * Problem, M2MAlg, Device, M2LAlg, BEMQuadrature and the Basic* solver templates are also declared at global
 * scope).
 */
#ifndef FMM_FACADE_HPP
#define FMM_FACADE_HPP

#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fmmcuda.h"

namespace fmm {

#ifdef FMM_REAL_IS_DOUBLE
typedef double real;
constexpr int kRealPrecision = FMM_FP64;
#else
typedef float real;
constexpr int kRealPrecision = FMM_FP32;
#endif

inline void check(fmm_status s)
{
   if(s != FMM_OK) throw std::runtime_error(std::string("fmmcuda: ") + fmm_last_error_string());
}

struct Vector3
{
   real x, y, z;

   Vector3(real x_ = 0, real y_ = 0, real z_ = 0) : x(x_), y(y_), z(z_) {}
   real& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
   real operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
   Vector3 operator+(const Vector3& r) const { return Vector3(x + r.x, y + r.y, z + r.z); }
   Vector3 operator-(const Vector3& r) const { return Vector3(x - r.x, y - r.y, z - r.z); }
   Vector3 operator*(real f) const { return Vector3(x * f, y * f, z * f); }
   Vector3 operator/(real f) const { return Vector3(x / f, y / f, z / f); }
   Vector3& operator+=(const Vector3& r) { x += r.x; y += r.y; z += r.z; return *this; }
   Vector3& operator-=(const Vector3& r) { x -= r.x; y -= r.y; z -= r.z; return *this; }
   Vector3& operator*=(real f) { x *= f; y *= f; z *= f; return *this; }
   Vector3& operator/=(real f) { x /= f; y /= f; z /= f; return *this; }
   real lengthSquared() const { return x * x + y * y + z * z; }
   real length() const { return std::sqrt(lengthSquared()); }
   Vector3 normalized() const { real l = length(); return l > 0 ? *this / l : Vector3(); }
   void normalize() { *this = normalized(); }
   /* (-y, x, 0): the azimuthal direction the reference uses for coil currents (vector3.cu:201-204) */
   Vector3 perp() const { return Vector3(-y, x, 0); }
   static real dot(const Vector3& a, const Vector3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
   static Vector3 cross(const Vector3& a, const Vector3& b)
   {
      return Vector3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
   }
   static real distanceSquared(const Vector3& a, const Vector3& b) { return (a - b).lengthSquared(); }
   static Vector3 xAxis() { return Vector3(1, 0, 0); }
   static Vector3 yAxis() { return Vector3(0, 1, 0); }
   static Vector3 zAxis() { return Vector3(0, 0, 1); }
};

/* A point with its integration weight; weight = volume * rule weight (quadrature.cpp:7-11). */
struct Quadrature : public Vector3
{
   real weight = 0;
   Quadrature() = default;
   Quadrature(const Vector3& coordinates, real volume, real w) : Vector3(coordinates), weight(volume * w) {}
};

/* A surface quadrature of the BEM problem (bem_quadrature.hpp): point, weight, field value and normal. */
struct BEMQuadrature : public Quadrature
{
   Vector3 B;
   Vector3 normal;
   BEMQuadrature() = default;
   BEMQuadrature(const Vector3& coordinates, real area, real w, const Vector3& B_, const Vector3& normal_)
      : Quadrature(coordinates, area, w), B(B_), normal(normal_)
   {
   }
};

enum class Problem { BioSavartLaplace = 0, BEM = 1 };
enum class M2MAlg { NoTranslation = 0, ComplexTranslation, RealTranslation, Layers, Matrices };
enum class Device { CPU = 0, GPU, Adaptive };
enum class M2LAlg { ComplexTranslation = 0, Matrices };

namespace detail {

/* Owns one fmm_plan. */
class PlanHandle
{
public:
   fmm_config cfg;
   fmm_plan* plan = nullptr;
   PlanHandle() { fmm_default_config(&cfg); cfg.precision = kRealPrecision; }
   ~PlanHandle() { reset(); }
   PlanHandle(const PlanHandle&) = delete;
   PlanHandle& operator=(const PlanHandle&) = delete;
   void reset()
   {
      if(plan) fmm_plan_destroy(plan);
      plan = nullptr;
   }
   fmm_plan* get()
   {
      if(!plan) check(fmm_plan_create(&cfg, &plan));
      return plan;
   }
};

template <class Q>
void packSources(const std::vector<Q>& q, std::vector<real>& xyz, std::vector<real>& w)
{
   xyz.resize(3 * q.size());
   w.resize(q.size());
   for(size_t i = 0; i < q.size(); i++)
   {
      xyz[3 * i] = q[i].x;
      xyz[3 * i + 1] = q[i].y;
      xyz[3 * i + 2] = q[i].z;
      w[i] = q[i].weight;
   }
}

/* BEM sources: only BEMQuadrature carries a field value and a normal. */
inline void setBemSources(fmm_plan* plan, const std::vector<BEMQuadrature>& q)
{
   std::vector<real> xyz(3 * q.size()), w(q.size()), B(3 * q.size()), n(3 * q.size());
   for(size_t i = 0; i < q.size(); i++)
   {
      for(int d = 0; d < 3; d++)
      {
         xyz[3 * i + d] = q[i][d];
         B[3 * i + d] = q[i].B[d];
         n[3 * i + d] = q[i].normal[d];
      }
      w[i] = q[i].weight;
   }
   check(fmm_set_bem_sources(plan, xyz.data(), w.data(), B.data(), n.data(), int64_t(q.size()), 0, nullptr));
}
template <class Q>
void setBemSources(fmm_plan*, const std::vector<Q>&)
{
   throw std::invalid_argument("fmm facade: Problem::BEM needs BEMQuadrature sources");
}

template <class P>
void packPoints(const P* p, size_t n, std::vector<real>& xyz)
{
   xyz.resize(3 * n);
   for(size_t i = 0; i < n; i++)
   {
      xyz[3 * i] = p[i].x;
      xyz[3 * i + 1] = p[i].y;
      xyz[3 * i + 2] = p[i].z;
   }
}

inline int leafCapacity(size_t referenceCapacity)
{
   return referenceCapacity > 1 ? int(referenceCapacity - 1) : 1;
}

}  // namespace detail

/* MultipoleSolver (multipole_solver.hpp:12-48): sources only; point queries. */
template <class QuadratureT = Quadrature, class PointT = Vector3>
class BasicMultipoleSolver
{
protected:
   std::vector<QuadratureT>& _quadratures;
   Problem _problem;
   detail::PlanHandle _plan;
   bool _sourcesUploaded = false;
   bool _multipolesAtLeavesAreReady = false;
   bool _multipolesAreReady = false;
   bool _upwardDone = false;   // the plan holds the tree and multipoles the treecode walks

public:
   bool log = false;
   int treecodeFlags = 0;      // fmm_treecode flags of calcA / calcB(current, point)
   const int harmonicOrder;
   const int harmonicLength;
   const size_t quadratureOctreeLeafCapacity;

   BasicMultipoleSolver(std::vector<QuadratureT>& quadratures, Problem problem = Problem::BioSavartLaplace,
                        size_t quadratureOctreeLeafCapacity_ = 1000, int order = 10)
      : _quadratures(quadratures), _problem(problem), harmonicOrder(order),
        harmonicLength((order + 1) * (order + 1)), quadratureOctreeLeafCapacity(quadratureOctreeLeafCapacity_)
   {
      _plan.cfg.order = order;
      _plan.cfg.leaf_capacity = detail::leafCapacity(quadratureOctreeLeafCapacity_);
   }
   virtual ~BasicMultipoleSolver() = default;

   /* The plan's configuration; changes take effect before the first phase runs
      (e.g. m2l_mode = FMM_M2L_BF16X3 for the tensor-core M2L of FP32 plans). */
   fmm_config& config() { return _plan.cfg; }
   fmm_plan* plan() { return _plan.get(); }

   virtual void calcMultipoleExpansionsAtLeaves() { _multipolesAtLeavesAreReady = true; }

   virtual void calclMultipoleExpansions(M2MAlg, Device = Device::CPU)
   {
      if(!_multipolesAtLeavesAreReady) throw std::runtime_error("Multipoles at leaves are not ready!");
      _multipolesAreReady = true;
   }

   virtual PointT calcA(real current, const PointT& point) { return pointQuery(current, point, 2); }
   virtual PointT calcB(real current, const PointT& point)
   {
      if(_problem == Problem::BEM) throw std::invalid_argument("fmm facade: a BEM solver evaluates calcA");
      return pointQuery(current, point, 1);
   }

   fmm_stats stats()
   {
      fmm_stats s{};
      check(fmm_get_stats(_plan.get(), &s));
      return s;
   }

protected:
   void uploadSources()
   {
      if(_sourcesUploaded) return;
      _sourcesUploaded = true;
      if(_problem == Problem::BEM)
      {
         detail::setBemSources(_plan.get(), _quadratures);
         return;
      }
      std::vector<real> xyz, w;
      detail::packSources(_quadratures, xyz, w);
      check(fmm_set_sources(_plan.get(), xyz.data(), w.data(), nullptr, int64_t(_quadratures.size()), 0, nullptr));
   }

   PointT pointQuery(real current, const PointT& point, int want)
   {
      if(!_multipolesAreReady) throw std::runtime_error("Multipoles are not ready!");
      if(!_upwardDone)
      {
         uploadSources();
         check(fmm_build_tree(_plan.get(), nullptr));
         check(fmm_upward(_plan.get(), nullptr));
         _upwardDone = true;
      }
      real xyz[3] = {point.x, point.y, point.z};
      real out[3];
      check(fmm_treecode(_plan.get(), double(current), want, xyz, 1, want == 1 ? out : nullptr,
                         want == 2 ? out : nullptr, treecodeFlags, 0, nullptr));
      PointT r;
      r.x = out[0];
      r.y = out[1];
      r.z = out[2];
      return r;
   }
};

/* FastMultipoleSolver (fast_multipole_solver.hpp:13-49): sources and target points; the reference's
   phases map to the plan's: calcMultipoleExpansionsAtLeaves -> fmm_build_tree + fmm_upward (P2M and
   M2M), calclMultipoleExpansions -> (done), calcLocalMultipoleExpansions -> fmm_downward (M2L, L2L),
   calcA / calcB(current) -> fmm_evaluate (L2P and the near field). */
template <class QuadratureT = Quadrature, class PointT = Vector3>
class BasicFastMultipoleSolver : public BasicMultipoleSolver<QuadratureT, PointT>
{
   typedef BasicMultipoleSolver<QuadratureT, PointT> Base;
   std::vector<PointT>& _points;
   bool _localMultipolesAreInitialized = false;
   bool _uploaded = false;

public:
   const size_t calculationPointOctreeLeafCapacity;

   BasicFastMultipoleSolver(std::vector<QuadratureT>& quadratures, std::vector<PointT>& points,
                            Problem problem = Problem::BioSavartLaplace, size_t quadratureOctreeLeafCapacity_ = 1000,
                            size_t calculationPointOctreeLeafCapacity_ = 100, int order = 10)
      : Base(quadratures, problem, quadratureOctreeLeafCapacity_, order), _points(points),
        calculationPointOctreeLeafCapacity(calculationPointOctreeLeafCapacity_)
   {
      this->_plan.cfg.target_leaf_capacity = detail::leafCapacity(calculationPointOctreeLeafCapacity_);
   }

   void calcMultipoleExpansionsAtLeaves() override
   {
      upload();
      check(fmm_build_tree(this->_plan.get(), nullptr));
      check(fmm_upward(this->_plan.get(), nullptr));
      this->_multipolesAtLeavesAreReady = true;
      this->_upwardDone = true;
   }

   void calcLocalMultipoleExpansions(M2LAlg, Device = Device::CPU)
   {
      if(!this->_multipolesAreReady) throw std::runtime_error("Multipoles are not ready!");
      check(fmm_downward(this->_plan.get(), nullptr));
      _localMultipolesAreInitialized = true;
   }

   using Base::calcA;
   using Base::calcB;
   virtual std::vector<std::pair<PointT, PointT>> calcA(real current) { return evaluate(current, 2); }
   virtual std::vector<std::pair<PointT, PointT>> calcB(real current) { return evaluate(current, 1); }
   /* calcBEM(current) (fast_multipole_solver.cpp:233-250): the BEM integral at the points, no current factor */
   virtual std::vector<std::pair<PointT, PointT>> calcBEM(real current)
   {
      if(this->_problem != Problem::BEM) throw std::invalid_argument("fmm facade: calcBEM needs Problem::BEM");
      (void)current;
      return evaluate(real(1), 2);
   }

private:
   void upload()
   {
      if(_uploaded) return;
      this->uploadSources();
      std::vector<real> xyz;
      detail::packPoints(_points.data(), _points.size(), xyz);
      check(fmm_set_targets(this->_plan.get(), xyz.data(), int64_t(_points.size()), 0, nullptr));
      _uploaded = true;
   }

   std::vector<std::pair<PointT, PointT>> evaluate(real current, int want)
   {
      if(!_localMultipolesAreInitialized) throw std::runtime_error("Local multipoles are not ready!");
      std::vector<real> out(3 * _points.size());
      check(fmm_evaluate(this->_plan.get(), double(current), want, want == 1 ? out.data() : nullptr,
                         want == 2 ? out.data() : nullptr, 0, nullptr));
      std::vector<std::pair<PointT, PointT>> res(_points.size());
      for(size_t i = 0; i < _points.size(); i++)
      {
         res[i].first = _points[i];
         res[i].second.x = out[3 * i];
         res[i].second.y = out[3 * i + 1];
         res[i].second.z = out[3 * i + 2];
      }
      return res;
   }
};

typedef BasicMultipoleSolver<> MultipoleSolver;
typedef BasicFastMultipoleSolver<> FastMultipoleSolver;

}  // namespace fmm

namespace math {

/* Direct Biot-Savart B at `point` from the quadratures with the azimuthal current direction
   (integration.cpp:101-111), on the GPU in `real` precision. */
template <class QuadratureT>
fmm::Vector3 calcBioSavartLaplace(fmm::real current, const fmm::Vector3& point, std::vector<QuadratureT>& quadratures)
{
   fmm::detail::PlanHandle h;
   std::vector<fmm::real> xyz, w;
   fmm::detail::packSources(quadratures, xyz, w);
   fmm::check(fmm_set_sources(h.get(), xyz.data(), w.data(), nullptr, int64_t(quadratures.size()), 0, nullptr));
   fmm::real p[3] = {point.x, point.y, point.z}, out[3];
   fmm::check(fmm_set_targets(h.get(), p, 1, 0, nullptr));
   fmm::check(fmm_direct(h.get(), double(current), 1, out, nullptr, 0, nullptr));
   return fmm::Vector3(out[0], out[1], out[2]);
}

}  // namespace math

namespace kernels {

typedef fmm::real real;
typedef std::vector<std::vector<real>> RealMatrix;
/* cuComplex / cuDoubleComplex layout */
struct Complex
{
   real x, y;
};

/* FMMCUDADLL/kernel_callers.hpp:7-9 */
inline std::vector<real> addVectors(const std::vector<real>& a, const std::vector<real>& b)
{
   if(a.size() != b.size()) throw std::invalid_argument("addVectors: sizes differ");
   std::vector<float> af(a.begin(), a.end()), bf(b.begin(), b.end()), cf(a.size());
   fmm::check(fmm_add_vectors(af.data(), bf.data(), cf.data(), int64_t(a.size())));
   return std::vector<real>(cf.begin(), cf.end());
}

/* translation_algorithms.hpp:13-25 */
inline void translateAllGPU(fmm::Vector3* result, const real* a, const fmm::Vector3* b, size_t harmonicCount,
                            size_t harmonicOrder)
{
   static_assert(sizeof(fmm::Vector3) == 3 * sizeof(real), "Vector3 must be three packed reals");
   fmm::check(fmm_translate_all(result, a, b, int64_t(harmonicCount), int(harmonicOrder), fmm::kRealPrecision, 0,
                                nullptr));
}
inline void translateAllCPU(fmm::Vector3* result, const real* a, const fmm::Vector3* b, size_t harmonicCount,
                            size_t harmonicOrder)
{
   translateAllGPU(result, a, b, harmonicCount, harmonicOrder);
}

/* translation_algorithms.hpp:41-61: column-major C (L x count) = B (L x L) * A (L x count) */
inline void translateAllGPUMatrixCuBLAS(real* result, const real* a, const real* b, size_t harmonicCount,
                                        size_t harmonicOrder)
{
   fmm::check(fmm_translate_all_matrix(result, a, b, int64_t(harmonicCount), int(harmonicOrder), 1,
                                       fmm::kRealPrecision, 0, nullptr));
}
inline void translateAllCPUMatrixBLAS(real* result, const real* a, const real* b, size_t harmonicCount,
                                      size_t harmonicOrder)
{
   translateAllGPUMatrixCuBLAS(result, a, b, harmonicCount, harmonicOrder);
}
/* The three-component overload: result[c] = B * a[c], c = 0..2. */
inline void translateAllGPUMatrixCuBLAS(RealMatrix& result, const RealMatrix& a, const real* b, size_t harmonicCount,
                                        size_t harmonicOrder)
{
   const size_t L = (harmonicOrder + 1) * (harmonicOrder + 1);
   const size_t n = harmonicCount * L;
   std::vector<real> in(a.size() * n), out(a.size() * n);
   for(size_t c = 0; c < a.size(); c++)
   {
      if(a[c].size() < n) throw std::invalid_argument("translateAllGPUMatrixCuBLAS: component shorter than count x L");
      std::copy(a[c].begin(), a[c].begin() + n, in.begin() + c * n);
   }
   fmm::check(fmm_translate_all_matrix(out.data(), in.data(), b, int64_t(harmonicCount), int(harmonicOrder),
                                       int64_t(a.size()), fmm::kRealPrecision, 0, nullptr));
   result.resize(a.size());
   for(size_t c = 0; c < a.size(); c++) result[c].assign(out.begin() + c * n, out.begin() + (c + 1) * n);
}

/* translation_algorithms.hpp:27-39: complex result (count x L) = a (count x L) * b (L x L), row-major */
inline void translateAllGPUMatrix(Complex* result, const Complex* a, const Complex* b, size_t harmonicCount,
                                  size_t harmonicOrder)
{
   fmm::check(fmm_translate_all_matrix_complex(result, a, b, int64_t(harmonicCount), int(harmonicOrder),
                                               fmm::kRealPrecision, 0, nullptr));
}
inline void translateAllCPUMatrix(std::vector<Complex>& result, const std::vector<Complex>& a,
                                  const std::vector<Complex>& b, size_t harmonicCount, size_t harmonicOrder)
{
   const size_t L = (harmonicOrder + 1) * (harmonicOrder + 1);
   if(a.size() < harmonicCount * L || b.size() < L * L) throw std::invalid_argument("translateAllCPUMatrix: sizes");
   result.resize(harmonicCount * L);
   translateAllGPUMatrix(result.data(), a.data(), b.data(), harmonicCount, harmonicOrder);
}

}  // namespace kernels

#ifndef FMM_FACADE_NO_GLOBAL_NAMES
using fmm::BasicFastMultipoleSolver;
using fmm::BasicMultipoleSolver;
using fmm::BEMQuadrature;
using fmm::FastMultipoleSolver;
using fmm::M2LAlg;
using fmm::M2MAlg;
using fmm::MultipoleSolver;
using fmm::Problem;
using fmm::Quadrature;
using fmm::real;
using fmm::Vector3;
using fmm::Device;
#endif

#endif /* FMM_FACADE_HPP */
