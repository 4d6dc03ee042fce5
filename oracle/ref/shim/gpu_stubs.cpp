// Link stubs for the reference's GPU entry points. The oracle build uses only the
// reference's CPU path; reaching any of these aborts loudly. The two index helpers
// and the sign factor are plain host functions the CPU path also calls.
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include "translation_algorithms.hpp"
#include "kernels.cuh"

namespace {
[[noreturn]] void gpuPathUnavailable(const char* what)
{
   std::fprintf(stderr, "reference GPU path '%s' is not built in the oracle\n", what);
   std::abort();
}
}

namespace kernels
{
void translateAllGPU(Vector3*, const real*, const Vector3*, size_t, size_t) { gpuPathUnavailable("translateAllGPU"); }
void translateAllGPUMatrix(Complex*, const Complex*, const Complex*, size_t, size_t)
{ gpuPathUnavailable("translateAllGPUMatrix"); }
void translateAllGPUMatrixCuBLAS(real*, const real*, const real*, size_t, size_t)
{ gpuPathUnavailable("translateAllGPUMatrixCuBLAS"); }
void translateAllGPUMatrixCuBLAS(RealMatrix&, const RealMatrix&, const real*, size_t, size_t)
{ gpuPathUnavailable("translateAllGPUMatrixCuBLAS"); }
size_t lmToIndex(int harmonicBegin, int l, int m) { return harmonicBegin + l * l + l + m; }
size_t lmToIndex(int l, int m) { return l * l + l + m; }
real strangeFactor(int m, int mu) { return std::pow(-1, -0.5 * (std::abs(m) - std::abs(mu) - std::abs(m - mu))); }
}
