// Quadrature sources generated on the device from the reference's tetrahedral torus mesh.
//
// The reference builds its coil on the host: Torus::buildHexahedra cuts a torus of square cross-section
// into n_length x n_width x n_height hexahedra and each hexahedron into five tetrahedra
// (FMM/FMMGPU/torus.cpp:52-117), and math::tetrahedraToQuadratures maps a basis rule on the unit
// tetrahedron into each of them (integration.cpp:34-42, 163-187). Here one thread per (tetrahedron,
// rule point) computes its hexahedron's corners, the tetrahedron, its volume and the mapped point in
// FP64 and writes the point and its weight straight into device memory, tetrahedron-major, so that a
// coil of any resolution goes to the solver without a host round trip.
#include "fmm_internal.cuh"

namespace fmm {

namespace {

constexpr int MAXRULE = 64;

struct Rule
{
   int k;
   double x[MAXRULE][3];
   double w[MAXRULE];
};

template <class T>
__global__ void kTorusQuadratures(double radius, double width, int nL, int nW, int nH, Rule rule, int64_t total,
                                  T* __restrict__ xyz, T* __restrict__ w)
{
   const int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
   if(e >= total) return;
   const int q = int(e % rule.k);
   const int64_t tet = e / rule.k;
   const int s = int(tet % 5);
   const int64_t hex = tet / 5;
   const int k = int(hex % nH), j = int((hex / nH) % nW), i = int(hex / (int64_t(nH) * nW));
   // torus.cpp:52-101: the step angle in degrees with the reference's PI literal, the inner radius, the
   // corners of hexahedron (i, j, k) on the rays at angles i and i + 1
   const double step = 360.0 / nL * REF_PI / 180.0;
   const double rIn = radius - width / 2.0;
   const double bottom = -width / 2.0, dz = width / nH, dw = width / nW;
   const double a0x = rIn * cos(step * i), a0y = rIn * sin(step * i);
   const double a1x = rIn * cos(step * (i + 1)), a1y = rIn * sin(step * (i + 1));
   const double l0 = sqrt(a0x * a0x + a0y * a0y), l1 = sqrt(a1x * a1x + a1y * a1y);
   const double u0x = a0x / l0, u0y = a0y / l0, u1x = a1x / l1, u1y = a1y / l1;
   const double zb = bottom + dz * k, zt = bottom + dz * (k + 1);
   double P[8][3];
   const double rx[2] = {a0x + u0x * dw * j, a0x + u0x * dw * (j + 1)};
   const double ry[2] = {a0y + u0y * dw * j, a0y + u0y * dw * (j + 1)};
   const double lx[2] = {a1x + u1x * dw * j, a1x + u1x * dw * (j + 1)};
   const double ly[2] = {a1y + u1y * dw * j, a1y + u1y * dw * (j + 1)};
   for(int h = 0; h < 2; h++)
   {
      const double zz = h ? zt : zb;
      P[4 * h + 0][0] = rx[0]; P[4 * h + 0][1] = ry[0]; P[4 * h + 0][2] = zz;   // right
      P[4 * h + 1][0] = rx[1]; P[4 * h + 1][1] = ry[1]; P[4 * h + 1][2] = zz;   // next right
      P[4 * h + 2][0] = lx[0]; P[4 * h + 2][1] = ly[0]; P[4 * h + 2][2] = zz;   // left
      P[4 * h + 3][0] = lx[1]; P[4 * h + 3][1] = ly[1]; P[4 * h + 3][2] = zz;   // next left
   }
   // the five tetrahedra of a hexahedron (torus.cpp:103-117)
   const int split[5][4] = {{0, 1, 3, 5}, {0, 3, 5, 6}, {0, 2, 3, 6}, {0, 4, 5, 6}, {3, 5, 6, 7}};
   const double* a = P[split[s][0]];
   const double* b = P[split[s][1]];
   const double* c = P[split[s][2]];
   const double* d = P[split[s][3]];
   // volume |(a - d) . ((b - d) x (c - d))| / 6 and x = a + (b - a) u + (c - a) v + (d - a) w
   const double ad[3] = {a[0] - d[0], a[1] - d[1], a[2] - d[2]};
   const double bd[3] = {b[0] - d[0], b[1] - d[1], b[2] - d[2]};
   const double cd[3] = {c[0] - d[0], c[1] - d[1], c[2] - d[2]};
   const double vol = fabs(ad[0] * (bd[1] * cd[2] - bd[2] * cd[1]) + ad[1] * (bd[2] * cd[0] - bd[0] * cd[2]) +
                           ad[2] * (bd[0] * cd[1] - bd[1] * cd[0])) / 6.0;
   const double u = rule.x[q][0], v = rule.x[q][1], t = rule.x[q][2];
   for(int dd = 0; dd < 3; dd++)
      xyz[3 * e + dd] = T(a[dd] + (b[dd] - a[dd]) * u + (c[dd] - a[dd]) * v + (d[dd] - a[dd]) * t);
   w[e] = T(vol * rule.w[q]);
}

}  // namespace

}  // namespace fmm

using namespace fmm;

extern "C" fmm_status fmm_torus_quadratures(double radius, double section_width, int n_length, int n_width,
                                            int n_height, const double* rule_x, const double* rule_w, int k,
                                            int precision, void* xyz, void* w, int on_device, void* stream)
{
   if(n_length < 1 || n_width < 1 || n_height < 1 || k < 1 || k > MAXRULE)
      return setError(FMM_E_INVALID, "fmm_torus_quadratures: mesh %d x %d x %d, rule of %d points (1..%d)", n_length,
                      n_width, n_height, k, MAXRULE);
   if(!rule_x || !rule_w || !xyz || !w) return setError(FMM_E_INVALID, "fmm_torus_quadratures: null argument");
   if(precision != FMM_FP32 && precision != FMM_FP64)
      return setError(FMM_E_INVALID, "fmm_torus_quadratures: unknown precision %d", precision);
   if(!(section_width > 0) || !(radius > section_width / 2))
      return setError(FMM_E_INVALID, "fmm_torus_quadratures: radius %g and section width %g", radius, section_width);
   const int64_t total = int64_t(n_length) * n_width * n_height * 5 * k;
   if(total > (int64_t(1) << 31) - 1) return setError(FMM_E_LIMIT, "fmm_torus_quadratures: %lld points", (long long)total);
   Rule rule{};
   rule.k = k;
   for(int q = 0; q < k; q++)
   {
      for(int d = 0; d < 3; d++) rule.x[q][d] = rule_x[3 * q + d];
      rule.w[q] = rule_w[q];
   }
   cudaStream_t st = (cudaStream_t)stream;
   const size_t es = precision == FMM_FP64 ? sizeof(double) : sizeof(float);
   void* dX = xyz;
   void* dW = w;
   DevBuf stage;
   if(!on_device)
   {
      FMM_TRY(stage.reserve(4 * es * size_t(total)));
      dX = stage.ptr;
      dW = (char*)stage.ptr + 3 * es * size_t(total);
   }
   const int blocks = int((total + 255) / 256);
   if(precision == FMM_FP64)
      kTorusQuadratures<double><<<blocks, 256, 0, st>>>(radius, section_width, n_length, n_width, n_height, rule, total,
                                                        (double*)dX, (double*)dW);
   else
      kTorusQuadratures<float><<<blocks, 256, 0, st>>>(radius, section_width, n_length, n_width, n_height, rule, total,
                                                       (float*)dX, (float*)dW);
   cudaError_t e = cudaGetLastError();
   if(e == cudaSuccess && !on_device)
   {
      e = cudaMemcpyAsync(xyz, dX, 3 * es * size_t(total), cudaMemcpyDeviceToHost, st);
      if(e == cudaSuccess) e = cudaMemcpyAsync(w, dW, es * size_t(total), cudaMemcpyDeviceToHost, st);
      if(e == cudaSuccess) e = cudaStreamSynchronize(st);
   }
   stage.release();
   if(e != cudaSuccess) return setError(FMM_E_CUDA, "fmm_torus_quadratures: %s", cudaGetErrorString(e));
   return FMM_OK;
}
