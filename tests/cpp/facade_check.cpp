// Drives the C++ facade (include/fmm_facade.hpp) the way the reference's own programs drive
// FastMultipoleSolver (FMM/FMMGPU/main.cpp:568-572) and its kernel seam. Reads
//   <dir>/quads.bin   n x 4 reals (x, y, z, weight)
//   <dir>/points.bin  m x 3 reals
//   <dir>/seam.bin    count, order, then count x L harmonics and count x L x 3 expansions (reals)
// and writes <dir>/fmm_B.bin (m x 3), <dir>/direct_B.bin (first 4 points x 3), <dir>/seam_out.bin
// (count x L x 3), <dir>/matrix_out.bin (3 x count x L for b = the identity plus 1 on the
// diagonal's neighbour), <dir>/tree_B.bin (MultipoleSolver::calcB(current, point), the treecode, at the
// first 8 points x 3) and <dir>/bem.bin (a BEM FastMultipoleSolver's calcBEM at the points, sources
// built from quads with field B = (1, 2, 3) and normal (0, 0, 1)). Exit status 0 only when every call
// and every call-order check behaved.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "fmm_facade.hpp"

template <class T>
static std::vector<T> readAll(const std::string& path)
{
   std::ifstream f(path, std::ios::binary);
   f.seekg(0, std::ios::end);
   size_t bytes = size_t(f.tellg());
   f.seekg(0);
   std::vector<T> v(bytes / sizeof(T));
   f.read(reinterpret_cast<char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
   return v;
}

template <class T>
static void writeAll(const std::string& path, const T* data, size_t n)
{
   std::ofstream f(path, std::ios::binary);
   f.write(reinterpret_cast<const char*>(data), std::streamsize(n * sizeof(T)));
}

int main(int argc, char** argv)
{
   if(argc < 2) return 2;
   const std::string dir = argv[1];
   auto q = readAll<real>(dir + "/quads.bin");
   auto p = readAll<real>(dir + "/points.bin");
   std::vector<Quadrature> quads(q.size() / 4);
   for(size_t i = 0; i < quads.size(); i++)
      quads[i] = Quadrature(Vector3(q[4 * i], q[4 * i + 1], q[4 * i + 2]), real(1), q[4 * i + 3]);
   std::vector<Vector3> points(p.size() / 3);
   for(size_t i = 0; i < points.size(); i++) points[i] = Vector3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);

   FastMultipoleSolver solver(quads, points, Problem::BioSavartLaplace, 33, 33, 10);
   bool orderChecked = false;
   try
   {
      solver.calcLocalMultipoleExpansions(M2LAlg::ComplexTranslation, Device::GPU);
   }
   catch(const std::runtime_error&)
   {
      orderChecked = true;
   }
   if(!orderChecked) return 3;
   solver.calcMultipoleExpansionsAtLeaves();
   solver.calclMultipoleExpansions(M2MAlg::Matrices, Device::GPU);
   solver.calcLocalMultipoleExpansions(M2LAlg::ComplexTranslation, Device::GPU);
   auto res = solver.calcB(real(1));
   std::vector<real> B(3 * res.size());
   for(size_t i = 0; i < res.size(); i++)
   {
      if(res[i].first.x != points[i].x || res[i].first.y != points[i].y || res[i].first.z != points[i].z) return 4;
      B[3 * i] = res[i].second.x;
      B[3 * i + 1] = res[i].second.y;
      B[3 * i + 2] = res[i].second.z;
   }
   writeAll(dir + "/fmm_B.bin", B.data(), B.size());

   std::vector<real> D;
   for(size_t i = 0; i < 4 && i < points.size(); i++)
   {
      Vector3 b = math::calcBioSavartLaplace(real(1), points[i], quads);
      D.push_back(b.x);
      D.push_back(b.y);
      D.push_back(b.z);
   }
   writeAll(dir + "/direct_B.bin", D.data(), D.size());

   auto s = readAll<real>(dir + "/seam.bin");
   const size_t count = size_t(s[0]), order = size_t(s[1]);
   const size_t L = (order + 1) * (order + 1);
   std::vector<Vector3> expansions(count * L), out(count * L);
   const real* harm = s.data() + 2;
   for(size_t i = 0; i < count * L; i++)
   {
      const real* e = s.data() + 2 + count * L + 3 * i;
      expansions[i] = Vector3(e[0], e[1], e[2]);
   }
   kernels::translateAllGPU(out.data(), harm, expansions.data(), count, order);
   writeAll(dir + "/seam_out.bin", &out[0].x, 3 * out.size());

   // the three-component matrix overload with b = I + (superdiagonal of ones)
   std::vector<real> bmat(L * L, real(0));
   for(size_t k = 0; k < L; k++)
   {
      bmat[k * L + k] = 1;
      if(k + 1 < L) bmat[k * L + k + 1] = 1;
   }
   kernels::RealMatrix comps(3, std::vector<real>(count * L)), prod;
   for(size_t c = 0; c < 3; c++)
      for(size_t i = 0; i < count * L; i++) comps[c][i] = (&expansions[i].x)[c];
   kernels::translateAllGPUMatrixCuBLAS(prod, comps, bmat.data(), count, order);
   std::vector<real> flat;
   for(auto& v : prod) flat.insert(flat.end(), v.begin(), v.end());
   writeAll(dir + "/matrix_out.bin", flat.data(), flat.size());

   // the reference's treecode point queries (multipole_solver.cpp:686-700)
   MultipoleSolver tree(quads, Problem::BioSavartLaplace, 33, 10);
   tree.calcMultipoleExpansionsAtLeaves();
   tree.calclMultipoleExpansions(M2MAlg::Matrices, Device::GPU);
   std::vector<real> TB;
   for(size_t i = 0; i < 8 && i < points.size(); i++)
   {
      Vector3 b = tree.calcB(real(2), points[i]);
      TB.push_back(b.x);
      TB.push_back(b.y);
      TB.push_back(b.z);
   }
   writeAll(dir + "/tree_B.bin", TB.data(), TB.size());

   // the BEM problem (Problem::BEM, calcBEM)
   std::vector<BEMQuadrature> bq(quads.size());
   for(size_t i = 0; i < quads.size(); i++)
      bq[i] = BEMQuadrature(quads[i], real(1), quads[i].weight, Vector3(1, 2, 3), Vector3(0, 0, 1));
   BasicFastMultipoleSolver<BEMQuadrature> bem(bq, points, Problem::BEM, 33, 33, 10);
   bem.calcMultipoleExpansionsAtLeaves();
   bem.calclMultipoleExpansions(M2MAlg::Matrices, Device::GPU);
   bem.calcLocalMultipoleExpansions(M2LAlg::ComplexTranslation, Device::GPU);
   auto bres = bem.calcBEM(real(1));
   std::vector<real> BF;
   for(auto& r : bres)
   {
      BF.push_back(r.second.x);
      BF.push_back(r.second.y);
      BF.push_back(r.second.z);
   }
   writeAll(dir + "/bem.bin", BF.data(), BF.size());

   auto sum = kernels::addVectors({1, 2, 3}, {10, 20, 30});
   if(sum.size() != 3 || sum[2] != real(33)) return 5;
   std::printf("facade ok: %zu targets, %zu seam items\n", points.size(), count);
   return 0;
}
