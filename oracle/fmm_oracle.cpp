// CPU restatement of the reference fast-multipole Biot-Savart solver (the oracle).
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or calls this
// file; it is imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg, and only as the checker.
//
// What is restated, each from the reference file and lines it follows (paths relative
// to FMM/FMMGPU/ of iamwhoamianamy/bachelors):
//   * real solid harmonics by the reference's own route (normalise, Legendre recurrence,
//     d^m P_l / dz^m recurrence, mirror, complex phase)          harmonics.cpp:79-199
//   * real <-> complex conversions                                harmonics.cpp:340-379
//   * M2M / M2L (l + lambda <= p) / L2L in complex form, with the
//     reference's sign factors                                    multipole_translator.cpp:3-32,143-176,195-255
//   * P2M: M_k += J * R_k(q - c) * w                               integration.cpp:137-161
//   * evaluation of A from a local expansion                      calculation_point_octree.cpp:192-212
//   * the direct Biot-Savart sum                                  integration.cpp:101-120
//   * output scaling mu0 / (4 pi) * I (B) and I / (4 pi) (A)      fast_multipole_solver.cpp:195-231
// and, in "standard" mode, the tree, interaction lists and analytic curl that the B200
// pipeline uses (one Morton octree over sources and targets, same-level M2L over the 316
// offsets, direct near field). That part has no reference counterpart; its definition is
// stated next to the code.
//
// Two modes:
//   compat = 1 reproduces the reference bit-for-bit in its arithmetic choices: the short
//     literal R_SQRT_2 = 0.70710678118 in realToComplex and 1/sqrt(2) in complexToReal
//     (math.hpp:16, harmonics.cpp:345,367), r += machine epsilon before normalising
//     (harmonics.cpp:83-88) and the missing complex phase at m = p (harmonics.cpp:189).
//   compat = 0 ("standard") uses exact constants, no epsilon, and the phase for all m <= p.
// The short literals PI = 3.14159265359 and MU0 = 1.2566370614e-6 (math.hpp:12-13) are used in
// both modes because they only set the overall output scale.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

typedef std::complex<double> cplx;
constexpr double REF_PI = 3.14159265359;
constexpr double REF_MU0 = 1.2566370614e-6;
constexpr double REF_R_SQRT_2 = 0.70710678118;

inline int idx(int l, int m) { return l * l + l + m; }
inline int nharm(int p) { return (p + 1) * (p + 1); }

// ---------------------------------------------------------------------------------------
// Harmonics, restated from harmonics.cpp:79-199. T is double or a forward-mode dual number
// (used to get the analytic gradient of the same formula for the curl checks).
// ---------------------------------------------------------------------------------------
struct Dual
{
   double v, d[3];
   Dual(double x = 0) : v(x), d{0, 0, 0} {}
};
inline Dual operator+(Dual a, Dual b) { Dual r(a.v + b.v); for(int i = 0; i < 3; i++) r.d[i] = a.d[i] + b.d[i]; return r; }
inline Dual operator-(Dual a, Dual b) { Dual r(a.v - b.v); for(int i = 0; i < 3; i++) r.d[i] = a.d[i] - b.d[i]; return r; }
inline Dual operator-(Dual a) { Dual r(-a.v); for(int i = 0; i < 3; i++) r.d[i] = -a.d[i]; return r; }
inline Dual operator*(Dual a, Dual b)
{ Dual r(a.v * b.v); for(int i = 0; i < 3; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
inline Dual operator/(Dual a, Dual b)
{ Dual r(a.v / b.v); for(int i = 0; i < 3; i++) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v); return r; }
inline Dual sqrtT(Dual a) { Dual r(std::sqrt(a.v)); for(int i = 0; i < 3; i++) r.d[i] = a.d[i] / (2 * r.v); return r; }
inline double sqrtT(double a) { return std::sqrt(a); }
inline double val(double a) { return a; }
inline double val(Dual a) { return a.v; }

double factorial(int n)
{
   double f = 1;
   for(int i = 2; i <= n; i++) f *= i;
   return f;
}

template <class T>
void solidHarmonics(int p, T x, T y, T z, bool regular, bool compat, T* out)
{
   // r = |point| (+ machine epsilon in the reference), point /= r
   T r = sqrtT(x * x + y * y + z * z);
   if(compat) r = r + T(DBL_EPSILON);
   T ux = x / r, uy = y / r, uz = z / r;
   std::vector<T> h(nharm(p), T(0));
   // Legendre polynomials P_l(z) into (l, 0)
   h[idx(0, 0)] = T(1);
   if(p >= 1) h[idx(1, 0)] = uz;
   for(int l = 2; l <= p; l++)
      h[idx(l, 0)] = (T(double(2 * l - 1)) * uz * h[idx(l - 1, 0)] - T(double(l - 1)) * h[idx(l - 2, 0)]) / T(double(l));
   // d^m P_l / dz^m for 1 <= m <= l
   if(p >= 1) { h[idx(1, -1)] = T(1); h[idx(1, 1)] = T(1); }
   for(int l = 2; l <= p; l++)
   {
      for(int m = 1; m < l; m++)
         h[idx(l, m)] = uz * h[idx(l - 1, m)] + T(double(l + m - 1)) * h[idx(l - 1, m - 1)];
      h[idx(l, l)] = T(double(2 * l - 1)) * h[idx(l - 1, l - 1)];
   }
   // mirror to -m
   for(int l = 2; l <= p; l++)
      for(int m = 1; m <= l; m++) h[idx(l, -m)] = h[idx(l, m)];
   // multiply by sqrt(2) Re / Im of (x + i y)^m; the reference stops at m < p
   int mmax = compat ? p - 1 : p;
   T er = T(std::sqrt(2.0)), ei = T(0);
   for(int m = 1; m <= mmax; m++)
   {
      T nr = er * ux - ei * uy;
      T ni = er * uy + ei * ux;
      er = nr; ei = ni;
      for(int l = m; l <= p; l++)
      {
         h[idx(l, m)] = h[idx(l, m)] * er;
         h[idx(l, -m)] = h[idx(l, -m)] * ei;
      }
   }
   // radial part and (-1)^l with factorial normalisation
   T mult = regular ? r : T(1) / r;
   T curr = regular ? T(1) : mult;
   for(int l = 0; l <= p; l++)
   {
      for(int m = 0; m <= l; m++)
      {
         double f = regular ? 1.0 / factorial(l + m) : factorial(l - m);
         h[idx(l, -m)] = h[idx(l, -m)] * curr * T(f);
         if(m > 0) h[idx(l, m)] = h[idx(l, m)] * curr * T(f);
      }
      curr = -(curr * mult);
   }
   for(int k = 0; k < nharm(p); k++) out[k] = h[k];
}

// ---------------------------------------------------------------------------------------
// Real <-> complex (harmonics.cpp:340-379) and the complex translations
// (multipole_translator.cpp:3-32, 143-176, 195-255).
// ---------------------------------------------------------------------------------------
void realToComplex(int p, const double* a, bool compat, cplx* c)
{
   double s = compat ? REF_R_SQRT_2 : 1.0 / std::sqrt(2.0);
   for(int l = 0; l <= p; l++)
   {
      c[idx(l, 0)] = cplx(a[idx(l, 0)], 0);
      for(int m = 1; m <= l; m++)
      {
         c[idx(l, m)] = cplx(a[idx(l, m)] * s, a[idx(l, -m)] * s);
         c[idx(l, -m)] = cplx(a[idx(l, m)] * s, -a[idx(l, -m)] * s);
      }
   }
}

void complexToReal(int p, const cplx* c, double* a)
{
   double s = 1.0 / std::sqrt(2.0);
   for(int l = 0; l <= p; l++)
   {
      a[idx(l, 0)] = c[idx(l, 0)].real();
      for(int m = 1; m <= l; m++)
      {
         a[idx(l, m)] = s * (c[idx(l, m)] + c[idx(l, -m)]).real();
         a[idx(l, -m)] = s * (c[idx(l, m)] - c[idx(l, -m)]).imag();
      }
   }
}

// (-1)^e for the non-negative integer e = -(..)/2 the reference computes with pow(-1, x)
inline double signPow(int twiceExponent)
{
   int e = -twiceExponent / 2;
   return (e % 2 == 0) ? 1.0 : -1.0;
}
inline double m2mFactor(int m, int mu) { return signPow(std::abs(m) - std::abs(mu) - std::abs(m - mu)); }
inline double m2lFactor(int m, int mu, int lambda)
{ return signPow(std::abs(m - mu) - std::abs(m) - std::abs(mu)) * ((lambda % 2) ? -1.0 : 1.0); }
inline double l2lFactor(int m, int mu, int lambda, int l)
{ return signPow(std::abs(mu) - std::abs(m - mu) - std::abs(m)) * (((lambda + l) % 2) ? -1.0 : 1.0); }

// res(l,m) = sum R(lambda,mu) * M(l-lambda, m-mu) * factor(m, mu)     (translateMultipole, a = R, b = M)
void m2mComplex(int p, const cplx* R, const cplx* M, cplx* res)
{
   for(int k = 0; k < nharm(p); k++) res[k] = 0;
   for(int l = 0; l <= p; l++)
      for(int m = -l; m <= l; m++)
         for(int lambda = 0; lambda <= l; lambda++)
         {
            int dl = l - lambda;
            for(int mu = -lambda; mu <= lambda; mu++)
            {
               int dm = m - mu;
               if(dm >= -dl && dm <= dl) res[idx(l, m)] += R[idx(lambda, mu)] * M[idx(dl, dm)] * m2mFactor(m, mu);
            }
         }
}

// res(l,m) = sum_{l+lambda<=p} M(lambda,mu) * I(l+lambda, m-mu) * factor(m, mu, lambda)
// `lim` is the largest l + lambda kept: p in the reference (Q4 truncation), up to 2p for the
// untruncated operator; I must hold irregular harmonics up to order lim.
void m2lComplex(int p, const cplx* M, const cplx* I, cplx* res, int lim)
{
   for(int k = 0; k < nharm(p); k++) res[k] = 0;
   for(int l = 0; l <= p; l++)
      for(int lambda = 0; lambda <= p; lambda++)
         for(int m = -l; m <= l; m++)
            for(int mu = -lambda; mu <= lambda; mu++)
            {
               int dl = l + lambda, dm = m - mu;
               if(dm >= -dl && dm <= dl && dl <= lim)
                  res[idx(l, m)] += M[idx(lambda, mu)] * I[idx(dl, dm)] * m2lFactor(m, mu, lambda);
            }
}

// res(l,m) = sum_{lambda>=l} L(lambda,mu) * R(lambda-l, m-mu) * factor(m, mu, lambda, l)
void l2lComplex(int p, const cplx* L, const cplx* R, cplx* res)
{
   for(int k = 0; k < nharm(p); k++) res[k] = 0;
   for(int l = 0; l <= p; l++)
      for(int lambda = l; lambda <= p; lambda++)
         for(int m = -l; m <= l; m++)
            for(int mu = -lambda; mu <= lambda; mu++)
            {
               int dl = lambda - l, dm = m - mu;
               if(dm >= -dl && dm <= dl)
                  res[idx(l, m)] += L[idx(lambda, mu)] * R[idx(dl, dm)] * l2lFactor(m, mu, lambda, l);
            }
}

enum class Op { M2M, M2L, L2L };

// Apply one translation to a 3-component expansion stored AoS [k][xyz] (the reference's
// HarmonicSeries<Vector3>), component by component, as the *WithComplex functions do.
int g_m2lLimitExtra = 0;  // extra l + lambda beyond p kept by M2L (0 = the reference's truncation)
int g_capT = 0;           // target leaf capacity (0: same as the source capacity)

void translate(Op op, int p, bool compat, const double* in, const double* t, double* out)
{
   int L = nharm(p);
   int ph = (op == Op::M2L) ? p + g_m2lLimitExtra : p;
   std::vector<double> h(nharm(ph)), comp(L), res(L);
   std::vector<cplx> hc(nharm(ph)), cc(L), rc(L);
   solidHarmonics<double>(ph, t[0], t[1], t[2], op != Op::M2L, compat, h.data());
   realToComplex(ph, h.data(), compat, hc.data());
   for(int d = 0; d < 3; d++)
   {
      for(int k = 0; k < L; k++) comp[k] = in[3 * k + d];
      realToComplex(p, comp.data(), compat, cc.data());
      if(op == Op::M2M) m2mComplex(p, hc.data(), cc.data(), rc.data());
      else if(op == Op::M2L) m2lComplex(p, cc.data(), hc.data(), rc.data(), ph);
      else l2lComplex(p, cc.data(), hc.data(), rc.data());
      complexToReal(p, rc.data(), res.data());
      for(int k = 0; k < L; k++) out[3 * k + d] = res[k];
   }
}

inline void azimuthal(double x, double y, double J[3])
{
   // perp(q).normalized() = (-y, x, 0) / |(-y, x, 0)| (vector3.cu:154-204); zero on the axis
   double l = std::sqrt(x * x + y * y);
   if(l != 0) { J[0] = -y / l; J[1] = x / l; J[2] = 0; }
   else { J[0] = J[1] = J[2] = 0; }
}

// A and curl A of a 3-component expansion evaluated with harmonics at d. For a local
// expansion the harmonics are regular; for a multipole they are irregular.
void evalExpansion(int p, bool regular, const double* coef, const double* d, double A[3], double curl[3],
                   bool compat = false)
{
   int L = nharm(p);
   std::vector<Dual> h(L);
   Dual x(d[0]), y(d[1]), z(d[2]);
   x.d[0] = 1; y.d[1] = 1; z.d[2] = 1;
   solidHarmonics<Dual>(p, x, y, z, regular, compat, h.data());
   double a[3] = {0, 0, 0}, g[3][3] = {{0}};  // g[c][j] = d A_c / d x_j
   for(int k = 0; k < L; k++)
      for(int c = 0; c < 3; c++)
      {
         a[c] += coef[3 * k + c] * h[k].v;
         for(int j = 0; j < 3; j++) g[c][j] += coef[3 * k + c] * h[k].d[j];
      }
   for(int c = 0; c < 3; c++) A[c] = a[c];
   curl[0] = g[2][1] - g[1][2];
   curl[1] = g[0][2] - g[2][0];
   curl[2] = g[1][0] - g[0][1];
}

// ---------------------------------------------------------------------------------------
// Standard-mode tree and interaction lists (the definition the B200 pipeline implements).
//
// One octree over the union of sources and targets inside the cube (center, half-width H).
// A point's integer cell at depth D = 21 is u = floor((x - (center - H)) * 2^21 / (2 H)),
// clamped to [0, 2^21 - 1], computed in double. The Morton key interleaves the bits with x
// lowest: octant = bx | by << 1 | bz << 2. A node splits when it holds more than `cap`
// sources or more than `cap` targets and its level is below D. Children are created for
// the octants that hold at least one source or target. Nodes are numbered level by level,
// in key order within a level.
//
// Lists, built top-down. Col(root) = {root}. For a node D with parent P:
//   * for C in Col(P): if C is a leaf it is a coarse candidate, else each child c of C is
//     adjacent to D -> Col(D), or not -> V(D) (M2L; offset in [-3,3]^3 minus [-1,1]^3);
//   * for S in A(P) (coarse leaves adjacent to P) and each coarse candidate S:
//     adjacent to D -> A(D), else -> X(D).
// Direct (P2P) interactions of a target leaf T: every leaf in Col(T), every leaf in A(T),
// every finer leaf S with T in A(S), every node D with T in X(D) (all sources below D),
// and every S in X(a) for T and each ancestor a of T. "Adjacent" means the closed boxes
// touch or overlap.
// ---------------------------------------------------------------------------------------
constexpr int MAXLEVEL = 21;

struct Node
{
   int level;
   uint64_t key;  // Morton prefix of length 3*level
   int64_t s0, s1, t0, t1;
   int parent;
   int child[8];
   int nchild;
   int64_t ix, iy, iz;  // integer coordinates at its level
   bool leaf() const { return nchild == 0; }
};

inline uint64_t mortonOf(int64_t ux, int64_t uy, int64_t uz)
{
   uint64_t k = 0;
   for(int b = MAXLEVEL - 1; b >= 0; b--)
      k = (k << 3) | uint64_t(((ux >> b) & 1) | (((uy >> b) & 1) << 1) | (((uz >> b) & 1) << 2));
   return k;
}

inline int64_t quantize(double x, double lo, double scale)
{
   double u = std::floor((x - lo) * scale);
   if(u < 0) u = 0;
   if(u > double((1 << MAXLEVEL) - 1)) u = double((1 << MAXLEVEL) - 1);
   return int64_t(u);
}

bool adjacent(const Node& a, const Node& b)
{
   // closed-box contact test on the integer grid of the finer node
   const Node& c = a.level <= b.level ? a : b;  // coarser
   const Node& f = a.level <= b.level ? b : a;  // finer
   int64_t s = int64_t(1) << (f.level - c.level);
   int64_t ci[3] = {c.ix, c.iy, c.iz}, fi[3] = {f.ix, f.iy, f.iz};
   for(int d = 0; d < 3; d++)
      if(fi[d] < ci[d] * s - 1 || fi[d] > (ci[d] + 1) * s) return false;
   return true;
}

struct Tree
{
   std::vector<Node> nodes;
   std::vector<int> levelStart;  // nodes of level l are [levelStart[l], levelStart[l+1])
   std::vector<int64_t> srcOrder, tgtOrder;  // sorted position -> input index
   std::vector<uint64_t> srcKey, tgtKey;     // sorted keys
   double center[3], H;
   std::vector<std::vector<int>> col, A, V, X, U, W;
   std::vector<std::vector<int>> vOffset;    // offset index (0..342) per V entry
};

void sortByKey(const double* xyz, int64_t n, double lo[3], double scale, std::vector<uint64_t>& keys,
               std::vector<int64_t>& order)
{
   std::vector<std::pair<uint64_t, int64_t>> kv(n);
   for(int64_t i = 0; i < n; i++)
   {
      int64_t u[3];
      for(int d = 0; d < 3; d++) u[d] = quantize(xyz[3 * i + d], lo[d], scale);
      kv[i] = {mortonOf(u[0], u[1], u[2]), i};
   }
   std::stable_sort(kv.begin(), kv.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
   keys.resize(n); order.resize(n);
   for(int64_t i = 0; i < n; i++) { keys[i] = kv[i].first; order[i] = kv[i].second; }
}

int64_t lowerBound(const std::vector<uint64_t>& keys, int64_t a, int64_t b, uint64_t v)
{
   return std::lower_bound(keys.begin() + a, keys.begin() + b, v) - keys.begin();
}

void buildTree(Tree& t, const double* src, int64_t n, const double* tgt, int64_t m, const double* center, double H,
               int cap, int capT)
{
   for(int d = 0; d < 3; d++) t.center[d] = center[d];
   t.H = H;
   double lo[3] = {center[0] - H, center[1] - H, center[2] - H};
   double scale = double(1 << MAXLEVEL) / (2.0 * H);
   sortByKey(src, n, lo, scale, t.srcKey, t.srcOrder);
   sortByKey(tgt, m, lo, scale, t.tgtKey, t.tgtOrder);
   Node root{};
   root.level = 0; root.key = 0; root.s0 = 0; root.s1 = n; root.t0 = 0; root.t1 = m; root.parent = -1;
   root.nchild = 0; root.ix = root.iy = root.iz = 0;
   t.nodes.push_back(root);
   t.levelStart = {0, 1};
   for(int level = 0; level < MAXLEVEL; level++)
   {
      int a = t.levelStart[level], b = t.levelStart[level + 1];
      for(int i = a; i < b; i++)
      {
         Node nd = t.nodes[i];
         if(!(nd.s1 - nd.s0 > cap || nd.t1 - nd.t0 > capT)) continue;
         int shift = 3 * (MAXLEVEL - level - 1);
         int64_t sb[9], tb[9];
         for(int c = 0; c <= 8; c++)
         {
            uint64_t bound = ((nd.key << 3) + uint64_t(c)) << shift;
            sb[c] = (c == 8) ? nd.s1 : lowerBound(t.srcKey, nd.s0, nd.s1, bound);
            tb[c] = (c == 8) ? nd.t1 : lowerBound(t.tgtKey, nd.t0, nd.t1, bound);
         }
         for(int c = 0; c < 8; c++)
         {
            if(sb[c + 1] - sb[c] + tb[c + 1] - tb[c] == 0) continue;
            Node ch{};
            ch.level = level + 1;
            ch.key = (nd.key << 3) | uint64_t(c);
            ch.s0 = sb[c]; ch.s1 = sb[c + 1]; ch.t0 = tb[c]; ch.t1 = tb[c + 1];
            ch.parent = i; ch.nchild = 0;
            ch.ix = 2 * nd.ix + (c & 1); ch.iy = 2 * nd.iy + ((c >> 1) & 1); ch.iz = 2 * nd.iz + ((c >> 2) & 1);
            t.nodes[i].child[t.nodes[i].nchild++] = int(t.nodes.size());
            t.nodes.push_back(ch);
         }
      }
      int end = int(t.nodes.size());
      if(end == b) break;
      t.levelStart.push_back(end);
   }
}

void buildLists(Tree& t)
{
   size_t N = t.nodes.size();
   t.col.assign(N, {}); t.A.assign(N, {}); t.V.assign(N, {}); t.X.assign(N, {});
   t.U.assign(N, {}); t.W.assign(N, {}); t.vOffset.assign(N, {});
   t.col[0].push_back(0);
   for(size_t i = 1; i < N; i++)
   {
      const Node& D = t.nodes[i];
      int P = D.parent;
      std::vector<int> coarse;
      for(int C : t.col[P])
      {
         const Node& cn = t.nodes[C];
         if(cn.leaf()) { coarse.push_back(C); continue; }
         for(int k = 0; k < cn.nchild; k++)
         {
            int c = cn.child[k];
            if(adjacent(t.nodes[c], D)) t.col[i].push_back(c);
            else
            {
               t.V[i].push_back(c);
               const Node& s = t.nodes[c];
               int ox = int(s.ix - D.ix), oy = int(s.iy - D.iy), oz = int(s.iz - D.iz);
               t.vOffset[i].push_back((ox + 3) + 7 * (oy + 3) + 49 * (oz + 3));
            }
         }
      }
      for(int S : t.A[P]) coarse.push_back(S);
      for(int S : coarse)
      {
         if(adjacent(t.nodes[S], D)) t.A[i].push_back(S);
         else t.X[i].push_back(S);
      }
   }
   // direct-interaction lists of target leaves
   for(size_t i = 0; i < N; i++)
   {
      if(!t.nodes[i].leaf()) continue;
      for(int C : t.col[i])
         if(t.nodes[C].leaf()) t.U[i].push_back(C);
      for(int S : t.A[i])
      {
         t.U[i].push_back(S);  // coarse adjacent leaf -> this leaf
         t.U[S].push_back(int(i));  // this (finer) leaf -> coarse adjacent leaf
      }
   }
   for(size_t i = 0; i < N; i++)
      for(int S : t.X[i]) t.W[S].push_back(int(i));  // all sources below node i -> targets of leaf S
}

// ---------------------------------------------------------------------------------------
// Direct Biot-Savart (integration.cpp:101-120) over source index range, for one target.
// ---------------------------------------------------------------------------------------
inline void directAccumulate(const double* x, const double* q, double w, const double* J, double B[3], double A[3])
{
   double d[3] = {x[0] - q[0], x[1] - q[1], x[2] - q[2]};
   double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
   if(r2 == 0) return;  // self term excluded
   double r = std::sqrt(r2);
   double inv3 = 1.0 / (r2 * r);
   B[0] += w * (J[1] * d[2] - J[2] * d[1]) * inv3;
   B[1] += w * (J[2] * d[0] - J[0] * d[2]) * inv3;
   B[2] += w * (J[0] * d[1] - J[1] * d[0]) * inv3;
   for(int c = 0; c < 3; c++) A[c] += w * J[c] / r;
}

void currentOf(const double* J, const double* xyz, int64_t i, double out[3])
{
   if(J) { out[0] = J[3 * i]; out[1] = J[3 * i + 1]; out[2] = J[3 * i + 2]; }
   else azimuthal(xyz[3 * i], xyz[3 * i + 1], out);
}

}  // namespace

extern "C" {

// Number of degrees beyond p that M2L keeps in l + lambda (0 reproduces the reference's
// l + lambda <= p truncation; p keeps the full operator). Process-wide setting.
void orc_set_m2l_extra(int extra) { g_m2lLimitExtra = extra; }
// Target leaf capacity of the standard-mode tree (0: the source capacity). Process-wide setting.
void orc_set_target_cap(int capT) { g_capT = capT; }

// Real solid harmonics (regular or irregular) of `xyz` up to order p: out[(p+1)^2].
void orc_solid_harmonics(int p, int regular, int compat, const double* xyz, double* out)
{
   solidHarmonics<double>(p, xyz[0], xyz[1], xyz[2], regular != 0, compat != 0, out);
}

// Gradient of the real solid harmonics: out[(p+1)^2][3] (d/dx, d/dy, d/dz), standard mode.
void orc_solid_harmonics_grad(int p, int regular, const double* xyz, double* out)
{
   std::vector<Dual> h(nharm(p));
   Dual x(xyz[0]), y(xyz[1]), z(xyz[2]);
   x.d[0] = 1; y.d[1] = 1; z.d[2] = 1;
   solidHarmonics<Dual>(p, x, y, z, regular != 0, false, h.data());
   for(int k = 0; k < nharm(p); k++)
      for(int j = 0; j < 3; j++) out[3 * k + j] = h[k].d[j];
}

// The same gradient in either convention (compat != 0: the reference's).
void orc_solid_harmonics_grad2(int p, int regular, int compat, const double* xyz, double* out)
{
   std::vector<Dual> h(nharm(p));
   Dual x(xyz[0]), y(xyz[1]), z(xyz[2]);
   x.d[0] = 1; y.d[1] = 1; z.d[2] = 1;
   solidHarmonics<Dual>(p, x, y, z, regular != 0, compat != 0, h.data());
   for(int k = 0; k < nharm(p); k++)
      for(int j = 0; j < 3; j++) out[3 * k + j] = h[k].d[j];
}

// P2M about `center` from n points xyz[3n] with weights w[n] and current directions J[3n]
// (J == nullptr: the reference's azimuthal direction). out[(p+1)^2][3].
void orc_p2m(int p, int compat, int64_t n, const double* xyz, const double* w, const double* J,
             const double* center, double* out)
{
   int L = nharm(p);
   std::vector<double> h(L);
   for(int k = 0; k < 3 * L; k++) out[k] = 0;
   for(int64_t i = 0; i < n; i++)
   {
      double d[3] = {xyz[3 * i] - center[0], xyz[3 * i + 1] - center[1], xyz[3 * i + 2] - center[2]};
      solidHarmonics<double>(p, d[0], d[1], d[2], true, compat != 0, h.data());
      double j[3];
      currentOf(J, xyz, i, j);
      for(int k = 0; k < L; k++)
         for(int c = 0; c < 3; c++) out[3 * k + c] += j[c] * h[k] * w[i];
   }
}

void orc_m2m(int p, int compat, const double* in, const double* t, double* out)
{ translate(Op::M2M, p, compat != 0, in, t, out); }
void orc_m2l(int p, int compat, const double* in, const double* t, double* out)
{ translate(Op::M2L, p, compat != 0, in, t, out); }
void orc_l2l(int p, int compat, const double* in, const double* t, double* out)
{ translate(Op::L2L, p, compat != 0, in, t, out); }

// Batched real-form M2M with caller-supplied translation harmonics, the operation of the
// reference's kernels::translateAllCPU / translateAllGPU (translation_algorithms_cpu.cpp:9-95,
// MultipoleTranslator::translateMultipole multipole_translator.cpp:34-109). Per item i:
// a[i] holds the real regular harmonics of the translation ((p+1)^2), b[i] the vector
// expansion ((p+1)^2 x 3, AoS) and result[i] the translated expansion. The reference reads a
// real-form entry (l, m != 0) as the complex number s (h[l,|m|] + i sign(m) h[l,-|m|]) with
// s = R_SQRT_2 = 0.70710678118 (kernels.cuh:84-112); its m = 0 outputs sum the raw real-form
// products; its m > 0 outputs add the (l, m) and conjugated (l, -m) complex sums and scale by s.
// The sign factor is (-1)^((|m - mu| + |mu| - |m|) / 2) (multipole_translator.cpp:143-146).
void orc_translate_all(int64_t count, int p, const double* a, const double* b, double* result)
{
   const int L = nharm(p);
   const double s = REF_R_SQRT_2;
   auto factor = [](int m, int mu) { return ((std::abs(m - mu) + std::abs(mu) - std::abs(m)) / 2) % 2 ? -1.0 : 1.0; };
   auto view = [&](const double* h, int l, int m) -> cplx {
      if(m == 0) return cplx(h[idx(l, 0)], 0.0);
      return cplx(h[idx(l, std::abs(m))] * s, h[idx(l, -std::abs(m))] * s * (m > 0 ? 1.0 : -1.0));
   };
#pragma omp parallel for schedule(static)
   for(int64_t it = 0; it < count; it++)
   {
      const double* ai = a + it * L;
      const double* bi = b + it * 3 * L;
      double* ri = result + it * 3 * L;
      std::vector<double> bc(L);
      for(int c = 0; c < 3; c++)
      {
         for(int k = 0; k < L; k++) bc[k] = bi[3 * k + c];
         for(int l = 0; l <= p; l++)
         {
            double zero = 0;
            for(int lam = 0; lam <= l; lam++)
            {
               const int dl = l - lam;
               for(int mu = -std::min(lam, dl); mu <= std::min(lam, dl); mu++)
                  zero += bc[idx(lam, mu)] * ai[idx(dl, mu)] * factor(0, mu);
            }
            ri[3 * idx(l, 0) + c] = zero;
            for(int m = 1; m <= l; m++)
            {
               cplx acc = 0;
               for(int lam = 0; lam <= l; lam++)
               {
                  const int dl = l - lam;
                  for(int mu = -lam; mu <= lam; mu++)
                  {
                     const cplx B = view(bc.data(), lam, mu);
                     if(std::abs(m - mu) <= dl) acc += B * view(ai, dl, m - mu) * factor(m, mu);
                     if(std::abs(-m - mu) <= dl) acc += std::conj(B * view(ai, dl, -m - mu)) * factor(-m, mu);
                  }
               }
               ri[3 * idx(l, m) + c] = acc.real() * s;
               ri[3 * idx(l, -m) + c] = acc.imag() * s;
            }
         }
      }
   }
}

// The matrix forms of the same seam (translateAllCPUMatrixBLAS / translateAllGPUMatrixCuBLAS,
// translation_algorithms_cpu.cpp:114-135, and translateAllCPUMatrix :98-112): with items stored
// one after another, result (count x L) = a (count x L) * b (L x L), all row-major. The column-major
// BLAS call C = B * A of the reference is this product read in the transposed layout.
void orc_translate_all_matrix(int64_t count, int L, const double* a, const double* b, double* result)
{
#pragma omp parallel for schedule(static)
   for(int64_t i = 0; i < count; i++)
      for(int j = 0; j < L; j++)
      {
         double acc = 0;
         for(int k = 0; k < L; k++) acc += a[i * L + k] * b[int64_t(k) * L + j];
         result[i * L + j] = acc;
      }
}

// A = sum_k coef_k H_k(d) and curl A (analytic), H regular (local) or irregular (multipole).
void orc_eval_expansion(int p, int regular, int compat, const double* coef, const double* d, double* A, double* curl)
{ evalExpansion(p, regular != 0, coef, d, A, curl, compat != 0); }

// Direct sums in FP64: B = mu0/(4 pi) I sum w J x (x - q)/|x - q|^3 and A = I/(4 pi) sum w J/|x - q|,
// skipping coincident pairs. Either output may be null.
void orc_direct(int64_t n, const double* src, const double* w, const double* J, int64_t m, const double* tgt,
                double current, double* outB, double* outA)
{
#pragma omp parallel for schedule(dynamic, 8)
   for(int64_t t = 0; t < m; t++)
   {
      double B[3] = {0, 0, 0}, A[3] = {0, 0, 0};
      for(int64_t i = 0; i < n; i++)
      {
         double j[3];
         currentOf(J, src, i, j);
         directAccumulate(tgt + 3 * t, src + 3 * i, w[i], j, B, A);
      }
      for(int c = 0; c < 3; c++)
      {
         if(outB) outB[3 * t + c] = B[c] * REF_MU0 / (4 * REF_PI) * current;
         if(outA) outA[3 * t + c] = A[c] / (4 * REF_PI) * current;
      }
   }
}

// Adjoint of the direct Biot-Savart sum (no reference counterpart: the reference has no
// gradients). With g_t = dLoss/dB(x_t) and c = mu0/(4 pi) I:
//   dLoss/dJ_q = c w_q sum_t g_t x (q - x_t) / |q - x_t|^3
//   dLoss/dq   = c w_q sum_t [ a / r^3 - 3 (e . a) e / r^5 ],  e = q - x_t, a = J_q x g_t
// plus, when J is the azimuthal direction of q (J == nullptr), the term c w_q (dJ/dq)^T C(q)
// with C(q) = sum_t g_t x (q - x_t) / r^3. Coincident pairs are skipped. Outputs [3n].
void orc_adjoint_direct(int64_t n, const double* src, const double* w, const double* J, int64_t m,
                        const double* tgt, const double* g, double current, double* dJ, double* dx)
{
   const double c = REF_MU0 / (4 * REF_PI) * current;
#pragma omp parallel for schedule(dynamic, 8)
   for(int64_t q = 0; q < n; q++)
   {
      double Jq[3];
      currentOf(J, src, q, Jq);
      double C[3] = {0, 0, 0}, G[3] = {0, 0, 0};
      for(int64_t t = 0; t < m; t++)
      {
         double e[3] = {src[3 * q] - tgt[3 * t], src[3 * q + 1] - tgt[3 * t + 1], src[3 * q + 2] - tgt[3 * t + 2]};
         double r2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
         if(r2 == 0) continue;
         double r = std::sqrt(r2), ir3 = 1.0 / (r2 * r), ir5 = ir3 / r2;
         const double* gt = g + 3 * t;
         C[0] += (gt[1] * e[2] - gt[2] * e[1]) * ir3;
         C[1] += (gt[2] * e[0] - gt[0] * e[2]) * ir3;
         C[2] += (gt[0] * e[1] - gt[1] * e[0]) * ir3;
         double a[3] = {Jq[1] * gt[2] - Jq[2] * gt[1], Jq[2] * gt[0] - Jq[0] * gt[2], Jq[0] * gt[1] - Jq[1] * gt[0]};
         double ea = e[0] * a[0] + e[1] * a[1] + e[2] * a[2];
         for(int d = 0; d < 3; d++) G[d] += a[d] * ir3 - 3 * ea * e[d] * ir5;
      }
      if(!J)
      {
         double x = src[3 * q], y = src[3 * q + 1];
         double rho2 = x * x + y * y;
         if(rho2 > 0)
         {
            double ir = 1.0 / (rho2 * std::sqrt(rho2));
            G[0] += (x * y * C[0] + y * y * C[1]) * ir;
            G[1] += (-x * x * C[0] - x * y * C[1]) * ir;
         }
      }
      for(int d = 0; d < 3; d++)
      {
         if(dJ) dJ[3 * q + d] = c * w[q] * C[d];
         if(dx) dx[3 * q + d] = c * w[q] * G[d];
      }
   }
}

// Standard-mode FMM (the B200 pipeline's definition) at order p, leaf capacity `cap`,
// root cube (center, H). Outputs in input order; either may be null. stats (may be null)
// receives: [0] nodes, [1] levels, [2] leaves, [3] V entries, [4] U entries, [5] W entries,
// [6] X entries, [7] direct pair evaluations.
void orc_fmm(int p, int cap, int64_t n, const double* src, const double* w, const double* J, int64_t m,
             const double* tgt, double current, const double* center, double H, double* outB, double* outA,
             double* stats)
{
   Tree t;
   buildTree(t, src, n, tgt, m, center, H, cap, g_capT > 0 ? g_capT : cap);
   buildLists(t);
   int N = int(t.nodes.size()), L = nharm(p);
   std::vector<double> M(size_t(N) * 3 * L, 0.0), Lc(size_t(N) * 3 * L, 0.0);
   std::vector<std::array<double, 3>> ctr(N);
   for(int i = 0; i < N; i++)
   {
      const Node& nd = t.nodes[i];
      double h = 2 * H / double(int64_t(1) << nd.level);
      int64_t ii[3] = {nd.ix, nd.iy, nd.iz};
      for(int d = 0; d < 3; d++) ctr[i][d] = center[d] - H + (double(ii[d]) + 0.5) * h;
   }
   // P2M at leaves
#pragma omp parallel for schedule(dynamic, 4)
   for(int i = 0; i < N; i++)
   {
      const Node& nd = t.nodes[i];
      if(!nd.leaf() || nd.s1 == nd.s0) continue;
      int64_t cnt = nd.s1 - nd.s0;
      std::vector<double> xyz(3 * cnt), ww(cnt), jj(3 * cnt);
      for(int64_t k = 0; k < cnt; k++)
      {
         int64_t s = t.srcOrder[nd.s0 + k];
         for(int d = 0; d < 3; d++) xyz[3 * k + d] = src[3 * s + d];
         ww[k] = w[s];
         currentOf(J, src, s, &jj[3 * k]);
      }
      orc_p2m(p, 0, cnt, xyz.data(), ww.data(), jj.data(), ctr[i].data(), &M[size_t(i) * 3 * L]);
   }
   // M2M bottom-up
   for(int level = int(t.levelStart.size()) - 2; level >= 1; level--)
   {
#pragma omp parallel for schedule(dynamic, 4)
      for(int i = t.levelStart[level]; i < t.levelStart[level + 1]; i++)
      {
         const Node& nd = t.nodes[i];
         if(nd.s1 == nd.s0) continue;
         std::vector<double> tmp(3 * L);
         double tr[3];
         for(int d = 0; d < 3; d++) tr[d] = ctr[i][d] - ctr[nd.parent][d];
         translate(Op::M2M, p, false, &M[size_t(i) * 3 * L], tr, tmp.data());
#pragma omp critical
         for(int k = 0; k < 3 * L; k++) M[size_t(nd.parent) * 3 * L + k] += tmp[k];
      }
   }
   // M2L over V lists
#pragma omp parallel for schedule(dynamic, 4)
   for(int i = 0; i < N; i++)
   {
      if(t.nodes[i].t1 == t.nodes[i].t0) continue;
      std::vector<double> tmp(3 * L);
      for(int S : t.V[i])
      {
         if(t.nodes[S].s1 == t.nodes[S].s0) continue;
         double tr[3];
         for(int d = 0; d < 3; d++) tr[d] = ctr[S][d] - ctr[i][d];
         translate(Op::M2L, p, false, &M[size_t(S) * 3 * L], tr, tmp.data());
         for(int k = 0; k < 3 * L; k++) Lc[size_t(i) * 3 * L + k] += tmp[k];
      }
   }
   // L2L top-down
   for(int level = 1; level + 1 < int(t.levelStart.size()); level++)
   {
#pragma omp parallel for schedule(dynamic, 4)
      for(int i = t.levelStart[level]; i < t.levelStart[level + 1]; i++)
      {
         const Node& nd = t.nodes[i];
         if(nd.t1 == nd.t0) continue;
         std::vector<double> tmp(3 * L);
         double tr[3];
         for(int d = 0; d < 3; d++) tr[d] = ctr[nd.parent][d] - ctr[i][d];
         translate(Op::L2L, p, false, &Lc[size_t(nd.parent) * 3 * L], tr, tmp.data());
         for(int k = 0; k < 3 * L; k++) Lc[size_t(i) * 3 * L + k] += tmp[k];
      }
   }
   // L2P + direct near field at target leaves
   double directPairs = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : directPairs)
   for(int i = 0; i < N; i++)
   {
      const Node& nd = t.nodes[i];
      if(!nd.leaf() || nd.t1 == nd.t0) continue;
      // source ranges that interact directly with this leaf
      std::vector<std::pair<int64_t, int64_t>> ranges;
      for(int S : t.U[i]) ranges.push_back({t.nodes[S].s0, t.nodes[S].s1});
      for(int D : t.W[i]) ranges.push_back({t.nodes[D].s0, t.nodes[D].s1});
      for(int a = i; a != -1; a = t.nodes[a].parent)
         for(int S : t.X[a]) ranges.push_back({t.nodes[S].s0, t.nodes[S].s1});
      for(int64_t k = nd.t0; k < nd.t1; k++)
      {
         int64_t tg = t.tgtOrder[k];
         const double* x = tgt + 3 * tg;
         double d[3] = {x[0] - ctr[i][0], x[1] - ctr[i][1], x[2] - ctr[i][2]};
         double A[3], B[3];
         evalExpansion(p, true, &Lc[size_t(i) * 3 * L], d, A, B);
         for(auto& r : ranges)
            for(int64_t s = r.first; s < r.second; s++)
            {
               int64_t si = t.srcOrder[s];
               double j[3];
               currentOf(J, src, si, j);
               // the direct kernel accumulates B = J x (x - q) / r^3 = curl(J / r)
               directAccumulate(x, src + 3 * si, w[si], j, B, A);
               directPairs += 1;
            }
         for(int c = 0; c < 3; c++)
         {
            if(outB) outB[3 * tg + c] = B[c] * REF_MU0 / (4 * REF_PI) * current;
            if(outA) outA[3 * tg + c] = A[c] / (4 * REF_PI) * current;
         }
      }
   }
   if(stats)
   {
      double v = 0, u = 0, ww = 0, x = 0, leaves = 0;
      for(int i = 0; i < N; i++)
      {
         v += t.V[i].size(); u += t.U[i].size(); ww += t.W[i].size(); x += t.X[i].size();
         leaves += t.nodes[i].leaf();
      }
      stats[0] = N; stats[1] = double(t.levelStart.size() - 1); stats[2] = leaves; stats[3] = v; stats[4] = u;
      stats[5] = ww; stats[6] = x; stats[7] = directPairs;
   }
}

// Tree and list structure for structural parity: per node (level, ix, iy, iz, s0, s1, t0, t1,
// parent, nchild) into nodeInfo[10 * nodes] (if non-null, capacity maxNodes) and list sizes
// (|V|, |U|, |W|, |X|) into listSizes[4 * nodes]. Also the sorted-position -> input maps.
// Returns the node count.
int64_t orc_tree(int cap, int64_t n, const double* src, int64_t m, const double* tgt, const double* center, double H,
                 int64_t maxNodes, int64_t* nodeInfo, int64_t* listSizes, int64_t* srcOrder, int64_t* tgtOrder)
{
   Tree t;
   buildTree(t, src, n, tgt, m, center, H, cap, g_capT > 0 ? g_capT : cap);
   buildLists(t);
   int64_t N = int64_t(t.nodes.size());
   if(N > maxNodes) return N;
   for(int64_t i = 0; i < N; i++)
   {
      const Node& nd = t.nodes[i];
      int64_t v[10] = {nd.level, nd.ix, nd.iy, nd.iz, nd.s0, nd.s1, nd.t0, nd.t1, nd.parent, nd.nchild};
      if(nodeInfo) std::memcpy(nodeInfo + 10 * i, v, sizeof(v));
      if(listSizes)
      {
         listSizes[4 * i] = int64_t(t.V[i].size()); listSizes[4 * i + 1] = int64_t(t.U[i].size());
         listSizes[4 * i + 2] = int64_t(t.W[i].size()); listSizes[4 * i + 3] = int64_t(t.X[i].size());
      }
   }
   if(srcOrder) std::memcpy(srcOrder, t.srcOrder.data(), sizeof(int64_t) * n);
   if(tgtOrder) std::memcpy(tgtOrder, t.tgtOrder.data(), sizeof(int64_t) * m);
   return N;
}

// Counts, for every (target, source) pair, how many times the standard-mode lists account
// for it (M2L at any ancestor pair, or direct). Every entry of count[m * n] must be 1.
void orc_coverage(int cap, int64_t n, const double* src, int64_t m, const double* tgt, const double* center, double H,
                  int32_t* count)
{
   Tree t;
   buildTree(t, src, n, tgt, m, center, H, cap, g_capT > 0 ? g_capT : cap);
   buildLists(t);
   std::memset(count, 0, sizeof(int32_t) * n * m);
   auto addRange = [&](int64_t t0, int64_t t1, int64_t s0, int64_t s1) {
      for(int64_t a = t0; a < t1; a++)
         for(int64_t b = s0; b < s1; b++) count[t.tgtOrder[a] * n + t.srcOrder[b]]++;
   };
   for(size_t i = 0; i < t.nodes.size(); i++)
   {
      const Node& D = t.nodes[i];
      for(int S : t.V[i]) addRange(D.t0, D.t1, t.nodes[S].s0, t.nodes[S].s1);
      if(D.leaf())
      {
         for(int S : t.U[i]) addRange(D.t0, D.t1, t.nodes[S].s0, t.nodes[S].s1);
         for(int S : t.W[i]) addRange(D.t0, D.t1, t.nodes[S].s0, t.nodes[S].s1);
      }
      for(int S : t.X[i]) addRange(D.t0, D.t1, t.nodes[S].s0, t.nodes[S].s1);
   }
}

}
