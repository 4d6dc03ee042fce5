#!/usr/bin/env bash
# Builds the reference FMM (FMM/FMMGPU of iamwhoamianamy/bachelors) CPU path as
# shared libraries under oracle/_ref/, for use as a checker and as the timed CPU
# baseline. Nothing built here is product code.
#
# The reference is a Visual Studio project; it is compiled here directly with g++
# from its own translation units after the minimal patches listed below, applied to
# a scratch copy under oracle/_ref/src_* (never to the reference tree):
#   real type      real.hpp               REAL_IS_FLOAT -> REAL_IS_DOUBLE for the FP64 build
#   C++17 ctors    harmonic_series.hpp    in-class "HarmonicSeries<T>(" -> "HarmonicSeries("
#   MSVC-only      *.cpp                  std::exception("msg") -> std::runtime_error("msg")
#   C++20 init     calculation_point_octree.cpp  emplace_back(a, b, this) -> push_back({a, b, this})
#   order          multipole_solver.hpp   harmonicOrder = 10 -> FMM_ORDER (compile-time -D)
#   factorials     factorials.{hpp,cpp}   size_t operator[] -> real operator[] (p >= 11 overflows otherwise)
# OpenBLAS is replaced by a naive CBLAS shim and the GPU entry points by aborting stubs.
#
# Usage: oracle/ref/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REPO="$(cd "$HERE/../.." && pwd)"
REF="${1:-/root/reference}"
SRC="$REF/FMM/FMMGPU"
OUT="$REPO/oracle/_ref"
if [ ! -d "$SRC" ]; then
   echo "reference sources not found at $SRC; skipping reference build" >&2
   exit 0
fi
mkdir -p "$OUT"
TUS="harmonics multipole_translator math factorials box quadrature integration quadrature_octree \
calculation_point_octree multipole_solver fast_multipole_solver translation_algorithms_cpu blass_callers \
tetrahedron triangle bem_quadrature reference_cylinder_data hexahedron torus basis_quadratures exeptions \
testing_helpers cylinder"
CUDA_INC=/usr/local/cuda/include
CUDA_LIB=/usr/local/cuda/lib64

prepare() { # $1 = dir, $2 = float|double
   local d="$1"
   rm -rf "$d"; mkdir -p "$d"
   cp "$SRC"/*.cpp "$SRC"/*.hpp "$SRC"/*.cuh "$SRC"/vector3.cu "$d"/
   rm -f "$d/main.cpp"
   # strip UTF-8 byte order marks
   sed -i '1s/^\xEF\xBB\xBF//' "$d"/*.cpp "$d"/*.hpp "$d"/*.cuh "$d"/vector3.cu
   if [ "$2" = double ]; then
      sed -i 's/^#define REAL_IS_FLOAT/\/\/#define REAL_IS_FLOAT/; s/^\/\/#define REAL_IS_DOUBLE/#define REAL_IS_DOUBLE/' "$d/real.hpp"
   fi
   sed -i 's/^   HarmonicSeries<T>(/   HarmonicSeries(/' "$d/harmonic_series.hpp"
   sed -i 's/std::exception("/std::runtime_error("/g' "$d"/*.cpp
   sed -i 's/result\.emplace_back(\*point, aInPoint , this);/result.push_back({*point, aInPoint, this});/; s/result\.emplace_back(\*point, res, this);/result.push_back({*point, res, this});/' "$d/calculation_point_octree.cpp"
   sed -i 's/const int harmonicOrder = 10;/const int harmonicOrder = FMM_ORDER;/' "$d/multipole_solver.hpp"
   sed -i 's/size_t operator\[\](size_t i) const;/real operator[](size_t i) const;/' "$d/factorials.hpp"
   sed -i 's/^size_t Factorials::operator\[\]/real Factorials::operator[]/' "$d/factorials.cpp"
   grep -q 'real operator\[\]' "$d/factorials.hpp"
   grep -q 'FMM_ORDER' "$d/multipole_solver.hpp"
}

build() { # $1 = float|double, $2 = order, $3 = output name
   local d="$OUT/src_$1"
   local o="$OUT/obj_$1_p$2"
   mkdir -p "$o"
   local flags="-std=c++17 -fpermissive -w -O3 -march=native -fopenmp -fPIC -DFMM_ORDER=$2 -I$d -I$HERE/shim -I$CUDA_INC"
   local objs=""
   for t in $TUS; do
      g++ $flags -c "$d/$t.cpp" -o "$o/$t.o" &
      objs="$objs $o/$t.o"
   done
   g++ $flags -x c++ -c "$d/vector3.cu" -o "$o/vector3.o" &
   g++ $flags -c "$HERE/shim/cblas_shim.cpp" -o "$o/cblas_shim.o" &
   g++ $flags -c "$HERE/shim/gpu_stubs.cpp" -o "$o/gpu_stubs.o" &
   g++ $flags -c "$HERE/ref_driver.cpp" -o "$o/ref_driver.o" &
   wait
   g++ -shared -fopenmp -o "$OUT/$3" $objs "$o/vector3.o" "$o/cblas_shim.o" "$o/gpu_stubs.o" "$o/ref_driver.o" \
      -L$CUDA_LIB -Wl,-rpath,$CUDA_LIB -lcublas -lcudart
   echo "built $OUT/$3"
}

prepare "$OUT/src_double" double
prepare "$OUT/src_float" float
# FP64 pipelines at the orders the tests and the CPU baseline use; FP32 for the FP32 workloads.
build double 10 libref_fmm_f64_p10.so
build double 12 libref_fmm_f64_p12.so
build double 16 libref_fmm_f64_p16.so
build float 12 libref_fmm_f32_p12.so
build float 16 libref_fmm_f32_p16.so
