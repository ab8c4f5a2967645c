// Test infrastructure (oracle): build configuration for compiling the
// reference's gravity sources directly (oracle/Makefile.ref) instead of through
// its CMake project. Values chosen for this oracle build: OpenMP on, FFTW on
// (served by oracle/fftw_shim), MPI/HDF5/CUDA/Python off. The macro names are
// those the reference's sources test (cmake/templates/build_config.hpp.in).
#pragma once

#define COSMOSIM_BUILD_PRESET "chui-b200-oracle"
#define COSMOSIM_BUILD_TYPE "Release"
#define COSMOSIM_CXX_FLAGS "-O3 -march=x86-64-v3 -fopenmp"
#define COSMOSIM_SOURCE_GIT "unknown"
#define COSMOSIM_SOURCE_IDENTITY "oracle-direct-build"
#define COSMOSIM_SOURCE_MANIFEST_SHA256 "unknown"
#define COSMOSIM_BUILD_COMPILER "GNU"
#define COSMOSIM_DEPENDENCY_PROVIDERS "fftw=oracle-shim"
#define COSMOSIM_ENABLE_NATIVE_CPU 0

#define COSMOSIM_ENABLE_MPI 0
#define COSMOSIM_HAVE_OPENMP 1
#define COSMOSIM_ENABLE_HDF5 0
#define COSMOSIM_HDF5_PARALLEL 0
#define COSMOSIM_ENABLE_FFTW 1
#define COSMOSIM_ENABLE_CUDA 0
#define COSMOSIM_ENABLE_PYTHON 0
#define COSMOSIM_ENABLE_TRACERS 0
#define COSMOSIM_ENABLE_TESTS 0
#define COSMOSIM_ENABLE_BENCHMARKS 0
#define COSMOSIM_ENABLE_LTO 0
#define COSMOSIM_ENABLE_PROFILING 0
