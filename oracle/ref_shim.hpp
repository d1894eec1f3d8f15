// Test infrastructure only: a CPU execution model for the reference's inline
// CUDA C kernels, so that they can be compiled by g++ and run on the host as
// the checker of the CUDA product.  Nothing in the product includes this.
//
// Each CUDA thread of a block runs as a ucontext fiber on one OS thread;
// __syncthreads() switches fibers until every live fiber of the block has
// reached the barrier.  `__shared__` becomes `static thread_local`, which all
// fibers of the block share because a block never leaves its OS thread.
// Blocks are spread over a pool of OS threads.
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
#include <functional>

struct vt_dim3 {
    unsigned x, y, z;
};

struct vt_fiber;
extern thread_local vt_fiber* vt_cur_fiber;
extern thread_local vt_dim3 vt_block_idx;
extern thread_local vt_dim3 vt_block_dim;
extern thread_local vt_dim3 vt_grid_dim;
const vt_dim3& vt_thread_idx();

#define threadIdx (vt_thread_idx())
#define blockIdx (vt_block_idx)
#define blockDim (vt_block_dim)
#define gridDim (vt_grid_dim)
#define __global__
#define __device__
#define __shared__ static thread_local

void __syncthreads();

// Runs `body` for every thread of every block.  `os_threads` <= 0 uses all
// hardware threads.
void vt_launch(vt_dim3 grid, vt_dim3 block, const std::function<void()>& body, int os_threads);

// CUDA math/builtins the kernels use that the C++ library spells otherwise.
inline void sincos(double x, double* s, double* c) { *s = std::sin(x); *c = std::cos(x); }
inline void sincosf(float x, float* s, float* c) { *s = std::sin(x); *c = std::cos(x); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
using std::cos;
using std::exp;
using std::fabs;
using std::sin;
using std::sqrt;

namespace pycuda {
template <class T>
using complex = std::complex<T>;
template <class T>
inline T real(const std::complex<T>& z) { return z.real(); }
template <class T>
inline T imag(const std::complex<T>& z) { return z.imag(); }
}  // namespace pycuda
