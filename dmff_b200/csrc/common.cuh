// Shared device helpers for the ADMP / PME engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#define DMFFB_DIELECTRIC 1389.35455846  // dmff/common/constants.py:3
#define DMFFB_SQRT3 1.7320508075688772
#define DMFFB_RT3_REF 1.73205080757      // dmff/admp/multipole.py:13 (truncated, used in C2_gl)
#define DMFFB_TWO_OVER_SQRTPI 1.1283791670955126

namespace dmffb {

// ------------------------------------------------------------------ math wrappers
__device__ __forceinline__ float d_erfc(float x) { return erfcf(x); }
__device__ __forceinline__ double d_erfc(double x) { return erfc(x); }
__device__ __forceinline__ float d_erf(float x) { return erff(x); }
__device__ __forceinline__ double d_erf(double x) { return erf(x); }
__device__ __forceinline__ float d_exp(float x) { return expf(x); }
__device__ __forceinline__ double d_exp(double x) { return exp(x); }
__device__ __forceinline__ float d_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double d_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float d_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double d_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float d_floor(float x) { return floorf(x); }
__device__ __forceinline__ double d_floor(double x) { return floor(x); }

// value + derivative with respect to the pair distance r
template <typename T>
struct Dl {
    T v, d;
    __device__ __forceinline__ Dl() {}
    __device__ __forceinline__ Dl(T v_, T d_) : v(v_), d(d_) {}
};
template <typename T> __device__ __forceinline__ Dl<T> operator+(Dl<T> a, Dl<T> b) { return Dl<T>(a.v + b.v, a.d + b.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator-(Dl<T> a, Dl<T> b) { return Dl<T>(a.v - b.v, a.d - b.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator*(Dl<T> a, Dl<T> b) { return Dl<T>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator*(T s, Dl<T> a) { return Dl<T>(s * a.v, s * a.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator+(T s, Dl<T> a) { return Dl<T>(s + a.v, a.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator-(Dl<T> a) { return Dl<T>(-a.v, -a.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator*(Dl<T> a, T s) { return Dl<T>(a.v * s, a.d * s); }
template <typename T> __device__ __forceinline__ Dl<T> operator+(Dl<T> a, T s) { return Dl<T>(a.v + s, a.d); }
template <typename T> __device__ __forceinline__ Dl<T> operator-(Dl<T> a, T s) { return Dl<T>(a.v - s, a.d); }

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Segmented sums over runs of equal keys in a warp.  A key may appear in several runs (rows
// skipped by a launch sit between rows of the same atom), so runs are identified by a run id:
// the number of run heads up to and including the lane.  After seg_sum, the head lane of each
// run holds that run's total.
__device__ __forceinline__ bool seg_head(int key) {
    const int lane = threadIdx.x & 31;
    int prev = __shfl_up_sync(0xffffffffu, key, 1);
    return lane == 0 || prev != key;
}
__device__ __forceinline__ int seg_run_id(int key) {
    const int lane = threadIdx.x & 31;
    const unsigned heads = __ballot_sync(0xffffffffu, seg_head(key));
    return __popc(heads & (0xffffffffu >> (31 - lane)));
}
template <typename T>
__device__ __forceinline__ T seg_sum(T v, int run) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T ov = __shfl_down_sync(0xffffffffu, v, o);
        int orun = __shfl_down_sync(0xffffffffu, run, o);
        if (lane + o < 32 && orun == run) v += ov;
    }
    return v;
}

// block-wide reduction of NV doubles into dst[] with one atomicAdd per value per block
template <int NV>
__device__ __forceinline__ void block_reduce_add(double (&v)[NV], double* dst) {
    __shared__ double sh[32][NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[wid][k] = v[k];
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nw ? sh[lane][k] : 0.0;
            s = warp_sum(s);
            if (lane == 0 && s != 0.0) atomicAdd(dst + k, s);
        }
    }
    __syncthreads();  // the shared buffer may be reused by the next call
}

// ------------------------------------------------------------------ box
struct Box {
    double h[9];     // rows = lattice vectors
    double hinv[9];  // inverse
};

template <typename T>
struct BoxT {
    T h[9], hinv[9];
};

// minimum image as the reference's pbc_shift (spatial.py:14-32): ds = dr hinv; n = floor(ds+1/2);
// dr = (ds - n) h.  Returns n through nout.
template <typename T>
__device__ __forceinline__ void pbc_shift(const BoxT<T>& b, T& x, T& y, T& z, T* nout) {
    T s0 = x * b.hinv[0] + y * b.hinv[3] + z * b.hinv[6];
    T s1 = x * b.hinv[1] + y * b.hinv[4] + z * b.hinv[7];
    T s2 = x * b.hinv[2] + y * b.hinv[5] + z * b.hinv[8];
    T n0 = d_floor(s0 + T(0.5)), n1 = d_floor(s1 + T(0.5)), n2 = d_floor(s2 + T(0.5));
    s0 -= n0; s1 -= n1; s2 -= n2;
    x = s0 * b.h[0] + s1 * b.h[3] + s2 * b.h[6];
    y = s0 * b.h[1] + s1 * b.h[4] + s2 * b.h[7];
    z = s0 * b.h[2] + s1 * b.h[5] + s2 * b.h[8];
    if (nout) { nout[0] = n0; nout[1] = n1; nout[2] = n2; }
}

}  // namespace dmffb
