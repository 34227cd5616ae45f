// Reciprocal convolution of the dipole-solve iterations in one thread-block cluster:
// real mesh -> forward 3-D FFT -> multiply by the influence function -> inverse 3-D FFT -> real
// mesh, for meshes of up to 64 points per axis (FP32).
//
// Each CG iteration of the induced-dipole solve convolves the spread dipole mesh with the
// Coulomb influence function G(k) = C(k^2) / |theta(k)|^2 (recip.py:440-466; the reference runs a
// full complex fftn of the mesh inside jax.grad, recip.py:450).  With cuFFT that is an R2C
// transform (three kernels), a convolution kernel and a C2R transform (three kernels) on a mesh
// that fits in L2: seven dependent launches of a few microseconds each.  Here one cluster of CL
// CTAs holds the whole half spectrum in distributed shared memory:
//   phase A (each CTA, its own x-planes x = c, c + CL, ...): load the plane's real rows, complex
//           FFT along z of the zero-imaginary rows (keeping kz < K3/2 + 1), FFT along y; the spread
//           mesh plane is cleared for the next spread;
//   cluster barrier;
//   phase B (each CTA, columns (ky, kz) = c, c + CL, ... in chunks): read the column's K1 values
//           from the CTAs that own them (DSMEM), FFT along x, multiply by G, inverse FFT along x,
//           write the column back (DSMEM);
//   cluster barrier;
//   phase C (each CTA, its planes): inverse FFT along y, Hermitian completion of every row and
//           inverse complex FFT along z, real part out to the global mesh.
// Transforms are unnormalised in both directions (the cuFFT convention the gather expects).
//
// Line FFTs: Stockham autosort over the factors of the line length (radices 4, 2, 3, 5, 7; meshes
// with another prime factor take cuFFT), one radix-R butterfly per thread and stage: inputs
// x[j + t N / R] times the stage twiddles W_{Ns R}^{t k} (k = j mod Ns, precomputed per stage in
// shared memory, conjugated for the inverse), a hard-coded R-point DFT, outputs to
// y[(j - k) R + k + u Ns].
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"

namespace dmffb {

constexpr int kFcMaxK = 64;      // largest mesh extent per axis
constexpr int kFcMaxFactors = 8;
constexpr int kFcThreads = 512;
constexpr int kFcChunk = 32;      // phase-B columns per round

struct FcPlan {
    int n;                         // line length
    int nf;                        // factors
    int f[kFcMaxFactors];          // radices in order
};

struct FftConvArgs {
    int K[3];
    int Kh;                        // K[2] / 2 + 1
    int cl;                        // CTAs in the cluster
    float* grid_in;                // [K1*K2*K3] spread mesh (cleared by the kernel)
    float* grid_out;               // [K1*K2*K3] convolved mesh
    const float* G;                // [K1*K2*Kh] influence function over the half spectrum
    FcPlan px, py, pz;
};

// radices 4, 2, 3, 5, 7 in that order; ok = false when another prime factor remains (such meshes
// take the cuFFT path)
__host__ inline FcPlan fc_plan(int n, bool* ok = nullptr) {
    FcPlan p;
    p.n = n;
    p.nf = 0;
    int m = n;
    for (int r : {4, 2, 3, 5, 7}) {
        while (m % r == 0 && p.nf < kFcMaxFactors) {
            p.f[p.nf++] = r;
            m /= r;
        }
    }
    if (ok) *ok = (m == 1);
    return p;
}

// twiddles of every stage of a line length: for stage s (span Ns, radix R) the R x Ns table
// W_{Ns R}^{t k} at off_s + k R + t; total size sum_s Ns R <= 2 n
__host__ __device__ inline int fc_tw_size(const FcPlan& p) {
    int ns = 1, tot = 0;
    for (int s = 0; s < p.nf; ++s) {
        tot += ns * p.f[s];
        ns *= p.f[s];
    }
    return tot;
}

__device__ inline void fc_twiddles(float2* tw, const FcPlan& p, int tid, int nth) {
    int ns = 1, off = 0;
    for (int s = 0; s < p.nf; ++s) {
        const int R = p.f[s];
        for (int e = tid; e < ns * R; e += nth) {
            const int k = e / R, t = e % R;
            double sn, cs;
            sincospi(-2.0 * (double)(t * k) / (double)(ns * R), &sn, &cs);
            tw[off + e] = make_float2((float)cs, (float)sn);
        }
        off += ns * R;
        ns *= R;
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// in-place DFT of R points, V[u] = sum_t v[t] exp(-+2 pi i t u / R)
template <int R>
__device__ __forceinline__ void fc_dft(float2 (&v)[R], bool inv) {
    const float sg = inv ? 1.f : -1.f;
    if (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = make_float2(a.x + b.x, a.y + b.y);
        v[1] = make_float2(a.x - b.x, a.y - b.y);
    } else if (R == 4) {
        const float2 a = v[0], b = v[1], c = v[2], d = v[3];
        const float2 s0 = make_float2(a.x + c.x, a.y + c.y), d0 = make_float2(a.x - c.x, a.y - c.y);
        const float2 s1 = make_float2(b.x + d.x, b.y + d.y), d1 = make_float2(b.x - d.x, b.y - d.y);
        // -i sg-rotation of d1: multiply by exp(sg i pi / 2) = sg i
        const float2 r1 = make_float2(-sg * d1.y, sg * d1.x);
        v[0] = make_float2(s0.x + s1.x, s0.y + s1.y);
        v[2] = make_float2(s0.x - s1.x, s0.y - s1.y);
        v[1] = make_float2(d0.x + r1.x, d0.y + r1.y);
        v[3] = make_float2(d0.x - r1.x, d0.y - r1.y);
    } else if (R == 3) {
        const float c1 = -0.5f, s1 = sg * 0.86602540378443865f;
        const float2 a = v[0], b = v[1], c = v[2];
        const float2 t = make_float2(b.x + c.x, b.y + c.y), u = make_float2(b.x - c.x, b.y - c.y);
        v[0] = make_float2(a.x + t.x, a.y + t.y);
        const float2 m = make_float2(a.x + c1 * t.x, a.y + c1 * t.y);
        v[1] = make_float2(m.x - s1 * u.y, m.y + s1 * u.x);
        v[2] = make_float2(m.x + s1 * u.y, m.y - s1 * u.x);
    } else if (R == 5) {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
        const float s1 = sg * 0.95105651629515357f, s2 = sg * 0.58778525229247313f;
        const float2 a = v[0];
        const float2 t1 = make_float2(v[1].x + v[4].x, v[1].y + v[4].y), u1 = make_float2(v[1].x - v[4].x, v[1].y - v[4].y);
        const float2 t2 = make_float2(v[2].x + v[3].x, v[2].y + v[3].y), u2 = make_float2(v[2].x - v[3].x, v[2].y - v[3].y);
        v[0] = make_float2(a.x + t1.x + t2.x, a.y + t1.y + t2.y);
        const float2 m1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        const float2 m2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        const float2 n1 = make_float2(s1 * u1.x + s2 * u2.x, s1 * u1.y + s2 * u2.y);
        const float2 n2 = make_float2(s2 * u1.x - s1 * u2.x, s2 * u1.y - s1 * u2.y);
        // V1 = m1 + i n1, V4 = m1 - i n1, V2 = m2 + i n2, V3 = m2 - i n2
        v[1] = make_float2(m1.x - n1.y, m1.y + n1.x);
        v[4] = make_float2(m1.x + n1.y, m1.y - n1.x);
        v[2] = make_float2(m2.x - n2.y, m2.y + n2.x);
        v[3] = make_float2(m2.x + n2.y, m2.y - n2.x);
    } else {  // R == 7: direct sum over cos / sin(2 pi m / 7)
        constexpr float c7[7] = {1.f, 0.62348980185873353f, -0.22252093395631440f, -0.90096886790241913f,
                                 -0.90096886790241913f, -0.22252093395631440f, 0.62348980185873353f};
        constexpr float s7[7] = {0.f, 0.78183148246802981f, 0.97492791218182361f, 0.43388373911755812f,
                                 -0.43388373911755812f, -0.97492791218182361f, -0.78183148246802981f};
        float2 w[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            float2 acc = v[0];
#pragma unroll
            for (int t = 1; t < R; ++t) {
                const float cs = c7[(t * u) % R], sn = sg * s7[(t * u) % R];
                acc.x += v[t].x * cs - v[t].y * sn;
                acc.y += v[t].x * sn + v[t].y * cs;
            }
            w[u] = acc;
        }
#pragma unroll
        for (int u = 0; u < R; ++u) v[u] = w[u];
    }
}

// one Stockham stage of radix R over nl lines: butterfly j of a line reads x[j + t N / R], twiddles
// by W_{Ns R}^{t k} (k = j mod Ns), transforms, and writes y[(j - k) R + k + u Ns]
template <int R>
__device__ inline void fc_stage(const float2* in, int lin, int ein, float2* out, int lout, int eout, int nl, int N,
                                int Ns, const float2* tw, bool inv, int tid, int nth) {
    const int nb = N / R;
    for (int e = tid; e < nl * nb; e += nth) {
        const int l = e / nb, j = e - l * nb;
        const int k = j % Ns;
        float2 v[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
            v[t] = in[l * lin + (j + t * nb) * ein];
            if (t > 0) {
                float2 w = tw[k * R + t];
                if (inv) w.y = -w.y;
                v[t] = cmul(v[t], w);
            }
        }
        fc_dft<R>(v, inv);
        const int d0 = (j - k) * R + k;
#pragma unroll
        for (int u = 0; u < R; ++u) out[l * lout + (d0 + u * Ns) * eout] = v[u];
    }
}

// nl lines of length p.n, line l at base[l * lstride] with element stride es, transformed in
// place through the dense scratch scr (>= nl * p.n elements, line-major); inverse = conjugate
// twiddles, unnormalised
__device__ inline void fc_lines(const FcPlan& p, float2* base, int nl, int lstride, int es, float2* scr,
                                const float2* tw, bool inverse, int tid, int nth) {
    const int N = p.n;
    if (N == 1) return;
    int Ns = 1, off = 0;
    for (int s = 0; s < p.nf; ++s) {
        const int R = p.f[s];
        const bool from_lines = (s % 2 == 0);
        const float2* in = from_lines ? base : scr;
        float2* out = from_lines ? scr : base;
        const int lin = from_lines ? lstride : N, ein = from_lines ? es : 1;
        const int lout = from_lines ? N : lstride, eout = from_lines ? 1 : es;
        switch (R) {
            case 2: fc_stage<2>(in, lin, ein, out, lout, eout, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 3: fc_stage<3>(in, lin, ein, out, lout, eout, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 4: fc_stage<4>(in, lin, ein, out, lout, eout, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 5: fc_stage<5>(in, lin, ein, out, lout, eout, nl, N, Ns, tw + off, inverse, tid, nth); break;
            default: fc_stage<7>(in, lin, ein, out, lout, eout, nl, N, Ns, tw + off, inverse, tid, nth); break;
        }
        __syncthreads();
        off += Ns * R;
        Ns *= R;
    }
    if (p.nf % 2 == 1) {  // the result sits in the scratch: copy it back to the lines
        for (int e = tid; e < nl * N; e += nth) {
            const int l = e / N, o = e - l * N;
            base[l * lstride + o * es] = scr[l * N + o];
        }
        __syncthreads();
    }
}

// Shared memory: [planes: P * K2 * Kh float2][work: max(2 * K2 * K3, 2 * chunk * K1) float2]
// [stage twiddles: 3 * 2 * kFcMaxK float2]
__host__ inline size_t fc_smem_bytes(const int K[3], int cl) {
    const int Kh = K[2] / 2 + 1;
    const int P = (K[0] + cl - 1) / cl;
    size_t work = (size_t)2 * K[1] * K[2];
    work = work > (size_t)2 * kFcChunk * K[0] ? work : (size_t)2 * kFcChunk * K[0];
    return ((size_t)P * K[1] * Kh + work + 3 * 2 * kFcMaxK) * sizeof(float2);
}

__global__ void __launch_bounds__(kFcThreads) k_fftconv_cluster(FftConvArgs a) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ float2 sm[];
    const int K1 = a.K[0], K2 = a.K[1], K3 = a.K[2], Kh = a.Kh, cl = a.cl;
    const int c = (int)cluster.block_rank();
    const int tid = threadIdx.x, nth = blockDim.x;
    const int P = (K1 + cl - 1) / cl;
    float2* planes = sm;                                  // [P][K2][Kh]
    float2* work = planes + (size_t)P * K2 * Kh;
    size_t wsz = (size_t)2 * K2 * K3;
    if (wsz < (size_t)2 * kFcChunk * K1) wsz = (size_t)2 * kFcChunk * K1;
    float2* twx = work + wsz;
    float2* twy = twx + 2 * kFcMaxK;
    float2* twz = twy + 2 * kFcMaxK;
    fc_twiddles(twx, a.px, tid, nth);
    fc_twiddles(twy, a.py, tid, nth);
    fc_twiddles(twz, a.pz, tid, nth);
    __syncthreads();
    const int my_planes = c < K1 ? (K1 - 1 - c) / cl + 1 : 0;
    // ---- phase A: z (real rows as complex, keep kz < Kh) then y, per owned plane
    for (int pl = 0; pl < my_planes; ++pl) {
        const int x = c + pl * cl;
        float2* rows = work;                              // [K2][K3]
        float2* scr = work + (size_t)K2 * K3;
        float* gin = a.grid_in + (size_t)x * K2 * K3;
        for (int e = tid; e < K2 * K3; e += nth) {
            rows[e] = make_float2(gin[e], 0.f);
            gin[e] = 0.f;                                 // the next spread starts from zero
        }
        __syncthreads();
        fc_lines(a.pz, rows, K2, K3, 1, scr, twz, false, tid, nth);
        float2* plane = planes + (size_t)pl * K2 * Kh;    // [K2][Kh]
        for (int e = tid; e < K2 * Kh; e += nth) plane[e] = rows[(e / Kh) * K3 + (e % Kh)];
        __syncthreads();
        fc_lines(a.py, plane, Kh, 1, Kh, scr, twy, false, tid, nth);
    }
    cluster.sync();
    // ---- phase B: columns (ky, kz) across the x-planes of the whole cluster
    const int ncol = K2 * Kh;
    for (int c0 = c; c0 < ncol; c0 += cl * kFcChunk) {
        int nc = 0;
        for (int q = 0; q < kFcChunk; ++q)
            if (c0 + q * cl < ncol) nc = q + 1;
        float2* col = work;                               // [nc][K1]
        float2* scr = work + (size_t)kFcChunk * K1;
        for (int e = tid; e < nc * K1; e += nth) {
            const int q = e / K1, x = e % K1;
            const int cc = c0 + q * cl;
            float2* remote = cluster.map_shared_rank(planes, x % cl);
            col[e] = remote[(size_t)(x / cl) * K2 * Kh + cc];
        }
        __syncthreads();
        fc_lines(a.px, col, nc, K1, 1, scr, twx, false, tid, nth);
        for (int e = tid; e < nc * K1; e += nth) {
            const int q = e / K1, kx = e % K1;
            const int cc = c0 + q * cl;
            const float g = a.G[(size_t)kx * ncol + cc];  // [kx][ky][kz] = kx * K2 * Kh + cc
            col[e].x *= g;
            col[e].y *= g;
        }
        __syncthreads();
        fc_lines(a.px, col, nc, K1, 1, scr, twx, true, tid, nth);
        for (int e = tid; e < nc * K1; e += nth) {
            const int q = e / K1, x = e % K1;
            const int cc = c0 + q * cl;
            float2* remote = cluster.map_shared_rank(planes, x % cl);
            remote[(size_t)(x / cl) * K2 * Kh + cc] = col[e];
        }
        __syncthreads();
    }
    cluster.sync();
    // ---- phase C: inverse y, then Hermitian rows and inverse z, real part out
    for (int pl = 0; pl < my_planes; ++pl) {
        const int x = c + pl * cl;
        float2* plane = planes + (size_t)pl * K2 * Kh;
        float2* rows = work;
        float2* scr = work + (size_t)K2 * K3;
        fc_lines(a.py, plane, Kh, 1, Kh, scr, twy, true, tid, nth);
        for (int e = tid; e < K2 * K3; e += nth) {
            const int y = e / K3, z = e % K3;
            const float2 v = z < Kh ? plane[y * Kh + z] : plane[y * Kh + (K3 - z)];
            rows[e] = z < Kh ? v : make_float2(v.x, -v.y);
        }
        __syncthreads();
        fc_lines(a.pz, rows, K2, K3, 1, scr, twz, true, tid, nth);
        float* gout = a.grid_out + (size_t)x * K2 * K3;
        for (int e = tid; e < K2 * K3; e += nth) gout[e] = rows[e].x;
        __syncthreads();
    }
}

// influence function table over the half spectrum (the multiplier of k_conv for Coulomb, k = 0
// excluded), kernel precision FP32
__global__ void k_fc_gtable(int K1, int K2, int K3, int Kh, Box b, const double* bmod, double kappa, double V,
                            float* G) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)K1 * K2 * Kh;
    if (idx >= total) return;
    const int k3 = (int)(idx % Kh);
    const int k2 = (int)((idx / Kh) % K2);
    const int k1 = (int)(idx / ((int64_t)Kh * K2));
    const int m1 = k1 < (K1 + 1) / 2 ? k1 : k1 - K1;
    const int m2 = k2 < (K2 + 1) / 2 ? k2 : k2 - K2;
    const int m3 = k3 < (K3 + 1) / 2 ? k3 : k3 - K3;
    const double TWO_PI = 6.283185307179586;
    double kv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) kv[c] = TWO_PI * (b.hinv[3 * c] * m1 + b.hinv[3 * c + 1] * m2 + b.hinv[3 * c + 2] * m3);
    const double ksq = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
    const double th = bmod[k1] * bmod[K1 + k2] * bmod[K1 + K2 + k3];
    double g = 0.0;
    if (!(m1 == 0 && m2 == 0 && m3 == 0)) {
        const double C = 2.0 * 3.141592653589793 / V / ksq * exp(-ksq / 4.0 / (kappa * kappa));
        g = C / (th * th);
    }
    G[idx] = (float)g;
}

}  // namespace dmffb
