// Reciprocal convolution of the dipole-solve iterations in three kernels of the engine's own
// FFT: real mesh -> forward 3-D FFT -> multiply by the influence function -> inverse 3-D FFT ->
// real mesh, for meshes of up to 64 points per axis (FP32).
//
// Each CG iteration of the induced-dipole solve convolves the spread dipole mesh with the
// Coulomb influence function G(k) = C(k^2) / |theta(k)|^2 (recip.py:440-466; the reference runs a
// full complex fftn of the mesh inside jax.grad, recip.py:450).  With cuFFT that is an R2C
// transform, a separate convolution kernel and a C2R transform on a mesh that fits in L2, each
// latency-bound.  Here:
//   k_fc_fwd_planes (one CTA per x-plane): two real rows packed per complex row, FFT along z,
//           half spectra separated, FFT along y, half spectrum out; the spread plane is cleared;
//   k_fc_columns (kFcCols spectrum columns (ky, kz) per CTA): FFT along x, times G, inverse FFT
//           along x, in place;
//   k_fc_inv_planes (one CTA per x-plane): inverse FFT along y, Hermitian completion of row pairs
//           packed as A + i B, inverse FFT along z, the two real rows out.
// Transforms are unnormalised in both directions (the cuFFT convention the gather expects).
//
// Line FFTs: Stockham autosort over the factors of the line length (radices 4, 2, 3, 5, 7, then a
// remaining prime as one generic stage of O(R) work per output), one radix-R butterfly per thread
// and stage for the hard-coded radices: inputs
// x[j + t N / R] times the stage twiddles W_{Ns R}^{t k} (k = j mod Ns, precomputed per stage in
// shared memory, conjugated for the inverse), a hard-coded R-point DFT, outputs to
// y[(j - k) R + k + u Ns].
#pragma once
#include <cmath>

#include "common.cuh"

namespace dmffb {

constexpr int kFcMaxK = 64;      // largest mesh extent per axis
constexpr int kFcMaxFactors = 8;
constexpr int kFcPlaneThreads = 512;
constexpr int kFcColThreads = 256;
constexpr int kFcCols = 8;        // spectrum columns per CTA of the column pass
constexpr int kFcTw = 2 * kFcMaxK;  // stage twiddles of one line length (sum over stages of Ns R < 2 n)

struct FcPlan {
    int n;                         // line length
    int nf;                        // factors
    int f[kFcMaxFactors];          // radices in order
};

struct FftConvArgs {
    int K[3];
    int Kh;                        // K[2] / 2 + 1
    float* grid_in;                // [K1*K2*K3] spread mesh (cleared by the forward pass)
    float* grid_out;               // [K1*K2*K3] convolved mesh
    float2* spec;                  // [K1][K2][Kh] half spectrum between the passes
    const float* G;                // [K1*K2*Kh] influence function over the half spectrum
    FcPlan px, py, pz;
    float2 tw[3][kFcTw];           // stage twiddles of the x, y and z line lengths
};

// radices 4, 2, 3, 5, 7 in that order, then the remaining factor (a prime above 7, n <= 64) as one
// generic stage; ok = false when n is out of range
__host__ inline FcPlan fc_plan(int n, bool* ok = nullptr) {
    FcPlan p;
    p.n = n;
    p.nf = 0;
    int m = n;
    for (int r : {4, 2, 3, 5, 7}) {
        while (m % r == 0 && p.nf < kFcMaxFactors - 1) {
            p.f[p.nf++] = r;
            m /= r;
        }
    }
    if (m > 1) p.f[p.nf++] = m;
    if (ok) *ok = n >= 2 && n <= kFcMaxK;
    return p;
}

__host__ __device__ inline bool fc_hardcoded(int R) { return R == 2 || R == 3 || R == 4 || R == 5 || R == 7; }

// stage twiddles of a line length, Ns R entries per stage (span Ns, radix R) at off_s (the sum of
// Ns R over the earlier stages, < 2 n in all): W_{Ns R}^{t k} at off_s + k R + t for a hard-coded
// radix, W_{Ns R}^m at off_s + m for the generic stage; FP64 on the host rounded to FP32
__host__ inline void fc_host_twiddles(const FcPlan& p, float2* tw) {
    int ns = 1, off = 0;
    for (int s = 0; s < p.nf; ++s) {
        const int R = p.f[s];
        for (int e = 0; e < ns * R; ++e) {
            const int k = e / R, t = e % R;
            const int m = fc_hardcoded(R) ? t * k : e;
            const double ang = -2.0 * 3.14159265358979323846 * (double)m / (double)(ns * R);
            tw[off + e] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        off += ns * R;
        ns *= R;
    }
}

// stage twiddles of one line length from the launch arguments into shared memory
__device__ inline void fc_load_twiddles(float2* dst, const float2* src, int tid, int nth) {
    for (int e = tid; e < kFcTw; e += nth) dst[e] = src[e];
}

// a / d for 0 <= a < 2^20 and 1 <= d <= 2^12 through the FP32 reciprocal rcp = 1 / d: (a + 1/2) / d
// lies at least 1 / (2 d) away from an integer, far above the rounding of the two FP32 operations
__device__ __forceinline__ int fc_div(int a, float rcp) { return __float2int_rd(((float)a + 0.5f) * rcp); }

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

// one Stockham stage of radix R over nl lines (line l at l * ls, element stride es, the same
// layout in and out): butterfly j of a line reads x[j + t N / R], twiddles by W_{Ns R}^{t k}
// (k = j mod Ns), transforms, and writes y[(j - k) R + k + u Ns].  Consecutive threads take
// consecutive lines when lines are interleaved (ls < es), else consecutive butterflies of a line.
template <int R>
__device__ inline void fc_stage(const float2* in, float2* out, int ls, int es, int nl, int N, int Ns,
                                const float2* tw, bool inv, int tid, int nth) {
    const int nb = N / R;
    const bool line_fast = ls < es;
    const float rnl = 1.f / (float)nl, rnb = 1.f / (float)nb, rns = 1.f / (float)Ns;
    for (int e = tid; e < nl * nb; e += nth) {
        int l, j;
        if (line_fast) {
            j = fc_div(e, rnl);
            l = e - j * nl;
        } else {
            l = fc_div(e, rnb);
            j = e - l * nb;
        }
        const int k = j - fc_div(j, rns) * Ns;
        float2 v[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
            v[t] = in[l * ls + (j + t * nb) * es];
            if (t > 0) {
                float2 w = tw[k * R + t];
                if (inv) w.y = -w.y;
                v[t] = cmul(v[t], w);
            }
        }
        fc_dft<R>(v, inv);
        const int d0 = (j - k) * R + k;
#pragma unroll
        for (int u = 0; u < R; ++u) out[l * ls + (d0 + u * Ns) * es] = v[u];
    }
}

// the generic stage (radix R not hard-coded, a prime above 7): one output per thread,
//     y[(j - k) R + k + u Ns] = sum_t x[j + t N / R] W_{Ns R}^{t (k + u Ns)},  k = j mod Ns,
// with W_{Ns R}^m read from the stage's table (conjugated for the inverse)
__device__ inline void fc_stage_generic(const float2* in, float2* out, int ls, int es, int nl, int N, int Ns, int R,
                                        const float2* tw, bool inv, int tid, int nth) {
    const int nb = N / R, span = Ns * R;
    const bool line_fast = ls < es;
    const float rnl = 1.f / (float)nl, rn = 1.f / (float)N, rnb = 1.f / (float)nb, rns = 1.f / (float)Ns;
    for (int e = tid; e < nl * N; e += nth) {
        int l, o;
        if (line_fast) {
            o = fc_div(e, rnl);
            l = e - o * nl;
        } else {
            l = fc_div(e, rn);
            o = e - l * N;
        }
        const int u = fc_div(o, rnb), j = o - u * nb;
        const int k = j - fc_div(j, rns) * Ns;
        const int m = k + u * Ns;
        float2 acc = make_float2(0.f, 0.f);
        int idx = 0;
        for (int t = 0; t < R; ++t) {
            const float2 v = in[l * ls + (j + t * nb) * es];
            float2 w = tw[idx];
            if (inv) w.y = -w.y;
            acc.x += v.x * w.x - v.y * w.y;
            acc.y += v.x * w.y + v.y * w.x;
            idx += m;
            if (idx >= span) idx -= span;
        }
        out[l * ls + ((j - k) * R + k + u * Ns) * es] = acc;
    }
}

// nl lines of length p.n, line l at base[l * ls] with element stride es, transformed in place
// through scratch scr of the same layout; inverse = conjugate twiddles, unnormalised.  Ends with
// a barrier.
__device__ inline void fc_lines(const FcPlan& p, float2* base, int nl, int ls, int es, float2* scr,
                                const float2* tw, bool inverse, int tid, int nth) {
    const int N = p.n;
    int Ns = 1, off = 0;
    for (int s = 0; s < p.nf; ++s) {
        const int R = p.f[s];
        const float2* in = (s % 2 == 0) ? base : scr;
        float2* out = (s % 2 == 0) ? scr : base;
        switch (R) {
            case 2: fc_stage<2>(in, out, ls, es, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 3: fc_stage<3>(in, out, ls, es, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 4: fc_stage<4>(in, out, ls, es, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 5: fc_stage<5>(in, out, ls, es, nl, N, Ns, tw + off, inverse, tid, nth); break;
            case 7: fc_stage<7>(in, out, ls, es, nl, N, Ns, tw + off, inverse, tid, nth); break;
            default: fc_stage_generic(in, out, ls, es, nl, N, Ns, R, tw + off, inverse, tid, nth); break;
        }
        __syncthreads();
        off += Ns * R;
        Ns *= R;
    }
    if (p.nf % 2 == 1) {  // the result sits in the scratch: copy it back to the lines
        const float rnl = 1.f / (float)nl, rn = 1.f / (float)N;
        for (int e = tid; e < nl * N; e += nth) {
            int l, o;
            if (ls < es) {
                o = fc_div(e, rnl);
                l = e - o * nl;
            } else {
                l = fc_div(e, rn);
                o = e - l * N;
            }
            base[l * ls + o * es] = scr[l * ls + o * es];
        }
        __syncthreads();
    }
}

// Shared memory of one plane pass (plane_smem_layout): rows [ceil(K2/2)][K3] (also the scratch of the
// y lines), the z scratch of the same size and the plane [K2][Kh].
struct FcPlaneSmem {
    float2 *rows, *scr, *plane;
};

__device__ inline FcPlaneSmem fc_plane_layout(const FftConvArgs& a, float2* sm) {
    const int K2 = a.K[1], K3 = a.K[2], Kh = a.Kh;
    size_t rsz = (size_t)((K2 + 1) / 2) * K3;
    if (rsz < (size_t)K2 * Kh) rsz = (size_t)K2 * Kh;
    FcPlaneSmem m;
    m.rows = sm;
    m.scr = sm + rsz;
    m.plane = sm + 2 * rsz;
    return m;
}

// Forward pass of x-plane x by one CTA: rows y = 2p, 2p + 1 of the real plane packed as one
// complex row (a + i b), FFT along z, the two half spectra separated
// (A = (C_k + conj C_{-k}) / 2, B = (C_k - conj C_{-k}) / 2i), FFT along y of the [K2][Kh] half
// plane, written to the spectrum W[x][ky][kz]; the spread mesh plane is cleared for the next
// spread.  Mesh and spectrum are read with coherent loads (a persistent caller writes them in the
// same launch).  Ends with a barrier of the CTA.
__device__ inline void fc_fwd_plane(const FftConvArgs& a, int x, float2* sm, const float2* twy, const float2* twz) {
    const int K2 = a.K[1], K3 = a.K[2], Kh = a.Kh;
    const int np = (K2 + 1) / 2;
    const int tid = threadIdx.x, nth = blockDim.x;
    const FcPlaneSmem m = fc_plane_layout(a, sm);
    float* gin = a.grid_in + (size_t)x * K2 * K3;
    const float rk3 = 1.f / (float)K3, rkh = 1.f / (float)Kh;
#pragma unroll 4
    for (int e = tid; e < np * K3; e += nth) {
        const int p = fc_div(e, rk3), z = e - p * K3;
        const int y1 = 2 * p + 1;
        const float re = gin[(2 * p) * K3 + z];
        const float im = y1 < K2 ? gin[y1 * K3 + z] : 0.f;
        m.rows[e] = make_float2(re, im);
    }
    __syncthreads();
    // the next spread starts from zero (this CTA has read its plane)
    for (int e = tid; e < K2 * K3; e += nth) gin[e] = 0.f;
    fc_lines(a.pz, m.rows, np, K3, 1, m.scr, twz, false, tid, nth);
    for (int e = tid; e < K2 * Kh; e += nth) {
        const int y = fc_div(e, rkh), kz = e - y * Kh;
        const float2* r = m.rows + (size_t)(y >> 1) * K3;
        const float2 c = r[kz], mm = r[kz == 0 ? 0 : K3 - kz];  // C_k and C_{-k}
        // even row: (C_k + conj C_-k) / 2; odd row: (C_k - conj C_-k) / 2i
        m.plane[e] = (y & 1) ? make_float2(0.5f * (c.y + mm.y), 0.5f * (mm.x - c.x))
                             : make_float2(0.5f * (c.x + mm.x), 0.5f * (c.y - mm.y));
    }
    __syncthreads();
    fc_lines(a.py, m.plane, Kh, 1, Kh, m.rows, twy, false, tid, nth);
    float2* w = a.spec + (size_t)x * K2 * Kh;
    for (int e = tid; e < K2 * Kh; e += nth) w[e] = m.plane[e];
    __syncthreads();
}

// Columns (ky, kz) = c0 .. c0 + kFcCols - 1 of the spectrum by one CTA: FFT along x, times the
// influence function, inverse FFT along x, in place.  Ends with a barrier of the CTA.
__device__ inline void fc_column_block(const FftConvArgs& a, int c0, float2* sm, const float2* twx) {
    const int K1 = a.K[0], ncol = a.K[1] * a.Kh;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int nc = min(kFcCols, ncol - c0);
    float2* col = sm;  // [K1][kFcCols]: line q at col + q, element stride kFcCols
    float2* scr = col + (size_t)kFcCols * K1;
#pragma unroll 4
    for (int e = tid; e < K1 * kFcCols; e += nth) {
        const int x = e / kFcCols, q = e - x * kFcCols;
        col[e] = q < nc ? a.spec[(size_t)x * ncol + c0 + q] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fc_lines(a.px, col, nc, 1, kFcCols, scr, twx, false, tid, nth);
    for (int e = tid; e < K1 * kFcCols; e += nth) {
        const int kx = e / kFcCols, q = e - kx * kFcCols;
        if (q < nc) {
            const float g = __ldg(a.G + (size_t)kx * ncol + c0 + q);
            col[e].x *= g;
            col[e].y *= g;
        }
    }
    __syncthreads();
    fc_lines(a.px, col, nc, 1, kFcCols, scr, twx, true, tid, nth);
    for (int e = tid; e < K1 * kFcCols; e += nth) {
        const int x = e / kFcCols, q = e - x * kFcCols;
        if (q < nc) a.spec[(size_t)x * ncol + c0 + q] = col[e];
    }
    __syncthreads();
}

// Inverse pass of x-plane x by one CTA: inverse FFT along y, the half spectra of rows 2p and
// 2p + 1 completed Hermitian (imaginary parts of kz = 0 and kz = K3 / 2 dropped, as a complex-to-
// real transform does) and packed as A + i B, inverse FFT along z, real and imaginary parts out as
// the two real rows.  Ends with a barrier of the CTA.
__device__ inline void fc_inv_plane(const FftConvArgs& a, int x, float2* sm, const float2* twy, const float2* twz) {
    const int K2 = a.K[1], K3 = a.K[2], Kh = a.Kh;
    const int np = (K2 + 1) / 2;
    const int tid = threadIdx.x, nth = blockDim.x;
    const FcPlaneSmem m = fc_plane_layout(a, sm);
    const float2* w = a.spec + (size_t)x * K2 * Kh;
#pragma unroll 4
    for (int e = tid; e < K2 * Kh; e += nth) m.plane[e] = w[e];
    __syncthreads();
    fc_lines(a.py, m.plane, Kh, 1, Kh, m.rows, twy, true, tid, nth);
    const bool even = (K3 % 2) == 0;
    const float rk3 = 1.f / (float)K3;
    for (int e = tid; e < np * K3; e += nth) {
        const int p = fc_div(e, rk3), z = e - p * K3;
        const int y0 = 2 * p, y1 = 2 * p + 1;
        const bool lo = z < Kh;
        const int zz = lo ? z : K3 - z;
        float2 A = m.plane[y0 * Kh + zz];
        float2 B = y1 < K2 ? m.plane[y1 * Kh + zz] : make_float2(0.f, 0.f);
        if (z == 0 || (even && z == K3 / 2)) {
            A.y = 0.f;
            B.y = 0.f;
        }
        if (!lo) {
            A.y = -A.y;
            B.y = -B.y;
        }
        m.rows[e] = make_float2(A.x - B.y, A.y + B.x);  // A + i B
    }
    __syncthreads();
    fc_lines(a.pz, m.rows, np, K3, 1, m.scr, twz, true, tid, nth);
    float* gout = a.grid_out + (size_t)x * K2 * K3;
    for (int e = tid; e < np * K3; e += nth) {
        const int p = fc_div(e, rk3), z = e - p * K3;
        const float2 v = m.rows[e];
        gout[(2 * p) * K3 + z] = v.x;
        if (2 * p + 1 < K2) gout[(2 * p + 1) * K3 + z] = v.y;
    }
    __syncthreads();
}

// bytes of the plane-pass working area (fc_plane_layout)
__host__ __device__ inline size_t fc_plane_work(const int K[3]) {
    const int np = (K[1] + 1) / 2, Kh = K[2] / 2 + 1;
    size_t rows = (size_t)np * K[2];
    if (rows < (size_t)K[1] * Kh) rows = (size_t)K[1] * Kh;
    return (2 * rows + (size_t)K[1] * Kh) * sizeof(float2);
}

// bytes of the column-pass working area
__host__ __device__ inline size_t fc_col_work(const int K[3]) { return (size_t)2 * kFcCols * K[0] * sizeof(float2); }

// shared memory of the stand-alone kernels: working area + the stage twiddles they use
__host__ inline size_t fc_plane_smem(const int K[3]) { return fc_plane_work(K) + 2 * kFcTw * sizeof(float2); }
__host__ inline size_t fc_col_smem(const int K[3]) { return fc_col_work(K) + kFcTw * sizeof(float2); }

__global__ void __launch_bounds__(kFcPlaneThreads) k_fc_fwd_planes(FftConvArgs a) {
    extern __shared__ float2 sm[];
    float2* twy = sm + fc_plane_work(a.K) / sizeof(float2);
    float2* twz = twy + kFcTw;
    fc_load_twiddles(twy, a.tw[1], threadIdx.x, blockDim.x);
    fc_load_twiddles(twz, a.tw[2], threadIdx.x, blockDim.x);
    __syncthreads();
    fc_fwd_plane(a, blockIdx.x, sm, twy, twz);
}

__global__ void __launch_bounds__(kFcColThreads) k_fc_columns(FftConvArgs a) {
    extern __shared__ float2 sm[];
    float2* twx = sm + fc_col_work(a.K) / sizeof(float2);
    fc_load_twiddles(twx, a.tw[0], threadIdx.x, blockDim.x);
    __syncthreads();
    fc_column_block(a, blockIdx.x * kFcCols, sm, twx);
}

__global__ void __launch_bounds__(kFcPlaneThreads) k_fc_inv_planes(FftConvArgs a) {
    extern __shared__ float2 sm[];
    float2* twy = sm + fc_plane_work(a.K) / sizeof(float2);
    float2* twz = twy + kFcTw;
    fc_load_twiddles(twy, a.tw[1], threadIdx.x, blockDim.x);
    fc_load_twiddles(twz, a.tw[2], threadIdx.x, blockDim.x);
    __syncthreads();
    fc_inv_plane(a, blockIdx.x, sm, twy, twz);
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
