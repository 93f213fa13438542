// parallel.cu -- parallel-beam projector family for sm_100a.
//
// Kernels (one warp per work item, lanes split into LZ lanes along z times
// 32/LZ lanes along the reduction axis; z is the contiguous axis of both the
// volume [nY][nX][nZ] and the sinogram [nR][nA][nZ], so a warp's tap loads are
// 128-bit vectors over consecutive z and coalesce into 512-byte requests):
//   k_forward      R1, rotate-and-sum with skimage-warp bilinear sampling
//                  (vamtoolbox/projector/Projector3DParallel.py:113-156)
//   k_backward_ref R2, pixel-driven np.interp backprojection + circle clip
//                  (Projector3DParallel.py:158-207)
//   k_adjoint      exact transpose of k_forward, gather form, no atomics
//   k_occ_*        occlusion sinogram (Projector3DParallel.py:77-111)
//
// Sample coordinates are evaluated in float64 with the same expressions in
// k_forward and k_adjoint (fma(c, k, fma(-s, j, m12)) etc.), so both see
// bit-identical tap weights and the adjoint is the transpose of the forward
// up to float32 summation order.  Weights and data are float32.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "vam_internal.cuh"

namespace vam {
namespace {

constexpr int kWarpsPerBlock = 8;
constexpr unsigned kFull = 0xffffffffu;

struct Layout {
    int VZ;        // floats per lane along z (4 or 1)
    int LZ;        // lanes along z (power of two)
    int lz_shift;  // log2(LZ)
    int zvec;      // number of VZ-vectors along z
    int zchunks;   // ceil(zvec / LZ)
};

Layout choose_layout(int nZ, bool aligned16) {
    Layout L;
    L.VZ = (nZ % 4 == 0 && aligned16) ? 4 : 1;
    L.zvec = nZ / L.VZ;
    int best = 1;
    double best_eff = -1.0;
    for (int lz = 32; lz >= 1; lz >>= 1) {
        if (lz > 1 && lz > 2 * L.zvec) continue;
        int ch = (L.zvec + lz - 1) / lz;
        double eff = (double)L.zvec / (double)(ch * lz);
        if (eff >= 0.87) { best = lz; best_eff = eff; break; }
        if (eff > best_eff + 1e-9) { best = lz; best_eff = eff; }
    }
    L.LZ = best;
    L.lz_shift = ilog2_pow2(best);
    L.zchunks = (L.zvec + best - 1) / best;
    return L;
}

struct Args {
    const float* in;
    float* out;
    const double4* trig;
    const uint8_t* circle;
    const float* mask;
    const float* occ;
    const uint8_t* occ_flag;
    const double* occ64;  // occ_mode 1: float64 minima [nR][nA] of the digitised 2-D occlusion
    int nY, nX, nZ, nA, C;
    int lz_shift, zvec, zchunks;
    float alpha, R;  // VAM_ABS_RAY
    int occ_mode, pad_;
};

template <int VZ>
__device__ __forceinline__ void load_vec(const float* p, float (&d)[VZ]) {
    static_assert(VZ == 1 || VZ == 4, "load_vec handles 1 or 4 floats; use load_vz for multiples of 4");
    if constexpr (VZ == 4) {
        float4 t = __ldg(reinterpret_cast<const float4*>(p));
        d[0] = t.x; d[1] = t.y; d[2] = t.z; d[3] = t.w;
    } else {
        d[0] = __ldg(p);
    }
}

template <int VZ>
__device__ __forceinline__ void store_vec(float* p, const float (&d)[VZ]) {
    if constexpr (VZ == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(d[0], d[1], d[2], d[3]);
    } else {
        *p = d[0];
    }
}

// Per-sample absorption factor of the RAY mode: exp(-a * max(0, s - s_entry)).
__device__ __forceinline__ unsigned long long pk_pair(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

__device__ __forceinline__ void fma_pair(unsigned long long& acc, unsigned long long w2, float a, float b) {
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(w2), "l"(pk_pair(a, b)));
}

__device__ __forceinline__ float ray_factor(float s, float s_entry, float alpha) {
    float d = s - s_entry;
    return d > 0.f ? expf(-alpha * d) : 1.f;
}

// [lo, hi] range of integer k for which the sample (row, col) = (rowb + c k,
// colb + s k) can touch the image (both coordinates inside (-1, n)), widened by
// one sample on each side; samples outside are exactly zero.
__device__ __forceinline__ void sample_range(double rowb, double colb, double c, double s, int nY,
                                             int nX, int kmax, int& lo, int& hi) {
    double a = 0.0, b = (double)kmax;
    if (fabs(c) > 1e-12) {
        double t0 = (-1.0 - rowb) / c, t1 = ((double)nY - rowb) / c;
        a = fmax(a, fmin(t0, t1));
        b = fmin(b, fmax(t0, t1));
    } else if (rowb <= -1.0 || rowb >= (double)nY) {
        lo = 1; hi = 0; return;
    }
    if (fabs(s) > 1e-12) {
        double t0 = (-1.0 - colb) / s, t1 = ((double)nX - colb) / s;
        a = fmax(a, fmin(t0, t1));
        b = fmin(b, fmax(t0, t1));
    } else if (colb <= -1.0 || colb >= (double)nX) {
        lo = 1; hi = 0; return;
    }
    if (!(a <= b)) { lo = 1; hi = 0; return; }
    lo = max(0, (int)floor(a) - 1);
    hi = min(kmax, (int)ceil(b) + 1);
}

// ---------------------------------------------------------------------------
// R1 forward
// ---------------------------------------------------------------------------
template <int VZ, bool OCC, int ABS>
__device__ __forceinline__ void k_forward_body(const Args& a, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const int LZ = 1 << a.lz_shift;
    const int LK = 32 >> a.lz_shift;
    const int zl = lane & (LZ - 1);
    const int kl = lane >> a.lz_shift;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int theta = by;
    const int zc = (int)(item % a.zchunks);
    const int j = (int)(item / a.zchunks);
    if (j >= a.nX) return;  // uniform per warp
    const int zv = zc * LZ + zl;
    const bool zok = zv < a.zvec;
    const int z0 = zok ? zv * VZ : 0;

    const double4 tr = a.trig[theta];
    const double c = tr.x, s = tr.y;
    const double rowb = fma(-s, (double)j, tr.w);
    const double colb = fma(c, (double)j, tr.z);

    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;

    int klo, khi;
    sample_range(rowb, colb, c, s, a.nY, a.nX, a.nY - 1, klo, khi);

    float s_entry = 0.f;
    bool live = true;
    if (ABS == VAM_ABS_RAY) {
        float t = (float)(j - a.C);
        if (fabsf(t) > a.R) live = false;
        else s_entry = -sqrtf(a.R * a.R - t * t);
    }
    int kstop[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) kstop[e] = INT_MAX;
    if (OCC && zok) {
#pragma unroll
        for (int e = 0; e < VZ; ++e) {
            const size_t oi = ((size_t)j * a.nA + theta) * a.nZ + z0 + e;
            float o = a.occ[oi];
            if (a.occ_flag[(size_t)theta * a.nZ + z0 + e] && !isnan(o)) kstop[e] = (int)o + a.C;
        }
    }

    if (live) {
        const float* vol = a.in;
        for (int k = klo + kl; k <= khi; k += LK) {
            const double row = fma(c, (double)k, rowb);
            const double col = fma(s, (double)k, colb);
            const double fr = floor(row), fc = floor(col);
            const int r0 = (int)fr, c0 = (int)fc;
            const bool rc = row > fr, cc = col > fc;
            const float dr = (float)(row - fr), dc = (float)(col - fc);
            const bool vr0 = (unsigned)r0 < (unsigned)a.nY, vr1 = rc && (unsigned)(r0 + 1) < (unsigned)a.nY;
            const bool vc0 = (unsigned)c0 < (unsigned)a.nX, vc1 = cc && (unsigned)(c0 + 1) < (unsigned)a.nX;
            float w00 = (1.f - dr) * (1.f - dc), w01 = (1.f - dr) * dc;
            float w10 = dr * (1.f - dc), w11 = dr * dc;
            if (ABS == VAM_ABS_MASK) {
                if (vr0 && vc0) w00 *= __ldg(a.mask + (size_t)r0 * a.nX + c0);
                if (vr0 && vc1) w01 *= __ldg(a.mask + (size_t)r0 * a.nX + c0 + 1);
                if (vr1 && vc0) w10 *= __ldg(a.mask + (size_t)(r0 + 1) * a.nX + c0);
                if (vr1 && vc1) w11 *= __ldg(a.mask + (size_t)(r0 + 1) * a.nX + c0 + 1);
            }
            float v[VZ];
#pragma unroll
            for (int e = 0; e < VZ; ++e) v[e] = 0.f;
            if (zok) {
                float t[VZ];
                if (vr0 && vc0) {
                    load_vec<VZ>(vol + ((size_t)r0 * a.nX + c0) * a.nZ + z0, t);
#pragma unroll
                    for (int e = 0; e < VZ; ++e) v[e] = fmaf(w00, t[e], v[e]);
                }
                if (vr0 && vc1) {
                    load_vec<VZ>(vol + ((size_t)r0 * a.nX + c0 + 1) * a.nZ + z0, t);
#pragma unroll
                    for (int e = 0; e < VZ; ++e) v[e] = fmaf(w01, t[e], v[e]);
                }
                if (vr1 && vc0) {
                    load_vec<VZ>(vol + ((size_t)(r0 + 1) * a.nX + c0) * a.nZ + z0, t);
#pragma unroll
                    for (int e = 0; e < VZ; ++e) v[e] = fmaf(w10, t[e], v[e]);
                }
                if (vr1 && vc1) {
                    load_vec<VZ>(vol + ((size_t)(r0 + 1) * a.nX + c0 + 1) * a.nZ + z0, t);
#pragma unroll
                    for (int e = 0; e < VZ; ++e) v[e] = fmaf(w11, t[e], v[e]);
                }
            }
            float f = 1.f;
            if (ABS == VAM_ABS_RAY) f = ray_factor((float)(k - a.C), s_entry, a.alpha);
#pragma unroll
            for (int e = 0; e < VZ; ++e) {
                float ve = (ABS == VAM_ABS_RAY) ? v[e] * f : v[e];
                if (OCC && k > kstop[e]) ve = 0.f;
                acc[e] += ve;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < VZ; ++e)
        for (int off = LZ; off < 32; off <<= 1) acc[e] += __shfl_xor_sync(kFull, acc[e], off);
    if (kl == 0 && zok) store_vec<VZ>(a.out + ((size_t)j * a.nA + theta) * a.nZ + z0, acc);
}

template <int VZ, bool OCC, int ABS>
__global__ void __launch_bounds__(256) k_forward(Args a) {
    k_forward_body<VZ, OCC, ABS>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// R1 forward, fast path: 32 lanes along z (VZ floats each), one lattice row
// (angle, detector) per warp, angle pairs (a, a+180) sampled from one lattice.
//
// The sample points of angle a+180 are those of angle a mirrored through the
// rotation centre: sample (j', k') of a+180 is lattice point (2C-j', 2C-k') of
// a (the warp matrices of Projector3DParallel.py:137-143 satisfy this
// identically), so one pass over a's lattice row gives both rays.  For odd N
// the k ranges coincide; for even N (2C = N) angle a sums k in [0, N-1] and
// a+180 sums k in [1, N] on the row j in [0, N]; the shared part k in [1, N-1]
// is accumulated once and the two end samples are added separately.
// ---------------------------------------------------------------------------
struct FastArgs {
    const float* vol;
    float* sino;
    const double4* trig;
    const int2* tasks;
    int nY, nX, nZ, nA, C;
    int RS;          // row stride of the volume in floats (nX * nZ)
    int zchunks;     // ceil(nZ / (32 * VZ))
    int even;        // N even
    float alpha, R;  // RAY absorption (tasks are unpaired then)
};

template <int VZ>
struct Acc {
    float v[VZ];
};

// One bilinear sample (all taps checked), added with weight f into acc.
// Lane-interleaved z vectors of the fast kernels: with Q = VZ / 4, lane l of
// a warp owns slices zbase + 4l + 128q + (0..3), q < Q, so every float4 load
// of the warp covers 512 contiguous bytes (four 128-byte lines).  p points at
// the lane's first slice; qn is the number of its vectors inside the volume.
// Six / five slices per lane (192- / 160-slice chunks, full chunks only): a
// float4 at zbase + 4l and a float2 at zbase + 128 + 2l or a float at
// zbase + 128 + l (a 256- / 128-byte run per warp).
template <int VZ>
__device__ __forceinline__ void load_vz(const float* __restrict__ p, float* d, int qn = VZ / 4) {
    if constexpr (VZ == 6 || VZ == 5) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        d[0] = t.x; d[1] = t.y; d[2] = t.z; d[3] = t.w;
        if constexpr (VZ == 6) {
            const float2 u = __ldg(reinterpret_cast<const float2*>(p + 128 - 2 * (int)(threadIdx.x & 31)));
            d[4] = u.x; d[5] = u.y;
        } else {
            d[4] = __ldg(p + 128 - 3 * (int)(threadIdx.x & 31));
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q) {
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q < qn) t = __ldg(reinterpret_cast<const float4*>(p + 128 * q));
        d[4 * q] = t.x; d[4 * q + 1] = t.y; d[4 * q + 2] = t.z; d[4 * q + 3] = t.w;
    }
}

// load_vz with an L1 evict-last priority: the forward's taps, which neighbouring bins and samples of
// the CTA read again (1.406 -> 1.373 ms at 256^3 x 360, identical results)
template <int VZ>
__device__ __forceinline__ void load_vz_keep(const float* __restrict__ p, float* d, int qn = VZ / 4) {
    if constexpr (VZ == 6 || VZ == 5) {
        float4 t;
        asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
            : "=f"(t.x), "=f"(t.y), "=f"(t.z), "=f"(t.w) : "l"(p));
        d[0] = t.x; d[1] = t.y; d[2] = t.z; d[3] = t.w;
        if constexpr (VZ == 6) {
            float2 u;
            asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];"
                : "=f"(u.x), "=f"(u.y) : "l"(p + 128 - 2 * (int)(threadIdx.x & 31)));
            d[4] = u.x; d[5] = u.y;
        } else {
            asm("ld.global.nc.L1::evict_last.f32 %0, [%1];" : "=f"(d[4]) : "l"(p + 128 - 3 * (int)(threadIdx.x & 31)));
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q) {
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q < qn)
            asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
                : "=f"(t.x), "=f"(t.y), "=f"(t.z), "=f"(t.w) : "l"(p + 128 * q));
        d[4 * q] = t.x; d[4 * q + 1] = t.y; d[4 * q + 2] = t.z; d[4 * q + 3] = t.w;
    }
}

template <int VZ>
__device__ __forceinline__ void store_vz(float* __restrict__ p, const float* d, int qn) {
    if constexpr (VZ == 6 || VZ == 5) {
        *reinterpret_cast<float4*>(p) = make_float4(d[0], d[1], d[2], d[3]);
        if constexpr (VZ == 6) *reinterpret_cast<float2*>(p + 128 - 2 * (int)(threadIdx.x & 31)) = make_float2(d[4], d[5]);
        else p[128 - 3 * (int)(threadIdx.x & 31)] = d[4];
        return;
    }
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q)
        if (q < qn) *reinterpret_cast<float4*>(p + 128 * q) = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
}

// First slice and number of in-range vectors of a lane in z-chunk zc (six / five slices per lane: full
// chunks, qn = 2 vectors).
template <int VZ>
__device__ __forceinline__ void lane_z(int zc, int lane, int nZ, int& z0, int& qn) {
    const int base = zc * 32 * VZ + 4 * lane;
    if constexpr (VZ == 6 || VZ == 5) {
        z0 = base;
        qn = 2;
        return;
    }
    qn = 0;
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q) qn += (base + 128 * q < nZ) ? 1 : 0;
    z0 = qn ? base : 0;
}

template <int VZ>
__device__ __forceinline__ void sample_checked(const FastArgs& a, const float* __restrict__ volz, double row,
                                               double col, float f, float (&acc)[VZ], int qn) {
    const double fr = floor(row), fc = floor(col);
    const int r0 = (int)fr, c0 = (int)fc;
    const bool rc = row > fr, cc = col > fc;
    const float dr = (float)(row - fr), dc = (float)(col - fc);
    const bool vr0 = (unsigned)r0 < (unsigned)a.nY, vr1 = rc && (unsigned)(r0 + 1) < (unsigned)a.nY;
    const bool vc0 = (unsigned)c0 < (unsigned)a.nX, vc1 = cc && (unsigned)(c0 + 1) < (unsigned)a.nX;
    const float w00 = (1.f - dr) * (1.f - dc) * f, w01 = (1.f - dr) * dc * f;
    const float w10 = dr * (1.f - dc) * f, w11 = dr * dc * f;
    float t[VZ];
    if (vr0 && vc0) {
        load_vz<VZ>(volz + (size_t)r0 * a.RS + (size_t)c0 * a.nZ, t, qn);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w00, t[e], acc[e]);
    }
    if (vr0 && vc1) {
        load_vz<VZ>(volz + (size_t)r0 * a.RS + (size_t)(c0 + 1) * a.nZ, t, qn);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w01, t[e], acc[e]);
    }
    if (vr1 && vc0) {
        load_vz<VZ>(volz + (size_t)(r0 + 1) * a.RS + (size_t)c0 * a.nZ, t, qn);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w10, t[e], acc[e]);
    }
    if (vr1 && vc1) {
        load_vz<VZ>(volz + (size_t)(r0 + 1) * a.RS + (size_t)(c0 + 1) * a.nZ, t, qn);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w11, t[e], acc[e]);
    }
}

template <int VZ, bool RAY>
__device__ __forceinline__ void k_forward_fast_body(const FastArgs& a, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const int item = bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = item % a.zchunks;
    const int j = item / a.zchunks;
    const int2 task = a.tasks[by];
    const bool paired = task.y >= 0;
    const int N = a.nY;
    const bool ext = paired && a.even;   // lattice row / column N is needed by the partner angle
    if (j > (ext ? N : N - 1)) return;   // uniform per warp
    int z0, qn;
    lane_z<VZ>(zc, lane, a.nZ, z0, qn);
    const bool zok = qn > 0;
    const float* __restrict__ volz = a.vol + z0;

    const double4 tr = a.trig[task.x];
    const double c = tr.x, s = tr.y;
    const double rowb = fma(-s, (double)j, tr.w);
    const double colb = fma(c, (double)j, tr.z);
    const int kmax = ext ? N : N - 1;
    int klo, khi;
    sample_range(rowb, colb, c, s, a.nY, a.nX, kmax, klo, khi);

    float s_entry = 0.f;
    if (RAY) {
        const float t = (float)(j - a.C);
        s_entry = fabsf(t) <= a.R ? -sqrtf(a.R * a.R - t * t) : 0.f;
        if (fabsf(t) > a.R) klo = 1, khi = 0;
    }
    float acc[VZ], e0[VZ], eN[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = e0[e] = eN[e] = 0.f;

    if (zok) {
        const int nYm1 = a.nY - 1, nXm1 = a.nX - 1;
        const int lo = max(klo, 1), hi = min(khi, N - 1);
        for (int k = lo; k <= hi; ++k) {
            const double row = fma(c, (double)k, rowb);
            const double col = fma(s, (double)k, colb);
            const float f = RAY ? ray_factor((float)(k - a.C), s_entry, a.alpha) : 1.f;
            const double fr = floor(row), fc = floor(col);
            const int r0 = (int)fr, c0 = (int)fc;
            if ((unsigned)r0 < (unsigned)nYm1 && (unsigned)c0 < (unsigned)nXm1) {
                // interior: all four taps in the image; a zero-weight ceil tap is
                // redirected to the floor tap so no unrelated value is read
                const float dr = (float)(row - fr), dc = (float)(col - fc);
                const int o00 = r0 * a.RS + c0 * a.nZ;
                const int dcol = (col > fc) ? a.nZ : 0;
                const int o10 = o00 + ((row > fr) ? a.RS : 0);
                float w00 = (1.f - dr) * (1.f - dc), w01 = (1.f - dr) * dc;
                float w10 = dr * (1.f - dc), w11 = dr * dc;
                if (RAY) { w00 *= f; w01 *= f; w10 *= f; w11 *= f; }
                float t0[VZ], t1[VZ], t2[VZ], t3[VZ];
                load_vz_keep<VZ>(volz + o00, t0, qn);
                load_vz_keep<VZ>(volz + o00 + dcol, t1, qn);
                load_vz_keep<VZ>(volz + o10, t2, qn);
                load_vz_keep<VZ>(volz + o10 + dcol, t3, qn);
#pragma unroll
                for (int e = 0; e < VZ; ++e) {
                    acc[e] = fmaf(w00, t0[e], acc[e]);
                    acc[e] = fmaf(w01, t1[e], acc[e]);
                    acc[e] = fmaf(w10, t2[e], acc[e]);
                    acc[e] = fmaf(w11, t3[e], acc[e]);
                }
            } else {
                sample_checked<VZ>(a, volz, row, col, f, acc, qn);
            }
        }
        if (klo <= 0 && khi >= 0) {
            const float f = RAY ? ray_factor((float)(0 - a.C), s_entry, a.alpha) : 1.f;
            sample_checked<VZ>(a, volz, rowb, colb, f, e0, qn);
        }
        if (ext && klo <= N && khi >= N)
            sample_checked<VZ>(a, volz, fma(c, (double)N, rowb), fma(s, (double)N, colb), 1.f, eN, qn);
    }
    if (!zok) return;
    if (j <= N - 1) {
        float o[VZ];
#pragma unroll
        for (int e = 0; e < VZ; ++e) o[e] = acc[e] + e0[e];
        store_vz<VZ>(a.sino + ((size_t)j * a.nA + task.x) * a.nZ + z0, o, qn);
    }
    if (paired) {
        // partner detector j' = 2C - j over lattice k in [2C-N+1, 2C]
        const int jp = 2 * a.C - j;
        if (jp >= 0 && jp <= N - 1) {
            float o[VZ];
#pragma unroll
            for (int e = 0; e < VZ; ++e) o[e] = acc[e] + (a.even ? eN[e] : e0[e]);
            store_vz<VZ>(a.sino + ((size_t)jp * a.nA + task.y) * a.nZ + z0, o, qn);
        }
    }
}

template <int VZ, bool RAY>
__global__ void __launch_bounds__(256) k_forward_fast(FastArgs a) {
    k_forward_fast_body<VZ, RAY>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Matched transpose, fast path: 32 lanes along z, one pixel per warp.
//
// The forward's tap weight of pixel (i, j) from lattice sample (J, K) is
// hat(i - row(J,K)) * hat(j - col(J,K)) with hat(d) = max(0, 1 - |d|) (the
// floor / ceil weights (1-dr), dr are exactly that).  The pixel's offset to
// its nearest lattice point (J0, K0) is formed once in float64 from the same
// coordinate expression the forward uses; the offsets to the 3 x 3 candidate
// lattice points follow in float32 by adding multiples of (s, -c) and
// (-c, -s), small numbers, so every candidate weight agrees with the
// forward's to ~1e-7 and the kernel gathers at most 3 detector rows per angle.
// ---------------------------------------------------------------------------
template <int VZ, bool RAY>
__device__ __forceinline__ void k_adjoint_fast_body(const Args& a, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zchunks = a.zchunks;
    const int zc = (int)(item % zchunks);
    const long p = item / zchunks;
    if (p >= (long)a.nY * a.nX) return;
    const int i = (int)(p / a.nX), j = (int)(p % a.nX);
    int z0, qn;
    lane_z<VZ>(zc, lane, a.nZ, z0, qn);
    const bool zok = qn > 0;
    const size_t rs = (size_t)a.nA * a.nZ;
    const int N = a.nY;
    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;
    const float* __restrict__ bz = a.in + z0;
    for (int th = 0; th < a.nA; ++th) {
        const double4 tr = a.trig[th];
        const double c = tr.x, s = tr.y;
        const double ri = (double)i - tr.w, ci = (double)j - tr.z;
        const double Jf = fma(-s, ri, c * ci), Kf = fma(c, ri, s * ci);
        const int J0 = __double2int_rn(Jf), K0 = __double2int_rn(Kf);
        const double row0 = fma(c, (double)K0, fma(-s, (double)J0, tr.w));
        const double col0 = fma(s, (double)K0, fma(c, (double)J0, tr.z));
        const float dr = (float)((double)i - row0), dc = (float)((double)j - col0);
        const float sf = (float)s, cf = (float)c;
#pragma unroll
        for (int da = -1; da <= 1; ++da) {
            const int J = J0 + da;
            if ((unsigned)J >= (unsigned)a.nX) continue;
            float s_entry = 0.f;
            if (RAY) {
                const float t = (float)(J - a.C);
                if (fabsf(t) > a.R) continue;
                s_entry = -sqrtf(a.R * a.R - t * t);
            }
            float W = 0.f;
#pragma unroll
            for (int db = -1; db <= 1; ++db) {
                const int K = K0 + db;
                if ((unsigned)K >= (unsigned)N) continue;
                const float er = fmaf((float)da, sf, fmaf(-(float)db, cf, dr));
                const float ec = fmaf(-(float)da, cf, fmaf(-(float)db, sf, dc));
                float w = fmaxf(0.f, 1.f - fabsf(er)) * fmaxf(0.f, 1.f - fabsf(ec));
                if (RAY) w *= ray_factor((float)(K - a.C), s_entry, a.alpha);
                W += w;
            }
            if (W != 0.f && zok) {
                float bv[VZ];
                load_vz<VZ>(bz + (size_t)J * rs + (size_t)th * a.nZ, bv, qn);
#pragma unroll
                for (int e = 0; e < VZ; ++e) acc[e] = fmaf(W, bv[e], acc[e]);
            }
        }
    }
    if (!zok) return;
    if (a.mask) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] *= m;
    }
    store_vz<VZ>(a.out + (size_t)p * a.nZ + z0, acc, qn);
}

template <int VZ, bool RAY>
__global__ void __launch_bounds__(256) k_adjoint_fast(Args a) {
    k_adjoint_fast_body<VZ, RAY>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// R2 backprojection, fast path: 32 lanes along z with VZ floats each (one
// pixel per warp, angles in sequence); same arithmetic as k_backward_ref.
// ---------------------------------------------------------------------------
template <int VZ, bool RAY>
__device__ __forceinline__ void k_backward_fast_body(const Args& a, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = (int)(item % a.zchunks);
    const long p = item / a.zchunks;
    if (p >= (long)a.nY * a.nX) return;
    const int i = (int)(p / a.nX), j = (int)(p % a.nX);
    int z0, qn;
    lane_z<VZ>(zc, lane, a.nZ, z0, qn);
    const bool zok = qn > 0;
    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;
    if (a.circle[p] && zok) {
        const double X = (double)(j - a.C), Y = (double)(i - a.C);
        const double tlo = (double)(-a.C), thi = (double)(a.nY - 1 - a.C);
        const int rs = a.nA * a.nZ, nYm1 = a.nY - 1;  // sinogram below 2^31 elements on this path
        const float* __restrict__ bz = a.in + z0;
#pragma unroll 2
        for (int th = 0; th < a.nA; ++th) {
            const double4 tr = a.trig[th];
            const double t = __dsub_rn(__dmul_rn(X, tr.x), __dmul_rn(Y, tr.y));
            // np.interp(left = right = 0): out-of-range angles read clamped rows with zero weight
            const bool ok = t >= tlo && t <= thi;
            const double ft = floor(t);
            const int j0 = min(max((int)fmax(fmin(ft, 1e9), -1e9) + a.C, 0), nYm1);
            float v0[VZ], v1[VZ];
            load_vz<VZ>(bz + j0 * rs + th * a.nZ, v0, qn);
            // t == floor(t): np.interp returns fp[j]; the second row is read with weight 0
            const float w = (float)(t - ft);
            load_vz<VZ>(bz + min(j0 + 1, nYm1) * rs + th * a.nZ, v1, qn);
            float f = ok ? 1.f : 0.f;
            if (RAY) {
                // |t| <= R is a discontinuity of the model: decide it on the float64 t
                if (ok && fabs(t) <= (double)a.R) {
                    const float sv = (float)__dadd_rn(__dmul_rn(X, tr.y), __dmul_rn(Y, tr.x));
                    f = ray_factor(sv, (float)(-sqrt((double)a.R * a.R - t * t)), a.alpha);
                } else {
                    f = 0.f;
                }
            }
            const float w1 = w * f, w0 = (1.f - w) * f;
#pragma unroll
            for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w1, v1[e], fmaf(w0, v0[e], acc[e]));
        }
    }
    if (!zok) return;
    if (a.mask) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = m * acc[e];
    }
    store_vz<VZ>(a.out + (size_t)p * a.nZ + z0, acc, qn);
}

template <int VZ, bool RAY>
__global__ void __launch_bounds__(256) k_backward_fast(Args a) {
    k_backward_fast_body<VZ, RAY>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Matched transpose from a weight table.
//
// k_adj_table evaluates, once per plan, for every pixel (i, j) and angle the
// forward's own tap weights: the candidate lattice samples (J, K) around the
// pixel's rotated position are evaluated with the forward's float64
// coordinate expression and float32 weights, (1-dr)(1-dc) etc. times the RAY
// factor, and summed per detector row J.  At most three rows J0-1..J0+1
// touch a pixel (|J - J*| < |cos| + |sin| <= sqrt 2).  k_adjoint_table is then
// a gather: per pixel and angle one 16-byte entry (broadcast over the warp)
// and at most three sinogram rows.
// ---------------------------------------------------------------------------
template <bool RAY>
__global__ void __launch_bounds__(256) k_adj_table(const double4* __restrict__ trig, float4* __restrict__ table, int nY,
                                                   int nX, int nA, int C, float alpha, float R) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;   // over (pixel, angle), angle fastest
    if (idx >= (long)nY * nX * nA) return;
    const int th = (int)(idx % nA);
    const long p = idx / nA;
    const int i = (int)(p / nX), j = (int)(p % nX);
    const double4 tr = trig[th];
    const double c = tr.x, s = tr.y;
    const double ri = (double)i - tr.w, ci = (double)j - tr.z;
    const int J0 = __double2int_rn(fma(-s, ri, c * ci)), K0 = __double2int_rn(fma(c, ri, s * ci));
    float W[3] = {0.f, 0.f, 0.f};
    for (int da = -1; da <= 1; ++da) {
        const int J = J0 + da;
        if ((unsigned)J >= (unsigned)nX) continue;
        float s_entry = 0.f;
        if (RAY) {
            const float t = (float)(J - C);
            if (fabsf(t) > R) continue;
            s_entry = -sqrtf(R * R - t * t);
        }
        const double rowb = fma(-s, (double)J, tr.w), colb = fma(c, (double)J, tr.z);
        for (int db = -2; db <= 2; ++db) {
            const int K = K0 + db;
            if ((unsigned)K >= (unsigned)nY) continue;
            const double row = fma(c, (double)K, rowb), col = fma(s, (double)K, colb);
            const double fr = floor(row), fc = floor(col);
            const int r0 = (int)fr, c0 = (int)fc;
            const bool rc = row > fr, cc = col > fc;
            if (!(i == r0 || (rc && i == r0 + 1))) continue;
            if (!(j == c0 || (cc && j == c0 + 1))) continue;
            const float dr = (float)(row - fr), dc = (float)(col - fc);
            float w = ((i == r0) ? (1.f - dr) : dr) * ((j == c0) ? (1.f - dc) : dc);
            if (RAY) w *= ray_factor((float)(K - C), s_entry, alpha);
            W[da + 1] += w;
        }
    }
    table[p * nA + th] = make_float4(__int_as_float(J0 - 1), W[0], W[1], W[2]);
}

template <int VZ>
__device__ __forceinline__ void k_adjoint_table_body(const Args& a, const float4* __restrict__ table, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = (int)(item % a.zchunks);
    const long p = item / a.zchunks;
    if (p >= (long)a.nY * a.nX) return;
    int z0, qn;
    lane_z<VZ>(zc, lane, a.nZ, z0, qn);
    if (qn == 0) return;
    const size_t rs = (size_t)a.nA * a.nZ;
    const float* __restrict__ bz = a.in + z0;
    const float4* __restrict__ tp = table + p * a.nA;
    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;
    if constexpr (VZ == 4) {
        // four slices per lane: the rows of an angle and the next angle's entry in flight together
        // (3.44 -> 3.09 ms at 256^3 x 360); with eight slices the extra row registers cost more
        // occupancy than the overlap gains (2.17 -> 2.33 ms), so that instance reads row by row
        float4 ent = __ldg(tp);
#pragma unroll 1
        for (int th = 0; th < a.nA; ++th) {
            // the next angle's entry is in flight while this angle's rows are read
            const float4 nxt = __ldg(tp + min(th + 1, a.nA - 1));
            const int J = __float_as_int(ent.x);
            const float w[3] = {ent.y, ent.z, ent.w};
            const float* __restrict__ row = bz + (size_t)J * rs + (size_t)th * a.nZ;
            // every row's loads are issued before any is consumed; a row of weight 0 is not read and its
            // zeros leave the sums unchanged (fma(0, 0, s) == s: the sums are never -0), so the result
            // equals summing the rows of nonzero weight in order
            float bv[3][VZ];
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                if (w[t] != 0.f) {
                    load_vz<VZ>(row + (size_t)t * rs, bv[t], qn);
                } else {
#pragma unroll
                    for (int e = 0; e < VZ; ++e) bv[t][e] = 0.f;
                }
            }
#pragma unroll
            for (int t = 0; t < 3; ++t)
#pragma unroll
                for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w[t], bv[t][e], acc[e]);
            ent = nxt;
        }
    } else {
#pragma unroll 2
        for (int th = 0; th < a.nA; ++th) {
            const float4 ent = __ldg(tp + th);
            const int J = __float_as_int(ent.x);
            const float w[3] = {ent.y, ent.z, ent.w};
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                if (w[t] != 0.f) {
                    float bv[VZ];
                    load_vz<VZ>(bz + (size_t)(J + t) * rs + (size_t)th * a.nZ, bv, qn);
#pragma unroll
                    for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w[t], bv[e], acc[e]);
                }
            }
        }
    }
    if (a.mask) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] *= m;
    }
    store_vz<VZ>(a.out + (size_t)p * a.nZ + z0, acc, qn);
}

// eight resident CTAs per SM (32 registers, no spills): 2.17 -> 1.91 ms at 256^3 x 360 with eight
// slices per lane, identical results
template <int VZ>
__global__ void __launch_bounds__(256, 8) k_adjoint_table(Args a, const float4* __restrict__ table) {
    k_adjoint_table_body<VZ>(a, table, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// R2 backprojection, batched: cos / sin of every angle staged in shared
// memory, and B angles per step whose detector-row loads are all issued
// before any is consumed, so each warp keeps 2B row loads in flight instead
// of waiting on one angle's float64 chain and loads at a time.
// ---------------------------------------------------------------------------
template <int VZ, int B, bool RAY>
__device__ __forceinline__ void k_backward_batched_body(const Args& a, unsigned bx, unsigned by) {
    extern __shared__ double2 s_cs[];
    for (int t = threadIdx.x; t < a.nA; t += blockDim.x) s_cs[t] = make_double2(a.trig[t].x, a.trig[t].y);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = (int)(item % a.zchunks);
    const long p = item / a.zchunks;
    if (p >= (long)a.nY * a.nX) return;
    const int i = (int)(p / a.nX), j = (int)(p % a.nX);
    int z0, qn;
    lane_z<VZ>(zc, lane, a.nZ, z0, qn);
    if (qn == 0) return;
    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;
    if (a.circle[p]) {
        const double X = (double)(j - a.C), Y = (double)(i - a.C);
        const double tlo = (double)(-a.C), thi = (double)(a.nY - 1 - a.C);
        // 32-bit offsets: the fast path is taken only for sinograms below 2^31 elements
        const int rs = a.nA * a.nZ, nYm1 = a.nY - 1;
        const float* __restrict__ bz = a.in + z0;
        for (int th0 = 0; th0 < a.nA; th0 += B) {
            int o0[B], o1[B];
            float w0[B], w1[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                // a batch past the last angle rereads the last angle with zero weights
                const int th = min(th0 + u, a.nA - 1);
                const double2 cs = s_cs[th];
                const double t = __dsub_rn(__dmul_rn(X, cs.x), __dmul_rn(Y, cs.y));
                // np.interp(left = right = 0): an angle outside [xp[0], xp[-1]] adds nothing; its taps
                // are clamped reads with zero weight instead of a branch
                const bool ok = th0 + u < a.nA && t >= tlo && t <= thi;
                const double ft = floor(t);
                const int j0 = min(max((int)fmax(fmin(ft, 1e9), -1e9) + a.C, 0), nYm1);
                const float w = (float)(t - ft);
                float f = 1.f;
                if (RAY) {
                    f = 0.f;
                    if (fabs(t) <= (double)a.R) {
                        const float sv = (float)__dadd_rn(__dmul_rn(X, cs.y), __dmul_rn(Y, cs.x));
                        f = ray_factor(sv, (float)(-sqrt((double)a.R * a.R - t * t)), a.alpha);
                    }
                }
                w1[u] = ok ? w * f : 0.f;        // t == floor(t): w = 0, the second row is not used
                w0[u] = ok ? (1.f - w) * f : 0.f;
                o0[u] = j0 * rs + th * a.nZ;
                o1[u] = min(j0 + 1, nYm1) * rs + th * a.nZ;
            }
            float v0[B][VZ], v1[B][VZ];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                load_vz<VZ>(bz + o0[u], v0[u], qn);
                load_vz<VZ>(bz + o1[u], v1[u], qn);
            }
            // acc += (1 - w) v0 + w v1 (times the ray factor): two FMAs per slice
#pragma unroll
            for (int u = 0; u < B; ++u)
#pragma unroll
                for (int e = 0; e < VZ; ++e) acc[e] = fmaf(w1[u], v1[u][e], fmaf(w0[u], v0[u][e], acc[e]));
        }
    }
    if (a.mask) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = m * acc[e];
    }
    store_vz<VZ>(a.out + (size_t)p * a.nZ + z0, acc, qn);
}

template <int VZ, int B, bool RAY>
__global__ void __launch_bounds__(256) k_backward_batched(Args a) {
    k_backward_batched_body<VZ, B, RAY>(a, blockIdx.x, blockIdx.y);
}

// Eight slices per lane without per-ray absorption, capped at 40 registers for six resident CTAs
// (a few spilled bytes): 1.61 -> 1.53 ms at 256^3 x 360, 0.65 -> 0.54 ms at 96^3 x 720, identical
// results.  The four-slice instances ran 3-6 % slower under the same cap and keep the default.
__global__ void __launch_bounds__(256, 6) k_backward_batched8(Args a) {
    k_backward_batched_body<8, 2, false>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// R2 backprojection from the plan's bin table: 2 x 2 pixel blocks share their
// detector rows.
//
// k_bwd_btable evaluates np.interp's bin once per plan: for every pixel
// inside the clip circle and every angle the same float64 t = x cos - y sin,
// floor j0 and float32 weight t - floor(t) as the batched kernel, no
// contribution where t leaves the detector (np.interp left = right = 0), and
// at the detector's last bin (t == xp[-1], weight 0) row nY - 2 with weight 1,
// which adds the same single row with the same rounding.  For one angle the
// four pixels of a 2 x 2 block have t within |cos| + |sin| <= sqrt(2) of each
// other, so their bins span at most three consecutive values and the block
// needs at most four detector rows (j_min .. j_max + 1) instead of eight.  The
// table holds, per block inside the circle and angle, 32 bytes: the offset of
// row j_min (j_min * nA * nZ + angle * nZ, -1 when no pixel of the block
// contributes), a code (bits 0-1: j_max - j_min; per pixel q three bits at
// 2 + 3q: bit 0 contributes, bits 1-2: j0 - j_min) and the four pixels'
// weights.  k_backward_blk loads the block's rows once per warp and runs, per
// pixel, (1 - w) * row j0 then w * row j0 + 1 as packed f32x2 FMAs (two fmaf
// roundings each), the order of k_backward_batched8, so the sums are
// bit-identical to it for finite data.  The warp walks the rows in passes
// d = 0 .. span (rows d and d + 1 live), applying each pixel in the pass of
// its own j0, so at most three rows are held in registers.  It replaced a
// per-pixel table kernel (8-byte entries, two rows per pixel and angle, L1
// bound at 90 %): 1.33 -> 0.92 ms at 256^3 x 360.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_bwd_btable(const double4* __restrict__ trig, const int* __restrict__ blist,
                                                    const int* __restrict__ cidx, int4* __restrict__ tab, int nbc,
                                                    int nA, int nY, int nX, int nZ, int C) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;  // over (block, angle), angle fastest
    if (idx >= (long)nbc * nA) return;
    const int th = (int)(idx % nA);
    const int blk = blist[idx / nA];
    const int nbx = (nX + 1) >> 1;
    const int bi = blk / nbx, bj = blk - bi * nbx;
    const double4 tr = trig[th];
    int j0s[4];
    float ws[4];
    bool val[4];
    int jmin = 1 << 30, jmax = -1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int i = 2 * bi + (q >> 1), j = 2 * bj + (q & 1);
        val[q] = i < nY && j < nX && cidx[(size_t)i * nX + j] >= 0;
        j0s[q] = 0;
        ws[q] = 0.f;
        if (val[q]) {
            const double X = (double)(j - C), Y = (double)(i - C);
            const double t = __dsub_rn(__dmul_rn(X, tr.x), __dmul_rn(Y, tr.y));
            if (!(t >= (double)(-C) && t <= (double)(nY - 1 - C))) {
                val[q] = false;
            } else {
                const double ft = floor(t);
                const int j0 = (int)ft + C;
                if (j0 == nY - 1) { j0s[q] = nY - 2; ws[q] = 1.f; }
                else { j0s[q] = j0; ws[q] = (float)(t - ft); }
                jmin = min(jmin, j0s[q]);
                jmax = max(jmax, j0s[q]);
            }
        }
    }
    if (jmax < 0) {
        tab[2 * idx] = make_int4(-1, 0, 0, 0);
        tab[2 * idx + 1] = make_int4(0, 0, 0, 0);
        return;
    }
    int code = jmax - jmin;  // <= 2
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (val[q]) code |= (1 | ((j0s[q] - jmin) << 1)) << (2 + 3 * q);
    tab[2 * idx] = make_int4(jmin * nA * nZ + th * nZ, code, __float_as_int(ws[0]), __float_as_int(ws[1]));
    tab[2 * idx + 1] = make_int4(__float_as_int(ws[2]), __float_as_int(ws[3]), 0, 0);
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// A lane's slices of one detector row: VZ / 4 float4 vectors at 4 l + 128 q (VZ = 4, 8), or a float4
// at 4 l and a float2 at 128 + 2 l (VZ = 6, 192-slice chunks) or a float at 128 + l (VZ = 5, 160-slice
// chunks).  The slice pairs of the packed FMAs: (VZ + 1) / 2, the fifth slice paired with a zero.
template <int VZ>
struct RowV {
    float4 v[VZ / 4];
    float2 t;  // VZ == 6, 5 (t.y = 0 for VZ == 5)
};

// the lane's vectors of one detector row (p: the row at the lane's first slice); vectors q >= qn (past
// nZ) read as zeros
template <int VZ>
__device__ __forceinline__ void load_row(RowV<VZ>& r, const float* __restrict__ p, int qn = VZ / 4) {
    if constexpr (VZ == 6) {
        r.v[0] = __ldg(reinterpret_cast<const float4*>(p));
        r.t = __ldg(reinterpret_cast<const float2*>(p + 128 - 2 * (int)(threadIdx.x & 31)));
    } else if constexpr (VZ == 5) {
        r.v[0] = __ldg(reinterpret_cast<const float4*>(p));
        r.t = make_float2(__ldg(p + 128 - 3 * (int)(threadIdx.x & 31)), 0.f);
    } else {
#pragma unroll
        for (int q = 0; q < VZ / 4; ++q)
            r.v[q] = q < qn ? __ldg(reinterpret_cast<const float4*>(p + 128 * q)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// acc (slice pairs) += (1 - w) * r0 then += w * r1: two packed FMAs per pair
template <int VZ>
__device__ __forceinline__ void lerp_rows(unsigned long long (&acc)[(VZ + 1) / 2], float w, const RowV<VZ>& r0,
                                          const RowV<VZ>& r1) {
    const unsigned long long w0 = pk_pair(1.f - w, 1.f - w), w1 = pk_pair(w, w);
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q) {
        fma_pair(acc[2 * q], w0, r0.v[q].x, r0.v[q].y);
        fma_pair(acc[2 * q + 1], w0, r0.v[q].z, r0.v[q].w);
    }
    if constexpr (VZ == 6 || VZ == 5) fma_pair(acc[2], w0, r0.t.x, r0.t.y);
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q) {
        fma_pair(acc[2 * q], w1, r1.v[q].x, r1.v[q].y);
        fma_pair(acc[2 * q + 1], w1, r1.v[q].z, r1.v[q].w);
    }
    if constexpr (VZ == 6 || VZ == 5) fma_pair(acc[2], w1, r1.t.x, r1.t.y);
}

// one warp per (2 x 2 block, z chunk of 32 VZ slices); FULL: nZ a multiple of 32 VZ, else the lanes
// past nZ in the last chunk load and store nothing.  The table entries
// arrive 32 angles at a time (lane l fetches angle k0 + l's 32 bytes, the next chunk in flight while
// this one is read), so no angle waits for its entry: eight slices per lane by cp.async into the warp's
// two shared-memory slots (no registers held: the body fits 80 registers, three CTAs per SM; 1.19 ->
// 0.92 ms at 256^3 x 360 against entries in registers at two CTAs), four slices in registers,
// broadcast by shuffles (0.21 -> 0.17 ms at 128^3 x 360 against the shared-memory slots).
constexpr int kBlkEnt = 64;  // int4 per slot: 32 angles x 32 bytes
template <int VZ, bool FULL>
__device__ __forceinline__ void k_backward_blk_body(const Args& a, const int4* __restrict__ tab,
                                                    const int* __restrict__ bcidx, unsigned bx) {
    __shared__ __align__(16) int4 s_ent[VZ == 8 ? kWarpsPerBlock : 1][2][kBlkEnt];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    // a CTA: 4 x 2 blocks (8 x 4 pixels, one block per warp) of one z chunk, so the warps of a CTA
    // read overlapping detector rows for the same angle at about the same time
    const int zc = (int)(bx % (unsigned)a.zchunks);
    const unsigned tile = bx / (unsigned)a.zchunks;
    const int nbx = (a.nX + 1) >> 1, nby = (a.nY + 1) >> 1;
    const int ntx = (nbx + 3) >> 2;
    const int bi = (int)(tile / ntx) * 2 + (wp >> 2), bj = (int)(tile % ntx) * 4 + (wp & 3);
    if (bi >= nby || bj >= nbx) return;
    const long blk = (long)bi * nbx + bj;
    int z0 = zc * 32 * VZ + 4 * lane, qn = VZ / 4;
    static_assert((VZ != 6 && VZ != 5) || FULL, "six / five slices per lane: full chunks only");
    if constexpr (!FULL) lane_z<VZ>(zc, lane, a.nZ, z0, qn);
    constexpr int NP = (VZ + 1) / 2;  // slice pairs
    unsigned long long acc[4][NP];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < NP; ++e) acc[q][e] = 0ull;
    const int pc = bcidx[blk];
    if (pc >= 0) {
        const int rs = a.nA * a.nZ;
        const float* __restrict__ bz = a.in + z0;
        const int4* __restrict__ e = tab + (size_t)pc * a.nA * 2;
        const int nA = a.nA;
        // one angle's rows and FMAs from its entry (e0: row offset, code, w0, w1; e1: w2, w3)
        auto angle = [&](const int4& e0, const int4& e1) {
            const int code = e0.y;
            const float w[4] = {__int_as_float(e0.z), __int_as_float(e0.w), __int_as_float(e1.x),
                                __int_as_float(e1.y)};
            const float* pr = bz + e0.x;
            const int span = code & 3;
            RowV<VZ> ra, rb, rc;
            load_row<VZ>(ra, pr, qn);
            load_row<VZ>(rb, pr + rs, qn);
            if (span >= 1) load_row<VZ>(rc, pr + 2 * rs, qn);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (((code >> (2 + 3 * q)) & 7) == 1) lerp_rows<VZ>(acc[q], w[q], ra, rb);
            if (span >= 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (((code >> (2 + 3 * q)) & 7) == 3) lerp_rows<VZ>(acc[q], w[q], rb, rc);
                if (span == 2) {
                    load_row<VZ>(ra, pr + 3 * rs, qn);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (((code >> (2 + 3 * q)) & 7) == 5) lerp_rows<VZ>(acc[q], w[q], rc, ra);
                }
            }
        };
        if constexpr (VZ == 8) {
            // entries by cp.async into the warp's two shared-memory slots: no registers held for them,
            // which lets the eight-slice body fit 80 registers (three CTAs per SM)
            int4* slot = &s_ent[wp][0][0];
            // chunk of angles k0 .. k0 + 31 into slot sl (one commit group per chunk, empty past the end)
            // the table is read once: evict-first in L2, so it does not push out sinogram lines that other
            // CTAs read again (DRAM 477 -> 459 MB per 256^3 x 360 launch, 0.934 -> 0.922 ms)
            unsigned long long pol;
            asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
            auto fetch = [&](int k0, int sl) {
                const int k = k0 + lane;
                int4* d = slot + sl * kBlkEnt + 2 * lane;
                if (k < nA) {
                    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(smem_addr(d)),
                                 "l"(e + 2 * k), "l"(pol) : "memory");
                    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(smem_addr(d + 1)),
                                 "l"(e + 2 * k + 1), "l"(pol) : "memory");
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            fetch(0, 0);
            fetch(32, 1);
#pragma unroll 1
            for (int k0 = 0, sl = 0; k0 < nA; k0 += 32, sl ^= 1) {
                const int kn = min(32, nA - k0);
                asm volatile("cp.async.wait_group 1;" ::: "memory");  // this chunk's copies (the next may fly)
                __syncwarp();
                const int4* es = slot + sl * kBlkEnt;
#pragma unroll 1
                for (int l = 0; l < kn; ++l) {
                    const int4 e0 = es[2 * l];
                    if (e0.x < 0) continue;  // uniform: every lane read the same entry
                    angle(e0, es[2 * l + 1]);
                }
                __syncwarp();  // every lane read the slot before it is refilled
                fetch(k0 + 64, sl);
            }
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncwarp();
        } else {
            // entries in registers (lane l: angle k0 + l, the next chunk in flight), broadcast by shuffles
            auto chunk = [&](int k0, int4& h0, int4& h1) {
                const int k = k0 + lane;
                if (k < nA) { h0 = __ldcs(e + 2 * k); h1 = __ldcs(e + 2 * k + 1); }
                else { h0 = make_int4(-1, 0, 0, 0); h1 = make_int4(0, 0, 0, 0); }
            };
            int4 h0, h1, g0, g1;
            chunk(0, h0, h1);
            chunk(32, g0, g1);
#pragma unroll 1
            for (int k0 = 0; k0 < nA; k0 += 32) {
                const int kn = min(32, nA - k0);
#pragma unroll 1
                for (int l = 0; l < kn; ++l) {
                    const int off = __shfl_sync(0xffffffffu, h0.x, l);
                    if (off < 0) continue;  // uniform: every lane read lane l's entry
                    const int4 e0 = make_int4(off, __shfl_sync(0xffffffffu, h0.y, l), __shfl_sync(0xffffffffu, h0.z, l),
                                              __shfl_sync(0xffffffffu, h0.w, l));
                    const int4 e1 = make_int4(__shfl_sync(0xffffffffu, h1.x, l), __shfl_sync(0xffffffffu, h1.y, l), 0, 0);
                    angle(e0, e1);
                }
                h0 = g0; h1 = g1;
                if (k0 + 64 < nA) chunk(k0 + 64, g0, g1);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int i = 2 * bi + (q >> 1), j = 2 * bj + (q & 1);
        if (i >= a.nY || j >= a.nX) continue;
        const long p = (long)i * a.nX + j;
        float v[2 * NP];
#pragma unroll
        for (int e2 = 0; e2 < NP; ++e2)
            asm("mov.b64 {%0, %1}, %2;" : "=f"(v[2 * e2]), "=f"(v[2 * e2 + 1]) : "l"(acc[q][e2]));
        if (a.mask) {
            const float m = __ldg(a.mask + p);
#pragma unroll
            for (int e2 = 0; e2 < VZ; ++e2) v[e2] = m * v[e2];
        }
        // streaming stores: the volume is not read again by this launch (0.924 -> 0.916 ms, DRAM reads
        // 399 -> 390 MB per 256^3 x 360 launch)
        float* dst = a.out + (size_t)p * a.nZ + z0;
        if constexpr (VZ == 6) {
            __stcs(reinterpret_cast<float4*>(dst), make_float4(v[0], v[1], v[2], v[3]));
            __stcs(reinterpret_cast<float2*>(dst + 128 - 2 * lane), make_float2(v[4], v[5]));
        } else if constexpr (VZ == 5) {
            __stcs(reinterpret_cast<float4*>(dst), make_float4(v[0], v[1], v[2], v[3]));
            __stcs(dst + 128 - 3 * lane, v[4]);
        } else {
#pragma unroll
            for (int q2 = 0; q2 < VZ / 4; ++q2)
                if (q2 < qn)
                    __stcs(reinterpret_cast<float4*>(dst + 128 * q2),
                           make_float4(v[4 * q2], v[4 * q2 + 1], v[4 * q2 + 2], v[4 * q2 + 3]));
        }
    }
}

template <int VZ, int MINB, bool FULL>
__global__ void __launch_bounds__(256, MINB) k_backward_blk(Args a, const int4* __restrict__ tab,
                                                            const int* __restrict__ bcidx) {
    k_backward_blk_body<VZ, FULL>(a, tab, bcidx, blockIdx.x);
}

// ---------------------------------------------------------------------------
// 2-D slices (nZ = 1): shared-memory tiles.
//
// With one slice there is no contiguous axis to put lanes on: a warp's taps
// land in up to 32 different cache lines.  These kernels stage, per tile, the
// region of the image (forward) or of the sinogram (backprojection) the tile's
// samples touch, with coalesced row loads, and gather from shared memory.
// The per-sample arithmetic is the generic kernels' (float64 coordinates and
// np.interp bin, float32 weights); taps that fall outside the staged region
// (not expected: the region is the tile's exact footprint plus a margin) are
// read from global memory with the same bounds checks.
// ---------------------------------------------------------------------------
constexpr int k2J = 64;     // forward: detector bins per tile
constexpr int k2K = 64;     // forward: samples per bin per tile
constexpr int k2Box = 96;   // forward: staged box side >= sqrt(2) (k2J + k2K - 2) + 5
constexpr int k2Stride = k2Box + 1;
constexpr int k2Smem = (k2Box * k2Stride + 4 * k2J) * 4;  // box + the k-group partial sums
constexpr int kB2 = 16;     // backprojection: pixel tile side
constexpr int kB2A = 32;    // backprojection: angles per staged block (one per lane when staging)
constexpr int kB2W = 30;    // backprojection: window bins per angle >= sqrt(2) (kB2 - 1) + 6
constexpr int kB2Smem = kB2A * kB2W * 4 + kB2A * 4 + kB2A * 16;

// grid (ceil(nX / k2J), nA); 256 threads = 64 bins x 4 groups of samples.
//
// Per tile the box [rlo, rlo + H) x [clo, clo + W) covers the footprint of all
// its samples with a margin of one pixel below and two above (rows and cols are
// affine in j and k, so the corners bound them); it is staged unclipped, with
// zeros outside the image, which is exactly the zero padding of the reference's
// warp, so every tap is an unconditional shared-memory read.  Each bin's
// coordinates are the reference's float64 values at the tile's first sample;
// the offsets along the ray are float32 (coordinate error below 2e-5 pixel on
// a continuous bilinear interpolant).
template <bool RAY>
__device__ __forceinline__ void k_forward_2d_body(const Args& a, unsigned bx, unsigned by) {
    extern __shared__ float s_f2[];
    float* box = s_f2;
    float* part = s_f2 + k2Box * k2Stride;
    const int theta = by;
    const int tj = threadIdx.x % k2J, tk = threadIdx.x / k2J;
    const int j0 = bx * k2J, j = j0 + tj;
    const int j1 = min(j0 + k2J, a.nX) - 1;
    const double4 tr = a.trig[theta];
    const double c = tr.x, s = tr.y;
    const float cf = (float)c, sf = (float)s;
    const double rowb = fma(-s, (double)j, tr.w), colb = fma(c, (double)j, tr.z);
    float s_entry = 0.f;
    bool live = j < a.nX;
    if (RAY) {
        const float t = (float)(j - a.C);
        if (fabsf(t) > a.R) live = false;
        else s_entry = -sqrtf(a.R * a.R - t * t);
    }
    const double rb0 = fma(-s, (double)j0, tr.w), rb1 = fma(-s, (double)j1, tr.w);
    const double cb0 = fma(c, (double)j0, tr.z), cb1 = fma(c, (double)j1, tr.z);
    auto to_int = [](double v) { return (int)fmax(fmin(floor(v), 1e9), -1e9); };
    float acc = 0.f;
    for (int k0 = 0; k0 < a.nY; k0 += k2K) {
        const int k1 = min(k0 + k2K, a.nY) - 1;
        double rmin = 1e300, rmax = -1e300, cmin = 1e300, cmax = -1e300;
        for (int q = 0; q < 4; ++q) {
            const double rb = (q & 1) ? rb1 : rb0, cb = (q & 1) ? cb1 : cb0;
            const double kk = (q & 2) ? (double)k1 : (double)k0;
            const double r = fma(c, kk, rb), cl = fma(s, kk, cb);
            rmin = fmin(rmin, r); rmax = fmax(rmax, r); cmin = fmin(cmin, cl); cmax = fmax(cmax, cl);
        }
        const int rlo = to_int(rmin) - 1, rhi = to_int(rmax) + 2;
        const int clo = to_int(cmin) - 1, chi = to_int(cmax) + 2;
        // the whole tile samples outside the image: every tap is zero padding (uniform)
        if (rhi < 0 || rlo > a.nY - 1 || chi < 0 || clo > a.nX - 1) continue;
        const int H = min(rhi - rlo + 1, k2Box), W = min(chi - clo + 1, k2Box);
        // warp w stages rows w, w + 8, ...; lanes run along the row (coalesced, no division)
        for (int r = (int)(threadIdx.x >> 5); r < H; r += kWarpsPerBlock) {
            const int gr = rlo + r;
            const bool rin = (unsigned)gr < (unsigned)a.nY;
            for (int cc = (int)(threadIdx.x & 31); cc < W; cc += 32) {
                const int gc = clo + cc;
                float v = 0.f;
                if (rin && (unsigned)gc < (unsigned)a.nX) {
                    const size_t g = (size_t)gr * a.nX + gc;
                    v = a.mask ? __ldg(a.mask + g) * __ldg(a.in + g) : __ldg(a.in + g);
                }
                box[r * k2Stride + cc] = v;
            }
        }
        __syncthreads();
        if (live) {
            const float rl0 = (float)(fma(c, (double)k0, rowb) - (double)rlo);
            const float cl0 = (float)(fma(s, (double)k0, colb) - (double)clo);
            for (int kk = tk; kk <= k1 - k0; kk += 4) {
                const float row = fmaf(cf, (float)kk, rl0), col = fmaf(sf, (float)kk, cl0);
                const float fr = floorf(row), fc = floorf(col);
                const float dr = row - fr, dc = col - fc;
                // clamped for memory safety only: the margins keep every weighted tap inside the box
                const int r0 = min(max((int)fr, 0), H - 2), c0 = min(max((int)fc, 0), W - 2);
                const float* t0 = box + r0 * k2Stride + c0;
                const float w00 = (1.f - dr) * (1.f - dc), w01 = (1.f - dr) * dc;
                const float w10 = dr * (1.f - dc), w11 = dr * dc;
                float v = w00 * t0[0];
                v = fmaf(w01, t0[1], v);
                v = fmaf(w10, t0[k2Stride], v);
                v = fmaf(w11, t0[k2Stride + 1], v);
                if (RAY) v *= ray_factor((float)(k0 + kk - a.C), s_entry, a.alpha);
                acc += v;
            }
        }
        __syncthreads();
    }
    part[tk * k2J + tj] = acc;
    __syncthreads();
    if (tk == 0 && j < a.nX) {
        const float sum = ((part[tj] + part[k2J + tj]) + part[2 * k2J + tj]) + part[3 * k2J + tj];
        a.out[(size_t)j * a.nA + theta] = sum;
    }
}

// The same tiles with the footprint box staged by one TMA tensor load per tile.
//
// A 2-D tensor map over the image (x = columns, y = rows, float32, zero fill
// outside) loads a 100 x 96 box into shared memory, signalled on an mbarrier:
// the box's x coordinate is the footprint's first column rounded down to a
// multiple of 4 (a tiled copy must start on a 16-byte boundary; the remainder
// is an offset into the box), its y coordinate the first row (negative and
// out-of-range coordinates read the fill value: exactly the reference's zero
// padding).  The samples are the plain tile kernel's, so the sums are
// bit-identical.  Replacing the block's bounds-checked row loads measured
// 0.75 -> 0.32 ms at 512^2 x 720, 0.44 -> 0.19 ms at 384^2 x 720 and
// 0.124 -> 0.049 ms at 256^2 x 360.  The tensor map needs rows a multiple of
// 16 bytes apart at a 16-byte aligned address: other images (and masked ones)
// are first copied into the plan's padded image, whose rows are nX rounded up
// to four floats (the map still ends at nX, so the padding is never read);
// 0.223 -> 0.105 ms at 363^2 x 360 with that copy.  The wait on the mbarrier
// is bounded: past the limit the block records VAM_STATUS_TIMEOUT in the
// plan's status word, waits (bounded) for its copy in flight and leaves its
// outputs unwritten.  A persistent batch runs the same body from its items'
// tensor maps (parameter space, like a direct launch's __grid_constant__ map).
constexpr int kTmaW = 100, kTmaH = 96;  // box: 100 columns (x, 400 B) x 96 rows
constexpr long kTmaWaitLimit = 1L << 24;  // try_wait polls before a block gives up
// dynamic shared memory of the TMA tile body: 128 B of alignment slack, the box, the k-group partial sums
// and the mbarrier
constexpr int k2SmemTma = 128 + kTmaH * kTmaW * 4 + 4 * k2J * 4 + 16;


__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    unsigned done = 0;
    for (long it = 0; it < kTmaWaitLimit && !done; ++it) {
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    }
    return done != 0;
}

// One block (tile of k2J bins x all samples, one angle) of the TMA-staged forward; tmap points to the
// image's tensor map in parameter space (a __grid_constant__ argument or a batch item).
template <bool RAY>
__device__ __forceinline__ void k_forward_2d_tma_body(const Args& a, const CUtensorMap* tmap, int* status,
                                                      unsigned bx, unsigned by) {
    extern __shared__ float s_f2[];
    float* box = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_f2) + 127) & ~(uintptr_t)127);
    float* part = box + kTmaH * kTmaW;
    unsigned long long* mbar = reinterpret_cast<unsigned long long*>(part + 4 * k2J);
    const unsigned bar = smem_addr(mbar);
    const int theta = by;
    const int tj = threadIdx.x % k2J, tk = threadIdx.x / k2J;
    const int j0 = bx * k2J, j = j0 + tj;
    const int j1 = min(j0 + k2J, a.nX) - 1;
    const double4 tr = a.trig[theta];
    const double c = tr.x, s = tr.y;
    const float cf = (float)c, sf = (float)s;
    const double rowb = fma(-s, (double)j, tr.w), colb = fma(c, (double)j, tr.z);
    float s_entry = 0.f;
    bool live = j < a.nX;
    if (RAY) {
        const float t = (float)(j - a.C);
        if (fabsf(t) > a.R) live = false;
        else s_entry = -sqrtf(a.R * a.R - t * t);
    }
    const double rb0 = fma(-s, (double)j0, tr.w), rb1 = fma(-s, (double)j1, tr.w);
    const double cb0 = fma(c, (double)j0, tr.z), cb1 = fma(c, (double)j1, tr.z);
    auto to_int = [](double v) { return (int)fmax(fmin(floor(v), 1e9), -1e9); };
    // the box may hold another body's generic-proxy writes (a persistent batch runs several bodies
    // in the same shared memory): order them before the tensor copies overwrite it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned phase = 0;
    bool failed = false;
    float acc = 0.f;
    for (int k0 = 0; k0 < a.nY; k0 += k2K) {
        const int k1 = min(k0 + k2K, a.nY) - 1;
        double rmin = 1e300, rmax = -1e300, cmin = 1e300, cmax = -1e300;
        for (int q = 0; q < 4; ++q) {
            const double rb = (q & 1) ? rb1 : rb0, cb = (q & 1) ? cb1 : cb0;
            const double kk = (q & 2) ? (double)k1 : (double)k0;
            const double r = fma(c, kk, rb), cl = fma(s, kk, cb);
            rmin = fmin(rmin, r); rmax = fmax(rmax, r); cmin = fmin(cmin, cl); cmax = fmax(cmax, cl);
        }
        const int rlo = to_int(rmin) - 1, rhi = to_int(rmax) + 2;
        const int clo = to_int(cmin) - 1, chi = to_int(cmax) + 2;
        // the whole tile samples outside the image: every tap is zero padding (uniform)
        if (rhi < 0 || rlo > a.nY - 1 || chi < 0 || clo > a.nX - 1) continue;
        const int H = min(rhi - rlo + 1, k2Box), W = min(chi - clo + 1, k2Box);
        const int cx = clo & ~3, cofs = clo - cx;  // the box's x on a 16-byte boundary, the remainder an offset
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"((unsigned)(kTmaH * kTmaW * 4)) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                ::"r"(smem_addr(box)), "l"(tmap), "r"(cx), "r"(rlo), "r"(bar) : "memory");
        }
        failed = !mbar_wait(bar, phase);
        phase ^= 1u;
        if (failed) break;  // uniform in practice; a block that gives up writes no outputs
        if (live) {
            const float rl0 = (float)(fma(c, (double)k0, rowb) - (double)rlo);
            const float cl0 = (float)(fma(s, (double)k0, colb) - (double)clo);
            for (int kk = tk; kk <= k1 - k0; kk += 4) {
                const float row = fmaf(cf, (float)kk, rl0), col = fmaf(sf, (float)kk, cl0);
                const float fr = floorf(row), fc = floorf(col);
                const float dr = row - fr, dc = col - fc;
                // clamped for memory safety only: the margins keep every weighted tap inside the box
                const int r0 = min(max((int)fr, 0), H - 2), c0 = min(max((int)fc, 0), W - 2);
                const float* t0 = box + r0 * kTmaW + c0 + cofs;
                const float w00 = (1.f - dr) * (1.f - dc), w01 = (1.f - dr) * dc;
                const float w10 = dr * (1.f - dc), w11 = dr * dc;
                float v = w00 * t0[0];
                v = fmaf(w01, t0[1], v);
                v = fmaf(w10, t0[kTmaW], v);
                v = fmaf(w11, t0[kTmaW + 1], v);
                if (RAY) v *= ray_factor((float)(k0 + kk - a.C), s_entry, a.alpha);
                acc += v;
            }
        }
        __syncthreads();  // every read of this box is done before the next copy overwrites it
    }
    if (failed) {
        mbar_wait(bar, phase ^ 1u);  // the copy may still be in flight: wait for it once more (bounded)
        if (threadIdx.x == 0) atomicOr(status, VAM_STATUS_TIMEOUT);
    } else {
        part[tk * k2J + tj] = acc;
        __syncthreads();
        if (tk == 0 && j < a.nX) {
            const float sum = ((part[tj] + part[k2J + tj]) + part[2 * k2J + tj]) + part[3 * k2J + tj];
            a.out[(size_t)j * a.nA + theta] = sum;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

template <bool RAY>
__global__ void __launch_bounds__(256) k_forward_2d_tma(Args a, const __grid_constant__ CUtensorMap tmap,
                                                        int* __restrict__ status) {
    k_forward_2d_tma_body<RAY>(a, &tmap, status, blockIdx.x, blockIdx.y);
}

template <bool RAY>
__global__ void __launch_bounds__(256) k_forward_2d(Args a) {
    k_forward_2d_body<RAY>(a, blockIdx.x, blockIdx.y);
}

// grid (ceil(nX / 16) * ceil(nY / 16)); 256 threads = one 16 x 16 pixel tile
template <bool RAY>
__device__ __forceinline__ void k_backward_2d_body(const Args& a, unsigned bx, unsigned by) {
    (void)by;
    extern __shared__ float s_b2[];
    float* win = s_b2;                                            // [kB2A][kB2W]
    int* wlo = reinterpret_cast<int*>(s_b2 + kB2A * kB2W);        // [kB2A] first staged detector row
    double2* cs = reinterpret_cast<double2*>(s_b2 + kB2A * kB2W + kB2A);  // [kB2A]
    const int tiles_x = (a.nX + kB2 - 1) / kB2;
    const int ti = bx / tiles_x, tjx = bx - ti * tiles_x;
    const int i0 = ti * kB2, jx0 = tjx * kB2;
    const int i = i0 + (int)threadIdx.x / kB2, j = jx0 + (int)threadIdx.x % kB2;
    const bool inside = i < a.nY && j < a.nX;
    const long p = (long)i * a.nX + j;
    const bool on = inside && a.circle[p];
    const double X = (double)(j - a.C), Y = (double)(i - a.C);
    const double tlo = (double)(-a.C), thi = (double)(a.nY - 1 - a.C);
    // tile corners for the windows
    const double Xa = (double)(jx0 - a.C), Xb = (double)(min(jx0 + kB2, a.nX) - 1 - a.C);
    const double Ya = (double)(i0 - a.C), Yb = (double)(min(i0 + kB2, a.nY) - 1 - a.C);
    float acc = 0.f;
    for (int th0 = 0; th0 < a.nA; th0 += kB2A) {
        const int na = min(kB2A, a.nA - th0);
        if (threadIdx.x < (unsigned)na) {
            const double4 tr = a.trig[th0 + threadIdx.x];
            cs[threadIdx.x] = make_double2(tr.x, tr.y);
            double tmin = 1e300, tmax = -1e300;
            for (int q = 0; q < 4; ++q) {
                const double x = (q & 1) ? Xb : Xa, y = (q & 2) ? Yb : Ya;
                const double t = __dsub_rn(__dmul_rn(x, tr.x), __dmul_rn(y, tr.y));
                tmin = fmin(tmin, t); tmax = fmax(tmax, t);
            }
            wlo[threadIdx.x] = max((int)fmax(fmin(floor(tmin), 1e9), -1e9) + a.C - 2, 0);
        }
        __syncthreads();
        // warp w stages window bins w, w + 8, ...; lane = angle (consecutive angles are contiguous)
        const int sa = (int)(threadIdx.x & 31);
        if (sa < na)
            for (int w = (int)(threadIdx.x >> 5); w < kB2W; w += kWarpsPerBlock) {
                const int row = wlo[sa] + w;
                win[sa * kB2W + w] = row < a.nY ? __ldg(a.in + (size_t)row * a.nA + th0 + sa) : 0.f;
            }
        __syncthreads();
        if (on) {
            for (int al = 0; al < na; ++al) {
                const double2 cc = cs[al];
                const double t = __dsub_rn(__dmul_rn(X, cc.x), __dmul_rn(Y, cc.y));
                if (!(t >= tlo && t <= thi)) continue;  // np.interp left = right = 0
                const double ft = floor(t);
                const int j0 = (int)ft + a.C;
                const int wi = j0 - wlo[al];
                const int th = th0 + al;
                auto row = [&](int r, int wr) -> float {
                    return (unsigned)wr < (unsigned)kB2W ? win[al * kB2W + wr] : __ldg(a.in + (size_t)r * a.nA + th);
                };
                float v = row(j0, wi);
                if (t != ft) v = fmaf((float)(t - ft), row(j0 + 1, wi + 1) - v, v);
                if (RAY) {
                    float f = 0.f;
                    if (fabs(t) <= (double)a.R) {
                        const float sv = (float)__dadd_rn(__dmul_rn(X, cc.y), __dmul_rn(Y, cc.x));
                        f = ray_factor(sv, (float)(-sqrt((double)a.R * a.R - t * t)), a.alpha);
                    }
                    v *= f;
                }
                acc += v;
            }
        }
        __syncthreads();
    }
    if (inside) {
        if (a.mask) acc = __ldg(a.mask + p) * acc;
        a.out[p] = acc;
    }
}

template <bool RAY>
__global__ void __launch_bounds__(256) k_backward_2d(Args a) {
    k_backward_2d_body<RAY>(a, blockIdx.x, blockIdx.y);
}

// out = mask (per pixel, broadcast over z) * x; with nZ % 4 == 0 and aligned buffers four
// slices of one pixel per thread and 16-byte load
__global__ void k_mask_mul(const float* __restrict__ x, const float* __restrict__ mask, float* __restrict__ out,
                           long npix, int nZ) {
    const long n = npix * nZ;
    const long stride = (long)gridDim.x * blockDim.x, t0 = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (nZ % 128 == 0 && (((uintptr_t)x | (uintptr_t)out) & 15) == 0) {
        // one warp per pixel row along z: no index division
        const int q = nZ / 4, lane = threadIdx.x & 31;
        const long nwarps = stride >> 5;
        for (long pix = t0 >> 5; pix < npix; pix += nwarps) {
            const float m = __ldg(mask + pix);
            const float4* xs = reinterpret_cast<const float4*>(x) + pix * q;
            float4* os = reinterpret_cast<float4*>(out) + pix * q;
            for (int i = lane; i < q; i += 32) {
                float4 v = __ldg(xs + i);
                v.x *= m; v.y *= m; v.z *= m; v.w *= m;
                os[i] = v;
            }
        }
        return;
    }
    for (long i = t0; i < n; i += stride) out[i] = mask[i / nZ] * x[i];
}

// rows of w floats of x (times mask, when given) into rows of wp >= w floats of out; the columns
// w .. wp - 1 are not written (the tensor map ends at w)
__device__ __forceinline__ void stage_rows(const float* __restrict__ x, const float* __restrict__ mask,
                                           float* __restrict__ out, long long npix, int w, int wp, long long t0,
                                           long long stride) {
    for (long long i = t0; i < npix; i += stride) {
        const long long y = i / w;
        const float v = mask ? mask[i] * x[i] : x[i];
        out[y * wp + (i - y * w)] = v;
    }
}

__global__ void k_stage_rows(const float* __restrict__ x, const float* __restrict__ mask, float* __restrict__ out,
                             long long npix, int w, int wp) {
    stage_rows(x, mask, out, npix, w, wp, (long long)blockIdx.x * blockDim.x + threadIdx.x,
               (long long)gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// R2 reference-parity backprojection
// ---------------------------------------------------------------------------
// np.interp(t, xp, fp, left=nan, right=nan) on the unit-spaced xp = k - C, in
// float64, for the occlusion sinogram (values are integers or NaN).
__device__ __forceinline__ double interp_nan(double t, double ft, int j0, int nY, int C, const float* occ,
                                             size_t stride) {
    if (t < (double)(-C) || t > (double)(nY - 1 - C)) return __longlong_as_double(0x7ff8000000000000LL);
    if (j0 == nY - 1 || t == ft) return (double)occ[(size_t)j0 * stride];
    double y0 = (double)occ[(size_t)j0 * stride], y1 = (double)occ[(size_t)(j0 + 1) * stride];
    // numpy evaluates slope*(x - xp[j]) + fp[j] without a fused multiply-add
    const double slope = y1 - y0;
    double res = __dadd_rn(__dmul_rn(slope, t - ft), y0);
    if (isnan(res)) {
        res = __dadd_rn(__dmul_rn(slope, t - (ft + 1.0)), y1);
        if (isnan(res) && y0 == y1) res = y0;
    }
    return res;
}

template <int VZ, bool OCC, int ABS>
__device__ __forceinline__ void k_backward_ref_body(const Args& a, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const int LZ = 1 << a.lz_shift;
    const int LK = 32 >> a.lz_shift;
    const int zl = lane & (LZ - 1);
    const int kl = lane >> a.lz_shift;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = (int)(item % a.zchunks);
    const long p = item / a.zchunks;
    if (p >= (long)a.nY * a.nX) return;
    const int i = (int)(p / a.nX), j = (int)(p % a.nX);
    const int zv = zc * LZ + zl;
    const bool zok = zv < a.zvec;
    const int z0 = zok ? zv * VZ : 0;
    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;

    if (a.circle[p]) {
        const double X = (double)(j - a.C), Y = (double)(i - a.C);
        const double tlo = (double)(-a.C), thi = (double)(a.nY - 1 - a.C);
        const size_t rs = (size_t)a.nA * a.nZ;  // sinogram row stride
        for (int th = kl; th < a.nA; th += LK) {
            const double4 tr = a.trig[th];
            const double t = __dsub_rn(__dmul_rn(X, tr.x), __dmul_rn(Y, tr.y));
            if (!(t >= tlo && t <= thi)) continue;  // np.interp left = right = 0
            const double ft = floor(t);
            const int j0 = (int)ft + a.C;
            const float* b0 = a.in + (size_t)j0 * rs + (size_t)th * a.nZ + z0;
            float v[VZ];
            if (zok) {
                load_vec<VZ>(b0, v);
                if (t != ft) {  // interior: fp[j] + (t - xp[j]) * (fp[j+1] - fp[j])
                    float v1[VZ];
                    load_vec<VZ>(b0 + rs, v1);
                    const float w = (float)(t - ft);
#pragma unroll
                    for (int e = 0; e < VZ; ++e) v[e] = fmaf(w, v1[e] - v[e], v[e]);
                }
            } else {
#pragma unroll
                for (int e = 0; e < VZ; ++e) v[e] = 0.f;
            }
            if (OCC && zok) {
                const double sv = __dadd_rn(__dmul_rn(X, tr.y), __dmul_rn(Y, tr.x));
                if (a.occ_mode == 1) {
                    // 2-D class (getOccShadow, Projector2DParallel.py:235-247): s against the minimum of t's
                    // np.digitize bin, which for t inside the detector is the interpolation bin j0; NaN
                    // (no occluder) compares false
                    if (sv > a.occ64[(size_t)j0 * a.nA + th]) v[0] = 0.f;
                } else {
#pragma unroll
                    for (int e = 0; e < VZ; ++e) {
                        const double o = interp_nan(t, ft, j0, a.nY, a.C, a.occ + (size_t)th * a.nZ + z0 + e, rs);
                        if (sv > floor(o)) v[e] = 0.f;
                    }
                }
            }
            if (ABS == VAM_ABS_RAY) {
                // |t| <= R is a discontinuity of the model: decide it on the float64 t
                float f = 0.f;
                if (fabs(t) <= (double)a.R) {
                    const float sv = (float)__dadd_rn(__dmul_rn(X, tr.y), __dmul_rn(Y, tr.x));
                    f = ray_factor(sv, (float)(-sqrt((double)a.R * a.R - t * t)), a.alpha);
                }
#pragma unroll
                for (int e = 0; e < VZ; ++e) v[e] *= f;
            }
#pragma unroll
            for (int e = 0; e < VZ; ++e) acc[e] += v[e];
        }
    }
#pragma unroll
    for (int e = 0; e < VZ; ++e)
        for (int off = LZ; off < 32; off <<= 1) acc[e] += __shfl_xor_sync(kFull, acc[e], off);
    if (ABS == VAM_ABS_MASK) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = m * acc[e];
    }
    if (kl == 0 && zok) store_vec<VZ>(a.out + (size_t)p * a.nZ + z0, acc);
}

template <int VZ, bool OCC, int ABS>
__global__ void __launch_bounds__(256) k_backward_ref(Args a) {
    k_backward_ref_body<VZ, OCC, ABS>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Matched transpose of k_forward
// ---------------------------------------------------------------------------
template <int VZ, bool OCC, int ABS>
__device__ __forceinline__ void k_adjoint_body(const Args& a, unsigned bx, unsigned by) {
    const int lane = threadIdx.x & 31;
    const int LZ = 1 << a.lz_shift;
    const int LK = 32 >> a.lz_shift;
    const int zl = lane & (LZ - 1);
    const int kl = lane >> a.lz_shift;
    const long item = (long)bx * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = (int)(item % a.zchunks);
    const long p = item / a.zchunks;
    if (p >= (long)a.nY * a.nX) return;
    const int i = (int)(p / a.nX), j = (int)(p % a.nX);
    const int zv = zc * LZ + zl;
    const bool zok = zv < a.zvec;
    const int z0 = zok ? zv * VZ : 0;
    const float Xf = (float)(j - a.C), Yf = (float)(i - a.C), Cf = (float)a.C;
    const size_t rs = (size_t)a.nA * a.nZ;
    float acc[VZ];
#pragma unroll
    for (int e = 0; e < VZ; ++e) acc[e] = 0.f;

    for (int th = kl; th < a.nA; th += LK) {
        const double4 tr = a.trig[th];
        const double c = tr.x, s = tr.y;
        const float cf = (float)c, sf = (float)s;
        // inverse rotation of the pixel into lattice coordinates (j*, k*)
        const float jf = Cf + cf * Xf - sf * Yf;
        const float kf = Cf + sf * Xf + cf * Yf;
        const int jlo = max(0, (int)ceilf(jf - 1.4143f)), jhi = min(a.nX - 1, (int)floorf(jf + 1.4143f));
        const int klo = max(0, (int)ceilf(kf - 1.4143f)), khi = min(a.nY - 1, (int)floorf(kf + 1.4143f));
        for (int jj = jlo; jj <= jhi; ++jj) {
            const double rowb = fma(-s, (double)jj, tr.w);
            const double colb = fma(c, (double)jj, tr.z);
            float s_entry = 0.f;
            if (ABS == VAM_ABS_RAY) {
                const float t = (float)(jj - a.C);
                if (fabsf(t) > a.R) continue;
                s_entry = -sqrtf(a.R * a.R - t * t);
            }
            int kstop[VZ];
#pragma unroll
            for (int e = 0; e < VZ; ++e) kstop[e] = INT_MAX;
            if (OCC && zok) {
#pragma unroll
                for (int e = 0; e < VZ; ++e) {
                    const float o = a.occ[(size_t)jj * rs + (size_t)th * a.nZ + z0 + e];
                    if (a.occ_flag[(size_t)th * a.nZ + z0 + e] && !isnan(o)) kstop[e] = (int)o + a.C;
                }
            }
            float W[VZ];
#pragma unroll
            for (int e = 0; e < VZ; ++e) W[e] = 0.f;
            const float rowbf = (float)rowb, colbf = (float)colb;
            for (int kk = klo; kk <= khi; ++kk) {
                // cheap float32 rejection (|error| << 1e-3), exact test below
                if (fabsf(fmaf(cf, (float)kk, rowbf) - (float)i) > 1.001f) continue;
                if (fabsf(fmaf(sf, (float)kk, colbf) - (float)j) > 1.001f) continue;
                const double row = fma(c, (double)kk, rowb);
                const double col = fma(s, (double)kk, colb);
                const double fr = floor(row), fc = floor(col);
                const int r0 = (int)fr, c0 = (int)fc;
                const bool rc = row > fr, cc = col > fc;
                if (!(i == r0 || (rc && i == r0 + 1))) continue;
                if (!(j == c0 || (cc && j == c0 + 1))) continue;
                const float dr = (float)(row - fr), dc = (float)(col - fc);
                const float wr = (i == r0) ? (1.f - dr) : dr;
                const float wc = (j == c0) ? (1.f - dc) : dc;
                float w = wr * wc;
                if (ABS == VAM_ABS_RAY) w *= ray_factor((float)(kk - a.C), s_entry, a.alpha);
#pragma unroll
                for (int e = 0; e < VZ; ++e) W[e] += (OCC && kk > kstop[e]) ? 0.f : w;
            }
            bool any = false;
#pragma unroll
            for (int e = 0; e < VZ; ++e) any |= (W[e] != 0.f);
            if (any && zok) {
                float bv[VZ];
                load_vec<VZ>(a.in + (size_t)jj * rs + (size_t)th * a.nZ + z0, bv);
#pragma unroll
                for (int e = 0; e < VZ; ++e) acc[e] = fmaf(W[e], bv[e], acc[e]);
            }
        }
    }
#pragma unroll
    for (int e = 0; e < VZ; ++e)
        for (int off = LZ; off < 32; off <<= 1) acc[e] += __shfl_xor_sync(kFull, acc[e], off);
    if (ABS == VAM_ABS_MASK) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = m * acc[e];
    }
    if (kl == 0 && zok) store_vec<VZ>(a.out + (size_t)p * a.nZ + z0, acc);
}

template <int VZ, bool OCC, int ABS>
__global__ void __launch_bounds__(256) k_adjoint(Args a) {
    k_adjoint_body<VZ, OCC, ABS>(a, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Occlusion sinogram: first row k where warp(insert) > 0, as (k - C); NaN if none.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_occ_sinogram(const float* __restrict__ ins, float* __restrict__ occ,
                                                      const double4* __restrict__ trig, int nY, int nX, int nZ,
                                                      int nA, int C) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;  // over (j, theta, z), z fastest
    if (idx >= (long)nX * nA * nZ) return;
    const int z = (int)(idx % nZ);
    const int th = (int)((idx / nZ) % nA);
    const int j = (int)(idx / ((long)nZ * nA));
    const double4 tr = trig[th];
    const double c = tr.x, s = tr.y;
    const double rowb = fma(-s, (double)j, tr.w);
    const double colb = fma(c, (double)j, tr.z);
    int klo, khi;
    sample_range(rowb, colb, c, s, nY, nX, nY - 1, klo, khi);
    float best = __int_as_float(0x7fc00000);
    // The "> 0" test is discontinuous in the coordinates, so they are formed
    // in skimage's unfused order, (M00*x + M01*y) + M02, bit-identical to the
    // reference (a fused multiply-add moves values off an integer by 1 ulp and
    // changes which neighbour gets a tiny positive weight).
    const double cj = __dmul_rn(c, (double)j), msj = __dmul_rn(-s, (double)j);
    for (int k = klo; k <= khi; ++k) {
        const double row = __dadd_rn(__dadd_rn(msj, __dmul_rn(c, (double)k)), tr.w);
        const double col = __dadd_rn(__dadd_rn(cj, __dmul_rn(s, (double)k)), tr.z);
        const double fr = floor(row), fc = floor(col);
        const int r0 = (int)fr, c0 = (int)fc;
        const bool rc = row > fr, cc = col > fc;
        // the bilinear value is > 0 iff a positive-weight tap is > 0
        auto tap = [&](int r, int cl) -> bool {
            return (unsigned)r < (unsigned)nY && (unsigned)cl < (unsigned)nX &&
                   ins[((size_t)r * nX + cl) * nZ + z] > 0.f;
        };
        bool hit = tap(r0, c0) || (cc && tap(r0, c0 + 1)) || (rc && tap(r0 + 1, c0)) ||
                   (rc && cc && tap(r0 + 1, c0 + 1));
        if (hit) { best = (float)(k - C); break; }
    }
    occ[idx] = best;
}

// occ_flag[theta][z] = any finite nonzero occ[j][theta][z] over j (Projector3DParallel.py:149)
__global__ void k_occ_flag(const float* __restrict__ occ, uint8_t* __restrict__ flag, int nX, int nA, int nZ) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)nA * nZ) return;
    uint8_t f = 0;
    for (int j = 0; j < nX; ++j) {
        const float o = occ[(size_t)j * nA * nZ + idx];
        if (!isnan(o) && o != 0.f) { f = 1; break; }
    }
    flag[idx] = f;
}

// ---------------------------------------------------------------------------
// The 2-D class's digitised occlusion sinogram (Projector2DParallel.py:70-143).
// Per angle every occluded pixel's detector coordinate t = x cos - y sin goes to
// its np.digitize bin over proj_t (index -1, i.e. the last bin's value, below
// the first bin), and each bin keeps the least s = x sin + y cos of its pixels.
// Slots: [nA][n + 1], slot 0 the wrapped index -1, slot 1 + k bin k; minima by
// atomicMin on an order-preserving integer key of the float64 s (exact and
// independent of the order of the atomics).
// ---------------------------------------------------------------------------
constexpr unsigned long long kOccEmpty = ~0ull;

__device__ __forceinline__ unsigned long long occ_key(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double occ_value(unsigned long long k) {
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__global__ void __launch_bounds__(256) k_occ2d_bin(const uint8_t* __restrict__ occlusion,
                                                   const double4* __restrict__ trig,
                                                   unsigned long long* __restrict__ slots, int n, int nA, int C) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // over (angle, pixel)
    if (idx >= (long long)nA * n * n) return;
    const int p = (int)(idx % ((long long)n * n));
    const int th = (int)(idx / ((long long)n * n));
    if (!occlusion[p]) return;
    const double X = (double)(p % n - C), Y = (double)(p / n - C);
    const double4 tr = trig[th];
    const double t = __dsub_rn(__dmul_rn(X, tr.x), __dmul_rn(Y, tr.y));
    const double s = __dadd_rn(__dmul_rn(X, tr.y), __dmul_rn(Y, tr.x));
    const int k = t < (double)(-C) ? 0 : 1 + min((int)floor(t) + C, n - 1);
    atomicMin(slots + (size_t)th * (n + 1) + k, occ_key(s));
}

// One thread per angle: the reference pairs the sorted unique bin indices with the per-bin minima
// sorted by bin value.  Without a wrapped index that is each bin's own minimum; with one (index -1,
// valued as the last bin) the minima shift by one bin, and if the last bin is occupied as well the
// two lists differ in length and the reference raises (flag bit 1).  An empty occlusion makes the
// reference take the minimum of an empty group (flag bit 2).
__global__ void k_occ2d_assign(const unsigned long long* __restrict__ slots, double* __restrict__ occ64,
                               float* __restrict__ occ, uint8_t* __restrict__ flag, int* __restrict__ err, int n,
                               int nA) {
    const int th = blockIdx.x * blockDim.x + threadIdx.x;
    if (th >= nA) return;
    const unsigned long long* sl = slots + (size_t)th * (n + 1);
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    for (int j = 0; j < n; ++j) occ64[(size_t)j * nA + th] = qnan;
    const unsigned long long wrap = sl[0];
    bool any = wrap != kOccEmpty;
    if (wrap == kOccEmpty) {
        for (int j = 0; j < n; ++j)
            if (sl[1 + j] != kOccEmpty) { occ64[(size_t)j * nA + th] = occ_value(sl[1 + j]); any = true; }
    } else if (sl[n] != kOccEmpty) {
        atomicOr(err, 1);
    } else {
        int prev = n - 1;
        for (int j = 0; j < n - 1; ++j) {
            if (sl[1 + j] == kOccEmpty) continue;
            occ64[(size_t)prev * nA + th] = occ_value(sl[1 + j]);
            prev = j;
        }
        occ64[(size_t)prev * nA + th] = occ_value(wrap);
    }
    if (!any) atomicOr(err, 2);
    // the forward's shadow test compares the integer sample coordinate k - C with the minimum:
    // k - C > v <=> k - C > floor(v), so the forward table holds floor(v) (exact in float32)
    for (int j = 0; j < n; ++j) {
        const double v = occ64[(size_t)j * nA + th];
        occ[(size_t)j * nA + th] = isnan(v) ? __double2float_rn(v) : (float)floor(v);
    }
    flag[th] = 1;
}

enum class Op { Forward, BackwardRef, Adjoint };

// Slices per lane of the fast kernels for nZ slices (0 = use the generic
// kernel): the widest vector whose lanes are at least min_eff busy.  The fast
// forward gathers about four times as many samples per second as the generic
// one, so it pays even with half of its lanes idle; the backprojectors' fast
// and generic kernels are closer, so they ask for busier lanes.
int fast_vz(int nZ, bool aligned, double min_eff) {
    if (!aligned || nZ % 4) return 0;
    auto eff = [&](int vz) {
        const int per = 32 * vz, ch = (nZ + per - 1) / per;
        return (double)nZ / (double)(ch * per);
    };
    if (eff(8) >= 0.74) return 8;
    if (eff(4) >= min_eff) return 4;
    return 0;
}

// ---------------------------------------------------------------------------
// Dispatch.  describe() decides which kernel body serves a call (fast or
// generic path, vector width, angle batch, weight table) and fills its
// arguments and grid; a direct call launches that one kernel, a batch runs the
// same body for many calls inside one persistent launch.  Both paths therefore
// compute bit-identical results.
// ---------------------------------------------------------------------------
enum Kind : int { KF_FAST = 0, KF_GEN, KB_BATCHED, KB_FAST, KB_GEN, KA_TABLE, KA_FAST, KA_GEN, KF_2D, KB_2D, KB_BTABLE };

struct Item {
    int kind;
    int vz;          // slices per lane of the template instance (1, 4 or 8)
    int ray, occ, absm, batch;
    unsigned gx, gy;  // the call's own grid (blocks of kWarpsPerBlock warps)
    unsigned smem;    // dynamic shared memory of the body
    int pre_nz;
    long long tstart;  // first ticket (virtual block) of the call inside a batch launch
    long long cost;    // estimated time of the call (batch ordering)
    int family;        // body family (k_batch instances): a bit of the FAM mask
    // pre-pass of the fast forward in mask mode: pre_out = mask * pre_in; of the 2-D tile forward
    // (pre_wp > 0): rows of pre_w floats of (mask *) pre_in into rows of pre_wp floats of pre_out
    const float* pre_in;
    const float* pre_mask;
    float* pre_out;
    long long pre_npix;
    int pre_w, pre_wp;
    Args a;
    FastArgs f;
    const float4* table;
    const int4* btab4;  // KB_BTABLE: the plan's 2 x 2 block bin table and its block index
    const int* bcidx;
    int* status;       // the plan's status word (kernels with bounded waits record timeouts there)
    int tma, tma_pad_;  // KF_2D: 1 when tmap describes a.in and the tiles are staged by TMA loads
    CUtensorMap tmap;   // read from parameter space, as a direct launch's __grid_constant__ argument
};
static_assert(sizeof(Item) % 8 == 0, "Item is copied to shared memory in 8-byte words");

bool image_tensor_map(const float* img, int nX, int nY, int row_stride, CUtensorMap& m);
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

int describe(vam_parallel_plan* plan, Op op, const float* in, float* out, Item& it, const char* name,
             bool noclip = false, bool in_batch = false) {
    VAM_REQUIRE(plan && in && out, VAM_ERR_ARG, std::string(name) + ": null argument");
    VAM_REQUIRE(!noclip || plan->d_ones, VAM_ERR_ARG, std::string(name) + ": no all-ones circle table");
    std::memset(&it, 0, sizeof(it));
    it.cost = (long long)plan->nY * plan->nX * plan->nZ * plan->nA;
    it.family = op == Op::Forward ? 1 : (op == Op::BackwardRef ? 2 : 4);
    it.gy = 1;
    // slices per lane: tuned (1 = generic kernel, 4 or 8 = fast kernel) or automatic (0)
    const bool fast_ok = (((uintptr_t)in | (uintptr_t)out) & 31) == 0 && plan->nZ % 4 == 0;
    const int want = op == Op::Forward ? plan->tune_fwd_vz : (op == Op::BackwardRef ? plan->tune_bwd_vz : plan->tune_adj_vz);
    int vzf = 0;
    if (fast_ok) {
        if (want == 4 || want == 8) vzf = want;
        else if (want == 0) vzf = fast_vz(plan->nZ, true, op == Op::Forward ? 0.45 : 0.74);
    }
    const bool ray = plan->abs_mode == VAM_ABS_RAY;
    // 2-D slice: shared-memory tiles when tuned to them (any width but 1), or automatically for
    // slices wide enough to fill the device with tiles (forward from 192, backprojection from 320 px)
    const bool tiles_2d = want == 0 ? plan->nX >= (op == Op::Forward ? 192 : 320) : want != 1;
    if (plan->nZ == 1 && !plan->has_occ && op != Op::Adjoint && tiles_2d && !noclip) {
        Args& a = it.a;
        a.in = in; a.out = out; a.trig = plan->d_trig; a.circle = plan->d_circle;
        a.mask = plan->abs_mode == VAM_ABS_MASK ? plan->d_mask : nullptr;
        a.nY = plan->nY; a.nX = plan->nX; a.nZ = 1; a.nA = plan->nA; a.C = plan->C;
        a.alpha = plan->abs_alpha; a.R = plan->abs_R;
        it.ray = ray;
        it.vz = 1;
        if (op == Op::Forward) {
            const bool aligned = (((uintptr_t)in) & 15) == 0 && plan->nX % 4 == 0;
            const bool use_tma = plan->tune_fwd_tma && tensor_map_encoder();
            const int wp = (plan->nX + 3) & ~3;
            if (plan->d_img_pad && use_tma && (a.mask || !aligned)) {
                // TMA rows start on 16-byte boundaries: stage (the masked) image once per call into
                // rows of a multiple of four floats
                it.pre_in = in; it.pre_mask = a.mask; it.pre_out = plan->d_img_pad;
                it.pre_npix = (long long)plan->nY * plan->nX; it.pre_nz = 1;
                it.pre_w = plan->nX; it.pre_wp = wp;
                a.in = plan->d_img_pad;
                a.mask = nullptr;
            } else if (a.mask) {  // stage the masked image once per call instead of per tile
                it.pre_in = in; it.pre_mask = plan->d_mask; it.pre_out = plan->d_vol_scratch;
                it.pre_npix = (long long)plan->nY * plan->nX; it.pre_nz = 1;
                a.in = plan->d_vol_scratch;
                a.mask = nullptr;
            }
            it.kind = KF_2D;
            it.family = 128;
            it.status = plan->d_status;
            it.tma = use_tma && image_tensor_map(a.in, a.nX, a.nY, it.pre_wp ? it.pre_wp : a.nX, it.tmap) ? 1 : 0;
            it.gx = (unsigned)((plan->nX + k2J - 1) / k2J);
            it.gy = (unsigned)plan->nA;
            it.smem = it.tma ? k2SmemTma : k2Smem;
        } else {
            it.kind = KB_2D;
            it.gx = (unsigned)(((plan->nX + kB2 - 1) / kB2) * ((plan->nY + kB2 - 1) / kB2));
            it.smem = kB2Smem;
        }
        return VAM_OK;
    }
    // the forward's slices per lane: also six / five where 192- / 160-slice chunks fill every lane
    // (tuned to 6 / 5, or automatic when 256-slice chunks would not)
    int fvz = vzf;
    if (fast_ok && plan->nZ % 192 == 0 && (want == 6 || (want == 0 && plan->nZ % 256 != 0))) fvz = 6;
    else if (fast_ok && plan->nZ % 160 == 0 && (want == 5 || (want == 0 && plan->nZ % 256 != 0))) fvz = 5;
    if (op == Op::Forward && !plan->has_occ && (long)plan->nY * plan->nX * plan->nZ < (1L << 31) && fvz) {
        FastArgs& a = it.f;
        a.vol = in;
        if (plan->abs_mode == VAM_ABS_MASK) {
            it.pre_in = in; it.pre_mask = plan->d_mask; it.pre_out = plan->d_vol_scratch;
            it.pre_npix = (long long)plan->nY * plan->nX; it.pre_nz = plan->nZ;
            a.vol = plan->d_vol_scratch;
        }
        a.sino = out; a.trig = plan->d_trig;
        a.nY = plan->nY; a.nX = plan->nX; a.nZ = plan->nZ; a.nA = plan->nA; a.C = plan->C;
        a.RS = plan->nX * plan->nZ;
        a.zchunks = (plan->nZ + 32 * fvz - 1) / (32 * fvz);
        a.even = (plan->nY % 2) == 0;
        a.alpha = plan->abs_alpha; a.R = plan->abs_R;
        a.tasks = ray ? plan->d_tasks_single : plan->d_tasks_paired;
        const long items = (long)(plan->nX + 1) * a.zchunks;
        it.kind = KF_FAST; it.vz = fvz; it.ray = ray;
        it.gx = (unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock);
        it.gy = (unsigned)(ray ? plan->nA : plan->n_tasks_paired);
        return VAM_OK;
    }
    // the block-table backprojection serves every nZ % 4 == 0, also where the automatic width of the
    // computed-bin kernels would fall back to the generic kernel (too many idle lanes)
    const bool blk_ok = op == Op::BackwardRef && fast_ok && !ray && plan->d_bwd_btab && plan->tune_bwd_table;
    if (op != Op::Forward && !plan->has_occ && (vzf || blk_ok) && !noclip &&
        (long long)plan->nY * plan->nA * plan->nZ < (1LL << 31)) {
        Args& a = it.a;
        a.in = in; a.out = out; a.trig = plan->d_trig; a.circle = plan->d_circle;
        a.mask = plan->abs_mode == VAM_ABS_MASK ? plan->d_mask : nullptr;
        a.nY = plan->nY; a.nX = plan->nX; a.nZ = plan->nZ; a.nA = plan->nA; a.C = plan->C;
        const int vzc = vzf ? vzf : 4;  // vzf == 0 only where the block table serves the call (blk_ok)
        a.zchunks = (plan->nZ + 32 * vzc - 1) / (32 * vzc);
        a.alpha = plan->abs_alpha; a.R = plan->abs_R;
        const long items = (long)plan->nY * plan->nX * a.zchunks;
        it.gx = (unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock);
        it.vz = vzf; it.ray = ray;
        if (op == Op::BackwardRef) {
            // the batched kernel stages cos / sin of every angle in shared memory (16 B per angle)
            const int batch = (size_t)plan->nA * sizeof(double2) <= 48 * 1024 ? plan->tune_bwd_batch : 1;
            if (blk_ok) {
                // the 2 x 2 block table: slices per lane as tuned (4 or 8), else eight for full 256-slice
                // chunks, six / five for full 192- / 160-slice chunks, eight from 160 slices up, four below
                // (256^3 x 360: 0.92 / 1.41 ms with 8 / 4; 192^3 x 720: 1.46 / 1.94; 96^3 x 720: 0.42 / 0.31)
                int bvz = 4;
                if (plan->tune_bwd_vz == 8 || plan->tune_bwd_vz == 4) bvz = plan->tune_bwd_vz;
                else if (plan->nZ % 256 == 0) bvz = 8;
                else if (plan->nZ % 192 == 0) bvz = 6;
                else if (plan->nZ % 160 == 0) bvz = 5;
                else if (plan->nZ >= 160) bvz = 8;
                it.kind = KB_BTABLE;
                it.vz = bvz;
                a.zchunks = (plan->nZ + 32 * bvz - 1) / (32 * bvz);
                const long ntx = ((plan->nX + 1) / 2 + 3) / 4, nty = ((plan->nY + 1) / 2 + 1) / 2;
                it.gx = (unsigned)(ntx * nty * a.zchunks);
                it.btab4 = plan->d_bwd_btab;
                it.bcidx = plan->d_bwd_bcidx;
            } else if (batch >= 2) {
                it.kind = KB_BATCHED;
                it.batch = vzf == 8 ? 2 : (batch >= 4 ? 4 : 2);
                it.smem = (unsigned)(sizeof(double2) * plan->nA);
            } else {
                it.kind = KB_FAST;
            }
        } else if (plan->d_adj_table && plan->adj_table_abs == plan->abs_mode && plan->tune_adj_table) {
            it.kind = KA_TABLE;
            it.table = plan->d_adj_table;
        } else {
            it.kind = KA_FAST;
        }
        return VAM_OK;
    }
    const bool aligned = (((uintptr_t)in | (uintptr_t)out) & 15) == 0;
    Layout L = choose_layout(plan->nZ, aligned);
    Args& a = it.a;
    a.in = in; a.out = out; a.trig = plan->d_trig; a.circle = noclip ? plan->d_ones : plan->d_circle;
    a.mask = plan->d_mask; a.occ = plan->d_occ; a.occ_flag = plan->d_occ_flag;
    a.occ64 = plan->d_occ64; a.occ_mode = plan->has_occ ? plan->occ_mode : 0;
    a.nY = plan->nY; a.nX = plan->nX; a.nZ = plan->nZ; a.nA = plan->nA; a.C = plan->C;
    a.lz_shift = L.lz_shift; a.zvec = L.zvec; a.zchunks = L.zchunks;
    a.alpha = plan->abs_alpha; a.R = plan->abs_R;
    const long items = (op == Op::Forward) ? (long)plan->nX * L.zchunks : (long)plan->nY * plan->nX * L.zchunks;
    it.kind = op == Op::Forward ? KF_GEN : (op == Op::BackwardRef ? KB_GEN : KA_GEN);
    it.vz = L.VZ; it.occ = plan->has_occ != 0; it.absm = plan->abs_mode;
    it.gx = (unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock);
    it.gy = op == Op::Forward ? (unsigned)plan->nA : 1u;
    return VAM_OK;
}

// ---- the body of a described call, for one block (bx, by) of its grid
// The bodies receive a local copy of their arguments: read once from the
// launch's parameter space into registers, instead of an indexed
// constant-cache load at every use inside the sample loops.
template <int FAM, int VZ, bool OCC, int ABS>
__device__ __forceinline__ void gen_body(const Item& it, unsigned bx, unsigned by) {
    const Args a = it.a;
    if constexpr ((FAM & 16) != 0) if (it.kind == KF_GEN) k_forward_body<VZ, OCC, ABS>(a, bx, by);
    if constexpr ((FAM & 8) != 0) if (it.kind == KB_GEN) k_backward_ref_body<VZ, OCC, ABS>(a, bx, by);
    if constexpr ((FAM & 4) != 0) if (it.kind == KA_GEN) k_adjoint_body<VZ, OCC, ABS>(a, bx, by);
}

template <int FAM, int VZ, int ABS>
__device__ __forceinline__ void lean_gen_body(const Item& it, const Args& a, unsigned bx, unsigned by) {
    if constexpr (FAM == 32) if (it.kind == KF_GEN) k_forward_body<VZ, false, ABS>(a, bx, by);
    if constexpr (FAM == 64) if (it.kind == KB_GEN) k_backward_ref_body<VZ, false, ABS>(a, bx, by);
}

template <int FAM, int VZ, bool OCC>
__device__ __forceinline__ void gen_body_fam(const Item& it, unsigned bx, unsigned by) {
    if (it.absm == VAM_ABS_MASK) gen_body<FAM, VZ, OCC, VAM_ABS_MASK>(it, bx, by);
    else if (it.absm == VAM_ABS_RAY) gen_body<FAM, VZ, OCC, VAM_ABS_RAY>(it, bx, by);
    else gen_body<FAM, VZ, OCC, VAM_ABS_NONE>(it, bx, by);
}

template <int FAM, bool RAY>
__device__ __forceinline__ void fast_body(const Item& it, unsigned bx, unsigned by) {
    if constexpr ((FAM & 1) != 0) {
        if (it.kind == KF_FAST) {
            const FastArgs f = it.f;
            if (it.vz == 8) k_forward_fast_body<8, RAY>(f, bx, by);
            else if (it.vz == 6) k_forward_fast_body<6, RAY>(f, bx, by);
            else if (it.vz == 5) k_forward_fast_body<5, RAY>(f, bx, by);
            else k_forward_fast_body<4, RAY>(f, bx, by);
        }
    }
    if constexpr ((FAM & 128) != 0) {
        if (it.kind == KF_2D) {
            const Args a = it.a;
            if (it.tma) k_forward_2d_tma_body<RAY>(a, &it.tmap, it.status, bx, by);
            else if constexpr (FAM == 511) k_forward_2d_body<RAY>(a, bx, by);
        }
    }
    if constexpr (FAM == 256 && !RAY) {
        if (it.kind == KB_BTABLE) {
            const Args a = it.a;
            const bool full = a.nZ % (32 * it.vz) == 0;
            if (it.vz == 8) { if (full) k_backward_blk_body<8, true>(a, it.btab4, it.bcidx, bx); else k_backward_blk_body<8, false>(a, it.btab4, it.bcidx, bx); }
            else if (it.vz == 6) k_backward_blk_body<6, true>(a, it.btab4, it.bcidx, bx);
            else if (it.vz == 5) k_backward_blk_body<5, true>(a, it.btab4, it.bcidx, bx);
            else { if (full) k_backward_blk_body<4, true>(a, it.btab4, it.bcidx, bx); else k_backward_blk_body<4, false>(a, it.btab4, it.bcidx, bx); }
        }
    }
    if constexpr ((FAM & 8) != 0 || ((FAM & 2) != 0 && !RAY)) {
        if (it.kind == KB_2D) {
            const Args a = it.a;
            k_backward_2d_body<RAY>(a, bx, by);
        } else if (it.kind == KB_BATCHED) {
            const Args a = it.a;
            if (it.vz == 8) k_backward_batched_body<8, 2, RAY>(a, bx, by);
            else if (it.batch == 4) k_backward_batched_body<4, 4, RAY>(a, bx, by);
            else k_backward_batched_body<4, 2, RAY>(a, bx, by);
        } else if (it.kind == KB_FAST) {
            const Args a = it.a;
            if (it.vz == 8) k_backward_fast_body<8, RAY>(a, bx, by);
            else k_backward_fast_body<4, RAY>(a, bx, by);
        }
    }
    if constexpr ((FAM & 4) != 0) {
        if (it.kind == KA_FAST) {
            const Args a = it.a;
            if (it.vz == 8) k_adjoint_fast_body<8, RAY>(a, bx, by);
            else k_adjoint_fast_body<4, RAY>(a, bx, by);
        }
    }
}

// FAM: the body families this instance carries -- 1 the fast forward, 128
// the 2-D forward, 2 the fast, batched and 2-D backprojections without per-ray
// absorption, 4 adjoint, 8 the other backprojections (generic with occlusion
// or per-ray absorption, fast with per-ray absorption), 16 the generic forward
// with occlusion or per-ray absorption, 32 / 64 the generic forward /
// backprojection without either, 256 the block-table backprojection (511: all
// bodies, for calls of mixed families); a batch launches one instance per family
// present, so no body is compiled around the registers of rarer ones and each
// keeps about its direct kernel's occupancy.
template <int FAM>
__device__ __forceinline__ void item_body(const Item& it, unsigned bx, unsigned by) {
    if (it.kind == KF_GEN || it.kind == KB_GEN || it.kind == KA_GEN) {
        if constexpr (FAM == 32 || FAM == 64) {
            // the lean generic families: no occlusion, no per-ray absorption
            const Args a = it.a;
            if (it.absm == VAM_ABS_MASK) {
                if (it.vz == 4) lean_gen_body<FAM, 4, VAM_ABS_MASK>(it, a, bx, by);
                else lean_gen_body<FAM, 1, VAM_ABS_MASK>(it, a, bx, by);
            } else {
                if (it.vz == 4) lean_gen_body<FAM, 4, VAM_ABS_NONE>(it, a, bx, by);
                else lean_gen_body<FAM, 1, VAM_ABS_NONE>(it, a, bx, by);
            }
        } else if constexpr ((FAM & (4 | 8 | 16)) != 0) {
            if (it.vz == 4) { if (it.occ) gen_body_fam<FAM, 4, true>(it, bx, by); else gen_body_fam<FAM, 4, false>(it, bx, by); }
            else { if (it.occ) gen_body_fam<FAM, 1, true>(it, bx, by); else gen_body_fam<FAM, 1, false>(it, bx, by); }
        }
    } else if (it.kind == KA_TABLE) {
        if constexpr ((FAM & 4) != 0) {
            const Args a = it.a;
            if (it.vz == 8) k_adjoint_table_body<8>(a, it.table, bx, by);
            else k_adjoint_table_body<4>(a, it.table, bx, by);
        }
    } else if (it.ray) {
        if constexpr (FAM != 2) fast_body<FAM, true>(it, bx, by);   // nor a per-ray absorption body
    } else {
        fast_body<FAM, false>(it, bx, by);
    }
}

// ---- direct call: one launch of the described body's own kernel
template <int VZ, bool OCC, int ABS>
void launch_gen3(const Item& it, dim3 grid, cudaStream_t st) {
    const dim3 block(kWarpsPerBlock * kWarp);
    if (it.kind == KF_GEN) k_forward<VZ, OCC, ABS><<<grid, block, 0, st>>>(it.a);
    else if (it.kind == KB_GEN) k_backward_ref<VZ, OCC, ABS><<<grid, block, 0, st>>>(it.a);
    else k_adjoint<VZ, OCC, ABS><<<grid, block, 0, st>>>(it.a);
}

template <int VZ, bool OCC>
void launch_gen2(const Item& it, dim3 grid, cudaStream_t st) {
    if (it.absm == VAM_ABS_MASK) launch_gen3<VZ, OCC, VAM_ABS_MASK>(it, grid, st);
    else if (it.absm == VAM_ABS_RAY) launch_gen3<VZ, OCC, VAM_ABS_RAY>(it, grid, st);
    else launch_gen3<VZ, OCC, VAM_ABS_NONE>(it, grid, st);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver
// library); null when the driver does not provide it
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* fp = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fp);
    });
    return fn;
}

// The tensor map of a [nY][nX] float32 image with rows row_stride floats apart, for
// k_forward_2d_tma's boxes: false (plain staging) unless the rows are a multiple of 16 bytes apart and
// the image starts on a 16-byte boundary.  A host-only call, so a captured launch carries the map in
// its parameters.
bool image_tensor_map(const float* img, int nX, int nY, int row_stride, CUtensorMap& m) {
    if ((((uintptr_t)img) & 15) != 0 || row_stride % 4 != 0 || row_stride < nX) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)nX, (cuuint64_t)nY};
    cuuint64_t strides[1] = {(cuuint64_t)row_stride * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)kTmaW, (cuuint32_t)kTmaH};
    cuuint32_t es[2] = {1, 1};
    return enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(img), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool RAY>
void launch_fast(const Item& it, dim3 grid, cudaStream_t st) {
    const dim3 block(kWarpsPerBlock * kWarp);
    switch (it.kind) {
        case KF_2D:
            if (it.tma) k_forward_2d_tma<RAY><<<grid, block, it.smem, st>>>(it.a, it.tmap, it.status);
            else k_forward_2d<RAY><<<grid, block, it.smem, st>>>(it.a);
            break;
        case KB_2D: k_backward_2d<RAY><<<grid, block, it.smem, st>>>(it.a); break;
        case KF_FAST:
            if (it.vz == 8) k_forward_fast<8, RAY><<<grid, block, 0, st>>>(it.f);
            else if (it.vz == 6) k_forward_fast<6, RAY><<<grid, block, 0, st>>>(it.f);
            else if (it.vz == 5) k_forward_fast<5, RAY><<<grid, block, 0, st>>>(it.f);
            else k_forward_fast<4, RAY><<<grid, block, 0, st>>>(it.f);
            break;
        case KB_BATCHED:
            if (it.vz == 8 && !RAY) k_backward_batched8<<<grid, block, it.smem, st>>>(it.a);
            else if (it.vz == 8) k_backward_batched<8, 2, RAY><<<grid, block, it.smem, st>>>(it.a);
            else if (it.batch == 4) k_backward_batched<4, 4, RAY><<<grid, block, it.smem, st>>>(it.a);
            else k_backward_batched<4, 2, RAY><<<grid, block, it.smem, st>>>(it.a);
            break;
        case KB_FAST:
            if (it.vz == 8) k_backward_fast<8, RAY><<<grid, block, 0, st>>>(it.a);
            else k_backward_fast<4, RAY><<<grid, block, 0, st>>>(it.a);
            break;
        case KA_FAST:
            if (it.vz == 8) k_adjoint_fast<8, RAY><<<grid, block, 0, st>>>(it.a);
            else k_adjoint_fast<4, RAY><<<grid, block, 0, st>>>(it.a);
            break;
        default: break;
    }
}

int launch_item(const Item& it, cudaStream_t st, const char* name) {
    if (it.pre_in && it.pre_wp) {
        k_stage_rows<<<(unsigned)std::min<long long>((it.pre_npix + 255) / 256, 148LL * 32), 256, 0, st>>>(
            it.pre_in, it.pre_mask, it.pre_out, it.pre_npix, it.pre_w, it.pre_wp);
        VAM_CHECK_LAUNCH("k_stage_rows");
    } else if (it.pre_in) {
        const long long n = it.pre_npix * it.pre_nz;
        k_mask_mul<<<(unsigned)std::min<long long>((n + 255) / 256, 148LL * 32), 256, 0, st>>>(
            it.pre_in, it.pre_mask, it.pre_out, (long)it.pre_npix, it.pre_nz);
        VAM_CHECK_LAUNCH("k_mask_mul");
    }
    const dim3 grid(it.gx, it.gy);
    if (it.kind == KF_GEN || it.kind == KB_GEN || it.kind == KA_GEN) {
        if (it.vz == 4) { if (it.occ) launch_gen2<4, true>(it, grid, st); else launch_gen2<4, false>(it, grid, st); }
        else { if (it.occ) launch_gen2<1, true>(it, grid, st); else launch_gen2<1, false>(it, grid, st); }
    } else if (it.kind == KA_TABLE) {
        const dim3 block(kWarpsPerBlock * kWarp);
        if (it.vz == 8) k_adjoint_table<8><<<grid, block, 0, st>>>(it.a, it.table);
        else k_adjoint_table<4><<<grid, block, 0, st>>>(it.a, it.table);
    } else if (it.kind == KB_BTABLE) {
        const dim3 block(kWarpsPerBlock * kWarp);
        const bool full = it.a.nZ % (32 * it.vz) == 0;
        if (it.vz == 8) {
            if (full) k_backward_blk<8, 3, true><<<grid, block, 0, st>>>(it.a, it.btab4, it.bcidx);
            else k_backward_blk<8, 3, false><<<grid, block, 0, st>>>(it.a, it.btab4, it.bcidx);
        } else if (it.vz == 6) {
            k_backward_blk<6, 3, true><<<grid, block, 0, st>>>(it.a, it.btab4, it.bcidx);
        } else if (it.vz == 5) {
            k_backward_blk<5, 3, true><<<grid, block, 0, st>>>(it.a, it.btab4, it.bcidx);
        } else {
            if (full) k_backward_blk<4, 3, true><<<grid, block, 0, st>>>(it.a, it.btab4, it.bcidx);
            else k_backward_blk<4, 3, false><<<grid, block, 0, st>>>(it.a, it.btab4, it.bcidx);
        }
    } else if (it.ray) {
        launch_fast<true>(it, grid, st);
    } else {
        launch_fast<false>(it, grid, st);
    }
    VAM_CHECK_LAUNCH(name);
    return VAM_OK;
}

int run(vam_parallel_plan* plan, Op op, const float* in, float* out, cudaStream_t st, const char* name,
        bool noclip = false) {
    VAM_REQUIRE(plan, VAM_ERR_ARG, std::string(name) + ": null argument");
    DeviceGuard g(plan->device);
    VAM_REQUIRE(g.ok, VAM_ERR_CUDA, std::string(name) + ": cannot select device");
    Item it;
    const int rc = describe(plan, op, in, out, it, name, noclip);
    if (rc != VAM_OK) return rc;
    return launch_item(it, st, name);
}

// ---------------------------------------------------------------------------
// Batched calls: persistent launches over the virtual blocks of many calls,
// one per kernel-body family (and per 48 calls), on streams forked from and
// joined to the caller's.
//
// Every call of a batch keeps its own grid; the calls' blocks are numbered
// consecutively (largest call first) into virtual blocks, and each resident
// CTA takes the next virtual block from a device counter (the work queue),
// finds its call by binary search and runs the call's body for that block.
// Calls of uneven size (2-D slices next to 3-D volumes, different angle
// counts) therefore fill the device together instead of one after another.
// A ticket is one block, as in a direct launch: the resident CTAs work on one
// window of consecutive blocks, whose sinogram or volume footprint stays in
// L2 (tickets of several blocks spread over a call's grid multiplied the DRAM
// reads of a 160^3 x 720 backprojection by 6.6); while at least two tickets
// per CTA remain, each CTA fetches its next ticket while its current block
// runs, which hides the counter's latency.
// ---------------------------------------------------------------------------
// The calls of one launch travel by value in the kernel's parameter space
// (__grid_constant__, up to 32 KB): a CTA reads its call's description through
// the constant cache, which keeps those reads off the L1 data path that the
// gather kernels saturate, and a graph capture records the list with the launch.
constexpr int kBatchMaxItems = 48;
struct BatchParams {
    int n;
    unsigned total;  // tickets (virtual blocks) of the launch, < 2^31
    unsigned* counter;
    Item items[kBatchMaxItems];
};

// the last call of a launch whose first ticket is <= t
__device__ __forceinline__ int batch_find(const BatchParams& P, unsigned t) {
    int lo = 0, hi = P.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.items[mid].tstart <= (long long)t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
static_assert(sizeof(BatchParams) < 32000, "batch parameters must fit the 32 KB kernel parameter space");

// Resident CTAs per SM each instance asks for, i.e. its register cap: the
// lean generic backprojection fits 40 registers (six CTAs, as its direct
// kernel: a 160^3 x 720 call ran 1.36x longer at four), the fast and 2-D
// backprojections and the 2-D forward 48 (five), the fast forward and the
// lean generic forward 64 (four); the heavy instances keep 80 (three), the
// block-table backprojection (four bodies: 4 or 8 slices, full or partial z
// chunks) 128 (two).
template <int FAM>
__global__ void __launch_bounds__(256, FAM == 64 ? 6 : (FAM == 2 || FAM == 128 ? 5 : (FAM == 1 || FAM == 32 ? 4 : (FAM == 256 ? 2 : 3))))
    k_batch(const __grid_constant__ BatchParams P) {
    __shared__ unsigned s_t[2];
    __shared__ int s_idx[2];
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(P.counter, 1u);
        s_t[0] = t;
        s_idx[0] = t < P.total ? batch_find(P, t) : 0;
    }
    __syncthreads();
    // s_t / s_idx alternate between two slots: slot s is read at the top of a round, slot s ^ 1 is
    // written at its end, and the barrier closing the round orders both
    for (int s = 0;; s ^= 1) {
        const unsigned t = s_t[s];
        if (t >= P.total) return;  // uniform: every thread read the same s_t
        // the next ticket is fetched while the block runs, except near the end of the queue, where
        // a CTA holding two tickets would run both blocks back to back while others find none
        const bool early = t + 2u * gridDim.x < P.total;
        unsigned next = 0;
        if (threadIdx.x == 0 && early) next = atomicAdd(P.counter, 1u);
        const Item& it = P.items[s_idx[s]];
        const unsigned b = t - (unsigned)it.tstart;  // a call's grid has < 2^31 blocks
        item_body<FAM>(it, b % it.gx, b / it.gx);
        if (threadIdx.x == 0) {
            if (!early) next = atomicAdd(P.counter, 1u);
            s_t[s ^ 1] = next;
            s_idx[s ^ 1] = next < P.total ? batch_find(P, next) : 0;
        }
        __syncthreads();  // also: the next block restages the body's shared memory
    }
}

using BatchKernel = void (*)(BatchParams);
BatchKernel batch_kernel(int fam) {
    switch (fam) {
        case 1: return k_batch<1>;
        case 2: return k_batch<2>;
        case 4: return k_batch<4>;
        case 8: return k_batch<8>;
        case 16: return k_batch<16>;
        case 32: return k_batch<32>;
        case 64: return k_batch<64>;
        case 128: return k_batch<128>;
        case 256: return k_batch<256>;
        default: return k_batch<511>;
    }
}

// mask pre-pass of every fast forward of a batch (blockIdx.y = call)
__global__ void k_batch_premask(const __grid_constant__ BatchParams P) {
    const Item& it = P.items[blockIdx.y];
    if (!it.pre_in) return;
    if (it.pre_wp) {
        stage_rows(it.pre_in, it.pre_mask, it.pre_out, it.pre_npix, it.pre_w, it.pre_wp,
                   (long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
        return;
    }
    const long long n = it.pre_npix * it.pre_nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        it.pre_out[i] = it.pre_mask[i / it.pre_nz] * it.pre_in[i];
}

// numpy linspace(-1, 1, n)[i]
double lin_m1_1(int i, int n) {
    if (n == 1) return -1.0;
    if (i == n - 1) return 1.0;
    volatile double step = 2.0 / (double)(n - 1);
    volatile double prod = (double)i * step;
    return prod + -1.0;
}

}  // namespace
}  // namespace vam

using namespace vam;

extern "C" int vam_parallel_plan_create(const vam_parallel_geom* geom, vam_parallel_plan** out) {
    clear_error();
    VAM_REQUIRE(geom && out, VAM_ERR_ARG, "vam_parallel_plan_create: null argument");
    *out = nullptr;
    VAM_REQUIRE(geom->n_y > 0 && geom->n_x > 0 && geom->n_z > 0 && geom->n_angles > 0, VAM_ERR_SHAPE,
                "vam_parallel_plan_create: sizes must be positive");
    VAM_REQUIRE(geom->n_x == geom->n_y, VAM_ERR_SHAPE,
                "vam_parallel_plan_create: the rotate-and-sum projector needs a square slice (n_x == n_y)");
    VAM_REQUIRE(geom->angles_deg, VAM_ERR_ARG, "vam_parallel_plan_create: angles_deg is null");
    VAM_REQUIRE((long)geom->n_y * geom->n_x * geom->n_z < (1L << 40), VAM_ERR_SHAPE,
                "vam_parallel_plan_create: volume too large");
    for (int i = 0; i < geom->n_angles; ++i)
        VAM_REQUIRE(std::isfinite(geom->angles_deg[i]), VAM_ERR_ARG, "vam_parallel_plan_create: non-finite angle");
    DeviceGuard g(geom->device);
    VAM_REQUIRE(g.ok, VAM_ERR_CUDA, "vam_parallel_plan_create: cannot select device");
    auto* p = new vam_parallel_plan();
    std::memset(p, 0, sizeof(*p));
    p->nY = geom->n_y; p->nX = geom->n_x; p->nZ = geom->n_z; p->nA = geom->n_angles;
    p->C = geom->n_y / 2;
    p->device = geom->device;
    p->adj_table_abs = -1;
    p->tune_bwd_batch = 2;
    p->tune_adj_table = 1;
    p->tune_bwd_table = 1;
    p->tune_fwd_tma = 1;
    // per-angle tables exactly as numpy evaluates them (Projector3DParallel.py:135-143)
    std::vector<double4> trig(p->nA);
    for (int i = 0; i < p->nA; ++i) {
        volatile double r = geom->angles_deg[i] * (M_PI / 180.0);
        double c = cos(r), s = sin(r);
        volatile double cs1 = c + s;
        volatile double cs2 = c - s;
        volatile double m02 = -(double)p->C * (cs1 - 1.0);
        volatile double m12 = -(double)p->C * (cs2 - 1.0);
        trig[i] = make_double4(c, s, m02, m12);
    }
    std::vector<uint8_t> circ((size_t)p->nY * p->nX);
    for (int i = 0; i < p->nY; ++i) {
        double a = lin_m1_1(i, p->nY);
        for (int j = 0; j < p->nX; ++j) {
            double b = lin_m1_1(j, p->nX);
            volatile double aa = a * a, bb = b * b;
            volatile double r2 = aa + bb;
            circ[(size_t)i * p->nX + j] = !(r2 > 1.0);
        }
    }
    // pair every angle with the one 180 degrees away (within 1e-9 degrees, mod 360)
    std::vector<int2> paired, single;
    {
        std::vector<int> used(p->nA, 0);
        for (int i = 0; i < p->nA; ++i) {
            single.push_back(make_int2(i, -1));
            if (used[i]) continue;
            used[i] = 1;
            int partner = -1;
            for (int k = i + 1; k < p->nA && partner < 0; ++k) {
                if (used[k]) continue;
                double d = std::fmod(geom->angles_deg[k] - geom->angles_deg[i] - 180.0, 360.0);
                if (d < 0) d += 360.0;
                if (d < 1e-9 || 360.0 - d < 1e-9) partner = k;
            }
            if (partner >= 0) used[partner] = 1;
            paired.push_back(make_int2(i, partner));
        }
    }
    p->n_tasks_paired = (int)paired.size();
    cudaError_t e = cudaMalloc(&p->d_trig, sizeof(double4) * p->nA);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_tasks_paired, sizeof(int2) * paired.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->d_tasks_single, sizeof(int2) * single.size());
    if (e == cudaSuccess) e = cudaMemcpy(p->d_tasks_paired, paired.data(), sizeof(int2) * paired.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_tasks_single, single.data(), sizeof(int2) * single.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_circle, circ.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_status, 0, sizeof(int));
    if (e == cudaSuccess && p->nZ == 1)
        e = cudaMalloc(&p->d_img_pad, sizeof(float) * (size_t)p->nY * (size_t)((p->nX + 3) & ~3));
    if (e == cudaSuccess) e = cudaMemcpy(p->d_trig, trig.data(), sizeof(double4) * p->nA, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_circle, circ.data(), circ.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        vam_parallel_plan_destroy(p);
        return set_error(VAM_ERR_NOMEM, std::string("vam_parallel_plan_create: ") + cudaGetErrorString(e));
    }
    *out = p;
    return VAM_OK;
}

extern "C" int vam_parallel_plan_destroy(vam_parallel_plan* p) {
    if (!p) return VAM_OK;
    DeviceGuard g(p->device);
    cudaFree(p->d_trig);
    cudaFree(p->d_circle);
    cudaFree(p->d_mask);
    cudaFree(p->d_occ);
    cudaFree(p->d_occ_flag);
    cudaFree(p->d_occ64);
    cudaFree(p->d_ones);
    cudaFree(p->d_tasks_paired);
    cudaFree(p->d_tasks_single);
    cudaFree(p->d_vol_scratch);
    cudaFree(p->d_adj_table);
    cudaFree(p->d_bwd_cidx);
    cudaFree(p->d_status);
    cudaFree(p->d_img_pad);
    cudaFree(p->d_bwd_btab);
    cudaFree(p->d_bwd_bcidx);
    delete p;
    return VAM_OK;
}

extern "C" int vam_parallel_set_absorption(vam_parallel_plan* p, int mode, const float* mask_dev,
                                           float alpha_per_px, float radius_px, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_parallel_set_absorption: null plan");
    VAM_REQUIRE(mode == VAM_ABS_NONE || mode == VAM_ABS_MASK || mode == VAM_ABS_RAY, VAM_ERR_ARG,
                "vam_parallel_set_absorption: unknown mode");
    DeviceGuard g(p->device);
    if (mode == VAM_ABS_MASK) {
        VAM_REQUIRE(mask_dev, VAM_ERR_ARG, "vam_parallel_set_absorption: MASK needs mask_dev");
        if (!p->d_mask) VAM_TRY_CUDA(cudaMalloc(&p->d_mask, sizeof(float) * (size_t)p->nY * p->nX));
        if (!p->d_vol_scratch)
            VAM_TRY_CUDA(cudaMalloc(&p->d_vol_scratch, sizeof(float) * (size_t)p->nY * p->nX * p->nZ));
        VAM_TRY_CUDA(cudaMemcpyAsync(p->d_mask, mask_dev, sizeof(float) * (size_t)p->nY * p->nX,
                                     cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    }
    if (mode == VAM_ABS_RAY) {
        VAM_REQUIRE(std::isfinite(alpha_per_px) && alpha_per_px >= 0.f && std::isfinite(radius_px) && radius_px > 0.f,
                    VAM_ERR_ARG, "vam_parallel_set_absorption: RAY needs alpha >= 0 and radius > 0");
    }
    p->abs_mode = mode;
    p->abs_alpha = alpha_per_px;
    p->abs_R = radius_px;
    return VAM_OK;
}

extern "C" int vam_parallel_set_occlusion(vam_parallel_plan* p, const float* insert_dev, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && insert_dev, VAM_ERR_ARG, "vam_parallel_set_occlusion: null argument");
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->nY * p->nA * p->nZ;
    if (!p->d_occ) VAM_TRY_CUDA(cudaMalloc(&p->d_occ, sizeof(float) * n));
    if (!p->d_occ_flag) VAM_TRY_CUDA(cudaMalloc(&p->d_occ_flag, (size_t)p->nA * p->nZ));
    cudaStream_t st = (cudaStream_t)stream;
    k_occ_sinogram<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(insert_dev, p->d_occ, p->d_trig, p->nY, p->nX,
                                                                   p->nZ, p->nA, p->C);
    VAM_CHECK_LAUNCH("k_occ_sinogram");
    const size_t nf = (size_t)p->nA * p->nZ;
    k_occ_flag<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(p->d_occ, p->d_occ_flag, p->nX, p->nA, p->nZ);
    VAM_CHECK_LAUNCH("k_occ_flag");
    p->has_occ = 1;
    p->occ_mode = 0;
    return VAM_OK;
}

extern "C" int vam_parallel_set_occlusion_2d(vam_parallel_plan* p, const uint8_t* occlusion_dev, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && occlusion_dev, VAM_ERR_ARG, "vam_parallel_set_occlusion_2d: null argument");
    VAM_REQUIRE(p->nZ == 1, VAM_ERR_SHAPE, "vam_parallel_set_occlusion_2d: the digitised occlusion is for 2-D plans (n_z == 1)");
    DeviceGuard g(p->device);
    const int n = p->nY;
    const size_t ns = (size_t)n * p->nA;
    if (!p->d_occ) VAM_TRY_CUDA(cudaMalloc(&p->d_occ, sizeof(float) * ns));
    if (!p->d_occ_flag) VAM_TRY_CUDA(cudaMalloc(&p->d_occ_flag, (size_t)p->nA));
    if (!p->d_occ64) VAM_TRY_CUDA(cudaMalloc(&p->d_occ64, sizeof(double) * ns));
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* slots = nullptr;
    int* d_err = nullptr;
    const size_t nslots = (size_t)(n + 1) * p->nA;
    VAM_TRY_CUDA(cudaMalloc(&slots, sizeof(unsigned long long) * nslots + 256));
    d_err = reinterpret_cast<int*>(reinterpret_cast<char*>(slots) + sizeof(unsigned long long) * nslots);
    int h_err = 0;
    cudaError_t e = cudaMemsetAsync(slots, 0xff, sizeof(unsigned long long) * nslots, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        const long long np = (long long)p->nA * n * n;
        k_occ2d_bin<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(occlusion_dev, p->d_trig, slots, n, p->nA, p->C);
        k_occ2d_assign<<<(unsigned)((p->nA + 127) / 128), 128, 0, st>>>(slots, p->d_occ64, p->d_occ, p->d_occ_flag,
                                                                        d_err, n, p->nA);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(slots);
    if (e != cudaSuccess) return set_error(VAM_ERR_CUDA, std::string("vam_parallel_set_occlusion_2d: ") + cudaGetErrorString(e));
    if (h_err & 2)
        return set_error(VAM_ERR_SHAPE, "vam_parallel_set_occlusion_2d: zero-size array to reduction operation minimum "
                                        "which has no identity (the occlusion is empty)");
    if (h_err & 1)
        return set_error(VAM_ERR_SHAPE, "vam_parallel_set_occlusion_2d: shape mismatch: occluded pixels below the "
                                        "first detector bin and in the last bin at the same angle");
    p->has_occ = 1;
    p->occ_mode = 1;
    return VAM_OK;
}

extern "C" int vam_parallel_clear_occlusion(vam_parallel_plan* p) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_parallel_clear_occlusion: null plan");
    p->has_occ = 0;
    return VAM_OK;
}

extern "C" int vam_parallel_get_occlusion_sinogram_2d(vam_parallel_plan* p, double* out_dev, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && out_dev, VAM_ERR_ARG, "vam_parallel_get_occlusion_sinogram_2d: null argument");
    VAM_REQUIRE(p->has_occ && p->occ_mode == 1, VAM_ERR_ARG,
                "vam_parallel_get_occlusion_sinogram_2d: no digitised 2-D occlusion set");
    DeviceGuard g(p->device);
    VAM_TRY_CUDA(cudaMemcpyAsync(out_dev, p->d_occ64, sizeof(double) * (size_t)p->nY * p->nA, cudaMemcpyDeviceToDevice,
                                 (cudaStream_t)stream));
    return VAM_OK;
}

extern "C" int vam_parallel_get_occlusion_sinogram(vam_parallel_plan* p, float* out_dev, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && out_dev, VAM_ERR_ARG, "vam_parallel_get_occlusion_sinogram: null argument");
    VAM_REQUIRE(p->has_occ, VAM_ERR_ARG, "vam_parallel_get_occlusion_sinogram: no occlusion set");
    DeviceGuard g(p->device);
    VAM_TRY_CUDA(cudaMemcpyAsync(out_dev, p->d_occ, sizeof(float) * (size_t)p->nY * p->nA * p->nZ,
                                 cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return VAM_OK;
}

extern "C" int vam_parallel_set_tuning(vam_parallel_plan* p, const vam_parallel_tuning* t) {
    clear_error();
    VAM_REQUIRE(p && t, VAM_ERR_ARG, "vam_parallel_set_tuning: null argument");
    auto vz_ok = [](int v) { return v == 0 || v == 1 || v == 4 || v == 8; };
    VAM_REQUIRE((vz_ok(t->forward_vz) || t->forward_vz == 6 || t->forward_vz == 5) && vz_ok(t->backward_vz) &&
                    vz_ok(t->adjoint_vz),
                VAM_ERR_ARG, "vam_parallel_set_tuning: vector widths must be 0 (auto), 1 (generic kernel), 4 or 8 "
                "(the forward also 6 or 5)");
    VAM_REQUIRE(t->backward_batch == 0 || t->backward_batch == 1 || t->backward_batch == 2 || t->backward_batch == 4,
                VAM_ERR_ARG, "vam_parallel_set_tuning: backward_batch must be 0 (auto), 1, 2 or 4");
    p->tune_fwd_vz = t->forward_vz;
    p->tune_bwd_vz = t->backward_vz;
    p->tune_adj_vz = t->adjoint_vz;
    p->tune_bwd_batch = t->backward_batch == 0 ? 2 : t->backward_batch;
    p->tune_adj_table = t->adjoint_table;
    p->tune_bwd_table = t->backward_table;
    p->tune_fwd_tma = t->forward_tma;
    return VAM_OK;
}

extern "C" int vam_parallel_get_tuning(vam_parallel_plan* p, vam_parallel_tuning* t) {
    clear_error();
    VAM_REQUIRE(p && t, VAM_ERR_ARG, "vam_parallel_get_tuning: null argument");
    t->forward_vz = p->tune_fwd_vz;
    t->backward_vz = p->tune_bwd_vz;
    t->adjoint_vz = p->tune_adj_vz;
    t->backward_batch = p->tune_bwd_batch;
    t->adjoint_table = p->tune_adj_table;
    t->backward_table = p->tune_bwd_table;
    t->forward_tma = p->tune_fwd_tma;
    return VAM_OK;
}

extern "C" int vam_parallel_prepare_adjoint(vam_parallel_plan* p, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_parallel_prepare_adjoint: null plan");
    DeviceGuard g(p->device);
    const size_t n = (size_t)p->nY * p->nX * p->nA;
    if (!p->d_adj_table) VAM_TRY_CUDA(cudaMalloc(&p->d_adj_table, sizeof(float4) * n));
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (p->abs_mode == VAM_ABS_RAY)
        k_adj_table<true><<<nb, 256, 0, st>>>(p->d_trig, p->d_adj_table, p->nY, p->nX, p->nA, p->C, p->abs_alpha, p->abs_R);
    else
        k_adj_table<false><<<nb, 256, 0, st>>>(p->d_trig, p->d_adj_table, p->nY, p->nX, p->nA, p->C, 0.f, 0.f);
    VAM_CHECK_LAUNCH("k_adj_table");
    p->adj_table_abs = p->abs_mode;
    return VAM_OK;
}

extern "C" int vam_parallel_status(vam_parallel_plan* p, int32_t* status) {
    clear_error();
    VAM_REQUIRE(p && status, VAM_ERR_ARG, "vam_parallel_status: null argument");
    DeviceGuard g(p->device);
    int v = 0;
    VAM_TRY_CUDA(cudaMemcpy(&v, p->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    VAM_TRY_CUDA(cudaMemset(p->d_status, 0, sizeof(int)));
    *status = v;
    return VAM_OK;
}

extern "C" int vam_parallel_prepare_backward(vam_parallel_plan* p, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_parallel_prepare_backward: null plan");
    VAM_REQUIRE((long long)p->nY * p->nA * p->nZ < (1LL << 31), VAM_ERR_NOTSUP,
                "vam_parallel_prepare_backward: the table holds 32-bit sinogram offsets (sinogram below 2^31 elements)");
    VAM_REQUIRE(p->nZ % 4 == 0, VAM_ERR_NOTSUP,
                "vam_parallel_prepare_backward: the table kernel runs four-slice vectors (nZ % 4 == 0)");
    DeviceGuard g(p->device);
    const int n = p->nY * p->nX;
    // the clip circle exactly as the plan's table (linspace(-1, 1) semantics)
    std::vector<int> cidx(n, -1);
    for (int i = 0, c = 0; i < p->nY; ++i) {
        const double a = lin_m1_1(i, p->nY);
        for (int j = 0; j < p->nX; ++j) {
            const double b = lin_m1_1(j, p->nX);
            volatile double aa = a * a, bb = b * b;
            volatile double r2 = aa + bb;
            if (!(r2 > 1.0)) cidx[(size_t)i * p->nX + j] = c++;
        }
    }
    // 2 x 2 blocks with at least one pixel inside the circle
    const int nbx = (p->nX + 1) / 2, nby = (p->nY + 1) / 2;
    std::vector<int> bcidx((size_t)nbx * nby, -1), blist;
    for (int bi = 0; bi < nby; ++bi)
        for (int bj = 0; bj < nbx; ++bj) {
            bool any = false;
            for (int q = 0; q < 4; ++q) {
                const int i = 2 * bi + (q >> 1), j = 2 * bj + (q & 1);
                any |= i < p->nY && j < p->nX && cidx[(size_t)i * p->nX + j] >= 0;
            }
            if (any) { bcidx[(size_t)bi * nbx + bj] = (int)blist.size(); blist.push_back(bi * nbx + bj); }
        }
    const int nbc = (int)blist.size();
    cudaStream_t st = (cudaStream_t)stream;
    if (!p->d_bwd_cidx) VAM_TRY_CUDA(cudaMalloc(&p->d_bwd_cidx, sizeof(int) * n));
    if (!p->d_bwd_bcidx) VAM_TRY_CUDA(cudaMalloc(&p->d_bwd_bcidx, sizeof(int) * bcidx.size()));
    if (!p->d_bwd_btab) VAM_TRY_CUDA(cudaMalloc(&p->d_bwd_btab, sizeof(int4) * 2 * (size_t)std::max(nbc, 1) * p->nA));
    int* d_blist = nullptr;
    VAM_TRY_CUDA(cudaMalloc(&d_blist, sizeof(int) * std::max(nbc, 1)));
    cudaError_t e = cudaMemcpyAsync(p->d_bwd_cidx, cidx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_bwd_bcidx, bcidx.data(), sizeof(int) * bcidx.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nbc) e = cudaMemcpyAsync(d_blist, blist.data(), sizeof(int) * nbc, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nbc) {
        const long tot = (long)nbc * p->nA;
        k_bwd_btable<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(p->d_trig, d_blist, p->d_bwd_cidx, p->d_bwd_btab,
                                                                    nbc, p->nA, p->nY, p->nX, p->nZ, p->C);
        e = cudaGetLastError();
    }
    // the host vectors and the block list are released after the copies and the build complete
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_blist);
    if (e != cudaSuccess)
        return set_error(VAM_ERR_CUDA, std::string("vam_parallel_prepare_backward: ") + cudaGetErrorString(e));
    return VAM_OK;
}

extern "C" int vam_parallel_forward(vam_parallel_plan* p, const float* vol, float* sino, vam_stream_t stream) {
    clear_error();
    return run(p, Op::Forward, vol, sino, (cudaStream_t)stream, "vam_parallel_forward");
}

extern "C" int vam_parallel_backward_ref(vam_parallel_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    return run(p, Op::BackwardRef, sino, vol, (cudaStream_t)stream, "vam_parallel_backward_ref");
}

extern "C" int vam_parallel_backward_ref_noclip(vam_parallel_plan* p, const float* sino, float* vol,
                                                vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_parallel_backward_ref_noclip: null plan");
    if (!p->d_ones) {
        DeviceGuard g(p->device);
        const size_t np = (size_t)p->nY * p->nX;
        VAM_TRY_CUDA(cudaMalloc(&p->d_ones, np));
        VAM_TRY_CUDA(cudaMemsetAsync(p->d_ones, 1, np, (cudaStream_t)stream));
    }
    return run(p, Op::BackwardRef, sino, vol, (cudaStream_t)stream, "vam_parallel_backward_ref_noclip", true);
}

extern "C" int vam_parallel_adjoint(vam_parallel_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    return run(p, Op::Adjoint, sino, vol, (cudaStream_t)stream, "vam_parallel_adjoint");
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
// launches (ticket counters) one list may need: 48 calls per launch, and one
// more launch at each of the <= 7 changes of body family
constexpr int kBatchMaxLaunches = 80;

// dynamic shared-memory sizes the batch kernels' residency is tabulated for
constexpr unsigned kSmemBuckets[4] = {0u, 16u * 1024, 40u * 1024, 48u * 1024};

// streams of a batch besides the caller's: the launches of one list run on up to
// kBatchSide + 1 streams, forked from and joined to the caller's stream
constexpr int kBatchSide = 3;

inline int smem_bucket(unsigned smem) {
    int k = 0;
    while (k < 3 && kSmemBuckets[k] < smem) ++k;
    return k;
}

struct vam_batch {
    int device;
    unsigned* d_counter;
    int sms;
    int per_sm[512][4];        // resident CTAs per SM of k_batch<fam> (fam 1 .. 256, 511) per
                               // dynamic shared-memory bucket (kSmemBuckets)
    std::vector<Item> host;    // the described calls of the last list, in queue order
    std::vector<int> group;    // first call of each launch (kBatchMaxItems calls per launch)
    std::vector<long long> tickets;  // tickets of each launch
    std::vector<int> fam;      // body family of each launch
    std::vector<unsigned> gsmem;  // dynamic shared memory of each launch (its calls' largest)
    long long blocks;          // blocks of all calls' grids
    unsigned smem;
    int any_pre;
    int ctas;                  // persistent CTAs of the last launch
    cudaStream_t side[kBatchSide];  // non-blocking streams for the launches after the first
    cudaEvent_t fork;               // recorded on the caller's stream before the launches
    cudaEvent_t join[kBatchSide];   // recorded on each side stream after its launches
};

static void batch_release(vam_batch* b) {
    for (int s = 0; s < kBatchSide; ++s) {
        if (b->side[s]) cudaStreamDestroy(b->side[s]);
        if (b->join[s]) cudaEventDestroy(b->join[s]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
}

extern "C" int vam_batch_create(int32_t device, vam_batch** out) {
    clear_error();
    VAM_REQUIRE(out, VAM_ERR_ARG, "vam_batch_create: null argument");
    *out = nullptr;
    DeviceGuard g(device);
    VAM_REQUIRE(g.ok, VAM_ERR_CUDA, "vam_batch_create: cannot select device");
    int sms = 0;
    VAM_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    int per_sm[512][4] = {};
    // residency for each dynamic shared-memory bucket up to the largest a call may ask for (48 KB,
    // the batched backprojection's trig table), queried once here, so a list never needs a
    // runtime query (which would not be allowed during graph capture); the opt-in limit is
    // raised first, as 48 KB plus the kernel's static shared memory exceeds the default
    for (int fam : {1, 2, 4, 8, 16, 32, 64, 128, 256, 511}) {
        VAM_TRY_CUDA(cudaFuncSetAttribute(batch_kernel(fam), cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        for (int k = 0; k < 4; ++k) {
            VAM_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[fam][k], batch_kernel(fam),
                                                                       kWarpsPerBlock * kWarp, kSmemBuckets[k]));
            VAM_REQUIRE(per_sm[fam][k] > 0, VAM_ERR_NOTSUP, "vam_batch_create: the batch kernel cannot be resident");
        }
    }
    auto* b = new vam_batch();
    b->device = device;
    b->sms = sms;
    std::memcpy(b->per_sm, per_sm, sizeof(per_sm));
    b->blocks = 0;
    b->smem = 0;
    b->any_pre = 0;
    b->ctas = 0;
    b->d_counter = nullptr;
    b->fork = nullptr;
    for (int s = 0; s < kBatchSide; ++s) b->side[s] = nullptr, b->join[s] = nullptr;
    cudaError_t e = cudaMalloc(&b->d_counter, sizeof(unsigned) * kBatchMaxLaunches);
    if (e != cudaSuccess) {
        batch_release(b);
        return set_error(VAM_ERR_NOMEM, std::string("vam_batch_create: ") + cudaGetErrorString(e));
    }
    e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int s = 0; s < kBatchSide && e == cudaSuccess; ++s) {
        e = cudaStreamCreateWithFlags(&b->side[s], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[s], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        batch_release(b);
        return set_error(VAM_ERR_CUDA, std::string("vam_batch_create: ") + cudaGetErrorString(e));
    }
    *out = b;
    return VAM_OK;
}

extern "C" int vam_batch_destroy(vam_batch* b) {
    if (!b) return VAM_OK;
    DeviceGuard g(b->device);
    batch_release(b);
    return VAM_OK;
}

namespace vam {
namespace {
// Relative time per sample of each body (fast forward = 1), measured on
// B200: the generic kernels gather fewer samples per second than the fast
// ones, and a single slice (nZ = 1) far fewer, so a batch orders its calls
// (longest first) by estimated time, not by samples.
double time_weight(const Item& it) {
    const bool slice = it.a.nZ == 1 || it.f.nZ == 1;
    switch (it.kind) {
        case KF_FAST: return 1.0;
        case KF_GEN: return slice ? 27.0 : 4.0;
        case KB_BATCHED: case KB_FAST: return 1.2;
        case KB_BTABLE: return 0.7;
        case KB_GEN: return slice ? 10.0 : 2.0;
        case KA_TABLE: return 1.5;
        case KA_FAST: return 3.5;
        case KF_2D: return 4.0;
        case KB_2D: return 2.0;
        default: return slice ? 27.0 : 4.0;
    }
}

// describe every call, order the queue, number the tickets; no CUDA call
int batch_prepare(vam_batch* b, const vam_work* work, int32_t n) {
    VAM_REQUIRE(n <= kBatchMaxItems * 64, VAM_ERR_SHAPE, "vam_batch: at most 3072 calls per list");
    std::vector<Item> items((size_t)n);
    for (int i = 0; i < n; ++i) {
        const vam_work& w = work[i];
        VAM_REQUIRE(w.plan, VAM_ERR_ARG, "vam_batch: work item without a plan");
        VAM_REQUIRE(w.plan->device == b->device, VAM_ERR_ARG, "vam_batch: plan on another device than the batch");
        VAM_REQUIRE(w.op >= VAM_OP_FORWARD && w.op <= VAM_OP_ADJOINT, VAM_ERR_ARG, "vam_batch: unknown op");
        const Op op = w.op == VAM_OP_FORWARD ? Op::Forward : (w.op == VAM_OP_BACKWARD_REF ? Op::BackwardRef : Op::Adjoint);
        const int rc = describe(w.plan, op, w.in, w.out, items[i], "vam_batch", false, true);
        if (rc != VAM_OK) return rc;
        const Item& d = items[i];
        // generic bodies with occlusion or per-ray absorption, and per-ray fast backprojections, go
        // to the heavy families (8 backward, 16 forward)
        const bool gen_heavy = d.occ || d.absm == VAM_ABS_RAY;
        if (d.kind == KB_GEN) items[i].family = gen_heavy ? 8 : 64;
        else if (d.family == 2 && d.ray) items[i].family = 8;
        if (d.kind == KF_GEN) items[i].family = gen_heavy ? 16 : 32;
        // the 2-D forward instance carries the TMA-staged body only; plain staging (no tensor map
        // encoder) runs in the all-bodies instance
        if (d.kind == KF_2D && !d.tma) items[i].family = 511;
        if (d.kind == KB_BTABLE) items[i].family = 256;

        VAM_REQUIRE((long long)items[i].gx * items[i].gy < (1LL << 31), VAM_ERR_SHAPE, "vam_batch: call grid too large");
        items[i].cost = (long long)std::llround((double)items[i].cost * time_weight(items[i]));
    }
    // a staged forward writes its plan's scratch: two such calls of one plan would share it
    std::vector<const float*> staged;
    for (const Item& it : items)
        if (it.pre_out) staged.push_back(it.pre_out);
    std::sort(staged.begin(), staged.end());
    VAM_REQUIRE(std::adjacent_find(staged.begin(), staged.end()) == staged.end(), VAM_ERR_ARG,
                "vam_batch: two forwards of one plan stage their input into the same scratch");
    // one launch per body family (each with the narrowest instance and its occupancy), and
    // within a family the largest call first, so the small ones fill the tail of the queue
    std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) {
        return x.family != y.family ? x.family < y.family : x.cost > y.cost;
    });
    b->group.clear();
    b->tickets.clear();
    b->fam.clear();
    b->gsmem.clear();
    b->smem = 0;
    b->any_pre = 0;
    b->blocks = 0;
    for (int g0 = 0, g1 = 0; g0 < n; g0 = g1) {
        g1 = g0 + 1;
        while (g1 < n && g1 - g0 < kBatchMaxItems && items[g1].family == items[g0].family) ++g1;
        int fam = 0;
        unsigned gsmem = 0;
        for (int i = g0; i < g1; ++i) {
            fam |= items[i].family;
            gsmem = std::max(gsmem, items[i].smem);
            b->any_pre |= items[i].pre_in != nullptr;
        }
        b->smem = std::max(b->smem, gsmem);
        if (fam & (fam - 1)) fam = 511;  // one family per launch; the all-bodies instance otherwise
        // tickets: one per block of each call's grid, the calls one after another
        long long total = 0;
        for (int i = g0; i < g1; ++i) {
            Item& it = items[i];
            const long long nb = (long long)it.gx * it.gy;
            it.tstart = total;
            total += nb;
            b->blocks += nb;
        }
        VAM_REQUIRE(total < (1LL << 31), VAM_ERR_SHAPE, "vam_batch: more than 2^31 blocks in one launch");
        b->group.push_back(g0);
        b->tickets.push_back(total);
        b->fam.push_back(fam);
        b->gsmem.push_back(gsmem);
    }
    VAM_REQUIRE((int)b->group.size() <= kBatchMaxLaunches, VAM_ERR_SHAPE, "vam_batch: too many launches for one list");
    b->host.swap(items);
    return VAM_OK;
}
}  // namespace
}  // namespace vam

extern "C" int vam_batch_prepare(vam_batch* b, const vam_work* work, int32_t n, vam_stream_t stream) {
    clear_error();
    (void)stream;
    VAM_REQUIRE(b && work && n > 0, VAM_ERR_ARG, "vam_batch_prepare: null argument or empty work list");
    return batch_prepare(b, work, n);
}

namespace vam {
namespace {
int batch_launch(vam_batch* b, int n, cudaStream_t st0, int lanes) {
    const int groups = (int)b->group.size();
    static BatchParams P;  // 15 KB: too large for the stack of every caller thread
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    for (int k = 0; k < groups; ++k) {
        cudaStream_t st = k % lanes == 0 ? st0 : b->side[k % lanes - 1];
        const int g0 = b->group[k];
        const int g1 = k + 1 < groups ? b->group[k + 1] : n;
        std::memset(&P, 0, sizeof(P));
        P.n = g1 - g0;
        P.total = (unsigned)b->tickets[k];
        P.counter = b->d_counter + k;
        std::memcpy(P.items, b->host.data() + g0, sizeof(Item) * (size_t)(g1 - g0));
        bool pre = false;
        long long pre_max = 0;
        for (int i = 0; i < P.n; ++i) {
            pre |= P.items[i].pre_in != nullptr;
            if (P.items[i].pre_in) pre_max = std::max(pre_max, P.items[i].pre_npix * P.items[i].pre_nz);
        }
        if (pre) {
            // about 8 elements per thread for the largest call (blockIdx.y = call)
            const long long gx = std::min<long long>(std::max<long long>((pre_max + 2047) / 2048, 1), 4096);
            k_batch_premask<<<dim3((unsigned)gx, (unsigned)P.n), 256, 0, st>>>(P);
            VAM_CHECK_LAUNCH("k_batch_premask");
        }
        const int fam = b->fam[k];
        const unsigned gsmem = b->gsmem[k];
        const long long ctas = std::min<long long>((long long)b->sms * b->per_sm[fam][smem_bucket(gsmem)], P.total);
        b->ctas = (int)ctas;
        batch_kernel(fam)<<<(unsigned)ctas, kWarpsPerBlock * kWarp, gsmem, st>>>(P);
        VAM_CHECK_LAUNCH("k_batch");
    }
    return VAM_OK;
}
}  // namespace
}  // namespace vam

extern "C" int vam_batch_submit(vam_batch* b, const vam_work* work, int32_t n, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(b && work && n > 0, VAM_ERR_ARG, "vam_batch_submit: null argument or empty work list");
    DeviceGuard g(b->device);
    VAM_REQUIRE(g.ok, VAM_ERR_CUDA, "vam_batch_submit: cannot select device");
    cudaStream_t st = (cudaStream_t)stream;
    const int rc = batch_prepare(b, work, n);
    if (rc != VAM_OK) return rc;
    const int groups = (int)b->group.size();
    VAM_TRY_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned) * groups, st));
    // Launch k runs on stream k mod lanes (the caller's stream, then the batch's own ones), forked
    // from and joined to the caller's stream: the calls of a list are independent, so the next
    // launch's CTAs take the SMs that the previous one's tail frees instead of waiting for its end.
    const int lanes = std::min(groups, kBatchSide + 1);
    if (lanes > 1) {
        VAM_TRY_CUDA(cudaEventRecord(b->fork, st));
        for (int s = 0; s + 1 < lanes; ++s) VAM_TRY_CUDA(cudaStreamWaitEvent(b->side[s], b->fork, 0));
    }
    const int rc_launch = batch_launch(b, n, st, lanes);
    // joined even after a failed launch, so a stream capture never ends with a side stream forked
    for (int s = 0; s + 1 < lanes; ++s) {
        VAM_TRY_CUDA(cudaEventRecord(b->join[s], b->side[s]));
        VAM_TRY_CUDA(cudaStreamWaitEvent(st, b->join[s], 0));
    }
    return rc_launch;
}

extern "C" int vam_batch_info(vam_batch* b, int64_t* virtual_blocks, int32_t* ctas) {
    clear_error();
    VAM_REQUIRE(b, VAM_ERR_ARG, "vam_batch_info: null argument");
    if (virtual_blocks) *virtual_blocks = b->blocks;
    if (ctas) *ctas = b->ctas;
    return VAM_OK;
}
