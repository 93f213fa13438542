// vecgeom.cu -- parallel-beam projector in ASTRA's vector geometry
// (parallel3d / parallel3d_vec), the model behind the reference's CUDA
// path Projector3DParallelCUDAAstra (vamtoolbox/projector/
// Projector3DParallelCUDA.py:13-72) and its inclined (laminography)
// geometry from genVectorsAstra (vamtoolbox/projector/genVectorsAstra.py:4-53).
//
// Model (restated from ASTRA's published geometry and projector
// descriptions; ASTRA itself is not available to pin against):
//  * volume [nY][nX][nZ] = ASTRA (col x, row y, slice z); voxel (i, j, k) is
//    centred at (i + 0.5 - nY/2, j + 0.5 - nX/2, k + 0.5 - nZ/2);
//  * detector [nU][nA][nV]; pixel (c, r) of angle a is centred at
//    d + (c - nU/2 + 0.5) u + (r - nV/2 + 0.5) v, its ray has direction ray;
//  * forward: Joseph-type line integral -- the ray is sampled on every voxel
//    plane across its dominant axis (largest |ray| component), bilinearly
//    within the plane with zero outside the volume, and the sum is scaled by
//    |ray| / |ray_dominant| (path length per plane);
//  * backward: voxel-driven -- each voxel centre is carried along the ray
//    onto the detector plane and the sinogram is sampled there bilinearly
//    (zero outside), summed over angles.
// All coordinates are affine in the loop indices: the plan holds, per angle,
// the coefficients of the in-plane sample position (forward) and of the
// detector position (backward), computed on the host in double.
#include "vam_internal.cuh"

#include <math.h>

#include <algorithm>
#include <vector>

using vam::clear_error;
using vam::set_error;

namespace {

constexpr int kThreads = 256;

// Forward, per angle: dominant axis (0 = x/i, 1 = y/j, 2 = z/k), the two
// in-plane continuous indices p = c0 + cc*c + cr*r + cs*s for s the plane
// index (first the lower-numbered remaining axis, then the other), and the
// path-length scale.
struct FwdAngle {
    float p0[4];   // c0, cc, cr, cs of in-plane axis A
    float p1[4];   // of in-plane axis B
    float scale;
    int axis;
    int pad[2];
};

// Backward, per angle: detector column / row continuous indices as affine
// functions of the voxel index (i, j, k).
struct BwdAngle {
    float u[4];    // u0, ui, uj, uk
    float v[4];    // v0, vi, vj, vk
};

__device__ __forceinline__ float affine(const float (&q)[4], float a, float b, float c) {
    return fmaf(q[3], c, fmaf(q[2], b, fmaf(q[1], a, q[0])));
}

// Bilinear sample of an [n0][n1] plane (element strides s0, s1, 32-bit
// offsets) at continuous indices (f0, f1), zero outside: interpolate along
// axis 1 in the two axis-0 rows, then across them.
__device__ __forceinline__ float bilerp(const float* __restrict__ base, float f0, float f1, int n0, int n1, int s0,
                                        int s1) {
    const float g0 = floorf(f0), g1 = floorf(f1);
    const int i0 = (int)g0, i1 = (int)g1;
    const float t0 = f0 - g0, t1 = f1 - g1;
    const bool a0 = (unsigned)i0 < (unsigned)n0, b0 = (unsigned)(i0 + 1) < (unsigned)n0;
    const bool a1 = (unsigned)i1 < (unsigned)n1, b1 = (unsigned)(i1 + 1) < (unsigned)n1;
    const int o = i0 * s0 + i1 * s1;
    const float x00 = (a0 && a1) ? __ldg(base + o) : 0.f;
    const float x01 = (a0 && b1) ? __ldg(base + o + s1) : 0.f;
    const float x10 = (b0 && a1) ? __ldg(base + o + s0) : 0.f;
    const float x11 = (b0 && b1) ? __ldg(base + o + s0 + s1) : 0.f;
    const float r0 = fmaf(t1, x01 - x00, x00), r1 = fmaf(t1, x11 - x10, x10);
    return fmaf(t0, r1 - r0, r0);
}

// bilerp where all four taps are known to lie inside the plane: the same arithmetic and loads, no
// bounds tests
__device__ __forceinline__ float bilerp_in(const float* __restrict__ base, float f0, float f1, int s0, int s1) {
    const float g0 = floorf(f0), g1 = floorf(f1);
    const int o = (int)g0 * s0 + (int)g1 * s1;
    const float t0 = f0 - g0, t1 = f1 - g1;
    const float x00 = __ldg(base + o), x01 = __ldg(base + o + s1);
    const float x10 = __ldg(base + o + s0), x11 = __ldg(base + o + s0 + s1);
    const float r0 = fmaf(t1, x01 - x00, x00), r1 = fmaf(t1, x11 - x10, x10);
    return fmaf(t0, r1 - r0, r0);
}

// Planes s in [lo, hi) on which f = f0 + m s stays inside [eps, n - 1 - eps] (so floor(f) and
// floor(f) + 1 are both valid indices), narrowed by one plane at each end against the rounding of
// the bound; the margin eps = 1e-3 in index units is far above the rounding of fmaf(m, s, f0).
__device__ __forceinline__ void inside_planes(float f0, float m, int n, int np, int& lo, int& hi) {
    const float a = 1e-3f, b = (float)(n - 1) - 1e-3f;
    if (!(b > a) || !isfinite(f0) || !isfinite(m)) { lo = 0; hi = 0; return; }
    if (fabsf(m) < 1e-20f) {
        if (f0 >= a && f0 <= b) { lo = 0; hi = np; } else { lo = 0; hi = 0; }
        return;
    }
    float s0 = (a - f0) / m, s1 = (b - f0) / m;
    if (m < 0.f) { const float t = s0; s0 = s1; s1 = t; }
    const float l = fmaxf(ceilf(s0) + 1.f, 0.f), h = fminf(floorf(s1) - 1.f, (float)(np - 1));
    if (!(h >= l)) { lo = 0; hi = 0; return; }
    lo = (int)l;
    hi = (int)h + 1;
}

// Linear sample along one axis (slice-exact geometries: the other in-plane
// coordinate is an integer voxel index on every sample).
__device__ __forceinline__ float lerp1(const float* __restrict__ base, float f, int n, int s) {
    const float g = floorf(f);
    const int i0 = (int)g;
    const float t = f - g;
    const float x0 = (unsigned)i0 < (unsigned)n ? __ldg(base + i0 * s) : 0.f;
    const float x1 = (unsigned)(i0 + 1) < (unsigned)n ? __ldg(base + (i0 + 1) * s) : 0.f;
    return fmaf(t, x1 - x0, x0);
}

// Forward: one thread per detector pixel (c, a, r), r fastest.  FLAT: every
// ray stays in the slice k = r (no inclination), the in-plane z coordinate
// is exact and only the horizontal axis is interpolated.
template <bool FLAT, bool HU>
__global__ void __launch_bounds__(kThreads) k_vec_forward(const float* __restrict__ vol, float* __restrict__ sino,
                                                          const FwdAngle* __restrict__ ang, int nY, int nX, int nZ,
                                                          int nU, int nA, int nV) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    const int c = blockIdx.z;
    if (r >= nV) return;
    const FwdAngle g = ang[a];
    const int sI = nX * nZ, sJ = nZ;
    const float fc = (float)c, fr = (float)r;
    float acc = 0.f;
    if (g.axis <= 1) {            // planes across i (axis 0) or j (axis 1); in-plane (other of i/j, k)
        const int plane = g.axis == 0 ? sI : sJ, hs = g.axis == 0 ? sJ : sI, nh = g.axis == 0 ? nX : nY;
        const int np = g.axis == 0 ? nY : nX;
        // HU: the horizontal coordinate has no row term, so it is the same for
        // every lane of the warp (computed from block indices and s only)
        const float h0 = affine(g.p0, fc, HU ? 0.f : fr, 0.f), k0 = affine(g.p1, fc, fr, 0.f);
        if (FLAT) {
#pragma unroll 4
            for (int s = 0; s < np; ++s) acc += lerp1(vol + s * plane + r, fmaf(g.p0[3], (float)s, h0), nh, hs);
        } else {
            // the planes where every lane's four taps are inside run without bounds tests; the sum keeps
            // its order, so the result is bit-identical
            int lo, hi, lo1, hi1;
            inside_planes(h0, g.p0[3], nh, np, lo, hi);
            inside_planes(k0, g.p1[3], nZ, np, lo1, hi1);
            lo = max(lo, lo1);
            hi = min(hi, hi1);
            const unsigned act = __activemask();
            lo = __reduce_max_sync(act, lo);
            hi = __reduce_min_sync(act, hi);
            if (hi < lo) hi = lo;
            auto checked = [&](int s) {
                return bilerp(vol + s * plane, fmaf(g.p0[3], (float)s, h0), fmaf(g.p1[3], (float)s, k0), nh, nZ, hs, 1);
            };
#pragma unroll 4
            for (int s = 0; s < lo; ++s) acc += checked(s);
#pragma unroll 4
            for (int s = lo; s < hi; ++s)
                acc += bilerp_in(vol + s * plane, fmaf(g.p0[3], (float)s, h0), fmaf(g.p1[3], (float)s, k0), hs, 1);
#pragma unroll 4
            for (int s = hi; s < np; ++s) acc += checked(s);
        }
    } else {                      // planes across k; in-plane (i, j)
        const float i0 = affine(g.p0, fc, fr, 0.f), j0 = affine(g.p1, fc, fr, 0.f);
        int lo, hi, lo1, hi1;
        inside_planes(i0, g.p0[3], nY, nZ, lo, hi);
        inside_planes(j0, g.p1[3], nX, nZ, lo1, hi1);
        lo = max(lo, lo1);
        hi = min(hi, hi1);
        const unsigned act = __activemask();
        lo = __reduce_max_sync(act, lo);
        hi = __reduce_min_sync(act, hi);
        if (hi < lo) hi = lo;
#pragma unroll 4
        for (int s = 0; s < lo; ++s)
            acc += bilerp(vol + s, fmaf(g.p0[3], (float)s, i0), fmaf(g.p1[3], (float)s, j0), nY, nX, sI, sJ);
#pragma unroll 4
        for (int s = lo; s < hi; ++s)
            acc += bilerp_in(vol + s, fmaf(g.p0[3], (float)s, i0), fmaf(g.p1[3], (float)s, j0), sI, sJ);
#pragma unroll 4
        for (int s = hi; s < nZ; ++s)
            acc += bilerp(vol + s, fmaf(g.p0[3], (float)s, i0), fmaf(g.p1[3], (float)s, j0), nY, nX, sI, sJ);
    }
    sino[(c * nA + a) * nV + r] = acc * g.scale;
}

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void mix4(float4& acc, float4 x0, float4 x1, float t) {
    acc.x += fmaf(t, x1.x - x0.x, x0.x);
    acc.y += fmaf(t, x1.y - x0.y, x0.y);
    acc.z += fmaf(t, x1.z - x0.z, x0.z);
    acc.w += fmaf(t, x1.w - x0.w, x0.w);
}

// Slice-exact forward with four detector rows (= four slices) per lane: the
// horizontal coordinate does not depend on the row, so one weight and two
// 16-byte loads serve four samples.  nZ % 4 == 0, 16-byte aligned arrays.
// Block = rows_per_block detector rows (c, a) x lanes_per_row lanes.
// six resident CTAs per SM (40 registers, no spills): 2.47 -> 2.31 ms at 256^3 x 360
__global__ void __launch_bounds__(kThreads, 6) k_vec_forward_flat4(const float* __restrict__ vol,
                                                                float* __restrict__ sino,
                                                                const FwdAngle* __restrict__ ang, int nY, int nX,
                                                                int nZ, int nU, int nA, int nV, int lanes_per_row) {
    const int rows_per_block = blockDim.x / lanes_per_row;
    const int row = blockIdx.x * rows_per_block + threadIdx.x / lanes_per_row;   // c * nA + a
    const int r = (threadIdx.x % lanes_per_row) * 4;
    if (row >= nU * nA || r >= nV) return;
    const int c = row / nA, a = row - c * nA;
    const FwdAngle g = ang[a];
    const int sI = nX * nZ, sJ = nZ;
    const int plane = g.axis == 0 ? sI : sJ, hs = g.axis == 0 ? sJ : sI, nh = g.axis == 0 ? nX : nY;
    const int np = g.axis == 0 ? nY : nX;
    const float h0 = affine(g.p0, (float)c, 0.f, 0.f);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 acc = zero;
#pragma unroll 4
    for (int s = 0; s < np; ++s) {
        const float fh = fmaf(g.p0[3], (float)s, h0);
        const float gh = floorf(fh);
        const int i0 = (int)gh;
        const float t = fh - gh;
        const float* pl = vol + s * plane + r;
        const float4 x0 = (unsigned)i0 < (unsigned)nh ? ld4(pl + i0 * hs) : zero;
        const float4 x1 = (unsigned)(i0 + 1) < (unsigned)nh ? ld4(pl + (i0 + 1) * hs) : zero;
        mix4(acc, x0, x1, t);
    }
    const float sc = g.scale;
    *reinterpret_cast<float4*>(sino + (c * nA + a) * nV + r) =
        make_float4(acc.x * sc, acc.y * sc, acc.z * sc, acc.w * sc);
}

// Slice-exact backward with four slices per lane (the detector column does
// not depend on k).
__global__ void __launch_bounds__(kThreads) k_vec_backward_flat4(const float* __restrict__ sino,
                                                                 float* __restrict__ vol,
                                                                 const BwdAngle* __restrict__ ang, int nY, int nX,
                                                                 int nZ, int nU, int nA, int nV, int lanes_per_row) {
    const int rows_per_block = blockDim.x / lanes_per_row;
    const int col = blockIdx.x * rows_per_block + threadIdx.x / lanes_per_row;   // i * nX + j
    const int k = (threadIdx.x % lanes_per_row) * 4;
    if (col >= nY * nX || k >= nZ) return;
    const int i = col / nX, j = col - i * nX;
    const float fi = (float)i, fj = (float)j;
    const int sC = nA * nV;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 acc = zero;
#pragma unroll 4
    for (int a = 0; a < nA; ++a) {
        const BwdAngle g = ang[a];
        const float fu = affine(g.u, fi, fj, 0.f);
        const float gu = floorf(fu);
        const int c0 = (int)gu;
        const float t = fu - gu;
        const float* pl = sino + a * nV + k;
        const float4 x0 = (unsigned)c0 < (unsigned)nU ? ld4(pl + c0 * sC) : zero;
        const float4 x1 = (unsigned)(c0 + 1) < (unsigned)nU ? ld4(pl + (c0 + 1) * sC) : zero;
        mix4(acc, x0, x1, t);
    }
    *reinterpret_cast<float4*>(vol + (i * nX + j) * nZ + k) = acc;
}

// Exact transpose of the forward (for gradients; ASTRA's backprojection is
// voxel-driven and is not): every ray walks the forward's samples and adds
// g * scale * weight to the taps it read.  Float atomics: exact up to the
// order of the additions.
__device__ __forceinline__ void scatter_bilerp(float* __restrict__ base, float f0, float f1, int n0, int n1, int s0,
                                               int s1, float v) {
    const float g0 = floorf(f0), g1 = floorf(f1);
    const int i0 = (int)g0, i1 = (int)g1;
    const float t0 = f0 - g0, t1 = f1 - g1;
    const bool a0 = (unsigned)i0 < (unsigned)n0, b0 = (unsigned)(i0 + 1) < (unsigned)n0;
    const bool a1 = (unsigned)i1 < (unsigned)n1, b1 = (unsigned)(i1 + 1) < (unsigned)n1;
    const int o = i0 * s0 + i1 * s1;
    const float r0 = v * (1.f - t0), r1 = v * t0;
    if (a0 && a1) atomicAdd(base + o, r0 * (1.f - t1));
    if (a0 && b1) atomicAdd(base + o + s1, r0 * t1);
    if (b0 && a1) atomicAdd(base + o + s0, r1 * (1.f - t1));
    if (b0 && b1) atomicAdd(base + o + s0 + s1, r1 * t1);
}

__global__ void __launch_bounds__(kThreads) k_vec_adjoint(const float* __restrict__ sino, float* __restrict__ vol,
                                                          const FwdAngle* __restrict__ ang, int nY, int nX, int nZ,
                                                          int nU, int nA, int nV) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    const int c = blockIdx.z;
    if (r >= nV) return;
    const FwdAngle g = ang[a];
    const float v = sino[(c * nA + a) * nV + r] * g.scale;
    if (v == 0.f) return;
    const int sI = nX * nZ, sJ = nZ;
    const float fc = (float)c, fr = (float)r;
    if (g.axis <= 1) {
        const int plane = g.axis == 0 ? sI : sJ, hs = g.axis == 0 ? sJ : sI, nh = g.axis == 0 ? nX : nY;
        const int np = g.axis == 0 ? nY : nX;
        const float h0 = affine(g.p0, fc, fr, 0.f), k0 = affine(g.p1, fc, fr, 0.f);
        for (int s = 0; s < np; ++s)
            scatter_bilerp(vol + s * plane, fmaf(g.p0[3], (float)s, h0), fmaf(g.p1[3], (float)s, k0), nh, nZ, hs, 1, v);
    } else {
        const float i0 = affine(g.p0, fc, fr, 0.f), j0 = affine(g.p1, fc, fr, 0.f);
        for (int s = 0; s < nZ; ++s)
            scatter_bilerp(vol + s, fmaf(g.p0[3], (float)s, i0), fmaf(g.p1[3], (float)s, j0), nY, nX, sI, sJ, v);
    }
}

// Backward: one thread per voxel (i, j, k), k fastest; angles looped.
// FLAT: the detector row of voxel slice k is exactly k.
template <bool FLAT, bool HU>
__global__ void __launch_bounds__(kThreads) k_vec_backward(const float* __restrict__ sino, float* __restrict__ vol,
                                                           const BwdAngle* __restrict__ ang, int nY, int nX, int nZ,
                                                           int nU, int nA, int nV) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if (k >= nZ) return;
    const float fi = (float)i, fj = (float)j, fk = (float)k;
    const int sC = nA * nV;
    float acc = 0.f;
#pragma unroll 4
    for (int a = 0; a < nA; ++a) {
        const BwdAngle g = ang[a];
        const float fu = affine(g.u, fi, fj, HU ? 0.f : fk);   // HU: no k term, warp-uniform
        const float* pl = sino + a * nV;
        if (FLAT)
            acc += lerp1(pl + k, fu, nU, sC);
        else
            acc += bilerp(pl, fu, affine(g.v, fi, fj, fk), nU, nV, sC, 1);
    }
    vol[(i * nX + j) * nZ + k] = acc;
}

// ---------------------------------------------------------------------------
// 2-D "line" model (the projector the reference's Projector2DParallelCUDAAstra
// builds, vamtoolbox/projector/Projector2DParallelCUDA.py:7-45): the weight of
// a (ray, pixel) pair is the length of the ray -- a zero-width line -- inside
// the unit pixel square.  ASTRA's 2-D frame: pixel (i, j) of an [nY][nX]
// image at (j - nX/2 + 1/2, nY/2 - i - 1/2) (row 0 on top), detector bin d at
// offset d - nT/2 + 1/2 along u = (cos a, sin a), rays along (sin a, -cos a).
// For a line at signed normal distance t from the pixel centre the chord is
// 1/A for |t| <= (A-B)/2, ((A+B)/2 - |t|) / (A B) up to (A+B)/2, then 0, with
// A = max(|cos|, |sin|), B = min.  Forward and backward evaluate the same t
// (fmaf(y, s, x c) - t_d) for a (ray, pixel) pair, so the backward is the
// forward's exact transpose.
// ---------------------------------------------------------------------------
struct LineAngle {
    float c, s;          // cos, sin
    float half_diff;     // (A - B) / 2
    float half_sum;      // (A + B) / 2
    float full;          // 1 / A
    float inv_ab;        // 1 / (A B), 0 when B == 0
    int along_x;         // |sin| >= |cos|: rays run mostly along x, one band per column
    int pad;
};

__device__ __forceinline__ float chord(float t, const LineAngle& g) {
    const float at = fabsf(t);
    if (at <= g.half_diff) return g.full;
    if (at >= g.half_sum) return 0.f;
    return (g.half_sum - at) * g.inv_ab;
}

__global__ void __launch_bounds__(kThreads) k_line2d_forward(const float* __restrict__ img, float* __restrict__ sino,
                                                             const LineAngle* __restrict__ ang, int nY, int nX,
                                                             int nT, int nA) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;   // a * nT + d (bins of one angle adjacent)
    if (gid >= nA * nT) return;
    const int a = gid / nT, d = gid - a * nT;
    const LineAngle g = ang[a];
    const float td = (float)d - 0.5f * (float)nT + 0.5f;
    const float x0 = 0.5f - 0.5f * (float)nX, y0 = 0.5f * (float)nY - 0.5f;   // centre of pixel (0, 0)
    float acc = 0.f;
    if (g.along_x) {
        for (int j = 0; j < nX; ++j) {
            const float x = x0 + (float)j;
            const float y = (td - x * g.c) / g.s;          // crossing of the column centre line
            const int ic = __float2int_rn(y0 - y);
#pragma unroll
            for (int q = -1; q <= 1; ++q) {
                const int i = ic + q;
                if ((unsigned)i >= (unsigned)nY) continue;
                const float yi = y0 - (float)i;
                const float w = chord(fmaf(yi, g.s, x * g.c) - td, g);
                if (w != 0.f) acc = fmaf(w, __ldg(img + i * nX + j), acc);
            }
        }
    } else {
        for (int i = 0; i < nY; ++i) {
            const float y = y0 - (float)i;
            const float x = (td - y * g.s) / g.c;          // crossing of the row centre line
            const int jc = __float2int_rn(x - x0);
#pragma unroll
            for (int q = -1; q <= 1; ++q) {
                const int j = jc + q;
                if ((unsigned)j >= (unsigned)nX) continue;
                const float xj = x0 + (float)j;
                const float w = chord(fmaf(y, g.s, xj * g.c) - td, g);
                if (w != 0.f) acc = fmaf(w, __ldg(img + i * nX + j), acc);
            }
        }
    }
    sino[d * nA + a] = acc;
}

__global__ void __launch_bounds__(kThreads) k_line2d_backward(const float* __restrict__ sino, float* __restrict__ img,
                                                              const LineAngle* __restrict__ ang, int nY, int nX,
                                                              int nT, int nA) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;   // i * nX + j
    if (gid >= nY * nX) return;
    const int i = gid / nX, j = gid - i * nX;
    const float x = 0.5f - 0.5f * (float)nX + (float)j, y = 0.5f * (float)nY - 0.5f - (float)i;
    const float dofs = 0.5f * (float)nT - 0.5f;
    float acc = 0.f;
    for (int a = 0; a < nA; ++a) {
        const LineAngle g = ang[a];
        const float tp = fmaf(y, g.s, x * g.c);
        const int dc = __float2int_rn(tp + dofs);
#pragma unroll
        for (int q = -1; q <= 1; ++q) {
            const int d = dc + q;
            if ((unsigned)d >= (unsigned)nT) continue;
            const float td = (float)d - 0.5f * (float)nT + 0.5f;
            const float w = chord(tp - td, g);
            if (w != 0.f) acc = fmaf(w, __ldg(sino + d * nA + a), acc);
        }
    }
    img[gid] = acc;
}

}  // namespace

struct vam_line2d_plan {
    int nY, nX, nT, nA, device;
    LineAngle* d_ang;
};

extern "C" int vam_line2d_plan_create(int32_t n_y, int32_t n_x, int32_t n_angles, const double* angles_deg,
                                      int32_t det_count, int32_t device, vam_line2d_plan** out) {
    clear_error();
    VAM_REQUIRE(angles_deg && out, VAM_ERR_ARG, "vam_line2d_plan_create: null argument");
    VAM_REQUIRE(n_y > 0 && n_x > 0 && n_angles > 0 && det_count > 0, VAM_ERR_SHAPE,
                "vam_line2d_plan_create: empty image, detector or angle set");
    VAM_REQUIRE((int64_t)n_y * n_x < (1ll << 31) && (int64_t)det_count * n_angles < (1ll << 31), VAM_ERR_SHAPE,
                "vam_line2d_plan_create: image or sinogram of 2^31 elements or more");
    std::vector<LineAngle> h(n_angles);
    for (int a = 0; a < n_angles; ++a) {
        VAM_REQUIRE(isfinite(angles_deg[a]), VAM_ERR_ARG, "vam_line2d_plan_create: non-finite angle");
        const double th = angles_deg[a] * 3.14159265358979323846 / 180.0;
        const double c = cos(th), sn = sin(th);
        const double A = fmax(fabs(c), fabs(sn)), B = fmin(fabs(c), fabs(sn));
        LineAngle& g = h[a];
        g.c = (float)c;
        g.s = (float)sn;
        g.half_diff = (float)((A - B) / 2.0);
        g.half_sum = (float)((A + B) / 2.0);
        g.full = (float)(1.0 / A);
        g.inv_ab = B > 1e-12 ? (float)(1.0 / (A * B)) : 0.f;
        g.along_x = fabs(sn) >= fabs(c);
        g.pad = 0;
    }
    vam::DeviceGuard dg(device);
    VAM_REQUIRE(dg.ok, VAM_ERR_CUDA, "vam_line2d_plan_create: cannot select the device");
    vam_line2d_plan* p = new vam_line2d_plan{n_y, n_x, det_count, n_angles, device, nullptr};
    if (cudaMalloc(&p->d_ang, sizeof(LineAngle) * n_angles) != cudaSuccess) {
        delete p;
        return set_error(VAM_ERR_NOMEM, "vam_line2d_plan_create: cudaMalloc failed");
    }
    if (cudaMemcpy(p->d_ang, h.data(), sizeof(LineAngle) * n_angles, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(p->d_ang);
        delete p;
        return set_error(VAM_ERR_CUDA, "vam_line2d_plan_create: table upload failed");
    }
    *out = p;
    return VAM_OK;
}

extern "C" int vam_line2d_plan_destroy(vam_line2d_plan* p) {
    clear_error();
    if (!p) return VAM_OK;
    vam::DeviceGuard dg(p->device);
    cudaFree(p->d_ang);
    delete p;
    return VAM_OK;
}

extern "C" int vam_line2d_forward(vam_line2d_plan* p, const float* img, float* sino, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && img && sino, VAM_ERR_ARG, "vam_line2d_forward: null argument");
    vam::DeviceGuard dg(p->device);
    const int n = p->nA * p->nT;
    k_line2d_forward<<<(n + kThreads - 1) / kThreads, kThreads, 0, (cudaStream_t)stream>>>(img, sino, p->d_ang, p->nY,
                                                                                        p->nX, p->nT, p->nA);
    VAM_CHECK_LAUNCH("vam_line2d_forward");
    return VAM_OK;
}

extern "C" int vam_line2d_backward(vam_line2d_plan* p, const float* sino, float* img, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && img && sino, VAM_ERR_ARG, "vam_line2d_backward: null argument");
    vam::DeviceGuard dg(p->device);
    const int n = p->nY * p->nX;
    k_line2d_backward<<<(n + kThreads - 1) / kThreads, kThreads, 0, (cudaStream_t)stream>>>(sino, img, p->d_ang,
                                                                                         p->nY, p->nX, p->nT, p->nA);
    VAM_CHECK_LAUNCH("vam_line2d_backward");
    return VAM_OK;
}

struct vam_vec_plan {
    int nY, nX, nZ, nU, nA, nV, device;
    bool flat_fwd, flat_bwd;
    bool hu_fwd, hu_bwd;     // horizontal coordinate independent of the detector row / voxel z
    FwdAngle* d_fwd;
    BwdAngle* d_bwd;
};

namespace {

// Lanes per detector row (or voxel column) for the four-wide kernels: the
// smallest power of two >= the float4 groups, at least one warp.
int lanes_for(int groups) {
    int l = 32;
    while (l < groups) l <<= 1;
    return l;
}

bool solve3(const double m[3][3], double inv[3][3]) {
    const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                       m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                       m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    if (!(fabs(det) > 1e-12)) return false;
    inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) / det;
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
    inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det;
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
    inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / det;
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
    return true;
}

}  // namespace

extern "C" int vam_vec_plan_create(const vam_vec_geom* geom, vam_vec_plan** out) {
    clear_error();
    VAM_REQUIRE(geom && out && geom->vectors, VAM_ERR_ARG, "vam_vec_plan_create: null argument");
    const int nY = geom->n_y, nX = geom->n_x, nZ = geom->n_z, nA = geom->n_angles;
    const int nU = geom->det_cols, nV = geom->det_rows;
    VAM_REQUIRE(nY > 0 && nX > 0 && nZ > 0 && nA > 0 && nU > 0 && nV > 0, VAM_ERR_SHAPE,
                "vam_vec_plan_create: empty volume, detector or angle set");
    VAM_REQUIRE(nA <= 65535 && nU <= 65535 && nY <= 65535 && nX <= 65535, VAM_ERR_SHAPE,
                "vam_vec_plan_create: dimension above 65535");
    VAM_REQUIRE((int64_t)nY * nX * nZ < (1ll << 31) && (int64_t)nU * nA * nV < (1ll << 31), VAM_ERR_SHAPE,
                "vam_vec_plan_create: volume or sinogram of 2^31 elements or more");
    const double cx = 0.5 - nY / 2.0, cy = 0.5 - nX / 2.0, cz = 0.5 - nZ / 2.0;   // voxel (0,0,0) centre
    std::vector<FwdAngle> fw(nA);
    std::vector<BwdAngle> bw(nA);
    bool flat_f = true, flat_b = true, hu_f = true, hu_b = true;
    // coefficients whose effect over the whole index range stays below 1e-6
    // voxel / pixel are rounding residue of an exact zero: snap them
    auto snap = [](float& c, double extent) {
        if (fabs((double)c) * extent < 1e-6) c = 0.f;
    };
    for (int a = 0; a < nA; ++a) {
        const double* q = geom->vectors + 12 * a;
        for (int t = 0; t < 12; ++t)
            VAM_REQUIRE(isfinite(q[t]), VAM_ERR_ARG, "vam_vec_plan_create: non-finite geometry vector");
        const double ray[3] = {q[0], q[1], q[2]}, d[3] = {q[3], q[4], q[5]};
        const double u[3] = {q[6], q[7], q[8]}, v[3] = {q[9], q[10], q[11]};
        // detector pixel (c, r) centre: P00 + c u + r v
        double P00[3];
        for (int t = 0; t < 3; ++t) P00[t] = d[t] + (0.5 - nU / 2.0) * u[t] + (0.5 - nV / 2.0) * v[t];
        const double ar[3] = {fabs(ray[0]), fabs(ray[1]), fabs(ray[2])};
        VAM_REQUIRE(ar[0] + ar[1] + ar[2] > 0, VAM_ERR_ARG, "vam_vec_plan_create: zero ray direction");
        const int ax = (ar[0] >= ar[1] && ar[0] >= ar[2]) ? 0 : (ar[1] >= ar[2] ? 1 : 2);
        const int pa = ax == 0 ? 1 : 0, pb = ax == 2 ? 1 : 2;   // in-plane axes, ascending
        const double cen[3] = {cx, cy, cz};
        FwdAngle& g = fw[a];
        g.axis = ax;
        g.scale = (float)(sqrt(ray[0] * ray[0] + ray[1] * ray[1] + ray[2] * ray[2]) / ar[ax]);
        // plane s of axis ax sits at world cen[ax] + s; a ray from P hits it at
        // P + ((cen[ax] + s - P[ax]) / ray[ax]) ray, whose continuous index on
        // axis b is (P[b] - cen[b]) + (cen[ax] + s - P[ax]) * ray[b] / ray[ax]
        for (int w = 0; w < 2; ++w) {
            const int b = w == 0 ? pa : pb;
            const double slope = ray[b] / ray[ax];
            float* p = w == 0 ? g.p0 : g.p1;
            p[0] = (float)((P00[b] - cen[b]) + (cen[ax] - P00[ax]) * slope);
            p[1] = (float)(u[b] - u[ax] * slope);
            p[2] = (float)(v[b] - v[ax] * slope);
            p[3] = (float)slope;
        }
        for (int w = 0; w < 2; ++w) {
            float* p = w == 0 ? g.p0 : g.p1;
            snap(p[0], 1.0);
            snap(p[1], nU);
            snap(p[2], nV);
            snap(p[3], std::max(nY, std::max(nX, nZ)));   // per plane, over every plane
        }
        if (g.p0[2] != 0.f) hu_f = false;
        // slice-exact: the z index of every sample is the detector row, and the
        // horizontal coordinate does not depend on the row
        if (!(ax != 2 && g.p1[0] == 0.f && g.p1[1] == 0.f && g.p1[2] == 1.f && g.p1[3] == 0.f && g.p0[2] == 0.f))
            flat_f = false;
        // backward: solve p - d = U u + V v + t ray; column index = U + nU/2 - 0.5
        const double M[3][3] = {{u[0], v[0], ray[0]}, {u[1], v[1], ray[1]}, {u[2], v[2], ray[2]}};
        double Mi[3][3];
        VAM_REQUIRE(solve3(M, Mi), VAM_ERR_ARG, "vam_vec_plan_create: ray parallel to the detector plane");
        BwdAngle& h = bw[a];
        for (int w = 0; w < 2; ++w) {
            const double* row = Mi[w];
            const double off = w == 0 ? nU / 2.0 - 0.5 : nV / 2.0 - 0.5;
            float* p = w == 0 ? h.u : h.v;
            p[0] = (float)(row[0] * (cx - d[0]) + row[1] * (cy - d[1]) + row[2] * (cz - d[2]) + off);
            p[1] = (float)row[0];
            p[2] = (float)row[1];
            p[3] = (float)row[2];
        }
        for (int w = 0; w < 2; ++w) {
            float* p = w == 0 ? h.u : h.v;
            snap(p[0], 1.0);
            snap(p[1], nY);
            snap(p[2], nX);
            snap(p[3], nZ);
        }
        if (h.u[3] != 0.f) hu_b = false;
        if (!(h.v[0] == 0.f && h.v[1] == 0.f && h.v[2] == 0.f && h.v[3] == 1.f && h.u[3] == 0.f)) flat_b = false;
    }
    if (nV != nZ) flat_f = flat_b = false;
    vam::DeviceGuard dg(geom->device);
    VAM_REQUIRE(dg.ok, VAM_ERR_CUDA, "vam_vec_plan_create: cannot select the device");
    vam_vec_plan* p = new vam_vec_plan{nY, nX, nZ, nU, nA, nV, geom->device, flat_f, flat_b, hu_f, hu_b,
                                       nullptr, nullptr};
    if (cudaMalloc(&p->d_fwd, sizeof(FwdAngle) * nA) != cudaSuccess ||
        cudaMalloc(&p->d_bwd, sizeof(BwdAngle) * nA) != cudaSuccess) {
        cudaFree(p->d_fwd);
        delete p;
        return set_error(VAM_ERR_NOMEM, "vam_vec_plan_create: cudaMalloc failed");
    }
    if (cudaMemcpy(p->d_fwd, fw.data(), sizeof(FwdAngle) * nA, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_bwd, bw.data(), sizeof(BwdAngle) * nA, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(p->d_fwd);
        cudaFree(p->d_bwd);
        delete p;
        return set_error(VAM_ERR_CUDA, "vam_vec_plan_create: table upload failed");
    }
    *out = p;
    return VAM_OK;
}

extern "C" int vam_vec_plan_destroy(vam_vec_plan* p) {
    clear_error();
    if (!p) return VAM_OK;
    vam::DeviceGuard dg(p->device);
    cudaFree(p->d_fwd);
    cudaFree(p->d_bwd);
    delete p;
    return VAM_OK;
}

extern "C" int vam_vec_plan_info(const vam_vec_plan* p, int32_t* flat_forward, int32_t* flat_backward) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_vec_plan_info: null plan");
    if (flat_forward) *flat_forward = p->flat_fwd;
    if (flat_backward) *flat_backward = p->flat_bwd;
    return VAM_OK;
}

extern "C" int vam_vec_forward(vam_vec_plan* p, const float* vol, float* sino, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && vol && sino, VAM_ERR_ARG, "vam_vec_forward: null argument");
    vam::DeviceGuard dg(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (p->flat_fwd && p->nV % 4 == 0 && p->nV / 4 <= kThreads && ((uintptr_t)vol & 15u) == 0 &&
        ((uintptr_t)sino & 15u) == 0) {
        const int lanes = lanes_for(p->nV / 4);
        const int rows = (int)((int64_t)p->nU * p->nA), per_block = kThreads / lanes;
        k_vec_forward_flat4<<<(rows + per_block - 1) / per_block, kThreads, 0, st>>>(
            vol, sino, p->d_fwd, p->nY, p->nX, p->nZ, p->nU, p->nA, p->nV, lanes);
        VAM_CHECK_LAUNCH("vam_vec_forward");
        return VAM_OK;
    }
    dim3 grid((p->nV + kThreads - 1) / kThreads, p->nA, p->nU);
    if (p->flat_fwd)
        k_vec_forward<true, false><<<grid, kThreads, 0, st>>>(vol, sino, p->d_fwd, p->nY, p->nX, p->nZ, p->nU,
                                                              p->nA, p->nV);
    else if (p->hu_fwd)
        k_vec_forward<false, true><<<grid, kThreads, 0, st>>>(vol, sino, p->d_fwd, p->nY, p->nX, p->nZ, p->nU,
                                                              p->nA, p->nV);
    else
        k_vec_forward<false, false><<<grid, kThreads, 0, st>>>(vol, sino, p->d_fwd, p->nY, p->nX, p->nZ, p->nU,
                                                               p->nA, p->nV);
    VAM_CHECK_LAUNCH("vam_vec_forward");
    return VAM_OK;
}

extern "C" int vam_vec_adjoint(vam_vec_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && vol && sino, VAM_ERR_ARG, "vam_vec_adjoint: null argument");
    vam::DeviceGuard dg(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    VAM_TRY_CUDA(cudaMemsetAsync(vol, 0, sizeof(float) * (size_t)p->nY * p->nX * p->nZ, st));
    dim3 grid((p->nV + kThreads - 1) / kThreads, p->nA, p->nU);
    k_vec_adjoint<<<grid, kThreads, 0, st>>>(sino, vol, p->d_fwd, p->nY, p->nX, p->nZ, p->nU, p->nA, p->nV);
    VAM_CHECK_LAUNCH("vam_vec_adjoint");
    return VAM_OK;
}

extern "C" int vam_vec_backward(vam_vec_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && vol && sino, VAM_ERR_ARG, "vam_vec_backward: null argument");
    vam::DeviceGuard dg(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (p->flat_bwd && p->nZ % 4 == 0 && p->nZ / 4 <= kThreads && ((uintptr_t)vol & 15u) == 0 &&
        ((uintptr_t)sino & 15u) == 0) {
        const int lanes = lanes_for(p->nZ / 4);
        const int cols = (int)((int64_t)p->nY * p->nX), per_block = kThreads / lanes;
        k_vec_backward_flat4<<<(cols + per_block - 1) / per_block, kThreads, 0, st>>>(
            sino, vol, p->d_bwd, p->nY, p->nX, p->nZ, p->nU, p->nA, p->nV, lanes);
        VAM_CHECK_LAUNCH("vam_vec_backward");
        return VAM_OK;
    }
    dim3 grid((p->nZ + kThreads - 1) / kThreads, p->nX, p->nY);
    if (p->flat_bwd)
        k_vec_backward<true, false><<<grid, kThreads, 0, st>>>(sino, vol, p->d_bwd, p->nY, p->nX, p->nZ, p->nU,
                                                               p->nA, p->nV);
    else if (p->hu_bwd)
        k_vec_backward<false, true><<<grid, kThreads, 0, st>>>(sino, vol, p->d_bwd, p->nY, p->nX, p->nZ, p->nU,
                                                               p->nA, p->nV);
    else
        k_vec_backward<false, false><<<grid, kThreads, 0, st>>>(sino, vol, p->d_bwd, p->nY, p->nX, p->nZ, p->nU,
                                                                p->nA, p->nV);
    VAM_CHECK_LAUNCH("vam_vec_backward");
    return VAM_OK;
}
