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
#include <vector>

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
    int nY, nX, nZ, nA, C;
    int lz_shift, zvec, zchunks;
    float alpha, R;  // VAM_ABS_RAY
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
__global__ void __launch_bounds__(256) k_forward(Args a) {
    const int lane = threadIdx.x & 31;
    const int LZ = 1 << a.lz_shift;
    const int LK = 32 >> a.lz_shift;
    const int zl = lane & (LZ - 1);
    const int kl = lane >> a.lz_shift;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int theta = blockIdx.y;
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
template <int VZ>
__device__ __forceinline__ void load_vz(const float* __restrict__ p, float* d, int qn = VZ / 4) {
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q) {
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q < qn) t = __ldg(reinterpret_cast<const float4*>(p + 128 * q));
        d[4 * q] = t.x; d[4 * q + 1] = t.y; d[4 * q + 2] = t.z; d[4 * q + 3] = t.w;
    }
}

template <int VZ>
__device__ __forceinline__ void store_vz(float* __restrict__ p, const float* d, int qn) {
#pragma unroll
    for (int q = 0; q < VZ / 4; ++q)
        if (q < qn) *reinterpret_cast<float4*>(p + 128 * q) = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
}

// First slice and number of in-range vectors of a lane in z-chunk zc.
template <int VZ>
__device__ __forceinline__ void lane_z(int zc, int lane, int nZ, int& z0, int& qn) {
    const int base = zc * 32 * VZ + 4 * lane;
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
__global__ void __launch_bounds__(256) k_forward_fast(FastArgs a) {
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int zc = item % a.zchunks;
    const int j = item / a.zchunks;
    const int2 task = a.tasks[blockIdx.y];
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
                load_vz<VZ>(volz + o00, t0, qn);
                load_vz<VZ>(volz + o00 + dcol, t1, qn);
                load_vz<VZ>(volz + o10, t2, qn);
                load_vz<VZ>(volz + o10 + dcol, t3, qn);
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
__global__ void __launch_bounds__(256) k_adjoint_fast(Args a) {
    const int lane = threadIdx.x & 31;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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

// ---------------------------------------------------------------------------
// R2 backprojection, fast path: 32 lanes along z with VZ floats each (one
// pixel per warp, angles in sequence); same arithmetic as k_backward_ref.
// ---------------------------------------------------------------------------
template <int VZ, bool RAY>
__global__ void __launch_bounds__(256) k_backward_fast(Args a) {
    const int lane = threadIdx.x & 31;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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
        const size_t rs = (size_t)a.nA * a.nZ;
        const float* __restrict__ bz = a.in + z0;
#pragma unroll 2
        for (int th = 0; th < a.nA; ++th) {
            const double4 tr = a.trig[th];
            const double t = __dsub_rn(__dmul_rn(X, tr.x), __dmul_rn(Y, tr.y));
            if (!(t >= tlo && t <= thi)) continue;
            const double ft = floor(t);
            const int j0 = (int)ft + a.C;
            const float* b0 = bz + (size_t)j0 * rs + (size_t)th * a.nZ;
            float v0[VZ], v1[VZ];
            load_vz<VZ>(b0, v0, qn);
            // t == floor(t): np.interp returns fp[j]; the second row is read with weight 0
            const float w = (float)(t - ft);
            load_vz<VZ>(b0 + (t != ft ? rs : 0), v1, qn);
            float f = 1.f;
            if (RAY) {
                // |t| <= R is a discontinuity of the model: decide it on the float64 t
                f = 0.f;
                if (fabs(t) <= (double)a.R) {
                    const float sv = (float)__dadd_rn(__dmul_rn(X, tr.y), __dmul_rn(Y, tr.x));
                    f = ray_factor(sv, (float)(-sqrt((double)a.R * a.R - t * t)), a.alpha);
                }
            }
#pragma unroll
            for (int e = 0; e < VZ; ++e) {
                const float v = fmaf(w, v1[e] - v0[e], v0[e]);
                acc[e] = RAY ? fmaf(v, f, acc[e]) : acc[e] + v;
            }
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
__global__ void __launch_bounds__(256) k_adjoint_table(Args a, const float4* __restrict__ table) {
    const int lane = threadIdx.x & 31;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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
    if (a.mask) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] *= m;
    }
    store_vz<VZ>(a.out + (size_t)p * a.nZ + z0, acc, qn);
}

// ---------------------------------------------------------------------------
// R2 backprojection, batched: cos / sin of every angle staged in shared
// memory, and B angles per step whose detector-row loads are all issued
// before any is consumed, so each warp keeps 2B row loads in flight instead
// of waiting on one angle's float64 chain and loads at a time.
// ---------------------------------------------------------------------------
template <int VZ, int B, bool RAY>
__global__ void __launch_bounds__(256) k_backward_batched(Args a) {
    extern __shared__ double2 s_cs[];
    for (int t = threadIdx.x; t < a.nA; t += blockDim.x) s_cs[t] = make_double2(a.trig[t].x, a.trig[t].y);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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
        const size_t rs = (size_t)a.nA * a.nZ;
        const float* __restrict__ bz = a.in + z0;
        for (int th0 = 0; th0 < a.nA; th0 += B) {
            size_t o0[B], o1[B];
            float w[B], f[B];
            bool ok[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int th = th0 + u;
                ok[u] = th < a.nA;
                const double2 cs = s_cs[ok[u] ? th : 0];
                const double t = __dsub_rn(__dmul_rn(X, cs.x), __dmul_rn(Y, cs.y));
                ok[u] = ok[u] && (t >= tlo && t <= thi);
                const double ft = floor(t);
                const int j0 = ok[u] ? (int)ft + a.C : 0;
                w[u] = (float)(t - ft);
                o0[u] = (size_t)j0 * rs + (size_t)th * a.nZ;
                o1[u] = o0[u] + ((t != ft) ? rs : 0);
                f[u] = 1.f;
                if (RAY) {
                    f[u] = 0.f;
                    if (fabs(t) <= (double)a.R) {
                        const float sv = (float)__dadd_rn(__dmul_rn(X, cs.y), __dmul_rn(Y, cs.x));
                        f[u] = ray_factor(sv, (float)(-sqrt((double)a.R * a.R - t * t)), a.alpha);
                    }
                }
            }
            float v0[B][VZ], v1[B][VZ];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                if (ok[u]) {
                    load_vz<VZ>(bz + o0[u], v0[u], qn);
                    load_vz<VZ>(bz + o1[u], v1[u], qn);
                } else {
#pragma unroll
                    for (int e = 0; e < VZ; ++e) v0[u][e] = v1[u][e] = 0.f;
                }
            }
#pragma unroll
            for (int u = 0; u < B; ++u)
#pragma unroll
                for (int e = 0; e < VZ; ++e) {
                    const float v = fmaf(w[u], v1[u][e] - v0[u][e], v0[u][e]);
                    acc[e] = RAY ? fmaf(v, f[u], acc[e]) : acc[e] + v;
                }
        }
    }
    if (a.mask) {
        const float m = __ldg(a.mask + p);
#pragma unroll
        for (int e = 0; e < VZ; ++e) acc[e] = m * acc[e];
    }
    store_vz<VZ>(a.out + (size_t)p * a.nZ + z0, acc, qn);
}

__global__ void k_mask_mul(const float* __restrict__ x, const float* __restrict__ mask, float* __restrict__ out,
                           long npix, int nZ) {
    const long n = npix * nZ;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = mask[i / nZ] * x[i];
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
__global__ void __launch_bounds__(256) k_backward_ref(Args a) {
    const int lane = threadIdx.x & 31;
    const int LZ = 1 << a.lz_shift;
    const int LK = 32 >> a.lz_shift;
    const int zl = lane & (LZ - 1);
    const int kl = lane >> a.lz_shift;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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
#pragma unroll
                for (int e = 0; e < VZ; ++e) {
                    const double o = interp_nan(t, ft, j0, a.nY, a.C, a.occ + (size_t)th * a.nZ + z0 + e, rs);
                    if (sv > floor(o)) v[e] = 0.f;
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

// ---------------------------------------------------------------------------
// Matched transpose of k_forward
// ---------------------------------------------------------------------------
template <int VZ, bool OCC, int ABS>
__global__ void __launch_bounds__(256) k_adjoint(Args a) {
    const int lane = threadIdx.x & 31;
    const int LZ = 1 << a.lz_shift;
    const int LK = 32 >> a.lz_shift;
    const int zl = lane & (LZ - 1);
    const int kl = lane >> a.lz_shift;
    const long item = (long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
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

enum class Op { Forward, BackwardRef, Adjoint };

template <int VZ, bool OCC, int ABS>
void launch_one(Op op, const Args& a, long items, cudaStream_t st) {
    dim3 block(kWarpsPerBlock * kWarp);
    if (op == Op::Forward) {
        dim3 grid((unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock), (unsigned)a.nA);
        k_forward<VZ, OCC, ABS><<<grid, block, 0, st>>>(a);
    } else {
        dim3 grid((unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock));
        if (op == Op::BackwardRef) k_backward_ref<VZ, OCC, ABS><<<grid, block, 0, st>>>(a);
        else k_adjoint<VZ, OCC, ABS><<<grid, block, 0, st>>>(a);
    }
}

template <int VZ, bool OCC>
void launch_abs(Op op, int abs_mode, const Args& a, long items, cudaStream_t st) {
    switch (abs_mode) {
        case VAM_ABS_MASK: launch_one<VZ, OCC, VAM_ABS_MASK>(op, a, items, st); break;
        case VAM_ABS_RAY: launch_one<VZ, OCC, VAM_ABS_RAY>(op, a, items, st); break;
        default: launch_one<VZ, OCC, VAM_ABS_NONE>(op, a, items, st); break;
    }
}

// VZ of the fast forward for nZ slices (0 = use the generic kernel)
int fast_vz(int nZ, bool aligned) {
    if (!aligned || nZ % 4) return 0;
    auto eff = [&](int vz) {
        const int per = 32 * vz, ch = (nZ + per - 1) / per;
        return (double)nZ / (double)(ch * per);
    };
    if (eff(8) >= 0.74) return 8;
    if (eff(4) >= 0.74) return 4;
    return 0;
}

int run_forward_fast(vam_parallel_plan* plan, const float* in, float* out, cudaStream_t st, int vz) {
    const float* vol = in;
    if (plan->abs_mode == VAM_ABS_MASK) {
        const long npix = (long)plan->nY * plan->nX;
        const long n = npix * plan->nZ;
        k_mask_mul<<<(unsigned)std::min<long>((n + 255) / 256, 148L * 32), 256, 0, st>>>(in, plan->d_mask,
                                                                                         plan->d_vol_scratch, npix, plan->nZ);
        VAM_CHECK_LAUNCH("k_mask_mul");
        vol = plan->d_vol_scratch;
    }
    FastArgs a;
    a.vol = vol; a.sino = out; a.trig = plan->d_trig;
    a.nY = plan->nY; a.nX = plan->nX; a.nZ = plan->nZ; a.nA = plan->nA; a.C = plan->C;
    a.RS = plan->nX * plan->nZ;
    a.zchunks = (plan->nZ + 32 * vz - 1) / (32 * vz);
    a.even = (plan->nY % 2) == 0;
    a.alpha = plan->abs_alpha; a.R = plan->abs_R;
    const bool ray = plan->abs_mode == VAM_ABS_RAY;
    a.tasks = ray ? plan->d_tasks_single : plan->d_tasks_paired;
    const int ntask = ray ? plan->nA : plan->n_tasks_paired;
    const long items = (long)(plan->nX + 1) * a.zchunks;
    dim3 grid((unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock), (unsigned)ntask);
    dim3 block(kWarpsPerBlock * kWarp);
    if (vz == 8) {
        if (ray) k_forward_fast<8, true><<<grid, block, 0, st>>>(a);
        else k_forward_fast<8, false><<<grid, block, 0, st>>>(a);
    } else {
        if (ray) k_forward_fast<4, true><<<grid, block, 0, st>>>(a);
        else k_forward_fast<4, false><<<grid, block, 0, st>>>(a);
    }
    VAM_CHECK_LAUNCH("k_forward_fast");
    return VAM_OK;
}

int run(vam_parallel_plan* plan, Op op, const float* in, float* out, cudaStream_t st, const char* name) {
    VAM_REQUIRE(plan && in && out, VAM_ERR_ARG, std::string(name) + ": null argument");
    DeviceGuard g(plan->device);
    VAM_REQUIRE(g.ok, VAM_ERR_CUDA, std::string(name) + ": cannot select device");
    int vzf = fast_vz(plan->nZ, (((uintptr_t)in | (uintptr_t)out) & 31) == 0);
    if (vzf) {  // tuned vector width (4 or 8 slices per lane), when it fits the slice count
        const int want = op == Op::Forward ? plan->tune_fwd_vz : (op == Op::BackwardRef ? plan->tune_bwd_vz : plan->tune_adj_vz);
        if (want == 4 || (want == 8 && fast_vz(plan->nZ, true) == 8)) vzf = want;
    }
    if (op == Op::Forward && !plan->has_occ && (long)plan->nY * plan->nX * plan->nZ < (1L << 31) && vzf)
        return run_forward_fast(plan, in, out, st, vzf);
    if (op != Op::Forward && !plan->has_occ && vzf) {
        Args a;
        std::memset(&a, 0, sizeof(a));
        a.in = in; a.out = out; a.trig = plan->d_trig; a.circle = plan->d_circle;
        a.mask = plan->abs_mode == VAM_ABS_MASK ? plan->d_mask : nullptr;
        a.nY = plan->nY; a.nX = plan->nX; a.nZ = plan->nZ; a.nA = plan->nA; a.C = plan->C;
        a.zchunks = (plan->nZ + 32 * vzf - 1) / (32 * vzf);
        a.alpha = plan->abs_alpha; a.R = plan->abs_R;
        const long items = (long)plan->nY * plan->nX * a.zchunks;
        dim3 grid((unsigned)((items + kWarpsPerBlock - 1) / kWarpsPerBlock)), block(kWarpsPerBlock * kWarp);
        const bool ray = plan->abs_mode == VAM_ABS_RAY;
        if (op == Op::BackwardRef) {
            // the batched kernel stages cos / sin of every angle in shared memory (16 B per angle)
            const int batch = (size_t)plan->nA * sizeof(double2) <= 48 * 1024 ? plan->tune_bwd_batch : 1;
            if (batch >= 2) {
                const size_t smem = sizeof(double2) * plan->nA;
                if (vzf == 8) {
                    if (ray) k_backward_batched<8, 2, true><<<grid, block, smem, st>>>(a);
                    else k_backward_batched<8, 2, false><<<grid, block, smem, st>>>(a);
                } else if (batch >= 4) {
                    if (ray) k_backward_batched<4, 4, true><<<grid, block, smem, st>>>(a);
                    else k_backward_batched<4, 4, false><<<grid, block, smem, st>>>(a);
                } else {
                    if (ray) k_backward_batched<4, 2, true><<<grid, block, smem, st>>>(a);
                    else k_backward_batched<4, 2, false><<<grid, block, smem, st>>>(a);
                }
            } else if (vzf == 8) { if (ray) k_backward_fast<8, true><<<grid, block, 0, st>>>(a); else k_backward_fast<8, false><<<grid, block, 0, st>>>(a); }
            else { if (ray) k_backward_fast<4, true><<<grid, block, 0, st>>>(a); else k_backward_fast<4, false><<<grid, block, 0, st>>>(a); }
        } else if (plan->d_adj_table && plan->adj_table_abs == plan->abs_mode && plan->tune_adj_table) {
            if (vzf == 8) k_adjoint_table<8><<<grid, block, 0, st>>>(a, plan->d_adj_table);
            else k_adjoint_table<4><<<grid, block, 0, st>>>(a, plan->d_adj_table);
        } else {
            if (vzf == 8) { if (ray) k_adjoint_fast<8, true><<<grid, block, 0, st>>>(a); else k_adjoint_fast<8, false><<<grid, block, 0, st>>>(a); }
            else { if (ray) k_adjoint_fast<4, true><<<grid, block, 0, st>>>(a); else k_adjoint_fast<4, false><<<grid, block, 0, st>>>(a); }
        }
        VAM_CHECK_LAUNCH(name);
        return VAM_OK;
    }
    const bool aligned = (((uintptr_t)in | (uintptr_t)out) & 15) == 0;
    Layout L = choose_layout(plan->nZ, aligned);
    Args a;
    a.in = in; a.out = out; a.trig = plan->d_trig; a.circle = plan->d_circle;
    a.mask = plan->d_mask; a.occ = plan->d_occ; a.occ_flag = plan->d_occ_flag;
    a.nY = plan->nY; a.nX = plan->nX; a.nZ = plan->nZ; a.nA = plan->nA; a.C = plan->C;
    a.lz_shift = L.lz_shift; a.zvec = L.zvec; a.zchunks = L.zchunks;
    a.alpha = plan->abs_alpha; a.R = plan->abs_R;
    long items = (op == Op::Forward) ? (long)plan->nX * L.zchunks : (long)plan->nY * plan->nX * L.zchunks;
    const bool occ = plan->has_occ != 0;
    if (L.VZ == 4) {
        if (occ) launch_abs<4, true>(op, plan->abs_mode, a, items, st);
        else launch_abs<4, false>(op, plan->abs_mode, a, items, st);
    } else {
        if (occ) launch_abs<1, true>(op, plan->abs_mode, a, items, st);
        else launch_abs<1, false>(op, plan->abs_mode, a, items, st);
    }
    VAM_CHECK_LAUNCH(name);
    return VAM_OK;
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
    cudaFree(p->d_tasks_paired);
    cudaFree(p->d_tasks_single);
    cudaFree(p->d_vol_scratch);
    cudaFree(p->d_adj_table);
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
    return VAM_OK;
}

extern "C" int vam_parallel_clear_occlusion(vam_parallel_plan* p) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_parallel_clear_occlusion: null plan");
    p->has_occ = 0;
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
    auto vz_ok = [](int v) { return v == 0 || v == 4 || v == 8; };
    VAM_REQUIRE(vz_ok(t->forward_vz) && vz_ok(t->backward_vz) && vz_ok(t->adjoint_vz), VAM_ERR_ARG,
                "vam_parallel_set_tuning: vector widths must be 0 (auto), 4 or 8");
    VAM_REQUIRE(t->backward_batch == 0 || t->backward_batch == 1 || t->backward_batch == 2 || t->backward_batch == 4,
                VAM_ERR_ARG, "vam_parallel_set_tuning: backward_batch must be 0 (auto), 1, 2 or 4");
    p->tune_fwd_vz = t->forward_vz;
    p->tune_bwd_vz = t->backward_vz;
    p->tune_adj_vz = t->adjoint_vz;
    p->tune_bwd_batch = t->backward_batch == 0 ? 2 : t->backward_batch;
    p->tune_adj_table = t->adjoint_table;
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

extern "C" int vam_parallel_forward(vam_parallel_plan* p, const float* vol, float* sino, vam_stream_t stream) {
    clear_error();
    return run(p, Op::Forward, vol, sino, (cudaStream_t)stream, "vam_parallel_forward");
}

extern "C" int vam_parallel_backward_ref(vam_parallel_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    return run(p, Op::BackwardRef, sino, vol, (cudaStream_t)stream, "vam_parallel_backward_ref");
}

extern "C" int vam_parallel_adjoint(vam_parallel_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    return run(p, Op::Adjoint, sino, vol, (cudaStream_t)stream, "vam_parallel_adjoint");
}
