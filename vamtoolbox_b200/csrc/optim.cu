// optim.cu -- fused bodies of the optimizer iterations (vamtoolbox/optimizer/*.py).
//
// Every reduction is a fixed two-level tree (per-block partials in the caller's
// workspace, then one block), so results are deterministic run to run and no
// value ever returns to the host: scalars such as max(x) or the BCLP loss stay
// in device memory and the consuming kernel reads them, which keeps a whole
// optimizer iteration capturable in one CUDA graph.
#include <float.h>
#include <math.h>

#include <cmath>
#include <mutex>
#include <string>

#include <initializer_list>

#include "vam_internal.cuh"

namespace vam {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1184;    // 148 SMs x 8
constexpr int kStats = 9;
constexpr size_t kWorkBytes = (size_t)kMaxBlocks * kStats * sizeof(double) + 1024;

// every non-null pointer 16-byte aligned (vector loads allowed)
bool aligned16(std::initializer_list<const void*> ptrs) {
    for (const void* q : ptrs)
        if (q && ((uintptr_t)q & 15)) return false;
    return true;
}

int blocks_for(int64_t n) {
    int64_t b = (n + (int64_t)kThreads * 8 - 1) / ((int64_t)kThreads * 8);
    if (b < 1) b = 1;
    if (b > kMaxBlocks) b = kMaxBlocks;
    return (int)b;
}

template <typename T, int OP>
__device__ __forceinline__ T red_op(T a, T b) {
    // NaN propagates like np.max / np.min: a NaN operand wins
    if (OP == VAM_RED_MAX) return (b != b) ? b : ((a > b || a != a) ? a : b);
    if (OP == VAM_RED_MIN) return (b != b) ? b : ((a < b || a != a) ? a : b);
    return a + b;
}

template <typename T, int OP>
__device__ __forceinline__ T red_identity() {
    if (OP == VAM_RED_MAX) return (T)-INFINITY;
    if (OP == VAM_RED_MIN) return (T)INFINITY;
    return (T)0;
}

// Block-wide reduction of one value per thread; result valid in thread 0.
template <typename T, int OP>
__device__ T block_reduce(T v) {
    __shared__ T sh[kThreads / 32];
    for (int off = 16; off > 0; off >>= 1) v = red_op<T, OP>(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? sh[l] : red_identity<T, OP>();
        for (int off = 16; off > 0; off >>= 1) v = red_op<T, OP>(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

// ---------------------------------------------------------------------------
// generic reduce
// ---------------------------------------------------------------------------
template <int OP>
__global__ void __launch_bounds__(kThreads) k_reduce_partial(const float* __restrict__ x, int64_t n,
                                                             double* __restrict__ part) {
    double acc = red_identity<double, OP>();
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads)
        acc = red_op<double, OP>(acc, (double)x[i]);
    acc = block_reduce<double, OP>(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

template <int OP>
__global__ void __launch_bounds__(kThreads) k_reduce_final(const double* __restrict__ part, int nb,
                                                           float* __restrict__ out) {
    double acc = red_identity<double, OP>();
    for (int i = threadIdx.x; i < nb; i += kThreads) acc = red_op<double, OP>(acc, part[i]);
    acc = block_reduce<double, OP>(acc);
    if (threadIdx.x == 0) out[0] = (float)acc;
}

// ---------------------------------------------------------------------------
// VER (metrics.py:47-76): min over gel, then count void >= min
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_ver_min(const float* __restrict__ x, const uint8_t* __restrict__ m,
                                                      int64_t n, double* __restrict__ part) {
    double mn = INFINITY;
    double cnt = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const uint8_t t = m[i];
        if (t == 1) mn = fmin(mn, (double)x[i]);
        cnt += (t != 0);
    }
    mn = block_reduce<double, VAM_RED_MIN>(mn);
    cnt = block_reduce<double, VAM_RED_SUM>(cnt);
    if (threadIdx.x == 0) { part[blockIdx.x] = mn; part[kMaxBlocks + blockIdx.x] = cnt; }
}

__global__ void __launch_bounds__(kThreads) k_ver_min_final(double* __restrict__ part, int nb) {
    double mn = INFINITY, cnt = 0.0;
    for (int i = threadIdx.x; i < nb; i += kThreads) { mn = fmin(mn, part[i]); cnt += part[kMaxBlocks + i]; }
    mn = block_reduce<double, VAM_RED_MIN>(mn);
    cnt = block_reduce<double, VAM_RED_SUM>(cnt);
    if (threadIdx.x == 0) { part[2 * kMaxBlocks] = mn; part[2 * kMaxBlocks + 1] = cnt; }
}

__global__ void __launch_bounds__(kThreads) k_ver_count(const float* __restrict__ x, const uint8_t* __restrict__ m,
                                                        int64_t n, double* __restrict__ part) {
    const float mn = (float)part[2 * kMaxBlocks];
    double cnt = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads)
        cnt += (m[i] == 2 && x[i] >= mn);
    cnt = block_reduce<double, VAM_RED_SUM>(cnt);
    if (threadIdx.x == 0) part[blockIdx.x] = cnt;
}

__global__ void __launch_bounds__(kThreads) k_ver_final(const double* __restrict__ part, int nb, float* __restrict__ out) {
    double cnt = 0.0;
    for (int i = threadIdx.x; i < nb; i += kThreads) cnt += part[i];
    cnt = block_reduce<double, VAM_RED_SUM>(cnt);
    if (threadIdx.x == 0) out[0] = (float)(cnt / part[2 * kMaxBlocks + 1]);
}

// ---------------------------------------------------------------------------
// IPDR (metrics.py:130-156): max - min over gel voxels
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_ipdr_partial(const float* __restrict__ x, const uint8_t* __restrict__ m,
                                                           int64_t n, double* __restrict__ part) {
    double mn = INFINITY, mx = -INFINITY;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        if (m[i] == 1) {
            const double v = (double)x[i];
            mn = fmin(mn, v);
            mx = fmax(mx, v);
        }
    }
    mn = block_reduce<double, VAM_RED_MIN>(mn);
    mx = block_reduce<double, VAM_RED_MAX>(mx);
    if (threadIdx.x == 0) { part[blockIdx.x] = mn; part[kMaxBlocks + blockIdx.x] = mx; }
}

__global__ void __launch_bounds__(kThreads) k_ipdr_final(const double* __restrict__ part, int nb, float* __restrict__ out) {
    double mn = INFINITY, mx = -INFINITY;
    for (int i = threadIdx.x; i < nb; i += kThreads) { mn = fmin(mn, part[i]); mx = fmax(mx, part[kMaxBlocks + i]); }
    mn = block_reduce<double, VAM_RED_MIN>(mn);
    mx = block_reduce<double, VAM_RED_MAX>(mx);
    if (threadIdx.x == 0) out[0] = (mn <= mx) ? (float)(mx - mn) : __int_as_float(0x7fc00000);
}

// ---------------------------------------------------------------------------
// BCLP dose pass (BCLP.py:293-437)
// ---------------------------------------------------------------------------
struct TableRef {
    const float* f;
    const float* m;
    const float* dm;
    int n;
    float f0, inv_step;
    int kind;                            // vam_response_kind
    double A, K, B, M, nu, C;            // closed-form parameters
};

// np.interp(d, f, y, left=y[0], right=y[-1]) on a uniformly spaced table
__device__ __forceinline__ void table_interp(const TableRef& t, float d, float& out_m, float& out_dm) {
    if (!(d > t.f[0])) {
        if (d == t.f[0] || !(d == d)) { out_m = d == d ? t.m[0] : d; out_dm = d == d ? t.dm[0] : d; return; }
        out_m = t.m[0]; out_dm = t.dm[0]; return;
    }
    if (!(d < t.f[t.n - 1])) { out_m = t.m[t.n - 1]; out_dm = t.dm[t.n - 1]; return; }
    int j = (int)((d - t.f0) * t.inv_step);
    j = min(max(j, 0), t.n - 2);
    while (j > 0 && t.f[j] > d) --j;
    while (j < t.n - 2 && t.f[j + 1] <= d) ++j;
    const float fj = t.f[j], fj1 = t.f[j + 1];
    if (fj == d) { out_m = t.m[j]; out_dm = t.dm[j]; return; }
    const float w = (d - fj) / (fj1 - fj);
    out_m = fmaf(w, t.m[j + 1] - t.m[j], t.m[j]);
    out_dm = fmaf(w, t.dm[j + 1] - t.dm[j], t.dm[j]);
}

// Closed-form response models in float64, in the reference's operation order
// (response.py:191-218 _map_glf / _dmapdf_glf, :239-250 linear, :252-262 identity).
// TABLE: the kernel instance for interpolation tables (no closed-form code, whose float64 registers
// would lower the table instance's occupancy); otherwise the kind is read from t at run time.
template <bool TABLE>
__device__ __forceinline__ void response_eval(const TableRef& t, float d, float& out_m, float& out_dm) {
    if (TABLE || t.kind == VAM_RESP_TABLE) {
        table_interp(t, d, out_m, out_dm);
        return;
    }
    if (t.kind == VAM_RESP_LINEAR) {
        out_m = (float)(t.M * (double)d + t.C);
        out_dm = (float)t.M;
        return;
    }
    if (t.kind == VAM_RESP_IDENTITY) {
        out_m = d;
        out_dm = 1.f;
        return;
    }
    const double e = exp(-t.B * ((double)d - t.M));
    const double onep = 1.0 + e;
    const double m = t.A + (t.K - t.A) / (t.nu == 1.0 ? onep : pow(onep, 1.0 / t.nu));
    const double c1 = t.nu == 1.0 ? 1.0 / (t.K - t.A) : pow(1.0 / (t.K - t.A), t.nu);
    const double y = m - t.A;
    const double c3 = t.nu == 1.0 ? y * y : pow(y, t.nu + 1.0);
    out_m = (float)m;
    out_dm = (float)(c1 * (t.B / t.nu) * c3 * e);
}

__device__ __forceinline__ float powabs(float a, float p) {
    if (p == 2.f) return a * a;
    if (p == 1.f) return a;
    if (p == 4.f) { float b = a * a; return b * b; }
    if (p == 3.f) return a * a * a;
    if (p == 0.f) return 1.f;
    return powf(a, p);
}

// Running sums of the BCLP loss / norm statistics (BCLP.py:277-346, 401-410).
struct DoseStats {
    double loss = 0, l0 = 0, l0e = 0, l1 = 0, l1e = 0, l2 = 0, l2e = 0, lf = 0, lfe = 0;
};

// One voxel of the fused dose pass: response, band error, gradient operand, statistics.
template <bool TABLE>
__device__ __forceinline__ void dose_voxel(const TableRef& tab, float d, float tgt, float ep, float w, float p,
                                           float& mp, float& op, DoseStats& S) {
    float dmp;
    response_eval<TABLE>(tab, d, mp, dmp);
    const float e = mp - tgt;
    const float ae = fabsf(e);
    const float eb = ae - ep;
    const bool v = eb > 0.f;
    const float aeb = fabsf(eb);
    op = 0.f;
    if (v) {
        const float sgn = (e > 0.f) ? 1.f : ((e < 0.f) ? -1.f : 0.f);
        op = w * powabs(aeb, p - 1.f) * sgn * dmp;
        S.loss += (double)(w * powabs(aeb, p));
        S.l0 += 1.0;
        S.l1 += aeb;
        S.l2 += (double)eb * eb;
        S.lf = fmax(S.lf, (double)aeb);
    }
    S.l0e += (ae > 0.f);
    S.l1e += ae;
    S.l2e += (double)e * e;
    if (ae > 0.f) S.lfe = fmax(S.lfe, (double)ae);
}

// vec: all arrays 16-byte aligned, so each thread takes four consecutive voxels per
// iteration with 16-byte loads (four independent loads in flight instead of one
// dependent chain at a time); the remaining n % 4 voxels go element by element.
template <bool TABLE>
__global__ void __launch_bounds__(kThreads) k_bclp_dose(const float* __restrict__ dose, const float* __restrict__ target,
                                                        int64_t n, TableRef tab, float eps, float weight, float p,
                                                        const float* __restrict__ eps_arr,
                                                        const float* __restrict__ w_arr, float* __restrict__ mapped,
                                                        float* __restrict__ operand, double* __restrict__ part, int vec) {
    DoseStats S;
    const int64_t stride = (int64_t)gridDim.x * kThreads;
    const int64_t t0 = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    const int64_t n4 = vec ? n / 4 : 0;
    for (int64_t i4 = t0; i4 < n4; i4 += stride) {
        const float4 d4 = __ldg(reinterpret_cast<const float4*>(dose) + i4);
        const float4 g4 = __ldg(reinterpret_cast<const float4*>(target) + i4);
        const float4 e4 = eps_arr ? __ldg(reinterpret_cast<const float4*>(eps_arr) + i4) : make_float4(eps, eps, eps, eps);
        const float4 w4 = w_arr ? __ldg(reinterpret_cast<const float4*>(w_arr) + i4)
                                : make_float4(weight, weight, weight, weight);
        float4 m4, o4;
        dose_voxel<TABLE>(tab, d4.x, g4.x, e4.x, w4.x, p, m4.x, o4.x, S);
        dose_voxel<TABLE>(tab, d4.y, g4.y, e4.y, w4.y, p, m4.y, o4.y, S);
        dose_voxel<TABLE>(tab, d4.z, g4.z, e4.z, w4.z, p, m4.z, o4.z, S);
        dose_voxel<TABLE>(tab, d4.w, g4.w, e4.w, w4.w, p, m4.w, o4.w, S);
        if (mapped) reinterpret_cast<float4*>(mapped)[i4] = m4;
        reinterpret_cast<float4*>(operand)[i4] = o4;
    }
    for (int64_t i = 4 * n4 + t0; i < n; i += stride) {
        float mp, op;
        dose_voxel<TABLE>(tab, dose[i], target[i], eps_arr ? eps_arr[i] : eps, w_arr ? w_arr[i] : weight, p, mp, op, S);
        if (mapped) mapped[i] = mp;
        operand[i] = op;
    }
    double vals[kStats] = {S.loss, S.l0, S.l0e, S.l1, S.l1e, S.l2, S.l2e, S.lf, S.lfe};
#pragma unroll
    for (int k = 0; k < kStats; ++k) {
        double r = (k >= 7) ? block_reduce<double, VAM_RED_MAX>(vals[k]) : block_reduce<double, VAM_RED_SUM>(vals[k]);
        if (threadIdx.x == 0) part[(size_t)k * kMaxBlocks + blockIdx.x] = r;
    }
}

__global__ void __launch_bounds__(kThreads) k_bclp_stats_final(const double* __restrict__ part, int nb,
                                                               float* __restrict__ stats) {
#pragma unroll
    for (int k = 0; k < kStats; ++k) {
        double acc = (k >= 7) ? 0.0 : 0.0;
        for (int i = threadIdx.x; i < nb; i += kThreads) {
            const double v = part[(size_t)k * kMaxBlocks + i];
            acc = (k >= 7) ? fmax(acc, v) : acc + v;
        }
        acc = (k >= 7) ? block_reduce<double, VAM_RED_MAX>(acc) : block_reduce<double, VAM_RED_SUM>(acc);
        if (threadIdx.x == 0) stats[k] = (float)acc;
    }
}

// g = clip(g - lr * pref * grad, lo, hi); pref from the device loss (BCLP.py:370-375)
__global__ void __launch_bounds__(kThreads) k_bclp_update(float* __restrict__ g, const float* __restrict__ grad,
                                                          int64_t n, float lr, float p, float q, float lo, float hi,
                                                          int has_hi, const float* __restrict__ stats, int vec) {
    const double S = (double)stats[0];
    const double L = pow(S, (double)q / (double)p);
    const float pref = (L != 0.0) ? (float)((double)q * pow(L, ((double)q - (double)p) / (double)q)) : 1.f;
    const float step = lr * pref;
    const float hv = has_hi ? hi : INFINITY;
    const int64_t stride = (int64_t)gridDim.x * kThreads;
    const int64_t t0 = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    const int64_t n4 = vec ? n / 4 : 0;  // 16-byte aligned: four values per thread and load
    for (int64_t i4 = t0; i4 < n4; i4 += stride) {
        float4 v = reinterpret_cast<const float4*>(g)[i4];
        const float4 d = __ldg(reinterpret_cast<const float4*>(grad) + i4);
        v.x = fminf(fmaxf(v.x - step * d.x, lo), hv);
        v.y = fminf(fmaxf(v.y - step * d.y, lo), hv);
        v.z = fminf(fmaxf(v.z - step * d.z, lo), hv);
        v.w = fminf(fmaxf(v.w - step * d.w, lo), hv);
        reinterpret_cast<float4*>(g)[i4] = v;
    }
    for (int64_t i = 4 * n4 + t0; i < n; i += stride) {
        float v = g[i] - step * grad[i];
        v = fmaxf(v, lo);
        if (has_hi) v = fminf(v, hi);
        g[i] = v;
    }
}

// ---------------------------------------------------------------------------
// CAL / OSMO helpers
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_cal_threshold(const float* __restrict__ x, const float* __restrict__ xmax,
                                                            const float* __restrict__ t, int64_t n, float d_h, float g,
                                                            float* __restrict__ out) {
    const float inv = 1.f / xmax[0];
    const float ig = 1.f / g;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const float y = x[i] * inv - d_h;
        out[i] = 1.f / (1.f + expf(-y * ig)) - t[i];
    }
}

__global__ void __launch_bounds__(kThreads) k_cal_update(float* __restrict__ b, const float* __restrict__ db,
                                                         const float* __restrict__ dbp, int64_t n, float lr, float m,
                                                         float mscale) {
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const float grad = db[i] * (1.f - m) + (dbp ? dbp[i] * mscale : 0.f);
        b[i] = fmaxf(b[i] - lr * grad, 0.f);
    }
}

__global__ void __launch_bounds__(kThreads) k_scale(float* __restrict__ x, const float* __restrict__ s, int64_t n,
                                                    int floor_on, float floor_val) {
    const float inv = 1.f / s[0];
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        float v = x[i] * inv;
        if (floor_on) v = fmaxf(v, floor_val);
        x[i] = v;
    }
}

__global__ void __launch_bounds__(kThreads) k_osmo_model(float* __restrict__ xm, const float* __restrict__ x,
                                                         const float* __restrict__ xmax, const uint8_t* __restrict__ m,
                                                         int64_t n, int gel, float d) {
    const float inv = xmax ? 1.f / xmax[0] : 1.f;
    const uint8_t sel = gel ? 1 : 2;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        if (m[i] != sel) continue;
        const float xv = x[i] * inv;
        if (gel) xm[i] += fmaxf(d - xv, 0.f);
        else xm[i] -= fmaxf(xv - d, 0.f);
    }
}

__global__ void k_append(const float* __restrict__ src, int n, float* __restrict__ arr, int* __restrict__ counter,
                         int cap) {
    const int row = counter[0];
    if (row < cap)
        for (int i = threadIdx.x; i < n; i += blockDim.x) arr[(size_t)row * n + i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) counter[0] = row + 1;
}

}  // namespace
}  // namespace vam

using namespace vam;

extern "C" int vam_append(const float* src, int32_t n, float* arr, int32_t* counter, int32_t cap, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(src && arr && counter, VAM_ERR_ARG, "vam_append: null argument");
    VAM_REQUIRE(n > 0 && cap > 0, VAM_ERR_SHAPE, "vam_append: n and cap_rows must be positive");
    k_append<<<1, 32, 0, (cudaStream_t)stream>>>(src, n, arr, counter, cap);
    VAM_CHECK_LAUNCH("vam_append");
    return VAM_OK;
}

extern "C" size_t vam_reduce_workspace_bytes(int64_t n) {
    (void)n;
    return kWorkBytes;
}

extern "C" int vam_reduce(const float* x, int64_t n, int op, float* out, void* work, size_t work_bytes,
                          vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && out && work, VAM_ERR_ARG, "vam_reduce: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_reduce: empty input");
    VAM_REQUIRE(work_bytes >= kWorkBytes, VAM_ERR_ARG, "vam_reduce: workspace too small");
    const int nb = blocks_for(n);
    cudaStream_t st = (cudaStream_t)stream;
    double* part = (double*)work;
    switch (op) {
        case VAM_RED_MAX:
            k_reduce_partial<VAM_RED_MAX><<<nb, kThreads, 0, st>>>(x, n, part);
            k_reduce_final<VAM_RED_MAX><<<1, kThreads, 0, st>>>(part, nb, out);
            break;
        case VAM_RED_MIN:
            k_reduce_partial<VAM_RED_MIN><<<nb, kThreads, 0, st>>>(x, n, part);
            k_reduce_final<VAM_RED_MIN><<<1, kThreads, 0, st>>>(part, nb, out);
            break;
        case VAM_RED_SUM:
            k_reduce_partial<VAM_RED_SUM><<<nb, kThreads, 0, st>>>(x, n, part);
            k_reduce_final<VAM_RED_SUM><<<1, kThreads, 0, st>>>(part, nb, out);
            break;
        default:
            return set_error(VAM_ERR_ARG, "vam_reduce: unknown op");
    }
    VAM_CHECK_LAUNCH("vam_reduce");
    return VAM_OK;
}

// ---------------------------------------------------------------------------
// Sinogram filter (util/data.py:302-370) around cuFFT's real transforms along the
// detector axis: the half spectrum times the real filter, and the epilogue that
// crops the padded inverse transform, scales, clips and converts to float32.
// ---------------------------------------------------------------------------
namespace vam {
namespace {

// X[k][m] *= h[k], X complex128 [nk][m] (row k = frequency k of every column)
__global__ void __launch_bounds__(kThreads) k_spectrum_scale(double2* __restrict__ X, const double* __restrict__ h,
                                                             int64_t m) {
    const double hk = h[blockIdx.y];
    double2* row = X + (int64_t)blockIdx.y * m;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < m; i += (int64_t)gridDim.x * kThreads) {
        double2 v = row[i];
        v.x *= hk;
        v.y *= hk;
        row[i] = v;
    }
}

// out[r][m] = clip(scale * y[r][m], lo, hi) as float32, rows r < n_rows of y [>= n_rows][m]
__global__ void __launch_bounds__(kThreads) k_filter_epilogue(const double* __restrict__ y, int64_t n, double scale,
                                                              int has_lo, double lo, int has_hi, double hi,
                                                              float* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        double v = y[i] * scale;
        if (has_lo) v = fmax(v, lo);
        if (has_hi) v = fmin(v, hi);
        out[i] = (float)v;
    }
}

}  // namespace
}  // namespace vam

extern "C" int vam_spectrum_scale(void* spectrum, const double* filter, int64_t n_freq, int64_t m, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(spectrum && filter, VAM_ERR_ARG, "vam_spectrum_scale: null argument");
    VAM_REQUIRE(n_freq > 0 && m > 0 && n_freq < 65536, VAM_ERR_SHAPE, "vam_spectrum_scale: 0 < n_freq < 65536, m > 0");
    const int64_t bx = std::min<int64_t>((m + kThreads - 1) / kThreads, 1024);
    k_spectrum_scale<<<dim3((unsigned)bx, (unsigned)n_freq), kThreads, 0, (cudaStream_t)stream>>>(
        static_cast<double2*>(spectrum), filter, m);
    VAM_CHECK_LAUNCH("vam_spectrum_scale");
    return VAM_OK;
}

extern "C" int vam_filter_epilogue(const double* y, int64_t n_rows, int64_t m, double scale, int has_lo, double lo,
                                   int has_hi, double hi, float* out, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(y && out, VAM_ERR_ARG, "vam_filter_epilogue: null argument");
    VAM_REQUIRE(n_rows > 0 && m > 0, VAM_ERR_SHAPE, "vam_filter_epilogue: empty input");
    const int64_t n = n_rows * m;
    k_filter_epilogue<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(y, n, scale, has_lo, lo, has_hi, hi, out);
    VAM_CHECK_LAUNCH("vam_filter_epilogue");
    return VAM_OK;
}

// ---------------------------------------------------------------------------
// No-allocation reduction: scratch in a static device array
// ---------------------------------------------------------------------------
namespace vam {
namespace {
constexpr int kNoAllocMaxBlocks = 4096;                       // 32 KiB of partials
constexpr int64_t kNoAllocPerBlock = (int64_t)kThreads * 8;  // inputs per partial
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks];

std::mutex g_noalloc_mu;
double* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_partials on the current device.  In host code
// the symbol is only a host-side stand-in, never a device pointer, so the
// address is looked up once per device and cached.  The same first call also
// loads the six reduction kernels this entry point launches (CUDA loads
// kernels lazily, on first use), so no later call of any op loads a module.
int noalloc_scratch(double** out) {
    int dev = -1;
    VAM_TRY_CUDA(cudaGetDevice(&dev));
    VAM_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, VAM_ERR_ARG, "vam_reduce_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            return set_error(VAM_ERR_CUDA, std::string("vam_reduce_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        const void* kernels[] = {(const void*)k_reduce_partial<VAM_RED_MAX>, (const void*)k_reduce_final<VAM_RED_MAX>,
                                 (const void*)k_reduce_partial<VAM_RED_MIN>, (const void*)k_reduce_final<VAM_RED_MIN>,
                                 (const void*)k_reduce_partial<VAM_RED_SUM>, (const void*)k_reduce_final<VAM_RED_SUM>};
        for (const void* k : kernels) {
            cudaFuncAttributes fa;
            e = cudaFuncGetAttributes(&fa, k);
            if (e != cudaSuccess)
                return set_error(VAM_ERR_CUDA, std::string("vam_reduce_noalloc: loading its kernels: ") + cudaGetErrorString(e));
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return VAM_OK;
}
}  // namespace
}  // namespace vam

extern "C" int vam_reduce_noalloc(const float* x, int64_t n, int op, float* out, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && out, VAM_ERR_ARG, "vam_reduce_noalloc: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_reduce_noalloc: empty input");
    VAM_REQUIRE(op == VAM_RED_MAX || op == VAM_RED_MIN || op == VAM_RED_SUM, VAM_ERR_ARG, "vam_reduce_noalloc: unknown op");
    const int64_t nb64 = (n + kNoAllocPerBlock - 1) / kNoAllocPerBlock;
    VAM_REQUIRE(nb64 <= kNoAllocMaxBlocks, VAM_ERR_SHAPE,
                "vam_reduce_noalloc: n = " + std::to_string((long long)n) + " exceeds the maximum of " +
                    std::to_string((long long)kNoAllocMaxBlocks * kNoAllocPerBlock) + " elements (static scratch of " +
                    std::to_string(kNoAllocMaxBlocks) + " partials)");
    double* part = nullptr;
    int rc = noalloc_scratch(&part);
    if (rc != VAM_OK) return rc;
    const int nb = (int)nb64;
    cudaStream_t st = (cudaStream_t)stream;
    switch (op) {
        case VAM_RED_MAX:
            k_reduce_partial<VAM_RED_MAX><<<nb, kThreads, 0, st>>>(x, n, part);
            k_reduce_final<VAM_RED_MAX><<<1, kThreads, 0, st>>>(part, nb, out);
            break;
        case VAM_RED_MIN:
            k_reduce_partial<VAM_RED_MIN><<<nb, kThreads, 0, st>>>(x, n, part);
            k_reduce_final<VAM_RED_MIN><<<1, kThreads, 0, st>>>(part, nb, out);
            break;
        default:
            k_reduce_partial<VAM_RED_SUM><<<nb, kThreads, 0, st>>>(x, n, part);
            k_reduce_final<VAM_RED_SUM><<<1, kThreads, 0, st>>>(part, nb, out);
            break;
    }
    VAM_CHECK_LAUNCH("vam_reduce_noalloc");
    return VAM_OK;
}

extern "C" int vam_metric_ipdr(const float* x, const uint8_t* mask, int64_t n, float* out, void* work,
                               size_t work_bytes, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && mask && out && work, VAM_ERR_ARG, "vam_metric_ipdr: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_metric_ipdr: empty input");
    VAM_REQUIRE(work_bytes >= kWorkBytes, VAM_ERR_ARG, "vam_metric_ipdr: workspace too small");
    const int nb = blocks_for(n);
    cudaStream_t st = (cudaStream_t)stream;
    double* part = (double*)work;
    k_ipdr_partial<<<nb, kThreads, 0, st>>>(x, mask, n, part);
    k_ipdr_final<<<1, kThreads, 0, st>>>(part, nb, out);
    VAM_CHECK_LAUNCH("vam_metric_ipdr");
    return VAM_OK;
}

extern "C" int vam_metric_ver(const float* x, const uint8_t* mask, int64_t n, float* out, void* work,
                              size_t work_bytes, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && mask && out && work, VAM_ERR_ARG, "vam_metric_ver: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_metric_ver: empty input");
    VAM_REQUIRE(work_bytes >= kWorkBytes, VAM_ERR_ARG, "vam_metric_ver: workspace too small");
    const int nb = blocks_for(n);
    cudaStream_t st = (cudaStream_t)stream;
    double* part = (double*)work;
    k_ver_min<<<nb, kThreads, 0, st>>>(x, mask, n, part);
    k_ver_min_final<<<1, kThreads, 0, st>>>(part, nb);
    k_ver_count<<<nb, kThreads, 0, st>>>(x, mask, n, part);
    k_ver_final<<<1, kThreads, 0, st>>>(part, nb, out);
    VAM_CHECK_LAUNCH("vam_metric_ver");
    return VAM_OK;
}

extern "C" int vam_bclp_dose_pass(const float* dose, const float* target, int64_t n, const vam_bclp_params* prm,
                                  float* mapped, float* operand, float* stats, void* work, size_t work_bytes,
                                  vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(dose && target && prm && operand && stats && work, VAM_ERR_ARG, "vam_bclp_dose_pass: null argument");
    VAM_REQUIRE(prm->response >= VAM_RESP_TABLE && prm->response <= VAM_RESP_IDENTITY, VAM_ERR_ARG,
                "vam_bclp_dose_pass: unknown response kind");
    VAM_REQUIRE(prm->response != VAM_RESP_TABLE ||
                    (prm->table_f && prm->table_map && prm->table_dmap && prm->n_table >= 2),
                VAM_ERR_ARG, "vam_bclp_dose_pass: response table needs >= 2 points");
    VAM_REQUIRE(prm->response != VAM_RESP_GLF || (prm->resp_K != prm->resp_A && prm->resp_nu != 0.0),
                VAM_ERR_ARG, "vam_bclp_dose_pass: generalised logistic needs K != A and nu != 0");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_bclp_dose_pass: empty input");
    VAM_REQUIRE(work_bytes >= kWorkBytes, VAM_ERR_ARG, "vam_bclp_dose_pass: workspace too small");
    VAM_REQUIRE(std::isfinite(prm->p) && prm->p > 0.f, VAM_ERR_ARG, "vam_bclp_dose_pass: p must be > 0");
    // table_f0 / table_inv_step seed the bin search as if the table were uniform
    // (np.linspace); the search then walks to the bin against the table values
    // themselves, so any strictly increasing table gives np.interp's bin.
    TableRef t;
    t.f = prm->table_f; t.m = prm->table_map; t.dm = prm->table_dmap; t.n = prm->n_table;
    t.f0 = prm->table_f0; t.inv_step = prm->table_inv_step;
    t.kind = prm->response;
    t.A = prm->resp_A; t.K = prm->resp_K; t.B = prm->resp_B; t.M = prm->resp_M; t.nu = prm->resp_nu; t.C = prm->resp_C;
    const int nb = blocks_for(n);
    cudaStream_t st = (cudaStream_t)stream;
    double* part = (double*)work;
    const bool vec = aligned16({dose, target, prm->eps_dev, prm->weight_dev, mapped, operand});
    if (t.kind == VAM_RESP_TABLE)
        k_bclp_dose<true><<<nb, kThreads, 0, st>>>(dose, target, n, t, prm->eps, prm->weight, prm->p, prm->eps_dev,
                                         prm->weight_dev, mapped, operand, part, vec);
    else
        k_bclp_dose<false><<<nb, kThreads, 0, st>>>(dose, target, n, t, prm->eps, prm->weight, prm->p, prm->eps_dev,
                                         prm->weight_dev, mapped, operand, part, vec);
    k_bclp_stats_final<<<1, kThreads, 0, st>>>(part, nb, stats);
    VAM_CHECK_LAUNCH("vam_bclp_dose_pass");
    return VAM_OK;
}

extern "C" int vam_bclp_sino_update(float* g, const float* grad, int64_t n, float lr, float p, float q, float lo,
                                    float hi, int has_hi, const float* stats, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(g && grad && stats, VAM_ERR_ARG, "vam_bclp_sino_update: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_bclp_sino_update: empty input");
    k_bclp_update<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(g, grad, n, lr, p, q, lo, hi, has_hi, stats,
                                                                         aligned16({g, grad}));
    VAM_CHECK_LAUNCH("vam_bclp_sino_update");
    return VAM_OK;
}

extern "C" int vam_cal_threshold(const float* x, const float* xmax, const float* target, int64_t n, float d_h,
                                 float g, float* out, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && xmax && target && out, VAM_ERR_ARG, "vam_cal_threshold: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_cal_threshold: empty input");
    k_cal_threshold<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(x, xmax, target, n, d_h, g, out);
    VAM_CHECK_LAUNCH("vam_cal_threshold");
    return VAM_OK;
}

extern "C" int vam_cal_sino_update(float* b, const float* db, const float* db_prev, int64_t n, float lr,
                                   float momentum, int32_t iter, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(b && db, VAM_ERR_ARG, "vam_cal_sino_update: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_cal_sino_update: empty input");
    const double m = momentum;
    const float mscale = (float)(m / (1.0 - std::pow(m, (double)iter + 1.0)));
    k_cal_update<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(b, db, momentum != 0.f ? db_prev : nullptr, n,
                                                                       lr, momentum, mscale);
    VAM_CHECK_LAUNCH("vam_cal_sino_update");
    return VAM_OK;
}

extern "C" int vam_scale_by_device(float* x, const float* s, int64_t n, int apply_floor, float floor_val,
                                   vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && s, VAM_ERR_ARG, "vam_scale_by_device: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_scale_by_device: empty input");
    k_scale<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(x, s, n, apply_floor, floor_val);
    VAM_CHECK_LAUNCH("vam_scale_by_device");
    return VAM_OK;
}

extern "C" int vam_osmo_model_update(float* xm, const float* x, const float* xmax, const uint8_t* mask, int64_t n,
                                     int gel, float d, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(xm && x && mask, VAM_ERR_ARG, "vam_osmo_model_update: null argument");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_osmo_model_update: empty input");
    k_osmo_model<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(xm, x, xmax, mask, n, gel, d);
    VAM_CHECK_LAUNCH("vam_osmo_model_update");
    return VAM_OK;
}
