// output.cu -- output formats of the sm_100a core: sinogram -> projector
// frames (vamtoolbox/imagesequence.py:85-401) and fan-beam rebinning
// (vamtoolbox/geometry.py:736-944).
//
// All of this is HBM-bound gather / scatter work.  Sinograms are [nR][nA][nZ]
// with z fastest, so every kernel puts consecutive threads on consecutive z:
// loads and stores of a warp are contiguous runs.  Arithmetic that the
// reference does in float64 numpy is done in double with explicit _rn
// intrinsics (no FMA contraction), in the reference's operation order, so
// the results are the reference's to the last bit where the reference's own
// order is known (rebinning, quantisation) and within a few ulps where it
// sits inside a compiled third-party routine (scipy's order-1 rotate,
// OpenCV's bilinear resize).
#include "vam_internal.cuh"

#include <math.h>

#include <algorithm>

using vam::set_error;
using vam::clear_error;

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }

template <typename T> __device__ __forceinline__ double ld(const T* p) { return (double)__ldg(p); }

// ---------------------------------------------------------------------------
// Plane rotation: ndimage.rotate(sino, angle, axes=(0, 2), reshape=True,
// order=1) as called by _rotate (imagesequence.py:396-401).  For output
// (o0, o1) of every angle plane the source point is
//   c0 = (m00*o0 + off0) + m01*o1,  c1 = (m10*o0 + off1) + m11*o1
// (rot_matrix and offset of scipy.ndimage.rotate); a point with c0 outside
// [0, nR-1] or c1 outside [0, nZ-1] reads the constant 0 (mode='constant');
// otherwise the order-1 spline is sum_k (x_k * w0_k) * w1_k over the four
// corners (lo,lo), (lo,hi), (hi,lo), (hi,hi) with w = 1-t / t, t = c - floor(c).
// Computed in double, stored in T like scipy's output array of the input dtype.
// flip_r / flip_z mirror the input first (_invertU / _invertV, :358-365).
// ---------------------------------------------------------------------------
struct RotArgs {
    double m00, m01, m10, m11, off0, off1;
    int nR, nA, nZ, oR, oZ, flip_r, flip_z;
};

template <typename T>
__global__ void __launch_bounds__(kThreads) k_sino_rotate(const T* __restrict__ in, T* __restrict__ out,
                                                          const RotArgs p) {
    const int row = blockIdx.x;                 // o0 * nA + a
    const int o0 = row / p.nA, a = row - o0 * p.nA;
    for (int o1 = threadIdx.x; o1 < p.oZ; o1 += blockDim.x) {
    const double c0 = dadd(dadd(dmul(p.m00, (double)o0), p.off0), dmul(p.m01, (double)o1));
    const double c1 = dadd(dadd(dmul(p.m10, (double)o0), p.off1), dmul(p.m11, (double)o1));
    double v = 0.0;
    if (c0 >= 0.0 && c0 <= (double)(p.nR - 1) && c1 >= 0.0 && c1 <= (double)(p.nZ - 1)) {
        const double f0 = floor(c0), f1 = floor(c1);
        const double t0 = dsub(c0, f0), t1 = dsub(c1, f1);
        const double a0 = dsub(1.0, t0), a1 = dsub(1.0, t1);
        int i0 = (int)f0, i1 = (int)f1;
        int j0 = min(i0 + 1, p.nR - 1), j1 = min(i1 + 1, p.nZ - 1);
        if (p.flip_r) { i0 = p.nR - 1 - i0; j0 = p.nR - 1 - j0; }
        if (p.flip_z) { i1 = p.nZ - 1 - i1; j1 = p.nZ - 1 - j1; }
        const size_t s = (size_t)p.nA * p.nZ;
        const T* base = in + (size_t)a * p.nZ;
        const double x00 = ld(base + i0 * s + i1), x01 = ld(base + i0 * s + j1);
        const double x10 = ld(base + j0 * s + i1), x11 = ld(base + j0 * s + j1);
        v = dmul(dmul(x00, a0), a1);
        v = dadd(v, dmul(dmul(x01, a0), t1));
        v = dadd(v, dmul(dmul(x10, t0), a1));
        v = dadd(v, dmul(dmul(x11, t0), t1));
    }
    out[((size_t)o0 * p.nA + a) * p.oZ + o1] = (T)v;
    }
}

// ---------------------------------------------------------------------------
// Plane resize: cv2.resize(plane, (oZ, oR), interpolation=INTER_LINEAR) of
// every angle plane, as called by _scaleSize (imagesequence.py:368-378).
// Per axis: f = (d + 0.5) * scale - 0.5 in double, s = floor(f), f -= s;
// s < 0 -> (s, f) = (0, 0); s >= n-1 -> (s, f) = (n-1, 0); weights (1-f, f).
// The z axis (plane width) is interpolated first, then the r axis:
// out = r0*wr0 + r1*wr1 with r_k = x[k][s]*wz0 + x[k][s+1]*wz1.  float
// planes use float weights and float arithmetic, double planes double; the
// result is stored as double either way, because _scaleSize collects the
// resized planes in a float64 np.zeros array.
// ---------------------------------------------------------------------------
struct ResizeArgs {
    double scale_r, scale_z;
    int nR, nA, nZ, oR, oZ, flip_r, flip_z;
};

__device__ __forceinline__ void axis_tap(int d, double scale, int n, int& s0, int& s1, double& f) {
    double fx = dsub(dmul(dadd((double)d, 0.5), scale), 0.5);
    double fl = floor(fx);
    int s = (int)fl;
    fx = dsub(fx, fl);
    if (s < 0) { s = 0; fx = 0.0; }
    if (s >= n - 1) { s = n - 1; fx = 0.0; }
    s0 = s;
    s1 = min(s + 1, n - 1);
    f = fx;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_sino_resize(const T* __restrict__ in, double* __restrict__ out,
                                                          const ResizeArgs p) {
    const int row = blockIdx.x;                            // y * nA + a
    const int y = row / p.nA, a = row - y * p.nA;
    int sr0, sr1;
    double fr;
    axis_tap(y, p.scale_r, p.nR, sr0, sr1, fr);
    for (int x = threadIdx.x; x < p.oZ; x += blockDim.x) {   // output z
    int sz0, sz1;
    double fz;
    axis_tap(x, p.scale_z, p.nZ, sz0, sz1, fz);
    int r0 = sr0, r1 = sr1;
    if (p.flip_r) { r0 = p.nR - 1 - r0; r1 = p.nR - 1 - r1; }
    if (p.flip_z) { sz0 = p.nZ - 1 - sz0; sz1 = p.nZ - 1 - sz1; }
    const size_t s = (size_t)p.nA * p.nZ;
    const T* b0 = in + r0 * s + (size_t)a * p.nZ;
    const T* b1 = in + r1 * s + (size_t)a * p.nZ;
    double v;
    if constexpr (sizeof(T) == 8) {
        const double wz1 = fz, wz0 = dsub(1.0, fz), wr1 = fr, wr0 = dsub(1.0, fr);
        const double q0 = dadd(dmul(b0[sz0], wz0), dmul(b0[sz1], wz1));
        const double q1 = dadd(dmul(b1[sz0], wz0), dmul(b1[sz1], wz1));
        v = dadd(dmul(q0, wr0), dmul(q1, wr1));
    } else {
        const float wz1 = (float)fz, wz0 = __fsub_rn(1.0f, wz1), wr1 = (float)fr, wr0 = __fsub_rn(1.0f, wr1);
        const float q0 = fadd(fmul(__ldg(b0 + sz0), wz0), fmul(__ldg(b0 + sz1), wz1));
        const float q1 = fadd(fmul(__ldg(b1 + sz0), wz0), fmul(__ldg(b1 + sz1), wz1));
        v = (double)fadd(fmul(q0, wr0), fmul(q1, wr1));
    }
    out[((size_t)y * p.nA + a) * p.oZ + x] = v;
    }
}

// ---------------------------------------------------------------------------
// Two order statistics (the k0-th and k1-th smallest, k1 in {k0, k0+1}) for
// np.percentile(..., method='linear') (imagesequence.py:129-133; numpy's
// _quantile takes exactly these two sorted elements and blends them).
// MSB-first radix select over order-preserving integer keys, 11-bit digits:
// one histogram pass per digit (shared-memory histogram, warp-aggregated
// increments, merged into a global histogram), one single-warp scan that
// picks the digit holding rank k.  The second rank is the first key unless
// the first key's run ends at k0, then it is min{key > key0} (one pass).
// NaN keys sort last (numpy's order); any NaN makes both outputs NaN, as
// np.percentile returns NaN for inputs holding NaN.  -0.0 is keyed as +0.0.
// The state lives in the caller's workspace; nothing syncs the host.
// ---------------------------------------------------------------------------
constexpr int kDigitBits = 11;
constexpr int kBins = 1 << kDigitBits;

struct SelState {
    unsigned long long prefix;     // key bits fixed so far
    unsigned long long min_above;  // min key > key0 (second rank)
    unsigned long long nan_count;
    long long k;                   // rank left inside the prefix range
    long long less;                // keys below the prefix range
    long long eq;                  // keys in the bin picked last
    unsigned int hist[kBins];
};

__device__ __forceinline__ uint32_t key_of(float x) {
    if (x != x) return 0xFFFFFFFFu;
    uint32_t b = __float_as_uint(x);
    if (b == 0x80000000u) b = 0u;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ unsigned long long key_of(double x) {
    if (x != x) return ~0ull;
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    if (b == 0x8000000000000000ull) b = 0ull;
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ float value_of(uint32_t k, float) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
__device__ __forceinline__ double value_of(unsigned long long k, double) {
    return __longlong_as_double((long long)((k & 0x8000000000000000ull) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
}

__global__ void k_sel_init(SelState* st, long long k0) {
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) st->hist[i] = 0u;
    if (threadIdx.x == 0) {
        st->prefix = 0ull;
        st->min_above = ~0ull;
        st->nan_count = 0ull;
        st->k = k0;
        st->less = 0;
        st->eq = 0;
    }
}

// Histogram of digit [shift, shift+width) over the keys whose bits above
// shift+width equal the prefix's (all keys when hi_shift >= key bits).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_sel_hist(const T* __restrict__ x, long long n, SelState* st,
                                                       int shift, int width, int first) {
    using K = decltype(key_of(T()));
    constexpr int kKeyBits = 8 * sizeof(K);
    __shared__ unsigned int sh[kBins];
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    const int hi = shift + width;
    const K want = hi >= kKeyBits ? (K)0 : (K)(st->prefix >> hi);
    const K dmask = (K)((1u << width) - 1u);
    const int lane = threadIdx.x & 31;
    unsigned long long nans = 0;
    // each warp takes 128 consecutive keys per step (4 coalesced loads in
    // flight per lane); the step index is uniform across the warp, so every
    // __match_any_sync sees all 32 lanes
    const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp_id * 128; base < n; base += n_warps * 128) {
        T v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const long long i = base + k * 32 + lane;
            v[k] = i < n ? x[i] : (T)0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int bin = kBins;   // no bin
            if (base + k * 32 + lane < n) {
                if (first && v[k] != v[k]) ++nans;
                const K key = key_of(v[k]);
                const bool match = hi >= kKeyBits ? true : (K)(key >> hi) == want;
                if (match) bin = (int)((key >> shift) & dmask);
            }
            if (!__any_sync(0xFFFFFFFFu, bin < kBins)) continue;   // no lane inside the prefix range
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, bin);
            if (bin < kBins && lane == __ffs(peers) - 1) atomicAdd(&sh[bin], (unsigned)__popc(peers));
        }
    }
    if (first && nans) atomicAdd(&st->nan_count, nans);
    __syncthreads();
    for (int i = threadIdx.x; i < (1 << width); i += blockDim.x)
        if (sh[i]) atomicAdd(&st->hist[i], sh[i]);
}

// One block of kBins / 2 threads: pick the bin holding rank k, fold it into
// the prefix, clear the histogram.
constexpr int kScanThreads = kBins / 2;

__global__ void __launch_bounds__(kScanThreads) k_sel_scan(SelState* st, int shift, int width) {
    __shared__ long long warp_sum[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nb = 1 << width;
    const long long k = st->k;   // read by every thread before the owner rewrites it
    const long long c0 = 2 * t < nb ? st->hist[2 * t] : 0;
    const long long c1 = 2 * t + 1 < nb ? st->hist[2 * t + 1] : 0;
    const long long mine = c0 + c1;
    long long incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < kScanThreads / 32 ? warp_sum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += v;
        }
        if (lane < kScanThreads / 32) warp_sum[lane] = w;   // inclusive prefix over warps
    }
    __syncthreads();
    incl += warp > 0 ? warp_sum[warp - 1] : 0;
    const long long excl = incl - mine;
    if (k >= excl && k < incl) {   // exactly one thread owns rank k
        const int b = k < excl + c0 ? 2 * t : 2 * t + 1;
        const long long below = k < excl + c0 ? excl : excl + c0;
        st->k = k - below;
        st->less += below;
        st->eq = b == 2 * t ? c0 : c1;
        st->prefix |= (unsigned long long)b << shift;
    }
    __syncthreads();
    if (2 * t < kBins) st->hist[2 * t] = 0u;
    if (2 * t + 1 < kBins) st->hist[2 * t + 1] = 0u;
}

// Second rank (k1 = k0 + 1) when it lies past the run of key0: min{key > key0}.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_sel_min_above(const T* __restrict__ x, long long n, SelState* st,
                                                            long long k1) {
    using K = decltype(key_of(T()));
    if (k1 < st->less + st->eq) return;     // key0's run already holds rank k1
    const K key0 = (K)st->prefix;
    K best = (K)~(K)0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {   // 4 loads in flight
        T v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = x[i + k * stride];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const K key = key_of(v[k]);
            if (key > key0 && key < best) best = key;
        }
    }
    for (; i < n; i += stride) {
        const K key = key_of(x[i]);
        if (key > key0 && key < best) best = key;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const K t = __shfl_xor_sync(0xFFFFFFFFu, best, o);
        best = t < best ? t : best;
    }
    if ((threadIdx.x & 31) == 0 && best != (K)~(K)0) atomicMin(&st->min_above, (unsigned long long)best);
}

template <typename T>
__global__ void k_sel_finish(SelState* st, long long k1, T* out) {
    using K = decltype(key_of(T()));
    const K key0 = (K)st->prefix;
    T v0 = value_of(key0, T());
    T v1 = v0;
    if (k1 >= st->less + st->eq) v1 = value_of((K)st->min_above, T());
    if (st->nan_count) {
        v0 = (T)NAN;
        v1 = (T)NAN;
    }
    out[0] = v0;
    out[1] = v1;
}

// ---------------------------------------------------------------------------
// Frames: for every angle a, frame[a][v][u] (uint8, N_v x N_u) is
//   0                                  when src_row[v] < 0 or src_col[u] < 0
//   byte(q(sino[src_col[u]][a][src_row[v]]))  otherwise
// (ImageSeq.__init__ :134-174 with _insertImage / _arrayInsertImage
// :303-355; the row / column tables carry the insertion offsets, the array
// copies (last copy wins) and the flips).  q replays the reference's numpy
// chain in its dtypes: x / norm * max (promote(T, norm dtype)), * scale,
// np.minimum(., max), astype(uint8/16/32), stored into a uint8 frame.
// byte(): NaN -> 0; t = trunc(v); -2^31 <= t < 2^31 -> low byte of (int32)t;
// wide (uint32 stage) and 2^31 <= t < 2^32 -> low byte of (uint32)t; else 0
// (the x86-64 conversion numpy's casts compile to, then the uint8 store).
// Thread layout: lane = frame row, warp = 32 frame columns, so every load
// instruction of a warp reads 32 consecutive z of one sinogram row and every
// thread stores 32 contiguous bytes.
// ---------------------------------------------------------------------------
struct QuantArgs {
    double norm_d, scale_d, max_d;
    float norm_f, scale_f, max_f;
    int in_f64;      // sinogram dtype is double
    int norm;        // divide by the percentile value and multiply by max
    int norm_f64;    // that stage computes in double
    int scale;       // multiply by the intensity scale
    int scale_f64;   // that stage computes in double
    int wide;        // bit depth > 16: the integer stage is uint32
};

__device__ __forceinline__ uint32_t low_byte(double v, int wide) {
    if (v != v) return 0u;
    const double t = trunc(v);
    if (t >= -2147483648.0 && t < 2147483648.0) return (uint32_t)(int32_t)t & 0xFFu;
    if (wide && t >= 2147483648.0 && t < 4294967296.0) return (uint32_t)(unsigned long long)t & 0xFFu;
    return 0u;
}

template <typename T>
__device__ __forceinline__ uint32_t quantise(T x, const QuantArgs& q) {
    bool f64 = q.in_f64;
    double vd = (double)x;
    float vf = (float)x;   // exact when T is float
    if (q.norm) {
        if (q.norm_f64) {
            vd = dmul(__ddiv_rn(vd, q.norm_d), q.max_d);
            f64 = true;
        } else {
            vf = fmul(__fdiv_rn(vf, q.norm_f), q.max_f);
        }
    }
    if (q.scale) {
        if (f64 || q.scale_f64) {
            if (!f64) vd = (double)vf;
            vd = dmul(vd, q.scale_d);
            f64 = true;
        } else {
            vf = fmul(vf, q.scale_f);
        }
    }
    if (f64) {
        vd = (vd != vd) ? vd : (vd < q.max_d ? vd : q.max_d);
        return low_byte(vd, q.wide);
    }
    vf = (vf != vf) ? vf : (vf < q.max_f ? vf : q.max_f);
    return low_byte((double)vf, q.wide);
}

struct FrameArgs {
    int nR, nA, nZ, n_u, n_v;
    int v0, v1;      // window rows [v0, v1)
    int u0, u1;      // window byte columns [u0, u1), multiples of the store width
    int vec16;       // n_u % 16 == 0: 16-byte stores, else 4-byte stores
    const int* src_col;
    const int* src_row;
    QuantArgs q;
};

// Window tile of the frames: lane = frame row, warp = 16 frame columns.
// Every load instruction of a warp reads 32 consecutive z of one sinogram row
// (the rows of a frame are consecutive z); every lane stores 16 contiguous
// bytes.  Rows / columns whose table entry is -1 (gaps between arrayed
// copies, store-width padding at the window edge) get zeros.
template <typename T>
__device__ __forceinline__ void frames_window_tile(const T* __restrict__ sino, uint8_t* __restrict__ frames,
                                                   const FrameArgs& p, int a, int tile_v, int tile_u) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int v = p.v0 + tile_v * 32 + lane;
    const int u0 = p.u0 + (tile_u * (kThreads / 32) + warp) * 16;
    if (u0 >= p.u1) return;
    int z = v < p.v1 ? __ldg(p.src_row + v) : -1;
    if (z >= p.nZ) z = -1;   // table entries outside the sinogram read as blank
    uint32_t word[4] = {0u, 0u, 0u, 0u};
    // column indices are the same for all lanes: one broadcast load each
    int r[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        r[j] = (u0 + j < p.u1) ? __ldg(p.src_col + u0 + j) : -1;
        if (r[j] >= p.nR) r[j] = -1;
    }
    if (z >= 0) {
        const T* col = sino + (size_t)a * p.nZ + z;
        const size_t rs = (size_t)p.nA * p.nZ;
        T x[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = r[j] >= 0 ? __ldg(col + (size_t)r[j] * rs) : (T)0;
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (r[j] >= 0) word[j >> 2] |= quantise(x[j], p.q) << (8 * (j & 3));
    }
    if (v >= p.v1) return;
    uint8_t* dst = frames + ((size_t)a * p.n_v + v) * p.n_u + u0;
    if (p.vec16) {
        *reinterpret_cast<uint4*>(dst) = make_uint4(word[0], word[1], word[2], word[3]);
    } else {
#pragma unroll
        for (int w = 0; w < 4; ++w)
            if (u0 + 4 * w < p.u1) reinterpret_cast<uint32_t*>(dst)[w] = word[w];
    }
}

// Frame row outside the window: zeros, contiguous 16-byte (4-byte when
// n_u % 16 != 0) stores by one warp.
__device__ __forceinline__ void frames_blank_row(uint8_t* __restrict__ frames, long long row, const FrameArgs& p) {
    const int lane = threadIdx.x & 31;
    const int v = (int)(row % p.n_v);
    const bool in_rows = v >= p.v0 && v < p.v1;
    uint8_t* dst = frames + row * p.n_u;
    if (p.vec16) {
        for (int u = lane * 16; u < p.n_u; u += 32 * 16)
            if (!(in_rows && u >= p.u0 && u < p.u1)) *reinterpret_cast<uint4*>(dst + u) = make_uint4(0u, 0u, 0u, 0u);
    } else {
        for (int u = lane * 4; u < p.n_u; u += 32 * 4)
            if (!(in_rows && u >= p.u0 && u < p.u1)) *reinterpret_cast<uint32_t*>(dst + u) = 0u;
    }
}

// One grid for both parts, so the quantiser arithmetic of the window tiles
// overlaps the store stream of the blank rows: blocks [0, n_win) are window
// tiles (a, tile row, tile column), the rest take 8 blank frame rows each.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_frames(const T* __restrict__ sino, uint8_t* __restrict__ frames,
                                                     const FrameArgs p, int tiles_u, int tiles_v, long long n_win,
                                                     long long n_rows) {
    const long long b = blockIdx.x;
    if (b < n_win) {
        const int tu = (int)(b % tiles_u);
        const long long rest = b / tiles_u;
        frames_window_tile<T>(sino, frames, p, (int)(rest / tiles_v), (int)(rest % tiles_v), tu);
        return;
    }
    const long long row = (b - n_win) * (kThreads / 32) + (threadIdx.x >> 5);
    if (row < n_rows) frames_blank_row(frames, row, p);
}

// ---------------------------------------------------------------------------
// Fan-beam rebinning (geometry.py:736-944): out[p][a][z] =
//   Tinv[p] * (D[p] * interp(p, a, z))
// interp = scipy.interpolate.interpn((xp, angles), b[..., z], (x_samp, theta_samp),
// method='linear', bounds_error=False, fill_value=0) evaluated as
//   ((x00*a0)*a1 + (x01*a0)*y1) + (x10*y0)*a1) + (x11*y0)*y1
// with (i, y) from the grid search done on the host, a = 1 - y, and 0 for an
// out-of-bounds sample.  b is the sinogram padded to nP rows: input row
// p - pad_lo, zero outside [0, nR).  Double arithmetic, stored in T.
// ---------------------------------------------------------------------------
struct RebinArgs {
    int nR, nA, nZ, nP, pad_lo;
    const int* xi;         // [nP] lower x-grid index, -1 = out of bounds
    const double* xw;      // [nP][4] y0, 1 - y0, dxv_dxp, 1 / T
    const int* ti;         // [nP][nA] lower angle-grid index, -1 = out of bounds
    const double* tw;      // [nP][nA][2] y1, 1 - y1
};

template <typename T>
__device__ __forceinline__ double rebin_sample(const double (&x)[4], bool inb, double a0, double y0, double a1,
                                               double y1, double dd, double tinv) {
    double v = 0.0;
    if (inb) {
        v = dmul(dmul(x[0], a0), a1);
        v = dadd(v, dmul(dmul(x[1], a0), y1));
        v = dadd(v, dmul(dmul(x[2], y0), a1));
        v = dadd(v, dmul(dmul(x[3], y0), y1));
    }
    return dmul(tinv, dmul(v, dd));
}

// One warp per output row (p, a), lanes along z, four z per lane in flight
// (16 loads); eight rows per block.
// four resident CTAs per SM (64 registers, a few spilled bytes; three at 72-75): 0.083 -> 0.076 ms for
// a float64 256 x 120 x 256 sinogram, identical results
template <typename T>
__global__ void __launch_bounds__(kThreads, 4) k_rebin_fan(const T* __restrict__ in, T* __restrict__ out,
                                                        const RebinArgs p) {
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);   // pp * nA + a
    if (row >= (long long)p.nP * p.nA) return;
    const int pp = (int)(row / p.nA);
    const int i0 = __ldg(p.xi + pp), j0 = __ldg(p.ti + row);
    const double y0 = __ldg(p.xw + 4 * pp), a0 = __ldg(p.xw + 4 * pp + 1);
    const double dd = __ldg(p.xw + 4 * pp + 2), tinv = __ldg(p.xw + 4 * pp + 3);
    const double y1 = __ldg(p.tw + 2 * row), a1 = __ldg(p.tw + 2 * row + 1);
    const bool inb = i0 >= 0 && j0 >= 0 && j0 + 1 < p.nA;
    const int r0 = i0 - p.pad_lo, r1 = i0 + 1 - p.pad_lo;
    const bool ok0 = inb && r0 >= 0 && r0 < p.nR, ok1 = inb && r1 >= 0 && r1 < p.nR;
    const size_t rs = (size_t)p.nA * p.nZ;
    const T* b00 = in + (size_t)(ok0 ? r0 : 0) * rs + (size_t)(inb ? j0 : 0) * p.nZ;
    const T* b10 = in + (size_t)(ok1 ? r1 : 0) * rs + (size_t)(inb ? j0 : 0) * p.nZ;
    T* o = out + (size_t)row * p.nZ;
    for (int z0 = lane; z0 < p.nZ; z0 += 4 * 32) {
        double x[4][4];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int z = z0 + h * 32;
            const bool zin = z < p.nZ;
            x[h][0] = ok0 && zin ? ld(b00 + z) : 0.0;
            x[h][1] = ok0 && zin ? ld(b00 + p.nZ + z) : 0.0;
            x[h][2] = ok1 && zin ? ld(b10 + z) : 0.0;
            x[h][3] = ok1 && zin ? ld(b10 + p.nZ + z) : 0.0;
        }
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int z = z0 + h * 32;
            if (z < p.nZ) o[z] = (T)rebin_sample<T>(x[h], inb, a0, y0, a1, y1, dd, tinv);
        }
    }
}

inline bool dtype_ok(int dtype) { return dtype == VAM_DTYPE_F32 || dtype == VAM_DTYPE_F64; }

int grid_stride_blocks() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 8;
}

}  // namespace

extern "C" int vam_sino_rotate(const void* in, int dtype, int32_t nR, int32_t nA, int32_t nZ, int32_t flip_r,
                               int32_t flip_z, const double* affine, void* out, int32_t oR, int32_t oZ,
                               vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(in && out && affine, VAM_ERR_ARG, "vam_sino_rotate: null argument");
    VAM_REQUIRE(dtype_ok(dtype), VAM_ERR_ARG, "vam_sino_rotate: dtype must be VAM_DTYPE_F32 or VAM_DTYPE_F64");
    VAM_REQUIRE(nR > 0 && nA > 0 && nZ > 0 && oR > 0 && oZ > 0, VAM_ERR_SHAPE, "vam_sino_rotate: empty shape");
    VAM_REQUIRE((int64_t)oR * nA < (1ll << 31), VAM_ERR_SHAPE, "vam_sino_rotate: oR * nA too large");
    for (int i = 0; i < 6; ++i)
        VAM_REQUIRE(isfinite(affine[i]), VAM_ERR_ARG, "vam_sino_rotate: non-finite affine coefficient");
    RotArgs p{affine[0], affine[1], affine[2], affine[3], affine[4], affine[5], nR, nA, nZ, oR, oZ,
              flip_r != 0, flip_z != 0};
    const unsigned grid = (unsigned)((int64_t)oR * nA);
    if (dtype == VAM_DTYPE_F64)
        k_sino_rotate<double><<<grid, kThreads, 0, (cudaStream_t)stream>>>((const double*)in, (double*)out, p);
    else
        k_sino_rotate<float><<<grid, kThreads, 0, (cudaStream_t)stream>>>((const float*)in, (float*)out, p);
    VAM_CHECK_LAUNCH("vam_sino_rotate");
    return VAM_OK;
}

extern "C" int vam_sino_resize(const void* in, int dtype, int32_t nR, int32_t nA, int32_t nZ, int32_t flip_r,
                               int32_t flip_z, void* out, int32_t oR, int32_t oZ, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(in && out, VAM_ERR_ARG, "vam_sino_resize: null argument");
    VAM_REQUIRE(dtype_ok(dtype), VAM_ERR_ARG, "vam_sino_resize: dtype must be VAM_DTYPE_F32 or VAM_DTYPE_F64");
    VAM_REQUIRE(nR > 0 && nA > 0 && nZ > 0 && oR > 0 && oZ > 0, VAM_ERR_SHAPE, "vam_sino_resize: empty shape");
    VAM_REQUIRE((int64_t)oR * nA < (1ll << 31), VAM_ERR_SHAPE, "vam_sino_resize: oR * nA too large");
    // OpenCV: inv_scale = dsize / ssize, scale = 1 / inv_scale
    ResizeArgs p{1.0 / ((double)oR / (double)nR), 1.0 / ((double)oZ / (double)nZ), nR, nA, nZ, oR, oZ,
                 flip_r != 0, flip_z != 0};
    const unsigned grid = (unsigned)((int64_t)oR * nA);
    if (dtype == VAM_DTYPE_F64)
        k_sino_resize<double><<<grid, kThreads, 0, (cudaStream_t)stream>>>((const double*)in, (double*)out, p);
    else
        k_sino_resize<float><<<grid, kThreads, 0, (cudaStream_t)stream>>>((const float*)in, (double*)out, p);
    VAM_CHECK_LAUNCH("vam_sino_resize");
    return VAM_OK;
}

extern "C" size_t vam_select_workspace_bytes(void) { return (sizeof(SelState) + 255) & ~(size_t)255; }

extern "C" int vam_select_pair(const void* x, int dtype, int64_t n, int64_t k0, int64_t k1, void* out, void* work,
                               size_t work_bytes, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(x && out && work, VAM_ERR_ARG, "vam_select_pair: null argument");
    VAM_REQUIRE(dtype_ok(dtype), VAM_ERR_ARG, "vam_select_pair: dtype must be VAM_DTYPE_F32 or VAM_DTYPE_F64");
    VAM_REQUIRE(n > 0, VAM_ERR_SHAPE, "vam_select_pair: empty input");
    VAM_REQUIRE(k0 >= 0 && k0 < n && (k1 == k0 || k1 == k0 + 1) && k1 < n, VAM_ERR_ARG,
                "vam_select_pair: ranks must satisfy 0 <= k0 <= k1 <= k0 + 1 < n + 1 and k1 < n");
    VAM_REQUIRE(work_bytes >= vam_select_workspace_bytes(), VAM_ERR_ARG, "vam_select_pair: workspace too small");
    VAM_REQUIRE(((uintptr_t)work & 7u) == 0, VAM_ERR_ARG, "vam_select_pair: workspace not 8-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    SelState* s = (SelState*)work;
    const int key_bits = dtype == VAM_DTYPE_F64 ? 64 : 32;
    const int blocks = (int)std::min<int64_t>(grid_stride_blocks(), (n + kThreads - 1) / kThreads);
    k_sel_init<<<1, kThreads, 0, st>>>(s, k0);
    for (int d = 0; d * kDigitBits < key_bits; ++d) {
        const int top = key_bits - d * kDigitBits;
        const int shift = std::max(top - kDigitBits, 0);
        const int width = top - shift;
        if (dtype == VAM_DTYPE_F64)
            k_sel_hist<double><<<blocks, kThreads, 0, st>>>((const double*)x, n, s, shift, width, d == 0);
        else
            k_sel_hist<float><<<blocks, kThreads, 0, st>>>((const float*)x, n, s, shift, width, d == 0);
        k_sel_scan<<<1, kScanThreads, 0, st>>>(s, shift, width);
    }
    if (dtype == VAM_DTYPE_F64) {
        if (k1 != k0) k_sel_min_above<double><<<blocks, kThreads, 0, st>>>((const double*)x, n, s, k1);
        k_sel_finish<double><<<1, 1, 0, st>>>(s, k1, (double*)out);
    } else {
        if (k1 != k0) k_sel_min_above<float><<<blocks, kThreads, 0, st>>>((const float*)x, n, s, k1);
        k_sel_finish<float><<<1, 1, 0, st>>>(s, k1, (float*)out);
    }
    VAM_CHECK_LAUNCH("vam_select_pair");
    return VAM_OK;
}

extern "C" int vam_imageseq_frames(const void* sino, int dtype, int32_t nR, int32_t nA, int32_t nZ,
                                   const vam_frame_params* prm, uint8_t* frames, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(sino && prm && frames && prm->src_col_dev && prm->src_row_dev, VAM_ERR_ARG,
                "vam_imageseq_frames: null argument");
    VAM_REQUIRE(dtype_ok(dtype), VAM_ERR_ARG, "vam_imageseq_frames: dtype must be VAM_DTYPE_F32 or VAM_DTYPE_F64");
    VAM_REQUIRE(nR > 0 && nA > 0 && nZ > 0, VAM_ERR_SHAPE, "vam_imageseq_frames: empty sinogram");
    VAM_REQUIRE(prm->n_u > 0 && prm->n_v > 0 && prm->n_u % 4 == 0, VAM_ERR_SHAPE,
                "vam_imageseq_frames: frame width must be a positive multiple of 4");
    VAM_REQUIRE(((uintptr_t)frames & 15u) == 0, VAM_ERR_ARG, "vam_imageseq_frames: frames not 16-byte aligned");
    VAM_REQUIRE(prm->bit_depth >= 0 && prm->bit_depth <= 32, VAM_ERR_ARG,
                "vam_imageseq_frames: bit_depth must be in [0, 32]");
    if (prm->has_norm) VAM_REQUIRE(prm->norm_dtype == VAM_DTYPE_F32 || prm->norm_dtype == VAM_DTYPE_F64,
                                   VAM_ERR_ARG, "vam_imageseq_frames: bad norm_dtype");
    VAM_REQUIRE(prm->box_v0 >= 0 && prm->box_v0 <= prm->box_v1 && prm->box_v1 <= prm->n_v &&
                prm->box_u0 >= 0 && prm->box_u0 <= prm->box_u1 && prm->box_u1 <= prm->n_u, VAM_ERR_ARG,
                "vam_imageseq_frames: window box outside the frame");
    FrameArgs p;
    p.nR = nR;
    p.nA = nA;
    p.nZ = nZ;
    p.n_u = prm->n_u;
    p.n_v = prm->n_v;
    p.vec16 = (prm->n_u % 16) == 0;
    const int w = p.vec16 ? 16 : 4;
    p.v0 = prm->box_v0;
    p.v1 = prm->box_v1;
    p.u0 = prm->box_u0 / w * w;
    p.u1 = std::min((prm->box_u1 + w - 1) / w * w, prm->n_u);
    if (p.v0 == p.v1 || p.u0 == p.u1) p.v0 = p.v1 = p.u0 = p.u1 = 0;   // empty window: all blank
    p.src_col = prm->src_col_dev;
    p.src_row = prm->src_row_dev;
    const double maxv = (double)((1ull << prm->bit_depth) - 1ull);
    QuantArgs& q = p.q;
    q.in_f64 = dtype == VAM_DTYPE_F64;
    q.norm = prm->has_norm != 0;
    q.norm_f64 = q.in_f64 || prm->norm_dtype == VAM_DTYPE_F64;
    q.norm_d = prm->norm_value;
    q.norm_f = (float)prm->norm_value;
    q.scale = prm->has_scale != 0;
    q.scale_f64 = prm->scale_is_f64 != 0;
    q.scale_d = prm->intensity_scale;
    q.scale_f = (float)prm->intensity_scale;
    q.max_d = maxv;
    q.max_f = (float)maxv;
    q.wide = prm->bit_depth > 16;
    cudaStream_t st = (cudaStream_t)stream;
    const bool has_blank = !(p.v0 == 0 && p.v1 == prm->n_v && p.u0 == 0 && p.u1 == prm->n_u);
    const long long n_rows = has_blank ? (long long)nA * prm->n_v : 0;
    const int tiles_u = (p.u1 - p.u0 + (kThreads / 32) * 16 - 1) / ((kThreads / 32) * 16);
    const int tiles_v = (p.v1 - p.v0 + 31) / 32;
    const long long n_win = (long long)nA * tiles_u * tiles_v;
    const long long blocks = n_win + (n_rows + kThreads / 32 - 1) / (kThreads / 32);
    VAM_REQUIRE(blocks < (1ll << 31), VAM_ERR_SHAPE, "vam_imageseq_frames: too many frame rows");
    if (blocks > 0) {
        if (dtype == VAM_DTYPE_F64)
            k_frames<double><<<(unsigned)blocks, kThreads, 0, st>>>((const double*)sino, frames, p, tiles_u,
                                                                    tiles_v, n_win, n_rows);
        else
            k_frames<float><<<(unsigned)blocks, kThreads, 0, st>>>((const float*)sino, frames, p, tiles_u,
                                                                   tiles_v, n_win, n_rows);
    }
    VAM_CHECK_LAUNCH("vam_imageseq_frames");
    return VAM_OK;
}

extern "C" int vam_rebin_fan(const void* in, int dtype, int32_t nR, int32_t nA, int32_t nZ, int32_t nP,
                             int32_t pad_lo, const int32_t* xi, const double* xw, const int32_t* ti,
                             const double* tw, void* out, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(in && out && xi && xw && ti && tw, VAM_ERR_ARG, "vam_rebin_fan: null argument");
    VAM_REQUIRE(dtype_ok(dtype), VAM_ERR_ARG, "vam_rebin_fan: dtype must be VAM_DTYPE_F32 or VAM_DTYPE_F64");
    VAM_REQUIRE(nR > 0 && nA > 0 && nZ > 0 && nP > 0, VAM_ERR_SHAPE, "vam_rebin_fan: empty shape");
    VAM_REQUIRE((int64_t)nP * nA < (1ll << 31), VAM_ERR_SHAPE, "vam_rebin_fan: nP * nA too large");
    RebinArgs p{nR, nA, nZ, nP, pad_lo, xi, xw, ti, tw};
    const unsigned blocks = (unsigned)(((int64_t)nP * nA + kThreads / 32 - 1) / (kThreads / 32));
    if (dtype == VAM_DTYPE_F64)
        k_rebin_fan<double><<<blocks, kThreads, 0, (cudaStream_t)stream>>>((const double*)in, (double*)out, p);
    else
        k_rebin_fan<float><<<blocks, kThreads, 0, (cudaStream_t)stream>>>((const float*)in, (float*)out, p);
    VAM_CHECK_LAUNCH("vam_rebin_fan");
    return VAM_OK;
}
