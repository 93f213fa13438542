// raytrace.cu -- curved-ray tracer in a graded-index medium, sm_100a.
//
// One thread per ray; every thread runs the reference's step loop
// (vamtoolbox/projector/pyTorchRayTrace.py:378-571 with the step of :738-832)
// to the step cap with the exit test every `check` steps, so the host never
// polls an active count and a whole forward or adjoint is one launch.
//
// Fields live in L2-resident device buffers owned by the plan: the index and
// its gradient packed as float4 texels (n, dn/dx, dn/dy, dn/dz) so one trilinear
// corner is one 16-byte load, the attenuation as float.  Rays are numbered
// (detector, angle, z) with z fastest (:1629-1632), so the 32 rays of a warp are
// 32 neighbouring z rows at one detector position and angle: their corner loads
// hit consecutive addresses of the [x][y][z] fields.
//
// Precision: ray state, field sampling and the deposited energy are float32;
// the voxel-index coordinates of the deposit / integrate step are float64 as
// in the reference (:1253-1260), because the floor/ceil neighbour rule counts a
// voxel twice at an exactly integral coordinate (:1262-1280) and float32
// rounding would create such coordinates where the reference has none.
#include <math.h>

#include <cmath>
#include <cstring>
#include <string>

#include "vam_internal.cuh"

struct vam_ray_plan {
    vam_ray_geom g;
    float energy0;
    float* d_x0;         // [nr][3]
    float* d_v0;         // [nr][3]
    float4* d_nfield;    // [nX][nY][nZ] (n, gx, gy, gz)
    float* d_afield;     // [nX][nY][nZ] attenuation (GRID)
    float* d_absorb;     // [nX][nY][nZ] absorption at the grid points
    float* d_scratch;    // [nX][nY][nZ] f * absorb, or the raw deposit
    // padded copies for the 3-D grid-medium kernels: the index texels with the last plane of each axis
    // repeated ([nX+1][nY+1][nZ+1], border padding), the attenuation and the f * absorb / deposit scratch
    // with a zero plane on both sides of each axis ([nX+2][nY+2][nZ+2], zero padding and dropped corners)
    float4* d_npad;
    float* d_apad;
    float* d_spad;
    unsigned long long* d_active;  // rays active at the cap (last call)
    vam_ray_medium med;  // kinds and analytic parameters (pointers unused after bind)
    int has_medium;
    // trajectory cache of the padded path (vam_ray_prepare_trajectories): per executed step of every ray its
    // position x_ip1 and exp(-attenuance), [max_num_step][num_rays] float4 (step-major: a warp's rays are
    // consecutive), the executed steps per ray and the rays active at the cap; valid until the medium changes
    float4* d_traj;
    int* d_traj_len;
    unsigned long long* d_traj_active;
    size_t traj_bytes;
    int64_t traj_rays;  // rays 0 .. traj_rays - 1 are cached (all, or a multiple of 32); the rest are traced
    int traj_valid;
};

namespace vam {
namespace {

struct RayArgs {
    const float* x0;
    const float* v0;
    const float4* nfield;
    const float* afield;
    int64_t nr;
    int nx, ny, nz;
    float norm[3];        // 2/span (0 for a 2D z axis)
    double half_span[3];  // span/2
    double inv_voxel[3];  // 1/voxel (0 for a 2D z axis)
    float half_span_f[3], inv_voxel_f[3];
    double bmax[3], bmin[3];  // exit bounds: max + voxel, min - voxel
    // the same bounds as float32 thresholds that decide every float32 x exactly
    // as the float64 compare does: x > bmax <=> x > bmax_f (bmax rounded down),
    // x < bmin <=> x < bmin_f (bmin rounded up)
    float bmax_f[3], bmin_f[3];
    float h;              // parameter step, float32 as the reference multiplies it
    float h_idx;          // step / voxel_x
    int max_steps, check, twod;
    int param, solver;
    int n_kind;
    float n_sur, lune_R, lune_p;
    int a_kind;
    float a_val, a_R;
    float energy0;
    unsigned long long* active;
};

constexpr int kRayThreads = 128;

// CFG selects how the medium and the integrator are known: 0 reads them from
// the arguments at run time, 1 is the common configuration fixed at compile
// time (grid index, grid attenuation, physical path length, forward symplectic
// Euler), so the step has no configuration branches.
constexpr int kCfgRuntime = 0, kCfgGridSymplectic = 1;
template <int CFG> __device__ __forceinline__ int n_kind(const RayArgs& a) { return CFG == kCfgGridSymplectic ? (int)VAM_INDEX_GRID : a.n_kind; }
template <int CFG> __device__ __forceinline__ int a_kind(const RayArgs& a) { return CFG == kCfgGridSymplectic ? (int)VAM_ALPHA_GRID : a.a_kind; }
template <int CFG> __device__ __forceinline__ int param(const RayArgs& a) { return CFG == kCfgGridSymplectic ? (int)VAM_PARAM_PHYSICAL : a.param; }
template <int CFG> __device__ __forceinline__ int solver(const RayArgs& a) { return CFG == kCfgGridSymplectic ? (int)VAM_ODE_SYMPLECTIC_EULER : a.solver; }

// grid_sample(align_corners=True) unnormalised coordinate of axis d
__device__ __forceinline__ float unnorm(float x, float nrm, int size, bool border) {
    float u = x * nrm;
    float ix = ((u + 1.f) * 0.5f) * (float)(size - 1);
    if (border) ix = fminf((float)(size - 1), fmaxf(ix, 0.f));
    return ix;
}

// Trilinear sample of the packed index texels with border padding.  The
// coordinate is clamped into [0, size-1], so the upper corner is out of range
// only when its weight is exactly 0; clamping its index keeps every load in
// bounds without a branch.
// u: the unclamped unnormalised coordinates (unnorm with border = false)
__device__ __forceinline__ float4 sample_n(const RayArgs& a, const float* u) {
    const float ix = fminf((float)(a.nx - 1), fmaxf(u[0], 0.f));
    const float iy = fminf((float)(a.ny - 1), fmaxf(u[1], 0.f));
    const float iz = fminf((float)(a.nz - 1), fmaxf(u[2], 0.f));
    const float fx = floorf(ix), fy = floorf(iy), fz = floorf(iz);
    const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
    const int x1 = min(x0 + 1, a.nx - 1), y1 = min(y0 + 1, a.ny - 1), z1 = min(z0 + 1, a.nz - 1);
    const float wx1 = ix - fx, wy1 = iy - fy, wz1 = iz - fz;
    const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
    const int sy = a.nz, sx = a.ny * a.nz;
    const float4* f = a.nfield;
    const float4 t000 = __ldg(f + x0 * sx + y0 * sy + z0), t100 = __ldg(f + x1 * sx + y0 * sy + z0);
    const float4 t010 = __ldg(f + x0 * sx + y1 * sy + z0), t110 = __ldg(f + x1 * sx + y1 * sy + z0);
    const float4 t001 = __ldg(f + x0 * sx + y0 * sy + z1), t101 = __ldg(f + x1 * sx + y0 * sy + z1);
    const float4 t011 = __ldg(f + x0 * sx + y1 * sy + z1), t111 = __ldg(f + x1 * sx + y1 * sy + z1);
    const float w000 = wx0 * wy0 * wz0, w100 = wx1 * wy0 * wz0, w010 = wx0 * wy1 * wz0, w110 = wx1 * wy1 * wz0;
    const float w001 = wx0 * wy0 * wz1, w101 = wx1 * wy0 * wz1, w011 = wx0 * wy1 * wz1, w111 = wx1 * wy1 * wz1;
    float4 r;
    r.x = w000 * t000.x + w100 * t100.x + w010 * t010.x + w110 * t110.x + w001 * t001.x + w101 * t101.x + w011 * t011.x + w111 * t111.x;
    r.y = w000 * t000.y + w100 * t100.y + w010 * t010.y + w110 * t110.y + w001 * t001.y + w101 * t101.y + w011 * t011.y + w111 * t111.y;
    r.z = w000 * t000.z + w100 * t100.z + w010 * t010.z + w110 * t110.z + w001 * t001.z + w101 * t101.z + w011 * t011.z + w111 * t111.z;
    r.w = w000 * t000.w + w100 * t100.w + w010 * t010.w + w110 * t110.w + w001 * t001.w + w101 * t101.w + w011 * t011.w + w111 * t111.w;
    return r;
}

// (n, grad n) at x for the configured index kind (medium.py:276-473)
__device__ __forceinline__ void grid_coords(const RayArgs& a, const float* x, float* u) {
    u[0] = unnorm(x[0], a.norm[0], a.nx, false);
    u[1] = unnorm(x[1], a.norm[1], a.ny, false);
    u[2] = unnorm(x[2], a.norm[2], a.nz, false);
}

// u: grid_coords(x), read only by the GRID kind
template <int CFG>
__device__ __forceinline__ void index_at(const RayArgs& a, const float* x, const float* u, float& n, float* gn) {
    if (n_kind<CFG>(a) == VAM_INDEX_GRID) {
        const float4 t = sample_n(a, u);
        n = t.x; gn[0] = t.y; gn[1] = t.z; gn[2] = t.w;
    } else if (n_kind<CFG>(a) == VAM_INDEX_LUNEBURG) {
        const float r = sqrtf(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (r < a.lune_R) {
            n = a.n_sur * powf(2.f - powf(r / a.lune_R, a.lune_p), 1.f / a.lune_p);
            const float k = -powf(a.n_sur / a.lune_R, a.lune_p) * powf(n, 1.f - a.lune_p) * powf(r, a.lune_p - 2.f);
            gn[0] = k * x[0]; gn[1] = k * x[1]; gn[2] = k * x[2];
        } else {
            n = (a.n_sur != 1.f) ? a.n_sur : 1.f;
            gn[0] = gn[1] = gn[2] = 0.f;
        }
    } else {
        n = a.n_sur;
        gn[0] = gn[1] = gn[2] = 0.f;
    }
}

// attenuation coefficient at x (medium.py:753-915; GRID uses zero padding)
// u: grid_coords(x), read only by the GRID kind
template <int CFG>
__device__ __forceinline__ float alpha_at(const RayArgs& a, const float* x, const float* u) {
    const int ak = a_kind<CFG>(a);
    if (ak == VAM_ALPHA_CYLINDER || ak == VAM_ALPHA_BALL) {
        float r2 = x[0] * x[0] + x[1] * x[1];
        if (ak == VAM_ALPHA_BALL) r2 += x[2] * x[2];
        return sqrtf(r2) < a.a_R ? a.a_val : 0.f;
    }
    if (ak != VAM_ALPHA_GRID) return 0.f;
    const float ix = u[0], iy = u[1], iz = u[2];
    // far outside the grid every corner is zero padding
    if (!(ix > -1.f && ix < (float)a.nx && iy > -1.f && iy < (float)a.ny && iz > -1.f && iz < (float)a.nz)) return 0.f;
    const float fx = floorf(ix), fy = floorf(iy), fz = floorf(iz);
    const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
    const float wx1 = ix - fx, wy1 = iy - fy, wz1 = iz - fz;
    // per-axis weights of the two corners, zeroed for a corner outside the grid
    const float ax0 = x0 >= 0 ? 1.f - wx1 : 0.f, ax1 = x0 + 1 < a.nx ? wx1 : 0.f;
    const float ay0 = y0 >= 0 ? 1.f - wy1 : 0.f, ay1 = y0 + 1 < a.ny ? wy1 : 0.f;
    const float az0 = z0 >= 0 ? 1.f - wz1 : 0.f, az1 = z0 + 1 < a.nz ? wz1 : 0.f;
    const int X0 = max(x0, 0), X1 = min(x0 + 1, a.nx - 1);
    const int Y0 = max(y0, 0), Y1 = min(y0 + 1, a.ny - 1);
    const int Z0 = max(z0, 0), Z1 = min(z0 + 1, a.nz - 1);
    const int sy = a.nz, sx = a.ny * a.nz;
    const float* f = a.afield;
    return ax0 * (ay0 * (az0 * __ldg(f + X0 * sx + Y0 * sy + Z0) + az1 * __ldg(f + X0 * sx + Y0 * sy + Z1)) +
                  ay1 * (az0 * __ldg(f + X0 * sx + Y1 * sy + Z0) + az1 * __ldg(f + X0 * sx + Y1 * sy + Z1))) +
           ax1 * (ay0 * (az0 * __ldg(f + X1 * sx + Y0 * sy + Z0) + az1 * __ldg(f + X1 * sx + Y0 * sy + Z1)) +
                  ay1 * (az0 * __ldg(f + X1 * sx + Y1 * sy + Z0) + az1 * __ldg(f + X1 * sx + Y1 * sy + Z1)));
}

// dv/dstep and dx/dstep of the three parametrisations (pyTorchRayTrace.py:694-735)
template <int CFG>
__device__ __forceinline__ void dv_dstep(const RayArgs& a, float n, const float* gn, float* dv) {
    if (param<CFG>(a) == VAM_PARAM_CANONICAL) { dv[0] = n * gn[0]; dv[1] = n * gn[1]; dv[2] = n * gn[2]; }
    else if (param<CFG>(a) == VAM_PARAM_OPTICAL) { dv[0] = gn[0] / n; dv[1] = gn[1] / n; dv[2] = gn[2] / n; }
    else { dv[0] = gn[0]; dv[1] = gn[1]; dv[2] = gn[2]; }
}

template <int CFG>
__device__ __forceinline__ void dx_dstep(const RayArgs& a, float n, const float* v, float* dx) {
    if (param<CFG>(a) == VAM_PARAM_CANONICAL) { dx[0] = v[0]; dx[1] = v[1]; dx[2] = v[2]; }
    else if (param<CFG>(a) == VAM_PARAM_OPTICAL) {
        const float in2 = 1.f / (n * n);
        dx[0] = v[0] * in2; dx[1] = v[1] * in2; dx[2] = v[2] * in2;
    } else { const float rn = 1.f / n; dx[0] = v[0] * rn; dx[1] = v[1] * rn; dx[2] = v[2] * rn; }
}

struct RayState {
    float xi[3], xp[3], vi[3], vp[3];
    float att, E, E0;
    bool active;
};

template <int CFG>
__device__ __forceinline__ void ray_init(const RayArgs& a, int64_t r, float E0, RayState& st) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        st.xi[d] = st.xp[d] = a.x0[r * 3 + d];
        st.vi[d] = st.vp[d] = a.v0[r * 3 + d];
    }
    st.att = 0.f;
    st.E0 = E0;
    st.E = E0;
    st.active = true;
    if (solver<CFG>(a) == VAM_ODE_LEAPFROG) {  // half step back in v (pyTorchRayTrace.py:816-828)
        float n, gn[3], dv[3], u[3];
        grid_coords(a, st.xp, u);
        index_at<CFG>(a, st.xp, u, n, gn);
        dv_dstep<CFG>(a, n, gn, dv);
#pragma unroll
        for (int d = 0; d < 3; ++d) st.vp[d] = st.vp[d] - dv[d] * a.h / 2.f;
    }
}

// One step of the configured ODE solver; returns the physical length ds and
// the attenuation alpha(x_i) used for the energy update.
template <int CFG>
__device__ __forceinline__ void ray_step(const RayArgs& a, RayState& st, float& ds, float& alpha) {
#pragma unroll
    for (int d = 0; d < 3; ++d) { st.xi[d] = st.xp[d]; st.vi[d] = st.vp[d]; }
    float n, gn[3], dv[3], dx[3], u[3];
    grid_coords(a, st.xi, u);
    index_at<CFG>(a, st.xi, u, n, gn);
    dv_dstep<CFG>(a, n, gn, dv);
#pragma unroll
    for (int d = 0; d < 3; ++d) st.vp[d] = st.vi[d] + dv[d] * a.h;
    if (solver<CFG>(a) == VAM_ODE_EULER) dx_dstep<CFG>(a, n, st.vi, dx);
    else dx_dstep<CFG>(a, n, st.vp, dx);
#pragma unroll
    for (int d = 0; d < 3; ++d) { dx[d] = dx[d] * a.h; st.xp[d] = st.xi[d] + dx[d]; }
    ds = sqrtf(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    alpha = alpha_at<CFG>(a, st.xi, u);
    st.att = st.att + alpha * ds;
    st.E = st.E0 * __expf(-st.att);
}

// Exit test of pyTorchRayTrace.py:1343-1424 (position past max+voxel moving
// outward, or below min-voxel moving inward's opposite).  The reference
// compares against float64 bounds; the float32 thresholds give the same answer
// for every float32 position.
__device__ __forceinline__ bool exited(const RayArgs& a, const RayState& st) {
    bool ex = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float x = st.xp[d];
        ex |= (x > a.bmax_f[d] && st.vp[d] > 0.f) || (x < a.bmin_f[d] && st.vp[d] < 0.f);
    }
    return ex;
}

// Trilinear corners of the deposit / integrate step at x_ip1, with the
// reference's floor / ceil neighbours (a voxel at an integral coordinate is
// visited twice, each time with weight 1 along that axis).
struct Corners {
    int lo[3], hi[3];
    float wlo[3], whi[3];
};

__device__ __forceinline__ void corners_at(const RayArgs& a, const float* x, Corners& c) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d == 2 && a.twod) {  // 2-D: the z index is exactly 0 (1/inf voxel), one neighbour
            c.lo[2] = c.hi[2] = 0;
            c.wlo[2] = c.whi[2] = 1.f;
            continue;
        }
        // float32 index; its error (< 3e-5 for grids up to 1024) only matters
        // for the floor / ceil decision near an integer, which is then redone
        // in float64 exactly as the reference forms it
        const float idxf = (x[d] + a.half_span_f[d]) * a.inv_voxel_f[d];
        const float flf = floorf(idxf);
        const float frf = idxf - flf;
        if (frf > 2e-4f && frf < 1.f - 2e-4f && fabsf(idxf) < 1.0e6f) {
            c.lo[d] = (int)flf;
            c.hi[d] = c.lo[d] + 1;
            c.wlo[d] = 1.f - frf;
            c.whi[d] = frf;
        } else {
            const double idx = ((double)x[d] + a.half_span[d]) * a.inv_voxel[d];
            const double fl = floor(idx), ce = ceil(idx);
            c.lo[d] = (int)fmax(fmin(fl, 2.0e9), -2.0e9);
            c.hi[d] = (int)fmax(fmin(ce, 2.0e9), -2.0e9);
            c.wlo[d] = (float)(1.0 - (idx - fl));
            c.whi[d] = (float)(1.0 - (ce - idx));
        }
    }
}

// The 4 (2-D) or 8 corners of a Corners set as element offsets into an
// [nx][ny][nz] field, their trilinear weights (x weight * y weight * z weight,
// the reference's product order) and whether each lies inside the grid.
// Offsets of outside corners are clamped into the grid and never dereferenced.
template <bool TWOD>
struct CornerList {
    static constexpr int kN = TWOD ? 4 : 8;
    int off[kN];
    float w[kN];
    bool in[kN];
};

template <bool TWOD>
__device__ __forceinline__ void corner_list(const RayArgs& a, const Corners& c, CornerList<TWOD>& L) {
    const int sx = a.ny * a.nz, sy = a.nz;
    const bool vx0 = (unsigned)c.lo[0] < (unsigned)a.nx, vx1 = (unsigned)c.hi[0] < (unsigned)a.nx;
    const bool vy0 = (unsigned)c.lo[1] < (unsigned)a.ny, vy1 = (unsigned)c.hi[1] < (unsigned)a.ny;
    const bool vz0 = TWOD || (unsigned)c.lo[2] < (unsigned)a.nz, vz1 = TWOD || (unsigned)c.hi[2] < (unsigned)a.nz;
    const int ox0 = min(max(c.lo[0], 0), a.nx - 1) * sx, ox1 = min(max(c.hi[0], 0), a.nx - 1) * sx;
    const int oy0 = min(max(c.lo[1], 0), a.ny - 1) * sy, oy1 = min(max(c.hi[1], 0), a.ny - 1) * sy;
    const int oz0 = TWOD ? 0 : min(max(c.lo[2], 0), a.nz - 1), oz1 = TWOD ? 0 : min(max(c.hi[2], 0), a.nz - 1);
#pragma unroll
    for (int cn = 0; cn < CornerList<TWOD>::kN; ++cn) {
        L.in[cn] = ((cn & 1) ? vx1 : vx0) && ((cn & 2) ? vy1 : vy0) && ((cn & 4) ? vz1 : vz0);
        L.off[cn] = ((cn & 1) ? ox1 : ox0) + ((cn & 2) ? oy1 : oy0) + ((cn & 4) ? oz1 : oz0);
        L.w[cn] = ((cn & 1) ? c.whi[0] : c.wlo[0]) * ((cn & 2) ? c.whi[1] : c.wlo[1]) *
                  ((cn & 4) ? c.whi[2] : c.wlo[2]);
    }
}

// ---------------------------------------------------------------------------
// integrate (forward)
// ---------------------------------------------------------------------------
template <bool TWOD, int CFG>
__global__ void __launch_bounds__(kRayThreads) k_ray_integrate(RayArgs a, const float* __restrict__ fa,
                                                               float* __restrict__ g) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= a.nr) return;
    RayState st;
    ray_init<CFG>(a, r, a.energy0, st);
    float integral = 0.f;
    int until_check = 0;  // the exit test runs at steps 0, check, 2 check, ...
    for (int step = 0; step < a.max_steps; ++step) {
        float ds, alpha;
        ray_step<CFG>(a, st, ds, alpha);
        Corners c;
        corners_at(a, st.xp, c);
        CornerList<TWOD> L;
        corner_list<TWOD>(a, c, L);
        const float eh = a.h_idx * st.E;
#pragma unroll
        for (int cn = 0; cn < CornerList<TWOD>::kN; ++cn)
            if (L.in[cn]) integral = fmaf(__ldg(fa + L.off[cn]), L.w[cn] * eh, integral);
        if (until_check == 0) {
            until_check = a.check;
            if (exited(a, st)) { st.active = false; break; }
        }
        --until_check;
    }
    g[r] = integral;
    if (st.active) atomicAdd(a.active, 1ULL);
}

// ---------------------------------------------------------------------------
// deposit (adjoint)
// ---------------------------------------------------------------------------
template <bool TWOD, int CFG>
__global__ void __launch_bounds__(kRayThreads) k_ray_deposit(RayArgs a, const float* __restrict__ gin,
                                                             float* __restrict__ dose) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= a.nr) return;
    RayState st;
    ray_init<CFG>(a, r, gin[r], st);
    const bool zero = st.E0 == 0.f;  // a zero-energy ray deposits nothing; still traced for the cap count
    int until_check = 0;
    for (int step = 0; step < a.max_steps; ++step) {
        float ds, alpha;
        ray_step<CFG>(a, st, ds, alpha);
        if (!zero) {
            Corners c;
            corners_at(a, st.xp, c);
            CornerList<TWOD> L;
            corner_list<TWOD>(a, c, L);
            const float eh = a.h_idx * st.E;
#pragma unroll
            for (int cn = 0; cn < CornerList<TWOD>::kN; ++cn)
                if (L.in[cn]) atomicAdd(dose + L.off[cn], L.w[cn] * eh);
        }
        if (until_check == 0) {
            until_check = a.check;
            if (exited(a, st)) { st.active = false; break; }
        }
        --until_check;
    }
    if (st.active) atomicAdd(a.active, 1ULL);
}

// ---------------------------------------------------------------------------
// d<w, integrate(f)>/d alpha_att: pass 1 totals, pass 2 suffix sums
// ---------------------------------------------------------------------------
template <bool TWOD, int CFG>
__global__ void __launch_bounds__(kRayThreads) k_ray_grad_att(RayArgs a, const float* __restrict__ fa,
                                                              const float* __restrict__ w, float* __restrict__ grad) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= a.nr) return;
    const float wr = w[r];
    if (wr == 0.f) return;
    float total = 0.f;
    for (int pass = 0; pass < 2; ++pass) {
        RayState st;
        ray_init<CFG>(a, r, a.energy0, st);
        float prefix = 0.f;
        int until_check = 0;
        for (int step = 0; step < a.max_steps; ++step) {
            if (!st.active) break;
            float ds, alpha;
            ray_step<CFG>(a, st, ds, alpha);
            Corners c;
            corners_at(a, st.xp, c);
            CornerList<TWOD> L;
            corner_list<TWOD>(a, c, L);
            const float eh = a.h_idx * st.E;
            float contrib = 0.f;
#pragma unroll
            for (int cn = 0; cn < CornerList<TWOD>::kN; ++cn)
                if (L.in[cn]) contrib = fmaf(__ldg(fa + L.off[cn]), L.w[cn] * eh, contrib);
            if (pass == 1 && ds > 0.f) {
                // att(step) = sum alpha(x_i) ds  ->  d integral / d alpha(x_i at this step)
                //   = -ds * (contributions of this and all later steps)
                const float suffix = total - prefix;
                const float coef = -wr * ds * suffix;
                if (coef != 0.f) {
                    const float ix = unnorm(st.xi[0], a.norm[0], a.nx, false);
                    const float iy = unnorm(st.xi[1], a.norm[1], a.ny, false);
                    const float iz = unnorm(st.xi[2], a.norm[2], a.nz, false);
                    const float fx = floorf(ix), fy = floorf(iy), fz = floorf(iz);
                    const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
                    const float wx1 = ix - fx, wy1 = iy - fy, wz1 = iz - fz;
                    for (int cz = 0; cz < 2; ++cz) {
                        const int Z = z0 + cz;
                        if ((unsigned)Z >= (unsigned)a.nz) continue;
                        for (int cy = 0; cy < 2; ++cy) {
                            const int Y = y0 + cy;
                            if ((unsigned)Y >= (unsigned)a.ny) continue;
                            for (int cx = 0; cx < 2; ++cx) {
                                const int X = x0 + cx;
                                if ((unsigned)X >= (unsigned)a.nx) continue;
                                const float tw = (cx ? wx1 : 1.f - wx1) * (cy ? wy1 : 1.f - wy1) * (cz ? wz1 : 1.f - wz1);
                                atomicAdd(grad + ((size_t)X * a.ny + Y) * a.nz + Z, coef * tw);
                            }
                        }
                    }
                }
            }
            prefix += contrib;
            if (until_check == 0) {
                until_check = a.check;
                if (exited(a, st)) st.active = false;
            }
            --until_check;
        }
        total = prefix;
    }
}

// ---------------------------------------------------------------------------
// record: the propagation matrix of the integrate operator, one CSR row per ray
// (pyTorchRayTrace.py:573-690, 901-937, 1146-1252).  Row r holds, in step
// order, the (voxel, weight) pairs ray r deposits with unit start energy:
// (h / voxel) * E(step) * trilinear corner weight, times the absorption at the
// voxel (the reference's right multiplication by a diagonal matrix); a voxel
// met twice (the floor / ceil double count, or two steps in one voxel) appears
// twice, as in the reference before it coalesces.  With count, pass 1 writes
// the row lengths; without, pass 2 fills cols / vals from row_ptr[r].
// ---------------------------------------------------------------------------
template <bool TWOD, int CFG>
__global__ void __launch_bounds__(kRayThreads) k_ray_record(RayArgs a, const float* __restrict__ absorb,
                                                            int64_t* __restrict__ count,
                                                            const int64_t* __restrict__ row_ptr,
                                                            int32_t* __restrict__ cols, float* __restrict__ vals) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= a.nr) return;
    RayState st;
    ray_init<CFG>(a, r, a.energy0, st);  // the reference's start energy: ray_density^-1 (2-D) or ^-2 (3-D)
    int64_t k = count ? 0 : row_ptr[r];
    int until_check = 0;
    for (int step = 0; step < a.max_steps; ++step) {
        float ds, alpha;
        ray_step<CFG>(a, st, ds, alpha);
        Corners c;
        corners_at(a, st.xp, c);
        CornerList<TWOD> L;
        corner_list<TWOD>(a, c, L);
        const float eh = a.h_idx * st.E;
#pragma unroll
        for (int cn = 0; cn < CornerList<TWOD>::kN; ++cn) {
            if (!L.in[cn]) continue;
            if (!count) {
                cols[k] = L.off[cn];
                vals[k] = L.w[cn] * eh * __ldg(absorb + L.off[cn]);
            }
            ++k;
        }
        if (until_check == 0) {
            until_check = a.check;
            if (exited(a, st)) { st.active = false; break; }
        }
        --until_check;
    }
    if (count) count[r] = k;
}

// Y[row][z] = sum over the row's entries of val * X[col][z]  (CSR times a z-tiled dense block).
// A warp per row; with one z per row the lanes split the row's entries and a shuffle tree sums them,
// otherwise the lanes run along z.  Fixed orders throughout: deterministic.
__global__ void __launch_bounds__(256) k_csr_spmm(int64_t nrows, const int64_t* __restrict__ row_ptr,
                                                  const int32_t* __restrict__ cols, const float* __restrict__ vals,
                                                  const float* __restrict__ X, int ztile, float* __restrict__ Y,
                                                  int vec4) {
    const int lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= nrows) return;
    const int64_t b = row_ptr[row], e = row_ptr[row + 1];
    if (ztile == 1) {
        float acc = 0.f;
        for (int64_t k = b + lane; k < e; k += 32) acc = fmaf(__ldg(vals + k), __ldg(X + __ldg(cols + k)), acc);
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) Y[row] = acc;
        return;
    }
    if (vec4) {  // ztile % 4 == 0, 16-byte aligned: a warp covers 128 columns of a row with one 512-byte load
        for (int z0 = 0; z0 < ztile; z0 += 128) {
            const int z = z0 + 4 * lane;
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            if (z < ztile)
                for (int64_t k = b; k < e; ++k) {
                    const float v = __ldg(vals + k);
                    const float4 xv = __ldg(reinterpret_cast<const float4*>(X + (int64_t)__ldg(cols + k) * ztile + z));
                    acc.x = fmaf(v, xv.x, acc.x); acc.y = fmaf(v, xv.y, acc.y);
                    acc.z = fmaf(v, xv.z, acc.z); acc.w = fmaf(v, xv.w, acc.w);
                }
            if (z < ztile) *reinterpret_cast<float4*>(Y + row * ztile + z) = acc;
        }
        return;
    }
    for (int z0 = 0; z0 < ztile; z0 += 32) {
        const int z = z0 + lane;
        float acc = 0.f;
        if (z < ztile)
            for (int64_t k = b; k < e; ++k)
                acc = fmaf(__ldg(vals + k), __ldg(X + (int64_t)__ldg(cols + k) * ztile + z), acc);
        if (z < ztile) Y[row * ztile + z] = acc;
    }
}

// ---------------------------------------------------------------------------
// 3-D grid media, physical path length, forward symplectic Euler: the step of
// the benchmark configuration on padded fields.  The padding turns every
// clamped or dropped trilinear corner into an in-bounds load of a border or
// zero cell, so a sample is one offset plus constant corner strides (z corners
// at +1 element, an immediate) with no per-corner bounds logic; the float4
// index texels are interpolated as two float2 halves with packed f32x2 FMAs.
// The values are the ones of k_ray_integrate / k_ray_deposit with
// kCfgGridSymplectic up to float32 summation order.
// ---------------------------------------------------------------------------
struct PadArgs {
    const float4* npad;  // [nx+1][ny+1][nz+1]
    const float* apad;   // [nx+2][ny+2][nz+2]
    int nsx, nsy;        // element strides of npad
    int psx, psy;        // element strides of apad and of the padded scratch
};

__device__ __forceinline__ unsigned long long pack2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}

__device__ __forceinline__ float2 unpack2(unsigned long long r) {
    float2 o;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
    return o;
}

// acc += w * (t.x, t.y) and w * (t.z, t.w): two packed FMAs (each half rounds like fmaf)
__device__ __forceinline__ void fma4(unsigned long long& a01, unsigned long long& a23, float w, const float4& t) {
    const unsigned long long ww = pack2(w, w);
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(a01) : "l"(ww), "l"(pack2(t.x, t.y)));
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(a23) : "l"(ww), "l"(pack2(t.z, t.w)));
}

// (n, grad n) at grid coordinates u (border padding): the texel block of the clamped coordinate.
// (Reading the attenuation corners here as well when the point is inside the grid, where both samples
// share corners and weights, measured slower: 25.2 against 23.5 ms at 128^3 x 360.)
__device__ __forceinline__ float4 sample_n_pad(const RayArgs& a, const PadArgs& q, const float* u) {
    const float ix = fminf((float)(a.nx - 1), fmaxf(u[0], 0.f));
    const float iy = fminf((float)(a.ny - 1), fmaxf(u[1], 0.f));
    const float iz = fminf((float)(a.nz - 1), fmaxf(u[2], 0.f));
    const float fx = floorf(ix), fy = floorf(iy), fz = floorf(iz);
    const float wx1 = ix - fx, wy1 = iy - fy, wz1 = iz - fz;
    const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
    const float4* p = q.npad + ((int)fx * q.nsx + (int)fy * q.nsy + (int)fz);
    const float4 t000 = __ldg(p), t001 = __ldg(p + 1);
    const float4 t010 = __ldg(p + q.nsy), t011 = __ldg(p + q.nsy + 1);
    const float4 t100 = __ldg(p + q.nsx), t101 = __ldg(p + q.nsx + 1);
    const float4 t110 = __ldg(p + q.nsx + q.nsy), t111 = __ldg(p + q.nsx + q.nsy + 1);
    const float w00 = wx0 * wy0, w01 = wx0 * wy1, w10 = wx1 * wy0, w11 = wx1 * wy1;
    unsigned long long a01 = 0ull, a23 = 0ull;
    fma4(a01, a23, w00 * wz0, t000);
    fma4(a01, a23, w10 * wz0, t100);
    fma4(a01, a23, w01 * wz0, t010);
    fma4(a01, a23, w11 * wz0, t110);
    fma4(a01, a23, w00 * wz1, t001);
    fma4(a01, a23, w10 * wz1, t101);
    fma4(a01, a23, w01 * wz1, t011);
    fma4(a01, a23, w11 * wz1, t111);
    const float2 r01 = unpack2(a01), r23 = unpack2(a23);
    return make_float4(r01.x, r01.y, r23.x, r23.y);
}

// attenuation at grid coordinates u (zero padding, medium.py:753-891)
__device__ __forceinline__ float alpha_pad(const RayArgs& a, const PadArgs& q, const float* u) {
    const float ix = u[0], iy = u[1], iz = u[2];
    if (!(ix > -1.f && ix < (float)a.nx && iy > -1.f && iy < (float)a.ny && iz > -1.f && iz < (float)a.nz)) return 0.f;
    const float fx = floorf(ix), fy = floorf(iy), fz = floorf(iz);
    const float wx1 = ix - fx, wy1 = iy - fy, wz1 = iz - fz;
    const float ax0 = 1.f - wx1, ay0 = 1.f - wy1, az0 = 1.f - wz1;
    const float* f = q.apad + (((int)fx + 1) * q.psx + ((int)fy + 1) * q.psy + ((int)fz + 1));
    return ax0 * (ay0 * (az0 * __ldg(f) + wz1 * __ldg(f + 1)) + wy1 * (az0 * __ldg(f + q.psy) + wz1 * __ldg(f + q.psy + 1))) +
           wx1 * (ay0 * (az0 * __ldg(f + q.psx) + wz1 * __ldg(f + q.psx + 1)) +
                  wy1 * (az0 * __ldg(f + q.psx + q.psy) + wz1 * __ldg(f + q.psx + q.psy + 1)));
}

__device__ __forceinline__ void ray_step_pad(const RayArgs& a, const PadArgs& q, RayState& st, float& ds) {
#pragma unroll
    for (int d = 0; d < 3; ++d) { st.xi[d] = st.xp[d]; st.vi[d] = st.vp[d]; }
    float u[3];
    grid_coords(a, st.xi, u);
    const float4 t = sample_n_pad(a, q, u);
    const float alpha = alpha_pad(a, q, u);
    st.vp[0] = st.vi[0] + t.y * a.h;
    st.vp[1] = st.vi[1] + t.z * a.h;
    st.vp[2] = st.vi[2] + t.w * a.h;
    const float rn = 1.f / t.x;
    float dx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { dx[d] = (st.vp[d] * rn) * a.h; st.xp[d] = st.xi[d] + dx[d]; }
    ds = sqrtf(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    st.att = st.att + alpha * ds;
    st.E = st.E0 * __expf(-st.att);
}

// The padded-scratch offset of the step's first deposit / integrate corner, the corner strides along
// x / y / z (0 where the floor / ceil neighbours coincide) and the eight weights times eh; false when
// every corner lies outside the grid (along some axis both neighbours are outside).
__device__ __forceinline__ bool pad_corners(const RayArgs& a, const PadArgs& q, const Corners& c, float eh, int& o,
                                            int& dx, int& dy, int& dz, float (&w)[8]) {
    const bool near = c.lo[0] >= -1 && c.hi[0] <= a.nx && c.lo[1] >= -1 && c.hi[1] <= a.ny && c.lo[2] >= -1 &&
                      c.hi[2] <= a.nz;
    if (!near) return false;
    o = (c.lo[0] + 1) * q.psx + (c.lo[1] + 1) * q.psy + (c.lo[2] + 1);
    dx = (c.hi[0] - c.lo[0]) * q.psx;
    dy = (c.hi[1] - c.lo[1]) * q.psy;
    dz = c.hi[2] - c.lo[2];
    const float wz0 = c.wlo[2] * eh, wz1 = c.whi[2] * eh;
    const float w00 = c.wlo[0] * c.wlo[1], w10 = c.whi[0] * c.wlo[1], w01 = c.wlo[0] * c.whi[1], w11 = c.whi[0] * c.whi[1];
    w[0] = w00 * wz0; w[1] = w10 * wz0; w[2] = w01 * wz0; w[3] = w11 * wz0;
    w[4] = w00 * wz1; w[5] = w10 * wz1; w[6] = w01 * wz1; w[7] = w11 * wz1;
    return true;
}

// r0: the first ray this launch traces (the rays before it come from the trajectory cache)
__global__ void __launch_bounds__(kRayThreads) k_ray_integrate_pad(RayArgs a, PadArgs q, const float* __restrict__ fpad,
                                                                   float* __restrict__ g, int64_t r0) {
    const int64_t r = r0 + (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= a.nr) return;
    RayState st;
    ray_init<kCfgGridSymplectic>(a, r, a.energy0, st);
    float integral = 0.f;
    int until_check = 0;
    for (int step = 0; step < a.max_steps; ++step) {
        float ds;
        ray_step_pad(a, q, st, ds);
        Corners c;
        corners_at(a, st.xp, c);
        int o, dx, dy, dz;
        float w[8];
        if (pad_corners(a, q, c, a.h_idx * st.E, o, dx, dy, dz, w)) {
            const float* f0 = fpad + o;
            const float* f1 = f0 + dx;
            integral = fmaf(__ldg(f0), w[0], integral);
            integral = fmaf(__ldg(f1), w[1], integral);
            integral = fmaf(__ldg(f0 + dy), w[2], integral);
            integral = fmaf(__ldg(f1 + dy), w[3], integral);
            integral = fmaf(__ldg(f0 + dz), w[4], integral);
            integral = fmaf(__ldg(f1 + dz), w[5], integral);
            integral = fmaf(__ldg(f0 + dy + dz), w[6], integral);
            integral = fmaf(__ldg(f1 + dy + dz), w[7], integral);
        }
        if (until_check == 0) {
            until_check = a.check;
            if (exited(a, st)) { st.active = false; break; }
        }
        --until_check;
    }
    g[r] = integral;
    if (st.active) atomicAdd(a.active, 1ULL);
}

__global__ void __launch_bounds__(kRayThreads) k_ray_deposit_pad(RayArgs a, PadArgs q, const float* __restrict__ gin,
                                                                 float* __restrict__ spad, int64_t r0) {
    const int64_t r = r0 + (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= a.nr) return;
    RayState st;
    ray_init<kCfgGridSymplectic>(a, r, gin[r], st);
    const bool zero = st.E0 == 0.f;
    int until_check = 0;
    for (int step = 0; step < a.max_steps; ++step) {
        float ds;
        ray_step_pad(a, q, st, ds);
        if (!zero) {
            Corners c;
            corners_at(a, st.xp, c);
            int o, dx, dy, dz;
            float w[8];
            if (pad_corners(a, q, c, a.h_idx * st.E, o, dx, dy, dz, w)) {
                float* s0 = spad + o;
                float* s1 = s0 + dx;
                atomicAdd(s0, w[0]);
                atomicAdd(s1, w[1]);
                atomicAdd(s0 + dy, w[2]);
                atomicAdd(s1 + dy, w[3]);
                atomicAdd(s0 + dz, w[4]);
                atomicAdd(s1 + dz, w[5]);
                atomicAdd(s0 + dy + dz, w[6]);
                atomicAdd(s1 + dy + dz, w[7]);
            }
        }
        if (until_check == 0) {
            until_check = a.check;
            if (exited(a, st)) { st.active = false; break; }
        }
        --until_check;
    }
    if (st.active) atomicAdd(a.active, 1ULL);
}

// ---------------------------------------------------------------------------
// Trajectory cache.  The rays' paths depend on the medium only, not on f or g, so
// the padded path can trace them once (k_ray_record_pad: the same ray_step_pad
// sequence and exit checks as the integrate / deposit kernels) and keep, per
// executed step, x_ip1 and exp(-attenuance); k_ray_integrate_traj and
// k_ray_deposit_traj then stream those records and run only the corner work of a
// step: the same corners_at / pad_corners on the same float32 values, the energy
// E0 * exp(-attenuance) as ray_step_pad forms it (the same exponential, recorded),
// the same accumulation order, so their results are bit-identical to the tracing
// kernels'.
// ---------------------------------------------------------------------------
// rays 0 .. m - 1 (m: the cached rays), records step-major with stride m
__global__ void __launch_bounds__(kRayThreads) k_ray_record_pad(RayArgs a, PadArgs q, float4* __restrict__ traj,
                                                                int* __restrict__ len,
                                                                unsigned long long* __restrict__ active, int64_t m) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= m) return;
    RayState st;
    ray_init<kCfgGridSymplectic>(a, r, 1.f, st);
    int until_check = 0, n = 0;
    for (int step = 0; step < a.max_steps; ++step) {
        float ds;
        ray_step_pad(a, q, st, ds);
        __stcs(traj + (size_t)step * m + r, make_float4(st.xp[0], st.xp[1], st.xp[2], __expf(-st.att)));
        n = step + 1;
        if (until_check == 0) {
            until_check = a.check;
            if (exited(a, st)) { st.active = false; break; }
        }
        --until_check;
    }
    len[r] = n;
    if (st.active) atomicAdd(active, 1ULL);
}

__global__ void __launch_bounds__(kRayThreads) k_ray_integrate_traj(RayArgs a, PadArgs q, const float4* __restrict__ traj,
                                                                    const int* __restrict__ len,
                                                                    const float* __restrict__ fpad, float* __restrict__ g,
                                                                    int64_t m) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    if (r >= m) return;
    const float E0 = a.energy0;
    const int n = len[r];
    float integral = 0.f;
    float4 t = n > 0 ? __ldcs(traj + r) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int step = 0; step < n; ++step) {
        // the next record in flight while this step's corners are gathered
        const float4 tn = step + 1 < n ? __ldcs(traj + (size_t)(step + 1) * m + r) : t;
        const float xp[3] = {t.x, t.y, t.z};
        const float E = E0 * t.w;
        Corners c;
        corners_at(a, xp, c);
        int o, dx, dy, dz;
        float w[8];
        if (pad_corners(a, q, c, a.h_idx * E, o, dx, dy, dz, w)) {
            const float* f0 = fpad + o;
            const float* f1 = f0 + dx;
            integral = fmaf(__ldg(f0), w[0], integral);
            integral = fmaf(__ldg(f1), w[1], integral);
            integral = fmaf(__ldg(f0 + dy), w[2], integral);
            integral = fmaf(__ldg(f1 + dy), w[3], integral);
            integral = fmaf(__ldg(f0 + dz), w[4], integral);
            integral = fmaf(__ldg(f1 + dz), w[5], integral);
            integral = fmaf(__ldg(f0 + dy + dz), w[6], integral);
            integral = fmaf(__ldg(f1 + dy + dz), w[7], integral);
        }
        t = tn;
    }
    g[r] = integral;
}

// The deposit from the records.  A warp's rays are consecutive z rows of one detector column and angle,
// so at one step lane l's upper-z corners are, as a rule, lane l + 1's lower-z corners (same x / y cells,
// z cell one higher): lane l + 1 then adds lane l's four upper weights to its own lower ones before its
// atomics and lane l issues only its lower four, about halving the atomics (the deposit's bound once the
// tracing is gone).  The sums are the tracing kernel's up to the order of float32 additions, which atomics
// leave open anyway.  Lanes walk to the warp's longest record, inactive ones with no corners.
// rays 0 .. m - 1; m is the ray count or a multiple of 32, so a warp's rays are all cached or none
__global__ void __launch_bounds__(kRayThreads) k_ray_deposit_traj(RayArgs a, PadArgs q, const float4* __restrict__ traj,
                                                                  const int* __restrict__ len,
                                                                  const float* __restrict__ gin, float* __restrict__ spad,
                                                                  int64_t m) {
    const int64_t r = (int64_t)blockIdx.x * kRayThreads + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool in = r < m;
    const float E0 = in ? gin[r] : 0.f;
    const int n = in && E0 != 0.f ? len[r] : 0;
    const int nmax = __reduce_max_sync(0xffffffffu, n);
    float4 t = n > 0 ? __ldcs(traj + r) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int step = 0; step < nmax; ++step) {
        const bool live = step < n;
        const float4 tn = step + 1 < n ? __ldcs(traj + (size_t)(step + 1) * m + r) : t;
        int o = 0, dx = 0, dy = 0, dz = 0;
        float w[8];
        bool ok = false;
        if (live) {
            const float xp[3] = {t.x, t.y, t.z};
            const float E = E0 * t.w;
            Corners c;
            corners_at(a, xp, c);
            ok = pad_corners(a, q, c, a.h_idx * E, o, dx, dy, dz, w);
        }
        if (!ok) {
#pragma unroll
            for (int k = 0; k < 8; ++k) w[k] = 0.f;
        }
        // lane l - 1's upper corners onto this lane's lower ones
        const int op = __shfl_up_sync(0xffffffffu, o, 1), dxp = __shfl_up_sync(0xffffffffu, dx, 1);
        const int dyp = __shfl_up_sync(0xffffffffu, dy, 1), dzp = __shfl_up_sync(0xffffffffu, dz, 1);
        const bool okp = __shfl_up_sync(0xffffffffu, ok, 1);
        float up[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) up[k] = __shfl_up_sync(0xffffffffu, w[4 + k], 1);
        const bool recv = lane > 0 && ok && okp && o == op + dzp && dx == dxp && dy == dyp;
        const bool sent = __shfl_down_sync(0xffffffffu, recv, 1) && lane < 31;
        if (ok) {
            if (recv) {
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] += up[k];
            }
            float* s0 = spad + o;
            float* s1 = s0 + dx;
            atomicAdd(s0, w[0]);
            atomicAdd(s1, w[1]);
            atomicAdd(s0 + dy, w[2]);
            atomicAdd(s1 + dy, w[3]);
            if (!sent) {
                atomicAdd(s0 + dz, w[4]);
                atomicAdd(s1 + dz, w[5]);
                atomicAdd(s0 + dy + dz, w[6]);
                atomicAdd(s1 + dy + dz, w[7]);
            }
        }
        t = tn;
    }
}

// padded [nx+1][ny+1][nz+1] texels: the last plane of each axis repeated (border padding)
__global__ void k_pad_n(const float4* __restrict__ src, float4* __restrict__ dst, int nx, int ny, int nz) {
    const int64_t n = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % (nz + 1)), y = (int)((i / (nz + 1)) % (ny + 1)), x = (int)(i / ((int64_t)(nz + 1) * (ny + 1)));
        dst[i] = src[((int64_t)min(x, nx - 1) * ny + min(y, ny - 1)) * nz + min(z, nz - 1)];
    }
}

// interior of a zero-bordered [nx+2][ny+2][nz+2] array: dst = a * b (b may be null)
__global__ void k_pad_mul(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ dst, int nx,
                          int ny, int nz) {
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz), y = (int)((i / nz) % ny), x = (int)(i / ((int64_t)nz * ny));
        dst[((int64_t)(x + 1) * (ny + 2) + (y + 1)) * (nz + 2) + (z + 1)] = b ? a[i] * b[i] : a[i];
    }
}

// dose = interior of the padded deposit * absorb
__global__ void k_unpad_mul(const float* __restrict__ spad, const float* __restrict__ b, float* __restrict__ out, int nx,
                            int ny, int nz) {
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz), y = (int)((i / nz) % ny), x = (int)(i / ((int64_t)nz * ny));
        out[i] = spad[((int64_t)(x + 1) * (ny + 2) + (y + 1)) * (nz + 2) + (z + 1)] * b[i];
    }
}

__global__ void k_mul(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] * b[i];
}

__global__ void k_mul_acc(const float* __restrict__ a, const float* __restrict__ b, float scale, float* __restrict__ out,
                          int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] += scale * (a[i] * b[i]);
}

__global__ void k_pack_n(const float* __restrict__ n, const float* __restrict__ g, float4* __restrict__ out, int64_t nv) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_float4(n[i], g[3 * i], g[3 * i + 1], g[3 * i + 2]);
}

RayArgs make_args(const vam_ray_plan* p) {
    RayArgs a;
    std::memset(&a, 0, sizeof(a));
    const vam_ray_geom& g = p->g;
    a.x0 = p->d_x0; a.v0 = p->d_v0; a.nfield = p->d_nfield; a.afield = p->d_afield;
    a.nr = g.num_rays;
    a.nx = g.n_x; a.ny = g.n_y; a.nz = g.n_z;
    a.twod = g.n_z == 1;
    for (int d = 0; d < 3; ++d) {
        const double span = g.coord_max[d] - g.coord_min[d];
        const double nrm = 2.0 / span;
        a.norm[d] = std::isfinite(nrm) ? (float)nrm : 0.f;
        a.half_span[d] = span / 2.0;
        const double iv = 1.0 / g.voxel[d];
        a.inv_voxel[d] = std::isfinite(iv) ? iv : 0.0;
        a.half_span_f[d] = (float)a.half_span[d];
        a.inv_voxel_f[d] = (float)a.inv_voxel[d];
        a.bmax[d] = g.coord_max[d] + g.voxel[d];
        a.bmin[d] = g.coord_min[d] - g.voxel[d];
        a.bmax_f[d] = (float)a.bmax[d];
        if (std::isfinite(a.bmax[d]) && (double)a.bmax_f[d] > a.bmax[d]) a.bmax_f[d] = std::nextafter(a.bmax_f[d], -INFINITY);
        a.bmin_f[d] = (float)a.bmin[d];
        if (std::isfinite(a.bmin[d]) && (double)a.bmin_f[d] < a.bmin[d]) a.bmin_f[d] = std::nextafter(a.bmin_f[d], INFINITY);
    }
    a.h = (float)g.step_size;
    a.h_idx = (float)(g.step_size / g.voxel[0]);
    a.max_steps = g.max_num_step;
    a.check = g.num_step_per_exit_check;
    a.param = g.parametrization;
    a.solver = g.ode_solver;
    a.n_kind = p->med.index_kind;
    a.n_sur = p->med.n_sur; a.lune_R = p->med.lune_R; a.lune_p = p->med.lune_p;
    a.a_kind = p->med.atten_kind;
    a.a_val = p->med.atten_value; a.a_R = p->med.atten_R;
    a.energy0 = p->energy0;
    a.active = p->d_active;
    return a;
}

bool grid_symplectic(const RayArgs& a) {
    return a.n_kind == VAM_INDEX_GRID && a.a_kind == VAM_ALPHA_GRID && a.param == VAM_PARAM_PHYSICAL &&
           a.solver == VAM_ODE_SYMPLECTIC_EULER;
}

int64_t padded_voxels(const vam_ray_geom& g) { return (int64_t)(g.n_x + 2) * (g.n_y + 2) * (g.n_z + 2); }

// the padded 3-D path serves the grid / symplectic configuration once its padded fields exist
// (32-bit element offsets: fewer than 2^31 padded voxels)
bool padded_path(const vam_ray_plan* p, const RayArgs& a) {
    return grid_symplectic(a) && !a.twod && p->d_npad && p->d_apad && p->d_spad &&
           padded_voxels(p->g) < ((int64_t)1 << 31);
}

PadArgs make_pad_args(const vam_ray_plan* p) {
    PadArgs q;
    const int ny = p->g.n_y, nz = p->g.n_z;
    q.npad = p->d_npad;
    q.apad = p->d_apad;
    q.nsx = (ny + 1) * (nz + 1);
    q.nsy = nz + 1;
    q.psx = (ny + 2) * (nz + 2);
    q.psy = nz + 2;
    return q;
}

// one of the four instances (2-D / 3-D x run-time / fixed configuration) of a ray kernel
#define VAM_RAY_LAUNCH(K, nb, st, ...)                                                                  \
    do {                                                                                                \
        if (grid_symplectic(a)) {                                                                       \
            if (a.twod) K<true, kCfgGridSymplectic><<<nb, kRayThreads, 0, st>>>(__VA_ARGS__);           \
            else K<false, kCfgGridSymplectic><<<nb, kRayThreads, 0, st>>>(__VA_ARGS__);                 \
        } else {                                                                                        \
            if (a.twod) K<true, kCfgRuntime><<<nb, kRayThreads, 0, st>>>(__VA_ARGS__);                  \
            else K<false, kCfgRuntime><<<nb, kRayThreads, 0, st>>>(__VA_ARGS__);                        \
        }                                                                                               \
    } while (0)

int ew_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b > 4736 ? 4736 : (b < 1 ? 1 : b));
}

}  // namespace
}  // namespace vam

using namespace vam;

extern "C" int vam_ray_plan_create(const vam_ray_geom* geom, const float* x0, const float* v0, float energy0,
                                   vam_ray_plan** out) {
    clear_error();
    VAM_REQUIRE(geom && x0 && v0 && out, VAM_ERR_ARG, "vam_ray_plan_create: null argument");
    *out = nullptr;
    const vam_ray_geom& g = *geom;
    VAM_REQUIRE(g.n_x > 1 && g.n_y > 1 && g.n_z >= 1 && g.num_rays > 0, VAM_ERR_SHAPE,
                "vam_ray_plan_create: grid needs n_x, n_y >= 2, n_z >= 1 and num_rays > 0");
    VAM_REQUIRE(g.max_num_step >= 0 && g.num_step_per_exit_check >= 1, VAM_ERR_ARG,
                "vam_ray_plan_create: max_num_step >= 0 and num_step_per_exit_check >= 1 required");
    VAM_REQUIRE(g.parametrization >= 0 && g.parametrization <= 2 && g.ode_solver >= 0 && g.ode_solver <= 2, VAM_ERR_ARG,
                "vam_ray_plan_create: unknown parametrization or ode_solver");
    VAM_REQUIRE(std::isfinite(g.step_size) && g.step_size > 0.0 && g.voxel[0] > 0.0 && g.voxel[1] > 0.0,
                VAM_ERR_ARG, "vam_ray_plan_create: step size and voxel must be positive");
    VAM_REQUIRE(g.n_z > 1 ? (std::isfinite(g.voxel[2]) && g.voxel[2] > 0.0) : true, VAM_ERR_ARG,
                "vam_ray_plan_create: 3D grid needs a finite voxel[2]");
    VAM_REQUIRE((int64_t)g.n_x * g.n_y * g.n_z < ((int64_t)1 << 31), VAM_ERR_SHAPE,
                "vam_ray_plan_create: the grid must have fewer than 2^31 voxels");
    DeviceGuard dg(g.device);
    VAM_REQUIRE(dg.ok, VAM_ERR_CUDA, "vam_ray_plan_create: cannot select device");
    auto* p = new vam_ray_plan();
    std::memset(p, 0, sizeof(*p));
    p->g = g;
    p->energy0 = energy0;
    const size_t nv = (size_t)g.n_x * g.n_y * g.n_z;
    cudaError_t e = cudaMalloc(&p->d_x0, sizeof(float) * 3 * g.num_rays);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_v0, sizeof(float) * 3 * g.num_rays);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_scratch, sizeof(float) * nv);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_absorb, sizeof(float) * nv);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_active, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemcpy(p->d_x0, x0, sizeof(float) * 3 * g.num_rays, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_v0, v0, sizeof(float) * 3 * g.num_rays, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->d_active, 0, sizeof(unsigned long long));
    if (e == cudaSuccess && g.n_z > 1) {
        e = cudaMalloc(&p->d_spad, sizeof(float) * padded_voxels(g));
        if (e == cudaSuccess) e = cudaMemset(p->d_spad, 0, sizeof(float) * padded_voxels(g));
    }
    if (e != cudaSuccess) {
        vam_ray_plan_destroy(p);
        return set_error(VAM_ERR_NOMEM, std::string("vam_ray_plan_create: ") + cudaGetErrorString(e));
    }
    *out = p;
    return VAM_OK;
}

extern "C" int vam_ray_plan_destroy(vam_ray_plan* p) {
    if (!p) return VAM_OK;
    DeviceGuard dg(p->g.device);
    cudaFree(p->d_x0);
    cudaFree(p->d_v0);
    cudaFree(p->d_nfield);
    cudaFree(p->d_afield);
    cudaFree(p->d_absorb);
    cudaFree(p->d_scratch);
    cudaFree(p->d_npad);
    cudaFree(p->d_apad);
    cudaFree(p->d_spad);
    cudaFree(p->d_active);
    cudaFree(p->d_traj);
    cudaFree(p->d_traj_len);
    cudaFree(p->d_traj_active);
    delete p;
    return VAM_OK;
}

extern "C" int vam_ray_set_medium(vam_ray_plan* p, const vam_ray_medium* m, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && m, VAM_ERR_ARG, "vam_ray_set_medium: null argument");
    VAM_REQUIRE(m->index_kind >= 0 && m->index_kind <= 2 && m->atten_kind >= 0 && m->atten_kind <= 3, VAM_ERR_ARG,
                "vam_ray_set_medium: unknown index or attenuation kind");
    VAM_REQUIRE(m->absorb_at_grid_dev, VAM_ERR_ARG, "vam_ray_set_medium: absorb_at_grid_dev is required");
    DeviceGuard dg(p->g.device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nv = (int64_t)p->g.n_x * p->g.n_y * p->g.n_z;
    if (m->index_kind == VAM_INDEX_GRID) {
        VAM_REQUIRE(m->n_grid_dev && m->grad_n_grid_dev, VAM_ERR_ARG, "vam_ray_set_medium: GRID index needs n and grad n");
        if (!p->d_nfield) VAM_TRY_CUDA(cudaMalloc(&p->d_nfield, sizeof(float4) * nv));
        k_pack_n<<<ew_blocks(nv), 256, 0, st>>>(m->n_grid_dev, m->grad_n_grid_dev, p->d_nfield, nv);
        VAM_CHECK_LAUNCH("k_pack_n");
        if (p->g.n_z > 1) {
            const int64_t np = (int64_t)(p->g.n_x + 1) * (p->g.n_y + 1) * (p->g.n_z + 1);
            if (!p->d_npad) VAM_TRY_CUDA(cudaMalloc(&p->d_npad, sizeof(float4) * np));
            k_pad_n<<<ew_blocks(np), 256, 0, st>>>(p->d_nfield, p->d_npad, p->g.n_x, p->g.n_y, p->g.n_z);
            VAM_CHECK_LAUNCH("k_pad_n");
        }
    } else {
        VAM_REQUIRE(std::isfinite(m->n_sur) && m->n_sur > 0.f, VAM_ERR_ARG, "vam_ray_set_medium: n_sur must be > 0");
    }
    if (m->atten_kind == VAM_ALPHA_GRID) {
        VAM_REQUIRE(m->atten_grid_dev, VAM_ERR_ARG, "vam_ray_set_medium: GRID attenuation needs atten_grid_dev");
        if (!p->d_afield) VAM_TRY_CUDA(cudaMalloc(&p->d_afield, sizeof(float) * nv));
        VAM_TRY_CUDA(cudaMemcpyAsync(p->d_afield, m->atten_grid_dev, sizeof(float) * nv, cudaMemcpyDeviceToDevice, st));
        if (p->g.n_z > 1) {
            const int64_t np = padded_voxels(p->g);
            if (!p->d_apad) VAM_TRY_CUDA(cudaMalloc(&p->d_apad, sizeof(float) * np));
            VAM_TRY_CUDA(cudaMemsetAsync(p->d_apad, 0, sizeof(float) * np, st));
            k_pad_mul<<<ew_blocks(nv), 256, 0, st>>>(p->d_afield, nullptr, p->d_apad, p->g.n_x, p->g.n_y, p->g.n_z);
            VAM_CHECK_LAUNCH("k_pad_mul");
        }
    }
    VAM_TRY_CUDA(cudaMemcpyAsync(p->d_absorb, m->absorb_at_grid_dev, sizeof(float) * nv, cudaMemcpyDeviceToDevice, st));
    p->med = *m;
    p->med.n_grid_dev = p->med.grad_n_grid_dev = p->med.atten_grid_dev = p->med.absorb_at_grid_dev = nullptr;
    p->has_medium = 1;
    p->traj_valid = 0;  // the paths follow the medium: a cached trajectory set is stale now
    return VAM_OK;
}

extern "C" int vam_ray_integrate(vam_ray_plan* p, const float* f, float* g, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && f && g, VAM_ERR_ARG, "vam_ray_integrate: null argument");
    VAM_REQUIRE(p->has_medium, VAM_ERR_ARG, "vam_ray_integrate: no medium bound (vam_ray_set_medium)");
    DeviceGuard dg(p->g.device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nv = (int64_t)p->g.n_x * p->g.n_y * p->g.n_z;
    VAM_TRY_CUDA(cudaMemsetAsync(p->d_active, 0, sizeof(unsigned long long), st));
    RayArgs a = make_args(p);
    const unsigned nb = (unsigned)((p->g.num_rays + kRayThreads - 1) / kRayThreads);
    if (padded_path(p, a)) {
        // a deposit leaves values in the border of d_spad: zero it, then write the interior
        VAM_TRY_CUDA(cudaMemsetAsync(p->d_spad, 0, sizeof(float) * padded_voxels(p->g), st));
        k_pad_mul<<<ew_blocks(nv), 256, 0, st>>>(f, p->d_absorb, p->d_spad, p->g.n_x, p->g.n_y, p->g.n_z);
        // the cached rays (0 .. traj_rays - 1) stream their records, the rest are traced; the count of
        // rays active at the cap starts from the cached rays' recorded count
        const int64_t m = p->traj_valid ? p->traj_rays : 0;
        if (m > 0) {
            VAM_TRY_CUDA(cudaMemcpyAsync(p->d_active, p->d_traj_active, sizeof(unsigned long long),
                                         cudaMemcpyDeviceToDevice, st));
            k_ray_integrate_traj<<<(unsigned)((m + kRayThreads - 1) / kRayThreads), kRayThreads, 0, st>>>(
                a, make_pad_args(p), p->d_traj, p->d_traj_len, p->d_spad, g, m);
            VAM_CHECK_LAUNCH("k_ray_integrate_traj");
        }
        if (m < p->g.num_rays) {
            k_ray_integrate_pad<<<(unsigned)((p->g.num_rays - m + kRayThreads - 1) / kRayThreads), kRayThreads, 0, st>>>(
                a, make_pad_args(p), p->d_spad, g, m);
            VAM_CHECK_LAUNCH("k_ray_integrate_pad");
        }
        return VAM_OK;
    }
    k_mul<<<ew_blocks(nv), 256, 0, st>>>(f, p->d_absorb, p->d_scratch, nv);
    VAM_RAY_LAUNCH(k_ray_integrate, nb, st, a, p->d_scratch, g);
    VAM_CHECK_LAUNCH("k_ray_integrate");
    return VAM_OK;
}

extern "C" int vam_ray_deposit(vam_ray_plan* p, const float* gin, float* dose, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && gin && dose, VAM_ERR_ARG, "vam_ray_deposit: null argument");
    VAM_REQUIRE(p->has_medium, VAM_ERR_ARG, "vam_ray_deposit: no medium bound (vam_ray_set_medium)");
    DeviceGuard dg(p->g.device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nv = (int64_t)p->g.n_x * p->g.n_y * p->g.n_z;
    VAM_TRY_CUDA(cudaMemsetAsync(p->d_active, 0, sizeof(unsigned long long), st));
    RayArgs a = make_args(p);
    const unsigned nb = (unsigned)((p->g.num_rays + kRayThreads - 1) / kRayThreads);
    if (padded_path(p, a)) {
        // deposits of corners outside the grid land in the zero border and are not copied out; the
        // border is zeroed again by the next call's memset
        VAM_TRY_CUDA(cudaMemsetAsync(p->d_spad, 0, sizeof(float) * padded_voxels(p->g), st));
        const int64_t m = p->traj_valid ? p->traj_rays : 0;
        if (m > 0) {
            VAM_TRY_CUDA(cudaMemcpyAsync(p->d_active, p->d_traj_active, sizeof(unsigned long long),
                                         cudaMemcpyDeviceToDevice, st));
            k_ray_deposit_traj<<<(unsigned)((m + kRayThreads - 1) / kRayThreads), kRayThreads, 0, st>>>(
                a, make_pad_args(p), p->d_traj, p->d_traj_len, gin, p->d_spad, m);
            VAM_CHECK_LAUNCH("k_ray_deposit_traj");
        }
        if (m < p->g.num_rays) {
            k_ray_deposit_pad<<<(unsigned)((p->g.num_rays - m + kRayThreads - 1) / kRayThreads), kRayThreads, 0, st>>>(
                a, make_pad_args(p), gin, p->d_spad, m);
            VAM_CHECK_LAUNCH("k_ray_deposit_pad");
        }
        k_unpad_mul<<<ew_blocks(nv), 256, 0, st>>>(p->d_spad, p->d_absorb, dose, p->g.n_x, p->g.n_y, p->g.n_z);
        VAM_CHECK_LAUNCH("k_unpad_mul");
        return VAM_OK;
    }
    VAM_TRY_CUDA(cudaMemsetAsync(p->d_scratch, 0, sizeof(float) * nv, st));
    VAM_RAY_LAUNCH(k_ray_deposit, nb, st, a, gin, p->d_scratch);
    VAM_CHECK_LAUNCH("k_ray_deposit");
    k_mul<<<ew_blocks(nv), 256, 0, st>>>(p->d_scratch, p->d_absorb, dose, nv);
    VAM_CHECK_LAUNCH("k_mul");
    return VAM_OK;
}

extern "C" int vam_ray_grad_alpha(vam_ray_plan* p, const float* f, const float* w, float* grad_att, float* grad_abs,
                                  vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && f && w, VAM_ERR_ARG, "vam_ray_grad_alpha: null argument");
    VAM_REQUIRE(p->has_medium, VAM_ERR_ARG, "vam_ray_grad_alpha: no medium bound (vam_ray_set_medium)");
    VAM_REQUIRE(!grad_att || p->med.atten_kind == VAM_ALPHA_GRID, VAM_ERR_NOTSUP,
                "vam_ray_grad_alpha: grad_att needs a GRID attenuation");
    DeviceGuard dg(p->g.device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nv = (int64_t)p->g.n_x * p->g.n_y * p->g.n_z;
    RayArgs a = make_args(p);
    const unsigned nb = (unsigned)((p->g.num_rays + kRayThreads - 1) / kRayThreads);
    if (grad_att) {
        k_mul<<<ew_blocks(nv), 256, 0, st>>>(f, p->d_absorb, p->d_scratch, nv);
        VAM_RAY_LAUNCH(k_ray_grad_att, nb, st, a, p->d_scratch, w, grad_att);
        VAM_CHECK_LAUNCH("k_ray_grad_att");
    }
    if (grad_abs) {
        VAM_TRY_CUDA(cudaMemsetAsync(p->d_scratch, 0, sizeof(float) * nv, st));
        VAM_TRY_CUDA(cudaMemsetAsync(p->d_active, 0, sizeof(unsigned long long), st));
        // deposit of w with unit start energy, times the forward's energy0:
        // sum_r w_r * energy0 * exp(-att) * (h/voxel) * w_corner at every voxel
        VAM_RAY_LAUNCH(k_ray_deposit, nb, st, a, w, p->d_scratch);
        VAM_CHECK_LAUNCH("k_ray_deposit");
        k_mul_acc<<<ew_blocks(nv), 256, 0, st>>>(p->d_scratch, f, p->energy0, grad_abs, nv);
        VAM_CHECK_LAUNCH("k_mul_acc");
    }
    return VAM_OK;
}

extern "C" int vam_ray_active_at_cap(vam_ray_plan* p, int64_t* out) {
    clear_error();
    VAM_REQUIRE(p && out, VAM_ERR_ARG, "vam_ray_active_at_cap: null argument");
    DeviceGuard dg(p->g.device);
    unsigned long long v = 0;
    VAM_TRY_CUDA(cudaMemcpy(&v, p->d_active, sizeof(v), cudaMemcpyDeviceToHost));
    *out = (int64_t)v;
    return VAM_OK;
}

extern "C" int vam_ray_prepare_trajectories(vam_ray_plan* p, int64_t limit_bytes, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_ray_prepare_trajectories: null plan");
    VAM_REQUIRE(p->has_medium, VAM_ERR_ARG, "vam_ray_prepare_trajectories: no medium bound (vam_ray_set_medium)");
    DeviceGuard dg(p->g.device);
    RayArgs a = make_args(p);
    VAM_REQUIRE(padded_path(p, a), VAM_ERR_NOTSUP,
                "vam_ray_prepare_trajectories: serves 3-D grid media with the physical path length and the "
                "symplectic Euler solver");
    const size_t steps = (size_t)std::max(a.max_steps, 1);
    const size_t per_ray = sizeof(float4) * steps + sizeof(int);
    VAM_REQUIRE(limit_bytes >= 0, VAM_ERR_ARG, "vam_ray_prepare_trajectories: negative byte limit");
    // every ray when they all fit, else the largest multiple of 32 rays (whole warps) from ray 0
    int64_t m = (int64_t)std::min<size_t>((size_t)p->g.num_rays, (size_t)limit_bytes / per_ray);
    if (m < p->g.num_rays) m -= m % 32;
    VAM_REQUIRE(m > 0, VAM_ERR_NOTSUP,
                "vam_ray_prepare_trajectories: one warp of rays needs " + std::to_string(per_ray * 32) +
                    " bytes, over the limit");
    const size_t bytes = per_ray * (size_t)m;
    p->traj_valid = 0;
    if (p->traj_bytes != bytes) {
        cudaFree(p->d_traj);
        cudaFree(p->d_traj_len);
        p->d_traj = nullptr;
        p->d_traj_len = nullptr;
        p->traj_bytes = 0;
        p->traj_valid = 0;
        cudaError_t e = cudaMalloc(&p->d_traj, sizeof(float4) * steps * (size_t)m);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_traj_len, sizeof(int) * (size_t)m);
        if (e != cudaSuccess) {
            cudaFree(p->d_traj);
            cudaFree(p->d_traj_len);
            p->d_traj = nullptr;
            p->d_traj_len = nullptr;
            cudaGetLastError();
            return set_error(VAM_ERR_NOMEM, std::string("vam_ray_prepare_trajectories: ") + cudaGetErrorString(e));
        }
        p->traj_bytes = bytes;
    }
    if (!p->d_traj_active) VAM_TRY_CUDA(cudaMalloc(&p->d_traj_active, sizeof(unsigned long long)));
    cudaStream_t st = (cudaStream_t)stream;
    VAM_TRY_CUDA(cudaMemsetAsync(p->d_traj_active, 0, sizeof(unsigned long long), st));
    const unsigned nb = (unsigned)((m + kRayThreads - 1) / kRayThreads);
    k_ray_record_pad<<<nb, kRayThreads, 0, st>>>(a, make_pad_args(p), p->d_traj, p->d_traj_len, p->d_traj_active, m);
    VAM_CHECK_LAUNCH("k_ray_record_pad");
    p->traj_rays = m;
    p->traj_valid = 1;
    return VAM_OK;
}

extern "C" int vam_ray_drop_trajectories(vam_ray_plan* p) {
    clear_error();
    VAM_REQUIRE(p, VAM_ERR_ARG, "vam_ray_drop_trajectories: null plan");
    DeviceGuard dg(p->g.device);
    cudaFree(p->d_traj);
    cudaFree(p->d_traj_len);
    p->d_traj = nullptr;
    p->d_traj_len = nullptr;
    p->traj_bytes = 0;
    p->traj_rays = 0;
    p->traj_valid = 0;
    return VAM_OK;
}

extern "C" int vam_ray_record_count(vam_ray_plan* p, int64_t* row_nnz, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && row_nnz, VAM_ERR_ARG, "vam_ray_record_count: null argument");
    VAM_REQUIRE(p->has_medium, VAM_ERR_ARG, "vam_ray_record_count: no medium bound (vam_ray_set_medium)");
    DeviceGuard dg(p->g.device);
    cudaStream_t st = (cudaStream_t)stream;
    RayArgs a = make_args(p);
    const unsigned nb = (unsigned)((p->g.num_rays + kRayThreads - 1) / kRayThreads);
    VAM_RAY_LAUNCH(k_ray_record, nb, st, a, p->d_absorb, row_nnz, nullptr, nullptr, nullptr);
    VAM_CHECK_LAUNCH("k_ray_record");
    return VAM_OK;
}

extern "C" int vam_ray_record_fill(vam_ray_plan* p, const int64_t* row_ptr, int32_t* cols, float* vals,
                                   vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && row_ptr && cols && vals, VAM_ERR_ARG, "vam_ray_record_fill: null argument");
    VAM_REQUIRE(p->has_medium, VAM_ERR_ARG, "vam_ray_record_fill: no medium bound (vam_ray_set_medium)");
    VAM_REQUIRE((int64_t)p->g.n_x * p->g.n_y * p->g.n_z < ((int64_t)1 << 31), VAM_ERR_SHAPE,
                "vam_ray_record_fill: column indices are 32-bit");
    DeviceGuard dg(p->g.device);
    cudaStream_t st = (cudaStream_t)stream;
    RayArgs a = make_args(p);
    const unsigned nb = (unsigned)((p->g.num_rays + kRayThreads - 1) / kRayThreads);
    VAM_RAY_LAUNCH(k_ray_record, nb, st, a, p->d_absorb, nullptr, row_ptr, cols, vals);
    VAM_CHECK_LAUNCH("k_ray_record");
    return VAM_OK;
}

extern "C" int vam_csr_spmm(int64_t nrows, const int64_t* row_ptr, const int32_t* cols, const float* vals,
                            const float* x, int32_t ztile, float* y, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(row_ptr && x && y && (cols || nrows == 0) && (vals || nrows == 0), VAM_ERR_ARG,
                "vam_csr_spmm: null argument");
    VAM_REQUIRE(nrows >= 0 && ztile >= 1, VAM_ERR_SHAPE, "vam_csr_spmm: nrows >= 0 and ztile >= 1 required");
    if (nrows == 0) return VAM_OK;
    const int64_t nb = (nrows + 7) / 8;
    VAM_REQUIRE(nb < ((int64_t)1 << 31), VAM_ERR_SHAPE, "vam_csr_spmm: too many rows");
    const int vec4 = ztile % 4 == 0 && (((uintptr_t)x | (uintptr_t)y) & 15) == 0;
    k_csr_spmm<<<(unsigned)nb, 256, 0, (cudaStream_t)stream>>>(nrows, row_ptr, cols, vals, x, ztile, y, vec4);
    VAM_CHECK_LAUNCH("k_csr_spmm");
    return VAM_OK;
}
