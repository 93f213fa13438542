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

// Bilinear tap helper on an [n0][n1] plane with strides s0, s1 (elements),
// zero outside.  Returns the weighted sum.
__device__ __forceinline__ float bilerp(const float* __restrict__ base, float f0, float f1, int n0, int n1,
                                        size_t s0, size_t s1) {
    const float g0 = floorf(f0), g1 = floorf(f1);
    const int i0 = (int)g0, i1 = (int)g1;
    const float t0 = f0 - g0, t1 = f1 - g1;
    const bool a0 = i0 >= 0 && i0 < n0, b0 = i0 + 1 >= 0 && i0 + 1 < n0;
    const bool a1 = i1 >= 0 && i1 < n1, b1 = i1 + 1 >= 0 && i1 + 1 < n1;
    const float* p = base + (ptrdiff_t)i0 * (ptrdiff_t)s0 + (ptrdiff_t)i1 * (ptrdiff_t)s1;
    const float x00 = (a0 && a1) ? __ldg(p) : 0.f;
    const float x01 = (a0 && b1) ? __ldg(p + s1) : 0.f;
    const float x10 = (b0 && a1) ? __ldg(p + s0) : 0.f;
    const float x11 = (b0 && b1) ? __ldg(p + s0 + s1) : 0.f;
    return (1.f - t0) * ((1.f - t1) * x00 + t1 * x01) + t0 * ((1.f - t1) * x10 + t1 * x11);
}

// Linear interpolation along one axis (slice-exact geometries: the other
// in-plane coordinate is an integer voxel index on every sample).
__device__ __forceinline__ float lerp1(const float* __restrict__ base, float f, int n, size_t s) {
    const float g = floorf(f);
    const int i0 = (int)g;
    const float t = f - g;
    const float x0 = (i0 >= 0 && i0 < n) ? __ldg(base + (ptrdiff_t)i0 * (ptrdiff_t)s) : 0.f;
    const float x1 = (i0 + 1 >= 0 && i0 + 1 < n) ? __ldg(base + (ptrdiff_t)(i0 + 1) * (ptrdiff_t)s) : 0.f;
    return (1.f - t) * x0 + t * x1;
}

// Forward: one thread per detector pixel (c, a, r), r fastest.  FLAT: every
// ray stays in the slice k = r (no inclination), the in-plane z coordinate
// is exact and only the horizontal axis is interpolated.
template <bool FLAT>
__global__ void __launch_bounds__(kThreads) k_vec_forward(const float* __restrict__ vol, float* __restrict__ sino,
                                                          const FwdAngle* __restrict__ ang, int nY, int nX, int nZ,
                                                          int nU, int nA, int nV) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    const int c = blockIdx.z;
    if (r >= nV) return;
    const FwdAngle g = ang[a];
    const size_t sI = (size_t)nX * nZ, sJ = (size_t)nZ, sK = 1;
    const float fc = (float)c, fr = (float)r;
    float acc = 0.f;
    if (g.axis == 0) {            // planes across i; in-plane (j, k)
        const float j0 = affine(g.p0, fc, fr, 0.f), k0 = affine(g.p1, fc, fr, 0.f);
#pragma unroll 4
        for (int s = 0; s < nY; ++s) {
            const float fj = fmaf(g.p0[3], (float)s, j0);
            const float* pl = vol + (size_t)s * sI;
            if (FLAT)
                acc += lerp1(pl + (size_t)r * sK, fj, nX, sJ);
            else
                acc += bilerp(pl, fj, fmaf(g.p1[3], (float)s, k0), nX, nZ, sJ, sK);
        }
    } else if (g.axis == 1) {     // planes across j; in-plane (i, k)
        const float i0 = affine(g.p0, fc, fr, 0.f), k0 = affine(g.p1, fc, fr, 0.f);
#pragma unroll 4
        for (int s = 0; s < nX; ++s) {
            const float fi = fmaf(g.p0[3], (float)s, i0);
            const float* pl = vol + (size_t)s * sJ;
            if (FLAT)
                acc += lerp1(pl + (size_t)r * sK, fi, nY, sI);
            else
                acc += bilerp(pl, fi, fmaf(g.p1[3], (float)s, k0), nY, nZ, sI, sK);
        }
    } else {                      // planes across k; in-plane (i, j)
        const float i0 = affine(g.p0, fc, fr, 0.f), j0 = affine(g.p1, fc, fr, 0.f);
        for (int s = 0; s < nZ; ++s)
            acc += bilerp(vol + (size_t)s * sK, fmaf(g.p0[3], (float)s, i0), fmaf(g.p1[3], (float)s, j0), nY, nX,
                          sI, sJ);
    }
    sino[((size_t)c * nA + a) * nV + r] = acc * g.scale;
}

// Backward: one thread per voxel (i, j, k), k fastest; angles looped.
// FLAT: the detector row of voxel slice k is exactly k.
template <bool FLAT>
__global__ void __launch_bounds__(kThreads) k_vec_backward(const float* __restrict__ sino, float* __restrict__ vol,
                                                           const BwdAngle* __restrict__ ang, int nY, int nX, int nZ,
                                                           int nU, int nA, int nV) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if (k >= nZ) return;
    const float fi = (float)i, fj = (float)j, fk = (float)k;
    const size_t sC = (size_t)nA * nV, sA = (size_t)nV;
    float acc = 0.f;
#pragma unroll 4
    for (int a = 0; a < nA; ++a) {
        const BwdAngle g = ang[a];
        const float fu = affine(g.u, fi, fj, fk);
        const float* pl = sino + (size_t)a * sA;
        if (FLAT)
            acc += lerp1(pl + k, fu, nU, sC);
        else
            acc += bilerp(pl, fu, affine(g.v, fi, fj, fk), nU, nV, sC, 1);
    }
    vol[((size_t)i * nX + j) * nZ + k] = acc;
}

}  // namespace

struct vam_vec_plan {
    int nY, nX, nZ, nU, nA, nV, device;
    bool flat_fwd, flat_bwd;
    FwdAngle* d_fwd;
    BwdAngle* d_bwd;
};

namespace {

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
    const double cx = 0.5 - nY / 2.0, cy = 0.5 - nX / 2.0, cz = 0.5 - nZ / 2.0;   // voxel (0,0,0) centre
    std::vector<FwdAngle> fw(nA);
    std::vector<BwdAngle> bw(nA);
    bool flat_f = true, flat_b = true;
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
        if (!(ax != 2 && g.p1[0] == 0.f && g.p1[1] == 0.f && g.p1[2] == 1.f && g.p1[3] == 0.f)) flat_f = false;
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
        if (!(h.v[0] == 0.f && h.v[1] == 0.f && h.v[2] == 0.f && h.v[3] == 1.f)) flat_b = false;
    }
    if (nV != nZ) flat_f = flat_b = false;
    vam::DeviceGuard dg(geom->device);
    VAM_REQUIRE(dg.ok, VAM_ERR_CUDA, "vam_vec_plan_create: cannot select the device");
    vam_vec_plan* p = new vam_vec_plan{nY, nX, nZ, nU, nA, nV, geom->device, flat_f, flat_b, nullptr, nullptr};
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
    dim3 grid((p->nV + kThreads - 1) / kThreads, p->nA, p->nU);
    if (p->flat_fwd)
        k_vec_forward<true><<<grid, kThreads, 0, (cudaStream_t)stream>>>(vol, sino, p->d_fwd, p->nY, p->nX, p->nZ,
                                                                        p->nU, p->nA, p->nV);
    else
        k_vec_forward<false><<<grid, kThreads, 0, (cudaStream_t)stream>>>(vol, sino, p->d_fwd, p->nY, p->nX, p->nZ,
                                                                         p->nU, p->nA, p->nV);
    VAM_CHECK_LAUNCH("vam_vec_forward");
    return VAM_OK;
}

extern "C" int vam_vec_backward(vam_vec_plan* p, const float* sino, float* vol, vam_stream_t stream) {
    clear_error();
    VAM_REQUIRE(p && vol && sino, VAM_ERR_ARG, "vam_vec_backward: null argument");
    vam::DeviceGuard dg(p->device);
    dim3 grid((p->nZ + kThreads - 1) / kThreads, p->nX, p->nY);
    if (p->flat_bwd)
        k_vec_backward<true><<<grid, kThreads, 0, (cudaStream_t)stream>>>(sino, vol, p->d_bwd, p->nY, p->nX, p->nZ,
                                                                         p->nU, p->nA, p->nV);
    else
        k_vec_backward<false><<<grid, kThreads, 0, (cudaStream_t)stream>>>(sino, vol, p->d_bwd, p->nY, p->nX, p->nZ,
                                                                          p->nU, p->nA, p->nV);
    VAM_CHECK_LAUNCH("vam_vec_backward");
    return VAM_OK;
}
