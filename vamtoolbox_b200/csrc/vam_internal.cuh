// vam_internal.cuh -- shared definitions of the sm_100a projection core.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/vam.h"

namespace vam {

// Records the message of the failing call (thread-local) and returns code.
int set_error(int code, const std::string& msg);
void clear_error();

#define VAM_TRY_CUDA(call)                                                                     \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return ::vam::set_error(VAM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define VAM_CHECK_LAUNCH(name)                                                                 \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess)                                                                 \
            return ::vam::set_error(VAM_ERR_CUDA, std::string(name) + " launch: " + cudaGetErrorString(e_)); \
    } while (0)

#define VAM_REQUIRE(cond, code, msg)                                                           \
    do {                                                                                       \
        if (!(cond)) return ::vam::set_error((code), (msg));                                   \
    } while (0)

// Makes `device` current for the scope of an entry point and restores the
// caller's device on exit.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != device) ok = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

constexpr int kWarp = 32;

__host__ __device__ inline int ilog2_pow2(int v) {
    int r = 0;
    while ((1 << r) < v) ++r;
    return r;
}

}  // namespace vam

// Plan of the parallel-beam projector family (lives on one device).
struct vam_parallel_plan {
    int nY, nX, nZ, nA, C, device;
    double4* d_trig;        // per angle: cos, sin, m02, m12 (skimage warp matrix offsets)
    uint8_t* d_circle;      // [nY][nX], 1 inside the inscribed circle (util/data.py:14-40)
    int abs_mode;           // vam_absorption_mode
    float abs_alpha, abs_R;
    float* d_mask;          // [nY][nX] for VAM_ABS_MASK
    float* d_occ;           // [nR][nA][nZ] occlusion sinogram, NaN = none
    uint8_t* d_occ_flag;    // [nA][nZ] forward shadow gate
    int has_occ;
    // 0: the 3-D class's occlusion (Projector3DParallel.py:77-111, 192-201); 1: the 2-D class's
    // digitised occlusion (Projector2DParallel.py:70-143, 235-247), nZ == 1 only, whose
    // backprojection compares s against the float64 minima in d_occ64 ([nR][nA])
    int occ_mode;
    double* d_occ64;
    uint8_t* d_ones;        // [nY][nX] all ones: the circle table of a backprojection without clipping
    // angle tasks of the fast forward: (a, b) with b the angle 180 degrees from a
    // (both sampled from a's lattice), or b = -1 for an unpaired angle
    int2* d_tasks_paired;
    int n_tasks_paired;
    int2* d_tasks_single;   // (a, -1) for every angle
    float* d_vol_scratch;   // [nY][nX][nZ] masked copy of the input (VAM_ABS_MASK)
    int* d_status;          // error bits the kernels record (VAM_STATUS_*), read by vam_parallel_status
    int4* d_bwd_btab;       // [blocks inside][nA][2] 2 x 2 block bin table (k_bwd_btable)
    int* d_bwd_bcidx;       // [(nY + 1) / 2][(nX + 1) / 2] compact block index, -1 outside the circle
    float* d_img_pad;       // nZ == 1: [nY][nX rounded up to 4] staged image of the TMA-tiled 2-D forward
    // matched-transpose weights: per pixel and angle, the first of <= 3
    // detector rows (as int bits) and their summed forward tap weights
    float4* d_adj_table;    // [nY*nX][nA]
    int adj_table_abs;      // absorption mode the table was built for (-1: none built)
    // reference-parity backprojection bins (k_bwd_btable): the clip circle's compact pixel index
    // (-1 outside) from which the block table is built
    int* d_bwd_cidx;
    // tuning (vam_parallel_set_tuning): vector widths 0 = automatic
    int tune_fwd_vz, tune_bwd_vz, tune_adj_vz, tune_bwd_batch, tune_adj_table, tune_bwd_table, tune_fwd_tma;
};
