/*
 * vam.h -- C ABI of the B200 (sm_100a) tomographic projection core.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream, returns an
 * int status (VAM_OK == 0) and is stream-ordered: nothing blocks the host, no
 * entry point allocates device memory after plan creation, so every compute
 * call may be captured in a CUDA graph.  Device pointers are marked `_dev`;
 * everything else is host memory.  `vam_stream_t` is ABI-compatible with
 * `cudaStream_t` (pass 0 for the legacy default stream).
 *
 * Array layouts follow the reference toolbox (C order, last index fastest):
 *   target volume      x[nY][nX][nZ]        (vamtoolbox/geometry.py:224)
 *   parallel sinogram  b[nR][nA][nZ], nR=nY (vamtoolbox/projector/Projector3DParallel.py:129-131)
 *   ray-traced grid    f[nX][nY][nZ]        (vamtoolbox/medium.py:37-40, xg shape)
 *   ray sinogram       g[nR*nA*nZr]         (vamtoolbox/projector/pyTorchRayTrace.py:1629-1632)
 */
#ifndef VAM_H
#define VAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* vam_stream_t;

enum vam_status {
    VAM_OK = 0,
    VAM_ERR_ARG = 1,      /* null pointer, bad enum, non-finite parameter      */
    VAM_ERR_SHAPE = 2,    /* inconsistent or unsupported sizes                  */
    VAM_ERR_CUDA = 3,     /* a CUDA runtime call failed (message has the name)  */
    VAM_ERR_TIMEOUT = 4,  /* a bounded device wait ran out                      */
    VAM_ERR_NOTSUP = 5,   /* option combination not implemented                 */
    VAM_ERR_NOMEM = 6     /* plan-time allocation failed                        */
};

/* Message of the last failing call on the calling host thread ("" if none). */
const char* vam_last_error_string(void);
/* Library version string, e.g. "vamcore 1.0 sm_100a". */
const char* vam_version(void);

/* ======================================================================= */
/* Parallel-beam projector family                                          */
/* ======================================================================= */

typedef struct vam_parallel_plan vam_parallel_plan;

typedef struct {
    int32_t n_y, n_x, n_z;     /* target array shape; the reference requires n_x == n_y */
    int32_t n_angles;
    const double* angles_deg;  /* host, n_angles projection angles in degrees */
    int32_t device;            /* CUDA device ordinal the plan lives on */
} vam_parallel_geom;

/* Builds per-angle tables (cos, sin, warp offsets), the inscribed-circle mask
 * and the workspace.  Replaces the constructor of
 * Projector3DParallelPython (vamtoolbox/projector/Projector3DParallel.py:57-75)
 * and Projector2DParallelPython (Projector2DParallel.py:47-68). */
int vam_parallel_plan_create(const vam_parallel_geom* geom, vam_parallel_plan** out);
int vam_parallel_plan_destroy(vam_parallel_plan* plan);

enum vam_absorption_mode {
    VAM_ABS_NONE = 0,
    VAM_ABS_MASK = 1,  /* radial mask exp(-a(R-r)): vamtoolbox/geometry.py:161-193,
                          applied as in Projector3DParallel.py:28-29,51-52          */
    VAM_ABS_RAY = 2    /* per-sample exp(-a*max(0, s - s_entry(t))), s_entry = -sqrt(R^2-t^2),
                          zero for |t|>R: the ray model of astra3Dabsorption.py:129-145
                          expressed in the projector's own (t, s) frame               */
};

/* Absorption weighting used by forward / backward_ref / adjoint.
 * MASK: mask_dev is an [nY][nX] device array (broadcast over z), copied.
 * RAY : alpha_per_px (1/pixel) and radius_px (container radius in pixels). */
int vam_parallel_set_absorption(vam_parallel_plan* plan, int mode, const float* mask_dev,
                                float alpha_per_px, float radius_px, vam_stream_t stream);

/* Occlusion from an attenuation field / insert: insert_dev is [nY][nX][nZ];
 * voxels > 0 are opaque.  Builds the occlusion sinogram of
 * Projector3DParallelPython.generateOccSinogram (Projector3DParallel.py:77-111)
 * on the device; later forward/backward_ref/adjoint calls apply the shadow
 * (Projector3DParallel.py:147-153, 192-201, 209-216). */
int vam_parallel_set_occlusion(vam_parallel_plan* plan, const float* insert_dev, vam_stream_t stream);
/* The 2-D class's digitised occlusion (Projector2DParallelPython.generateOccSinogram,
 * Projector2DParallel.py:70-143) for a plan with n_z == 1: occlusion_dev is
 * [nY][nX] bytes, nonzero = occluded.  Per angle each occluded pixel's
 * detector coordinate t = x cos - y sin is binned with np.digitize over the
 * detector axis and each bin keeps its least s = x sin + y cos, assigned to
 * the bins in the reference's order (a coordinate below the first bin counts
 * as the last bin's value).  Later forward / adjoint calls zero samples past
 * the bin's minimum (Projector2DParallel.py:145-186); backward_ref zeroes
 * pixels whose s exceeds the minimum of t's bin (getOccShadow, :235-247).
 * Reads back an error flag, so it synchronises the stream.  VAM_ERR_SHAPE
 * where the reference raises ValueError: an empty occlusion, or occluded
 * pixels below the first bin and in the last bin at one angle. */
int vam_parallel_set_occlusion_2d(vam_parallel_plan* plan, const uint8_t* occlusion_dev, vam_stream_t stream);
/* Copies the float64 bin minima of the digitised 2-D occlusion ([nY][nA], NaN
 * where a bin holds no occluded pixel: the reference's occ_sinogram) into
 * out_dev.  VAM_ERR_ARG unless vam_parallel_set_occlusion_2d succeeded. */
int vam_parallel_get_occlusion_sinogram_2d(vam_parallel_plan* plan, double* out_dev, vam_stream_t stream);
int vam_parallel_clear_occlusion(vam_parallel_plan* plan);
/* Copies the occlusion sinogram ([nR][nA][nZ], NaN where a column has no
 * occluder) into out_dev.  VAM_ERR_ARG if no occlusion is set. */
int vam_parallel_get_occlusion_sinogram(vam_parallel_plan* plan, float* out_dev, vam_stream_t stream);

/* Status bits kernels with bounded waits record in their plan. */
enum vam_status_bits {
    VAM_STATUS_TIMEOUT = 1  /* a block gave up waiting for its shared-memory copy and left its outputs
                               unwritten (a stalled copy; not expected in normal operation) */
};
/* Reads and clears the plan's status word (synchronises the device).  The 2-D
 * tile forward stages its image boxes with TMA copies waited on with a bounded
 * poll; a caller that must know every output was written checks this after
 * its calls. */
int vam_parallel_status(vam_parallel_plan* plan, int32_t* status);

/* Builds the plan's backprojection bin table: for every 2 x 2 block of pixels
 * with a pixel inside the clip circle and every angle, np.interp's bin of
 * t = x cos - y sin (float64, the reference's expression) of each of the four
 * pixels as the offset of the block's least bin row, a code of the pixels' bin
 * offsets and their float32 weights, 32 bytes per block and angle (148.5 MB at
 * 256^3 x 360).  Later backprojections (nZ % 4 == 0, no per-ray absorption)
 * read the table and share each block's at most four detector rows among its
 * pixels instead of evaluating the float64 bins (identical results).
 * Allocates: call before any stream capture.  VAM_ERR_NOTSUP when the plan's
 * sinogram has 2^31 elements or more, or nZ % 4 != 0. */
int vam_parallel_prepare_backward(vam_parallel_plan* plan, vam_stream_t stream);

/* R1 forward: rotate-and-sum Radon transform with bilinear sampling, zero
 * outside the image, detector width nY.  Replaces
 * Projector3DParallelPython.forward (Projector3DParallel.py:113-156). */
int vam_parallel_forward(vam_parallel_plan* plan, const float* vol_dev, float* sino_dev,
                         vam_stream_t stream);

/* R2 reference-parity backprojection: pixel-driven, linear interpolation
 * along the detector with zero outside (np.interp left=right=0), then the
 * inscribed-circle clip.  Replaces Projector3DParallelPython.backward
 * (Projector3DParallel.py:158-207).  Not the transpose of R1. */
int vam_parallel_backward_ref(vam_parallel_plan* plan, const float* sino_dev, float* vol_dev,
                              vam_stream_t stream);

/* R2 without the inscribed-circle clip: Projector2DParallelPython.backward(b,
 * clipping=False) (Projector2DParallel.py:188, 230-231).  The first call
 * allocates the plan's all-ones pixel table. */
int vam_parallel_backward_ref_noclip(vam_parallel_plan* plan, const float* sino_dev, float* vol_dev,
                                     vam_stream_t stream);

/* Matched transpose of R1 (<A x, y> == <x, A^T y>), gather form, no atomics.
 * No counterpart in the reference (its backward is R2); used for autograd. */
int vam_parallel_adjoint(vam_parallel_plan* plan, const float* sino_dev, float* vol_dev,
                         vam_stream_t stream);

/* Launch shapes of the parallel-beam kernels, chosen per problem by an
 * autotuner (vamtoolbox_b200/autotune.py times the candidates on the device
 * and caches the winner per device and problem shape).  Vector widths are the
 * slices each lane of a fast kernel carries (4 or 8; 1 = the generic kernel;
 * 0 = automatic; the fast kernels need nZ % 4 == 0; for a single slice any
 * value but 0 and 1 selects the shared-memory tile kernels, which 0 picks from
 * 192 (forward) and 320 (backprojection) pixels up); backward_batch is the
 * number of angles whose detector rows one warp loads together (1, 2 or 4);
 * adjoint_table selects the table-driven transpose once it is prepared.
 * No counterpart in the reference. */
typedef struct {
    int32_t forward_vz, backward_vz, adjoint_vz;
    int32_t backward_batch;
    int32_t adjoint_table;
    int32_t backward_table;  /* 1: the backprojection reads its bins from the plan's table
                                (vam_parallel_prepare_backward) when it is built, with backward_vz 4
                                or 8 slices per lane (0: 8 from 160 slices up); 0: computes them */
    int32_t forward_tma;     /* 1: the 2-D tile forward stages its boxes with TMA tensor copies (an image
                                whose rows are not 16-byte multiples, or in mask mode, is first copied
                                into the plan's padded image); 0: with plain loads.  Bit-identical. */
} vam_parallel_tuning;
int vam_parallel_set_tuning(vam_parallel_plan* plan, const vam_parallel_tuning* tuning);
int vam_parallel_get_tuning(vam_parallel_plan* plan, vam_parallel_tuning* tuning);

/* Batched calls over many plans (targets of uneven size, different angle
 * counts, 2-D slices next to 3-D volumes) in persistent launches fed by
 * device work queues: one launch per kernel-body family present in the list,
 * each compiled with only that family's bodies (their registers, their
 * occupancy).  Each work item is one forward / backward_ref / adjoint
 * call exactly as the single-plan entry points describe it, and produces
 * bit-identical results; items run concurrently, so no item may read another
 * item's output or write another item's input or output.  A forward that
 * stages its input in its plan's scratch (mask mode; a 2-D slice whose width
 * is not a multiple of four or whose input is not 16-byte aligned) makes that
 * plan appear at most once per batch with VAM_OP_FORWARD: a list with two
 * such calls of one plan is refused (VAM_ERR_ARG).
 *
 * The calls' descriptions travel by value in the launch's parameters (48
 * calls per launch; longer lists and further families become further
 * launches), so a submit makes no CUDA call but a counter reset, the launches
 * and an event fork / join: the launches after the first run on up to three
 * streams the batch owns, forked from the caller's stream and joined back to
 * it before the submit returns, so each launch fills the SMs the previous
 * one's tail frees.  A submit is therefore ordered on the caller's stream,
 * allocates nothing and may be captured in a CUDA graph with any list.  A
 * batch object (its queue counters and streams) is driven from one stream at
 * a time.
 *
 * Replaces running the reference's per-target projector calls one target at a
 * time (vamtoolbox/projector/Projector3DParallel.py:113-207 per target). */
typedef struct vam_batch vam_batch;
enum { VAM_OP_FORWARD = 0, VAM_OP_BACKWARD_REF = 1, VAM_OP_ADJOINT = 2 };
typedef struct {
    vam_parallel_plan* plan;
    int32_t op;        /* VAM_OP_* */
    const float* in;   /* volume (forward) or sinogram, device */
    float* out;        /* sinogram (forward) or volume, device */
} vam_work;
int vam_batch_create(int32_t device, vam_batch** out);
int vam_batch_destroy(vam_batch* batch);
int vam_batch_submit(vam_batch* batch, const vam_work* work, int32_t n, vam_stream_t stream);
/* validate and describe a work list without launching (reports a bad list before a capture) */
int vam_batch_prepare(vam_batch* batch, const vam_work* work, int32_t n, vam_stream_t stream);
/* blocks (over all calls' grids) of the last submitted list and persistent CTAs of its launch */
int vam_batch_info(vam_batch* batch, int64_t* virtual_blocks, int32_t* ctas);

/* Builds the plan's matched-transpose weight table (16 bytes per pixel and
 * angle: the detector rows that sample the pixel and their summed forward
 * weights), after which vam_parallel_adjoint is a pure gather.  Allocates;
 * call once before capturing adjoint calls in a graph, and again after
 * vam_parallel_set_absorption.  Without it the adjoint enumerates the
 * sampling lattice on the fly.  No counterpart in the reference. */
int vam_parallel_prepare_adjoint(vam_parallel_plan* plan, vam_stream_t stream);

/* ======================================================================= */
/* Curved-ray tracer (graded-index medium)                                 */
/* ======================================================================= */

typedef struct vam_ray_plan vam_ray_plan;

enum vam_ray_param { VAM_PARAM_PHYSICAL = 0, VAM_PARAM_CANONICAL = 1, VAM_PARAM_OPTICAL = 2 };
enum vam_ray_solver { VAM_ODE_SYMPLECTIC_EULER = 0, VAM_ODE_EULER = 1, VAM_ODE_LEAPFROG = 2 };
enum vam_index_kind { VAM_INDEX_HOMOGENEOUS = 0, VAM_INDEX_GRID = 1, VAM_INDEX_LUNEBURG = 2 };
enum vam_alpha_kind { VAM_ALPHA_ZERO = 0, VAM_ALPHA_CYLINDER = 1, VAM_ALPHA_BALL = 2, VAM_ALPHA_GRID = 3 };

typedef struct {
    int32_t n_x, n_y, n_z;      /* grid shape (nZ == 1 for a 2D problem) */
    double coord_min[3];        /* xv[0], yv[0], zv[0]   (vamtoolbox/medium.py:44-51) */
    double coord_max[3];        /* xv[-1], yv[-1], zv[-1] */
    double voxel[3];            /* xv[1]-xv[0] ...; voxel[2] = +inf in 2D (medium.py:52-56) */
    double step_size;           /* parameter step h (pyTorchRayTrace.py:44-46) */
    int32_t max_num_step;       /* step cap (pyTorchRayTrace.py:47-49) */
    int32_t num_step_per_exit_check; /* exit test cadence (pyTorchRayTrace.py:233) */
    int32_t parametrization;    /* enum vam_ray_param */
    int32_t ode_solver;         /* enum vam_ray_solver */
    int64_t num_rays;
    int32_t device;
} vam_ray_geom;

typedef struct {
    int32_t index_kind;         /* enum vam_index_kind (vamtoolbox/medium.py:276-473) */
    float n_sur;                /* homogeneous / Luneburg surround index */
    float lune_R, lune_p;       /* Luneburg radius (physical) and power */
    const float* n_grid_dev;    /* [nX][nY][nZ] index samples (GRID) */
    const float* grad_n_grid_dev; /* [nX][nY][nZ][3] gradient samples (GRID) */
    int32_t atten_kind;         /* enum vam_alpha_kind (medium.py:753-915) */
    float atten_value;          /* alpha_internal for CYLINDER / BALL */
    float atten_R;              /* physical radius for CYLINDER / BALL */
    const float* atten_grid_dev;/* [nX][nY][nZ] (GRID, zero padding) */
    const float* absorb_at_grid_dev; /* [nX][nY][nZ] absorption coefficient at the grid
                                        points: pyTorchRayTrace.py:458-462, 515-519 */
} vam_ray_medium;

/* Ray starting states: x0_dev, v0_dev are [num_rays][3] float32 (the
 * RayState.setupRaysParallel layout, pyTorchRayTrace.py:1515-1666), copied
 * into the plan; energy0 is the per-ray initial energy of the forward
 * (ray_density^-1 in 2D or ^-2 in 3D, :1682-1686).  The plan owns a grid-sized
 * scratch buffer and a float4 texel copy of the index field. */
int vam_ray_plan_create(const vam_ray_geom* geom, const float* x0_dev, const float* v0_dev,
                        float energy0, vam_ray_plan** out);
int vam_ray_plan_destroy(vam_ray_plan* plan);

/* Binds the medium (IndexModel / AttenuationModel / absorption at the grid
 * points, vamtoolbox/medium.py:276-915) to the plan: grid fields are copied
 * into the plan's packed layout, so later calls read the plan, not the
 * caller's buffers.  Call again after changing a field. */
int vam_ray_set_medium(vam_ray_plan* plan, const vam_ray_medium* medium, vam_stream_t stream);

/* R6 forward (integrate): g[r] = sum over steps and trilinear corners of
 * f[corner] * alpha_abs[corner] * (h/voxel_x) * w_corner * E(s).  Replaces
 * PyTorchRayTracingPropagator.forward (pyTorchRayTrace.py:87-107) ->
 * integrateEnergyUntilExit (:471-571).  f is not modified (the reference
 * multiplies its input in place, :515-519). */
int vam_ray_integrate(vam_ray_plan* plan, const float* f_dev, float* g_dev, vam_stream_t stream);

/* R5 adjoint (deposit): dose = alpha_abs * sum over rays/steps/corners of
 * g[r] * (h/voxel_x) * w_corner * E(s), accumulated with float32 atomics.
 * Replaces PyTorchRayTracingPropagator.backward (pyTorchRayTrace.py:109-133)
 * -> depositEnergyUntilExit (:378-469).  dose_dev is overwritten. */
int vam_ray_deposit(vam_ray_plan* plan, const float* g_dev, float* dose_dev, vam_stream_t stream);

/* Gradients of L = sum_r w[r] * integrate(f)[r]:
 *   grad_att_dev[v] += dL/d alpha_att[v]  (GRID attenuation only), through the
 *                      exp(-integral alpha ds) energy decay, each ray's path
 *                      traced twice (total, then suffix sums) instead of stored;
 *   grad_abs_dev[v] += dL/d alpha_abs[v] = f[v] * sum of the deposit of w at v.
 * Either output may be null.  No counterpart in the reference (it has no
 * differentiable ray tracer). */
int vam_ray_grad_alpha(vam_ray_plan* plan, const float* f_dev, const float* w_dev,
                       float* grad_att_dev, float* grad_abs_dev, vam_stream_t stream);

/* Number of rays still active when the step cap was reached in the last
 * integrate/deposit call (the reference logs an ERROR for this,
 * pyTorchRayTrace.py:464-467).  Synchronises the device. */
int vam_ray_active_at_cap(vam_ray_plan* plan, int64_t* out_count);

/* Trajectory cache of a plan on a 3-D grid medium with the physical path
 * length and the symplectic Euler solver: the rays are traced once (the same
 * steps and exit checks as vam_ray_integrate) and each executed step's
 * position x_ip1 and attenuance are kept, 16 bytes per ray and step
 * (max_num_step x num_rays x 16 B: 36 GB at 128^3 x 360 rays x 384 steps).
 * While it is valid, vam_ray_integrate and vam_ray_deposit stream the records
 * instead of re-tracing (bit-identical results); vam_ray_set_medium
 * invalidates it (prepare again to refresh it).  When not every ray fits in
 * limit_bytes (16 B per step of the cap plus 4 B per ray), the cache holds
 * rays 0 .. m - 1 for the largest multiple of 32 rays m that fits and the
 * remaining rays are traced every call (same results).  VAM_ERR_NOTSUP when
 * the configuration has no padded path or not even 32 rays fit,
 * VAM_ERR_NOMEM when the device cannot hold it (the plan then traces as
 * before).  Allocates: call before any stream capture.
 * vam_ray_drop_trajectories frees it.  The reference re-traces every call
 * (pyTorchRayTrace.py:378-571). */
int vam_ray_prepare_trajectories(vam_ray_plan* plan, int64_t limit_bytes, vam_stream_t stream);
int vam_ray_drop_trajectories(vam_ray_plan* plan);

/* The propagation matrix of vam_ray_integrate, one CSR row per ray, replacing
 * PyTorchRayTracingPropagator.buildPropagationMatrix / recordEnergyUntilExit
 * (vamtoolbox/projector/pyTorchRayTrace.py:169-197, 573-690, 901-937,
 * 1146-1252): row r lists, in step order, the voxels (C-order index over the
 * [n_x][n_y][n_z] grid) ray r deposits into, starting with the plan's
 * energy0, and the weights (h / voxel) * E * trilinear weight * absorption at
 * the voxel; a
 * voxel met twice appears twice (the reference sums them when it coalesces).
 * vam_ray_record_count writes row_nnz[num_rays] (device); the caller forms
 * row_ptr[num_rays + 1] (exclusive scan) and vam_ray_record_fill writes
 * cols / vals.  Column indices are 32-bit (grids below 2^31 voxels). */
int vam_ray_record_count(vam_ray_plan* plan, int64_t* row_nnz_dev, vam_stream_t stream);
int vam_ray_record_fill(vam_ray_plan* plan, const int64_t* row_ptr_dev, int32_t* cols_dev, float* vals_dev,
                        vam_stream_t stream);

/* y[row][z] = sum_k vals[k] * x[cols[k]][z] over the CSR row, for a dense x of
 * ztile columns per matrix column (the algebraic propagator's z tiling:
 * PyTorchAlgebraicPropagator.forward / backward,
 * vamtoolbox/projector/pyTorchAlgebraicPropagation.py:146-181; the backward
 * passes the transposed matrix in CSR form).  Deterministic. */
int vam_csr_spmm(int64_t nrows, const int64_t* row_ptr_dev, const int32_t* cols_dev, const float* vals_dev,
                 const float* x_dev, int32_t ztile, float* y_dev, vam_stream_t stream);

/* ======================================================================= */
/* Optimizer iteration bodies (vamtoolbox/optimizer/*.py)                   */
/* ======================================================================= */

/* Workspace for the reductions below, in bytes, for arrays of n elements. */
size_t vam_reduce_workspace_bytes(int64_t n);

enum vam_reduce_op { VAM_RED_MAX = 0, VAM_RED_MIN = 1, VAM_RED_SUM = 2 };

/* out_dev[0] = op over x[0..n) (float, deterministic two-level tree). */
int vam_reduce(const float* x_dev, int64_t n, int op, float* out_dev, void* work_dev,
               size_t work_bytes, vam_stream_t stream);

/* Sinogram filtering along the detector axis (vamtoolbox/util/data.py:302-370,
 * filterSinogram: zero-pad each detector column to a power of two >= 2 nR,
 * multiply its spectrum by the real filter of _get_fourier_filter, :373-438,
 * invert, crop).  The transforms are cuFFT's real-to-complex / complex-to-real
 * pair over the padded axis; these two kernels are the steps around them.
 * vam_spectrum_scale: spectrum_dev complex128 [n_freq][m] (re, im pairs),
 * row k multiplied in place by filter_dev[k] (float64). */
int vam_spectrum_scale(void* spectrum_dev, const double* filter_dev, int64_t n_freq, int64_t m,
                       vam_stream_t stream);
/* out_dev[r][j] = clip(scale * y_dev[r][j], lo, hi) as float32 for the first
 * n_rows rows of y_dev ([>= n_rows][m], float64): the crop of the padded
 * inverse transform, the reference's normalisations (BCLP's pi / (2 n_angles))
 * and constraints (clip at 0 / the bounds) in one pass.  has_lo / has_hi
 * select the bounds. */
int vam_filter_epilogue(const double* y_dev, int64_t n_rows, int64_t m, double scale, int has_lo, double lo,
                        int has_hi, double hi, float* out_dev, vam_stream_t stream);

/* Same reduction as vam_reduce for callers that cannot allocate device memory:
 * a printer host that reserves all device memory for its projection buffers
 * before a print starts, so cudaMalloc would fail, and that must not trigger
 * cudaMalloc's implicit device synchronisation while a layer is exposing; or
 * a plug-in that is handed fixed buffers and has no allocator of its own.  No counterpart in the
 * reference.  Its scratch is one static device array of 4096 doubles (32 KiB)
 * inside the library, held on every GPU that loads it until process exit; one
 * partial per 2048 inputs, so n is limited to 8388608 elements (larger n:
 * VAM_ERR_SHAPE, nothing launched).  Allocates nothing and calls no
 * allocating routine.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and loads the entry point's kernels for every
 * op; make that first call before any stream capture.  The address is cached
 * per device ordinal for the life of the process: after cudaDeviceReset on a
 * device the cached address is stale, so do not call this entry point on a
 * device that was reset after its first call.  All calls share the one array:
 * calls that overlap on the GPU (different streams, no ordering) race; each
 * call writes every partial it reads, so nothing carries over between calls. */
int vam_reduce_noalloc(const float* x_dev, int64_t n, int op, float* out_dev, vam_stream_t stream);

/* Volumetric error rate (vamtoolbox/metrics.py:47-87): out_dev[0] =
 * #(void >= min(gel)) / (#gel + #void).  mask_dev: 1 = gel, 2 = void, 0 = outside. */
int vam_metric_ver(const float* x_dev, const uint8_t* mask_dev, int64_t n, float* out_dev,
                   void* work_dev, size_t work_bytes, vam_stream_t stream);

/* In-part dose range (vamtoolbox/metrics.py:130-156, layerwise=False): out_dev[0] =
 * max(x[gel]) - min(x[gel]).  mask_dev as for vam_metric_ver.  With no gel voxel
 * out_dev[0] is NaN (the reference's np.min raises on the empty selection). */
int vam_metric_ipdr(const float* x_dev, const uint8_t* mask_dev, int64_t n, float* out_dev,
                    void* work_dev, size_t work_bytes, vam_stream_t stream);

/* Response model of the BCLP dose pass (vamtoolbox/response.py:12-399). */
enum vam_response_kind {
    VAM_RESP_TABLE = 0,     /* type="interpolation": np.interp on the table, nearest-value extrapolation */
    VAM_RESP_GLF = 1,       /* type="analytical", form="gen_log_fun": A + (K-A) / (1 + exp(-B(f-M)))^(1/nu) */
    VAM_RESP_LINEAR = 2,    /* type="analytical", form="linear": M f + C */
    VAM_RESP_IDENTITY = 3   /* type="analytical", form="identity": f */
};

/* BCLP state update, one pass over the dose (vamtoolbox/optimizer/BCLP.py:277-437):
 * mapped = response(dose), e = mapped - f_T,
 * eb = |e| - eps, v = eb > 0, operand = v*w*|eb|^(p-1)*sign(e)*dresponse(dose).
 * stats_dev[0..8] = { sum v*w*|eb|^p, l0, l0_eps0, l1, l1_eps0, l2^2, l2_eps0^2, lf, lf_eps0 }.
 * Scalars: eps / weight are arrays when eps_dev / weight_dev are non-null.
 * The response is the table (VAM_RESP_TABLE) or a closed form evaluated in
 * float64 per voxel (response.py:191-279: _map_glf / _dmapdf_glf, _map_lin /
 * _dmapdf_lin, _map_id / _dmapdf_id). */
typedef struct {
    const float* table_f;       /* device, n_table strictly increasing sample points */
    const float* table_map;     /* device, response at the sample points */
    const float* table_dmap;    /* device, derivative at the sample points */
    int32_t n_table;
    float table_f0;             /* table_f[0] (host copy, seeds the bin search) */
    float table_inv_step;       /* (n_table - 1) / (table_f[n-1] - table_f[0]) */
    float eps, weight, p;
    const float* eps_dev;       /* optional per-voxel eps */
    const float* weight_dev;    /* optional per-voxel weight */
    int32_t response;           /* vam_response_kind; the table fields are unused unless VAM_RESP_TABLE */
    double resp_A, resp_K, resp_B, resp_M, resp_nu;  /* VAM_RESP_GLF; VAM_RESP_LINEAR uses resp_M */
    double resp_C;              /* VAM_RESP_LINEAR offset */
} vam_bclp_params;

int vam_bclp_dose_pass(const float* dose_dev, const float* target_dev, int64_t n,
                       const vam_bclp_params* prm, float* mapped_dev, float* operand_dev,
                       float* stats_dev, void* work_dev, size_t work_bytes, vam_stream_t stream);

/* g = clip(g - lr * pref * grad, lo, hi) with pref = q*L^((q-p)/q), L =
 * stats_dev[0]^(q/p), and pref = 1 when L == 0 (BCLP.py:370-375, 477-534).
 * has_hi == 0 means no upper bound. */
int vam_bclp_sino_update(float* g_dev, const float* grad_dev, int64_t n, float lr, float p,
                         float q, float lo, float hi, int has_hi, const float* stats_dev,
                         vam_stream_t stream);

/* Elementwise helpers used by CAL / OSMO / PM iteration bodies. */
/* y = 1/(1+exp(-(x*scale_dev[0]^-1 - d)/g)) - t   (CAL.py:147-175 with x normalised by a device max) */
int vam_cal_threshold(const float* x_dev, const float* xmax_dev, const float* target_dev, int64_t n,
                      float d_h, float g, float* out_dev, vam_stream_t stream);
/* b = clip(b - lr*(db*(1-m) + db_prev*m/(1-m^(it+1))), 0)   (CAL.py:177-186) */
int vam_cal_sino_update(float* b_dev, const float* db_dev, const float* db_prev_dev, int64_t n,
                        float lr, float momentum, int32_t iter, vam_stream_t stream);
/* x = max(x/scale_dev[0], floor_val) when apply_floor, else x/scale_dev[0] */
int vam_scale_by_device(float* x_dev, const float* scale_dev, int64_t n, int apply_floor,
                        float floor_val, vam_stream_t stream);
/* OSMO model update (OSMO.py:36-109), with xn = x / xmax_dev[0] (xmax_dev may be
 * null when x is already normalised): gel voxels (mask == 1, gel != 0)
 * xm += max(d_h - xn, 0); void voxels (mask == 2, gel == 0) xm -= max(xn - d_l, 0). */
int vam_osmo_model_update(float* xm_dev, const float* x_dev, const float* xmax_dev,
                          const uint8_t* mask_dev, int64_t n, int gel, float d, vam_stream_t stream);

/* Graph-friendly log append: row = counter_dev[0]; if row < cap_rows,
 * arr_dev[row*n + i] = src_dev[i] for i < n; then counter_dev[0] += 1.  Lets a
 * captured iteration record per-iteration scalars (loss, norms, VER) without
 * per-iteration kernel arguments (BCLP.py LogPerf :14-135, CAL.py / OSMO.py error arrays). */
int vam_append(const float* src_dev, int32_t n, float* arr_dev, int32_t* counter_dev, int32_t cap_rows,
               vam_stream_t stream);

/* ======================================================================= */
/* Vector-geometry parallel beam: the model of the reference's CUDA path    */
/* (ASTRA parallel3d / parallel3d_vec, incl. inclined / laminography rays)  */
/* ======================================================================= */

typedef struct vam_vec_plan vam_vec_plan;

typedef struct {
    int32_t n_y, n_x, n_z;      /* target array [nY][nX][nZ] = ASTRA (col x, row y, slice z) */
    int32_t n_angles;
    int32_t det_cols, det_rows; /* detector nU x nV; the sinogram is [nU][nA][nV] */
    const double* vectors;      /* host, n_angles x 12: ray direction, detector centre, u (pixel (0,0)->(0,1)),
                                   v (pixel (0,0)->(1,0)), as the rows genVectorsAstra builds
                                   (vamtoolbox/projector/genVectorsAstra.py:4-53) */
    int32_t device;
} vam_vec_geom;

/* Per-angle affine sampling tables for the model of
 * Projector3DParallelCUDAAstra (vamtoolbox/projector/Projector3DParallelCUDA.py:13-72):
 * voxel (i, j, k) centred at (i + 0.5 - nY/2, j + 0.5 - nX/2, k + 0.5 - nZ/2),
 * detector pixel (c, r) at d + (c - nU/2 + 0.5) u + (r - nV/2 + 0.5) v.
 * VAM_ERR_ARG for a ray parallel to the detector plane. */
int vam_vec_plan_create(const vam_vec_geom* geom, vam_vec_plan** out);
int vam_vec_plan_destroy(vam_vec_plan* plan);
/* Whether forward / backward use the slice-exact kernels (no inclination). */
int vam_vec_plan_info(const vam_vec_plan* plan, int32_t* flat_forward, int32_t* flat_backward);

/* Line integrals, Joseph-type: every ray sampled on each voxel plane across
 * its dominant axis, bilinear in the plane (zero outside), times
 * |ray| / |ray_dominant|; replaces astra.create_sino3d_gpu
 * (Projector3DParallelCUDA.py:40-54).  vol [nY][nX][nZ] -> sino [nU][nA][nV]. */
int vam_vec_forward(vam_vec_plan* plan, const float* vol_dev, float* sino_dev, vam_stream_t stream);

/* Voxel-driven backprojection: each voxel centre carried along the ray onto
 * the detector, the sinogram sampled there bilinearly (zero outside), summed
 * over angles; replaces astra.creators.create_backprojection3d_gpu
 * (Projector3DParallelCUDA.py:56-72). */
int vam_vec_backward(vam_vec_plan* plan, const float* sino_dev, float* vol_dev, vam_stream_t stream);

/* Exact transpose of vam_vec_forward (<A x, y> = <x, A^T y> up to float
 * summation order): every ray adds its value times the forward's weights to
 * the voxels the forward read (float atomics).  No counterpart in the
 * reference (ASTRA's backprojection above is voxel-driven); used for
 * gradients. */
int vam_vec_adjoint(vam_vec_plan* plan, const float* sino_dev, float* vol_dev, vam_stream_t stream);

/* 2-D "line" model of the reference's Projector2DParallelCUDAAstra
 * (vamtoolbox/projector/Projector2DParallelCUDA.py:7-45, ASTRA's "line"
 * projector): the weight of a (ray, pixel) pair is the length of the ray, a
 * zero-width line, inside the unit pixel.  ASTRA's 2-D frame: pixel (i, j) of
 * [nY][nX] at (j - nX/2 + 1/2, nY/2 - i - 1/2), detector bin d at offset
 * d - nT/2 + 1/2 along (cos a, sin a), rays along (sin a, -cos a).  The
 * backward is the forward's exact transpose (astra create_backprojection with
 * that projector).  img [nY][nX], sino [nT][nA]. */
typedef struct vam_line2d_plan vam_line2d_plan;
int vam_line2d_plan_create(int32_t n_y, int32_t n_x, int32_t n_angles, const double* angles_deg, int32_t det_count,
                           int32_t device, vam_line2d_plan** out);
int vam_line2d_plan_destroy(vam_line2d_plan* plan);
int vam_line2d_forward(vam_line2d_plan* plan, const float* img_dev, float* sino_dev, vam_stream_t stream);
int vam_line2d_backward(vam_line2d_plan* plan, const float* sino_dev, float* img_dev, vam_stream_t stream);

/* ======================================================================= */
/* Output formats: projector frames (vamtoolbox/imagesequence.py) and      */
/* fan-beam rebinning (vamtoolbox/geometry.py:736-944)                     */
/* ======================================================================= */

/* Element type of the sinograms handled below (the reference keeps the
 * caller's numpy dtype through these steps). */
enum vam_dtype { VAM_DTYPE_F32 = 0, VAM_DTYPE_F64 = 1 };

/* Order-1 rotation of every (r, z) plane of a sinogram [nR][nA][nZ] into
 * [oR][nA][oZ], zero outside the input: ndimage.rotate(sino, angle,
 * axes=(0, 2), reshape=True, order=1) as called by ImageSeq's _rotate
 * (vamtoolbox/imagesequence.py:396-401).  affine (host, 6 doubles) =
 * {m00, m01, m10, m11, off0, off1}: output (o0, o1) samples the input at
 * ((m00*o0 + off0) + m01*o1, (m10*o0 + off1) + m11*o1), scipy's rot_matrix
 * and offset.  flip_r / flip_z mirror the input first (_invertU / _invertV,
 * imagesequence.py:358-365).  Double arithmetic, stored in dtype. */
int vam_sino_rotate(const void* in_dev, int dtype, int32_t nR, int32_t nA, int32_t nZ, int32_t flip_r,
                    int32_t flip_z, const double* affine, void* out_dev, int32_t oR, int32_t oZ,
                    vam_stream_t stream);

/* Bilinear resize of every (r, z) plane to [oR][nA][oZ]: cv2.resize(plane,
 * (oZ, oR), interpolation=INTER_LINEAR) as called by _scaleSize
 * (imagesequence.py:368-378): half-pixel centres, edge clamp, z interpolated
 * before r, in the input's dtype.  out_dev is always double [oR][nA][oZ]:
 * _scaleSize collects the planes in a float64 array.  flip_r / flip_z as above. */
int vam_sino_resize(const void* in_dev, int dtype, int32_t nR, int32_t nA, int32_t nZ, int32_t flip_r,
                    int32_t flip_z, void* out_dev, int32_t oR, int32_t oZ, vam_stream_t stream);

/* Workspace of vam_select_pair, in bytes (independent of n). */
size_t vam_select_workspace_bytes(void);

/* out_dev[0], out_dev[1] (dtype) = the k0-th and k1-th smallest of x[0..n)
 * (0-based, k1 == k0 or k0 + 1): the two sorted elements np.percentile
 * (method 'linear') blends, imagesequence.py:129-133.  NaN sorts last and
 * any NaN makes both outputs NaN (np.percentile returns NaN then).  Radix
 * select on the device; stream-ordered, no host synchronisation.
 * work_dev: vam_select_workspace_bytes(), 8-byte aligned. */
int vam_select_pair(const void* x_dev, int dtype, int64_t n, int64_t k0, int64_t k1, void* out_dev,
                    void* work_dev, size_t work_bytes, vam_stream_t stream);

typedef struct {
    int32_t n_u, n_v;             /* frame width (multiple of 4) and height, ImageConfig (imagesequence.py:55-58) */
    const int32_t* src_col_dev;   /* [n_u] sinogram row r shown in frame column u, -1 = blank */
    const int32_t* src_row_dev;   /* [n_v] sinogram z shown in frame row v, -1 = blank */
    int32_t bit_depth;            /* 0..32; max value 2^bit_depth - 1 (imagesequence.py:127) */
    int32_t has_norm;             /* divide by norm_value, multiply by the max value (:129-133) */
    double norm_value;            /* the percentile value */
    int32_t norm_dtype;           /* vam_dtype of the percentile value (numpy promotes the array to it) */
    int32_t has_scale;            /* multiply by intensity_scale (:135-138) */
    double intensity_scale;
    int32_t scale_is_f64;         /* the scale is a float64 numpy scalar (promotes a float32 array) */
    int32_t box_v0, box_v1;       /* frame rows [v0, v1) and columns [u0, u1) that may show the image; */
    int32_t box_u0, box_u1;       /* outside this box every pixel is 0 whatever the tables say */
} vam_frame_params;

/* frames_dev[a][v][u] (uint8, 16-byte aligned, nA frames of n_v x n_u) from
 * the sinogram [nR][nA][nZ]: 0 where src_row[v] or src_col[u] is -1, else
 * the quantised sino[src_col[u]][a][src_row[v]]: ImageSeq.__init__
 * (imagesequence.py:127-174), whose chain x / norm * max, * scale,
 * np.minimum(., max), astype(uint8/16/32) and the store into a uint8 frame
 * (low byte) is replayed in the reference's dtypes; the insertion offsets,
 * array copies and flips of _insertImage / _arrayInsertImage (:303-355) are
 * carried by the two tables.  The blank area outside the box
 * is written with contiguous zero stores, the box by the gather kernel; a
 * box equal to the frame makes it one gather pass (used to fetch just the
 * image window, frame = window). */
int vam_imageseq_frames(const void* sino_dev, int dtype, int32_t nR, int32_t nA, int32_t nZ,
                        const vam_frame_params* prm, uint8_t* frames_dev, vam_stream_t stream);

/* Fan-beam rebinning, rebinFanBeam (vamtoolbox/geometry.py:736-944):
 * out[p][a][z] = tinv[p] * (dxv[p] * interp) for p < nP (the vial width in
 * projector pixels), interp being interpn's bilinear sample of the sinogram
 * padded to nP rows (input row p - pad_lo, zero outside [0, nR)).  Tables
 * from the host grid search: xi_dev[nP] lower x index (-1: out of bounds),
 * xw_dev[nP][4] = {y0, 1 - y0, dxv_dxp, 1/T}, ti_dev[nP][nA] lower angle index
 * (-1: out of bounds), tw_dev[nP][nA][2] = {y1, 1 - y1}.  out_dev [nP][nA][nZ]. */
int vam_rebin_fan(const void* in_dev, int dtype, int32_t nR, int32_t nA, int32_t nZ, int32_t nP,
                  int32_t pad_lo, const int32_t* xi_dev, const double* xw_dev, const int32_t* ti_dev,
                  const double* tw_dev, void* out_dev, vam_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* VAM_H */
