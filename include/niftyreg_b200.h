/* niftyreg_b200: B200-native F3D objective-and-gradient evaluation behind a C ABI.
 *
 * Every entry point takes plain pointers and sizes and returns an nrb_status. Array arguments
 * are DEVICE pointers unless the parameter name ends in _host. `stream` is a cudaStream_t passed
 * as void* (NULL = the legacy default stream); every call is asynchronous on that stream unless
 * it returns a host value, in which case it synchronises the stream first.
 *
 * Data layout (identical to NiftyReg's NIfTI buffers, so a platform plugin can hand over its
 * arrays without reshaping):
 *   - scalar volume: float32, x fastest, [nz][ny][nx];
 *   - vector image (deformation field, spatial/voxel gradient, control-point grid and its
 *     gradient): three planes [x | y | z], each laid out as a scalar volume;
 *   - mask: int32 per reference voxel, -1 = inactive, NULL = every voxel active;
 *   - matrices: row-major float[16] in the NIfTI mat44 layout.
 *
 * Each declaration names the reference interface it replaces (paths relative to the NiftyReg
 * source tree). */
#ifndef NIFTYREG_B200_H
#define NIFTYREG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum nrb_status {
    NRB_OK = 0,
    NRB_ERR_INVALID = 1,      /* bad argument: null pointer, non-positive size, bins < 5 ... */
    NRB_ERR_UNSUPPORTED = 2,  /* geometry outside the F3D layout (grid not axis-aligned ...) */
    NRB_ERR_CUDA = 3,         /* a CUDA call failed; nrb_last_error() has the text */
    NRB_ERR_NO_DEVICE = 4,    /* no CUDA device, or not an sm_100 device */
    NRB_ERR_OOM = 5           /* device allocation failed */
} nrb_status;

/* Geometry of one registration level: the reference image (which is also the geometry of the
 * warped image, the deformation field and the voxel-based gradients), the floating image and
 * the cubic B-spline control-point grid. *_xyz is voxel->mm, *_ijk mm->voxel (NiftyReg picks
 * the sform when sform_code > 0, else the qform: reg-lib/Content.h GetXYZMatrix/GetIJKMatrix).
 * Mirrors the three NiftiImage members of F3dContent (reg-lib/F3dContent.h:5-30). */
typedef struct nrb_geometry {
    int32_t ref_dim[3];
    float ref_pixdim[3];
    float ref_xyz[16];
    float ref_ijk[16];
    int32_t flo_dim[3];
    float flo_pixdim[3];
    float flo_xyz[16];
    float flo_ijk[16];
    int32_t cpp_dim[3];
    float cpp_pixdim[3]; /* control-point spacing in mm */
    float cpp_xyz[16];
    float cpp_ijk[16];
} nrb_geometry;

/* Packed per-evaluation scalars written by the objective kernels (device memory). */
typedef struct nrb_objective {
    double nmi;          /* (H_ref + H_war) / H_joint, unweighted */
    double entropy[4];   /* H_ref, H_war, H_joint, total histogram mass (_reg_nmi.cpp:303-346) */
    double be;           /* approximate bending energy, unweighted (_regul.cpp:72-153) */
    double objective;    /* sim_weight * nmi - be_weight * be (_reg_f3d.cpp:443-462) */
    double max_grad_len; /* largest node-gradient length of the last gradient evaluation */
} nrb_objective;

/* ---- library ------------------------------------------------------------------------------ */

/* Text of the last error on this thread (empty string when none). */
const char *nrb_last_error(void);
/* Selects and checks the CUDA device (replaces CudaContext::SetCudaIdx,
 * reg-lib/cuda/CudaContext.cpp:38-91 and Platform::SetGpuIdx, reg-lib/Platform.cpp:66-93). */
nrb_status nrb_set_device(int device);
/* 1 when the library was built for sm_100a and a B200-class device is present. */
int nrb_device_ok(void);
/* Returns the current device's unused memory in the library's own memory pool to the driver,
 * keeping at most keep_bytes mapped (the pool otherwise keeps what registrations and batches
 * freed, up to the largest working set it has held, for the next ones). Work already queued
 * keeps its memory. No counterpart in the reference. */
nrb_status nrb_memory_trim(size_t keep_bytes);

/* ---- deformation and resampling (Compute, reg-lib/Compute.h:6-49) ------------------------ */

/* Cubic B-spline deformation field (positions in mm) from the control-point positions.
 * Replaces Compute::GetDeformationField(false, true) (reg-lib/Compute.cpp:83-90) ->
 * reg_spline_getDeformationField (reg-lib/cpu/_reg_localTrans.cpp:1457-1538).
 * def: 3 * nvox(ref) floats. Masked voxels receive 0. */
nrb_status nrb_get_deformation_field(const nrb_geometry *g, const float *cpp, const int32_t *mask,
                                     float *def, void *stream);

/* Trilinear warp of the floating image by a deformation field, padding outside the floating
 * volume. Replaces Compute::ResampleImage(1, padding) (reg-lib/Compute.cpp:8-15) ->
 * ResampleImage3D (reg-lib/cpu/_reg_resampling.cpp:316-464). Masked voxels are untouched. */
nrb_status nrb_resample_image(const nrb_geometry *g, const float *flo, const float *def,
                              const int32_t *mask, float padding, float *warped, void *stream);

/* Warp of the floating image by a deformation field with interpolation `order`: 0 nearest,
 * 1 linear, 3 cubic spline; any other order returns NRB_ERR_UNSUPPORTED. The reference's float
 * operations are kept unfused, so the result is bit-identical to the reference's. Replaces
 * Compute::ResampleImage(order, padding) (reg-lib/Compute.cpp:8-15) -> ResampleImage3D
 * (reg-lib/cpu/_reg_resampling.cpp:316-464) with interpNearestNeighKernel / interpLinearKernel /
 * interpCubicSplineKernel (:60-97). Masked voxels are untouched. */
nrb_status nrb_resample_image_order(const nrb_geometry *g, const float *flo, const float *def,
                                    const int32_t *mask, int order, float padding, float *warped,
                                    void *stream);

/* Spatial gradient (floating voxel units) of the trilinearly warped floating image, NaN -> 0.
 * Replaces Compute::GetImageGradient(1, padding, 0) (reg-lib/Compute.cpp:129-138) ->
 * TrilinearImageGradient (reg-lib/cpu/_reg_resampling.cpp:1797-1915). grad: 3 * nvox(ref). */
nrb_status nrb_get_image_gradient(const nrb_geometry *g, const float *flo, const float *def,
                                  const int32_t *mask, float padding, float *grad, void *stream);

/* ---- intensity rescale (reg_nmi::InitialiseMeasure, reg-lib/cpu/_reg_nmi.cpp:91-158) ------ */

/* In-place rescale of the finite values of a volume to [new_min, new_max] in double precision.
 * Replaces reg_intensityRescale (reg-lib/cpu/_reg_tools.cpp:92-174). */
nrb_status nrb_intensity_rescale(float *img, int64_t nvox, float new_min, float new_max,
                                 void *stream);

/* ---- NMI measure (reg_nmi, reg-lib/cpu/_reg_nmi.h:19-84) ---------------------------------- */

/* Workspace of one NMI measure: joint histogram counts, FP64 probability/log tables,
 * entropies. Replaces the histogram arrays reg_nmi allocates in InitialiseMeasure. */
typedef struct nrb_nmi nrb_nmi;
nrb_status nrb_nmi_create(int ref_bins, int flo_bins, nrb_nmi **out);
void nrb_nmi_destroy(nrb_nmi *nmi);

/* Joint histogram of (reference, warped) over active voxels, 3-tap B-spline smoothing, FP64
 * entropies; writes the log table used by the gradient and the scalars into `obj` (device,
 * may be NULL). Replaces reg_nmi::GetSimilarityMeasureValueFw (reg-lib/cpu/_reg_nmi.cpp:385-398
 * -> reg_getNmiValue :160-347, approximated Parzen window). If nmi_host is non-NULL the stream
 * is synchronised and the NMI is returned there. */
nrb_status nrb_nmi_value(nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                         const float *warped, const int32_t *mask, nrb_objective *obj,
                         double *nmi_host, void *stream);

/* Adds weight * dNMI/d(warped) * spatial gradient to vgrad, using the log table of the last
 * nrb_nmi_value call (the 4x4 Parzen window in FP32 on an FP32 copy of the table when it fits in
 * 96 KB of shared memory, in FP64 otherwise; the normalisation constant in FP64). Replaces reg_getVoxelBasedNmiGradient3d (reg-lib/cpu/_reg_nmi.cpp:501-593),
 * which reg_nmi::GetVoxelBasedSimilarityMeasureGradientFw (:623-638) runs after recomputing the
 * histogram. */
nrb_status nrb_nmi_voxel_gradient(nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                                  const float *warped, const float *warped_grad,
                                  const int32_t *mask, double weight, float *vgrad, void *stream);

/* Copies the last histogram state to the host: pro/log are ref_bins*flo_bins + ref_bins +
 * flo_bins doubles (joint | reference marginal | floating marginal), ent is 4 doubles. Any
 * pointer may be NULL. Synchronises the stream. Test and debug use. */
nrb_status nrb_nmi_read_tables(nrb_nmi *nmi, double *pro_host, double *log_host,
                               double *ent_host, void *stream);

/* ---- voxel -> node gradient (Compute::ConvolveVoxelBasedMeasureGradient) ------------------ */

/* One axis (0, 1, 2) of the density-normalised cubic B-spline convolution of a vector image,
 * spacing in mm; in place over the whole volume. Replaces reg_tools_kernelConvolution with
 * ConvKernelType::Cubic and one active axis (reg-lib/cpu/_reg_tools.cpp:831-1112). */
nrb_status nrb_kernel_convolution_cubic(float *img, int nvol, const int32_t dim[3],
                                        const float pixdim[3], float spacing_mm, int axis,
                                        void *stream);

/* Same result as nrb_kernel_convolution_cubic, but it allocates nothing: no device or host
 * allocation, no allocator of any library. It has no counterpart in the reference; it exists
 * for callers that must not allocate at the time of the call (while recording a stream
 * capture, under an exhausted memory cap, inside a memory pool the caller owns). Its scratch
 * is one fixed array per device, reserved when the library's module loads (16 MiB + 2 KiB):
 *  - one volume of at most NRB_STATIC_CONV_MAX_VOXELS voxels, a kernel of at most
 *    NRB_STATIC_CONV_MAX_TAPS taps (radius 255); larger requests return NRB_ERR_UNSUPPORTED
 *    and launch nothing;
 *  - the first call on each device looks the scratch up (cudaGetSymbolAddress) with that
 *    device current; make that first call before any stream capture begins;
 *  - nothing in the scratch has to start at zero;
 *  - calls on one device share the scratch: two calls whose work can overlap (unordered
 *    streams, several host threads) race and produce garbage. Order them on one stream. */
#define NRB_STATIC_CONV_MAX_VOXELS 2097152
#define NRB_STATIC_CONV_MAX_TAPS 511
nrb_status nrb_kernel_convolution_cubic_static(float *img, int nvol, const int32_t dim[3],
                                               const float pixdim[3], float spacing_mm, int axis,
                                               void *stream);

/* Node gradient = weight * reorient(trilinear sample at the node of the x-, y- then z-convolved
 * voxel gradient). The convolution is evaluated only at the voxels the node sampling reads.
 * Overwrites node_grad (3 * nvox(cpp)). vgrad is read only. Replaces
 * Compute::ConvolveVoxelBasedMeasureGradient (reg-lib/Compute.cpp:230-281) ->
 * reg_tools_kernelConvolution x3 + reg_voxelCentricToNodeCentric
 * (reg-lib/cpu/_reg_localTrans.cpp:1540-1685). Scratch comes from `ws`
 * (nrb_workspace_create). */
typedef struct nrb_workspace nrb_workspace;
nrb_status nrb_workspace_create(const nrb_geometry *g, nrb_workspace **out);
void nrb_workspace_destroy(nrb_workspace *ws);
nrb_status nrb_convolve_voxel_based_gradient(nrb_workspace *ws, const nrb_geometry *g,
                                             const float *vgrad, float weight, float *node_grad,
                                             void *stream);

/* ---- regularisation (Compute::ApproxBendingEnergy*, reg-lib/Compute.cpp:40-51) ------------- */

/* Approximate bending energy of the grid positions, unweighted, FP64 sum. Written to
 * obj->be when obj is non-NULL; returned in be_host (synchronising) when non-NULL.
 * Replaces reg_spline_approxBendingEnergy (reg-lib/cpu/_reg_localTrans_regul.cpp:155-177). */
nrb_status nrb_approx_bending_energy(nrb_workspace *ws, const nrb_geometry *g, const float *cpp,
                                     nrb_objective *obj, double *be_host, void *stream);

/* node_grad += weight/#nodes * d(BE)/d(displacement). Replaces
 * reg_spline_approxBendingEnergyGradient (reg-lib/cpu/_reg_localTrans_regul.cpp:453-482). */
nrb_status nrb_approx_bending_energy_gradient(nrb_workspace *ws, const nrb_geometry *g,
                                              const float *cpp, float weight, float *node_grad,
                                              void *stream);

/* ---- optimiser support (Compute.cpp:91-183, Optimiser.cpp:231-317) ------------------------- */

/* Largest Euclidean length of the node gradient (float), into obj->max_grad_len and/or
 * max_host. Replaces Compute::GetMaximalLength (reg-lib/Compute.cpp:140-146). */
nrb_status nrb_get_maximal_length(const float *node_grad, int64_t nnode, nrb_objective *obj,
                                  double *max_host, void *stream);
/* node_grad /= max length; the length is read from obj->max_grad_len when max_len < 0.
 * Replaces Compute::NormaliseGradient (reg-lib/Compute.cpp:148-176). */
nrb_status nrb_normalise_gradient(float *node_grad, int64_t nnode, double max_len,
                                  const nrb_objective *obj, void *stream);
/* cur = best + scale * grad over n values. Replaces Compute::UpdateControlPointPosition
 * (reg-lib/Compute.cpp:91-127, all axes optimised). */
nrb_status nrb_update_control_point_position(float *cur, const float *best, const float *grad,
                                             float scale, int64_t n, void *stream);
/* Conjugate-gradient direction update with FP64 dot products in a fixed reduction order.
 * first_call != 0: g1 = g2 = -grad. Replaces ConjugateGradient<float>::UpdateGradientValues
 * (reg-lib/Optimiser.cpp:231-317; CUDA counterpart reg-lib/cuda/CudaOptimiser.cu:198-290). */
nrb_status nrb_conjugate_gradient(nrb_workspace *ws, float *grad, float *g1, float *g2, int64_t n,
                                  int first_call, void *stream);

/* ---- fused F3D evaluations (reg_f3d, reg-lib/_reg_f3d.cpp) -------------------------------- */

/* One objective evaluation: bending energy of cpp, deformation field, trilinear warp, joint
 * histogram and entropies fused into one pass over the reference voxels (the deformation field
 * and warped image are never written to HBM). Replaces reg_f3d::GetObjectiveFunctionValue
 * (reg-lib/_reg_f3d.cpp:443-462) with WarpFloatingImage (reg-lib/_reg_base.cpp:688-708) and
 * ComputeSimilarityMeasure (:469-494). Writes obj on the device; obj_host (optional) receives a
 * copy after a stream synchronisation. */
nrb_status nrb_f3d_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                             const float *ref, const float *flo, const int32_t *mask,
                             const float *cpp, float padding, double sim_weight,
                             double be_weight, nrb_objective *obj, nrb_objective *obj_host,
                             void *stream);

/* One gradient evaluation into node_grad: the joint histogram is recomputed at cpp (as
 * reg_nmi::GetVoxelBasedSimilarityMeasureGradientFw does), then warp + spatial gradient + NMI
 * voxel gradient run fused in one pass into vgrad (3 * nvox(ref) floats of caller memory),
 * then the voxel->node convolution (weighted by sim_weight) overwrites node_grad and the
 * bending-energy gradient (be_weight) is added. Replaces reg_f3d::GetObjectiveFunctionGradient
 * (reg-lib/_reg_f3d.cpp:553-576). */
nrb_status nrb_f3d_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                            const float *ref, const float *flo, const int32_t *mask,
                            const float *cpp, float padding, double sim_weight,
                            double be_weight, float *vgrad, float *node_grad, void *stream);

/* ---- whole registration (reg_f3d<float>::Run, reg-lib/_reg_base.cpp:727-818) -------------- */

typedef struct nrb_f3d_params {
    int32_t levels;           /* -ln: pyramid levels (all performed) */
    int32_t max_iterations;   /* -maxit: finest-level budget, doubled per coarser level */
    float bending_energy;     /* -be */
    float spacing[3];         /* -sx/-sy/-sz: negative = voxels, positive = mm */
    int32_t ref_bins;         /* --rbn (the +4 Parzen margin is added internally) */
    int32_t flo_bins;         /* --fbn */
    float padding;            /* -pad: warped padding value (NaN by default) */
    int32_t verbose;
    int32_t host_loop;        /* 0 (default): each level's optimisation runs as one CUDA graph
                               * with the optimiser state on the device; 1: the host takes every
                               * line-search branch (one synchronising read per evaluation).
                               * Both take the same steps. Per-kernel timing forces 1. */
    int32_t floating_margin;  /* voxels of the padding value laid around each level's floating
                               * image in a padded device copy (default 8, at most 64; 0: no
                               * copy). Samples that reach into the margin take the kernels'
                               * plain load path instead of the clamped one; the results are the
                               * same bit for bit. */
    int32_t batch_gradient_percent; /* nrb_f3d_register_batch: a level's gradient stage runs
                               * once this share (%) of the pairs still active waits for a
                               * gradient, or when no pair has a line-search step left (default
                               * 50; 1..100). Scheduling only: results do not depend on it. */
    int32_t floating_texture; /* 1 (default): each level's padded floating copy is also held as
                               * a layered texture, and the fused passes fetch each slice's 2x2
                               * footprint with one gather; 0: plain loads. The same values are
                               * read either way, so the results are identical. */
    int32_t autotune;         /* 1 (default): the first level of each shape times the objective
                               * and gradient walks over a candidate set (block height, z-chunk,
                               * resident blocks) and keeps the fastest in the process's walk
                               * table (nrb_autotune_entries); 0: the cost model's plans. The
                               * walk plan moves no value, so results are identical either way. */
    int32_t batch_group_mb;   /* nrb_f3d_register_batch and the grouping server: when > 0, a
                               * group of pairs registered together holds at most this many MB of
                               * finest-level images (reference + floating); a pair larger than
                               * that is a group of its own. 0 (default): no cap; larger groups
                               * measured faster on every mix tried. Scheduling only: results do
                               * not depend on it. */
} nrb_f3d_params;

typedef struct nrb_f3d_result {
    int32_t cpp_dim[3];       /* final grid dims; the grid is 3 * prod(cpp_dim) floats */
    double final_nmi;         /* NMI at the best position of the finest level */
    double final_be;          /* unweighted BE there */
    double final_objective;
    int64_t objective_evaluations;
    int64_t gradient_evaluations;
    double seconds;           /* host wall time of the whole call */
} nrb_f3d_result;

/* ---- walk autotuner (no counterpart in the reference) --------------------------------------
 * One entry per level shape registered in this process with autotune on: the fastest measured
 * objective and gradient walks and the times of the cost model's own plans beside them. */
typedef struct nrb_walk_entry {
    int32_t ref_dim[3];
    int32_t cpp_dim[3];
    int32_t bins[2];          /* user bins (reference, floating) */
    int32_t obj_ty, obj_zchunk, obj_resident;    /* block height (warps), z-chunk, resident blocks (0: occupancy) */
    float obj_us, obj_model_us;                  /* device us per launch: tuned, cost model's plan */
    int32_t grad_ty, grad_zchunk, grad_resident;
    float grad_us, grad_model_us;
    int32_t candidates;       /* walks timed */
} nrb_walk_entry;
/* Copies up to `capacity` entries into out (may be NULL) and returns the number of entries. */
int nrb_autotune_entries(nrb_walk_entry *out, int capacity);
/* Empties the table: the next registration of each shape tunes again. */
void nrb_autotune_clear(void);

/* Default parameters of reg_f3d<float> (reg-lib/_reg_base.cpp:17-70, _reg_f3d.cpp:18-40). */
void nrb_f3d_default_params(nrb_f3d_params *p);

/* Final grid dims for a registration of this reference (for sizing cpp_out_host). */
nrb_status nrb_f3d_grid_dims(const int32_t ref_dim[3], const float ref_pixdim[3],
                             const nrb_f3d_params *p, int32_t cpp_dim_out[3]);

/* Full F3D registration from HOST images (identity orientation, origin 0, the given voxel
 * size): pyramid, per-level grid refinement, conjugate-gradient line search, all on the
 * device. Host<->device copies are part of the call. cpp_out_host receives the final
 * control-point positions (3 * prod(cpp_dim) floats, capacity cpp_capacity floats). */
nrb_status nrb_f3d_register_host(const float *ref_host, const float *flo_host,
                                 const int32_t dim[3], const float pixdim[3],
                                 const nrb_f3d_params *p, float *cpp_out_host,
                                 int64_t cpp_capacity, nrb_f3d_result *result);

/* The same registration from images already resident on the device. */
nrb_status nrb_f3d_register_device(const float *ref, const float *flo, const int32_t dim[3],
                                   const float pixdim[3], const nrb_f3d_params *p,
                                   float *cpp_out, int64_t cpp_capacity, nrb_f3d_result *result,
                                   void *stream);

/* The final warped image of a registration, on the device: the deformation field of the
 * control-point grid `cpp` over the reference geometry of `g` (nrb_get_deformation_field), then
 * the floating image `flo` (device, original intensities) resampled with interpolation `order`
 * and `padding` (nrb_resample_image_order). Replaces reg_f3d<T>::GetWarpedImage
 * (reg-lib/_reg_f3d.cpp:503-515), which the reference runs on the CPU with order 3 (cubic
 * spline). For a grid from nrb_f3d_register_*, `g` holds the grid of nrb_f3d_grid_dims with the
 * spacing the registration used. One pass: the positions are computed as nrb_get_deformation_field
 * computes them and resampled at once (no deformation field in memory, no allocation).
 * warped: nvox(ref) floats. */
nrb_status nrb_f3d_warped_image(const nrb_geometry *g, const float *flo, const float *cpp, int order,
                                float padding, float *warped, void *stream);

/* ---- NIfTI-1 images (reg-io/_reg_ReadWriteImage.cpp, reg-io/niftilib) ----------------------- */

/* A host image as the request path of a registration carries it. */
typedef struct nrb_image {
    int32_t dim[3];         /* nx, ny, nz (absent axes 1) */
    int32_t nvol;           /* volumes: product of dims 4..7 (1: scalar image, 3: vector image) */
    float pixdim[3];        /* spacing in mm */
    float xyz[16];          /* voxel -> mm: the sform when sform_code > 0, else the qform, else the
                             * spacings on the diagonal (Content::GetXYZMatrix's choice) */
    float ijk[16];          /* mm -> voxel */
    int32_t sform_code;     /* as read (xyz is the sform when > 0) */
    int32_t qform_code;     /* as read (xyz is the qform when > 0 and sform_code is 0) */
    int32_t intent_code;    /* NIfTI intent (1007: vector) */
    float intent_p1;        /* NiftyReg transformation type for a grid (2: cubic B-spline grid) */
    float intent_p2;        /* squaring number of a velocity grid (NiftyReg's use), else 0 */
    char intent_name[16];   /* "NREG_TRANS" for NiftyReg transformations */
    float *data;            /* host float32, nvol * nx * ny * nz, x fastest; owned by the library
                             * after nrb_image_read (free with nrb_image_free), by the caller when
                             * passed to nrb_image_write */
} nrb_image;

/* Reads a single-file NIfTI-1 image (.nii or .nii.gz) as reg_io_ReadImageFile does
 * (reg-io/_reg_ReadWriteImage.cpp:51-81, with reg_checkAndCorrectDimension,
 * reg-lib/cpu/_reg_tools.cpp:13-71): any integer or real datatype converted to float and scaled
 * by scl_slope / scl_inter (slope 0 = 1); micron and metre spacings converted to mm. */
nrb_status nrb_image_read(const char *path, nrb_image *out);
/* Frees the data of an image from nrb_image_read. */
void nrb_image_free(nrb_image *img);
/* Writes a float32 single-file NIfTI-1 image (.nii, or .nii.gz compressed): xyz as the sform
 * (code sform_code, else qform_code, else 1), no qform, nvol > 1 as the 5th axis with the intent fields, the
 * layout NiftyReg uses for grids and deformation fields (reg_io_WriteImageFile,
 * reg-io/_reg_ReadWriteImage.cpp:83-120). */
nrb_status nrb_image_write(const char *path, const nrb_image *img);

/* reg_f3d<float>::Run on two host images with their own dims, spacings and orientations (from
 * nrb_image_read, or filled by the caller: xyz is used as given, as an sform when sform_code > 0),
 * each pyramid built along its own axes, the grid oriented like the reference
 * (reg_createControlPointGrid, reg-lib/cpu/_reg_localTrans.cpp:21-128). Results, allocated by the
 * library (free with nrb_image_free): cpp_out (required) the final control-point grid, a vector
 * image of 3 planes tagged as NiftyReg tags grids (intent 1007, "NREG_TRANS", p1 = 2);
 * warped_out (optional, may be NULL) the input floating image warped by it with cubic-spline
 * interpolation on the reference geometry (reg_f3d::GetWarpedImage). Replaces reg_f3d::Run +
 * GetControlPointPositionImage + GetWarpedImage (reg-lib/_reg_f3d.cpp:503-523). */
nrb_status nrb_f3d_register_images(const nrb_image *ref, const nrb_image *flo, const nrb_f3d_params *p,
                                   nrb_image *cpp_out, nrb_image *warped_out, nrb_f3d_result *result);

/* The image pyramid of reg_createImagePyramid<float> (reg-lib/cpu/_reg_tools.cpp:1705-1733) for a
 * device image with dims, spacings and voxel -> mm matrix xyz (NULL: identity orientation at
 * origin 0): level levels-1 is the input, each coarser level is Gaussian-smoothed (sigma 0.7355
 * voxel) and nearest-neighbour downsampled from the next finer one along every axis whose size / 2
 * is at least 32 (reg_downsampleImage, _reg_tools.cpp:1343-1500). out receives the levels end to
 * end, coarsest first; dims_out (3 per level), xyz_out (16 per level) and total_out (floats of
 * out) may be NULL; with out == NULL only the headers and the total are computed (host only). */
nrb_status nrb_image_pyramid(const float *img, const int32_t dim[3], const float pixdim[3],
                             const float xyz[16], int levels, float *out, int64_t capacity,
                             int32_t *dims_out, float *xyz_out, int64_t *total_out, void *stream);

/* The node values of reg_spline_refineControlPointGrid3D (reg-lib/cpu/_reg_localTrans.cpp:
 * 1809-2119): a grid of old_dim nodes (three planes) refined onto new_dim nodes at half the
 * spacing, as the registration does between pyramid levels. new_dim comes from the finer
 * reference (nrb_f3d_grid_header) and lies in [1, 2 * old_dim]; out must not alias old. */
nrb_status nrb_refine_control_point_grid(const float *old, const int32_t old_dim[3], float *out,
                                         const int32_t new_dim[3], void *stream);

/* Dims, spacing and voxel -> mm matrix of the final (finest-level) control-point grid that
 * nrb_f3d_register_images returns for this reference and these parameters, from the header alone
 * (host only): reg_createControlPointGrid over the coarsest reference
 * (reg-lib/cpu/_reg_localTrans.cpp:21-128), refined onto each finer reference (:1808-2238). */
nrb_status nrb_f3d_grid_header(const nrb_image *ref, const nrb_f3d_params *p, int32_t dim_out[3],
                               float pixdim_out[3], float xyz_out[16]);

/* A registration request on files, the way reg_f3d -ref -flo -cpp -res runs it
 * (reg-apps/reg_f3d.cpp): both images read with nrb_image_read, nrb_f3d_register_images, the grid
 * written to cpp_path and, when res_path is not NULL, the warped image to res_path (NIfTI-1,
 * .nii or .nii.gz). */
nrb_status nrb_f3d_register_files(const char *ref_path, const char *flo_path, const nrb_f3d_params *p,
                                  const char *cpp_path, const char *res_path, nrb_f3d_result *result);

/* ---- F3D2: symmetric registration with stationary velocity fields (reg_f3d2) --------------- */

/* Deformation field (positions in mm) on the reference grid of g (g->ref_*) from the cubic
 * B-spline velocity grid vel on g->cpp_*: the flow at every voxel, divided by 2^N, squared N times
 * by composition. *steps is N (the grid's intent_p2); with update_step_number (or *steps == 0)
 * it is first set to the smallest N >= 6 with max |flow| / 2^N < 0.28 mm. Replaces
 * Compute::GetDefFieldFromVelocityGrid (reg-lib/Compute.cpp:223-228) ->
 * reg_spline_getDefFieldFromVelocityGrid (reg-lib/cpu/_reg_localTrans.cpp:3583-3613).
 * def: 3 * nvox(ref) floats. Synchronises the stream when it updates N. */
nrb_status nrb_get_def_field_from_velocity_grid(const nrb_geometry *g, const float *vel,
                                                int update_step_number, int32_t *steps, float *def,
                                                void *stream);

/* update(x) <- apply(update(x)): trilinear in the voxel space of apply (dim, xyz voxel -> mm,
 * ijk mm -> voxel), positions outside extrapolated linearly from the border. apply and update
 * are distinct 3 * nvox buffers. Replaces Compute::DefFieldCompose (reg-lib/Compute.cpp:394-397)
 * -> reg_defField_compose (reg-lib/cpu/_reg_localTrans.cpp:2334-2480). */
nrb_status nrb_def_field_compose(const int32_t dim[3], const float xyz[16], const float ijk[16],
                                 const float *apply, float *update, void *stream);

/* The voxel-based gradient vgrad (3 * nvox(ref), on g->ref_*) transported along the opposite
 * transformation, whose velocity grid vel_other lies on g->cpp_*: with its intermediate fields
 * phi_0..phi_{N-1} (N = steps), vgrad <- vgrad + J(phi_i) * vgrad(phi_i) for i = 0..N-1, then
 * vgrad / 2^N. Replaces Compute::ExponentiateGradient (reg-lib/Compute.cpp:288-330). */
nrb_status nrb_exponentiate_gradient(const nrb_geometry *g, const float *vel_other, int32_t steps,
                                     float *vgrad, void *stream);

/* Forward and backward velocity grids (same dims; matrices g_fw->cpp_xyz and g_bw->cpp_xyz) made
 * opposite: as displacements, fw <- (fw - bw) / 2 and bw <- (bw - fw) / 2. Replaces
 * Compute::SymmetriseVelocityFields (reg-lib/Compute.cpp:356-392). */
nrb_status nrb_symmetrise_velocity_fields(const nrb_geometry *g_fw, float *fw,
                                          const nrb_geometry *g_bw, float *bw, void *stream);

/* reg_f3d2<float>::Run (reg-lib/_reg_f3d2.cpp, the -vel and -sym variant of reg_f3d) on two host
 * images: forward and backward velocity grids over the union of both fields of view
 * (reg_createSymmetricControlPointGrids, reg-lib/cpu/_reg_localTrans.cpp:133-357), symmetric NMI
 * (forward + backward) minus the bending energy of both grids, gradients exponentiated along the
 * opposite transformation, grids symmetrised after every update. Images in any orientation; the
 * velocity grids are axis-aligned in the world.
 * Results allocated by the library (free with nrb_image_free): cpp_fw_out and cpp_bw_out
 * (required) the final velocity grids, intent_p1 = 6 (SPLINE_VEL_GRID), intent_p2 the squaring
 * number; warped_fw_out / warped_bw_out (optional) the floating image on the reference grid and
 * the reference image on the floating grid, cubic spline (reg_f3d2::GetWarpedImage). The result's
 * final_nmi is the symmetric NMI (forward + backward); final_be the sum of both grids' energies. */
nrb_status nrb_f3d2_register_images(const nrb_image *ref, const nrb_image *flo, const nrb_f3d_params *p,
                                    nrb_image *cpp_fw_out, nrb_image *cpp_bw_out, nrb_image *warped_fw_out,
                                    nrb_image *warped_bw_out, nrb_f3d_result *result);

/* Dims, spacing and voxel -> mm matrix of the final (finest-level) velocity grids that
 * nrb_f3d2_register_images returns for these images and parameters, from the headers alone (host
 * only, no device work): reg_createSymmetricControlPointGrids over the coarsest pyramid images
 * (reg-lib/cpu/_reg_localTrans.cpp:133-357), refined once per finer level
 * (reg_spline_refineControlPointGrid without a reference, :1809-2229). Data is not read. */
nrb_status nrb_f3d2_grid_header(const nrb_image *ref, const nrb_image *flo, const nrb_f3d_params *p,
                                int32_t dim_out[3], float pixdim_out[3], float xyz_out[16]);

/* A reg_f3d -vel request on files (reg-apps/reg_f3d.cpp:647-705): both images read with
 * nrb_image_read, nrb_f3d2_register_images, the forward velocity grid written to cpp_path and the
 * backward one beside it with "_backward" before the extension (a.nii.gz -> a_backward.nii.gz);
 * when res_path is not NULL the warped floating image to res_path and the warped reference to its
 * "_backward" name. */
nrb_status nrb_f3d2_register_files(const char *ref_path, const char *flo_path, const nrb_f3d_params *p,
                                   const char *cpp_path, const char *res_path, nrb_f3d_result *result);

/* ---- batched and served registrations (no counterpart in the reference) -------------------- */

/* One registration request: host images (valid until the request completes), the reference's
 * geometry (identity orientation, origin 0) and where the final grid goes. */
typedef struct nrb_pair {
    const float *ref_host;
    const float *flo_host;
    int32_t dim[3];
    float pixdim[3];
    float *cpp_out_host;      /* 3 * prod(cpp_dim) floats (nrb_f3d_grid_dims), or NULL */
    int64_t cpp_capacity;
} nrb_pair;

/* Peak device bytes one registration of this size needs (the admission unit of a server). */
nrb_status nrb_f3d_footprint(const int32_t dim[3], const float pixdim[3], const nrb_f3d_params *p,
                             int64_t *bytes);

/* A registration server on the current device (no counterpart in the reference: reg_f3d
 * registers one pair per process). `slots` workers, each with its own stream, take requests in
 * arrival order: a free worker takes the queue's head once its footprint fits in what is left of
 * hbm_budget_bytes (<= 0: 80% of the free device memory; a request always runs when nothing else
 * does), together with the queued requests that can share its group (the same parameters, a
 * volume within a factor of two of the head's, up to max_group requests, within the budget), and
 * registers the group as nrb_f3d_register_batch does. Requests that arrive while groups run wait
 * for the next free worker and run beside them; each result is the one nrb_f3d_register_host
 * gives for the same request alone. nrb_server_create uses max_group = 16. While servers exist
 * on a device, the library's memory pool there keeps freed memory up to the budget (release
 * threshold); its previous threshold comes back when the last server is destroyed. The
 * application's default memory pool is not touched. */
typedef struct nrb_server nrb_server;
nrb_status nrb_server_create(int slots, int64_t hbm_budget_bytes, nrb_server **out);
nrb_status nrb_server_create_grouped(int slots, int max_group, int64_t hbm_budget_bytes, nrb_server **out);
nrb_status nrb_server_submit(nrb_server *s, const nrb_pair *req, const nrb_f3d_params *p,
                             int64_t *ticket);
/* Blocks until the request ends; queue_seconds = submit -> admission, latency_seconds =
 * submit -> result. A ticket is waited on once: a second wait on it (another thread, or after
 * the first returned) returns NRB_ERR_INVALID. */
nrb_status nrb_server_wait(nrb_server *s, int64_t ticket, nrb_f3d_result *result,
                           double *queue_seconds, double *latency_seconds);
/* Peak admitted footprint and peak number of concurrent registrations so far. */
nrb_status nrb_server_stats(nrb_server *s, int64_t *peak_bytes, int32_t *peak_active);
/* Largest group registered together so far. */
nrb_status nrb_server_peak_group(nrb_server *s, int32_t *peak_group);
/* Finishes the queued requests, then stops the workers. */
void nrb_server_destroy(nrb_server *s);

/* n registrations advanced together (no counterpart in the reference, which registers one pair
 * per reg_f3d run). The pairs are taken in order of size in groups of at most `concurrency`
 * (<= 64) whose summed footprints fit in hbm_budget_bytes (<= 0: 80% of the free device memory)
 * and, when p->batch_group_mb is set, whose finest-level images fit in it; a group runs level
 * by level, each level as one CUDA graph in which every stage -- the line-search
 * objective, its finalize, the gradient, the node convolution, the conjugate-gradient direction
 * -- is one launch over all the pairs that need it. When the pairs make two or more groups that
 * each fit in half the budget, two host threads run the groups, so that one group's uploads,
 * pyramids and level set-up overlap the other's graphs on the device; otherwise the groups run
 * one after another with the whole budget. Each pair's arithmetic is that of its plain
 * registration, so results[i] and pairs[i].cpp_out_host equal nrb_f3d_register_host's for pair i
 * alone, bit for bit. The pairs of a group share the parameters, so they share the bin counts;
 * they may differ in size and spacing. */
nrb_status nrb_f3d_register_batch(const nrb_pair *pairs, int n, const nrb_f3d_params *p,
                                  int concurrency, int64_t hbm_budget_bytes,
                                  nrb_f3d_result *results);

/* Number of kernel launches issued by this library in this process so far. */
int64_t nrb_kernel_launch_count(void);

/* Per-kernel CUDA-event timing (no counterpart in the reference, which only offers the wall
 * clocks of reg-apps/reg_benchmark.cpp). While enabled, every launch of the timed kernels is
 * bracketed by events on its own stream; enabling clears the counters. nrb_timing_read returns,
 * for "objective", "gradient", "finalize", "conv", "be_value" or "be_gradient", the launches,
 * their summed device time and the algorithmic bytes those launches had to move. */
void nrb_timing_enable(int on);
nrb_status nrb_timing_read(const char *kernel, int64_t *launches, double *total_ms,
                           double *algorithmic_bytes);

#ifdef __cplusplus
}
#endif
#endif /* NIFTYREG_B200_H */
