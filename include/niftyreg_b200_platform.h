/* NiftyReg's reg_f3d on the B200 platform: a C entry of libniftyreg_b200_platform.so, the
 * reference's registration library (reg-lib, reg-io) built from its own sources with the B200
 * platform's classes (niftyreg_b200/platform) in place of reg-lib/Platform.cpp. reg_f3d<float>,
 * its conjugate-gradient optimiser and pyramid driver run unchanged; on the B200 platform every
 * Compute / measure / optimiser step is one call of niftyreg_b200.h on the device.
 *
 * Plain pointers and sizes; every array is a HOST array. */
#ifndef NIFTYREG_B200_PLATFORM_H
#define NIFTYREG_B200_PLATFORM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NRB_PLATFORM_CPU 0   /* PlatformType::Cpu (reg-lib/Platform.h:10) */
#define NRB_PLATFORM_B200 1  /* the B200 platform (PlatformType value 3) */
#define NRB_PLATFORM_MAX_LEVELS 8

/* The reg_f3d settings the F3D hot path uses (reg-apps/reg_f3d.cpp options in brackets). */
typedef struct nrb_platform_params {
    int32_t platform;        /* NRB_PLATFORM_CPU or NRB_PLATFORM_B200 [-platf] */
    int32_t gpu;             /* device index for the B200 platform, -1: the current one [-gpuid] */
    int32_t levels;          /* pyramid levels, all performed [-ln] */
    int32_t max_iterations;  /* finest-level budget, doubled per coarser level [-maxit] */
    float bending_energy;    /* [-be] */
    float linear_energy;     /* [-le]; must be 0 on the B200 platform */
    float spacing;           /* control-point spacing: negative = voxels, positive = mm [-sx] */
    int32_t bins;            /* NMI bins of both images [--rbn/--fbn] */
    int32_t verbose;         /* 0: DoNotPrintOutInformation */
    float padding;           /* warped padding value, NaN by default [-pad] */
} nrb_platform_params;

typedef struct nrb_platform_result {
    int32_t cpp_dim[3];      /* final grid dims; the grid is 3 * prod(cpp_dim) floats */
    double final_nmi;        /* best NMI of the last level (bestWMeasure / similarity weight) */
    int64_t objective_evaluations;  /* reg_f3d::GetObjectiveFunctionValue calls */
    int64_t gradient_evaluations;   /* reg_f3d::GetObjectiveFunctionGradient calls */
    double seconds;          /* host wall time around reg_f3d<float>::Run */
    double level_seconds[NRB_PLATFORM_MAX_LEVELS];
} nrb_platform_result;

/* Text of the last error (a NiftyReg fatal error or a CUDA error) on this thread. */
const char *nrb_platform_last_error(void);

/* reg_f3d<float>::Run (reg-lib/_reg_base.cpp:727-818) on a reference and a floating image of
 * the same geometry: dims (nx, ny, nz), spacing and voxel->mm matrix `xyz` (row-major, used as
 * sform and qform). The final control-point positions go to cpp_out (capacity cpp_capacity
 * floats). Returns 0, or -1 with nrb_platform_last_error() set. */
int nrb_platform_f3d_register(const float *ref, const float *flo, const int32_t dim[3], const float pixdim[3],
                              const float xyz[16], const nrb_platform_params *p, float *cpp_out,
                              int64_t cpp_capacity, nrb_platform_result *result);

#ifdef __cplusplus
}
#endif

#endif
