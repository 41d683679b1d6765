/* Test infrastructure only: plain-C restatement of the NiftyReg F3D objective-and-gradient path.
 * It is the checker for the CUDA kernels and is never linked into the product.
 *
 * Conventions: volumes are float32, x fastest ([nz][ny][nx]); vector images are planar
 * ([x plane | y plane | z plane]); matrices are row-major float[16] (NIfTI mat44 layout);
 * masks are int32 with -1 = inactive, NULL = every voxel active. */
#ifndef NRB_ORACLE_H
#define NRB_ORACLE_H
#include <stddef.h>

void orc_bspline_basis(float t, float b[4]);
int orc_deformation_field(const float *cpp, const int cdim[3], const float cpix[3],
                          const int rdim[3], const float rpix[3], const int *mask, float *def);
int orc_resample_linear(const float *flo, const int fdim[3], const float flo_ijk[16],
                        const float *def, const int rdim[3], const int *mask, float pad,
                        float *warped);
int orc_resample_order(const float *flo, const int fdim[3], const float flo_ijk[16], const float *def,
                       const int rdim[3], const int *mask, float pad, int order, float *warped);
int orc_image_gradient_linear(const float *flo, const int fdim[3], const float flo_ijk[16],
                              const float *def, const int rdim[3], const int *mask, float pad,
                              float *grad);
void orc_intensity_rescale(float *img, size_t n, float new_min, float new_max);
double orc_nmi_value(const float *ref, const float *war, size_t n, const int *mask, int ref_bins,
                     int flo_bins, double *pro, double *logh, double *ent);
void orc_nmi_voxel_gradient(const float *ref, const float *war, const float *wgrad, size_t n,
                            const int *mask, int ref_bins, int flo_bins, const double *logh,
                            const double *ent, double weight, float *vgrad);
void orc_kernel_convolution_cubic(float *img, int nvol, const int dim[3], const float pix[3],
                                  float spacing_mm, int axis, const int *mask);
void orc_voxel_to_node(float *node, const int cdim[3], const float grid_xyz[16],
                       const float *voxel, const int rdim[3], const float rpix[3],
                       const float ref_ijk[16], const float reorient[16], float weight,
                       int update);
void orc_convolve_to_nodes(float *vgrad, const int rdim[3], const float rpix[3],
                           const float ref_ijk[16], const int cdim[3], const float cpix[3],
                           const float grid_xyz[16], const float flo_ijk[16], float weight,
                           float *node);
double orc_be_value(const float *cpp, const int cdim[3]);
void orc_be_gradient(const float *cpp, const int cdim[3], const float grid_xyz[16], float weight,
                     float *grad);
double orc_max_length(const float *grad, size_t nnode, int ox, int oy, int oz);
void orc_normalise_gradient(float *grad, size_t nnode, double maxlen, int ox, int oy, int oz);
void orc_update_control_points(float *cur, const float *best, const float *grad, float scale,
                               size_t nvox);
void orc_cg_update(float *grad, float *g1, float *g2, size_t nvox, int first_call);

/* F3D2 (reg_f3d2): velocity fields */
int orc_velocity_squaring_steps(float lo, float hi);
int orc_velocity_def_field(const float *vel, const int gdim[3], const float gxyz[16], int steps, int update,
                           const int fdim[3], const float fxyz[16], float *def, int *steps_out);
void orc_def_compose(const int dim[3], const float xyz[16], const float *apply, float *update);
int orc_exponentiate_gradient(const int fdim[3], const float fxyz[16], const float *vel, const int gdim[3],
                              const float gxyz[16], int steps, float *vgrad);
void orc_symmetrise(const int gdim[3], const float fw_xyz[16], const float bw_xyz[16], float *fw, float *bw);

#endif
