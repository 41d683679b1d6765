// Test infrastructure only: a C-ABI adapter over the reference NiftyReg CPU library, compiled
// together with the reference's own sources into oracle/_ref/libnrref.so by oracle/Makefile.
// It lets the tests and the CPU baseline call the reference's hot-path functions on plain float
// arrays. Nothing in the product links or loads this file.
//
// Geometry convention of every entry point: an image is (dim[3], pixdim[3], xyz[16]) where xyz
// is the row-major voxel->mm matrix. The shim installs it as the image's sform (sform_code 1)
// and lets the reference derive sto_ijk itself with nifti_mat44_inverse.
#include <omp.h>
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>
#include "_reg_f3d.h"
#include "_reg_f3d2.h"
#include "_reg_localTrans.h"
#include "_reg_localTrans_regul.h"
#include "_reg_nmi.h"
#include "_reg_resampling.h"
#include "_reg_tools.h"
#include "Compute.h"
#include "F3dContent.h"

namespace {

mat44 ToMat(const float *m) {
    mat44 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r.m[i][j] = m[4 * i + j];
    return r;
}

// Scalar (nu = 1) or vector (nu = 3) float image with an sform built from xyz.
NiftiImage MakeImage(const int *dim, const float *pix, const float *xyz, int nu = 1) {
    std::vector<NiftiImage::dim_t> dims{ dim[0], dim[1], dim[2] };
    if (nu > 1) { dims.push_back(1); dims.push_back(nu); }
    NiftiImage img(dims, NIFTI_TYPE_FLOAT32);
    img.setPixDim(NiftiDim::X, pix[0]);
    img.setPixDim(NiftiDim::Y, pix[1]);
    img.setPixDim(NiftiDim::Z, pix[2]);
    img->sform_code = 1;
    img->sto_xyz = ToMat(xyz);
    img->sto_ijk = nifti_mat44_inverse(img->sto_xyz);
    // a qform consistent with the sform keeps every reference code path well defined
    img->qform_code = 1;
    nifti_mat44_to_quatern(img->sto_xyz, &img->quatern_b, &img->quatern_c, &img->quatern_d,
                           &img->qoffset_x, &img->qoffset_y, &img->qoffset_z, nullptr, nullptr,
                           nullptr, &img->qfac);
    img->qto_xyz = nifti_quatern_to_mat44(img->quatern_b, img->quatern_c, img->quatern_d,
                                          img->qoffset_x, img->qoffset_y, img->qoffset_z,
                                          pix[0], pix[1], pix[2], img->qfac);
    img->qto_ijk = nifti_mat44_inverse(img->qto_xyz);
    return img;
}

size_t Nvox(const int *d) { return size_t(d[0]) * d[1] * d[2]; }

// Exposes the protected histogram buffers of reg_nmi and lets a caller evaluate NMI on
// intensities that are already rescaled to [2, bins-3].
class ShimNmi: public reg_nmi {
public:
    void Setup(NiftiImage& ref, NiftiImage& war, NiftiImage& warGrad, NiftiImage& voxGrad,
               int *mask, int refBins, int floBins, double weight, bool approx) {
        SetTimePointWeight(0, weight);
        SetReferenceBinNumber(refBins, 0);
        SetFloatingBinNumber(floBins, 0);
        // InitialiseMeasure rescales the images it is given: hand it throw-away copies, then
        // point the measure at the caller's already-rescaled reference.
        refCopy = NiftiImage(ref, NiftiImage::Copy::Image);
        floCopy = NiftiImage(war, NiftiImage::Copy::Image);
        InitialiseMeasure(refCopy, floCopy, mask, war, warGrad, voxGrad);
        this->referenceImage = ref;
        if (approx) ApproximatePw(); else DoNotApproximatePw();
    }
    double *Pro() { return jointHistogramPro[0]; }
    double *Log() { return jointHistogramLog[0]; }
    double *Ent() { return entropyValues[0]; }
    int Total() { return totalBinNumber[0]; }
private:
    NiftiImage refCopy, floCopy;
};

// reg_f3d with evaluation counters and access to the final objective terms.
class ShimF3d: public reg_f3d<float> {
public:
    ShimF3d(): reg_f3d<float>(1, 1) {}
    double GetObjectiveFunctionValue() override { ++objCalls; return reg_f3d<float>::GetObjectiveFunctionValue(); }
    void GetObjectiveFunctionGradient() override { ++gradCalls; reg_f3d<float>::GetObjectiveFunctionGradient(); }
    // marks the start of every pyramid level for the per-level statistics
    float InitCurrentLevel(int level) override {
        if (level >= 0) marks.push_back({ std::chrono::steady_clock::now(), objCalls, gradCalls });
        return reg_f3d<float>::InitCurrentLevel(level);
    }
    double FinalWMeasure() const { return this->bestWMeasure; }
    double FinalWBE() const { return bestWBE; }
    double SimilarityWeight() const { return this->similarityWeight; }
    struct Mark {
        std::chrono::steady_clock::time_point t;
        long obj, grad;
    };
    std::vector<Mark> marks;
    long objCalls = 0, gradCalls = 0;
};

class ShimF3d2: public reg_f3d2<float> {
public:
    ShimF3d2(): reg_f3d2<float>(1, 1) {}
    double GetObjectiveFunctionValue() override { ++objCalls; return reg_f3d2<float>::GetObjectiveFunctionValue(); }
    void GetObjectiveFunctionGradient() override { ++gradCalls; reg_f3d2<float>::GetObjectiveFunctionGradient(); }
    double FinalWMeasure() const { return this->bestWMeasure; }
    double FinalWBE() const { return this->bestWBE; }
    double SimilarityWeight() const { return this->similarityWeight; }
    long objCalls = 0, gradCalls = 0;
};

// a cubic B-spline velocity grid as reg_f3d2 tags it
NiftiImage MakeVelocityGrid(const int *gdim, const float *gpix, const float *gxyz, const float *vel, int steps) {
    NiftiImage grid = MakeImage(gdim, gpix, gxyz, 3);
    memcpy(grid->data, vel, grid->nvox * sizeof(float));
    grid->intent_code = NIFTI_INTENT_VECTOR;
    grid->intent_p1 = SPLINE_VEL_GRID;
    grid->intent_p2 = float(steps);
    return grid;
}

}  // namespace

extern "C" {

int ref_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

// _reg_localTrans.cpp:21-128
int ref_create_control_point_grid(const int *rdim, const float *rpix, const float *rxyz,
                                  const float *spacing, int *cdim, float *cpix, float *cxyz,
                                  float *cpp_out, size_t cap) {
    NiftiImage ref = MakeImage(rdim, rpix, rxyz);
    NiftiImage grid;
    reg_createControlPointGrid<float>(grid, ref, spacing);
    cdim[0] = grid->nx; cdim[1] = grid->ny; cdim[2] = grid->nz;
    cpix[0] = grid->dx; cpix[1] = grid->dy; cpix[2] = grid->dz;
    const mat44& m = grid->sform_code > 0 ? grid->sto_xyz : grid->qto_xyz;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) cxyz[4 * i + j] = m.m[i][j];
    if (cpp_out) {
        if (cap < grid->nvox) return -1;
        memcpy(cpp_out, grid->data, grid->nvox * sizeof(float));
    }
    return 0;
}

// _reg_localTrans.cpp:1457-1538
int ref_deformation_field(const float *cpp, const int *cdim, const float *cpix, const float *cxyz,
                          const int *rdim, const float *rpix, const float *rxyz,
                          const int *mask, float *def_out) {
    NiftiImage grid = MakeImage(cdim, cpix, cxyz, 3);
    memcpy(grid->data, cpp, grid->nvox * sizeof(float));
    NiftiImage def = MakeImage(rdim, rpix, rxyz, 3);
    reg_spline_getDeformationField(grid, def, const_cast<int *>(mask), false, true);
    memcpy(def_out, def->data, def->nvox * sizeof(float));
    return 0;
}

// _reg_resampling.cpp:638-692
int ref_resample(const float *flo, const int *fdim, const float *fpix, const float *fxyz,
                 const float *def, const int *rdim, const float *rpix, const float *rxyz,
                 const int *mask, float pad, float *warped_inout) {
    NiftiImage fimg = MakeImage(fdim, fpix, fxyz);
    memcpy(fimg->data, flo, Nvox(fdim) * sizeof(float));
    NiftiImage dimg = MakeImage(rdim, rpix, rxyz, 3);
    memcpy(dimg->data, def, 3 * Nvox(rdim) * sizeof(float));
    NiftiImage wimg = MakeImage(rdim, rpix, rxyz);
    memcpy(wimg->data, warped_inout, Nvox(rdim) * sizeof(float));
    reg_resampleImage(fimg, wimg, dimg, mask, 1, pad);
    memcpy(warped_inout, wimg->data, Nvox(rdim) * sizeof(float));
    return 0;
}

// reg_io_ReadImageFile's reading of a single-file NIfTI image (reg-io/_reg_ReadWriteImage.cpp:
// 51-81): niftilib, then reg_checkAndCorrectDimension; the voxel -> mm matrix Content picks (the
// sform when sform_code > 0, else the qform); data converted to float (reg_tools_changeDatatype)
// and scaled by scl_slope / scl_inter as the intensity rescale does. With data == nullptr only the
// sizes are returned.
int ref_image_read(const char *path, int *dim, int *nvol, float *pixdim, float *xyz, float *data) {
    nifti_image *im = nifti_image_read(path, data != nullptr);
    if (!im) return -1;
    reg_checkAndCorrectDimension(im);
    for (int i = 0; i < 3; ++i) {
        dim[i] = im->dim[i + 1];
        pixdim[i] = im->pixdim[i + 1];
    }
    long long nv = 1;
    for (int i = 4; i <= 7; ++i) nv *= im->dim[i] > 0 ? im->dim[i] : 1;
    *nvol = (int)nv;
    const mat44& m = im->sform_code > 0 ? im->sto_xyz : im->qto_xyz;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) xyz[4 * i + j] = m.m[i][j];
    if (data) {
        reg_tools_changeDatatype<float>(im);
        const float slope = im->scl_slope == 0 ? 1.f : im->scl_slope, inter = im->scl_inter;
        const float *src = static_cast<float *>(im->data);
        for (size_t i = 0; i < im->nvox; ++i)
            data[i] = (slope == 1.f && inter == 0.f) ? src[i] : (float)((double)src[i] * slope + inter);
    }
    nifti_image_free(im);
    return 0;
}

// _reg_resampling.cpp:638-692 with the interpolation order (0 nearest, 1 linear, 3 cubic spline)
int ref_resample_order(const float *flo, const int *fdim, const float *fpix, const float *fxyz,
                       const float *def, const int *rdim, const float *rpix, const float *rxyz,
                       const int *mask, float pad, int order, float *warped_inout) {
    NiftiImage fimg = MakeImage(fdim, fpix, fxyz);
    memcpy(fimg->data, flo, Nvox(fdim) * sizeof(float));
    NiftiImage dimg = MakeImage(rdim, rpix, rxyz, 3);
    memcpy(dimg->data, def, 3 * Nvox(rdim) * sizeof(float));
    NiftiImage wimg = MakeImage(rdim, rpix, rxyz);
    memcpy(wimg->data, warped_inout, Nvox(rdim) * sizeof(float));
    reg_resampleImage(fimg, wimg, dimg, mask, order, pad);
    memcpy(warped_inout, wimg->data, Nvox(rdim) * sizeof(float));
    return 0;
}

// _reg_resampling.cpp:2328-2384
int ref_image_gradient(const float *flo, const int *fdim, const float *fpix, const float *fxyz,
                       const float *def, const int *rdim, const float *rpix, const float *rxyz,
                       const int *mask, float pad, float *grad_out) {
    NiftiImage fimg = MakeImage(fdim, fpix, fxyz);
    memcpy(fimg->data, flo, Nvox(fdim) * sizeof(float));
    NiftiImage dimg = MakeImage(rdim, rpix, rxyz, 3);
    memcpy(dimg->data, def, 3 * Nvox(rdim) * sizeof(float));
    NiftiImage gimg = MakeImage(rdim, rpix, rxyz, 3);
    reg_getImageGradient(fimg, gimg, dimg, mask, 1, pad, 0);
    memcpy(grad_out, gimg->data, 3 * Nvox(rdim) * sizeof(float));
    return 0;
}

// _reg_tools.cpp:92-174
int ref_intensity_rescale(float *img, const int *dim, float new_min, float new_max) {
    const float pix[3] = { 1, 1, 1 };
    const float eye[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
    NiftiImage im = MakeImage(dim, pix, eye);
    memcpy(im->data, img, Nvox(dim) * sizeof(float));
    reg_intensityRescale(im, 0, new_min, new_max);
    memcpy(img, im->data, Nvox(dim) * sizeof(float));
    return 0;
}

// _reg_nmi.cpp:160-398. Images must already be rescaled to [2, bins-3].
double ref_nmi_value(const float *ref, const float *war, const int *dim, const int *mask,
                     int ref_bins, int flo_bins, int approx, double *pro_out, double *log_out,
                     double *ent_out) {
    const float pix[3] = { 1, 1, 1 };
    const float eye[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
    NiftiImage r = MakeImage(dim, pix, eye), w = MakeImage(dim, pix, eye);
    NiftiImage wg = MakeImage(dim, pix, eye, 3), vg = MakeImage(dim, pix, eye, 3);
    memcpy(r->data, ref, Nvox(dim) * sizeof(float));
    memcpy(w->data, war, Nvox(dim) * sizeof(float));
    std::unique_ptr<int[]> m(new int[Nvox(dim)]());
    if (mask) memcpy(m.get(), mask, Nvox(dim) * sizeof(int));
    ShimNmi nmi;
    nmi.Setup(r, w, wg, vg, m.get(), ref_bins, flo_bins, 1.0, approx != 0);
    const double v = nmi.GetSimilarityMeasureValueFw();
    if (pro_out) memcpy(pro_out, nmi.Pro(), nmi.Total() * sizeof(double));
    if (log_out) memcpy(log_out, nmi.Log(), nmi.Total() * sizeof(double));
    if (ent_out) memcpy(ent_out, nmi.Ent(), 4 * sizeof(double));
    return v;
}

// _reg_nmi.cpp:501-638: recomputes the histogram, then adds the voxel-wise NMI gradient.
int ref_nmi_voxel_gradient(const float *ref, const float *war, const float *war_grad,
                           const int *dim, const int *mask, int ref_bins, int flo_bins,
                           double weight, float *vgrad_inout) {
    const float pix[3] = { 1, 1, 1 };
    const float eye[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
    NiftiImage r = MakeImage(dim, pix, eye), w = MakeImage(dim, pix, eye);
    NiftiImage wg = MakeImage(dim, pix, eye, 3), vg = MakeImage(dim, pix, eye, 3);
    memcpy(r->data, ref, Nvox(dim) * sizeof(float));
    memcpy(w->data, war, Nvox(dim) * sizeof(float));
    memcpy(wg->data, war_grad, 3 * Nvox(dim) * sizeof(float));
    memcpy(vg->data, vgrad_inout, 3 * Nvox(dim) * sizeof(float));
    std::unique_ptr<int[]> m(new int[Nvox(dim)]());
    if (mask) memcpy(m.get(), mask, Nvox(dim) * sizeof(int));
    ShimNmi nmi;
    nmi.Setup(r, w, wg, vg, m.get(), ref_bins, flo_bins, weight, true);
    nmi.GetVoxelBasedSimilarityMeasureGradientFw(0);
    memcpy(vgrad_inout, vg->data, 3 * Nvox(dim) * sizeof(float));
    return 0;
}

// Compute.cpp:230-281: cubic-spline convolution of the voxel-based gradient along x, y, z with
// the grid spacing, then voxel->node sampling, reorientation by the floating ijk matrix and
// weighting. vgrad_inout receives the convolved voxel gradient, node_out the node gradient.
int ref_convolve_to_nodes(float *vgrad_inout, const int *rdim, const float *rpix, const float *rxyz,
                          const int *fdim, const float *fpix, const float *fxyz,
                          const int *cdim, const float *cpix, const float *cxyz,
                          float weight, float *node_out) {
    NiftiImage r = MakeImage(rdim, rpix, rxyz), f = MakeImage(fdim, fpix, fxyz);
    NiftiImage g = MakeImage(cdim, cpix, cxyz, 3);
    F3dContent con(r, f, g);
    memcpy(con.GetVoxelBasedMeasureGradient()->data, vgrad_inout, 3 * Nvox(rdim) * sizeof(float));
    Compute compute(con);
    compute.ConvolveVoxelBasedMeasureGradient(weight);
    memcpy(vgrad_inout, con.GetVoxelBasedMeasureGradient()->data, 3 * Nvox(rdim) * sizeof(float));
    memcpy(node_out, con.GetTransformationGradient()->data, 3 * Nvox(cdim) * sizeof(float));
    return 0;
}

// _reg_tools.cpp:831-1112, one axis (0, 1 or 2) of the cubic kernel with spacing in mm.
int ref_kernel_convolution_cubic(float *img_inout, int nvol, const int *dim, const float *pix,
                                 float spacing, int axis) {
    const float eye[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
    NiftiImage im = MakeImage(dim, pix, eye, nvol);
    memcpy(im->data, img_inout, size_t(nvol) * Nvox(dim) * sizeof(float));
    std::vector<float> sigma(nvol, spacing);
    bool axes[3] = { axis == 0, axis == 1, axis == 2 };
    reg_tools_kernelConvolution(im, sigma.data(), ConvKernelType::Cubic, nullptr, nullptr, axes);
    memcpy(img_inout, im->data, size_t(nvol) * Nvox(dim) * sizeof(float));
    return 0;
}

// _reg_localTrans_regul.cpp:155-177
double ref_be_value(const float *cpp, const int *cdim, const float *cpix, const float *cxyz) {
    NiftiImage g = MakeImage(cdim, cpix, cxyz, 3);
    memcpy(g->data, cpp, g->nvox * sizeof(float));
    return reg_spline_approxBendingEnergy(g);
}

// _reg_localTrans_regul.cpp:453-482 (adds into grad_inout)
int ref_be_gradient(const float *cpp, const int *cdim, const float *cpix, const float *cxyz,
                    float weight, float *grad_inout) {
    NiftiImage g = MakeImage(cdim, cpix, cxyz, 3);
    memcpy(g->data, cpp, g->nvox * sizeof(float));
    NiftiImage gr = MakeImage(cdim, cpix, cxyz, 3);
    memcpy(gr->data, grad_inout, gr->nvox * sizeof(float));
    reg_spline_approxBendingEnergyGradient(g, gr, weight);
    memcpy(grad_inout, gr->data, gr->nvox * sizeof(float));
    return 0;
}

// reg_createImagePyramid<float> (_reg_tools.cpp:1705-1733) with `levels` levels, all performed:
// the levels end to end in out (coarsest first), their dims and sform matrices; out may be null
// to query the total. Returns the total float count, or -1 when cap is too small.
long long ref_image_pyramid(const float *img, const int *dim, const float *pix, const float *xyz, int levels,
                            float *out, size_t cap, int *dims_out, float *xyz_out) {
    NiftiImage im = MakeImage(dim, pix, xyz);
    memcpy(im->data, img, Nvox(dim) * sizeof(float));
    std::vector<NiftiImage> pyr(levels);
    reg_createImagePyramid<float>(im, pyr, unsigned(levels), unsigned(levels));
    size_t total = 0;
    for (int l = 0; l < levels; ++l) {
        dims_out[3 * l] = pyr[l]->nx;
        dims_out[3 * l + 1] = pyr[l]->ny;
        dims_out[3 * l + 2] = pyr[l]->nz;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) xyz_out[16 * l + 4 * i + j] = pyr[l]->sto_xyz.m[i][j];
        total += pyr[l]->nvox;
    }
    if (!out) return (long long)total;
    if (cap < total) return -1;
    size_t off = 0;
    for (int l = 0; l < levels; ++l) {
        memcpy(out + off, pyr[l]->data, pyr[l]->nvox * sizeof(float));
        off += pyr[l]->nvox;
    }
    return (long long)total;
}

// _reg_localTrans.cpp:2121-2170 (grid refinement onto the reference image)
int ref_refine_grid(const float *cpp, const int *cdim, const float *cpix, const float *cxyz,
                    const int *rdim, const float *rpix, const float *rxyz,
                    int *cdim_out, float *cpix_out, float *cxyz_out, float *cpp_out, size_t cap) {
    NiftiImage g = MakeImage(cdim, cpix, cxyz, 3);
    memcpy(g->data, cpp, g->nvox * sizeof(float));
    NiftiImage r = MakeImage(rdim, rpix, rxyz);
    reg_spline_refineControlPointGrid(g, r);
    cdim_out[0] = g->nx; cdim_out[1] = g->ny; cdim_out[2] = g->nz;
    cpix_out[0] = g->dx; cpix_out[1] = g->dy; cpix_out[2] = g->dz;
    const mat44& m = g->sform_code > 0 ? g->sto_xyz : g->qto_xyz;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) cxyz_out[4 * i + j] = m.m[i][j];
    if (cap < g->nvox) return -1;
    memcpy(cpp_out, g->data, g->nvox * sizeof(float));
    return 0;
}

// Full F3D registration through reg_f3d<float>::Run (_reg_base.cpp:727-818).
// params: [0] levels, [1] max iterations (finest level), [2] bending-energy weight,
//         [3] linear-energy weight, [4] bins, [5] spacing (negative: voxels), [6] verbose
// stats:  [0] final NMI (best wSIM / similarity weight), [1] final wBE, [2] objective
//         evaluations, [3] gradient evaluations, [4] wall seconds, then per level l
//         [5 + 3l] objective evaluations, [6 + 3l] gradient evaluations, [7 + 3l] seconds
//         (stats must hold 5 + 3 * levels doubles)
int ref_f3d_register(const float *ref, const float *flo, const int *dim, const float *pix,
                     const float *xyz, const double *params, int *cdim_out, float *cpp_out,
                     size_t cap, double *stats) {
    NiftiImage r = MakeImage(dim, pix, xyz), f = MakeImage(dim, pix, xyz);
    memcpy(r->data, ref, Nvox(dim) * sizeof(float));
    memcpy(f->data, flo, Nvox(dim) * sizeof(float));
    ShimF3d reg;
    reg.SetReferenceImage(r);
    reg.SetFloatingImage(f);
    reg.SetLevelNumber(unsigned(params[0]));
    reg.SetLevelToPerform(unsigned(params[0]));
    reg.SetMaximalIterationNumber(unsigned(params[1]));
    reg.SetBendingEnergyWeight(float(params[2]));
    reg.SetLinearEnergyWeight(float(params[3]));
    reg.UseNMISetReferenceBinNumber(0, int(params[4]));
    reg.UseNMISetFloatingBinNumber(0, int(params[4]));
    reg.SetSpacing(0, float(params[5]));
    if (params[6] == 0) reg.DoNotPrintOutInformation();
    const auto t0 = std::chrono::steady_clock::now();
    reg.Run();
    const auto t1 = std::chrono::steady_clock::now();
    NiftiImage grid = reg.GetControlPointPositionImage();
    cdim_out[0] = grid->nx; cdim_out[1] = grid->ny; cdim_out[2] = grid->nz;
    if (cpp_out) {
        if (cap < grid->nvox) return -1;
        memcpy(cpp_out, grid->data, grid->nvox * sizeof(float));
    }
    stats[0] = reg.SimilarityWeight() > 0 ? reg.FinalWMeasure() / reg.SimilarityWeight() : 0;
    stats[1] = reg.FinalWBE();
    stats[2] = double(reg.objCalls);
    stats[3] = double(reg.gradCalls);
    stats[4] = std::chrono::duration<double>(t1 - t0).count();
    reg.marks.push_back({ t1, reg.objCalls, reg.gradCalls });
    for (size_t l = 0; l + 1 < reg.marks.size(); ++l) {
        stats[5 + 3 * l] = double(reg.marks[l + 1].obj - reg.marks[l].obj);
        stats[6 + 3 * l] = double(reg.marks[l + 1].grad - reg.marks[l].grad);
        stats[7 + 3 * l] = std::chrono::duration<double>(reg.marks[l + 1].t - reg.marks[l].t).count();
    }
    return 0;
}

// the same registration with a reference and a floating image of their own dims, spacings and
// voxel -> mm matrices (both sform images); also returns the final grid's voxel -> mm matrix
int ref_f3d_register2(const float *ref, const int *rdim, const float *rpix, const float *rxyz, const float *flo,
                      const int *fdim, const float *fpix, const float *fxyz, const double *params, int *cdim_out,
                      float *cpp_out, size_t cap, float *cxyz_out, double *stats) {
    NiftiImage r = MakeImage(rdim, rpix, rxyz), f = MakeImage(fdim, fpix, fxyz);
    memcpy(r->data, ref, Nvox(rdim) * sizeof(float));
    memcpy(f->data, flo, Nvox(fdim) * sizeof(float));
    ShimF3d reg;
    reg.SetReferenceImage(r);
    reg.SetFloatingImage(f);
    reg.SetLevelNumber(unsigned(params[0]));
    reg.SetLevelToPerform(unsigned(params[0]));
    reg.SetMaximalIterationNumber(unsigned(params[1]));
    reg.SetBendingEnergyWeight(float(params[2]));
    reg.SetLinearEnergyWeight(float(params[3]));
    reg.UseNMISetReferenceBinNumber(0, int(params[4]));
    reg.UseNMISetFloatingBinNumber(0, int(params[4]));
    reg.SetSpacing(0, float(params[5]));
    if (params[6] == 0) reg.DoNotPrintOutInformation();
    reg.Run();
    NiftiImage grid = reg.GetControlPointPositionImage();
    cdim_out[0] = grid->nx; cdim_out[1] = grid->ny; cdim_out[2] = grid->nz;
    if (cap < grid->nvox) return -1;
    memcpy(cpp_out, grid->data, grid->nvox * sizeof(float));
    const mat44& m = grid->sform_code > 0 ? grid->sto_xyz : grid->qto_xyz;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) cxyz_out[4 * i + j] = m.m[i][j];
    stats[0] = reg.SimilarityWeight() > 0 ? reg.FinalWMeasure() / reg.SimilarityWeight() : 0;
    stats[1] = reg.FinalWBE();
    stats[2] = double(reg.objCalls);
    stats[3] = double(reg.gradCalls);
    return 0;
}

// reg_spline_getDefFieldFromVelocityGrid on a deformation field of the given geometry
int ref_velocity_def_field(const float *vel, const int *gdim, const float *gpix, const float *gxyz, int steps,
                           int update, const int *fdim, const float *fpix, const float *fxyz, float *def_out,
                           int *steps_out) {
    NiftiImage grid = MakeVelocityGrid(gdim, gpix, gxyz, vel, steps);
    NiftiImage field = MakeImage(fdim, fpix, fxyz, 3);
    reg_spline_getDefFieldFromVelocityGrid(grid, field, update != 0);
    memcpy(def_out, field->data, field->nvox * sizeof(float));
    *steps_out = int(grid->intent_p2);
    return 0;
}

// reg_defField_compose: update <- apply(update)
int ref_def_compose(const int *dim, const float *pix, const float *xyz, const float *apply, float *update) {
    NiftiImage a = MakeImage(dim, pix, xyz, 3), u = MakeImage(dim, pix, xyz, 3);
    memcpy(a->data, apply, a->nvox * sizeof(float));
    memcpy(u->data, update, u->nvox * sizeof(float));
    reg_defField_compose(a, u, nullptr);
    memcpy(update, u->data, u->nvox * sizeof(float));
    return 0;
}

// Compute::ExponentiateGradient (reg-lib/Compute.cpp:288-330, no affine) with the reference's
// own functions, in its order, on a gradient image of the given geometry
int ref_exponentiate_gradient(const int *fdim, const float *fpix, const float *fxyz, const float *vel,
                              const int *gdim, const float *gpix, const float *gxyz, int steps, float *vgrad) {
    NiftiImage grid = MakeVelocityGrid(gdim, gpix, gxyz, vel, steps);
    NiftiImage field = MakeImage(fdim, fpix, fxyz, 3);
    NiftiImage grad = MakeImage(fdim, fpix, fxyz, 3);
    memcpy(grad->data, vgrad, grad->nvox * sizeof(float));
    const size_t compNum = size_t(fabs(grid->intent_p2));
    NiftiImage tempGrad(grad, NiftiImage::Copy::ImageInfoAndAllocData);
    std::unique_ptr<NiftiImage[]> tempDef(new NiftiImage[compNum + 1]);
    for (size_t i = 0; i <= compNum; ++i) tempDef[i] = NiftiImage(field, NiftiImage::Copy::ImageInfoAndAllocData);
    reg_spline_getIntermediateDefFieldFromVelGrid(grid, tempDef.get());
    for (size_t i = 0; i < compNum; ++i) {
        reg_resampleGradient(grad, tempGrad, tempDef[i], 1, 0);
        reg_tools_addImageToImage(tempGrad, grad, grad);
    }
    reg_tools_divideValueToImage(grad, grad, pow(2, compNum));
    memcpy(vgrad, grad->data, grad->nvox * sizeof(float));
    return 0;
}

// Compute::SymmetriseVelocityFields (reg-lib/Compute.cpp:356-392) with the reference's functions
int ref_symmetrise(const int *gdim, const float *gpix, const float *fw_xyz, const float *bw_xyz, float *fw,
                   float *bw) {
    NiftiImage g = MakeImage(gdim, gpix, fw_xyz, 3), gb = MakeImage(gdim, gpix, bw_xyz, 3);
    memcpy(g->data, fw, g->nvox * sizeof(float));
    memcpy(gb->data, bw, gb->nvox * sizeof(float));
    NiftiImage warpedTrans(gb, NiftiImage::Copy::ImageInfoAndAllocData);
    NiftiImage warpedTransBw(g, NiftiImage::Copy::ImageInfoAndAllocData);
    reg_getDisplacementFromDeformation(g);
    reg_getDisplacementFromDeformation(gb);
    warpedTrans.copyData(g);
    warpedTransBw.copyData(gb);
    reg_tools_subtractImageFromImage(gb, warpedTrans, gb);
    reg_tools_subtractImageFromImage(g, warpedTransBw, g);
    reg_tools_multiplyValueToImage(gb, gb, 0.5f);
    reg_tools_multiplyValueToImage(g, g, 0.5f);
    reg_getDeformationFromDisplacement(g);
    reg_getDeformationFromDisplacement(gb);
    memcpy(fw, g->data, g->nvox * sizeof(float));
    memcpy(bw, gb->data, gb->nvox * sizeof(float));
    return 0;
}

// reg_createSymmetricControlPointGrids (no affine): dims and voxel -> mm of the grids, and the
// forward grid's identity positions
int ref_symmetric_grids(const int *rdim, const float *rpix, const float *rxyz, const int *fdim, const float *fpix,
                        const float *fxyz, const float *spacing, int *gdim, float *gxyz, float *cpp_out,
                        size_t cap) {
    NiftiImage r = MakeImage(rdim, rpix, rxyz), f = MakeImage(fdim, fpix, fxyz);
    NiftiImage fw, bw;
    reg_createSymmetricControlPointGrids<float>(fw, bw, r, f, nullptr, spacing);
    gdim[0] = fw->nx; gdim[1] = fw->ny; gdim[2] = fw->nz;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) gxyz[4 * i + j] = fw->sto_xyz.m[i][j];
    if (cpp_out) {
        if (cap < fw->nvox) return -1;
        memcpy(cpp_out, fw->data, fw->nvox * sizeof(float));
    }
    return 0;
}

// reg_f3d2<float> (the -vel / -sym registration): final grids, the forward grid's voxel -> mm,
// the squaring number and [final symmetric NMI, final weighted BE, objective calls, gradient calls]
int ref_f3d2_register(const float *ref, const int *rdim, const float *rpix, const float *rxyz, const float *flo,
                      const int *fdim, const float *fpix, const float *fxyz, const double *params, int *cdim_out,
                      float *fw_out, float *bw_out, size_t cap, float *cxyz_out, int *steps_out, double *stats) {
    NiftiImage r = MakeImage(rdim, rpix, rxyz), f = MakeImage(fdim, fpix, fxyz);
    memcpy(r->data, ref, Nvox(rdim) * sizeof(float));
    memcpy(f->data, flo, Nvox(fdim) * sizeof(float));
    ShimF3d2 reg;
    reg.SetReferenceImage(r);
    reg.SetFloatingImage(f);
    reg.SetLevelNumber(unsigned(params[0]));
    reg.SetLevelToPerform(unsigned(params[0]));
    reg.SetMaximalIterationNumber(unsigned(params[1]));
    reg.SetBendingEnergyWeight(float(params[2]));
    reg.SetLinearEnergyWeight(float(params[3]));
    reg.UseNMISetReferenceBinNumber(0, int(params[4]));
    reg.UseNMISetFloatingBinNumber(0, int(params[4]));
    reg.SetSpacing(0, float(params[5]));
    if (params[6] == 0) reg.DoNotPrintOutInformation();
    reg.Run();
    NiftiImage fw = reg.GetControlPointPositionImage(), bw = reg.GetBackwardControlPointPositionImage();
    cdim_out[0] = fw->nx; cdim_out[1] = fw->ny; cdim_out[2] = fw->nz;
    if (cap < fw->nvox || cap < bw->nvox) return -1;
    memcpy(fw_out, fw->data, fw->nvox * sizeof(float));
    memcpy(bw_out, bw->data, bw->nvox * sizeof(float));
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) cxyz_out[4 * i + j] = fw->sto_xyz.m[i][j];
    *steps_out = int(fw->intent_p2);
    stats[0] = reg.SimilarityWeight() > 0 ? reg.FinalWMeasure() / reg.SimilarityWeight() : 0;
    stats[1] = reg.FinalWBE();
    stats[2] = double(reg.objCalls);
    stats[3] = double(reg.gradCalls);
    return 0;
}

}  // extern "C"
