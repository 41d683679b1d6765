// Test infrastructure only: one whole F3D objective-and-gradient evaluation through the
// reference's own functions, in FLOAT32 or FLOAT64. Compiled into both reference builds by
// oracle/Makefile: oracle/_ref/libnrref.so (the reference's default SSE build) and
// oracle/_ref64/libnrref64.so (the same sources without the SSE path, which is single precision
// only, reg-lib/cpu/_reg_localTrans.cpp:1466-1469). Nothing in the product links or loads this
// file.
//
// ref64_evaluate is the FP64 oracle: the evaluation through the reference's FLOAT64
// instantiations, from the same float inputs the single-precision path receives;
// ref32_evaluate is the same chain on FLOAT32 images, i.e. what reg_f3d<float> computes per
// gradient evaluation (_reg_base.cpp:497-548, _reg_f3d.cpp:553-576) in that build:
//   deformation field      reg_spline_getDeformationField -> <double>   (_reg_localTrans.cpp:1517-1523)
//   warp, spatial gradient reg_resampleImage / reg_getImageGradient, std::visit on double
//                          (_reg_resampling.cpp:676-687, 2366-2380)
//   NMI value and tables   reg_nmi on double images                     (_reg_nmi.cpp:361-375)
//   NMI voxel gradient     reg_getVoxelBasedNmiGradient3d<double>       (_reg_nmi.cpp:595-621)
//   convolution to nodes   reg_tools_kernelConvolution on double along x, y, z with the grid
//                          spacing, then reg_voxelCentricToNodeCentric<double> reoriented by the
//                          floating image's ijk matrix (Compute.cpp:230-281, _reg_tools.cpp:
//                          1336-1339, _reg_localTrans.cpp:1686-1705)
//   bending energy         reg_spline_approxBendingEnergy[Gradient] on a double grid
//                          (_reg_localTrans_regul.cpp:155-177, 453-482)
// The geometry convention is the one of ref_shim.cpp: (dim[3], pixdim[3], xyz[16] row-major
// voxel -> mm), installed as the sform.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>
#include "_reg_localTrans.h"
#include "_reg_localTrans_regul.h"
#include "_reg_nmi.h"
#include "_reg_resampling.h"
#include "_reg_tools.h"

namespace {

mat44 ToMat64(const float *m) {
    mat44 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r.m[i][j] = m[4 * i + j];
    return r;
}

// scalar (nu = 1) or vector (nu = 3) image of type T with an sform built from xyz
template <class T>
NiftiImage MakeImageT(const int *dim, const float *pix, const float *xyz, int nu = 1) {
    std::vector<NiftiImage::dim_t> dims{ dim[0], dim[1], dim[2] };
    if (nu > 1) { dims.push_back(1); dims.push_back(nu); }
    NiftiImage img(dims, sizeof(T) == 8 ? NIFTI_TYPE_FLOAT64 : NIFTI_TYPE_FLOAT32);
    img.setPixDim(NiftiDim::X, pix[0]);
    img.setPixDim(NiftiDim::Y, pix[1]);
    img.setPixDim(NiftiDim::Z, pix[2]);
    img->sform_code = 1;
    img->sto_xyz = ToMat64(xyz);
    img->sto_ijk = nifti_mat44_inverse(img->sto_xyz);
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

template <class T>
void Fill(NiftiImage& img, const float *src) {
    T *d = static_cast<T *>(img->data);
    for (size_t i = 0; i < img->nvox; ++i) d[i] = src[i];
}

template <class T>
void Out(const NiftiImage& img, double *dst) {
    const T *s = static_cast<const T *>(img->data);
    for (size_t i = 0; i < img->nvox; ++i) dst[i] = s[i];
}

// reg_nmi on images that already hold intensities in [2, bins - 3]: InitialiseMeasure rescales
// the images it is given, so it receives copies and the measure then points at the caller's.
class EvalNmi: public reg_nmi {
public:
    void Setup(NiftiImage& ref, NiftiImage& war, NiftiImage& warGrad, NiftiImage& voxGrad, int *mask, int refBins,
               int floBins) {
        SetTimePointWeight(0, 1.0);
        SetReferenceBinNumber(refBins, 0);
        SetFloatingBinNumber(floBins, 0);
        refCopy = NiftiImage(ref, NiftiImage::Copy::Image);
        floCopy = NiftiImage(war, NiftiImage::Copy::Image);
        InitialiseMeasure(refCopy, floCopy, mask, war, warGrad, voxGrad);
        this->referenceImage = ref;
        ApproximatePw();
    }
    const double *Ent() const { return entropyValues[0]; }

private:
    NiftiImage refCopy, floCopy;
};

size_t Nvox(const int *d) { return size_t(d[0]) * d[1] * d[2]; }

// values_out: [0] NMI, [1] bending energy (unweighted), [2] objective = sim_weight * NMI -
// be_weight * BE, [3] H_ref, [4] H_war, [5] H_joint, [6] histogram total. def_out (3N),
// warped_out (N) and node_out (3C) may be null.
template <class T>
int Evaluate(const float *ref, const int *rdim, const float *rpix, const float *rxyz, const float *flo,
             const int *fdim, const float *fpix, const float *fxyz, const float *cpp, const int *cdim,
             const float *cpix, const float *cxyz, int ref_bins, int flo_bins, double sim_weight,
             double be_weight, float pad, double *def_out, double *warped_out, double *node_out,
             double *values_out) {
    const size_t nv = Nvox(rdim);
    NiftiImage r = MakeImageT<T>(rdim, rpix, rxyz), f = MakeImageT<T>(fdim, fpix, fxyz);
    Fill<T>(r, ref);
    Fill<T>(f, flo);
    NiftiImage grid = MakeImageT<T>(cdim, cpix, cxyz, 3);
    Fill<T>(grid, cpp);
    std::unique_ptr<int[]> mask(new int[nv]());

    NiftiImage def = MakeImageT<T>(rdim, rpix, rxyz, 3);
    reg_spline_getDeformationField(grid, def, mask.get(), false, true);
    NiftiImage war = MakeImageT<T>(rdim, rpix, rxyz);
    reg_resampleImage(f, war, def, mask.get(), 1, pad);
    NiftiImage wgrad = MakeImageT<T>(rdim, rpix, rxyz, 3);
    reg_getImageGradient(f, wgrad, def, mask.get(), 1, pad, 0);
    NiftiImage vgrad = MakeImageT<T>(rdim, rpix, rxyz, 3);  // zero-filled

    EvalNmi nmi;
    nmi.Setup(r, war, wgrad, vgrad, mask.get(), ref_bins, flo_bins);
    const double v = nmi.GetSimilarityMeasureValueFw();
    nmi.GetVoxelBasedSimilarityMeasureGradientFw(0);

    // Compute::ConvolveImage: one cubic-kernel pass per axis with the grid spacing of that axis
    const float spacing[3] = { grid->dx, grid->dy, grid->dz };
    for (int axis = 0; axis < 3; ++axis) {
        float s[3] = { spacing[axis], spacing[axis], spacing[axis] };
        bool active[3] = { axis == 0, axis == 1, axis == 2 };
        reg_tools_kernelConvolution(vgrad, s, ConvKernelType::Cubic, nullptr, nullptr, active);
    }
    NiftiImage node = MakeImageT<T>(cdim, cpix, cxyz, 3);
    mat44 *reorient = f->sform_code > 0 ? &f->sto_ijk : &f->qto_ijk;
    reg_voxelCentricToNodeCentric(node, vgrad, (float)sim_weight, false, reorient);
    const double be = reg_spline_approxBendingEnergy(grid);
    if (be_weight > 0) reg_spline_approxBendingEnergyGradient(grid, node, (float)be_weight);

    const double *ent = nmi.Ent();
    values_out[0] = v;
    values_out[1] = be;
    values_out[2] = (sim_weight > 0 ? sim_weight * v : 0.0) - (be_weight > 0 ? be_weight * be : 0.0);
    values_out[3] = ent[0];
    values_out[4] = ent[1];
    values_out[5] = ent[2];
    values_out[6] = ent[3];
    if (def_out) Out<T>(def, def_out);
    if (warped_out) Out<T>(war, warped_out);
    if (node_out) Out<T>(node, node_out);
    return 0;
}

}  // namespace

extern "C" {

int ref64_evaluate(const float *ref, const int *rdim, const float *rpix, const float *rxyz, const float *flo,
                   const int *fdim, const float *fpix, const float *fxyz, const float *cpp, const int *cdim,
                   const float *cpix, const float *cxyz, int ref_bins, int flo_bins, double sim_weight,
                   double be_weight, float pad, double *def_out, double *warped_out, double *node_out,
                   double *values_out) {
    return Evaluate<double>(ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz, cpp, cdim, cpix, cxyz, ref_bins,
                            flo_bins, sim_weight, be_weight, pad, def_out, warped_out, node_out, values_out);
}

int ref32_evaluate(const float *ref, const int *rdim, const float *rpix, const float *rxyz, const float *flo,
                   const int *fdim, const float *fpix, const float *fxyz, const float *cpp, const int *cdim,
                   const float *cpix, const float *cxyz, int ref_bins, int flo_bins, double sim_weight,
                   double be_weight, float pad, double *def_out, double *warped_out, double *node_out,
                   double *values_out) {
    return Evaluate<float>(ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz, cpp, cdim, cpix, cxyz, ref_bins,
                           flo_bins, sim_weight, be_weight, pad, def_out, warped_out, node_out, values_out);
}

}  // extern "C"
