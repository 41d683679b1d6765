// Test infrastructure only: the reference's own CUDA platform as a comparison arm. Compiled with
// the reference's CPU library, its reg-lib/cuda sources (sm_100a) and Platform.cpp rebuilt with
// USE_CUDA into oracle/_refcuda/libnrref_cuda.so by oracle/Makefile (target refcuda). Nothing in
// the product links or loads this file.
#include <chrono>
#include <cstring>
#include <vector>
#include "_reg_f3d.h"

namespace {

mat44 ToMatC(const float *m) {
    mat44 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r.m[i][j] = m[4 * i + j];
    return r;
}

// float image with an sform built from xyz (and a consistent qform)
NiftiImage MakeImageC(const int *dim, const float *pix, const float *xyz) {
    std::vector<NiftiImage::dim_t> dims{ dim[0], dim[1], dim[2] };
    NiftiImage img(dims, NIFTI_TYPE_FLOAT32);
    img.setPixDim(NiftiDim::X, pix[0]);
    img.setPixDim(NiftiDim::Y, pix[1]);
    img.setPixDim(NiftiDim::Z, pix[2]);
    img->sform_code = 1;
    img->sto_xyz = ToMatC(xyz);
    img->sto_ijk = nifti_mat44_inverse(img->sto_xyz);
    img->qform_code = 1;
    nifti_mat44_to_quatern(img->sto_xyz, &img->quatern_b, &img->quatern_c, &img->quatern_d, &img->qoffset_x,
                           &img->qoffset_y, &img->qoffset_z, nullptr, nullptr, nullptr, &img->qfac);
    img->qto_xyz = nifti_quatern_to_mat44(img->quatern_b, img->quatern_c, img->quatern_d, img->qoffset_x,
                                          img->qoffset_y, img->qoffset_z, pix[0], pix[1], pix[2], img->qfac);
    img->qto_ijk = nifti_mat44_inverse(img->qto_xyz);
    return img;
}

// reg_f3d<float> with evaluation counters (the counted callbacks of its optimiser loop) and a
// mark at the start of every pyramid level
class CudaShimF3d: public reg_f3d<float> {
public:
    CudaShimF3d(): reg_f3d<float>(1, 1) {}
    double GetObjectiveFunctionValue() override { ++objCalls; return reg_f3d<float>::GetObjectiveFunctionValue(); }
    void GetObjectiveFunctionGradient() override { ++gradCalls; reg_f3d<float>::GetObjectiveFunctionGradient(); }
    float InitCurrentLevel(int level) override {
        if (level >= 0) marks.push_back({ std::chrono::steady_clock::now(), objCalls, gradCalls });
        return reg_f3d<float>::InitCurrentLevel(level);
    }
    double FinalWMeasure() const { return this->bestWMeasure; }
    double SimilarityWeight() const { return this->similarityWeight; }
    struct Mark {
        std::chrono::steady_clock::time_point t;
        long obj, grad;
    };
    std::vector<Mark> marks;
    long objCalls = 0, gradCalls = 0;
};

}  // namespace

extern "C" {

// reg_f3d<float>::Run on the reference's CUDA platform (PlatformType::Cuda). params and stats as
// ref_f3d_register: params [0] levels, [1] max iterations, [2] BE, [3] LE, [4] bins, [5] spacing,
// [6] verbose; stats [0] final NMI, [1] 0, [2] objective evaluations, [3] gradient evaluations,
// [4] seconds around Run, then per level (objective evaluations, gradient evaluations, seconds).
// Returns 0.
int refcuda_f3d_register(const float *ref, const float *flo, const int *dim, const float *pix, const float *xyz,
                         const double *params, int *cdim_out, float *cpp_out, size_t cap, double *stats) {
    NiftiImage r = MakeImageC(dim, pix, xyz), f = MakeImageC(dim, pix, xyz);
    const size_t n = size_t(dim[0]) * dim[1] * dim[2];
    memcpy(r->data, ref, n * sizeof(float));
    memcpy(f->data, flo, n * sizeof(float));
    CudaShimF3d reg;
    reg.SetPlatformType(PlatformType::Cuda);
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
    cdim_out[0] = grid->nx;
    cdim_out[1] = grid->ny;
    cdim_out[2] = grid->nz;
    if (cpp_out) {
        if (cap < grid->nvox) return -1;
        memcpy(cpp_out, grid->data, grid->nvox * sizeof(float));
    }
    stats[0] = reg.SimilarityWeight() > 0 ? reg.FinalWMeasure() / reg.SimilarityWeight() : 0;
    stats[1] = 0;
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

}  // extern "C"
