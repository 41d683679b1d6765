// nrb_platform_f3d_register: reg_f3d<float>::Run on the CPU or the B200 platform of this build.
#include <chrono>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "B200Platform.h"
#include "_reg_f3d.h"
#include "niftyreg_b200_platform.h"

namespace {

thread_local std::string g_error;

// float image of the given geometry, sform and qform both from xyz
NiftiImage MakeImage(const int32_t *dim, const float *pixdim, const float *xyz, const float *data) {
    std::vector<NiftiImage::dim_t> dims{ dim[0], dim[1], dim[2] };
    NiftiImage img(dims, NIFTI_TYPE_FLOAT32);
    img.setPixDim(NiftiDim::X, pixdim[0]);
    img.setPixDim(NiftiDim::Y, pixdim[1]);
    img.setPixDim(NiftiDim::Z, pixdim[2]);
    mat44 m;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) m.m[r][c] = xyz[4 * r + c];
    img->sform_code = 1;
    img->sto_xyz = m;
    img->sto_ijk = nifti_mat44_inverse(m);
    img->qform_code = 1;
    nifti_mat44_to_quatern(m, &img->quatern_b, &img->quatern_c, &img->quatern_d, &img->qoffset_x, &img->qoffset_y,
                           &img->qoffset_z, nullptr, nullptr, nullptr, &img->qfac);
    img->qto_xyz = nifti_quatern_to_mat44(img->quatern_b, img->quatern_c, img->quatern_d, img->qoffset_x,
                                          img->qoffset_y, img->qoffset_z, pixdim[0], pixdim[1], pixdim[2], img->qfac);
    img->qto_ijk = nifti_mat44_inverse(img->qto_xyz);
    std::memcpy(img->data, data, size_t(dim[0]) * dim[1] * dim[2] * sizeof(float));
    return img;
}

// reg_f3d<float> that counts the optimiser's callbacks and marks the start of each level
class CountingF3d: public reg_f3d<float> {
public:
    CountingF3d(): reg_f3d<float>(1, 1) {}
    double GetObjectiveFunctionValue() override {
        ++objective;
        return reg_f3d<float>::GetObjectiveFunctionValue();
    }
    void GetObjectiveFunctionGradient() override {
        ++gradient;
        reg_f3d<float>::GetObjectiveFunctionGradient();
    }
    float InitCurrentLevel(int level) override {
        if (level >= 0) starts.push_back(std::chrono::steady_clock::now());
        return reg_f3d<float>::InitCurrentLevel(level);
    }
    double FinalNmi() const { return this->similarityWeight > 0 ? this->bestWMeasure / this->similarityWeight : 0; }
    int64_t objective = 0, gradient = 0;
    std::vector<std::chrono::steady_clock::time_point> starts;
};

}  // namespace

extern "C" const char *nrb_platform_last_error(void) {
    return g_error.c_str();
}

extern "C" int nrb_platform_f3d_register(const float *ref, const float *flo, const int32_t dim[3],
                                         const float pixdim[3], const float xyz[16], const nrb_platform_params *p,
                                         float *cpp_out, int64_t cpp_capacity, nrb_platform_result *result) {
    g_error.clear();
    try {
        if (!ref || !flo || !dim || !pixdim || !xyz || !p || !result)
            throw std::invalid_argument("nrb_platform_f3d_register: null argument");
        if (p->platform != NRB_PLATFORM_CPU && p->platform != NRB_PLATFORM_B200)
            throw std::invalid_argument("nrb_platform_f3d_register: unknown platform");
        if (p->levels < 1 || p->levels > NRB_PLATFORM_MAX_LEVELS)
            throw std::invalid_argument("nrb_platform_f3d_register: levels must be in [1, 8]");
        NiftiImage r = MakeImage(dim, pixdim, xyz, ref), f = MakeImage(dim, pixdim, xyz, flo);
        CountingF3d reg;
        // the platform first: the NMI measure below is created by the platform's measure creator
        reg.SetPlatformType(p->platform == NRB_PLATFORM_B200 ? PlatformB200 : PlatformType::Cpu);
        if (p->platform == NRB_PLATFORM_B200 && p->gpu >= 0) reg.SetGpuIdx(unsigned(p->gpu));
        reg.SetReferenceImage(r);
        reg.SetFloatingImage(f);
        reg.SetLevelNumber(unsigned(p->levels));
        reg.SetLevelToPerform(unsigned(p->levels));
        reg.SetMaximalIterationNumber(unsigned(p->max_iterations));
        reg.SetBendingEnergyWeight(p->bending_energy);
        reg.SetLinearEnergyWeight(p->linear_energy);
        reg.UseNMISetReferenceBinNumber(0, p->bins);
        reg.UseNMISetFloatingBinNumber(0, p->bins);
        reg.SetSpacing(0, p->spacing);
        reg.SetWarpedPaddingValue(p->padding);
        if (!p->verbose) reg.DoNotPrintOutInformation();
        const auto t0 = std::chrono::steady_clock::now();
        reg.Run();
        const auto t1 = std::chrono::steady_clock::now();
        NiftiImage grid = reg.GetControlPointPositionImage();
        result->cpp_dim[0] = grid->nx;
        result->cpp_dim[1] = grid->ny;
        result->cpp_dim[2] = grid->nz;
        if (cpp_out) {
            if (cpp_capacity < int64_t(grid->nvox))
                throw std::invalid_argument("nrb_platform_f3d_register: cpp_out too small");
            std::memcpy(cpp_out, grid->data, grid->nvox * sizeof(float));
        }
        result->final_nmi = reg.FinalNmi();
        result->objective_evaluations = reg.objective;
        result->gradient_evaluations = reg.gradient;
        result->seconds = std::chrono::duration<double>(t1 - t0).count();
        for (int l = 0; l < NRB_PLATFORM_MAX_LEVELS; ++l) result->level_seconds[l] = 0;
        reg.starts.push_back(t1);
        for (size_t l = 0; l + 1 < reg.starts.size() && l < NRB_PLATFORM_MAX_LEVELS; ++l)
            result->level_seconds[l] = std::chrono::duration<double>(reg.starts[l + 1] - reg.starts[l]).count();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}
