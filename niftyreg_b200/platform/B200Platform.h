// The B200 platform for NiftyReg's reg_f3d: subclasses of the reference's Content, Compute,
// reg_nmi, MeasureCreator and Optimiser interfaces whose every method forwards to one call of
// the C ABI in niftyreg_b200.h, and the factories that the Platform class hands out for it.
//
// Seam (reference paths relative to the NiftyReg source tree):
//   reg-lib/Platform.h:10-19        PlatformType; the B200 platform takes the next value (3)
//   reg-lib/Platform.cpp:20-162     Platform: factories per type, CreateOptimiser
//   reg-lib/ComputeFactory.h        -> B200ComputeFactory
//   reg-lib/ContentCreatorFactory.h -> B200ContentCreatorFactory (F3D content)
//   reg-lib/MeasureCreatorFactory.hpp, MeasureCreator.hpp -> B200MeasureCreator (NMI)
//   reg-lib/Optimiser.hpp:28-143    -> B200Optimiser, B200ConjugateGradient (device DOFs)
// reg_f3d<float>, its optimiser loop (reg-lib/_reg_base.cpp:727-818) and the pyramid driver run
// unchanged; the images, deformation field, warped image, gradients and control-point grid live
// on the device for the whole level, as on the reference's CUDA platform
// (reg-lib/cuda/CudaF3dContent.cpp, CudaCompute.cu, _reg_nmi_gpu.cu, CudaOptimiser.cu).
//
// Scope: single-channel F3D with NMI, bending energy, linear interpolation, all axes optimised.
// Anything else (Jacobian or linear-energy penalties, landmarks, other measures, velocity
// fields, gradient smoothing, perturbation) raises the reference's fatal error rather than
// running on the host.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "ComputeFactory.h"
#include "ContentCreatorFactory.h"
#include "F3dContent.h"
#include "MeasureCreatorFactory.hpp"
#include "Optimiser.hpp"
#include "Platform.h"
#include "_reg_nmi.h"
#include "niftyreg_b200.h"

// The platform's PlatformType value: the enum's next entry after OpenCl (reg-lib/Platform.h:10).
inline constexpr PlatformType PlatformB200 = static_cast<PlatformType>(3);

namespace nrb_platform {

// A non-zero status of the C ABI becomes the reference's fatal error (a std::runtime_error).
void Check(nrb_status s, const char *what);
// A CUDA runtime error likewise.
void CheckCuda(cudaError_t e, const char *what);

// A device allocation owned by one object (freed with it).
struct DeviceArray {
    void *ptr = nullptr;
    size_t bytes = 0;
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    ~DeviceArray() { Free(); }
    void Allocate(size_t n);
    void Free();
    float *f() const { return static_cast<float*>(ptr); }
    int32_t *i() const { return static_cast<int32_t*>(ptr); }
};

}  // namespace nrb_platform

// F3D content on the device (mirrors CudaF3dContent, reg-lib/cuda/CudaF3dContent.h). Layout is
// the NIfTI buffers' own (planar vector images), so host<->device transfers are flat copies.
// Getters of device-resident images download first; Update*() uploads.
class B200F3dContent: public F3dContent {
public:
    B200F3dContent(NiftiImage& referenceIn, NiftiImage& floatingIn, NiftiImage& controlPointGridIn,
                   NiftiImage *localWeightSimIn = nullptr, int *referenceMaskIn = nullptr,
                   mat44 *transformationMatrixIn = nullptr, size_t bytesIn = sizeof(float));
    ~B200F3dContent() override;

    // Content / DefContent / F3dContent getters: download the device copy
    NiftiImage& GetDeformationField() override;
    NiftiImage& GetWarped() override;
    NiftiImage& GetWarpedGradient() override;
    NiftiImage& GetVoxelBasedMeasureGradient() override;
    NiftiImage& GetControlPointGrid() override;
    NiftiImage& GetTransformationGradient() override;
    // host -> device
    void UpdateDeformationField() override;
    void UpdateWarped() override;
    void UpdateWarpedGradient() override;
    void UpdateVoxelBasedMeasureGradient() override;
    void UpdateControlPointGrid() override;
    void UpdateTransformationGradient() override;
    void ZeroTransformationGradient() override;
    void ZeroVoxelBasedMeasureGradient() override;
    bool IsCurrentComputationDoubleCapable() override { return false; }

    // the reference and floating intensities after the measure rescaled the host copies
    void UploadImages();

    // Lazy deformation field and warped image. B200Compute::GetDeformationField and a linear
    // ResampleImage record the request; the NMI value of a recorded warp is then one fused pass
    // over the voxels (nrb_f3d_objective) that writes neither array, and the first reader of
    // either array computes it from the control points of the request. Control points that
    // change while a request is open are first saved, so a later reader still sees the field of
    // the request's control points.
    void MarkDeformationPending();
    bool MarkWarpPending(float padding);  // false when no field is pending (warp now instead)
    bool WarpPending() const { return pendingDef && pendingWarp; }
    const float* PendingControlPoints() const { return fromSnapshot ? snapDev.f() : cppDev.f(); }
    float PendingPadding() const { return pendingPad; }
    void BeforeControlPointsChange();
    void MaterialiseDeformation();
    void MaterialiseWarp();
    bool FusedObjectiveOk() const { return fusedOk; }
    void DisableFusedObjective() { fusedOk = false; }

    const nrb_geometry& Geometry() const { return geom; }
    nrb_workspace* Workspace() const { return ws; }
    cudaStream_t Stream() const { return stream; }
    float* ReferenceDevice() const { return refDev.f(); }
    float* FloatingDevice() const { return floDev.f(); }
    const int32_t* MaskDevice() const { return maskDev.i(); }
    float* DeformationFieldDevice() const { return defDev.f(); }
    float* WarpedDevice() const { return warpedDev.f(); }
    float* WarpedGradientDevice() const { return warpedGradDev.f(); }
    float* VoxelBasedGradientDevice() const { return voxelGradDev.f(); }
    float* GetControlPointGridDevice() const { return cppDev.f(); }
    float* GetTransformationGradientDevice() const { return transGradDev.f(); }
    size_t NodeNumber() const { return nodeNumber; }

private:
    void Download(NiftiImage& img, const nrb_platform::DeviceArray& dev);
    void Upload(nrb_platform::DeviceArray& dev, const NiftiImage& img);

    nrb_geometry geom{};
    nrb_workspace *ws = nullptr;
    cudaStream_t stream = nullptr;
    size_t nodeNumber = 0;
    nrb_platform::DeviceArray refDev, floDev, maskDev, defDev, warpedDev, warpedGradDev, voxelGradDev,
        cppDev, transGradDev;
    nrb_platform::DeviceArray snapDev;  // the control points of an open request, once they change
    bool pendingDef = false, pendingWarp = false, fromSnapshot = false;
    float pendingPad = 0.f;
    bool fusedOk = true;  // the fused objective applies (a grid aligned with the reference)
};

// Compute on the device (reg-lib/Compute.h:6-49; CUDA counterpart reg-lib/cuda/CudaCompute.h).
class B200Compute: public Compute {
public:
    explicit B200Compute(Content& conIn): Compute(conIn) {}

    void ResampleImage(int interpolation, float paddingValue) override;
    double GetJacobianPenaltyTerm(bool approx) override;
    void JacobianPenaltyTermGradient(float weight, bool approx) override;
    double CorrectFolding(bool approx) override;
    double ApproxBendingEnergy() override;
    void ApproxBendingEnergyGradient(float weight) override;
    double ApproxLinearEnergy() override;
    void ApproxLinearEnergyGradient(float weight) override;
    double GetLandmarkDistance(size_t landmarkNumber, float *landmarkReference, float *landmarkFloating) override;
    void LandmarkDistanceGradient(size_t landmarkNumber, float *landmarkReference, float *landmarkFloating,
                                  float weight) override;
    void GetDeformationField(bool composition, bool bspline) override;
    void UpdateControlPointPosition(float *currentDof, const float *bestDof, const float *gradient, const float scale,
                                    const bool optimiseX, const bool optimiseY, const bool optimiseZ) override;
    void GetImageGradient(int interpolation, float paddingValue, int activeTimePoint) override;
    double GetMaximalLength(bool optimiseX, bool optimiseY, bool optimiseZ) override;
    void NormaliseGradient(double maxGradLength, bool optimiseX, bool optimiseY, bool optimiseZ) override;
    void SmoothGradient(float sigma) override;
    void GetApproximatedGradient(InterfaceOptimiser& opt) override;
    void GetDefFieldFromVelocityGrid(const bool updateStepNumber) override;
    void ConvolveVoxelBasedMeasureGradient(float weight) override;
    void ExponentiateGradient(Content& conBw) override;
    void UpdateVelocityField(float scale, bool optimiseX, bool optimiseY, bool optimiseZ) override;
    void BchUpdate(float scale, int bchUpdateValue) override;
    void SymmetriseVelocityFields(Content& conBw) override;
    void GetAffineDeformationField(bool compose) override;

protected:
    void DefFieldCompose(const NiftiImage& defField) override;
    NiftiImage ResampleGradient(int interpolation, float padding) override;
    void VoxelCentricToNodeCentric(float weight) override;

private:
    B200F3dContent& Con() { return dynamic_cast<B200F3dContent&>(con); }
};

// NMI on the device (reg-lib/cpu/_reg_nmi.h:19-84; CUDA counterpart reg-lib/cuda/_reg_nmi_gpu.h).
// InitialiseMeasure is the base class's (bin numbers, host intensity rescale); Bind then attaches
// the content's device buffers and a device histogram workspace.
class reg_nmi_b200: public reg_nmi {
public:
    ~reg_nmi_b200() override;
    void Bind(B200F3dContent& con);
    double GetSimilarityMeasureValueFw() override;
    double GetSimilarityMeasureValueBw() override;
    void GetVoxelBasedSimilarityMeasureGradientFw(int currentTimePoint) override;
    void GetVoxelBasedSimilarityMeasureGradientBw(int currentTimePoint) override;

private:
    B200F3dContent *bound = nullptr;
    nrb_nmi *nmi = nullptr;
};

class B200MeasureCreator: public MeasureCreator {
public:
    reg_measure* Create(const MeasureType measureType) override;
    void Initialise(reg_measure& measure, DefContent& con, DefContent *conBw = nullptr) override;
};

// Gradient ascent with the DOFs on the device (reg-lib/Optimiser.hpp:28-104; CUDA counterpart
// reg-lib/cuda/CudaOptimiser.hpp:13-58). The base class's line search (Optimise) runs as is.
class B200Optimiser: public Optimiser<float> {
public:
    explicit B200Optimiser(B200F3dContent& conIn): con(conIn) {}
    ~B200Optimiser() override;
    void Initialise(size_t nvox, int ndim, bool optX, bool optY, bool optZ, size_t maxIt, size_t startIt,
                    InterfaceOptimiser *intOpt, float *cppData, float *gradData, size_t nvoxBw, float *cppDataBw,
                    float *gradDataBw) override;
    void StoreCurrentDof() override;
    void RestoreBestDof() override;
    void Perturbation(float length) override;

protected:
    B200F3dContent& con;
    nrb_platform::DeviceArray best;
};

// Conjugate gradient with the DOFs and both direction arrays on the device
// (reg-lib/Optimiser.hpp:105-143, Optimiser.cpp:186-340; CUDA counterpart
// reg-lib/cuda/CudaOptimiser.hpp:59-96, which derives from the CUDA gradient ascent the same way).
class B200ConjugateGradient: public B200Optimiser {
public:
    using B200Optimiser::B200Optimiser;
    void Initialise(size_t nvox, int ndim, bool optX, bool optY, bool optZ, size_t maxIt, size_t startIt,
                    InterfaceOptimiser *intOpt, float *cppData, float *gradData, size_t nvoxBw, float *cppDataBw,
                    float *gradDataBw) override;
    void Optimise(float maxLength, float smallLength, float& startLength) override;
    void RestartOptimisation() override { firstCall = true; }

protected:
    void UpdateGradientValues() override;

private:
    nrb_platform::DeviceArray dir1, dir2;
    bool firstCall = true;
};

class B200ComputeFactory: public ComputeFactory {
public:
    Compute* Produce(Content& con) override { return new B200Compute(con); }
};

class B200F3dContentCreator: public F3dContentCreator {
public:
    F3dContent* Create(NiftiImage& reference, NiftiImage& floating, NiftiImage& controlPointGrid,
                       NiftiImage *localWeightSim = nullptr, int *referenceMask = nullptr,
                       mat44 *transformationMatrix = nullptr, size_t bytes = sizeof(float)) override {
        return new B200F3dContent(reference, floating, controlPointGrid, localWeightSim, referenceMask,
                                  transformationMatrix, bytes);
    }
};

class B200ContentCreatorFactory: public ContentCreatorFactory {
public:
    ContentCreator* Produce(const ContentType conType) override;
};

class B200MeasureCreatorFactory: public MeasureCreatorFactory {
public:
    MeasureCreator* Produce() override { return new B200MeasureCreator(); }
};
