// The B200 platform's classes: each method is one call of the C ABI (niftyreg_b200.h) on the
// content's stream. Reference interfaces are cited in B200Platform.h.
#include "B200Platform.h"

#include <cstring>

namespace nrb_platform {

void Check(nrb_status s, const char *what) {
    if (s != NRB_OK)
        NR_FATAL_ERROR(std::string("B200 platform: ") + what + ": " + nrb_last_error());
}

void CheckCuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        NR_FATAL_ERROR(std::string("B200 platform: ") + what + ": " + cudaGetErrorString(e));
}

void DeviceArray::Allocate(size_t n) {
    Free();
    if (n == 0) return;
    CheckCuda(cudaMalloc(&ptr, n), "cudaMalloc");
    bytes = n;
}

void DeviceArray::Free() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

[[noreturn]] static void NotOnB200(const std::string& what) {
    NR_FATAL_ERROR(what + " is not available on the B200 platform");
    throw std::logic_error(what);  // FatalError throws; this keeps the compiler's noreturn promise
}

// dims, spacing and both orientation matrices of an image, as Content picks them
// (sform when sform_code > 0, else qform: reg-lib/Content.h GetXYZMatrix/GetIJKMatrix)
static void FillGeometry(const NiftiImage& img, int32_t dim[3], float pix[3], float xyz[16], float ijk[16]) {
    nifti_image *n = const_cast<nifti_image*>(static_cast<const nifti_image*>(img));
    dim[0] = n->nx;
    dim[1] = n->ny;
    dim[2] = n->nz;
    pix[0] = n->dx;
    pix[1] = n->dy;
    pix[2] = n->dz;
    const mat44 *m = Content::GetXYZMatrix(*n), *mi = Content::GetIJKMatrix(*n);
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            xyz[4 * r + c] = m->m[r][c];
            ijk[4 * r + c] = mi->m[r][c];
        }
}

}  // namespace nrb_platform

using namespace nrb_platform;

/* ---------------------------------------------------------------------------------------------
 * B200F3dContent
 * ------------------------------------------------------------------------------------------- */
B200F3dContent::B200F3dContent(NiftiImage& referenceIn, NiftiImage& floatingIn, NiftiImage& controlPointGridIn,
                               NiftiImage *localWeightSimIn, int *referenceMaskIn, mat44 *transformationMatrixIn,
                               size_t bytesIn):
    Content(referenceIn, floatingIn, referenceMaskIn, transformationMatrixIn, sizeof(float)),
    DefContent(referenceIn, floatingIn, localWeightSimIn, referenceMaskIn, transformationMatrixIn, sizeof(float)),
    F3dContent(referenceIn, floatingIn, controlPointGridIn, localWeightSimIn, referenceMaskIn, transformationMatrixIn,
               sizeof(float)) {
    if (reference->nt != 1 || floating->nt != 1)
        NotOnB200("A multi-channel image");
    if (reference->nz < 2)
        NotOnB200("A 2D registration");
    if (localWeightSim)
        NotOnB200("A local similarity weight image");
    if (transformationMatrix)
        NotOnB200("An affine-only content");
    if (reference->datatype != NIFTI_TYPE_FLOAT32)
        reference.changeDatatype(NIFTI_TYPE_FLOAT32);
    if (floating->datatype != NIFTI_TYPE_FLOAT32)
        floating.changeDatatype(NIFTI_TYPE_FLOAT32);
    if (controlPointGrid->datatype != NIFTI_TYPE_FLOAT32)
        NotOnB200("A double-precision control-point grid");

    FillGeometry(reference, geom.ref_dim, geom.ref_pixdim, geom.ref_xyz, geom.ref_ijk);
    FillGeometry(floating, geom.flo_dim, geom.flo_pixdim, geom.flo_xyz, geom.flo_ijk);
    FillGeometry(controlPointGrid, geom.cpp_dim, geom.cpp_pixdim, geom.cpp_xyz, geom.cpp_ijk);
    nodeNumber = controlPointGrid.nVoxelsPerVolume();

    CheckCuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    Check(nrb_workspace_create(&geom, &ws), "nrb_workspace_create");

    const size_t nvox = reference.nVoxelsPerVolume();
    refDev.Allocate(nvox * sizeof(float));
    floDev.Allocate(floating.nVoxelsPerVolume() * sizeof(float));
    maskDev.Allocate(nvox * sizeof(int32_t));
    defDev.Allocate(3 * nvox * sizeof(float));
    warpedDev.Allocate(nvox * sizeof(float));
    warpedGradDev.Allocate(3 * nvox * sizeof(float));
    voxelGradDev.Allocate(3 * nvox * sizeof(float));
    cppDev.Allocate(3 * nodeNumber * sizeof(float));
    snapDev.Allocate(3 * nodeNumber * sizeof(float));
    transGradDev.Allocate(3 * nodeNumber * sizeof(float));
    for (DeviceArray *a : { &defDev, &warpedDev, &warpedGradDev, &voxelGradDev, &transGradDev })
        CheckCuda(cudaMemsetAsync(a->ptr, 0, a->bytes, stream), "cudaMemsetAsync");
    UploadImages();
    CheckCuda(cudaMemcpyAsync(maskDev.ptr, referenceMask, nvox * sizeof(int32_t), cudaMemcpyHostToDevice, stream),
              "mask upload");
    Upload(cppDev, controlPointGrid);
    CheckCuda(cudaStreamSynchronize(stream), "content upload");
}

B200F3dContent::~B200F3dContent() {
    // the grid goes back to the NiftiImage shared with reg_f3d (as CudaF3dContent's destructor)
    if (cppDev.ptr && controlPointGrid) {
        cudaMemcpyAsync(controlPointGrid->data, cppDev.ptr, cppDev.bytes, cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
    }
    for (DeviceArray *a : { &refDev, &floDev, &maskDev, &defDev, &warpedDev, &warpedGradDev, &voxelGradDev, &cppDev,
                            &snapDev, &transGradDev })
        a->Free();
    nrb_workspace_destroy(ws);
    if (stream) cudaStreamDestroy(stream);
}

void B200F3dContent::Download(NiftiImage& img, const DeviceArray& dev) {
    const size_t n = std::min(dev.bytes, size_t(img.totalBytes()));
    CheckCuda(cudaMemcpyAsync(img->data, dev.ptr, n, cudaMemcpyDeviceToHost, stream), "download");
    CheckCuda(cudaStreamSynchronize(stream), "download");
}

void B200F3dContent::Upload(DeviceArray& dev, const NiftiImage& img) {
    const size_t n = std::min(dev.bytes, size_t(img.totalBytes()));
    CheckCuda(cudaMemcpyAsync(dev.ptr, img->data, n, cudaMemcpyHostToDevice, stream), "upload");
}

void B200F3dContent::UploadImages() {
    Upload(refDev, reference);
    Upload(floDev, floating);
    CheckCuda(cudaStreamSynchronize(stream), "image upload");
}

void B200F3dContent::MarkDeformationPending() {
    // a new request supersedes an open one (reg_f3d reads the warp of a request before it asks
    // for the next field)
    pendingDef = true;
    pendingWarp = false;
    fromSnapshot = false;
}

bool B200F3dContent::MarkWarpPending(float padding) {
    if (!pendingDef) return false;
    pendingWarp = true;
    pendingPad = padding;
    return true;
}

void B200F3dContent::BeforeControlPointsChange() {
    if (!pendingDef || fromSnapshot) return;
    CheckCuda(cudaMemcpyAsync(snapDev.ptr, cppDev.ptr, cppDev.bytes, cudaMemcpyDeviceToDevice, stream),
              "control-point snapshot");
    fromSnapshot = true;
}

void B200F3dContent::MaterialiseDeformation() {
    if (!pendingDef) return;
    Check(nrb_get_deformation_field(&geom, PendingControlPoints(), maskDev.i(), defDev.f(), stream),
          "nrb_get_deformation_field");
    pendingDef = false;
    fromSnapshot = false;
}

void B200F3dContent::MaterialiseWarp() {
    // a recorded warp is of the recorded field, which may already have been computed
    MaterialiseDeformation();
    if (!pendingWarp) return;
    Check(nrb_resample_image(&geom, floDev.f(), defDev.f(), maskDev.i(), pendingPad, warpedDev.f(), stream),
          "nrb_resample_image");
    pendingWarp = false;
}

NiftiImage& B200F3dContent::GetDeformationField() {
    MaterialiseDeformation();
    Download(deformationField, defDev);
    return deformationField;
}
NiftiImage& B200F3dContent::GetWarped() {
    MaterialiseWarp();
    Download(warped, warpedDev);
    return warped;
}
NiftiImage& B200F3dContent::GetWarpedGradient() { Download(warpedGradient, warpedGradDev); return warpedGradient; }
NiftiImage& B200F3dContent::GetVoxelBasedMeasureGradient() {
    Download(voxelBasedMeasureGradient, voxelGradDev);
    return voxelBasedMeasureGradient;
}
NiftiImage& B200F3dContent::GetControlPointGrid() { Download(controlPointGrid, cppDev); return controlPointGrid; }
NiftiImage& B200F3dContent::GetTransformationGradient() {
    Download(transformationGradient, transGradDev);
    return transformationGradient;
}
void B200F3dContent::UpdateDeformationField() {
    MaterialiseWarp();  // a recorded warp is of the recorded field
    Upload(defDev, deformationField);
}
void B200F3dContent::UpdateWarped() {
    MaterialiseDeformation();
    pendingWarp = false;
    Upload(warpedDev, warped);
}
void B200F3dContent::UpdateWarpedGradient() { Upload(warpedGradDev, warpedGradient); }
void B200F3dContent::UpdateVoxelBasedMeasureGradient() { Upload(voxelGradDev, voxelBasedMeasureGradient); }
void B200F3dContent::UpdateControlPointGrid() {
    BeforeControlPointsChange();
    Upload(cppDev, controlPointGrid);
}
void B200F3dContent::UpdateTransformationGradient() { Upload(transGradDev, transformationGradient); }
void B200F3dContent::ZeroTransformationGradient() {
    CheckCuda(cudaMemsetAsync(transGradDev.ptr, 0, transGradDev.bytes, stream), "cudaMemsetAsync");
}
void B200F3dContent::ZeroVoxelBasedMeasureGradient() {
    CheckCuda(cudaMemsetAsync(voxelGradDev.ptr, 0, voxelGradDev.bytes, stream), "cudaMemsetAsync");
}

/* ---------------------------------------------------------------------------------------------
 * B200Compute
 * ------------------------------------------------------------------------------------------- */
void B200Compute::GetDeformationField(bool composition, bool bspline) {
    if (composition || !bspline)
        NotOnB200("A composed or non-B-spline deformation field");
    Con().MarkDeformationPending();
}

void B200Compute::ResampleImage(int interpolation, float paddingValue) {
    B200F3dContent& c = Con();
    if (interpolation == 1 && c.MarkWarpPending(paddingValue)) return;
    c.MaterialiseDeformation();
    if (interpolation == 1)
        Check(nrb_resample_image(&c.Geometry(), c.FloatingDevice(), c.DeformationFieldDevice(), c.MaskDevice(),
                                 paddingValue, c.WarpedDevice(), c.Stream()),
              "nrb_resample_image");
    else
        Check(nrb_resample_image_order(&c.Geometry(), c.FloatingDevice(), c.DeformationFieldDevice(), c.MaskDevice(),
                                       interpolation, paddingValue, c.WarpedDevice(), c.Stream()),
              "nrb_resample_image_order");
}

void B200Compute::GetImageGradient(int interpolation, float paddingValue, int activeTimePoint) {
    if (interpolation != 1)
        NotOnB200("A non-linear image gradient");
    if (activeTimePoint != 0)
        NotOnB200("A multi-channel image gradient");
    B200F3dContent& c = Con();
    c.MaterialiseDeformation();
    Check(nrb_get_image_gradient(&c.Geometry(), c.FloatingDevice(), c.DeformationFieldDevice(), c.MaskDevice(),
                                 paddingValue, c.WarpedGradientDevice(), c.Stream()),
          "nrb_get_image_gradient");
}

double B200Compute::ApproxBendingEnergy() {
    B200F3dContent& c = Con();
    double be = 0;
    Check(nrb_approx_bending_energy(c.Workspace(), &c.Geometry(), c.GetControlPointGridDevice(), nullptr, &be,
                                    c.Stream()),
          "nrb_approx_bending_energy");
    return be;
}

void B200Compute::ApproxBendingEnergyGradient(float weight) {
    B200F3dContent& c = Con();
    Check(nrb_approx_bending_energy_gradient(c.Workspace(), &c.Geometry(), c.GetControlPointGridDevice(), weight,
                                             c.GetTransformationGradientDevice(), c.Stream()),
          "nrb_approx_bending_energy_gradient");
}

void B200Compute::ConvolveVoxelBasedMeasureGradient(float weight) {
    B200F3dContent& c = Con();
    Check(nrb_convolve_voxel_based_gradient(c.Workspace(), &c.Geometry(), c.VoxelBasedGradientDevice(), weight,
                                            c.GetTransformationGradientDevice(), c.Stream()),
          "nrb_convolve_voxel_based_gradient");
}

double B200Compute::GetMaximalLength(bool optimiseX, bool optimiseY, bool optimiseZ) {
    if (!optimiseX && !optimiseY && !optimiseZ) return 0;
    if (!(optimiseX && optimiseY && optimiseZ))
        NotOnB200("Optimising a subset of the axes");
    B200F3dContent& c = Con();
    double len = 0;
    Check(nrb_get_maximal_length(c.GetTransformationGradientDevice(), int64_t(c.NodeNumber()), nullptr, &len,
                                 c.Stream()),
          "nrb_get_maximal_length");
    return len;
}

void B200Compute::NormaliseGradient(double maxGradLength, bool optimiseX, bool optimiseY, bool optimiseZ) {
    if (maxGradLength == 0 || (!optimiseX && !optimiseY && !optimiseZ)) return;
    if (!(optimiseX && optimiseY && optimiseZ))
        NotOnB200("Optimising a subset of the axes");
    B200F3dContent& c = Con();
    Check(nrb_normalise_gradient(c.GetTransformationGradientDevice(), int64_t(c.NodeNumber()), maxGradLength,
                                 nullptr, c.Stream()),
          "nrb_normalise_gradient");
}

void B200Compute::UpdateControlPointPosition(float *currentDof, const float *bestDof, const float *gradient,
                                             const float scale, const bool optimiseX, const bool optimiseY,
                                             const bool optimiseZ) {
    if (!(optimiseX && optimiseY && optimiseZ))
        NotOnB200("Optimising a subset of the axes");
    B200F3dContent& c = Con();
    c.BeforeControlPointsChange();
    Check(nrb_update_control_point_position(currentDof, bestDof, gradient, scale, 3 * int64_t(c.NodeNumber()),
                                            c.Stream()),
          "nrb_update_control_point_position");
}

double B200Compute::GetJacobianPenaltyTerm(bool) { NotOnB200("The Jacobian penalty"); }
void B200Compute::JacobianPenaltyTermGradient(float, bool) { NotOnB200("The Jacobian penalty gradient"); }
double B200Compute::CorrectFolding(bool) { NotOnB200("Folding correction"); }
double B200Compute::ApproxLinearEnergy() { NotOnB200("The linear energy"); }
void B200Compute::ApproxLinearEnergyGradient(float) { NotOnB200("The linear energy gradient"); }
double B200Compute::GetLandmarkDistance(size_t, float*, float*) { NotOnB200("The landmark distance"); }
void B200Compute::LandmarkDistanceGradient(size_t, float*, float*, float) { NotOnB200("The landmark gradient"); }
void B200Compute::SmoothGradient(float) { NotOnB200("Gradient smoothing"); }
void B200Compute::GetApproximatedGradient(InterfaceOptimiser&) { NotOnB200("The approximated gradient"); }
void B200Compute::GetDefFieldFromVelocityGrid(const bool) { NotOnB200("A velocity field"); }
void B200Compute::ExponentiateGradient(Content&) { NotOnB200("Gradient exponentiation"); }
void B200Compute::UpdateVelocityField(float, bool, bool, bool) { NotOnB200("A velocity field update"); }
void B200Compute::BchUpdate(float, int) { NotOnB200("The BCH update"); }
void B200Compute::SymmetriseVelocityFields(Content&) { NotOnB200("Velocity field symmetrisation"); }
void B200Compute::GetAffineDeformationField(bool) { NotOnB200("An affine deformation field"); }
void B200Compute::DefFieldCompose(const NiftiImage&) { NotOnB200("Deformation field composition"); }
NiftiImage B200Compute::ResampleGradient(int, float) { NotOnB200("Gradient resampling"); }
void B200Compute::VoxelCentricToNodeCentric(float) {
    NotOnB200("The separate voxel-to-node step (ConvolveVoxelBasedMeasureGradient does both)");
}

/* ---------------------------------------------------------------------------------------------
 * reg_nmi_b200 and its creator
 * ------------------------------------------------------------------------------------------- */
reg_nmi_b200::~reg_nmi_b200() {
    nrb_nmi_destroy(nmi);
}

void reg_nmi_b200::Bind(B200F3dContent& con) {
    if (this->referenceTimePoints != 1)
        NotOnB200("A multi-channel NMI");
    nrb_nmi_destroy(nmi);
    nmi = nullptr;
    bound = &con;
    Check(nrb_nmi_create(this->referenceBinNumber[0], this->floatingBinNumber[0], &nmi), "nrb_nmi_create");
}

double reg_nmi_b200::GetSimilarityMeasureValueFw() {
    if (this->timePointWeights[0] <= 0) return 0;
    B200F3dContent& c = *bound;
    if (c.WarpPending() && c.FusedObjectiveOk()) {
        // field, warp and histogram in one pass; the same histogram, so the same NMI and tables
        // as the three steps would give
        nrb_objective o;
        const nrb_status s = nrb_f3d_objective(c.Workspace(), nmi, &c.Geometry(), c.ReferenceDevice(),
                                               c.FloatingDevice(), c.MaskDevice(), c.PendingControlPoints(),
                                               c.PendingPadding(), 1.0, 0.0, nullptr, &o, c.Stream());
        if (s == NRB_OK) return this->timePointWeights[0] * o.nmi;
        if (s != NRB_ERR_UNSUPPORTED) Check(s, "nrb_f3d_objective");
        c.DisableFusedObjective();  // a grid not aligned with the reference: the three steps
    }
    c.MaterialiseWarp();
    double value = 0;
    Check(nrb_nmi_value(nmi, &c.Geometry(), c.ReferenceDevice(), c.WarpedDevice(), c.MaskDevice(), nullptr, &value,
                        c.Stream()),
          "nrb_nmi_value");
    return this->timePointWeights[0] * value;
}

void reg_nmi_b200::GetVoxelBasedSimilarityMeasureGradientFw(int currentTimePoint) {
    if (currentTimePoint != 0)
        NotOnB200("A multi-channel NMI gradient");
    if (this->timePointWeights[0] <= 0) return;
    B200F3dContent& c = *bound;
    c.MaterialiseWarp();
    // the histogram at the current warp first, as reg_nmi::GetVoxelBasedSimilarityMeasureGradientFw
    Check(nrb_nmi_value(nmi, &c.Geometry(), c.ReferenceDevice(), c.WarpedDevice(), c.MaskDevice(), nullptr, nullptr,
                        c.Stream()),
          "nrb_nmi_value");
    Check(nrb_nmi_voxel_gradient(nmi, &c.Geometry(), c.ReferenceDevice(), c.WarpedDevice(), c.WarpedGradientDevice(),
                                 c.MaskDevice(), this->timePointWeights[0], c.VoxelBasedGradientDevice(), c.Stream()),
          "nrb_nmi_voxel_gradient");
}

double reg_nmi_b200::GetSimilarityMeasureValueBw() { NotOnB200("A symmetric NMI"); }
void reg_nmi_b200::GetVoxelBasedSimilarityMeasureGradientBw(int) { NotOnB200("A symmetric NMI gradient"); }

reg_measure* B200MeasureCreator::Create(const MeasureType measureType) {
    if (measureType == MeasureType::Nmi)
        return new reg_nmi_b200();
    NotOnB200("This similarity measure");
}

void B200MeasureCreator::Initialise(reg_measure& measure, DefContent& con, DefContent *conBw) {
    if (conBw)
        NotOnB200("A symmetric measure");
    auto *nmi = dynamic_cast<reg_nmi_b200*>(&measure);
    auto *c = dynamic_cast<B200F3dContent*>(&con);
    if (!nmi || !c)
        NotOnB200("A measure or content of another platform");
    // bins and the intensity rescale to [2, bins - 3] on the host images (the reference's own
    // reg_nmi::InitialiseMeasure), then the rescaled images go to the device
    nmi->InitialiseMeasure(c->Content::GetReference(), c->Content::GetFloating(), c->Content::GetReferenceMask(),
                           c->Content::GetWarped(), c->DefContent::GetWarpedGradient(),
                           c->DefContent::GetVoxelBasedMeasureGradient(), c->DefContent::GetLocalWeightSim());
    c->UploadImages();
    nmi->Bind(*c);
}

ContentCreator* B200ContentCreatorFactory::Produce(const ContentType conType) {
    if (conType == ContentType::F3d)
        return new B200F3dContentCreator();
    NotOnB200("This content type");
}

/* ---------------------------------------------------------------------------------------------
 * optimisers
 * ------------------------------------------------------------------------------------------- */
B200Optimiser::~B200Optimiser() {
    this->bestDof = nullptr;  // device memory (best): not the base class's to free
}

// the state Optimiser<T>::Initialise sets (reg-lib/Optimiser.cpp:48-89), the best DOFs in device
// memory; ends with the first objective evaluation
void B200Optimiser::Initialise(size_t nvox, int ndim, bool optX, bool optY, bool optZ, size_t maxIt, size_t startIt,
                               InterfaceOptimiser *intOpt, float *cppData, float *gradData, size_t nvoxBw,
                               float *cppDataBw, float *gradDataBw) {
    if (!(optX && optY && optZ))
        NotOnB200("Optimising a subset of the axes");
    if (nvoxBw > 0 && cppDataBw && gradDataBw)
        NotOnB200("A symmetric optimisation");
    this->dofNumber = nvox;
    this->ndim = ndim;
    this->optimiseX = optX;
    this->optimiseY = optY;
    this->optimiseZ = optZ;
    this->maxIterationNumber = maxIt;
    this->currentIterationNumber = startIt;
    this->currentDof = cppData;
    this->gradient = gradData;
    this->isSymmetric = false;
    best.Allocate(nvox * sizeof(float));
    this->bestDof = best.f();
    this->StoreCurrentDof();
    this->intOpt = intOpt;
    this->bestObjFunctionValue = this->currentObjFunctionValue = this->intOpt->GetObjectiveFunctionValue();
}

void B200Optimiser::StoreCurrentDof() {
    CheckCuda(cudaMemcpyAsync(this->bestDof, this->currentDof, this->dofNumber * sizeof(float),
                              cudaMemcpyDeviceToDevice, con.Stream()),
              "StoreCurrentDof");
}

void B200Optimiser::RestoreBestDof() {
    con.BeforeControlPointsChange();
    CheckCuda(cudaMemcpyAsync(this->currentDof, this->bestDof, this->dofNumber * sizeof(float),
                              cudaMemcpyDeviceToDevice, con.Stream()),
              "RestoreBestDof");
}

void B200Optimiser::Perturbation(float) { NotOnB200("Perturbation"); }

void B200ConjugateGradient::Initialise(size_t nvox, int ndim, bool optX, bool optY, bool optZ, size_t maxIt,
                                       size_t startIt, InterfaceOptimiser *intOpt, float *cppData, float *gradData,
                                       size_t nvoxBw, float *cppDataBw, float *gradDataBw) {
    B200Optimiser::Initialise(nvox, ndim, optX, optY, optZ, maxIt, startIt, intOpt, cppData, gradData, nvoxBw,
                              cppDataBw, gradDataBw);
    firstCall = true;
    dir1.Allocate(nvox * sizeof(float));
    dir2.Allocate(nvox * sizeof(float));
}

// ConjugateGradient<T>::Optimise (reg-lib/Optimiser.cpp:318-322): direction update, then the
// base line search
void B200ConjugateGradient::Optimise(float maxLength, float smallLength, float& startLength) {
    this->UpdateGradientValues();
    Optimiser<float>::Optimise(maxLength, smallLength, startLength);
}

void B200ConjugateGradient::UpdateGradientValues() {
    Check(nrb_conjugate_gradient(con.Workspace(), this->gradient, dir1.f(), dir2.f(), int64_t(this->dofNumber),
                                 firstCall ? 1 : 0, con.Stream()),
          "nrb_conjugate_gradient");
    firstCall = false;
}
