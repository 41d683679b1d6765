// The Platform class of reg-lib/Platform.h, implemented for a build with the B200 platform: the
// CPU platform's factories as the reference's own Platform.cpp makes them, and the B200 ones for
// PlatformB200. A library built with this file in place of reg-lib/Platform.cpp exposes the B200
// platform to reg_f3d through SetPlatformType(PlatformB200), with no other change to the
// reference sources. The member layout and the methods' meaning are reg-lib/Platform.h's; the
// CPU branch of CreateOptimiser hands the optimiser the NIfTI buffers, the B200 branch the
// content's device arrays (reg-lib/Platform.cpp:111-162).
#include <type_traits>

#include "B200Platform.h"
#include "CpuKernelFactory.h"

Platform::Platform(const PlatformType platformTypeIn) {
    platformType = platformTypeIn;
    if (platformType == PlatformType::Cpu) {
        platformName = "CPU";
        computeFactory = new ComputeFactory();
        contentCreatorFactory = new ContentCreatorFactory();
        kernelFactory = new CpuKernelFactory();
        measureCreatorFactory = new MeasureCreatorFactory();
    } else if (platformType == PlatformB200) {
        platformName = "B200";
        SetGpuIdx(999);
        computeFactory = new B200ComputeFactory();
        contentCreatorFactory = new B200ContentCreatorFactory();
        kernelFactory = new CpuKernelFactory();  // reg_aladin's kernels; not on the F3D path
        measureCreatorFactory = new B200MeasureCreatorFactory();
    } else {
        NR_FATAL_ERROR("Unsupported platform type");
    }
}

Platform::~Platform() {
    delete computeFactory;
    delete contentCreatorFactory;
    delete kernelFactory;
    delete measureCreatorFactory;
}

std::string Platform::GetName() const {
    return platformName;
}

PlatformType Platform::GetPlatformType() const {
    return platformType;
}

// 999 keeps the current device (the CUDA runtime's, device 0 in a fresh process)
void Platform::SetGpuIdx(unsigned gpuIdxIn) {
    if (platformType != PlatformB200) {
        gpuIdx = 999;
        return;
    }
    int device = 0;
    if (gpuIdxIn != 999) {
        gpuIdx = gpuIdxIn;
        device = int(gpuIdxIn);
    } else if (cudaGetDevice(&device) != cudaSuccess) {
        device = 0;
    }
    nrb_platform::Check(nrb_set_device(device), "nrb_set_device");
}

Compute* Platform::CreateCompute(Content& con) const {
    return computeFactory->Produce(con);
}

ContentCreator* Platform::CreateContentCreator(const ContentType conType) const {
    return contentCreatorFactory->Produce(conType);
}

Kernel* Platform::CreateKernel(const std::string& name, Content *con) const {
    return kernelFactory->Produce(name, con);
}

MeasureCreator* Platform::CreateMeasureCreator() const {
    return measureCreatorFactory->Produce();
}

template<typename Type>
Optimiser<Type>* Platform::CreateOptimiser(F3dContent& con, InterfaceOptimiser& opt, size_t maxIterationNumber,
                                           bool useConjGradient, bool optimiseX, bool optimiseY, bool optimiseZ,
                                           F3dContent *conBw) const {
    nifti_image *grid = con.F3dContent::GetControlPointGrid();
    nifti_image *gridBw = conBw ? static_cast<nifti_image*>(conBw->F3dContent::GetControlPointGrid()) : nullptr;
    Optimiser<Type> *optimiser = nullptr;
    Type *dof = nullptr, *grad = nullptr, *dofBw = nullptr, *gradBw = nullptr;
    if (platformType == PlatformType::Cpu) {
        optimiser = useConjGradient ? new ConjugateGradient<Type>() : new Optimiser<Type>();
        dof = static_cast<Type*>(grid->data);
        grad = static_cast<Type*>(con.GetTransformationGradient()->data);
        if (conBw) {
            dofBw = static_cast<Type*>(gridBw->data);
            gradBw = static_cast<Type*>(conBw->GetTransformationGradient()->data);
        }
    } else if (platformType == PlatformB200) {
        if constexpr (std::is_same_v<Type, float>) {
            if (conBw)
                NR_FATAL_ERROR("A symmetric optimisation is not available on the B200 platform");
            auto& b = dynamic_cast<B200F3dContent&>(con);
            optimiser = useConjGradient ? static_cast<Optimiser<float>*>(new B200ConjugateGradient(b))
                                        : static_cast<Optimiser<float>*>(new B200Optimiser(b));
            dof = b.GetControlPointGridDevice();
            grad = b.GetTransformationGradientDevice();
        } else {
            NR_FATAL_ERROR("The B200 platform optimises single-precision grids only");
        }
    }
    optimiser->Initialise(grid->nvox, grid->nz > 1 ? 3 : 2, optimiseX, optimiseY, optimiseZ, maxIterationNumber, 0,
                          &opt, dof, grad, gridBw ? gridBw->nvox : 0, dofBw, gradBw);
    return optimiser;
}
template Optimiser<float>* Platform::CreateOptimiser(F3dContent&, InterfaceOptimiser&, size_t, bool, bool, bool, bool,
                                                     F3dContent*) const;
template Optimiser<double>* Platform::CreateOptimiser(F3dContent&, InterfaceOptimiser&, size_t, bool, bool, bool,
                                                      bool, F3dContent*) const;
