// ref_gpu_standins.cu -- stand-ins for three reference functions that
// EnstrophyAnalyzer::run (EnstrophyAnalyzer.cu:63-98) refers to.
//
// TEST INFRASTRUCTURE ONLY (oracle).  The same-device reference library
// (oracle/Makefile, target `refgpu`) compiles EnstrophyAnalyzer.cu unmodified
// for its enstrophyKernel; its run(), which the harness never calls, needs
// Parameter::getParD, vf::cuda::CudaGrid's constructor and
// calculateMacroscopicQuantitiesCompressible, whose reference definitions
// pull in the whole parameter and output code.  These definitions only let
// the library load; reaching one aborts.
#include <cstdlib>

#include <cuda_helper/CudaGrid.h>

#include "Parameter/Parameter.h"
#include "PostProcessor/MacroscopicQuantities.cuh"

std::shared_ptr<LBMSimulationParameter> Parameter::getParD(int)
{
    std::abort();
}

vf::cuda::CudaGrid::CudaGrid(unsigned int, unsigned int)
{
    std::abort();
}

void calculateMacroscopicQuantitiesCompressible(real*, real*, real*, real*, real*, unsigned int*, unsigned int*,
                                                unsigned int*, unsigned int*, unsigned long long, unsigned int, real*,
                                                bool)
{
    std::abort();
}
