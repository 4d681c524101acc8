// CASolverFactoryGPU.cpp -- CASolverFactory::createSolver with the GPU codes.
//
// Codes 7 / 8 / 9 build a CUDASolver (plain CUDA-core / tcgen05 tensor core /
// bit-packed); every other code goes to the reference's own factory
// (src/CellularAutomata/CASolverFactory.cpp:6-121), reached here under the
// name ltl_reference_createSolver.  In the reference tree a maintainer would
// instead add the three `case` blocks (codes 7, 8, 9, each returning a
// CUDASolver) to that switch; the renamed symbol lets the test build link both
// without editing the reference's sources.
#include "CellularAutomata/CASolverFactory.h"
#include "CUDASolver.h"
#include "Memory/Allocators/CPUAllocator.h"

extern "C" CASolver* ltl_reference_createSolver(int code, int deviceId, int n, int halo, int nThreads);

CASolver* CASolverFactory::createSolver(int code, int deviceId, int n, int halo, int nThreads) {
    int variant = -1;
    switch (code) {
        case 7: variant = LTL_VARIANT_PLAIN; break;
        case 8: variant = LTL_VARIANT_TENSOR; break;
        case 9: variant = LTL_VARIANT_PACKED; break;
        default: return ltl_reference_createSolver(code, deviceId, n, halo, nThreads);
    }
    CPUAllocator<int>* cpuAllocator = new CPUAllocator<int>();
    Allocator<int>* allocator = reinterpret_cast<Allocator<int>*>(cpuAllocator);
    CADataDomain<int>* hostVisible = new CADataDomain<int>(allocator, n, halo);
    hostVisible->allocate();
    CUDASolver* s = new CUDASolver(deviceId, n, variant, hostVisible);
    if (!s->ok()) {
        delete s;
        return nullptr;
    }
    return s;
}
