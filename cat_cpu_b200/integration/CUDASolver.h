// CUDASolver.h -- the GPU solvers of libltl_b200 as a drop-in CASolver for the
// reference tree (kezada94/CAT_cpu, src/CellularAutomata/Solvers/).
//
// Compiled against the reference's own headers; it implements the abstract
// interface of CASolver (src/CellularAutomata/Solvers/CASolver.h:7-28) on top of
// the C ABI in include/ltl.h.  Radius and rule come from the reference's
// compile-time macros RADIUS / SMIN / SMAX / BMIN / BMAX (Makefile:10-14).
#pragma once

#include "CellularAutomata/Solvers/CASolver.h"
#include "Memory/CADataDomain.h"
#include "ltl.h"

#include <vector>

class CUDASolver : public CASolver {
   public:
    // variant: LTL_VARIANT_PLAIN / LTL_VARIANT_TENSOR / LTL_VARIANT_PACKED
    CUDASolver(int deviceId, int n, int variant, CADataDomain<int>* hostVisible);
    ~CUDASolver();
    bool ok() const { return ctx_ != nullptr; }

    // Called by every OpenMP thread inside CPUBenchmark's parallel region
    // (CPUBenchmark.cpp:66-82): thread 0 queues all steps on the GPU and waits
    // for them, then the team meets at a barrier, so the benchmark timer (thread
    // 0, after its own barrier) includes device completion.
    void doSteps(int stepNumber) override;
    void doStep() override;

   protected:
    void CAStepAlgorithm() override;
    void swapPointers() override;
    void fillHorizontalBoundaryConditions() override;
    void fillVerticalBoundaryConditions() override;
    void copyCurrentStateToHostVisibleData() override;
    void copyHostVisibleDataToCurrentState() override;
    void preamble() override;

   private:
    ltl_ctx* ctx_ = nullptr;
    int n_ = 0;
    std::vector<uint8_t> staging_;
};
