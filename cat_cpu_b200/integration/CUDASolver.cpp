// CUDASolver.cpp -- see CUDASolver.h.
#include "CUDASolver.h"

#include <cstdio>
#include <omp.h>

CUDASolver::CUDASolver(int deviceId, int n, int variant, CADataDomain<int>* hostVisible) : n_(n) {
    hostVisibleData = hostVisible;
    staging_.resize((size_t)n * n);
    int rc = ltl_create(&ctx_, deviceId, n, RADIUS, SMIN, SMAX, BMIN, BMAX, variant);
    if (rc != LTL_OK) {
        std::fprintf(stderr, "CUDASolver: ltl_create failed (%d): %s\n", rc, ltl_last_error());
        ctx_ = nullptr;
    }
}

CUDASolver::~CUDASolver() {
    if (ctx_) ltl_destroy(ctx_);
}

void CUDASolver::doSteps(int stepNumber) {
    if (omp_get_thread_num() == 0) {
        int rc = ltl_step(ctx_, stepNumber);
        if (rc == LTL_OK) rc = ltl_synchronize(ctx_);
        if (rc != LTL_OK) std::fprintf(stderr, "CUDASolver: step failed (%d): %s\n", rc, ltl_last_error());
    }
#pragma omp barrier
}

void CUDASolver::doStep() { doSteps(1); }

// The step, the torus halo and the buffer swap all happen on the device inside
// ltl_step; the per-phase hooks of the CPU solvers have nothing left to do.
void CUDASolver::CAStepAlgorithm() {}
void CUDASolver::swapPointers() {}
void CUDASolver::fillHorizontalBoundaryConditions() {}
void CUDASolver::fillVerticalBoundaryConditions() {}
void CUDASolver::preamble() {}

// int host grid (reference layout, halo of the domain) <-> uint8 device grid
void CUDASolver::copyHostVisibleDataToCurrentState() {
    for (int i = 0; i < n_; ++i)
        for (int j = 0; j < n_; ++j) staging_[(size_t)i * n_ + j] = (uint8_t)(hostVisibleData->getInnerElementAt(i, j) != 0);
    int rc = ltl_upload(ctx_, staging_.data(), (size_t)n_);
    if (rc != LTL_OK) std::fprintf(stderr, "CUDASolver: upload failed (%d): %s\n", rc, ltl_last_error());
}

void CUDASolver::copyCurrentStateToHostVisibleData() {
    int rc = ltl_download(ctx_, staging_.data(), (size_t)n_);
    if (rc != LTL_OK) std::fprintf(stderr, "CUDASolver: download failed (%d): %s\n", rc, ltl_last_error());
    for (int i = 0; i < n_; ++i)
        for (int j = 0; j < n_; ++j) hostVisibleData->setInnerElementAt(i, j, staging_[(size_t)i * n_ + j]);
}
