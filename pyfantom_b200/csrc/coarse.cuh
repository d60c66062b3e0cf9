// Element-level operator of multigrid level 1 (coarse.cu).
#pragma once

#include "common.cuh"
#include "elemop.cuh"

namespace pf {

struct CoarseOp {
    Grid fine, g;                 // fine grid and level-1 grid
    int tsize = 8;                // bytes per value of the V-cycle precision
    double coef[150];             // the distinct nonzeros of B0 (Walsh-basis child-0 matrix)
    void* Eh = nullptr;           // Ehat [8][coarse elements], V-cycle precision
    int* dmap = nullptr;          // coarse element -> dirty index or -1
    int* dlist = nullptr;         // dirty index -> coarse element
    double* M = nullptr;          // dirty matrices, physical basis, FP64 [cap][576]
    void* Wd = nullptr;           // dirty matrices, Walsh basis [576][cap], V-cycle precision
    int* count = nullptr;         // device: number of dirty elements, number of identity nodes
    int* h_count = nullptr;       // pinned copy
    int* bcount = nullptr;        // per-block counts of the flag compactions
    int cap = 0, ndirty = 0;
    // identity rows R (I - Z) P of the constrained fine DOFs, applied per coarse node in the
    // physical basis (kept out of the Walsh-basis dirty matrices, where their O(1) entries
    // would swamp the O(E_min) stiffness of void elements in FP32)
    const uint8_t* nflag = nullptr;  // coarse node touches a constrained fine node
    int* nmap = nullptr;             // coarse node -> identity index or -1
    int* nlist = nullptr;            // identity index -> coarse node
    void* S = nullptr;               // [3 * 27][icap] coefficients, V-cycle precision
    int icap = 0, nident = 0;
};

// PF_OK if K0 has the structure of an isotropic box element (coefficients in coef[150])
int coarse_factorise(const Op* op, double* coef);
int coarse_create(const Op* op, int fp32, CoarseOp** out);
void coarse_destroy(CoarseOp* c);
// Ehat and the dirty matrices for E; *realloc set when the dirty storage moved
int coarse_setup(CoarseOp* c, const double* E, const uint8_t* mask, const uint8_t* elem_flag,
                 const uint8_t* node_flag, const double* K0_dev, cudaStream_t st, bool* realloc);
template <typename T>
int launch_coarse_matvec(const CoarseOp* c, const Grid& g, const T* u, const Epi<T>& epi, cudaStream_t st);

}  // namespace pf
